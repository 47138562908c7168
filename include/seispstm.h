/*
 * seispstm.h - C ABI of the B200 Kirchhoff pre-stack time migration library
 * (libseispstm.so, CUDA sm_100a).
 *
 * The library replaces the compute of SeisProc's PSTM hot path: the Python
 * signatures it sits under are
 *   MigrationEngine.migrate_bin_full   processors/migration/migration_engine.py:225-360
 *   migrate_kirchhoff_full             processors/migration/kirchhoff_kernel.py:459-854
 *   normalize_by_fold                  processors/migration/kirchhoff_kernel.py:437-456
 *   KirchhoffMigrator._migrate_chunk   processors/migration/kirchhoff_migrator.py:256-404
 * and the host binding that calls these entry points lives in the Python
 * package seisproc_b200 (ctypes).  SeisProc's PSTM path has no native FFI of its
 * own (it is pure PyTorch), so these signatures are new; each one names the
 * reference function whose work it performs.
 *
 * Conventions
 *  - Plain C types only; every array argument is a DEVICE pointer unless
 *    stated otherwise.  `stream` is a cudaStream_t passed as void*.
 *  - Traces are (n_samples, n_traces) sample-major float32, the reference's
 *    layout (views/migration_monitor_dialog.py:254 transposes into it).
 *  - Images and folds are (n_times, n_il, n_xl) float32, il-major columns
 *    (migration_engine.py:295-301).
 *  - Velocities are V_rms at the output samples, addressed as
 *    velocity[k * v_stride_t + c * v_stride_c] with k the output sample and
 *    c = il * n_xl + xl the column; both strides 0 means a constant velocity.
 *  - No C++ exception crosses this boundary.  Every entry point returns a
 *    pstm_status; pstm_last_error() gives the message of the last failure on
 *    the calling thread.
 *  - Calls are asynchronous on `stream` unless stated; a plan must not be used
 *    by two calls that overlap in time.
 */
#ifndef SEISPSTM_H_
#define SEISPSTM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SEISPSTM_ABI_VERSION 1

typedef enum pstm_status {
  PSTM_OK = 0,
  PSTM_EINVAL = 1,   /* invalid argument or configuration (reference raises ValueError) */
  PSTM_ENOMEM = 2,   /* device allocation failed */
  PSTM_ETIMEOUT = 3, /* a bounded device-side wait expired; the result is invalid */
  PSTM_EBOUNDS = 4,  /* a device-side bounds check fired; the result is invalid */
  PSTM_ECUDA = 5,    /* CUDA runtime error */
  PSTM_ENOTSUP = 6   /* combination not built into this library */
} pstm_status;

typedef enum pstm_dtype {
  PSTM_F32 = 0,
  PSTM_BF16 = 1,
  PSTM_F16 = 2,
  PSTM_F64 = 3
} pstm_dtype;

/* Amplitude weight (models/migration_config.py:40-45 WeightMode).
 * OBLIQUITY_SPREADING is migrate_kirchhoff_full's weight
 *   (z/(r_s+e)) (z/(r_r+e)) / (r_s r_r + e)          kirchhoff_kernel.py:690-693
 * SPREADING is KirchhoffMigrator's 1/(sqrt(r_s^2 r_r^2) + e)   kirchhoff_migrator.py:378 */
typedef enum pstm_weight {
  PSTM_WEIGHT_OBLIQUITY_SPREADING = 0,
  PSTM_WEIGHT_SPREADING = 1,
  PSTM_WEIGHT_OBLIQUITY = 2,
  PSTM_WEIGHT_NONE = 3
} pstm_weight;

/* Sample-index clamp.
 * FULL:      idx = (t - in_t0)/in_dt clamped to [0, n_samples - 1.001]   kirchhoff_kernel.py:707-709
 * MIGRATOR:  idx = (t - in_t0)/in_dt clamped to [0, n_samples - 2]       kirchhoff_migrator.py:381 */
typedef enum pstm_clamp { PSTM_CLAMP_FULL = 0, PSTM_CLAMP_MIGRATOR = 1 } pstm_clamp;

typedef struct pstm_grid {
  int32_t n_il, n_xl, n_times;
  /* world coordinates of column (il, xl):
   *   x = origin_x + il * il_dx + xl * xl_dx,  y = origin_y + il * il_dy + xl * xl_dy
   * migrate_bin_full's grid (azimuth ignored) is il_dx = il_spacing, xl_dy = xl_spacing. */
  double origin_x, origin_y;
  double il_dx, il_dy, xl_dx, xl_dy;
  double t0_ms, dt_ms; /* output time axis: t0 = t0_ms + k * dt_ms */
} pstm_grid;

typedef struct pstm_params {
  int32_t n_samples;           /* input samples per trace */
  double in_t0_ms, in_dt_ms;   /* input trace time axis */
  double max_aperture_m;       /* per-leg aperture h_s < A and h_r < A (kirchhoff_kernel.py:635) */
  double max_angle_deg;        /* atan2(h, z + 1e-6) < theta on both legs (:670-685) */
  int32_t time_dependent_aperture; /* A(z) = min(A, z tan theta) (:674-680) */
  int32_t weight;              /* pstm_weight */
  int32_t clamp;               /* pstm_clamp */
  int32_t storage;             /* pstm_dtype of the in-kernel trace copy: F32, BF16 or F16 */
  int32_t antialias;           /* 1: causal-integrated triangle anti-alias filter */
  double aa_dx, aa_dy;         /* output spacing used for the operator-dip half-width */
  double aa_max_halfwidth;     /* cap on the triangle half-width, in input samples */
  int32_t variant;             /* kernel shape id; 0 = built-in heuristic */
  int32_t forward_only;        /* 1: the plan only migrates.  float32 rows are then staged in
                                  intercept form, one FMA per tap and ~3 % faster; the
                                  demigration stays its transpose to ~1e-5 (not float rounding)
                                  and pstm_velocity_gradient rejects the plan; a batch takes
                                  it when every class plan is forward_only.
                                  0: (x, dx) rows, migration and demigration an exact float
                                  transpose pair (dot-product tests, least squares). */
  double taper_width;          /* 0: hard masks only (what the reference migrators apply).
                                  In (0, 1): also the aperture controller's cosine tapers
                                  (processors/migration/aperture.py:228-270) of both legs:
                                  distance from A (1 - w) to A, angle atan2(h, |z|) from
                                  theta (1 - w) to theta.  Float32 storage, migration only
                                  (demigration, V-gradient, batches and the anti-alias
                                  filter refuse it); the fold still counts hard-masked
                                  pairs.  The offset taper is per trace: scale the traces. */
  double ray_gradient;         /* 0: straight rays, t = (r_s + r_r) / V (DSR).  k != 0: rays
                                  in v(z) = v0 + k z, one-way time arccosh(1 + k r^2 /
                                  (2 v0 z)) / k, v0 = the velocity passed (constant), z =
                                  v0 t0 / 2: the traveltime table the reference migrator
                                  interpolates by default (traveltime_lut.py:141-167,
                                  kirchhoff_migrator.py:146-175, 346-365).  Float32,
                                  migration only, like taper_width (and not with it). */
} pstm_params;

typedef struct pstm_geometry {
  int64_t n_traces;
  int32_t coord_dtype; /* PSTM_F32 or PSTM_F64; world coordinates, device pointers */
  const void* source_x;
  const void* source_y;
  const void* receiver_x;
  const void* receiver_y;
} pstm_geometry;

typedef struct pstm_plan_stats {
  int64_t n_traces;
  int64_t n_tiles;
  int64_t list_entries;     /* total (tile, trace) candidate pairs after culling */
  int64_t device_bytes;     /* scratch owned by the plan */
  int32_t tile_il, tile_xl; /* columns per tile */
  int32_t t_window;         /* output samples per CTA window */
  int32_t variant;
} pstm_plan_stats;

typedef struct pstm_plan pstm_plan;

/* Library ABI version (SEISPSTM_ABI_VERSION). */
int32_t pstm_abi_version(void);

/* Copies the last error message of the calling thread into buf (NUL-terminated,
 * truncated to n bytes); returns its full length. */
int32_t pstm_last_error(char* buf, size_t n);

/* Builds a migration plan: converts the world coordinates to grid-local float32
 * (the grid origin is subtracted in float64), bins traces by midpoint, sorts
 * them spatially and builds, for every output tile, the list of traces whose
 * legs can fall inside the aperture of any of its columns.  Replaces the
 * per-tile midpoint pre-filter of kirchhoff_kernel.py:572-602.  Allocates the
 * plan's device scratch; synchronises `stream` once to size the lists. */
pstm_status pstm_plan_create(pstm_plan** plan, const pstm_grid* grid, const pstm_params* params,
                             const pstm_geometry* geometry, void* stream);

pstm_status pstm_plan_destroy(pstm_plan* plan);

pstm_status pstm_plan_get_stats(const pstm_plan* plan, pstm_plan_stats* stats);

/* Plans take their device memory from a stream-ordered pool per device, which
 * keeps up to 16 GiB of freed memory mapped so that the next plan reuses it
 * (building and destroying plans per bin then maps nothing new).  This returns
 * the current device's pooled memory beyond keep_bytes to the driver.  No
 * counterpart in the reference (its buffers are torch tensors, cached by
 * torch's allocator; torch.cuda.empty_cache is the analogue). */
pstm_status pstm_trim_memory(int64_t keep_bytes);

/* Copies traces first .. first + count - 1 of a host (n_samples, n_traces)
 * float32 array (the reference's sample-major layout) into a device
 * (n_samples, count) array, as one strided asynchronous copy on `stream` (the
 * host array should be page-locked for the copy to be asynchronous).  It lets
 * a caller upload a bin in blocks of traces and migrate each block (one plan
 * per block) while the next one is in flight; no counterpart in the reference. */
pstm_status pstm_copy_trace_columns(float* dst, const float* src, int64_t n_samples,
                                   int64_t n_traces, int64_t first, int64_t count,
                                   void* stream);

/* Loads traces into the plan's spatially sorted, trace-major device copy in the
 * plan's storage dtype (per-trace float32 scale for BF16/F16; for the
 * anti-alias filter, the trend-removed double integral).  `traces` is
 * (n_samples, n_traces) float32, or (n_traces, n_samples) if trace_major. */
pstm_status pstm_load_traces(pstm_plan* plan, const float* traces, int32_t trace_major,
                             void* stream);

/* Forward migration (data -> image): the work of migrate_kirchhoff_full
 * (kirchhoff_kernel.py:459-854) on the traces last loaded into the plan.
 * image and fold are (n_times, n_il, n_xl) float32 and are overwritten.
 * fold may be NULL. */
pstm_status pstm_migrate_loaded(pstm_plan* plan, const float* velocity, int64_t v_stride_t,
                                int64_t v_stride_c, float* image, float* fold, void* stream);

/* pstm_load_traces + pstm_migrate_loaded in one call. */
pstm_status pstm_migrate(pstm_plan* plan, const float* traces, int32_t trace_major,
                         const float* velocity, int64_t v_stride_t, int64_t v_stride_c,
                         float* image, float* fold, void* stream);

/* Fold only: number of traces inside the aperture and angle masks per output
 * sample (kirchhoff_kernel.py:724-726). */
pstm_status pstm_fold(pstm_plan* plan, const float* velocity, int64_t v_stride_t,
                      int64_t v_stride_c, float* fold, void* stream);

/* Adjoint of pstm_migrate (image -> data, Kirchhoff demigration): scatters
 * w * image(t0, x) into samples i0 and i0+1 of every trace inside the masks.
 * traces_out is (n_samples, n_traces) float32 (or trace-major) and is
 * overwritten.  No reference counterpart exists (the reference has no adjoint);
 * it is the exact transpose of the forward operator. */
pstm_status pstm_demigrate(pstm_plan* plan, const float* image, const float* velocity,
                           int64_t v_stride_t, int64_t v_stride_c, float* traces_out,
                           int32_t trace_major, void* stream);

/* Gradient of <grad_image, migrate(traces; V)> with respect to V_rms at every
 * output sample (traveltime and weight recomputed, masks held fixed), for the
 * OBLIQUITY_SPREADING weight.  Uses the traces last loaded into the plan.
 * grad_velocity is (n_times, n_il, n_xl) float32, overwritten. */
pstm_status pstm_velocity_gradient(pstm_plan* plan, const float* grad_image,
                                   const float* velocity, int64_t v_stride_t,
                                   int64_t v_stride_c, float* grad_velocity, void* stream);

/* Synchronises `stream`, then reads and clears the plan's device-side error
 * flags: PSTM_ETIMEOUT (a bounded wait for a trace copy expired),
 * PSTM_EBOUNDS, or PSTM_EINVAL for a velocity that is not positive and finite
 * or whose depth V*t0/2 decreases with t0.  Results computed since the last
 * check are invalid when this does not return PSTM_OK. */
pstm_status pstm_check(pstm_plan* plan, void* stream);

/* image / fold where fold >= min_fold, else image unchanged (out may alias image).
 * kirchhoff_kernel.py:437-456. */
pstm_status pstm_normalize_by_fold(const float* image, const float* fold, float* out, int64_t n,
                                   float min_fold, void* stream);

/* Divide by max(fold, min_fold) and zero where fold < min_fold:
 * MigrationResult.apply_fold_normalization / KirchhoffMigrator.migrate_dataset
 * (base_migrator.py:317-349, kirchhoff_migrator.py:496-501). */
pstm_status pstm_normalize_mute(const float* image, const float* fold, float* out, int64_t n,
                                float min_fold, void* stream);

/* ---- velocity ingestion ------------------------------------------------- */

/* V_rms at every output sample, out[k * n_cols + c] (float32), resampled on the
 * device from a velocity model `model` laid out (nz, nx, ny) C-order float32 on
 * its own (time, x, y) axes.  It replaces the point-by-point scipy evaluation
 * of models/velocity_model.py:181-245 (RegularGridInterpolator, linear,
 * fill_value=None: linear extrapolation beyond the axis ends) for the 2-D and
 * 3-D models that utils/velocity_io.py:1007-1173 reads.  The per-axis tables
 * come from the host: for output time k, iz[k] is the model interval
 * (clamped to [0, nz - 2]) and wz[k] the fraction within it (outside [0, 1]
 * when extrapolating); ix/wx and iy/wy likewise per output column.  A 2-D
 * model passes ny = 1 and iy = wy = NULL.  An axis of length 1 is constant
 * along it.  All pointers are device pointers; the blend is float64, rounded
 * once to float32. */
pstm_status pstm_velocity_grid(const float* model, int32_t nz, int32_t nx, int32_t ny,
                               const int32_t* iz, const double* wz, int32_t n_t,
                               const int32_t* ix, const double* wx, const int32_t* iy,
                               const double* wy, int64_t n_cols, float* out, void* stream);

/* ---- time-domain RMS operator (compatibility entry) -------------------- */

/* Sizes and parameters of pstm_time_rms_migrate.  Input sample i is at time
 * i * dt_ms (input traces start at t = 0); output time k at t_min_ms + k * dt_ms. */
typedef struct pstm_time_rms_params {
  int64_t n_samples;              /* input samples per trace, <= 2^24 */
  int64_t n_traces;
  int64_t n_points;               /* output points n_il * n_xl, il-major */
  int32_t n_times;                /* output times */
  int32_t tile;                   /* output points per tile (consecutive) */
  double dt_ms, t_min_ms;
  double max_aperture_m, max_angle_deg;
  int32_t time_dependent_aperture;
} pstm_time_rms_params;

/* The reference's time-domain RMS operator, migrate_kirchhoff_time_domain_rms
 * (processors/migration/kirchhoff_kernel.py:1313-1783, behind
 * MigrationEngine.migrate_bin_time_domain_rms, migration_engine.py:633-802) --
 * a different operator from pstm_migrate's Kirchhoff summation.  For each
 * (tile, trace) pair every input sample maps to
 * t_out = sqrt(t_in^2 + 4 h_eff^2 / V_rms(t_in)^2) for every output point of
 * the tile (h = point-to-midpoint distance, h_eff^2 = h^2 + half-offset^2),
 * masked by output range, aperture and angle, weighted by z / (r^3 + 1e-10),
 * and added at the truncated output index into the TRACE's own midpoint
 * column, with fold counted alongside.  The index arithmetic is the
 * reference's float32 sequence with IEEE rounding, so a contribution lands
 * where the reference puts it except in the rare cases where the reference's
 * CPU square root (torch's, not correctly rounded on every input) rounds an
 * output time across an integer index.
 *
 * Device pointers: traces (n_samples, n_traces) float32 sample-major;
 * mid_x/mid_y/half_offset_sq per trace; out_x/out_y per output point; v_rms
 * per input sample.  The caller forms the pairs the reference's per-tile
 * trace selection yields (midpoint within aperture + tile radius + 100 m of
 * the tile centre, the nearest max_traces_per_tile kept), sorted by the
 * trace's column: pair q is (pair_trace[q], pair_tile[q]), and segment g,
 * pairs seg_off[g] .. seg_off[g + 1] - 1 (n_segments + 1 offsets), all have
 * column seg_col[g] (il * n_xl + xl), one segment per column.  Pairs or
 * segments out of range are skipped.  image and fold, (n_times, n_points)
 * float32, are overwritten.  Requires 2 n_times + 3 n_samples <= 58112 (the
 * per-column sums and the staged trace live in shared memory). */
pstm_status pstm_time_rms_migrate(const pstm_time_rms_params* params, const float* traces,
                                  const float* mid_x, const float* mid_y,
                                  const float* half_offset_sq, const float* out_x,
                                  const float* out_y, const float* v_rms,
                                  const int32_t* pair_trace, const int32_t* pair_tile,
                                  int64_t n_pairs, const int64_t* seg_off,
                                  const int32_t* seg_col, int64_t n_segments, float* image,
                                  float* fold, void* stream);

/* ---- batched migration: many plans in one persistent launch ------------- */
typedef struct pstm_batch pstm_batch;

/* Groups plans that share the kernel shape, storage, weight, clamp, time axis
 * and trace length -- typically the offset/azimuth classes of one survey, each
 * with its own geometry, traces and output image -- for pstm_batch_migrate.
 * images[i] / folds[i] (folds may be NULL, or contain NULL entries) are the
 * per-class outputs, velocity the V_rms shared by all classes.  Builds the
 * device work list of (class, tile, window) items ordered by descending
 * trace-list length.  No reference counterpart: the reference migrates bins
 * one at a time (views/migration_monitor_dialog.py:201-430). */
pstm_status pstm_batch_create(pstm_batch** batch, pstm_plan* const* plans, int32_t n_plans,
                              float* const* images, float* const* folds, const float* velocity,
                              int64_t v_stride_t, int64_t v_stride_c, void* stream);

/* Migrates every class of the batch with the traces last loaded into each plan
 * (pstm_load_traces): one launch of the persistent kernel (one CTA per SM,
 * items pulled from a device queue), then the per-class folds.  Contains no
 * allocation and no host synchronisation, so it can be captured in a CUDA
 * graph.  Device-side errors are reported by pstm_check on the member plans. */
pstm_status pstm_batch_migrate(pstm_batch* batch, void* stream);

pstm_status pstm_batch_destroy(pstm_batch* batch);

/* Number of plans in the batch. */
int32_t pstm_batch_size(const pstm_batch* batch);

/* Number of kernel launches issued by this library since load (for accounting). */
int64_t pstm_launch_count(void);

/* Size of the device scratch array used by pstm_migrate_noalloc. */
#define PSTM_NOALLOC_SCRATCH_BYTES (16u << 20)

/* Forward migration + fold (as pstm_plan_create + pstm_migrate + pstm_check) that
 * allocates no device memory.  It has no counterpart in the reference.
 *
 * It is for callers that must not allocate while they run.  Examples: a process
 * whose caching allocator (PyTorch's, or an application's memory pool) already
 * owns the device's free memory; a real-time path that cannot take the
 * device-wide synchronisation cudaFree implies; code issuing work where
 * allocation is not allowed.  The caller still passes the inputs (traces
 * (n_samples, n_traces) float32 sample-major, coordinates, velocity) and the
 * outputs (image, fold; fold may be NULL).
 *
 * Its scratch lives in one static device array of PSTM_NOALLOC_SCRATCH_BYTES,
 * which every GPU that loads the library holds until the process exits.
 * Problems that need more reject with PSTM_EINVAL.  The scratch holds the
 * grid-local geometry (16 B/trace), the per-tile trace lists (sized for the
 * worst case, 4 B per tile per trace) and the staged float32 trace rows;
 * storage must be PSTM_F32.  Non-finite coordinates reject with PSTM_EINVAL, as
 * in pstm_plan_create.  The first call on a device looks up the array's
 * device address (cudaGetSymbolAddress).  All calls share the array: calls
 * whose work overlaps on the GPU race, and the array keeps the last call's
 * contents (the error flag is cleared on every call).  The call synchronises
 * `stream` before it returns, to report device-side errors, so it cannot be
 * captured in a CUDA graph (a plan with pstm_migrate can). */
pstm_status pstm_migrate_noalloc(const pstm_grid* grid, const pstm_params* params,
                                 const pstm_geometry* geometry, const float* traces,
                                 const float* velocity, int64_t v_stride_t, int64_t v_stride_c,
                                 float* image, float* fold, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SEISPSTM_H_ */
