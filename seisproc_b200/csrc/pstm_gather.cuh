// Kernel arguments and device helpers shared by the gather kernels (forward,
// V-gradient, batched, adjoint) and the fold kernel.
#pragma once
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <type_traits>

#include "pstm_common.cuh"
#include "pstm_internal.h"

namespace pstm {

// The aperture controller's cosine tapers (opt-in; the reference migrators
// construct the controller and never apply it): distance taper from d0 to the
// aperture dmax, angle taper from a0 to the maximum angle amax (radians), both
// legs; tan2 = tan^2(a0).  processors/migration/aperture.py:228-270.
struct TaperArgs {
  float d0, dinv, dmax;
  float a0, ainv, amax, tan2;
};

constexpr uint32_t kMagicBitsC = 0x4B000000u;  // float bits of 2^23

struct KArgs {
  const float4* geo;
  const int* list;
  const int64_t* off;
  const void* traces;
  const float* scales;
  int S;
  int n_samples;
  int n_il, n_xl, n_times;
  int tiles_xl, tile_il, tile_xl;
  float il_dx, il_dy, xl_dx, xl_dy;
  float out_t0, out_dt, in_t0, in_dt;
  const float* vel;
  long long vst, vsc;
  float aperture, tan_theta;
  int tda;
  float clamp_hi;
  float* out;
  float* fold_out;  // forward: fold written alongside the image when non-null
  const float* in_img;
  float* accum;
  int* err;
  int ring_stages, ring_rows;  // pipelined kernel: stages x rows per stage
  // anti-alias: output spacing (m) per axis, max half-width (samples), row pad
  float aa_dx, aa_dy, aa_lmax;
  int aa_pad;
  int row_origin;  // expanded rows: intercept origin (entry index)
  TaperArgs tp;    // plans built with a taper width
  // curved rays (plans built with a ray gradient k): k, and 1000 / (k in_dt)
  // turning the summed arccosh of the two legs into an input sample index
  float cr_k, cr_scale;
  long long n_traces;  // rows staged (bounds of the list entries)
  int inject;          // checked test build only: the fault to simulate (0 = none)
  int hist16;          // fold histogram in 16-bit halves (every tile list < 65536 traces)
};

// Faults the checked test build can simulate (pstm_test_set_injection); the
// product build never reads KArgs::inject.
enum Inject { INJ_NONE = 0, INJ_MISSING_COPY = 1, INJ_NO_CLAMP = 2, INJ_BAD_LIST_ENTRY = 3 };

// Trace-list entry at position pos.  The checked build (PSTM_BOUNDS_CHECK)
// verifies it before any use -- an entry outside [0, n_traces) raises
// PSTM_ERR_BOUNDS and is replaced by 0 -- and can simulate a corrupted first
// entry of the lists to exercise that path.
__device__ __forceinline__ int list_entry(const KArgs& A, int64_t pos) {
  int jj = A.list[pos];
#ifdef PSTM_BOUNDS_CHECK
  if (A.inject == INJ_BAD_LIST_ENTRY && pos == 0)
    jj = (int)(A.n_traces + 1000 < 0x7fffffffLL ? A.n_traces + 1000 : 0x7fffffffLL);
  if (jj < 0 || (long long)jj >= A.n_traces) {
    set_error(A.err, PSTM_ERR_BOUNDS);
    jj = 0;
  }
#endif
  return jj;
}

// Checked build: the entry index a staged-row read addresses (from the float
// bits of the floored index) must lie in [lo, hi] of the row as staged;
// otherwise PSTM_ERR_BOUNDS is raised and the read goes to entry 0 instead.
// The product build compiles this to nothing.
struct RowCheck {
  int lo, hi;
  int* err;
};
__device__ __forceinline__ uint32_t checked_addr(uint32_t addr, uint32_t bits, uint32_t base,
                                                 int shift, const RowCheck& rc) {
#ifdef PSTM_BOUNDS_CHECK
  const int e = (int)(bits - kMagicBitsC);
  if (e < rc.lo || e > rc.hi) {
    set_error(rc.err, PSTM_ERR_BOUNDS);
    return base + (kMagicBitsC << shift);
  }
#endif
  return addr;
}

__device__ __forceinline__ float vel_at(const KArgs& A, int k, int c) {
  return __ldg(A.vel + (long long)k * A.vst + (long long)c * A.vsc);
}

// Threshold on max(h_s, h_r) at output sample k of column c: the per-leg
// aperture (constant or min(A, z tan(theta))) and the angle limit
// h < tan(theta) (z + 1e-6), all strict.
__device__ __forceinline__ float threshold(const KArgs& A, int c, int k) {
  const float v = vel_at(A, k, c);
  const float z = depth_of(v, out_time_ms(k, A.out_dt, A.out_t0));
  const float ang = __fmul_rn(A.tan_theta, __fadd_rn(z, 1e-6f));
  const float ap = A.tda ? fminf(A.aperture, __fmul_rn(z, A.tan_theta)) : A.aperture;
  return fminf(ap, ang);
}

__device__ __forceinline__ void column_xy(const KArgs& A, int il, int xl, float& x, float& y) {
  x = __fadd_rn(__fmul_rn((float)il, A.il_dx), __fmul_rn((float)xl, A.xl_dx));
  y = __fadd_rn(__fmul_rn((float)il, A.il_dy), __fmul_rn((float)xl, A.xl_dy));
}

// Squared leg distances rounded as the reference forms them (dx^2 + dy^2 in
// float32, no contraction).
__device__ __forceinline__ void leg_h2(float xc, float yc, float4 g, float& hs2, float& hr2) {
  const float dxs = __fsub_rn(xc, g.x), dys = __fsub_rn(yc, g.y);
  const float dxr = __fsub_rn(xc, g.z), dyr = __fsub_rn(yc, g.w);
  hs2 = __fadd_rn(__fmul_rn(dxs, dxs), __fmul_rn(dys, dys));
  hr2 = __fadd_rn(__fmul_rn(dxr, dxr), __fmul_rn(dyr, dyr));
}

// First window index kk in [0, nk) with hmax < thr[kk] (thr non-decreasing), or nk.
__device__ __forceinline__ int first_valid(const float* thr, int nk, float hmax) {
  int lo = 0, hi = nk;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (hmax < thr[mid])
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

// Tile -> column of local column index cl.
__device__ __forceinline__ bool tile_column(const KArgs& A, int tile, int cl, int& il, int& xl) {
  const int ti = tile / A.tiles_xl, tx = tile - ti * A.tiles_xl;
  il = ti * A.tile_il + cl / A.tile_xl;
  xl = tx * A.tile_xl + cl % A.tile_xl;
  return cl < A.tile_il * A.tile_xl && il < A.n_il && xl < A.n_xl;
}

// First staged sample of a window starting at output sample k0: traveltimes
// satisfy t >= |t0|, so no sample below floor((t0(k0) - in_t0)/in_dt) - 1 is read.
__device__ __forceinline__ int window_lo(const KArgs& A, int k0, int align) {
  const float t = out_time_ms(k0, A.out_dt, A.out_t0);
  float lof = floorf((t - A.in_t0) / A.in_dt) - 2.0f;
  int lo = lof > 0.0f ? (int)lof : 0;
  lo = min(lo, A.n_samples - 2);
  lo = max(lo, 0);
  return lo - lo % align;
}

enum WMode { W_OBL_SPREAD = 0, W_SPREAD = 1, W_OBL = 2, W_NONE = 3 };
enum Op { OP_FWD = 0, OP_ADJ = 1, OP_VGRAD = 2 };

constexpr float kMagic = 8388608.0f;  // 2^23
constexpr uint32_t kMagicBits = 0x4B000000u;
constexpr float kRadicandFloor = 1e-12f;  // keeps rsqrt finite at r = 0 (m^2)

// 1 up to start, 0.5 (1 + cos(pi (x - start) / (end - start))) up to end, 0
// beyond (inv = 1 / (end - start)): the aperture controller's cosine edge.
__device__ __forceinline__ float cos_edge(float x, float start, float inv, float end) {
  if (x <= start) return 1.0f;
  if (x > end) return 0.0f;
  return 0.5f * (1.0f + cospif((x - start) * inv));
}

// Angle taper of one leg at one output sample, angle = atan2(h, |z|); z^2 comes
// from the lane's constants (pre-scaled: zz = a^2 (z^2 + f), aa = a^2; else
// zz = z^2 + f).  Below the taper start (h^2 <= z^2 tan^2(a0)) it is 1 without
// the arctangent.
// The taper zone proper, called rather than inlined: the unrolled sweeps
// would otherwise carry dozens of copies of the arctangent and cosine.
static __device__ __noinline__ float angle_taper_zone(float h2, float z2, float a0, float ainv,
                                                      float amax) {
  return cos_edge(atan2f(sqrtf(h2), sqrtf(fmaxf(z2, 0.0f))), a0, ainv, amax);
}

template <bool PRE>
__device__ __forceinline__ float leg_angle_taper(float h2, float zz, float aa,
                                                 const TaperArgs& tp) {
  const float z2s = PRE ? fmaf(-aa, kRadicandFloor, zz) : zz - kRadicandFloor;
  const float h2s = PRE ? h2 * aa : h2;
  if (h2s <= z2s * tp.tan2) return 1.0f;
  return angle_taper_zone(h2, PRE ? z2s / aa : z2s, tp.a0, tp.ainv, tp.amax);
}

inline KArgs make_args(const Plan* p, const float* vel, int64_t vst, int64_t vsc) {
  KArgs A;
  A.geo = p->geo;
  A.list = p->tile_list;
  A.off = p->tile_off;
  A.traces = p->traces;
  A.scales = p->scales;
  A.S = p->row_stride;
  A.n_samples = p->n_samples;
  A.n_il = p->grid.n_il;
  A.n_xl = p->grid.n_xl;
  A.n_times = p->grid.n_times;
  A.tiles_xl = p->tiles_xl;
  A.tile_il = p->shape.tile_il;
  A.tile_xl = p->shape.tile_xl;
  A.il_dx = p->il_dx;
  A.il_dy = p->il_dy;
  A.xl_dx = p->xl_dx;
  A.xl_dy = p->xl_dy;
  A.out_t0 = (float)p->grid.t0_ms;
  A.out_dt = (float)p->grid.dt_ms;
  A.in_t0 = (float)p->params.in_t0_ms;
  A.in_dt = (float)p->params.in_dt_ms;
  A.vel = vel;
  A.vst = vst;
  A.vsc = vsc;
  A.aperture = (float)p->params.max_aperture_m;
  A.tan_theta = p->tan_theta;
  A.tda = p->params.time_dependent_aperture;
  A.clamp_hi = p->params.clamp == PSTM_CLAMP_MIGRATOR ? (float)(p->n_samples - 2)
                                                      : (float)((double)p->n_samples - 1.001);
  A.out = nullptr;
  A.fold_out = nullptr;
  A.in_img = nullptr;
  A.accum = p->accum;
  A.err = p->err;
  A.ring_stages = A.ring_rows = 0;
  A.aa_dx = (float)p->params.aa_dx;
  A.aa_dy = (float)p->params.aa_dy;
  A.aa_lmax = (float)p->params.aa_max_halfwidth;
  A.aa_pad = p->aa_pad;
  A.row_origin = p->row_origin;
  {
    const double tw = p->params.taper_width;
    const double ap = p->params.max_aperture_m, th = p->params.max_angle_deg * M_PI / 180.0;
    const double d0 = ap * (1.0 - tw), a0 = th * (1.0 - tw);
    A.tp.d0 = (float)d0;
    A.tp.dinv = tw > 0 ? (float)(1.0 / (ap - d0)) : 0.0f;
    A.tp.dmax = (float)ap;
    A.tp.a0 = (float)a0;
    A.tp.ainv = tw > 0 ? (float)(1.0 / (th - a0)) : 0.0f;
    A.tp.amax = (float)th;
    A.tp.tan2 = (float)(std::tan(a0) * std::tan(a0));
  }
  A.n_traces = p->n_traces;
  A.inject = test_injection();
  A.hist16 = p->longest_list < 65536 ? 1 : 0;
  A.cr_k = (float)p->params.ray_gradient;
  A.cr_scale = p->params.ray_gradient != 0
                   ? (float)(1000.0 / (p->params.ray_gradient * p->params.in_dt_ms))
                   : 0.0f;
  return A;
}

// The lower clamp is only needed when an output time precedes the first input
// sample (idx could fall below -1).
inline bool needs_lowclamp(const Plan* p) {
  return p->grid.t0_ms < p->params.in_t0_ms - 1e-9;
}


inline pstm_status cuda_fail(cudaError_t e, const char* what, std::string* why) {
  *why = std::string(what) + ": " + cudaGetErrorString(e);
  return PSTM_ECUDA;
}

}  // namespace pstm
