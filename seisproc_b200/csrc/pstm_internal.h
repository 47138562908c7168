// Internal (C++) view of a PSTM plan shared by the plan builder and the
// migration kernels.  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/seispstm.h"

namespace pstm {

// Kernel shape of one migration CTA: COLS columns (tile_il x tile_xl) x WPC
// warps per column, each warp owning 64*M consecutive output samples.
struct Shape {
  int id;
  int cols, wpc, m;
  int tile_il, tile_xl;
  int t_window() const { return wpc * 64 * m; }
  int threads() const { return cols * wpc * 32; }
};

constexpr int kGuard = 2;        // guard entries before the first staged sample
constexpr int kBlockTraces = 32;  // trace rows per pipeline stage, at most

struct Plan {
  int device = 0;
  pstm_grid grid{};
  pstm_params params{};
  int64_t n_traces = 0;
  int n_samples = 0;
  int row_stride = 0;  // elements per staged trace row (multiple of 8)
  int aa_pad = 0;      // anti-alias rows: integral entries before sample 0 (and after N)
  int row_origin = 0;  // expanded rows: entry q holds (x - (q - row_origin) dx, dx)
  int elt_bytes = 4;
  Shape shape{};
  int tiles_il = 0, tiles_xl = 0;
  int64_t n_tiles = 0;
  int n_windows = 0;
  // grid-local column coordinate steps (world origin subtracted in float64)
  float il_dx = 0, il_dy = 0, xl_dx = 0, xl_dy = 0;
  float tan_theta = 0;
  // device buffers
  float4* geo = nullptr;         // (sx, sy, rx, ry) local, spatially sorted
  int* perm = nullptr;           // sorted -> original trace index
  int* inv_perm = nullptr;       // original -> sorted
  int64_t* tile_off = nullptr;   // n_tiles + 1
  int* tile_list = nullptr;      // sorted trace indices per tile
  int64_t list_entries = 0;
  // longest tile list; below 65536 the forward kernel's fold histogram
  // counts in 16-bit halves (every count is at most the list length)
  int64_t longest_list = INT64_MAX;
  void* traces = nullptr;        // n_traces x row_stride, storage dtype
  float* scales = nullptr;       // per sorted trace (BF16/F16), else nullptr
  float* accum = nullptr;        // adjoint accumulation rows (n_traces x row_stride f32)
  // adjoint: tiles holding each block of adj_tb consecutive sorted traces, and
  // the per-call column table (z'^2, a', g, threshold) per output sample
  int adj_tb = 0;
  int64_t* adj_off = nullptr;    // n_trace_blocks + 1
  int* adj_tiles = nullptr;
  int64_t n_adj_tiles = 0;
  float4* adj_table = nullptr;   // n_times x n_il x n_xl, column-major
  int* err = nullptr;            // device error flags
  int64_t bytes = 0;
  bool traces_loaded = false;
};

// launchers (pstm_migrate.cu)
// forward migration; fold (nullable) is counted in the same launch
pstm_status launch_forward(Plan* p, const float* vel, int64_t vst, int64_t vsc, float* image,
                           float* fold, cudaStream_t s, std::string* why);
pstm_status launch_fold(Plan* p, const float* vel, int64_t vst, int64_t vsc, float* fold,
                        cudaStream_t s, std::string* why);
pstm_status launch_adjoint(Plan* p, const float* image, const float* vel, int64_t vst,
                           int64_t vsc, cudaStream_t s, std::string* why);
pstm_status launch_vgrad(Plan* p, const float* grad_image, const float* vel, int64_t vst,
                         int64_t vsc, float* grad_v, cudaStream_t s, std::string* why);
pstm_status launch_velocity_check(Plan* p, const float* vel, int64_t vst, int64_t vsc,
                                  cudaStream_t s, std::string* why);
bool shape_for_variant(int variant, int n_xl, int n_times, Shape* out);
// Fault simulated by the checked test build's kernels (set by its
// pstm_test_set_injection); always 0 in the product build.
int test_injection();
size_t forward_smem_bytes(const Plan* p);
size_t forward_smem_budget(const Plan* p);  // per-CTA shared memory of the plan's shape
void count_launch();
// Device memory of plans and their temporaries: stream-ordered allocations from
// a library pool per device that keeps up to kPoolKeepBytes of freed memory
// mapped for the next plan (pstm_trim_memory returns it).
constexpr uint64_t kPoolKeepBytes = uint64_t(16) << 30;
cudaError_t dev_malloc(void** ptr, size_t bytes, cudaStream_t s);
void dev_free(void* ptr, cudaStream_t s);
void set_last_error(const std::string& msg);  // message returned by pstm_last_error
pstm_status ensure_trace_storage(Plan* p, cudaStream_t s);  // staged rows allocated once

}  // namespace pstm
