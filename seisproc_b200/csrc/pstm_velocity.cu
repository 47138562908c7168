// V_rms(t0, x, y) on the output grid, resampled on the device from a velocity
// model given on its own (time, x[, y]) axes.
//
// The reference evaluates a 2-D or 3-D velocity model point by point with
// scipy's RegularGridInterpolator, linear, fill_value=None (linear
// extrapolation beyond the axis ends): models/velocity_model.py:181-245.  Its
// per-axis step (which interval, and the fraction within it) depends on one
// coordinate only, so the host computes it once per output time and once per
// output column (O(n_t + n_cols), in float64), and this kernel forms the
// n_t x n_cols blends -- the part that grows with the grid.  The blend is
// evaluated in float64 and rounded once to float32, as the reference's float64
// interpolation followed by .astype(float32) does.
//
// Work split: a thread owns one output column and loops over a run of output
// times, so the column's x/y tables are read once and the time tables are
// warp-uniform; the model (a few MB at most) stays in L2.  Writes are the
// HBM traffic: 4 bytes per output sample, coalesced along columns.  The
// float64 blend is factored as time-lerp(lateral blend, lateral blend), the
// same trilinear value as the sum over eight corners to float64 rounding.
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "pstm_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kTimesPerBlock = 32;

__global__ void __launch_bounds__(kThreads)
    velocity_grid_kernel(const float* __restrict__ model, int nz, int nx, int ny,
                         const int32_t* __restrict__ iz, const double* __restrict__ wz, int n_t,
                         const int32_t* __restrict__ ix, const double* __restrict__ wx,
                         const int32_t* __restrict__ iy, const double* __restrict__ wy,
                         int64_t n_cols, float* __restrict__ out) {
  const int64_t c = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  if (c >= n_cols) return;
  const int k0 = blockIdx.y * kTimesPerBlock;
  const int k1 = min(k0 + kTimesPerBlock, n_t);
  // An axis of length 1 is constant along it (both corners are index 0).
  // Interval indices are clamped to [0, n - 2]: the host tables already are,
  // and the clamp keeps every model read in bounds whatever the caller passes.
  const int64_t sx = ny, sz = (int64_t)nx * ny;
  const int64_t dx1 = nx > 1 ? sx : 0, dy1 = ny > 1 ? 1 : 0, dz1 = nz > 1 ? sz : 0;
  const double fx = wx[c];
  const double fy = iy ? wy[c] : 0.0;
  const int jx = min(max(ix[c], 0), max(nx - 2, 0));
  const int jy = iy ? min(max(iy[c], 0), max(ny - 2, 0)) : 0;
  const float* col = model + (int64_t)jx * sx + jy;
  // lateral corner weights of this column, (x, y) = (0,0), (0,1), (1,0), (1,1)
  const double w00 = (1.0 - fx) * (1.0 - fy), w01 = (1.0 - fx) * fy;
  const double w10 = fx * (1.0 - fy), w11 = fx * fy;
  auto lateral = [&](const float* q) {
    return w00 * (double)__ldg(q) + w01 * (double)__ldg(q + dy1) +
           w10 * (double)__ldg(q + dx1) + w11 * (double)__ldg(q + dx1 + dy1);
  };
  // The model's time axis is coarse next to the output's, so consecutive
  // output times share a model interval: the two lateral blends at its ends
  // are formed once per interval (warp-uniform: every lane has the same k) and
  // each output time is one lerp between them.
  int cur = -1;
  double v0 = 0.0, v1 = 0.0;
  for (int k = k0; k < k1; ++k) {
    const int jz = min(max(iz[k], 0), max(nz - 2, 0));
    if (jz != cur) {
      cur = jz;
      v0 = lateral(col + (int64_t)jz * sz);
      v1 = lateral(col + (int64_t)jz * sz + dz1);
    }
    const double fz = wz[k];
    out[(int64_t)k * n_cols + c] = (float)((1.0 - fz) * v0 + fz * v1);
  }
}

pstm_status bad(const char* msg) {
  pstm::set_last_error(msg);
  return PSTM_EINVAL;
}

}  // namespace

extern "C" pstm_status pstm_velocity_grid(const float* model, int32_t nz, int32_t nx, int32_t ny,
                                          const int32_t* iz, const double* wz, int32_t n_t,
                                          const int32_t* ix, const double* wx, const int32_t* iy,
                                          const double* wy, int64_t n_cols, float* out,
                                          void* stream) {
  if (nz < 1 || nx < 1 || ny < 1 || n_t < 0 || n_cols < 0 || !model || !out ||
      (n_t > 0 && (!iz || !wz)) || (n_cols > 0 && (!ix || !wx)) || (!iy != !wy) ||
      (ny > 1 && !iy))
    return bad("pstm_velocity_grid: bad arguments");
  if (n_t == 0 || n_cols == 0) return PSTM_OK;
  const dim3 grid((unsigned)((n_cols + kThreads - 1) / kThreads),
                  (unsigned)((n_t + kTimesPerBlock - 1) / kTimesPerBlock));
  if (grid.y > 65535u) return bad("pstm_velocity_grid: more than 2097120 output times");
  velocity_grid_kernel<<<grid, kThreads, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      model, nz, nx, ny, iz, wz, n_t, ix, wx, iy, wy, n_cols, out);
  pstm::count_launch();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    pstm::set_last_error(std::string("velocity_grid_kernel: ") + cudaGetErrorString(e));
    return PSTM_ECUDA;
  }
  return PSTM_OK;
}
