// Time-domain RMS operator: every input sample of a trace mapped to an output
// time t_out = sqrt(t_in^2 + 4 h_eff^2 / V_rms(t_in)^2) and scattered into the
// trace's own midpoint column, once per output point of each tile whose trace
// list holds the trace.
//
// This is the reference's migrate_kirchhoff_time_domain_rms
// (processors/migration/kirchhoff_kernel.py:1313-1783; per-sample arithmetic
// _time_domain_batch_kernel :1217-1287), a different operator from the
// Kirchhoff summation of pstm_gather2.cuh.  Its output time index truncates a
// float32 expression, so the index arithmetic here repeats the reference's
// float32 operations in the reference's order with explicitly rounded IEEE
// intrinsics (no FMA contraction): each contribution lands at the reference's
// index, except where torch's CPU float32 sqrt (not correctly rounded on
// every input) rounds t_out across an integer index in the reference's own
// CPU run -- a few in 10^7.  The sums differ only in order.
//
// Work split.  All contributions of a trace land in ONE column (its midpoint
// bin), so the caller's (tile, trace) pairs are sorted by that column and a CTA
// owns one column: its n_times image and fold sums live in shared memory
// (float red.shared for the image, integer atomics for the fold) and are
// stored once at the end -- no global atomics, no zeroing pass over the
// touched columns.  Per pair the CTA stages the trace (a strided column of the
// sample-major input, read once per pair and reused by every output point of
// the tile); per output point the horizontal terms are formed once (uniform
// across the CTA) and the threads sweep the input samples.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <string>

#include "pstm_internal.h"

namespace {

constexpr int kThreads = 256;

struct TdConst {
  float dt, t_min, lim, aperture, theta, tan_lo, tan_hi;
  int fast_angle;  // the angle test may start with the tangent comparison
  int tda;         // time-dependent aperture
  float tan_theta;
};

// atan2(h, z1) < theta for h >= 0.  Away from the limit the comparison with
// z1 tan(theta) decides it (margins of 1e-4 relative, far above the rounding
// of either form); within the margins atan2f decides, as the reference does.
__device__ __forceinline__ bool angle_ok(float h, float z1, const TdConst& k) {
  if (k.fast_angle && z1 > 0.f) {
    if (h < z1 * k.tan_lo) return true;
    if (h > z1 * k.tan_hi) return false;
  }
  return atan2f(h, z1) < k.theta;
}

__global__ void __launch_bounds__(kThreads)
    time_rms_kernel(const float* __restrict__ traces, int64_t n_traces, int n_s,
                    const float* __restrict__ mid_x, const float* __restrict__ mid_y,
                    const float* __restrict__ hoff_sq, const float* __restrict__ out_x,
                    const float* __restrict__ out_y, int64_t n_points, int tile,
                    const float* __restrict__ v_rms, const int32_t* __restrict__ pair_trace,
                    const int32_t* __restrict__ pair_tile, int64_t n_pairs,
                    const int64_t* __restrict__ seg_off, const int32_t* __restrict__ seg_col,
                    int n_times, TdConst k, float* __restrict__ image,
                    float* __restrict__ fold) {
  extern __shared__ float smem[];
  float* img = smem;                                       // n_times
  uint32_t* cnt = reinterpret_cast<uint32_t*>(img + n_times);  // n_times
  float* vs = reinterpret_cast<float*>(cnt + n_times);    // n_s: V_rms
  float* vsq = vs + n_s;                                   // n_s: V_rms^2
  float* row = vsq + n_s;                                  // n_s: this pair's trace
  const int col = seg_col[blockIdx.x];
  if (col < 0 || col >= n_points) return;
  const int64_t q0 = min(max(seg_off[blockIdx.x], (int64_t)0), n_pairs);
  const int64_t q1 = min(max(seg_off[blockIdx.x + 1], q0), n_pairs);

  for (int i = threadIdx.x; i < n_times; i += kThreads) {
    img[i] = 0.f;
    cnt[i] = 0u;
  }
  for (int s = threadIdx.x; s < n_s; s += kThreads) {
    const float v = v_rms[s];
    vs[s] = v;
    vsq[s] = __fmul_rn(v, v);
  }

  for (int64_t q = q0; q < q1; ++q) {
    const int j = pair_trace[q];
    const int t = pair_tile[q];
    if (j < 0 || j >= n_traces || t < 0 || (int64_t)t * tile >= n_points) continue;
    __syncthreads();  // the previous pair's row is no longer read
    for (int s = threadIdx.x; s < n_s; s += kThreads) row[s] = __ldg(traces + (int64_t)s * n_traces + j);
    __syncthreads();
    const float mx = mid_x[j], my = mid_y[j], ho = hoff_sq[j];
    const int64_t p0 = (int64_t)t * tile;
    const int64_t p1 = min(p0 + tile, n_points);
    for (int64_t p = p0; p < p1; ++p) {
      // kirchhoff_kernel.py:1588-1594: h^2 = dx^2 + dy^2, h_eff^2 = h^2 + half-offset^2
      const float dx = __fsub_rn(out_x[p], mx);
      const float dy = __fsub_rn(out_y[p], my);
      const float h_sq = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
      const float h = __fsqrt_rn(h_sq);
      // both aperture forms require h < max_aperture (the time-dependent one is
      // clamped to it), so a point beyond it contributes nothing
      if (!(h < k.aperture)) continue;
      // :1243 time_shift^2 = 4 h_eff^2 1e6 / V^2, evaluated left to right
      const float c = __fmul_rn(__fmul_rn(4.f, __fadd_rn(h_sq, ho)), 1e6f);
      for (int s = threadIdx.x; s < n_s; s += kThreads) {
        const float t_in = __fmul_rn((float)s, k.dt);           // :1633 (t_min 0)
        const float t_out = __fsqrt_rn(__fadd_rn(__fmul_rn(t_in, t_in), __fdiv_rn(c, vsq[s])));
        const float idx = __fdiv_rn(__fsub_rn(t_out, k.t_min), k.dt);  // :1250
        if (!(idx >= 0.f && idx < k.lim)) continue;                    // :1253
        const float v = vs[s];
        if (k.tda) {  // :1256-1259 aperture(t) = t_out V / 2000 tan(theta), <= max
          const float ap = fminf(__fmul_rn(__fdiv_rn(__fmul_rn(t_out, v), 2000.f), k.tan_theta),
                                 k.aperture);
          if (!(h < ap)) continue;
        }
        const float z = __fdiv_rn(__fmul_rn(v, t_out), 2000.f);        // :1264
        if (!angle_ok(h, __fadd_rn(z, 1e-6f), k)) continue;            // :1267-1268
        const float r_sq = __fadd_rn(__fmul_rn(z, z), h_sq);            // :1274-1276
        const float w = __fdiv_rn(z, __fadd_rn(__fmul_rn(__fsqrt_rn(r_sq), r_sq), 1e-10f));
        const int ki = (int)idx;                                       // :1282 truncation
        atomicAdd(img + ki, __fmul_rn(row[s], w));
        atomicAdd(cnt + ki, 1u);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n_times; i += kThreads) {
    image[(int64_t)i * n_points + col] = img[i];
    fold[(int64_t)i * n_points + col] = (float)cnt[i];
  }
}

pstm_status bad(const char* msg) {
  pstm::set_last_error(msg);
  return PSTM_EINVAL;
}

}  // namespace

extern "C" pstm_status pstm_time_rms_migrate(const pstm_time_rms_params* p, const float* traces,
                                             const float* mid_x, const float* mid_y,
                                             const float* half_offset_sq, const float* out_x,
                                             const float* out_y, const float* v_rms,
                                             const int32_t* pair_trace, const int32_t* pair_tile,
                                             int64_t n_pairs, const int64_t* seg_off,
                                             const int32_t* seg_col, int64_t n_segments,
                                             float* image, float* fold, void* stream) {
  if (!p) return bad("pstm_time_rms_migrate: params is NULL");
  if (p->n_samples < 1 || p->n_samples > (1 << 24) || p->n_traces < 0 ||
      p->n_traces > INT32_MAX || p->n_points < 1 || p->n_points > INT32_MAX || p->n_times < 1 ||
      p->tile < 1 || !(p->dt_ms > 0.0) || !std::isfinite(p->t_min_ms) ||
      std::isnan(p->max_aperture_m) || !std::isfinite(p->max_angle_deg))
    return bad("pstm_time_rms_migrate: bad sizes or parameters");
  if (!image || !fold) return bad("pstm_time_rms_migrate: image/fold is NULL");
  if (n_pairs < 0 || n_segments < 0 || n_segments > INT32_MAX)
    return bad("pstm_time_rms_migrate: bad pair/segment counts");
  if (n_segments > 0 && (!traces || !mid_x || !mid_y || !half_offset_sq || !out_x || !out_y ||
                         !v_rms || !pair_trace || !pair_tile || !seg_off || !seg_col))
    return bad("pstm_time_rms_migrate: NULL input");
  const size_t smem = sizeof(float) * (2 * (size_t)p->n_times + 3 * (size_t)p->n_samples);
  if (smem > 227 * 1024)
    return bad("pstm_time_rms_migrate: 2 n_times + 3 n_samples exceeds 58112 (shared memory)");
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const size_t bytes = sizeof(float) * (size_t)p->n_times * (size_t)p->n_points;
  cudaError_t e = cudaMemsetAsync(image, 0, bytes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(fold, 0, bytes, s);
  if (e != cudaSuccess) {
    pstm::set_last_error(std::string("pstm_time_rms_migrate: ") + cudaGetErrorString(e));
    return PSTM_ECUDA;
  }
  if (n_segments == 0) return PSTM_OK;

  TdConst k;
  k.dt = (float)p->dt_ms;
  k.t_min = (float)p->t_min_ms;
  k.lim = (float)((double)p->n_times - 0.001);
  k.aperture = (float)p->max_aperture_m;
  const double rad = p->max_angle_deg * (M_PI / 180.0);
  k.theta = (float)rad;
  k.tan_theta = (float)std::tan(rad);
  k.fast_angle = (p->max_angle_deg > 0.0 && p->max_angle_deg < 80.0) ? 1 : 0;
  k.tan_lo = k.fast_angle ? (float)(std::tan(rad) * (1.0 - 1e-4)) : 0.f;
  k.tan_hi = k.fast_angle ? (float)(std::tan(rad) * (1.0 + 1e-4)) : 0.f;
  k.tda = p->time_dependent_aperture ? 1 : 0;

  e = cudaFuncSetAttribute(time_rms_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
  if (e != cudaSuccess) {
    pstm::set_last_error(std::string("time_rms_kernel: ") + cudaGetErrorString(e));
    return PSTM_ECUDA;
  }
  time_rms_kernel<<<(unsigned)n_segments, kThreads, smem, s>>>(
      traces, p->n_traces, (int)p->n_samples, mid_x, mid_y, half_offset_sq, out_x, out_y,
      p->n_points, p->tile, v_rms, pair_trace, pair_tile, n_pairs, seg_off, seg_col, p->n_times,
      k, image, fold);
  pstm::count_launch();
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    pstm::set_last_error(std::string("time_rms_kernel: ") + cudaGetErrorString(e));
    return PSTM_ECUDA;
  }
  return PSTM_OK;
}
