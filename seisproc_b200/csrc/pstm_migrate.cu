// Kirchhoff PSTM gather kernels for sm_100a: forward migration, fold,
// demigration (adjoint) and the V_rms gradient.
//
// One CTA owns an output tile: COLS columns x a window of WPC*64*M output
// samples.  Warp w works on column w / WPC and on 64*M consecutive samples;
// lane l holds samples (k, k+32) of every 64-sample group as one packed f32x2
// register pair, so the image accumulators stay in registers for the whole
// trace loop and the two samples of a pair are computed by one f32x2 op.
//
// Traces arrive through the tile's pre-culled trace list in blocks of
// kBlockTraces.  The TMA engine (cp.async.bulk, completion on an mbarrier)
// copies each trace row of the block from HBM into shared memory; the CTA then
// expands the rows into (x[i], x[i+1]-x[i]) float2 entries so that one 64-bit
// shared load plus one FFMA produces a linearly interpolated amplitude.  While
// the CTA computes on block b, the bulk copy of block b+1 is in flight.
//
// Per (column, trace) the aperture and angle masks of the reference
// (kirchhoff_kernel.py:635, 670-685) reduce to one threshold test
// max(h_s, h_r) < thr(t0) whose threshold grows with t0, so every trace
// contributes to a suffix [k_start, n_times) of the column.  k_start is found
// once per (column, trace) by binary search over a per-CTA threshold table, and
// the fold kernel counts the same k_start values.
//
// Per contributing pair the forward kernel spends 2 MUFU rsqrt and about 9
// FP32-pipe instructions (f32x2 ops count once per pair of samples): DSR time
// t = (r_s + r_r)/V with r = rr * rsqrt(rr), the 2^23 floor trick for the
// sample index, one LDS.64 and one FFMA for the interpolation, and the
// obliquity x spreading weight z^2 (q_s q_r)^2 with the z^2 factor applied once
// per output sample in the epilogue.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <string>

#include "pstm_gather2.cuh"

namespace pstm {

static std::atomic<int64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
int64_t launch_total() { return g_launches.load(); }

static std::atomic<int> g_inject{0};
int test_injection() { return g_inject.load(std::memory_order_relaxed); }

// ---------------------------------------------------------------------------
// Fold: number of traces inside the masks per output sample.  Counts the same
// k_start values as the gather kernel (same threshold table and search).
// ---------------------------------------------------------------------------
template <int COLS, int T>
__global__ void __launch_bounds__(256) pstm_fold_kernel(const KArgs A) {
  extern __shared__ __align__(128) unsigned char smem[];
  float* thr = reinterpret_cast<float*>(smem);
  int* hist = reinterpret_cast<int*>(smem + COLS * T * 4);
  const int tile = blockIdx.x;
  const int k0 = blockIdx.y * T;
  const int kend = min(k0 + T, A.n_times);
  const int nk = kend - k0;
  for (int e = threadIdx.x; e < COLS * T; e += blockDim.x) {
    const int q = e / T, kk = e - q * T;
    int qil, qxl;
    float v = -1.0f;
    if (kk < nk && tile_column(A, tile, q, qil, qxl)) v = threshold(A, qil * A.n_xl + qxl, k0 + kk);
    thr[e] = v;
    hist[e] = 0;
  }
  __syncthreads();
  const int64_t off0 = A.off[tile];
  const int n_list = (int)(A.off[tile + 1] - off0);
  float qx[COLS], qy[COLS];
  bool ok[COLS];
#pragma unroll
  for (int q = 0; q < COLS; ++q) {
    int qil, qxl;
    ok[q] = tile_column(A, tile, q, qil, qxl);
    qx[q] = qy[q] = 0.f;
    if (ok[q]) column_xy(A, qil, qxl, qx[q], qy[q]);
  }
  for (int t = threadIdx.x; t < n_list; t += blockDim.x) {
    const float4 g = __ldg(A.geo + list_entry(A, off0 + t));
#pragma unroll
    for (int q = 0; q < COLS; ++q) {
      if (!ok[q]) continue;
      float hs2, hr2;
      leg_h2(qx[q], qy[q], g, hs2, hr2);
      const int kk = first_valid(thr + q * T, nk, sqrtf(fmaxf(hs2, hr2)));
      if (kk < nk) atomicAdd(hist + q * T + kk, 1);
    }
  }
  __syncthreads();
  // inclusive prefix over the window, one warp per column
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_c = A.n_il * A.n_xl;
  for (int q = warp; q < COLS; q += blockDim.x / 32) {
    int qil, qxl;
    if (!tile_column(A, tile, q, qil, qxl)) continue;
    const int c = qil * A.n_xl + qxl;
    int carry = 0;
    for (int base = 0; base < nk; base += 32) {
      int v = (base + lane < nk) ? hist[q * T + base + lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      v += carry;
      if (base + lane < nk) A.out[(long long)(k0 + base + lane) * n_c + c] = (float)v;
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
  }
}

// Non-decreasing depth z(t0) per column keeps every mask a suffix in t0; a
// velocity model that breaks it (or is not positive and finite) is rejected.
__global__ void pstm_velocity_check_kernel(const KArgs A, int n_cols_checked) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)A.n_times * n_cols_checked;
  if (e >= total) return;
  const int c = (int)(e / A.n_times), k = (int)(e % A.n_times);
  const float v = vel_at(A, k, c);
  if (!(v > 0.f) || !(v < 3.0e38f)) {
    set_error(A.err, PSTM_ERR_VELOCITY);
    return;
  }
  if (k + 1 < A.n_times) {
    const float z0 = depth_of(v, out_time_ms(k, A.out_dt, A.out_t0));
    const float z1 = depth_of(vel_at(A, k + 1, c), out_time_ms(k + 1, A.out_dt, A.out_t0));
    if (z1 < z0) set_error(A.err, PSTM_ERR_VELOCITY);
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
// Kernel shapes: {id, cols, wpc, m, tile_il, tile_xl}.
static const Shape kShapes[] = {
    {1, 8, 2, 8, 2, 4},  // 8 columns (2x4) x 1024 samples, 16 warps
    {2, 4, 4, 4, 2, 2},  // 4 columns (2x2) x 1024 samples, 16 warps
    {3, 16, 1, 8, 4, 4},  // 16 columns (4x4) x 512 samples, 16 warps
    {4, 4, 2, 4, 2, 2},  // 4 columns (2x2) x 512 samples, 8 warps
    {5, 8, 2, 8, 8, 1},  // 2D lines: 8 inlines x 1024 samples
    {6, 4, 2, 4, 4, 1},  // 2D lines: 4 inlines x 512 samples
    {7, 2, 4, 2, 2, 1},  // 2D lines: 2 inlines x 512 samples
    {8, 4, 4, 4, 4, 1},  // 2D lines: 4 inlines x 1024 samples
    {9, 16, 1, 8, 16, 1},  // 2D lines: 16 inlines x 512 samples
    {10, 16, 1, 4, 4, 4},  // 16 columns (4x4) x 256 samples
    {11, 16, 1, 2, 4, 4},  // 16 columns (4x4) x 128 samples
    {12, 16, 1, 4, 16, 1},  // 2D lines: 16 inlines x 256 samples
    {13, 8, 1, 8, 2, 4},  // 8 columns (2x4) x 512 samples, 8 warps, two CTAs per SM
};

bool shape_for_variant(int variant, int n_xl, int n_times, Shape* out) {
  if (variant == 0) {
    // heuristic: 4 x 4 tiles for 3D grids, inline strips for 2D lines
    const bool line = n_xl < 2;
    if (line)
      variant = n_times <= 512 ? 9 : 8;
    else
      variant = 3;  // 16 columns x 512 samples: fastest measured for 500 and 1000 samples
  }
  for (const Shape& s : kShapes) {
    if (s.id == variant) {
      *out = s;
      return true;
    }
  }
  return false;
}

size_t forward_smem_budget(const Plan* p) { return (size_t)smem_budget(p->shape.threads()); }

size_t forward_smem_bytes(const Plan* p) {
  // pipelined forward kernel: the smallest ring (2 stages x 1 row) must fit
  // (the adjoint keeps as many float rows as fit, at least one)
  const int T = p->shape.t_window();
  return (size_t)smem2_layout(p->shape.cols, T, p->row_stride, p->elt_bytes, 2, 1).total;
}

pstm_status launch_velocity_check(Plan* p, const float* vel, int64_t vst, int64_t vsc,
                                  cudaStream_t s, std::string* why) {
  KArgs A = make_args(p, vel, vst, vsc);
  const int ncols = vsc != 0 ? p->grid.n_il * p->grid.n_xl : 1;
  const long long total = (long long)p->grid.n_times * ncols;
  const int threads = 256;
  pstm_velocity_check_kernel<<<(unsigned)((total + threads - 1) / threads), threads, 0, s>>>(A,
                                                                                            ncols);
  count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? PSTM_OK : cuda_fail(e, "velocity check", why);
}

template <int COLS>
static cudaError_t fold_one(const Plan* p, const KArgs& A, cudaStream_t s) {
  constexpr int T = 1024;
  auto kern = pstm_fold_kernel<COLS, T>;
  const int bytes = COLS * T * 8;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)p->n_tiles, (unsigned)((p->grid.n_times + T - 1) / T));
  kern<<<grid, 256, bytes, s>>>(A);
  count_launch();
  return cudaGetLastError();
}

pstm_status launch_fold(Plan* p, const float* vel, int64_t vst, int64_t vsc, float* fold,
                        cudaStream_t s, std::string* why) {
  KArgs A = make_args(p, vel, vst, vsc);
  A.out = fold;
  cudaError_t e;
  switch (p->shape.cols) {
    case 2:
      e = fold_one<2>(p, A, s);
      break;
    case 4:
      e = fold_one<4>(p, A, s);
      break;
    case 8:
      e = fold_one<8>(p, A, s);
      break;
    case 16:
      e = fold_one<16>(p, A, s);
      break;
    default:
      e = cudaErrorInvalidValue;
  }
  return e == cudaSuccess ? PSTM_OK : cuda_fail(e, "fold kernel", why);
}

}  // namespace pstm

#ifdef PSTM_CHECKED_BUILD
// The checked test build (libseispstm_checked.so: bounds checks on, 50 ms wait
// limit) exports one more entry point: the fault its kernels simulate on the
// next launches, so the tests can drive the failure paths without faulting a
// GPU -- a stage copy that is never issued (the bounded waits expire:
// PSTM_ETIMEOUT), the upper index clamp left out (staged-row reads beyond the
// row, caught by the bounds checks: PSTM_EBOUNDS), a trace-list entry out of
// range (caught before it is used: PSTM_EBOUNDS).  0 restores normal runs.
extern "C" pstm_status pstm_test_set_injection(int32_t kind) {
  if (kind < pstm::INJ_NONE || kind > pstm::INJ_BAD_LIST_ENTRY) return PSTM_EINVAL;
  pstm::g_inject.store(kind);
  return PSTM_OK;
}
#endif
