// Kirchhoff demigration: the exact transpose of the forward gather, organised
// by traces.
//
// The forward kernel owns output columns and streams traces past them; its
// transpose scatters image samples into trace samples.  Scattering from a
// column-owning CTA would leave every trace row with one partial sum per tile
// that lists it (hundreds), summed by global atomics.  Here a CTA owns up to
// 16 traces instead (fewer when rows are long): their accumulation rows stay
// in shared memory while the CTA visits every tile whose list holds one of
// them (the plan's per-trace-block tile lists, built once), and each row is
// written out once, with plain stores.  Within a tile the warps take the forward kernel's (column, time
// segment) roles and recompute exactly the forward traveltimes, masks and
// weights; per output sample pair they add g(1 - f) and g f into the two
// staged samples the forward kernel interpolates (`red.shared.add.f32`), where
// g is the image sample times the forward epilogue factor times the weight.
//
// Per-column constants come from a table built per call: for every output
// sample (z'^2, a', g, threshold) with the same arithmetic the forward kernel
// uses, laid out column-major so that a warp's 32 consecutive samples load as
// one coalesced request.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <string>

#include "pstm_gather2.cuh"

namespace pstm {
namespace {

constexpr int kAdjMaxTraces = 16;   // traces (shared-memory rows) per CTA, at most
constexpr int kAdjSmemBudget = 200 * 1024;
constexpr int kAdjGuard = 4;    // floats before each row: index -1 lands there and is dropped

__global__ void adj_pair_kernel(const int64_t* off, const int* list, int tb, uint64_t* keys) {
  const int tile = blockIdx.x;
  const int64_t a = off[tile], b = off[tile + 1];
  for (int64_t e = a + threadIdx.x; e < b; e += blockDim.x)
    keys[e] = ((uint64_t)(list[e] / tb) << 32) | (uint32_t)tile;
}

// blk_off[b] = first unique (block, tile) key of trace block b; tiles[u] = its tile.
__global__ void adj_off_kernel(const uint64_t* uniq, int64_t n_uniq, int n_blocks,
                               int64_t* blk_off, int* tiles) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n_uniq) tiles[i] = (int)(uint32_t)uniq[i];
  if (i <= n_blocks) {
    int64_t lo = 0, hi = n_uniq;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if ((int64_t)(uniq[mid] >> 32) < i)
        lo = mid + 1;
      else
        hi = mid;
    }
    blk_off[i] = lo;
  }
}

// (z'^2, a', g, threshold) per output sample, column-major: the forward kernel's
// per-lane constants and epilogue factor times the image sample.
template <int WM>
__global__ void adj_table_kernel(const KArgs A, const float* __restrict__ image,
                                 float4* __restrict__ tab) {
  const int n_c = A.n_il * A.n_xl;
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;  // image order k * n_c + c
  if (e >= (int64_t)A.n_times * n_c) return;
  const int k = (int)(e / n_c), c = (int)(e - (int64_t)k * n_c);
  const float v = vel_at(A, k, c);
  const float z = depth_of(v, out_time_ms(k, A.out_dt, A.out_t0));
  float zz = fmaf(z, z, kRadicandFloor);
  float aa = 1000.0f / (v * A.in_dt);
  float fl = 1.0f;
  if (WM == W_OBL_SPREAD || WM == W_OBL) fl = z * z;
  if constexpr (kPrescaled<OP_FWD, WM>) {
    const float a2 = __fmul_rn(aa, aa);
    zz = __fmul_rn(zz, a2);
    aa = a2;
    if (WM == W_OBL_SPREAD || WM == W_OBL) fl *= WM == W_OBL_SPREAD ? a2 * a2 : a2;
  }
  tab[(int64_t)c * A.n_times + k] = make_float4(zz, aa, image[e] * fl, threshold(A, c, k));
}

__device__ __forceinline__ void red_add(uint32_t addr, float v) {
  asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(addr), "f"(v) : "memory");
}

// Pending contributions of a lane: acc0 to sample `cur`, acc1 to `cur + 1`.
// The lane's samples are consecutive in k, so their indices mostly repeat or
// step by one; contributions are merged in registers and a shared-memory add
// is issued only when the index moves on, and only for a non-zero sum (masked
// samples carry zero weight; adding 0 leaves a float unchanged, so skipping it
// changes no result and saves the compare-and-swap loop a float add to shared
// memory compiles to).
struct AdjRun {
  uint32_t cur;  // address of sample cur
  float acc0, acc1;
};

__device__ __forceinline__ void adj_push(AdjRun& r, uint32_t a, float g0, float g1) {
  const bool same = a == r.cur;
  const bool next = a == r.cur + 4;
  if (!same && r.acc0 != 0.f) red_add(r.cur, r.acc0);
  if (!same && !next && r.acc1 != 0.f) red_add(r.cur + 4, r.acc1);
  r.acc0 = same ? r.acc0 + g0 : (next ? r.acc1 + g0 : g0);
  r.acc1 = same ? r.acc1 + g1 : g1;
  r.cur = a;
}

// One trace over a lane's 2M consecutive output samples (pairs (2i, 2i+1)):
// the forward sweep's traveltime, index and weight, then the transposed
// interpolation.  A sample contributes when h < threshold(k) -- the forward
// kernel's mask, as its thresholds are non-decreasing in k.
template <int M, int WM, bool LOWC>
__device__ __forceinline__ void adj_sweep(const f2 (&zz)[M], const f2 (&aa)[M], const f2 (&gg)[M],
                                          const f2 (&th)[M], float hs2, float hr2, float h,
                                          uint32_t rbase, f2 bb, float hi_c, float lo_c) {
  const f2 magic2 = f2_bcast(kMagic);
  const f2 hs2b = f2_bcast(hs2), hr2b = f2_bcast(hr2);
  AdjRun run;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    f2 qs, qr, id;
    if constexpr (kPrescaled<OP_FWD, WM>) {
      const f2 rrs = f2_fma(hs2b, aa[i], zz[i]);
      const f2 rrr = f2_fma(hr2b, aa[i], zz[i]);
      qs = f2{rsqrt_approx(rrs.x), rsqrt_approx(rrs.y)};
      qr = f2{rsqrt_approx(rrr.x), rsqrt_approx(rrr.y)};
      id = f2_fma(rrr, qr, f2_fma(rrs, qs, bb));
    } else {
      const f2 rrs = f2_add(hs2b, zz[i]);
      const f2 rrr = f2_add(hr2b, zz[i]);
      qs = f2{rsqrt_approx(rrs.x), rsqrt_approx(rrs.y)};
      qr = f2{rsqrt_approx(rrr.x), rsqrt_approx(rrr.y)};
      const f2 sum = f2_fma(rrr, qr, f2_mul(rrs, qs));
      id = f2_fma(sum, aa[i], bb);
    }
    id.x = fminf(id.x, hi_c);
    id.y = fminf(id.y, hi_c);
    if constexpr (LOWC) {
      id.x = fmaxf(id.x, lo_c);
      id.y = fmaxf(id.y, lo_c);
    }
    const f2 tm = f2_add_rm(id, magic2);
    const f2 fr = f2_sub(id, f2_sub(tm, magic2));
    const f2 p = f2_mul(qs, qr);
    f2 w;
    if constexpr (WM == W_OBL_SPREAD) {
      w = f2_mul(p, p);
    } else if constexpr (WM == W_OBL) {
      w = p;
    } else if constexpr (WM == W_SPREAD) {
      w = f2{p.x * rcp_approx(fmaf(1e-6f, p.x, 1.0f)), p.y * rcp_approx(fmaf(1e-6f, p.y, 1.0f))};
    } else {
      w = f2{1.0f, 1.0f};
    }
    w.x = h < th[i].x ? w.x : 0.f;
    w.y = h < th[i].y ? w.y : 0.f;
    const f2 g = f2_mul(gg[i], w);
    const f2 g1 = f2_mul(g, fr);
    const f2 g0v = f2_sub(g, g1);
    const uint32_t a0 = rbase + (__float_as_uint(tm.x) << 2);
    const uint32_t a1 = rbase + (__float_as_uint(tm.y) << 2);
    if (i == 0) {
      run.cur = a0;
      run.acc0 = g0v.x;
      run.acc1 = g1.x;
    } else {
      adj_push(run, a0, g0v.x, g1.x);
    }
    adj_push(run, a1, g0v.y, g1.y);
  }
  if (run.acc0 != 0.f) red_add(run.cur, run.acc0);
  if (run.acc1 != 0.f) red_add(run.cur + 4, run.acc1);
}

// Lane l of warp (column, segment ts) takes the 2M consecutive samples of
// chunk l * WPC + ts of each window: a column's warps interleave chunks (equal
// shares of shallow and deep samples), and the lanes of one scatter are 2M
// samples apart, so they rarely hit the same trace sample.  Warps visit the
// CTA's traces in rotated order, so two warps rarely update one row at once.
template <int COLS, int WPC, int M, int WM, bool LOWC, int MINB>
__global__ void __launch_bounds__(COLS* WPC * 32, MINB)
    pstm_adjoint_kernel(const KArgs A, const float4* __restrict__ tab,
                        const int64_t* __restrict__ blk_off, const int* __restrict__ blk_tiles,
                        int64_t n_traces, int n_windows, int tb) {
  constexpr int T = WPC * 64 * M;
  constexpr int SPL = 2 * M;  // samples per lane per window
  extern __shared__ __align__(16) float rows[];
  __shared__ float4 gsh[kAdjMaxTraces];
  const int RS = A.S + 8;  // floats per row: guard, samples, padding
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t j0 = (int64_t)blockIdx.x * tb;
  const int nt = (int)(n_traces - j0 < tb ? n_traces - j0 : tb);
  for (int e = tid; e < tb * RS; e += blockDim.x) rows[e] = 0.f;
  if (tid < nt) gsh[tid] = __ldg(A.geo + j0 + tid);
  __syncthreads();

  const int cl = warp / WPC, ts = warp % WPC;
  const f2 bb = f2_bcast(-A.in_t0 / A.in_dt);  // whole rows: no staging offset
  const float hi_c = A.clamp_hi, lo_c = 0.0f;
  const uint32_t rbase0 = smem_addr(rows) + kAdjGuard * 4 - (kMagicBits << 2);
  const int kl0 = (lane * WPC + ts) * SPL;  // first sample of this lane in a window

  const int64_t q1 = blk_off[blockIdx.x + 1];
  for (int64_t q = blk_off[blockIdx.x]; q < q1; ++q) {
    const int tile = blk_tiles[q];
    int il, xl;
    if (!tile_column(A, tile, cl, il, xl)) continue;  // warp-uniform
    const int c = il * A.n_xl + xl;
    float xc, yc;
    column_xy(A, il, xl, xc, yc);
    float hs2 = 0.f, hr2 = 0.f, hmax = 3.0e38f;
    if (lane < nt) {
      leg_h2(xc, yc, gsh[lane], hs2, hr2);
      hmax = sqrtf(fmaxf(hs2, hr2));
    }
    const float4* tc = tab + (int64_t)c * A.n_times;
    for (int win = 0; win < n_windows; ++win) {
      const int k0 = win * T;
      if (k0 + ts * SPL >= A.n_times) continue;  // warp-uniform: no sample of this warp
      f2 zz[M], aa[M], gg[M], th[M];
      float tmax = -1.0f;
#pragma unroll
      for (int i = 0; i < M; ++i) {
        // samples past the end take the last sample's constants (so their
        // indices stay inside the row) with no image value and no threshold
        const int ka = k0 + kl0 + 2 * i, kb = ka + 1;
        float4 qa = __ldg(tc + min(ka, A.n_times - 1));
        float4 qb = __ldg(tc + min(kb, A.n_times - 1));
        if (ka >= A.n_times) qa.z = 0.f, qa.w = -1.f;
        if (kb >= A.n_times) qb.z = 0.f, qb.w = -1.f;
        zz[i] = f2{qa.x, qb.x};
        aa[i] = f2{qa.y, qb.y};
        gg[i] = f2{qa.z, qb.z};
        th[i] = f2{qa.w, qb.w};
        tmax = fmaxf(tmax, fmaxf(qa.w, qb.w));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) tmax = fmaxf(tmax, __shfl_xor_sync(0xffffffffu, tmax, o));
      for (int u = 0; u < nt; ++u) {
        const int t = (u + warp) % nt;
        const float h = __shfl_sync(0xffffffffu, hmax, t);
        if (!(h < tmax)) continue;  // no contributing sample for this warp
        const float hs = __shfl_sync(0xffffffffu, hs2, t);
        const float hr = __shfl_sync(0xffffffffu, hr2, t);
        adj_sweep<M, WM, LOWC>(zz, aa, gg, th, hs, hr, h, rbase0 + (uint32_t)(t * RS * 4), bb,
                               hi_c, lo_c);
      }
    }
  }
  __syncthreads();
  // each trace row belongs to this CTA alone: plain stores
  const int ns = A.n_samples;
  for (int e = tid; e < nt * ns; e += blockDim.x) {
    const int t = e / ns, s = e - t * ns;
    A.accum[(j0 + t) * A.S + s] = rows[t * RS + kAdjGuard + s];
  }
}

template <int COLS, int WPC, int M, int WM, int MINB>
cudaError_t adj_launch(const Plan* p, const KArgs& A, const float4* tab, cudaStream_t s) {
  auto kern = needs_lowclamp(p) ? pstm_adjoint_kernel<COLS, WPC, M, WM, true, MINB>
                                : pstm_adjoint_kernel<COLS, WPC, M, WM, false, MINB>;
  const int tb = p->adj_tb;
  const int T = WPC * 64 * M;  // output samples per window of this kernel shape
  const int n_windows = (p->grid.n_times + T - 1) / T;
  const int smem = tb * (p->row_stride + 8) * (int)sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return e;
  const int64_t nb = (p->n_traces + tb - 1) / tb;
  kern<<<(unsigned)nb, COLS * WPC * 32, smem, s>>>(A, tab, p->adj_off, p->adj_tiles, p->n_traces,
                                                  n_windows, tb);
  count_launch();
  return cudaGetLastError();
}

// MINB: CTAs per SM the register budget is sized for.
template <int COLS, int WPC, int M, int MINB = 1>
cudaError_t adj_wm(const Plan* p, const KArgs& A, const float4* tab, cudaStream_t s) {
  switch (p->params.weight) {
    case W_OBL_SPREAD:
      return adj_launch<COLS, WPC, M, W_OBL_SPREAD, MINB>(p, A, tab, s);
    case W_SPREAD:
      return adj_launch<COLS, WPC, M, W_SPREAD, MINB>(p, A, tab, s);
    case W_OBL:
      return adj_launch<COLS, WPC, M, W_OBL, MINB>(p, A, tab, s);
    case W_NONE:
      return adj_launch<COLS, WPC, M, W_NONE, MINB>(p, A, tab, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t adj_dispatch(const Plan* p, const KArgs& A, const float4* tab, cudaStream_t s) {
  switch (p->shape.id) {
    case 1:
    case 5:
    case 13:
      return adj_wm<8, 2, 8>(p, A, tab, s);
    case 2:
    case 8:
      return adj_wm<4, 4, 4>(p, A, tab, s);
    case 4:
    case 6:
      return adj_wm<4, 2, 4>(p, A, tab, s);
    case 7:
      return adj_wm<2, 4, 2>(p, A, tab, s);
    case 3:
    case 9:
    case 10:
    case 11:
    case 12:
      // 16-column tiles, whatever the forward window: 4 samples per lane (128-sample windows) at 40 registers, three CTAs
      // (48 warps) per SM to hide the latency of the shared-memory adds:
      // 1.65x faster than 16 samples per lane at 128 registers and one CTA
      // per SM (two CTAs at 8 samples per lane: 1.6x)
      return adj_wm<16, 1, 2, 3>(p, A, tab, s);
  }
  return cudaErrorInvalidValue;
}

template <int WM>
cudaError_t table_launch(const KArgs& A, const float* image, float4* tab, cudaStream_t s) {
  const int64_t n = (int64_t)A.n_times * A.n_il * A.n_xl;
  adj_table_kernel<WM><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(A, image, tab);
  count_launch();
  return cudaGetLastError();
}

// Per-trace-block tile lists: unique (trace block, tile) pairs of the tile lists.
cudaError_t build_block_lists(Plan* p, cudaStream_t s) {
  int tb = kAdjMaxTraces;
  while (tb > 1 && tb * (p->row_stride + 8) * (int)sizeof(float) > kAdjSmemBudget) tb >>= 1;
  p->adj_tb = tb;
  const int64_t E = p->list_entries;
  const int64_t nb = (p->n_traces + tb - 1) / tb;
  uint64_t *keys = nullptr, *sorted = nullptr;
  int64_t* n_sel = nullptr;
  void* tmp = nullptr;
  struct Free {
    void** ptrs[4];
    cudaStream_t s;
    ~Free() {
      for (auto pp : ptrs) dev_free(*pp, s);
    }
  } fr{{(void**)&keys, (void**)&sorted, (void**)&n_sel, &tmp}, s};
  cudaError_t e;
  if ((e = dev_malloc((void**)&p->adj_off, (nb + 1) * sizeof(int64_t), s)) != cudaSuccess)
    return e;
  p->bytes += (nb + 1) * sizeof(int64_t);
  if (E == 0) {
    p->n_adj_tiles = 0;
    return cudaMemsetAsync(p->adj_off, 0, (nb + 1) * sizeof(int64_t), s);
  }
  if (E > INT32_MAX) return cudaErrorInvalidValue;
  if ((e = dev_malloc((void**)&keys, E * sizeof(uint64_t), s)) != cudaSuccess) return e;
  if ((e = dev_malloc((void**)&sorted, E * sizeof(uint64_t), s)) != cudaSuccess) return e;
  if ((e = dev_malloc((void**)&n_sel, sizeof(int64_t), s)) != cudaSuccess) return e;
  adj_pair_kernel<<<(unsigned)p->n_tiles, 256, 0, s>>>(p->tile_off, p->tile_list, tb, keys);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  int end_bit = 32;
  while (end_bit < 64 && (uint64_t(1) << (end_bit - 32)) <= (uint64_t)nb) ++end_bit;
  size_t sort_bytes = 0, uniq_bytes = 0;
  e = cub::DeviceRadixSort::SortKeys(nullptr, sort_bytes, keys, sorted, (int)E, 0, end_bit, s);
  if (e != cudaSuccess) return e;
  e = cub::DeviceSelect::Unique(nullptr, uniq_bytes, sorted, keys, n_sel, (int)E, s);
  if (e != cudaSuccess) return e;
  if ((e = dev_malloc(&tmp, std::max(sort_bytes, uniq_bytes), s)) != cudaSuccess) return e;
  e = cub::DeviceRadixSort::SortKeys(tmp, sort_bytes, keys, sorted, (int)E, 0, end_bit, s);
  if (e != cudaSuccess) return e;
  e = cub::DeviceSelect::Unique(tmp, uniq_bytes, sorted, keys, n_sel, (int)E, s);
  if (e != cudaSuccess) return e;
  int64_t n_uniq = 0;
  e = cudaMemcpyAsync(&n_uniq, n_sel, sizeof(int64_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return e;
  if ((e = dev_malloc((void**)&p->adj_tiles, std::max<int64_t>(n_uniq, 1) * sizeof(int), s)) !=
      cudaSuccess)
    return e;
  p->bytes += std::max<int64_t>(n_uniq, 1) * sizeof(int);
  p->n_adj_tiles = n_uniq;
  const int64_t n_thr = std::max<int64_t>(n_uniq, nb + 1);
  adj_off_kernel<<<(unsigned)((n_thr + 255) / 256), 256, 0, s>>>(keys, n_uniq, (int)nb, p->adj_off,
                                                                 p->adj_tiles);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  count_launch();
  return cudaStreamSynchronize(s);
}

}  // namespace

pstm_status launch_adjoint(Plan* p, const float* image, const float* vel, int64_t vst,
                           int64_t vsc, cudaStream_t s, std::string* why) {
  cudaError_t e = cudaSuccess;
  if (!p->adj_off) {
    e = build_block_lists(p, s);
    if (e != cudaSuccess) {
      dev_free(p->adj_off, s);
      dev_free(p->adj_tiles, s);
      p->adj_off = nullptr;
      p->adj_tiles = nullptr;
      return cuda_fail(e, "adjoint trace-block lists", why);
    }
  }
  const size_t tab_elems = (size_t)p->grid.n_times * p->grid.n_il * p->grid.n_xl;
  if (!p->adj_table) {
    e = dev_malloc((void**)&p->adj_table, tab_elems * sizeof(float4), s);
    if (e != cudaSuccess) {
      p->adj_table = nullptr;
      return cuda_fail(e, "adjoint column table", why);
    }
    p->bytes += (int64_t)(tab_elems * sizeof(float4));
  }
  KArgs A = make_args(p, vel, vst, vsc);
  A.in_img = image;
  switch (p->params.weight) {
    case W_OBL_SPREAD:
      e = table_launch<W_OBL_SPREAD>(A, image, p->adj_table, s);
      break;
    case W_SPREAD:
      e = table_launch<W_SPREAD>(A, image, p->adj_table, s);
      break;
    case W_OBL:
      e = table_launch<W_OBL>(A, image, p->adj_table, s);
      break;
    default:
      e = table_launch<W_NONE>(A, image, p->adj_table, s);
  }
  if (e == cudaSuccess && p->n_traces > 0) e = adj_dispatch(p, A, p->adj_table, s);
  return e == cudaSuccess ? PSTM_OK : cuda_fail(e, "adjoint kernel", why);
}

}  // namespace pstm
