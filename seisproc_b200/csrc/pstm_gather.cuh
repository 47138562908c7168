// Gather-kernel template shared by the forward, adjoint and V-gradient
// translation units (each instantiates one op, so they compile in parallel).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <type_traits>

#include "pstm_common.cuh"
#include "pstm_internal.h"

namespace pstm {

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
  const float* in_img;
  float* accum;
  int* err;
  int ring_stages, ring_rows;  // pipelined kernel: stages x rows per stage
  // anti-alias: output spacing (m) per axis, max half-width (samples), row pad
  float aa_dx, aa_dy, aa_lmax;
  int aa_pad;
};

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

template <int COLS, int WPC, int M>
struct Geom {
  static constexpr int NW = COLS * WPC;
  static constexpr int NT = NW * 32;
  static constexpr int T = WPC * 64 * M;
  static constexpr int B = kBlockTraces;
};

// Shared-memory carve-up (bytes), identical for every op.
struct SmemLayout {
  int setup, thr, jj, raw, exp, total;
};
__host__ __device__ inline SmemLayout smem_layout(int cols, int T, int S, int elt, int op) {
  SmemLayout L;
  int o = 16;  // mbarrier
  L.setup = o;
  o += cols * kBlockTraces * 16;
  L.thr = o;
  o += cols * T * 4;
  L.jj = o;
  o += 2 * kBlockTraces * 4;
  o = (o + 127) & ~127;
  L.raw = o;
  if (op != OP_ADJ) o += kBlockTraces * S * elt;
  o = (o + 127) & ~127;
  L.exp = o;
  o += kBlockTraces * (S + kGuard + 2) * (op == OP_ADJ ? 4 : 8);
  L.total = o;
  return L;
}

// ---------------------------------------------------------------------------
// Forward / adjoint / V-gradient gather kernel.
// ---------------------------------------------------------------------------
template <int COLS, int WPC, int M, typename ST, int WM, bool LOWCLAMP, int OP>
__global__ void __launch_bounds__(COLS* WPC * 32, 1) pstm_gather_kernel(const KArgs A) {
  using G = Geom<COLS, WPC, M>;
  constexpr int B = G::B;
  constexpr int T = G::T;
  extern __shared__ __align__(128) unsigned char smem[];
  const int S = A.S;
  const int E = S + kGuard + 2;  // expanded entries per trace row
  const SmemLayout L = smem_layout(COLS, T, S, (int)sizeof(ST), OP);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem);
  float4* setup = reinterpret_cast<float4*>(smem + L.setup);
  float* thr = reinterpret_cast<float*>(smem + L.thr);
  int* jjs = reinterpret_cast<int*>(smem + L.jj);
  ST* raw = reinterpret_cast<ST*>(smem + L.raw);
  float2* exps = reinterpret_cast<float2*>(smem + L.exp);     // forward / vgrad
  float* tacc = reinterpret_cast<float*>(smem + L.exp);       // adjoint
  __shared__ int abort_flag;

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int tile = blockIdx.x;
  const int k0 = blockIdx.y * T;
  const int kend = min(k0 + T, A.n_times);
  const int nk = kend - k0;
  const int cl = warp / WPC, ts = warp % WPC;
  int il, xl;
  const bool col_ok = tile_column(A, tile, cl, il, xl);
  const int c = il * A.n_xl + xl;
  float xc = 0.f, yc = 0.f;
  if (col_ok) column_xy(A, il, xl, xc, yc);
  const int n_c = A.n_il * A.n_xl;

  if (tid == 0) {
    abort_flag = 0;
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  // threshold table for this window
  for (int e = tid; e < COLS * T; e += G::NT) {
    const int q = e / T, kk = e - q * T;
    int qil, qxl;
    float v = -1.0f;
    if (kk < nk && tile_column(A, tile, q, qil, qxl)) v = threshold(A, qil * A.n_xl + qxl, k0 + kk);
    thr[e] = v;
  }

  // per-lane output-sample constants: z^2 + floor (radicand), a = 1000/(V dt_in)
  const int kw = k0 + ts * 64 * M;
  f2 zz[M], aa[M], acc[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int klo = kw + 64 * i + lane, khi = klo + 32;
    const int kl = min(klo, A.n_times - 1), kh = min(khi, A.n_times - 1);
    const int cc = col_ok ? c : 0;
    const float vl = vel_at(A, kl, cc), vh = vel_at(A, kh, cc);
    const float zl = depth_of(vl, out_time_ms(kl, A.out_dt, A.out_t0));
    const float zh = depth_of(vh, out_time_ms(kh, A.out_dt, A.out_t0));
    zz[i] = f2{fmaf(zl, zl, kRadicandFloor), fmaf(zh, zh, kRadicandFloor)};
    aa[i] = f2{1000.0f / (vl * A.in_dt), 1000.0f / (vh * A.in_dt)};
    acc[i] = f2{0.f, 0.f};
    if (OP == OP_ADJ) {
      // image value times the per-sample weight factor that the forward kernel
      // applies in its epilogue
      float ml = 0.f, mh = 0.f;
      if (col_ok && klo < A.n_times) ml = A.in_img[(long long)klo * n_c + c];
      if (col_ok && khi < A.n_times) mh = A.in_img[(long long)khi * n_c + c];
      if (WM == W_OBL_SPREAD || WM == W_OBL) {
        ml *= zl * zl;
        mh *= zh * zh;
      }
      acc[i] = f2{ml, mh};
    }
  }

  const int align = Storage<ST>::kAlign;
  const int lo = window_lo(A, k0, align);
  const int rowlen = S - lo;                      // staged elements per trace
  const int nent = (A.n_samples - lo) + kGuard;   // expanded entries used
  const float bias = (float)(kGuard - lo);
  const float bconst = -A.in_t0 / A.in_dt + bias;
  const float hi_c = A.clamp_hi + bias;
  const float lo_c = bias;  // idx >= 0
  const int64_t off0 = A.off[tile];
  const int n_list = (int)(A.off[tile + 1] - off0);
  const int nb = (n_list + B - 1) / B;

  __syncthreads();

  auto issue = [&](int b) {
    const int cnt = min(B, n_list - b * B);
    int* jb = jjs + (b & 1) * B;
    for (int t = 0; t < cnt; ++t) jb[t] = A.list[off0 + (int64_t)b * B + t];
    if (OP != OP_ADJ) {
      const uint32_t bytes = (uint32_t)(rowlen * (int)sizeof(ST));
      mbar_arrive_expect_tx(bar, bytes * cnt);
      const ST* src = reinterpret_cast<const ST*>(A.traces);
      for (int t = 0; t < cnt; ++t)
        bulk_g2s(raw + t * S, src + (int64_t)jb[t] * S + lo, bytes, bar);
    }
  };

  if (tid == 0 && nb > 0) issue(0);

  const f2 magic2 = f2_bcast(kMagic);
  const f2 bb = f2_bcast(bconst);

  for (int b = 0; b < nb; ++b) {
    const int cnt = min(B, n_list - b * B);
    const int* jb = jjs + (b & 1) * B;
    if (OP != OP_ADJ) {
      if (tid == 0) {
        if (!mbar_wait(bar, b & 1)) {
          set_error(A.err, PSTM_ERR_TIMEOUT);
          mbar_wait(bar, b & 1);  // give the copy in flight one more bounded chance
          abort_flag = 1;
        }
      }
      __syncthreads();
      if (abort_flag) return;
      // expand rows into (x[i], x[i+1]-x[i]) entries, guards hold x[lo]
      for (int e = tid; e < cnt * nent; e += G::NT) {
        const int t = e / nent, q = e - t * nent;
        const ST* row = raw + t * S;
        const float sc = A.scales ? __ldg(A.scales + jb[t]) : 1.0f;
        float a, d;
        if (q < kGuard) {
          a = Storage<ST>::load(row, 0) * sc;
          d = 0.f;
        } else {
          const int i = q - kGuard;  // staged position; sample lo + i
          a = Storage<ST>::load(row, i) * sc;
          d = (lo + i + 1 < A.n_samples) ? Storage<ST>::load(row, i + 1) * sc - a : 0.f;
        }
        exps[t * E + q] = make_float2(a, d);
      }
    } else {
      for (int e = tid; e < cnt * E; e += G::NT) tacc[e] = 0.f;
    }
    // per (column, trace): leg distances and first contributing sample
    for (int e = tid; e < COLS * cnt; e += G::NT) {
      const int q = e / cnt, t = e - q * cnt;
      int qil, qxl;
      float hs2 = 0.f, hr2 = 0.f;
      int ks = kend;
      if (tile_column(A, tile, q, qil, qxl)) {
        float qx, qy;
        column_xy(A, qil, qxl, qx, qy);
        leg_h2(qx, qy, __ldg(A.geo + jb[t]), hs2, hr2);
        ks = k0 + first_valid(thr + q * T, nk, sqrtf(fmaxf(hs2, hr2)));
      }
      setup[q * B + t] = make_float4(hs2, hr2, __int_as_float(ks), 0.f);
    }
    __syncthreads();
    if (tid == 0 && b + 1 < nb) {
      if (OP != OP_ADJ) fence_proxy_async();
      issue(b + 1);  // next block's trace indices (+ its bulk copies)
    }

    if (col_ok) {
      // One straight-line sweep over all M groups per trace (no branch between
      // groups, so the compiler can interleave their MUFU/LDS chains).  Traces
      // whose first contributing sample lies inside this warp's range take the
      // masked sweep; samples before k_start get weight 0.
      for (int t = 0; t < cnt; ++t) {
        const float4 su = setup[cl * B + t];
        const int ks = __float_as_int(su.z);
        if (ks >= kw + 64 * M) continue;
        const uint32_t ebase =
            (OP == OP_ADJ ? smem_addr(tacc + t * E) - (kMagicBits << 2)
                          : smem_addr(exps + t * E) - (kMagicBits << 3));
        const f2 hs2b = f2_bcast(su.x), hr2b = f2_bcast(su.y);
        auto sweep = [&](auto masked_tag) {
          constexpr bool MASKED = decltype(masked_tag)::value;
#pragma unroll
          for (int i = 0; i < M; ++i) {
            const f2 rrs = f2_add(hs2b, zz[i]);
            const f2 rrr = f2_add(hr2b, zz[i]);
            const f2 qs = f2{rsqrt_approx(rrs.x), rsqrt_approx(rrs.y)};
            const f2 qr = f2{rsqrt_approx(rrr.x), rsqrt_approx(rrr.y)};
            const f2 sum = f2_fma(rrr, qr, f2_mul(rrs, qs));
            f2 id = f2_fma(sum, aa[i], bb);
            const f2 id_raw = id;
            id.x = fminf(id.x, hi_c);
            id.y = fminf(id.y, hi_c);
            if (LOWCLAMP) {
              id.x = fmaxf(id.x, lo_c);
              id.y = fmaxf(id.y, lo_c);
            }
            const f2 tm = f2_add_rm(id, magic2);
            const f2 fr = f2_sub(id, f2_sub(tm, magic2));
            const f2 p = f2_mul(qs, qr);
            f2 w;  // weight without the per-sample z^2 factor
            if (WM == W_OBL_SPREAD) {
              w = f2_mul(p, p);
            } else if (WM == W_OBL) {
              w = p;
            } else if (WM == W_SPREAD) {
              w = f2{p.x * rcp_approx(fmaf(1e-6f, p.x, 1.0f)),
                     p.y * rcp_approx(fmaf(1e-6f, p.y, 1.0f))};
            } else {
              w = f2{1.0f, 1.0f};
            }
            if constexpr (MASKED) {
              const int klo = kw + 64 * i + lane;
              w.x = klo >= ks ? w.x : 0.f;
              w.y = klo + 32 >= ks ? w.y : 0.f;
            }
            if (OP == OP_FWD) {
              const f2 e0 = lds_f2(ebase + (__float_as_uint(tm.x) << 3));
              const f2 e1 = lds_f2(ebase + (__float_as_uint(tm.y) << 3));
              const f2 amp = f2{fmaf(fr.x, e0.y, e0.x), fmaf(fr.y, e1.y, e1.x)};
              acc[i] = f2_fma(amp, w, acc[i]);
            } else if (OP == OP_ADJ) {
              const f2 g = f2_mul(acc[i], w);
              const uint32_t a0 = ebase + (__float_as_uint(tm.x) << 2);
              const uint32_t a1 = ebase + (__float_as_uint(tm.y) << 2);
              const float g0 = g.x * fr.x, g1 = g.y * fr.y;
              asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a0), "f"(g.x - g0) : "memory");
              asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a0 + 4), "f"(g0) : "memory");
              asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a1), "f"(g.y - g1) : "memory");
              asm volatile("red.shared.add.f32 [%0], %1;" ::"r"(a1 + 4), "f"(g1) : "memory");
            } else {  // OP_VGRAD (obliquity x spreading)
              const f2 e0 = lds_f2(ebase + (__float_as_uint(tm.x) << 3));
              const f2 e1 = lds_f2(ebase + (__float_as_uint(tm.y) << 3));
              const f2 amp = f2{fmaf(fr.x, e0.y, e0.x), fmaf(fr.y, e1.y, e1.x)};
              // slope of the interpolant in samples; zero where the index is clamped
              const f2 slope = f2{(id_raw.x < hi_c && id_raw.x > lo_c) ? e0.y : 0.f,
                                  (id_raw.y < hi_c && id_raw.y > lo_c) ? e1.y : 0.f};
              const f2 q2 = f2_fma(qs, qs, f2_mul(qr, qr));
              const f2 one_m = f2_sub(f2_bcast(1.0f), f2_mul(zz[i], q2));
              const f2 hq = f2_fma(hs2b, qs, f2_mul(hr2b, qr));
              // 2 amp (1 - z^2 (qs^2 + qr^2)) - slope a (hs^2 qs + hr^2 qr)
              const f2 term = f2_sub(f2_mul(f2_bcast(2.0f), f2_mul(amp, one_m)),
                                     f2_mul(f2_mul(slope, aa[i]), hq));
              acc[i] = f2_fma(term, w, acc[i]);
            }
          }
        };
        if (ks <= kw)
          sweep(std::false_type{});
        else
          sweep(std::true_type{});
      }
    }
    __syncthreads();
    if (OP == OP_ADJ) {
      // flush the block's trace accumulators into the sorted trace rows;
      // entries below the first staged sample stand for x[0]
      for (int e = tid; e < cnt * nent; e += G::NT) {
        const int t = e / nent, q = e - t * nent;
        float v = tacc[t * E + q];
        int smp;
        if (q < kGuard) {
          smp = lo;  // guards are only ever hit when lo == 0
        } else {
          smp = lo + q - kGuard;
        }
        if (v != 0.f && smp < A.n_samples) atomicAdd(A.accum + (int64_t)jb[t] * S + smp, v);
      }
      __syncthreads();
    }
  }

  if (OP == OP_ADJ || !col_ok) return;
  const int n_c2 = n_c;
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int klo = kw + 64 * i + lane, khi = klo + 32;
    float fl = 1.f, fh = 1.f;
    if (WM == W_OBL_SPREAD || WM == W_OBL || OP == OP_VGRAD) {
      const int kl = min(klo, A.n_times - 1), kh = min(khi, A.n_times - 1);
      const float vl = vel_at(A, kl, c), vh = vel_at(A, kh, c);
      const float zl = depth_of(vl, out_time_ms(kl, A.out_dt, A.out_t0));
      const float zh = depth_of(vh, out_time_ms(kh, A.out_dt, A.out_t0));
      fl = zl * zl;
      fh = zh * zh;
      if (OP == OP_VGRAD) {
        fl = klo < A.n_times ? fl / vl * A.in_img[(long long)klo * n_c2 + c] : 0.f;
        fh = khi < A.n_times ? fh / vh * A.in_img[(long long)khi * n_c2 + c] : 0.f;
      }
    }
    if (klo < A.n_times) A.out[(long long)klo * n_c2 + c] = acc[i].x * fl;
    if (khi < A.n_times) A.out[(long long)khi * n_c2 + c] = acc[i].y * fh;
  }
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
  A.in_img = nullptr;
  A.accum = p->accum;
  A.err = p->err;
  A.ring_stages = A.ring_rows = 0;
  A.aa_dx = (float)p->params.aa_dx;
  A.aa_dy = (float)p->params.aa_dy;
  A.aa_lmax = (float)p->params.aa_max_halfwidth;
  A.aa_pad = p->aa_pad;
  return A;
}

template <int COLS, int WPC, int M, typename ST, int WM, bool LC, int OP>
inline cudaError_t launch_one(const Plan* p, const KArgs& A, cudaStream_t s) {
  auto kern = pstm_gather_kernel<COLS, WPC, M, ST, WM, LC, OP>;
  const int T = WPC * 64 * M;
  const SmemLayout L = smem_layout(COLS, T, p->row_stride, (int)sizeof(ST), OP);
  cudaError_t e =
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)p->n_tiles, (unsigned)((p->grid.n_times + T - 1) / T));
  kern<<<grid, COLS * WPC * 32, L.total, s>>>(A);
  count_launch();
  return cudaGetLastError();
}

template <int COLS, int WPC, int M, typename ST, int OP>
inline cudaError_t dispatch_wm(const Plan* p, const KArgs& A, bool lowclamp, cudaStream_t s) {
  const int wm = p->params.weight;
  if constexpr (OP == OP_VGRAD || !std::is_same<ST, float>::value) {
    // 16-bit storage and the velocity gradient are built for the reference
    // weight only
    if (wm != W_OBL_SPREAD) return cudaErrorNotSupported;
    return lowclamp ? launch_one<COLS, WPC, M, ST, W_OBL_SPREAD, true, OP>(p, A, s)
                    : launch_one<COLS, WPC, M, ST, W_OBL_SPREAD, false, OP>(p, A, s);
  } else {
#define PSTM_WM(W)                                                          \
  if (wm == W)                                                              \
    return lowclamp ? launch_one<COLS, WPC, M, ST, W, true, OP>(p, A, s)    \
                    : launch_one<COLS, WPC, M, ST, W, false, OP>(p, A, s);
  PSTM_WM(W_OBL_SPREAD)
  PSTM_WM(W_SPREAD)
  PSTM_WM(W_OBL)
  PSTM_WM(W_NONE)
#undef PSTM_WM
    return cudaErrorInvalidValue;
  }
}

template <int COLS, int WPC, int M, int OP>
inline cudaError_t dispatch_st(const Plan* p, const KArgs& A, bool lowclamp, cudaStream_t s) {
  if constexpr (OP == OP_ADJ) {
    return dispatch_wm<COLS, WPC, M, float, OP>(p, A, lowclamp, s);
  } else {
    switch (p->params.storage) {
      case PSTM_F32:
        return dispatch_wm<COLS, WPC, M, float, OP>(p, A, lowclamp, s);
      case PSTM_BF16:
        return dispatch_wm<COLS, WPC, M, __nv_bfloat16, OP>(p, A, lowclamp, s);
      case PSTM_F16:
        return dispatch_wm<COLS, WPC, M, __half, OP>(p, A, lowclamp, s);
    }
    return cudaErrorInvalidValue;
  }
}

template <int OP>
inline cudaError_t dispatch_shape(const Plan* p, const KArgs& A, bool lowclamp, cudaStream_t s) {
  switch (p->shape.id) {
    case 1:
    case 5:
      return dispatch_st<8, 2, 8, OP>(p, A, lowclamp, s);
    case 2:
    case 8:
      return dispatch_st<4, 4, 4, OP>(p, A, lowclamp, s);
    case 4:
    case 6:
      return dispatch_st<4, 2, 4, OP>(p, A, lowclamp, s);
    case 7:
      return dispatch_st<2, 4, 2, OP>(p, A, lowclamp, s);
  }
  return cudaErrorInvalidValue;
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
