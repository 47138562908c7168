// Warp-specialised gather kernel (forward migration and V-gradient).
//
// The rows of the tile's trace list stream through a ring of up to 4
// shared-memory stages (up to 32 rows each) by 1-D TMA bulk copies issued by
// warp 0 (one row per lane); `full[s]` completes on the copies' byte count, `empty[s]`
// when every warp has finished the stage.  Warps never synchronise with each
// other otherwise (warp 0 waits on `empty` before refilling): each one computes
// the per-(column, trace) set-up for 32 list entries at a time (one lane per
// trace: leg distances and the first contributing sample by binary search in
// the CTA's threshold table), then sweeps the traces, taking each trace's
// set-up from its lane by shuffle.  Samples are read straight from the staged
// row: float32 rows hold expanded (x[i], x[i+1] - x[i]) entries (one 8-byte
// load per sample), the anti-alias integral rows each linear piece as intercept
// and slope in the index frame (one load and one FMA per tap), 16-bit rows
// plain samples (two loads and a lerp).
#pragma once
#include "pstm_gather.cuh"

namespace pstm {

constexpr int kMaxStages = 4;
// Every staged row is preceded by 16 zero bytes, so an index in (-1, 0) -- an
// output time equal to the first input time, rounded -- reads x[-1] = 0 with
// weight (1 - f) ~ 0 instead of leaving the row.
constexpr int kRowGuard = 16;
constexpr int kSmemBudget = 227 * 1024;

// CTAs per SM a kernel shape is built for: 256-thread CTAs run two per SM
// (128 registers each, half the shared-memory ring each), so one CTA's stage
// waits overlap the other's sweeps; 512-thread CTAs run one.
__host__ __device__ constexpr int ctas_per_sm(int threads) { return threads <= 256 ? 2 : 1; }
// Dynamic shared memory one CTA of the shape may take (the SM's 228 KB shared
// by its CTAs, less the 1 KB the hardware reserves per CTA).
__host__ __device__ constexpr int smem_budget(int threads) {
  return ctas_per_sm(threads) == 1 ? kSmemBudget : (228 * 1024) / 2 - 1024;
}

struct Smem2 {
  int bars, thr, hist, raw, total;
};
// Bytes per fold-histogram entry: 16-bit counts when every tile list is
// shorter than 65536 traces (no count can exceed its list's length).
inline int hist_entry_bytes(bool hist16) { return hist16 ? 2 : 4; }
// Ring of `stages` stages of `sb` trace rows each; `hb` bytes per fold
// histogram entry.
__host__ __device__ inline Smem2 smem2_layout(int cols, int T, int S, int elt, int stages, int sb,
                                              int hb = 4) {
  Smem2 L;
  int o = 0;
  L.bars = o;
  o += 2 * kMaxStages * 8 + 16;
  o = (o + 15) & ~15;
  L.thr = o;
  o += cols * T * 4;
  L.hist = o;  // fold histogram of first contributing samples
  o += cols * T * hb;
  o = (o + 127) & ~127;
  L.raw = o;
  o += stages * sb * (S * elt + kRowGuard);
  L.total = o;
  return L;
}

// Ring of the largest stages (up to 32 rows), then the most stages (up to 4,
// at least 2), that fits: large stages measured faster than deeper rings of
// smaller ones (fewer barrier round trips per trace; on the 3D workload 2 x 10
// rows ran 1 % faster than 2 x 8 and 3 x 8 slower than 2 x 8).  Stage sizes
// other than 1 are even, so a stage's traces are always swept in pairs.
inline bool ring_shape(int cols, int T, int S, int elt, int* stages, int* sb,
                       int budget = kSmemBudget, int hb = 4) {
  static_assert(kBlockTraces == 32, "one bulk copy per lane of warp 0");
  static const int kRows[] = {32, 24, 16, 12, 10, 8, 6, 4, 2, 1};
  for (const int b : kRows)
    for (int st = kMaxStages; st >= 2; --st)
      if (smem2_layout(cols, T, S, elt, st, b, hb).total <= budget) {
        *stages = st;
        *sb = b;
        return true;
      }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Forward sweeps with a weight that is a power of p = q_s q_r (or none) run on
// traveltimes pre-scaled by the index scale a = 1000 / (V dt): the per-sample
// tables hold a^2 (z^2 + eps) and a^2 and the power of a comes back in the
// epilogue, which saves an FP32 op per sample pair.
template <int OP, int WM>
constexpr bool kPrescaled = OP == OP_FWD && (WM == W_OBL_SPREAD || WM == W_OBL || WM == W_NONE);

template <typename ST>
__device__ __forceinline__ float lds_elem(uint32_t addr);
template <>
__device__ __forceinline__ float lds_elem<float>(uint32_t addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(addr));
  return v;
}
template <>
__device__ __forceinline__ float lds_elem<__nv_bfloat16>(uint32_t addr) {
  unsigned short h;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(h) : "r"(addr));
  return __uint_as_float(((uint32_t)h) << 16);
}
template <>
__device__ __forceinline__ float lds_elem<__half>(uint32_t addr) {
  unsigned short h;
  asm volatile("ld.shared.u16 %0, [%1];" : "=h"(h) : "r"(addr));
  return __half2float(__ushort_as_half(h));
}

// One straight-line sweep over the M sample groups of a warp for NTR traces at
// once (their dependency chains interleave).  Per trace n: squared leg
// distances hs2[n], hr2[n], the shared-memory address of its staged row minus
// the bit pattern of 2^23 (so the index's float bits address the sample), its
// first contributing sample kst[n] (samples before it get weight 0 when
// MASKED) and, for f16 storage, its scale.  A MASKED sweep starts at group g0,
// the first 64-sample group holding a contributing sample of any of its traces
// (warp-uniform, so the skipped groups cost one uniform branch each).
template <int M, typename ST, int WM, bool LOWC, bool MASKED, int OP, int NTR, bool TAPER,
          bool CURVED = false>
__device__ __forceinline__ void sweep_traces(f2 (&acc)[M], const f2 (&zz)[M], const f2 (&aa)[M],
                                             const float (&hs2)[NTR], const float (&hr2)[NTR],
                                             const uint32_t (&rbase)[NTR], const int (&kst)[NTR],
                                             const float (&sc)[NTR], f2 bb, f2 magic2,
                                             float hi_c, float lo_c, int kw, int lane, int g0,
                                             const TaperArgs& tp, float cr_scale = 0.f,
                                             RowCheck rc = RowCheck{}) {
  // curved rays: zz = z^2 + f, aa = k / (2 v0 max(z, 1e-6)); no pre-scaling
  constexpr bool PRE = kPrescaled<OP, WM> && !CURVED;
  constexpr int ES = (int)sizeof(ST);
  constexpr int SHIFT = ES == 8 ? 3 : (ES == 4 ? 2 : 1);
#pragma unroll
  for (int i = 0; i < M; ++i) {
    if constexpr (MASKED) {
      if (i < g0) continue;
    }
#pragma unroll
    for (int n = 0; n < NTR; ++n) {
      const f2 hs2b = f2_bcast(hs2[n]), hr2b = f2_bcast(hr2[n]);
      f2 rrs, rrr, qs, qr, id;
      if constexpr (CURVED) {
        // one-way times in v(z) = v0 + k z: arccosh(1 + k r^2 / (2 v0 z)) / k
        rrs = f2_add(hs2b, zz[i]);
        rrr = f2_add(hr2b, zz[i]);
        qs = f2{rsqrt_approx(rrs.x), rsqrt_approx(rrs.y)};
        qr = f2{rsqrt_approx(rrr.x), rsqrt_approx(rrr.y)};
        const f2 xs = f2_fma(rrs, aa[i], f2_bcast(1.0f));
        const f2 xr = f2_fma(rrr, aa[i], f2_bcast(1.0f));
        const f2 tt = f2{acoshf(fmaxf(xs.x, 1.0f)) + acoshf(fmaxf(xr.x, 1.0f)),
                         acoshf(fmaxf(xs.y, 1.0f)) + acoshf(fmaxf(xr.y, 1.0f))};
        id = f2_fma(tt, f2_bcast(cr_scale), bb);
      } else if constexpr (PRE) {
        // zz = a^2 (z^2 + eps), aa = a^2: rr' = a^2 rr, q' = q / a, and
        // rr'_s q'_s + rr'_r q'_r = a (r_s + r_r), the index less its offset
        rrs = f2_fma(hs2b, aa[i], zz[i]);
        rrr = f2_fma(hr2b, aa[i], zz[i]);
        qs = f2{rsqrt_approx(rrs.x), rsqrt_approx(rrs.y)};
        qr = f2{rsqrt_approx(rrr.x), rsqrt_approx(rrr.y)};
        id = f2_fma(rrr, qr, f2_fma(rrs, qs, bb));
      } else {
        rrs = f2_add(hs2b, zz[i]);
        rrr = f2_add(hr2b, zz[i]);
        qs = f2{rsqrt_approx(rrs.x), rsqrt_approx(rrs.y)};
        qr = f2{rsqrt_approx(rrr.x), rsqrt_approx(rrr.y)};
        const f2 sum = f2_fma(rrr, qr, f2_mul(rrs, qs));
        id = f2_fma(sum, aa[i], bb);
      }
      const f2 id_raw = id;
      id.x = fminf(id.x, hi_c);
      id.y = fminf(id.y, hi_c);
      if constexpr (LOWC) {
        id.x = fmaxf(id.x, lo_c);
        id.y = fmaxf(id.y, lo_c);
      }
      const f2 tm = f2_add_rm(id, magic2);
      const uint32_t a0 = checked_addr(rbase[n] + (__float_as_uint(tm.x) << SHIFT),
                                       __float_as_uint(tm.x), rbase[n], SHIFT, rc);
      const uint32_t a1 = checked_addr(rbase[n] + (__float_as_uint(tm.y) << SHIFT),
                                       __float_as_uint(tm.y), rbase[n], SHIFT, rc);
      f2 dx, amp;
      if constexpr (std::is_same<ST, float2>::value) {
        // expanded rows: one 8-byte load gives (x[i0], x[i0+1] - x[i0])
        const f2 fr = f2_sub(id, f2_sub(tm, magic2));
        const f2 e0 = lds_f2(a0), e1 = lds_f2(a1);
        dx = f2{e0.y, e1.y};
        amp = f2{fmaf(fr.x, e0.y, e0.x), fmaf(fr.y, e1.y, e1.x)};
      } else if constexpr (std::is_same<ST, RowIcpt>::value) {
        // intercept rows (id is the entry coordinate less q0): one FMA per tap
        const f2 e0 = lds_f2(a0), e1 = lds_f2(a1);
        dx = f2{e0.y, e1.y};
        amp = f2{fmaf(id.x, e0.y, e0.x), fmaf(id.y, e1.y, e1.x)};
      } else {
        const f2 fr = f2_sub(id, f2_sub(tm, magic2));
        const f2 x0 = f2{lds_elem<ST>(a0), lds_elem<ST>(a1)};
        const f2 x1 = f2{lds_elem<ST>(a0 + ES), lds_elem<ST>(a1 + ES)};
        dx = f2_sub(x1, x0);
        amp = f2_fma(fr, dx, x0);
      }
      const f2 p = f2_mul(qs, qr);
      if constexpr (PRE) {
        // weight p^2 (obliquity x spreading; the a^4 z^2 factor comes in the
        // epilogue), p (obliquity) or 1; formed while the taps load
        f2 w = p;
        if constexpr (WM == W_OBL_SPREAD) w = f2_mul(p, p);
        if constexpr (WM == W_NONE) w = f2_bcast(1.0f);
        // per-trace factor: f16 scale, or the distance tapers of both legs
        if constexpr (std::is_same<ST, __half>::value || TAPER) w = f2_mul(w, f2_bcast(sc[n]));
        if constexpr (TAPER) {
          w.x *= leg_angle_taper<true>(hs2[n], zz[i].x, aa[i].x, tp) *
                 leg_angle_taper<true>(hr2[n], zz[i].x, aa[i].x, tp);
          w.y *= leg_angle_taper<true>(hs2[n], zz[i].y, aa[i].y, tp) *
                 leg_angle_taper<true>(hr2[n], zz[i].y, aa[i].y, tp);
        }
        if constexpr (MASKED) {
          const int klo = kw + 64 * i + lane;
          w.x = klo >= kst[n] ? w.x : 0.f;
          w.y = klo + 32 >= kst[n] ? w.y : 0.f;
        }
        acc[i] = f2_fma(amp, w, acc[i]);
        continue;
      }
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
      if constexpr (std::is_same<ST, __half>::value || TAPER) w = f2_mul(w, f2_bcast(sc[n]));
      if constexpr (TAPER) {
        w.x *= leg_angle_taper<false>(hs2[n], zz[i].x, aa[i].x, tp) *
               leg_angle_taper<false>(hr2[n], zz[i].x, aa[i].x, tp);
        w.y *= leg_angle_taper<false>(hs2[n], zz[i].y, aa[i].y, tp) *
               leg_angle_taper<false>(hr2[n], zz[i].y, aa[i].y, tp);
      }
      if constexpr (MASKED) {
        const int klo = kw + 64 * i + lane;
        w.x = klo >= kst[n] ? w.x : 0.f;
        w.y = klo + 32 >= kst[n] ? w.y : 0.f;
      }
      if constexpr (OP == OP_FWD) {
        acc[i] = f2_fma(amp, w, acc[i]);
      } else {  // OP_VGRAD
        const f2 slope = f2{(id_raw.x < hi_c && id_raw.x > lo_c) ? dx.x : 0.f,
                            (id_raw.y < hi_c && id_raw.y > lo_c) ? dx.y : 0.f};
        const f2 q2 = f2_fma(qs, qs, f2_mul(qr, qr));
        const f2 one_m = f2_sub(f2_bcast(1.0f), f2_mul(zz[i], q2));
        const f2 hq = f2_fma(hs2b, qs, f2_mul(hr2b, qr));
        const f2 term = f2_sub(f2_mul(f2_bcast(2.0f), f2_mul(amp, one_m)),
                               f2_mul(f2_mul(slope, aa[i]), hq));
        acc[i] = f2_fma(term, w, acc[i]);
      }
    }
  }
}

// The sweep of a warp's M groups for NTR traces, entered through a jump table:
// groups g0..g1 (g0 holding the earliest first contributing sample of the
// traces, g1 the latest) masked by sample index, the groups after g1 plain
// (every sample contributes); g1 < 0 runs every group plain.  One
// straight-line block, no per-group branch in the plain part: against masking
// every group from g0 on it issues 4.6 % fewer instructions (the sample masks'
// compares and selects) and ran 0.8 % faster on the 3D workload.
#define PSTM_SWEEP_GROUP(I, MK)                                                                 \
  if constexpr ((I) < M) {                                                                      \
    sweep_traces<1, ST, WM, LOWC, MK, OP, NTR, TAPER, CURVED>(                                  \
        reinterpret_cast<f2(&)[1]>(acc[(I) % M]), reinterpret_cast<const f2(&)[1]>(zz[(I) % M]), \
        reinterpret_cast<const f2(&)[1]>(aa[(I) % M]), hs2, hr2, rbase, kst, sc, bb, magic2,     \
        hi_c, lo_c, kw + 64 * (I), lane, 0, tp, cr_scale, rc);                                  \
  }
template <int M, typename ST, int WM, bool LOWC, int OP, int NTR, bool TAPER, bool CURVED>
__device__ __forceinline__ void sweep_split(f2 (&acc)[M], const f2 (&zz)[M], const f2 (&aa)[M],
                                            const float (&hs2)[NTR], const float (&hr2)[NTR],
                                            const uint32_t (&rbase)[NTR], const int (&kst)[NTR],
                                            const float (&sc)[NTR], f2 bb, f2 magic2, float hi_c,
                                            float lo_c, int kw, int lane, int g0, int g1,
                                            const TaperArgs& tp, float cr_scale, RowCheck rc) {
  static_assert(M <= 8, "the jump table covers up to 8 groups");
  if (g1 < 0) goto plain0;
  switch (g0 < 0 ? 0 : g0) {
    case 0: PSTM_SWEEP_GROUP(0, true) if (g1 <= 0) goto plain1; [[fallthrough]];
    case 1: PSTM_SWEEP_GROUP(1, true) if (g1 <= 1) goto plain2; [[fallthrough]];
    case 2: PSTM_SWEEP_GROUP(2, true) if (g1 <= 2) goto plain3; [[fallthrough]];
    case 3: PSTM_SWEEP_GROUP(3, true) if (g1 <= 3) goto plain4; [[fallthrough]];
    case 4: PSTM_SWEEP_GROUP(4, true) if (g1 <= 4) goto plain5; [[fallthrough]];
    case 5: PSTM_SWEEP_GROUP(5, true) if (g1 <= 5) goto plain6; [[fallthrough]];
    case 6: PSTM_SWEEP_GROUP(6, true) if (g1 <= 6) goto plain7; [[fallthrough]];
    case 7: PSTM_SWEEP_GROUP(7, true) [[fallthrough]];
    default: goto done;
  }
plain0: PSTM_SWEEP_GROUP(0, false)
plain1: PSTM_SWEEP_GROUP(1, false)
plain2: PSTM_SWEEP_GROUP(2, false)
plain3: PSTM_SWEEP_GROUP(3, false)
plain4: PSTM_SWEEP_GROUP(4, false)
plain5: PSTM_SWEEP_GROUP(5, false)
plain6: PSTM_SWEEP_GROUP(6, false)
plain7: PSTM_SWEEP_GROUP(7, false)
done:;
}
#undef PSTM_SWEEP_GROUP

// One output tile x time window: the body shared by the per-plan grid kernel
// (one CTA per tile/window) and the persistent batched kernel (one work item
// at a time).  Barriers are (re)initialised on entry; every bulk copy issued
// for the item has landed when it returns.
// Anti-aliased sweep (float32 rows of the trend-removed double integral I2):
// per sample the triangle half-width L = clamp(a * max(|gx|, |gy|), 1, Lmax)
// with gx = (x - s_x) dx q_s + (x - r_x) dx q_r (the operator dip along the
// inline axis times the inline spacing; gy likewise), then
//   amp = (I2(idx + L) - 2 I2(idx) + I2(idx - L)) / L^2
// from three linearly interpolated taps on the staged row.
template <int M, bool LOWC, bool MASKED, int NTR>
__device__ __forceinline__ void sweep_aa(f2 (&acc)[M], const f2 (&zz)[M], const f2 (&aa)[M],
                                         const float (&hs2)[NTR], const float (&hr2)[NTR],
                                         const float (&gxs)[NTR], const float (&gxr)[NTR],
                                         const float (&gys)[NTR], const float (&gyr)[NTR],
                                         const uint32_t (&rbase)[NTR], const int (&kst)[NTR],
                                         f2 bb, f2 magic2, float hi_c, float lo_c, float lmax,
                                         int kw, int lane, int g0, RowCheck rc = RowCheck{}) {
  auto tap = [&](f2 pos, uint32_t base) {
    // expanded rows: intercept and slope of I2's piece, one FMA of the position
    const f2 tm = f2_add_rm(pos, magic2);
    const f2 e0 = lds_f2(checked_addr(base + (__float_as_uint(tm.x) << 3),
                                      __float_as_uint(tm.x), base, 3, rc));
    const f2 e1 = lds_f2(checked_addr(base + (__float_as_uint(tm.y) << 3),
                                      __float_as_uint(tm.y), base, 3, rc));
    return f2{fmaf(pos.x, e0.y, e0.x), fmaf(pos.y, e1.y, e1.x)};
  };
#pragma unroll
  for (int i = 0; i < M; ++i) {
    if constexpr (MASKED) {
      if (i < g0) continue;
    }
#pragma unroll
    for (int n = 0; n < NTR; ++n) {
      // pre-scaled as the plain sweep: zz = a^2 (z^2 + eps), aa = a^2, q' = q / a;
      // g' = g / a, so L = a max(|g_x|, |g_y|) = aa max(|g'_x|, |g'_y|)
      const f2 rrs = f2_fma(f2_bcast(hs2[n]), aa[i], zz[i]);
      const f2 rrr = f2_fma(f2_bcast(hr2[n]), aa[i], zz[i]);
      const f2 qs = f2{rsqrt_approx(rrs.x), rsqrt_approx(rrs.y)};
      const f2 qr = f2{rsqrt_approx(rrr.x), rsqrt_approx(rrr.y)};
      f2 id = f2_fma(rrr, qr, f2_fma(rrs, qs, bb));
      id.x = fminf(id.x, hi_c);
      id.y = fminf(id.y, hi_c);
      if constexpr (LOWC) {
        id.x = fmaxf(id.x, lo_c);
        id.y = fmaxf(id.y, lo_c);
      }
      const f2 gx = f2_fma(f2_bcast(gxs[n]), qs, f2_mul(f2_bcast(gxr[n]), qr));
      const f2 gy = f2_fma(f2_bcast(gys[n]), qs, f2_mul(f2_bcast(gyr[n]), qr));
      f2 L = f2_mul(f2{fmaxf(fabsf(gx.x), fabsf(gy.x)), fmaxf(fabsf(gx.y), fabsf(gy.y))}, aa[i]);
      L.x = fminf(fmaxf(L.x, 1.0f), lmax);
      L.y = fminf(fmaxf(L.y, 1.0f), lmax);
      const f2 il = f2{rcp_approx(L.x), rcp_approx(L.y)};
      const f2 y0 = tap(f2_sub(id, L), rbase[n]);
      const f2 y1 = tap(id, rbase[n]);
      const f2 y2 = tap(f2_add(id, L), rbase[n]);
      const f2 amp = f2_mul(f2_fma(f2_bcast(-2.0f), y1, f2_add(y0, y2)), f2_mul(il, il));
      const f2 p = f2_mul(qs, qr);
      f2 w = f2_mul(p, p);
      if constexpr (MASKED) {
        const int klo = kw + 64 * i + lane;
        w.x = klo >= kst[n] ? w.x : 0.f;
        w.y = klo + 32 >= kst[n] ? w.y : 0.f;
      }
      acc[i] = f2_fma(amp, w, acc[i]);
    }
  }
}

template <int COLS, int WPC, int M, typename ST, int WM, bool LOWC, int OP, bool AA = false,
          bool TAPER = false, bool CURVED = false>
__device__ __forceinline__ void gather_tile(const KArgs& A, const int tile, const int win,
                                            unsigned char* smem) {
  constexpr int NW = COLS * WPC;
  constexpr int T = WPC * 64 * M;
  constexpr int ES = (int)sizeof(ST);
  constexpr int SHIFT = ES == 8 ? 3 : (ES == 4 ? 2 : 1);
  static_assert(kRowGuard % 16 == 0, "row data must stay 16-byte aligned");
  const int S = A.S;
  const int B = A.ring_rows, kStages = A.ring_stages;
  const bool h16 = A.hist16 != 0;
  const Smem2 L = smem2_layout(COLS, T, S, ES, kStages, B, h16 ? 2 : 4);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + L.bars);
  uint64_t* empty = full + kMaxStages;
  int* abort_flag = reinterpret_cast<int*>(empty + kMaxStages);
  float* thr = reinterpret_cast<float*>(smem + L.thr);
  int* hist = reinterpret_cast<int*>(smem + L.hist);
  const bool want_fold = A.fold_out != nullptr;
  unsigned char* raw = smem + L.raw;
  const int RP = S * ES + kRowGuard;  // bytes per staged row incl. its guard

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int k0 = win * T;
  const int kend = min(k0 + T, A.n_times);
  const int nk = kend - k0;
  const int n_c = A.n_il * A.n_xl;
  const int64_t off0 = A.off[tile];
  const int n_list = (int)(A.off[tile + 1] - off0);
  const int nb = (n_list + B - 1) / B;
  // anti-alias rows are staged whole (they carry the integral's padding)
  const int lo = AA ? 0 : window_lo(A, k0, Storage<ST>::kAlign);
  const int rowlen = S - lo;

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, NW);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  for (int r = tid; r < kStages * B; r += blockDim.x)
    *reinterpret_cast<uint4*>(raw + r * RP) = make_uint4(0u, 0u, 0u, 0u);
  for (int e = tid; e < COLS * T; e += blockDim.x) {
    const int q = e / T, kk = e - q * T;
    int qil, qxl;
    float v = -1.0f;
    if (kk < nk && tile_column(A, tile, q, qil, qxl)) v = threshold(A, qil * A.n_xl + qxl, k0 + kk);
    thr[e] = v;
    if (want_fold && (!h16 || (e & 1) == 0)) hist[h16 ? e >> 1 : e] = 0;
  }
  __syncthreads();

  // Lane 0 of warp 0 issues the bulk copies: the first kStages blocks now, and
  // block b + kStages into stage b % kStages once every warp has released
  // block b (warp 0 waits for that, so it never runs ahead of the others by
  // more than the ring).
  const uint32_t bytes = (uint32_t)(rowlen * ES);
  auto issue = [&](int b) {
    const int s = b % kStages;
    const int cnt = min(B, n_list - b * B);
    if (lane == 0) mbar_arrive_expect_tx(full + s, bytes * cnt);
    __syncwarp();
#ifdef PSTM_BOUNDS_CHECK
    // simulated fault: block 1 of the first item is never copied, so the
    // consumers' bounded waits on its stage expire
    if (A.inject == INJ_MISSING_COPY && tile == 0 && win == 0 && b == 1) return;
#endif
    if (lane < cnt) {
      const int jj = list_entry(A, off0 + (int64_t)b * B + lane);
      bulk_g2s(raw + (s * B + lane) * RP + kRowGuard,
               reinterpret_cast<const ST*>(A.traces) + (int64_t)jj * S + lo, bytes, full + s);
    }
  };
  if (warp == 0)
    for (int b = 0; b < min(nb, kStages); ++b) issue(b);

  // -------------------------------------------------------------- consumers
  // Warp -> (column, time segment).  The scheduler of warp w is w % 4; the
  // shallow segments mask out more samples than the deep ones, so every
  // scheduler gets warps of all segments (when there are enough warps).
  constexpr bool kMix = NW % (4 * WPC) == 0;
  const int cl = kMix ? (warp & 3) + 4 * (warp / (4 * WPC)) : warp / WPC;
  const int ts = kMix ? (warp >> 2) % WPC : (warp + (WPC / 2) * (warp / WPC)) % WPC;
  int il, xl;
  const bool col_ok = tile_column(A, tile, cl, il, xl);
  const int c = col_ok ? il * A.n_xl + xl : 0;
  float xc = 0.f, yc = 0.f;
  if (col_ok) column_xy(A, il, xl, xc, yc);
  const int kw = k0 + ts * 64 * M;
  const bool warp_live = col_ok && kw < A.n_times;

  f2 zz[M], aa[M], acc[M];
#pragma unroll
  for (int i = 0; i < M; ++i) {
    const int kl = min(kw + 64 * i + lane, A.n_times - 1), kh = min(kl + 32, A.n_times - 1);
    const float vl = vel_at(A, kl, c), vh = vel_at(A, kh, c);
    const float zl = depth_of(vl, out_time_ms(kl, A.out_dt, A.out_t0));
    const float zh = depth_of(vh, out_time_ms(kh, A.out_dt, A.out_t0));
    zz[i] = f2{fmaf(zl, zl, kRadicandFloor), fmaf(zh, zh, kRadicandFloor)};
    aa[i] = f2{1000.0f / (vl * A.in_dt), 1000.0f / (vh * A.in_dt)};
    if constexpr (CURVED) {
      // aa holds k / (2 v0 max(z, 1e-6)) for the curved-ray argument
      aa[i] = f2{A.cr_k / (2.0f * vl * fmaxf(zl, 1e-6f)), A.cr_k / (2.0f * vh * fmaxf(zh, 1e-6f))};
    } else if constexpr (kPrescaled<OP, WM>) {
      aa[i] = f2_mul(aa[i], aa[i]);
      zz[i] = f2_mul(zz[i], aa[i]);
    }
    acc[i] = f2{0.f, 0.f};
  }
  // Index frame of the sweeps: the staged position idx - lo (16-bit rows), or
  // idx + 1 - lo (expanded float32 rows, sample i at entry i + 1).  For the
  // anti-alias integral (sample i at entry i + pad, intercept form) the entry
  // coordinate less the rows' intercept origin q0, with the rounding-down add
  // of 2^23 + q0 - lo yielding the staged entry's index in the float's bits.
  // Intercept-form float32 rows (sample i at entry i + 1) take the anti-alias
  // frame with q0 = the plan's row origin.
  constexpr bool kIcpt = std::is_same<ST, RowIcpt>::value;
  constexpr bool kExpanded = std::is_same<ST, float2>::value || kIcpt;
  const float shift = AA ? (float)A.aa_pad - (float)A.row_origin
                     : kIcpt ? 1.0f - (float)A.row_origin
                             : (kExpanded ? 1.0f : 0.0f) - (float)lo;
  const f2 mg = f2_bcast(AA || kIcpt ? kMagic + (float)(A.row_origin - lo) : kMagic);
  const float bconst = -A.in_t0 / A.in_dt + shift;
  const f2 bb = f2_bcast(bconst);
#ifdef PSTM_BOUNDS_CHECK
  // simulated fault: no upper clamp, so late samples index past the staged row
  const float hi_c = A.inject == INJ_NO_CLAMP ? 1.0e30f : A.clamp_hi + shift;
#else
  const float hi_c = A.clamp_hi + shift;
#endif
  const float lo_c = shift;  // idx >= 0 (LOWC: output times before the first input)
  // entries a staged-row read may address: the guard before the row, then
  // the rowlen entries copied (16-bit and plain float32 rows read two)
  const RowCheck rck{-kRowGuard / ES, rowlen - (ES == 8 ? 1 : 2), A.err};
  const float* thr_c = thr + cl * T;
  const uint32_t raw_base = smem_addr(raw) + kRowGuard - (kMagicBits << SHIFT);
  const int kwe = kw + 64 * M;

  bool aborted = false;
  int slot = 0, stage = 0, blk = 0;
  uint32_t phase = 0;
  // the next chunk's list entries and geometry are fetched while the current
  // chunk computes
  int jj_next = (lane < n_list) ? list_entry(A, off0 + lane) : 0;
  float4 g_next = make_float4(0.f, 0.f, 0.f, 0.f);
  if (warp_live && lane < n_list) g_next = __ldg(A.geo + jj_next);
  for (int p0 = 0; p0 < n_list && !aborted; p0 += 32) {
    // set-up of 32 list entries, one per lane
    float hs2 = 0.f, hr2 = 0.f;
    float gxs = 0.f, gxr = 0.f, gys = 0.f, gyr = 0.f;  // AA: dip coefficients
    int ks = 0x7fffffff;  // no contribution in this window
    float tsc = 1.0f;
    const int jj = jj_next;
    if (p0 + lane < n_list) {
      if (warp_live) {
        leg_h2(xc, yc, g_next, hs2, hr2);
        const int fv = first_valid(thr_c, nk, sqrtf(fmaxf(hs2, hr2)));
        if (fv < nk) {
          ks = k0 + fv;
          // fold: one warp per column counts where each trace starts
          if (want_fold && ts == 0) {
            // 16-bit counts: entry e is half e & 1 of word e / 2 (T is even)
            const int e = cl * T + fv;
            if (h16)
              atomicAdd(reinterpret_cast<unsigned*>(hist) + (e >> 1), 1u << (16 * (e & 1)));
            else
              atomicAdd(hist + e, 1);
          }
        }
        if constexpr (AA) {
          gxs = (xc - g_next.x) * A.aa_dx;
          gxr = (xc - g_next.z) * A.aa_dx;
          gys = (yc - g_next.y) * A.aa_dy;
          gyr = (yc - g_next.w) * A.aa_dy;
        }
      }
      if (A.scales) tsc = __ldg(A.scales + jj);
      if constexpr (TAPER) {
        // the distance tapers of both legs: one factor per (column, trace)
        if (warp_live)
          tsc *= cos_edge(sqrtf(hs2), A.tp.d0, A.tp.dinv, A.tp.dmax) *
                 cos_edge(sqrtf(hr2), A.tp.d0, A.tp.dinv, A.tp.dmax);
      }
    }
    const int pn = p0 + 32 + lane;
    if (pn < n_list) jj_next = list_entry(A, off0 + pn);
    const int nt = min(32, n_list - p0);
    bool prefetched = false;  // the next chunk's geometry is loaded a few traces in
    for (int t = 0; t < nt;) {
      const int p = p0 + t;
      if (!prefetched && t >= 4) {
        if (warp_live && pn < n_list) g_next = __ldg(A.geo + jj_next);
        prefetched = true;
      }
      if (slot == 0) {
        bool ok = true;
        if (lane == 0) ok = mbar_wait(full + stage, phase);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (!ok) {
          if (lane == 0) {
            set_error(A.err, PSTM_ERR_TIMEOUT);
            *abort_flag = 1;
          }
          aborted = true;
          break;
        }
      }
      int adv;
      if constexpr (AA) {
        // two traces of the same stage when available
        const bool pair = (slot + 1 < B) && (t + 1 < nt);
        const int ka = __shfl_sync(0xffffffffu, ks, t);
        const int kb = __shfl_sync(0xffffffffu, ks, pair ? t + 1 : t);
        const bool la = ka < kwe, lb = pair && kb < kwe;
        const uint32_t rb0 = raw_base + (uint32_t)((stage * B + slot) * RP);
        // anti-aliased sweeps take one trace at a time (three taps per sample)
        for (int q = 0; q < (pair ? 2 : 1); ++q) {
          const int u = t + q;
          const int kq = q ? kb : ka;
          if (!(q ? lb : la)) continue;
          const float hs[1] = {__shfl_sync(0xffffffffu, hs2, u)};
          const float hr[1] = {__shfl_sync(0xffffffffu, hr2, u)};
          const float g0[1] = {__shfl_sync(0xffffffffu, gxs, u)};
          const float g1[1] = {__shfl_sync(0xffffffffu, gxr, u)};
          const float g2[1] = {__shfl_sync(0xffffffffu, gys, u)};
          const float g3[1] = {__shfl_sync(0xffffffffu, gyr, u)};
          const uint32_t rb[1] = {rb0 + (uint32_t)(q * RP)};
          const int kk[1] = {kq};
          if (kq > kw)
            sweep_aa<M, LOWC, true, 1>(acc, zz, aa, hs, hr, g0, g1, g2, g3, rb, kk, bb, mg, hi_c,
                                       lo_c, A.aa_lmax, kw, lane, (kq - kw) >> 6, rck);
          else
            sweep_aa<M, LOWC, false, 1>(acc, zz, aa, hs, hr, g0, g1, g2, g3, rb, kk, bb, mg, hi_c,
                                        lo_c, A.aa_lmax, kw, lane, 0, rck);
        }
        adv = pair ? 2 : 1;
      } else {
        // the traces of this stage (within the chunk) that reach the warp's
        // window, two at a time in list order; the others are skipped
        const int t_end = min(nt, t + (B - slot));
        const unsigned live = __ballot_sync(0xffffffffu, lane >= t && lane < t_end && ks < kwe);
        if (live == 0) {
          adv = t_end - t;
        } else {
          // staged row of chunk position u: slot + (u - t) of this stage
          const uint32_t rbs = raw_base + (uint32_t)((stage * B + slot - t) * RP);
          const int a = __ffs(live) - 1;
          const unsigned rest = live & (live - 1);
          const int ka = __shfl_sync(0xffffffffu, ks, a);
          if (rest) {
            const int b = __ffs(rest) - 1;
            const int kb = __shfl_sync(0xffffffffu, ks, b);
            const float hs[2] = {__shfl_sync(0xffffffffu, hs2, a), __shfl_sync(0xffffffffu, hs2, b)};
            const float hr[2] = {__shfl_sync(0xffffffffu, hr2, a), __shfl_sync(0xffffffffu, hr2, b)};
            const float sc[2] = {__shfl_sync(0xffffffffu, tsc, a), __shfl_sync(0xffffffffu, tsc, b)};
            const uint32_t rb[2] = {rbs + (uint32_t)(a * RP), rbs + (uint32_t)(b * RP)};
            const int kk[2] = {ka, kb};
            const int kmax = max(ka, kb);
            sweep_split<M, ST, WM, LOWC, OP, 2, TAPER, CURVED>(
                acc, zz, aa, hs, hr, rb, kk, sc, bb, mg, hi_c, lo_c, kw, lane,
                (min(ka, kb) - kw) >> 6, kmax > kw ? (kmax - kw) >> 6 : -1, A.tp, A.cr_scale, rck);
            adv = b + 1 - t;
          } else {
            const float hs[1] = {__shfl_sync(0xffffffffu, hs2, a)};
            const float hr[1] = {__shfl_sync(0xffffffffu, hr2, a)};
            const float sc[1] = {__shfl_sync(0xffffffffu, tsc, a)};
            const uint32_t rb[1] = {rbs + (uint32_t)(a * RP)};
            const int kk[1] = {ka};
            const int g = ka > kw ? (ka - kw) >> 6 : -1;
            sweep_split<M, ST, WM, LOWC, OP, 1, TAPER, CURVED>(acc, zz, aa, hs, hr, rb, kk, sc, bb,
                                                               mg, hi_c, lo_c, kw, lane, g, g,
                                                               A.tp, A.cr_scale, rck);
            adv = t_end - t;
          }
        }
      }
      t += adv;
      slot += adv;
      if (slot == B || p + adv == n_list) {
        __syncwarp();
        if (lane == 0) mbar_arrive(empty + stage);
        if (warp == 0 && blk + kStages < nb) {
          bool ok = true;
          if (lane == 0) ok = mbar_wait(empty + stage, phase);
          ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
          if (!ok) {
            if (lane == 0) {
              set_error(A.err, PSTM_ERR_TIMEOUT);
              *abort_flag = 1;
            }
            aborted = true;
            break;
          }
          issue(blk + kStages);
        }
        ++blk;
        slot = 0;
        if (++stage == kStages) {
          stage = 0;
          phase ^= 1u;
        }
      }
    }
    if (!prefetched && warp_live && pn < n_list) g_next = __ldg(A.geo + jj_next);
  }
  if (aborted) {
    // leave no bulk copy in flight into this CTA's shared memory
    if (warp == 0 && lane == 0)
      for (int b = blk; b < min(nb, blk + kStages); ++b)
        mbar_wait(full + b % kStages, (b / kStages) & 1);
  }
  if (want_fold) {
    // fold = running count of the traces started so far (every warp of the
    // CTA reaches this barrier, aborted or not)
    __syncthreads();
    if (warp < COLS && !*abort_flag) {
      int qil, qxl;
      if (tile_column(A, tile, warp, qil, qxl)) {
        const int qc = qil * A.n_xl + qxl;
        int carry = 0;
        for (int base = 0; base < nk; base += 32) {
          int v = 0;
          if (base + lane < nk) {
            const int e = warp * T + base + lane;
            v = h16 ? (int)((reinterpret_cast<const unsigned*>(hist)[e >> 1] >> (16 * (e & 1))) &
                            0xffffu)
                    : hist[e];
          }
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += u;
          }
          v += carry;
          if (base + lane < nk) A.fold_out[(long long)(k0 + base + lane) * n_c + qc] = (float)v;
          carry = __shfl_sync(0xffffffffu, v, 31);
        }
      }
    }
  }
  if (aborted || !warp_live) return;
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
      if constexpr (kPrescaled<OP, WM> && !CURVED) {
        // the pre-scaled weight p' = p / a^2: multiply by a^4 (p^2) or a^2 (p)
        const float al = 1000.0f / (vl * A.in_dt), ah = 1000.0f / (vh * A.in_dt);
        const float al2 = al * al, ah2 = ah * ah;
        fl *= WM == W_OBL_SPREAD ? al2 * al2 : al2;
        fh *= WM == W_OBL_SPREAD ? ah2 * ah2 : ah2;
      }
      if (OP == OP_VGRAD) {
        fl = klo < A.n_times ? fl / vl * A.in_img[(long long)klo * n_c + c] : 0.f;
        fh = khi < A.n_times ? fh / vh * A.in_img[(long long)khi * n_c + c] : 0.f;
      }
    }
    if (klo < A.n_times) A.out[(long long)klo * n_c + c] = acc[i].x * fl;
    if (khi < A.n_times) A.out[(long long)khi * n_c + c] = acc[i].y * fh;
  }
}

template <int COLS, int WPC, int M, typename ST, int WM, bool LOWC, int OP, bool AA = false,
          bool TAPER = false, bool CURVED = false>
__global__ void __launch_bounds__(COLS* WPC * 32, ctas_per_sm(COLS* WPC * 32))
    pstm_gather2_kernel(const KArgs A) {
  extern __shared__ __align__(128) unsigned char smem[];
  gather_tile<COLS, WPC, M, ST, WM, LOWC, OP, AA, TAPER, CURVED>(A, blockIdx.x, blockIdx.y, smem);
}

// Persistent batched kernel: CTAs pull (class, tile, window) work items from a
// device queue (items ordered by descending trace-list length) until none is
// left.  Each class has its own plan data and output image in descs[class].
template <int COLS, int WPC, int M, typename ST, int WM, bool LOWC, int OP>
__global__ void __launch_bounds__(COLS* WPC * 32, ctas_per_sm(COLS* WPC * 32))
    pstm_batch_kernel(const KArgs* __restrict__ descs, const int4* __restrict__ items, int n_items,
                      int* __restrict__ counter) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int next;
  __shared__ KArgs a;
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(counter, 1);
    __syncthreads();
    const int it = next;
    if (it >= n_items) break;
    const int4 w = items[it];
    if (threadIdx.x == 0) a = descs[w.x];
    __syncthreads();
    gather_tile<COLS, WPC, M, ST, WM, LOWC, OP>(a, w.y, w.z, smem);
    __syncthreads();
    if (threadIdx.x == 0) {  // every phase has completed: retire the barriers before re-use
      uint64_t* bars = reinterpret_cast<uint64_t*>(smem);
      for (int s = 0; s < a.ring_stages; ++s) {
        mbar_inval(bars + s);
        mbar_inval(bars + kMaxStages + s);
      }
    }
  }
}

template <int COLS, int WPC, int M, typename ST, int WM, int OP, bool AA = false,
          bool TAPER = false, bool CURVED = false>
inline cudaError_t launch2_one(const Plan* p, const KArgs& A, cudaStream_t s) {
  auto kern = needs_lowclamp(p)
                  ? pstm_gather2_kernel<COLS, WPC, M, ST, WM, true, OP, AA, TAPER, CURVED>
                  : pstm_gather2_kernel<COLS, WPC, M, ST, WM, false, OP, AA, TAPER, CURVED>;
  const int T = WPC * 64 * M;
  KArgs A2 = A;
  const int hb = hist_entry_bytes(A.hist16 != 0);
  if (!ring_shape(COLS, T, p->row_stride, (int)sizeof(ST), &A2.ring_stages, &A2.ring_rows,
                  smem_budget(COLS * WPC * 32), hb))
    return cudaErrorInvalidValue;
  const Smem2 L = smem2_layout(COLS, T, p->row_stride, (int)sizeof(ST), A2.ring_stages,
                               A2.ring_rows, hb);
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L.total);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)p->n_tiles, (unsigned)((p->grid.n_times + T - 1) / T));
  kern<<<grid, COLS * WPC * 32, L.total, s>>>(A2);
  count_launch();
  return cudaGetLastError();
}

template <int COLS, int WPC, int M, typename ST, int OP, bool TAPER = false, bool CURVED = false>
inline cudaError_t dispatch2_wm(const Plan* p, const KArgs& A, cudaStream_t s) {
  const int wm = p->params.weight;
  constexpr bool k32 = std::is_same<ST, float>::value || std::is_same<ST, float2>::value ||
                      std::is_same<ST, RowIcpt>::value;
  if constexpr (OP == OP_VGRAD || !k32) {
    if (wm != W_OBL_SPREAD) return cudaErrorNotSupported;
    return launch2_one<COLS, WPC, M, ST, W_OBL_SPREAD, OP, false, TAPER, CURVED>(p, A, s);
  } else {
    switch (wm) {
      case W_OBL_SPREAD:
        return launch2_one<COLS, WPC, M, ST, W_OBL_SPREAD, OP, false, TAPER, CURVED>(p, A, s);
      case W_SPREAD:
        return launch2_one<COLS, WPC, M, ST, W_SPREAD, OP, false, TAPER, CURVED>(p, A, s);
      case W_OBL:
        return launch2_one<COLS, WPC, M, ST, W_OBL, OP, false, TAPER, CURVED>(p, A, s);
      case W_NONE:
        return launch2_one<COLS, WPC, M, ST, W_NONE, OP, false, TAPER, CURVED>(p, A, s);
    }
    return cudaErrorInvalidValue;
  }
}

// Forward launch over intercept-form float32 rows (forward_only plans),
// instantiated in its own translation unit (pstm_gather_fwd_icpt.cu).
cudaError_t launch_forward_icpt(const Plan* p, const KArgs& A, cudaStream_t s);
// Forward launch with the aperture tapers (float32 plans with a taper width),
// instantiated in pstm_gather_fwd_taper.cu.
cudaError_t launch_forward_taper(const Plan* p, const KArgs& A, cudaStream_t s);
// Forward launch with curved-ray traveltimes (float32 plans with a ray
// gradient), instantiated in pstm_gather_fwd_taper.cu as well.
cudaError_t launch_forward_curved(const Plan* p, const KArgs& A, cudaStream_t s);

template <int COLS, int WPC, int M, int OP>
inline cudaError_t dispatch2_st(const Plan* p, const KArgs& A, cudaStream_t s) {
  if (p->params.antialias) {
    if constexpr (OP == OP_FWD)
      return launch2_one<COLS, WPC, M, float2, W_OBL_SPREAD, OP, true>(p, A, s);
    else
      return cudaErrorNotSupported;
  }
  switch (p->params.storage) {
    case PSTM_F32:
      // plans stage expanded (x, dx) rows, forward_only plans intercept-form
      // rows; the no-allocation path plain rows
      if (p->elt_bytes != 8) return dispatch2_wm<COLS, WPC, M, float, OP>(p, A, s);
      if (p->params.taper_width > 0) {
        if constexpr (OP == OP_FWD)
          return launch_forward_taper(p, A, s);
        else
          return cudaErrorNotSupported;
      }
      if (p->params.ray_gradient != 0) {
        if constexpr (OP == OP_FWD)
          return launch_forward_curved(p, A, s);
        else
          return cudaErrorNotSupported;
      }
      if (p->row_origin != 0) {
        if constexpr (OP == OP_FWD)
          return launch_forward_icpt(p, A, s);
        else
          return cudaErrorNotSupported;
      }
      return dispatch2_wm<COLS, WPC, M, float2, OP>(p, A, s);
    case PSTM_BF16:
      return dispatch2_wm<COLS, WPC, M, __nv_bfloat16, OP>(p, A, s);
    case PSTM_F16:
      return dispatch2_wm<COLS, WPC, M, __half, OP>(p, A, s);
  }
  return cudaErrorInvalidValue;
}

template <int OP>
inline cudaError_t dispatch2_shape(const Plan* p, const KArgs& A, cudaStream_t s) {
  switch (p->shape.id) {
    case 1:
    case 5:
      return dispatch2_st<8, 2, 8, OP>(p, A, s);
    case 2:
    case 8:
      return dispatch2_st<4, 4, 4, OP>(p, A, s);
    case 4:
    case 6:
      return dispatch2_st<4, 2, 4, OP>(p, A, s);
    case 7:
      return dispatch2_st<2, 4, 2, OP>(p, A, s);
    case 3:
    case 9:
      return dispatch2_st<16, 1, 8, OP>(p, A, s);
    case 10:
    case 12:
      return dispatch2_st<16, 1, 4, OP>(p, A, s);
    case 11:
      return dispatch2_st<16, 1, 2, OP>(p, A, s);
    case 13:
      return dispatch2_st<8, 1, 8, OP>(p, A, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace pstm
