// Shared device helpers for the sm_100a PSTM kernels: packed f32x2 arithmetic,
// mbarrier / bulk-copy (TMA) wrappers with bounded waits, and the error flag.
#pragma once
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#define PSTM_ERR_TIMEOUT 1
#define PSTM_ERR_BOUNDS 2
#define PSTM_ERR_VELOCITY 4
#define PSTM_ERR_COORDS 8

// Bounded waits on an mbarrier give up after this many nanoseconds of the
// global timer (2 s: far beyond any legitimate wait for one pipeline stage;
// the checked test build shortens it).
#ifndef PSTM_WAIT_NS
#define PSTM_WAIT_NS 2000000000ull
#endif

namespace pstm {

// ----------------------------------------------------------------- f32x2 ---
// Blackwell executes add/mul/fma on a pair of f32 lanes in one instruction.
struct f2 {
  float x, y;
};

__device__ __forceinline__ unsigned long long pk(f2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1,%2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ f2 upk(unsigned long long r) {
  f2 a;
  asm("mov.b64 {%0,%1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}
// round toward -inf: used for the 2^23 floor trick
__device__ __forceinline__ f2 f2_add_rm(f2 a, f2 b) {
  unsigned long long d;
  asm("add.rm.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}
__device__ __forceinline__ f2 f2_sub(f2 a, f2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)));
  return upk(d);
}
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(pk(a)), "l"(pk(b)), "l"(pk(c)));
  return upk(d);
}
__device__ __forceinline__ f2 f2_bcast(float v) { return f2{v, v}; }

// MUFU reciprocal square root (approximate, ~2 ulp).
__device__ __forceinline__ float rsqrt_approx(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// ------------------------------------------------------ shared-memory I/O ---
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ f2 lds_f2(uint32_t addr) {
  f2 v;
  asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr));
  return v;
}

// ------------------------------------------------------------- mbarrier ---
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// Returns true when the phase with parity `parity` has completed, false if the
// bounded spin ran out.
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// A waiting thread is suspended by the hardware (up to the hint, in ns) until
// the phase completes, so waiting warps do not spin on issue slots.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_addr(bar);
  const uint32_t hint_ns = 20000;
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity), "r"(hint_ns)
        : "memory");
    if (done) return true;
    const uint64_t now = global_ns();
    if (it == 0)
      t0 = now;
    else if (now - t0 > PSTM_WAIT_NS)
      return false;
  }
}

// 1-D bulk copy global -> shared (TMA engine), completion signalled on `bar`.
// dst, src 16-byte aligned; bytes a multiple of 16.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ------------------------------------------------------------- storage ---
template <typename T>
struct Storage;
template <>
struct Storage<float> {
  static constexpr int kAlign = 4;  // elements per 16 bytes
  __device__ __forceinline__ static float load(const float* p, int i) { return p[i]; }
};
// float32 samples expanded to (x[i], x[i+1] - x[i]) entries: one 8-byte load
// gives both interpolation taps
template <>
struct Storage<float2> {
  static constexpr int kAlign = 2;  // entries per 16 bytes
};
// float32 samples expanded into intercept form, for plans that only migrate:
// entry q holds (x[q-1] - (q - q0) d, d) with d = x[q] - x[q-1] and q0 the
// plan's row origin, so the interpolant at entry coordinate e is one FMA,
// (e - q0) d + c
struct RowIcpt {
  float c, d;
};
template <>
struct Storage<RowIcpt> {
  static constexpr int kAlign = 2;  // entries per 16 bytes
};
template <>
struct Storage<__nv_bfloat16> {
  static constexpr int kAlign = 8;
  __device__ __forceinline__ static float load(const __nv_bfloat16* p, int i) {
    return __bfloat162float(p[i]);
  }
};
template <>
struct Storage<__half> {
  static constexpr int kAlign = 8;
  __device__ __forceinline__ static float load(const __half* p, int i) {
    return __half2float(p[i]);
  }
};

__device__ __forceinline__ void set_error(int* err, int code) {
  if (err) atomicOr(err, code);
}

// Output time axis exactly as the reference forms it in float32
// (migration_engine.py:305-306): t = k*dt + t0 (ms), z = V * (t/1000) / 2.
__device__ __forceinline__ float out_time_ms(int k, float dt_ms, float t0_ms) {
  return __fadd_rn(__fmul_rn(static_cast<float>(k), dt_ms), t0_ms);
}
__device__ __forceinline__ float depth_of(float v, float t_ms) {
  return __fdiv_rn(__fmul_rn(v, __fdiv_rn(t_ms, 1000.0f)), 2.0f);
}

}  // namespace pstm
