// Device helpers shared by the dense-stereo kernels.
//
// Bit-exactness rules (Lux.Engine computes in .NET floats, one rounding per operation, no FMA):
//   * every kernel is compiled with --fmad=false; products and sums additionally go through __fmul_rn / __fadd_rn
//     where the reference's operation order matters, so no contraction can change a result;
//   * (int)f follows .NET 9+ (truncate, saturate, NaN -> 0), which is what cvt.rzi.s32.f32 does;
//   * divisions are IEEE round-to-nearest (__fdiv_rn), as the reference's `/`.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define LUX_DEV __device__ __forceinline__

namespace lux {

LUX_DEV uint32_t fbits(float f) { return __float_as_uint(f); }
LUX_DEV float ffrom(uint32_t u) { return __uint_as_float(u); }
LUX_DEV int f2i(float f) { return __float2int_rz(f); }  // .NET (int)f

// .NET Math.Max/Min on floats: NaN propagates.
LUX_DEV float cs_maxf(float a, float b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a == b) return signbit(a) ? b : a;
  return a > b ? a : b;
}
LUX_DEV float cs_minf(float a, float b) {
  if (a != a) return a;
  if (b != b) return b;
  if (a == b) return signbit(a) ? a : b;
  return a < b ? a : b;
}

// IntelApprox.RcpBits (Lux.Engine/Imaging/IntelApprox.cs:21-29): rcp_entry given the table entry of b,
// r = table[(b >> 11) & 0xfff], fetched by the caller (from a shared-memory copy); rcp_bits with the table in global memory.
LUX_DEV uint32_t rcp_entry(uint32_t b, uint32_t r) {
  uint32_t sign = b & 0x80000000u, e = (b >> 23) & 0xff, m = b & 0x7fffff;
  if (e == 0xff) return m != 0 ? (b | 0x400000u) : sign;
  if (e == 0) return sign | 0x7f800000u;
  int re = (int)((r >> 23) & 0xff) - ((int)e - 127);
  if (re <= 0) return sign;
  return sign | ((uint32_t)re << 23) | (r & 0x7fffff);
}
LUX_DEV uint32_t rcp_bits(uint32_t b, const uint32_t* __restrict__ table) {
  uint32_t sign = b & 0x80000000u, e = (b >> 23) & 0xff, m = b & 0x7fffff;
  if (e == 0xff) return m != 0 ? (b | 0x400000u) : sign;
  if (e == 0) return sign | 0x7f800000u;
  uint32_t r = __ldg(table + (m >> 11));
  int re = (int)((r >> 23) & 0xff) - ((int)e - 127);
  if (re <= 0) return sign;
  return sign | ((uint32_t)re << 23) | (r & 0x7fffff);
}
LUX_DEV float rcp_approx(float x, const uint32_t* __restrict__ table) { return ffrom(rcp_bits(fbits(x), table)); }

// The fast 2^x of the adaptive P2 (DenseStereoSgm.cs:269-272): e clamped by MathF.Min/Max, n = (int)e - (e < 0).
LUX_DEV float sgm_exp2(float e) {
  const float E3 = __uint_as_float(0x3d9fcb52u), E2 = __uint_as_float(0x3e677e26u), E1 = __uint_as_float(0x3f322226u),
              E0 = __uint_as_float(0x3f7ffb19u);
  int ei = f2i(e) + (e < 0.0f ? -1 : 0);
  float f = __fsub_rn(e, (float)ei);
  float poly = __fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(__fadd_rn(__fmul_rn(E3, f), E2), f), E1), f), E0);
  return ffrom(fbits(poly) + ((uint32_t)ei << 23));
}

// P2 of one path step (DenseStereoSgm.cs:266-273): S = (|Δ0·w0| + |Δ2·w2|) + |Δ1·w1|, P2 = (int)(p2Base·2^-S).
LUX_DEV int sgm_p2(const float g[4], const float n[4], const float gw[4], float p2base) {
  float d0 = __fmul_rn(__fsub_rn(g[0], n[0]), gw[0]);
  float d1 = __fmul_rn(__fsub_rn(g[1], n[1]), gw[1]);
  float d2 = __fmul_rn(__fsub_rn(g[2], n[2]), gw[2]);
  float S = __fadd_rn(__fadd_rn(fabsf(d0), fabsf(d2)), fabsf(d1));
  float e = cs_maxf(cs_minf(-S, 128.0f), -126.0f);
  float E = sgm_exp2(e);
  return f2i(__fmul_rn(p2base, E));
}

// Bounded spin on a device-scope flag: returns false when the deadline (ns of %globaltimer) passes.
LUX_DEV uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
LUX_DEV int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
LUX_DEV void st_release(int* p, int v) { asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory"); }
// CTA-scope acquire / release on shared memory: the hand-over between warps of one block.
LUX_DEV int ld_acquire_cta(const int* p) {
  int v;
  asm volatile("ld.acquire.cta.shared.s32 %0, [%1];" : "=r"(v) : "r"((unsigned)__cvta_generic_to_shared(p)) : "memory");
  return v;
}
LUX_DEV void st_release_cta(int* p, int v) {
  asm volatile("st.release.cta.shared.s32 [%0], %1;" ::"r"((unsigned)__cvta_generic_to_shared(p)), "r"(v) : "memory");
}
// Waits (bounded) until the shared counter *p >= target. Returns false on timeout or when *stop is set. The sleep
// between polls doubles from 32 ns to 256 ns: the waiting warps leave the issue slots to the warps that have work.
LUX_DEV bool wait_shared_at_least(const int* p, int target, const volatile int* stop, uint64_t timeout_ns) {
  if (ld_acquire_cta(p) >= target) return true;
  const uint64_t t0 = global_ns();
  unsigned sleep_ns = 32;
  for (unsigned it = 0;; it++) {
    __nanosleep(sleep_ns);
    if (sleep_ns < 256) sleep_ns <<= 1;
    if (ld_acquire_cta(p) >= target) return true;
    if ((it & 15) == 15) {
      if (*stop) return false;
      if (global_ns() - t0 > timeout_ns) return false;
    }
  }
}

// Shared-memory mbarriers: the hand-over between warps of one block. arrive releases (CTA scope) what the arriving
// thread and, through a preceding __syncwarp, its warp wrote; a successful try_wait acquires it. A thread in try_wait is
// suspended by the hardware until the phase completes or a time limit passes, so waiting warps take no issue slots.
LUX_DEV uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
LUX_DEV void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
LUX_DEV void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// true once the phase of parity `parity` has completed
LUX_DEV bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for a phase: gives up when *stop is set or after timeout_ns (then sets *err = 11 and *stop).
LUX_DEV bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* stop, int* err, uint64_t timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (unsigned it = 0;; it++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 7) == 7) {
      if (*stop) return false;
      if (global_ns() - t0 > timeout_ns) {
        atomicCAS(err, 0, 11);
        *stop = 1;
        return false;
      }
    }
  }
}

// Asynchronous global -> shared copies (cp.async): the data is the issuing thread's after cp.async.wait_group, and the
// warp's after a following __syncwarp.
LUX_DEV void cp_async8(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
LUX_DEV void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
LUX_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
LUX_DEV void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Waits until *flag >= target and returns the value it saw (which may be larger); on timeout, or when another block
// already failed, returns -1 (setting *err = code on timeout). Spins are bounded by wall time.
LUX_DEV int wait_at_least_value(const int* flag, int target, int* err, int code, uint64_t timeout_ns) {
  int v = ld_acquire(flag);
  if (v >= target) return v;
  const uint64_t t0 = global_ns();
  for (;;) {
    __nanosleep(32);
    v = ld_acquire(flag);
    if (v >= target) return v;
    if (*(volatile int*)err != 0) return -1;
    if (global_ns() - t0 > timeout_ns) {
      atomicCAS(err, 0, code);
      return -1;
    }
  }
}

// Waits until *flag >= target; on timeout sets *err = code and returns false. Spins are bounded by wall time.
LUX_DEV bool wait_at_least(const int* flag, int target, int* err, int code, uint64_t timeout_ns) {
  if (ld_acquire(flag) >= target) return true;
  uint64_t t0 = global_ns();
  for (;;) {
    __nanosleep(64);
    if (ld_acquire(flag) >= target) return true;
    if (*(volatile int*)err != 0) return false;  // another block already failed: stop waiting
    if (global_ns() - t0 > timeout_ns) {
      atomicCAS(err, 0, code);
      return false;
    }
  }
}

}  // namespace lux
