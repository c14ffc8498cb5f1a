// sm_100a building blocks: mbarriers with bounded waits, TMA tile loads, tcgen05 (TMEM alloc,
// UMMA descriptors, MMA issue/commit, TMEM loads).  Inline PTX, no library dependency.
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "common.cuh"

namespace afqmc {
namespace tc {

// ---------------------------------------------------------------------------------------------
// error flag of a bounded wait that gave up (written to device memory, read by the host)
// ---------------------------------------------------------------------------------------------
constexpr unsigned kTimeoutFlag = 1u;
// cycle budget of one wait (about 2-3 s at B200 clocks)
constexpr long long kWaitCycles = 4000000000ll;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for the phase with the given parity; gives up after `budget` cycles (kWaitCycles unless a
// caller passes less), sets *err and returns false.  `abort` lets a role stop waiting once
// another role has reported a failure.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned* err,
                                          volatile int* abort, long long budget = kWaitCycles) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (abort && *abort) return false;
    if (clock64() - t0 > budget) {
      if (err) atomicOr(err, kTimeoutFlag);
      if (abort) *abort = 1;
      return false;
    }
  }
}

// The same wait for a whole warp, with one outcome for all its lanes: the epilogue warps follow a
// wait with warp-collective tensor-memory loads, which every lane must take part in.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, unsigned parity, unsigned* err,
                                               volatile int* abort) {
  const bool ok = mbar_wait(bar, parity, err, abort);
  return __all_sync(0xffffffffu, ok) != 0;
}

// ---------------------------------------------------------------------------------------------
// TMA
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar,
                                            int x, int y, int z) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
      : "memory");
}

// the same load with an L2 cache policy (from make_policy_*)
__device__ __forceinline__ void tma_load_3d_hint(void* dst, const CUtensorMap* map, uint64_t* bar,
                                                 int x, int y, int z, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%3, %4, %5}], [%2], %6;" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z),
      "l"(policy)
      : "memory");
}

// L2 policies: keep the lines in L2 ahead of others / evict them first
__device__ __forceinline__ uint64_t make_policy_evict_last() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}
__device__ __forceinline__ uint64_t make_policy_evict_first() {
  uint64_t pol;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
  return pol;
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ---------------------------------------------------------------------------------------------
// tcgen05
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(dst_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// UMMA shared-memory descriptor, K-major operand in the 128-byte swizzle layout written by TMA:
// rows of 128 bytes, 8-row groups 1024 bytes apart (SBO), tile base 1024-byte aligned.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= uint64_t((saddr & 0x3FFFF) >> 4);      // start address      [0,14)
  d |= uint64_t(1) << 16;                      // LBO (unused here)  [16,30)
  d |= uint64_t(1024 >> 4) << 32;              // SBO = 1024 B       [32,46)
  d |= uint64_t(1) << 46;                      // version = 1        [46,48)
  d |= uint64_t(2) << 61;                      // SWIZZLE_128B       [61,64)
  return d;
}

// Instruction descriptor: kind::tf32, D = F32, A = B = TF32, K-major, M x N, optional A negate.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (neg_a ? (1u << 13) : 0u) |
         (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Instruction descriptor: kind::f16, D = F32, A = B = F16, K-major, M x N, optional A negate.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N, bool neg_a) {
  return (1u << 4) | (0u << 7) | (0u << 10) | (neg_a ? (1u << 13) : 0u) |
         (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// one MMA of the split arithmetic in either operand format (same shapes, same descriptors: a
// K step is 32 bytes of the 128-byte swizzle row in both, 8 TF32 or 16 FP16 elements)
template <bool F16>
__device__ __forceinline__ void mma_split(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate) {
  if constexpr (F16)
    mma_f16(d_tmem, adesc, bdesc, idesc, accumulate);
  else
    mma_tf32(d_tmem, adesc, bdesc, idesc, accumulate);
}

template <bool F16>
__host__ __device__ constexpr uint32_t idesc_split(int M, int N, bool neg_a) {
  return F16 ? idesc_f16(M, N, neg_a) : idesc_tf32(M, N, neg_a);
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns per thread
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
// 32 lanes x 32 bits, 8 consecutive columns per thread
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}
// the load of CW (8 or 16) consecutive columns
template <int CW>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[CW]) {
  static_assert(CW == 8 || CW == 16, "column chunk of 8 or 16");
  if constexpr (CW == 16)
    tmem_ld16(taddr, v);
  else
    tmem_ld8(taddr, v);
}
__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns per thread (warp-collective)
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16};" ::"r"(taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15]))
      : "memory");
}
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(
                   taddr),
               "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
               "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
               "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
               : "memory");
}
template <int CW>
__device__ __forceinline__ void tmem_st(uint32_t taddr, const float (&v)[CW]) {
  static_assert(CW == 8 || CW == 16, "column chunk of 8 or 16");
  if constexpr (CW == 16)
    tmem_st16(taddr, v);
  else
    tmem_st8(taddr, v);
}
__device__ __forceinline__ void tmem_st_wait() {
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// TF32 split: x = hi + lo with hi = x rounded to TF32 (10-bit mantissa, round to nearest) and
// lo = (x - hi) rounded to TF32 as well.  The tensor core reads only the 19 most significant bits
// of an FP32 operand, dropping the rest: an unrounded lo would be truncated toward zero there,
// which biases every product toward smaller magnitudes.  Rounded, both terms carry unbiased
// errors and hi + lo keeps 22 significant bits of x.
__host__ __device__ __forceinline__ float tf32_hi(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) {  // finite: round mantissa to 10 bits
    u += 0x1000u;
    u &= 0xffffe000u;
  }
  float r;
  memcpy(&r, &u, 4);
  return r;
}

__host__ __device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
  hi = tf32_hi(x);
  lo = tf32_hi(x - hi);
}

// FP16 split of a value already scaled into the FP16 range (|x| < 2^15): x = hi + lo with
// hi = FP16(x) and lo = FP16(x - hi), 22 significant bits like the TF32 split; the tensor core
// multiplies FP16 values exactly and accumulates in FP32.
__device__ __forceinline__ void f16_split(float x, __half& hi, __half& lo) {
  hi = __float2half_rn(x);
  lo = __float2half_rn(x - __half2float(hi));
}

// 2^e with |x| * 2^e in [2^13, 2^14) for the largest |x| of a row or tensor (1 for zero)
__host__ __device__ inline int f16_scale_exponent(float amax) {
  if (!(amax > 0.f)) return 0;
  int e;
  frexpf(amax, &e);  // amax = f * 2^e, f in [0.5, 1)
  return 14 - e;
}

}  // namespace tc
}  // namespace afqmc
