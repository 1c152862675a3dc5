// gjx_device.cuh -- sm_100a device primitives of the blocked one-sided Jacobi.
//
// Every arithmetic routine here produces the same bits as the corresponding
// reference routine (share/device_code_common*.hpp): the operations are IEEE
// correctly rounded (__fma_rn, __ddiv_rn, __dsqrt_rn, __drcp_rn) and are
// applied in the reference's order, so a block-pair step computed here equals
// the reference's bit for bit.  This file is compiled with --fmad=false so
// that no a*b+c is contracted behind our back.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gjx_internal.h"

namespace gjx {

// sqrt(2^-53), sqrt(2/2^-53) = 2^27, sqrt(32)*2^-53, 2/sqrt(3), 1/2:
// correctly rounded values of the definitions in share/HypJacL.hpp:21-59.
constexpr double kSqrtHeps = 0x1.6a09e667f3bcdp-27;
constexpr double kSqrt2Heps = 0x1.0p+27;
constexpr double kMyTol = 0x1.6a09e667f3bcdp-51;
constexpr double kCoshIFix = 0x1.279a74590331cp+0;
constexpr double kTanh1Fix = 0.5;


// ---------------------------------------------------------------------------
// correctly rounded 1/sqrt
// ---------------------------------------------------------------------------

// Is 1/sqrt(F) above the midpoint (2Y+1) * 2^-80, i.e. (2Y+1)^2 * F < 2^160?
__device__ __forceinline__ bool above_mid(const unsigned long long y2p1, const unsigned long long F)
{
  const unsigned long long Pl = y2p1 * y2p1;             // (2Y+1)^2 < 2^108
  const unsigned long long Ph = __umul64hi(y2p1, y2p1);
  const unsigned long long lo_hi = __umul64hi(Pl, F);    // (Pl * F) >> 64
  const unsigned long long hh_lo = Ph * F;               // Ph * F < 2^98
  const unsigned long long hh_hi = __umul64hi(Ph, F);
  const unsigned long long T_lo = hh_lo + lo_hi;         // (P * F) >> 64
  const unsigned long long T_hi = hh_hi + (T_lo < hh_lo ? 1ull : 0ull);
  return T_hi < (1ull << 32);                            // (P * F) >> 64 < 2^96
}

// 1/sqrt(a) rounded to nearest.  Our own method: a = F * 2^e, e even,
// F in [2^52, 2^54); 1/sqrt(F) = Y * 2^-79 with a 53-bit Y is bracketed by an
// estimate from two correctly rounded operations and fixed by exact integer
// tests of the rounding midpoints (the sign of 1 - m^2 F).  Any correctly
// rounded 1/sqrt returns these bits.
__device__ __forceinline__ double rsqrt_rn(const double a)
{
  if (!(a > 0.0) || isinf(a)) {
    if (isnan(a))
      return a + a;
    if (a == 0.0)
      return copysign(__longlong_as_double(0x7ff0000000000000ll), a);
    if (a < 0.0)
      return __longlong_as_double((long long)0xfff8000000000000ull);
    return 0.0; // +inf
  }
  const unsigned long long bits = (unsigned long long)__double_as_longlong(a);
  int E = (int)((bits >> 52) & 0x7FFu);
  unsigned long long F = bits & 0xFFFFFFFFFFFFFull;
  if (E)
    F |= (1ull << 52);
  else {
    const int sh = __clzll((long long)F) - 11;
    F <<= sh;
    E = 1 - sh;
  }
  int e = E - 1075;
  if (e & 1) {
    F <<= 1;
    --e;
  }
  if (F == (1ull << 52))
    return scalbn(1.0, -26 - e / 2);
  const double est = __drcp_rn(__dsqrt_rn(__ull2double_rn(F)));
  long long Y = __double2ll_rz(scalbn(est, 79));
  if (Y >= (1ll << 53))
    Y = (1ll << 53) - 1;
  if (Y < (1ll << 52))
    Y = (1ll << 52);
  // the estimate is within two ulps: at most a few corrections, bounded
  for (int i = 0; (i < 4) && above_mid((unsigned long long)(2 * Y + 1), F); ++i)
    ++Y;
  for (int i = 0; (i < 4) && (Y > (1ll << 52)) && !above_mid((unsigned long long)(2 * Y - 1), F); ++i)
    --Y;
  return scalbn(__ll2double_rn(Y), -79 - e / 2);
}

// ---------------------------------------------------------------------------
// 32-lane butterfly sum (share/device_code_common_Kepler.hpp:26-74): lane i
// adds lane i^16, i^8, i^4, i^2, i^1; the result is lane 0's, broadcast.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sum32(double v)
{
  v = v + __shfl_xor_sync(0xffffffffu, v, 16);
  v = v + __shfl_xor_sync(0xffffffffu, v, 8);
  v = v + __shfl_xor_sync(0xffffffffu, v, 4);
  v = v + __shfl_xor_sync(0xffffffffu, v, 2);
  v = v + __shfl_xor_sync(0xffffffffu, v, 1);
  return __shfl_sync(0xffffffffu, v, 0);
}

// ---------------------------------------------------------------------------
// 2x2 rotations (share/device_code_common_rotate.hpp:16-64, USE_RSQRT form).
// Return 1 for a "big" rotation (c != 1), 0 otherwise.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int rotT(const double Apq, const double Dp, const double Dq, double &c, double &t)
{
  const double h = Dq - Dp;
  const double ct2 = __ddiv_rn(h, Apq * 2.0);
  const double CT2 = fabs(ct2);
  if (CT2 < kSqrtHeps) {
    const double cot = CT2 + 1.0;
    t = copysign(__drcp_rn(cot), ct2);
    c = rsqrt_rn(__fma_rn(t, t, 1.0));
    return 1;
  }
  else if (CT2 >= kSqrt2Heps) {
    const double cot = CT2 * 2.0;
    c = 1.0;
    t = copysign(__drcp_rn(cot), ct2);
    return 0;
  }
  else {
    const double cot = CT2 + __dsqrt_rn(__fma_rn(CT2, CT2, 1.0));
    t = copysign(__drcp_rn(cot), ct2);
    c = rsqrt_rn(__fma_rn(t, t, 1.0));
    return (c < 1.0);
  }
}

__device__ __forceinline__ int rotH(const double Apq, const double Dp, const double Dq, double &c, double &t)
{
  const double h = Dq + Dp;
  const double ct2 = -__ddiv_rn(h, Apq * 2.0);
  const double CT2 = fabs(ct2);
  if (CT2 >= kSqrt2Heps) {
    const double cot = CT2 * 2.0;
    c = 1.0;
    t = copysign(__drcp_rn(cot), ct2);
    return 0;
  }
  else if (CT2 > 1.0) {
    const double cot = CT2 + __dsqrt_rn(__fma_rn(CT2, CT2, -1.0));
    t = copysign(__drcp_rn(cot), ct2);
    c = rsqrt_rn(__fma_rn(-t, t, 1.0));
    return (c > 1.0);
  }
  else {
    c = kCoshIFix;
    t = kTanh1Fix;
    return 1;
  }
}

// ---------------------------------------------------------------------------
// mbarrier + bulk-copy (TMA engine) helpers, with bounded waits
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, const uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, const uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, const uint32_t parity)
{
  uint32_t done;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(done)
               : "r"(smem_u32(bar)), "r"(parity)
               : "memory");
  return done != 0u;
}

// Wait for the phase with the given parity, at most ~limit_cycles.  Returns
// false on timeout (the caller records an error and stops waiting).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, const uint32_t parity,
                                                  const long long limit_cycles)
{
  if (mbar_try_wait(bar, parity))
    return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit_cycles)
      return false;
  }
  return true;
}

// 1-D bulk copy global -> shared, completing bytes on the mbarrier.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, const uint32_t bytes, uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

} // namespace gjx
