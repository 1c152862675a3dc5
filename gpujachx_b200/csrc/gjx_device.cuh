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

// 2^k as a double, k in [-1022, 1023]
__device__ __forceinline__ double pow2(const int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// 1/sqrt(a) rounded to nearest.  Our own method.  Scale a = f * 4^k with
// f in [1, 4), so that 1/sqrt(f) = Y * 2^-53 lies in (1/2, 1) with Y a
// 53-bit integer after rounding.  From the hardware-assisted estimate y:
//   * fast path (after P. Markstein, "IA-64 and Elementary Functions"):
//     e = 1 - f y^2 by two FMAs on y^2 = yh + yl (error below 2^-103), then
//     1/sqrt(f) = y (1 + e/2 + O(e^2)); in ulps the correction is
//     d = 2^53 y e / 2 within 2^-48, so Y = y 2^53 + rint(d) unless d lies
//     within 2^-40 of a half-integer;
//   * otherwise (almost never), the exact test: 1/sqrt(f) lies above the
//     midpoint (2Y+1) * 2^-54 iff (2Y+1)^2 * F < 2^160, F = f 2^52, decided
//     in integers.
// Any correctly rounded 1/sqrt returns these bits.
static __device__ __noinline__ long long rsqrt_fix_exact(long long Y, const unsigned long long F)
{
  for (int i = 0; (i < 4) && above_mid((unsigned long long)(2 * Y + 1), F); ++i)
    ++Y;
  for (int i = 0; (i < 4) && (Y > (1ll << 52)) && !above_mid((unsigned long long)(2 * Y - 1), F); ++i)
    --Y;
  return Y;
}

// the whole method, every input class; the slow path of rsqrt_rn below
static __device__ __noinline__ double rsqrt_rn_full(const double a)
{
  unsigned long long bits = (unsigned long long)__double_as_longlong(a);
  if ((bits >> 63) || ((bits >> 52) == 0x7FFu) || !(bits << 1)) { // negative, inf, nan, zero
    if (isnan(a))
      return a + a;
    if (a == 0.0)
      return copysign(__longlong_as_double(0x7ff0000000000000ll), a);
    if (a < 0.0)
      return __longlong_as_double((long long)0xfff8000000000000ull);
    return 0.0; // +inf
  }
  int sh = 0; // a = a' * 2^-sh with a' normal
  double an = a;
  if (!(bits >> 52)) {
    an = a * pow2(108);
    bits = (unsigned long long)__double_as_longlong(an);
    sh = 108;
  }
  const double ya = rsqrt(an);              // estimate of 1/sqrt(a'), within an ulp
  const int eu = (int)(bits >> 52) - 1023; // a' = m * 2^eu, m in [1, 2)
  const int k2 = eu & ~1;                  // a' = f * 2^k2, f in [1, 4)
  const double f = __longlong_as_double((long long)((bits & 0xFFFFFFFFFFFFFull) | ((unsigned long long)(1023 + (eu - k2)) << 52)));
  const int kk = (k2 - sh) / 2; // a = f * 4^kk exactly (k2 - sh is even)
  if (f == 1.0)
    return pow2(-kk);
  const double y = ya * pow2(k2 / 2); // estimate of 1/sqrt(f), in (1/2, 1] (exact scaling)
  const double yh = y * y;
  const double yl = __fma_rn(y, y, -yh);
  const double e = __fma_rn(-f, yl, __fma_rn(-f, yh, 1.0));
  const double d = (y * (0.5 * e)) * pow2(53);
  const double dr = rint(d);
  double Yd = __fma_rn(y, pow2(53), dr); // y 2^53 + rint(d): an integer below 2^54, exact
  if (fabs(d - dr) > 0.5 - 0x1.0p-40 || Yd >= pow2(53) || Yd < pow2(52)) {
    long long Y = (long long)fmin(fmax(Yd, pow2(52)), pow2(53) - 1.0);
    Yd = (double)rsqrt_fix_exact(Y, (unsigned long long)(f * pow2(52)));
  }
  return Yd * pow2(-53 - kk); // exact scaling into the normal range
}

// Fast path: the estimate from the hardware approximation (relative error
// about 2^-20, measured) refined by one second-order Newton step to about
// an ulp, then the same rounding decision as rsqrt_rn_full (after Markstein).
// The residual e = 1 - f y^2 is formed from a and the unscaled estimate ya
// (f y^2 = a ya^2: the power-of-4 scalings cancel), so the scaling of y into
// (1/2, 1] runs beside it; Y = rint(y 2^53 + d) comes from one FMA whose
// result lies in [2^52, 2^53), where doubles are the integers.  Powers of 4
// (f = 1) give 2^-kk exactly.  Whatever the decision cannot settle -- signs,
// zeros, subnormals, inf, NaN, exponents beyond +-960 (where a ya^2 could
// leave the normal range) and the rare ambiguous roundings -- goes to
// rsqrt_rn_full in one branch at the end (the fast path's values for those
// inputs are discarded), so the result is the correctly rounded 1/sqrt(a)
// either way.
__device__ __forceinline__ double rsqrt_rn(const double a)
{
  const unsigned long long bits = (unsigned long long)__double_as_longlong(a);
  const unsigned long long ef = bits >> 52; // sign and exponent field
  double y0;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y0) : "d"(a));
  const double h0 = a * y0;
  const double r0 = __fma_rn(-h0, y0, 1.0);
  const double ya = __fma_rn(y0 * r0, __fma_rn(0.375, r0, 0.5), y0); // y0 (1 + r0/2 + 3 r0^2/8)
  const int eu = (int)ef - 1023;
  const int kk = (eu & ~1) / 2; // a = f * 4^kk, f in [1, 4)
  // e = 1 - f y^2 with y^2 = yh + yl split exactly (y = ya 2^kk, f = a 4^-kk)
  const double yh = ya * ya;
  const double yl = __fma_rn(ya, ya, -yh);
  const double e = __fma_rn(-a, yl, __fma_rn(-a, yh, 1.0));
  const double y52 = ya * pow2(52 + kk); // y 2^52 (exact), beside the residual
  // the correction in ulps of y, (y (e/2)) 2^53 = (y 2^52) e
  const double d = y52 * e;
  // Y = y 2^53 + rint(d): y 2^53 is an integer, and the FMA rounds the sum
  // in [2^52, 2^53) to an integer (ties cannot occur: they are refused below)
  const double Yd = __fma_rn(y52, 2.0, d);
  const double dr = Yd - 2.0 * y52; // rint(d), exact
  // a power of 4 (f = 1, e.g. 1 + t^2 = 1 for a tiny rotation angle): 2^-kk exactly
  const bool p4 = !(bits & 0xFFFFFFFFFFFFFull) && !(eu & 1);
  const double res = p4 ? pow2(-kk) : Yd * pow2(-53 - kk);
  if ((ef - 1ull > 2045ull) || (eu < -960) || (eu > 960) ||
      (!p4 && (!(fabs(d) < 0x1.0p50) || fabs(d - dr) > 0.5 - 0x1.0p-40 || Yd >= pow2(53) || Yd < pow2(52))))
    return rsqrt_rn_full(a);
  return res;
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
// The three cases of each are evaluated without branching (the operands of
// the case that applies are selected, then the same operations run), so the
// 16 lanes that compute 16 rotations at once never diverge.
__device__ __forceinline__ int rotT(const double Apq, const double Dp, const double Dq, double &c, double &t)
{
  const double h = Dq - Dp;
  const double ct2 = __ddiv_rn(h, Apq * 2.0);
  const double CT2 = fabs(ct2);
  const bool small = CT2 < kSqrtHeps, large = CT2 >= kSqrt2Heps;
  const double cot_mid = CT2 + __dsqrt_rn(__fma_rn(CT2, CT2, 1.0));
  const double cot = small ? (CT2 + 1.0) : (large ? (CT2 * 2.0) : cot_mid);
  t = copysign(__drcp_rn(cot), ct2);
  const double cr = rsqrt_rn(__fma_rn(t, t, 1.0));
  c = large ? 1.0 : cr;
  return small ? 1 : (large ? 0 : (cr < 1.0));
}

__device__ __forceinline__ int rotH(const double Apq, const double Dp, const double Dq, double &c, double &t)
{
  const double h = Dq + Dp;
  const double ct2 = -__ddiv_rn(h, Apq * 2.0);
  const double CT2 = fabs(ct2);
  const bool large = CT2 >= kSqrt2Heps, mid = !large && (CT2 > 1.0);
  const double cot_mid = CT2 + __dsqrt_rn(__fma_rn(CT2, CT2, -1.0));
  const double cot = large ? (CT2 * 2.0) : cot_mid;
  const double tt = copysign(__drcp_rn(cot), ct2);
  const double cr = rsqrt_rn(__fma_rn(-tt, tt, 1.0));
  c = large ? 1.0 : (mid ? cr : kCoshIFix);
  t = (large || mid) ? tt : kTanh1Fix;
  return large ? 0 : (mid ? (cr > 1.0) : 1);
}

// one inner rotation, as the lanes that compute it hand it to those that apply it
struct Rot {
  double c, t, t_;
  int mode; // 0 nothing, 1 rotate, 2 swap columns
  int scale, swap;
};

// rotT for the lanes with trig, rotH for the others, in one chain.  The two
// formulas take the same operations up to signs -- Dq - Dp is Dq + (-Dp)
// exactly, the quotient negated, +1 or -1 under the square root, t t + 1 or
// -t t + 1 under the reciprocal square root -- and their special cases are
// selects, so each lane gets exactly the operations of its own formula while
// a warp whose lanes need both kinds runs one chain of divides and square
// roots instead of two.
__device__ __forceinline__ int rotTH(const bool trig, const double Apq, const double Dp, const double Dq, double &c,
                                     double &t)
{
  const double h = Dq + (trig ? -Dp : Dp);
  const double qt = __ddiv_rn(h, Apq * 2.0);
  const double ct2 = trig ? qt : -qt;
  const double CT2 = fabs(ct2);
  const bool large = CT2 >= kSqrt2Heps;
  const bool small = trig && (CT2 < kSqrtHeps);      // rotT's first case
  const bool mid = !trig && !large && (CT2 > 1.0);  // rotH's middle case
  const double cot_mid = CT2 + __dsqrt_rn(__fma_rn(CT2, CT2, trig ? 1.0 : -1.0));
  const double cot = small ? (CT2 + 1.0) : (large ? (CT2 * 2.0) : cot_mid);
  const double tt = copysign(__drcp_rn(cot), ct2);
  const double cr = rsqrt_rn(__fma_rn(trig ? tt : -tt, tt, 1.0));
  c = large ? 1.0 : ((trig || mid) ? cr : kCoshIFix);
  t = (trig || large || mid) ? tt : kTanh1Fix;
  return trig ? (small ? 1 : (large ? 0 : (cr < 1.0))) : (large ? 0 : (mid ? (cr > 1.0) : 1));
}

// rotT (trig) or rotH; when the lanes of the warp need different kinds, the
// merged chain of rotTH (each is a long dependent chain of divisions and
// square roots)
__device__ __forceinline__ int rot_either(const bool trig, const double Apq, const double Dp, const double Dq,
                                          double &c, double &t)
{
  if (__all_sync(0xffffffffu, trig))
    return rotT(Apq, Dp, Dq, c, t);
  if (__all_sync(0xffffffffu, !trig))
    return rotH(Apq, Dp, Dq, c, t);
  return rotTH(trig, Apq, Dp, Dq, c, t);
}

template <bool SORT>
__device__ __forceinline__ Rot inner_rot(const double Dp, const double Dq, const double Apq, const unsigned p,
                                         const unsigned q, const int definite, const unsigned npos, unsigned &ts_out,
                                         unsigned &tb_out)
{
  // branch-free: the two half-warps handle different pairs, so every choice
  // below is a select of values computed by both (no divergent paths)
  Rot r;
  const double Dp_ = __dsqrt_rn(Dp), Dq_ = __dsqrt_rn(Dq), Apq_ = fabs(Apq), Dpq_ = Dp_ * Dq_;
  const int ts = !(Apq_ < (Dpq_ * kMyTol));
  int tb;
  if (!SORT) {
    // the rotation is computed whether or not it is applied (no side
    // effects), so that its latency overlaps the relative test
    const bool trig = definite || ((p < npos) && (q < npos)) || ((p >= npos) && (q >= npos));
    double c, t;
    const int b = rot_either(trig, Apq, Dp, Dq, c, t);
    r.c = ts ? c : 1.0;
    r.t = ts ? t : 0.0;
    r.t_ = ts ? (trig ? -t : t) : 0.0;
    tb = ts ? b : 0;
    r.mode = ts;
    r.scale = tb;
    r.swap = 0;
  }
  else {
    const int def = definite ? definite : ((p < npos) && (q < npos)) ? +1 : ((p >= npos) && (q >= npos)) ? -1 : 0;
    double c, t;
    const int b = rot_either(def != 0, Apq, Dp, Dq, c, t);
    const double t_ = def ? -t : t;
    const double Dp2 = __fma_rn(t, Apq, Dp), Dq2 = __fma_rn(t_, Apq, Dq); // used when ts and def
    const int swp = !((!def) || ((def > 0) && (Dp2 >= Dq2)) || ((def < 0) && (Dp2 <= Dq2)));
    const int order = ((def > 0) && (Dp < Dq)) || ((def < 0) && (Dq < Dp));
    r.c = ts ? c : 1.0;
    r.t = ts ? t : 0.0;
    r.t_ = ts ? t_ : 0.0;
    tb = ts ? b : 0;
    r.mode = ts ? 1 : (order ? 2 : 0);
    r.scale = tb;
    r.swap = ts ? swp : 0;
  }
  ts_out = (unsigned)ts;
  tb_out = (unsigned)tb;
  return r;
}

// a named barrier for the nthreads threads of a warp group (id 0 with all the
// CTA's threads is __syncthreads)
__device__ __forceinline__ void bar_sync(const unsigned id, const unsigned nthreads)
{
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
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

__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"((uint32_t)__cvta_generic_to_shared(bar)) : "memory");
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

// 16-byte asynchronous copy global -> shared (both 16-byte aligned), L2 only
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// one arrival on the mbarrier once all prior cp.async of this thread completed
__device__ __forceinline__ void cp_async_arrive(uint64_t *bar)
{
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// TMA tensor copy of a 3-D box at (c0, c1, c2) of the tensor map (kernel
// parameter space) into shared memory, completing bytes on the mbarrier.
// c0 * element size must be a multiple of 16 bytes (c0 = 0 here).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *tm, const int c0, const int c1,
                                            const int c2, uint64_t *bar)
{
  asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
               "[%5];" ::"r"(smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
               : "memory");
}

// TMA tensor store of a 3-D box of shared memory to (c0, c1, c2) of the
// tensor map, in this thread's current bulk async-group; elements of the box
// outside the tensor are not written.  c0 = 0 here; no coordinate is negative.
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *tm, const void *src, const int c0, const int c1,
                                             const int c2)
{
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(tm)),
               "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}

// close this thread's bulk async-group
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// this thread's bulk groups have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// all but this thread's most recent bulk group have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_but1() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }

// this thread's bulk groups are complete (their global writes performed),
// and ordered before this thread's later generic-proxy operations
__device__ __forceinline__ void bulk_wait_all()
{
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// this thread's shared-memory writes become visible to the async proxy (a TMA
// store issued after a barrier)
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

} // namespace gjx
