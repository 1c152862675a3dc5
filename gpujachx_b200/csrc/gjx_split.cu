// gjx_split.cu -- the split-precision form (gjx_hypJacL2_split).
//
// The same blocked one-sided Jacobi as the plain form, with its two dense
// contractions -- the Gram matrix of each pivot block pair and the update of
// G and V by the pair's accumulated transform -- run on the tensor cores as
// exact integer products of 8-bit slices (tcgen05.mma kind::i8, int32
// accumulators in tensor memory), recombined in FP64.  What stays native
// FP64: the Cholesky factor of each pair's Gram matrix, the inner 2x2
// rotations and their relative convergence test (the plain form's rotT /
// rotH / inner_rot), the J-signed hyperbolic formulas, the column norms and D.
//
// Geometry: blocks of 32 columns, pairs of 64 (twice the reference's 16 and
// 32: with wider pairs each byte of G and V moved per sweep carries twice the
// arithmetic, and a 64 x 64 Gram fills the tensor core's operand shapes).
// The outer pivot tables are the loaded family's for n1 = ncol / 32, the
// inner ones the family's for 64 columns.
//
// Slicing (Ozaki's scheme, balanced digits).  A column c of the operand is
// scaled by 2^-e_c, e_c the exponent bound of its largest |entry| (|a| <
// 2^e_c), so each entry becomes x = a 2^-e_c in (-1, 1); v = rint(x 2^55) is a
// 56-bit integer, written as v = sum_t d_t 2^(49 - 7t), t = 0..7: d_0 in
// [-64, 64], d_1..d_7 in [-64, 63] (balanced base-128 digits).  Each digit
// plane is an int8 matrix.  A product of two such operands is
//   sum_k v_ik w_kj = sum_(t,u) 2^(98 - 7(t+u)) sum_k d_t,ik d_u,kj,
// and the slice products with t + u <= 7 are kept: 36 int8 x int8 -> int32
// products, summed exactly per group g = t + u in 8 int32 accumulators, then
// F = sum_g 2^-7g S_g in FP64 (Horner, low groups first) and a power-of-two
// scale.  The slicing error is 2^-56 of the column's scale per entry, the
// truncation of the groups g >= 8 about 2^-55 of the product's scale: the
// order of FP64 rounding.  The scales are tracked exactly: the update kernel
// folds the largest |entry| of every column it writes into a per-column word
// (atomic max of the high words), read by the next step (by step parity).
//
// Kernels, per outer step:
//   sp_pair_kernel    one CTA per block pair: the Gram matrix (TMA tensor
//                     copies of 64-row tiles, slicing into K-major digit
//                     planes, 26 MMAs of 128 x 64 x 32 per 32 rows: the A
//                     operand stacks planes t and t + 4, so one MMA yields
//                     groups t + u and t + 4 + u), its Cholesky factor, the
//                     inner sweep(s), and the digit planes of the update's B
//                     operand diag(2^e) V_loc (for G and for V) in global
//                     memory;
//   sp_update_kernel  one CTA per 128 rows of a pair's columns of G or V: the
//                     FP64 tile by TMA, sliced, 72 MMAs of 128 x 64 x 32, the
//                     epilogue back to FP64 in place by TMA stores, and the
//                     tile's column maxima.
// Every wait is bounded (kWait cycles): on a timeout the kernel sets the
// error word and leaves.
#include <cudaTypedefs.h>
#include <mutex>
#include <string>
#include <vector>

#include "gjx.h"
#include "gjx_device.cuh"
#include "gjx_internal.h"

namespace gjx {
namespace split {

constexpr unsigned kThreads = 256u;
constexpr unsigned kBW = 32u;    // columns per block
constexpr unsigned kW = 64u;     // columns per block pair
constexpr unsigned kDig = 8u;    // digits per value
constexpr long long kWait = 2000000000ll;
constexpr unsigned kTmemCols = 512u; // 8 accumulators x 64 columns
// sum_{t=1..7} 64 * 2^(49 - 7t): added before cutting the low digits so that
// each becomes a field in [0, 127] standing for the digit + 64
constexpr long long kDigitBias = 64ll * ((1ll << 42) + (1ll << 35) + (1ll << 28) + (1ll << 21) + (1ll << 14) +
                                         (1ll << 7) + 1ll);

struct Params {
  CUtensorMap tmGram; // 3-D view (64 rows, tiles, columns) of G, box {66, 1, 16} (the plain form's)
  CUtensorMap tmG;    // 2-D view (rows, columns) of G, box {128, 32}
  CUtensorMap tmV;    // the same of V
  const uint16_t *strat1; // [steps1][pairs][2], blocks of 32 columns
  const uint8_t *strat0;  // [s0steps][32][2], 64 columns
  unsigned long long *cvg;
  int *err;
  uint32_t *cmaxG; // [2][ncol]: high word of the largest |entry| of each column, by step parity
  uint32_t *cmaxV; // [2][ncol]
  uint8_t *bop;    // per pair: the update's B operands (G, then V): kBopBytes each
  unsigned nrow, ncol, nplus, pairs, step, parity, s0steps, nswp0;
  unsigned tilesG, tilesV; // 128-row tiles of G and of V
  int gdefinite;
  int accv;
};

// ---- the update's B operand in global memory: 8 digit planes (K-major,
// 64 x 64 bytes each, core matrices of 8 rows x 16 bytes, LBO 128, SBO 512)
// then the 64 column exponents h_j
constexpr uint32_t kBPlane = 4096u;
constexpr uint32_t kBopBytes = kDig * kBPlane + 256u;

// ---------------------------------------------------------------------------
// tcgen05 helpers
// ---------------------------------------------------------------------------
// shared-memory matrix descriptor, no swizzle (K-major canonical layout:
// core matrices of 8 rows x 16 bytes; lbo = byte step between core matrices
// along K, sbo = along M/N)
__device__ __forceinline__ uint64_t sdesc(const uint32_t saddr, const uint32_t lbo, const uint32_t sbo)
{
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46); // version 1 (sm_100), base offset 0, no swizzle
}

// instruction descriptor: kind::i8, s8 x s8 -> s32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_i8(const unsigned M, const unsigned N)
{
  return (2u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(const uint32_t dtmem, const uint64_t a, const uint64_t b, const uint32_t idesc,
                                       const uint32_t accumulate)
{
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(dtmem),
               "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
               : "memory");
}

// one arrival on the mbarrier when every MMA issued so far by this thread is complete
__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// by one whole warp: allocate the CTA's 512 TMEM columns, address into *dst
__device__ __forceinline__ void tmem_alloc(uint32_t *dst)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(kTmemCols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(const uint32_t taddr)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(kTmemCols) : "memory");
}

// 16 consecutive 32-bit columns of this warp's 32 lanes (one row per thread)
__device__ __forceinline__ void tmem_ld16(const uint32_t taddr, int (&v)[16])
{
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
               "%14, %15}, [%16];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                 "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                 "=r"(v[15])
               : "r"(taddr)
               : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 2-D TMA tensor copy / store of the box at (c0, c1)
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *tm, const int c0, const int c1,
                                            uint64_t *bar)
{
  asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
               "[%4];" ::"r"(smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap *tm, const void *src, const int c0, const int c1)
{
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(
                   reinterpret_cast<uint64_t>(tm)),
               "r"(smem_u32(src)), "r"(c0), "r"(c1)
               : "memory");
}

// ---------------------------------------------------------------------------
// digits
// ---------------------------------------------------------------------------
// exponent bound of a column from the high word of its largest |entry|:
// every entry is below 2^e (a zero or subnormal column: e = -1022)
__device__ __forceinline__ int col_exp(const uint32_t hw) { return (int)((hw >> 20) & 0x7FFu) - 1022; }

// 2^k for k in [-1022, 1023]
__device__ __forceinline__ double p2(const int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// x * 2^k exactly (no intermediate over- or underflow for the k used here:
// |k| <= 2100, two factors of at most 2^1050 each side)
__device__ __forceinline__ double scale2(const double x, const int k)
{
  const int k1 = k / 2;
  return (x * p2(k1)) * p2(k - k1);
}

// the 56-bit integer of a * 2^(55 - e) (|a| < 2^e), biased for digit cutting
__device__ __forceinline__ long long biased_int(const double a, const int e)
{
  long long v = __double2ll_rn(scale2(a, 55 - e));
  v = max(min(v, 1ll << 55), -(1ll << 55)); // |a| < 2^e holds by construction; never exceed the digit range
  return v + kDigitBias;
}

// plane t's bytes of four values (the words w[0..3] from biased_int): byte j
// of the result is digit t of value j as an int8
template <unsigned T> __device__ __forceinline__ uint32_t plane_word(const long long (&w)[4])
{
  if (T == 0u) { // d_0 = w >> 49 in [-64, 64]: its 8 low bits
    uint32_t r = 0u;
#pragma unroll
    for (unsigned j = 0u; j < 4u; ++j)
      r |= ((uint32_t)(w[j] >> 49) & 0xFFu) << (8u * j);
    return r;
  }
  else { // field f = bits [49 - 7T, 56 - 7T) in [0, 127] stands for f - 64: sign-extend (f ^ 64) from 7 bits
    uint32_t r = 0u;
#pragma unroll
    for (unsigned j = 0u; j < 4u; ++j)
      r |= ((uint32_t)(w[j] >> (49u - 7u * T)) & 0x7Fu) << (8u * j);
    r ^= 0x40404040u;
    return r | ((r & 0x40404040u) << 1);
  }
}

// 16 values -> 16 bytes of each of the 8 planes
__device__ __forceinline__ void digits16(const long long (&w)[16], uint4 (&out)[kDig])
{
#define GJX_PLANE(T)                                                                                                 \
  {                                                                                                                  \
    uint32_t q[4];                                                                                                   \
    _Pragma("unroll") for (unsigned k = 0u; k < 4u; ++k)                                                             \
    {                                                                                                                \
      const long long ww[4] = {w[4u * k], w[4u * k + 1u], w[4u * k + 2u], w[4u * k + 3u]};                           \
      q[k] = plane_word<T>(ww);                                                                                      \
    }                                                                                                                \
    out[T] = make_uint4(q[0], q[1], q[2], q[3]);                                                                     \
  }
  GJX_PLANE(0u) GJX_PLANE(1u) GJX_PLANE(2u) GJX_PLANE(3u) GJX_PLANE(4u) GJX_PLANE(5u) GJX_PLANE(6u) GJX_PLANE(7u)
#undef GJX_PLANE
}

// F = sum_g 2^-7g S_g, low groups first
__device__ __forceinline__ double recombine(const int (&s)[kDig])
{
  double f = (double)s[7];
#pragma unroll
  for (int g = 6; g >= 0; --g)
    f = __fma_rn(f, 0x1.0p-7, (double)s[g]);
  return f;
}

__device__ __forceinline__ uint32_t abs_hi(const double x)
{
  return (uint32_t)(__double_as_longlong(x) >> 32) & 0x7FFFFFFFu;
}

// ---------------------------------------------------------------------------
// sp_pair_kernel
// ---------------------------------------------------------------------------
// Gram staging: 3 stages of one 64-row tile of the pair's 64 columns, four
// boxes {66 rows, 1 tile, 16 columns}: column c at c * 66 doubles (528 bytes,
// an odd number of 16-byte granules: 8 consecutive columns in 8 bank groups)
constexpr unsigned kGStages = 3u;
constexpr uint32_t kGBox = 66u * 16u * 8u;         // 8448 bytes
constexpr uint32_t kGStageBytes = 4u * kGBox;       // 33792
// digit planes of a 64-row tile: 2 chunks of 32 rows x 8 planes x 2 KB; the
// planes of a chunk in the order 0, 4, 1, 5, 2, 6, 3, 7 so that planes t and
// t + 4 form one 128-row A operand
constexpr uint32_t kGPlane = 2048u;
constexpr uint32_t kGChunk = kDig * kGPlane;        // 16384
constexpr uint32_t kGTilePlanes = 2u * kGChunk;     // 32768
constexpr unsigned kGPlaneBufs = 2u;
constexpr uint32_t kOffGStage = 0u;
constexpr uint32_t kOffGPlanes = kGStages * kGStageBytes;                     // 101376
constexpr uint32_t kOffGEnd = kOffGPlanes + kGPlaneBufs * kGTilePlanes;       // 166912
// after the Gram (reusing the staging): R and V_loc (64 x 64, ld 65), the
// groups 4..7 of the bottom accumulator halves (int32 [4][64][64])
constexpr unsigned kLd = 65u;
constexpr uint32_t kOffR = 0u;
constexpr uint32_t kOffVl = kOffR + 64u * kLd * 8u;                          // 33280
constexpr uint32_t kOffBot = kOffVl + 64u * kLd * 8u;                        // 66560, 65536 bytes
static_assert(kOffBot + 65536u <= kOffGEnd, "Gram epilogue scratch must fit");
// fixed region after it
constexpr uint32_t kOffS0 = kOffGEnd;                                        // inner table, 64 steps x 64 bytes
constexpr uint32_t kOffScale = kOffS0 + 4096u;                               // 64 int: e_c of G; 64 int: of V
constexpr uint32_t kOffRed = kOffScale + 512u;                               // 64 unsigned
constexpr uint32_t kOffBar = kOffRed + 256u;                                 // 8 mbarriers
constexpr uint32_t kOffTmem = kOffBar + 64u;
constexpr uint32_t kPairSmem = kOffTmem + 16u;
static_assert(kPairSmem <= 227u * 1024u, "shared memory of sp_pair_kernel");

__device__ __forceinline__ void set_err(const Params &P) { atomicExch(P.err, kErrWaitTimeout); }

// signature of block pair (i, j) of 32-column blocks (as the plain form's
// block_signature with blocks of 32)
__device__ __forceinline__ void pair_signature(const Params &P, const unsigned iBlk, const unsigned jBlk,
                                               int &definite, unsigned &npos)
{
  const unsigned ifc0 = iBlk * kBW, ifc1 = jBlk * kBW, nplus = P.nplus;
  if (P.gdefinite) {
    definite = P.gdefinite;
    npos = 0u;
  }
  else if (nplus <= ifc0) {
    npos = 0u;
    definite = -1;
  }
  else if (nplus <= ifc0 + kBW) {
    npos = nplus - ifc0;
    definite = 0;
  }
  else if (nplus <= ifc1) {
    npos = kBW;
    definite = 0;
  }
  else if (nplus <= ifc1 + kBW) {
    npos = kBW + (nplus - ifc1);
    definite = 0;
  }
  else {
    npos = 2u * kBW;
    definite = +1;
  }
}

// the inner sweep(s) on R (64 x 64) accumulating V_loc: per inner step warp w
// takes pairs 4w .. 4w + 3; lane x holds rows x and x + 32; quarter c of the
// warp (lanes 8c .. 8c + 7) evaluates pair 4w + c's rotation, every lane
// applies all four.  One barrier per step.
template <bool SORT>
__device__ void inner64(double *const R, double *const Vl, const uint8_t *const s0, const unsigned s0steps,
                        const unsigned nswp, const int definite, const unsigned npos, unsigned *const red,
                        unsigned &blk_s, unsigned &blk_b)
{
  const unsigned tid = threadIdx.x, x = tid & 31u, w = tid >> 5;
  blk_s = 0u;
  blk_b = 0u;
  for (unsigned swp = 0u; swp < nswp; ++swp) {
    unsigned ws = 0u, wb = 0u;
    for (unsigned step = 0u; step < s0steps; ++step) {
      const uint8_t *const st = s0 + step * 64u;
      unsigned p[4], q[4];
      double gp0[4], gp1[4], gq0[4], gq1[4], vp0[4], vp1[4], vq0[4], vq1[4], d[4][3];
#pragma unroll
      for (unsigned c = 0u; c < 4u; ++c) {
        const unsigned k = 4u * w + c;
        p[c] = st[2u * k];
        q[c] = st[2u * k + 1u];
        gp0[c] = R[p[c] * kLd + x];
        gp1[c] = R[p[c] * kLd + x + 32u];
        gq0[c] = R[q[c] * kLd + x];
        gq1[c] = R[q[c] * kLd + x + 32u];
        vp0[c] = Vl[p[c] * kLd + x];
        vp1[c] = Vl[p[c] * kLd + x + 32u];
        vq0[c] = Vl[q[c] * kLd + x];
        vq1[c] = Vl[q[c] * kLd + x + 32u];
        d[c][0] = __fma_rn(gp1[c], gp1[c], gp0[c] * gp0[c]);
        d[c][1] = __fma_rn(gq1[c], gq1[c], gq0[c] * gq0[c]);
        d[c][2] = __fma_rn(gp1[c], gq1[c], gp0[c] * gq0[c]);
      }
#pragma unroll
      for (unsigned o = 16u; o; o >>= 1u)
#pragma unroll
        for (unsigned c = 0u; c < 4u; ++c)
#pragma unroll
          for (unsigned i = 0u; i < 3u; ++i)
            d[c][i] += __shfl_xor_sync(0xffffffffu, d[c][i], o);
      const unsigned mc = x >> 3; // this lane's pair among the warp's four
      double Dp = d[0][0], Dq = d[0][1], Apq = d[0][2];
      unsigned pm = p[0], qm = q[0];
#pragma unroll
      for (unsigned c = 1u; c < 4u; ++c)
        if (mc == c) {
          Dp = d[c][0];
          Dq = d[c][1];
          Apq = d[c][2];
          pm = p[c];
          qm = q[c];
        }
      unsigned a_s = 0u, a_b = 0u;
      const Rot mine = inner_rot<SORT>(Dp, Dq, Apq, pm, qm, definite, npos, a_s, a_b);
      if ((x & 7u) == 0u) {
        ws += a_s;
        wb += a_b;
      }
#pragma unroll
      for (unsigned c = 0u; c < 4u; ++c) {
        Rot r;
        r.c = __shfl_sync(0xffffffffu, mine.c, 8u * c);
        r.t = __shfl_sync(0xffffffffu, mine.t, 8u * c);
        r.t_ = __shfl_sync(0xffffffffu, mine.t_, 8u * c);
        const int fl = __shfl_sync(0xffffffffu, mine.mode | (mine.scale << 2) | (mine.swap << 3), 8u * c);
        r.mode = fl & 3;
        r.scale = (fl >> 2) & 1;
        r.swap = (fl >> 3) & 1;
        if (r.mode == 0)
          continue;
        const unsigned pp = p[c], qq = q[c];
        if (r.mode == 2) {
          R[pp * kLd + x] = gq0[c];
          R[pp * kLd + x + 32u] = gq1[c];
          R[qq * kLd + x] = gp0[c];
          R[qq * kLd + x + 32u] = gp1[c];
          Vl[pp * kLd + x] = vq0[c];
          Vl[pp * kLd + x + 32u] = vq1[c];
          Vl[qq * kLd + x] = vp0[c];
          Vl[qq * kLd + x + 32u] = vp1[c];
          continue;
        }
        double np0 = __fma_rn(r.t_, gq0[c], gp0[c]), nq0 = __fma_rn(r.t, gp0[c], gq0[c]);
        double np1 = __fma_rn(r.t_, gq1[c], gp1[c]), nq1 = __fma_rn(r.t, gp1[c], gq1[c]);
        double mp0 = __fma_rn(r.t_, vq0[c], vp0[c]), mq0 = __fma_rn(r.t, vp0[c], vq0[c]);
        double mp1 = __fma_rn(r.t_, vq1[c], vp1[c]), mq1 = __fma_rn(r.t, vp1[c], vq1[c]);
        if (r.scale) {
          np0 *= r.c;
          nq0 *= r.c;
          np1 *= r.c;
          nq1 *= r.c;
          mp0 *= r.c;
          mq0 *= r.c;
          mp1 *= r.c;
          mq1 *= r.c;
        }
        const unsigned dp = r.swap ? qq : pp, dq = r.swap ? pp : qq;
        R[dp * kLd + x] = np0;
        R[dp * kLd + x + 32u] = np1;
        R[dq * kLd + x] = nq0;
        R[dq * kLd + x + 32u] = nq1;
        Vl[dp * kLd + x] = mp0;
        Vl[dp * kLd + x + 32u] = mp1;
        Vl[dq * kLd + x] = mq0;
        Vl[dq * kLd + x + 32u] = mq1;
      }
      __syncthreads();
    }
    ws = __reduce_add_sync(0xffffffffu, ws);
    wb = __reduce_add_sync(0xffffffffu, wb);
    if (x == 0u) {
      red[2u * w] = ws;
      red[2u * w + 1u] = wb;
    }
    __syncthreads();
    unsigned tot_s = 0u, tot_b = 0u;
#pragma unroll
    for (unsigned k = 0u; k < 8u; ++k) {
      tot_s += red[2u * k];
      tot_b += red[2u * k + 1u];
    }
    __syncthreads();
    if (!tot_s)
      break;
    blk_s += tot_s;
    blk_b += tot_b;
  }
}

// the update's B operand diag(2^e_k) V_loc of one matrix: 8 digit planes
// (K-major, n = output column j, k = pair column) and the exponents h_j,
// written to global memory.  Thread (j = tid / 4, kg = tid % 4) takes
// k = 16 kg .. 16 kg + 15 of column j.
__device__ void bop_write(const double *const Vl, const int *const e, uint8_t *const out)
{
  const unsigned tid = threadIdx.x, j = tid >> 2, kg = tid & 3u;
  double b[16];
  uint32_t hw = 0u;
#pragma unroll
  for (unsigned i = 0u; i < 16u; ++i) {
    const unsigned k = 16u * kg + i;
    b[i] = scale2(Vl[j * kLd + k], e[k]);
    hw = max(hw, abs_hi(b[i]));
  }
  hw = max(hw, __shfl_xor_sync(0xffffffffu, hw, 1));
  hw = max(hw, __shfl_xor_sync(0xffffffffu, hw, 2));
  const int h = col_exp(hw);
  long long w[16];
#pragma unroll
  for (unsigned i = 0u; i < 16u; ++i)
    w[i] = biased_int(b[i], h);
  uint4 pl[kDig];
  digits16(w, pl);
#pragma unroll
  for (unsigned t = 0u; t < kDig; ++t)
    *reinterpret_cast<uint4 *>(out + t * kBPlane + (j >> 3) * 512u + kg * 128u + (j & 7u) * 16u) = pl[t];
  if (kg == 0u)
    reinterpret_cast<int *>(out + kDig * kBPlane)[j] = h;
}

template <bool SORT, bool ACCV>
__global__ void __launch_bounds__(kThreads, 1) sp_pair_kernel(const __grid_constant__ Params P)
{
  extern __shared__ __align__(1024) unsigned char sm[];
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const unsigned pair = blockIdx.x;
  const uint16_t *const blk = P.strat1 + ((size_t)P.step * P.pairs + pair) * 2u;
  const unsigned iBlk = blk[0], jBlk = blk[1];
  uint64_t *const bar = reinterpret_cast<uint64_t *>(sm + kOffBar); // [0..2] stage full, [3..4] planes free
  uint32_t *const tmem_holder = reinterpret_cast<uint32_t *>(sm + kOffTmem);
  int *const eG = reinterpret_cast<int *>(sm + kOffScale);
  int *const eV = eG + 64;
  unsigned *const red = reinterpret_cast<unsigned *>(sm + kOffRed);
  uint8_t *const s0 = sm + kOffS0;
  const unsigned ntiles = (P.nrow + 63u) / 64u;
  __shared__ int s_fail;

  if (tid == 0u) {
    s_fail = 0;
    for (unsigned i = 0u; i < 5u; ++i)
      mbar_init(&bar[i], 1u);
    mbar_fence_init();
  }
  // column scales and the inner table
  if (tid < 64u) {
    const unsigned gc = (tid < kBW) ? iBlk * kBW + tid : jBlk * kBW + tid - kBW;
    eG[tid] = col_exp(P.cmaxG[P.parity * P.ncol + gc]);
    eV[tid] = ACCV ? col_exp(P.cmaxV[P.parity * P.ncol + gc]) : 0;
  }
  for (unsigned i = tid; i < P.s0steps * 64u; i += kThreads)
    s0[i] = P.strat0[i];
  if (warp == 0u)
    tmem_alloc(tmem_holder);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  const uint32_t sbase = smem_u32(sm);

  // first copies: tiles 0 .. kGStages - 1
  if (tid == 0u) {
    for (unsigned i = 0u; i < kGStages && i < ntiles; ++i) {
      mbar_arrive_expect_tx(&bar[i], kGStageBytes);
      unsigned char *const dst = sm + kOffGStage + i * kGStageBytes;
      tma_load_3d(dst, &P.tmGram, 0, (int)i, (int)(iBlk * kBW), &bar[i]);
      tma_load_3d(dst + kGBox, &P.tmGram, 0, (int)i, (int)(iBlk * kBW + 16u), &bar[i]);
      tma_load_3d(dst + 2u * kGBox, &P.tmGram, 0, (int)i, (int)(jBlk * kBW), &bar[i]);
      tma_load_3d(dst + 3u * kGBox, &P.tmGram, 0, (int)i, (int)(jBlk * kBW + 16u), &bar[i]);
    }
  }
  // slicing task of this thread: column x, rows 16 rg .. 16 rg + 15 of the tile
  const unsigned x = tid & 63u, rg = tid >> 6;
  const int ex = eG[x];
  constexpr uint32_t kId = idesc_i8(128u, 64u);
  for (unsigned i = 0u; i < ntiles; ++i) {
    const unsigned s = i % kGStages, b = i & 1u;
    int bad = !mbar_wait_bounded(&bar[s], (i / kGStages) & 1u, kWait);
    if (i >= 2u && !mbar_wait_bounded(&bar[3u + b], ((i - 2u) >> 1) & 1u, kWait))
      bad = 1;
    if (__syncthreads_or(bad)) { // every thread leaves the loop together
      if (tid == 0u)
        s_fail = 1;
      break;
    }
    {
      const double *const col = reinterpret_cast<const double *>(sm + kOffGStage + s * kGStageBytes) + x * 66u;
      long long w[16];
#pragma unroll
      for (unsigned k = 0u; k < 8u; ++k) {
        const double2 v = *reinterpret_cast<const double2 *>(col + 16u * rg + 2u * k);
        w[2u * k] = biased_int(v.x, ex);
        w[2u * k + 1u] = biased_int(v.y, ex);
      }
      uint4 pl[kDig];
      digits16(w, pl);
      uint8_t *const dst = sm + kOffGPlanes + b * kGTilePlanes + (rg >> 1) * kGChunk + (x >> 3) * 256u +
                           (rg & 1u) * 128u + (x & 7u) * 16u;
#pragma unroll
      for (unsigned t = 0u; t < kDig; ++t) {
        const unsigned slot = (t < 4u) ? 2u * t : 2u * (t - 4u) + 1u;
        *reinterpret_cast<uint4 *>(dst + slot * kGPlane) = pl[t];
      }
    }
    fence_async_shared();
    __syncthreads();
    if (tid == 0u) {
      // the stage is read: refill it with tile i + kGStages
      if (i + kGStages < ntiles) {
        mbar_arrive_expect_tx(&bar[s], kGStageBytes);
        unsigned char *const dst = sm + kOffGStage + s * kGStageBytes;
        const int tile = (int)(i + kGStages);
        tma_load_3d(dst, &P.tmGram, 0, tile, (int)(iBlk * kBW), &bar[s]);
        tma_load_3d(dst + kGBox, &P.tmGram, 0, tile, (int)(iBlk * kBW + 16u), &bar[s]);
        tma_load_3d(dst + 2u * kGBox, &P.tmGram, 0, tile, (int)(jBlk * kBW), &bar[s]);
        tma_load_3d(dst + 3u * kGBox, &P.tmGram, 0, tile, (int)(jBlk * kBW + 16u), &bar[s]);
      }
      tc_fence_after();
#pragma unroll 1
      for (unsigned kc = 0u; kc < 2u; ++kc) {
        const uint32_t base = sbase + kOffGPlanes + b * kGTilePlanes + kc * kGChunk;
#pragma unroll 1
        for (unsigned t = 0u; t < 4u; ++t) {
          const uint64_t a = sdesc(base + 2u * t * kGPlane, 128u, 256u);
#pragma unroll 1
          for (unsigned u = 0u; u + t < kDig; ++u) {
            const unsigned slot = (u < 4u) ? 2u * u : 2u * (u - 4u) + 1u;
            const uint64_t bd = sdesc(base + slot * kGPlane, 128u, 256u);
            mma_i8(tmem + (t + u) * 64u, a, bd, kId, (i == 0u && kc == 0u && t == 0u) ? 0u : 1u);
          }
        }
      }
      mma_commit(&bar[3u + b]);
    }
  }
  // the last commit covers every MMA
  __syncthreads();
  int bad = s_fail;
  if (!bad && ntiles) {
    const unsigned last = ntiles - 1u;
    bad = !mbar_wait_bounded(&bar[3u + (last & 1u)], (last >> 1) & 1u, kWait);
  }
  const bool failed = __syncthreads_or(bad) != 0;
  tc_fence_after();

  // Gram epilogue: warps 2, 3, 6, 7 (TMEM lanes 64..127: the planes t + 4)
  // park their groups 4..7 in shared memory; warps 0, 1, 4, 5 add them to
  // their groups and form the FP64 Gram entries (x = row, y = column)
  double *const R = reinterpret_cast<double *>(sm + kOffR);
  double *const Vl = reinterpret_cast<double *>(sm + kOffVl);
  int *const bot = reinterpret_cast<int *>(sm + kOffBot);
  const unsigned q4 = warp & 3u, half = warp >> 2;
  if (!failed && q4 >= 2u) {
    const unsigned xr = (q4 - 2u) * 32u + lane;
#pragma unroll 1
    for (unsigned g = 0u; g < 4u; ++g)
#pragma unroll 1
      for (unsigned ch = 0u; ch < 2u; ++ch) {
        int v[16];
        tmem_ld16(tmem + ((q4 * 32u) << 16) + g * 64u + half * 32u + ch * 16u, v);
        tmem_wait_ld();
#pragma unroll
        for (unsigned k = 0u; k < 16u; ++k)
          bot[(g * 64u + half * 32u + ch * 16u + k) * 64u + xr] = v[k];
      }
  }
  tc_fence_before();
  __syncthreads();
  if (!failed && q4 < 2u) {
    const unsigned xr = q4 * 32u + lane;
#pragma unroll 1
    for (unsigned ch = 0u; ch < 2u; ++ch) {
      int acc[kDig][16];
#pragma unroll
      for (unsigned g = 0u; g < kDig; ++g)
        tmem_ld16(tmem + ((q4 * 32u) << 16) + g * 64u + half * 32u + ch * 16u, acc[g]);
      tmem_wait_ld();
#pragma unroll
      for (unsigned k = 0u; k < 16u; ++k) {
        const unsigned y = half * 32u + ch * 16u + k;
        int sg[kDig];
#pragma unroll
        for (unsigned g = 0u; g < kDig; ++g)
          sg[g] = acc[g][k] + ((g >= 4u) ? bot[((g - 4u) * 64u + y) * 64u + xr] : 0);
        R[y * kLd + xr] = scale2(recombine(sg), eG[xr] + eG[y] - 12);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0u)
    tmem_dealloc(tmem);
  if (failed) {
    if (tid == 0u)
      set_err(P);
    return;
  }

  // Cholesky of the Gram matrix (lower triangle, in place): column k of L,
  // then the trailing update, two barriers per column.  A pivot that is not
  // positive (a column dependent on the previous ones to working accuracy)
  // gives a zero column of L.
  __shared__ double s_inv;
  for (unsigned k = 0u; k < 64u; ++k) {
    if (tid == 0u) {
      const double d = R[k * kLd + k];
      const double piv = d > 0.0 ? __dsqrt_rn(d) : 0.0;
      R[k * kLd + k] = piv;
      s_inv = piv > 0.0 ? __drcp_rn(piv) : 0.0;
    }
    __syncthreads();
    const double inv = s_inv;
    if (tid > k && tid < 64u)
      R[k * kLd + tid] *= inv;
    __syncthreads();
    // A(i, j) -= L(i, k) L(j, k), k < j <= i
    for (unsigned e = tid; e < 64u * 64u; e += kThreads) {
      const unsigned i = e & 63u, j = e >> 6;
      if (j > k && i >= j)
        R[j * kLd + i] = __fma_rn(-R[k * kLd + i], R[k * kLd + j], R[j * kLd + i]);
    }
    __syncthreads();
  }
  // R = L^T (upper), V_loc = I
  for (unsigned e = tid; e < 64u * 64u; e += kThreads) {
    const unsigned i = e & 63u, j = e >> 6; // R(i, j) = L(j, i) for i <= j: both from the lower triangle
    Vl[j * kLd + i] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (unsigned e = tid; e < 64u * 64u; e += kThreads) {
    const unsigned i = e & 63u, j = e >> 6;
    if (i < j)
      R[j * kLd + i] = R[i * kLd + j]; // upper (i, j) <- lower (j, i)
  }
  __syncthreads();
  for (unsigned e = tid; e < 64u * 64u; e += kThreads) {
    const unsigned i = e & 63u, j = e >> 6;
    if (i > j)
      R[j * kLd + i] = 0.0;
  }
  __syncthreads();

  int definite;
  unsigned npos;
  pair_signature(P, iBlk, jBlk, definite, npos);
  unsigned blk_s = 0u, blk_b = 0u;
  inner64<SORT>(R, Vl, s0, P.s0steps, P.nswp0, definite, npos, red, blk_s, blk_b);

  // the update's B operands, the counters, and the next step's column maxima cleared
  uint8_t *const bop = P.bop + (size_t)pair * (ACCV ? 2u : 1u) * kBopBytes;
  bop_write(Vl, eG, bop);
  if (ACCV)
    bop_write(Vl, eV, bop + kBopBytes);
  if (tid < 64u) {
    const unsigned gc = (tid < kBW) ? iBlk * kBW + tid : jBlk * kBW + tid - kBW;
    P.cmaxG[(P.parity ^ 1u) * P.ncol + gc] = 0u;
    if (ACCV)
      P.cmaxV[(P.parity ^ 1u) * P.ncol + gc] = 0u;
  }
  if (tid == 0u && blk_s) {
    if (blk_b)
      atomicAdd(P.cvg, (((unsigned long long)blk_b) << 32) | blk_s);
    else
      atomicAdd(reinterpret_cast<unsigned *>(P.cvg), blk_s);
  }
}

// ---------------------------------------------------------------------------
// sp_update_kernel: C = A B for one 128-row tile of a pair's 64 columns of G
// (tiles 0 .. tilesG - 1) or of V (the rest), A the FP64 tile, B = V_loc
// (its digit planes diag(2^e) V_loc from sp_pair_kernel).  C replaces A.
// ---------------------------------------------------------------------------
constexpr uint32_t kUStage = 128u * 64u * 8u;     // FP64 tile, column c at c * 128 doubles
constexpr uint32_t kUAPlane = 8192u;               // 128 x 64 bytes, K-major, LBO 128, SBO 512
constexpr uint32_t kOffUStage = 0u;
constexpr uint32_t kOffUA = kUStage;                            // 65536
constexpr uint32_t kOffUB = kOffUA + kDig * kUAPlane;           // 131072
constexpr uint32_t kOffUScale = kOffUB + kBopBytes;             // 163840 + 256: 64 int e_k, then 64 uint col max
constexpr uint32_t kOffUBar = kOffUScale + 512u;
constexpr uint32_t kOffUTmem = kOffUBar + 32u;
constexpr uint32_t kUpdSmem = kOffUTmem + 16u;
static_assert(kUpdSmem <= 227u * 1024u, "shared memory of sp_update_kernel");

template <bool ACCV>
__global__ void __launch_bounds__(kThreads, 1) sp_update_kernel(const __grid_constant__ Params P)
{
  extern __shared__ __align__(1024) unsigned char sm[];
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const unsigned pair = blockIdx.y, tile = blockIdx.x;
  const bool isV = tile >= P.tilesG;
  const unsigned row0 = (isV ? tile - P.tilesG : tile) * 128u;
  const uint16_t *const blk = P.strat1 + ((size_t)P.step * P.pairs + pair) * 2u;
  const unsigned iBlk = blk[0], jBlk = blk[1];
  const CUtensorMap *const tm = isV ? &P.tmV : &P.tmG;
  uint32_t *const cmax = isV ? P.cmaxV : P.cmaxG;
  uint64_t *const bar = reinterpret_cast<uint64_t *>(sm + kOffUBar); // [0] loads, [1] MMAs
  uint32_t *const tmem_holder = reinterpret_cast<uint32_t *>(sm + kOffUTmem);
  int *const ek = reinterpret_cast<int *>(sm + kOffUScale);
  uint32_t *const cm = reinterpret_cast<uint32_t *>(sm + kOffUScale + 256u);
  const uint8_t *const bsrc = P.bop + ((size_t)pair * (ACCV ? 2u : 1u) + (isV ? 1u : 0u)) * kBopBytes;

  if (tid == 0u) {
    mbar_init(&bar[0], 1u);
    mbar_init(&bar[1], 1u);
    mbar_fence_init();
  }
  if (tid < 64u) {
    const unsigned gc = (tid < kBW) ? iBlk * kBW + tid : jBlk * kBW + tid - kBW;
    ek[tid] = col_exp(cmax[P.parity * P.ncol + gc]);
    cm[tid] = 0u;
  }
  if (warp == 0u)
    tmem_alloc(tmem_holder);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  const uint32_t sbase = smem_u32(sm);
  if (tid == 0u) {
    mbar_arrive_expect_tx(&bar[0], kUStage + kBopBytes);
    tma_load_2d(sm + kOffUStage, tm, (int)row0, (int)(iBlk * kBW), &bar[0]);
    tma_load_2d(sm + kOffUStage + kUStage / 2u, tm, (int)row0, (int)(jBlk * kBW), &bar[0]);
    bulk_g2s(sm + kOffUB, bsrc, kBopBytes, &bar[0]);
  }
  const bool ok_load = mbar_wait_bounded(&bar[0], 0u, kWait);
  if (__syncthreads_or(!ok_load)) {
    if (tid == 0u)
      set_err(P);
    tc_fence_before();
    __syncthreads();
    if (warp == 0u)
      tmem_dealloc(tmem);
    return;
  }
  // slicing: thread takes rows r = tid % 128 of pair columns 16 kg .. 16 kg + 15, kg = tid / 128 and + 2
  {
    const double *const st = reinterpret_cast<const double *>(sm + kOffUStage);
    const unsigned r = tid & 127u;
#pragma unroll 1
    for (unsigned kg = tid >> 7; kg < 4u; kg += 2u) {
      long long w[16];
#pragma unroll
      for (unsigned i = 0u; i < 16u; ++i) {
        const unsigned k = 16u * kg + i;
        w[i] = biased_int(st[k * 128u + r], ek[k]);
      }
      uint4 pl[kDig];
      digits16(w, pl);
      uint8_t *const dst = sm + kOffUA + (r >> 3) * 512u + kg * 128u + (r & 7u) * 16u;
#pragma unroll
      for (unsigned t = 0u; t < kDig; ++t)
        *reinterpret_cast<uint4 *>(dst + t * kUAPlane) = pl[t];
    }
  }
  fence_async_shared();
  __syncthreads();
  if (tid == 0u) {
    tc_fence_after();
    constexpr uint32_t kId = idesc_i8(128u, 64u);
#pragma unroll 1
    for (unsigned t = 0u; t < kDig; ++t)
#pragma unroll 1
      for (unsigned u = 0u; u + t < kDig; ++u)
#pragma unroll 1
        for (unsigned kh = 0u; kh < 2u; ++kh) {
          const uint64_t a = sdesc(sbase + kOffUA + t * kUAPlane + kh * 256u, 128u, 512u);
          const uint64_t b = sdesc(sbase + kOffUB + u * kBPlane + kh * 256u, 128u, 512u);
          mma_i8(tmem + (t + u) * 64u, a, b, kId, (t == 0u && kh == 0u) ? 0u : 1u);
        }
    mma_commit(&bar[1]);
  }
  const bool ok_mma = mbar_wait_bounded(&bar[1], 0u, kWait);
  const bool failed = __syncthreads_or(!ok_mma) != 0;
  tc_fence_after();
  if (!failed) {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. (rows of the tile), columns 32 (w / 4) ..
    const unsigned q4 = warp & 3u, half = warp >> 2, r = q4 * 32u + lane;
    const int *const h = reinterpret_cast<const int *>(sm + kOffUB + kDig * kBPlane);
    double *const st = reinterpret_cast<double *>(sm + kOffUStage);
#pragma unroll 1
    for (unsigned ch = 0u; ch < 2u; ++ch) {
      int acc[kDig][16];
#pragma unroll
      for (unsigned g = 0u; g < kDig; ++g)
        tmem_ld16(tmem + ((q4 * 32u) << 16) + g * 64u + half * 32u + ch * 16u, acc[g]);
      tmem_wait_ld();
#pragma unroll
      for (unsigned k = 0u; k < 16u; ++k) {
        const unsigned j = half * 32u + ch * 16u + k;
        int sg[kDig];
#pragma unroll
        for (unsigned g = 0u; g < kDig; ++g)
          sg[g] = acc[g][k];
        const double c = scale2(recombine(sg), h[j] - 12);
        st[j * 128u + r] = c;
        // rows beyond the matrix (zero-filled input) give 0 and change no maximum
        const uint32_t m = __reduce_max_sync(0xffffffffu, abs_hi(c));
        if (lane == 0u)
          atomicMax(&cm[j], m);
      }
    }
  }
  tc_fence_before();
  fence_async_shared();
  __syncthreads();
  if (warp == 0u)
    tmem_dealloc(tmem);
  if (failed) {
    if (tid == 0u)
      set_err(P);
    return;
  }
  if (tid == 0u) {
    tma_store_2d(tm, sm + kOffUStage, (int)row0, (int)(iBlk * kBW));
    tma_store_2d(tm, sm + kOffUStage + kUStage / 2u, (int)row0, (int)(jBlk * kBW));
    bulk_commit();
  }
  if (tid < 64u) {
    const unsigned gc = (tid < kBW) ? iBlk * kBW + tid : jBlk * kBW + tid - kBW;
    if (cm[tid])
      atomicMax(&cmax[(P.parity ^ 1u) * P.ncol + gc], cm[tid]);
  }
  if (tid == 0u)
    bulk_wait_all();
}

// the largest |entry| of every column (high words), one warp per column
__global__ void sp_colmax_kernel(const double *const A, const unsigned nrow, const unsigned ncol, const unsigned ld,
                                 uint32_t *const out)
{
  const unsigned c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31u;
  if (c >= ncol)
    return;
  uint32_t m = 0u;
  for (unsigned r = lane; r < nrow; r += 32u)
    m = max(m, abs_hi(A[(size_t)c * ld + r]));
  m = __reduce_max_sync(0xffffffffu, m);
  if (lane == 0u)
    out[c] = m;
}

__global__ void sp_fill_kernel(uint32_t *const a, const unsigned n, const uint32_t v)
{
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    a[i] = v;
}

} // namespace split

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

using namespace split;

struct SplitCtx {
  bool configured = false;
  unsigned long long version = ~0ull; // strategy version of the tables below
  unsigned n1 = 0u, steps0 = 0u, steps1 = 0u;
  uint8_t *d_s0 = nullptr;
  uint16_t *d_s1 = nullptr;
  size_t s1_cap = 0u;
  uint32_t *d_cmax = nullptr; // [G: 2 ncol][V: 2 ncol]
  size_t cmax_cap = 0u;
  uint8_t *d_bop = nullptr;
  size_t bop_cap = 0u;
  unsigned long long *d_cnt = nullptr, *h_cnt = nullptr;
};
std::mutex g_split_mtx;
std::vector<SplitCtx> g_split_dev;
thread_local std::string g_split_err;

int cuda_fail(const cudaError_t e, const char *what)
{
  g_split_err = std::string(what) + ": " + cudaGetErrorString(e);
  set_error(g_split_err.c_str());
  return GJX_ERR_CUDA;
}

#define SP_CUDA(call, what)                                                                                          \
  do {                                                                                                               \
    const cudaError_t e_ = (call);                                                                                   \
    if (e_ != cudaSuccess)                                                                                           \
      return cuda_fail(e_, what);                                                                                    \
  } while (0)

template <typename T> int grow(T *&p, size_t &cap, const size_t n, const char *what)
{
  if (n <= cap)
    return 0;
  if (p)
    SP_CUDA(cudaFree(p), what);
  p = nullptr;
  cap = 0u;
  SP_CUDA(cudaMalloc(&p, n * sizeof(T)), what);
  cap = n;
  return 0;
}

// 2-D view (rows, columns) of a column-major matrix, box {128 rows, 32 columns}
cudaError_t make_tile_map(CUtensorMap *tm, const double *base, const unsigned nrow, const unsigned ncol,
                          const unsigned ld)
{
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    const cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess)
      return e;
    if (q != cudaDriverEntryPointSuccess || !fn)
      return cudaErrorNotSupported;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[2] = {nrow, ncol};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(double)};
  const cuuint32_t box[2] = {128u, 32u};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <bool S, bool A> cudaError_t set_attrs()
{
  cudaError_t e = cudaFuncSetAttribute(sp_pair_kernel<S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kPairSmem);
  if (e != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(sp_update_kernel<A>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUpdSmem);
}

template <bool S, bool A> cudaError_t launch_step(const Params &p, const cudaStream_t st)
{
  sp_pair_kernel<S, A><<<p.pairs, kThreads, kPairSmem, st>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return e;
  sp_update_kernel<A><<<dim3(p.tilesG + p.tilesV, p.pairs), kThreads, kUpdSmem, st>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_split_step(const bool sort, const bool accv, const Params &p, const cudaStream_t st)
{
  if (sort)
    return accv ? launch_step<true, true>(p, st) : launch_step<true, false>(p, st);
  return accv ? launch_step<false, true>(p, st) : launch_step<false, false>(p, st);
}

int split_sweeps(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                 double *const dG, const unsigned lddG, double *const dV, const unsigned lddV, double *const dD,
                 const cudaStream_t st, unsigned *const glbSwp, unsigned long long *const glb_s,
                 unsigned long long *const glb_b)
{
  const bool cdsort = (routine & GJX_CDSORT_1) != 0u, full = (routine & GJX_FULL_SVD) != 0u,
             blk_ori = (routine & GJX_BLK_ORI) != 0u;
  int dev = 0;
  SP_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if ((size_t)dev >= g_split_dev.size())
    g_split_dev.resize((size_t)dev + 1u);
  SplitCtx &c = g_split_dev[(size_t)dev];
  if (!c.configured) {
    SP_CUDA((set_attrs<true, true>()), "split kernel attributes");
    SP_CUDA((set_attrs<true, false>()), "split kernel attributes");
    SP_CUDA((set_attrs<false, true>()), "split kernel attributes");
    SP_CUDA((set_attrs<false, false>()), "split kernel attributes");
    SP_CUDA(cudaMalloc(&c.d_s0, 64u * 64u), "cudaMalloc(split inner table)");
    SP_CUDA(cudaMalloc(&c.d_cnt, 2u * sizeof(unsigned long long)), "cudaMalloc(split counters)");
    SP_CUDA(cudaHostAlloc(&c.h_cnt, 2u * sizeof(unsigned long long), cudaHostAllocPortable), "cudaHostAlloc");
    c.configured = true;
  }
  const unsigned n1 = ncol / kBW;
  {
    std::vector<uint8_t> s0;
    std::vector<uint16_t> s1;
    unsigned steps0 = 0u, steps1 = 0u;
    unsigned long long ver = 0ull;
    // the tables are read again when the loaded families or n1 change
    {
      if (const int r = family_tables(kW, n1, s0, steps0, s1, steps1, ver))
        return r;
      if (steps0 > 64u) {
        set_error("inner table of more than 64 steps");
        return GJX_ERR_NO_STRAT;
      }
      if (c.version != ver || c.n1 != n1) {
        if (const int r = grow(c.d_s1, c.s1_cap, s1.size(), "cudaMalloc(split outer table)"))
          return r;
        SP_CUDA(cudaMemcpyAsync(c.d_s0, s0.data(), s0.size(), cudaMemcpyHostToDevice, st), "upload inner table");
        SP_CUDA(cudaMemcpyAsync(c.d_s1, s1.data(), s1.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, st),
                "upload outer table");
        SP_CUDA(cudaStreamSynchronize(st), "upload tables");
        c.version = ver;
        c.n1 = n1;
        c.steps0 = steps0;
        c.steps1 = steps1;
      }
    }
  }
  const unsigned pairs = n1 / 2u;
  if (const int r = grow(c.d_cmax, c.cmax_cap, 4u * (size_t)ncol, "cudaMalloc(column maxima)"))
    return r;
  if (const int r = grow(c.d_bop, c.bop_cap, (size_t)pairs * (full ? 2u : 1u) * kBopBytes, "cudaMalloc(B operands)"))
    return r;

  Params p{};
  SP_CUDA(make_gram_map(&p.tmGram, dG, nrow, ncol, lddG), "Gram tensor map of G");
  SP_CUDA(make_tile_map(&p.tmG, dG, nrow, ncol, lddG), "tile tensor map of G");
  if (full)
    SP_CUDA(make_tile_map(&p.tmV, dV, ncol, ncol, lddV), "tile tensor map of V");
  p.strat1 = c.d_s1;
  p.strat0 = c.d_s0;
  p.cvg = c.d_cnt;
  p.err = reinterpret_cast<int *>(c.d_cnt + 1);
  p.cmaxG = c.d_cmax;
  p.cmaxV = c.d_cmax + 2u * (size_t)ncol;
  p.bop = c.d_bop;
  p.nrow = nrow;
  p.ncol = ncol;
  p.nplus = nplus;
  p.pairs = pairs;
  p.s0steps = c.steps0;
  p.nswp0 = blk_ori ? 1u : kNSweep;
  p.tilesG = (nrow + 127u) / 128u;
  p.tilesV = full ? (ncol + 127u) / 128u : 0u;
  p.gdefinite = (nplus ? ((nplus < ncol) ? 0 : +1) : -1);
  p.accv = full ? 1 : 0;

  if (full) {
    SP_CUDA(launch_initV(dV, ncol, lddV, st), "initV");
    sp_fill_kernel<<<(ncol + 255u) / 256u, 256u, 0u, st>>>(p.cmaxV, ncol, 0x3FF00000u); // |V| <= 1 = max
    SP_CUDA(cudaGetLastError(), "column maxima of V");
  }
  sp_colmax_kernel<<<(ncol + 7u) / 8u, 256u, 0u, st>>>(dG, nrow, ncol, lddG, p.cmaxG);
  SP_CUDA(cudaGetLastError(), "column maxima of G");
  SP_CUDA(cudaMemsetAsync(c.d_cnt + 1, 0, sizeof(unsigned long long), st), "clear error word");
  *glb_s = 0ull;
  *glb_b = 0ull;
  unsigned swp = 0u, gstep = 0u;
  while (swp < kNSweep) {
    SP_CUDA(cudaMemsetAsync(c.d_cnt, 0, sizeof(unsigned long long), st), "clear counter");
    for (unsigned s = 0u; s < c.steps1; ++s, ++gstep) {
      p.step = s;
      p.parity = gstep & 1u;
      SP_CUDA(launch_split_step(cdsort, full, p, st), "split step");
    }
    ++swp;
    SP_CUDA(cudaMemcpyAsync(c.h_cnt, c.d_cnt, 2u * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
            "read counters");
    SP_CUDA(cudaStreamSynchronize(st), "split sweep");
    if ((int)c.h_cnt[1]) {
      set_error("a split-form kernel timed out waiting for its copies or products");
      return GJX_ERR_DEVICE;
    }
    const unsigned long long cvg = c.h_cnt[0];
    *glb_s += (unsigned)cvg;
    *glb_b += (unsigned)(cvg >> 32u);
    if (!(unsigned)(cvg >> 32u))
      break;
  }
  *glbSwp = swp;
  SP_CUDA(launch_initD(dG, dD, nrow, ncol, nplus, lddG, st), "initD");
  SP_CUDA(cudaStreamSynchronize(st), "initD");
  return 0;
}

} // namespace
} // namespace gjx

extern "C" int gjx_hypJacL2_split(const unsigned routine, const unsigned nrow, const unsigned ncol,
                                  const unsigned nplus, double *const dG, const unsigned lddG, double *const dV,
                                  const unsigned lddV, double *const dD, void *const stream, unsigned *const glbSwp,
                                  unsigned long long *const glb_s, unsigned long long *const glb_b)
{
  if (const int r = gjx::check_dev_args(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, glbSwp, glb_s, glb_b))
    return r;
  if (ncol % 64u) {
    gjx::set_error("the split form takes ncol a multiple of 64 (blocks of 32 columns, an even number of them)");
    return -3;
  }
  if (nrow > 61440u) {
    gjx::set_error("the split form takes nrow <= 61440 (its int32 accumulators hold 8 x 4225 x nrow)");
    return -2;
  }
  std::lock_guard<std::mutex> lk(gjx::g_split_mtx);
  return gjx::split_sweeps(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, static_cast<cudaStream_t>(stream),
                           glbSwp, glb_s, glb_b);
}
