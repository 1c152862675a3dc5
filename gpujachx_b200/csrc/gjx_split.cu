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
// 2^e_c), so each entry becomes x = a 2^-e_c in (-1, 1); v = rint(x 2^54) is a
// 55-bit integer, written as v = sum_t d_t 2^(8 (6 - t)), t = 0..6: d_0 in
// [-64, 65], d_1..d_6 in [-128, 127] (balanced base-256 digits: with 128
// added to each of the six low bytes of v, digit t is byte 6 - t of the sum
// with its top bit flipped, so cutting a value is a handful of byte
// permutes).  Each digit plane is an int8 matrix.  A product of two such
// operands is
//   sum_k v_ik w_kj = sum_(t,u) 2^(96 - 8(t+u)) sum_k d_t,ik d_u,kj,
// and the slice products with t + u <= 6 are kept: 28 int8 x int8 -> int32
// products, summed exactly per group g = t + u in 7 int32 accumulators, then
// combined in int64 (groups 0-3 and 4-6), two conversions, one FMA and a
// power-of-two scale.  The slicing error is 2^-55 of the column's scale per
// entry, the dropped groups g >= 7 weigh about 2^-56 of the product's scale:
// the order of FP64 rounding.  The scales are tracked exactly: the update
// kernel folds the largest |entry| of every column it writes into a
// per-column word (atomic max of the high words), read by the next step (by
// step parity).  The int32 group sums bound the Gram's rows: 7 x 2^14 x nrow
// < 2^31, nrow <= 16384.
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
//   sp_update_kernel  a persistent grid over the 128-row tiles of every pair's
//                     columns of G and V: the FP64 tile by TMA (two ahead),
//                     sliced, 72 MMAs of 128 x 64 x 32, the epilogue back to
//                     FP64 in place, and the columns' maxima.
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
constexpr unsigned kDig = 7u;    // digits per value
constexpr long long kWait = 2000000000ll;
constexpr unsigned kTmemCols = 512u; // 8 accumulators x 64 columns
// 128 in each of the six low bytes: added to v so that each low byte holds
// its digit + 128
constexpr long long kDigitBias = 128ll * 0x010101010101ll;
constexpr unsigned kMaxRows = 16384u; // int32 group sums of the Gram matrix: 7 x 2^14 x nrow < 2^31

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
  double *G, *V;
  unsigned ldG, ldV;
  unsigned nrow, ncol, nplus, pairs, step, parity, s0steps, nswp0;
  unsigned tilesG, tilesV; // 128-row tiles of G and of V
  int gdefinite;
  int accv;
  unsigned sms; // CTAs of the persistent update grid
  long long *clk; // [0..4] block 0 of sp_pair_kernel: clock64 at the phase ends; [5..9] CTA 0 of
                  // sp_update_kernel, sums over the call (gjx_split_phase_cycles)
};

// ---- the update's B operand in global memory: for each half of the output
// columns (32 each) the 7 digit planes side by side (K-major, 32 x 64 bytes
// each, core matrices of 8 rows x 16 bytes, LBO 128, SBO 512), then the 64
// column exponents h_j
constexpr uint32_t kBHalfPlane = 2048u;
constexpr uint32_t kBHalf = kDig * kBHalfPlane; // 14336
constexpr uint32_t kBPlane = 4096u;              // both halves of a digit
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
// every entry is below 2^e; columns below 2^-969 (zero ones among them) are
// given e = -969, so that 2^(54 - e) and its inverse stay normal
__device__ __forceinline__ int col_exp(const uint32_t hw) { return max((int)((hw >> 20) & 0x7FFu) - 1022, -969); }

// 2^k for k in [-1022, 1023]
__device__ __forceinline__ double p2(const int k) { return __longlong_as_double((long long)(k + 1023) << 52); }

// x * 2^k exactly (no intermediate over- or underflow for the k used here:
// |k| <= 2100, two factors of at most 2^1050 each side)
__device__ __forceinline__ double scale2(const double x, const int k)
{
  const int k1 = k / 2;
  return (x * p2(k1)) * p2(k - k1);
}

// 2^(54 - e) for a column with exponent bound e
__device__ __forceinline__ double cut_factor(const int e) { return p2(54 - e); }

// the 55-bit integer of a * f (f = cut_factor(e), |a| < 2^e: |a f| < 2^54),
// biased for digit cutting
__device__ __forceinline__ long long biased_int(const double a, const double f)
{
  return __double2ll_rn(a * f) + kDigitBias;
}

// plane T's bytes of four biased values: byte j of the result is digit T of
// value j as an int8 (byte 6 - T of the value; the low digits' top bits flipped)
template <unsigned T> __device__ __forceinline__ uint32_t plane_word(const long long w0, const long long w1,
                                                                     const long long w2, const long long w3)
{
  constexpr unsigned B = 6u - T;             // byte of the value
  constexpr unsigned sel = (B & 3u) | ((4u + (B & 3u)) << 4); // bytes B of x and of y, to bytes 0 and 1
  const uint32_t x0 = (B >= 4u) ? (uint32_t)((unsigned long long)w0 >> 32) : (uint32_t)w0;
  const uint32_t x1 = (B >= 4u) ? (uint32_t)((unsigned long long)w1 >> 32) : (uint32_t)w1;
  const uint32_t x2 = (B >= 4u) ? (uint32_t)((unsigned long long)w2 >> 32) : (uint32_t)w2;
  const uint32_t x3 = (B >= 4u) ? (uint32_t)((unsigned long long)w3 >> 32) : (uint32_t)w3;
  const uint32_t lo = __byte_perm(x0, x1, sel), hi = __byte_perm(x2, x3, sel);
  const uint32_t r = __byte_perm(lo, hi, 0x5410u);
  return (T == 0u) ? r : (r ^ 0x80808080u);
}

// 16 biased values -> 16 bytes of each of the 7 planes
__device__ __forceinline__ void digits16(const long long (&w)[16], uint4 (&out)[kDig])
{
#define GJX_PLANE(T)                                                                                                 \
  out[T] = make_uint4(plane_word<T>(w[0], w[1], w[2], w[3]), plane_word<T>(w[4], w[5], w[6], w[7]),                \
                      plane_word<T>(w[8], w[9], w[10], w[11]), plane_word<T>(w[12], w[13], w[14], w[15]));
  GJX_PLANE(0u) GJX_PLANE(1u) GJX_PLANE(2u) GJX_PLANE(3u) GJX_PLANE(4u) GJX_PLANE(5u) GJX_PLANE(6u)
#undef GJX_PLANE
}

// sum_g 2^-8g S_g, times 2^24: groups 0-3 and 4-6 each summed exactly in
// int64, then two conversions and one FMA
__device__ __forceinline__ double recombine(const int s0, const int s1, const int s2, const int s3, const int s4,
                                           const int s5, const int s6)
{
  const long long H = ((long long)s0 << 24) + ((long long)s1 << 16) + ((long long)s2 << 8) + (long long)s3;
  const long long L = ((long long)s4 << 16) + ((long long)s5 << 8) + (long long)s6;
  return __fma_rn(__ll2double_rn(L), 0x1.0p-24, __ll2double_rn(H));
}

__device__ __forceinline__ uint32_t abs_hi(const double x)
{
  return (uint32_t)(__double_as_longlong(x) >> 32) & 0x7FFFFFFFu;
}

// ---------------------------------------------------------------------------
// sp_pair_kernel
// ---------------------------------------------------------------------------
// Gram staging: kGStages stages of one 64-row tile of the pair's 64 columns, four
// boxes {66 rows, 1 tile, 16 columns}: column c at c * 66 doubles (528 bytes,
// an odd number of 16-byte granules: 8 consecutive columns in 8 bank groups)
constexpr unsigned kGStages = 3u;
constexpr unsigned kBarPlanes = kGStages; // [2] mbarriers after the stages': a plane buffer's MMAs done
constexpr uint32_t kGBox = 66u * 16u * 8u;         // 8448 bytes
constexpr uint32_t kGStageBytes = 4u * kGBox;       // 33792
// digit planes of a 64-row tile: 2 chunks of 32 rows x 8 plane slots x 2 KB
// (K-major: 64 columns x 32 rows; slot 7 is never written).  The planes of a
// chunk lie in digit order, so planes t, t + 1 form one 128-row A operand and
// planes u .. u + 3 one 256-column B operand.
constexpr uint32_t kGPlane = 2048u;
constexpr uint32_t kGChunk = 8u * kGPlane;          // 16384
constexpr uint32_t kGTilePlanes = 2u * kGChunk;     // 32768
constexpr unsigned kGPlaneBufs = 2u;
constexpr uint32_t kOffGStage = 0u;
constexpr uint32_t kOffGPlanes = kGStages * kGStageBytes;                     // 101376
constexpr uint32_t kOffGEnd = kOffGPlanes + kGPlaneBufs * kGTilePlanes;       // 166912
// after the Gram (reusing the staging): R and V_loc (64 x 64, ld 65), the
// bottom halves of accumulator blocks 0..5 (int32 [6][64][64]: groups 1..6)
constexpr unsigned kLd = 65u;
constexpr uint32_t kOffR = 0u;
constexpr uint32_t kOffVl = kOffR + 64u * kLd * 8u;                          // 33280
constexpr uint32_t kOffBot = kOffVl + 64u * kLd * 8u;                        // 66560, 98304 bytes
static_assert(kOffBot + 6u * 64u * 64u * 4u <= kOffGEnd, "Gram epilogue scratch must fit");
// fixed region after it
constexpr uint32_t kOffS0 = kOffGEnd;                                        // inner table, 64 steps x 64 bytes
constexpr uint32_t kOffScale = kOffS0 + 4096u;                               // 64 int: e_c of G; 64 int: of V
constexpr uint32_t kOffRed = kOffScale + 512u;                               // 64 unsigned
constexpr uint32_t kOffBar = kOffRed + 256u;                                 // 8 mbarriers
constexpr uint32_t kOffTmem = kOffBar + 64u;
static_assert(kGStages + 2u <= 8u, "stage and plane-buffer mbarriers must fit their region");
constexpr uint32_t kOffRot = kOffTmem + 16u;                                 // 8 warps x 16 doubles: rotations
constexpr uint32_t kPairSmem = kOffRot + 1024u;
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
// applies all four.  The twelve sums go through a reduce-scatter (at level 16
// each half keeps its two pairs' products, at level 8 each quarter its own,
// levels 4, 2, 1 within the quarter: the same operands in the same order as
// the full butterfly, with 18 shuffles instead of 60), and the four rotations
// reach every lane through rs (16 doubles of this warp's own shared memory;
// lane 8c writes pair c's), not through shuffles.  One barrier per step.
template <bool SORT>
__device__ void inner64(double *const R, double *const Vl, const uint8_t *const s0, const unsigned s0steps,
                        const unsigned nswp, const int definite, const unsigned npos, unsigned *const red,
                        unsigned &blk_s, unsigned &blk_b, double *const rs)
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
      const bool up = x >= 16u, odd = ((x >> 3) & 1u) != 0u;
      double h[2][3], sm3[3];
#pragma unroll
      for (unsigned j = 0u; j < 2u; ++j)
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i) {
          const double other = __shfl_xor_sync(0xffffffffu, up ? d[j][i] : d[2u + j][i], 16);
          h[j][i] = (up ? d[2u + j][i] : d[j][i]) + other;
        }
#pragma unroll
      for (unsigned i = 0u; i < 3u; ++i) {
        const double other = __shfl_xor_sync(0xffffffffu, odd ? h[0][i] : h[1][i], 8);
        sm3[i] = (odd ? h[1][i] : h[0][i]) + other;
      }
#pragma unroll
      for (unsigned o = 4u; o; o >>= 1u)
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i)
          sm3[i] += __shfl_xor_sync(0xffffffffu, sm3[i], o);
      const unsigned mc = x >> 3; // this lane's pair among the warp's four
      unsigned pm = p[0], qm = q[0];
#pragma unroll
      for (unsigned c = 1u; c < 4u; ++c)
        if (mc == c) {
          pm = p[c];
          qm = q[c];
        }
      unsigned a_s = 0u, a_b = 0u;
      const Rot mine = inner_rot<SORT>(sm3[0], sm3[1], sm3[2], pm, qm, definite, npos, a_s, a_b);
      if ((x & 7u) == 0u) {
        ws += a_s;
        wb += a_b;
        double *const e = rs + 4u * mc;
        e[0] = mine.c;
        e[1] = mine.t;
        e[2] = mine.t_;
        e[3] = __longlong_as_double((long long)(mine.mode | (mine.scale << 2) | (mine.swap << 3)));
      }
      __syncwarp();
#pragma unroll
      for (unsigned c = 0u; c < 4u; ++c) {
        const double2 ct = *reinterpret_cast<const double2 *>(rs + 4u * c);
        const double2 tf = *reinterpret_cast<const double2 *>(rs + 4u * c + 2u);
        Rot r;
        r.c = ct.x;
        r.t = ct.y;
        r.t_ = tf.x;
        const int fl = (int)__double_as_longlong(tf.y);
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

// the update's B operand diag(2^e_k) V_loc of one matrix: its digit planes
// (K-major, n = output column j, k = pair column; the columns of each half
// apart) and the exponents h_j, written to global memory.  Thread
// (j = tid / 4, kg = tid % 4) takes k = 16 kg .. 16 kg + 15 of column j.
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
  const double f = cut_factor(h);
  long long w[16];
#pragma unroll
  for (unsigned i = 0u; i < 16u; ++i)
    w[i] = biased_int(b[i], f);
  uint4 pl[kDig];
  digits16(w, pl);
#pragma unroll
  for (unsigned t = 0u; t < kDig; ++t)
    *reinterpret_cast<uint4 *>(out + (j >> 5) * kBHalf + t * kBHalfPlane + ((j & 31u) >> 3) * 512u + kg * 128u +
                               (j & 7u) * 16u) = pl[t];
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
  uint64_t *const bar = reinterpret_cast<uint64_t *>(sm + kOffBar); // stages full, then planes free
  uint32_t *const tmem_holder = reinterpret_cast<uint32_t *>(sm + kOffTmem);
  int *const eG = reinterpret_cast<int *>(sm + kOffScale);
  int *const eV = eG + 64;
  unsigned *const red = reinterpret_cast<unsigned *>(sm + kOffRed);
  uint8_t *const s0 = sm + kOffS0;
  const unsigned ntiles = (P.nrow + 63u) / 64u;
  __shared__ int s_fail;

  const bool rec = pair == 0u && tid == 0u;
  long long t_start = 0;
  if (rec)
    t_start = clock64();
  if (tid == 0u) {
    s_fail = 0;
    for (unsigned i = 0u; i < kGStages + 2u; ++i)
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
  const double fx = cut_factor(eG[x]);
  unsigned i_stop = ntiles; // the tiles taken in (all, unless a wait gave up)
  for (unsigned i = 0u; i < ntiles; ++i) {
    const unsigned s = i % kGStages, b = i & 1u;
    int bad = !mbar_wait_bounded(&bar[s], (i / kGStages) & 1u, kWait);
    if (i >= 2u && !mbar_wait_bounded(&bar[kBarPlanes + b], ((i - 2u) >> 1) & 1u, kWait))
      bad = 1;
    if (__syncthreads_or(bad)) { // every thread leaves the loop together
      if (tid == 0u)
        s_fail = 1;
      i_stop = i;
      break;
    }
    {
      const double *const col = reinterpret_cast<const double *>(sm + kOffGStage + s * kGStageBytes) + x * 66u;
      long long w[16];
#pragma unroll
      for (unsigned k = 0u; k < 8u; ++k) {
        const double2 v = *reinterpret_cast<const double2 *>(col + 16u * rg + 2u * k);
        w[2u * k] = biased_int(v.x, fx);
        w[2u * k + 1u] = biased_int(v.y, fx);
      }
      uint4 pl[kDig];
      digits16(w, pl);
      uint8_t *const dst = sm + kOffGPlanes + b * kGTilePlanes + (rg >> 1) * kGChunk + (x >> 3) * 256u +
                           (rg & 1u) * 128u + (x & 7u) * 16u;
#pragma unroll
      for (unsigned t = 0u; t < kDig; ++t)
        *reinterpret_cast<uint4 *>(dst + t * kGPlane) = pl[t];
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
      // A = planes 2p (rows 0-63) and 2p + 1 (rows 64-127; for p = 3 the
      // unused slot 7), B = planes u0 .. u0 + n - 1 side by side: D block
      // 2p + u0 + i gets group 2p + u0 + i in its top rows and group
      // 2p + u0 + i + 1 in its bottom rows.  Every (t, u) with t + u <= 6 is
      // covered; what lands in groups >= 7 is never read.
      const uint64_t d0 = sdesc(sbase + kOffGPlanes + b * kGTilePlanes, 128u, 256u);
      const uint32_t first = (i == 0u) ? 0u : 1u;
#pragma unroll
      for (unsigned kc = 0u; kc < 2u; ++kc) {
        const uint64_t dc = d0 + ((kc * kGChunk) >> 4);
        const uint32_t acc0 = (kc == 0u) ? first : 1u;
#define GJX_GMMA(P, U0, NN, ACC)                                                                                     \
  mma_i8(tmem + (2u * (P) + (U0)) * 64u, dc + ((2u * (P) * kGPlane) >> 4), dc + (((U0) * kGPlane) >> 4),             \
         idesc_i8(128u, (NN) * 64u), (ACC))
        GJX_GMMA(0u, 0u, 4u, acc0);
        GJX_GMMA(0u, 4u, 3u, acc0);
        GJX_GMMA(1u, 0u, 4u, 1u);
        GJX_GMMA(1u, 4u, 1u, 1u);
        GJX_GMMA(2u, 0u, 3u, 1u);
        GJX_GMMA(3u, 0u, 1u, 1u);
#undef GJX_GMMA
      }
      mma_commit(&bar[kBarPlanes + b]);
    }
  }
  // the last commit covers every MMA
  __syncthreads();
  int bad = s_fail;
  if (!bad && ntiles) {
    const unsigned last = ntiles - 1u;
    bad = !mbar_wait_bounded(&bar[kBarPlanes + (last & 1u)], (last >> 1) & 1u, kWait);
  }
  const bool failed = __syncthreads_or(bad) != 0;
  tc_fence_after();
  if (rec)
    P.clk[0] = clock64() - t_start;

  // Gram epilogue: warps 2, 3, 6, 7 (TMEM lanes 64..127: the odd planes)
  // park blocks 0..5 (groups 1..6) in shared memory; warps 0, 1, 4, 5 add
  // them to their blocks' groups and form the FP64 Gram entries (x = row,
  // y = column)
  double *const R = reinterpret_cast<double *>(sm + kOffR);
  double *const Vl = reinterpret_cast<double *>(sm + kOffVl);
  int *const bot = reinterpret_cast<int *>(sm + kOffBot);
  const unsigned q4 = warp & 3u, half = warp >> 2;
  if (!failed && q4 >= 2u) {
    const unsigned xr = (q4 - 2u) * 32u + lane;
#pragma unroll 1
    for (unsigned g = 0u; g < 6u; ++g)
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
        sg[0] = acc[0][k];
#pragma unroll
        for (unsigned g = 1u; g < kDig; ++g)
          sg[g] = acc[g][k] + bot[((g - 1u) * 64u + y) * 64u + xr];
        R[y * kLd + xr] = scale2(recombine(sg[0], sg[1], sg[2], sg[3], sg[4], sg[5], sg[6]), eG[xr] + eG[y] - 36);
      }
    }
  }
  if (failed && tid == 0u) {
    // before the shared memory and TMEM are given up: the copies still in
    // flight (tiles i_stop .. i_stop + kGStages - 1, as issued) and the MMAs
    // of the last tile taken complete (bounded)
    for (unsigned t = i_stop; t < ntiles && t < i_stop + kGStages; ++t)
      (void)mbar_wait_bounded(&bar[t % kGStages], (t / kGStages) & 1u, kWait / 8);
    if (i_stop > 0u)
      (void)mbar_wait_bounded(&bar[kBarPlanes + ((i_stop - 1u) & 1u)], ((i_stop - 1u) >> 1) & 1u, kWait / 8);
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
  if (rec)
    P.clk[1] = clock64() - t_start;

  // Cholesky of the Gram matrix (lower triangle, in place), one barrier per
  // column: in round k warp 0 updates column k + 1 by column k and pivots it
  // (L(i, j) = A(i, j) / sqrt(A(j, j)), by the reciprocal), while warps 1..7
  // update columns k + 2 .. 63 by column k.  A pivot that is not positive (a
  // column dependent on the previous ones to working accuracy) gives a zero
  // column of L.  Lane x holds rows x and x + 32.
  {
    const auto pivot = [&](const unsigned j) {
      __syncwarp();
      const double d = R[j * kLd + j];
      const double piv = d > 0.0 ? __dsqrt_rn(d) : 0.0, inv = piv > 0.0 ? __drcp_rn(piv) : 0.0;
      __syncwarp();
#pragma unroll
      for (unsigned h = 0u; h < 2u; ++h) {
        const unsigned i = lane + 32u * h;
        if (i > j)
          R[j * kLd + i] *= inv;
        else if (i == j)
          R[j * kLd + j] = piv;
      }
    };
    if (warp == 0u)
      pivot(0u);
    __syncthreads();
    for (unsigned k = 0u; k + 1u < 64u; ++k) {
      if (warp == 0u) {
        const unsigned j = k + 1u;
        const double ljk = R[k * kLd + j];
#pragma unroll
        for (unsigned h = 0u; h < 2u; ++h) {
          const unsigned i = lane + 32u * h;
          if (i >= j)
            R[j * kLd + i] = __fma_rn(-R[k * kLd + i], ljk, R[j * kLd + i]);
        }
        pivot(j);
      }
      else {
        // the columns of a round are independent: three at a time, so that
        // their shared-memory loads overlap (each entry's operations unchanged)
        const double l0 = R[k * kLd + lane], l1 = R[k * kLd + lane + 32u];
        unsigned j = k + 1u + warp;
#pragma unroll 1
        for (; j + 14u < 64u; j += 21u) {
          double ljk[3], a0[3], a1[3];
#pragma unroll
          for (unsigned u = 0u; u < 3u; ++u) {
            const unsigned jj = j + 7u * u;
            ljk[u] = R[k * kLd + jj];
            a0[u] = R[jj * kLd + lane];
            a1[u] = R[jj * kLd + lane + 32u];
          }
#pragma unroll
          for (unsigned u = 0u; u < 3u; ++u) {
            const unsigned jj = j + 7u * u;
            if (lane >= jj)
              R[jj * kLd + lane] = __fma_rn(-l0, ljk[u], a0[u]);
            if (lane + 32u >= jj)
              R[jj * kLd + lane + 32u] = __fma_rn(-l1, ljk[u], a1[u]);
          }
        }
#pragma unroll 1
        for (; j < 64u; j += 7u) {
          const double ljk = R[k * kLd + j];
          if (lane >= j)
            R[j * kLd + lane] = __fma_rn(-l0, ljk, R[j * kLd + lane]);
          if (lane + 32u >= j)
            R[j * kLd + lane + 32u] = __fma_rn(-l1, ljk, R[j * kLd + lane + 32u]);
        }
      }
      __syncthreads();
    }
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

  if (rec)
    P.clk[2] = clock64() - t_start;
  int definite;
  unsigned npos;
  pair_signature(P, iBlk, jBlk, definite, npos);
  unsigned blk_s = 0u, blk_b = 0u;
  inner64<SORT>(R, Vl, s0, P.s0steps, P.nswp0, definite, npos, red, blk_s, blk_b,
                reinterpret_cast<double *>(sm + kOffRot) + 16u * warp);
  if (rec)
    P.clk[3] = clock64() - t_start;

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
  if (rec)
    P.clk[4] = clock64() - t_start;
}

// ---------------------------------------------------------------------------
// sp_update_kernel: C = A B for 128-row tiles of the pairs' 64 columns of G
// and V, A the FP64 tile, B = V_loc (its digit planes diag(2^e) V_loc from
// sp_pair_kernel); C replaces A.  A persistent grid: CTA c takes a
// contiguous run of the items (pair, tile), tiles of a pair in order (G's,
// then V's), so its B operand changes rarely.  Two warp groups work on
// consecutive items at once:
//   warps 4-7 (cutters) wait for the FP64 tile of item i (TMA, two items
//     ahead, double-buffered), cut it into the 7 digit planes of A, and one
//     lane issues the MMAs: for each half of the output columns and each
//     digit t of A, one 128 x 32 (7 - t) x 32 MMA per K half against the B
//     planes t..6 side by side -- 28 MMAs, the half's 7 int32 group sums in
//     224 TMEM columns;
//   warps 0-3 (epilogue) take each half as soon as its MMAs complete, sum its
//     groups in int64, convert exactly, scale, store the row straight to
//     global memory (a warp writes 256 contiguous bytes per column) and fold
//     the magnitudes into the columns' maxima, then free the half's TMEM.
// So the cutting of item i + 1 and the MMAs of one half overlap the
// epilogue of the other.  Every wait is bounded; on a timeout the kernel
// sets the error word and both groups leave.
// ---------------------------------------------------------------------------
constexpr uint32_t kUStage = 128u * 64u * 8u;                  // FP64 tile, column c at c * 128 doubles
constexpr uint32_t kUAPlane = 8192u;                            // 128 x 64 bytes, K-major, LBO 128, SBO 512
constexpr uint32_t kOffUStage = 0u;                             // two tiles
constexpr uint32_t kOffUA = 2u * kUStage;                       // 131072
constexpr uint32_t kOffUB = kOffUA + kDig * kUAPlane;           // 188416
constexpr uint32_t kOffUFk = kOffUB + kBopBytes;                // 64 double: cut factors of A's columns
constexpr uint32_t kOffUFo = kOffUFk + 512u;                    // [2][64] double: output scales, by item parity
constexpr uint32_t kOffUCm = kOffUFo + 1024u;                   // [4][64] uint: maxima of the row quarters
constexpr uint32_t kOffUBar = kOffUCm + 1024u;                  // 10 mbarriers
constexpr uint32_t kOffUTmem = kOffUBar + 80u;
constexpr uint32_t kOffUFlag = kOffUTmem + 16u;
constexpr uint32_t kUpdSmem = kOffUFlag + 16u;
static_assert(kUpdSmem <= 227u * 1024u, "shared memory of sp_update_kernel");
// mbarriers
constexpr unsigned kBarFull = 0u;  // [2] FP64 tiles (TMA bytes)
constexpr unsigned kBarB = 2u;     // B operand (bulk copy bytes)
constexpr unsigned kBarMma = 3u;   // [2] the MMAs of a half (tcgen05.commit)
constexpr unsigned kBarFree = 5u;  // [2] a half's TMEM drained (4 epilogue warps)
constexpr unsigned kBarMeta = 7u;  // [2] an item's output scales written (cutters), by item parity

struct Item {
  unsigned pair, iBlk, jBlk, row0, rows, key;
  bool isV;
};

__device__ __forceinline__ Item item_of(const Params &P, const unsigned k)
{
  const unsigned tiles = P.tilesG + P.tilesV;
  Item it;
  it.pair = k / tiles;
  const unsigned t = k - it.pair * tiles;
  it.isV = t >= P.tilesG;
  it.row0 = (it.isV ? t - P.tilesG : t) * 128u;
  it.rows = it.isV ? P.ncol : P.nrow;
  it.key = 2u * it.pair + (it.isV ? 1u : 0u);
  const uint16_t *const blk = P.strat1 + ((size_t)P.step * P.pairs + it.pair) * 2u;
  it.iBlk = blk[0];
  it.jBlk = blk[1];
  return it;
}

__device__ __forceinline__ void load_tile(const Params &P, const Item &it, unsigned char *const dst, uint64_t *bar)
{
  const CUtensorMap *const tm = it.isV ? &P.tmV : &P.tmG;
  mbar_arrive_expect_tx(bar, kUStage);
  tma_load_2d(dst, tm, (int)it.row0, (int)(it.iBlk * kBW), bar);
  tma_load_2d(dst + kUStage / 2u, tm, (int)it.row0, (int)(it.jBlk * kBW), bar);
}

// int64 t (|t| < 2^51) as a double, exactly: the bits of 1.5 * 2^52 + t minus 1.5 * 2^52
__device__ __forceinline__ double exact_ll(const long long t)
{
  return __longlong_as_double(t + 0x4338000000000000ll) - 0x1.8p+52;
}

// sum_g 2^-8g S_g (g = 0..6) in FP64: T0 = S0 2^8 + S1, T1 = S2 2^8 + S3,
// T2 = S4 2^16 + S5 2^8 + S6 are exact int64 (below 2^48) and convert exactly;
// two roundings
__device__ __forceinline__ double recombine_u(const int s0, const int s1, const int s2, const int s3, const int s4,
                                             const int s5, const int s6)
{
  const long long t0 = (long long)s0 * 256ll + (long long)s1;
  const long long t1 = (long long)s2 * 256ll + (long long)s3;
  const long long t2 = (long long)s4 * 65536ll + (long long)s5 * 256ll + (long long)s6;
  return __fma_rn(exact_ll(t0), 0x1.0p-8, __fma_rn(exact_ll(t1), 0x1.0p-24, exact_ll(t2) * 0x1.0p-48));
}

// a bounded wait that gives up at once when the other group has aborted
__device__ __forceinline__ bool wait_or_abort(uint64_t *bar, const uint32_t parity, volatile int *abort_flag)
{
  if (mbar_try_wait(bar, parity))
    return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort_flag || clock64() - t0 > kWait)
      return false;
  }
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// named barrier id of n threads that also ORs their predicates: the same
// answer in every participating thread
__device__ __forceinline__ bool bar_or(const unsigned id, const unsigned n, const bool pred)
{
  uint32_t r;
  asm volatile("{\n\t.reg .pred p, q;\n\t"
               "setp.ne.u32 p, %1, 0;\n\t"
               "barrier.cta.red.or.pred q, %2, %3, p;\n\t"
               "selp.u32 %0, 1, 0, q;\n\t}"
               : "=r"(r)
               : "r"((uint32_t)pred), "r"(id), "r"(n)
               : "memory");
  return r != 0u;
}

template <bool ACCV>
__global__ void __launch_bounds__(kThreads, 1) sp_update_kernel(const __grid_constant__ Params P)
{
  extern __shared__ __align__(1024) unsigned char sm[];
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const unsigned nitems = P.pairs * (P.tilesG + P.tilesV);
  const unsigned per = nitems / gridDim.x, extra = nitems % gridDim.x;
  const unsigned it0 = blockIdx.x * per + min(blockIdx.x, extra);
  const unsigned it1 = it0 + per + (blockIdx.x < extra ? 1u : 0u);
  uint64_t *const bar = reinterpret_cast<uint64_t *>(sm + kOffUBar);
  uint32_t *const tmem_holder = reinterpret_cast<uint32_t *>(sm + kOffUTmem);
  volatile int *const abort_flag = reinterpret_cast<volatile int *>(sm + kOffUFlag);
  double *const fk = reinterpret_cast<double *>(sm + kOffUFk);
  double *const fo = reinterpret_cast<double *>(sm + kOffUFo);
  uint32_t *const cm = reinterpret_cast<uint32_t *>(sm + kOffUCm);
  const int *const hcol = reinterpret_cast<const int *>(sm + kOffUB + kDig * kBPlane);

  if (tid == 0u) {
    for (unsigned i = 0u; i < 3u; ++i)
      mbar_init(&bar[i], 1u);
    mbar_init(&bar[kBarMma], 1u);
    mbar_init(&bar[kBarMma + 1u], 1u);
    mbar_init(&bar[kBarFree], 4u);
    mbar_init(&bar[kBarFree + 1u], 4u);
    mbar_init(&bar[kBarMeta], 1u);
    mbar_init(&bar[kBarMeta + 1u], 1u);
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == 0u)
    tmem_alloc(tmem_holder);
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  const uint32_t sbase = smem_u32(sm);

  if (warp >= 4u) {
    // ------------------------------- cutters -------------------------------
    const unsigned ct = tid - 128u; // 0..127: row ct of the tile
    const bool lead = ct == 0u;
    // the lead's count of the asynchronous work it started and saw finish, for
    // the drain on the failure path: tile loads per buffer (issued, landed),
    // B loads, commits per half -- scalars, so that they stay in registers
    unsigned li0 = 0u, li1 = 0u, ld0 = 0u, ld1 = 0u, b_iss = 0u, b_done = 0u, mi0 = 0u, mi1 = 0u;
    // CTA 0's lead: cycles waiting for the tensor core or the epilogue (free planes, free TMEM),
    // cutting, waiting for copies (tiles, B)
    const bool timed = lead && blockIdx.x == 0u;
    long long c_mma = 0, c_cut = 0, c_copy = 0, tc = 0;
    if (lead)
      for (unsigned k = it0; k < it1 && k < it0 + 2u; ++k) {
        load_tile(P, item_of(P, k), sm + kOffUStage + (k - it0) * kUStage, &bar[kBarFull + (k - it0)]);
        li0 += (k == it0) ? 1u : 0u;
        li1 += (k == it0) ? 0u : 1u;
      }
    auto col_word = [&](const Item &x) -> uint32_t {
      const unsigned gc = (ct < kBW) ? x.iBlk * kBW + ct : x.jBlk * kBW + ct - kBW;
      return (x.isV ? P.cmaxV : P.cmaxG)[P.parity * P.ncol + gc];
    };
    uint32_t next_cmax = (ct < 64u && it0 < it1) ? col_word(item_of(P, it0)) : 0u;
    unsigned key = ~0u, nb = 0u;
    for (unsigned k = it0, n = 0u; k < it1; ++k, ++n) {
      const Item it = item_of(P, k);
      const unsigned buf = n & 1u;
      bool ok = true;
      if (timed)
        tc = clock64();
      // the previous item's MMAs are complete: A and B are free
      if (n > 0u)
        ok = wait_or_abort(&bar[kBarMma + 1u], (n - 1u) & 1u, abort_flag);
      if (timed) {
        c_mma += clock64() - tc;
        tc = clock64();
      }
      const bool newb = it.key != key;
      if (ok && newb && lead) {
        mbar_arrive_expect_tx(&bar[kBarB], kBopBytes);
        bulk_g2s(sm + kOffUB, P.bop + ((size_t)it.pair * (ACCV ? 2u : 1u) + (it.isV ? 1u : 0u)) * kBopBytes,
                 kBopBytes, &bar[kBarB]);
        ++b_iss;
      }
      if (ct < 64u)
        fk[ct] = cut_factor(col_exp(next_cmax));
      if (ok && newb) {
        ok = wait_or_abort(&bar[kBarB], nb & 1u, abort_flag);
        b_done += ok ? 1u : 0u;
      }
      if (ok) {
        ok = wait_or_abort(&bar[kBarFull + buf], (n >> 1) & 1u, abort_flag);
        ld0 += (ok && !buf) ? 1u : 0u;
        ld1 += (ok && buf) ? 1u : 0u;
      }
      if (timed) {
        c_copy += clock64() - tc;
        tc = clock64();
      }
      if (newb) {
        key = it.key;
        ++nb;
      }
      if (ct < 64u) // this item's output scales, for the epilogue
        fo[buf * 64u + ct] = p2(hcol[ct] - 12);
      // fk and fo written, every cutter's waits done; one decision for all
      if (bar_or(1u, 128u, !ok || *abort_flag)) {
        *abort_flag = 1;
        break;
      }
      if (lead)
        mbar_arrive(&bar[kBarMeta + buf]);
      // the tile's rows into the digit planes of A: row ct, pair columns 16 kg .. 16 kg + 15
      {
        const double *const st = reinterpret_cast<const double *>(sm + kOffUStage + buf * kUStage);
#pragma unroll 1
        for (unsigned kg = 0u; kg < 4u; ++kg) {
          long long w[16];
#pragma unroll
          for (unsigned i = 0u; i < 16u; ++i) {
            const unsigned c = 16u * kg + i;
            w[i] = biased_int(st[c * 128u + ct], fk[c]);
          }
          uint4 pl[kDig];
          digits16(w, pl);
          uint8_t *const dst = sm + kOffUA + (ct >> 3) * 512u + kg * 128u + (ct & 7u) * 16u;
#pragma unroll
          for (unsigned t = 0u; t < kDig; ++t)
            *reinterpret_cast<uint4 *>(dst + t * kUAPlane) = pl[t];
        }
      }
      fence_async_shared();
      bar_sync(1u, 128u);
      if (timed) {
        c_cut += clock64() - tc;
        tc = clock64();
      }
      if (ct < 64u && k + 1u < it1)
        next_cmax = col_word(item_of(P, k + 1u));
      if (lead) {
        if (k + 2u < it1) { // the tile is cut: its buffer takes the item two ahead
          load_tile(P, item_of(P, k + 2u), sm + kOffUStage + buf * kUStage, &bar[kBarFull + buf]);
          li0 += buf ? 0u : 1u;
          li1 += buf ? 1u : 0u;
        }
        const uint64_t a0 = sdesc(sbase + kOffUA, 128u, 512u), b0 = sdesc(sbase + kOffUB, 128u, 512u);
#pragma unroll
        for (unsigned h = 0u; h < 2u; ++h) {
          // the half's TMEM is drained by the epilogue of the previous item
          if (n > 0u && !wait_or_abort(&bar[kBarFree + h], (n - 1u) & 1u, abort_flag)) {
            *abort_flag = 1;
            break;
          }
          tc_fence_after();
#pragma unroll
          for (unsigned kh = 0u; kh < 2u; ++kh)
#pragma unroll
            for (unsigned t = 0u; t < kDig; ++t)
              mma_i8(tmem + h * 224u + t * 32u, a0 + ((t * kUAPlane + kh * 256u) >> 4),
                     b0 + ((h * kBHalf + kh * 256u) >> 4), idesc_i8(128u, 32u * (kDig - t)),
                     (t == 0u && kh == 0u) ? 0u : 1u);
          mma_commit(&bar[kBarMma + h]);
          mi0 += h ? 0u : 1u;
          mi1 += h ? 1u : 0u;
        }
        if (timed)
          c_mma += clock64() - tc;
      }
    }
    if (timed) {
      atomicAdd(reinterpret_cast<unsigned long long *>(P.clk + 5), (unsigned long long)c_mma);
      atomicAdd(reinterpret_cast<unsigned long long *>(P.clk + 6), (unsigned long long)c_cut);
      atomicAdd(reinterpret_cast<unsigned long long *>(P.clk + 7), (unsigned long long)c_copy);
      atomicAdd(reinterpret_cast<unsigned long long *>(P.clk + 9), (unsigned long long)(it1 - it0));
    }
    if (lead && *abort_flag) {
      // before the shared memory and TMEM are given up, what was started
      // completes (bounded): the tile loads and the B load not yet waited
      // for, and each half's last MMAs
      if (li0 > ld0)
        (void)mbar_wait_bounded(&bar[kBarFull], (li0 - 1u) & 1u, kWait / 8);
      if (li1 > ld1)
        (void)mbar_wait_bounded(&bar[kBarFull + 1u], (li1 - 1u) & 1u, kWait / 8);
      if (b_iss > b_done)
        (void)mbar_wait_bounded(&bar[kBarB], (b_iss - 1u) & 1u, kWait / 8);
      if (mi0 > 0u)
        (void)mbar_wait_bounded(&bar[kBarMma], (mi0 - 1u) & 1u, kWait / 8);
      if (mi1 > 0u)
        (void)mbar_wait_bounded(&bar[kBarMma + 1u], (mi1 - 1u) & 1u, kWait / 8);
    }
  }
  else {
    // ------------------------------ epilogue -------------------------------
    const unsigned q4 = warp, r = q4 * 32u + lane; // TMEM lanes of this warp: the tile's rows
    const bool etimed = tid == 0u && blockIdx.x == 0u;
    long long c_epi = 0, te = 0;
    for (unsigned k = it0, n = 0u; k < it1; ++k, ++n) {
      const Item it = item_of(P, k);
      const unsigned buf = n & 1u;
      if (bar_or(2u, 128u, !wait_or_abort(&bar[kBarMeta + buf], (n >> 1) & 1u, abort_flag))) {
        *abort_flag = 1;
        break;
      }
      double *const out = it.isV ? P.V : P.G;
      const size_t ld = it.isV ? P.ldV : P.ldG;
      const bool inside = it.row0 + r < it.rows;
      bool ok = true;
#pragma unroll 1
      for (unsigned h = 0u; h < 2u && ok; ++h) {
        if (bar_or(2u, 128u, !wait_or_abort(&bar[kBarMma + h], n & 1u, abort_flag))) {
          *abort_flag = 1;
          ok = false;
          break;
        }
        tc_fence_after();
        if (etimed)
          te = clock64();
        double *const colh = out + (size_t)((h ? it.jBlk : it.iBlk) * kBW) * ld + it.row0 + r;
#pragma unroll 1
        for (unsigned ch = 0u; ch < 2u; ++ch) {
          const unsigned j0 = h * 32u + ch * 16u;
          int acc[kDig][16];
#pragma unroll
          for (unsigned g = 0u; g < kDig; ++g)
            tmem_ld16(tmem + ((q4 * 32u) << 16) + h * 224u + g * 32u + ch * 16u, acc[g]);
          double f[16];
#pragma unroll
          for (unsigned kk = 0u; kk < 16u; ++kk)
            f[kk] = fo[buf * 64u + j0 + kk];
          tmem_wait_ld();
#pragma unroll
          for (unsigned kk = 0u; kk < 16u; ++kk) {
            const double c = recombine_u(acc[0][kk], acc[1][kk], acc[2][kk], acc[3][kk], acc[4][kk], acc[5][kk],
                                         acc[6][kk]) * f[kk];
            if (inside)
              colh[(size_t)(ch * 16u + kk) * ld] = c;
            const uint32_t m = __reduce_max_sync(0xffffffffu, abs_hi(c)); // rows beyond the matrix hold 0
            if (lane == 0u)
              cm[q4 * 64u + j0 + kk] = m;
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0u)
          mbar_arrive(&bar[kBarFree + h]);
        if (etimed)
          c_epi += clock64() - te;
      }
      if (!ok)
        break;
      bar_sync(2u, 128u); // the item's row-quarter maxima are written
      if (r < 64u) {
        const uint32_t m = max(max(cm[r], cm[64u + r]), max(cm[128u + r], cm[192u + r]));
        const unsigned gc = (r < kBW) ? it.iBlk * kBW + r : it.jBlk * kBW + r - kBW;
        if (m)
          atomicMax(&(it.isV ? P.cmaxV : P.cmaxG)[(P.parity ^ 1u) * P.ncol + gc], m);
      }
      bar_sync(2u, 128u);
    }
    if (etimed)
      atomicAdd(reinterpret_cast<unsigned long long *>(P.clk + 8), (unsigned long long)c_epi);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0u)
    tmem_dealloc(tmem);
  if (*abort_flag && tid == 0u)
    set_err(P);
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
  long long *d_clk = nullptr;  // 16 words: phase clocks of the last pair launch, update phase sums
  std::vector<cudaEvent_t> ev; // profiling: two per outer step
};
std::mutex g_split_mtx;
std::vector<SplitCtx> g_split_dev;
long long *g_last_clk = nullptr; // the clock words of the last call's device
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

template <bool S, bool A>
cudaError_t launch_step(const Params &p, const cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1)
{
  sp_pair_kernel<S, A><<<p.pairs, kThreads, kPairSmem, st>>>(p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return e;
  if (e0 && (e = cudaEventRecord(e0, st)) != cudaSuccess)
    return e;
  const unsigned items = p.pairs * (p.tilesG + p.tilesV);
  sp_update_kernel<A><<<items < p.sms ? items : p.sms, kThreads, kUpdSmem, st>>>(p);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return e;
  return e1 ? cudaEventRecord(e1, st) : cudaSuccess;
}

// one outer step: the pair kernel, then the update kernel (between events
// e0 and e1 when profiling)
cudaError_t launch_split_step(const bool sort, const bool accv, const Params &p, const cudaStream_t st,
                              cudaEvent_t e0, cudaEvent_t e1)
{
  if (sort)
    return accv ? launch_step<true, true>(p, st, e0, e1) : launch_step<true, false>(p, st, e0, e1);
  return accv ? launch_step<false, true>(p, st, e0, e1) : launch_step<false, false>(p, st, e0, e1);
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
    SP_CUDA(cudaMalloc(&c.d_clk, 16u * sizeof(long long)), "cudaMalloc(split clocks)");
    SP_CUDA(cudaMemset(c.d_clk, 0, 16u * sizeof(long long)), "clear split clocks");
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
  p.clk = c.d_clk;
  g_last_clk = c.d_clk;
  p.G = dG;
  p.V = full ? dV : nullptr;
  p.ldG = lddG;
  p.ldV = full ? lddV : 0u;
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
  int nsm = 148;
  SP_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev), "SM count");
  p.sms = (unsigned)nsm;

  if (full) {
    SP_CUDA(launch_initV(dV, ncol, lddV, st), "initV");
    sp_fill_kernel<<<(ncol + 255u) / 256u, 256u, 0u, st>>>(p.cmaxV, ncol, 0x3FF00000u); // |V| <= 1 = max
    SP_CUDA(cudaGetLastError(), "column maxima of V");
  }
  sp_colmax_kernel<<<(ncol + 7u) / 8u, 256u, 0u, st>>>(dG, nrow, ncol, lddG, p.cmaxG);
  SP_CUDA(cudaGetLastError(), "column maxima of G");
  SP_CUDA(cudaMemsetAsync(c.d_cnt + 1, 0, sizeof(unsigned long long), st), "clear error word");
  SP_CUDA(cudaMemsetAsync(c.d_clk + 5, 0, 5u * sizeof(long long), st), "clear update clocks");
  *glb_s = 0ull;
  *glb_b = 0ull;
  const bool prof = profiling();
  if (prof)
    while (c.ev.size() < 2u * c.steps1) {
      cudaEvent_t e = nullptr;
      SP_CUDA(cudaEventCreate(&e), "cudaEventCreate");
      c.ev.push_back(e);
    }
  profile_add(full ? 4u : 2u, 0u, 0.0); // initV, maxima of V; maxima of G, initD
  unsigned swp = 0u, gstep = 0u;
  while (swp < kNSweep) {
    SP_CUDA(cudaMemsetAsync(c.d_cnt, 0, sizeof(unsigned long long), st), "clear counter");
    for (unsigned s = 0u; s < c.steps1; ++s, ++gstep) {
      p.step = s;
      p.parity = gstep & 1u;
      SP_CUDA(launch_split_step(cdsort, full, p, st, prof ? c.ev[2u * s] : nullptr,
                                prof ? c.ev[2u * s + 1u] : nullptr),
              "split step");
    }
    ++swp;
    SP_CUDA(cudaMemcpyAsync(c.h_cnt, c.d_cnt, 2u * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st),
            "read counters");
    SP_CUDA(cudaStreamSynchronize(st), "split sweep");
    double ms = 0.0;
    if (prof)
      for (unsigned s = 0u; s < c.steps1; ++s) {
        float t = 0.0f;
        SP_CUDA(cudaEventElapsedTime(&t, c.ev[2u * s], c.ev[2u * s + 1u]), "cudaEventElapsedTime");
        ms += t;
      }
    profile_add(2ull * c.steps1, prof ? c.steps1 : 0u, ms);
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
  if (nrow > gjx::split::kMaxRows) {
    gjx::set_error("the split form takes nrow <= 16384 (its int32 Gram accumulators hold 7 x 2^14 x nrow)");
    return -2;
  }
  std::lock_guard<std::mutex> lk(gjx::g_split_mtx);
  return gjx::split_sweeps(routine, nrow, ncol, nplus, dG, lddG, dV, lddV, dD, static_cast<cudaStream_t>(stream),
                           glbSwp, glb_s, glb_b);
}

/* Cycles (clock64) from the start of block pair 0's CTA in the last
 * sp_pair_kernel launch of the last gjx_hypJacL2_split call to the end of:
 * [0] the Gram products, [1] the Gram epilogue, [2] the Cholesky factor,
 * [3] the inner sweeps, [4] the B operands; then CTA 0 of the update kernel
 * summed over the call: [5] waiting for its tile and B copies, [6] cutting
 * the tiles, [7] the products, [8] the epilogues, [9] items.  0 or
 * GJX_ERR_CUDA. */
extern "C" int gjx_split_phase_cycles(long long *out10)
{
  std::lock_guard<std::mutex> lk(gjx::g_split_mtx);
  if (!gjx::g_last_clk) {
    for (int i = 0; i < 10; ++i)
      out10[i] = 0;
    return 0;
  }
  const cudaError_t e = cudaMemcpy(out10, gjx::g_last_clk, 10u * sizeof(long long), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? 0 : GJX_ERR_CUDA;
}
