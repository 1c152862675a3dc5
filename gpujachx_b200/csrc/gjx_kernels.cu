// gjx_kernels.cu -- sm_100a kernels of the blocked one-sided Jacobi (H)SVD.
//
// One block pair (i, j) of an outer step is processed by a cluster of NSPLIT
// CTAs (NSPLIT = 4 or 2 when the step has few pairs, so that more SMs work on
// each pair; 1 when the pairs already fill the GPU), 256 threads each:
//
//   1. Gram matrix of the M x 32 column pair [G_i G_j], lower triangle only
//      (the Cholesky never reads the upper one).  Each CTA streams the whole
//      pair through shared memory in 64-row tiles (TMA tensor copies into a
//      bank-skewed, zero-padded layout, mbarrier completion, 4 stages of 2
//      tiles) and computes its share of the 528 entries; every
//      entry is one FMA chain in the reference's row order
//      (share/device_code_common_Cholesky.hpp:4-56).  A lane holds the
//      chains (x0..x0+3, y) of one column y (2-CTA clusters), also of a
//      second column (one CTA per pair), or (x0, x0+1; y) (4-CTA clusters):
//      the operands of the x columns are shared by the warp, the y columns
//      slide through a row window, and all operands come as 16-byte row
//      pairs.  The shares are exchanged through distributed shared memory,
//      then one cluster barrier.
//   2. 32x32 Cholesky by the CTA with a one-column look-ahead: warp 0 updates
//      and pivots the next column while warps 1-7 update the rest
//      (share/device_code_common_Cholesky.hpp:58-158).
//   3. Inner Jacobi sweep(s) on R: per inner step each warp sums the dot
//      products of its two pairs by register butterflies in the reference's
//      order, half-warps compute the two rotations (branch-free; trigonometric
//      or hyperbolic, optional KISS sorting) and every lane applies both to its
//      row of R and V_loc; one barrier per step (share/device_code_nosort.hpp,
//      share/device_code_cdsort.hpp, share/device_code_cdsort_KISS.hpp).
//      Steps 2 and 3 are deterministic, so every CTA of the cluster computes
//      them itself and holds the same V_loc bit for bit.
//   4. [G_i G_j] <- [G_i G_j] V_loc (and V likewise): 256-row stages brought
//      in by TMA tensor copies, the stages dealt out to the CTAs of the
//      cluster (the first one in flight during steps 2 and 3); each output
//      is a 32-FMA chain in the reference's skewed order
//      (share/device_code_common.hpp:146-185), computed in 4x8 register
//      tiles along anti-diagonals, put back in place of the stage's operands
//      and written out by TMA tensor stores that overlap the next stage.
//
// pair_step2 runs two block pairs in one CTA (the batched form, and steps
// with more pairs than SMs): steps 1 and 4 of the two one after the other on
// all warps, steps 2 and 3 concurrently on two groups of 4 warps.
//
// All arithmetic is in the reference's order, so results are bit-identical.
#include <cooperative_groups.h>
#include <cudaTypedefs.h>

#include "gjx_device.cuh"
#include "gjx_internal.h"
#include "gjx_qr.cuh"

namespace cg = cooperative_groups;

namespace gjx {

constexpr unsigned kThreads = 256u;
constexpr long long kWaitLimit = 2000000000ll; // ~1 s of cycles per wait

// Gram staging: a stage holds 2 tiles of 64 rows of the 32 columns, brought
// in by the TMA engine: per tile and block one box {66 rows, 1 tile, 16
// columns} of the 3-D view (64 rows, tiles, columns) of G.  Rows 64-65 lie
// outside the view and are zero-filled, so column c of a tile starts at
// c * 66.  The column stride of 66 doubles (33 16-byte granules, odd) puts the
// row pairs of 8 consecutive columns in 8 bank groups.  4 stages in flight;
// the copies are issued by a thread of warp 7, which computes no Gram entry.
constexpr unsigned kGramTiles = 2u;
constexpr unsigned kGramStages = 4u;
constexpr unsigned kGramColLd = 66u;
constexpr unsigned kGramTileLd = 32u * kGramColLd;
constexpr unsigned kGramStage = kGramTiles * kGramTileLd; // doubles
constexpr uint32_t kGramBoxBytes = 66u * 16u * 8u;
constexpr unsigned kIssuer = 224u; // lane 0 of warp 7

// Update staging: 256 rows x 32 columns; the 32-row piece p of column c
// starts at c*272 + p*34 (2 doubles of skew per piece spread the banks).
// One TMA tensor copy per block and stage: a 3-D view (32 rows, pieces,
// columns) of the matrix and a box of {34, 8, 16} lands exactly in this
// layout (rows 32 and 33 of a piece box lie outside the view: zero fill).
constexpr unsigned kUpdRows = 256u;
constexpr unsigned kUpdColLd = 272u;
constexpr unsigned kUpdStages = 2u;
constexpr unsigned kUpdStage = 32u * kUpdColLd; // doubles
constexpr unsigned kVTLd = 34u;                 // B^T rows (V_loc transposed)
constexpr uint32_t kUpdBoxBytes = 34u * 8u * 16u * 8u;

constexpr unsigned kRegion =
    (kGramStages * kGramStage > kUpdStages * kUpdStage) ? kGramStages * kGramStage : kUpdStages * kUpdStage;


// shared memory map (in doubles)
constexpr unsigned kOffR = kRegion;        // R, 32x32 (later B^T, 32x34)
constexpr unsigned kOffVl = kOffR + 32u * kVTLd;
constexpr unsigned kOffS0 = kOffVl + 1024u; // strat0 copy, 1024 bytes
constexpr unsigned kOffRed = kOffS0 + 128u; // 32 unsigned
constexpr unsigned kOffBar = kOffRed + 16u; // 8 mbarriers
constexpr unsigned kSmemDoubles = kOffBar + 8u;

size_t l1_smem_bytes() { return (size_t)kSmemDoubles * sizeof(double); }

// the step kernels of 2- and 4-CTA clusters keep a third update buffer after
// the rest (128-byte aligned), 227 KB in all
constexpr unsigned kOffUpd3 = (kSmemDoubles + 15u) & ~15u;
constexpr unsigned kSmemDoubles3 = kOffUpd3 + kUpdStage;
static_assert(kSmemDoubles3 * sizeof(double) <= 227u * 1024u, "the third update buffer must fit");
template <unsigned NSPLIT> struct UpdBuffers {
  static constexpr unsigned value = (NSPLIT > 1u) ? 3u : 2u;
};
size_t step_smem_bytes(const unsigned nsplit)
{
  return (size_t)((nsplit > 1u) ? kSmemDoubles3 : kSmemDoubles) * sizeof(double);
}

#define E32(A, r, c) (A)[(c) * 32u + (r)]

// ---------------------------------------------------------------------------
// Gram: one 64-row tile (at offset base of the stage) for the 4 entries
// (x0+u, y), u < 4, of one lane.  Entry (x, y) adds G[r,y]*G[r,x] for
// r = x, x+1, ..., x+63 (mod 64), the reference's order.  With k = r - x0
// (0..66, taken mod 64) chain u takes the k in [u, u+63] in increasing order.
// Operands come in 16-byte pairs of rows (k, k+1), k even (a pair never
// straddles a piece): one pair of column y and one of each column x0+u per
// two rows; the pairs of k + 4 are in flight while those of k are used.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void gram_tile(const double *const st, const unsigned base, const unsigned x0,
                                          const unsigned y, double (&acc)[4])
{
  const double *const yp = st + base + y * kGramColLd;
  const double *const xp = st + base + x0 * kGramColLd;
  double2 Yb[3], Xb[3][4];
#pragma unroll
  for (unsigned q = 0u; q < 2u; ++q) {
    const unsigned o = (x0 + 2u * q) & 63u;
    Yb[q] = *reinterpret_cast<const double2 *>(yp + o);
#pragma unroll
    for (unsigned u = 0u; u < 4u; ++u)
      Xb[q][u] = *reinterpret_cast<const double2 *>(xp + u * kGramColLd + o);
  }
#pragma unroll
  for (unsigned kp = 0u; kp < 34u; ++kp) { // pairs k = 2kp, 2kp + 1
    if (kp + 2u < 34u) {
      const unsigned q = (kp + 2u) % 3u;
      const unsigned o = (x0 + 2u * (kp + 2u)) & 63u;
      Yb[q] = *reinterpret_cast<const double2 *>(yp + o);
#pragma unroll
      for (unsigned u = 0u; u < 4u; ++u)
        if (2u * (kp + 2u) + 1u >= u && 2u * (kp + 2u) <= u + 63u)
          Xb[q][u] = *reinterpret_cast<const double2 *>(xp + u * kGramColLd + o);
    }
    const unsigned q = kp % 3u;
#pragma unroll
    for (unsigned h = 0u; h < 2u; ++h) {
      const unsigned k = 2u * kp + h;
      const double yv = h ? Yb[q].y : Yb[q].x;
#pragma unroll
      for (unsigned u = 0u; u < 4u; ++u)
        if (k >= u && k <= u + 63u)
          acc[u] = __fma_rn(yv, h ? Xb[q][u].y : Xb[q][u].x, acc[u]);
    }
  }
}

// The same for the 8 chains (x0+u, y0) and (x0+u, y1) of a lane (one CTA per
// block pair): both columns share the diagonal operands, so each 16-byte
// diagonal load feeds 4 FMAs instead of 2.
__device__ __forceinline__ void gram_tile2(const double *const st, const unsigned base, const unsigned x0,
                                           const unsigned y0, const unsigned y1, double (&acc)[4][2])
{
  const double *const yp0 = st + base + y0 * kGramColLd;
  const double *const yp1 = st + base + y1 * kGramColLd;
  const double *const xp = st + base + x0 * kGramColLd;
  double2 Yb[3][2], Xb[3][4];
#pragma unroll
  for (unsigned q = 0u; q < 2u; ++q) {
    const unsigned o = (x0 + 2u * q) & 63u;
    Yb[q][0] = *reinterpret_cast<const double2 *>(yp0 + o);
    Yb[q][1] = *reinterpret_cast<const double2 *>(yp1 + o);
#pragma unroll
    for (unsigned u = 0u; u < 4u; ++u)
      Xb[q][u] = *reinterpret_cast<const double2 *>(xp + u * kGramColLd + o);
  }
#pragma unroll
  for (unsigned kp = 0u; kp < 34u; ++kp) { // pairs k = 2kp, 2kp + 1
    if (kp + 2u < 34u) {
      const unsigned q = (kp + 2u) % 3u;
      const unsigned o = (x0 + 2u * (kp + 2u)) & 63u;
      Yb[q][0] = *reinterpret_cast<const double2 *>(yp0 + o);
      Yb[q][1] = *reinterpret_cast<const double2 *>(yp1 + o);
#pragma unroll
      for (unsigned u = 0u; u < 4u; ++u)
        if (2u * (kp + 2u) + 1u >= u && 2u * (kp + 2u) <= u + 63u)
          Xb[q][u] = *reinterpret_cast<const double2 *>(xp + u * kGramColLd + o);
    }
    const unsigned q = kp % 3u;
#pragma unroll
    for (unsigned h = 0u; h < 2u; ++h) {
      const unsigned k = 2u * kp + h;
#pragma unroll
      for (unsigned v = 0u; v < 2u; ++v) {
        const double yv = h ? Yb[q][v].y : Yb[q][v].x;
#pragma unroll
        for (unsigned u = 0u; u < 4u; ++u)
          if (k >= u && k <= u + 63u)
            acc[u][v] = __fma_rn(yv, h ? Xb[q][u].y : Xb[q][u].x, acc[u][v]);
      }
    }
  }
}

// Lanes of gram_tile2 (one CTA per pair): x-block b (rows 4b..4b+3) has
// 2(b+1) lanes; its lane j takes columns y0 = j and y1 = j + 2(b+1), i.e. all
// y = 0..4b+3 (entries with y > x are computed and dropped).  72 lanes in 3
// warps: x-blocks (7, 6, 0), (5, 4, 3), (2, 1).
__device__ __forceinline__ bool gram_lane2(const unsigned warp, const unsigned lane, unsigned &x0, unsigned &y0,
                                           unsigned &y1)
{
  if (warp >= 3u)
    return false;
  unsigned first = 0u;
#pragma unroll
  for (unsigned i = 0u; i < 3u; ++i) {
    const int b = (warp == 0u) ? ((i == 0u) ? 7 : (i == 1u) ? 6 : 0)
                               : (warp == 1u) ? ((i == 0u) ? 5 : (i == 1u) ? 4 : 3) : ((i == 0u) ? 2 : (i == 1u) ? 1 : -1);
    if (b < 0)
      return false;
    const unsigned nl = 2u * (unsigned)b + 2u;
    if (lane < first + nl) {
      const unsigned j = lane - first;
      x0 = 4u * (unsigned)b;
      y0 = j;
      y1 = j + nl;
      return true;
    }
    first += nl;
  }
  return false;
}

// The 2 chains (x0, y) and (x0+1, y) of a lane, in acc[0] and acc[1]
// (4-CTA clusters: each CTA has a quarter of the entries, and thinner lane
// tiles give it 3 warps): chain u takes the k in [u, u+63], so 33 row pairs.
__device__ __forceinline__ void gram_tile_n2(const double *const st, const unsigned base, const unsigned x0,
                                             const unsigned y, double (&acc)[4])
{
  const double *const yp = st + base + y * kGramColLd;
  const double *const xp = st + base + x0 * kGramColLd;
  double2 Yb[3], Xb[3][2];
#pragma unroll
  for (unsigned q = 0u; q < 2u; ++q) {
    const unsigned o = (x0 + 2u * q) & 63u;
    Yb[q] = *reinterpret_cast<const double2 *>(yp + o);
#pragma unroll
    for (unsigned u = 0u; u < 2u; ++u)
      Xb[q][u] = *reinterpret_cast<const double2 *>(xp + u * kGramColLd + o);
  }
#pragma unroll
  for (unsigned kp = 0u; kp < 33u; ++kp) { // pairs k = 2kp, 2kp + 1
    if (kp + 2u < 33u) {
      const unsigned q = (kp + 2u) % 3u;
      const unsigned o = (x0 + 2u * (kp + 2u)) & 63u;
      Yb[q] = *reinterpret_cast<const double2 *>(yp + o);
#pragma unroll
      for (unsigned u = 0u; u < 2u; ++u)
        if (2u * (kp + 2u) + 1u >= u && 2u * (kp + 2u) <= u + 63u)
          Xb[q][u] = *reinterpret_cast<const double2 *>(xp + u * kGramColLd + o);
    }
    const unsigned q = kp % 3u;
#pragma unroll
    for (unsigned h = 0u; h < 2u; ++h) {
      const unsigned k = 2u * kp + h;
      const double yv = h ? Yb[q].y : Yb[q].x;
#pragma unroll
      for (unsigned u = 0u; u < 2u; ++u)
        if (k >= u && k <= u + 63u)
          acc[u] = __fma_rn(yv, h ? Xb[q][u].y : Xb[q][u].x, acc[u]);
    }
  }
}

// Lanes of gram_tile_n2 in a 4-CTA cluster: x-block b (rows 2b, 2b+1) has the
// lanes y = 0..2b+1 (entries with y > x are computed and dropped); CTA r
// takes x-blocks 15-r (warp 0), 8+r then r (warp 1) and 7-r (warp 2): 68
// lanes in every CTA.
__device__ __forceinline__ bool gram_lane_q(const unsigned rank, const unsigned warp, const unsigned lane,
                                            unsigned &x0, unsigned &y)
{
  unsigned b, first = 0u;
  if (warp == 0u)
    b = 15u - rank;
  else if (warp == 1u) {
    const unsigned n1 = 2u * (8u + rank) + 2u;
    b = (lane < n1) ? 8u + rank : rank;
    first = (lane < n1) ? 0u : n1;
  }
  else if (warp == 2u)
    b = 7u - rank;
  else
    return false;
  if (lane >= first + 2u * b + 2u)
    return false;
  x0 = 2u * b;
  y = lane - first;
  return true;
}

// Lanes of gram_tile (2-CTA clusters): x-block xb (rows 4xb..4xb+3)
// has the lanes y = 0..4xb+3 (entries with y > x are computed and dropped).
// A warp takes a primary x-block p (lanes 0..4p+3) and possibly a secondary
// one s (the next 4s+4 lanes), so that the 4 operands of column x0+u are
// shared by the warp.
//   rank 0: (7), (6,0), (1); rank 1: (5), (4,2), (3)
template <unsigned NSPLIT>
__device__ __forceinline__ bool gram_lane_of(const unsigned rank, const unsigned warp, const unsigned lane,
                                             unsigned &x0, unsigned &y)
{
  static_assert(NSPLIT == 2u, "the lane map of 2-CTA clusters");
  if (warp >= 3u) // rank 0: (7), (6,0), (1); rank 1: (5), (4,2), (3)
    return false;
  const int p = (rank == 0u) ? ((warp == 2u) ? 1 : 7 - (int)warp) : 5 - (int)warp;
  const int sb = (warp == 1u) ? (rank == 0u ? 0 : 2) : -1;
  const unsigned np = 4u * (unsigned)p + 4u;
  if (lane < np) {
    x0 = 4u * (unsigned)p;
    y = lane;
    return true;
  }
  if (sb >= 0 && lane < np + 4u * (unsigned)sb + 4u) {
    x0 = 4u * (unsigned)sb;
    y = lane - np;
    return true;
  }
  return false;
}

// ---------------------------------------------------------------------------
// Right-looking Cholesky of the lower triangle held in R, by the whole CTA,
// with a one-column look-ahead: in round k warp 0 updates column k+1 by
// column k and pivots it (x > k+1: times rsqrt_rn(A(k+1,k+1)), the diagonal
// its square root) while warps 1..7 update columns k+2..31 by column k,
// A(x,j) = fma(-A(x,k), A(j,k), A(x,j)) for x >= j.  Every entry receives
// the reference's operations in the reference's order
// (share/device_code_common_Cholesky.hpp:58-158); one barrier per column.
// Afterwards R = L^T with zeros below the diagonal.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void chol_pivot(double *const R, const unsigned j, const unsigned x, const double a)
{
  const double ajj = __shfl_sync(0xffffffffu, a, j);
  const double rs = rsqrt_rn(ajj), sq = __dsqrt_rn(ajj);
  if (x > j)
    E32(R, x, j) = a * rs;
  else if (x == j)
    E32(R, j, j) = sq;
}


// by a group of NW warps (thread gt of the group, named barrier bar): the
// group's warp 0 pivots, warps 1..NW-1 update the trailing columns
template <unsigned NW>
__device__ __forceinline__ void chol32_grp(double *const R, const unsigned gt, const unsigned bar)
{
  const unsigned w = gt >> 5, x = gt & 31u;
  if (w == 0u)
    chol_pivot(R, 0u, x, E32(R, x, 0u));
  bar_sync(bar, NW * 32u);
#pragma unroll 1
  for (unsigned k = 0u; k + 1u < 32u; ++k) {
    if (w == 0u) {
      const unsigned j = k + 1u;
      double a = E32(R, x, j);
      if (x >= j)
        a = __fma_rn(-E32(R, x, k), E32(R, j, k), a);
      chol_pivot(R, j, x, a);
    }
    else {
      // the columns of a round are independent: four at a time, so that
      // their shared-memory loads overlap (each entry's operations unchanged)
      const double xk = -E32(R, x, k);
      unsigned j = k + 1u + w;
#pragma unroll 1
      for (; j + 3u * (NW - 1u) < 32u; j += 4u * (NW - 1u)) {
        double ajk[4], axj[4];
#pragma unroll
        for (unsigned u = 0u; u < 4u; ++u) {
          ajk[u] = E32(R, j + u * (NW - 1u), k);
          axj[u] = E32(R, x, j + u * (NW - 1u));
        }
#pragma unroll
        for (unsigned u = 0u; u < 4u; ++u)
          if (x >= j + u * (NW - 1u))
            E32(R, x, j + u * (NW - 1u)) = __fma_rn(xk, ajk[u], axj[u]);
      }
#pragma unroll 1
      for (; j < 32u; j += NW - 1u)
        if (x >= j)
          E32(R, x, j) = __fma_rn(xk, E32(R, j, k), E32(R, x, j));
    }
    bar_sync(bar, NW * 32u);
  }
  constexpr unsigned NV = 1024u / (NW * 32u);
  double v[NV];
#pragma unroll
  for (unsigned i = 0u; i < NV; ++i) { // element (x = col of R^T, y = row) = (i*NW*32 + gt)
    const unsigned e = i * NW * 32u + gt, xx = e >> 5, yy = e & 31u;
    v[i] = (xx >= yy) ? E32(R, xx, yy) : 0.0;
  }
  bar_sync(bar, NW * 32u);
#pragma unroll
  for (unsigned i = 0u; i < NV; ++i) {
    const unsigned e = i * NW * 32u + gt, xx = e >> 5, yy = e & 31u;
    E32(R, yy, xx) = v[i];
  }
}

// ---------------------------------------------------------------------------
// Inner Jacobi sweep(s) on R (32x32) accumulating V_loc.  Per inner step (16
// disjoint column pairs) warp w owns pairs w and w + 8, lane x = row x:
//   the six dot products (Dp, Dq, Apq of both pairs) by register butterflies
//   in the reference's order (share/device_code_common_Kepler.hpp:26-74:
//   lane i adds lane i^16, ^8, ^4, ^2, ^1; IEEE addition commutes, so every
//   lane ends with lane 0's bits); lanes 0-15 compute pair w's rotation
//   (branch-free), lanes 16-31 pair w+8's; the halves trade them with one
//   shuffle; each lane applies both to its row of R and V_loc from the values
//   it loaded at the start of the step.  One barrier per step.
// Every operation is the reference's (share/device_code_nosort.hpp:4-222,
// share/device_code_cdsort.hpp:25-167, share/device_code_cdsort_KISS.hpp).
// ---------------------------------------------------------------------------
// apply rotation r to row x of columns p, q of R (values Gp, Gq, already
// loaded) and of V_loc (Vp, Vq); mode 0 leaves them, 2 swaps the columns
__device__ __forceinline__ void inner_apply(double *const R, double *const Vl, const unsigned p, const unsigned q,
                                            const Rot &r, const unsigned x, const double Gp, const double Gq,
                                            const double Vp, const double Vq)
{
  if (r.mode == 0)
    return;
  if (r.mode == 2) {
    E32(R, x, p) = Gq;
    E32(R, x, q) = Gp;
    E32(Vl, x, p) = Vq;
    E32(Vl, x, q) = Vp;
    return;
  }
  double np = __fma_rn(r.t_, Gq, Gp), nq = __fma_rn(r.t, Gp, Gq);
  double vp = __fma_rn(r.t_, Vq, Vp), vq = __fma_rn(r.t, Vp, Vq);
  if (r.scale) {
    np = r.c * np;
    nq = r.c * nq;
    vp = r.c * vp;
    vq = r.c * vq;
  }
  const unsigned dp = r.swap ? q : p, dq = r.swap ? p : q;
  E32(R, x, dp) = np;
  E32(R, x, dq) = nq;
  E32(Vl, x, dp) = vp;
  E32(Vl, x, dq) = vq;
}

// by a group of NW warps (8 or 4; lane x, warp w of the group, named barrier
// bar): warp w takes the NC = 8 / NW couples of pairs (w + c NW, w + c NW + 8)
// of each inner step, interleaved
template <bool SORT, unsigned NW>
__device__ __forceinline__ void inner_sweeps(double *const R, double *const Vl, const uint8_t *const s0,
                                             const unsigned s0steps, const unsigned nswp, const int definite,
                                             const unsigned npos, unsigned *const red, const unsigned x,
                                             const unsigned w, const unsigned bar, unsigned &blk_s, unsigned &blk_b)
{
  constexpr unsigned NC = 8u / NW;
  blk_s = 0u;
  blk_b = 0u;
  const bool hb = x >= 16u; // this half computes the couple's second pair (else its first)
  for (unsigned swp = 0u; swp < nswp; ++swp) {
    unsigned ws = 0u, wb = 0u; // lanes 0 and 16: their pairs' counts
    for (unsigned step = 0u; step < s0steps; ++step) {
      const uint8_t *const st = s0 + step * 32u;
      unsigned pa[NC], qa[NC], pb[NC], qb[NC];
      double Gpa[NC], Gqa[NC], Gpb[NC], Gqb[NC], Vpa[NC], Vqa[NC], Vpb[NC], Vqb[NC], v[NC][3];
#pragma unroll
      for (unsigned c = 0u; c < NC; ++c) {
        const unsigned a = w + c * NW;
        pa[c] = st[2u * a];
        qa[c] = st[2u * a + 1u];
        pb[c] = st[2u * a + 16u];
        qb[c] = st[2u * a + 17u];
        Gpa[c] = E32(R, x, pa[c]);
        Gqa[c] = E32(R, x, qa[c]);
        Gpb[c] = E32(R, x, pb[c]);
        Gqb[c] = E32(R, x, qb[c]);
        // V_loc of the same rows, loaded now so that the application waits for no load
        Vpa[c] = E32(Vl, x, pa[c]);
        Vqa[c] = E32(Vl, x, qa[c]);
        Vpb[c] = E32(Vl, x, pb[c]);
        Vqb[c] = E32(Vl, x, qb[c]);
        // the butterfly as a reduce-scatter: at the first level (lane ^ 16)
        // each lane keeps the products of its half's pair and receives the
        // partner's products of the same pair; the other four levels stay
        // within the half.  Every lane adds the same operands in the same
        // order as the full butterfly would, with half the shuffles.
        const double va[3] = {__fma_rn(Gpa[c], Gpa[c], 0.0), __fma_rn(Gqa[c], Gqa[c], 0.0),
                              __fma_rn(Gpa[c], Gqa[c], 0.0)};
        const double vb[3] = {__fma_rn(Gpb[c], Gpb[c], 0.0), __fma_rn(Gqb[c], Gqb[c], 0.0),
                              __fma_rn(Gpb[c], Gqb[c], 0.0)};
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i) {
          const double other = __shfl_xor_sync(0xffffffffu, hb ? va[i] : vb[i], 16);
          v[c][i] = (hb ? vb[i] : va[i]) + other;
        }
      }
#pragma unroll
      for (unsigned k = 8u; k; k >>= 1u) {
        double o[NC][3];
#pragma unroll
        for (unsigned c = 0u; c < NC; ++c)
#pragma unroll
          for (unsigned i = 0u; i < 3u; ++i)
            o[c][i] = __shfl_xor_sync(0xffffffffu, v[c][i], k);
#pragma unroll
        for (unsigned c = 0u; c < NC; ++c)
#pragma unroll
          for (unsigned i = 0u; i < 3u; ++i)
            v[c][i] = v[c][i] + o[c][i];
      }
      Rot r[NC];
#pragma unroll
      for (unsigned c = 0u; c < NC; ++c) {
        unsigned a_s, a_b;
        r[c] = inner_rot<SORT>(v[c][0], v[c][1], v[c][2], hb ? pb[c] : pa[c], hb ? qb[c] : qa[c], definite, npos, a_s,
                               a_b);
        if (x == 0u || x == 16u) {
          ws += a_s;
          wb += a_b;
        }
      }
#pragma unroll
      for (unsigned c = 0u; c < NC; ++c) {
        Rot o;
        o.c = __shfl_xor_sync(0xffffffffu, r[c].c, 16);
        o.t = __shfl_xor_sync(0xffffffffu, r[c].t, 16);
        o.t_ = __shfl_xor_sync(0xffffffffu, r[c].t_, 16);
        const int fl = __shfl_xor_sync(0xffffffffu, r[c].mode | (r[c].scale << 2) | (r[c].swap << 3), 16);
        o.mode = fl & 3;
        o.scale = (fl >> 2) & 1;
        o.swap = (fl >> 3) & 1;
        const Rot m = r[c]; // a value: selecting between two lvalues would take their addresses
        inner_apply(R, Vl, pa[c], qa[c], hb ? o : m, x, Gpa[c], Gqa[c], Vpa[c], Vqa[c]);
        inner_apply(R, Vl, pb[c], qb[c], hb ? m : o, x, Gpb[c], Gqb[c], Vpb[c], Vqb[c]);
      }
      bar_sync(bar, NW * 32u);
    }
    ws = __reduce_add_sync(0xffffffffu, ws);
    wb = __reduce_add_sync(0xffffffffu, wb);
    if (x == 0u) {
      red[2u * w] = ws;
      red[2u * w + 1u] = wb;
    }
    bar_sync(bar, NW * 32u);
    unsigned tot_s = 0u, tot_b = 0u;
#pragma unroll
    for (unsigned k = 0u; k < NW; ++k) {
      tot_s += red[2u * k];
      tot_b += red[2u * k + 1u];
    }
    bar_sync(bar, NW * 32u);
    if (tot_s) {
      blk_s += tot_s;
      blk_b += tot_b;
    }
    else
      break;
  }
}

// by a group of 4 warps (lane x, warp w of the group, named barrier bar):
// warp w takes pairs w, w + 4, w + 8, w + 12 of each inner step, and quarter
// k of the warp (lanes 8k .. 8k + 7) computes pair w + 4k's rotation.  The
// twelve dot products go through a reduce-scatter: at level 16 each half
// keeps its two pairs' products (lanes 0-15 pairs w, w + 4), at level 8 each
// quarter its own pair's, levels 4, 2, 1 stay within the quarter -- the same
// operands in the same order as the full butterfly, with one rotation to
// evaluate per warp and step.  Every lane then applies the four rotations.
// The four rotations of a warp reach its lanes through shared memory (rs: 16
// doubles of this warp's own; the lane 8k writes pair k's, every lane reads
// all four back with broadcast loads), not through shuffles.
template <bool SORT>
__device__ __forceinline__ void inner_sweeps_q(double *const R, double *const Vl, const uint8_t *const s0,
                                               const unsigned s0steps, const unsigned nswp, const int definite,
                                               const unsigned npos, unsigned *const red, const unsigned x,
                                               const unsigned w, const unsigned bar, unsigned &blk_s,
                                               unsigned &blk_b, double *const rs)
{
  blk_s = 0u;
  blk_b = 0u;
  const bool up = x >= 16u, odd = ((x >> 3) & 1u) != 0u;
  const unsigned mine = w + 4u * (x >> 3); // the pair this lane's quarter evaluates
  for (unsigned swp = 0u; swp < nswp; ++swp) {
    unsigned ws = 0u, wb = 0u; // lanes 0, 8, 16, 24: their pairs' counts
    for (unsigned step = 0u; step < s0steps; ++step) {
      const uint8_t *const st = s0 + step * 32u;
      unsigned p[4], q[4];
      double Gp[4], Gq[4], Vp[4], Vq[4], v[4][3];
#pragma unroll
      for (unsigned k = 0u; k < 4u; ++k) {
        p[k] = st[2u * (w + 4u * k)];
        q[k] = st[2u * (w + 4u * k) + 1u];
        Gp[k] = E32(R, x, p[k]);
        Gq[k] = E32(R, x, q[k]);
        Vp[k] = E32(Vl, x, p[k]);
        Vq[k] = E32(Vl, x, q[k]);
        v[k][0] = __fma_rn(Gp[k], Gp[k], 0.0);
        v[k][1] = __fma_rn(Gq[k], Gq[k], 0.0);
        v[k][2] = __fma_rn(Gp[k], Gq[k], 0.0);
      }
      const unsigned pm = st[2u * mine], qm = st[2u * mine + 1u];
      double h[2][3], s[3];
#pragma unroll
      for (unsigned j = 0u; j < 2u; ++j)
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i) {
          const double other = __shfl_xor_sync(0xffffffffu, up ? v[j][i] : v[2u + j][i], 16);
          h[j][i] = (up ? v[2u + j][i] : v[j][i]) + other;
        }
#pragma unroll
      for (unsigned i = 0u; i < 3u; ++i) {
        const double other = __shfl_xor_sync(0xffffffffu, odd ? h[0][i] : h[1][i], 8);
        s[i] = (odd ? h[1][i] : h[0][i]) + other;
      }
#pragma unroll
      for (unsigned k = 4u; k; k >>= 1u) {
        double o[3];
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i)
          o[i] = __shfl_xor_sync(0xffffffffu, s[i], k);
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i)
          s[i] = s[i] + o[i];
      }
      unsigned a_s, a_b;
      const Rot r = inner_rot<SORT>(s[0], s[1], s[2], pm, qm, definite, npos, a_s, a_b);
      if (!(x & 7u)) {
        ws += a_s;
        wb += a_b;
        double *const e = rs + 4u * (x >> 3);
        e[0] = r.c;
        e[1] = r.t;
        e[2] = r.t_;
        e[3] = __longlong_as_double((long long)(r.mode | (r.scale << 2) | (r.swap << 3)));
      }
      __syncwarp();
#pragma unroll
      for (unsigned k = 0u; k < 4u; ++k) {
        const double2 ct = *reinterpret_cast<const double2 *>(rs + 4u * k);
        const double2 tf = *reinterpret_cast<const double2 *>(rs + 4u * k + 2u);
        Rot o;
        o.c = ct.x;
        o.t = ct.y;
        o.t_ = tf.x;
        const int f = (int)__double_as_longlong(tf.y);
        o.mode = f & 3;
        o.scale = (f >> 2) & 1;
        o.swap = (f >> 3) & 1;
        inner_apply(R, Vl, p[k], q[k], o, x, Gp[k], Gq[k], Vp[k], Vq[k]);
      }
      bar_sync(bar, 128u);
    }
    ws = __reduce_add_sync(0xffffffffu, ws);
    wb = __reduce_add_sync(0xffffffffu, wb);
    if (x == 0u) {
      red[2u * w] = ws;
      red[2u * w + 1u] = wb;
    }
    bar_sync(bar, 128u);
    unsigned tot_s = 0u, tot_b = 0u;
#pragma unroll
    for (unsigned k = 0u; k < 4u; ++k) {
      tot_s += red[2u * k];
      tot_b += red[2u * k + 1u];
    }
    bar_sync(bar, 128u);
    if (tot_s) {
      blk_s += tot_s;
      blk_b += tot_b;
    }
    else
      break;
  }
}

// by a group of 2 warps (lane x, warp w of the group, named barrier bar):
// warp w takes pairs w, w + 2, ..., w + 14 of each inner step, and eighth k
// of the warp (lanes 4k .. 4k + 3) computes pair w + 2k's rotation.  The
// reduce-scatter of inner_sweeps_q goes one level further: at level 16 each
// half keeps four pairs' products, at 8 each quarter two, at 4 each eighth
// its own, levels 2 and 1 stay within the eighth -- the same operands in the
// same order as the full butterfly.  Every lane then applies the eight
// rotations to its row.
// The eight rotations of a warp reach its lanes through shared memory (rs:
// 32 doubles of this warp's own; lane 4k writes pair k's), as in
// inner_sweeps_q.
template <bool SORT>
__device__ __forceinline__ void inner_sweeps_e(double *const R, double *const Vl, const uint8_t *const s0,
                                               const unsigned s0steps, const unsigned nswp, const int definite,
                                               const unsigned npos, unsigned *const red, const unsigned x,
                                               const unsigned w, const unsigned bar, unsigned &blk_s,
                                               unsigned &blk_b, double *const rs)
{
  blk_s = 0u;
  blk_b = 0u;
  const bool up = x >= 16u, odd8 = ((x >> 3) & 1u) != 0u, odd4 = ((x >> 2) & 1u) != 0u;
  const unsigned mine = w + 2u * (x >> 2); // the pair this lane's eighth evaluates
  for (unsigned swp = 0u; swp < nswp; ++swp) {
    unsigned ws = 0u, wb = 0u; // lanes 0, 4, ..., 28: their pairs' counts
    for (unsigned step = 0u; step < s0steps; ++step) {
      const uint8_t *const st = s0 + step * 32u;
      unsigned p[8], q[8];
      double Gp[8], Gq[8], Vp[8], Vq[8], v[8][3];
#pragma unroll
      for (unsigned k = 0u; k < 8u; ++k) {
        p[k] = st[2u * (w + 2u * k)];
        q[k] = st[2u * (w + 2u * k) + 1u];
        Gp[k] = E32(R, x, p[k]);
        Gq[k] = E32(R, x, q[k]);
        Vp[k] = E32(Vl, x, p[k]);
        Vq[k] = E32(Vl, x, q[k]);
        v[k][0] = __fma_rn(Gp[k], Gp[k], 0.0);
        v[k][1] = __fma_rn(Gq[k], Gq[k], 0.0);
        v[k][2] = __fma_rn(Gp[k], Gq[k], 0.0);
      }
      const unsigned pm = st[2u * mine], qm = st[2u * mine + 1u];
      double h4[4][3], h2[2][3], s[3];
#pragma unroll
      for (unsigned j = 0u; j < 4u; ++j)
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i) {
          const double other = __shfl_xor_sync(0xffffffffu, up ? v[j][i] : v[4u + j][i], 16);
          h4[j][i] = (up ? v[4u + j][i] : v[j][i]) + other;
        }
#pragma unroll
      for (unsigned j = 0u; j < 2u; ++j)
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i) {
          const double other = __shfl_xor_sync(0xffffffffu, odd8 ? h4[j][i] : h4[2u + j][i], 8);
          h2[j][i] = (odd8 ? h4[2u + j][i] : h4[j][i]) + other;
        }
#pragma unroll
      for (unsigned i = 0u; i < 3u; ++i) {
        const double other = __shfl_xor_sync(0xffffffffu, odd4 ? h2[0][i] : h2[1][i], 4);
        s[i] = (odd4 ? h2[1][i] : h2[0][i]) + other;
      }
#pragma unroll
      for (unsigned k = 2u; k; k >>= 1u) {
        double o[3];
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i)
          o[i] = __shfl_xor_sync(0xffffffffu, s[i], k);
#pragma unroll
        for (unsigned i = 0u; i < 3u; ++i)
          s[i] = s[i] + o[i];
      }
      unsigned a_s, a_b;
      const Rot r = inner_rot<SORT>(s[0], s[1], s[2], pm, qm, definite, npos, a_s, a_b);
      if (!(x & 3u)) {
        ws += a_s;
        wb += a_b;
        double *const e = rs + 4u * (x >> 2);
        e[0] = r.c;
        e[1] = r.t;
        e[2] = r.t_;
        e[3] = __longlong_as_double((long long)(r.mode | (r.scale << 2) | (r.swap << 3)));
      }
      __syncwarp();
#pragma unroll
      for (unsigned k = 0u; k < 8u; ++k) {
        const double2 ct = *reinterpret_cast<const double2 *>(rs + 4u * k);
        const double2 tf = *reinterpret_cast<const double2 *>(rs + 4u * k + 2u);
        Rot o;
        o.c = ct.x;
        o.t = ct.y;
        o.t_ = tf.x;
        const int f = (int)__double_as_longlong(tf.y);
        o.mode = f & 3;
        o.scale = (f >> 2) & 1;
        o.swap = (f >> 3) & 1;
        inner_apply(R, Vl, p[k], q[k], o, x, Gp[k], Gq[k], Vp[k], Vq[k]);
      }
      bar_sync(bar, 64u);
    }
    ws = __reduce_add_sync(0xffffffffu, ws);
    wb = __reduce_add_sync(0xffffffffu, wb);
    if (x == 0u) {
      red[2u * w] = ws;
      red[2u * w + 1u] = wb;
    }
    bar_sync(bar, 64u);
    const unsigned tot_s = red[0] + red[2], tot_b = red[1] + red[3];
    bar_sync(bar, 64u);
    if (tot_s) {
      blk_s += tot_s;
      blk_b += tot_b;
    }
    else
      break;
  }
}

// ---------------------------------------------------------------------------
// Update of one 256-row stage: warp rg (0..7), lane = sub + 8*cg.  The thread
// owns rows sub*32 + rg*4 + (0..3) and columns cg*8 + (0..7); entry (u, v)
// adds A[r, s] * B[s, c] for s = (x + c + k) mod 32, k = 0..31, x = r mod 32,
// i.e. the anti-diagonal index t = u + v + k reads column s = x0 + c0 + t.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void update_stage(const double *const st, const double *const VT, const unsigned rg,
                                             const unsigned sub, const unsigned cg, double (&acc)[4][8])
{
  const unsigned x0 = rg * 4u, c0 = cg * 8u;
  const double *const ab = st + sub * 34u + x0;
  const double *const bb = VT + c0;
#pragma unroll
  for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
    for (unsigned v = 0u; v < 8u; ++v)
      acc[u][v] = +0.0;
#pragma unroll
  for (unsigned t = 0u; t < 42u; ++t) {
    const unsigned s = (x0 + c0 + t) & 31u;
    const double2 a01 = *reinterpret_cast<const double2 *>(ab + s * kUpdColLd);
    const double2 a23 = *reinterpret_cast<const double2 *>(ab + s * kUpdColLd + 2u);
    const double a[4] = {a01.x, a01.y, a23.x, a23.y};
    const double2 b01 = *reinterpret_cast<const double2 *>(bb + s * kVTLd);
    const double2 b23 = *reinterpret_cast<const double2 *>(bb + s * kVTLd + 2u);
    const double2 b45 = *reinterpret_cast<const double2 *>(bb + s * kVTLd + 4u);
    const double2 b67 = *reinterpret_cast<const double2 *>(bb + s * kVTLd + 6u);
    const double b[8] = {b01.x, b01.y, b23.x, b23.y, b45.x, b45.y, b67.x, b67.y};
#pragma unroll
    for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
      for (unsigned v = 0u; v < 8u; ++v) {
        if ((t >= u + v) && (t - u - v < 32u))
          acc[u][v] = __fma_rn(a[u], b[v], acc[u][v]);
      }
  }
}

// the stage's results in place of its operands: the thread's 4 rows x 8
// columns go where update_stage read them; warp rg read only its own rows
// (rg*4 .. rg*4+3 of each 32-row piece), so after __syncwarp nothing that
// another lane still needs is overwritten.  A TMA store then writes the stage
// back (rows 32-33 of a piece lie outside the view and are not written).
__device__ __forceinline__ void update_put(double *const st, const double (&acc)[4][8], const unsigned rg,
                                           const unsigned sub, const unsigned cg8)
{
  double *const o = st + sub * 34u + rg * 4u;
#pragma unroll
  for (unsigned v = 0u; v < 8u; ++v) {
    double *const col = o + (cg8 * 8u + v) * kUpdColLd;
    *reinterpret_cast<double2 *>(col) = make_double2(acc[0][v], acc[1][v]);
    *reinterpret_cast<double2 *>(col + 2u) = make_double2(acc[2][v], acc[3][v]);
  }
}

// the signature of block pair (iBlk, jBlk): global if the matrix is definite,
// else block-local (share/device_code_nosort_solveV.hpp:33-67)
__device__ __forceinline__ void block_signature(const StepParams &P, const unsigned iBlk, const unsigned jBlk,
                                                int &definite, unsigned &npos)
{
  const unsigned ifc0 = iBlk * kNColB, ifc1 = jBlk * kNColB, nplus = P.nplus;
  if (P.gdefinite) {
    definite = P.gdefinite;
    npos = 0u;
  }
  else if (nplus <= ifc0) {
    npos = 0u;
    definite = -1;
  }
  else if (nplus <= ifc0 + kNColB) {
    npos = nplus - ifc0;
    definite = 0;
  }
  else if (nplus <= ifc1) {
    npos = kNColB;
    definite = 0;
  }
  else if (nplus <= ifc1 + kNColB) {
    npos = kNColB + (nplus - ifc1);
    definite = 0;
  }
  else {
    npos = 2u * kNColB;
    definite = +1;
  }
}

// a block pair's rotation counts into its matrix's sweep counter: big << 32 |
// small, or the low word alone when no rotation was big, as the reference
__device__ __forceinline__ void add_counts(const StepParams &P, const unsigned blk_s, const unsigned blk_b)
{
  if (!blk_s)
    return;
  if (blk_b)
    atomicAdd(P.cvg, (((unsigned long long)blk_b) << 32) | blk_s);
  else
    atomicAdd(reinterpret_cast<unsigned *>(P.cvg), blk_s);
}

// ---------------------------------------------------------------------------
// The block-pair step kernel.
// ---------------------------------------------------------------------------
// NBUF update buffers: 2 in the region of the Gram stages, a third (NBUF = 3)
// at kOffUpd3 where the launch provides it
template <bool SORT, bool ACCV, unsigned NSPLIT, unsigned NBUF = 2u, unsigned FAC = 0u>
__device__ __forceinline__ void pair_step(const StepParams &P, const unsigned step, const unsigned pair,
                                          const unsigned rank, double *const sm)
{
  static_assert(FAC == 0u || NSPLIT == 1u, "the QR factor is one CTA's");
  static_assert(NBUF == 2u || NBUF == 3u, "2 or 3 update buffers");
  double *const stg = sm;
  double *const R = sm + kOffR;
  double *const Vl = sm + kOffVl;
  uint8_t *const s0 = reinterpret_cast<uint8_t *>(sm + kOffS0);
  unsigned *const red = reinterpret_cast<unsigned *>(sm + kOffRed);
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kOffBar);

  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const size_t pidx = ((size_t)step * P.pairs + pair) * 2u;
  const unsigned iBlk = P.strat1[pidx + 0u], jBlk = P.strat1[pidx + 1u];

  for (unsigned i = tid; i < 256u; i += kThreads)
    reinterpret_cast<uint32_t *>(s0)[i] = reinterpret_cast<const uint32_t *>(P.strat0)[i];
  if (tid == 0u) {
    for (unsigned b = 0u; b < 8u; ++b)
      mbar_init(&bars[b], 1u); // one arrival with the expected bytes, the TMA engine completes it
    mbar_fence_init();
  }
  __syncthreads();

  int failed = 0;
  if constexpr (FAC != 0u) {
    // ----------------- 1'. QR factor (the -DUSE_QR builds) -----------------
    qr_factor_cta(P.G + (size_t)iBlk * kNColB * P.ldG, P.G + (size_t)jBlk * kNColB * P.ldG, P.ldG, P.nrow, R, stg);
  }
  else {
  // ------------------------------ 1. Gram --------------------------------
  const unsigned ntile = P.nrow >> 6; // 64-row tiles
  // chains per lane: 8 with one CTA per pair (gram_tile2), 4 with 2 CTAs
  // (gram_tile), 2 with 4 CTAs (gram_tile_n2); 3 Gram warps each
  unsigned gx0 = 0u, gy = 0u, gy1 = 0u;
  const unsigned gwarps = 3u;
  bool gthr;
  if constexpr (NSPLIT == 1u)
    gthr = gram_lane2(warp, lane, gx0, gy, gy1);
  else if constexpr (NSPLIT == 4u)
    gthr = gram_lane_q(rank, warp, lane, gx0, gy);
  else
    gthr = gram_lane_of<NSPLIT>(rank, warp, lane, gx0, gy);
  double gacc[4] = {+0.0, +0.0, +0.0, +0.0};
  double gacc2[4][2] = {{+0.0, +0.0}, {+0.0, +0.0}, {+0.0, +0.0}, {+0.0, +0.0}};

  const unsigned ngst = (ntile + kGramTiles - 1u) / kGramTiles; // stages of 2 tiles
  // thread 0: the TMA engine brings stage k, per tile block i's and block j's
  // 16 columns as one box each
  auto issue_gram = [&](const unsigned k) {
    const unsigned s = k % kGramStages;
    const unsigned nt = min(kGramTiles, ntile - k * kGramTiles);
    double *const st = stg + s * kGramStage;
    mbar_arrive_expect_tx(&bars[s], nt * 2u * kGramBoxBytes);
    for (unsigned t = 0u; t < nt; ++t) {
      const int tile = (int)(k * kGramTiles + t);
      tma_load_3d(st + t * kGramTileLd, &P.tmGram, 0, tile, (int)(iBlk * kNColB), &bars[s]);
      tma_load_3d(st + t * kGramTileLd + 16u * kGramColLd, &P.tmGram, 0, tile, (int)(jBlk * kNColB), &bars[s]);
    }
  };

  if (tid == kIssuer)
    for (unsigned k = 0u; k + 1u < kGramStages && k < ngst; ++k)
      issue_gram(k);
  unsigned k = 0u;
  for (; k < ngst; ++k) {
    if (tid == kIssuer && k + kGramStages - 1u < ngst)
      issue_gram(k + kGramStages - 1u); // into the buffer released at the end of stage k - 1
    int fail = 0;
    if (warp < gwarps) {
      if (!mbar_wait_bounded(&bars[k % kGramStages], (k / kGramStages) & 1u, kWaitLimit))
        fail = 1;
      else if (gthr) {
        const unsigned nt = min(kGramTiles, ntile - k * kGramTiles);
        for (unsigned t = 0u; t < nt; ++t) {
          if constexpr (NSPLIT == 1u)
            gram_tile2(stg + (k % kGramStages) * kGramStage, t * kGramTileLd, gx0, gy, gy1, gacc2);
          else if constexpr (NSPLIT == 4u)
            gram_tile_n2(stg + (k % kGramStages) * kGramStage, t * kGramTileLd, gx0, gy, gacc);
          else
            gram_tile(stg + (k % kGramStages) * kGramStage, t * kGramTileLd, gx0, gy, gacc);
        }
      }
    }
    failed = __syncthreads_or(fail); // uniform decision
    if (failed)
      break;
  }
  if (failed && tid == 0u) { // let the copies in flight land (bounded) before anything else, report
    for (unsigned q = k; q < ngst && q < k + kGramStages; ++q)
      (void)mbar_wait_bounded(&bars[q % kGramStages], (q / kGramStages) & 1u, kWaitLimit / 8);
    atomicOr(P.err, kErrWaitTimeout);
  }
  // our share of the lower triangle, into our R and the other CTAs' R
  if constexpr (NSPLIT == 1u) {
    if (gthr) {
#pragma unroll
      for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
        for (unsigned v = 0u; v < 2u; ++v) {
          const unsigned y = v ? gy1 : gy;
          if (gx0 + u >= y)
            R[y * 32u + gx0 + u] = gacc2[u][v];
        }
    }
  }
  else if (gthr) {
#pragma unroll
    for (unsigned u = 0u; u < ((NSPLIT == 4u) ? 2u : 4u); ++u)
      if (gx0 + u >= gy) {
        const unsigned o = gy * 32u + gx0 + u;
        R[o] = gacc[u];
        if (NSPLIT > 1u) {
          cg::cluster_group cl = cg::this_cluster();
#pragma unroll
          for (unsigned q = 1u; q < NSPLIT; ++q)
            cl.map_shared_rank(R, (rank + q) % NSPLIT)[o] = gacc[u];
        }
      }
  }
  }
  if (NSPLIT > 1u)
    cg::this_cluster().sync(); // release our writes, acquire the others'
  else
    __syncthreads();
  if (failed)
    return; // the error word is set; the host reports it

  // the first update stage of this CTA: its rows do not change before the
  // update, so the copy overlaps the Cholesky and the inner sweeps
  const unsigned nG = (P.nrow + kUpdRows - 1u) / kUpdRows;
  const unsigned nV = ACCV ? (P.ncol + kUpdRows - 1u) / kUpdRows : 0u;
  const unsigned nst = nG + nV;
  const unsigned nmine = (nst > rank) ? (nst - rank + NSPLIT - 1u) / NSPLIT : 0u;
  auto ubuf = [&](const unsigned s) { return (NBUF == 3u && s == 2u) ? sm + kOffUpd3 : stg + s * kUpdStage; };
  auto issue_upd = [&](const unsigned i) { // one thread: this CTA's i-th stage, 2 tensor copies
    const unsigned k = rank + i * NSPLIT, s = i % NBUF;
    const bool isG = k < nG;
    const CUtensorMap *const tm = isG ? &P.tmG : &P.tmV;
    const int piece = (int)(((isG ? k : (k - nG)) * kUpdRows) >> 5);
    double *const st = ubuf(s);
    mbar_arrive_expect_tx(&bars[4u + s], 2u * kUpdBoxBytes);
    tma_load_3d(st, tm, 0, piece, (int)(iBlk * kNColB), &bars[4u + s]);
    tma_load_3d(st + 16u * kUpdColLd, tm, 0, piece, (int)(jBlk * kNColB), &bars[4u + s]);
  };
  if (tid == 0u && nmine > 0u)
    issue_upd(0u);

  // ---------------------------- 2. Cholesky -------------------------------
  for (unsigned i = tid; i < 1024u; i += kThreads)
    Vl[i] = ((i >> 5) == (i & 31u)) ? 1.0 : 0.0;
  if constexpr (FAC == 0u)
    chol32_grp<8u>(R, tid, 0u);
  __syncthreads();

  // --------------------------- 3. inner sweeps ----------------------------
  int definite;
  unsigned npos;
  block_signature(P, iBlk, jBlk, definite, npos);
  unsigned blk_s, blk_b;
  if (FAC == 2u && SORT && definite) // -DUSE_DRMAC: Drmac's sweep in the definite sorting kernels
    drmac_sweeps(R, Vl, s0, P.s0steps, P.nswp0, definite, red, lane, warp, blk_s, blk_b);
  else
    inner_sweeps<SORT, 8u>(R, Vl, s0, P.s0steps, P.nswp0, definite, npos, red, lane, warp, 0u, blk_s, blk_b);

  if (rank == 0u && tid == 0u)
    add_counts(P, blk_s, blk_b);
  if (!SORT && !blk_s) { // no rotation: the block pair is unchanged
    if (tid == 0u && nmine > 0u && !mbar_wait_bounded(&bars[4u], 0u, kWaitLimit))
      atomicOr(P.err, kErrWaitTimeout); // the prefetched copy has landed before we leave
    return;
  }

  // ------------------------------ 4. update -------------------------------
  double *const VT = R; // R is dead; B^T[s][c] = V_loc[s][c]
  for (unsigned i = tid; i < 1024u; i += kThreads) {
    const unsigned c = i >> 5, s = i & 31u;
    VT[s * kVTLd + c] = E32(Vl, s, c);
  }

  __syncthreads(); // VT ready
  // stage i: thread 0 issues the copy of stage i + 1 into its buffer once the
  // store that last used that buffer has read it out (with 2 buffers the
  // store of stage i - 1, issued just before; with 3 that of stage i - 2, a
  // stage ago); the warps compute stage i and put the results in place;
  // after the barrier thread 0 stores them with two tensor copies, which
  // overlap the next stage's arithmetic
  const unsigned rg = warp, sub = lane & 7u, cg8 = lane >> 3;
  for (unsigned i = 0u; i < nmine; ++i) {
    if (tid == 0u && i + 1u < nmine) {
      if (NBUF == 3u)
        bulk_wait_read_but1();
      else
        bulk_wait_read();
      issue_upd(i + 1u);
    }
    // a warp computes only if all its lanes saw the stage land
    const int fail = !__all_sync(0xffffffffu, mbar_wait_bounded(&bars[4u + (i % NBUF)], (i / NBUF) & 1u,
                                                                kWaitLimit));
    double *const sb = ubuf(i % NBUF);
    if (!fail) {
      double acc[4][8]; // the whole warp computes (rows past the end: not stored)
      update_stage(sb, VT, rg, sub, cg8, acc);
      __syncwarp();
      update_put(sb, acc, rg, sub, cg8);
      fence_async_shared();
    }
    if (__syncthreads_or(fail)) { // uniform decision; drain (bounded), report
      if (tid == 0u) {
        (void)mbar_wait_bounded(&bars[4u + (i % NBUF)], (i / NBUF) & 1u, kWaitLimit / 8);
        if (i + 1u < nmine)
          (void)mbar_wait_bounded(&bars[4u + ((i + 1u) % NBUF)], ((i + 1u) / NBUF) & 1u, kWaitLimit / 8);
        bulk_wait_all();
        atomicOr(P.err, kErrWaitTimeout);
      }
      return;
    }
    if (tid == 0u) {
      const unsigned k = rank + i * NSPLIT;
      const bool isG = k < nG;
      const CUtensorMap *const tm = isG ? &P.tmG : &P.tmV;
      const int piece = (int)(((isG ? k : (k - nG)) * kUpdRows) >> 5);
      tma_store_3d(tm, sb, 0, piece, (int)(iBlk * kNColB));
      tma_store_3d(tm, sb + 16u * kUpdColLd, 0, piece, (int)(jBlk * kNColB));
      bulk_commit();
    }
  }
  if (tid == 0u)
    bulk_wait_all(); // the stores are complete before the block pair counts as done
}

// ---------------------------------------------------------------------------
// Two block pairs in one CTA (batched form; pair A of matrix PA, pair B of
// matrix PB).  The Grams and the updates run on all 8 warps, A's then B's,
// as one stream of stages each (the copies of B's first stages overlap A's
// last ones).  The Cholesky factorisations and the inner sweeps, chains of
// dependent divides and square roots that leave the SM's pipes mostly idle,
// run concurrently: warps 0-3 take pair A (named barrier 1), warps 4-7 pair B
// (barrier 2).  Every entry of R, V_loc and the updated columns is computed
// with the same operations in the same order as by pair_step, so each matrix
// gets the bits it would get alone.
// ---------------------------------------------------------------------------
constexpr unsigned kOffR2 = kSmemDoubles; // pair B's R (later B^T), V_loc, counters
constexpr unsigned kOffVl2 = kOffR2 + 32u * kVTLd;
constexpr unsigned kOffRed2 = kOffVl2 + 1024u;
constexpr unsigned kOffRot2 = kOffRed2 + 16u; // the rotations of the 8 warps (inner_sweeps_q), 16 doubles each
constexpr unsigned kSmemDoubles2 = kOffRot2 + 128u;

size_t batch2_smem_bytes() { return (size_t)kSmemDoubles2 * sizeof(double); }

template <bool SORT, bool ACCV>
__device__ __forceinline__ void pair_step2(const StepParams &PA, const unsigned stepA, const unsigned pairA,
                                           const StepParams &PB, const unsigned stepB, const unsigned pairB,
                                           double *const sm)
{
  double *const stg = sm;
  uint8_t *const s0 = reinterpret_cast<uint8_t *>(sm + kOffS0);
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kOffBar);
  unsigned *const flags = reinterpret_cast<unsigned *>(sm + kOffRed2) + 30u; // [g]: pair g updates

  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  size_t pidx = ((size_t)stepA * PA.pairs + pairA) * 2u;
  const unsigned iA = PA.strat1[pidx + 0u], jA = PA.strat1[pidx + 1u];
  pidx = ((size_t)stepB * PB.pairs + pairB) * 2u;
  const unsigned iB = PB.strat1[pidx + 0u], jB = PB.strat1[pidx + 1u];

  for (unsigned i = tid; i < 256u; i += kThreads)
    reinterpret_cast<uint32_t *>(s0)[i] = reinterpret_cast<const uint32_t *>(PA.strat0)[i];
  if (tid == 0u) {
    for (unsigned b = 0u; b < 8u; ++b)
      mbar_init(&bars[b], 1u);
    mbar_fence_init();
  }
  __syncthreads();

  // ------------------------------ 1. Grams --------------------------------
  // stages 0 .. ngA-1 are A's, ngA .. ngA+ngB-1 B's
  const unsigned ntA = PA.nrow >> 6, ntB = PB.nrow >> 6;
  const unsigned ngA = (ntA + kGramTiles - 1u) / kGramTiles, ngB = (ntB + kGramTiles - 1u) / kGramTiles;
  const unsigned ng = ngA + ngB;
  unsigned gx0 = 0u, gy = 0u, gy1 = 0u;
  const bool gthr = gram_lane2(warp, lane, gx0, gy, gy1);
  double gacc[4][2] = {{+0.0, +0.0}, {+0.0, +0.0}, {+0.0, +0.0}, {+0.0, +0.0}};
  auto stage_tiles = [&](const unsigned k) {
    return (k < ngA) ? min(kGramTiles, ntA - k * kGramTiles) : min(kGramTiles, ntB - (k - ngA) * kGramTiles);
  };
  auto issue_gram = [&](const unsigned k) {
    const unsigned s = k % kGramStages;
    const bool a = k < ngA;
    const unsigned t0 = (a ? k : (k - ngA)) * kGramTiles, nt = stage_tiles(k);
    const CUtensorMap *const tm = a ? &PA.tmGram : &PB.tmGram;
    const int ci = (int)((a ? iA : iB) * kNColB), cj = (int)((a ? jA : jB) * kNColB);
    double *const st = stg + s * kGramStage;
    mbar_arrive_expect_tx(&bars[s], nt * 2u * kGramBoxBytes);
    for (unsigned t = 0u; t < nt; ++t) {
      tma_load_3d(st + t * kGramTileLd, tm, 0, (int)(t0 + t), ci, &bars[s]);
      tma_load_3d(st + t * kGramTileLd + 16u * kGramColLd, tm, 0, (int)(t0 + t), cj, &bars[s]);
    }
  };
  auto put_gram = [&](double *const R) { // our share of the lower triangle
    if (gthr) {
#pragma unroll
      for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
        for (unsigned v = 0u; v < 2u; ++v) {
          const unsigned y = v ? gy1 : gy;
          if (gx0 + u >= y)
            R[y * 32u + gx0 + u] = gacc[u][v];
          gacc[u][v] = +0.0;
        }
    }
  };

  if (tid == kIssuer)
    for (unsigned k = 0u; k + 1u < kGramStages && k < ng; ++k)
      issue_gram(k);
  unsigned k = 0u;
  int failed = 0;
  for (; k < ng; ++k) {
    if (tid == kIssuer && k + kGramStages - 1u < ng)
      issue_gram(k + kGramStages - 1u);
    int fail = 0;
    if (warp < 3u) {
      if (!mbar_wait_bounded(&bars[k % kGramStages], (k / kGramStages) & 1u, kWaitLimit))
        fail = 1;
      else if (gthr) {
        const unsigned nt = stage_tiles(k);
        for (unsigned t = 0u; t < nt; ++t)
          gram_tile2(stg + (k % kGramStages) * kGramStage, t * kGramTileLd, gx0, gy, gy1, gacc);
      }
      if (k + 1u == ngA)
        put_gram(sm + kOffR);
      else if (k + 1u == ng)
        put_gram(sm + kOffR2);
    }
    failed = __syncthreads_or(fail);
    if (failed)
      break;
  }
  if (failed) {
    if (tid == 0u) {
      for (unsigned q = k; q < ng && q < k + kGramStages; ++q)
        (void)mbar_wait_bounded(&bars[q % kGramStages], (q / kGramStages) & 1u, kWaitLimit / 8);
      atomicOr(PA.err, kErrWaitTimeout);
      atomicOr(PB.err, kErrWaitTimeout);
    }
    return;
  }

  // A's first update stage, in flight during the serial phases
  const unsigned nGA = (PA.nrow + kUpdRows - 1u) / kUpdRows, nGB = (PB.nrow + kUpdRows - 1u) / kUpdRows;
  const unsigned nstA = nGA + (ACCV ? (PA.ncol + kUpdRows - 1u) / kUpdRows : 0u);
  const unsigned nstB = nGB + (ACCV ? (PB.ncol + kUpdRows - 1u) / kUpdRows : 0u);
  // update stage geometry: pair g's i-th stage
  auto stage_geom = [&](const unsigned g, const unsigned i, double *&ci, double *&cj, size_t &ld, unsigned &base,
                        unsigned &rows, const CUtensorMap *&tm, int &piece) {
    const StepParams &P = g ? PB : PA;
    const unsigned nG = g ? nGB : nGA, iBlk = g ? iB : iA, jBlk = g ? jB : jA;
    if (i < nG) {
      ci = P.G + (size_t)iBlk * kNColB * P.ldG;
      cj = P.G + (size_t)jBlk * kNColB * P.ldG;
      ld = P.ldG;
      base = i * kUpdRows;
      rows = min(kUpdRows, P.nrow - base);
      tm = &P.tmG;
    }
    else {
      ci = P.V + (size_t)iBlk * kNColB * P.ldV;
      cj = P.V + (size_t)jBlk * kNColB * P.ldV;
      ld = P.ldV;
      base = (i - nG) * kUpdRows;
      rows = min(kUpdRows, P.ncol - base);
      tm = &P.tmV;
    }
    piece = (int)(base >> 5);
  };
  auto issue_upd = [&](const unsigned q, const unsigned g, const unsigned i) { // stream position q
    double *ci, *cj;
    size_t ld;
    unsigned base, rows;
    const CUtensorMap *tm;
    int piece;
    stage_geom(g, i, ci, cj, ld, base, rows, tm, piece);
    const unsigned s = q % kUpdStages;
    double *const st = stg + s * kUpdStage;
    mbar_arrive_expect_tx(&bars[4u + s], 2u * kUpdBoxBytes);
    tma_load_3d(st, tm, 0, piece, (int)((g ? iB : iA) * kNColB), &bars[4u + s]);
    tma_load_3d(st + 16u * kUpdColLd, tm, 0, piece, (int)((g ? jB : jA) * kNColB), &bars[4u + s]);
  };
  if (tid == 0u)
    issue_upd(0u, 0u, 0u);

  // ------------------- 2.-3. Cholesky and inner sweeps --------------------
  {
    const unsigned grp = warp >> 2, gt = tid & 127u, gw = warp & 3u;
    const StepParams &P = grp ? PB : PA;
    double *const R = sm + (grp ? kOffR2 : kOffR);
    double *const Vl = sm + (grp ? kOffVl2 : kOffVl);
    unsigned *const red = reinterpret_cast<unsigned *>(sm + (grp ? kOffRed2 : kOffRed));
    for (unsigned i = gt; i < 1024u; i += 128u)
      Vl[i] = ((i >> 5) == (i & 31u)) ? 1.0 : 0.0;
    chol32_grp<4u>(R, gt, 1u + grp);
    bar_sync(1u + grp, 128u);
    int definite;
    unsigned npos;
    block_signature(P, grp ? iB : iA, grp ? jB : jA, definite, npos);
    unsigned blk_s, blk_b;
    inner_sweeps_q<SORT>(R, Vl, s0, P.s0steps, P.nswp0, definite, npos, red, lane, gw, 1u + grp, blk_s, blk_b,
                         sm + kOffRot2 + 16u * warp);
    if (gt == 0u) {
      add_counts(P, blk_s, blk_b);
      flags[grp] = (SORT || blk_s) ? 1u : 0u;
    }
  }
  __syncthreads();
  const bool updA = flags[0] != 0u, updB = flags[1] != 0u;
  // the stream of update stages: A's (or, when A is unchanged, its prefetched
  // first stage, waited for and dropped), then B's
  const unsigned qa = updA ? nstA : 1u, nq = qa + (updB ? nstB : 0u);
  if (nq == 1u && !updA) {
    if (tid == 0u && !mbar_wait_bounded(&bars[4u], 0u, kWaitLimit))
      atomicOr(PA.err, kErrWaitTimeout);
    return;
  }

  // ------------------------------ 4. updates ------------------------------
  for (unsigned i = tid; i < 2048u; i += kThreads) { // both R are dead: B^T[s][c] = V_loc[s][c]
    const unsigned g = i >> 10, c = (i >> 5) & 31u, s_ = i & 31u;
    (sm + (g ? kOffR2 : kOffR))[s_ * kVTLd + c] = E32(sm + (g ? kOffVl2 : kOffVl), s_, c);
  }
  __syncthreads();
  const unsigned rg = warp, sub = lane & 7u, cg8 = lane >> 3;
  for (unsigned q = 0u; q < nq; ++q) {
    if (tid == 0u && q + 1u < nq) {
      const unsigned q1 = q + 1u;
      bulk_wait_read(); // the store of stage q - 1 has read the buffer stage q + 1 lands in
      if (q1 < qa)
        issue_upd(q1, 0u, q1);
      else
        issue_upd(q1, 1u, q1 - qa);
    }
    const int fail = !__all_sync(0xffffffffu, mbar_wait_bounded(&bars[4u + (q % kUpdStages)], (q / kUpdStages) & 1u,
                                                                kWaitLimit));
    const unsigned g = (q < qa) ? 0u : 1u;
    const bool work = g == 1u || updA;
    double *const sb = stg + (q % kUpdStages) * kUpdStage;
    if (!fail && work) {
      double acc[4][8];
      update_stage(sb, sm + (g ? kOffR2 : kOffR), rg, sub, cg8, acc);
      __syncwarp();
      update_put(sb, acc, rg, sub, cg8);
      fence_async_shared();
    }
    if (__syncthreads_or(fail)) {
      if (tid == 0u) {
        (void)mbar_wait_bounded(&bars[4u + (q % kUpdStages)], (q / kUpdStages) & 1u, kWaitLimit / 8);
        if (q + 1u < nq)
          (void)mbar_wait_bounded(&bars[4u + ((q + 1u) % kUpdStages)], ((q + 1u) / kUpdStages) & 1u,
                                  kWaitLimit / 8);
        bulk_wait_all();
        atomicOr(g ? PB.err : PA.err, kErrWaitTimeout);
      }
      return;
    }
    if (tid == 0u && work) {
      double *ci, *cj;
      size_t ld;
      unsigned base, rows;
      const CUtensorMap *tm;
      int piece;
      stage_geom(g, g ? q - qa : q, ci, cj, ld, base, rows, tm, piece);
      tma_store_3d(tm, sb, 0, piece, (int)((g ? iB : iA) * kNColB));
      tma_store_3d(tm, sb + 16u * kUpdColLd, 0, piece, (int)((g ? jB : jA) * kNColB));
      bulk_commit();
    }
  }
  if (tid == 0u)
    bulk_wait_all();
}

// one launch per outer step: block pair blockIdx.x / NSPLIT, cluster rank
// blockIdx.x % NSPLIT
template <bool SORT, bool ACCV, unsigned NSPLIT>
__global__ void __launch_bounds__(kThreads, 1) l1_step_kernel(const __grid_constant__ StepParams P)
{
  extern __shared__ __align__(128) double sm[];
  const unsigned rank = (NSPLIT > 1u) ? (blockIdx.x % NSPLIT) : 0u;
  pair_step<SORT, ACCV, NSPLIT, UpdBuffers<NSPLIT>::value>(P, P.step, blockIdx.x / NSPLIT, rank, sm);
}

// one launch per outer step, two block pairs per CTA (a step with more pairs
// than SMs: one wave instead of two, and the two pairs' serial phases
// overlap): CTA c takes pairs 2c and 2c + 1 through pair_step2, or the last
// pair alone through pair_step
template <bool SORT, bool ACCV>
__global__ void __launch_bounds__(kThreads, 1) l1_step2_kernel(const __grid_constant__ StepParams P)
{
  extern __shared__ __align__(128) double sm[];
  const unsigned a = 2u * blockIdx.x;
  if (a + 1u < P.pairs)
    pair_step2<SORT, ACCV>(P, P.step, a, P, P.step, a + 1u, sm);
  else
    pair_step<SORT, ACCV, 1u>(P, P.step, a, 0u, sm);
}

// ---------------------------------------------------------------------------
// One launch for a whole sweep.  Cluster c takes block pair c of every outer
// step in turn.  A block is rewritten by exactly one pair per step, so pair
// (i, j) of step s may start once both blocks have been written by all CTAs
// of their step s-1 pairs: P.ver counts those CTAs (NSPLIT per step).
// Thread 0 of each CTA waits for the counts (bounded); the CTAs of a cluster
// agree through distributed shared memory and a cluster barrier, so they
// leave together on an error (pair_step has one cluster barrier on every
// path).  Writers fence their stores before counting; readers acquire the
// counts and fence the async proxy before their tile copies.  All clusters
// are resident at once (cooperative launch, checked on the host).
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire(const unsigned *p)
{
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// the reference's alternative builds (P.variant: 1 -DUSE_QR, 2 -DUSE_DRMAC):
// one CTA per block pair, the QR factor in place of the Gram and Cholesky
template <bool SORT, bool ACCV, unsigned FAC>
__global__ void __launch_bounds__(kThreads, 1) l1_var_kernel(const __grid_constant__ StepParams P)
{
  extern __shared__ __align__(128) double sm[];
  pair_step<SORT, ACCV, 1u, 2u, FAC>(P, P.step, blockIdx.x, 0u, sm);
}

template <bool SORT, bool ACCV, unsigned NSPLIT>
__global__ void __launch_bounds__(kThreads, 1) l1_sweep_kernel(const __grid_constant__ StepParams P)
{
  extern __shared__ __align__(128) double sm[];
  __shared__ unsigned agree[NSPLIT]; // [r]: CTA r of the cluster may proceed
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kOffBar);
  const unsigned rank = (NSPLIT > 1u) ? (blockIdx.x % NSPLIT) : 0u;
  const unsigned pair = blockIdx.x / NSPLIT;
  for (unsigned step = 0u; step < P.steps1; ++step) {
    const size_t pidx = ((size_t)step * P.pairs + pair) * 2u;
    const unsigned iB = P.strat1[pidx + 0u], jB = P.strat1[pidx + 1u];
    if (threadIdx.x == 0u) {
      const unsigned need = NSPLIT * step;
      unsigned ok = (*(volatile int *)P.err == 0) ? 1u : 0u;
      const long long t0 = clock64();
      while (ok && (ld_acquire(P.ver + iB) < need || ld_acquire(P.ver + jB) < need)) {
        if (*(volatile int *)P.err)
          ok = 0u;
        else if (clock64() - t0 > kWaitLimit) {
          atomicOr(P.err, kErrWaitTimeout);
          ok = 0u;
        }
        else
          __nanosleep(64);
      }
      for (unsigned q = 0u; q < NSPLIT; ++q)
        cg::this_cluster().map_shared_rank(agree, q)[rank] = ok;
    }
    if (NSPLIT > 1u)
      cg::this_cluster().sync();
    else
      __syncthreads();
    unsigned all = 1u;
    for (unsigned q = 0u; q < NSPLIT; ++q)
      all &= agree[q];
    if (!all)
      break; // the same decision in every CTA of the cluster
    asm volatile("fence.proxy.async;" ::: "memory"); // the copies below read what other SMs wrote
    pair_step<SORT, ACCV, NSPLIT, UpdBuffers<NSPLIT>::value>(P, step, pair, rank, sm);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0u) {
      __threadfence();
      atomicAdd(P.ver + iB, 1u);
      atomicAdd(P.ver + jB, 1u);
      for (unsigned k = 0u; k < 8u; ++k)
        mbar_inval(&bars[k]);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Batched form: each launch advances every active matrix of a batch by one
// outer step of its own sweep (matrix b: step kstep[b] mod steps1), so small
// matrices run their short sweeps back to back while large ones progress.  A
// persistent grid (one CTA per SM) takes the block pairs -- (matrix << 16) |
// pair, largest matrices first -- from a work queue, W at a time: with W = 2
// two live pairs go through pair_step2 together, a lone one through
// pair_step with one CTA, so every matrix gets the bits it would get alone.
// Converged matrices are skipped.  The mbarriers are invalidated after each
// item (both step forms initialise them).
// ---------------------------------------------------------------------------
template <bool SORT, bool ACCV, unsigned W>
__global__ void __launch_bounds__(kThreads, 1) l1_batch_kernel(const __grid_constant__ BatchStep B)
{
  extern __shared__ __align__(128) double sm[];
  __shared__ unsigned item;
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kOffBar);
  for (;;) {
    if (threadIdx.x == 0u)
      item = atomicAdd(B.queue, W);
    __syncthreads();
    const unsigned it = item;
    const bool stop = (it >= B.nitems) || (*(volatile int *)B.err != 0);
    __syncthreads(); // every thread has read item
    if (stop)
      break;
    const uint32_t e0 = B.items[it];
    const unsigned b0 = e0 >> 16u;
    const bool live0 = !B.done[b0];
    uint32_t e1 = 0u;
    bool live1 = false;
    if (W == 2u && it + 1u < B.nitems) {
      e1 = B.items[it + 1u];
      live1 = !B.done[e1 >> 16u];
    }
    if (!live0 && !live1)
      continue;
    if (live0 && live1 && B.mats[b0].p.strat0 == B.mats[e1 >> 16u].p.strat0) {
      const BatchMat &ma = B.mats[b0], &mb = B.mats[e1 >> 16u];
      pair_step2<SORT, ACCV>(ma.p, B.kstep[b0] % ma.steps1, e0 & 0xffffu, mb.p, B.kstep[e1 >> 16u] % mb.steps1,
                             e1 & 0xffffu, sm);
    }
    else {
      for (unsigned h = 0u; h < 2u; ++h) {
        const bool live = h ? live1 : live0;
        if (!live)
          continue;
        const uint32_t e = h ? e1 : e0;
        const BatchMat &m = B.mats[e >> 16u];
        pair_step<SORT, ACCV, 1u>(m.p, B.kstep[e >> 16u] % m.steps1, e & 0xffffu, 0u, sm);
        __syncthreads();
        if (threadIdx.x == 0u)
          for (unsigned k = 0u; k < 8u; ++k)
            mbar_inval(&bars[k]);
        __syncthreads();
      }
      continue;
    }
    __syncthreads();
    if (threadIdx.x == 0u)
      for (unsigned k = 0u; k < 8u; ++k)
        mbar_inval(&bars[k]);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// One block pair on a CTA of 4 warps (batched form, two such CTAs per SM).
// The arithmetic is that of pair_step with one CTA per pair -- the Gram
// chains of gram_tile2 on warps 0-2 (warp 3 issues the tile copies), the
// Cholesky factorisation and quarter-warp inner sweeps of pair_step2's warp
// groups, pair_step's update tiles (warp w takes row groups w and w + 4 of
// every stage) -- so every matrix gets the bits of its single call.  Shared
// memory (86 KB): the Gram's 4 stages of one 64-row tile, later one update
// buffer; R, V_loc.  With one buffer a stage's copy waits for the store of
// the stage before; the other CTA of the SM runs meanwhile, and its serial
// phases (Cholesky, inner sweeps: chains of divides and square roots that
// leave the pipes idle) overlap this CTA's Gram and update, and the reverse.
// ---------------------------------------------------------------------------
constexpr unsigned kNThreads = 128u;
constexpr unsigned kNGStages = 4u;
constexpr unsigned kNIssuer = 96u; // lane 0 of warp 3
constexpr unsigned kNRegion = (kNGStages * kGramTileLd > kUpdStage) ? kNGStages * kGramTileLd : kUpdStage;
constexpr unsigned kNOffR = kNRegion; // R, 32x32 (later B^T, 32x34)
constexpr unsigned kNOffVl = kNOffR + 32u * kVTLd;
constexpr unsigned kNOffS0 = kNOffVl + 1024u;
constexpr unsigned kNOffRed = kNOffS0 + 128u;
constexpr unsigned kNOffBar = kNOffRed + 16u; // [0..3] Gram stages, [4] the update buffer
constexpr unsigned kNOffRot = kNOffBar + 8u; // the rotations of the 4 warps (inner_sweeps_q), 16 doubles each
constexpr unsigned kNSmemDoubles = kNOffRot + 64u;
static_assert(2u * (kNSmemDoubles * sizeof(double) + 1024u) <= 228u * 1024u, "two CTAs per SM");
size_t batchn_smem_bytes() { return (size_t)kNSmemDoubles * sizeof(double); }

template <bool SORT, bool ACCV>
__device__ __forceinline__ void pair_step_n(const StepParams &P, const unsigned step, const unsigned pair,
                                            double *const sm)
{
  double *const stg = sm;
  double *const R = sm + kNOffR;
  double *const Vl = sm + kNOffVl;
  uint8_t *const s0 = reinterpret_cast<uint8_t *>(sm + kNOffS0);
  unsigned *const red = reinterpret_cast<unsigned *>(sm + kNOffRed);
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kNOffBar);
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const size_t pidx = ((size_t)step * P.pairs + pair) * 2u;
  const unsigned iBlk = P.strat1[pidx + 0u], jBlk = P.strat1[pidx + 1u];

  for (unsigned i = tid; i < 256u; i += kNThreads)
    reinterpret_cast<uint32_t *>(s0)[i] = reinterpret_cast<const uint32_t *>(P.strat0)[i];
  if (tid == 0u) {
    for (unsigned b = 0u; b < 5u; ++b)
      mbar_init(&bars[b], 1u);
    mbar_fence_init();
  }
  __syncthreads();

  // ------------------------------ 1. Gram --------------------------------
  const unsigned ntile = P.nrow >> 6;
  unsigned gx0 = 0u, gy = 0u, gy1 = 0u;
  const bool gthr = gram_lane2(warp, lane, gx0, gy, gy1);
  double gacc[4][2] = {{+0.0, +0.0}, {+0.0, +0.0}, {+0.0, +0.0}, {+0.0, +0.0}};
  auto issue_gram = [&](const unsigned k) { // tile k into stage k mod 4
    const unsigned s = k % kNGStages;
    double *const st = stg + s * kGramTileLd;
    mbar_arrive_expect_tx(&bars[s], 2u * kGramBoxBytes);
    tma_load_3d(st, &P.tmGram, 0, (int)k, (int)(iBlk * kNColB), &bars[s]);
    tma_load_3d(st + 16u * kGramColLd, &P.tmGram, 0, (int)k, (int)(jBlk * kNColB), &bars[s]);
  };
  if (tid == kNIssuer)
    for (unsigned k = 0u; k + 1u < kNGStages && k < ntile; ++k)
      issue_gram(k);
  unsigned k = 0u;
  int failed = 0;
  for (; k < ntile; ++k) {
    if (tid == kNIssuer && k + kNGStages - 1u < ntile)
      issue_gram(k + kNGStages - 1u); // into the stage released after tile k - 1
    int fail = 0;
    if (warp < 3u) {
      if (!mbar_wait_bounded(&bars[k % kNGStages], (k / kNGStages) & 1u, kWaitLimit))
        fail = 1;
      else if (gthr)
        gram_tile2(stg + (k % kNGStages) * kGramTileLd, 0u, gx0, gy, gy1, gacc);
    }
    failed = __syncthreads_or(fail);
    if (failed)
      break;
  }
  if (failed) {
    if (tid == 0u) { // the copies in flight land (bounded) before anything else, report
      for (unsigned q = k; q < ntile && q < k + kNGStages; ++q)
        (void)mbar_wait_bounded(&bars[q % kNGStages], (q / kNGStages) & 1u, kWaitLimit / 8);
      atomicOr(P.err, kErrWaitTimeout);
    }
    return;
  }
  if (gthr) {
#pragma unroll
    for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
      for (unsigned v = 0u; v < 2u; ++v) {
        const unsigned y = v ? gy1 : gy;
        if (gx0 + u >= y)
          R[y * 32u + gx0 + u] = gacc[u][v];
      }
  }
  __syncthreads();

  // the first update stage: its rows do not change before the update, so the
  // copy overlaps the Cholesky and the inner sweeps
  const unsigned nG = (P.nrow + kUpdRows - 1u) / kUpdRows;
  const unsigned nst = nG + (ACCV ? (P.ncol + kUpdRows - 1u) / kUpdRows : 0u);
  auto issue_upd = [&](const unsigned i) {
    const bool isG = i < nG;
    const CUtensorMap *const tm = isG ? &P.tmG : &P.tmV;
    const int piece = (int)(((isG ? i : (i - nG)) * kUpdRows) >> 5);
    mbar_arrive_expect_tx(&bars[4], 2u * kUpdBoxBytes);
    tma_load_3d(stg, tm, 0, piece, (int)(iBlk * kNColB), &bars[4]);
    tma_load_3d(stg + 16u * kUpdColLd, tm, 0, piece, (int)(jBlk * kNColB), &bars[4]);
  };
  if (tid == 0u && nst > 0u)
    issue_upd(0u);

  // ------------------- 2.-3. Cholesky and inner sweeps --------------------
  for (unsigned i = tid; i < 1024u; i += kNThreads)
    Vl[i] = ((i >> 5) == (i & 31u)) ? 1.0 : 0.0;
  chol32_grp<4u>(R, tid, 0u);
  __syncthreads();
  int definite;
  unsigned npos;
  block_signature(P, iBlk, jBlk, definite, npos);
  unsigned blk_s, blk_b;
  inner_sweeps_q<SORT>(R, Vl, s0, P.s0steps, P.nswp0, definite, npos, red, lane, warp, 0u, blk_s, blk_b,
                       sm + kNOffRot + 16u * warp);
  if (tid == 0u)
    add_counts(P, blk_s, blk_b);
  if (!SORT && !blk_s) { // no rotation: the block pair is unchanged
    if (tid == 0u && nst > 0u && !mbar_wait_bounded(&bars[4], 0u, kWaitLimit))
      atomicOr(P.err, kErrWaitTimeout); // the prefetched copy has landed before we leave
    return;
  }

  // ------------------------------ 4. update -------------------------------
  for (unsigned i = tid; i < 1024u; i += kNThreads) { // R is dead: B^T[s][c] = V_loc[s][c]
    const unsigned c = i >> 5, s_ = i & 31u;
    R[s_ * kVTLd + c] = E32(Vl, s_, c);
  }
  __syncthreads();
  const unsigned sub = lane & 7u, cg8 = lane >> 3;
  for (unsigned i = 0u; i < nst; ++i) {
    if (tid == 0u && i > 0u) {
      bulk_wait_read(); // the store of stage i - 1 has read the buffer out
      issue_upd(i);
    }
    const int fail = !__all_sync(0xffffffffu, mbar_wait_bounded(&bars[4], i & 1u, kWaitLimit));
    if (!fail) {
#pragma unroll 1
      for (unsigned h = 0u; h < 2u; ++h) { // row groups warp and warp + 4
        double acc[4][8];
        update_stage(stg, R, warp + 4u * h, sub, cg8, acc);
        __syncwarp();
        update_put(stg, acc, warp + 4u * h, sub, cg8);
      }
      fence_async_shared();
    }
    if (__syncthreads_or(fail)) {
      if (tid == 0u) {
        (void)mbar_wait_bounded(&bars[4], i & 1u, kWaitLimit / 8);
        bulk_wait_all();
        atomicOr(P.err, kErrWaitTimeout);
      }
      return;
    }
    if (tid == 0u) {
      const bool isG = i < nG;
      const CUtensorMap *const tm = isG ? &P.tmG : &P.tmV;
      const int piece = (int)(((isG ? i : (i - nG)) * kUpdRows) >> 5);
      tma_store_3d(tm, stg, 0, piece, (int)(iBlk * kNColB));
      tma_store_3d(tm, stg + 16u * kUpdColLd, 0, piece, (int)(jBlk * kNColB));
      bulk_commit();
    }
  }
  if (tid == 0u)
    bulk_wait_all(); // the stores are complete before the block pair counts as done
}

// The batched step on CTAs of 4 warps, two per SM: a CTA takes one block pair
// at a time from the queue (the same queue, items and skips as
// l1_batch_kernel).  The mbarriers are invalidated after each item.
template <bool SORT, bool ACCV>
__global__ void __launch_bounds__(kNThreads, 2) l1_batchn_kernel(const __grid_constant__ BatchStep B)
{
  extern __shared__ __align__(128) double sm[];
  __shared__ unsigned item;
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kNOffBar);
  for (;;) {
    if (threadIdx.x == 0u)
      item = atomicAdd(B.queue, 1u);
    __syncthreads();
    const unsigned it = item;
    const bool stop = (it >= B.nitems) || (*(volatile int *)B.err != 0);
    __syncthreads(); // every thread has read item
    if (stop)
      break;
    const uint32_t e = B.items[it];
    const unsigned b = e >> 16u;
    if (B.done[b])
      continue;
    const BatchMat &m = B.mats[b];
    pair_step_n<SORT, ACCV>(m.p, B.kstep[b] % m.steps1, e & 0xffffu, sm);
    __syncthreads();
    if (threadIdx.x == 0u)
      for (unsigned k = 0u; k < 5u; ++k)
        mbar_inval(&bars[k]);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Two block pairs on a CTA of 4 warps (batched form, two such CTAs per SM:
// four pairs in flight per SM).  Pair A of matrix PA, pair B of matrix PB:
// their Grams (gram_tile2 on warps 0-2, copies by warp 3) and updates (warp w
// takes row groups w and w + 4 of every stage) run on the 4 warps, A's then
// B's, as one stream of tiles and one of stages; their Cholesky
// factorisations and inner sweeps run concurrently, warps 0-1 on A (named
// barrier 1), warps 2-3 on B (barrier 2), with the eighth-warp reduce-scatter
// of inner_sweeps_e.  Every entry gets the operations of pair_step in the
// same order, so each matrix gets the bits of its single call.  Shared
// memory (104 KB): the Gram's 4 stages of one tile, later one update buffer;
// A's and B's R, V_loc and counters.
// ---------------------------------------------------------------------------
constexpr unsigned kN2OffRA = kNRegion;
constexpr unsigned kN2OffVlA = kN2OffRA + 32u * kVTLd;
constexpr unsigned kN2OffRB = kN2OffVlA + 1024u;
constexpr unsigned kN2OffVlB = kN2OffRB + 32u * kVTLd;
constexpr unsigned kN2OffS0 = kN2OffVlB + 1024u;
constexpr unsigned kN2OffRed = kN2OffS0 + 128u; // [0..3] A's counts, [4..7] B's, [8..9] flags
constexpr unsigned kN2OffBar = kN2OffRed + 8u;  // [0..3] Gram stages, [4] the update buffer
constexpr unsigned kN2OffRot = kN2OffBar + 8u; // the rotations of the 4 warps (inner_sweeps_e), 32 doubles each
constexpr unsigned kN2SmemDoubles = kN2OffRot + 128u;
static_assert(2u * (kN2SmemDoubles * sizeof(double) + 1024u) <= 228u * 1024u, "two CTAs per SM");
size_t batchn2_smem_bytes() { return (size_t)kN2SmemDoubles * sizeof(double); }

template <bool SORT, bool ACCV>
__device__ __forceinline__ void pair_step2n(const StepParams &PA, const unsigned stepA, const unsigned pairA,
                                            const StepParams &PB, const unsigned stepB, const unsigned pairB,
                                            double *const sm)
{
  double *const stg = sm;
  uint8_t *const s0 = reinterpret_cast<uint8_t *>(sm + kN2OffS0);
  unsigned *const red = reinterpret_cast<unsigned *>(sm + kN2OffRed);
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kN2OffBar);
  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  size_t pidx = ((size_t)stepA * PA.pairs + pairA) * 2u;
  const unsigned iA = PA.strat1[pidx + 0u], jA = PA.strat1[pidx + 1u];
  pidx = ((size_t)stepB * PB.pairs + pairB) * 2u;
  const unsigned iB = PB.strat1[pidx + 0u], jB = PB.strat1[pidx + 1u];

  for (unsigned i = tid; i < 256u; i += kNThreads)
    reinterpret_cast<uint32_t *>(s0)[i] = reinterpret_cast<const uint32_t *>(PA.strat0)[i];
  if (tid == 0u) {
    for (unsigned b = 0u; b < 5u; ++b)
      mbar_init(&bars[b], 1u);
    mbar_fence_init();
  }
  __syncthreads();

  // ------------------------------ 1. Grams --------------------------------
  // tiles 0 .. ntA-1 are A's, ntA .. ntA+ntB-1 B's
  const unsigned ntA = PA.nrow >> 6, ntB = PB.nrow >> 6, nt = ntA + ntB;
  unsigned gx0 = 0u, gy = 0u, gy1 = 0u;
  const bool gthr = gram_lane2(warp, lane, gx0, gy, gy1);
  double gacc[4][2] = {{+0.0, +0.0}, {+0.0, +0.0}, {+0.0, +0.0}, {+0.0, +0.0}};
  auto issue_gram = [&](const unsigned k) {
    const unsigned s = k % kNGStages;
    const bool a = k < ntA;
    const CUtensorMap *const tm = a ? &PA.tmGram : &PB.tmGram;
    const int tile = (int)(a ? k : (k - ntA));
    double *const st = stg + s * kGramTileLd;
    mbar_arrive_expect_tx(&bars[s], 2u * kGramBoxBytes);
    tma_load_3d(st, tm, 0, tile, (int)((a ? iA : iB) * kNColB), &bars[s]);
    tma_load_3d(st + 16u * kGramColLd, tm, 0, tile, (int)((a ? jA : jB) * kNColB), &bars[s]);
  };
  auto put_gram = [&](double *const R) { // our share of the lower triangle
    if (gthr) {
#pragma unroll
      for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
        for (unsigned v = 0u; v < 2u; ++v) {
          const unsigned y = v ? gy1 : gy;
          if (gx0 + u >= y)
            R[y * 32u + gx0 + u] = gacc[u][v];
          gacc[u][v] = +0.0;
        }
    }
  };
  if (tid == kNIssuer)
    for (unsigned k = 0u; k + 1u < kNGStages && k < nt; ++k)
      issue_gram(k);
  unsigned k = 0u;
  int failed = 0;
  for (; k < nt; ++k) {
    if (tid == kNIssuer && k + kNGStages - 1u < nt)
      issue_gram(k + kNGStages - 1u);
    int fail = 0;
    if (warp < 3u) {
      if (!mbar_wait_bounded(&bars[k % kNGStages], (k / kNGStages) & 1u, kWaitLimit))
        fail = 1;
      else if (gthr)
        gram_tile2(stg + (k % kNGStages) * kGramTileLd, 0u, gx0, gy, gy1, gacc);
      if (k + 1u == ntA)
        put_gram(sm + kN2OffRA);
      else if (k + 1u == nt)
        put_gram(sm + kN2OffRB);
    }
    failed = __syncthreads_or(fail);
    if (failed)
      break;
  }
  if (failed) {
    if (tid == 0u) {
      for (unsigned q = k; q < nt && q < k + kNGStages; ++q)
        (void)mbar_wait_bounded(&bars[q % kNGStages], (q / kNGStages) & 1u, kWaitLimit / 8);
      atomicOr(PA.err, kErrWaitTimeout);
      atomicOr(PB.err, kErrWaitTimeout);
    }
    return;
  }

  // the update stages: A's, then B's; A's first one in flight during the
  // serial phases
  const unsigned nGA = (PA.nrow + kUpdRows - 1u) / kUpdRows, nGB = (PB.nrow + kUpdRows - 1u) / kUpdRows;
  const unsigned nstA = nGA + (ACCV ? (PA.ncol + kUpdRows - 1u) / kUpdRows : 0u);
  const unsigned nstB = nGB + (ACCV ? (PB.ncol + kUpdRows - 1u) / kUpdRows : 0u);
  auto stage_at = [&](const unsigned g, const unsigned i, const CUtensorMap *&tm, int &piece) {
    const StepParams &P = g ? PB : PA;
    const unsigned nG = g ? nGB : nGA;
    const bool isG = i < nG;
    tm = isG ? &P.tmG : &P.tmV;
    piece = (int)(((isG ? i : (i - nG)) * kUpdRows) >> 5);
  };
  auto issue_upd = [&](const unsigned g, const unsigned i) {
    const CUtensorMap *tm;
    int piece;
    stage_at(g, i, tm, piece);
    mbar_arrive_expect_tx(&bars[4], 2u * kUpdBoxBytes);
    tma_load_3d(stg, tm, 0, piece, (int)((g ? iB : iA) * kNColB), &bars[4]);
    tma_load_3d(stg + 16u * kUpdColLd, tm, 0, piece, (int)((g ? jB : jA) * kNColB), &bars[4]);
  };
  if (tid == 0u && nstA > 0u)
    issue_upd(0u, 0u);

  // ------------------- 2.-3. Cholesky and inner sweeps --------------------
  {
    const unsigned grp = warp >> 1, gt = tid & 63u, gw = warp & 1u;
    const StepParams &P = grp ? PB : PA;
    double *const R = sm + (grp ? kN2OffRB : kN2OffRA);
    double *const Vl = sm + (grp ? kN2OffVlB : kN2OffVlA);
    for (unsigned i = gt; i < 1024u; i += 64u)
      Vl[i] = ((i >> 5) == (i & 31u)) ? 1.0 : 0.0;
    chol32_grp<2u>(R, gt, 1u + grp);
    bar_sync(1u + grp, 64u);
    int definite;
    unsigned npos;
    block_signature(P, grp ? iB : iA, grp ? jB : jA, definite, npos);
    unsigned blk_s, blk_b;
    inner_sweeps_e<SORT>(R, Vl, s0, P.s0steps, P.nswp0, definite, npos, red + 4u * grp, lane, gw, 1u + grp, blk_s,
                         blk_b, sm + kN2OffRot + 32u * warp);
    if (gt == 0u) {
      add_counts(P, blk_s, blk_b);
      red[8u + grp] = (SORT || blk_s) ? 1u : 0u;
    }
  }
  __syncthreads();
  const bool updA = red[8] != 0u, updB = red[9] != 0u;
  // the stream of update stages: A's (or, when A is unchanged, its prefetched
  // first stage, waited for and dropped), then B's
  const unsigned qa = updA ? nstA : (nstA > 0u ? 1u : 0u), nq = qa + (updB ? nstB : 0u);
  if (nq == qa && !updA) {
    if (tid == 0u && qa > 0u && !mbar_wait_bounded(&bars[4], 0u, kWaitLimit))
      atomicOr(PA.err, kErrWaitTimeout);
    return;
  }

  // ------------------------------ 4. updates ------------------------------
  for (unsigned i = tid; i < 2048u; i += kNThreads) { // both R are dead: B^T[s][c] = V_loc[s][c]
    const unsigned g = i >> 10, c = (i >> 5) & 31u, s_ = i & 31u;
    (sm + (g ? kN2OffRB : kN2OffRA))[s_ * kVTLd + c] = E32(sm + (g ? kN2OffVlB : kN2OffVlA), s_, c);
  }
  __syncthreads();
  const unsigned sub = lane & 7u, cg8 = lane >> 3;
  for (unsigned q = 0u; q < nq; ++q) {
    const unsigned g = (q < qa) ? 0u : 1u, i = g ? q - qa : q;
    if (tid == 0u && q > 0u) {
      bulk_wait_read(); // the store of stage q - 1 has read the buffer out
      issue_upd(g, i);
    }
    const int fail = !__all_sync(0xffffffffu, mbar_wait_bounded(&bars[4], q & 1u, kWaitLimit));
    const bool work = g == 1u || updA;
    if (!fail && work) {
#pragma unroll 1
      for (unsigned h = 0u; h < 2u; ++h) { // row groups warp and warp + 4
        double acc[4][8];
        update_stage(stg, sm + (g ? kN2OffRB : kN2OffRA), warp + 4u * h, sub, cg8, acc);
        __syncwarp();
        update_put(stg, acc, warp + 4u * h, sub, cg8);
      }
      fence_async_shared();
    }
    if (__syncthreads_or(fail)) {
      if (tid == 0u) {
        (void)mbar_wait_bounded(&bars[4], q & 1u, kWaitLimit / 8);
        bulk_wait_all();
        atomicOr(g ? PB.err : PA.err, kErrWaitTimeout);
      }
      return;
    }
    if (tid == 0u && work) {
      const CUtensorMap *tm;
      int piece;
      stage_at(g, i, tm, piece);
      tma_store_3d(tm, stg, 0, piece, (int)((g ? iB : iA) * kNColB));
      tma_store_3d(tm, stg + 16u * kUpdColLd, 0, piece, (int)((g ? jB : jA) * kNColB));
      bulk_commit();
    }
  }
  if (tid == 0u)
    bulk_wait_all();
}

// The batched step on CTAs of 4 warps, two per SM, two block pairs per CTA
// at a time (items taken in twos from the queue, as l1_batch_kernel with W =
// 2): two live pairs with the same inner table through pair_step2n, a lone
// one through pair_step_n.  The mbarriers are invalidated after each item.
template <bool SORT, bool ACCV>
__global__ void __launch_bounds__(kNThreads, 2) l1_batchn2_kernel(const __grid_constant__ BatchStep B)
{
  extern __shared__ __align__(128) double sm[];
  __shared__ unsigned item;
  auto inval = [&](uint64_t *const bars) {
    __syncthreads();
    if (threadIdx.x == 0u)
      for (unsigned k = 0u; k < 5u; ++k)
        mbar_inval(&bars[k]);
    __syncthreads();
  };
  for (;;) {
    if (threadIdx.x == 0u)
      item = atomicAdd(B.queue, 2u);
    __syncthreads();
    const unsigned it = item;
    const bool stop = (it >= B.nitems) || (*(volatile int *)B.err != 0);
    __syncthreads(); // every thread has read item
    if (stop)
      break;
    const uint32_t e0 = B.items[it];
    const bool live0 = !B.done[e0 >> 16u];
    uint32_t e1 = 0u;
    bool live1 = false;
    if (it + 1u < B.nitems) {
      e1 = B.items[it + 1u];
      live1 = !B.done[e1 >> 16u];
    }
    if (live0 && live1 && B.mats[e0 >> 16u].p.strat0 == B.mats[e1 >> 16u].p.strat0) {
      const BatchMat &ma = B.mats[e0 >> 16u], &mb = B.mats[e1 >> 16u];
      pair_step2n<SORT, ACCV>(ma.p, B.kstep[e0 >> 16u] % ma.steps1, e0 & 0xffffu, mb.p,
                              B.kstep[e1 >> 16u] % mb.steps1, e1 & 0xffffu, sm);
      inval(reinterpret_cast<uint64_t *>(sm + kN2OffBar));
      continue;
    }
    for (unsigned h = 0u; h < 2u; ++h) {
      if (!(h ? live1 : live0))
        continue;
      const uint32_t e = h ? e1 : e0;
      const BatchMat &m = B.mats[e >> 16u];
      pair_step_n<SORT, ACCV>(m.p, B.kstep[e >> 16u] % m.steps1, e & 0xffffu, sm);
      inval(reinterpret_cast<uint64_t *>(sm + kNOffBar));
    }
  }
}

// One launch per sweep of the whole batch (the dataflow form): the CTAs take
// (matrix, step, pair) items in queue order -- step-major, every matrix's
// step s before any step s + 1 -- and an item waits until both of its blocks
// have been written by its matrix's step s - 1 (per-block counts of the
// sweep, release / acquire, bounded waits).  Steps of different matrices, and
// the pairs of consecutive steps of one matrix whose blocks are ready,
// overlap.  An item waits only on items taken earlier, by running CTAs, so
// the launch needs no co-residency.  Two items go through pair_step2 when
// neither can depend on the other (different matrices, or the same step).
template <bool SORT, bool ACCV, unsigned W>
__global__ void __launch_bounds__(kThreads, 1) l1_batch_flow_kernel(const __grid_constant__ BatchFlow B)
{
  extern __shared__ __align__(128) double sm[];
  __shared__ unsigned item, ok;
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kOffBar);
  const unsigned tid = threadIdx.x;
  // thread 0: wait until item h's blocks are written by its previous step
  auto ready = [&](const uint32_t e, const unsigned stp) -> bool {
    const unsigned b = e >> 16u, q = e & 0xffffu;
    const BatchMat &m = B.mats[b];
    const size_t pidx = ((size_t)stp * m.p.pairs + q) * 2u;
    const unsigned *const v = B.ver + B.vofs[b];
    const unsigned iB = m.p.strat1[pidx], jB = m.p.strat1[pidx + 1u];
    const long long t0 = clock64();
    while (ld_acquire(v + iB) < stp || ld_acquire(v + jB) < stp) {
      if (*(volatile int *)B.err)
        return false;
      if (clock64() - t0 > kWaitLimit) {
        atomicOr(B.err, kErrWaitTimeout);
        return false;
      }
      __nanosleep(64);
    }
    return true;
  };
  auto written = [&](const uint32_t e, const unsigned stp) { // thread 0, after the pair's stores completed
    const unsigned b = e >> 16u, q = e & 0xffffu;
    const BatchMat &m = B.mats[b];
    const size_t pidx = ((size_t)stp * m.p.pairs + q) * 2u;
    unsigned *const v = B.ver + B.vofs[b];
    __threadfence();
    atomicAdd(v + m.p.strat1[pidx], 1u);
    atomicAdd(v + m.p.strat1[pidx + 1u], 1u);
  };
  auto inval = [&]() {
    __syncthreads();
    if (tid == 0u)
      for (unsigned k = 0u; k < 8u; ++k)
        mbar_inval(&bars[k]);
    __syncthreads();
  };
  for (;;) {
    if (tid == 0u)
      item = atomicAdd(B.queue, W);
    __syncthreads();
    const unsigned it = item;
    const bool stop = (it >= B.nitems) || (*(volatile int *)B.err != 0);
    __syncthreads();
    if (stop)
      break;
    uint32_t e[2] = {B.items[it], 0u};
    unsigned st[2] = {B.isteps[it], 0u};
    bool live[2] = {!B.done[e[0] >> 16u], false};
    if (W == 2u && it + 1u < B.nitems) {
      e[1] = B.items[it + 1u];
      st[1] = B.isteps[it + 1u];
      live[1] = !B.done[e[1] >> 16u];
    }
    const unsigned b0 = e[0] >> 16u, b1 = e[1] >> 16u;
    const bool both = live[0] && live[1] && (b0 != b1 || st[0] == st[1]) &&
                      B.mats[b0].p.strat0 == B.mats[b1].p.strat0;
    if (both) {
      if (tid == 0u)
        ok = ready(e[0], st[0]) && ready(e[1], st[1]);
      __syncthreads();
      if (!ok)
        break;
      asm volatile("fence.proxy.async;" ::: "memory"); // the copies below read what other SMs wrote
      const BatchMat &ma = B.mats[b0], &mb = B.mats[b1];
      pair_step2<SORT, ACCV>(ma.p, st[0], e[0] & 0xffffu, mb.p, st[1], e[1] & 0xffffu, sm);
      __threadfence();
      __syncthreads();
      if (tid == 0u) {
        written(e[0], st[0]);
        written(e[1], st[1]);
      }
      inval();
      continue;
    }
    bool go = true;
    for (unsigned h = 0u; h < 2u && go; ++h) {
      if (!live[h])
        continue;
      if (tid == 0u)
        ok = ready(e[h], st[h]);
      __syncthreads();
      if (!ok) {
        go = false;
        break;
      }
      asm volatile("fence.proxy.async;" ::: "memory");
      const BatchMat &m = B.mats[e[h] >> 16u];
      pair_step<SORT, ACCV, 1u>(m.p, st[h], e[h] & 0xffffu, 0u, sm);
      __threadfence();
      __syncthreads();
      if (tid == 0u)
        written(e[h], st[h]);
      inval();
    }
    if (!go)
      break;
  }
}

// The dataflow form on CTAs of 4 warps, two per SM: one item at a time, the
// same queue, readiness waits and write counts as l1_batch_flow_kernel.
template <bool SORT, bool ACCV>
__global__ void __launch_bounds__(kNThreads, 2) l1_batchn_flow_kernel(const __grid_constant__ BatchFlow B)
{
  extern __shared__ __align__(128) double sm[];
  __shared__ unsigned item, ok;
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kNOffBar);
  const unsigned tid = threadIdx.x;
  for (;;) {
    if (tid == 0u)
      item = atomicAdd(B.queue, 1u);
    __syncthreads();
    const unsigned it = item;
    const bool stop = (it >= B.nitems) || (*(volatile int *)B.err != 0);
    __syncthreads();
    if (stop)
      break;
    const uint32_t e = B.items[it];
    const unsigned stp = B.isteps[it], b = e >> 16u, q = e & 0xffffu;
    if (B.done[b])
      continue;
    const BatchMat &m = B.mats[b];
    const size_t pidx = ((size_t)stp * m.p.pairs + q) * 2u;
    unsigned *const v = B.ver + B.vofs[b];
    const unsigned iB = m.p.strat1[pidx], jB = m.p.strat1[pidx + 1u];
    if (tid == 0u) { // both blocks written by the matrix's previous step (bounded)
      ok = 1u;
      const long long t0 = clock64();
      while (ld_acquire(v + iB) < stp || ld_acquire(v + jB) < stp) {
        if (*(volatile int *)B.err) {
          ok = 0u;
          break;
        }
        if (clock64() - t0 > kWaitLimit) {
          atomicOr(B.err, kErrWaitTimeout);
          ok = 0u;
          break;
        }
        __nanosleep(64);
      }
    }
    __syncthreads();
    if (!ok)
      break;
    asm volatile("fence.proxy.async;" ::: "memory"); // the copies below read what other SMs wrote
    pair_step_n<SORT, ACCV>(m.p, stp, q, sm);
    __threadfence();
    __syncthreads();
    if (tid == 0u) {
      __threadfence();
      atomicAdd(v + iB, 1u);
      atomicAdd(v + jB, 1u);
      for (unsigned k = 0u; k < 5u; ++k)
        mbar_inval(&bars[k]);
    }
    __syncthreads();
  }
}

// The dataflow form on CTAs of 4 warps, two per SM, two items at a time:
// two independent items (different matrices, or the same step, and the same
// inner table) through pair_step2n, else one after the other through
// pair_step_n; the readiness waits and write counts of l1_batch_flow_kernel.
template <bool SORT, bool ACCV>
__global__ void __launch_bounds__(kNThreads, 2) l1_batchn2_flow_kernel(const __grid_constant__ BatchFlow B)
{
  extern __shared__ __align__(128) double sm[];
  __shared__ unsigned item, ok;
  const unsigned tid = threadIdx.x;
  auto blocks = [&](const uint32_t e, const unsigned stp, unsigned &iB, unsigned &jB) {
    const BatchMat &m = B.mats[e >> 16u];
    const size_t pidx = ((size_t)stp * m.p.pairs + (e & 0xffffu)) * 2u;
    iB = m.p.strat1[pidx];
    jB = m.p.strat1[pidx + 1u];
  };
  // thread 0: both blocks of the item written by its matrix's previous step (bounded)
  auto ready = [&](const uint32_t e, const unsigned stp) -> bool {
    unsigned iB, jB;
    blocks(e, stp, iB, jB);
    const unsigned *const v = B.ver + B.vofs[e >> 16u];
    const long long t0 = clock64();
    while (ld_acquire(v + iB) < stp || ld_acquire(v + jB) < stp) {
      if (*(volatile int *)B.err)
        return false;
      if (clock64() - t0 > kWaitLimit) {
        atomicOr(B.err, kErrWaitTimeout);
        return false;
      }
      __nanosleep(64);
    }
    return true;
  };
  auto written = [&](const uint32_t e, const unsigned stp) { // thread 0, after the pair's stores completed
    unsigned iB, jB;
    blocks(e, stp, iB, jB);
    unsigned *const v = B.ver + B.vofs[e >> 16u];
    __threadfence();
    atomicAdd(v + iB, 1u);
    atomicAdd(v + jB, 1u);
  };
  auto inval = [&](uint64_t *const bars) {
    __syncthreads();
    if (tid == 0u)
      for (unsigned k = 0u; k < 5u; ++k)
        mbar_inval(&bars[k]);
    __syncthreads();
  };
  for (;;) {
    if (tid == 0u)
      item = atomicAdd(B.queue, 2u);
    __syncthreads();
    const unsigned it = item;
    const bool stop = (it >= B.nitems) || (*(volatile int *)B.err != 0);
    __syncthreads();
    if (stop)
      break;
    uint32_t e[2] = {B.items[it], 0u};
    unsigned st[2] = {B.isteps[it], 0u};
    bool live[2] = {!B.done[e[0] >> 16u], false};
    if (it + 1u < B.nitems) {
      e[1] = B.items[it + 1u];
      st[1] = B.isteps[it + 1u];
      live[1] = !B.done[e[1] >> 16u];
    }
    const unsigned b0 = e[0] >> 16u, b1 = e[1] >> 16u;
    const bool both = live[0] && live[1] && (b0 != b1 || st[0] == st[1]) &&
                      B.mats[b0].p.strat0 == B.mats[b1].p.strat0;
    if (both) {
      if (tid == 0u)
        ok = ready(e[0], st[0]) && ready(e[1], st[1]);
      __syncthreads();
      if (!ok)
        break;
      asm volatile("fence.proxy.async;" ::: "memory"); // the copies below read what other SMs wrote
      const BatchMat &ma = B.mats[b0], &mb = B.mats[b1];
      pair_step2n<SORT, ACCV>(ma.p, st[0], e[0] & 0xffffu, mb.p, st[1], e[1] & 0xffffu, sm);
      __threadfence();
      __syncthreads();
      if (tid == 0u) {
        written(e[0], st[0]);
        written(e[1], st[1]);
      }
      inval(reinterpret_cast<uint64_t *>(sm + kN2OffBar));
      continue;
    }
    bool go = true;
    for (unsigned h = 0u; h < 2u && go; ++h) {
      if (!live[h])
        continue;
      if (tid == 0u)
        ok = ready(e[h], st[h]);
      __syncthreads();
      if (!ok) {
        go = false;
        break;
      }
      asm volatile("fence.proxy.async;" ::: "memory");
      const BatchMat &m = B.mats[e[h] >> 16u];
      pair_step_n<SORT, ACCV>(m.p, st[h], e[h] & 0xffffu, sm);
      __threadfence();
      __syncthreads();
      if (tid == 0u)
        written(e[h], st[h]);
      inval(reinterpret_cast<uint64_t *>(sm + kNOffBar));
    }
    if (!go)
      break;
  }
}

// after a sweep of the dataflow form: per matrix still sweeping, the sweep's
// counter folded into its totals and the convergence test (no big rotation,
// or the sweep cap); its block counts and the queue cleared for the next
__global__ void batch_flow_end_kernel(const BatchSweep S, unsigned *const ver, const unsigned *const vofs)
{
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0u)
    S.queue[0] = 0u;
  if (i >= S.nmat || S.done[i])
    return;
  const unsigned n1 = S.mats[i].p.pairs * 2u;
  for (unsigned k = 0u; k < n1; ++k)
    ver[vofs[i] + k] = 0u;
  const unsigned long long c = S.cvg[i];
  S.cvg[i] = 0ull;
  const unsigned small = (unsigned)c, big = (unsigned)(c >> 32u);
  S.glb_s[i] += small;
  S.glb_b[i] += big;
  const unsigned sw = ++S.sweeps[i];
  if (!big || sw >= kNSweep)
    S.done[i] = 1u;
  else
    atomicAdd(S.active, 1u);
}

// after a launch of the batch: one step more for every active matrix; at the
// end of its sweep, its totals and the convergence test (no big rotation in
// the sweep, or the sweep cap); the work queue cleared for the next launch
__global__ void batch_sweep_end_kernel(const BatchSweep S)
{
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0u)
    S.queue[0] = 0u;
  if (i >= S.nmat || S.done[i])
    return;
  const unsigned k = ++S.kstep[i];
  if (k % S.mats[i].steps1) { // the sweep goes on
    atomicAdd(S.active, 1u);
    return;
  }
  const unsigned long long c = S.cvg[i];
  S.cvg[i] = 0ull;
  const unsigned small = (unsigned)c, big = (unsigned)(c >> 32u);
  S.glb_s[i] += small;
  S.glb_b[i] += big;
  const unsigned sw = ++S.sweeps[i];
  if (!big || sw >= kNSweep)
    S.done[i] = 1u;
  else
    atomicAdd(S.active, 1u);
}

// ---------------------------------------------------------------------------
// U = G diag(1/||g_c||), D_c = +-||g_c||^2 (share/device_code_common.hpp:187-219)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) initD_kernel(double *const G, double *const D, const unsigned nrow,
                                                    const unsigned ncol, const unsigned nplus, const unsigned ldG)
{
  const unsigned c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const unsigned l = threadIdx.x & 31u;
  if (c >= ncol)
    return;
  double *const g = G + (size_t)c * ldG;
  double x = +0.0;
  for (unsigned r = l; r < nrow; r += 32u) {
    const double y = g[r];
    x = __fma_rn(y, y, x);
  }
  const double y = sum32(x);
  const double nrm = __dsqrt_rn(y);
  for (unsigned r = l; r < nrow; r += 32u)
    g[r] = __ddiv_rn(g[r], nrm);
  if (!l)
    D[c] = (c < nplus) ? y : -y;
}

__global__ void initV_kernel(double *const V, const unsigned ncol, const unsigned ldV)
{
  const size_t n = (size_t)ncol * ncol;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const unsigned c = (unsigned)(i / ncol), r = (unsigned)(i % ncol);
    V[(size_t)c * ldV + r] = (r == c) ? 1.0 : 0.0;
  }
}

// initD for a batch: block b normalises the columns of matrix b, one warp
// per column, the same arithmetic as initD_kernel
__global__ void __launch_bounds__(256) initD_batch_kernel(const BatchMat *const M, const unsigned nmat,
                                                          const uint32_t *const done_ok)
{
  const BatchMat &m = M[blockIdx.x];
  if (blockIdx.x >= nmat || !done_ok[blockIdx.x])
    return;
  const unsigned l = threadIdx.x & 31u;
  for (unsigned c = threadIdx.x >> 5; c < m.p.ncol; c += blockDim.x >> 5) {
    double *const g = m.p.G + (size_t)c * m.p.ldG;
    double x = +0.0;
    for (unsigned r = l; r < m.p.nrow; r += 32u) {
      const double y = g[r];
      x = __fma_rn(y, y, x);
    }
    const double y = sum32(x);
    const double nrm = __dsqrt_rn(y);
    for (unsigned r = l; r < m.p.nrow; r += 32u)
      g[r] = __ddiv_rn(g[r], nrm);
    if (!l)
      m.D[c] = (c < m.p.nplus) ? y : -y;
  }
}

__global__ void initV_batch_kernel(const BatchMat *const M, const unsigned nmat)
{
  for (unsigned b = blockIdx.y; b < nmat; b += gridDim.y) {
    const BatchMat &m = M[b];
    if (!m.p.V)
      continue;
    const size_t n = (size_t)m.p.ncol * m.p.ncol;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
      const unsigned c = (unsigned)(i / m.p.ncol), r = (unsigned)(i % m.p.ncol);
      m.p.V[(size_t)c * m.p.ldV + r] = (r == c) ? 1.0 : 0.0;
    }
  }
}

// The failure path of the bounded waits, exercised on purpose: each CTA
// waits on an mbarrier that expects one arrival nobody makes, with the given
// cycle limit, records whether the wait gave up and in how many cycles, and
// invalidates the barrier.  Nothing faults or hangs; the context stays usable.
__global__ void wait_selftest_kernel(const long long limit, int *const timed_out, long long *const cycles)
{
  __shared__ uint64_t bar;
  if (threadIdx.x == 0u) {
    mbar_init(&bar, 1u);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0u) {
    const long long t0 = clock64();
    const bool ok = mbar_wait_bounded(&bar, 0u, limit);
    cycles[blockIdx.x] = clock64() - t0;
    if (!ok)
      atomicAdd(timed_out, 1);
    mbar_inval(&bar);
  }
}

// uniform values in (-1, 1) from a counter hash (splitmix64), for the
// autotuner's timed runs
__global__ void fill_random_kernel(double *const a, const size_t n, const unsigned long long seed)
{
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9e3779b97f4a7c15ull * (i + 1u);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    a[i] = (double)(long long)(z >> 11) * 0x1.0p-52 - 1.0;
  }
}

__global__ void rsqrt_test_kernel(const double *const in, double *const out, const unsigned n)
{
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    out[i] = rsqrt_rn(in[i]);
}

// ---------------------------------------------------------------------------
// launchers and tensor maps
// ---------------------------------------------------------------------------
cudaError_t make_update_map(CUtensorMap *tm, const double *base, const unsigned nrow, const unsigned ncol,
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
  // (rows within a 32-row piece, pieces, columns); box {34, 8, 16}
  const cuuint64_t dims[3] = {32u, nrow / 32u, ncol};
  const cuuint64_t strides[2] = {32u * sizeof(double), (cuuint64_t)ld * sizeof(double)};
  const cuuint32_t box[3] = {34u, 8u, 16u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3u, const_cast<double *>(base), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (r == CUDA_SUCCESS) ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t make_gram_map(CUtensorMap *tm, const double *base, const unsigned nrow, const unsigned ncol,
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
  // (rows within a 64-row tile, tiles, columns); box {66, 1, 16}
  const cuuint64_t dims[3] = {64u, nrow / 64u, ncol};
  const cuuint64_t strides[2] = {64u * sizeof(double), (cuuint64_t)ld * sizeof(double)};
  const cuuint32_t box[3] = {66u, 1u, 16u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r = encode(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3u, const_cast<double *>(base), dims, strides, box,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return (r == CUDA_SUCCESS) ? cudaSuccess : cudaErrorInvalidValue;
}

template <bool S, bool A, unsigned N> static cudaError_t set_smem(const int bytes)
{
  return cudaFuncSetAttribute(l1_step_kernel<S, A, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <bool S, bool A> static cudaError_t set_smem2()
{
  return cudaFuncSetAttribute(l1_step2_kernel<S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)batch2_smem_bytes());
}

template <bool S, bool A, unsigned F> static cudaError_t set_smem_var(const int bytes)
{
  return cudaFuncSetAttribute(l1_var_kernel<S, A, F>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t l1_configure()
{
  const int b = (int)l1_smem_bytes();
  cudaError_t e;
  if ((e = set_smem_var<false, false, 1u>(b)) || (e = set_smem_var<false, true, 1u>(b)) ||
      (e = set_smem_var<true, false, 1u>(b)) || (e = set_smem_var<true, true, 1u>(b)) ||
      (e = set_smem_var<false, false, 2u>(b)) || (e = set_smem_var<false, true, 2u>(b)) ||
      (e = set_smem_var<true, false, 2u>(b)) || (e = set_smem_var<true, true, 2u>(b)))
    return e;
  if ((e = set_smem2<false, false>()) || (e = set_smem2<false, true>()) || (e = set_smem2<true, false>()) ||
      (e = set_smem2<true, true>()))
    return e;
  const int b3 = (int)step_smem_bytes(2u);
  if ((e = set_smem<false, false, 1u>(b)) || (e = set_smem<false, true, 1u>(b)) || (e = set_smem<true, false, 1u>(b)) ||
      (e = set_smem<true, true, 1u>(b)) || (e = set_smem<false, false, 2u>(b3)) || (e = set_smem<false, true, 2u>(b3)) ||
      (e = set_smem<true, false, 2u>(b3)) || (e = set_smem<true, true, 2u>(b3)) ||
      (e = set_smem<false, false, 4u>(b3)) || (e = set_smem<false, true, 4u>(b3)) ||
      (e = set_smem<true, false, 4u>(b3)) || (e = set_smem<true, true, 4u>(b3)))
    return e;
  return cudaSuccess;
}

template <bool S, bool A, unsigned N> static cudaError_t launch(const StepParams &p, cudaStream_t s)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(p.pairs * N);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = step_smem_bytes(N);
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = N;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, l1_step_kernel<S, A, N>, p);
}

template <bool S, bool A> static cudaError_t set_smem_batch()
{
  cudaError_t e = cudaFuncSetAttribute(l1_batch_kernel<S, A, 1u>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)l1_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(l1_batch_kernel<S, A, 2u>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)batch2_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(l1_batchn_kernel<S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)batchn_smem_bytes());
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(l1_batchn2_kernel<S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)batchn2_smem_bytes());
  return e;
}

cudaError_t batch_configure()
{
  cudaError_t e;
  if ((e = set_smem_batch<false, false>()) || (e = set_smem_batch<false, true>()) ||
      (e = set_smem_batch<true, false>()) || (e = set_smem_batch<true, true>()))
    return e;
  return cudaSuccess;
}

template <bool S, bool A>
static void batch_launch(const unsigned width, const BatchStep &b, const unsigned ctas, cudaStream_t s)
{
  if (width == kWidthHalf)
    l1_batchn_kernel<S, A><<<ctas, kNThreads, batchn_smem_bytes(), s>>>(b);
  else if (width == kWidthHalf2)
    l1_batchn2_kernel<S, A><<<ctas, kNThreads, batchn2_smem_bytes(), s>>>(b);
  else if (width == 2u)
    l1_batch_kernel<S, A, 2u><<<ctas, kThreads, batch2_smem_bytes(), s>>>(b);
  else
    l1_batch_kernel<S, A, 1u><<<ctas, kThreads, l1_smem_bytes(), s>>>(b);
}

cudaError_t launch_batch_step(const bool sort, const bool accv, const unsigned width, const BatchStep &b,
                              const unsigned ctas, cudaStream_t s)
{
  if (sort) {
    if (accv)
      batch_launch<true, true>(width, b, ctas, s);
    else
      batch_launch<true, false>(width, b, ctas, s);
  }
  else if (accv)
    batch_launch<false, true>(width, b, ctas, s);
  else
    batch_launch<false, false>(width, b, ctas, s);
  return cudaGetLastError();
}

template <bool S, bool A> static cudaError_t set_smem_flow()
{
  cudaError_t e = cudaFuncSetAttribute(l1_batch_flow_kernel<S, A, 1u>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)l1_smem_bytes());
  if (e != cudaSuccess)
    return e;
  e = cudaFuncSetAttribute(l1_batch_flow_kernel<S, A, 2u>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)batch2_smem_bytes());
  if (e != cudaSuccess)
    return e;
  e = cudaFuncSetAttribute(l1_batchn_flow_kernel<S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)batchn_smem_bytes());
  if (e != cudaSuccess)
    return e;
  return cudaFuncSetAttribute(l1_batchn2_flow_kernel<S, A>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)batchn2_smem_bytes());
}

cudaError_t flow_configure()
{
  cudaError_t e;
  if ((e = set_smem_flow<false, false>()) || (e = set_smem_flow<false, true>()) || (e = set_smem_flow<true, false>()) ||
      (e = set_smem_flow<true, true>()))
    return e;
  return cudaSuccess;
}

template <bool S, bool A>
static void flow_launch(const unsigned width, const BatchFlow &b, const unsigned ctas, cudaStream_t s)
{
  if (width == kWidthHalf)
    l1_batchn_flow_kernel<S, A><<<ctas, kNThreads, batchn_smem_bytes(), s>>>(b);
  else if (width == kWidthHalf2)
    l1_batchn2_flow_kernel<S, A><<<ctas, kNThreads, batchn2_smem_bytes(), s>>>(b);
  else if (width == 2u)
    l1_batch_flow_kernel<S, A, 2u><<<ctas, kThreads, batch2_smem_bytes(), s>>>(b);
  else
    l1_batch_flow_kernel<S, A, 1u><<<ctas, kThreads, l1_smem_bytes(), s>>>(b);
}

cudaError_t launch_batch_flow(const bool sort, const bool accv, const unsigned width, const BatchFlow &b,
                              const unsigned ctas, cudaStream_t s)
{
  if (sort) {
    if (accv)
      flow_launch<true, true>(width, b, ctas, s);
    else
      flow_launch<true, false>(width, b, ctas, s);
  }
  else if (accv)
    flow_launch<false, true>(width, b, ctas, s);
  else
    flow_launch<false, false>(width, b, ctas, s);
  return cudaGetLastError();
}

cudaError_t launch_batch_flow_end(const BatchSweep &w, unsigned *ver, const unsigned *vofs, cudaStream_t s)
{
  batch_flow_end_kernel<<<(w.nmat + 255u) / 256u, 256u, 0, s>>>(w, ver, vofs);
  return cudaGetLastError();
}

cudaError_t launch_batch_sweep_end(const BatchSweep &w, cudaStream_t s)
{
  batch_sweep_end_kernel<<<(w.nmat + 255u) / 256u, 256u, 0, s>>>(w);
  return cudaGetLastError();
}

cudaError_t launch_batch_initV(const BatchMat *m, unsigned nmat, cudaStream_t s)
{
  initV_batch_kernel<<<dim3(8u, nmat < 4096u ? nmat : 4096u), 256u, 0, s>>>(m, nmat);
  return cudaGetLastError();
}

cudaError_t launch_batch_initD(const BatchMat *m, unsigned nmat, const uint32_t *ok, cudaStream_t s)
{
  initD_batch_kernel<<<nmat, 256u, 0, s>>>(m, nmat, ok);
  return cudaGetLastError();
}

template <bool S, bool A, unsigned N> static cudaLaunchConfig_t sweep_cfg(const StepParams &p, cudaStream_t s,
                                                                         cudaLaunchAttribute *at)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(p.pairs * N);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = step_smem_bytes(N);
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = N;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeCooperative;
  at[1].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 2;
  return cfg;
}

template <bool S, bool A, unsigned N> static bool sweep_fits(const StepParams &p)
{
  if (cudaFuncSetAttribute(l1_sweep_kernel<S, A, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)step_smem_bytes(N)) != cudaSuccess)
    return false;
  cudaLaunchAttribute at[2];
  cudaLaunchConfig_t cfg = sweep_cfg<S, A, N>(p, nullptr, at);
  cfg.numAttrs = 1; // the occupancy query takes the cluster shape
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, l1_sweep_kernel<S, A, N>, &cfg) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return (unsigned)clusters >= p.pairs;
}

template <bool S, bool A, unsigned N> static cudaError_t sweep_launch(const StepParams &p, cudaStream_t s)
{
  cudaLaunchAttribute at[2];
  cudaLaunchConfig_t cfg = sweep_cfg<S, A, N>(p, s, at);
  return cudaLaunchKernelEx(&cfg, l1_sweep_kernel<S, A, N>, p);
}

bool sweep_kernel_fits(const bool sort, const bool accv, const StepParams &p)
{
  if (p.split == 4u) {
    if (sort)
      return accv ? sweep_fits<true, true, 4u>(p) : sweep_fits<true, false, 4u>(p);
    return accv ? sweep_fits<false, true, 4u>(p) : sweep_fits<false, false, 4u>(p);
  }
  if (p.split == 2u) {
    if (sort)
      return accv ? sweep_fits<true, true, 2u>(p) : sweep_fits<true, false, 2u>(p);
    return accv ? sweep_fits<false, true, 2u>(p) : sweep_fits<false, false, 2u>(p);
  }
  if (sort)
    return accv ? sweep_fits<true, true, 1u>(p) : sweep_fits<true, false, 1u>(p);
  return accv ? sweep_fits<false, true, 1u>(p) : sweep_fits<false, false, 1u>(p);
}

cudaError_t launch_l1_sweep(const bool sort, const bool accv, const StepParams &p, cudaStream_t s)
{
  if (p.split == 4u) {
    if (sort)
      return accv ? sweep_launch<true, true, 4u>(p, s) : sweep_launch<true, false, 4u>(p, s);
    return accv ? sweep_launch<false, true, 4u>(p, s) : sweep_launch<false, false, 4u>(p, s);
  }
  if (p.split == 2u) {
    if (sort)
      return accv ? sweep_launch<true, true, 2u>(p, s) : sweep_launch<true, false, 2u>(p, s);
    return accv ? sweep_launch<false, true, 2u>(p, s) : sweep_launch<false, false, 2u>(p, s);
  }
  if (sort)
    return accv ? sweep_launch<true, true, 1u>(p, s) : sweep_launch<true, false, 1u>(p, s);
  return accv ? sweep_launch<false, true, 1u>(p, s) : sweep_launch<false, false, 1u>(p, s);
}

unsigned l1_split(const unsigned pairs)
{
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    (void)cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return (4u * pairs <= (unsigned)sms) ? 4u : (2u * pairs <= (unsigned)sms) ? 2u : 1u;
}

template <bool S, bool A> static cudaError_t launch2(const StepParams &p, cudaStream_t s)
{
  l1_step2_kernel<S, A><<<(p.pairs + 1u) / 2u, kThreads, batch2_smem_bytes(), s>>>(p);
  return cudaGetLastError();
}

template <bool S, bool A, unsigned F> static cudaError_t launch_var(const StepParams &p, cudaStream_t s)
{
  l1_var_kernel<S, A, F><<<p.pairs, kThreads, l1_smem_bytes(), s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_l1_step(const bool sort, const bool accv, const StepParams &p, cudaStream_t s)
{
  if (p.variant == 1u) {
    if (sort)
      return accv ? launch_var<true, true, 1u>(p, s) : launch_var<true, false, 1u>(p, s);
    return accv ? launch_var<false, true, 1u>(p, s) : launch_var<false, false, 1u>(p, s);
  }
  if (p.variant == 2u) {
    if (sort)
      return accv ? launch_var<true, true, 2u>(p, s) : launch_var<true, false, 2u>(p, s);
    return accv ? launch_var<false, true, 2u>(p, s) : launch_var<false, false, 2u>(p, s);
  }
  const unsigned n = p.split;
  if (n == 1u && p.width == 2u) {
    if (sort)
      return accv ? launch2<true, true>(p, s) : launch2<true, false>(p, s);
    return accv ? launch2<false, true>(p, s) : launch2<false, false>(p, s);
  }
  if (n == 4u) {
    if (sort)
      return accv ? launch<true, true, 4u>(p, s) : launch<true, false, 4u>(p, s);
    return accv ? launch<false, true, 4u>(p, s) : launch<false, false, 4u>(p, s);
  }
  if (n == 2u) {
    if (sort)
      return accv ? launch<true, true, 2u>(p, s) : launch<true, false, 2u>(p, s);
    return accv ? launch<false, true, 2u>(p, s) : launch<false, false, 2u>(p, s);
  }
  if (sort)
    return accv ? launch<true, true, 1u>(p, s) : launch<true, false, 1u>(p, s);
  return accv ? launch<false, true, 1u>(p, s) : launch<false, false, 1u>(p, s);
}

cudaError_t launch_initD(double *G, double *D, unsigned nrow, unsigned ncol, unsigned nplus, unsigned ldG,
                         cudaStream_t s)
{
  const unsigned wpb = 8u;
  initD_kernel<<<(ncol + wpb - 1u) / wpb, 32u * wpb, 0, s>>>(G, D, nrow, ncol, nplus, ldG);
  return cudaGetLastError();
}

cudaError_t launch_initV(double *V, unsigned ncol, unsigned ldV, cudaStream_t s)
{
  const size_t n = (size_t)ncol * ncol;
  unsigned blocks = (unsigned)((n + 255u) / 256u);
  if (blocks > 4096u)
    blocks = 4096u;
  initV_kernel<<<blocks, 256u, 0, s>>>(V, ncol, ldV);
  return cudaGetLastError();
}

cudaError_t launch_wait_selftest(long long limit, int *timed_out, long long *cycles, unsigned ctas, cudaStream_t s)
{
  wait_selftest_kernel<<<ctas, 32u, 0, s>>>(limit, timed_out, cycles);
  return cudaGetLastError();
}

cudaError_t launch_fill_random(double *a, size_t n, unsigned long long seed, cudaStream_t s)
{
  fill_random_kernel<<<1024u, 256u, 0, s>>>(a, n, seed);
  return cudaGetLastError();
}

cudaError_t launch_rsqrt_test(const double *in, double *out, unsigned n, cudaStream_t s)
{
  rsqrt_test_kernel<<<(n + 255u) / 256u, 256u, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

} // namespace gjx
