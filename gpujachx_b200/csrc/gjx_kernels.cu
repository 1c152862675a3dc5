// gjx_kernels.cu -- sm_100a kernels of the blocked one-sided Jacobi (H)SVD.
//
// One CTA of 512 threads processes one block pair (i, j) of an outer step:
//
//   1. Gram matrix of the M x 32 column pair [G_i G_j] (lower triangle only:
//      the Cholesky never reads the upper one), streamed through shared
//      memory in 64-row tiles by the TMA engine (cp.async.bulk + mbarrier,
//      4 stages); each of the 528 entries is one FMA chain in the
//      reference's row order (share/device_code_common_Cholesky.hpp:4-56),
//      computed in 4x4 register tiles with a sliding row window;
//   2. 32x32 Cholesky in one warp, rows in registers, shuffles for the
//      pivots (share/device_code_common_Cholesky.hpp:58-158);
//   3. inner Jacobi sweep(s) over the 32 columns of R, one warp per column
//      pair, warp-shuffle dot products, trigonometric or hyperbolic
//      rotations, optional KISS sorting (share/device_code_nosort.hpp,
//      share/device_code_cdsort.hpp, share/device_code_cdsort_KISS.hpp);
//   4. [G_i G_j] <- [G_i G_j] V_loc (and V likewise), 256-row stages
//      brought in by the TMA engine, each output a 32-FMA chain in the
//      reference's skewed order (share/device_code_common.hpp:146-185),
//      computed in 4x8 register tiles along anti-diagonals.
//
// All arithmetic is in the reference's order, so results are bit-identical.
#include "gjx_device.cuh"
#include "gjx_internal.h"

namespace gjx {

constexpr unsigned kThreads = 512u;
constexpr long long kWaitLimit = 2000000000ll; // ~1 s of cycles per wait

// Gram staging: column c of a 64-row tile at gcol_off(c), rows 0..95 where
// rows 64..95 repeat rows 0..31, so a chain starting at row x never wraps.
constexpr unsigned kGramStages = 4u;
constexpr unsigned kGramColLd = 112u;
constexpr unsigned kGramStage = 32u * kGramColLd; // doubles
constexpr uint32_t kGramTxBytes = 32u * (512u + 256u);
__device__ __forceinline__ unsigned gcol_off(const unsigned c) { return c * kGramColLd + 2u * ((c >> 2) & 7u); }

// Update staging: 256 rows x 32 columns; the 32-row piece p of a column
// starts at p*34 (2 doubles of skew per piece spreads the banks).
constexpr unsigned kUpdRows = 256u;
constexpr unsigned kUpdColLd = 272u;
constexpr unsigned kUpdStages = 2u;
constexpr unsigned kUpdStage = 32u * kUpdColLd; // doubles
constexpr unsigned kVTLd = 34u;                 // B^T rows (V_loc transposed)

constexpr unsigned kRegion =
    (kGramStages * kGramStage > kUpdStages * kUpdStage) ? kGramStages * kGramStage : kUpdStages * kUpdStage;

// shared memory map (doubles, then bytes)
constexpr unsigned kOffR = kRegion;        // R, 32x32 (later B^T, 32x34)
constexpr unsigned kOffVl = kOffR + 32u * kVTLd;
constexpr unsigned kOffS0 = kOffVl + 1024u; // strat0 copy, 1024 bytes
constexpr unsigned kOffRed = kOffS0 + 128u; // 32 unsigned
constexpr unsigned kOffBar = kOffRed + 16u; // 8 mbarriers
constexpr unsigned kOffFlag = kOffBar + 8u;
constexpr unsigned kSmemDoubles = kOffFlag + 2u;

size_t l1_smem_bytes() { return (size_t)kSmemDoubles * sizeof(double); }

#define E32(A, r, c) (A)[(c) * 32u + (r)]

// ---------------------------------------------------------------------------
// Gram: one 64-row tile for the thread's 4x4 block of entries (x0+u, y0+v).
// Entry (x, y) adds G[r,y]*G[r,x] for r = x, x+1, ..., x+63 (mod 64).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void gram_tile(const double *const st, const unsigned x0, const unsigned y0,
                                          double (&acc)[4][4])
{
  const double *xp[4], *yp[4];
#pragma unroll
  for (unsigned u = 0u; u < 4u; ++u)
    xp[u] = st + gcol_off(x0 + u) + x0 + u;
#pragma unroll
  for (unsigned v = 0u; v < 4u; ++v)
    yp[v] = st + gcol_off(y0 + v) + x0;
  double W[4][4]; // W[slot][v]: row x0 + (j..j+3), slot = row mod 4
#pragma unroll
  for (unsigned m = 0u; m < 4u; ++m)
#pragma unroll
    for (unsigned v = 0u; v < 4u; ++v)
      W[m][v] = yp[v][m];
#pragma unroll
  for (unsigned j = 0u; j < 64u; ++j) {
    double X[4];
#pragma unroll
    for (unsigned u = 0u; u < 4u; ++u)
      X[u] = xp[u][j];
#pragma unroll
    for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
      for (unsigned v = 0u; v < 4u; ++v)
        acc[u][v] = __fma_rn(W[(j + u) & 3u][v], X[u], acc[u][v]);
    if (j < 63u) {
#pragma unroll
      for (unsigned v = 0u; v < 4u; ++v)
        W[j & 3u][v] = yp[v][j + 4u];
    }
  }
}

// ---------------------------------------------------------------------------
// Cholesky of the lower triangle held in R, by one warp: lane x keeps row x.
// Afterwards R = L^T with zeros below the diagonal.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void chol32_warp(double *const R, const unsigned x)
{
  double a[32];
#pragma unroll
  for (unsigned j = 0u; j < 32u; ++j)
    a[j] = (j <= x) ? E32(R, x, j) : 0.0;
#pragma unroll
  for (unsigned k = 0u; k < 32u; ++k) {
    const double akk = __shfl_sync(0xffffffffu, a[k], k);
    const double rs = rsqrt_rn(akk);
    const double sq = __dsqrt_rn(akk);
    if (x > k)
      a[k] = a[k] * rs;
    else if (x == k)
      a[k] = sq;
#pragma unroll
    for (unsigned j = k + 1u; j < 32u; ++j) {
      const double ajk = __shfl_sync(0xffffffffu, a[k], j);
      if (x >= j)
        a[j] = __fma_rn(-a[k], ajk, a[j]);
    }
  }
  __syncwarp();
#pragma unroll
  for (unsigned y = 0u; y < 32u; ++y)
    E32(R, y, x) = (x >= y) ? a[y] : 0.0;
}

// ---------------------------------------------------------------------------
// Inner Jacobi sweep(s).  Warp y owns column pair y of each inner step, lane
// x row x.  definite != 0: all pairs trigonometric (J = +-I on the block);
// otherwise columns < npos are +1 and the others -1.
// ---------------------------------------------------------------------------
template <bool SORT>
__device__ __forceinline__ void inner_sweeps(double *const R, double *const Vl, const uint8_t *const s0,
                                             const unsigned s0steps, const unsigned nswp, const int definite,
                                             const unsigned npos, unsigned *const red, const unsigned x,
                                             const unsigned y, unsigned &blk_s, unsigned &blk_b)
{
  blk_s = 0u;
  blk_b = 0u;
  for (unsigned swp = 0u; swp < nswp; ++swp) {
    unsigned ws = 0u, wb = 0u;
    for (unsigned step = 0u; step < s0steps; ++step) {
      const unsigned p = s0[(step * 16u + y) * 2u + 0u];
      const unsigned q = s0[(step * 16u + y) * 2u + 1u];
      const double Gp = E32(R, x, p), Gq = E32(R, x, q);
      const double Vp = E32(Vl, x, p), Vq = E32(Vl, x, q);
      const double Dp = sum32(__fma_rn(Gp, Gp, 0.0));
      const double Dq = sum32(__fma_rn(Gq, Gq, 0.0));
      const double Apq = sum32(__fma_rn(Gp, Gq, 0.0));
      const double Dp_ = __dsqrt_rn(Dp), Dq_ = __dsqrt_rn(Dq), Apq_ = fabs(Apq), Dpq_ = Dp_ * Dq_;
      const int ts = !(Apq_ < (Dpq_ * kMyTol));
      int tb = 0;
      if (!SORT) {
        if (ts) {
          const bool trig = definite || ((p < npos) && (q < npos)) || ((p >= npos) && (q >= npos));
          double c, t, t_;
          if (trig) {
            tb = rotT(Apq, Dp, Dq, c, t);
            t_ = -t;
          }
          else {
            tb = rotH(Apq, Dp, Dq, c, t);
            t_ = t;
          }
          double np = __fma_rn(t_, Gq, Gp), nq = __fma_rn(t, Gp, Gq);
          double vp = __fma_rn(t_, Vq, Vp), vq = __fma_rn(t, Vp, Vq);
          if (tb) {
            np = c * np;
            nq = c * nq;
            vp = c * vp;
            vq = c * vq;
          }
          E32(R, x, p) = np;
          E32(R, x, q) = nq;
          E32(Vl, x, p) = vp;
          E32(Vl, x, q) = vq;
        }
      }
      else {
        int def;
        if (definite)
          def = definite;
        else if ((p < npos) && (q < npos))
          def = +1;
        else if ((p >= npos) && (q >= npos))
          def = -1;
        else
          def = 0;
        if (ts) {
          double c, t, t_, Dp2 = Dp, Dq2 = Dq;
          if (def) {
            tb = rotT(Apq, Dp, Dq, c, t);
            t_ = -t;
            Dp2 = __fma_rn(t, Apq, Dp);
            Dq2 = __fma_rn(t_, Apq, Dq);
          }
          else {
            tb = rotH(Apq, Dp, Dq, c, t);
            t_ = t;
          }
          double np = __fma_rn(t_, Gq, Gp), nq = __fma_rn(t, Gp, Gq);
          double vp = __fma_rn(t_, Vq, Vp), vq = __fma_rn(t, Vp, Vq);
          if (tb) {
            np = c * np;
            nq = c * nq;
            vp = c * vp;
            vq = c * vq;
          }
          const bool keep = (!def) || ((def > 0) && (Dp2 >= Dq2)) || ((def < 0) && (Dp2 <= Dq2));
          const unsigned dp = keep ? p : q, dq = keep ? q : p;
          E32(R, x, dp) = np;
          E32(R, x, dq) = nq;
          E32(Vl, x, dp) = vp;
          E32(Vl, x, dq) = vq;
        }
        else if (((def > 0) && (Dp < Dq)) || ((def < 0) && (Dq < Dp))) {
          E32(R, x, p) = Gq;
          E32(R, x, q) = Gp;
          E32(Vl, x, p) = Vq;
          E32(Vl, x, q) = Vp;
        }
      }
      ws += (unsigned)ts;
      wb += (unsigned)tb;
      __syncthreads();
    }
    if (x == 0u) {
      red[y] = ws;
      red[16u + y] = wb;
    }
    __syncthreads();
    unsigned tot_s = 0u, tot_b = 0u;
#pragma unroll
    for (unsigned i = 0u; i < 16u; ++i) {
      tot_s += red[i];
      tot_b += red[16u + i];
    }
    __syncthreads();
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

// ---------------------------------------------------------------------------
// The block-pair step kernel.
// ---------------------------------------------------------------------------
template <bool SORT, bool ACCV>
__global__ void __launch_bounds__(kThreads, 1) l1_step_kernel(const StepParams P)
{
  extern __shared__ __align__(128) double sm[];
  double *const stg = sm;
  double *const R = sm + kOffR;
  double *const Vl = sm + kOffVl;
  uint8_t *const s0 = reinterpret_cast<uint8_t *>(sm + kOffS0);
  unsigned *const red = reinterpret_cast<unsigned *>(sm + kOffRed);
  uint64_t *const bars = reinterpret_cast<uint64_t *>(sm + kOffBar);

  const unsigned tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
  const size_t pidx = ((size_t)P.step * P.pairs + blockIdx.x) * 2u;
  const unsigned iBlk = P.strat1[pidx + 0u], jBlk = P.strat1[pidx + 1u];
  double *const Gi = P.G + (size_t)iBlk * kNColB * P.ldG;
  double *const Gj = P.G + (size_t)jBlk * kNColB * P.ldG;

  for (unsigned i = tid; i < 256u; i += kThreads)
    reinterpret_cast<uint32_t *>(s0)[i] = reinterpret_cast<const uint32_t *>(P.strat0)[i];
  if (tid == 0u) {
    for (unsigned b = 0u; b < 8u; ++b)
      mbar_init(&bars[b], 1u);
    mbar_fence_init();
  }
  __syncthreads();

  // ------------------------------ 1. Gram --------------------------------
  const unsigned ntile = P.nrow >> 6;
  const bool gthr = (warp < 4u) && (lane < 9u);
  unsigned gx0 = 0u, gy0 = 0u;
  if (gthr) { // 36 tiles of 4x4 covering the lower triangle, (xb, yb <= xb)
    const unsigned t = lane * 4u + warp;
    unsigned xb = 0u;
    while (((xb + 1u) * (xb + 2u)) / 2u <= t)
      ++xb;
    gx0 = 4u * xb;
    gy0 = 4u * (t - (xb * (xb + 1u)) / 2u);
  }
  double gacc[4][4];
#pragma unroll
  for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
    for (unsigned v = 0u; v < 4u; ++v)
      gacc[u][v] = +0.0;

  auto issue_gram = [&](const unsigned T) { // warp 0
    const unsigned s = T % kGramStages;
    double *const st = stg + s * kGramStage;
    if (lane == 0u)
      mbar_arrive_expect_tx(&bars[s], kGramTxBytes);
    __syncwarp();
    const double *const src = ((lane < 16u) ? (Gi + (size_t)lane * P.ldG) : (Gj + (size_t)(lane - 16u) * P.ldG)) +
                              (size_t)T * 64u;
    double *const dst = st + gcol_off(lane);
    bulk_g2s(dst, src, 512u, &bars[s]);
    bulk_g2s(dst + 64u, src, 256u, &bars[s]);
  };

  unsigned issued = 0u;
  if (warp == 0u)
    for (; (issued < kGramStages - 1u) && (issued < ntile); ++issued)
      issue_gram(issued);
  else
    issued = (kGramStages - 1u < ntile) ? (kGramStages - 1u) : ntile;

  unsigned T = 0u;
  int failed = 0;
  for (; T < ntile; ++T) {
    if (issued < ntile) {
      if (warp == 0u)
        issue_gram(issued);
      ++issued;
    }
    int fail = 0;
    if (warp < 4u) {
      if (!mbar_wait_bounded(&bars[T % kGramStages], (T / kGramStages) & 1u, kWaitLimit))
        fail = 1;
      else if (gthr)
        gram_tile(stg + (T % kGramStages) * kGramStage, gx0, gy0, gacc);
    }
    failed = __syncthreads_or(fail); // uniform decision
    if (failed)
      break;
  }
  if (failed) { // drain the copies still in flight (bounded), then report
    if (warp == 0u && lane == 0u) {
      for (unsigned U = T; U < issued; ++U)
        (void)mbar_wait_bounded(&bars[U % kGramStages], (U / kGramStages) & 1u, kWaitLimit / 8);
      atomicOr(P.err, kErrWaitTimeout);
    }
    return;
  }
  if (gthr) {
#pragma unroll
    for (unsigned u = 0u; u < 4u; ++u)
#pragma unroll
      for (unsigned v = 0u; v < 4u; ++v)
        if (gx0 + u >= gy0 + v)
          E32(R, gx0 + u, gy0 + v) = gacc[u][v];
  }
  __syncthreads();

  // ---------------------------- 2. Cholesky -------------------------------
  if (warp == 0u)
    chol32_warp(R, lane);
  else
    for (unsigned i = tid - 32u; i < 1024u; i += kThreads - 32u)
      Vl[i] = ((i >> 5) == (i & 31u)) ? 1.0 : 0.0;
  __syncthreads();

  // --------------------------- 3. inner sweeps ----------------------------
  int definite;
  unsigned npos;
  if (P.gdefinite) {
    definite = P.gdefinite;
    npos = 0u;
  }
  else { // block-local signature (share/device_code_nosort_solveV.hpp:33-67)
    const unsigned ifc0 = iBlk * kNColB, ifc1 = jBlk * kNColB, nplus = P.nplus;
    if (nplus <= ifc0) {
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
  unsigned blk_s, blk_b;
  inner_sweeps<SORT>(R, Vl, s0, P.s0steps, P.nswp0, definite, npos, red, lane, warp, blk_s, blk_b);

  if (tid == 0u && blk_s) {
    if (blk_b)
      atomicAdd(P.cvg, (((unsigned long long)blk_b) << 32) | blk_s);
    else
      atomicAdd(reinterpret_cast<unsigned *>(P.cvg), blk_s); // low word, as the reference
  }
  if (!SORT && !blk_s)
    return; // no rotation: the block pair is unchanged

  // ------------------------------ 4. update -------------------------------
  double *const VT = R; // R is dead; B^T[s][c] = V_loc[s][c]
  for (unsigned i = tid; i < 1024u; i += kThreads) {
    const unsigned c = i >> 5, s = i & 31u;
    VT[s * kVTLd + c] = E32(Vl, s, c);
  }

  const unsigned nG = (P.nrow + kUpdRows - 1u) / kUpdRows;
  const unsigned nV = ACCV ? (P.ncol + kUpdRows - 1u) / kUpdRows : 0u;
  const unsigned nst = nG + nV;
  double *const Vi = ACCV ? (P.V + (size_t)iBlk * kNColB * P.ldV) : nullptr;
  double *const Vj = ACCV ? (P.V + (size_t)jBlk * kNColB * P.ldV) : nullptr;

  // stage k: rows [base, base + rows) of G (k < nG) or V
  auto stage_geom = [&](const unsigned k, double *&ci, double *&cj, size_t &ld, unsigned &base, unsigned &rows) {
    if (k < nG) {
      ci = Gi;
      cj = Gj;
      ld = P.ldG;
      base = k * kUpdRows;
      rows = min(kUpdRows, P.nrow - base);
    }
    else {
      ci = Vi;
      cj = Vj;
      ld = P.ldV;
      base = (k - nG) * kUpdRows;
      rows = min(kUpdRows, P.ncol - base);
    }
  };
  auto issue_upd = [&](const unsigned k) { // warp 0
    double *ci, *cj;
    size_t ld;
    unsigned base, rows;
    stage_geom(k, ci, cj, ld, base, rows);
    const unsigned s = k % kUpdStages, pieces = rows >> 5;
    double *const st = stg + s * kUpdStage;
    if (lane == 0u)
      mbar_arrive_expect_tx(&bars[4u + s], 32u * pieces * 256u);
    __syncwarp();
    const double *const src = ((lane < 16u) ? (ci + (size_t)lane * ld) : (cj + (size_t)(lane - 16u) * ld)) + base;
    double *const dst = st + lane * kUpdColLd;
    for (unsigned pc = 0u; pc < pieces; ++pc)
      bulk_g2s(dst + pc * 34u, src + pc * 32u, 256u, &bars[4u + s]);
  };

  __syncthreads(); // VT ready; the Gram stages are free
  if (warp == 0u)
    issue_upd(0u);
  const unsigned rg = warp, sub = lane & 7u, cg = lane >> 3;
  for (unsigned k = 0u; k < nst; ++k) {
    if (warp == 0u && k + 1u < nst)
      issue_upd(k + 1u);
    int fail = 0;
    if (warp < 8u) {
      if (!mbar_wait_bounded(&bars[4u + (k % kUpdStages)], (k / kUpdStages) & 1u, kWaitLimit))
        fail = 1;
      else {
        double *ci, *cj;
        size_t ld;
        unsigned base, rows;
        stage_geom(k, ci, cj, ld, base, rows);
        if (sub * 32u < rows) {
          double acc[4][8];
          update_stage(stg + (k % kUpdStages) * kUpdStage, VT, rg, sub, cg, acc);
          const unsigned r0 = base + sub * 32u + rg * 4u;
#pragma unroll
          for (unsigned v = 0u; v < 8u; ++v) {
            const unsigned c = cg * 8u + v;
            double *const col = ((c < 16u) ? (ci + (size_t)c * ld) : (cj + (size_t)(c - 16u) * ld)) + r0;
            *reinterpret_cast<double2 *>(col) = make_double2(acc[0][v], acc[1][v]);
            *reinterpret_cast<double2 *>(col + 2u) = make_double2(acc[2][v], acc[3][v]);
          }
        }
      }
    }
    if (__syncthreads_or(fail)) { // uniform decision; drain (bounded), report
      if (warp == 0u && lane == 0u) {
        (void)mbar_wait_bounded(&bars[4u + (k % kUpdStages)], (k / kUpdStages) & 1u, kWaitLimit / 8);
        if (k + 1u < nst)
          (void)mbar_wait_bounded(&bars[4u + ((k + 1u) % kUpdStages)], ((k + 1u) / kUpdStages) & 1u,
                                  kWaitLimit / 8);
        atomicOr(P.err, kErrWaitTimeout);
      }
      return;
    }
  }
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

__global__ void rsqrt_test_kernel(const double *const in, double *const out, const unsigned n)
{
  const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    out[i] = rsqrt_rn(in[i]);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
cudaError_t l1_configure()
{
  const int bytes = (int)l1_smem_bytes();
  cudaError_t e;
  if ((e = cudaFuncSetAttribute(l1_step_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
    return e;
  if ((e = cudaFuncSetAttribute(l1_step_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
    return e;
  if ((e = cudaFuncSetAttribute(l1_step_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)))
    return e;
  return cudaFuncSetAttribute(l1_step_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

cudaError_t launch_l1_step(const bool sort, const bool accv, const StepParams &p, cudaStream_t s)
{
  const dim3 grid(p.pairs), block(kThreads);
  const size_t sh = l1_smem_bytes();
  if (sort) {
    if (accv)
      l1_step_kernel<true, true><<<grid, block, sh, s>>>(p);
    else
      l1_step_kernel<true, false><<<grid, block, sh, s>>>(p);
  }
  else {
    if (accv)
      l1_step_kernel<false, true><<<grid, block, sh, s>>>(p);
    else
      l1_step_kernel<false, false><<<grid, block, sh, s>>>(p);
  }
  return cudaGetLastError();
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

cudaError_t launch_rsqrt_test(const double *in, double *out, unsigned n, cudaStream_t s)
{
  rsqrt_test_kernel<<<(n + 255u) / 256u, 256u, 0, s>>>(in, out, n);
  return cudaGetLastError();
}

} // namespace gjx
