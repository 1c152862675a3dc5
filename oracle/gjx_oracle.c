/*
 * gjx_oracle.c -- CPU restatement of the GPUJACHx hierarchically blocked
 * one-sided Jacobi (H)SVD, plain FP64 path, operation for operation.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is compiled
 * into oracle/_build/libgjx_oracle.so and may be loaded only by tests/,
 * __graft_entry__.smoke() and the CPU-baseline / reference arm of bench.py,
 * always as the checker or the timed CPU baseline, never as a product path.
 * The product (gpujachx_b200, libgjx.so) never links or calls it.
 *
 * Parity: pinned.  Its outputs are compared bit for bit with the reference
 * (sources under share/ and 1/ built for sm_100a and run on a B200) through
 * the golden fixtures in tests/golden/, which record the reference's own
 * outputs (see tests/golden/make_golden.py).
 *
 * Every routine restates the reference arithmetic in the same order, so that
 * the results are identical bit for bit; the citations give the reference
 * file:line each routine follows (paths relative to the reference repo):
 *   - the 32-lane xor-butterfly sum          share/device_code_common_Kepler.hpp:26-74
 *   - trigonometric / hyperbolic rotations  share/device_code_common_rotate.hpp:16-64 (USE_RSQRT)
 *   - correctly rounded 1/sqrt              share/device_code_common.hpp:89-133 (same results;
 *                                            the method here is our own exact integer midpoint test)
 *   - Gram matrix of a column pair          share/device_code_common_Cholesky.hpp:4-56
 *   - 32x32 Cholesky and transposition      share/device_code_common_Cholesky.hpp:58-158
 *   - inner (L0) Jacobi, no sorting          share/device_code_nosort.hpp:4-222
 *   - inner (L0) Jacobi, KISS sorting        share/device_code_cdsort_KISS.hpp:4-260,
 *                                            share/device_code_cdsort.hpp:10-167
 *   - block-pair kernels (L1)                share/device_code_{nosort,cdsort}_{solveV,accumV}.hpp
 *   - Cannon-like update G <- G*V_loc        share/device_code_common.hpp:146-185
 *   - column normalisation and D            share/device_code_common.hpp:187-219
 *   - V = I                                  share/device_code_common.hpp:221-230
 *   - sweep driver and argument checks      1/HypJacL2.cu:13-202
 *   - strategy table loading                 share/HypJacL.cu:11-121, share/my_utils.cu:30-61
 *   - QR factor of the pair (-DUSE_QR):      share/device_code_common_QR.hpp:4-94 (dPeelOff,
 *     Householder QR of 32-row chunks merged  dFactorize), share/device_code_common_Kepler.hpp:326-371
 *     by Givens rotations                     (dQR32), share/device_code_common_rotate.hpp:120-155
 *                                            (dGivens)
 *   - scaled norms and cosines (-DUSE_QR,    share/device_code_common_Kepler.hpp:76-324 (dMax32,
 *     -DUSE_DRMAC)                            dMin32, dSSQ32, dNRM2_32, dCOSA),
 *                                            share/device_code_common_scale.hpp:7-58
 *   - Drmac's inner sweep for the definite   share/device_code_cdsort_Drmac.hpp:4-316,
 *     sorting kernels (-DUSE_DRMAC)           share/device_code_common_rotate.hpp:5-8 (tCot2)
 *
 * The variant (gjxo_set_variant): 0 the default build (Gram + Cholesky), 1
 * the -DUSE_QR build, 2 the -DUSE_DRMAC build (which implies USE_QR).
 *
 * Build: gcc -O2 -fopenmp -ffp-contract=off -fno-fast-math (no contraction of
 * a*b+c into fma anywhere: every fma below is explicit).
 */

#include <dlfcn.h>
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define O_NSWEEP 30u

/* the two products of a Givens rotation in dPeelOff (c a + s b, c b - s a),
 * as the reference's nvcc build contracts them */
#ifndef O_GIVENS_A
#define O_GIVENS_A(c, a, s, b) fma((c), (a), (s) * (b))
#endif
#ifndef O_GIVENS_B
#define O_GIVENS_B(c, b, s, a) fma((c), (b), -((s) * (a)))
#endif
#define O_NCOLB 16u

/* sqrt(2^-53), 2^27 = sqrt(2 / 2^-53), sqrt(32) * 2^-53, 2/sqrt(3), 1/2:
 * the correctly rounded values of the definitions in share/HypJacL.hpp:21-59 */
static const double O_SQRT_HEPS = 0x1.6a09e667f3bcdp-27;
static const double O_SQRT_2_HEPS = 0x1.0p+27;
static const double O_MYTOL = 0x1.6a09e667f3bcdp-51;
static const double O_COSHI_FIX = 0x1.279a74590331cp+0;
static const double O_TANH1_FIX = 0.5;

/* ---------------------------------------------------------------------- */
/* correctly rounded 1/sqrt(a)                                             */
/* ---------------------------------------------------------------------- */

/* (2Y+1)^2 * F < 2^160 ?  i.e. is 1/sqrt(F) above the midpoint (2Y+1)*2^-80 */
static int o_above_mid(uint64_t Y2p1, uint64_t F)
{
  const unsigned __int128 P = (unsigned __int128)Y2p1 * Y2p1; /* < 2^108 */
  const uint64_t Pl = (uint64_t)P, Ph = (uint64_t)(P >> 64);
  const unsigned __int128 lo = (unsigned __int128)Pl * F;    /* < 2^118 */
  const unsigned __int128 hi = (unsigned __int128)Ph * F;    /* < 2^98 */
  const unsigned __int128 T = hi + (lo >> 64);               /* product >> 64 */
  return T < ((unsigned __int128)1 << 96);
}

/*
 * rsqrt rounded to nearest.  a = F * 2^e with e even and F in [2^52, 2^54);
 * 1/sqrt(F) lies in (2^-27, 2^-26] and, below 2^-26, equals Y * 2^-79 for a
 * 53-bit Y in [2^52, 2^53).  Starting from the estimate 1/sqrt(F) (two
 * correctly rounded operations, within two ulps), Y is moved until
 * 1/sqrt(F) lies between the midpoints (2Y-1)*2^-80 and (2Y+1)*2^-80; the
 * side of a midpoint m is decided exactly, in integers, by the sign of
 * 1 - m^2 * F.  No midpoint is ever hit exactly ((2Y+1)^2 * F = 2^160 would
 * need an odd square dividing a power of two), so the result is the
 * correctly rounded 1/sqrt(a).
 */
double gjxo_rsqrt_rn(const double a)
{
  if (isnan(a))
    return a + a;
  if (a == 0.0)
    return copysign(INFINITY, a);
  if (a < 0.0)
    return -NAN;
  if (isinf(a))
    return 0.0;

  uint64_t bits;
  memcpy(&bits, &a, sizeof(bits));
  int E = (int)((bits >> 52) & 0x7FFu);
  uint64_t F = bits & 0xFFFFFFFFFFFFFull;
  if (E) {
    F |= (1ull << 52);
  }
  else { /* subnormal: normalise */
    E = 1;
    while (!(F & (1ull << 52))) {
      F <<= 1;
      --E;
    }
  }
  int e = E - 1075; /* a = F * 2^e */
  if (e & 1) {
    F <<= 1;
    --e;
  }
  if (F == (1ull << 52)) /* a = 2^(52+e), an exact power of four */
    return ldexp(1.0, -26 - e / 2);

  const double est = 1.0 / sqrt((double)F); /* in [2^-27, 2^-26] */
  int64_t Y = (int64_t)ldexp(est, 79);
  if (Y >= (int64_t)(1ull << 53))
    Y = (int64_t)(1ull << 53) - 1;
  if (Y < (int64_t)(1ull << 52))
    Y = (int64_t)(1ull << 52);
  while (o_above_mid((uint64_t)(2 * Y + 1), F))
    ++Y;
  while ((Y > (int64_t)(1ull << 52)) && !o_above_mid((uint64_t)(2 * Y - 1), F))
    --Y;
  return ldexp((double)Y, -79 - e / 2);
}

/* ---------------------------------------------------------------------- */
/* 32-lane butterfly sum: lane i adds lane i^16, ^8, ^4, ^2, ^1; lane 0    */
/* ---------------------------------------------------------------------- */

double gjxo_sum32(const double *const v)
{
  double t[32];
  for (unsigned i = 0u; i < 32u; ++i)
    t[i] = v[i];
  for (unsigned k = 16u; k; k >>= 1u)
    for (unsigned i = 0u; i < k; ++i)
      t[i] = t[i] + t[i + k];
  return t[0];
}

/* ---------------------------------------------------------------------- */
/* 2x2 rotations                                                           */
/* ---------------------------------------------------------------------- */

int gjxo_rotT(const double Apq, const double Dp, const double Dq, double *const c, double *const t)
{
  const double h = Dq - Dp;
  const double ct2 = h / scalbn(Apq, 1);
  const double CT2 = fabs(ct2);
  if (CT2 < O_SQRT_HEPS) {
    const double cot = CT2 + 1.0;
    *t = copysign(1.0 / cot, ct2);
    *c = gjxo_rsqrt_rn(fma(*t, *t, 1.0));
    return 1;
  }
  else if (CT2 >= O_SQRT_2_HEPS) {
    const double cot = scalbn(CT2, 1);
    *c = 1.0;
    *t = copysign(1.0 / cot, ct2);
    return 0;
  }
  else {
    const double cot = CT2 + sqrt(fma(CT2, CT2, 1.0));
    *t = copysign(1.0 / cot, ct2);
    *c = gjxo_rsqrt_rn(fma(*t, *t, 1.0));
    return (*c < 1.0);
  }
}

int gjxo_rotH(const double Apq, const double Dp, const double Dq, double *const c, double *const t)
{
  const double h = Dq + Dp;
  const double ct2 = -(h / scalbn(Apq, 1));
  const double CT2 = fabs(ct2);
  if (CT2 >= O_SQRT_2_HEPS) {
    const double cot = scalbn(CT2, 1);
    *c = 1.0;
    *t = copysign(1.0 / cot, ct2);
    return 0;
  }
  else if (CT2 > 1.0) {
    const double cot = CT2 + sqrt(fma(CT2, CT2, -1.0));
    *t = copysign(1.0 / cot, ct2);
    *c = gjxo_rsqrt_rn(fma(-*t, *t, 1.0));
    return (*c > 1.0);
  }
  else {
    *c = O_COSHI_FIX;
    *t = O_TANH1_FIX;
    return 1;
  }
}

/* ---------------------------------------------------------------------- */
/* the variant builds: QR factor, scaled norms, Drmac's inner sweep          */
/* ---------------------------------------------------------------------- */

#define E32(A, r, c) (A)[(c) * 32u + (r)]

static int o_variant = 0; /* 0 Cholesky, 1 QR, 2 Drmac (+ QR) */
static void o_swap(double *const X, const unsigned p, const unsigned q);

void gjxo_set_variant(const int v) { o_variant = v; }

/* share/HypJacL.hpp:55-90: the decimal literals of the reference */
static const double O_MU_ = 1.4916681462400414314624091158735E-154;
static const double O_NU_ = 2.370187977027293260705088939015E+153;
static const double O_MU_EPS = 1.0020841800044863889980540256751E-292;
static const double O_NU_8 = 2.24711641857789464E+307;

/* max |x| and min |x| (x != 0) over the 32 lanes: order-free (exact) */
static double o_max32(const double *const x)
{
  double m = fabs(x[0]);
  for (unsigned l = 1u; l < 32u; ++l)
    m = fmax(m, fabs(x[l]));
  return m;
}

static double o_min32(const double *const x)
{
  double m = (x[0] == 0.0) ? DBL_MAX : fabs(x[0]);
  for (unsigned l = 1u; l < 32u; ++l)
    m = fmin(m, (x[l] == 0.0) ? DBL_MAX : fabs(x[l]));
  return m;
}

/* the butterfly sum of the lanes' squares (each square rounded first) */
static double o_ssq_lanes(const double *const x)
{
  double v[32];
  for (unsigned l = 0u; l < 32u; ++l)
    v[l] = x[l] * x[l];
  return gjxo_sum32(v);
}

/* share/device_code_common_scale.hpp:7-58 */
static int o_find_scl(const double x, const double t)
{
  int x_n, t_n;
  const double x_m = frexp(x, &x_n);
  const double t_m = frexp(t, &t_n);
  return ((x <= t) ? ((t_n - x_n) + (x_m < t_m)) : ((t_n - x_n) - (x_m > t_m)));
}

static int o_find_scl2(const double x)
{
  const int scl = ilogb(x);
  return (scl + (scl & 1));
}

static void o_normalize2(int *const scl, double *const ssq)
{
  const int scl_ = o_find_scl2(*ssq);
  *scl += scl_;
  *ssq = scalbn(*ssq, -scl_);
}

static int o_cmp_scl(const int s1, const int s2, const double x1, const double x2)
{
  if (s1 < s2)
    return -1;
  if (s2 < s1)
    return 1;
  if (x1 < x2)
    return -1;
  if (x2 < x1)
    return 1;
  return 0;
}

static void o_sum_scl(const int s1, const int s2, const double x1, const double x2, int *const s, double *const x)
{
  if (o_cmp_scl(s1, s2, x1, x2) <= 0) {
    *s = s2;
    *x = scalbn(x1, s1 - s2) + x2;
  }
  else {
    *s = s1;
    *x = scalbn(x2, s2 - s1) + x1;
  }
}

/* the lanes' |x| selected (and scaled) into the three magnitude ranges
 * (share/device_code_common_Kepler.hpp:178-208) */
static double o_ssq_range(const double *const x, const int range, const int scl)
{
  double v[32];
  for (unsigned l = 0u; l < 32u; ++l) {
    const double a = fabs(x[l]);
    if (range == 0)
      v[l] = (a < O_MU_) ? scalbn(a, scl) : 0.0;
    else if (range == 1)
      v[l] = ((a >= O_MU_) && (a <= O_NU_)) ? a : 0.0;
    else
      v[l] = (a > O_NU_) ? scalbn(a, scl) : 0.0;
  }
  return o_ssq_lanes(v);
}

/* share/device_code_common_Kepler.hpp:210-268: ssq * 2^scl = sum of squares */
static int o_SSQ32(double *const ssq, const double *const x)
{
  const double M = o_max32(x);
  if (M == 0.0) {
    *ssq = 0.0;
    return INT_MIN;
  }
  const double m = o_min32(x);
  const int lo = (m < O_MU_), hi = (M > O_NU_);
  int sc0, sc1, sc2, scl;
  double sq0, sq1, sq2;
  if (hi) {
    sc2 = o_find_scl(M, O_NU_);
    sq2 = o_ssq_range(x, 2, sc2);
    sc2 *= -2;
    if (m > O_NU_) {
      scl = sc2;
      *ssq = sq2;
    }
    else {
      sc1 = 0;
      sq1 = o_ssq_range(x, 1, 0);
      if (sq1 > 0.0) {
        o_normalize2(&sc1, &sq1);
        o_normalize2(&sc2, &sq2);
        o_sum_scl(sc1, sc2, sq1, sq2, &scl, ssq);
      }
      else {
        scl = sc2;
        *ssq = sq2;
      }
    }
  }
  else if (lo) {
    sc0 = o_find_scl(m, O_MU_);
    sq0 = o_ssq_range(x, 0, sc0);
    sc0 *= -2;
    if (M < O_MU_) {
      scl = sc0;
      *ssq = sq0;
    }
    else {
      sc1 = 0;
      sq1 = o_ssq_range(x, 1, 0);
      if (sq1 > 0.0) {
        o_normalize2(&sc1, &sq1);
        o_normalize2(&sc0, &sq0);
        o_sum_scl(sc0, sc1, sq0, sq1, &scl, ssq);
      }
      else {
        scl = sc0;
        *ssq = sq0;
      }
    }
  }
  else {
    scl = 0;
    *ssq = o_ssq_lanes(x);
  }
  return scl;
}

/* share/device_code_common_Kepler.hpp:278-283 */
double gjxo_nrm2_32(const double *const x)
{
  double ssq;
  const int scl = o_SSQ32(&ssq, x) / 2;
  return scalbn(sqrt(ssq), scl);
}

/* share/device_code_common_Kepler.hpp:285-324 (Ap >= Aq in o_cosa_) */
static double o_cosa_(const double Ap, const double Aq, const double *const x, const double *const y)
{
  double z[32];
  int big, small;
  if (Aq >= 1.0) {
    big = ((Ap * Aq) >= DBL_MAX);
    small = 0;
  }
  else {
    big = 0;
    small = ((Ap * Aq) <= O_MU_EPS);
  }
  if (big) {
    for (unsigned l = 0u; l < 32u; ++l)
      z[l] = (fabs(x[l]) >= fabs(y[l])) ? ((x[l] / Ap) * y[l]) : ((y[l] / Ap) * x[l]);
    return gjxo_sum32(z) / Aq;
  }
  if (small) {
    for (unsigned l = 0u; l < 32u; ++l)
      z[l] = (fabs(x[l]) >= fabs(y[l])) ? (x[l] * (y[l] / Aq)) : (y[l] * (x[l] / Aq));
    return gjxo_sum32(z) / Ap;
  }
  for (unsigned l = 0u; l < 32u; ++l)
    z[l] = x[l] * y[l];
  return (gjxo_sum32(z) / Aq) / Ap;
}

double gjxo_cosa(const double Ap, const double Aq, const double *const x, const double *const y)
{
  return (Ap >= Aq) ? o_cosa_(Ap, Aq, x, y) : o_cosa_(Aq, Ap, y, x);
}

/* share/device_code_common_rotate.hpp:120-155 */
static void o_givens(const double f, const double g, double *const c, double *const s, double *const r)
{
  const double f_ = fabs(f), g_ = fabs(g);
  if (f_ >= g_) {
    if (g_ == 0.0) {
      *c = copysign(1.0, f);
      *s = 0.0;
      *r = f_;
    }
    else {
      const double g_f = g_ / f_;
      *r = f_ * sqrt(fma(g_f, g_f, 1.0));
      *c = f / *r;
      *s = g / *r;
    }
  }
  else {
    if (f_ == 0.0) {
      *c = 0.0;
      *s = copysign(1.0, g);
      *r = g_;
    }
    else {
      const double f_g = f_ / g_;
      *r = g_ * sqrt(fma(f_g, f_g, 1.0));
      *c = f / *r;
      *s = g / *r;
    }
  }
}

/* share/device_code_common_Kepler.hpp:326-371: Householder QR of a 32 x 32
 * block, reflector k applied to columns k+1..31, column k set to -beta e_k */
void gjxo_qr32(double *const A)
{
  for (unsigned k = 0u; k < 31u; ++k) {
    double Axk[32], Axk_[32];
    for (unsigned x = 0u; x < 32u; ++x) {
      Axk[x] = E32(A, x, k);
      Axk_[x] = (x >= k) ? Axk[x] : 0.0;
    }
    const double nrm2 = gjxo_nrm2_32(Axk_);
    if (!(nrm2 > 0.0))
      continue;
    const double alpha = E32(A, k, k);
    const double beta = copysign(nrm2, alpha);
    const double alpha_beta = alpha + beta;
    const double tau = alpha_beta / beta;
    double Vxk[32];
    for (unsigned x = 0u; x < 32u; ++x)
      Vxk[x] = (x == k) ? 1.0 : ((x > k) ? (Axk_[x] / alpha_beta) : 0.0);
    for (unsigned j = k + 1u; j < 32u; ++j) {
      double v[32];
      for (unsigned x = 0u; x < 32u; ++x)
        v[x] = Vxk[x] * E32(A, x, j);
      const double dp = gjxo_sum32(v);
      const double _tdp = -(tau * dp);
      for (unsigned x = 0u; x < 32u; ++x)
        E32(A, x, j) = fma(_tdp, Vxk[x], E32(A, x, j));
    }
    for (unsigned x = 0u; x < 32u; ++x)
      E32(A, x, k) = (x == k) ? -beta : ((x > k) ? 0.0 : Axk[x]);
  }
}

/* share/device_code_common_QR.hpp:4-66: the triangular R1 (a QR-factored
 * chunk) merged into R0 by Givens rotations along the diagonals: in step k
 * row x of R0 and row x - k of R1 (x >= k) are rotated so that R1(x-k, x)
 * vanishes, in every column >= x */
static void o_peel(double *const R0, double *const R1)
{
  for (unsigned k = 0u; k < 32u; ++k)
    for (unsigned x = k; x < 32u; ++x) {
      const unsigned xk = x - k;
      double c, s, r;
      o_givens(E32(R0, x, x), E32(R1, xk, x), &c, &s, &r);
      for (unsigned j = x + 1u; j < 32u; ++j) {
        const double a = E32(R0, x, j), b = E32(R1, xk, j);
        E32(R0, x, j) = O_GIVENS_A(c, a, s, b);
        E32(R1, xk, j) = O_GIVENS_B(c, b, s, a);
      }
      E32(R0, x, x) = r;
      E32(R1, xk, x) = 0.0;
    }
}

/* share/device_code_common_QR.hpp:68-92 (dFactorize): R of the pair's rows */
void gjxo_qr_factor(double *const Gi, double *const Gj, const size_t ld, const unsigned nrow, double *const A)
{
  double W[1024];
  for (unsigned y = 0u; y < 32u; ++y)
    for (unsigned x = 0u; x < 32u; ++x)
      E32(A, x, y) = ((y < O_NCOLB) ? Gi + y * ld : Gj + (y - O_NCOLB) * ld)[x];
  gjxo_qr32(A);
  for (unsigned i = 32u; i < nrow; i += 32u) {
    for (unsigned y = 0u; y < 32u; ++y)
      for (unsigned x = 0u; x < 32u; ++x)
        E32(W, x, y) = ((y < O_NCOLB) ? Gi + y * ld : Gj + (y - O_NCOLB) * ld)[i + x];
    gjxo_qr32(W);
    o_peel(A, W);
  }
}

/* share/device_code_cdsort_Drmac.hpp:4-316: the definite sorting sweep with
 * scaled norms and cosines; def = +1 (descending) or -1 (ascending) */
static void o_drmac(double *const G, double *const V, const unsigned char *const strat0, const unsigned s0steps,
                    const unsigned nswp, const int def, unsigned *const s, unsigned *const b)
{
  unsigned blk_s = 0u, blk_b = 0u;
  for (unsigned swp = 0u; swp < nswp; ++swp) {
    unsigned swp_s = 0u, swp_b = 0u;
    for (unsigned step = 0u; step < s0steps; ++step)
      for (unsigned y = 0u; y < 16u; ++y) {
        const unsigned p = strat0[(step * 16u + y) * 2u + 0u];
        const unsigned q = strat0[(step * 16u + y) * 2u + 1u];
        double Gp[32], Gq[32], Vp[32], Vq[32];
        for (unsigned x = 0u; x < 32u; ++x) {
          Gp[x] = E32(G, x, p);
          Gq[x] = E32(G, x, q);
          Vp[x] = E32(V, x, p);
          Vq[x] = E32(V, x, q);
        }
        const double Ap = gjxo_nrm2_32(Gp), Aq = gjxo_nrm2_32(Gq), CosA = gjxo_cosa(Ap, Aq, Gp, Gq);
        const int transf_s = (fabs(CosA) >= O_MYTOL);
        swp_s += (unsigned)transf_s;
        int transf_b = 0;
        if (transf_s) {
          const double Aq_p = Aq / Ap, Ap_q = Ap / Aq, ct2 = (Aq_p - Ap_q) / scalbn(CosA, 1);
          if (ct2 <= O_NU_8) {
            const double CT2 = fabs(ct2);
            double c, t;
            if (CT2 < O_SQRT_HEPS) {
              const double cot = CT2 + 1.0;
              t = copysign(1.0 / cot, ct2);
              c = gjxo_rsqrt_rn(fma(t, t, 1.0));
              transf_b = 1;
            }
            else if (CT2 >= O_SQRT_2_HEPS) {
              const double cot = scalbn(CT2, 1);
              c = 1.0;
              t = copysign(1.0 / cot, ct2);
            }
            else {
              const double cot = CT2 + sqrt(fma(CT2, CT2, 1.0));
              t = copysign(1.0 / cot, ct2);
              c = gjxo_rsqrt_rn(fma(t, t, 1.0));
              transf_b = (c < 1.0);
            }
            const double t_ = -t, tCosA = t * CosA, tCosA_ = -tCosA;
            const double Ap_ = Ap * sqrt(fma(tCosA_, Aq_p, 1.0)), Aq_ = Aq * sqrt(fma(tCosA, Ap_q, 1.0));
            const int keep = (def > 0) ? (Ap_ >= Aq_) : (Ap_ <= Aq_);
            const unsigned dp = keep ? p : q, dq = keep ? q : p;
            for (unsigned x = 0u; x < 32u; ++x) {
              const double np = fma(t_, Gq[x], Gp[x]), nq = fma(t, Gp[x], Gq[x]);
              const double mp = fma(t_, Vq[x], Vp[x]), mq = fma(t, Vp[x], Vq[x]);
              E32(G, x, dp) = transf_b ? (c * np) : np;
              E32(G, x, dq) = transf_b ? (c * nq) : nq;
              E32(V, x, dp) = transf_b ? (c * mp) : mp;
              E32(V, x, dq) = transf_b ? (c * mq) : mq;
            }
          }
          else if ((def > 0) ? (Ap >= Aq) : (Ap <= Aq)) {
            const double t_ = CosA, t = -t_;
            for (unsigned x = 0u; x < 32u; ++x) {
              E32(G, x, q) = Aq * fma(t, Gp[x] / Ap, Gq[x] / Aq);
              E32(V, x, p) = fma(t_, Vq[x], Vp[x]);
              E32(V, x, q) = fma(t, Vp[x], Vq[x]);
            }
          }
          else {
            const double t = CosA, t_ = -t;
            for (unsigned x = 0u; x < 32u; ++x) {
              E32(G, x, q) = Ap * fma(t_, Gq[x] / Aq, Gp[x] / Ap);
              E32(G, x, p) = Gq[x];
              E32(V, x, q) = fma(t_, Vq[x], Vp[x]);
              E32(V, x, p) = fma(t, Vp[x], Vq[x]);
            }
          }
        }
        else if ((def > 0) ? (Ap < Aq) : (Aq < Ap)) {
          o_swap(G, p, q);
          o_swap(V, p, q);
        }
        swp_b += (unsigned)transf_b;
      }
    if (swp_s) {
      blk_s += swp_s;
      blk_b += swp_b;
    }
    else
      break;
  }
  *s = blk_s;
  *b = blk_b;
}

/* ---------------------------------------------------------------------- */
/* block-pair (L1) building blocks                                         */
/* ---------------------------------------------------------------------- */

/* local column c of the pair [G_i G_j] */
static inline double *o_col(double *const Gi, double *const Gj, const size_t ld, const unsigned c)
{
  return (c < O_NCOLB) ? (Gi + c * ld) : (Gj + (c - O_NCOLB) * ld);
}

/* lower triangle (and diagonal) of the Gram matrix, each element summed over
 * the rows of every 64-row tile starting at tile row x (the element's row) */
void gjxo_gram(double *const Gi, double *const Gj, const size_t ld, const unsigned nrow, double *const A)
{
  for (unsigned x = 0u; x < 32u; ++x) {
    const double *const cx = o_col(Gi, Gj, ld, x);
    for (unsigned y = 0u; y <= x; ++y) {
      const double *const cy = o_col(Gi, Gj, ld, y);
      double acc = +0.0;
      for (unsigned b = 0u; b < nrow; b += 64u)
        for (unsigned j = 0u; j < 64u; ++j) {
          const unsigned r = b + ((x + j) & 63u);
          acc = fma(cy[r], cx[r], acc);
        }
      E32(A, x, y) = acc;
    }
    for (unsigned y = x + 1u; y < 32u; ++y)
      E32(A, x, y) = 0.0; /* never read */
  }
}

/* right-looking Cholesky of the lower triangle, then R = L^T (zero below) */
void gjxo_chol32(double *const A)
{
  for (unsigned k = 0u; k < 32u; ++k) {
    const double Akk = E32(A, k, k);
    const double rs = gjxo_rsqrt_rn(Akk);
    for (unsigned x = k + 1u; x < 32u; ++x)
      E32(A, x, k) = E32(A, x, k) * rs;
    E32(A, k, k) = sqrt(Akk);
    for (unsigned j = k + 1u; j < 32u; ++j) {
      const double Ajk = E32(A, j, k);
      for (unsigned x = j; x < 32u; ++x)
        E32(A, x, j) = fma(-E32(A, x, k), Ajk, E32(A, x, j));
    }
  }
  double R[1024];
  for (unsigned x = 0u; x < 32u; ++x)
    for (unsigned y = 0u; y < 32u; ++y)
      E32(R, y, x) = ((x >= y) ? E32(A, x, y) : 0.0);
  memcpy(A, R, sizeof(R));
}

/* what the pair (p,q) of one inner step computes from the columns */
typedef struct {
  double Dp, Dq, Apq;
  int transf_s;
} o_dots;

static o_dots o_dot(const double *const G, const unsigned p, const unsigned q)
{
  double vp[32], vq[32], vpq[32];
  for (unsigned x = 0u; x < 32u; ++x) {
    const double Gp = E32(G, x, p), Gq = E32(G, x, q);
    vp[x] = fma(Gp, Gp, +0.0);
    vq[x] = fma(Gq, Gq, +0.0);
    vpq[x] = fma(Gp, Gq, +0.0);
  }
  o_dots d;
  d.Dp = gjxo_sum32(vp);
  d.Dq = gjxo_sum32(vq);
  d.Apq = gjxo_sum32(vpq);
  const double Dp_ = sqrt(d.Dp), Dq_ = sqrt(d.Dq), Apq_ = fabs(d.Apq), Dpq_ = Dp_ * Dq_;
  d.transf_s = !(Apq_ < (Dpq_ * O_MYTOL));
  return d;
}

/* apply the 2x2 transform to columns p,q of X (R or V_loc); when swap, the
 * two new columns exchange places; when scale, multiply by c */
static void o_rot(double *const X, const unsigned p, const unsigned q, const double c, const double tp,
                  const double tq, const int scale, const int swap)
{
  /* new_p = fma(tp, Xq, Xp), new_q = fma(tq, Xp, Xq) */
  const unsigned dp = swap ? q : p, dq = swap ? p : q;
  for (unsigned x = 0u; x < 32u; ++x) {
    const double Xp = E32(X, x, p), Xq = E32(X, x, q);
    const double np = fma(tp, Xq, Xp), nq = fma(tq, Xp, Xq);
    E32(X, x, dp) = scale ? (c * np) : np;
    E32(X, x, dq) = scale ? (c * nq) : nq;
  }
}

static void o_swap(double *const X, const unsigned p, const unsigned q)
{
  for (unsigned x = 0u; x < 32u; ++x) {
    const double t = E32(X, x, p);
    E32(X, x, p) = E32(X, x, q);
    E32(X, x, q) = t;
  }
}

/*
 * Inner (L0) Jacobi on R (32x32) accumulating V_loc.
 *   mode 0: no sorting, trigonometric            (dDefJacL0)
 *   mode 1: no sorting, mixed signs with npos    (dHypJacL0)
 *   mode 2: KISS sorting, definite = +1 / -1     (dDefJacL0posd / negd)
 *   mode 3: sorting, mixed signs with npos       (dHypJacL0s)
 * Returns the rotation counts of the block (small in *s, big in *b).
 */
void gjxo_inner(double *const G, double *const V, const unsigned char *const strat0, const unsigned s0steps,
                const unsigned nswp, const int mode, const int definite, const unsigned npos,
                unsigned *const s, unsigned *const b)
{
  unsigned blk_s = 0u, blk_b = 0u;
  for (unsigned swp = 0u; swp < nswp; ++swp) {
    unsigned swp_s = 0u, swp_b = 0u;
    for (unsigned step = 0u; step < s0steps; ++step) {
      for (unsigned y = 0u; y < 16u; ++y) {
        const unsigned p = strat0[(step * 16u + y) * 2u + 0u];
        const unsigned q = strat0[(step * 16u + y) * 2u + 1u];
        o_dots d = o_dot(G, p, q);
        swp_s += (unsigned)d.transf_s;
        int transf_b = 0;
        if (mode == 0 || mode == 1) {
          if (d.transf_s) {
            const int trig = (mode == 0) || (((p < npos) && (q < npos)) || ((p >= npos) && (q >= npos)));
            double c, t, t_;
            if (trig) {
              transf_b = gjxo_rotT(d.Apq, d.Dp, d.Dq, &c, &t);
              t_ = -t;
            }
            else {
              transf_b = gjxo_rotH(d.Apq, d.Dp, d.Dq, &c, &t);
              t_ = t;
            }
            o_rot(G, p, q, c, t_, t, transf_b, 0);
            o_rot(V, p, q, c, t_, t, transf_b, 0);
          }
        }
        else {
          int def;
          if (mode == 2)
            def = definite;
          else if ((p < npos) && (q < npos))
            def = +1;
          else if ((p >= npos) && (q >= npos))
            def = -1;
          else
            def = 0;
          if (d.transf_s) {
            double c, t, t_;
            double Dp = d.Dp, Dq = d.Dq;
            if (def) {
              transf_b = gjxo_rotT(d.Apq, Dp, Dq, &c, &t);
              t_ = -t;
              Dp = fma(t, d.Apq, Dp);
              Dq = fma(t_, d.Apq, Dq);
            }
            else {
              transf_b = gjxo_rotH(d.Apq, Dp, Dq, &c, &t);
              t_ = t;
            }
            const int keep = (!def || ((def > 0) && (Dp >= Dq)) || ((def < 0) && (Dp <= Dq)));
            o_rot(G, p, q, c, t_, t, transf_b, !keep);
            o_rot(V, p, q, c, t_, t, transf_b, !keep);
          }
          else if (((def > 0) && (d.Dp < d.Dq)) || ((def < 0) && (d.Dq < d.Dp))) {
            o_swap(G, p, q);
            o_swap(V, p, q);
          }
        }
        swp_b += (unsigned)transf_b;
      }
    }
    if (swp_s) {
      blk_s += swp_s;
      blk_b += swp_b;
    }
    else
      break;
  }
  *s = blk_s;
  *b = blk_b;
}

/* rows of the pair <- rows * B, each element a 32-term chain starting at
 * column (c + r) mod 32 */
void gjxo_update(double *const Gi, double *const Gj, const size_t ld, const unsigned nrow, const double *const B)
{
  double row[32];
  for (unsigned r = 0u; r < nrow; ++r) {
    const unsigned x = r & 31u;
    for (unsigned c = 0u; c < 32u; ++c)
      row[c] = o_col(Gi, Gj, ld, c)[r];
    for (unsigned c = 0u; c < 32u; ++c) {
      double acc = +0.0;
      unsigned p = (c + x) & 31u;
      for (unsigned k = 0u; k < 32u; ++k) {
        acc = fma(row[p], E32(B, p, c), acc);
        p = (p + 1u) & 31u;
      }
      o_col(Gi, Gj, ld, c)[r] = acc;
    }
  }
}

/* one block pair of one outer step; returns the counters like the atomics */
static void o_pair(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                   double *const G, const size_t ldG, double *const V, const size_t ldV,
                   const unsigned iBlk, const unsigned jBlk, const unsigned char *const strat0,
                   const unsigned s0steps, const unsigned nswp0, const int gdefinite,
                   unsigned *const s, unsigned *const b)
{
  const int cdsort = (routine & 1u) != 0u, full = (routine & 2u) != 0u;
  double *const Gi = G + (size_t)iBlk * O_NCOLB * ldG, *const Gj = G + (size_t)jBlk * O_NCOLB * ldG;
  double A[1024], Vl[1024];
  if (o_variant) /* -DUSE_QR / -DUSE_DRMAC builds */
    gjxo_qr_factor(Gi, Gj, ldG, nrow, A);
  else {
    gjxo_gram(Gi, Gj, ldG, nrow, A);
    gjxo_chol32(A);
  }
  for (unsigned i = 0u; i < 1024u; ++i)
    Vl[i] = ((i >> 5u) == (i & 31u)) ? 1.0 : 0.0;

  int definite;
  unsigned npos;
  if (gdefinite) {
    definite = gdefinite;
    npos = 0u;
  }
  else { /* share/device_code_nosort_solveV.hpp:33-67 */
    const unsigned ifc0 = iBlk * O_NCOLB, ifc1 = jBlk * O_NCOLB;
    if (nplus <= ifc0) {
      npos = 0u;
      definite = -1;
    }
    else if (nplus <= (ifc0 + O_NCOLB)) {
      npos = nplus - ifc0;
      definite = 0;
    }
    else if (nplus <= ifc1) {
      npos = O_NCOLB;
      definite = 0;
    }
    else if (nplus <= (ifc1 + O_NCOLB)) {
      npos = O_NCOLB + (nplus - ifc1);
      definite = 0;
    }
    else {
      npos = 2u * O_NCOLB;
      definite = +1;
    }
  }

  const int mode = cdsort ? (definite ? 2 : 3) : (definite ? 0 : 1);
  if (mode == 2 && o_variant == 2)
    o_drmac(A, Vl, strat0, s0steps, nswp0, definite, s, b);
  else
    gjxo_inner(A, Vl, strat0, s0steps, nswp0, mode, definite, npos, s, b);

  if (cdsort || *s) {
    gjxo_update(Gi, Gj, ldG, nrow, Vl);
    if (full) {
      double *const Vi = V + (size_t)iBlk * O_NCOLB * ldV, *const Vj = V + (size_t)jBlk * O_NCOLB * ldV;
      gjxo_update(Vi, Vj, ldV, ncol, Vl);
    }
  }
}

/* U = G diag(1/||g||), D = +-||g||^2 (lane-strided sums, then butterfly) */
void gjxo_initD(double *const G, const size_t ldG, const unsigned nrow, const unsigned ncol,
                const unsigned nplus, double *const D)
{
  for (unsigned c = 0u; c < ncol; ++c) {
    double *const g = G + (size_t)c * ldG;
    double lane[32];
    for (unsigned l = 0u; l < 32u; ++l) {
      double x = +0.0;
      for (unsigned r = l; r < nrow; r += 32u)
        x = fma(g[r], g[r], x);
      lane[l] = x;
    }
    const double y = gjxo_sum32(lane);
    const double nrm = sqrt(y);
    for (unsigned r = 0u; r < nrow; ++r)
      g[r] = g[r] / nrm;
    D[c] = (c < nplus) ? y : -y;
  }
}

/*
 * The sweep driver: 1/HypJacL2.cu:13-202 with the kernel launches replaced by
 * a loop over the block pairs of each step (parallel: the pairs are disjoint).
 * G is nrow x ncol with leading dimension ldG, V ncol x ncol with ldV.
 * strat0: [s0steps][16][2] bytes; strat1: [s1steps][s1pairs][2] uint16.
 * Returns 0, or the reference's negative argument codes.
 */
int gjxo_hypJacL2(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                  double *const G, const unsigned ldG, double *const V, const unsigned ldV, double *const D,
                  const unsigned char *const strat0, const unsigned s0steps,
                  const unsigned short *const strat1, const unsigned s1steps, const unsigned s1pairs,
                  unsigned *const glbSwp, unsigned long long *const glb_s, unsigned long long *const glb_b,
                  const int nthreads)
{
  if (routine >= 16u)
    return -1;
  const int full = (routine & 2u) != 0u, blk_ori = (routine & 8u) != 0u;
  if (!nrow || (nrow % 64u))
    return -2;
  if (!ncol || (ncol > nrow) || (ncol % 32u))
    return -3;
  if (nplus > ncol)
    return -4;
  if (!G)
    return -5;
  if (ldG < nrow)
    return -6;
  if (full) {
    if (!V)
      return -7;
    if (ldV < ncol)
      return -8;
  }
  if (!D)
    return -9;
  if (!glbSwp)
    return -10;
  if (!glb_s)
    return -11;
  if (!glb_b)
    return -12;

#ifdef _OPENMP
  if (nthreads > 0)
    omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif

  const unsigned nswp0 = blk_ori ? 1u : O_NSWEEP;
  if (full)
    for (unsigned c = 0u; c < ncol; ++c)
      for (unsigned r = 0u; r < ncol; ++r)
        V[(size_t)c * ldV + r] = (r == c) ? 1.0 : 0.0;

  const int gdefinite = (nplus ? ((nplus < ncol) ? 0 : +1) : -1);
  unsigned *const ps = (unsigned *)malloc(sizeof(unsigned) * 2u * s1pairs);
  if (!ps)
    return 1;

  *glb_s = 0ull;
  *glb_b = 0ull;
  unsigned blk_swp = 0u;
  while (blk_swp < O_NSWEEP) {
    unsigned long long cvg = 0ull;
    for (unsigned stp = 0u; stp < s1steps; ++stp) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1)
#endif
      for (int pr = 0; pr < (int)s1pairs; ++pr) {
        const unsigned iBlk = strat1[((size_t)stp * s1pairs + (unsigned)pr) * 2u + 0u];
        const unsigned jBlk = strat1[((size_t)stp * s1pairs + (unsigned)pr) * 2u + 1u];
        o_pair(routine, nrow, ncol, nplus, G, ldG, V, ldV, iBlk, jBlk, strat0, s0steps, nswp0, gdefinite,
               ps + 2u * (unsigned)pr, ps + 2u * (unsigned)pr + 1u);
      }
      for (unsigned pr = 0u; pr < s1pairs; ++pr) {
        const unsigned s = ps[2u * pr], b = ps[2u * pr + 1u];
        if (s) {
          if (b)
            cvg += (((unsigned long long)b) << 32u) | s;
          else /* 32-bit add to the low word */
            cvg = (cvg & 0xFFFFFFFF00000000ull) | (unsigned)((unsigned)cvg + s);
        }
      }
    }
    ++blk_swp;
    const unsigned cvg_s = (unsigned)cvg, cvg_b = (unsigned)(cvg >> 32u);
    *glb_s += cvg_s;
    *glb_b += cvg_b;
    if (!cvg_b)
      break;
  }
  free(ps);
  *glbSwp = blk_swp;
  gjxo_initD(G, ldG, nrow, ncol, nplus, D);
  return 0;
}

/* one outer step only (the timed sample of the CPU baseline) */
void gjxo_outer_step(const unsigned routine, const unsigned nrow, const unsigned ncol, const unsigned nplus,
                     double *const G, const unsigned ldG, double *const V, const unsigned ldV,
                     const unsigned char *const strat0, const unsigned s0steps,
                     const unsigned short *const strat1, const unsigned stp, const unsigned s1pairs,
                     unsigned long long *const cvg_s, unsigned long long *const cvg_b, const int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0)
    omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  const unsigned nswp0 = (routine & 8u) ? 1u : O_NSWEEP;
  const int gdefinite = (nplus ? ((nplus < ncol) ? 0 : +1) : -1);
  unsigned long long s_tot = 0ull, b_tot = 0ull;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : s_tot, b_tot)
#endif
  for (int pr = 0; pr < (int)s1pairs; ++pr) {
    unsigned s = 0u, b = 0u;
    const unsigned iBlk = strat1[((size_t)stp * s1pairs + (unsigned)pr) * 2u + 0u];
    const unsigned jBlk = strat1[((size_t)stp * s1pairs + (unsigned)pr) * 2u + 1u];
    o_pair(routine, nrow, ncol, nplus, G, ldG, V, ldV, iBlk, jBlk, strat0, s0steps, nswp0, gdefinite, &s, &b);
    s_tot += s;
    b_tot += b;
  }
  *cvg_s = s_tot;
  *cvg_b = b_tot;
}

/*
 * Strategy tables from strat.so: symbol "<name>%05u", bytes for n <= 256,
 * uint16 above (share/HypJacL.cu:84-120, share/my_utils.cu:50-61).  Returns
 * the number of steps copied into out ([steps][n/2][2] uint16), or < 0.
 */
int gjxo_load_strat(const char *const sdy, const char *const name, const unsigned n,
                    unsigned short *const out, const unsigned cap_entries)
{
  unsigned steps;
  if (!strcmp(name, "mmstep"))
    steps = n;
  else if (!strcmp(name, "BrentL") || !strcmp(name, "colcyc") || !strcmp(name, "cycloc") ||
           !strcmp(name, "rowcyc") || !strcmp(name, "cycwor"))
    steps = n - 1u;
  else
    return -1;
  if (!n || (n & 1u))
    return -2;
  const unsigned entries = steps * (n / 2u) * 2u;
  if (entries > cap_entries)
    return -3;
  void *const h = dlopen(sdy, RTLD_LAZY);
  if (!h)
    return -4;
  char sym[16];
  (void)snprintf(sym, sizeof(sym), "%s%05u", name, n);
  const void *const p = dlsym(h, sym);
  if (!p) {
    dlclose(h);
    return -5;
  }
  for (unsigned i = 0u; i < entries; ++i)
    out[i] = (n <= 256u) ? ((const unsigned char *)p)[i] : ((const unsigned short *)p)[i];
  dlclose(h);
  return (int)steps;
}
