// gjx_qr.cuh -- the pivot-block factor and inner sweep of the reference's
// alternative builds, selected at run time (gjx_set_variant):
//
//   variant 1 (-DUSE_QR): R of the pair [G_i G_j] by a Householder QR of its
//     first 32 rows and of every further 32-row chunk, each chunk's R merged
//     into the running R by Givens rotations along the diagonals
//     (share/device_code_common_QR.hpp:4-94, dQR32 at
//     share/device_code_common_Kepler.hpp:326-371, dGivens at
//     share/device_code_common_rotate.hpp:120-155);
//   variant 2 (-DUSE_DRMAC, implies USE_QR): in addition, the definite
//     sorting sweep measures each pair by its scaled norms and cosine
//     (share/device_code_cdsort_Drmac.hpp:4-316 with dNRM2_32 / dCOSA of
//     share/device_code_common_Kepler.hpp:76-324 and the scaling helpers of
//     share/device_code_common_scale.hpp:7-58).
//
// Every result has the reference's bits: the warp sums are the reference's
// butterfly (sum32), maxima and minima are exact in any order, and each
// product, quotient, square root and FMA is the reference's, in its order
// (its nvcc build contracts the two Givens products c a + s b, c b - s a into
// fma(c, a, s b) and fma(c, b, -(s a)); written out here).  A block pair is
// one CTA of 8 warps; lane x holds row x.
#pragma once

#include <cfloat>
#include <climits>

#include "gjx_device.cuh"

namespace gjx {

// share/HypJacL.hpp:55-90, the reference's decimal literals
constexpr double kMu = 1.4916681462400414314624091158735E-154;
constexpr double kNu = 2.370187977027293260705088939015E+153;
constexpr double kMuEps = 1.0020841800044863889980540256751E-292;
constexpr double kNu8 = 2.24711641857789464E+307;

// max |x| and min |x| (x != 0, else DBL_MAX) over the warp, broadcast
__device__ __forceinline__ double max32(double x)
{
  x = fabs(x);
#pragma unroll
  for (unsigned o = 16u; o; o >>= 1u)
    x = fmax(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

__device__ __forceinline__ double min32(double x)
{
  x = (x == 0.0) ? DBL_MAX : fabs(x);
#pragma unroll
  for (unsigned o = 16u; o; o >>= 1u)
    x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

// share/device_code_common_scale.hpp:7-58
__device__ __forceinline__ int find_scl(const double x, const double t)
{
  int x_n, t_n;
  const double x_m = frexp(x, &x_n);
  const double t_m = frexp(t, &t_n);
  return (x <= t) ? ((t_n - x_n) + (x_m < t_m)) : ((t_n - x_n) - (x_m > t_m));
}

__device__ __forceinline__ void normalize2(int &scl, double &ssq)
{
  const int e = ilogb(ssq);
  const int scl_ = e + (e & 1);
  scl += scl_;
  ssq = scalbn(ssq, -scl_);
}

__device__ __forceinline__ void sum_scl(const int s1, const int s2, const double x1, const double x2, int &s,
                                        double &x)
{
  const int cmp = (s1 < s2) ? -1 : (s2 < s1) ? 1 : (x1 < x2) ? -1 : (x2 < x1) ? 1 : 0;
  if (cmp <= 0) {
    s = s2;
    x = scalbn(x1, s1 - s2) + x2;
  }
  else {
    s = s1;
    x = scalbn(x2, s2 - s1) + x1;
  }
}

// the warp sum of the squares of this lane's |x| in one magnitude range
// (0: below mu, scaled by 2^scl; 1: [mu, nu]; 2: above nu, scaled)
__device__ __forceinline__ double ssq_range(const double x, const int range, const int scl)
{
  const double a = fabs(x);
  double v;
  if (range == 0)
    v = (a < kMu) ? scalbn(a, scl) : 0.0;
  else if (range == 1)
    v = ((a >= kMu) && (a <= kNu)) ? a : 0.0;
  else
    v = (a > kNu) ? scalbn(a, scl) : 0.0;
  return sum32(__dmul_rn(v, v));
}

// share/device_code_common_Kepler.hpp:210-268: ssq * 2^scl = sum of squares
__device__ __forceinline__ int ssq32(double &ssq, const double x)
{
  const double M = max32(x);
  if (M == 0.0) {
    ssq = 0.0;
    return INT_MIN;
  }
  const double m = min32(x);
  const bool lo = (m < kMu), hi = (M > kNu);
  int sc0, sc1, sc2, scl;
  double sq0, sq1, sq2;
  if (hi) {
    sc2 = find_scl(M, kNu);
    sq2 = ssq_range(x, 2, sc2);
    sc2 *= -2;
    if (m > kNu) {
      scl = sc2;
      ssq = sq2;
    }
    else {
      sc1 = 0;
      sq1 = ssq_range(x, 1, 0);
      if (sq1 > 0.0) {
        normalize2(sc1, sq1);
        normalize2(sc2, sq2);
        sum_scl(sc1, sc2, sq1, sq2, scl, ssq);
      }
      else {
        scl = sc2;
        ssq = sq2;
      }
    }
  }
  else if (lo) {
    sc0 = find_scl(m, kMu);
    sq0 = ssq_range(x, 0, sc0);
    sc0 *= -2;
    if (M < kMu) {
      scl = sc0;
      ssq = sq0;
    }
    else {
      sc1 = 0;
      sq1 = ssq_range(x, 1, 0);
      if (sq1 > 0.0) {
        normalize2(sc1, sq1);
        normalize2(sc0, sq0);
        sum_scl(sc0, sc1, sq0, sq1, scl, ssq);
      }
      else {
        scl = sc0;
        ssq = sq0;
      }
    }
  }
  else {
    scl = 0;
    ssq = sum32(__dmul_rn(x, x));
  }
  return scl;
}

// share/device_code_common_Kepler.hpp:278-283: the 2-norm of the warp's x
__device__ __forceinline__ double nrm2_32(const double x)
{
  double ssq;
  const int scl = ssq32(ssq, x) / 2;
  return scalbn(__dsqrt_rn(ssq), scl);
}

// share/device_code_common_Kepler.hpp:285-324: cos of the angle between the
// warp's x and y (norms Ap, Aq), guarded against over- and underflow
__device__ __forceinline__ double cosa_(const double Ap, const double Aq, const double x, const double y)
{
  bool big, small;
  if (Aq >= 1.0) {
    big = (__dmul_rn(Ap, Aq) >= DBL_MAX);
    small = false;
  }
  else {
    big = false;
    small = (__dmul_rn(Ap, Aq) <= kMuEps);
  }
  if (big) {
    const double z = (fabs(x) >= fabs(y)) ? __dmul_rn(__ddiv_rn(x, Ap), y) : __dmul_rn(__ddiv_rn(y, Ap), x);
    return __ddiv_rn(sum32(z), Aq);
  }
  if (small) {
    const double z = (fabs(x) >= fabs(y)) ? __dmul_rn(x, __ddiv_rn(y, Aq)) : __dmul_rn(y, __ddiv_rn(x, Aq));
    return __ddiv_rn(sum32(z), Ap);
  }
  return __ddiv_rn(__ddiv_rn(sum32(__dmul_rn(x, y)), Aq), Ap);
}

__device__ __forceinline__ double cosa(const double Ap, const double Aq, const double x, const double y)
{
  return (Ap >= Aq) ? cosa_(Ap, Aq, x, y) : cosa_(Aq, Ap, y, x);
}

// share/device_code_common_rotate.hpp:120-155
__device__ __forceinline__ void givens(const double f, const double g, double &c, double &s, double &r)
{
  const double f_ = fabs(f), g_ = fabs(g);
  if (f_ >= g_) {
    if (g_ == 0.0) {
      c = copysign(1.0, f);
      s = 0.0;
      r = f_;
    }
    else {
      const double g_f = __ddiv_rn(g_, f_);
      r = __dmul_rn(f_, __dsqrt_rn(__fma_rn(g_f, g_f, 1.0)));
      c = __ddiv_rn(f, r);
      s = __ddiv_rn(g, r);
    }
  }
  else {
    if (f_ == 0.0) {
      c = 0.0;
      s = copysign(1.0, g);
      r = g_;
    }
    else {
      const double f_g = __ddiv_rn(f_, g_);
      r = __dmul_rn(g_, __dsqrt_rn(__fma_rn(f_g, f_g, 1.0)));
      c = __ddiv_rn(f, r);
      s = __ddiv_rn(g, r);
    }
  }
}

// Householder QR of the 32 x 32 block A (column major) by the CTA: reflector
// k from column k (norm by nrm2_32), applied to columns k+1..31 (warp w
// takes columns k+1+w, k+9+w, ...), column k set to -beta e_k.  All warps
// compute the reflector; two barriers per column.
__device__ __forceinline__ void qr32_cta(double *const A, const unsigned warp, const unsigned x)
{
  for (unsigned k = 0u; k < 31u; ++k) {
    const double Axk = A[k * 32u + x];
    const double Axk_ = (x >= k) ? Axk : 0.0;
    const double nrm2 = nrm2_32(Axk_);
    double beta = 0.0, alpha_beta = 0.0, tau = 0.0;
    if (nrm2 > 0.0) {
      const double alpha = A[k * 32u + k];
      beta = copysign(nrm2, alpha);
      alpha_beta = alpha + beta;
      tau = __ddiv_rn(alpha_beta, beta);
    }
    __syncthreads(); // column k and A(k, k) are read
    if (nrm2 > 0.0) {
      const double Vxk = (x == k) ? 1.0 : ((x > k) ? __ddiv_rn(Axk_, alpha_beta) : 0.0);
      for (unsigned j = k + 1u + warp; j < 32u; j += 8u) {
        const double Axy = A[j * 32u + x];
        const double dp = sum32(__dmul_rn(Vxk, Axy));
        const double _tdp = -__dmul_rn(tau, dp);
        A[j * 32u + x] = __fma_rn(_tdp, Vxk, Axy);
      }
      if (warp == 0u)
        A[k * 32u + x] = (x == k) ? -beta : ((x > k) ? 0.0 : Axk);
    }
    __syncthreads();
  }
}

// share/device_code_common_QR.hpp:4-66: the triangular R1 merged into R0: in
// step k, lane x >= k rotates row x of R0 with row x - k of R1 so that
// R1(x-k, x) vanishes, in every column >= x (warp w takes columns w, w+8, ...)
__device__ __forceinline__ void peel_cta(double *const R0, double *const R1, const unsigned warp, const unsigned x)
{
  for (unsigned k = 0u; k < 32u; ++k) {
    const bool act = x >= k;
    const unsigned xk = x - k;
    double c = 0.0, s = 0.0, r = 0.0;
    if (act)
      givens(R0[x * 32u + x], R1[x * 32u + xk], c, s, r);
    __syncthreads(); // every lane's diagonal pair is read
    if (act)
      for (unsigned j = warp; j < 32u; j += 8u) {
        if (j > x) {
          const double a = R0[j * 32u + x], b = R1[j * 32u + xk];
          R0[j * 32u + x] = __fma_rn(c, a, __dmul_rn(s, b));
          R1[j * 32u + xk] = __fma_rn(c, b, -__dmul_rn(s, a));
        }
        else if (j == x) {
          R0[x * 32u + x] = r;
          R1[x * 32u + xk] = 0.0;
        }
      }
    __syncthreads();
  }
}

// share/device_code_common_QR.hpp:68-92 (dFactorize): R of the pair's rows
// into R (32 x 32, column major), W a 32 x 32 scratch
__device__ __forceinline__ void qr_factor_cta(const double *const Gi, const double *const Gj, const size_t ld,
                                              const unsigned nrow, double *const R, double *const W)
{
  const unsigned tid = threadIdx.x, warp = tid >> 5, x = tid & 31u;
  auto load = [&](double *const dst, const unsigned row0) {
    for (unsigned i = tid; i < 1024u; i += 256u) {
      const unsigned y = i >> 5, r = i & 31u;
      dst[i] = ((y < 16u) ? Gi + (size_t)y * ld : Gj + (size_t)(y - 16u) * ld)[row0 + r];
    }
  };
  load(R, 0u);
  __syncthreads();
  qr32_cta(R, warp, x);
  for (unsigned row0 = 32u; row0 < nrow; row0 += 32u) {
    load(W, row0);
    __syncthreads();
    qr32_cta(W, warp, x);
    peel_cta(R, W, warp, x);
  }
}

// share/device_code_cdsort_Drmac.hpp:4-316: the definite sorting sweep(s)
// with scaled norms and cosines (def = +1 descending, -1 ascending); warp w
// takes pairs w and w + 8 of each inner step, one after the other.  Counts as
// the reference's (small in blk_s, big in blk_b).
__device__ __forceinline__ void drmac_sweeps(double *const G, double *const V, const uint8_t *const s0,
                                             const unsigned s0steps, const unsigned nswp, const int def,
                                             unsigned *const red, const unsigned x, const unsigned w,
                                             unsigned &blk_s, unsigned &blk_b)
{
  blk_s = 0u;
  blk_b = 0u;
  for (unsigned swp = 0u; swp < nswp; ++swp) {
    unsigned ws = 0u, wb = 0u;
    for (unsigned step = 0u; step < s0steps; ++step) {
#pragma unroll 1
      for (unsigned h = 0u; h < 2u; ++h) {
        const unsigned y = w + 8u * h;
        const unsigned p = s0[(step * 16u + y) * 2u], q = s0[(step * 16u + y) * 2u + 1u];
        const double Gp = G[p * 32u + x], Gq = G[q * 32u + x], Vp = V[p * 32u + x], Vq = V[q * 32u + x];
        const double Ap = nrm2_32(Gp), Aq = nrm2_32(Gq), CosA = cosa(Ap, Aq, Gp, Gq);
        const int transf_s = (fabs(CosA) >= kMyTol);
        int transf_b = 0;
        if (transf_s) {
          const double Aq_p = __ddiv_rn(Aq, Ap), Ap_q = __ddiv_rn(Ap, Aq);
          const double ct2 = __ddiv_rn(Aq_p - Ap_q, scalbn(CosA, 1));
          if (ct2 <= kNu8) {
            const double CT2 = fabs(ct2);
            double c, t;
            if (CT2 < kSqrtHeps) {
              t = copysign(__drcp_rn(CT2 + 1.0), ct2);
              c = rsqrt_rn(__fma_rn(t, t, 1.0));
              transf_b = 1;
            }
            else if (CT2 >= kSqrt2Heps) {
              c = 1.0;
              t = copysign(__drcp_rn(scalbn(CT2, 1)), ct2);
            }
            else {
              t = copysign(__drcp_rn(CT2 + __dsqrt_rn(__fma_rn(CT2, CT2, 1.0))), ct2);
              c = rsqrt_rn(__fma_rn(t, t, 1.0));
              transf_b = (c < 1.0);
            }
            const double t_ = -t, tCosA = __dmul_rn(t, CosA), tCosA_ = -tCosA;
            const double Ap_ = __dmul_rn(Ap, __dsqrt_rn(__fma_rn(tCosA_, Aq_p, 1.0)));
            const double Aq_ = __dmul_rn(Aq, __dsqrt_rn(__fma_rn(tCosA, Ap_q, 1.0)));
            const bool keep = (def > 0) ? (Ap_ >= Aq_) : (Ap_ <= Aq_);
            const unsigned dp = keep ? p : q, dq = keep ? q : p;
            double np = __fma_rn(t_, Gq, Gp), nq = __fma_rn(t, Gp, Gq);
            double mp = __fma_rn(t_, Vq, Vp), mq = __fma_rn(t, Vp, Vq);
            if (transf_b) {
              np = __dmul_rn(c, np);
              nq = __dmul_rn(c, nq);
              mp = __dmul_rn(c, mp);
              mq = __dmul_rn(c, mq);
            }
            G[dp * 32u + x] = np;
            G[dq * 32u + x] = nq;
            V[dp * 32u + x] = mp;
            V[dq * 32u + x] = mq;
          }
          else if ((def > 0) ? (Ap >= Aq) : (Ap <= Aq)) {
            const double t_ = CosA, t = -t_;
            G[q * 32u + x] = __dmul_rn(Aq, __fma_rn(t, __ddiv_rn(Gp, Ap), __ddiv_rn(Gq, Aq)));
            V[p * 32u + x] = __fma_rn(t_, Vq, Vp);
            V[q * 32u + x] = __fma_rn(t, Vp, Vq);
          }
          else {
            const double t = CosA, t_ = -t;
            G[q * 32u + x] = __dmul_rn(Ap, __fma_rn(t_, __ddiv_rn(Gq, Aq), __ddiv_rn(Gp, Ap)));
            G[p * 32u + x] = Gq;
            V[q * 32u + x] = __fma_rn(t_, Vq, Vp);
            V[p * 32u + x] = __fma_rn(t, Vp, Vq);
          }
        }
        else if ((def > 0) ? (Ap < Aq) : (Aq < Ap)) {
          G[p * 32u + x] = Gq;
          G[q * 32u + x] = Gp;
          V[p * 32u + x] = Vq;
          V[q * 32u + x] = Vp;
        }
        if (x == 0u) {
          ws += (unsigned)transf_s;
          wb += (unsigned)transf_b;
        }
      }
      __syncthreads();
    }
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

} // namespace gjx
