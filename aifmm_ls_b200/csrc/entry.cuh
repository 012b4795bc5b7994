// entry.cuh -- device evaluation of one Lippmann-Schwinger matrix entry.
//
// Replaces LS2DTree::getMatrixEntry (LS/LS_Assembly.hpp:474-541) reached through
// userkernel::getMatrixEntry (kernel.hpp:130-136):
//   near (leaf j adjacent to leaf i, self included): table(dir)(ii, jj) * kappa^2 q(x_i) (+1 on the diagonal)
//   far: (i/4) kappa^2 q(x_i) sum_{n=-60}^{60} M(n+60, jj) (J_n(R) + i Y_n(R)) e^{i n theta}
//        R = kappa |x_i - c_j|, theta = atan2(x_i - c_j)
//   |entry| < 1e-16 -> 0.
// Bessel functions of integer order replace the reference's per-order Boost
// calls (LS/LS_Assembly.hpp:39-65): J_n by Miller's backward recurrence
// normalised with J_0 + 2 sum J_2k = 1; Y_0, Y_1 from the Neumann series in the
// same J values, then Y_n by forward recurrence.  (CUDA's y0/y1 carry an
// absolute error of ~1e-12 for large arguments, too coarse for 1e-14 entries.)
// The n and -n terms are paired, J_{-n} = (-1)^n J_n, Y_{-n} = (-1)^n Y_n.
#pragma once
#include "common.cuh"

#define AIFMM_SERIES 60

// W_n = M_n e^{in theta} + (-1)^n M_{-n} e^{-in theta}   (n >= 1), W_0 = M_0
__device__ __forceinline__ double2 series_w(const double2* __restrict__ Mc, int n, double2 e) {
  double2 mp = __ldg(&Mc[AIFMM_SERIES + n]);
  double2 mm = __ldg(&Mc[AIFMM_SERIES - n]);
  double2 a = cmul(mp, e);
  double2 b = cmul(mm, cconj(e));
  return (n & 1) ? csub(a, b) : cadd(a, b);
}

// sum_{n=-60}^{60} Mc[n+60] H_n(R) e^{in th}
// Pass 1 (downward): Miller's recurrence for J_N..J_0 accumulating sum J_n W_n,
// the normalisation J_0 + 2 sum J_2k and the Neumann sums that give Y_0, Y_1
// (Y_0 = (2/pi)[(ln(R/2)+gamma) J_0 - 2 sum_k (-1)^k J_2k / k],
//  Y_1 = -Y_0' = -(2/(pi R)) J_0 + (2/pi)[(ln(R/2)+gamma) J_1 + sum_k (-1)^k (J_2k-1 - J_2k+1) / k]).
// Pass 2 (upward): Y_n by forward recurrence accumulating sum Y_n W_n.
__device__ __forceinline__ double2 far_series(double R, double th, const double2* __restrict__ Mc) {
  const int NS = AIFMM_SERIES;
  double s1, c1;
  sincos(th, &s1, &c1);
  const double2 e1 = make_double2(c1, s1);
  const double2 e1c = cconj(e1);
  // ---- pass 1
  const double big = fmax((double)NS, R);
  int N = (int)(big + 24.0 + 10.0 * cbrt(big));
  N += (N & 1);
  double jp1 = 0.0, jcur = 1.0e-250;
  double norm = 2.0 * jcur;                          // N is even
  double S0 = ((N / 2) & 1 ? -jcur : jcur) / (N / 2);  // seed term of sum (-1)^k J_2k / k
  double S1 = 0.0;
  double2 acc = make_double2(0.0, 0.0);
  double sn, cn;
  sincos((double)NS * th, &sn, &cn);
  double2 en = make_double2(cn, sn);  // e^{i 60 th}
  for (int k = N; k >= 1; --k) {
    const double jnew = ((2.0 * k) / R) * jcur - jp1;  // J_{k-1}
    jp1 = jcur; jcur = jnew;
    const int m = k - 1;
    if ((m & 1) == 0) {
      norm += (m == 0 ? 1.0 : 2.0) * jnew;
      if (m >= 2) { const int kk = m >> 1; S0 += ((kk & 1) ? -jnew : jnew) / kk; }
    } else {
      const int k1 = (m + 1) >> 1, k2 = (m - 1) >> 1;
      S1 += ((k1 & 1) ? -jnew : jnew) / k1;
      if (k2 >= 1) S1 -= ((k2 & 1) ? -jnew : jnew) / k2;
    }
    if (m <= NS) {
      if (m < NS) {
        if (((m + 1) & 15) == 0) { sincos((double)(m + 1) * th, &sn, &cn); en = make_double2(cn, sn); }
        en = cmul(en, e1c);  // e^{i m th}
      }
      const double2 w = (m == 0) ? __ldg(&Mc[NS]) : series_w(Mc, m, en);
      acc.x = fma(jnew, w.x, acc.x); acc.y = fma(jnew, w.y, acc.y);
    }
    if (fabs(jcur) > 1.0e200) {  // rescale to stay in range
      jcur *= 1.0e-200; jp1 *= 1.0e-200; norm *= 1.0e-200;
      acc.x *= 1.0e-200; acc.y *= 1.0e-200; S0 *= 1.0e-200; S1 *= 1.0e-200;
    }
  }
  const double inorm = 1.0 / norm;
  const double2 SJ = make_double2(acc.x * inorm, acc.y * inorm);
  const double J0 = jcur * inorm, J1 = jp1 * inorm;
  S0 *= inorm; S1 *= inorm;
  const double kTwoOverPi = 0.63661977236758134307553505349;
  const double kEuler = 0.57721566490153286060651209008;
  const double lg = log(0.5 * R) + kEuler;
  double ym = kTwoOverPi * (lg * J0 - 2.0 * S0);
  double yc = -kTwoOverPi / R * J0 + kTwoOverPi * (lg * J1 + S1);
  // ---- pass 2
  const double2 w0 = __ldg(&Mc[NS]);
  double2 SY = make_double2(ym * w0.x, ym * w0.y);
  double2 e = e1;
  const double inv = 2.0 / R;
  for (int n = 1; n <= NS; ++n) {
    if ((n & 15) == 0) { sincos((double)n * th, &sn, &cn); e = make_double2(cn, sn); }
    const double2 w = series_w(Mc, n, e);
    SY.x = fma(yc, w.x, SY.x); SY.y = fma(yc, w.y, SY.y);
    const double yn = (n * inv) * yc - ym;
    ym = yc; yc = yn;
    e = cmul(e, e1);
  }
  // sum (J_n + i Y_n) W_n = SJ + i SY
  return make_double2(SJ.x - SY.y, SJ.y + SY.x);
}

__device__ __forceinline__ int near_dir(int dx, int dy) {
  // neighbour numbering of FMM2DTree (0=(-1,-1) 1=(0,-1) 2=(1,-1) 3=(1,0) 4=(1,1)
  // 5=(0,1) 6=(-1,1) 7=(-1,0)) and 8 = self, the index of LS_Assembly.hpp's N_centers
  const int tab[9] = {0, 1, 2, 7, 8, 3, 6, 5, 4};
  return tab[(dy + 1) * 3 + (dx + 1)];
}

// PHI = true: the system matrix A (findPhi, LS_Assembly.hpp:506-511, 528-533);
// PHI = false: the bare integral operator G of the same entry (no kappa^2 q(x_i)
// factor, no identity), the operator the reference applies to the solution to
// get the scattered field (hybrid.cpp:263-281).
template <bool PHI = true>
__device__ __forceinline__ double2 lsa_entry(int i, int j, const EntryCtx& c) {
  const int rank = c.rank;
  const int li = i / rank, ii = i - li * rank;
  const int lj = j / rank, jj = j - lj * rank;
  const int2 a = __ldg(&c.leafxy[li]);
  const int2 b = __ldg(&c.leafxy[lj]);
  const int dx = b.x - a.x, dy = b.y - a.y;
  const double qi = __ldg(&c.q[i]);
  if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1) {
    const int dir = near_dir(dx, dy);
    double2 e = __ldg(&c.nearT[(size_t)dir * rank * rank + ii + (size_t)jj * rank]);
    if (PHI) {
      // entry*kappa*kappa*q evaluated left to right (LS_Assembly.hpp:508)
      e.x = e.x * c.kappa; e.y = e.y * c.kappa;
      e.x = e.x * c.kappa; e.y = e.y * c.kappa;
      e.x = e.x * qi; e.y = e.y * qi;
      if (i == j) e.x = 1.0 + e.x;
    }
    if (hypot(e.x, e.y) < 1e-16) e = make_double2(0.0, 0.0);
    return e;
  }
  const double2 ri = __ldg(&c.pts[i]);
  const double2 cj = __ldg(&c.leafc[lj]);
  const double ddy = ri.y - cj.y, ddx = ri.x - cj.x;
  const double th = atan2(ddy, ddx);
  const double R = c.kappa * sqrt(ddy * ddy + ddx * ddx);
  double2 s = far_series(R, th, c.M + (size_t)jj * (2 * AIFMM_SERIES + 1));
  // *= I/4 (exact), then *= kappa*kappa*q (LS_Assembly.hpp:529-531)
  s = make_double2(-0.25 * s.y, 0.25 * s.x);
  if (PHI) {
    const double kq = c.kappa * c.kappa * qi;
    s.x *= kq; s.y *= kq;
    if (i == j) s.x += 1.0;
  }
  if (hypot(s.x, s.y) < 1e-16) s = make_double2(0.0, 0.0);
  return s;
}
