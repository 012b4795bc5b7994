/*
 * aifmm_oracle.cpp -- CPU oracle for the AIFMM-LS direct solver.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker for the CUDA product path.
 * It restates, in plain C++17 with OpenMP and without Eigen/Boost, the
 * reference's algorithm for the 2-D Lippmann-Schwinger AIFMM solver
 * (vaishna77/AIFMM_LS).  Each routine cites the reference file:line it follows.
 * Abbreviations: F = FMM2DTree_find_error.hpp, LSA = LS/LS_Assembly.hpp.
 *
 * Parity pinning: the Gauss-Legendre rule is checked bit-for-bit against the
 * reference's table and the Bessel values against mpmath fixtures.  The rest is
 * "parity unpinned" against the reference itself (it cannot be compiled here:
 * Eigen and Boost are absent) and is validated against a dense direct solve.
 *
 * Third-party semantics restated from their published descriptions:
 *  - Eigen ColPivHouseholderQR: Householder QR with column pivoting and the
 *    LAPACK xGEQP3 norm downdating of LAPACK Working Note 176; pivot = first
 *    remaining column of largest updated norm; rank() counts |R_ii| above
 *    threshold*max|R_ii|; solve() uses only the exactly-nonzero pivots.
 *  - Eigen PartialPivLU: Gaussian elimination with partial (row) pivoting.
 *  - Boost cyl_bessel_j / cyl_neumann for integer orders: recurrences below,
 *    J by Miller's backward recurrence normalised by J0 + 2 sum J_2k = 1 (or
 *    forward recurrence when x exceeds the order), Y by forward recurrence.
 */
#include "aifmm_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <utility>
#include <memory>
#include <vector>
#include <omp.h>

namespace {

using cd = std::complex<double>;
const cd I1(0.0, 1.0);
const double PI = 3.1415926535897932384;  // LSA:30
// relative tolerance under which two pivot candidates (ACA entries, QR column
// norms) are treated as equal; the first index then wins
const double PIVOT_TIE = 1e-11;

// --------------------------------------------------------------------------
// Dense complex matrix (column-major), zero-initialised.
// --------------------------------------------------------------------------
struct Mat {
  int r = 0, c = 0;
  std::vector<cd> a;
  Mat() {}
  Mat(int r_, int c_) : r(r_), c(c_), a((size_t)r_ * c_) {}
  cd& operator()(int i, int j) { return a[(size_t)i + (size_t)j * r]; }
  const cd& operator()(int i, int j) const { return a[(size_t)i + (size_t)j * r]; }
  long size() const { return (long)r * c; }
};

Mat mul(const Mat& A, const Mat& B) {
  Mat C(A.r, B.c);
  if (A.c != B.r) { fprintf(stderr, "oracle mul dim mismatch %dx%d * %dx%d\n", A.r, A.c, B.r, B.c); abort(); }
  for (int j = 0; j < B.c; ++j)
    for (int k = 0; k < A.c; ++k) {
      cd b = B(k, j);
      if (b == cd(0.0, 0.0)) continue;
      for (int i = 0; i < A.r; ++i) C(i, j) += A(i, k) * b;
    }
  return C;
}
Mat adj(const Mat& A) {
  Mat B(A.c, A.r);
  for (int j = 0; j < A.c; ++j)
    for (int i = 0; i < A.r; ++i) B(j, i) = std::conj(A(i, j));
  return B;
}
Mat sub(const Mat& A, const Mat& B) {
  if (A.r != B.r || A.c != B.c) { fprintf(stderr, "oracle sub dim mismatch %dx%d - %dx%d\n", A.r, A.c, B.r, B.c); abort(); }
  Mat C = A;
  for (size_t i = 0; i < C.a.size(); ++i) C.a[i] -= B.a[i];
  return C;
}
Mat neg(const Mat& A) {
  Mat C = A;
  for (auto& v : C.a) v = -v;
  return C;
}
Mat add(const Mat& A, const Mat& B) {
  if (A.r != B.r || A.c != B.c) { fprintf(stderr, "oracle add dim mismatch\n"); abort(); }
  Mat C = A;
  for (size_t i = 0; i < C.a.size(); ++i) C.a[i] += B.a[i];
  return C;
}
Mat block(const Mat& A, int i0, int j0, int rr, int cc) {
  Mat B(rr, cc);
  for (int j = 0; j < cc; ++j)
    for (int i = 0; i < rr; ++i) B(i, j) = A(i0 + i, j0 + j);
  return B;
}
Mat hcat(const Mat& A, const Mat& B) {
  if (A.r != B.r) { fprintf(stderr, "oracle hcat dim mismatch\n"); abort(); }
  Mat C(A.r, A.c + B.c);
  std::copy(A.a.begin(), A.a.end(), C.a.begin());
  std::copy(B.a.begin(), B.a.end(), C.a.begin() + A.a.size());
  return C;
}
double fnorm(const Mat& A) {
  double s = 0.0;
  for (const auto& v : A.a) s += std::norm(v);
  return std::sqrt(s);
}
Mat identity(int n) {
  Mat A(n, n);
  for (int i = 0; i < n; ++i) A(i, i) = 1.0;
  return A;
}

// --------------------------------------------------------------------------
// Householder QR with column pivoting (semantics of Eigen::ColPivHouseholderQR,
// restated from LAPACK xGEQP3 / LAWN 176 and Eigen's documented behaviour).
// --------------------------------------------------------------------------
struct ColPivQR {
  Mat qr;                 // R on/above the diagonal, Householder essentials below
  std::vector<cd> tau;    // reflector coefficients: G_k = I - tau_k v_k v_k^H
  std::vector<int> perm;  // A*P = Q*R; perm[i] = original column at position i
  int nzp = 0;            // exactly-nonzero pivots (used by solve)
  double maxpivot = 0.0;
  bool user_threshold = false;
  double thr = 0.0;

  explicit ColPivQR(const Mat& A) { compute(A); }

  void compute(const Mat& A) {
    qr = A;
    const int rows = A.r, cols = A.c, size = std::min(rows, cols);
    tau.assign(size, cd(0, 0));
    perm.resize(cols);
    for (int i = 0; i < cols; ++i) perm[i] = i;
    std::vector<double> nu(cols), nd(cols);
    double maxnorm = 0.0;
    for (int j = 0; j < cols; ++j) {
      double s = 0.0;
      for (int i = 0; i < rows; ++i) s += std::norm(qr(i, j));
      nu[j] = nd[j] = std::sqrt(s);
      if (j == 0 || nu[j] > maxnorm) maxnorm = nu[j];
    }
    const double eps = DBL_EPSILON;
    double thr_helper = rows > 0 ? (maxnorm * eps) * (maxnorm * eps) / rows : 0.0;
    const double downdate_thr = std::sqrt(eps);
    nzp = size;
    maxpivot = 0.0;
    for (int k = 0; k < size; ++k) {
      double mxn = 0.0;
      for (int j = k; j < cols; ++j) mxn = std::max(mxn, nu[j]);
      int big = k;
      for (int j = k; j < cols; ++j)
        if (nu[j] >= mxn * (1.0 - PIVOT_TIE)) { big = j; break; }
      double bigsq = nu[big] * nu[big];
      if (nzp == size && bigsq < thr_helper * (double)(rows - k)) nzp = k;
      if (big != k) {
        for (int i = 0; i < rows; ++i) std::swap(qr(i, k), qr(i, big));
        std::swap(nu[k], nu[big]);
        std::swap(nd[k], nd[big]);
        std::swap(perm[k], perm[big]);
      }
      // reflector for qr(k:rows, k)
      cd c0 = qr(k, k);
      double tailsq = 0.0;
      for (int i = k + 1; i < rows; ++i) tailsq += std::norm(qr(i, k));
      double beta;
      cd t;
      const double tiny = DBL_MIN;
      if (tailsq <= tiny && c0.imag() * c0.imag() <= tiny) {
        t = 0.0;
        beta = c0.real();
        for (int i = k + 1; i < rows; ++i) qr(i, k) = 0.0;
      } else {
        beta = std::sqrt(std::norm(c0) + tailsq);
        if (c0.real() >= 0.0) beta = -beta;
        cd den = c0 - beta;
        for (int i = k + 1; i < rows; ++i) qr(i, k) /= den;
        t = std::conj((beta - c0) / beta);
      }
      tau[k] = t;
      qr(k, k) = beta;
      if (std::abs(beta) > maxpivot) maxpivot = std::abs(beta);
      // apply G_k = I - t v v^H to the trailing columns
      for (int j = k + 1; j < cols; ++j) {
        cd w = qr(k, j);
        for (int i = k + 1; i < rows; ++i) w += std::conj(qr(i, k)) * qr(i, j);
        qr(k, j) -= t * w;
        for (int i = k + 1; i < rows; ++i) qr(i, j) -= t * qr(i, k) * w;
      }
      // norm downdate (LAWN 176)
      for (int j = k + 1; j < cols; ++j) {
        if (nu[j] != 0.0) {
          double tmp = std::abs(qr(k, j)) / nu[j];
          tmp = (1.0 + tmp) * (1.0 - tmp);
          if (tmp < 0.0) tmp = 0.0;
          double r = nu[j] / nd[j];
          double tmp2 = tmp * r * r;
          if (tmp2 <= downdate_thr) {
            double s = 0.0;
            for (int i = k + 1; i < rows; ++i) s += std::norm(qr(i, j));
            nd[j] = std::sqrt(s);
            nu[j] = nd[j];
          } else {
            nu[j] *= std::sqrt(tmp);
          }
        }
      }
    }
  }
  void setThreshold(double t) { user_threshold = true; thr = t; }
  double threshold() const {
    return user_threshold ? thr : (double)std::min(qr.r, qr.c) * DBL_EPSILON;
  }
  int rank() const {
    double pre = std::abs(maxpivot) * threshold();
    int res = 0;
    for (int i = 0; i < nzp; ++i) res += (std::abs(qr(i, i)) > pre);
    return res;
  }
  // c <- G_k c (rows k..), k = 0..len-1 in order  (computes Q^H c)
  void applyQH(Mat& C, int len) const {
    for (int k = 0; k < len; ++k) {
      const cd t = tau[k];
      for (int j = 0; j < C.c; ++j) {
        cd w = C(k, j);
        for (int i = k + 1; i < qr.r; ++i) w += std::conj(qr(i, k)) * C(i, j);
        C(k, j) -= t * w;
        for (int i = k + 1; i < qr.r; ++i) C(i, j) -= t * qr(i, k) * w;
      }
    }
  }
  // full unitary Q = G_0^H G_1^H ... G_{size-1}^H  (rows x rows)
  Mat householderQ() const {
    Mat Q = identity(qr.r);
    const int size = (int)tau.size();
    for (int k = size - 1; k >= 0; --k) {
      const cd t = std::conj(tau[k]);
      for (int j = 0; j < Q.c; ++j) {
        cd w = Q(k, j);
        for (int i = k + 1; i < qr.r; ++i) w += std::conj(qr(i, k)) * Q(i, j);
        Q(k, j) -= t * w;
        for (int i = k + 1; i < qr.r; ++i) Q(i, j) -= t * qr(i, k) * w;
      }
    }
    return Q;
  }
  Mat matrixR() const {
    Mat R(qr.r, qr.c);
    for (int j = 0; j < qr.c; ++j)
      for (int i = 0; i <= std::min(j, qr.r - 1); ++i) R(i, j) = qr(i, j);
    return R;
  }
  Mat solve(const Mat& B) const {
    Mat X(qr.c, B.c);
    if (nzp == 0) return X;
    Mat C = B;
    applyQH(C, nzp);
    for (int j = 0; j < C.c; ++j) {
      for (int i = nzp - 1; i >= 0; --i) {
        cd s = C(i, j);
        for (int l = i + 1; l < nzp; ++l) s -= qr(i, l) * C(l, j);
        C(i, j) = s / qr(i, i);
      }
    }
    for (int i = 0; i < nzp; ++i)
      for (int j = 0; j < C.c; ++j) X(perm[i], j) = C(i, j);
    return X;
  }
};

// Gaussian elimination with partial pivoting (Eigen::PartialPivLU semantics).
struct PartialLU {
  Mat lu;
  std::vector<int> piv;
  explicit PartialLU(const Mat& A) : lu(A), piv(A.r) {
    const int n = A.r;
    for (int k = 0; k < n; ++k) {
      int p = k;
      double best = std::abs(lu(k, k));
      for (int i = k + 1; i < n; ++i) {
        double v = std::abs(lu(i, k));
        if (v > best) { best = v; p = i; }
      }
      piv[k] = p;
      if (p != k)
        for (int j = 0; j < n; ++j) std::swap(lu(k, j), lu(p, j));
      cd d = lu(k, k);
      if (d != cd(0, 0))
        for (int i = k + 1; i < n; ++i) lu(i, k) /= d;
      for (int j = k + 1; j < n; ++j) {
        cd u = lu(k, j);
        for (int i = k + 1; i < n; ++i) lu(i, j) -= lu(i, k) * u;
      }
    }
  }
  Mat solve(const Mat& B) const {
    const int n = lu.r;
    Mat X = B;
    for (int k = 0; k < n; ++k)
      if (piv[k] != k)
        for (int j = 0; j < X.c; ++j) std::swap(X(k, j), X(piv[k], j));
    for (int j = 0; j < X.c; ++j) {
      for (int i = 0; i < n; ++i) {
        cd s = X(i, j);
        for (int l = 0; l < i; ++l) s -= lu(i, l) * X(l, j);
        X(i, j) = s;
      }
      for (int i = n - 1; i >= 0; --i) {
        cd s = X(i, j);
        for (int l = i + 1; l < n; ++l) s -= lu(i, l) * X(l, j);
        X(i, j) = s / lu(i, i);
      }
    }
    return X;
  }
};

// --------------------------------------------------------------------------
// Gauss-Legendre rule (reference table LS/Gauss_Legendre_Nodes_and_Weights.hpp,
// case 10 at :210; order: -x_0, +x_0, -x_1, +x_1, ... by increasing |x|).
// --------------------------------------------------------------------------
void gauss_legendre(int n, std::vector<double>& nodes, std::vector<double>& weights) {
  std::vector<long double> xs, ws;
  for (int i = 0; i < (n + 1) / 2; ++i) {
    long double x = cosl(PI * (i + 0.75L) / (n + 0.5L));
    long double pp = 0;
    for (int it = 0; it < 100; ++it) {
      long double p0 = 1.0L, p1 = x;
      for (int k = 2; k <= n; ++k) {
        long double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1; p1 = p2;
      }
      pp = n * (x * p1 - p0) / (x * x - 1.0L);
      long double dx = p1 / pp;
      x -= dx;
      if (fabsl(dx) < 1e-21L) break;
    }
    {
      long double p0 = 1.0L, p1 = x;
      for (int k = 2; k <= n; ++k) {
        long double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1; p1 = p2;
      }
      pp = n * (x * p1 - p0) / (x * x - 1.0L);
    }
    xs.push_back(x);  // decreasing positive roots
    ws.push_back(2.0L / ((1.0L - x * x) * pp * pp));
  }
  // order by increasing |x|
  std::vector<int> idx(xs.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = (int)i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return fabsl(xs[a]) < fabsl(xs[b]); });
  nodes.clear(); weights.clear();
  for (int id : idx) {
    long double x = fabsl(xs[id]);
    if (x < 1e-30L) { nodes.push_back(0.0); weights.push_back((double)ws[id]); continue; }
    nodes.push_back((double)(-x)); weights.push_back((double)ws[id]);
    nodes.push_back((double)x);    weights.push_back((double)ws[id]);
  }
}

// --------------------------------------------------------------------------
// Bessel functions of integer order (replaces LSA:39-65 besselJ/besselY).
// --------------------------------------------------------------------------
void bessel_jy_all(int nmax, double xd, double* J, double* Y) {
  const long double x = xd;
  // Y_0, Y_1 and forward recurrence (stable for Y)
  long double y0 = std::cyl_neumannl(0.0L, x), y1 = std::cyl_neumannl(1.0L, x);
  Y[0] = (double)y0;
  if (nmax >= 1) Y[1] = (double)y1;
  long double ym = y0, yc = y1;
  for (int n = 1; n < nmax; ++n) {
    long double yn = (2.0L * n / x) * yc - ym;
    ym = yc; yc = yn;
    Y[n + 1] = (double)yn;
  }
  if (x > (long double)nmax + 5.0L) {
    // forward recurrence for J is stable for n < x
    long double j0 = std::cyl_bessel_jl(0.0L, x), j1 = std::cyl_bessel_jl(1.0L, x);
    J[0] = (double)j0;
    if (nmax >= 1) J[1] = (double)j1;
    long double jm = j0, jc = j1;
    for (int n = 1; n < nmax; ++n) {
      long double jn = (2.0L * n / x) * jc - jm;
      jm = jc; jc = jn;
      J[n + 1] = (double)jn;
    }
    return;
  }
  // Miller's backward recurrence, normalised by J0 + 2*sum J_2k = 1
  const double big = std::max((double)nmax, xd);
  int N = (int)(big + 40.0 + 12.0 * std::cbrt(big + 1.0));
  if (N % 2) ++N;
  std::vector<long double> jj(N + 2, 0.0L);
  long double jp1 = 0.0L, jc = 1e-300L, sum = 0.0L;
  jj[N] = jc;
  for (int k = N; k >= 1; --k) {
    long double jm = (2.0L * k / x) * jc - jp1;
    jp1 = jc; jc = jm;
    jj[k - 1] = jm;
    if (fabsl(jm) > 1e300L) {  // rescale
      for (int t = k - 1; t <= N; ++t) jj[t] *= 1e-300L;
      jc *= 1e-300L; jp1 *= 1e-300L;
    }
  }
  for (int k = 0; k <= N; k += 2) sum += (k == 0 ? 1.0L : 2.0L) * jj[k];
  for (int n = 0; n <= nmax; ++n) J[n] = (double)(jj[n] / sum);
}

double besselJn_signed(int n, double x) {  // LSA:39-51 semantics for a single order
  int m = n < 0 ? -n : n;
  double v = std::cyl_bessel_j((double)m, x);
  if (n < 0 && (m % 2)) v = -v;
  return v;
}

// --------------------------------------------------------------------------
// Contrast functions (LS/LS_functions.hpp:1-120).
// --------------------------------------------------------------------------
struct P2 { double x, y; };

double q_gaussian(P2 r) { double R2 = r.x * r.x + r.y * r.y; return 1.5 * std::exp(-160.0 * R2); }
double q_multiple_gaussians(P2 r) {
  static const double cx[20] = {-1.17182014706864, -0.861066625441127, -1.14533939124057, -0.856639124568525,
    -0.620066350133170, -0.457064031294315, -0.482782006538245, -0.635070123186999, 0.108594058866164,
    -0.0315722590552472, -0.177274727610547, 0.0342987980936911, 0.369662097773613, 0.591444264226524,
    0.401225715100565, 0.666822699314234, 1.10327781188617, 0.827519268441487, 0.873411278211136, 1.09482906183464};
  static const double cy[20] = {-0.361066625441127, 0.0719520938231629, 0.354660608759432, 1.14336087543147,
    -1.12006635013317, -0.457064031294315, 0.364929876813001, 0.802261227250738, -0.394084977497864,
    -0.0315722590552472, 0.322725272389453, 1.03429879809369, -1.13033790222639, 0.0137164199764117,
    0.401225715100565, 1.16682269931423, -0.345187707108795, -0.172480731558513, 0.373411278211136, 1.09482906183464};
  double q = 0.0, a = 0.0013;
  for (int i = 0; i < 20; ++i) {
    double R2 = (r.x - cx[i]) * (r.x - cx[i]) + (r.y - cy[i]) * (r.y - cy[i]);
    q += 1.5 * std::exp(-R2 / a);
  }
  return q;
}
double q_flatbump(P2 r) { double R2 = r.x * r.x + r.y * r.y; return 0.5 * std::erfc(5.0 * (R2 - 1.0)); }
double q_cavity(P2 r) {
  double R = std::sqrt(r.x * r.x + r.y * r.y), th = std::atan2(r.y, r.x);
  return (1.0 - std::pow(std::sin(0.5 * th), 500)) * std::exp(-2000 * (0.1 - R * R) * (0.1 - R * R));
}
double q_lens(P2 r) { double R = std::sqrt(r.x * r.x + r.y * r.y); return 4 * (r.y - 0.1) * (1.0 - std::erf(25.0 * (R - 0.3))); }
double q_plasma(P2 r) {
  double C = 0.4987;
  double psi = 1.0 - (r.x - 0.15 * (1 - r.x * r.x)) * (r.x - 0.15 * (1 - r.x * r.x)) - C * (1.0 + 0.3 * r.x) * (1.0 + 0.3 * r.x) * r.y * r.y;
  const double a[5] = {0.45, 0.195, 0.51, 0.195, 0.63}, x[5] = {0.8, 0.54, -0.14, -0.5, 0.18}, y[5] = {0.0, -0.28, 0.7, -0.01, 0.8};
  if (psi <= 0.05) return 0.0;
  double g = 0.0;
  for (int i = 0; i < 5; ++i) {
    double t = (r.x - x[i]) * (r.x - x[i]) + (r.y - y[i]) * (r.y - y[i]);
    g += a[i] * std::exp(-t / 0.01);
  }
  return -1.5 * (psi - 0.05) - g * std::cos(0.9 * r.y);
}

double contrast(const orc_params& p, P2 r) {
  switch (p.q_kind) {
    case ORC_Q_GAUSSIAN160: return q_gaussian(r);
    case ORC_Q_MULTI_GAUSS: return q_multiple_gaussians(r);
    case ORC_Q_PLASMA: return q_plasma(r);
    case ORC_Q_FLATBUMP: return q_flatbump(r);
    case ORC_Q_CAVITY: return q_cavity(r);
    case ORC_Q_GAUSS_AW: { double R2 = r.x * r.x + r.y * r.y; return p.q_amp * std::exp(-p.q_width * R2); }
    case ORC_Q_DISK: { double R2 = r.x * r.x + r.y * r.y; return R2 < p.q_radius * p.q_radius ? p.q_amp : 0.0; }
    default: return q_lens(r);
  }
}

// --------------------------------------------------------------------------
// Adaptive tensor Gauss-Legendre quadrature over [-1,1]^2 (LS/domain2D.hpp:46-138).
// A panel is split into four; the parent is accepted when |I_parent - sum I_child|
// < eps (absolute, :111), otherwise each child is refined.  The integral is the
// sum of accepted panels' own estimates in depth-first order.
// --------------------------------------------------------------------------
struct GL10 {
  std::vector<double> x, w;
  GL10() { gauss_legendre(10, x, w); }
};
const GL10& gl10() { static GL10 g; return g; }

template <class F>
cd panel_integral(const F& f, double xc, double yc, double xr, double yr) {
  const GL10& g = gl10();
  double xn[10], yn[10];
  for (int l = 0; l < 10; ++l) { xn[l] = xc + xr * g.x[l]; yn[l] = yc + yr * g.x[l]; }
  cd s(0.0, 0.0);
  for (int m = 0; m < 10; ++m)
    for (int n = 0; n < 10; ++n) s += g.w[m] * g.w[n] * f(xn[m], yn[n]);
  s *= (xr * yr);
  return s;
}

template <class F>
void refine(const F& f, double xc, double yc, double xr, double yr, cd Ip, double eps, cd& acc) {
  double hx = 0.5 * xr, hy = 0.5 * yr;
  double cxs[4] = {xc - hx, xc + hx, xc + hx, xc - hx};
  double cys[4] = {yc - hy, yc - hy, yc + hy, yc + hy};
  cd Ic[4];
  for (int l = 0; l < 4; ++l) Ic[l] = panel_integral(f, cxs[l], cys[l], hx, hy);
  cd err = Ip;
  for (int l = 0; l < 4; ++l) err -= Ic[l];
  if (std::abs(err) < eps) { acc += Ip; return; }
  for (int l = 0; l < 4; ++l) refine(f, cxs[l], cys[l], hx, hy, Ic[l], eps, acc);
}

template <class F>
cd adaptive_integral(const F& f, double eps) {
  cd root = panel_integral(f, 0.0, 0.0, 1.0, 1.0);
  cd acc(0.0, 0.0);
  refine(f, 0.0, 0.0, 1.0, 1.0, root, eps, acc);
  return acc;
}

double chebT(double x, int n) { return std::cos(n * std::acos(x)); }  // LS/FarFieldInteraction.hpp:96-98

double round6(double v) {  // Eigen text output at default stream precision + read back (LSA:1178-1228)
  char buf[64];
  snprintf(buf, sizeof buf, "%.6g", v);
  return strtod(buf, nullptr);
}

struct Tables {
  int rank = 0, nb = 0;
  std::vector<cd> M;     // 121 x rank (column-major)
  std::vector<cd> near;  // 9 x (rank x rank), column-major per table
  std::vector<double> qpinv;  // NB x rank
};

std::vector<std::pair<int, int>> basis_list(int degree) {  // LS/FarFieldInteraction.hpp:46-54
  std::vector<std::pair<int, int>> v;
  for (int d = 0; d < degree; ++d)
    for (int a = 0; a < d + 1; ++a) v.push_back({a, d - a});
  return v;
}

std::vector<double> cheb1d(int n) {  // LSA:567-570
  std::vector<double> c(n);
  for (int k = 0; k < n; ++k) c[k] = -std::cos((k + 0.5) / n * PI);
  return c;
}

// pseudo-inverse of the full-column-rank Chebyshev Vandermonde Q (rank x NB)
// (LS/FarFieldInteraction.hpp:138-150) via Householder least squares.
std::vector<double> q_pinv(int n_cheb, int degree) {
  auto bl = basis_list(degree);
  auto c = cheb1d(n_cheb);
  int rank = n_cheb * n_cheb, nb = (int)bl.size();
  Mat Q(rank, nb);
  for (int i = 0; i < rank; ++i) {
    double x = c[i % n_cheb], y = c[i / n_cheb];
    for (int l = 0; l < nb; ++l) Q(i, l) = chebT(x, bl[l].first) * chebT(y, bl[l].second);
  }
  ColPivQR qr(Q);
  Mat X = qr.solve(identity(rank));  // least-squares solution = pinv for full column rank
  std::vector<double> out((size_t)nb * rank);
  for (int j = 0; j < rank; ++j)
    for (int l = 0; l < nb; ++l) out[l + (size_t)j * nb] = X(l, j).real();
  return out;
}

Tables compute_tables(const orc_params& p, bool do_round) {
  Tables T;
  const int n = p.n_cheb, rank = n * n;
  auto bl = basis_list(p.degree);
  const int nb = (int)bl.size();
  T.rank = rank; T.nb = nb;
  T.qpinv = q_pinv(n, p.degree);
  std::vector<double> rad(p.depth + 2);
  rad[0] = p.L;
  for (int j = 1; j < (int)rad.size(); ++j) rad[j] = rad[j - 1] / 2.0;
  const double rl = rad[p.depth];
  const double kappa = p.kappa;
  const double eps = 1e-7;  // LS/FarFieldInteraction.hpp:37, LS/NearFieldInteraction1.hpp:112
  // far field C (121 x NB) at the leaf level (LS/FarFieldInteraction.hpp:115-135)
  std::vector<cd> C((size_t)121 * nb);
#pragma omp parallel for schedule(dynamic)
  for (int t = 0; t < 121 * nb; ++t) {
    int nn = t / nb - 60, l = t % nb;
    int a = bl[l].first, b = bl[l].second;
    auto f = [&](double x, double y) -> cd {
      double R2 = x * x + y * y;
      double normX = std::sqrt(R2);
      double argJ = kappa * rl * normX;
      double th = std::atan2(y, x);
      cd e = std::exp(-I1 * double(nn) * th);
      return besselJn_signed(nn, argJ) * e * chebT(x, a) * chebT(y, b);
    };
    cd integral = adaptive_integral(f, eps);
    C[(size_t)(nn + 60) + (size_t)l * 121] = rl * rl * integral;
  }
  T.M.assign((size_t)121 * rank, cd(0, 0));
  for (int j = 0; j < rank; ++j)
    for (int r = 0; r < 121; ++r) {
      cd s(0, 0);
      for (int l = 0; l < nb; ++l) s += C[(size_t)r + (size_t)l * 121] * T.qpinv[l + (size_t)j * nb];
      T.M[(size_t)r + (size_t)j * 121] = s;
    }
  // near field colleague tables (LSA:1290-1343, LS/NearFieldInteraction1.hpp:98-128)
  const double Nc[9][2] = {{-2, -2}, {0, -2}, {2, -2}, {2, 0}, {2, 2}, {0, 2}, {-2, 2}, {-2, 0}, {0, 0}};
  auto c = cheb1d(n);
  std::vector<cd> V((size_t)9 * rank * nb);
#pragma omp parallel for schedule(dynamic)
  for (int t = 0; t < 9 * rank * nb; ++t) {
    int dir = t / (rank * nb), i = (t / nb) % rank, l = t % nb;
    double cbx = Nc[dir][0] * rl, cby = Nc[dir][1] * rl;
    double ax = rl * c[i % n] + 0.0, ay = rl * c[i / n] + 0.0;
    double Xx = (ax - cbx) / rl, Xy = (ay - cby) / rl;
    int a = bl[l].first, b = bl[l].second;
    auto f = [&](double x, double y) -> cd {
      double R2 = (Xx - x) * (Xx - x) + (Xy - y) * (Xy - y);
      double R = std::sqrt(R2);
      double arg = kappa * rl * R;
      cd h(std::cyl_bessel_j(0.0, arg), std::cyl_neumann(0.0, arg));
      return h * chebT(x, a) * chebT(y, b);
    };
    V[(size_t)t] = adaptive_integral(f, eps);
  }
  T.near.assign((size_t)9 * rank * rank, cd(0, 0));
  for (int dir = 0; dir < 9; ++dir)
    for (int j = 0; j < rank; ++j)
      for (int i = 0; i < rank; ++i) {
        cd s(0, 0);
        for (int l = 0; l < nb; ++l) {
          cd v = V[(size_t)dir * rank * nb + (size_t)i * nb + l];
          cd vt = v * I1 * rl * rl / 4.0;
          s += vt * T.qpinv[l + (size_t)j * nb];
        }
        T.near[(size_t)dir * rank * rank + i + (size_t)j * rank] = s;
      }
  if (do_round) {
    for (auto& v : T.M) v = cd(round6(v.real()), round6(v.imag()));
    for (auto& v : T.near) v = cd(round6(v.real()), round6(v.imag()));
  }
  return T;
}

// --------------------------------------------------------------------------
// Problem: geometry, matrix entries (LSA:474-541) and the AIFMM solver (F).
// --------------------------------------------------------------------------
struct Box {
  int neighbors[8];
  int inner[16];
  int outer[24];
  bool Eliminated = false;
  int NumMultipoles = 0, NumLocals = 0;
  std::vector<int> chargeLocations;
  std::vector<int> in_check, in_charge, out_check, out_charge;
  Mat Ac, Ar, L2P, P2M, L2P_f, L2M_f;
  std::map<int, Mat> M2L, P2P, M2P, P2L, P2M_f, M2M_f;
  Mat particle_rhs, multipole_rhs, local_rhs;
  Mat particles, multipoles, locals;
  int rank_in_aca = 0, rank_out_aca = 0;
  // the L2P_f of neighbour n formed when this box was eliminated, kept for a
  // solve with new right-hand sides against the same factors (orc_solve_again)
  Mat Lf[8];
};

// neighbour numbering of F:11-74 / F:168-1046: 0=(-1,-1) 1=(0,-1) 2=(1,-1)
// 3=(1,0) 4=(1,1) 5=(0,1) 6=(-1,1) 7=(-1,0)
const int NB_DX[8] = {-1, 0, 1, 1, 1, 0, -1, -1};
const int NB_DY[8] = {-1, -1, -1, 0, 1, 1, 1, 0};

// counter-clockwise ring position of offset (dx,dy) on the ring of radius d,
// starting at (-d,-d): this is the inner (d=2) / outer (d=3) slot numbering of
// the interaction lists assigned in F:168-1046.
int ring_slot(int dx, int dy, int d) {
  if (dy == -d) return dx + d;                 // bottom edge, left to right
  if (dx == d) return 2 * d + (dy + d);        // right edge, bottom to top
  if (dy == d) return 4 * d + (d - dx);        // top edge, right to left
  return 6 * d + (d - dy);                     // left edge, top to bottom
}

struct Problem {
  orc_params p;
  Tables T;
  int depth, rank, nleaf1d, N;
  std::vector<double> rad;
  std::vector<P2> pts;
  std::vector<double> q;     // contrast at points
  std::vector<P2> leafc;     // leaf centres
  std::vector<std::vector<Box>> tree;
  std::vector<int> nBoxes;
  double tol;
  std::vector<std::pair<int, int>> P2Pq, P2L_M2Pq;
  int nrhs = 1;
  double perturb = 0.0;        // relative entry perturbation (sensitivity studies only)
  bool full_compress = false;  // eliminate_phase (F:2374) instead of the driver's _efficient
  // Reorderings that the GPU solver uses, restated here so that tests can show
  // they change no bit of the result (test-only; 0 = the reference's order):
  //   1: back substitution in waves of mutually non-adjacent boxes;
  //   2: the factorisation of P2P[k][k] and its solves with the right-hand side
  //      and the neighbour blocks before the recompressions of step k;
  //   4: the factorisation of L2M_f and its solves before the x-phase fill-ins.
  int schedule = 0;
  long ncompress = 0;
  struct XEarly { bool on = false; std::unique_ptr<ColPivQR> qr; Mat Xb; Mat S[8]; } xe;
  struct ZEarly { bool on = false; Mat Yneg, Yrhs, Z[8]; } ze;

  static void box_xy(int k, int level, int& ix, int& iy) {
    ix = iy = 0;
    for (int l = 0; l < level; ++l) {
      int c = (k >> (2 * (level - 1 - l))) & 3;
      ix = 2 * ix + ((c == 1 || c == 2) ? 1 : 0);
      iy = 2 * iy + ((c >= 2) ? 1 : 0);
    }
  }
  static int box_index(int ix, int iy, int level) {
    int k = 0;
    for (int l = level - 1; l >= 0; --l) {
      int bx = (ix >> l) & 1, by = (iy >> l) & 1;
      int c = by ? (bx ? 2 : 3) : (bx ? 1 : 0);
      k = 4 * k + c;
    }
    return k;
  }

  Problem(const orc_params& pp, const Tables& TT) : p(pp), T(TT) {
    depth = p.depth;
    rank = p.n_cheb * p.n_cheb;
    nleaf1d = 1 << depth;
    rad.resize(depth + 2);
    rad[0] = p.L;
    for (int j = 1; j < (int)rad.size(); ++j) rad[j] = rad[j - 1] / 2.0;
    // uniform quadtree, Morton order (LSA:808-890), leaf centres
    int nleaf = 1 << (2 * depth);
    leafc.resize(nleaf);
    for (int k = 0; k < nleaf; ++k) {
      P2 cc = {0.0, 0.0};
      double r = p.L;
      for (int l = 0; l < depth; ++l) {
        int c = (k >> (2 * (depth - 1 - l))) & 3;
        if (c == 0) { cc.x = cc.x - 0.5 * r; cc.y = cc.y - 0.5 * r; }
        else if (c == 1) { cc.x = cc.x + 0.5 * r; cc.y = cc.y - 0.5 * r; }
        else if (c == 2) { cc.x = cc.x + 0.5 * r; cc.y = cc.y + 0.5 * r; }
        else { cc.x = cc.x - 0.5 * r; cc.y = cc.y + 0.5 * r; }
        r = 0.5 * r;
      }
      leafc[k] = cc;
    }
    // grid points (LSA:1074-1087): local index y*n + x
    auto c = cheb1d(p.n_cheb);
    N = nleaf * rank;
    pts.resize(N);
    q.resize(N);
    for (int k = 0; k < nleaf; ++k)
      for (int j = 0; j < p.n_cheb; ++j)
        for (int i = 0; i < p.n_cheb; ++i) {
          P2 t;
          t.x = rad[depth] * c[i] + leafc[k].x;
          t.y = rad[depth] * c[j] + leafc[k].y;
          pts[(size_t)k * rank + j * p.n_cheb + i] = t;
        }
    for (int i = 0; i < N; ++i) q[i] = contrast(p, pts[i]);
    tol = std::pow(10, -1.0 * p.tol_pow);
  }

  cd entry(int i, int j) const {
    cd e = entry0(i, j);
    if (perturb != 0.0) {
      // deterministic pseudo-random relative perturbation in [-perturb, perturb]
      unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ull ^ ((unsigned long long)j + 0x632BE59BD9B4E019ull) * 0xBF58476D1CE4E5B9ull;
      h ^= h >> 31; h *= 0x94D049BB133111EBull; h ^= h >> 29;
      double u = (double)(h >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
      e *= (1.0 + perturb * u);
    }
    return e;
  }
  // LSA:474-541.  phi = the kernel's findPhi switch: true for the system matrix,
  // false for the bare operator G used for the scattered field (LSA:506-511, 528-533)
  cd entry0(int i, int j, bool phi = true) const {
    const int li = i / rank, ii = i % rank, lj = j / rank, jj = j % rank;
    int xi, yi, xj, yj;
    box_xy(li, depth, xi, yi);
    box_xy(lj, depth, xj, yj);
    int dx = xj - xi, dy = yj - yi;
    const P2 ri = pts[i];
    if (std::abs(dx) <= 1 && std::abs(dy) <= 1) {
      int dir = 8;
      for (int d = 0; d < 8; ++d)
        if (NB_DX[d] == dx && NB_DY[d] == dy) dir = d;
      cd e = T.near[(size_t)dir * rank * rank + ii + (size_t)jj * rank];
      if (phi) {
        e = e * p.kappa * p.kappa * q[i];  // LSA:508, evaluated left to right
        if (i == j) e = 1.0 + e;
      }
      if (std::abs(e) < 1e-16) e = 0.0;
      return e;
    }
    const P2 cj = leafc[lj];
    double th = std::atan2(ri.y - cj.y, ri.x - cj.x);
    double R2 = (ri.y - cj.y) * (ri.y - cj.y) + (ri.x - cj.x) * (ri.x - cj.x);
    double R = p.kappa * std::sqrt(R2);
    double J[61], Y[61], cs[61], sn[61];
    bessel_jy_all(60, R, J, Y);
    for (int n = 0; n <= 60; ++n) { cs[n] = std::cos(n * th); sn[n] = std::sin(n * th); }
    cd s(0.0, 0.0);
    const cd* Mc = &T.M[(size_t)jj * 121];
    for (int n = -60; n <= 60; ++n) {
      int m = n < 0 ? -n : n;
      double sg = (n < 0 && (m & 1)) ? -1.0 : 1.0;
      cd h(sg * J[m], sg * Y[m]);
      cd e(cs[m], n < 0 ? -sn[m] : sn[m]);
      cd t = h * e;
      s += Mc[n + 60] * t;
    }
    s *= I1 / 4.0;
    if (phi) {
      s *= p.kappa * p.kappa * q[i];  // LSA:531
      if (i == j) s += 1.0;
    }
    if (std::abs(s) < 1e-16) s = 0.0;
    return s;
  }

  std::vector<cd> getRow(int i, const std::vector<int>& cols) const {
    std::vector<cd> r(cols.size());
#pragma omp parallel for if (cols.size() > 64)
    for (int k = 0; k < (int)cols.size(); ++k) r[k] = entry(i, cols[k]);
    return r;
  }
  std::vector<cd> getCol(int j, const std::vector<int>& rows) const {
    std::vector<cd> c(rows.size());
#pragma omp parallel for if (rows.size() > 64)
    for (int k = 0; k < (int)rows.size(); ++k) c[k] = entry(rows[k], j);
    return c;
  }
  Mat getMatrix(const std::vector<int>& rows, const std::vector<int>& cols) const {
    Mat A((int)rows.size(), (int)cols.size());
#pragma omp parallel for collapse(2) if (rows.size() * cols.size() > 256)
    for (int j = 0; j < (int)cols.size(); ++j)
      for (int i = 0; i < (int)rows.size(); ++i) A(i, j) = entry(rows[i], cols[j]);
    return A;
  }

  // ---------------- tree and interaction lists (F:127-1070) ----------------
  void createTree() {
    tree.assign(depth + 1, {});
    nBoxes.assign(depth + 1, 0);
    for (int j = 0; j <= depth; ++j) {
      nBoxes[j] = 1 << (2 * j);
      tree[j].resize(nBoxes[j]);
      int n1 = 1 << j;
      for (int k = 0; k < nBoxes[j]; ++k) {
        Box& b = tree[j][k];
        for (int& v : b.neighbors) v = -1;
        for (int& v : b.inner) v = -1;
        for (int& v : b.outer) v = -1;
        if (j == 0) continue;
        int x, y;
        box_xy(k, j, x, y);
        for (int d = 0; d < 8; ++d) {
          int nx = x + NB_DX[d], ny = y + NB_DY[d];
          if (nx >= 0 && ny >= 0 && nx < n1 && ny < n1) b.neighbors[d] = box_index(nx, ny, j);
        }
        if (j < 2) continue;
        // interaction list: children of the parent's neighbours that are not
        // neighbours (distance 2 -> inner ring, distance 3 -> outer ring)
        int px = x / 2, py = y / 2;
        for (int ddy = -1; ddy <= 1; ++ddy)
          for (int ddx = -1; ddx <= 1; ++ddx) {
            if (ddx == 0 && ddy == 0) continue;
            int qx = px + ddx, qy = py + ddy;
            if (qx < 0 || qy < 0 || qx >= n1 / 2 || qy >= n1 / 2) continue;
            for (int cy = 0; cy < 2; ++cy)
              for (int cx = 0; cx < 2; ++cx) {
                int ox = 2 * qx + cx - x, oy = 2 * qy + cy - y;
                int d = std::max(std::abs(ox), std::abs(oy));
                int id = box_index(2 * qx + cx, 2 * qy + cy, j);
                if (d == 2) b.inner[ring_slot(ox, oy, 2)] = id;
                else if (d == 3) b.outer[ring_slot(ox, oy, 3)] = id;
              }
          }
      }
    }
    // leaf charge locations (F:1072-1090)
    for (int k = 0; k < nBoxes[depth]; ++k) {
      auto& cl = tree[depth][k].chargeLocations;
      cl.resize(rank);
      for (int i = 0; i < rank; ++i) cl[i] = k * rank + i;
    }
  }

  // ---------------- ACA (ACA.hpp:368-577) ----------------
  static void maxAbs(const std::vector<cd>& v, const std::set<int>& allowed, int& index) {
    // ACA.hpp:27-40: first maximum of |v| over allowed indices in ascending order.
    // Magnitudes within PIVOT_TIE (relative) of the maximum count as tied, so that
    // mathematically equal candidates (mirror-symmetric grids and contrasts) are
    // resolved by index rather than by rounding noise.
    if (allowed.empty()) { index = 0; return; }
    double mx = 0.0;
    for (int i : allowed) mx = std::max(mx, std::abs(v[i]));
    const double cut = mx * (1.0 - PIVOT_TIE);
    for (int i : allowed)
      if (std::abs(v[i]) >= cut) { index = i; return; }
    index = *allowed.begin();
  }
  static cd dotc(const std::vector<cd>& a, const std::vector<cd>& b) {
    cd s(0, 0);
    for (size_t i = 0; i < a.size(); ++i) s += std::conj(a[i]) * b[i];
    return s;
  }
  static double vnorm(const std::vector<cd>& a) {
    double s = 0;
    for (auto& v : a) s += std::norm(v);
    return std::sqrt(s);
  }

  void aca(const std::vector<int>& rowsI, const std::vector<int>& colsI, std::vector<int>& row_bases,
           std::vector<int>& col_bases, int& rank_out, Mat& Ac, Mat& Ar) const {
    const double tol_robust = 1e-12;  // ACA.hpp:23
    const double tol_ACA = tol;
    int N1 = (int)rowsI.size(), N2 = (int)colsI.size();
    std::vector<std::vector<cd>> Uvec, Vvec, AcVec, ArVec;
    int cr = 0;
    int mn = std::min(N1, N2);
    std::set<int> rem_r, rem_c;
    for (int l = 0; l < N1; ++l) rem_r.insert(l);
    for (int l = 0; l < N2; ++l) rem_c.insert(l);
    std::vector<cd> row, col, u, v;
    int row_index = 0, col_index = 0;
    if (N1 < N2) {
      int l;
      for (l = 0; l < N1; ++l) {
        row_index = l;
        row = getRow(rowsI[row_index], colsI);
        maxAbs(row, rem_c, col_index);
        if (std::abs(row[col_index]) > tol_robust) break;
      }
      if (l == N1) { rank_out = 0; Ac = Mat(N1, 0); Ar = Mat(0, N2); return; }
      v.resize(N2);
      for (int s = 0; s < N2; ++s) v[s] = row[s] / row[col_index];
      row_bases.push_back(row_index);
      col_bases.push_back(col_index);
      col = getCol(colsI[col_index], rowsI);
      u = col;
      Uvec.push_back(u); Vvec.push_back(v);
      AcVec.push_back(col); ArVec.push_back(row);
      rem_c.erase(col_index); rem_r.erase(row_index);
      cr = 1;
      double normS = 0.0, prev = DBL_MAX;
      maxAbs(col, rem_r, row_index);
      while (std::abs(row[col_index]) > tol_ACA && std::abs(col[row_index]) > tol_ACA &&
             std::abs(prev - normS) >= tol_ACA * prev && cr < mn) {
        row_bases.push_back(row_index);
        row = getRow(rowsI[row_index], colsI);
        std::vector<cd> row_temp = row;
        for (int l2 = 0; l2 < cr; ++l2)
          for (int s = 0; s < N2; ++s) row[s] -= Uvec[l2][row_index] * Vvec[l2][s];
        maxAbs(row, rem_c, col_index);
        col_bases.push_back(col_index);
        for (int s = 0; s < N2; ++s) v[s] = row[s] / row[col_index];
        col = getCol(colsI[col_index], rowsI);
        std::vector<cd> col_temp = col;
        for (int l2 = 0; l2 < cr; ++l2)
          for (int s = 0; s < N1; ++s) col[s] -= Vvec[l2][col_index] * Uvec[l2][s];
        u = col;
        if (vnorm(u) < tol_robust || vnorm(v) < tol_robust) {
          row_bases.pop_back(); col_bases.pop_back();
          break;
        }
        Uvec.push_back(u); Vvec.push_back(v);
        AcVec.push_back(col_temp); ArVec.push_back(row_temp);
        ++cr;
        rem_c.erase(col_index); rem_r.erase(row_index);
        if (cr != 2) prev = normS;
        double un = vnorm(u), vn = vnorm(v);
        normS = normS * normS + (un * vn) * (un * vn);
        for (int l2 = 0; l2 < cr; ++l2) normS += 2 * std::abs(dotc(Uvec[l2], u) * dotc(Vvec[l2], v));
        normS = std::sqrt(normS);
        maxAbs(col, rem_r, row_index);
      }
    } else {
      int l;
      for (l = 0; l < N2; ++l) {
        col_index = l;
        col = getCol(colsI[col_index], rowsI);
        maxAbs(col, rem_r, row_index);
        if (std::abs(col[row_index]) > tol_robust) break;
      }
      if (l == N2) { rank_out = 0; Ac = Mat(N1, 0); Ar = Mat(0, N2); return; }
      col_bases.push_back(col_index);
      v.resize(N1);
      for (int s = 0; s < N1; ++s) v[s] = col[s] / col[row_index];
      row_bases.push_back(row_index);
      row = getRow(rowsI[row_index], colsI);
      u = row;
      Uvec.push_back(u); Vvec.push_back(v);
      AcVec.push_back(col); ArVec.push_back(row);
      cr = 1;
      rem_r.erase(row_index); rem_c.erase(col_index);
      double normS = 0.0, prev = DBL_MAX;
      maxAbs(row, rem_c, col_index);
      while (std::abs(row[col_index]) > tol_ACA && std::abs(col[row_index]) > tol_ACA &&
             std::abs(prev - normS) >= tol_ACA * prev && cr < mn) {
        col_bases.push_back(col_index);
        col = getCol(colsI[col_index], rowsI);
        std::vector<cd> col_temp = col;
        for (int l2 = 0; l2 < cr; ++l2)
          for (int s = 0; s < N1; ++s) col[s] -= Uvec[l2][col_index] * Vvec[l2][s];
        maxAbs(col, rem_r, row_index);
        row_bases.push_back(row_index);
        for (int s = 0; s < N1; ++s) v[s] = col[s] / col[row_index];
        row = getRow(rowsI[row_index], colsI);
        std::vector<cd> row_temp = row;
        for (int l2 = 0; l2 < cr; ++l2)
          for (int s = 0; s < N2; ++s) row[s] -= Vvec[l2][row_index] * Uvec[l2][s];
        u = row;
        if (vnorm(u) < tol_robust || vnorm(v) < tol_robust) {
          col_bases.pop_back(); row_bases.pop_back();
          break;
        }
        Uvec.push_back(u); Vvec.push_back(v);
        AcVec.push_back(col_temp); ArVec.push_back(row_temp);
        ++cr;
        rem_r.erase(row_index); rem_c.erase(col_index);
        if (cr != 2) prev = normS;
        double un = vnorm(u), vn = vnorm(v);
        normS = normS * normS + (un * vn) * (un * vn);
        for (int l2 = 0; l2 < cr; ++l2) normS += 2 * std::abs(dotc(Uvec[l2], u) * dotc(Vvec[l2], v));
        normS = std::sqrt(normS);
        maxAbs(row, rem_c, col_index);
      }
    }
    rank_out = cr;
    Ac = Mat(N1, cr);
    Ar = Mat(cr, N2);
    for (int i = 0; i < cr; ++i) {
      for (int s = 0; s < N1; ++s) Ac(s, i) = AcVec[i][s];
      for (int s = 0; s < N2; ++s) Ar(i, s) = ArVec[i][s];
    }
  }

  // ---------------- bases (F:1105-1336) ----------------
  void rows_for(int j, int k, bool incoming_check, std::vector<int>& out) const {
    // F:1182-1228: the leaf's own points, else the children's incoming check
    // points (incoming_check) or outgoing charge points
    if (j == depth) {
      out.insert(out.end(), tree[j][k].chargeLocations.begin(), tree[j][k].chargeLocations.end());
    } else {
      for (int c = 0; c < 4; ++c) {
        const Box& ch = tree[j + 1][4 * k + c];
        const auto& v = incoming_check ? ch.in_check : ch.out_charge;
        out.insert(out.end(), v.begin(), v.end());
      }
    }
  }
  void il_nodes(int j, int k, bool incoming_check, std::vector<int>& out) const {
    const Box& b = tree[j][k];
    for (int in = 0; in < 16; ++in)
      if (b.inner[in] != -1) rows_for(j, b.inner[in], incoming_check, out);
    for (int on = 0; on < 24; ++on)
      if (b.outer[on] != -1) rows_for(j, b.outer[on], incoming_check, out);
  }
  void getNodes_outgoing_box(int j, int k) {  // F:1230-1281
    Box& b = tree[j][k];
    std::vector<int> boxA, IL;
    rows_for(j, k, false, boxA);
    il_nodes(j, k, true, IL);
    std::vector<int> rb, cb;
    int cr;
    Mat Ac;
    aca(IL, boxA, rb, cb, cr, Ac, b.Ar);
    b.rank_out_aca = cr;
    if (cr > 0) {
      for (int r : rb) b.out_check.push_back(IL[r]);
      for (int c : cb) b.out_charge.push_back(boxA[c]);
    }
  }
  void getNodes_incoming_box(int j, int k) {  // F:1283-1336
    Box& b = tree[j][k];
    std::vector<int> boxA, IL;
    rows_for(j, k, true, boxA);
    il_nodes(j, k, false, IL);
    std::vector<int> rb, cb;
    int cr;
    Mat Ar;
    aca(boxA, IL, rb, cb, cr, b.Ac, Ar);
    b.rank_in_aca = cr;
    if (cr > 0) {
      for (int r : rb) b.in_check.push_back(boxA[r]);
      for (int c : cb) b.in_charge.push_back(IL[c]);
    }
  }
  void get_L2P_P2M_box(int j, int k) {  // F:1105-1128
    Box& b = tree[j][k];
    if (b.in_check.size() < b.out_check.size()) {
      b.out_check.resize(b.in_check.size());
      b.out_charge.resize(b.in_check.size());
    } else {
      b.in_check.resize(b.out_check.size());
      b.in_charge.resize(b.out_check.size());
    }
    const int r = (int)b.in_check.size();
    Mat temp1 = block(b.Ac, 0, 0, b.Ac.r, r);
    b.L2P = Mat(b.Ac.r, r);
    if (r > 0) {
      Mat D1 = getMatrix(b.in_check, b.in_charge);
      PartialLU lu(adj(D1));
      b.L2P = adj(lu.solve(adj(temp1)));
    }
    Mat temp2 = block(b.Ar, 0, 0, (int)b.out_check.size(), b.Ar.c);
    b.P2M = Mat((int)b.out_check.size(), b.Ar.c);
    if (!b.out_check.empty()) {
      Mat D2 = getMatrix(b.out_check, b.out_charge);
      PartialLU lu(D2);
      b.P2M = lu.solve(temp2);
    }
  }
  void getNodes() {  // F:1137-1158 (boxes of one level are independent)
    for (int j = depth; j >= 2; --j) {
#pragma omp parallel for schedule(dynamic)
      for (int k = 0; k < nBoxes[j]; ++k) getNodes_outgoing_box(j, k);
#pragma omp parallel for schedule(dynamic)
      for (int k = 0; k < nBoxes[j]; ++k) getNodes_incoming_box(j, k);
#pragma omp parallel for schedule(dynamic)
      for (int k = 0; k < nBoxes[j]; ++k) get_L2P_P2M_box(j, k);
    }
  }
  void assemble_M2L() {  // F:1338-1361
    for (int j = 2; j <= depth; ++j) {
#pragma omp parallel for schedule(dynamic)
      for (int k = 0; k < nBoxes[j]; ++k) {
        Box& b = tree[j][k];
        std::vector<std::pair<int, Mat>> blocks;
        for (int in = 0; in < 16; ++in)
          if (b.inner[in] != -1) { int kIL = b.inner[in]; blocks.push_back({kIL, getMatrix(b.in_check, tree[j][kIL].out_charge)}); }
        for (int on = 0; on < 24; ++on)
          if (b.outer[on] != -1) { int kIL = b.outer[on]; blocks.push_back({kIL, getMatrix(b.in_check, tree[j][kIL].out_charge)}); }
        for (auto& pr : blocks) b.M2L[pr.first] = pr.second;
      }
    }
  }
  void initialise_phase() {  // F:1703-1727
    for (int j = 2; j <= depth; ++j)
      for (int k = 0; k < nBoxes[j]; ++k) {
        Box& b = tree[j][k];
        b.NumMultipoles = b.P2M.r;
        b.NumLocals = b.L2P.c;
        b.local_rhs = Mat(b.NumMultipoles, nrhs);
        b.multipole_rhs = Mat(b.NumLocals, nrhs);
      }
  }
  void initialise_P2P_Leaf_Level() {  // F:1729-1741
#pragma omp parallel for schedule(dynamic)
    for (int k = 0; k < nBoxes[depth]; ++k) {
      Box& b = tree[depth][k];
      std::vector<std::pair<int, Mat>> blocks;
      for (int n = 0; n < 8; ++n) {
        int nn = b.neighbors[n];
        if (nn != -1) blocks.push_back({nn, getMatrix(b.chargeLocations, tree[depth][nn].chargeLocations)});
      }
      blocks.push_back({k, getMatrix(b.chargeLocations, b.chargeLocations)});
      for (auto& pr : blocks) b.P2P[pr.first] = pr.second;
    }
  }
  Mat mosaic(int j, int k, int nn) {  // F:1743-1794
    int nr = 0, nc = 0;
    for (int a = 0; a < 4; ++a) nr += tree[j + 1][4 * k + a].NumLocals;
    for (int b = 0; b < 4; ++b) nc += tree[j + 1][4 * nn + b].NumMultipoles;
    Mat P(nr, nc);
    int ri = 0;
    for (int a = 0; a < 4; ++a) {
      int ci = 0;
      Box& ch = tree[j + 1][4 * k + a];
      for (int b = 0; b < 4; ++b) {
        int cb = 4 * nn + b;
        int rr = ch.NumLocals, cc = tree[j + 1][cb].NumMultipoles;
        if (rr > 0 && cc > 0) {
          const Mat& src = ch.M2L[cb];
          if (src.r != rr || src.c != cc) { fprintf(stderr, "oracle mosaic: M2L block %d->%d is %dx%d, want %dx%d\n", 4 * k + a, cb, src.r, src.c, rr, cc); abort(); }
          for (int y = 0; y < cc; ++y)
            for (int x = 0; x < rr; ++x) P(ri + x, ci + y) = src(x, y);
        }
        ci += cc;
      }
      ri += ch.NumLocals;
    }
    return P;
  }
  void initialise_P2P_NonLeafLevel(int j) {
    for (int k = 0; k < nBoxes[j]; ++k) {
      Box& b = tree[j][k];
      for (int n = 0; n < 8; ++n) {
        int nn = b.neighbors[n];
        if (nn != -1) b.P2P[nn] = mosaic(j, k, nn);
      }
      b.P2P[k] = mosaic(j, k, k);
    }
    // F:1798-1807
    for (int k = 0; k < nBoxes[j]; ++k) {
      int len = 0;
      for (int c = 0; c < 4; ++c) len += tree[j + 1][4 * k + c].NumLocals;
      Mat r(len, nrhs);
      int o = 0;
      for (int c = 0; c < 4; ++c) {
        const Mat& m = tree[j + 1][4 * k + c].multipole_rhs;
        for (int s = 0; s < nrhs; ++s)
          for (int i = 0; i < m.r; ++i) r(o + i, s) = m(i, s);
        o += m.r;
      }
      tree[j][k].particle_rhs = r;
    }
  }

  bool is_well_separated(int j, int k, int l) const {  // F:2077-2088
    if (k == l) return false;
    for (int i = 0; i < 8; ++i)
      if (tree[j][k].neighbors[i] == l) return false;
    return true;
  }

  // ---------------- elimination (F:1814-2372) ----------------
  // The reference leaves several blocks uninitialised in the no-QR branches
  // (Eigen Mat(r,c)); the value those statements stand for is a product with
  // an empty inner dimension, i.e. zero, which is what is stored here.
  // schedule bit 2: what eliminate_x computes from P2P[k][k], the right-hand side
  // and the neighbour blocks alone, computed before the step's recompressions
  void x_early(int j, int k) {
    xe.on = false;
    Box& B = tree[j][k];
    if (B.P2P[k].size() == 0) return;
    xe.qr.reset(new ColPivQR(B.P2P[k]));
    xe.Xb = xe.qr->solve(B.particle_rhs);
    for (int n = 0; n < 8; ++n) {
      int nn = B.neighbors[n];
      if (nn == -1) continue;
      xe.S[n] = tree[j][nn].Eliminated ? xe.qr->solve(B.M2P[nn]) : xe.qr->solve(B.P2P[nn]);
    }
    xe.on = true;
  }
  void eliminate_x(int j, int k) {
    Box& B = tree[j][k];
    if (B.P2P[k].size() != 0) {
      std::unique_ptr<ColPivQR> own;
      if (!xe.on) own.reset(new ColPivQR(B.P2P[k]));
      const ColPivQR& QR = xe.on ? *xe.qr : *own;
      // QR^{-1} of the right-hand side and of X[k][nn] for neighbour n
      auto solve_rhs = [&]() { return xe.on ? xe.Xb : QR.solve(B.particle_rhs); };
      auto solve_nb = [&](int n, const Mat& src) { return xe.on ? xe.S[n] : QR.solve(src); };
      // F:1961-1987
      B.L2M_f = neg(mul(B.P2M, QR.solve(B.L2P)));
      for (int n = 0; n < 8; ++n) {
        int nn = B.neighbors[n];
        if (nn == -1) continue;
        if (!tree[j][nn].Eliminated) B.P2M_f[nn] = neg(mul(B.P2M, solve_nb(n, B.P2P[nn])));
        else B.M2M_f[nn] = neg(mul(B.P2M, solve_nb(n, B.M2P[nn])));
      }
      B.local_rhs = neg(mul(B.P2M, solve_rhs()));
      Mat Xb = solve_rhs();
      Mat XL = QR.solve(B.L2P);
      // QR^{-1} X[k][pp] for every neighbour pp (the reference re-solves these
      // for every equation nn; the value is the same)
      Mat W[8];
      for (int pI = 0; pI < 8; ++pI) {
        int pp = B.neighbors[pI];
        if (pp == -1) continue;
        W[pI] = solve_nb(pI, tree[j][pp].Eliminated ? B.M2P[pp] : B.P2P[pp]);
      }
      xe.on = false;
      if (schedule & 4) z_early(j, k);
      for (int n = 0; n < 8; ++n) {
        int nn = B.neighbors[n];
        if (nn == -1) continue;
        Box& Nn = tree[j][nn];
        // F:2004-2011
        if (!Nn.Eliminated) Nn.L2P_f = neg(mul(Nn.P2P[k], XL));
        else Nn.L2P_f = neg(mul(Nn.P2L[k], XL));
        B.Lf[n] = Nn.L2P_f;
        // F:2013-2075
        for (int pI = 0; pI < 8; ++pI) {
          int pp = B.neighbors[pI];
          if (pp == -1) continue;
          Box& Pp = tree[j][pp];
          if (!Nn.Eliminated) {
            if (!Pp.Eliminated) {
              Mat upd = mul(Nn.P2P[k], W[pI]);
              if (Nn.P2P[pp].size() == 0) Nn.P2P[pp] = neg(upd);
              else Nn.P2P[pp] = sub(Nn.P2P[pp], upd);
              if (is_well_separated(j, nn, pp) && nn < pp && fnorm(Nn.P2P[pp]) > 1e-10) P2Pq.push_back({nn, pp});
            } else {
              Mat upd = mul(Nn.P2P[k], W[pI]);
              if (Nn.M2P[pp].size() == 0) Nn.M2P[pp] = neg(upd);
              else Nn.M2P[pp] = sub(Nn.M2P[pp], upd);
            }
          } else {
            if (!Pp.Eliminated) {
              Mat upd = mul(Nn.P2L[k], W[pI]);
              if (Nn.P2L[pp].size() == 0) Nn.P2L[pp] = neg(upd);
              else Nn.P2L[pp] = sub(Nn.P2L[pp], upd);
              if (is_well_separated(j, nn, pp) && fnorm(Nn.P2L[pp]) > 1e-10) P2L_M2Pq.push_back({nn, pp});
            } else {
              Nn.M2L[pp] = sub(Nn.M2L[pp], mul(Nn.P2L[k], W[pI]));
            }
          }
        }
        // F:1995-2002
        if (!Nn.Eliminated) Nn.particle_rhs = sub(Nn.particle_rhs, mul(Nn.P2P[k], Xb));
        else Nn.multipole_rhs = sub(Nn.multipole_rhs, mul(Nn.P2L[k], Xb));
      }
    } else {
      // F:1843-1957 (box k carries no unknowns at this level)
      B.L2M_f = Mat(B.P2M.r, B.L2P.c);
      for (int n = 0; n < 8; ++n) {
        int nn = B.neighbors[n];
        if (nn == -1) continue;
        if (!tree[j][nn].Eliminated) B.P2M_f[nn] = Mat(B.P2M.r, B.P2P[nn].c);
        else B.M2M_f[nn] = Mat(B.P2M.r, B.M2P[nn].c);
      }
      B.local_rhs = Mat(B.P2M.r, nrhs);
      for (int n = 0; n < 8; ++n) {
        int nn = B.neighbors[n];
        if (nn == -1) continue;
        Box& Nn = tree[j][nn];
        if (!Nn.Eliminated) Nn.L2P_f = Mat(Nn.P2P[k].r, B.L2P.c);
        else Nn.L2P_f = Mat(Nn.P2L[k].r, B.L2P.c);
        B.Lf[n] = Nn.L2P_f;
        for (int pI = 0; pI < 8; ++pI) {
          int pp = B.neighbors[pI];
          if (pp == -1) continue;
          Box& Pp = tree[j][pp];
          if (!Nn.Eliminated) {
            if (!Pp.Eliminated) {
              if (Nn.P2P[pp].size() == 0) Nn.P2P[pp] = Mat(Nn.P2P[k].r, B.P2P[pp].c);
              if (is_well_separated(j, nn, pp) && nn < pp && fnorm(Nn.P2P[pp]) > 1e-10) P2Pq.push_back({nn, pp});
            } else {
              if (Nn.M2P[pp].size() == 0) Nn.M2P[pp] = Mat(Nn.P2P[k].r, B.M2P[pp].c);
            }
          } else {
            if (!Pp.Eliminated) {
              if (Nn.P2L[pp].size() == 0) Nn.P2L[pp] = Mat(Nn.P2L[k].r, B.P2P[pp].c);
              if (is_well_separated(j, nn, pp) && fnorm(Nn.P2L[pp]) > 1e-10) P2L_M2Pq.push_back({nn, pp});
            } else {
              (void)Nn.M2L[pp];
            }
          }
        }
      }
    }
  }

  // The factorisation of L2M_f and its solves (F:2251-2279): they read only box
  // k's own blocks and write only box k's own blocks.
  void z_solves(int j, int k, Mat& Yneg, Mat& Yrhs, Mat* Z) {
    Box& B = tree[j][k];
    ColPivQR QR2(B.L2M_f);
    const int r = B.NumMultipoles;
    // F:2255-2279
    B.M2L[k] = QR2.solve(neg(identity(r)));
    for (int n = 0; n < 8; ++n) {
      int nn = B.neighbors[n];
      if (nn == -1) continue;
      if (!tree[j][nn].Eliminated) {
        B.P2L[nn] = QR2.solve(B.P2M_f[nn]);
        if (is_well_separated(j, k, nn) && fnorm(B.P2L[nn]) > 1e-10) P2L_M2Pq.push_back({k, nn});
      } else {
        B.M2L[nn] = QR2.solve(B.M2M_f[nn]);
      }
    }
    // F:2251-2253
    B.multipole_rhs = QR2.solve(B.local_rhs);
    Yneg = QR2.solve(neg(identity(r)));
    Yrhs = QR2.solve(B.local_rhs);
    for (int pI = 0; pI < 8; ++pI) {
      int pp = B.neighbors[pI];
      if (pp == -1) continue;
      Z[pI] = tree[j][pp].Eliminated ? QR2.solve(B.M2M_f[pp]) : QR2.solve(B.P2M_f[pp]);
    }
  }
  // schedule bit 4: z_solves before the x-phase fill-ins of the neighbours' blocks
  void z_early(int j, int k) {
    ze.on = false;
    if (tree[j][k].L2M_f.size() == 0) return;
    z_solves(j, k, ze.Yneg, ze.Yrhs, ze.Z);
    ze.on = true;
  }
  void eliminate_z(int j, int k) {
    Box& B = tree[j][k];
    if (B.L2M_f.size() > 0) {
      Mat Yneg, Yrhs, Z[8];
      if (ze.on) {
        Yneg = ze.Yneg;
        Yrhs = ze.Yrhs;
        for (int q = 0; q < 8; ++q) Z[q] = ze.Z[q];
      } else {
        z_solves(j, k, Yneg, Yrhs, Z);
      }
      ze.on = false;
      for (int n = 0; n < 8; ++n) {
        int nn = B.neighbors[n];
        if (nn == -1) continue;
        Box& Nn = tree[j][nn];
        // F:2348-2372
        Mat fy = mul(Nn.L2P_f, Yneg);
        if (!Nn.Eliminated) {
          if (Nn.M2P[k].size() == 0) Nn.M2P[k] = neg(fy);
          else Nn.M2P[k] = sub(Nn.M2P[k], fy);
        } else {
          if (Nn.M2L[k].size() == 0) Nn.M2L[k] = neg(fy);
          else Nn.M2L[k] = sub(Nn.M2L[k], fy);
        }
        // F:2296-2346
        for (int pI = 0; pI < 8; ++pI) {
          int pp = B.neighbors[pI];
          if (pp == -1) continue;
          Box& Pp = tree[j][pp];
          if (!Nn.Eliminated) {
            if (!Pp.Eliminated) {
              Nn.P2P[pp] = sub(Nn.P2P[pp], mul(Nn.L2P_f, Z[pI]));
              if (is_well_separated(j, nn, pp) && nn < pp && fnorm(Nn.P2P[pp]) > 1e-10) P2Pq.push_back({nn, pp});
            } else {
              Nn.M2P[pp] = sub(Nn.M2P[pp], mul(Nn.L2P_f, Z[pI]));
            }
          } else {
            if (!Pp.Eliminated) {
              Nn.P2L[pp] = sub(Nn.P2L[pp], mul(Nn.L2P_f, Z[pI]));
              if (is_well_separated(j, nn, pp) && fnorm(Nn.P2L[pp]) > 1e-10) P2L_M2Pq.push_back({nn, pp});
            } else {
              Nn.M2L[pp] = sub(Nn.M2L[pp], mul(Nn.L2P_f, Z[pI]));
            }
          }
        }
        // F:2287-2294
        if (!Nn.Eliminated) Nn.particle_rhs = sub(Nn.particle_rhs, mul(Nn.L2P_f, Yrhs));
        else Nn.multipole_rhs = sub(Nn.multipole_rhs, mul(Nn.L2P_f, Yrhs));
      }
    } else {
      // F:2116-2242 (box k has rank zero)
      B.M2L[k] = Mat(0, B.NumMultipoles);
      for (int n = 0; n < 8; ++n) {
        int nn = B.neighbors[n];
        if (nn == -1) continue;
        if (!tree[j][nn].Eliminated) {
          B.P2L[nn] = Mat(0, B.P2M_f[nn].c);
        } else {
          B.M2L[nn] = Mat(0, B.M2M_f[nn].c);
        }
      }
      B.multipole_rhs = Mat(0, nrhs);
      for (int n = 0; n < 8; ++n) {
        int nn = B.neighbors[n];
        if (nn == -1) continue;
        Box& Nn = tree[j][nn];
        if (!Nn.Eliminated) {
          if (Nn.M2P[k].size() == 0) Nn.M2P[k] = Mat(Nn.L2P_f.r, B.NumMultipoles);
        } else {
          if (Nn.M2L[k].size() == 0) Nn.M2L[k] = Mat(Nn.L2P_f.r, B.NumMultipoles);
        }
        for (int pI = 0; pI < 8; ++pI) {
          int pp = B.neighbors[pI];
          if (pp == -1) continue;
          Box& Pp = tree[j][pp];
          if (!Nn.Eliminated) {
            if (!Pp.Eliminated) {
              (void)Nn.P2P[pp];
              if (is_well_separated(j, nn, pp) && nn < pp && fnorm(Nn.P2P[pp]) > 1e-10) P2Pq.push_back({nn, pp});
            } else {
              (void)Nn.M2P[pp];
            }
          } else {
            if (!Pp.Eliminated) {
              (void)Nn.P2L[pp];
              if (is_well_separated(j, nn, pp) && fnorm(Nn.P2L[pp]) > 1e-10) P2L_M2Pq.push_back({nn, pp});
            } else {
              (void)Nn.M2L[pp];
            }
          }
        }
      }
    }
  }

  // ---------------- recompression (F:1424-1699) ----------------
  void compress_P2P(int j, int k, int b, Mat& new_L2P, Mat& new_P2Mt, Mat& M2L) {  // F:1532-1559
    Box& K = tree[j][k];
    Box& Bb = tree[j][b];
    Mat A_col = hcat(K.L2P, K.P2P[b]);
    ColPivQR qc(A_col);
    qc.setThreshold(tol);
    Mat Qc = qc.householderQ();
    new_L2P = block(Qc, 0, 0, Qc.r, qc.rank());
    Mat Rk_prime = mul(adj(new_L2P), K.P2P[b]);
    Mat Rk = mul(adj(new_L2P), K.L2P);
    Mat A_row = hcat(adj(Bb.P2M), adj(Rk_prime));
    ColPivQR qrw(A_row);
    qrw.setThreshold(tol);
    Mat Qr = qrw.householderQ();
    new_P2Mt = block(Qr, 0, 0, Qr.r, qrw.rank());
    Mat Rn = mul(adj(new_P2Mt), adj(Bb.P2M));
    Mat Rn_prime = mul(adj(new_P2Mt), adj(Rk_prime));
    M2L = add(mul(mul(Rk, K.M2L[b]), adj(Rn)), adj(Rn_prime));
  }
  void compress_M2P(int j, int k, int b, Mat& new_L2P, Mat& M2L) {  // F:1561-1575
    Box& K = tree[j][k];
    Mat A_col = hcat(K.L2P, K.M2P[b]);
    ColPivQR qc(A_col);
    qc.setThreshold(tol);
    Mat Qc = qc.householderQ();
    new_L2P = block(Qc, 0, 0, Qc.r, qc.rank());
    Mat Rk_prime = mul(adj(new_L2P), K.M2P[b]);
    Mat Rk = mul(adj(new_L2P), K.L2P);
    M2L = add(mul(Rk, K.M2L[b]), Rk_prime);
  }
  void compress_P2L(int j, int k, int b, Mat& new_P2Mt, Mat& M2L) {  // F:1577-1591
    Box& K = tree[j][k];
    Box& Bb = tree[j][b];
    Mat A_row = hcat(adj(Bb.P2M), adj(K.P2L[b]));
    ColPivQR qrw(A_row);
    qrw.setThreshold(tol);
    Mat Qr = qrw.householderQ();
    new_P2Mt = block(Qr, 0, 0, Qr.r, qrw.rank());
    Mat Rn = mul(adj(new_P2Mt), adj(Bb.P2M));
    Mat Rn_prime = mul(adj(new_P2Mt), adj(K.P2L[b]));
    M2L = add(mul(K.M2L[b], adj(Rn)), adj(Rn_prime));
  }
  void update_other_M2Ls_at_k(int j, int k, int b, const Mat& nL) {  // F:1594-1630
    Box& K = tree[j][k];
    Mat T = mul(adj(nL), K.L2P);
    for (int in = 0; in < 16; ++in)
      if (K.inner[in] != -1 && K.inner[in] != b) K.M2L[K.inner[in]] = mul(T, K.M2L[K.inner[in]]);
    for (int on = 0; on < 24; ++on)
      if (K.outer[on] != -1 && K.outer[on] != b) K.M2L[K.outer[on]] = mul(T, K.M2L[K.outer[on]]);
    for (int n = 0; n < 8; ++n) {
      int kN = K.neighbors[n];
      if (kN != -1 && tree[j][kN].Eliminated && K.Eliminated) K.M2L[kN] = mul(T, K.M2L[kN]);
    }
    if (K.Eliminated) K.M2L[k] = mul(T, K.M2L[k]);
  }
  void update_other_M2Ls_at_b(int j, int k, int b, const Mat& nP) {  // F:1632-1669
    Box& Bb = tree[j][b];
    Mat T = mul(Bb.P2M, nP);
    for (int in = 0; in < 16; ++in) {
      int kIL = Bb.inner[in];
      if (kIL != -1 && kIL != k) tree[j][kIL].M2L[b] = mul(tree[j][kIL].M2L[b], T);
    }
    for (int on = 0; on < 24; ++on) {
      int kIL = Bb.outer[on];
      if (kIL != -1 && kIL != b) tree[j][kIL].M2L[b] = mul(tree[j][kIL].M2L[b], T);
    }
    for (int n = 0; n < 8; ++n) {
      int kN = Bb.neighbors[n];
      if (kN != -1 && tree[j][kN].Eliminated && Bb.Eliminated) tree[j][kN].M2L[b] = mul(tree[j][kN].M2L[b], T);
    }
    if (Bb.Eliminated) Bb.M2L[b] = mul(Bb.M2L[b], T);
  }
  void update_parent_L2P(int j, int k, const Mat& nL) {  // F:1671-1684
    int kP = k / 4, ck = k % 4;
    Box& P = tree[j - 1][kP];
    std::vector<Mat> U(4);
    int ri = 0;
    for (int c = 0; c < 4; ++c) {
      int nl = tree[j][kP * 4 + c].NumLocals;
      U[c] = block(P.L2P, ri, 0, nl, P.L2P.c);
      ri += nl;
    }
    U[ck] = mul(mul(adj(nL), tree[j][k].L2P), U[ck]);
    int tot = U[0].r + U[1].r + U[2].r + U[3].r;
    Mat out(tot, U[0].c);
    int o = 0;
    for (int c = 0; c < 4; ++c) {
      for (int y = 0; y < U[c].c; ++y)
        for (int x = 0; x < U[c].r; ++x) out(o + x, y) = U[c](x, y);
      o += U[c].r;
    }
    P.L2P = out;
  }
  void update_parent_P2M(int j, int b, const Mat& nP) {  // F:1686-1699
    int bP = b / 4, cb = b % 4;
    Box& P = tree[j - 1][bP];
    std::vector<Mat> V(4);
    int ci = 0;
    for (int c = 0; c < 4; ++c) {
      int nm = tree[j][bP * 4 + c].NumMultipoles;
      V[c] = block(P.P2M, 0, ci, P.P2M.r, nm);
      ci += nm;
    }
    V[cb] = mul(mul(V[cb], tree[j][b].P2M), nP);
    int tot = V[0].c + V[1].c + V[2].c + V[3].c;
    Mat out(V[0].r, tot);
    int o = 0;
    for (int c = 0; c < 4; ++c) {
      for (int y = 0; y < V[c].c; ++y)
        for (int x = 0; x < V[c].r; ++x) out(x, o + y) = V[c](x, y);
      o += V[c].c;
    }
    P.P2M = out;
  }
  static void equalise(Mat& L, Mat& Pt) {  // the "_modified" truncation in F:1445-1460
    if (L.c < Pt.c) Pt = block(Pt, 0, 0, Pt.r, L.c);
    else L = block(L, 0, 0, L.r, Pt.c);
  }
  void compress_P2P_Two_Ways(int j, int k, int b) {  // F:1424-1490
    Mat nLk, nPtb, M2Lkb, nLb, nPtk, M2Lbk;
    compress_P2P(j, k, b, nLk, nPtb, M2Lkb);
    compress_P2P(j, b, k, nLb, nPtk, M2Lbk);
    equalise(nLk, nPtk);
    equalise(nLb, nPtb);
    Box& K = tree[j][k];
    Box& Bb = tree[j][b];
    K.M2L[b] = block(M2Lkb, 0, 0, nLk.c, nPtb.c);
    update_other_M2Ls_at_k(j, k, b, nLk);
    update_other_M2Ls_at_b(j, k, b, nPtb);
    if (j > 2) { update_parent_L2P(j, k, nLk); update_parent_P2M(j, b, nPtb); }
    K.L2P = nLk;
    Bb.P2M = adj(nPtb);
    K.NumLocals = K.L2P.c;
    Bb.NumMultipoles = Bb.P2M.r;
    Bb.M2L[k] = block(M2Lbk, 0, 0, nLb.c, nPtk.c);
    update_other_M2Ls_at_k(j, b, k, nLb);
    update_other_M2Ls_at_b(j, b, k, nPtk);
    if (j > 2) { update_parent_L2P(j, b, nLb); update_parent_P2M(j, k, nPtk); }
    Bb.L2P = nLb;
    K.P2M = adj(nPtk);
    Bb.NumLocals = Bb.L2P.c;
    K.NumMultipoles = K.P2M.r;
  }
  void compress_M2P_P2L(int j, int k, int b) {  // F:1492-1530
    Mat nLk, M2Lkb, nPtk, M2Lbk;
    compress_M2P(j, k, b, nLk, M2Lkb);
    compress_P2L(j, b, k, nPtk, M2Lbk);
    equalise(nLk, nPtk);
    Box& K = tree[j][k];
    Box& Bb = tree[j][b];
    K.M2L[b] = block(M2Lkb, 0, 0, nLk.c, M2Lkb.c);
    update_other_M2Ls_at_k(j, k, b, nLk);
    if (j > 2) update_parent_L2P(j, k, nLk);
    K.L2P = nLk;
    K.NumLocals = K.L2P.c;
    Bb.M2L[k] = block(M2Lbk, 0, 0, M2Lbk.r, nPtk.c);
    update_other_M2Ls_at_b(j, b, k, nPtk);
    if (j > 2) update_parent_P2M(j, k, nPtk);
    K.P2M = adj(nPtk);
    K.NumMultipoles = K.P2M.r;
  }

  void eliminate_phase_efficient() {  // F:2407-2451
    ncompress = 0;
    for (int j = depth; j >= 2; --j) {
      if (j != depth) initialise_P2P_NonLeafLevel(j);
      for (int k = 0; k < nBoxes[j]; ++k) {
        if (schedule & 2) x_early(j, k);
        for (size_t i = 0; i < P2Pq.size(); ++i) {
          int nn = P2Pq[i].first, pp = P2Pq[i].second;
          if (k == nn || k == pp) {
            P2Pq.erase(P2Pq.begin() + i);
            --i;
            if (tree[j][nn].P2P[pp].size() != 0) {
              ++ncompress;
              compress_P2P_Two_Ways(j, nn, pp);
              tree[j][nn].P2P[pp] = Mat();
              tree[j][pp].P2P[nn] = Mat();
            }
          }
        }
        for (size_t i = 0; i < P2L_M2Pq.size(); ++i) {
          int nn = P2L_M2Pq[i].first, pp = P2L_M2Pq[i].second;
          if (k == nn || k == pp) {
            P2L_M2Pq.erase(P2L_M2Pq.begin() + i);
            --i;
            if (tree[j][nn].P2L[pp].size() != 0) {
              ++ncompress;
              compress_M2P_P2L(j, pp, nn);
              tree[j][nn].P2L[pp] = Mat();
              tree[j][pp].M2P[nn] = Mat();
            }
          }
        }
        P2Pq.clear();
        P2L_M2Pq.clear();
        tree[j][k].Eliminated = true;
        eliminate_x(j, k);
        eliminate_z(j, k);
      }
    }
    solve_base(2);
  }

  void eliminate_phase() {  // F:2374-2405 (compress every queued pair after each box)
    for (int j = depth; j >= 2; --j) {
      if (j != depth) initialise_P2P_NonLeafLevel(j);
      for (int k = 0; k < nBoxes[j]; ++k) {
        tree[j][k].Eliminated = true;
        eliminate_x(j, k);
        eliminate_z(j, k);
        for (size_t i = 0; i < P2Pq.size(); ++i) {
          int nn = P2Pq[i].first, pp = P2Pq[i].second;
          if (tree[j][nn].P2P[pp].size() == 0) continue;  // duplicate entry
          compress_P2P_Two_Ways(j, nn, pp);
          tree[j][nn].P2P[pp] = Mat();
          tree[j][pp].P2P[nn] = Mat();
        }
        P2Pq.clear();
        for (size_t i = 0; i < P2L_M2Pq.size(); ++i) {
          int nn = P2L_M2Pq[i].first, pp = P2L_M2Pq[i].second;
          if (tree[j][nn].P2L[pp].size() == 0) continue;  // duplicate entry
          compress_M2P_P2L(j, pp, nn);
          tree[j][nn].P2L[pp] = Mat();
          tree[j][pp].M2P[nn] = Mat();
        }
        P2L_M2Pq.clear();
      }
    }
    solve_base(2);
  }

  void solve_base(int j) {  // F:2453-2485
    int NM = 0, NL = 0;
    for (int k = 0; k < nBoxes[j]; ++k) { NM += tree[j][k].NumMultipoles; NL += tree[j][k].NumLocals; }
    if (NL == 0 || NM == 0) {
      // the reference leaves the (empty) multipole vectors unset here
      for (int k = 0; k < nBoxes[j]; ++k) tree[j][k].multipoles = Mat(tree[j][k].NumMultipoles, nrhs);
      return;
    }
    Mat A(NL, NM), b(NL, nrhs);
    int ri = 0;
    for (int r = 0; r < nBoxes[j]; ++r) {
      Box& R = tree[j][r];
      int si = 0;
      for (int s = 0; s < nBoxes[j]; ++s) {
        int nc = tree[j][s].NumMultipoles;
        if (R.NumLocals > 0 && nc > 0) {
          const Mat& m = R.M2L[s];
          if (m.r != R.NumLocals || m.c != nc) { fprintf(stderr, "oracle base: M2L %d->%d is %dx%d\n", r, s, m.r, m.c); abort(); }
          for (int y = 0; y < nc; ++y)
            for (int x = 0; x < R.NumLocals; ++x) A(ri + x, si + y) = m(x, y);
        }
        si += nc;
      }
      for (int t = 0; t < nrhs; ++t)
        for (int x = 0; x < R.NumLocals; ++x) b(ri + x, t) = R.multipole_rhs(x, t);
      ri += R.NumLocals;
    }
    ColPivQR qr(A);
    Mat m = qr.solve(b);
    int o = 0;
    for (int k = 0; k < nBoxes[j]; ++k) {
      tree[j][k].multipoles = block(m, o, 0, tree[j][k].NumMultipoles, nrhs);
      o += tree[j][k].NumMultipoles;
    }
  }

  // A solve with new right-hand sides against the factors of the last solve:
  // the right-hand-side updates that the elimination made box by box
  // (F:1968, 1997-2001, 2252, 2289-2293), gathered per receiving box.  Box nn
  // subtracted X[t][nn] QRx^-1 r_nn and L2P_f[t] y_nn from every neighbour t;
  // those blocks are frozen once nn is eliminated, except L2P_f, kept in Lf.
  void solve_again() {
    for (int j = depth; j >= 2; --j) {
      const int nb = nBoxes[j];
      std::vector<Mat> xb(nb), y(nb);
      if (j != depth)
        for (int k = 0; k < nb; ++k) {
          int len = 0;
          for (int c = 0; c < 4; ++c) len += tree[j + 1][4 * k + c].multipole_rhs.r;
          Mat r(len, nrhs);
          int o = 0;
          for (int c = 0; c < 4; ++c) {
            const Mat& m = tree[j + 1][4 * k + c].multipole_rhs;
            for (int t = 0; t < nrhs; ++t)
              for (int x = 0; x < m.r; ++x) r(o + x, t) = m(x, t);
            o += m.r;
          }
          tree[j][k].particle_rhs = r;
        }
      for (int k = 0; k < nb; ++k) {
        Box& B = tree[j][k];
        for (int n = 0; n < 8; ++n) {
          const int nn = B.neighbors[n];
          if (nn == -1 || nn > k) continue;
          const Box& Nn = tree[j][nn];
          if (xb[nn].size()) B.particle_rhs = sub(B.particle_rhs, mul(B.P2P[nn], xb[nn]));
          if (y[nn].size()) B.particle_rhs = sub(B.particle_rhs, mul(Nn.Lf[(n + 4) & 7], y[nn]));
        }
        if (B.P2P[k].size() == 0) { xb[k] = Mat(0, nrhs); y[k] = Mat(0, nrhs); continue; }
        ColPivQR qr(B.P2P[k]);
        xb[k] = qr.solve(B.particle_rhs);
        if (B.L2M_f.size() != 0) y[k] = ColPivQR(B.L2M_f).solve(neg(mul(B.P2M, xb[k])));
        else y[k] = Mat(0, nrhs);
      }
      for (int k = 0; k < nb; ++k) {
        Box& B = tree[j][k];
        Mat m = y[k];
        for (int n = 0; n < 8; ++n) {
          const int nn = B.neighbors[n];
          if (nn == -1 || nn < k) continue;
          const Box& Nn = tree[j][nn];
          if (xb[nn].size() && m.r) m = sub(m, mul(B.P2L[nn], xb[nn]));
          if (y[nn].size() && m.r) m = sub(m, mul(Nn.Lf[(n + 4) & 7], y[nn]));
        }
        B.multipole_rhs = m;
      }
    }
    solve_base(2);
    for (int j = 2; j <= depth; ++j)
      for (int k = 0; k < nBoxes[j]; ++k) tree[j][k].Eliminated = true;
    back_substitution_phase();
  }

  void back_substitution_phase() {  // F:2487-2532
    for (int j = 2; j <= depth; ++j) {
      if (!(schedule & 1)) {
        for (int k = nBoxes[j] - 1; k >= 0; --k) back_substitute_box(j, k);
        continue;
      }
      // schedule bit 1: box k reads the particles of its larger-index neighbours
      // and the multipoles of the others, so wave(k) = 1 + max wave of its
      // larger-index neighbours orders every read after its write
      std::vector<int> wave(nBoxes[j], 0);
      int nw = 0;
      for (int k = nBoxes[j] - 1; k >= 0; --k) {
        for (int n = 0; n < 8; ++n) {
          int nn = tree[j][k].neighbors[n];
          if (nn > k) wave[k] = std::max(wave[k], wave[nn] + 1);
        }
        nw = std::max(nw, wave[k] + 1);
      }
      for (int w = 0; w < nw; ++w)
        for (int k = 0; k < nBoxes[j]; ++k)  // increasing order inside a wave
          if (wave[k] == w) back_substitute_box(j, k);
    }
  }
  void back_substitute_box(int j, int k) {
    Box& B = tree[j][k];
    if (B.P2P[k].size() != 0) {
      ColPivQR qr(B.P2P[k]);
      Mat rhs1 = B.particle_rhs;
      for (int n = 0; n < 8; ++n) {
        int nn = B.neighbors[n];
        if (nn == -1) continue;
        if (!tree[j][nn].Eliminated) rhs1 = sub(rhs1, mul(B.P2P[nn], tree[j][nn].particles));
        else rhs1 = sub(rhs1, mul(B.M2P[nn], tree[j][nn].multipoles));
      }
      Mat rhs2 = sub(B.multipoles, mul(B.P2M, qr.solve(rhs1)));
      Mat Atemp = neg(mul(B.P2M, qr.solve(B.L2P)));
      if (Atemp.size() != 0) {
        ColPivQR aq(Atemp);
        B.locals = aq.solve(rhs2);
      } else {
        B.locals = Mat(0, nrhs);
      }
      B.particles = qr.solve(sub(rhs1, mul(B.L2P, B.locals)));
    } else {
      B.particles = Mat(0, nrhs);
    }
    B.Eliminated = false;
    if (j != depth) {
      int o = 0;
      for (int c = 0; c < 4; ++c) {
        Box& ch = tree[j + 1][4 * k + c];
        ch.multipoles = block(B.particles, o, 0, ch.NumMultipoles, nrhs);
        o += ch.NumMultipoles;
      }
    }
  }
};

}  // namespace

// ============================================================================
// C interface
// ============================================================================
extern "C" {

int orc_gauss_legendre(int n, double* nodes, double* weights) {
  std::vector<double> x, w;
  gauss_legendre(n, x, w);
  for (int i = 0; i < n; ++i) { nodes[i] = x[i]; weights[i] = w[i]; }
  return 0;
}

int orc_bessel_jy(int nmax, double x, double* J, double* Y) {
  bessel_jy_all(nmax, x, J, Y);
  return 0;
}

int orc_tables(const orc_params* p, int round6_, double* M, double* near_tab, double* qpinv) {
  Tables T = compute_tables(*p, round6_ != 0);
  for (size_t i = 0; i < T.M.size(); ++i) { M[2 * i] = T.M[i].real(); M[2 * i + 1] = T.M[i].imag(); }
  for (size_t i = 0; i < T.near.size(); ++i) { near_tab[2 * i] = T.near[i].real(); near_tab[2 * i + 1] = T.near[i].imag(); }
  if (qpinv) std::copy(T.qpinv.begin(), T.qpinv.end(), qpinv);
  return 0;
}

void* orc_create(const orc_params* p, const double* M, const double* near_tab) {
  Tables T;
  T.rank = p->n_cheb * p->n_cheb;
  T.nb = p->degree * (p->degree + 1) / 2;
  T.M.resize((size_t)121 * T.rank);
  T.near.resize((size_t)9 * T.rank * T.rank);
  for (size_t i = 0; i < T.M.size(); ++i) T.M[i] = cd(M[2 * i], M[2 * i + 1]);
  for (size_t i = 0; i < T.near.size(); ++i) T.near[i] = cd(near_tab[2 * i], near_tab[2 * i + 1]);
  return new Problem(*p, T);
}

void orc_destroy(void* h) { delete static_cast<Problem*>(h); }

int orc_num_points(void* h) { return static_cast<Problem*>(h)->N; }

int orc_set_perturbation(void* h, double rel) {
  static_cast<Problem*>(h)->perturb = rel;
  return 0;
}

int orc_set_variant(void* h, int full_compress) {
  static_cast<Problem*>(h)->full_compress = full_compress != 0;
  return 0;
}

int orc_set_schedule(void* h, int flags) {
  static_cast<Problem*>(h)->schedule = flags;
  return 0;
}

long orc_compressions(void* h) { return static_cast<Problem*>(h)->ncompress; }

int orc_grid_points(void* h, double* xy) {
  Problem* P = static_cast<Problem*>(h);
  for (int i = 0; i < P->N; ++i) { xy[2 * i] = P->pts[i].x; xy[2 * i + 1] = P->pts[i].y; }
  return 0;
}

int orc_contrast(void* h, double* q) {
  Problem* P = static_cast<Problem*>(h);
  std::copy(P->q.begin(), P->q.end(), q);
  return 0;
}

int orc_rhs_plane_wave(void* h, int nrhs, const double* theta, double* b) {
  Problem* P = static_cast<Problem*>(h);
  const double k = P->p.kappa;
  for (int s = 0; s < nrhs; ++s) {
    double ct = std::cos(theta[s]), st = std::sin(theta[s]);
    if (theta[s] == 0.0) { ct = 1.0; st = 0.0; }
    for (int i = 0; i < P->N; ++i) {
      // LS/LS_functions.hpp:113-120 with the incidence direction (cos t, sin t)
      double ph = P->pts[i].x * ct + P->pts[i].y * st;
      cd inc = std::exp(I1 * k * ph);
      cd v = -1.0 * k * k * P->q[i] * inc;
      b[2 * ((size_t)s * P->N + i)] = v.real();
      b[2 * ((size_t)s * P->N + i) + 1] = v.imag();
    }
  }
  return 0;
}

int orc_entries(void* h, long n, const int* I, const int* J, double* out) {
  Problem* P = static_cast<Problem*>(h);
#pragma omp parallel for schedule(dynamic, 256)
  for (long t = 0; t < n; ++t) {
    cd v = P->entry(I[t], J[t]);
    out[2 * t] = v.real();
    out[2 * t + 1] = v.imag();
  }
  return 0;
}

int orc_dense_matvec(void* h, int nrhs, const double* x, double* y) {
  Problem* P = static_cast<Problem*>(h);
  const int N = P->N;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < N; ++i) {
    std::vector<cd> acc(nrhs, cd(0, 0));
    for (int j = 0; j < N; ++j) {
      cd a = P->entry(i, j);
      if (a == cd(0, 0)) continue;
      for (int s = 0; s < nrhs; ++s) acc[s] += a * cd(x[2 * ((size_t)s * N + j)], x[2 * ((size_t)s * N + j) + 1]);
    }
    for (int s = 0; s < nrhs; ++s) { y[2 * ((size_t)s * N + i)] = acc[s].real(); y[2 * ((size_t)s * N + i) + 1] = acc[s].imag(); }
  }
  return 0;
}

// hybrid.cpp:263-281: U_total = U_incidence + G Phi with G the findPhi = false
// operator, dense with exact entries; the incidence direction is (cos t, sin t)
int orc_total_field(void* h, int nrhs, const double* theta, const double* phi, double* u) {
  Problem* P = static_cast<Problem*>(h);
  const int N = P->N;
  const double k = P->p.kappa;
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < N; ++i) {
    std::vector<cd> acc(nrhs, cd(0, 0));
    for (int j = 0; j < N; ++j) {
      cd g = P->entry0(i, j, false);
      if (g == cd(0, 0)) continue;
      for (int s = 0; s < nrhs; ++s) acc[s] += g * cd(phi[2 * ((size_t)s * N + j)], phi[2 * ((size_t)s * N + j) + 1]);
    }
    for (int s = 0; s < nrhs; ++s) {
      double ct = std::cos(theta[s]), st = std::sin(theta[s]);
      if (theta[s] == 0.0) { ct = 1.0; st = 0.0; }
      const cd inc = std::exp(I1 * k * (P->pts[i].x * ct + P->pts[i].y * st));  // LS/LS_functions.hpp:113-116
      const cd v = inc + acc[s];
      u[2 * ((size_t)s * N + i)] = v.real();
      u[2 * ((size_t)s * N + i) + 1] = v.imag();
    }
  }
  return 0;
}

int orc_solve(void* h, int nrhs, const double* b, double* x, double* times) {
  Problem* P = static_cast<Problem*>(h);
  P->nrhs = nrhs;
  const int N = P->N, rank = P->rank;
  double t0 = omp_get_wtime();
  P->createTree();
  double t1 = omp_get_wtime();
  // leaf rhs (F:1092-1103)
  for (int k = 0; k < P->nBoxes[P->depth]; ++k) {
    Mat r(rank, nrhs);
    for (int s = 0; s < nrhs; ++s)
      for (int i = 0; i < rank; ++i) {
        size_t g = (size_t)s * N + (size_t)k * rank + i;
        r(i, s) = cd(b[2 * g], b[2 * g + 1]);
      }
    P->tree[P->depth][k].particle_rhs = r;
  }
  P->getNodes();
  P->assemble_M2L();
  P->initialise_phase();
  P->initialise_P2P_Leaf_Level();
  double t2 = omp_get_wtime();
  if (P->full_compress) P->eliminate_phase();
  else P->eliminate_phase_efficient();
  double t3 = omp_get_wtime();
  P->back_substitution_phase();
  double t4 = omp_get_wtime();
  for (int k = 0; k < P->nBoxes[P->depth]; ++k) {
    const Mat& px = P->tree[P->depth][k].particles;
    for (int s = 0; s < nrhs; ++s)
      for (int i = 0; i < rank; ++i) {
        size_t g = (size_t)s * N + (size_t)k * rank + i;
        cd v = i < px.r ? px(i, s) : cd(0, 0);
        x[2 * g] = v.real();
        x[2 * g + 1] = v.imag();
      }
  }
  if (times) { times[0] = t1 - t0; times[1] = t2 - t1; times[2] = t3 - t2; times[3] = t4 - t3; }
  return 0;
}

// A solve with new right-hand sides against the factors of the last orc_solve.
int orc_solve_again(void* h, int nrhs, const double* b, double* x) {
  Problem* P = static_cast<Problem*>(h);
  P->nrhs = nrhs;
  const int N = P->N, rank = P->rank;
  for (int k = 0; k < P->nBoxes[P->depth]; ++k) {
    Mat r(rank, nrhs);
    for (int s = 0; s < nrhs; ++s)
      for (int i = 0; i < rank; ++i) {
        size_t g = (size_t)s * N + (size_t)k * rank + i;
        r(i, s) = cd(b[2 * g], b[2 * g + 1]);
      }
    P->tree[P->depth][k].particle_rhs = r;
  }
  P->solve_again();
  for (int k = 0; k < P->nBoxes[P->depth]; ++k) {
    const Mat& px = P->tree[P->depth][k].particles;
    for (int s = 0; s < nrhs; ++s)
      for (int i = 0; i < rank; ++i) {
        size_t g = (size_t)s * N + (size_t)k * rank + i;
        cd v = i < px.r ? px(i, s) : cd(0, 0);
        x[2 * g] = v.real();
        x[2 * g + 1] = v.imag();
      }
  }
  return 0;
}

// Dense matrix implied by the compressed representation before elimination
// (near blocks exact, far blocks U_k^{(j)} M2L^{(j)} V_b^{(j)} through the
// nested transfer operators).  Used to check the elimination algebra.
int orc_compressed_dense(const orc_params* p, const double* Mt, const double* nt, double* out) {
  Problem* P = static_cast<Problem*>(orc_create(p, Mt, nt));
  P->nrhs = 1;
  P->createTree();
  P->getNodes();
  P->assemble_M2L();
  P->initialise_phase();
  const int N = P->N, rank = P->rank, D = P->depth, nleaf = P->nBoxes[D];
  std::vector<std::vector<Mat>> U(D + 1), V(D + 1);
  U[D].resize(nleaf); V[D].resize(nleaf);
  for (int k = 0; k < nleaf; ++k) { U[D][k] = P->tree[D][k].L2P; V[D][k] = P->tree[D][k].P2M; }
  for (int j = D - 1; j >= 2; --j) {
    U[j].resize(nleaf); V[j].resize(nleaf);
    for (int k = 0; k < nleaf; ++k) {
      int ac = k >> (2 * (D - j - 1)), an = ac >> 2, c = ac & 3;
      Box& A = P->tree[j][an];
      int off = 0, offm = 0;
      for (int cc = 0; cc < c; ++cc) { off += P->tree[j + 1][4 * an + cc].NumLocals; offm += P->tree[j + 1][4 * an + cc].NumMultipoles; }
      U[j][k] = mul(U[j + 1][k], block(A.L2P, off, 0, P->tree[j + 1][ac].NumLocals, A.L2P.c));
      V[j][k] = mul(block(A.P2M, 0, offm, A.P2M.r, P->tree[j + 1][ac].NumMultipoles), V[j + 1][k]);
    }
  }
#pragma omp parallel for schedule(dynamic)
  for (int a = 0; a < nleaf; ++a)
    for (int b = 0; b < nleaf; ++b) {
      Mat blk(rank, rank);
      int xa, ya, xb, yb;
      Problem::box_xy(a, D, xa, ya); Problem::box_xy(b, D, xb, yb);
      if (std::abs(xa - xb) <= 1 && std::abs(ya - yb) <= 1) {
        for (int y = 0; y < rank; ++y)
          for (int x = 0; x < rank; ++x) blk(x, y) = P->entry(a * rank + x, b * rank + y);
      } else {
        for (int j = D; j >= 2; --j) {
          int A_ = a >> (2 * (D - j)), B_ = b >> (2 * (D - j)), xA, yA, xB, yB;
          Problem::box_xy(A_, j, xA, yA); Problem::box_xy(B_, j, xB, yB);
          if (std::max(std::abs(xA - xB), std::abs(yA - yB)) >= 2 &&
              std::max(std::abs(xA / 2 - xB / 2), std::abs(yA / 2 - yB / 2)) <= 1) {
            auto it = P->tree[j][A_].M2L.find(B_);
            if (it != P->tree[j][A_].M2L.end() && it->second.size() > 0) blk = mul(mul(U[j][a], it->second), V[j][b]);
            break;
          }
        }
      }
      for (int y = 0; y < rank; ++y)
        for (int x = 0; x < rank; ++x) {
          size_t g = (size_t)(a * rank + x) + (size_t)(b * rank + y) * N;
          out[2 * g] = blk(x, y).real();
          out[2 * g + 1] = blk(x, y).imag();
        }
    }
  delete P;
  return 0;
}

int orc_level_ranks(void* h, int level, int* rank_in, int* rank_out) {
  Problem* P = static_cast<Problem*>(h);
  if (level < 2 || level > P->depth || P->tree.empty()) return -1;
  for (int k = 0; k < P->nBoxes[level]; ++k) {
    rank_in[k] = P->tree[level][k].rank_in_aca;
    rank_out[k] = P->tree[level][k].rank_out_aca;
  }
  return 0;
}

int orc_box_lists(void* h, int level, int box, int* out48) {
  Problem* P = static_cast<Problem*>(h);
  if (P->tree.empty()) P->createTree();
  if (level < 0 || level > P->depth) return -1;
  const Box& b = P->tree[level][box];
  for (int i = 0; i < 8; ++i) out48[i] = b.neighbors[i];
  for (int i = 0; i < 16; ++i) out48[8 + i] = b.inner[i];
  for (int i = 0; i < 24; ++i) out48[24 + i] = b.outer[i];
  return 0;
}

int orc_box_skeleton(void* h, int level, int box, int which, int* out, int cap) {
  Problem* P = static_cast<Problem*>(h);
  if (level < 2 || level > P->depth || P->tree.empty()) return -1;
  const Box& b = P->tree[level][box];
  const std::vector<int>* v = which == 0 ? &b.in_check : which == 1 ? &b.in_charge : which == 2 ? &b.out_check : &b.out_charge;
  int n = (int)v->size();
  for (int i = 0; i < n && i < cap; ++i) out[i] = (*v)[i];
  return n;
}

}  // extern "C"
