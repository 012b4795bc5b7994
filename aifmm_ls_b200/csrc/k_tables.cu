// k_tables.cu -- leaf-level interaction tables by adaptive Gauss-Legendre
// quadrature on the GPU (one warp per integral, explicit depth-first stack).
//
// Replaces the reference's precomputation, which is what getMatrixEntry reads
// for a uniform tree (only the leaf level's tables are ever used):
//  * far field: C(n, l) = r^2 int_{[-1,1]^2} J_n(kappa r |P|) e^{-in theta_P} T_a(x) T_b(y) dP
//    (LS/FarFieldInteraction.hpp:62-74, 115-135), M = C Q^+ (:152-160)
//  * near field, 9 colleague directions: V(i, l) = int H0(kappa r |X_i - P|) T_a T_b dP
//    (LS/NearFieldInteraction1.hpp:98-128), table = (i r^2/4) V Q^+ (LS/LS_Assembly.hpp:1290-1317)
//  * quadrature: LS/domain2D.hpp:46-138 -- a panel is split in four; the parent is
//    accepted when |I_parent - sum I_child| < 1e-7, otherwise every child is refined;
//    the result is the sum of accepted panels' own estimates in depth-first order.
#include "kernels.h"

namespace {

struct QuadParams {
  int n_cheb, rank, nb;       // nb = degree (degree + 1) / 2
  double kappa, r;            // wavenumber, leaf half width
  const double* gl_x;         // 10 Gauss-Legendre nodes (reference order)
  const double* gl_w;
  const int2* basis;          // (a, b) per basis function
  const double* cheb;         // n_cheb 1-D Chebyshev nodes
  double2* C;                 // 121 x nb (column-major)
  double2* V;                 // 9 * rank x nb  (row = dir * rank + i)
  int* status;                // nonzero on stack overflow / panel budget exhausted
};

__device__ double cheb_T(double x, int n) { return cos(n * acos(x)); }

// J_n(x) for a single order n >= 0 (x >= 0)
__device__ double jn_single(int n, double x) {
  if (x == 0.0) return n == 0 ? 1.0 : 0.0;
  if (x <= 8.0) {
    // power series: sum_k (-1)^k (x/2)^{2k+n} / (k! (n+k)!)
    double lead = 1.0, h = 0.5 * x;
    for (int k = 1; k <= n; ++k) lead *= h / k;
    double t = lead, s = lead, q = -h * h;
    for (int k = 1; k < 200; ++k) {
      t *= q / ((double)k * (double)(n + k));
      s += t;
      if (fabs(t) < 1e-18 * fabs(s)) break;
    }
    return s;
  }
  if (n < x) {
    double a = j0(x), b = j1(x);
    if (n == 0) return a;
    for (int k = 1; k < n; ++k) { double c = (2.0 * k / x) * b - a; a = b; b = c; }
    return b;
  }
  int N = (int)(fmax((double)n, x) + 24.0 + 10.0 * cbrt(fmax((double)n, x)));
  N += (N & 1);
  double jp1 = 0.0, jc = 1e-250, norm = 2.0 * jc, want = 0.0;
  for (int k = N; k >= 1; --k) {
    double jm = ((2.0 * k) / x) * jc - jp1;
    jp1 = jc; jc = jm;
    if (((k - 1) & 1) == 0) norm += (k - 1 == 0 ? 1.0 : 2.0) * jm;
    if (k - 1 == n) want = jm;
    if (fabs(jc) > 1e200) { jc *= 1e-200; jp1 *= 1e-200; norm *= 1e-200; want *= 1e-200; }
  }
  return want / norm;
}

struct Panel { double xc, yc, xr, yr; double2 I; };

template <bool FAR>
__device__ double2 integrand(const QuadParams& P, int task, double x, double y) {
  if (FAR) {
    const int nn = task / P.nb - 60, l = task % P.nb;
    const int2 ab = P.basis[l];
    const double R2 = x * x + y * y;
    const double normX = sqrt(R2);
    const double argJ = P.kappa * P.r * normX;
    const double th = atan2(y, x);
    const int m = nn < 0 ? -nn : nn;
    double jv = jn_single(m, argJ);
    if (nn < 0 && (m & 1)) jv = -jv;
    double s, c;
    sincos((double)m * th, &s, &c);
    // exp(-I n theta) = (cos(n theta), -sin(n theta))
    double2 e = make_double2(c, nn >= 0 ? -s : s);
    double2 v = make_double2(jv * e.x, jv * e.y);
    const double ta = cheb_T(x, ab.x), tb = cheb_T(y, ab.y);
    v.x *= ta; v.y *= ta;
    v.x *= tb; v.y *= tb;
    return v;
  } else {
    const int rank = P.rank, n = P.n_cheb;
    const int dir = task / (rank * P.nb);
    const int i = (task / P.nb) % rank;
    const int l = task % P.nb;
    const int2 ab = P.basis[l];
    const double Nc[9][2] = {{-2, -2}, {0, -2}, {2, -2}, {2, 0}, {2, 2}, {0, 2}, {-2, 2}, {-2, 0}, {0, 0}};
    const double cbx = Nc[dir][0] * P.r, cby = Nc[dir][1] * P.r;
    const double ax = P.r * P.cheb[i % n] + 0.0, ay = P.r * P.cheb[i / n] + 0.0;
    const double Xx = (ax - cbx) / P.r, Xy = (ay - cby) / P.r;
    const double R2 = (Xx - x) * (Xx - x) + (Xy - y) * (Xy - y);
    const double R = sqrt(R2);
    const double arg = P.kappa * P.r * R;
    double2 h = make_double2(j0(arg), y0(arg));
    const double ta = cheb_T(x, ab.x), tb = cheb_T(y, ab.y);
    h.x *= ta; h.y *= ta;
    h.x *= tb; h.y *= tb;
    return h;
  }
}

// integral over one panel; all 32 lanes participate, result valid in every lane.
// The 100 weighted values are summed by one lane in the reference's (m, n) order.
template <bool FAR>
__device__ double2 panel_integral(const QuadParams& P, int task, double xc, double yc, double xr, double yr,
                                  double2* buf /* 100 per warp */) {
  const int lane = threadIdx.x & 31;
  for (int p = lane; p < 100; p += 32) {
    const int m = p / 10, n = p % 10;
    const double x = xc + xr * P.gl_x[m];
    const double y = yc + yr * P.gl_x[n];
    const double w = P.gl_w[m] * P.gl_w[n];
    double2 f = integrand<FAR>(P, task, x, y);
    buf[p] = make_double2(w * f.x, w * f.y);
  }
  __syncwarp();
  double2 s = make_double2(0.0, 0.0);
  if (lane == 0) {
    for (int p = 0; p < 100; ++p) { s.x += buf[p].x; s.y += buf[p].y; }
    const double a = xr * yr;
    s.x *= a; s.y *= a;
  }
  __syncwarp();
  s.x = __shfl_sync(0xffffffffu, s.x, 0);
  s.y = __shfl_sync(0xffffffffu, s.y, 0);
  return s;
}

constexpr int kStack = 160;
constexpr int kWarps = 4;

template <bool FAR>
__global__ void __launch_bounds__(32 * kWarps) quad_kernel(QuadParams P, int ntasks, double eps) {
  __shared__ double2 sbuf[kWarps][100];
  __shared__ Panel sstack[kWarps][kStack];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int task = blockIdx.x * kWarps + w;
  if (task >= ntasks) return;
  double2* buf = sbuf[w];
  Panel* st = sstack[w];
  double2 acc = make_double2(0.0, 0.0);
  double2 root = panel_integral<FAR>(P, task, 0.0, 0.0, 1.0, 1.0, buf);
  int top = 0;
  if (lane == 0) st[0] = Panel{0.0, 0.0, 1.0, 1.0, root};
  top = 1;
  __syncwarp();
  long budget = 400000;
  bool failed = false;
  while (top > 0) {
    Panel pa = st[top - 1];
    __syncwarp();
    --top;
    const double hx = 0.5 * pa.xr, hy = 0.5 * pa.yr;
    const double cx[4] = {pa.xc - hx, pa.xc + hx, pa.xc + hx, pa.xc - hx};
    const double cy[4] = {pa.yc - hy, pa.yc - hy, pa.yc + hy, pa.yc + hy};
    double2 ic[4];
    for (int l = 0; l < 4; ++l) ic[l] = panel_integral<FAR>(P, task, cx[l], cy[l], hx, hy, buf);
    double2 err = pa.I;
    for (int l = 0; l < 4; ++l) err = csub(err, ic[l]);
    if (--budget <= 0 || top + 4 > kStack) failed = true;
    if (hypot(err.x, err.y) < eps || failed) {
      acc = cadd(acc, pa.I);
    } else {
      if (lane == 0)
        for (int l = 3; l >= 0; --l) st[top + (3 - l)] = Panel{cx[l], cy[l], hx, hy, ic[l]};
      top += 4;
      __syncwarp();
    }
    if (failed) break;
  }
  if (lane == 0) {
    if (failed) atomicExch(P.status, 1);
    if (FAR) {
      const int nn = task / P.nb, l = task % P.nb;
      const double rr = P.r * P.r;
      P.C[nn + (size_t)l * 121] = make_double2(rr * acc.x, rr * acc.y);
    } else {
      P.V[task] = acc;  // (dir*rank + i) * nb + l  -> row-major V[row][l]
    }
  }
}

// Q (rank x nb) Chebyshev Vandermonde at the leaf nodes, Q^+ = (Q^T Q)^{-1} Q^T by
// Cholesky (Q has orthogonal columns on tensor Chebyshev nodes, so this is benign),
// then M = C Q^+ and near = (V * i r^2 / 4) Q^+ .  One CTA.
__global__ void tables_finish_kernel(QuadParams P, double* qpinv_out, double2* M, double2* nearT) {
  extern __shared__ double sm[];
  const int rank = P.rank, nb = P.nb, n = P.n_cheb;
  double* Q = sm;                    // rank x nb
  double* G = Q + rank * nb;         // nb x nb
  double* Qp = G + nb * nb;          // nb x rank
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int t = tid; t < rank * nb; t += nt) {
    int i = t % rank, l = t / rank;
    int2 ab = P.basis[l];
    Q[i + l * rank] = cheb_T(P.cheb[i % n], ab.x) * cheb_T(P.cheb[i / n], ab.y);
  }
  __syncthreads();
  for (int t = tid; t < nb * nb; t += nt) {
    int a = t % nb, b = t / nb;
    double s = 0.0;
    for (int i = 0; i < rank; ++i) s += Q[i + a * rank] * Q[i + b * rank];
    G[a + b * nb] = s;
  }
  __syncthreads();
  if (tid == 0) {  // Cholesky G = L L^T in place (lower)
    for (int k = 0; k < nb; ++k) {
      double d = G[k + k * nb];
      for (int p = 0; p < k; ++p) d -= G[k + p * nb] * G[k + p * nb];
      d = sqrt(d);
      G[k + k * nb] = d;
      for (int i = k + 1; i < nb; ++i) {
        double s = G[i + k * nb];
        for (int p = 0; p < k; ++p) s -= G[i + p * nb] * G[k + p * nb];
        G[i + k * nb] = s / d;
      }
    }
  }
  __syncthreads();
  for (int col = tid; col < rank; col += nt) {  // solve G x = Q^T e_col
    double x[64];
    for (int a = 0; a < nb; ++a) x[a] = Q[col + a * rank];
    for (int a = 0; a < nb; ++a) {
      double s = x[a];
      for (int p = 0; p < a; ++p) s -= G[a + p * nb] * x[p];
      x[a] = s / G[a + a * nb];
    }
    for (int a = nb - 1; a >= 0; --a) {
      double s = x[a];
      for (int p = a + 1; p < nb; ++p) s -= G[p + a * nb] * x[p];
      x[a] = s / G[a + a * nb];
    }
    for (int a = 0; a < nb; ++a) Qp[a + col * nb] = x[a];
  }
  __syncthreads();
  for (int t = tid; t < nb * rank; t += nt) qpinv_out[t] = Qp[t];
  for (int t = tid; t < 121 * rank; t += nt) {
    int r = t % 121, j = t / 121;
    double2 s = make_double2(0.0, 0.0);
    for (int l = 0; l < nb; ++l) {
      double2 c = P.C[r + (size_t)l * 121];
      double qv = Qp[l + j * nb];
      s.x += c.x * qv; s.y += c.y * qv;
    }
    M[r + (size_t)j * 121] = s;
  }
  const double rB = P.r;
  for (int t = tid; t < 9 * rank * rank; t += nt) {
    int dir = t / (rank * rank), rem = t % (rank * rank);
    int i = rem % rank, j = rem / rank;
    double2 s = make_double2(0.0, 0.0);
    for (int l = 0; l < nb; ++l) {
      double2 v = P.V[((size_t)dir * rank + i) * nb + l];
      // ((V * I) * r) * r / 4  (LS_Assembly.hpp:1313)
      double2 vt = make_double2(-v.y, v.x);
      vt.x = vt.x * rB; vt.y = vt.y * rB;
      vt.x = vt.x * rB; vt.y = vt.y * rB;
      vt.x = vt.x / 4.0; vt.y = vt.y / 4.0;
      double qv = Qp[l + j * nb];
      s.x += vt.x * qv; s.y += vt.y * qv;
    }
    nearT[(size_t)dir * rank * rank + i + (size_t)j * rank] = s;
  }
}

}  // namespace

// Host launcher: all pointers are device pointers.  Returns a CUDA error code.
int aifmm_launch_tables(int n_cheb, int degree, double kappa, double r, const double* gl_x, const double* gl_w,
                        const int2* basis, const double* cheb, double2* Cwork, double2* Vwork, int* status,
                        double* qpinv, double2* M, double2* nearT, cudaStream_t stream) {
  QuadParams P;
  P.n_cheb = n_cheb; P.rank = n_cheb * n_cheb; P.nb = degree * (degree + 1) / 2;
  P.kappa = kappa; P.r = r; P.gl_x = gl_x; P.gl_w = gl_w; P.basis = basis; P.cheb = cheb;
  P.C = Cwork; P.V = Vwork; P.status = status;
  const double eps = 1e-7;  // LS/FarFieldInteraction.hpp:37, LS/NearFieldInteraction1.hpp:112
  int nfar = 121 * P.nb, nnear = 9 * P.rank * P.nb;
  quad_kernel<true><<<(nfar + kWarps - 1) / kWarps, 32 * kWarps, 0, stream>>>(P, nfar, eps);
  quad_kernel<false><<<(nnear + kWarps - 1) / kWarps, 32 * kWarps, 0, stream>>>(P, nnear, eps);
  size_t smem = sizeof(double) * ((size_t)P.rank * P.nb + P.nb * P.nb + P.nb * P.rank);
  if (smem > 200 * 1024 || P.nb > 64) return (int)cudaErrorInvalidValue;
  cudaFuncSetAttribute(tables_finish_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  tables_finish_kernel<<<1, 256, smem, stream>>>(P, qpinv, M, nearT);
  return (int)cudaGetLastError();
}
