// k_geom.cu -- grid points, contrast and plane-wave right-hand sides on the device.
//
// Replaces LS2DTree::createUniformTree / assignLeafChargeLocations
// (LS/LS_Assembly.hpp:808-890, 1074-1087: Morton order, children 0 BL, 1 BR,
// 2 TR, 3 TL; leaf nodes r * cheb + centre, local index y*n + x) and the
// contrast / right-hand side functions of LS/LS_functions.hpp:1-120.
#include <algorithm>

#include "kernels.h"

namespace {

__device__ double q_of(int kind, double amp, double width, double radius, double x, double y) {
  switch (kind) {
    case Q_GAUSSIAN160: { double R2 = x * x + y * y; return 1.5 * exp(-160.0 * R2); }
    case Q_MULTI_GAUSS: {
      const double cx[20] = {-1.17182014706864, -0.861066625441127, -1.14533939124057, -0.856639124568525,
        -0.620066350133170, -0.457064031294315, -0.482782006538245, -0.635070123186999, 0.108594058866164,
        -0.0315722590552472, -0.177274727610547, 0.0342987980936911, 0.369662097773613, 0.591444264226524,
        0.401225715100565, 0.666822699314234, 1.10327781188617, 0.827519268441487, 0.873411278211136, 1.09482906183464};
      const double cy[20] = {-0.361066625441127, 0.0719520938231629, 0.354660608759432, 1.14336087543147,
        -1.12006635013317, -0.457064031294315, 0.364929876813001, 0.802261227250738, -0.394084977497864,
        -0.0315722590552472, 0.322725272389453, 1.03429879809369, -1.13033790222639, 0.0137164199764117,
        0.401225715100565, 1.16682269931423, -0.345187707108795, -0.172480731558513, 0.373411278211136, 1.09482906183464};
      double q = 0.0, a = 0.0013;
      for (int i = 0; i < 20; ++i) {
        double R2 = (x - cx[i]) * (x - cx[i]) + (y - cy[i]) * (y - cy[i]);
        q += 1.5 * exp(-R2 / a);
      }
      return q;
    }
    case Q_PLASMA: {
      double C = 0.4987;
      double psi = 1.0 - (x - 0.15 * (1 - x * x)) * (x - 0.15 * (1 - x * x)) - C * (1.0 + 0.3 * x) * (1.0 + 0.3 * x) * y * y;
      const double a[5] = {0.45, 0.195, 0.51, 0.195, 0.63}, px[5] = {0.8, 0.54, -0.14, -0.5, 0.18},
                   py[5] = {0.0, -0.28, 0.7, -0.01, 0.8};
      if (psi <= 0.05) return 0.0;
      double g = 0.0;
      for (int i = 0; i < 5; ++i) {
        double t = (x - px[i]) * (x - px[i]) + (y - py[i]) * (y - py[i]);
        g += a[i] * exp(-t / 0.01);
      }
      return -1.5 * (psi - 0.05) - g * cos(0.9 * y);
    }
    case Q_FLATBUMP: { double R2 = x * x + y * y; return 0.5 * erfc(5.0 * (R2 - 1.0)); }
    case Q_CAVITY: {
      double R = sqrt(x * x + y * y), th = atan2(y, x);
      return (1.0 - pow(sin(0.5 * th), 500)) * exp(-2000 * (0.1 - R * R) * (0.1 - R * R));
    }
    case Q_GAUSS_AW: { double R2 = x * x + y * y; return amp * exp(-width * R2); }
    case Q_DISK: { double R2 = x * x + y * y; return R2 < radius * radius ? amp : 0.0; }
    default: { double R = sqrt(x * x + y * y); return 4 * (y - 0.1) * (1.0 - erf(25.0 * (R - 0.3))); }
  }
}

__global__ void geometry_kernel(int n_cheb, int depth, double L, int q_kind, double q_amp, double q_width,
                                double q_radius, const double* __restrict__ cheb, double2* pts, double* q,
                                double2* leafc, int2* leafxy, int nleaf) {
  const int rank = n_cheb * n_cheb;
  const long tot = (long)nleaf * rank;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int k = (int)(t / rank), l = (int)(t % rank);
    double cx = 0.0, cy = 0.0, r = L, rl = L;
    int ix = 0, iy = 0;
    for (int lev = 0; lev < depth; ++lev) {
      const int c = (k >> (2 * (depth - 1 - lev))) & 3;
      if (c == 0) { cx = cx - 0.5 * r; cy = cy - 0.5 * r; }
      else if (c == 1) { cx = cx + 0.5 * r; cy = cy - 0.5 * r; }
      else if (c == 2) { cx = cx + 0.5 * r; cy = cy + 0.5 * r; }
      else { cx = cx - 0.5 * r; cy = cy + 0.5 * r; }
      r = 0.5 * r;
      ix = 2 * ix + ((c == 1 || c == 2) ? 1 : 0);
      iy = 2 * iy + ((c >= 2) ? 1 : 0);
    }
    for (int lev = 0; lev < depth; ++lev) rl = rl / 2.0;
    if (l == 0) { leafc[k] = make_double2(cx, cy); leafxy[k] = make_int2(ix, iy); }
    const double px = rl * cheb[l % n_cheb] + cx;
    const double py = rl * cheb[l / n_cheb] + cy;
    pts[t] = make_double2(px, py);
    q[t] = q_of(q_kind, q_amp, q_width, q_radius, px, py);
  }
}

// b(i, s) = -kappa^2 q(x_i) exp(i kappa (x cos t_s + y sin t_s))   (LS/LS_functions.hpp:113-120)
__global__ void rhs_kernel(const double2* __restrict__ pts, const double* __restrict__ q, double kappa, int N, int nrhs,
                           const double* __restrict__ theta, double2* b) {
  const long tot = (long)N * nrhs;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % N), s = (int)(t / N);
    double ct = cos(theta[s]), st = sin(theta[s]);
    if (theta[s] == 0.0) { ct = 1.0; st = 0.0; }
    const double ph = pts[i].x * ct + pts[i].y * st;
    double sn, cs;
    sincos(kappa * ph, &sn, &cs);
    const double a = -1.0 * kappa * kappa * q[i];
    b[t] = make_double2(a * cs, a * sn);
  }
}

// u_inc = exp(i kappa (x cos t + y sin t)) at every grid point (LS/LS_functions.hpp:113-116
// is the t = 0 case)
__global__ void incident_kernel(const double2* __restrict__ pts, double kappa, int N, int nrhs,
                                const double* __restrict__ theta, double2* u) {
  const long tot = (long)N * nrhs;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % N), s = (int)(t / N);
    double ct = cos(theta[s]), st = sin(theta[s]);
    if (theta[s] == 0.0) { ct = 1.0; st = 0.0; }
    const double ph = pts[i].x * ct + pts[i].y * st;
    double sn, cs;
    sincos(kappa * ph, &sn, &cs);
    u[t] = make_double2(cs, sn);
  }
}

// dst[g.x, g.x + g.z) = src[g.y, g.y + g.z) for every segment g: one warp per segment
__global__ void gather_segments_kernel(const int* __restrict__ src, const int4* __restrict__ segs, long nseg,
                                       int* __restrict__ dst) {
  const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  for (long w = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nseg; w += nwarps) {
    const int4 g = segs[w];
    for (int i = lane; i < g.z; i += 32) dst[(long)g.x + i] = src[(long)g.y + i];
  }
}

}  // namespace

int aifmm_launch_incident_field(const double2* pts, double kappa, int N, int nrhs, const double* theta, double2* u,
                                cudaStream_t s) {
  const long tot = (long)N * nrhs;
  long blocks = (tot + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  if (blocks < 1) return 0;
  incident_kernel<<<(int)blocks, 256, 0, s>>>(pts, kappa, N, nrhs, theta, u);
  return (int)cudaGetLastError();
}

int aifmm_launch_gather_segments(const int* src, const int4* segs, long nseg, int* dst, cudaStream_t s) {
  if (nseg <= 0) return 0;
  long blocks = (nseg * 32 + 255) / 256;
  if (blocks > 148L * 32) blocks = 148L * 32;
  gather_segments_kernel<<<(int)blocks, 256, 0, s>>>(src, segs, nseg, dst);
  return (int)cudaGetLastError();
}

int aifmm_launch_geometry(int n_cheb, int depth, double L, int q_kind, double q_amp, double q_width, double q_radius,
                          const double* cheb, double2* pts, double* q, double2* leafc, int2* leafxy,
                          cudaStream_t s) {
  const int nleaf = 1 << (2 * depth);
  const long tot = (long)nleaf * n_cheb * n_cheb;
  long blocks = (tot + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  geometry_kernel<<<(int)blocks, 256, 0, s>>>(n_cheb, depth, L, q_kind, q_amp, q_width, q_radius, cheb, pts, q,
                                              leafc, leafxy, nleaf);
  return (int)cudaGetLastError();
}

int aifmm_launch_rhs_plane_wave(const double2* pts, const double* q, double kappa, int N, int nrhs,
                                const double* theta, double2* b, cudaStream_t s) {
  const long tot = (long)N * nrhs;
  long blocks = (tot + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  rhs_kernel<<<(int)blocks, 256, 0, s>>>(pts, q, kappa, N, nrhs, theta, b);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------- error norms
// find_error (FMM2DTree_find_error.hpp:2534-2581): ||x - x_true||^2 and
// ||x_true||^2 over an n x nrhs block with column strides ldx / ldt.  Each of a
// fixed number of CTAs sums a fixed slice in a fixed order, and one CTA adds
// the slices in order, so the result does not depend on timing.
namespace {
constexpr int kErrCtas = 148, kErrThreads = 256;

__device__ double block_sum_err(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  v = 0.0;
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;
}

__global__ void __launch_bounds__(kErrThreads) err_partial_kernel(const double2* __restrict__ x, long ldx,
                                                                  const double2* __restrict__ t, long ldt, long n,
                                                                  int nrhs, double* part) {
  __shared__ double sh[kErrThreads / 32];
  const long tot = n * nrhs;
  double se = 0.0, st = 0.0;
  for (long e = blockIdx.x * (long)kErrThreads + threadIdx.x; e < tot; e += (long)kErrCtas * kErrThreads) {
    const long i = e % n, c = e / n;
    const double2 a = x[i + c * ldx], b = t[i + c * ldt];
    const double dr = a.x - b.x, di = a.y - b.y;
    se += dr * dr + di * di;
    st += b.x * b.x + b.y * b.y;
  }
  se = block_sum_err(se, sh);
  st = block_sum_err(st, sh);
  if (threadIdx.x == 0) { part[2 * blockIdx.x] = se; part[2 * blockIdx.x + 1] = st; }
}

__global__ void err_final_kernel(const double* __restrict__ part, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double se = 0.0, st = 0.0;
    for (int b = 0; b < kErrCtas; ++b) { se += part[2 * b]; st += part[2 * b + 1]; }
    out[0] = se;
    out[1] = st;
  }
}
}  // namespace

size_t aifmm_error_norms_scratch_bytes() { return sizeof(double) * 2 * kErrCtas; }

int aifmm_launch_error_norms(const double2* x, long ldx, const double2* t, long ldt, long n, int nrhs, double* part,
                             double* out2, cudaStream_t s) {
  err_partial_kernel<<<kErrCtas, kErrThreads, 0, s>>>(x, ldx, t, ldt, n, nrhs, part);
  err_final_kernel<<<1, 32, 0, s>>>(part, out2);
  return (int)cudaGetLastError();
}

// ---------------------------------------------------------------- column kernels (GMRES)
// For nrhs independent Krylov processes run in lockstep: column c of an
// N x nrhs block (column stride ld) belongs to process c.  One CTA per column
// sums its products in a fixed order, so results do not depend on timing.
namespace {
constexpr int kColThreads = 512;

__global__ void __launch_bounds__(kColThreads) coldot_kernel(const double2* __restrict__ a, long lda,
                                                             const double2* __restrict__ b, long ldb, long n,
                                                             double2* out) {
  __shared__ double sh[kColThreads / 32];
  const int c = blockIdx.x;
  const double2* x = a + c * lda;
  const double2* y = b + c * ldb;
  double re = 0.0, im = 0.0;
  for (long i = threadIdx.x; i < n; i += kColThreads) {  // conj(x) y
    const double2 u = x[i], v = y[i];
    re += u.x * v.x + u.y * v.y;
    im += u.x * v.y - u.y * v.x;
  }
  re = block_sum_err(re, sh);
  im = block_sum_err(im, sh);
  if (threadIdx.x == 0) out[c] = make_double2(re, im);
}

// y(:, c) = alpha_c x(:, c) + beta_c y(:, c) with per-column complex coefficients
__global__ void colaxpby_kernel(const double2* __restrict__ x, long ldx, double2* y, long ldy, long n, int nrhs,
                                const double2* __restrict__ alpha, const double2* __restrict__ beta) {
  const long tot = n * nrhs;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < tot; e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, c = e / n;
    const double2 a = alpha[c], b = beta[c], u = x[i + c * ldx];
    double2* v = y + i + c * ldy;
    const double2 w = *v;
    *v = make_double2(a.x * u.x - a.y * u.y + b.x * w.x - b.y * w.y, a.x * u.y + a.y * u.x + b.x * w.y + b.y * w.x);
  }
}
}  // namespace

int aifmm_launch_coldot(const double2* a, long lda, const double2* b, long ldb, long n, int nrhs, double2* out,
                        cudaStream_t s) {
  coldot_kernel<<<nrhs, kColThreads, 0, s>>>(a, lda, b, ldb, n, out);
  return (int)cudaGetLastError();
}

int aifmm_launch_colaxpby(const double2* x, long ldx, double2* y, long ldy, long n, int nrhs, const double2* alpha,
                          const double2* beta, cudaStream_t s) {
  const long tot = n * nrhs;
  const int blocks = (int)std::min<long>((tot + 255) / 256, 148L * 16);
  colaxpby_kernel<<<blocks, 256, 0, s>>>(x, ldx, y, ldy, n, nrhs, alpha, beta);
  return (int)cudaGetLastError();
}
