// k_geom.cu -- grid points, contrast and plane-wave right-hand sides on the device.
//
// Replaces LS2DTree::createUniformTree / assignLeafChargeLocations
// (LS/LS_Assembly.hpp:808-890, 1074-1087: Morton order, children 0 BL, 1 BR,
// 2 TR, 3 TL; leaf nodes r * cheb + centre, local index y*n + x) and the
// contrast / right-hand side functions of LS/LS_functions.hpp:1-120.
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
