// k_dense.cu -- batched small dense complex linear algebra for the bases and the
// hierarchical elimination.
//
//  * Householder QR with column pivoting: the semantics of Eigen's
//    ColPivHouseholderQR as used by FMM2DTree_find_error.hpp (:1535, :1819,
//    :2092, :2477, :2493, :2510): pivot = first remaining column of largest
//    (downdated) norm, LAPACK xGEQP3 norm downdating (LAPACK Working Note 176),
//    reflector G = I - tau v v^H with beta = -sign(Re a_kk) |x|, exactly-nonzero
//    pivot count from the eps-scaled initial column norm, rank() = #|R_ii| >
//    threshold * max|R_ii|, solve() using only the nonzero pivots.
//  * QR solves, explicit Q (householderQ().block(...)).
//  * Partial-pivoting LU solves for the interpolative operators
//    (get_L2P_P2M_box, :1105-1128).
//  * Batched GEMM / GEAM / Frobenius norms.
// One CTA per factorisation; everything else is batched over descriptor lists.
#include <algorithm>
#include <cfloat>
#include "kernels.h"
#include "entry.cuh"

namespace {

constexpr int kT = 256;
constexpr int kW = kT / 32;
constexpr double kPivotTie = 1e-11;  // same pivot tie tolerance as the ACA

// Real-type constants of the two forms: machine epsilon, the smallest normal
// number, and the range inside which a product may be inverted directly.
template <typename R> struct rl;
template <> struct rl<double> {
  static constexpr double eps = DBL_EPSILON, tiny = DBL_MIN, lo = 1e-290, hi = 1e290;
};
template <> struct rl<float> {
  static constexpr float eps = FLT_EPSILON, tiny = FLT_MIN, lo = 1e-35f, hi = 1e35f;
};

// Norms, reflector scalars and pivot reciprocals are computed in double for both
// forms: complex64 blocks of the contrast's far corners hold values near 1e-25,
// whose squares underflow FP32 and whose reciprocals overflow it.  The O(m n)
// column updates stay in the blocks' own precision.
__device__ __forceinline__ double cabs2d(double2 a) { return cabs2(a); }
__device__ __forceinline__ double cabs2d(float2 a) { const double x = a.x, y = a.y; return x * x + y * y; }
__device__ __forceinline__ double2 c2d(double2 a) { return a; }
__device__ __forceinline__ double2 c2d(float2 a) { return make_double2(a.x, a.y); }

template <typename R>
__device__ __forceinline__ R warp_sum(R x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}
template <typename C>
__device__ __forceinline__ C warp_sum2(C x) {
  for (int o = 16; o > 0; o >>= 1) {
    x.x += __shfl_xor_sync(0xffffffffu, x.x, o);
    x.y += __shfl_xor_sync(0xffffffffu, x.y, o);
  }
  return x;
}

template <typename R>
__device__ R block_sum(R x, R* sh) {
  x = warp_sum(x);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = x;
  __syncthreads();
  if (threadIdx.x == 0) { R r = 0; for (int w = 0; w < kW; ++w) r += sh[w]; sh[kW] = r; }
  __syncthreads();
  R r = sh[kW];
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------- QR factor
// The factorisation runs on A (lda), nu/nd (norm arrays) and perm, either in
// global memory or staged in shared memory (qr_factor_smem_kernel).
template <typename C>
__device__ void qr_factor_body(const QRJob& J, C* A, int lda, double* nu, double* nd, int* perm) {
  __shared__ double sh[kW + 1];
  __shared__ double sv[kW]; __shared__ int si[kW];
  __shared__ C s_tau;
  __shared__ int s_big;
  C* tau = static_cast<C*>(J.tau);
  const int m = J.m, n = J.n, size = min(m, n);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int j = tid; j < n; j += kT) perm[j] = j;
  // initial column norms (one warp per column)
  for (int j = w; j < n; j += kW) {
    double s = 0.0;
    for (int i = lane; i < m; i += 32) s += cabs2d(A[i + (size_t)j * lda]);
    s = warp_sum(s);
    if (lane == 0) { nu[j] = sqrt(s); nd[j] = nu[j]; }
  }
  __syncthreads();
  double maxnorm = 0.0;
  for (int j = 0; j < n; ++j) maxnorm = fmax(maxnorm, nu[j]);
  const double eps = rl<typename cplx<C>::R>::eps;  // the precision of the data
  const double thr_helper = m > 0 ? (maxnorm * eps) * (maxnorm * eps) / m : 0.0;
  const double downdate_thr = sqrt(eps);
  int nzp = size;
  double maxpivot = 0.0;
  for (int k = 0; k < size; ++k) {
    // pivot: first largest updated norm among columns k..n-1
    double bv = -1.0; int bi = -1;
    for (int j = k + tid; j < n; j += kT) {
      double v = nu[j];
      if (bi < 0 || v > bv) { bv = v; bi = j; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      double ov = __shfl_down_sync(0xffffffffu, bv, o);
      int oi = __shfl_down_sync(0xffffffffu, bi, o);
      if (oi >= 0 && (bi < 0 || ov > bv || (ov == bv && oi < bi))) { bv = ov; bi = oi; }
    }
    if (lane == 0) { sv[w] = bv; si[w] = bi; }
    __syncthreads();
    if (tid == 0) {
      double v = sv[0]; int i = si[0];
      for (int q = 1; q < kW; ++q)
        if (si[q] >= 0 && (i < 0 || sv[q] > v || (sv[q] == v && si[q] < i))) { v = sv[q]; i = si[q]; }
      // norms within kPivotTie of the largest count as tied: first index wins
      const double cut = v * (1.0 - kPivotTie);
      for (int j = k; j < n; ++j)
        if (nu[j] >= cut) { i = j; break; }
      s_big = i;
    }
    __syncthreads();
    const int big = s_big;
    if (nzp == size && nu[big] * nu[big] < thr_helper * (double)(m - k)) nzp = k;
    if (big != k) {
      for (int i = tid; i < m; i += kT) {
        C t = A[i + (size_t)k * lda];
        A[i + (size_t)k * lda] = A[i + (size_t)big * lda];
        A[i + (size_t)big * lda] = t;
      }
      __syncthreads();
      if (tid == 0) {
        double t = nu[k]; nu[k] = nu[big]; nu[big] = t;
        t = nd[k]; nd[k] = nd[big]; nd[big] = t;
        int p = perm[k]; perm[k] = perm[big]; perm[big] = p;
      }
    }
    // reflector for A(k:m, k)
    double tail = 0.0;
    for (int i = k + 1 + tid; i < m; i += kT) tail += cabs2d(A[i + (size_t)k * lda]);
    tail = block_sum(tail, sh);
    const double2 c0 = c2d(A[k + (size_t)k * lda]);
    double beta;
    if (tail <= DBL_MIN && c0.y * c0.y <= DBL_MIN) {
      beta = c0.x;
      if (tid == 0) { s_tau = cplx<C>::mk(0.0, 0.0); }
      for (int i = k + 1 + tid; i < m; i += kT) A[i + (size_t)k * lda] = cplx<C>::mk(0.0, 0.0);
    } else {
      beta = sqrt(cabs2(c0) + tail);
      if (c0.x >= 0.0) beta = -beta;
      const double2 den = make_double2(c0.x - beta, c0.y);
      if (tid == 0) {
        s_tau = cplx<C>::from(cconj(cdiv(make_double2(beta - c0.x, -c0.y), make_double2(beta, 0.0))));
      }
      for (int i = k + 1 + tid; i < m; i += kT)
        A[i + (size_t)k * lda] = cplx<C>::from(cdiv(c2d(A[i + (size_t)k * lda]), den));
    }
    __syncthreads();
    const C t = s_tau;
    if (tid == 0) { A[k + (size_t)k * lda] = cplx<C>::mk(beta, 0.0); tau[k] = t; }
    maxpivot = fmax(maxpivot, fabs(beta));
    // apply G = I - t v v^H to columns k+1.. (one warp per column), then downdate norms
    for (int j = k + 1 + w; j < n; j += kW) {
      C* col = A + (size_t)j * lda;
      const C* v = A + (size_t)k * lda;
      C s = cplx<C>::mk(0.0, 0.0);
      for (int i = k + 1 + lane; i < m; i += 32) s = cfmac(v[i], col[i], s);
      s = warp_sum2(s);
      const C wv = cadd(col[k], s);
      const C tw = cmul(t, wv);
      for (int i = k + 1 + lane; i < m; i += 32) col[i] = csub(col[i], cmul(cmul(t, v[i]), wv));
      __syncwarp();
      if (lane == 0) col[k] = csub(col[k], tw);
      __syncwarp();
      // LAWN 176 downdate
      double upd = nu[j];
      if (upd != 0.0) {
        const double2 rkj = c2d(col[k]);
        double tmp = hypot(rkj.x, rkj.y) / upd;
        tmp = (1.0 + tmp) * (1.0 - tmp);
        if (tmp < 0.0) tmp = 0.0;
        double rr = upd / nd[j];
        double tmp2 = tmp * rr * rr;
        if (tmp2 <= downdate_thr) {
          double ss = 0.0;
          for (int i = k + 1 + lane; i < m; i += 32) ss += cabs2d(col[i]);
          ss = warp_sum(ss);
          if (lane == 0) { nd[j] = sqrt(ss); nu[j] = nd[j]; }
        } else if (lane == 0) {
          nu[j] = upd * sqrt(tmp);
        }
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    const double thr = J.thr > 0.0 ? J.thr : (double)size * eps;
    const double pre = fabs(maxpivot) * thr;
    int rk = 0;
    for (int i = 0; i < nzp; ++i) rk += (cabsd(A[i + (size_t)i * lda]) > pre);
    J.info[0] = nzp;
    J.info[1] = rk;
    if (J.maxpiv) J.maxpiv[0] = maxpivot;
  }
}

template <typename C>
__global__ void __launch_bounds__(kT) qr_factor_kernel(const QRJob* __restrict__ jobs) {
  const QRJob J = jobs[blockIdx.x];
  qr_factor_body<C>(J, static_cast<C*>(J.a), J.lda, J.norms, J.norms + J.n, J.perm);
}

// Jobs whose matrix fits in shared memory, one barrier per pivot step.
// The matrix sits in shared memory by original column ("slot"); a column swap
// only exchanges the positions that two slots carry.  Each pivot step:
//   1. every warp selects the pivot from the shared norms/positions and builds
//      the reflector from the pivot column into its own buffer (all warps get the
//      same bits: same data, same reduction order), so no warp waits for another;
//   2. warp (k mod warps) writes the finished pivot column -- R above, beta on,
//      the reflector below the diagonal -- straight to global memory;
//   3. the four lanes of a group apply the reflector to each column the group
//      owns (slots g, g + 64, ...; rows interleaved over the lanes) and downdate
//      its norm;
//   4. one barrier.
// Norms and positions are double-buffered by step parity, so a warp running
// ahead never changes what a slower warp is still scanning.  Columns left at
// positions >= min(m, n) are written out at the end.
// Arithmetic: pivot ties as in qr_factor_body; the reflector scalars tau and
// 1/(a_kk - beta) come from one division; the norm downdate of LAPACK Working
// Note 176 is evaluated without divisions -- with T = (nu - |r|)(nu + |r|) (the
// LAWN quantity (1 - (|r|/nu)^2) times nu^2), the column is recomputed when
// T <= sqrt(eps) nd^2 and otherwise nu becomes sqrt(T).
constexpr int kQrGroups = kT / 4;
__host__ __device__ __forceinline__ int qr_smem_ld(int m) { return m + ((12 - (m & 7)) & 7); }  // ld = 4 (mod 8)

template <typename C>
__device__ void qr_smem_body(const QRJob& J, C* qsm) {
  const int m = J.m, n = J.n, size = min(m, n);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, p = tid & 3, g = tid >> 2;
  const int ld = qr_smem_ld(m);
  const unsigned full = 0xffffffffu, gm = 0xfu << (lane & ~3);
  C* A = qsm;                                                    // ld x n, by slot
  C* V = A + (size_t)ld * n;                                     // kW x m: each warp's reflector
  double* snu2 = reinterpret_cast<double*>(V + (size_t)kW * m);  // 2 x n: norms, by step parity
  double* snd = snu2 + 2 * n;                                    // n: norms at the last recompute
  double* srd = snd + n;                                         // size: |R_kk|
  int* spos2 = reinterpret_cast<int*>(srd + size);               // 2 x n: positions, by step parity
  const C* Ja = static_cast<const C*>(J.a);
  C* Jout = static_cast<C*>(J.a);
  C* Jtau = static_cast<C*>(J.tau);
  for (int e = tid; e < m * n; e += kT) {
    const int i = e % m, j = e / m;
    A[i + (size_t)j * ld] = Ja[i + (size_t)j * J.lda];
  }
  __syncthreads();
  for (int s = g; s < n; s += kQrGroups) {
    const C* col = A + (size_t)s * ld;
    double q = 0.0;
    for (int i = p; i < m; i += 4) q += cabs2d(col[i]);
    q += __shfl_xor_sync(gm, q, 1);
    q += __shfl_xor_sync(gm, q, 2);
    if (p == 0) { snu2[s] = snd[s] = sqrt(q); spos2[s] = s; }
  }
  __syncthreads();
  const int nscan = (n + 31) >> 5;
  double maxnorm = 0.0;
  for (int q = 0; q < nscan; ++q) { const int s = lane + 32 * q; if (s < n) maxnorm = fmax(maxnorm, snu2[s]); }
  for (int o = 16; o > 0; o >>= 1) maxnorm = fmax(maxnorm, __shfl_xor_sync(full, maxnorm, o));
  const double eps = rl<typename cplx<C>::R>::eps;  // the precision of the data
  const double thr_helper = m > 0 ? (maxnorm * eps) * (maxnorm * eps) / m : 0.0;
  const double downdate_thr = sqrt(eps);
  C* vw = V + (size_t)w * m;
  int nzp = size;
  double maxpivot = 0.0;
  for (int k = 0; k < size; ++k) {
    const double* snu = snu2 + (k & 1) * n;
    const int* spos = spos2 + (k & 1) * n;
    double* snu_n = snu2 + ((k + 1) & 1) * n;
    int* spos_n = spos2 + ((k + 1) & 1) * n;
    // 1. pivot: largest norm at positions >= k, the first position within the
    //    tie tolerance.  Norms are non-negative: their bit patterns order like
    //    their values, so the maximum is two unsigned warp reductions.
    unsigned hi = 0, lo = 0;
    for (int q = 0; q < nscan; ++q) {
      const int s = lane + 32 * q;
      if (s < n && spos[s] >= k) {
        const double v = snu[s];
        const unsigned h = (unsigned)__double2hiint(v), l = (unsigned)__double2loint(v);
        if (h > hi || (h == hi && l > lo)) { hi = h; lo = l; }
      }
    }
    const unsigned mh = __reduce_max_sync(full, hi);
    const unsigned ml = __reduce_max_sync(full, hi == mh ? lo : 0u);
    const double cut = __hiloint2double((int)mh, (int)ml) * (1.0 - kPivotTie);
    unsigned key = 0xffffffffu;
    for (int q = 0; q < nscan; ++q) {
      const int s = lane + 32 * q;
      if (s < n) {
        const int ps = spos[s];
        if (ps >= k && snu[s] >= cut) key = min(key, (unsigned)ps * 1024u + (unsigned)s);
      }
    }
    key = __reduce_min_sync(full, key);
    const int big = (int)(key >> 10), bslot = (int)(key & 1023u);
    const double nub = snu[bslot];
    if (nzp == size && nub * nub < thr_helper * (double)(m - k)) nzp = k;
    //    reflector for the pivot column, rows k..m-1
    const C* pc = A + (size_t)bslot * ld;
    double tail = 0.0;
    for (int i = k + 1 + lane; i < m; i += 32) tail += cabs2d(pc[i]);
    for (int o = 16; o > 0; o >>= 1) tail += __shfl_xor_sync(full, tail, o);
    const double2 c0 = c2d(pc[k]);
    double beta;
    C t;
    if (tail <= DBL_MIN && c0.y * c0.y <= DBL_MIN) {
      beta = c0.x;
      t = cplx<C>::mk(0.0, 0.0);
      for (int i = k + 1 + lane; i < m; i += 32) vw[i] = cplx<C>::mk(0.0, 0.0);
    } else {
      beta = sqrt(cabs2(c0) + tail);
      if (c0.x >= 0.0) beta = -beta;
      const double2 den = make_double2(c0.x - beta, c0.y);
      const double dd = cabs2(den);
      const double prod = beta * dd;
      double ib, idd;  // 1/beta, 1/|den|^2
      if (fabs(prod) > 1e-290 && fabs(prod) < 1e290) {
        const double q = 1.0 / prod;
        ib = dd * q;
        idd = beta * q;
      } else {
        ib = 1.0 / beta;
        idd = 1.0 / dd;
      }
      t = cplx<C>::from(make_double2((beta - c0.x) * ib, c0.y * ib));  // conj((beta - a_kk) / beta)
      const double2 rden = make_double2(den.x * idd, -den.y * idd);    // 1 / (a_kk - beta)
      for (int i = k + 1 + lane; i < m; i += 32) vw[i] = cplx<C>::from(cmul(c2d(pc[i]), rden));
    }
    maxpivot = fmax(maxpivot, fabs(beta));
    __syncwarp();
    // 2. the finished pivot column goes to position k
    if (w == (k & (kW - 1))) {
      C* out = Jout + (size_t)k * J.lda;
      for (int i = lane; i < m; i += 32) out[i] = i < k ? pc[i] : (i == k ? cplx<C>::mk(beta, 0.0) : vw[i]);
      if (lane == 0) { Jtau[k] = t; J.perm[k] = bslot; srd[k] = fabs(beta); }
    }
    // 3. G = I - t v v^H on the columns at positions > k; norm downdates
    for (int s = g; s < n; s += kQrGroups) {
      int ps = spos[s];
      if (ps == big) ps = k;
      else if (ps == k) ps = big;
      if (ps > k) {
        C* col = A + (size_t)s * ld;
        const int i0 = k + 1 + ((p - (k + 1)) & 3);  // this lane's first row below k
        C d0 = cplx<C>::mk(0.0, 0.0), d1 = cplx<C>::mk(0.0, 0.0);
        int i = i0;
        for (; i + 4 < m; i += 8) { d0 = cfmac(vw[i], col[i], d0); d1 = cfmac(vw[i + 4], col[i + 4], d1); }
        if (i < m) d0 = cfmac(vw[i], col[i], d0);
        C d = cadd(d0, d1);
        d.x += __shfl_xor_sync(gm, d.x, 1); d.y += __shfl_xor_sync(gm, d.y, 1);
        d.x += __shfl_xor_sync(gm, d.x, 2); d.y += __shfl_xor_sync(gm, d.y, 2);
        const C akj = col[k];
        const C tw = cmul(t, cadd(akj, d));
        for (int r = i0; r < m; r += 4) col[r] = csub(col[r], cmul(vw[r], tw));
        const C rkj = csub(akj, tw);
        __syncwarp(gm);
        if (p == 0) col[k] = rkj;
        double nu = snu[s], nd = snd[s];
        if (nu != 0.0) {
          const double ar = sqrt(cabs2d(rkj));
          double tt = (nu - ar) * (nu + ar);
          if (tt < 0.0) tt = 0.0;
          if (tt <= downdate_thr * (nd * nd)) {
            double q = 0.0;
            for (int r = i0; r < m; r += 4) q += cabs2d(col[r]);
            q += __shfl_xor_sync(gm, q, 1);
            q += __shfl_xor_sync(gm, q, 2);
            nd = sqrt(q);
            nu = nd;
          } else {
            nu = sqrt(tt);
          }
        }
        if (p == 0) { snu_n[s] = nu; snd[s] = nd; }
      }
      if (p == 0) spos_n[s] = ps;
    }
    __syncthreads();
  }
  // 4. columns that were never pivots (positions >= size)
  const int* spos = spos2 + (size & 1) * n;
  for (int s = g; s < n; s += kQrGroups) {
    const int ps = spos[s];
    if (ps >= size) {
      const C* col = A + (size_t)s * ld;
      C* out = Jout + (size_t)ps * J.lda;
      for (int i = p; i < m; i += 4) out[i] = col[i];
      if (p == 0) J.perm[ps] = s;
    }
  }
  if (tid == 0) {
    const double thr = J.thr > 0.0 ? J.thr : (double)size * eps;
    const double pre = fabs(maxpivot) * thr;
    int rk = 0;
    for (int i = 0; i < nzp; ++i) rk += (srd[i] > pre);
    J.info[0] = nzp;
    J.info[1] = rk;
    if (J.maxpiv) J.maxpiv[0] = maxpivot;
  }
}

template <typename C>
__global__ void __launch_bounds__(kT) qr_factor_smem_kernel(const QRJob* __restrict__ jobs) {
  extern __shared__ double2 qsm[];
  const QRJob J = jobs[blockIdx.x];
  qr_smem_body<C>(J, reinterpret_cast<C*>(qsm));
}

// ---------------------------------------------------------------- fused compression
// CTA-wide building blocks on global-memory operands (written earlier by the
// same CTA; a __syncthreads separates producer and consumer).

// C (m x n, ldc) = alpha op(A) op(B) + beta C; op 1 = conjugate transpose.
// Accumulation over k in increasing order, as gemm_kernel.
template <typename C>
__device__ void cta_gemm(C* Cm, int ldc, int m, int n, int k, const C* A, int lda, int opA,
                         const C* B, int ldb, int opB, double2 alpha_, double2 beta_) {
  const bool zero_beta = beta_.x == 0.0 && beta_.y == 0.0;
  const C alpha = cplx<C>::from(alpha_), beta = cplx<C>::from(beta_);
  for (int o = threadIdx.x; o < m * n; o += kT) {
    const int i = o % m, jj = o / m;
    C acc = cplx<C>::mk(0.0, 0.0);
#pragma unroll 4
    for (int kk = 0; kk < k; ++kk) {
      const C a = opA ? cconj(A[kk + (size_t)i * lda]) : A[i + (size_t)kk * lda];
      const C b = opB ? cconj(B[jj + (size_t)kk * ldb]) : B[kk + (size_t)jj * ldb];
      acc = cfma(a, b, acc);
    }
    C v = cmul(alpha, acc);
    if (!zero_beta) v = cadd(v, cmul(beta, Cm[i + (size_t)jj * ldc]));
    Cm[i + (size_t)jj * ldc] = v;
  }
}

size_t aifmm_formq_smem_bytes(int m, int size, int ncols, int es) {
  return (size_t)es * ((size_t)(m | 1) * size + size + (size_t)m * ncols);
}

// Q(:, 0:ncols) = householderQ() of an m x n factor (reflectors below the
// diagonal of qr, coefficients tau): column c is G_0^H ... G_min(c, size-1)^H e_c.
// The factor is staged in shared memory; the four lanes of a group build one
// column (rows interleaved), reducing the reflector dot products by shuffles.
template <typename C>
__device__ void cta_formq(const C* qr, int ldq, int m, int n, const C* tau, C* Q, int ldQ, int ncols, C* sm) {
  const int size = min(m, n), ldf = m | 1;
  const int tid = threadIdx.x, lane = tid & 31, p = tid & 3, g = tid >> 2;
  const unsigned gm = 0xfu << (lane & ~3);
  C* F = sm;
  C* ts = F + (size_t)ldf * size;
  C* Qs = ts + size;
  for (int e = tid; e < m * size; e += kT) {
    const int i = e % m, j = e / m;
    F[i + (size_t)j * ldf] = qr[i + (size_t)j * ldq];
  }
  for (int k = tid; k < size; k += kT) ts[k] = cconj(tau[k]);
  for (int e = tid; e < m * ncols; e += kT) {
    const int i = e % m, j = e / m;
    Qs[e] = cplx<C>::mk(i == j ? 1.0 : 0.0, 0.0);
  }
  __syncthreads();
  for (int cc = g; cc < ncols; cc += kQrGroups) {
    C* q = Qs + (size_t)cc * m;
    for (int k = min(size - 1, cc); k >= 0; --k) {
      const C* v = F + (size_t)k * ldf;
      const int i0 = k + 1 + ((p - (k + 1)) & 3);
      C d = cplx<C>::mk(0.0, 0.0);
      for (int i = i0; i < m; i += 4) d = cfmac(v[i], q[i], d);
      d.x += __shfl_xor_sync(gm, d.x, 1); d.y += __shfl_xor_sync(gm, d.y, 1);
      d.x += __shfl_xor_sync(gm, d.x, 2); d.y += __shfl_xor_sync(gm, d.y, 2);
      const C qk = q[k];
      const C tw = cmul(ts[k], cadd(qk, d));
      for (int i = i0; i < m; i += 4) q[i] = csub(q[i], cmul(v[i], tw));
      __syncwarp(gm);
      if (p == 0) q[k] = csub(qk, tw);
      __syncwarp(gm);
    }
  }
  __syncthreads();
  for (int e = tid; e < m * ncols; e += kT) {
    const int i = e % m, j = e / m;
    Q[i + (size_t)j * ldQ] = Qs[e];
  }
}

template <typename C>
__global__ void __launch_bounds__(kT) compress_p2p_kernel(const CompressJob* __restrict__ jobs) {
  extern __shared__ double2 csm_raw[];
  C* csm = reinterpret_cast<C*>(csm_raw);
  const CompressJob J = jobs[blockIdx.x];
  const int m = J.m, rK = J.rK, c = J.c, rb = J.rb, n1 = rK + c;
  const int tid = threadIdx.x;
  const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
  const C* L2P = static_cast<const C*>(J.L2P);
  const C* Pkb = static_cast<const C*>(J.Pkb);
  const C* P2M = static_cast<const C*>(J.P2M);
  const C* M2L = static_cast<const C*>(J.M2L);
  C* Acol = static_cast<C*>(J.Acol);
  C* Arow = static_cast<C*>(J.Arow);
  C* tau = static_cast<C*>(J.tau);
  C* nL = static_cast<C*>(J.nL);
  C* nPt = static_cast<C*>(J.nPt);
  C* Rkp = static_cast<C*>(J.Rkp);
  C* Rk = static_cast<C*>(J.Rk);
  C* Rn = static_cast<C*>(J.Rn);
  C* Rnp = static_cast<C*>(J.Rnp);
  C* Tm = static_cast<C*>(J.Tm);
  C* M2Lo = static_cast<C*>(J.M2Lo);
  // [L2P_k | P2P_kb]
  for (int e = tid; e < m * n1; e += kT) {
    const int i = e % m, col = e / m;
    Acol[e] = col < rK ? L2P[i + (size_t)col * J.ldL] : Pkb[i + (size_t)(col - rK) * J.ldP];
  }
  __syncthreads();
  QRJob q{};
  q.a = Acol; q.lda = m; q.m = m; q.n = n1; q.tau = tau; q.perm = J.perm; q.info = J.info; q.thr = J.tol;
  qr_smem_body<C>(q, csm);
  __syncthreads();
  const int rc = J.info[1];
  const int ldc_ = max(rc, 1);
  cta_formq<C>(Acol, m, m, n1, tau, nL, m, rc, csm);
  __syncthreads();
  cta_gemm<C>(Rkp, ldc_, rc, c, m, nL, m, 1, Pkb, J.ldP, 0, one, zero);   // R' = nL^H P2P_kb
  cta_gemm<C>(Rk, ldc_, rc, rK, m, nL, m, 1, L2P, J.ldL, 0, one, zero);   // R = nL^H L2P_k
  __syncthreads();
  // [P2M_b^H | R'^H]
  const int n2 = rb + rc;
  for (int e = tid; e < c * n2; e += kT) {
    const int i = e % c, col = e / c;
    Arow[e] = col < rb ? cconj(P2M[col + (size_t)i * J.ldM]) : cconj(Rkp[(col - rb) + (size_t)i * ldc_]);
  }
  __syncthreads();
  q.a = Arow; q.lda = c; q.m = c; q.n = n2; q.info = J.info + 2;
  qr_smem_body<C>(q, csm);
  __syncthreads();
  const int rr = J.info[3];
  const int ldr_ = max(rr, 1);
  cta_formq<C>(Arow, c, c, n2, tau, nPt, c, rr, csm);
  __syncthreads();
  cta_gemm<C>(Rn, ldr_, rr, rb, c, nPt, c, 1, P2M, J.ldM, 1, one, zero);    // nPt^H P2M_b^H
  cta_gemm<C>(Rnp, ldr_, rr, rc, c, nPt, c, 1, Rkp, ldc_, 1, one, zero);    // nPt^H R'^H
  cta_gemm<C>(Tm, ldc_, rc, rb, rK, Rk, ldc_, 0, M2L, J.ldT, 0, one, zero);  // R M2L_kb
  __syncthreads();
  cta_gemm<C>(M2Lo, J.ldO, rc, rr, rb, Tm, ldc_, 0, Rn, ldr_, 1, one, zero);
  __syncthreads();
  for (int e = tid; e < rc * rr; e += kT) {
    const int i = e % rc, jj = e / rc;
    C* o = M2Lo + i + (size_t)jj * J.ldO;
    *o = cadd(cconj(Rnp[jj + (size_t)i * ldr_]), *o);
  }
  if (tid == 0) { J.ranks[0] = rc; J.ranks[1] = rr; }
}

// ---------------------------------------------------------------- QR solve (warp per column, registers)
// One warp per right-hand side; lane l holds rows l, l+32, ... of its column in
// registers (RPL rows per lane, m <= 32*RPL).  The first nzp columns of the
// factor and tau are staged once per CTA in shared memory.  Only warp shuffles
// synchronise: Q^H b reflector by reflector, then column-oriented back
// substitution with R, then the column permutation.
template <typename C, int RPL>
__global__ void __launch_bounds__(kT) qr_solve_warp_kernel(const SolveJob* __restrict__ jobs,
                                                           const int* __restrict__ cta_off, int njobs) {
  extern __shared__ double2 fsm_raw[];
  int lo = 0, hi = njobs - 1;
  while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (cta_off[mid] <= (int)blockIdx.x) lo = mid; else hi = mid - 1; }
  const SolveJob J = jobs[lo];
  const C* Jqr = static_cast<const C*>(J.qr);
  const C* Jtau = static_cast<const C*>(J.tau);
  const C* JB = static_cast<const C*>(J.B);
  const int m = J.m, n = J.n, nzp = J.info[0];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int c = (blockIdx.x - cta_off[lo]) * kW + w;
  const int ldf = m | 1;
  // 1 / R_kk in double (a complex64 pivot near 1e-40 has no FP32 reciprocal), so
  // that back substitution only multiplies; then the factor and tau
  double2* rinv = fsm_raw;
  C* F = reinterpret_cast<C*>(rinv + nzp);  // m x nzp, ld = m|1
  C* tau = F + (size_t)ldf * nzp;
  for (int e = threadIdx.x; e < m * nzp; e += kT) {
    const int i = e % m, j = e / m;
    F[i + (size_t)j * ldf] = Jqr[i + (size_t)j * J.ldq];
  }
  for (int k = threadIdx.x; k < nzp; k += kT) {
    tau[k] = Jtau[k];
    rinv[k] = cdiv(make_double2(1.0, 0.0), c2d(Jqr[k + (size_t)k * J.ldq]));
  }
  __syncthreads();
  if (c >= J.nrhs) return;
  C* x = static_cast<C*>(J.X) + (size_t)c * J.ldx;
  if (nzp == 0) {
    for (int i = lane; i < n; i += 32) x[i] = cplx<C>::mk(0.0, 0.0);
    return;
  }
  C b[RPL];
#pragma unroll
  for (int r = 0; r < RPL; ++r) {
    const int i = lane + 32 * r;
    b[r] = i < m ? (JB ? JB[i + (size_t)c * J.ldb] : cplx<C>::mk(i == c ? 1.0 : 0.0, 0.0)) : cplx<C>::mk(0.0, 0.0);
  }
  for (int k = 0; k < nzp; ++k) {
    const C* v = F + (size_t)k * ldf;
    C s = cplx<C>::mk(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int i = lane + 32 * r;
      if (i > k && i < m) s = cfmac(v[i], b[r], s);
    }
    s = warp_sum2(s);
    const int ok = k & 31, rk = k >> 5;
    C bk = cplx<C>::mk(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < RPL; ++r) if (r == rk) bk = b[r];
    bk.x = __shfl_sync(0xffffffffu, bk.x, ok);
    bk.y = __shfl_sync(0xffffffffu, bk.y, ok);
    const C tw = cmul(tau[k], cadd(bk, s));
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int i = lane + 32 * r;
      if (i > k && i < m) b[r] = csub(b[r], cmul(v[i], tw));
      else if (i == k) b[r] = csub(b[r], tw);
    }
  }
  for (int i = nzp - 1; i >= 0; --i) {
    const int oi = i & 31, ri = i >> 5;
    C bi = cplx<C>::mk(0.0, 0.0);
#pragma unroll
    for (int r = 0; r < RPL; ++r) if (r == ri) bi = b[r];
    bi.x = __shfl_sync(0xffffffffu, bi.x, oi);
    bi.y = __shfl_sync(0xffffffffu, bi.y, oi);
    const C xi = cplx<C>::from(cmul(c2d(bi), rinv[i]));
    const C* Rc = F + (size_t)i * ldf;
#pragma unroll
    for (int r = 0; r < RPL; ++r) {
      const int l = lane + 32 * r;
      if (l < i) b[r] = csub(b[r], cmul(Rc[l], xi));
      else if (l == i) b[r] = xi;
    }
  }
  for (int i = lane; i < n; i += 32) x[i] = cplx<C>::mk(0.0, 0.0);
  __syncwarp();
  const C alpha = cplx<C>::from(J.alpha);
#pragma unroll
  for (int r = 0; r < RPL; ++r) {
    const int i = lane + 32 * r;
    if (i < nzp) x[J.perm[i]] = cmul(alpha, b[r]);
  }
}

// ---------------------------------------------------------------- QR solve
// one warp per right-hand side column
template <typename C>
__global__ void __launch_bounds__(kT) qr_solve_kernel(const SolveJob* __restrict__ jobs, const int* __restrict__ col_off,
                                                      int njobs, int total_cols) {
  const int gw = blockIdx.x * kW + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (gw >= total_cols) return;
  int lo = 0, hi = njobs - 1;
  while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (col_off[mid] <= gw) lo = mid; else hi = mid - 1; }
  const SolveJob J = jobs[lo];
  const C* Jqr = static_cast<const C*>(J.qr);
  const C* Jtau = static_cast<const C*>(J.tau);
  const C* JB = static_cast<const C*>(J.B);
  const int c = gw - col_off[lo];
  const int m = J.m, n = J.n;
  const int nzp = J.info[0];
  C* x = static_cast<C*>(J.X) + (size_t)c * J.ldx;
  if (nzp == 0) {
    for (int i = lane; i < n; i += 32) x[i] = cplx<C>::mk(0.0, 0.0);
    return;
  }
  C* wv = static_cast<C*>(J.work) + (size_t)c * m;
  for (int i = lane; i < m; i += 32)
    wv[i] = JB ? JB[i + (size_t)c * J.ldb] : cplx<C>::mk(i == c ? 1.0 : 0.0, 0.0);
  __syncwarp();
  // Q^H b with the first nzp reflectors
  for (int k = 0; k < nzp; ++k) {
    const C* v = Jqr + (size_t)k * J.ldq;
    C s = cplx<C>::mk(0.0, 0.0);
    for (int i = k + 1 + lane; i < m; i += 32) s = cfmac(v[i], wv[i], s);
    s = warp_sum2(s);
    const C t = Jtau[k];
    const C w = cadd(wv[k], s);
    __syncwarp();
    for (int i = k + 1 + lane; i < m; i += 32) wv[i] = csub(wv[i], cmul(cmul(t, v[i]), w));
    if (lane == 0) wv[k] = csub(wv[k], cmul(t, w));
    __syncwarp();
  }
  // back substitution with R(0:nzp, 0:nzp), column oriented
  for (int i = nzp - 1; i >= 0; --i) {
    C xi = cplx<C>::from(cdiv(c2d(wv[i]), c2d(Jqr[i + (size_t)i * J.ldq])));
    __syncwarp();
    if (lane == 0) wv[i] = xi;
    for (int l = lane; l < i; l += 32) wv[l] = csub(wv[l], cmul(Jqr[l + (size_t)i * J.ldq], xi));
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) x[i] = cplx<C>::mk(0.0, 0.0);
  __syncwarp();
  const C alpha = cplx<C>::from(J.alpha);
  for (int i = lane; i < nzp; i += 32) x[J.perm[i]] = cmul(alpha, wv[i]);
}

// ---------------------------------------------------------------- form Q
template <typename C>
__global__ void __launch_bounds__(kT) formq_kernel(const FormQJob* __restrict__ jobs, const int* __restrict__ col_off,
                                                   int njobs, int total_cols) {
  const int gw = blockIdx.x * kW + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (gw >= total_cols) return;
  int lo = 0, hi = njobs - 1;
  while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (col_off[mid] <= gw) lo = mid; else hi = mid - 1; }
  const FormQJob J = jobs[lo];
  const C* Jqr = static_cast<const C*>(J.qr);
  const C* Jtau = static_cast<const C*>(J.tau);
  const int c = gw - col_off[lo];
  const int ncols = J.ncols >= 0 ? J.ncols : J.ncols_dev[0];
  if (c >= ncols) return;
  const int m = J.m, size = min(J.m, J.n);
  C* q = static_cast<C*>(J.Q) + (size_t)c * J.ldQ;
  for (int i = lane; i < m; i += 32) q[i] = cplx<C>::mk(i == c ? 1.0 : 0.0, 0.0);
  __syncwarp();
  for (int k = min(size - 1, c); k >= 0; --k) {
    const C* v = Jqr + (size_t)k * J.ldq;
    C s = cplx<C>::mk(0.0, 0.0);
    for (int i = k + 1 + lane; i < m; i += 32) s = cfmac(v[i], q[i], s);
    s = warp_sum2(s);
    const C t = cconj(Jtau[k]);
    const C w = cadd(q[k], s);
    __syncwarp();
    for (int i = k + 1 + lane; i < m; i += 32) q[i] = csub(q[i], cmul(cmul(t, v[i]), w));
    if (lane == 0) q[k] = csub(q[k], cmul(t, w));
    __syncwarp();
  }
}

// ---------------------------------------------------------------- GEMM
// C = alpha sum_t op(A_t) op(B_t) + beta C over a list of GEMMs, one 32 x 32
// tile of C per CTA (16 x 16 threads, 2 x 2 outputs each).  The k dimension of
// all terms is walked in chunks of 32; the next chunk's global loads are issued
// into registers before the current chunk is multiplied out of shared memory,
// so one load latency hides behind each chunk's arithmetic.  Accumulation runs
// over k in increasing order, term after term.
// Output tile TM x TN(SJ) with TN = 16 SJ: SJ = 2 gives 32 x 32 tiles, SJ = 1
// gives 32 x 16 tiles for thin products (a block times a few right-hand sides).
constexpr int TM = 32, TK = 32;
template <int SJ>
__device__ __forceinline__ void gemm_fetch(const GemmTerm& T, int k0, int row0, int col0, int m, int n,
                                           double2 (&ra)[4], double2 (&rb)[2 * SJ]) {
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int e = threadIdx.x + 256 * u;
    const int kk = e / TM, ii = e % TM, gi = row0 + ii, gk = k0 + kk;
    ra[u] = make_double2(0.0, 0.0);
    const double2* A = static_cast<const double2*>(T.A);
    if (gi < m && gk < T.k) ra[u] = T.opA ? cconj(A[gk + (size_t)gi * T.lda]) : A[gi + (size_t)gk * T.lda];
  }
#pragma unroll
  for (int u = 0; u < 2 * SJ; ++u) {
    const int e = threadIdx.x + 256 * u;
    const int jj = e / TK, kb = e % TK, gj = col0 + jj, gkb = k0 + kb;
    rb[u] = make_double2(0.0, 0.0);
    const double2* B = static_cast<const double2*>(T.B);
    if (gj < n && gkb < T.k) rb[u] = T.opB ? cconj(B[gj + (size_t)gkb * T.ldb]) : B[gkb + (size_t)gj * T.ldb];
  }
}
// d += a b for one m8n8k4 FP64 tensor-core product (each lane: one A element,
// one B element, two accumulators)
__device__ __forceinline__ void dmma884(double (&d)[2], double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}
template <int SJ>
__global__ void __launch_bounds__(256) gemm_kernel(const GemmDesc* __restrict__ ds, const GemmTerm* __restrict__ terms,
                                                   const int* __restrict__ tile_off, int nd) {
  constexpr int TN = 16 * SJ;
  const int bid = blockIdx.x;
  int lo = 0, hi = nd - 1;
  while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (tile_off[mid] <= bid) lo = mid; else hi = mid - 1; }
  const GemmDesc D = ds[lo];
  const int t = bid - tile_off[lo];
  const int tiles_m = (D.m + TM - 1) / TM;
  const int tm = t % tiles_m, tn = t / tiles_m;
  __shared__ double2 As[TK][TM + 1];
  __shared__ double2 Bs[TK][TN + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int si = warp & 3, sj0 = SJ * (warp >> 2);
  double cr[SJ][2], ci[SJ][2];
#pragma unroll
  for (int q = 0; q < SJ; ++q) cr[q][0] = cr[q][1] = ci[q][0] = ci[q][1] = 0.0;
  const int row0 = tm * TM, col0 = tn * TN;
  int tt = 0, k0 = 0;
  GemmTerm T{};
  bool have = false;
  for (; tt < D.nterms; ++tt) { T = terms[D.term0 + tt]; if (T.k > 0) { have = true; break; } }
  double2 ra[4], rb[2 * SJ];
  if (have) gemm_fetch<SJ>(T, k0, row0, col0, D.m, D.n, ra, rb);
  while (have) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = threadIdx.x + 256 * u;
      As[e / TM][e % TM] = ra[u];
    }
#pragma unroll
    for (int u = 0; u < 2 * SJ; ++u) {
      const int e = threadIdx.x + 256 * u;
      Bs[e % TK][e / TK] = rb[u];
    }
    __syncthreads();
    // issue the next chunk's loads (possibly the next term's) before the arithmetic
    k0 += TK;
    bool next = true;
    if (k0 >= T.k) {
      next = false;
      k0 = 0;
      for (++tt; tt < D.nterms; ++tt) { T = terms[D.term0 + tt]; if (T.k > 0) { next = true; break; } }
    }
    if (next) gemm_fetch<SJ>(T, k0, row0, col0, D.m, D.n, ra, rb);
    // FP64 tensor cores: mma.sync m8n8k4 (DMMA).  Warp w owns the 8x8 output
    // sub-tiles (si, sj0 .. sj0 + SJ - 1) of the tile; a complex product is four
    // real products, Cr += Ar Br + (-Ai) Bi and Ci += Ar Bi + Ai Br.
    // Fragments (PTX ISA, mma.m8n8k4 .f64): A row = lane/4, col = lane%4;
    // B row = lane%4, col = lane/4; C row = lane/4, cols 2(lane%4) + {0, 1}.
#pragma unroll
    for (int k4 = 0; k4 < TK; k4 += 4) {
      const double2 a = As[k4 + (lane & 3)][si * 8 + (lane >> 2)];
      const double ar = a.x, ai = a.y, nai = -a.y;
#pragma unroll
      for (int q = 0; q < SJ; ++q) {
        const double2 b = Bs[k4 + (lane & 3)][(sj0 + q) * 8 + (lane >> 2)];
        dmma884(cr[q], ar, b.x);
        dmma884(cr[q], nai, b.y);
        dmma884(ci[q], ar, b.y);
        dmma884(ci[q], ai, b.x);
      }
    }
    __syncthreads();
    have = next;
  }
  const bool zero_beta = D.beta.x == 0.0 && D.beta.y == 0.0;
#pragma unroll
  for (int q = 0; q < SJ; ++q)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int gi = row0 + si * 8 + (lane >> 2), gj = col0 + (sj0 + q) * 8 + 2 * (lane & 3) + h;
      if (gi < D.m && gj < D.n) {
        double2* c = static_cast<double2*>(D.C) + gi + (size_t)gj * D.ldc;
        double2 v = cmul(D.alpha, make_double2(cr[q][h], ci[q][h]));
        if (!zero_beta) v = cadd(v, cmul(D.beta, *c));
        *c = v;
      }
    }
}

// The complex64 products of the mixed form: the same tiles and descriptor
// lists, FP32 fused multiply-adds with FP32 accumulation on the CUDA cores
// (these products are a few tens of rows deep: their time is the launch and
// the load latency, not the arithmetic).  Thread t computes rows t % 32 of
// the tile in columns t / 32 + 8 q.
template <int SJ>
__global__ void __launch_bounds__(256) gemm_f32_kernel(const GemmDesc* __restrict__ ds,
                                                       const GemmTerm* __restrict__ terms,
                                                       const int* __restrict__ tile_off, int nd) {
  constexpr int TN = 16 * SJ, NQ = TN / 8;
  const int bid = blockIdx.x;
  int lo = 0, hi = nd - 1;
  while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (tile_off[mid] <= bid) lo = mid; else hi = mid - 1; }
  const GemmDesc D = ds[lo];
  const int t = bid - tile_off[lo];
  const int tiles_m = (D.m + TM - 1) / TM;
  const int tm = t % tiles_m, tn = t / tiles_m;
  __shared__ float2 As[TK][TM + 1];
  __shared__ float2 Bs[TK][TN + 1];
  const int ti = threadIdx.x & 31, tj = threadIdx.x >> 5;
  float2 acc[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) acc[q] = make_float2(0.f, 0.f);
  const int row0 = tm * TM, col0 = tn * TN;
  for (int tt = 0; tt < D.nterms; ++tt) {
    const GemmTerm T = terms[D.term0 + tt];
    const float2* A = static_cast<const float2*>(T.A);
    const float2* B = static_cast<const float2*>(T.B);
    for (int k0 = 0; k0 < T.k; k0 += TK) {
      for (int e = threadIdx.x; e < TK * TM; e += 256) {
        const int kk = e / TM, ii = e % TM, gi = row0 + ii, gk = k0 + kk;
        float2 v = make_float2(0.f, 0.f);
        if (gi < D.m && gk < T.k) v = T.opA ? cconj(A[gk + (size_t)gi * T.lda]) : A[gi + (size_t)gk * T.lda];
        As[kk][ii] = v;
      }
      for (int e = threadIdx.x; e < TK * TN; e += 256) {
        const int jj = e / TK, kb = e % TK, gj = col0 + jj, gk = k0 + kb;
        float2 v = make_float2(0.f, 0.f);
        if (gj < D.n && gk < T.k) v = T.opB ? cconj(B[gj + (size_t)gk * T.ldb]) : B[gk + (size_t)gj * T.ldb];
        Bs[kb][jj] = v;
      }
      __syncthreads();
      const int kmax = min(TK, T.k - k0);
      for (int kk = 0; kk < kmax; ++kk) {
        const float2 a = As[kk][ti];
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] = cfma(a, Bs[kk][tj + 8 * q], acc[q]);
      }
      __syncthreads();
    }
  }
  const bool zero_beta = D.beta.x == 0.0 && D.beta.y == 0.0;
  const float2 alpha = cplx<float2>::from(D.alpha), beta = cplx<float2>::from(D.beta);
  const int gi = row0 + ti;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    const int gj = col0 + tj + 8 * q;
    if (gi < D.m && gj < D.n) {
      float2* c = static_cast<float2*>(D.C) + gi + (size_t)gj * D.ldc;
      float2 v = cmul(alpha, acc[q]);
      if (!zero_beta) v = cadd(v, cmul(beta, *c));
      *c = v;
    }
  }
}

// ---------------------------------------------------------------- GEAM
// Element sizes per descriptor: the arithmetic is complex128, a complex64
// operand is widened on load and a complex64 result rounded on store.
__device__ __forceinline__ double2 ld_any(const void* p, size_t i, int es) {
  return es == 16 ? static_cast<const double2*>(p)[i] : cplx<double2>::from(static_cast<const float2*>(p)[i]);
}
__device__ __forceinline__ void st_any(void* p, size_t i, int es, double2 v) {
  if (es == 16) static_cast<double2*>(p)[i] = v;
  else static_cast<float2*>(p)[i] = cplx<float2>::from(v);
}
__global__ void geam_kernel(const GeamDesc* __restrict__ ds, const long long* __restrict__ off, int nd,
                            long long total) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nd - 1;
    while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (off[mid] <= e) lo = mid; else hi = mid - 1; }
    const GeamDesc D = ds[lo];
    long long loc = e - off[lo];
    int i = (int)(loc % D.m), j = (int)(loc / D.m);
    double2 a = D.opA ? cconj(ld_any(D.A, j + (size_t)i * D.lda, D.esA)) : ld_any(D.A, i + (size_t)j * D.lda, D.esA);
    if (D.rs) a = cscale(a, D.rs[i]);
    if (D.cs) a = cscale(a, D.cs[j]);
    double2 v = cmul(D.alpha, a);
    const size_t ci = i + (size_t)j * D.ldc;
    if (!(D.beta.x == 0.0 && D.beta.y == 0.0)) v = cadd(v, cmul(D.beta, ld_any(D.C, ci, D.esC)));
    st_any(D.C, ci, D.esC, v);
  }
}

// ---------------------------------------------------------------- norms
__global__ void __launch_bounds__(kT) norm_kernel(const NormDesc* __restrict__ ds) {
  const NormDesc D = ds[blockIdx.x];
  __shared__ double sh[kW + 1];
  double s = 0.0;
  for (long long e = threadIdx.x; e < (long long)D.m * D.n; e += kT) {
    int i = (int)(e % D.m), j = (int)(e / D.m);
    s += cabs2(ld_any(D.A, i + (size_t)j * D.lda, D.es));
  }
  s = block_sum(s, sh);
  if (threadIdx.x == 0) {
    D.out[0] = sqrt(s);  // may be mapped host memory
    __threadfence_system();
  }
}

// ---------------------------------------------------------------- equilibration
// one CTA per block, one thread per column (mode 0) or row (mode 1)
__global__ void __launch_bounds__(kT) equilibrate_kernel(const EquilDesc* __restrict__ ds) {
  const EquilDesc D = ds[blockIdx.x];
  const int cnt = D.mode == 0 ? D.n : D.m, len = D.mode == 0 ? D.m : D.n;
  for (int c = threadIdx.x; c < cnt; c += kT) {
    double q = 0.0;
    for (int e = 0; e < len; ++e) {
      const double2 a = D.mode == 0 ? D.A[e + (size_t)c * D.lda] : D.A[c + (size_t)e * D.lda];
      const double f = D.scale ? D.scale[e] : 1.0;
      q += cabs2(a) * (f * f);
    }
    const double nrm = sqrt(q);
    const bool ok = nrm > 0.0 && nrm < 1e300;
    D.s[c] = ok ? 1.0 / nrm : 1.0;
    D.is[c] = ok ? nrm : 1.0;
  }
}

// ---------------------------------------------------------------- skeleton LU solve
__global__ void __launch_bounds__(kT) skel_lu_kernel(const SkelLUJob* __restrict__ jobs, EntryCtx ctx) {
  const SkelLUJob J = jobs[blockIdx.x];
  const int r = J.r, m = J.m;
  if (r == 0) return;
  double2* D = J.work;             // r x r
  double2* X = J.work + (size_t)r * r;  // r x m
  const int tid = threadIdx.x;
  __shared__ int s_p;
  for (int e = tid; e < r * r; e += kT) {
    int i = e % r, j = e / r;
    if (J.adjD) D[i + (size_t)j * r] = cconj(lsa_entry(J.rows[j], J.cols[i], ctx));
    else D[i + (size_t)j * r] = lsa_entry(J.rows[i], J.cols[j], ctx);
  }
  for (int e = tid; e < r * m; e += kT) {
    int i = e % r, j = e / r;
    X[i + (size_t)j * r] = J.adjB ? cconj(J.B[j + (size_t)i * J.ldb]) : J.B[i + (size_t)j * J.ldb];
  }
  __syncthreads();
  // LU with partial pivoting (first row of largest modulus), row swaps applied to X
  for (int k = 0; k < r; ++k) {
    if (tid == 0) {
      int p = k; double best = cabsd(D[k + (size_t)k * r]);
      for (int i = k + 1; i < r; ++i) { double v = cabsd(D[i + (size_t)k * r]); if (v > best) { best = v; p = i; } }
      s_p = p;
      J.piv[k] = p;
    }
    __syncthreads();
    const int p = s_p;
    if (p != k) {
      for (int j = tid; j < r; j += kT) { double2 t = D[k + (size_t)j * r]; D[k + (size_t)j * r] = D[p + (size_t)j * r]; D[p + (size_t)j * r] = t; }
      for (int j = tid; j < m; j += kT) { double2 t = X[k + (size_t)j * r]; X[k + (size_t)j * r] = X[p + (size_t)j * r]; X[p + (size_t)j * r] = t; }
    }
    __syncthreads();
    const double2 d = D[k + (size_t)k * r];
    for (int i = k + 1 + tid; i < r; i += kT) {
      if (!(d.x == 0.0 && d.y == 0.0)) D[i + (size_t)k * r] = cdiv(D[i + (size_t)k * r], d);
    }
    __syncthreads();
    for (int e = tid; e < (r - k - 1) * (r - k - 1); e += kT) {
      int i = k + 1 + e % (r - k - 1), j = k + 1 + e / (r - k - 1);
      D[i + (size_t)j * r] = csub(D[i + (size_t)j * r], cmul(D[i + (size_t)k * r], D[k + (size_t)j * r]));
    }
    __syncthreads();
  }
  // forward (unit lower) and back substitution, one thread per right-hand side column
  for (int j = tid; j < m; j += kT) {
    double2* x = X + (size_t)j * r;
    for (int i = 0; i < r; ++i) {
      double2 s = x[i];
      for (int l = 0; l < i; ++l) s = csub(s, cmul(D[i + (size_t)l * r], x[l]));
      x[i] = s;
    }
    for (int i = r - 1; i >= 0; --i) {
      double2 s = x[i];
      for (int l = i + 1; l < r; ++l) s = csub(s, cmul(D[i + (size_t)l * r], x[l]));
      x[i] = cdiv(s, D[i + (size_t)i * r]);
    }
  }
  __syncthreads();
  for (int e = tid; e < r * m; e += kT) {
    int i = e % r, j = e / r;
    if (J.adjX) J.X[j + (size_t)i * J.ldx] = cconj(X[i + (size_t)j * r]);
    else J.X[i + (size_t)j * J.ldx] = X[i + (size_t)j * r];
  }
}

}  // namespace

namespace {
// the element size of a batch: 16 (complex128) or 8 (complex64)
bool valid_es(int es) { return es == 16 || es == 8; }
// opt a kernel into the large dynamic shared memory once per process
template <typename K>
void smem_attr_once(K kernel, bool& done) {
  if (!done) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    done = true;
  }
}
}  // namespace

int aifmm_launch_qr_factor(const QRJob* d_jobs, int njobs, int es, cudaStream_t s) {
  if (njobs <= 0) return 0;
  if (!valid_es(es)) return (int)cudaErrorInvalidValue;
  if (es == 16) qr_factor_kernel<double2><<<njobs, kT, 0, s>>>(d_jobs);
  else qr_factor_kernel<float2><<<njobs, kT, 0, s>>>(d_jobs);
  return (int)cudaGetLastError();
}

namespace {
template <typename C>
int launch_solve_warp(const SolveJob* d_jobs, const int* d_cta_off, int njobs, int total_ctas, int rpl, size_t smem,
                      cudaStream_t s) {
  static bool attr[8] = {false, false, false, false, false, false, false, false};
  switch (rpl) {
#define AIFMM_SOLVE_CASE(R)                                                               \
    case R:                                                                               \
      smem_attr_once(qr_solve_warp_kernel<C, R>, attr[R]);                                \
      qr_solve_warp_kernel<C, R><<<total_ctas, kT, smem, s>>>(d_jobs, d_cta_off, njobs);  \
      break;
    AIFMM_SOLVE_CASE(1) AIFMM_SOLVE_CASE(2) AIFMM_SOLVE_CASE(3) AIFMM_SOLVE_CASE(4)
    AIFMM_SOLVE_CASE(5) AIFMM_SOLVE_CASE(6) AIFMM_SOLVE_CASE(7)
#undef AIFMM_SOLVE_CASE
    default: return (int)cudaErrorInvalidValue;
  }
  return (int)cudaGetLastError();
}
}  // namespace

int aifmm_launch_qr_solve_warp(const SolveJob* d_jobs, const int* d_cta_off, int njobs, int total_ctas, int mmax,
                               int nzpmax, int es, cudaStream_t s) {
  if (njobs <= 0 || total_ctas <= 0) return 0;
  if (!valid_es(es)) return (int)cudaErrorInvalidValue;
  const size_t smem = (size_t)es * ((size_t)(mmax | 1) * nzpmax + (size_t)nzpmax) + sizeof(double2) * nzpmax + 64;
  const int rpl = (mmax + 31) / 32;
  return es == 16 ? launch_solve_warp<double2>(d_jobs, d_cta_off, njobs, total_ctas, rpl, smem, s)
                  : launch_solve_warp<float2>(d_jobs, d_cta_off, njobs, total_ctas, rpl, smem, s);
}

size_t aifmm_qr_smem_bytes(int m, int n, int es) {
  if (n > 1024) return ~size_t(0);  // pivot keys hold a column index below 1024
  return (size_t)es * ((size_t)qr_smem_ld(m) * n + (size_t)kW * m) +
         sizeof(double) * (3 * (size_t)n + (size_t)std::min(m, n)) + sizeof(int) * 2 * (size_t)n;
}
int aifmm_launch_qr_factor_smem(const QRJob* d_jobs, int njobs, size_t smem, int es, cudaStream_t s) {
  if (njobs <= 0) return 0;
  if (!valid_es(es)) return (int)cudaErrorInvalidValue;
  static bool attr[2] = {false, false};
  if (es == 16) {
    smem_attr_once(qr_factor_smem_kernel<double2>, attr[0]);
    qr_factor_smem_kernel<double2><<<njobs, kT, smem, s>>>(d_jobs);
  } else {
    smem_attr_once(qr_factor_smem_kernel<float2>, attr[1]);
    qr_factor_smem_kernel<float2><<<njobs, kT, smem, s>>>(d_jobs);
  }
  return (int)cudaGetLastError();
}
int aifmm_launch_qr_solve(const SolveJob* d_jobs, const int* d_col_off, int njobs, int total_cols, int es,
                          cudaStream_t s) {
  if (njobs <= 0 || total_cols <= 0) return 0;
  if (!valid_es(es)) return (int)cudaErrorInvalidValue;
  const int grid = (total_cols + kW - 1) / kW;
  if (es == 16) qr_solve_kernel<double2><<<grid, kT, 0, s>>>(d_jobs, d_col_off, njobs, total_cols);
  else qr_solve_kernel<float2><<<grid, kT, 0, s>>>(d_jobs, d_col_off, njobs, total_cols);
  return (int)cudaGetLastError();
}
size_t aifmm_compress_smem_bytes(int m, int rK, int c, int rb, int es) {
  const int n1 = rK + c, s1 = std::min(m, n1), n2 = rb + s1, s2 = std::min(c, n2);
  if (m > 1024 || c > 1024) return 0;
  size_t b = std::max(aifmm_qr_smem_bytes(m, n1, es), aifmm_qr_smem_bytes(c, n2, es));
  b = std::max(b, aifmm_formq_smem_bytes(m, s1, s1, es));
  b = std::max(b, aifmm_formq_smem_bytes(c, s2, s2, es));
  return b <= (size_t(200) << 10) ? b : 0;
}
int aifmm_launch_compress_p2p(const CompressJob* d_jobs, int njobs, size_t smem, int es, cudaStream_t s) {
  if (njobs <= 0) return 0;
  if (!valid_es(es)) return (int)cudaErrorInvalidValue;
  static bool attr[2] = {false, false};
  if (es == 16) {
    smem_attr_once(compress_p2p_kernel<double2>, attr[0]);
    compress_p2p_kernel<double2><<<njobs, kT, smem, s>>>(d_jobs);
  } else {
    smem_attr_once(compress_p2p_kernel<float2>, attr[1]);
    compress_p2p_kernel<float2><<<njobs, kT, smem, s>>>(d_jobs);
  }
  return (int)cudaGetLastError();
}
int aifmm_launch_formq(const FormQJob* d_jobs, const int* d_col_off, int njobs, int total_cols, int es,
                       cudaStream_t s) {
  if (njobs <= 0 || total_cols <= 0) return 0;
  if (!valid_es(es)) return (int)cudaErrorInvalidValue;
  const int grid = (total_cols + kW - 1) / kW;
  if (es == 16) formq_kernel<double2><<<grid, kT, 0, s>>>(d_jobs, d_col_off, njobs, total_cols);
  else formq_kernel<float2><<<grid, kT, 0, s>>>(d_jobs, d_col_off, njobs, total_cols);
  return (int)cudaGetLastError();
}
int aifmm_launch_gemm(const GemmDesc* d, const GemmTerm* d_terms, const int* d_tile_off, int nd, int total_tiles,
                      cudaStream_t s, int tile_cols, int es) {
  if (nd <= 0 || total_tiles <= 0) return 0;
  if (!valid_es(es)) return (int)cudaErrorInvalidValue;
  if (es == 16) {
    if (tile_cols == 16) gemm_kernel<1><<<total_tiles, 256, 0, s>>>(d, d_terms, d_tile_off, nd);
    else gemm_kernel<2><<<total_tiles, 256, 0, s>>>(d, d_terms, d_tile_off, nd);
  } else {
    if (tile_cols == 16) gemm_f32_kernel<1><<<total_tiles, 256, 0, s>>>(d, d_terms, d_tile_off, nd);
    else gemm_f32_kernel<2><<<total_tiles, 256, 0, s>>>(d, d_terms, d_tile_off, nd);
  }
  return (int)cudaGetLastError();
}
int aifmm_launch_geam(const GeamDesc* d, const long long* d_off, int nd, long long total, cudaStream_t s) {
  if (nd <= 0 || total <= 0) return 0;
  long long blocks = (total + 255) / 256;
  if (blocks > 148LL * 32) blocks = 148LL * 32;
  geam_kernel<<<(int)blocks, 256, 0, s>>>(d, d_off, nd, total);
  return (int)cudaGetLastError();
}
int aifmm_launch_equilibrate(const EquilDesc* d, int nd, cudaStream_t s) {
  if (nd <= 0) return 0;
  equilibrate_kernel<<<nd, kT, 0, s>>>(d);
  return (int)cudaGetLastError();
}
int aifmm_launch_norms(const NormDesc* d, int nd, cudaStream_t s) {
  if (nd <= 0) return 0;
  norm_kernel<<<nd, kT, 0, s>>>(d);
  return (int)cudaGetLastError();
}
int aifmm_launch_skel_lu(const SkelLUJob* d, int nd, const EntryCtx& ctx, cudaStream_t s) {
  if (nd <= 0) return 0;
  skel_lu_kernel<<<nd, kT, 0, s>>>(d, ctx);
  return (int)cudaGetLastError();
}
