// k_aca.cu -- batched partially pivoted ACA skeletonisation (K3).
//
// Replaces LowRank::ACA_only_nodes (ACA.hpp:368-577) as called by
// getNodes_outgoing_box / getNodes_incoming_box (FMM2DTree_find_error.hpp:1230-1336).
// One CTA per (box, direction); all boxes of a level in one launch.
//
// The reference has two mirror-image branches: rows first when N1 < N2
// (ACA.hpp:397-481), columns first otherwise (:482-568).  Both are the same
// procedure on A or A^T, written here once in terms of a "primary" index set
// (the one scanned first) and a "secondary" one:
//   * scan primary indices in order for the first vector whose largest entry
//     over the secondary set exceeds tol_robust = 1e-12 (ACA.hpp:399-413);
//   * v = P / P[pivot], u = S (unmodified first column / row);
//   * loop while |P[s_piv]| > tol, |S[p_next]| > tol, |prev - normS| >= tol*prev,
//     rank < min(N1, N2): residual P and S against the previous terms, pivots
//     = first maximum of |.| over the remaining indices in ascending order
//     (ACA.hpp:27-40), stop when |u| or |v| < tol_robust;
//   * normS bookkeeping exactly as ACA.hpp:472-478 (the sum over l includes the
//     new term, prev_normS is not updated when the rank becomes 2).
// The unmodified rows (Ar) or columns (Ac) are the outputs the solver keeps.
#include <cfloat>
#include "kernels.h"
#include "entry.cuh"


namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

struct ArgMax { double v; int i; };

__device__ __forceinline__ ArgMax better(ArgMax a, ArgMax b) {
  if (b.i < 0) return a;
  if (a.i < 0) return b;
  if (b.v > a.v) return b;
  if (a.v > b.v) return a;
  return a.i <= b.i ? a : b;
}

__device__ ArgMax block_argmax_strict(ArgMax x, ArgMax* sh) {
  for (int o = 16; o > 0; o >>= 1) {
    ArgMax y;
    y.v = __shfl_down_sync(0xffffffffu, x.v, o);
    y.i = __shfl_down_sync(0xffffffffu, x.i, o);
    x = better(x, y);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    ArgMax r = sh[0];
    for (int k = 1; k < kWarps; ++k) r = better(r, sh[k]);
    sh[kWarps] = r;
  }
  __syncthreads();
  ArgMax r = sh[kWarps];
  __syncthreads();
  return r;
}

__device__ int block_min_int(int x, int* sh) {
  for (int o = 16; o > 0; o >>= 1) x = min(x, __shfl_down_sync(0xffffffffu, x, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    int r = sh[0];
    for (int k = 1; k < kWarps; ++k) r = min(r, sh[k]);
    sh[kWarps] = r;
  }
  __syncthreads();
  int r = sh[kWarps];
  __syncthreads();
  return r;
}

// Pivot choice of ACA.hpp:27-40 with a relative tie tolerance: the first index
// whose magnitude is within kPivotTie of the maximum (the first maximum when
// values differ by more).  Each thread passes the candidates it owns through
// `cand(i) -> magnitude or -1 if not allowed`, evaluated twice.
constexpr double kPivotTie = 1e-11;
template <class F>
__device__ ArgMax block_pick(int n, F cand, ArgMax* sa, int* si) {
  ArgMax am{-1.0, -1};
  for (int t = threadIdx.x; t < n; t += kThreads) {
    double v = cand(t);
    if (v >= 0.0) am = better(am, ArgMax{v, t});
  }
  ArgMax best = block_argmax_strict(am, sa);
  if (best.i < 0) return best;
  const double cut = best.v * (1.0 - kPivotTie);
  int first = 0x7fffffff;
  for (int t = threadIdx.x; t < n; t += kThreads) {
    double v = cand(t);
    if (v >= 0.0 && v >= cut) { first = t; break; }
  }
  first = block_min_int(first, si);
  return ArgMax{best.v, first};
}

__device__ double block_sum(double x, double* sh) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int k = 0; k < kWarps; ++k) r += sh[k];
    sh[kWarps] = r;
  }
  __syncthreads();
  double r = sh[kWarps];
  __syncthreads();
  return r;
}

// entry of the primary vector p at secondary position s
__device__ __forceinline__ double2 ent(const AcaJob& J, bool rows_first, int p, int s, const EntryCtx& c) {
  return rows_first ? lsa_entry(J.rows[p], J.cols[s], c) : lsa_entry(J.rows[s], J.cols[p], c);
}

__global__ void __launch_bounds__(kThreads) aca_kernel(const AcaJob* __restrict__ jobs, double tol, EntryCtx ctx) {
  const AcaJob J = jobs[blockIdx.x];
  __shared__ ArgMax sa[kWarps + 1];
  __shared__ double sd[kWarps + 1];
  __shared__ int si[kWarps + 1];
  double2* coef = J.coef;
  double2* dots_u = J.dots_u;
  double2* dots_v = J.dots_v;
  const double tol_robust = 1e-12;  // ACA.hpp:23
  const int tid = threadIdx.x;
  const bool rows_first = J.n1 < J.n2;
  const int np = rows_first ? J.n1 : J.n2;   // primary count
  const int ns = rows_first ? J.n2 : J.n1;   // secondary count
  const int rmax = min(J.n1, J.n2);
  // the outputs' side: in rows-first mode rows are primary vectors
  const bool keepP = (J.want_rows != 0) == rows_first;
  if (tid == 0) { J.rank[0] = 0; J.rank[1] = rows_first ? 1 : 2; }
  if (rmax == 0) return;
  for (int t = tid; t < np; t += kThreads) J.remP[t] = 1;
  for (int t = tid; t < ns; t += kThreads) J.remS[t] = 1;
  __syncthreads();
  // ---- first primary vector with a non-negligible entry
  int p0 = -1, spiv = -1;
  for (int l = 0; l < np; ++l) {
    for (int s = tid; s < ns; s += kThreads) J.P[s] = ent(J, rows_first, l, s, ctx);
    __syncthreads();
    ArgMax r = block_pick(ns, [&](int s) { double2 v = J.P[s]; return hypot(v.x, v.y); }, sa, si);
    if (r.v > tol_robust) { p0 = l; spiv = r.i; break; }
  }
  if (p0 < 0) return;  // rank 0
  // v = P / P[spiv]; U[0] = S = secondary vector at spiv
  const double2 piv0 = J.P[spiv];
  for (int s = tid; s < ns; s += kThreads) {
    double2 pv = J.P[s];
    J.V[s] = cdiv(pv, piv0);
    if (keepP) {
      if (J.want_rows) J.out[0 + (size_t)s * rmax] = pv; else J.out[s] = pv;
    }
  }
  for (int t = tid; t < np; t += kThreads) {
    double2 sv = ent(J, rows_first, t, spiv, ctx);
    J.S[t] = sv;
    J.U[t] = sv;
    if (!keepP) {
      if (J.want_rows) J.out[0 + (size_t)t * rmax] = sv; else J.out[t] = sv;
    }
  }
  if (tid == 0) {
    J.prim_bases[0] = p0; J.sec_bases[0] = spiv;
    J.remS[spiv] = 0; J.remP[p0] = 0;
  }
  __syncthreads();
  int rank = 1;
  double normS = 0.0, prev = DBL_MAX;
  // next primary pivot: max |S| over remaining primary indices
  ArgMax rn = block_pick(np, [&](int t) { double2 v = J.S[t]; return J.remP[t] ? hypot(v.x, v.y) : -1.0; }, sa, si);
  int pnext = rn.i < 0 ? 0 : rn.i;
  double pivP = hypot(J.P[spiv].x, J.P[spiv].y);
  while (true) {
    double sp = hypot(J.S[pnext].x, J.S[pnext].y);
    if (!(pivP > tol && sp > tol && fabs(prev - normS) >= tol * prev && rank < rmax)) break;
    // ---- primary vector at pnext, residual against previous terms
    for (int l = tid; l < rank; l += kThreads) coef[l] = J.U[(size_t)l * np + pnext];
    __syncthreads();
    for (int s = tid; s < ns; s += kThreads) {
      double2 pv = ent(J, rows_first, pnext, s, ctx);
      if (keepP) {
        if (J.want_rows) J.out[rank + (size_t)s * rmax] = pv; else J.out[s + (size_t)rank * ns] = pv;
      }
      for (int l = 0; l < rank; ++l) pv = csub(pv, cmul(coef[l], J.V[(size_t)l * ns + s]));
      J.P[s] = pv;
    }
    __syncthreads();
    ArgMax r2 = block_pick(ns, [&](int s) { double2 v = J.P[s]; return J.remS[s] ? hypot(v.x, v.y) : -1.0; }, sa, si);
    const int snew = r2.i < 0 ? 0 : r2.i;
    const double2 pivot = J.P[snew];
    double vn2 = 0.0;
    for (int s = tid; s < ns; s += kThreads) {
      double2 v = cdiv(J.P[s], pivot);
      J.V[(size_t)rank * ns + s] = v;
      vn2 += cabs2(v);
    }
    for (int l = tid; l < rank; l += kThreads) coef[l] = J.V[(size_t)l * ns + snew];
    __syncthreads();
    double un2 = 0.0;
    for (int t = tid; t < np; t += kThreads) {
      double2 sv = ent(J, rows_first, t, snew, ctx);
      if (!keepP) {
        if (J.want_rows) J.out[rank + (size_t)t * rmax] = sv; else J.out[t + (size_t)rank * np] = sv;
      }
      for (int l = 0; l < rank; ++l) sv = csub(sv, cmul(coef[l], J.U[(size_t)l * np + t]));
      J.S[t] = sv;
      J.U[(size_t)rank * np + t] = sv;
      un2 += cabs2(sv);
    }
    const double un = sqrt(block_sum(un2, sd));
    const double vn = sqrt(block_sum(vn2, sd));
    if (un < tol_robust || vn < tol_robust) break;  // term rejected, bases not committed
    if (tid == 0) {
      J.prim_bases[rank] = pnext; J.sec_bases[rank] = snew;
      J.remS[snew] = 0; J.remP[pnext] = 0;
    }
    ++rank;
    // normS update (ACA.hpp:472-478): dots of every stored term with the new one
    for (int l = threadIdx.x >> 5; l < rank; l += kWarps) {
      double2 du = make_double2(0.0, 0.0), dv = make_double2(0.0, 0.0);
      const double2* ul = J.U + (size_t)l * np;
      const double2* un_ = J.U + (size_t)(rank - 1) * np;
      for (int t = threadIdx.x & 31; t < np; t += 32) du = cfmac(ul[t], un_[t], du);
      const double2* vl = J.V + (size_t)l * ns;
      const double2* vn_ = J.V + (size_t)(rank - 1) * ns;
      for (int s = threadIdx.x & 31; s < ns; s += 32) dv = cfmac(vl[s], vn_[s], dv);
      for (int o = 16; o > 0; o >>= 1) {
        du.x += __shfl_down_sync(0xffffffffu, du.x, o); du.y += __shfl_down_sync(0xffffffffu, du.y, o);
        dv.x += __shfl_down_sync(0xffffffffu, dv.x, o); dv.y += __shfl_down_sync(0xffffffffu, dv.y, o);
      }
      if ((threadIdx.x & 31) == 0) { dots_u[l] = du; dots_v[l] = dv; }
    }
    __syncthreads();
    if (rank != 2) prev = normS;
    double ns_ = normS * normS + (un * vn) * (un * vn);
    for (int l = 0; l < rank; ++l) {
      double2 pr = cmul(dots_u[l], dots_v[l]);
      ns_ += 2 * hypot(pr.x, pr.y);
    }
    normS = sqrt(ns_);
    __syncthreads();
    // next primary pivot
    ArgMax r3 = block_pick(np, [&](int t) { double2 v = J.S[t]; return J.remP[t] ? hypot(v.x, v.y) : -1.0; }, sa, si);
    pnext = r3.i < 0 ? 0 : r3.i;
    pivP = hypot(J.P[snew].x, J.P[snew].y);
    spiv = snew;
  }
  if (tid == 0) J.rank[0] = rank;
}

}  // namespace

int aifmm_launch_aca(const AcaJob* d_jobs, int njobs, double tol, const EntryCtx& ctx, cudaStream_t stream) {
  if (njobs <= 0) return 0;
  aca_kernel<<<njobs, kThreads, 0, stream>>>(d_jobs, tol, ctx);
  return (int)cudaGetLastError();
}
