// k_entries.cu -- batched matrix-entry assembly (K1).
//
// Replaces kernel::getRow / getCol / getMatrix (kernel.hpp:54-86) and the block
// assemblies built on them: leaf P2P blocks (FMM2DTree_find_error.hpp:1729-1741),
// M2L blocks (:1338-1361), the skeleton blocks of get_L2P_P2M_box (:1105-1128),
// and the dense product of the find_error fixture generator
// (FMM2DTree_gen_rhs_x.hpp:2864-2871).
#include "kernels.h"
#include "entry.cuh"


namespace {

__global__ void block_entries_kernel(const BlockDesc* __restrict__ d, const long long* __restrict__ off, int nd,
                                     long long total, EntryCtx ctx) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = nd - 1;
    while (lo < hi) {  // last descriptor with off <= e
      int mid = (lo + hi + 1) >> 1;
      if (off[mid] <= e) lo = mid; else hi = mid - 1;
    }
    const BlockDesc b = d[lo];
    const long long loc = e - off[lo];
    const int r = (int)(loc % b.nr), c = (int)(loc / b.nr);
    double2 v = lsa_entry(__ldg(&b.rows[r]), __ldg(&b.cols[c]), ctx);
    if (b.adjoint) b.out[c + (size_t)r * b.ldo] = cconj(v);
    else b.out[r + (size_t)c * b.ldo] = v;
  }
}

__global__ void list_entries_kernel(const int* __restrict__ I, const int* __restrict__ J, long n, double2* out,
                                    EntryCtx ctx) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    out[t] = lsa_entry(I[t], J[t], ctx);
}

// y(:, s) = A x(:, s) for nrhs columns (x, y: N x nrhs column-major).
// Each CTA owns 128 target rows and a slice of source points; partial sums are
// combined with atomics.
constexpr int kMvRows = 128;
constexpr int kMvMaxRhs = 8;
template <bool PHI>
__global__ void __launch_bounds__(kMvRows) dense_matvec_kernel(const double2* __restrict__ x, double2* y, int N,
                                                                int nrhs, int cols_per_slice, EntryCtx ctx) {
  const int i = blockIdx.x * kMvRows + threadIdx.x;
  const int j0 = blockIdx.y * cols_per_slice;
  const int j1 = min(N, j0 + cols_per_slice);
  if (i >= N) return;
  double2 acc[kMvMaxRhs];
  for (int s = 0; s < kMvMaxRhs; ++s) acc[s] = make_double2(0.0, 0.0);
  for (int j = j0; j < j1; ++j) {
    double2 a = lsa_entry<PHI>(i, j, ctx);
    if (a.x == 0.0 && a.y == 0.0) continue;
    for (int s = 0; s < nrhs; ++s) acc[s] = cfma(a, __ldg(&x[j + (size_t)s * N]), acc[s]);
  }
  for (int s = 0; s < nrhs; ++s) {
    atomicAdd(&y[i + (size_t)s * N].x, acc[s].x);
    atomicAdd(&y[i + (size_t)s * N].y, acc[s].y);
  }
}

}  // namespace

int aifmm_launch_block_entries(const BlockDesc* d_desc, const long long* d_off, int nd, long long total,
                               const EntryCtx& ctx, cudaStream_t stream) {
  if (nd <= 0 || total <= 0) return 0;
  long long blocks = (total + 255) / 256;
  if (blocks > 148LL * 64) blocks = 148LL * 64;
  block_entries_kernel<<<(int)blocks, 256, 0, stream>>>(d_desc, d_off, nd, total, ctx);
  return (int)cudaGetLastError();
}

int aifmm_launch_list_entries(const int* I, const int* J, long n, double2* out, const EntryCtx& ctx,
                              cudaStream_t stream) {
  if (n <= 0) return 0;
  long blocks = (n + 255) / 256;
  if (blocks > 148L * 64) blocks = 148L * 64;
  list_entries_kernel<<<(int)blocks, 256, 0, stream>>>(I, J, n, out, ctx);
  return (int)cudaGetLastError();
}

namespace {
template <bool PHI>
int launch_matvec(const double2* x, double2* y, int N, int nrhs, const EntryCtx& ctx, cudaStream_t stream) {
  if (nrhs > kMvMaxRhs) return (int)cudaErrorInvalidValue;
  const int row_blocks = (N + kMvRows - 1) / kMvRows;
  // enough slices to give every SM several CTAs
  int slices = (148 * 8 + row_blocks - 1) / row_blocks;
  if (slices < 1) slices = 1;
  int cps = (N + slices - 1) / slices;
  slices = (N + cps - 1) / cps;
  dim3 grid(row_blocks, slices);
  dense_matvec_kernel<PHI><<<grid, kMvRows, 0, stream>>>(x, y, N, nrhs, cps, ctx);
  return (int)cudaGetLastError();
}
}  // namespace

int aifmm_launch_dense_matvec(const double2* x, double2* y, int N, int nrhs, const EntryCtx& ctx,
                              cudaStream_t stream) {
  if (nrhs > kMvMaxRhs) return (int)cudaErrorInvalidValue;
  cudaMemsetAsync(y, 0, sizeof(double2) * (size_t)N * nrhs, stream);
  return launch_matvec<true>(x, y, N, nrhs, ctx, stream);
}
int aifmm_launch_green_matvec_add(const double2* x, double2* y, int N, int nrhs, const EntryCtx& ctx,
                                  cudaStream_t stream) {
  return launch_matvec<false>(x, y, N, nrhs, ctx, stream);
}
