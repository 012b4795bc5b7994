// kernels.h -- descriptor structs and launchers shared by the host orchestrator
// and the CUDA kernels of the AIFMM-LS B200 solver.
#pragma once
#include "common.cuh"

// ---- K1 entries
struct BlockDesc {        // A(rows, cols) into out (column-major, ldo) or its adjoint
  const int* rows;
  const int* cols;
  int nr, nc;
  double2* out;
  int ldo;
  int adjoint;
};

// ---- K3 ACA
struct AcaJob {
  const int* rows;   // N1 global point indices
  const int* cols;   // N2 global point indices
  int n1, n2;
  int want_rows;     // 1: keep unmodified rows (Ar, rank x N2, ld = rmax); 0: columns (Ac, N1 x rank, ld = N1)
  double2* out;
  double2* U;        // rmax x n_prim
  double2* V;        // rmax x n_sec
  double2* P;        // n_sec
  double2* S;        // n_prim
  double2* coef;     // rmax + 1
  double2* dots_u;   // rmax + 1
  double2* dots_v;   // rmax + 1
  unsigned char* remP;
  unsigned char* remS;
  int* prim_bases;   // rmax
  int* sec_bases;    // rmax
  int* rank;         // [0] rank (-1: too large), [1] branch (1 rows first, 2 columns first)
};

// ---- dense
// The factorisation kernels serve both forms: complex128 blocks (the plain
// form) and complex64 blocks (the mixed form).  Their descriptors hold untyped
// element pointers; each launcher takes the element size es (16 or 8 bytes)
// of its whole batch.  Scalars (alpha, beta, thresholds) are always double.
struct QRJob {
  void* a; int lda;
  int m, n;
  void* tau;
  int* perm;
  double* norms;     // 2n reals of the element's real type
  double thr;        // 0 -> min(m,n)*eps
  int* info;         // [0] nonzero pivots, [1] rank
  double* maxpiv;
};

struct SolveJob {        // X = alpha * QR^{-1} B
  const void* qr; int ldq; int m, n;
  const void* tau; const int* perm; const int* info;
  const void* B; int ldb;   // nullptr -> identity
  void* X; int ldx;
  int nrhs;
  double2 alpha;
  void* work;            // m x nrhs
};

struct FormQJob {
  const void* qr; int ldq; int m, n;
  const void* tau;
  void* Q; int ldQ;
  const int* ncols_dev;
  int ncols;             // < 0 -> read ncols_dev[0]
};

struct GemmTerm {        // op(A) (m x k) * op(B) (k x n); op 0 = N, 1 = conjugate transpose
  const void* A; const void* B;
  int lda, ldb, opA, opB, k;
};
struct GemmDesc {        // C = alpha * sum_t op(A_t) op(B_t) + beta * C
  void* C; int ldc; int m, n;
  double2 alpha, beta;
  int term0, nterms;
};

// C = alpha op(A) + beta C; A and C may differ in element size (the copies
// between the complex128 assembly and complex64 factors convert)
struct GeamDesc {
  const void* A; void* C;
  int lda, ldc, opA, m, n;
  int esA, esC;
  double2 alpha, beta;
  const double* rs;      // optional (nullptr: 1): C(i, j) = alpha rs[i] op(A)(i, j) cs[j] + beta C(i, j)
  const double* cs;
};

// Frobenius norm of a block of either element size, accumulated in double
struct NormDesc { const void* A; int lda, m, n; int es; double* out; };

// Equilibration of a complex128 block: mode 0, the column norms of diag(scale) A
// (scale over rows, may be nullptr); mode 1, the row norms of A diag(scale)
// (scale over columns).  s = 1 / norm and is = norm per column (row); a zero
// norm gives s = is = 1.
struct EquilDesc { const double2* A; int lda, m, n; int mode; const double* scale; double* s; double* is; };

struct SkelLUJob {       // X = D^{-1} B, D = A(rows, cols) or its adjoint
  const int* rows; const int* cols; int r;
  int adjD;
  const double2* B; int ldb; int adjB;
  int m;
  double2* X; int ldx; int adjX;
  double2* work;         // r*r + r*m
  int* piv;
};

// One direction of compress_P2P (FMM2DTree_find_error.hpp:1532-1559) in one CTA:
// column QR of [L2P_k | P2P_kb] with threshold tol -> rank rc, nL = Q(:, :rc);
// R' = nL^H P2P_kb, R = nL^H L2P_k; row QR of [P2M_b^H | R'^H] -> rank rr,
// nPt = Q(:, :rr); M2L' = R M2L_kb (nPt^H P2M_b^H)^H + (nPt^H R'^H)^H.
struct CompressJob {
  const void* L2P; int ldL;        // m x rK
  const void* Pkb; int ldP;        // m x c
  const void* P2M; int ldM;        // rb x c
  const void* M2L; int ldT;        // rK x rb
  int m, rK, c, rb;
  double tol;
  void* nL;                        // out: m x rc (ld m), room for min(m, rK + c) columns
  void* nPt;                       // out: c x rr (ld c), room for min(c, rb + min(m, rK + c)) columns
  void* M2Lo; int ldO;             // out: rc x rr
  int* ranks;                      // out: rc, rr
  // scratch
  void* Acol;                      // m x (rK + c)
  void* Arow;                      // c x (rb + rc)
  void* tau; int* perm; int* info;
  void* Rkp; void* Rk; void* Rn; void* Rnp; void* Tm;
};

// launchers (return a cudaError_t value)
int aifmm_launch_tables(int n_cheb, int degree, double kappa, double r, const double* gl_x, const double* gl_w,
                        const int2* basis, const double* cheb, double2* Cwork, double2* Vwork, int* status,
                        double* qpinv, double2* M, double2* nearT, cudaStream_t stream);
int aifmm_launch_block_entries(const BlockDesc* d_desc, const long long* d_off, int nd, long long total,
                               const EntryCtx& ctx, cudaStream_t stream);
int aifmm_launch_list_entries(const int* I, const int* J, long n, double2* out, const EntryCtx& ctx,
                              cudaStream_t stream);
int aifmm_launch_dense_matvec(const double2* x, double2* y, int N, int nrhs, const EntryCtx& ctx,
                              cudaStream_t stream);
// y += G x with G the entries without kappa^2 q and identity (findPhi = false)
int aifmm_launch_green_matvec_add(const double2* x, double2* y, int N, int nrhs, const EntryCtx& ctx,
                                  cudaStream_t stream);
int aifmm_launch_aca(const AcaJob* d_jobs, int njobs, double tol, const EntryCtx& ctx, cudaStream_t stream);
int aifmm_launch_qr_factor(const QRJob* d_jobs, int njobs, int es, cudaStream_t s);
int aifmm_launch_qr_solve(const SolveJob* d_jobs, const int* d_col_off, int njobs, int total_cols, int es,
                          cudaStream_t s);
size_t aifmm_qr_smem_bytes(int m, int n, int es);
// one warp per right-hand side (8 per CTA), the column in registers; m <= 224 and
// the factor's first nzp columns must fit in shared memory
int aifmm_launch_qr_solve_warp(const SolveJob* d_jobs, const int* d_cta_off, int njobs, int total_ctas, int mmax,
                               int nzpmax, int es, cudaStream_t s);
// one CTA per factorisation, the matrix in shared memory (aifmm_qr_smem_bytes)
int aifmm_launch_qr_factor_smem(const QRJob* d_jobs, int njobs, size_t smem, int es, cudaStream_t s);
// shared memory the fused compression needs for these sizes (0: does not fit)
size_t aifmm_compress_smem_bytes(int m, int rK, int c, int rb, int es);
int aifmm_launch_compress_p2p(const CompressJob* d_jobs, int njobs, size_t smem, int es, cudaStream_t s);
int aifmm_launch_formq(const FormQJob* d_jobs, const int* d_col_off, int njobs, int total_cols, int es, cudaStream_t s);
// tile_cols: output tile width, 32 (32 x 32 tiles) or 16 (32 x 16 tiles for thin products)
int aifmm_launch_gemm(const GemmDesc* d, const GemmTerm* d_terms, const int* d_tile_off, int nd, int total_tiles,
                      cudaStream_t s, int tile_cols, int es = 16);
int aifmm_launch_geam(const GeamDesc* d, const long long* d_off, int nd, long long total, cudaStream_t s);
int aifmm_launch_norms(const NormDesc* d, int nd, cudaStream_t s);
int aifmm_launch_equilibrate(const EquilDesc* d, int nd, cudaStream_t s);
int aifmm_launch_skel_lu(const SkelLUJob* d, int nd, const EntryCtx& ctx, cudaStream_t s);
