/*
 * aifmm_b200.h -- C ABI of the B200 AIFMM-LS direct solver.
 *
 * A drop-in for the reference's (vaishna77/AIFMM_LS) solver path: the
 * userkernel / LS2DTree matrix (kernel.hpp, LS/LS_Assembly.hpp) and the
 * FMM2DTree build -> assemble -> eliminate -> back-substitute flow
 * (FMM2DTree_find_error.hpp).  Every entry point below names the reference
 * interface it replaces.  Plain C types only: complex numbers are interleaved
 * (re, im) doubles, matrices are column-major, point sets are (x, y) pairs.
 *
 * Pointer arguments that carry bulk data accept either host or device memory,
 * selected with AIFMM_PTR_DEVICE in `flags`; everything else is host memory.
 * Calls on one handle must not overlap (one CUDA stream per handle); separate
 * handles are independent.  Every call returns a status; aifmm_last_error()
 * gives the message of the last failure on a handle.
 */
#ifndef AIFMM_B200_H
#define AIFMM_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define AIFMM_ABI_VERSION 1

typedef enum {
  AIFMM_OK = 0,
  AIFMM_ERR_ARG = 1,       /* invalid argument */
  AIFMM_ERR_CUDA = 2,      /* CUDA runtime failure (message in aifmm_last_error) */
  AIFMM_ERR_STATE = 3,     /* call out of order (e.g. solve before assemble) */
  AIFMM_ERR_NOMEM = 4,     /* device allocation failed */
  AIFMM_ERR_NUMERIC = 5,   /* inconsistent block shapes / quadrature budget exhausted */
  AIFMM_ERR_NODEVICE = 6   /* no CUDA device */
} aifmm_status;

enum { AIFMM_PTR_HOST = 0, AIFMM_PTR_DEVICE = 1,
       /* factorize / factorize_solve: keep a copy of the assembled blocks so that the
        * handle can be factored again without re-assembling (the elimination consumes
        * them otherwise) */
       AIFMM_KEEP_ASSEMBLY = 2 };

/* aifmm_solve: replay a CUDA graph of the whole solve for this right-hand-side count.
 * The first such solve after a factorisation records the graph (one ordinary solve
 * plus the capture); the graph, its descriptors and its per-solve buffers stay on the
 * device until the factors are dropped (build_tree / assemble / factorize / destroy). */
enum { AIFMM_SOLVE_GRAPH = 4 };

/* Factorisation precision (aifmm_factorize).  FP64: complex128 throughout, the
 * reference's arithmetic.  C64: the mixed form -- the elimination, its factors and
 * aifmm_solve run in complex64 (recompression tolerance at least 1e-6); the assembly,
 * the compressed product and aifmm_solve_refined's GMRES stay complex128, so a
 * refined solve recovers FP64 accuracy against the compressed matrix. */
enum { AIFMM_PRECISION_FP64 = 0, AIFMM_PRECISION_C64 = 1 };

/* Contrast functions q(x): 0..5 are the reference's Qchoice values
 * (LS/LS_functions.hpp:99-112: gaussian 1.5 exp(-160|x|^2), multipleGaussians,
 * plasma, flatBump, cavity, lens); 10: amp*exp(-width*|x|^2); 11: amp*[|x| < radius]. */
enum { AIFMM_Q_GAUSSIAN160 = 0, AIFMM_Q_MULTI_GAUSS = 1, AIFMM_Q_PLASMA = 2, AIFMM_Q_FLATBUMP = 3,
       AIFMM_Q_CAVITY = 4, AIFMM_Q_LENS = 5, AIFMM_Q_GAUSS_AW = 10, AIFMM_Q_DISK = 11 };

/* Problem description: the reference driver's argv
 * (testFMM2D_find_error.cpp:44-52: nChebNodes kappa degreeOfBases L Qchoice TOL_POW nLevelsUniform)
 * plus the parameters of the extra contrast kinds. */
typedef struct {
  int n_cheb;      /* Chebyshev nodes per leaf per dimension (nChebNodes) */
  double kappa;    /* wavenumber */
  int degree;      /* degreeOfBases: NB = degree*(degree+1)/2 polynomial bases */
  double L;        /* half width of the domain */
  int depth;       /* nLevelsUniform: leaf level of the uniform quadtree */
  int tol_pow;     /* ACA and recompression tolerance 10^-tol_pow (TOL_POW) */
  int q_kind;      /* contrast (see enum) */
  double q_amp, q_width, q_radius;
} aifmm_desc;

typedef struct aifmm_problem aifmm_problem;

/* Replaces userkernel(...) (kernel.hpp:106-128) -> LS2DTree(...) (LS/LS_Assembly.hpp:234-277)
 * and FMM2DTree(...) (FMM2DTree_find_error.hpp:106-125): uniform tree, Chebyshev grid,
 * contrast; binds a CUDA device.  The caller owns the handle. */
aifmm_status aifmm_problem_create(const aifmm_desc* desc, int device, aifmm_problem** out);
aifmm_status aifmm_problem_destroy(aifmm_problem* p);
const char* aifmm_last_error(const aifmm_problem* p);
const char* aifmm_status_string(aifmm_status s);

/* Replaces evaluatePrecomputations / writeMToFile / getNeighborInteractions followed by
 * readMFromFile / readNeighborInteractions (LS/LS_Assembly.hpp:270-276, 1166-1228, 1320-1459):
 * leaf-level far-field coefficients M (121 x rank) and the 9 colleague near tables
 * (rank x rank each), by adaptive Gauss-Legendre quadrature on the GPU.  round6 != 0
 * applies the reference's text round trip (6 significant digits) to both. */
aifmm_status aifmm_tables_compute(aifmm_problem* p, int round6);
/* No counterpart in the reference.  The tables of aifmm_tables_compute(p, 0) (no
 * 6-digit round trip) written to caller-provided device buffers M_dev (121 x rank
 * complex) and near_dev (9 x rank x rank complex), without any device or host
 * allocation.  It is meant for callers that cannot let a library call cudaMalloc:
 * applications that reserve all device memory up front and hand it out through
 * their own allocator, and latency-sensitive loops that cannot accept the device
 * synchronisation cudaMalloc / cudaFree may cause.
 *  - Scratch is one fixed 1 MiB device array inside the library, held by every GPU
 *    that loads the library until the process exits; problems whose scratch
 *    (C 121 x NB, V 9 rank x NB, Q^+ NB x rank, 256-byte aligned) exceeds it are
 *    rejected with AIFMM_ERR_ARG (e.g. 16 x 16 nodes with degree >= 10).
 *  - The first call on a device looks up the array's device address; make that
 *    first call before any stream capture.
 *  - Runs on the handle's stream and returns when the tables are written.
 *  - All calls share the array: calls that overlap on the GPU (other handles,
 *    other host threads) race and must be serialised by the caller.
 *  - aifmm_last_error() is not updated by this call; the status is the error. */
aifmm_status aifmm_tables_compute_noalloc(aifmm_problem* p, double* M_dev, double* near_dev);
/* Supply / read the tables (host memory, interleaved complex, column-major:
 * M is 121 x rank, near is 9 consecutive rank x rank tables). */
aifmm_status aifmm_tables_set(aifmm_problem* p, const double* M, const double* near_tables);
aifmm_status aifmm_tables_get(aifmm_problem* p, double* M, double* near_tables);

/* userkernel::N (kernel.hpp:102) */
aifmm_status aifmm_num_points(const aifmm_problem* p, int* n_points);
/* userkernel::gridPoints (kernel.hpp:103; LS/LS_Assembly.hpp:1074-1087): N x 2 doubles (host) */
aifmm_status aifmm_grid_points(aifmm_problem* p, double* xy);
/* userKernel::RHSFunction (LS/LS_functions.hpp:113-120) for plane waves exp(i kappa (x cos t + y sin t)):
 * b is N x nrhs complex; theta is host memory. */
aifmm_status aifmm_rhs_plane_wave(aifmm_problem* p, int nrhs, const double* theta, double* b, int flags);

/* userkernel::getMatrixEntry (kernel.hpp:130-136 -> LS/LS_Assembly.hpp:474-541) for n (I, J) pairs */
aifmm_status aifmm_entries(aifmm_problem* p, long n, const int* I, const int* J, double* out, int flags);
/* kernel::getMatrix (kernel.hpp:74-86): out is nr x nc complex, column-major (getRow / getCol are nr = 1 / nc = 1) */
aifmm_status aifmm_get_matrix(aifmm_problem* p, int nr, const int* rows, int nc, const int* cols, double* out,
                              int flags);

/* FMM2DTree::createTree + assign_Tree_Interactions (FMM2DTree_find_error.hpp:127-1070) */
aifmm_status aifmm_build_tree(aifmm_problem* p);
/* FMM2DTree::assignLeafChargeLocations, getNodes (ACA skeletons, L2P/P2M), assemble_M2L,
 * initialise_phase, initialise_P2P_Leaf_Level (FMM2DTree_find_error.hpp:1072-1361, 1714-1741) */
aifmm_status aifmm_assemble(aifmm_problem* p);
/* FMM2DTree::assign_Leaf_rhs, eliminate_phase_efficient, back_substitution_phase
 * (FMM2DTree_find_error.hpp:1092-1103, 2407-2532) for nrhs right-hand sides at once:
 * b and x are N x nrhs complex (column-major). */
aifmm_status aifmm_factorize_solve(aifmm_problem* p, int nrhs, const double* b, double* x, int flags);

/* FMM2DTree::eliminate_phase_efficient and the base-level factorisation of
 * solve_particles_at_base_level (FMM2DTree_find_error.hpp:2407-2485) without a
 * right-hand side: the factors (QR of every P2P[k][k] and L2M_f, the fill-in
 * blocks the right-hand side passes through, the base-level QR) stay on the
 * device until the next build_tree / assemble / factorize.  precision:
 * AIFMM_PRECISION_FP64 or AIFMM_PRECISION_C64.  flags: AIFMM_KEEP_ASSEMBLY. */
aifmm_status aifmm_factorize(aifmm_problem* p, int precision, int flags);
/* The right-hand-side half of the reference's solve with kept factors:
 * assign_Leaf_rhs, the right-hand-side updates of eliminate_x / eliminate_z
 * (FMM2DTree_find_error.hpp:1968, 1997-2001, 2252, 2289-2293), the base-level
 * solve (:2453-2485) and back_substitution_phase (:2487-2532), for nrhs
 * right-hand sides at once.  b and x are N x nrhs complex with column strides ldb
 * and ldx (>= N), host or device memory (flags).  Any number of solves may follow
 * one aifmm_factorize.  stream (a cudaStream_t, may be NULL): the solve starts after
 * the work already queued on it, and work queued on it afterwards sees x. */
aifmm_status aifmm_solve(aifmm_problem* p, int nrhs, const double* b, long ldb, double* x, long ldx, void* stream,
                         int flags);
/* No counterpart in the reference: pick the batched GEMM's output-tile width (32 x 16 or
 * 32 x 32) for this handle by timing both on batches shaped like the problem's products
 * (thin: blocks times 8 right-hand sides; wide: block times block), at the leaf rank
 * and at four times it.  ms (may be NULL): 4 timings in ms, [thin 16, thin 32, wide 16,
 * wide 32]; tile_cols (may be NULL): the chosen widths [thin, wide].  Results do not
 * depend on the choice beyond rounding: both widths sum every product in the same order. */
aifmm_status aifmm_autotune(aifmm_problem* p, double* ms, int* tile_cols);
/* No counterpart in the reference: the recompression tolerance of the next
 * factorisations, 10^-tol_pow (0: the description's tol_pow, which always stays the
 * assembly's ACA tolerance).  A looser factorisation is a cheaper preconditioner for
 * aifmm_solve_refined. */
aifmm_status aifmm_set_factor_tolerance(aifmm_problem* p, int tol_pow);
/* No counterpart in the reference (its hybrid.cpp:199 calls a matvec of a DFMM class
 * that is not in the repository): y = A_c x, the product with the compressed matrix
 * the assembly represents -- leaf near-field blocks plus the interaction-list M2L
 * blocks of every level through the nested L2P / P2M bases (FMM2DTree_find_error.hpp:
 * 1105-1361, 1729-1741) -- in FP64.  Needs the kept assembly: call after
 * aifmm_factorize(p, precision, AIFMM_KEEP_ASSEMBLY).  x, y: N x nrhs complex with
 * column strides ldx, ldy; host or device memory (flags). */
aifmm_status aifmm_compressed_matvec(aifmm_problem* p, int nrhs, const double* x, long ldx, double* y, long ldy,
                                     int flags);
/* No counterpart in the reference: right-preconditioned restarted GMRES (restart 30; with
 * complex64 factors the first cycle is 10) on A_c x = b in FP64, with the kept factorisation as the preconditioner
 * and the direct solve as the starting guess, until every column's relative residual
 * ||b - A_c x|| / ||b|| <= rtol or maxit preconditioned products.  A restart cycle that
 * does not halve the worst true residual ends the solve with AIFMM_ERR_NUMERIC (the
 * factors are not an effective preconditioner; x is not written).  Needs
 * aifmm_factorize(p, precision, AIFMM_KEEP_ASSEMBLY).  *iterations and *relres (the
 * worst column's final relative residual) may be NULL.  b, x as aifmm_solve. */
aifmm_status aifmm_solve_refined(aifmm_problem* p, int nrhs, const double* b, long ldb, double* x, long ldx,
                                 double rtol, int maxit, int* iterations, double* relres, int flags);
/* FMM2DTree::error_check (FMM2DTree_find_error.hpp:2534-2581): *rel = ||x - x_true|| /
 * ||x_true|| (Frobenius norms over the nrhs columns; x and x_true N x nrhs complex with
 * column strides ldx and ldt, host or device memory). */
aifmm_status aifmm_find_error(aifmm_problem* p, int nrhs, const double* x, long ldx, const double* x_true, long ldt,
                              double* rel, int flags);

/* No counterpart in the reference: return the assembly's reusable workspaces and the
 * kept copy of the assembled blocks (AIFMM_KEEP_ASSEMBLY) to the device, keeping the
 * factors.  For a handle that from now on only solves (a cached factorisation).  After
 * a complex64 factorisation the kept copy stays: its refined solves need it. */
aifmm_status aifmm_trim(aifmm_problem* p);
/* No counterpart in the reference: return the assembly's reusable workspaces only; the
 * kept copy of the assembled blocks stays (for aifmm_solve_refined and
 * aifmm_compressed_matvec on a handle that keeps its factors). */
aifmm_status aifmm_release_workspaces(aifmm_problem* p);

/* No counterpart in the reference (its products are Eigen expressions inside the
 * elimination, e.g. FMM2DTree_find_error.hpp:1961-2075): the solver's batched complex
 * GEMM kernel (FP64 tensor cores) on one product, C = alpha op(A) op(B) + beta C,
 * op 0 = as is, 1 = conjugate transpose; column-major, alpha and beta are one
 * complex number each (host).  For checking the kernel against another BLAS. */
aifmm_status aifmm_zgemm(aifmm_problem* p, int opA, int opB, int m, int n, int k, const double* alpha,
                         const double* A, int lda, const double* B, int ldb, const double* beta, double* C, int ldc,
                         int flags);

/* The dense product of the find_error fixture generator (FMM2DTree_gen_rhs_x.hpp:2864-2871):
 * y = A x with exact entries, x and y N x nrhs complex (nrhs <= 8). */
aifmm_status aifmm_dense_matvec(aifmm_problem* p, int nrhs, const double* x, double* y, int flags);

/* The total field from a solution (hybrid.cpp:263-281, with the kernel's findPhi
 * switch of LS/LS_Assembly.hpp:474-541 off): u = u_inc + G phi, where
 * u_inc = exp(i kappa (x cos t_s + y sin t_s)) for angle theta[s] (the reference's
 * IncidenceFunction, LS/LS_functions.hpp:113-116, is t = 0) and G is the operator
 * whose entries are the system entries without the kappa^2 q(x_i) factor and the
 * identity.  Dense with exact entries; theta is a host array of nrhs angles; phi
 * and u are N x nrhs complex (nrhs <= 8). */
aifmm_status aifmm_total_field(aifmm_problem* p, int nrhs, const double* theta, const double* phi, double* u,
                               int flags);

/* Introspection: ranks of the ACA skeletons of a level after assemble (incoming, outgoing,
 * before the rank equalisation of get_L2P_P2M_box) and the skeleton point lists
 * (which: 0 incoming check, 1 incoming charge, 2 outgoing check, 3 outgoing charge). */
aifmm_status aifmm_level_ranks(aifmm_problem* p, int level, int* rank_in, int* rank_out);
aifmm_status aifmm_box_skeleton(aifmm_problem* p, int level, int box, int which, int* out, int cap, int* count);
/* Wall time of the last phases in ms: [0] build_tree [1] tables [2] assemble [3] factorize_solve
 * [4] factorize [5] solve (6 values). */
aifmm_status aifmm_phase_times(const aifmm_problem* p, double* ms);
/* Number of kernel launches issued by the last factorize_solve and by the last assemble. */
aifmm_status aifmm_launch_counts(const aifmm_problem* p, long* factor_solve, long* assemble);
/* Number of kernel launches issued by the last factorize and by the last solve. */
aifmm_status aifmm_launch_counts_split(const aifmm_problem* p, long* factorize, long* solve);
/* CUDA-event timing of one kind of kernel launch (0 QR factorisation, 1 QR solve,
 * 2 GEMM) on the handle's stream while enabled; reading returns the launches, the
 * summed device time (ms) and the summed algorithmic flops since it was enabled. */
aifmm_status aifmm_kernel_profile(aifmm_problem* p, int kind, int enable);
aifmm_status aifmm_kernel_profile_read(aifmm_problem* p, int kind, long* launches, double* ms, double* flops);
/* Host-side statistics of the last factorize_solve: [0] ms waiting in stream syncs,
 * [1] number of syncs, [2] ms in pending-pair handling (recompression), [3] ms in the
 * per-box elimination, [4] ms in back substitution, [5] recompressions, [6] total ms,
 * [7] kernel launches; of the last assemble: [8] ms building index lists on the host,
 * [9] ms in the ACA (launch to ranks on the host), [10] ms for the interpolative
 * operators, [11] ms for the M2L and P2P block entries, [12] ms of ACA kernel time
 * (CUDA events); device memory held by the handle: [13] bytes of the block pool, [14] bytes
 * of its workspaces (the assembly's reusable buffers, per-step scratch, descriptor
 * ring).  n <= 15 values are written. */
aifmm_status aifmm_stats(const aifmm_problem* p, double* out, int n);
/* The CUDA stream the handle works on (cudaStream_t). */
aifmm_status aifmm_get_stream(const aifmm_problem* p, void** stream);

/* ---- Serving loop (no counterpart in the reference, which solves one problem with
 * one right-hand side per process run, testFMM2D_find_error.cpp:41-176).
 * Factorisations stay resident on the device under a caller-chosen key; solve
 * requests against a key are batched continuously (every solve queued for a key
 * when a worker takes it runs as one multi-RHS aifmm_solve); factorisations are
 * admitted by device footprint and the least recently used idle one is evicted to
 * make room (a later solve on an evicted key factors it again).  Workers drive
 * their own handles and streams, so different keys overlap on the GPU.  All calls
 * are thread-safe. */
typedef struct aifmm_server aifmm_server;
/* hbm_budget_bytes <= 0: 80% of the device memory free at creation.  workers: host
 * threads (each runs one request at a time).  max_batch_rhs: right-hand sides per
 * batched solve (and the largest nrhs of one request). */
aifmm_status aifmm_server_create(int device, double hbm_budget_bytes, int workers, int max_batch_rhs,
                                 aifmm_server** out);
/* Runs the queued requests to completion, then stops the workers and frees every factor. */
aifmm_status aifmm_server_destroy(aifmm_server* s);
/* How many workers may run factorisations at once (default: all but one, so that
 * solves are never all stuck behind factorisations; 1 worker: that one). */
aifmm_status aifmm_server_set_factor_workers(aifmm_server* s, int n);
/* The form of the factorisations admitted from now on: AIFMM_PRECISION_FP64 (direct
 * solves with FP64 factors, the default) or AIFMM_PRECISION_C64 (complex64 factors
 * kept with the complex128 assembly for trees of depth <= 3, FP64 factors kept with it
 * for deeper trees -- complex64 factors do not precondition those, measured -- and every
 * solve aifmm_solve_refined to relative residual rtol; a key whose complex64 refinement
 * stagnates is refactored in FP64 from its kept assembly and refined again).  Keys
 * factored earlier keep their form. */
aifmm_status aifmm_server_set_form(aifmm_server* s, int precision, double rtol);
/* Queue a factorisation of desc under key (tables with the 6-digit round trip, tree,
 * assembly, FP64 factorisation); replaces an earlier one under the same key. */
aifmm_status aifmm_server_factorize(aifmm_server* s, long long key, const aifmm_desc* desc, long* request);
/* Queue nrhs right-hand sides against key (which must have been submitted for
 * factorisation).  b and x: host memory, N x nrhs complex, column-major; both must
 * stay valid until the request is waited for. */
aifmm_status aifmm_server_solve(aifmm_server* s, long long key, int nrhs, const double* b, double* x,
                                long* request);
/* Wait up to timeout_s seconds for a request.  AIFMM_ERR_STATE: not finished yet (wait
 * again).  Otherwise *result is the request's status, *latency_ms the time from
 * submission to completion and *batch_rhs the right-hand sides of the batch a solve
 * ran in (any output pointer may be NULL); the request is then forgotten. */
aifmm_status aifmm_server_wait(aifmm_server* s, long request, double timeout_s, aifmm_status* result,
                               double* latency_ms, int* batch_rhs);
/* [0] p50 and [1] p99 solve latency (ms), [2] p50 and [3] p99 factorisation latency,
 * [4] solves and [5] factorisations completed, [6] evictions, [7] solve batches,
 * [8] mean right-hand sides per batch, [9] device bytes held by factors, [10] resident
 * factorisations, [11] failed requests, [12] mean GMRES iterations per refined batch,
 * [13] mixed-form keys refactored in FP64.  n <= 14 values are written. */
aifmm_status aifmm_server_stats(aifmm_server* s, double* out, int n);

#ifdef __cplusplus
}
#endif
#endif /* AIFMM_B200_H */
