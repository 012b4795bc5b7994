/*
 * aifmm_oracle.h -- C interface of the CPU oracle for the AIFMM-LS direct solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA product
 * path is compared against.  Only the test suite, the smoke check and the CPU
 * baseline leg of the benchmark may load it; the product library never links
 * or calls it.
 *
 * Parity status: the Gauss-Legendre rule is pinned bit-for-bit against the
 * reference's own table (LS/Gauss_Legendre_Nodes_and_Weights.hpp, case 10) and
 * the Bessel values against high-precision (mpmath) fixtures.  Everything else
 * (quadrature tables, ACA, elimination) is a restatement of the reference's
 * algorithm with no reference-produced golden outputs to compare with, because
 * the reference cannot be compiled without Eigen and Boost: parity of those
 * stages is therefore unpinned against the reference itself and is checked
 * against a dense direct solve instead.
 */
#ifndef AIFMM_ORACLE_H
#define AIFMM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Contrast kinds.  0..5 are the reference's Qchoice values
 * (LS/LS_functions.hpp:99-112); 10 and 11 are the Gaussian and disk contrasts
 * with free parameters used by the larger workloads. */
enum {
  ORC_Q_GAUSSIAN160 = 0, ORC_Q_MULTI_GAUSS = 1, ORC_Q_PLASMA = 2,
  ORC_Q_FLATBUMP = 3, ORC_Q_CAVITY = 4, ORC_Q_LENS = 5,
  ORC_Q_GAUSS_AW = 10,   /* amp * exp(-width*|x|^2) */
  ORC_Q_DISK = 11        /* amp * [|x| < radius] */
};

typedef struct {
  int n_cheb;        /* Chebyshev nodes per leaf per dimension */
  double kappa;      /* wavenumber */
  int degree;        /* polynomial degree of the basis (NB = d(d+1)/2) */
  double L;          /* half width of the domain */
  int depth;         /* uniform quadtree depth (leaf level) */
  int tol_pow;       /* ACA / RRQR tolerance = 10^-tol_pow */
  int q_kind;        /* contrast kind (see enum) */
  double q_amp, q_width, q_radius;
} orc_params;

/* Gauss-Legendre n-point rule by Newton iteration (nodes in the reference's
 * interleaved -x,+x order). */
int orc_gauss_legendre(int n, double* nodes, double* weights);

/* J_n(x), Y_n(x) for n = 0..nmax (reference precision recurrences). */
int orc_bessel_jy(int nmax, double x, double* J, double* Y);

/* Leaf-level tables: M (121 x rank, complex, column-major, interleaved re/im),
 * near (9 x rank x rank, complex, column-major per table), Qpinv (NB x rank).
 * round6 != 0 applies the reference's 6-significant-digit text round trip. */
int orc_tables(const orc_params* p, int round6, double* M, double* near_tab, double* qpinv);

void* orc_create(const orc_params* p, const double* M, const double* near_tab);
void orc_destroy(void* h);
int orc_num_points(void* h);
int orc_grid_points(void* h, double* xy);
/* contrast values at the grid points */
int orc_contrast(void* h, double* q);
/* plane-wave right-hand side b = -kappa^2 q exp(i kappa (x cos t + y sin t)) */
int orc_rhs_plane_wave(void* h, int nrhs, const double* theta, double* b);
int orc_entries(void* h, long n, const int* I, const int* J, double* out);
/* y = A x for nrhs right-hand sides (dense, exact entries) */
int orc_dense_matvec(void* h, int nrhs, const double* x, double* y);
/* u = u_inc + G phi (the total field of hybrid.cpp:263-281; G = entries with findPhi off) */
int orc_total_field(void* h, int nrhs, const double* theta, const double* phi, double* u);
/* Full pipeline: assemble, eliminate_phase_efficient (with the rhs carried),
 * base solve, back substitution.  times[4] = tree, assemble, factor, solve (s). */
int orc_solve(void* h, int nrhs, const double* b, double* x, double* times);
/* a solve with new right-hand sides against the factors of the last orc_solve */
int orc_solve_again(void* h, int nrhs, const double* b, double* x);
/* Multiply every matrix entry by (1 + rel*u), u a fixed pseudo-random number in
 * [-1, 1] per (i, j): used to measure how strongly the algorithm amplifies
 * last-bit differences in the entries. */
int orc_set_perturbation(void* h, double rel);
/* 0: eliminate_phase_efficient (the reference driver's choice, default);
 * 1: eliminate_phase (compress every queued pair after each box). */
int orc_set_variant(void* h, int full_compress);
/* Test-only reorderings used by the GPU solver (1: back substitution in waves;
 * 2: P2P[k][k] factorisation and its right-hand-side / neighbour solves before the
 * step's recompressions; 4: L2M_f factorisation and its solves before the x-phase
 * fill-ins).  0 is the reference's order. */
int orc_set_schedule(void* h, int flags);
/* recompressions performed by the last solve */
long orc_compressions(void* h);
/* dense N x N matrix (column-major complex) implied by the compressed
 * representation before elimination */
int orc_compressed_dense(const orc_params* p, const double* M, const double* near_tab, double* out);
/* Introspection after orc_solve: per box ranks of a level (after getNodes). */
int orc_level_ranks(void* h, int level, int* rank_in, int* rank_out);
/* neighbour (8), inner (16) and outer (24) interaction lists of one box */
int orc_box_lists(void* h, int level, int box, int* out48);
/* skeleton point lists of one box (incoming check / charge, outgoing check / charge) */
int orc_box_skeleton(void* h, int level, int box, int which, int* out, int cap);

#ifdef __cplusplus
}
#endif
#endif
