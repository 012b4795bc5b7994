"""The compressed product y = A_c x and GMRES refinement against it.

A_c is the matrix the assembly represents before elimination (leaf near field
plus the interaction-list M2L blocks through the nested bases).  The oracle
builds it densely (orc_compressed_dense); the GPU product must agree with that
dense product to 1e-10 relative (FP64; the bases L2P = Ac D^-1 carry the
conditioning of the skeleton blocks D).  The refined solve -- a factorisation
at a looser recompression tolerance used as the preconditioner of GMRES on
A_c x = b -- must reach its residual target and land within the compression
tolerance of the FP64 oracle's solution.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tree(p, tabs):
    import aifmm_ls_b200 as A
    from oracle import oracle as O
    names = {v: k for k, v in O.Q_KINDS.items()}
    K = A.LSKernel(n_cheb=p.n_cheb, kappa=p.kappa, degree=p.degree, L=p.L, depth=p.depth, tol_pow=p.tol_pow,
                   q_kind=names[p.q_kind], q_amp=p.q_amp, q_width=p.q_width, q_radius=p.q_radius)
    K.tables_set(*tabs[:2])
    T = A.FMM2DTree(K)
    T.createTree()
    T.assemble()
    return K, T


@pytest.mark.parametrize("q_kind,kappa,tol_pow,depth", [("gaussian160", 10.0, 8, 3), ("gaussian160", 10.0, 8, 4),
                                                         ("gauss_aw", 20.0, 10, 3)])
def test_compressed_matvec_matches_oracle(oracle_mod, table_cache, q_kind, kappa, tol_pow, depth):
    p, tabs = table_cache(depth=depth, q_kind=q_kind, kappa=kappa, tol_pow=tol_pow)
    K, T = _tree(p, tabs)
    T.factorize(keep_assembly=True)
    rng = np.random.default_rng(3)
    x = rng.standard_normal((2, K.N)) + 1j * rng.standard_normal((2, K.N))
    y = T.compressed_matvec(x)
    Ac = oracle_mod.Problem(p, *tabs[:2]).compressed_dense()
    yo = (Ac @ x.T).T
    rel = np.linalg.norm(y - yo) / np.linalg.norm(yo)
    print("%s depth %d: |A_c x (GPU) - A_c x (oracle, dense)| = %.2e" % (q_kind, depth, rel))
    assert rel <= 1e-10


def test_refined_solve_reaches_its_residual(oracle_mod, table_cache):
    """Benchmark physics at depth 4 (Gaussian 1.5 exp(-32|x|^2), kappa 40, assembly
    tolerance 1e-10), factorised at recompression tolerance 1e-6."""
    p, tabs = table_cache(depth=4, q_kind="gauss_aw", kappa=40.0, tol_pow=10)
    K, T = _tree(p, tabs)
    T.set_factor_tolerance(6)
    T.factorize(keep_assembly=True)
    b = K.rhs_plane_wave([0.2, 2.9])
    x, iters, relres = T.solve_refined(b, rtol=1e-10, maxit=60)
    r = b - T.compressed_matvec(x)
    true_rel = np.max(np.linalg.norm(r, axis=1) / np.linalg.norm(b, axis=1))
    print("refined solve: %d GMRES iterations, reported %.2e, recomputed %.2e" % (iters, relres, true_rel))
    assert relres <= 1e-10 and true_rel <= 2e-10
    # the loosely factored direct solve alone is far from that
    x_direct = T.solve_factored(b)
    r0 = np.max(np.linalg.norm(b - T.compressed_matvec(x_direct), axis=1) / np.linalg.norm(b, axis=1))
    assert r0 > 1e3 * true_rel
    # the FP64 direct solve (tolerance 1e-10 throughout) drops fill-ins between
    # well-separated boxes (F:2442-2443), so it solves A_c only approximately
    P = oracle_mod.Problem(p, *tabs[:2])
    xo, _ = P.solve(b)
    print("refined (factor tol 1e-6) vs FP64 direct oracle (tol 1e-10): %.2e; direct at 1e-6 vs oracle %.2e"
          % (np.linalg.norm(x - xo) / np.linalg.norm(xo), np.linalg.norm(x_direct - xo) / np.linalg.norm(xo)))


@pytest.mark.parametrize("q_kind,kappa,tol_pow", [("gauss_aw", 40.0, 10), ("disk", 20.0, 8)])
def test_refined_solve_converges_to_the_compressed_system(oracle_mod, table_cache, q_kind, kappa, tol_pow):
    """GMRES refinement converges to A_c^-1 b, the solution of the compressed
    system the assembly represents: against the oracle's dense A_c, solved
    densely, to the residual target times the conditioning (1e-8 here)."""
    p, tabs = table_cache(depth=3, q_kind=q_kind, kappa=kappa, tol_pow=tol_pow)
    K, T = _tree(p, tabs)
    T.set_factor_tolerance(max(tol_pow - 4, 4))
    T.factorize(keep_assembly=True)
    b = K.rhs_plane_wave([0.7, 3.1])
    x, iters, relres = T.solve_refined(b, rtol=1e-11, maxit=60)
    Ac = oracle_mod.Problem(p, *tabs[:2]).compressed_dense()
    xd = np.linalg.solve(Ac, b.T).T
    rel = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    print("%s: refined (%d iterations, residual %.1e) vs dense A_c solve %.2e" % (q_kind, iters, relres, rel))
    assert relres <= 1e-11
    assert rel <= 1e-8
