"""The mixed form: complex64 factorisation, FP64 refinement.

aifmm_factorize(p, AIFMM_PRECISION_C64, ...) runs the elimination, its factors
and the direct solves in complex64 (after an equilibration of the bases), at a
recompression tolerance of at least 1e-6; aifmm_solve_refined then runs GMRES in
FP64 against the complex128 compressed product with those factors as the
preconditioner.  The bar where the form applies (shallow trees): the refined
solution lands where the FP64 refined solution lands -- on the dense solve of
the oracle's compressed matrix A_c, to 1e-8 relative.  Where it does not (deeper
trees: the elimination's internal growth times FP32 rounding), the refined
solve must report the stagnation instead of returning a wrong answer.
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


@pytest.mark.parametrize("q_kind,kappa,tol_pow", [("gauss_aw", 40.0, 10), ("disk", 20.0, 8)])
def test_mixed_refined_solve_converges_to_the_compressed_system(oracle_mod, table_cache, q_kind, kappa, tol_pow):
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=3, q_kind=q_kind, kappa=kappa, tol_pow=tol_pow)
    K, T = _tree(p, tabs)
    T.factorize(keep_assembly=True, precision=A.PRECISION_C64)
    b = K.rhs_plane_wave([0.7, 3.1])
    x, iters, relres = T.solve_refined(b, rtol=1e-11, maxit=80)
    Ac = oracle_mod.Problem(p, *tabs[:2]).compressed_dense()
    xd = np.linalg.solve(Ac, b.T).T
    rel = np.linalg.norm(x - xd) / np.linalg.norm(xd)
    print("%s: complex64 factors, refined (%d iterations, residual %.1e) vs dense A_c solve %.2e"
          % (q_kind, iters, relres, rel))
    assert relres <= 1e-11
    assert rel <= 1e-8


def test_mixed_matches_fp64_refined_on_benchmark_physics(table_cache):
    """Depth 3, Gaussian 1.5 exp(-32|x|^2), kappa 40, assembly tolerance 1e-10: the
    complex64 and FP64 (factor tolerance 1e-6) refined solutions to residual 1e-10
    agree to 1e-8."""
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=3, q_kind="gauss_aw", kappa=40.0, tol_pow=10)
    b = None
    out = {}
    for prec in (A.PRECISION_FP64, A.PRECISION_C64):
        K, T = _tree(p, tabs)
        T.set_factor_tolerance(6)
        T.factorize(keep_assembly=True, precision=prec)
        if b is None:
            b = K.rhs_plane_wave([0.2, 2.9, 4.4])
        x, iters, relres = T.solve_refined(b, rtol=1e-10, maxit=80)
        r = b - T.compressed_matvec(x)
        true_rel = np.max(np.linalg.norm(r, axis=1) / np.linalg.norm(b, axis=1))
        out[prec] = x
        print("precision %d: %d GMRES iterations, residual %.2e (recomputed %.2e)" % (prec, iters, relres, true_rel))
        assert relres <= 1e-10 and true_rel <= 2e-10
    d_ref = np.linalg.norm(out[A.PRECISION_C64] - out[A.PRECISION_FP64]) / np.linalg.norm(out[A.PRECISION_FP64])
    print("refined: complex64 vs FP64 factors %.2e" % d_ref)
    assert d_ref <= 1e-8


def test_mixed_refinement_reports_stagnation_on_a_deep_tree(table_cache):
    """Depth 4 of the same physics: the elimination's internal growth times FP32
    rounding leaves the complex64 direct solve far from linear, so GMRES cannot
    converge; the refined solve must say so (AIFMM_ERR_NUMERIC, after its short
    first cycle and one more) instead of returning a wrong answer."""
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=4, q_kind="gauss_aw", kappa=40.0, tol_pow=10)
    K, T = _tree(p, tabs)
    T.set_factor_tolerance(6)
    T.factorize(keep_assembly=True, precision=A.PRECISION_C64)
    b = K.rhs_plane_wave([0.2])
    with pytest.raises(A.AifmmError) as ei:
        T.solve_refined(b, rtol=1e-10, maxit=80)
    assert ei.value.status == 5  # AIFMM_ERR_NUMERIC
    print("depth 4 complex64:", ei.value)
    # the same handle refactored in FP64 refines to the target
    T.factorize(keep_assembly=True, precision=A.PRECISION_FP64)
    x, iters, relres = T.solve_refined(b, rtol=1e-10, maxit=80)
    assert relres <= 1e-10


def test_mixed_graph_solve_is_the_eager_solve(table_cache):
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=3, q_kind="gaussian160", kappa=10.0, tol_pow=8)
    K, T = _tree(p, tabs)
    T.factorize(keep_assembly=True, precision=A.PRECISION_C64)
    b = K.rhs_plane_wave([0.0, 1.3, 2.2])
    x0 = T.solve_factored(b)
    x1 = T.solve_factored(b, graph=True)
    x2 = T.solve_factored(b, graph=True)
    assert np.array_equal(x0, x1) and np.array_equal(x1, x2)
    # complex64 arithmetic: the solution carries no more than FP32 precision
    xr = np.asarray(x0)
    assert np.array_equal(xr.real.astype(np.float32).astype(np.float64), xr.real)


def test_fp64_after_mixed_on_one_handle(table_cache):
    """Refactoring a handle in FP64 after a complex64 factorisation gives the bits
    of a fresh FP64 handle (the kept assembly stays complex128)."""
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=3, q_kind="gauss_aw", kappa=20.0, tol_pow=10)
    K, T = _tree(p, tabs)
    b = K.rhs_plane_wave([0.4])
    T.factorize(keep_assembly=True, precision=A.PRECISION_C64)
    x32 = T.solve_factored(b)
    T.factorize(keep_assembly=True, precision=A.PRECISION_FP64)
    x64 = T.solve_factored(b)
    K2, T2 = _tree(p, tabs)
    T2.factorize(keep_assembly=True)
    x64b = T2.solve_factored(b)
    assert np.array_equal(x64, x64b)
    assert not np.array_equal(x32, x64)
