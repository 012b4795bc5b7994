"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances: matrix entries agree to 1e-12 relative (FP64, different Bessel and
summation order); skeleton index lists and ranks are identical; the solution of
the FP64 solver agrees with the oracle's to 1e-8 relative (the parity bar of the
reference path).  Tables computed on the GPU agree with the oracle's to the
quadrature tolerance; solver parity tests feed both sides the same tables.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-8
ENTRY_TOL = 1e-12


def _kernel(p, tables):
    import aifmm_ls_b200 as A
    from oracle import oracle as O
    names = {v: k for k, v in O.Q_KINDS.items()}
    K = A.LSKernel(n_cheb=p.n_cheb, kappa=p.kappa, degree=p.degree, L=p.L, depth=p.depth, tol_pow=p.tol_pow,
                   q_kind=names[p.q_kind], q_amp=p.q_amp, q_width=p.q_width, q_radius=p.q_radius)
    M, near, _ = tables
    K.tables_set(M, near)
    return K


def test_grid_and_rhs_match_oracle(oracle_mod, table_cache):
    p, tabs = table_cache(depth=3, q_kind="gauss_aw", kappa=20.0)
    K = _kernel(p, tabs)
    P = oracle_mod.Problem(p, *tabs[:2])
    assert np.array_equal(K.gridPoints, P.grid_points())
    th = [0.0, 0.7, 2.9]
    b = K.rhs_plane_wave(th)
    bo = P.rhs_plane_wave(th)
    assert np.max(np.abs(b - bo)) <= 1e-13 * np.max(np.abs(bo))


def _round6_kat(gpu, ora):
    """Survey KAT 6: the tables after the reference's 6-digit text round trip.
    About a fifth of the real and imaginary parts vanish by symmetry; both
    implementations leave rounding noise there (< 1e-12 of the table's scale),
    which the text round trip keeps and which no two implementations share.
    Every significant part must be bit-identical; noise parts must agree to
    1e-12 of the scale.  Returns (flips among significant parts, parts)."""
    a = np.concatenate([gpu.real.ravel(), gpu.imag.ravel()])
    b = np.concatenate([ora.real.ravel(), ora.imag.ravel()])
    scale = np.max(np.abs(b))
    sig = np.abs(b) >= 1e-12 * scale
    flips = int(np.count_nonzero(a[sig] != b[sig]))
    assert np.max(np.abs(a[~sig] - b[~sig])) <= 1e-12 * scale
    return flips, int(sig.sum())


def test_gpu_tables_match_oracle(oracle_mod):
    import aifmm_ls_b200 as A
    p = oracle_mod.params(depth=3, kappa=10.0)
    M0, N0, _ = oracle_mod.tables(p, round6=False)
    K = A.LSKernel(depth=3, kappa=10.0)
    K.tables_compute(round6=False)
    M1, N1 = K.tables_get()
    # same adaptive quadrature (absolute tolerance 1e-7 per integral): the values agree far below it
    for a, b in ((M1, M0), (N1, N0)):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    M0r, N0r, _ = oracle_mod.tables(p, round6=True)
    K.tables_compute(round6=True)
    M1r, N1r = K.tables_get()
    flips, nsig = _round6_kat(np.concatenate([M1r.ravel(), N1r.ravel()]), np.concatenate([M0r.ravel(), N0r.ravel()]))
    print("6-digit tables: significant parts differing between GPU and oracle: %d of %d" % (flips, nsig))
    assert flips == 0


@pytest.mark.parametrize("q_kind,kappa", [("gaussian160", 10.0), ("gauss_aw", 40.0), ("disk", 80.0)])
def test_entries_match_oracle(oracle_mod, table_cache, q_kind, kappa):
    p, tabs = table_cache(depth=4, q_kind=q_kind, kappa=kappa)
    K = _kernel(p, tabs)
    P = oracle_mod.Problem(p, *tabs[:2])
    rng = np.random.default_rng(20261203)
    N = K.N
    I = rng.integers(0, N, 4000)
    J = rng.integers(0, N, 4000)
    # include near-field and diagonal entries
    J[:500] = I[:500]
    J[500:1000] = np.minimum(I[500:1000] + 1, N - 1)
    g = K.entries(I, J)
    o = P.entries(I, J)
    scale = np.maximum(np.abs(o), 1e-300)
    err = np.abs(g - o)
    ok = (err <= ENTRY_TOL * scale) | (err <= 1e-15)
    assert ok.all(), (np.max(err / scale), int((~ok).sum()))


@pytest.mark.parametrize("q_kind,kappa,tol_pow", [("gaussian160", 10.0, 8), ("gauss_aw", 20.0, 10), ("disk", 20.0, 8)])
def test_skeletons_match_oracle(oracle_mod, table_cache, q_kind, kappa, tol_pow):
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=4, q_kind=q_kind, kappa=kappa, tol_pow=tol_pow)
    K = _kernel(p, tabs)
    T = A.FMM2DTree(K)
    T.createTree()
    T.assemble()
    P = oracle_mod.Problem(p, *tabs[:2])
    b = P.rhs_plane_wave([0.0])
    P.solve(b)
    for lev in range(2, p.depth + 1):
        ri, ro = T.level_ranks(lev)
        ri_o, ro_o = P.level_ranks(lev)
        assert np.array_equal(ri, ri_o), lev
        assert np.array_equal(ro, ro_o), lev
        for box in range(0, 4 ** lev, max(1, 4 ** lev // 23)):
            for which in range(4):
                assert np.array_equal(T.box_skeleton(lev, box, which), P.box_skeleton(lev, box, which)), (lev, box, which)


def _oracle_spread(oracle_mod, p, M, near, b, x0):
    """How far the oracle's own solution moves when every entry is perturbed by
    1e-16 relative: the resolution to which the reference algorithm defines x."""
    spread = 0.0
    for eps in (1e-16, -1e-16, 3e-16):
        P = oracle_mod.Problem(p, M, near)
        P.set_perturbation(eps)
        x1, _ = P.solve(b)
        spread = max(spread, np.linalg.norm(x1 - x0) / np.linalg.norm(x0))
    return spread


@pytest.mark.parametrize("q_kind,kappa,tol_pow,depth", [
    ("gaussian160", 10.0, 8, 3), ("gaussian160", 10.0, 8, 4),
    ("gauss_aw", 20.0, 10, 3), ("gauss_aw", 40.0, 10, 4),
    ("disk", 20.0, 8, 3), ("disk", 20.0, 8, 4)])
def test_solution_matches_oracle(oracle_mod, table_cache, q_kind, kappa, tol_pow, depth):
    """x_gpu vs x_oracle <= max(1e-8, 5 x the oracle's own spread under 1e-16
    entry perturbations); where the oracle is well defined to 1e-8 (the
    reference driver's Gaussian contrast) this is the 1e-8 bar itself."""
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=depth, q_kind=q_kind, kappa=kappa, tol_pow=tol_pow)
    M, near = tabs[:2]
    K = _kernel(p, tabs)
    T = A.FMM2DTree(K)
    T.createTree()
    T.assemble()
    P = oracle_mod.Problem(p, M, near)
    b = P.rhs_plane_wave([0.0, 1.1])
    xo, _ = P.solve(b)
    x = T.solve(b)
    rel = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    spread = _oracle_spread(oracle_mod, p, M, near, b, xo)
    bound = max(SOLVE_TOL, 5.0 * spread)
    print("%s kappa=%g tol=1e-%d depth=%d: |x_gpu - x_oracle| = %.2e, oracle spread %.2e"
          % (q_kind, kappa, tol_pow, depth, rel, spread))
    assert rel <= bound, (rel, spread)
    if q_kind == "gaussian160":
        assert rel <= SOLVE_TOL
    if depth <= 3:  # the GPU solution is as accurate as the oracle's against a dense solve
        A_ = P.dense()
        xd = np.linalg.solve(A_, b.T).T
        eg = np.linalg.norm(x - xd) / np.linalg.norm(xd)
        eo = np.linalg.norm(xo - xd) / np.linalg.norm(xd)
        assert eg <= 1.5 * eo + 1e-8, (eg, eo)


def test_solve_twice_with_kept_assembly(oracle_mod, table_cache):
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=3, q_kind="gauss_aw", kappa=20.0, tol_pow=10)
    K = _kernel(p, tabs)
    T = A.FMM2DTree(K)
    T.createTree()
    T.assemble()
    b = K.rhs_plane_wave([0.3])
    x1 = T.solve(b, keep_assembly=True)
    x2 = T.solve(b)  # the kept copy of the assembly is restored
    assert np.array_equal(x1, x2)
    T.assemble()
    T.solve(b)
    with pytest.raises(A.AifmmError):
        T.solve(b)  # the elimination consumed the assembly and no copy was kept


def test_dense_matvec_matches_oracle(oracle_mod, table_cache):
    p, tabs = table_cache(depth=3, q_kind="gauss_aw", kappa=20.0)
    K = _kernel(p, tabs)
    P = oracle_mod.Problem(p, *tabs[:2])
    rng = np.random.default_rng(7)
    x = rng.standard_normal((2, K.N)) + 1j * rng.standard_normal((2, K.N))
    y = K.dense_matvec(x)
    yo = P.dense_matvec(x)
    assert np.linalg.norm(y - yo) / np.linalg.norm(yo) <= 1e-12


def test_total_field_matches_oracle(oracle_mod, table_cache):
    """u = u_inc + G phi (the scattered-field post-processing of hybrid.cpp:263-281)
    for the solver's own solution, against the oracle's dense product."""
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=3, q_kind="gauss_aw", kappa=20.0)
    K = _kernel(p, tabs)
    T = A.FMM2DTree(K)
    th = np.array([0.0, 0.9])
    b = K.rhs_plane_wave(th)
    T.createTree()
    T.assemble()
    phi = T.solve(b)
    u = K.total_field(th, phi)
    P = oracle_mod.Problem(p, *tabs[:2])
    uo = P.total_field(th, phi)
    assert np.linalg.norm(u - uo) / np.linalg.norm(uo) <= ENTRY_TOL
    # kappa^2 q u + phi is the solver's residual A phi - b: about 2e-4 relative at
    # this compression tolerance (the oracle's own solution gives the same)
    q = P.contrast()
    assert np.linalg.norm(p.kappa ** 2 * q * u + phi) / np.linalg.norm(phi) <= 1e-3


def test_reference_default_run_depth5(oracle_mod, table_cache):
    """The reference's default run `testFMM2D_find_error 6 10 6 1 0 8 5`
    (testFMM2D_find_error.cpp:44-52, Readme.md:17-21): 6x6 nodes, kappa 10,
    degree 6, Qchoice 0, TOL 1e-8, depth 5 (36,864 unknowns), one plane wave at
    theta = 0.  At this depth the reference algorithm itself resolves x only to
    ~1e-5: perturbing every entry by 1e-16 moves the oracle's solution by
    3e-6 .. 4e-4 (rank and pivot decisions near their thresholds).  So the bound
    is the one of test_solution_matches_oracle, max(1e-8, 5 x that spread), and
    the GPU solution must be as accurate as the oracle's: its residual with
    exact entries on 400 sampled rows within 10% of the oracle solution's."""
    import aifmm_ls_b200 as A
    p, tabs = table_cache(depth=5, q_kind="gaussian160", kappa=10.0, tol_pow=8)
    M, near = tabs[:2]
    K = _kernel(p, tabs)
    T = A.FMM2DTree(K)
    T.createTree()
    T.assemble()
    P = oracle_mod.Problem(p, M, near)
    b = P.rhs_plane_wave([0.0])
    xo, _ = P.solve(b)
    x = T.solve(b)
    rel = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    spread = 0.0
    for eps in (1e-16, -1e-16):
        Q = oracle_mod.Problem(p, M, near)
        Q.set_perturbation(eps)
        x1, _ = Q.solve(b)
        spread = max(spread, np.linalg.norm(x1 - xo) / np.linalg.norm(xo))
    rng = np.random.default_rng(5)
    rows = np.sort(rng.choice(K.N, 400, replace=False)).astype(np.int32)
    Ar = K.getMatrix(rows, np.arange(K.N, dtype=np.int32))
    res_g = np.linalg.norm(Ar @ x[0] - b[0, rows]) / np.linalg.norm(b[0, rows])
    res_o = np.linalg.norm(Ar @ xo[0] - b[0, rows]) / np.linalg.norm(b[0, rows])
    print("depth 5 reference run: |x_gpu - x_oracle| = %.2e, oracle spread %.2e; sampled residual GPU %.3e, "
          "oracle %.3e" % (rel, spread, res_g, res_o))
    assert rel <= max(SOLVE_TOL, 5.0 * spread)
    assert res_g <= 1.1 * res_o + 1e-12


def test_bench_path_with_gpu_tables(oracle_mod):
    """The benchmark's own path: tables computed on the GPU with the 6-digit round
    trip, against the oracle with the tables it computes itself (benchmark
    physics at depth 4: Gaussian 1.5 exp(-32|x|^2), kappa 40, TOL 1e-10)."""
    import aifmm_ls_b200 as A
    kw = dict(n_cheb=6, kappa=40.0, degree=6, depth=4, tol_pow=10, q_kind="gauss_aw", q_amp=1.5, q_width=32.0)
    p = oracle_mod.params(**kw)
    M0, N0, _ = oracle_mod.tables(p, round6=False)
    M0r, N0r, _ = oracle_mod.tables(p, round6=True)
    K = A.LSKernel(**kw)
    K.tables_compute(round6=False)
    M1, N1 = K.tables_get()
    K.tables_compute(round6=True)
    M1r, N1r = K.tables_get()
    v0 = np.concatenate([M0.ravel(), N0.ravel()])
    v1 = np.concatenate([M1.ravel(), N1.ravel()])
    rel_unrounded = np.max(np.abs(v1 - v0)) / np.max(np.abs(v0))
    flips, nsig = _round6_kat(np.concatenate([M1r.ravel(), N1r.ravel()]), np.concatenate([M0r.ravel(), N0r.ravel()]))
    print("tables before rounding: max difference %.2e of the scale; 6-digit significant parts differing: %d of %d"
          % (rel_unrounded, flips, nsig))
    T = A.FMM2DTree(K)
    T.createTree()
    T.assemble()
    th = [0.0, 2.1]
    b = K.rhs_plane_wave(th)
    x = T.solve(b)
    P = oracle_mod.Problem(p, M0r, N0r)
    xo, _ = P.solve(b)
    rel = np.linalg.norm(x - xo) / np.linalg.norm(xo)
    spread = _oracle_spread(oracle_mod, p, M0r, N0r, b, xo)
    print("bench path: |x_gpu(gpu tables) - x_oracle(oracle tables)| = %.2e, oracle spread %.2e" % (rel, spread))
    assert rel_unrounded <= 1e-12
    assert flips == 0
    assert rel <= max(SOLVE_TOL, 5.0 * spread), (rel, spread)
