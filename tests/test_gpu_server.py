"""The serving loop (aifmm_server_*): factors resident on the device, solve
requests batched continuously, admission by device memory with LRU eviction.

Each right-hand side must come out the same alone (its own factorize + solve on
a fresh handle) and in the mix (batched with other requests, other keys'
work overlapping on the GPU).  The solver's kernels compute every column of a
multi-RHS solve independently and in a fixed order, so the bar is bit-for-bit.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROBLEMS = {
    1: dict(n_cheb=6, kappa=10.0, degree=6, depth=3, tol_pow=8, q_kind="gaussian160"),
    2: dict(n_cheb=6, kappa=20.0, degree=6, depth=3, tol_pow=8, q_kind="disk", q_amp=2.0, q_radius=0.5),
    3: dict(n_cheb=6, kappa=40.0, degree=6, depth=4, tol_pow=10, q_kind="gauss_aw", q_amp=1.5, q_width=32.0),
}


def _alone(kw, b):
    import aifmm_ls_b200 as A
    K = A.LSKernel(**kw)
    K.tables_compute(round6=True)
    T = A.FMM2DTree(K)
    T.createTree()
    T.assemble()
    T.factorize()
    return T.solve_factored(b)


def _rhs(key, nrhs, seed):
    import aifmm_ls_b200 as A
    K = A.LSKernel(**PROBLEMS[key])
    rng = np.random.default_rng(seed)
    return K.rhs_plane_wave(rng.uniform(0, 2 * np.pi, nrhs))


def test_results_same_alone_and_in_the_mix():
    import aifmm_ls_b200 as A
    S = A.Server(workers=3, max_batch_rhs=16)
    try:
        for key, kw in PROBLEMS.items():
            S.factorize(key, **kw)
        rng = np.random.default_rng(11)
        jobs = [(int(rng.integers(1, 4)), int(rng.integers(1, 5)), s) for s in range(24)]
        rhs = {s: _rhs(key, nr, 100 + s) for key, nr, s in jobs}
        ids = {}
        lock = threading.Lock()

        def submit(part):
            for key, nr, s in part:
                rid = S.solve(key, rhs[s])
                with lock:
                    ids[s] = (key, rid)

        threads = [threading.Thread(target=submit, args=(jobs[i::3],)) for i in range(3)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        out, batch = {}, {}
        for s, (key, rid) in ids.items():
            st, lat, br, x = S.wait(rid)
            assert st == 0, st
            out[s], batch[s] = x, br
        stats = S.stats()
        print("server:", stats)
        assert stats["solves"] == len(jobs)
        assert stats["batches"] < len(jobs)  # requests were batched
        for key, nr, s in jobs:
            x_alone = _alone(PROBLEMS[key], rhs[s])
            assert np.array_equal(out[s], x_alone), (key, s, batch[s])
    finally:
        S.close()


def test_lru_eviction_and_factoring_again():
    import aifmm_ls_b200 as A
    # room for one depth-3 factorisation (the server's estimate) but not two
    est = (4 ** 3 * 36) * 36 * 1100.0 + (64 << 20)
    S = A.Server(workers=1, hbm_budget_bytes=1.5 * est)
    try:
        b1 = _rhs(1, 2, 5)
        b2 = _rhs(2, 1, 6)
        assert S.wait(S.factorize(1, **PROBLEMS[1]))[0] == 0
        x1 = S.wait(S.solve(1, b1))[3]
        assert S.wait(S.factorize(2, **PROBLEMS[2]))[0] == 0  # evicts key 1
        x2 = S.wait(S.solve(2, b2))[3]
        st, lat, br, x1b = S.wait(S.solve(1, b1))  # key 1 is factored again from its kept description
        assert st == 0
        stats = S.stats()
        print("server:", stats)
        assert stats["evictions"] >= 2 and stats["resident"] == 1
        assert np.array_equal(x1, x1b)
        assert np.array_equal(x1, _alone(PROBLEMS[1], b1))
        assert np.array_equal(x2, _alone(PROBLEMS[2], b2))
    finally:
        S.close()


def test_failed_requests_do_not_stop_the_server():
    import aifmm_ls_b200 as A
    S = A.Server(workers=2, hbm_budget_bytes=2e9)
    try:
        bad = S.factorize(7, n_cheb=1, depth=3)  # invalid description
        huge = S.factorize(8, n_cheb=16, depth=8)  # larger than the budget
        with pytest.raises(A.AifmmError):
            S.solve(99, np.zeros((1, 10), np.complex128))  # never factored
        assert S.wait(bad)[0] == 1  # AIFMM_ERR_ARG
        assert S.wait(huge)[0] == 4  # AIFMM_ERR_NOMEM
        ok = S.factorize(1, **PROBLEMS[1])
        b = _rhs(1, 1, 9)
        rid = S.solve(1, b)
        assert S.wait(ok)[0] == 0
        st, lat, br, x = S.wait(rid)
        assert st == 0
        assert np.array_equal(x, _alone(PROBLEMS[1], b))
        assert S.stats()["failed"] == 2
    finally:
        S.close()


def test_mixed_form_results_alone_and_in_the_mix():
    """The mixed form (complex64 factors, each solve refined to relative residual
    1e-8 against the compressed product): every result in the mix meets that
    residual on a handle of its own and agrees with the same right-hand side
    solved alone to the tolerance times the conditioning.  Complex64 factors
    serve the depth-3 keys; the depth-4 key gets FP64 factors (complex64 ones do
    not precondition it), refined the same way."""
    import aifmm_ls_b200 as A
    rtol = 1e-8
    S = A.Server(workers=3, max_batch_rhs=16, precision=A.PRECISION_C64, rtol=rtol)
    try:
        for key, kw in PROBLEMS.items():
            S.factorize(key, **kw)
        rng = np.random.default_rng(21)
        jobs = [(int(rng.integers(1, 4)), int(rng.integers(1, 4)), s) for s in range(12)]
        rhs = {s: _rhs(key, nr, 300 + s) for key, nr, s in jobs}
        ids = {s: (key, S.solve(key, rhs[s])) for key, nr, s in jobs}
        out = {}
        for s, (key, rid) in ids.items():
            st, lat, br, x = S.wait(rid)
            assert st == 0, st
            out[s] = x
        stats = S.stats()
        print("server (mixed):", stats)
        assert stats["solves"] == len(jobs) and stats["mean_gmres_iterations"] >= 1
        assert stats["promoted_to_fp64"] == 0 and stats["failed"] == 0
    finally:
        S.close()
    handles = {}
    for key, nr, s in jobs:
        if key not in handles:
            K = A.LSKernel(**PROBLEMS[key])
            K.tables_compute(round6=True)
            T = A.FMM2DTree(K)
            T.createTree()
            T.assemble()
            prec = A.PRECISION_C64 if PROBLEMS[key]["depth"] <= 3 else A.PRECISION_FP64
            T.factorize(keep_assembly=True, precision=prec)
            handles[key] = (K, T)
        K, T = handles[key]
        b = rhs[s]
        x_alone, iters, relres = T.solve_refined(b, rtol=rtol, maxit=90)
        res = np.max(np.linalg.norm(b - T.compressed_matvec(out[s]), axis=1) / np.linalg.norm(b, axis=1))
        diff = np.linalg.norm(out[s] - x_alone) / np.linalg.norm(x_alone)
        assert res <= 1.5 * rtol, (key, s, res)
        assert diff <= 1e-6, (key, s, diff)
