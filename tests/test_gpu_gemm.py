"""The solver's batched complex GEMM (FP64 tensor cores, mma.sync m8n8k4)
against numpy, on the shapes the elimination produces (Schur-complement
fill-ins -X[nn][k] QR^-1 X[k][pp], FMM2DTree_find_error.hpp:1961-2075) and on
ragged ones: sizes that are not multiples of the 32x32 tile or of k = 4, both
conjugate-transpose operands, and accumulation into C (beta != 0).
Tolerance: 1e-13 relative to |alpha| |A| |B| + |beta| |C| (FP64, summation
order differs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k", [(36, 36, 36), (1, 1, 1), (7, 33, 5), (64, 8, 72), (100, 37, 131), (36, 8, 0)])
@pytest.mark.parametrize("opA,opB", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_zgemm_matches_numpy(m, n, k, opA, opB):
    import aifmm_ls_b200 as A
    K = A.LSKernel(depth=2)
    rng = np.random.default_rng(m * 1000 + n * 10 + k + 7 * opA + 3 * opB)
    cn = lambda *s: rng.standard_normal(s) + 1j * rng.standard_normal(s)
    Am = cn(k, m) if opA else cn(m, k)
    Bm = cn(n, k) if opB else cn(k, n)
    C0 = cn(m, n)
    alpha, beta = -1.0 + 0.5j, 0.75 - 0.25j
    C = K.zgemm(Am, Bm, C0, alpha=alpha, beta=beta, opA=opA, opB=opB)
    oa = Am.conj().T if opA else Am
    ob = Bm.conj().T if opB else Bm
    want = alpha * (oa @ ob) + beta * C0
    scale = abs(alpha) * np.abs(oa) @ np.abs(ob) + abs(beta) * np.abs(C0)
    assert np.all(np.abs(C - want) <= 1e-13 * scale + 1e-300), np.max(np.abs(C - want) / scale)


def test_autotune_picks_a_width_and_products_stay_exact():
    import aifmm_ls_b200 as A
    K = A.LSKernel(depth=4)
    ms, widths = K.autotune()
    print("GEMM tile timings (ms) [thin 16, thin 32, wide 16, wide 32]:", ms, "chosen:", widths)
    assert np.all(ms > 0) and set(widths.tolist()) <= {16, 32}
    rng = np.random.default_rng(1)
    for m, n, k in ((36, 8, 36), (144, 144, 144), (37, 3, 70)):
        Am = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
        Bm = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
        C = K.zgemm(Am, Bm)
        scale = np.abs(Am) @ np.abs(Bm)
        assert np.all(np.abs(C - Am @ Bm) <= 1e-13 * scale)
