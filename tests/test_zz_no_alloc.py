"""The allocation-free table entry point (aifmm_tables_compute_noalloc).

Some callers cannot let a library call cudaMalloc: applications that reserve
the GPU's memory up front and hand it out through their own allocator, and
latency-sensitive loops that cannot accept the device synchronisation that
cudaMalloc / cudaFree may cause.  This entry point keeps its scratch in a fixed
1 MiB device array inside the library; the caller passes the output buffers.
It must produce the same tables as aifmm_tables_compute(p, round6=0), call
after call (the array keeps the previous call's contents), and reject problems
whose scratch exceeds the array.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(K, M_dev, N_dev):
    import aifmm_ls_b200 as A
    return A.load().aifmm_tables_compute_noalloc(K.h, ctypes.c_void_p(M_dev.data_ptr()),
                                                 ctypes.c_void_p(N_dev.data_ptr()))


@pytest.mark.parametrize("n_cheb,kappa,depth", [(6, 10.0, 3), (8, 40.0, 4)])
def test_noalloc_tables_match_allocating_entry_point(n_cheb, kappa, depth):
    import torch
    import aifmm_ls_b200 as A
    K = A.LSKernel(n_cheb=n_cheb, kappa=kappa, degree=6, depth=depth)
    K.tables_compute(round6=False)
    M_ref, N_ref = K.tables_get()
    rank = n_cheb * n_cheb
    # the caller owns the outputs; the entry point itself allocates nothing
    M_dev = torch.empty(121 * rank * 2, dtype=torch.float64, device="cuda")
    N_dev = torch.empty(9 * rank * rank * 2, dtype=torch.float64, device="cuda")
    for _ in range(2):  # two calls in a row: the shared scratch must not carry state
        M_dev.fill_(float("nan"))
        N_dev.fill_(float("nan"))
        torch.cuda.synchronize()
        assert _noalloc(K, M_dev, N_dev) == 0
        M = M_dev.cpu().numpy().view(np.complex128).reshape(121, rank, order="F")
        Nt = N_dev.cpu().numpy().view(np.complex128)
        Nt = np.stack([Nt[d * rank * rank:(d + 1) * rank * rank].reshape(rank, rank, order="F") for d in range(9)])
        # same kernels, same order of operations: agreement to the last bit (tolerance 0)
        assert np.max(np.abs(M - M_ref)) <= 0.0
        assert np.max(np.abs(Nt - N_ref)) <= 0.0


def test_noalloc_rejects_problems_larger_than_its_scratch():
    import torch
    import aifmm_ls_b200 as A
    K = A.LSKernel(n_cheb=16, kappa=10.0, degree=10, depth=2)  # V alone is 9*256*55*16 B ~ 2 MB > 1 MiB
    rank = 256
    M_dev = torch.empty(121 * rank * 2, dtype=torch.float64, device="cuda")
    N_dev = torch.empty(9 * rank * rank * 2, dtype=torch.float64, device="cuda")
    assert _noalloc(K, M_dev, N_dev) == 1  # AIFMM_ERR_ARG
