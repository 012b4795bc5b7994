"""Device memory of a handle stays flat over repeated solve cycles.

bench.py and a serving loop call createTree -> assemble -> solve many times on
one handle.  Every block of the previous tree (bases, ACA factors, the
elimination's blocks and factorisations, the kept copy of the assembly) must go
back to the handle's pool when the tree is rebuilt, and the assembly's
per-level workspaces are kept and reused, so after the first cycle no cycle
takes more device memory than the one before.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_repeated_cycles_keep_device_memory_flat(table_cache):
    import torch
    import aifmm_ls_b200 as A
    p, (M, near, _) = table_cache(depth=4, q_kind="gauss_aw", kappa=20.0, tol_pow=10)
    K = A.LSKernel(n_cheb=6, kappa=20.0, degree=6, depth=4, tol_pow=10, q_kind="gauss_aw", q_amp=1.5, q_width=32.0)
    K.tables_set(M, near)
    T = A.FMM2DTree(K)
    b = K.rhs_plane_wave([0.3, 1.7])
    held, free, xs = [], [], []
    for cycle in range(8):
        T.createTree()
        T.assemble()
        xs.append(T.solve(b, keep_assembly=(cycle % 2 == 1)))
        st = T.stats()
        held.append(st["pool_bytes"] + st["workspace_bytes"])
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
    print("bytes held by the handle per cycle:", held)
    assert all(h == held[1] for h in held[1:]), held
    # the device's free memory agrees (within what other allocations of this process may move)
    assert max(free[1:]) - min(free[1:]) <= 64 << 20, free
    for x in xs[1:]:
        assert np.array_equal(x, xs[0])
