"""aifmm_ls_b200 -- B200-native AIFMM direct solver for the 2-D Lippmann-Schwinger equation.

Python face of the C ABI in include/aifmm_b200.h (libaifmm_b200.so, built
in-tree for sm_100a).  The classes mirror the reference's surface:

* ``LSKernel`` -- ``userkernel`` (kernel.hpp:90-193): grid points, the matrix
  entries ``getMatrixEntry`` / ``getRow`` / ``getCol`` / ``getMatrix`` and the
  leaf-level quadrature tables of LS/LS_Assembly.hpp.
* ``FMM2DTree`` -- ``FMM2DTree<userkernel>`` (FMM2DTree_find_error.hpp): the
  build / assemble / eliminate / back-substitute flow and ``error_check``.

There is no CPU fallback: every call goes to the CUDA library and raises
``AifmmError`` when it is missing or fails.
"""
import ctypes
import os

import numpy as np

__all__ = ["AifmmError", "LSKernel", "FMM2DTree", "Server", "Desc", "load", "lib_path", "Q_KINDS"]

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "lib", "libaifmm_b200.so")
_lib = None

PTR_HOST, PTR_DEVICE, KEEP_ASSEMBLY, SOLVE_GRAPH = 0, 1, 2, 4
PRECISION_FP64 = 0
PRECISION_C64 = 1   # the mixed form: complex64 elimination, FP64 refinement (solve_refined)
Q_KINDS = {"gaussian160": 0, "multi_gauss": 1, "plasma": 2, "flatbump": 3, "cavity": 4, "lens": 5,
           "gauss_aw": 10, "disk": 11}


class AifmmError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("aifmm status %d: %s" % (status, msg))
        self.status = status


class Desc(ctypes.Structure):
    """aifmm_desc: the reference driver's argv (testFMM2D_find_error.cpp:44-52) plus contrast parameters."""
    _fields_ = [("n_cheb", ctypes.c_int), ("kappa", ctypes.c_double), ("degree", ctypes.c_int),
                ("L", ctypes.c_double), ("depth", ctypes.c_int), ("tol_pow", ctypes.c_int),
                ("q_kind", ctypes.c_int), ("q_amp", ctypes.c_double), ("q_width", ctypes.c_double),
                ("q_radius", ctypes.c_double)]


# every entry point of include/aifmm_b200.h with its ctypes signature
_P = ctypes.POINTER
_d = _P(ctypes.c_double)
_i = _P(ctypes.c_int)
_v = ctypes.c_void_p
SIGNATURES = {
    "aifmm_problem_create": ([_P(Desc), ctypes.c_int, _P(_v)], ctypes.c_int),
    "aifmm_problem_destroy": ([_v], ctypes.c_int),
    "aifmm_last_error": ([_v], ctypes.c_char_p),
    "aifmm_status_string": ([ctypes.c_int], ctypes.c_char_p),
    "aifmm_tables_compute": ([_v, ctypes.c_int], ctypes.c_int),
    "aifmm_tables_set": ([_v, _d, _d], ctypes.c_int),
    "aifmm_tables_get": ([_v, _d, _d], ctypes.c_int),
    "aifmm_tables_compute_noalloc": ([_v, _v, _v], ctypes.c_int),
    "aifmm_num_points": ([_v, _i], ctypes.c_int),
    "aifmm_grid_points": ([_v, _d], ctypes.c_int),
    "aifmm_rhs_plane_wave": ([_v, ctypes.c_int, _d, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_entries": ([_v, ctypes.c_long, _i, _i, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_get_matrix": ([_v, ctypes.c_int, _i, ctypes.c_int, _i, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_build_tree": ([_v], ctypes.c_int),
    "aifmm_assemble": ([_v], ctypes.c_int),
    "aifmm_factorize_solve": ([_v, ctypes.c_int, _d, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_factorize": ([_v, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "aifmm_solve": ([_v, ctypes.c_int, _d, ctypes.c_long, _d, ctypes.c_long, _v, ctypes.c_int], ctypes.c_int),
    "aifmm_find_error": ([_v, ctypes.c_int, _d, ctypes.c_long, _d, ctypes.c_long, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_zgemm": ([_v, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, _d, ctypes.c_int,
                     _d, ctypes.c_int, _d, _d, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "aifmm_trim": ([_v], ctypes.c_int),
    "aifmm_release_workspaces": ([_v], ctypes.c_int),
    "aifmm_set_factor_tolerance": ([_v, ctypes.c_int], ctypes.c_int),
    "aifmm_autotune": ([_v, _d, _i], ctypes.c_int),
    "aifmm_compressed_matvec": ([_v, ctypes.c_int, _d, ctypes.c_long, _d, ctypes.c_long, ctypes.c_int], ctypes.c_int),
    "aifmm_solve_refined": ([_v, ctypes.c_int, _d, ctypes.c_long, _d, ctypes.c_long, ctypes.c_double, ctypes.c_int,
                             _i, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_server_create": ([ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _P(_v)], ctypes.c_int),
    "aifmm_server_destroy": ([_v], ctypes.c_int),
    "aifmm_server_set_factor_workers": ([_v, ctypes.c_int], ctypes.c_int),
    "aifmm_server_set_form": ([_v, ctypes.c_int, ctypes.c_double], ctypes.c_int),
    "aifmm_server_factorize": ([_v, ctypes.c_longlong, _P(Desc), _P(ctypes.c_long)], ctypes.c_int),
    "aifmm_server_solve": ([_v, ctypes.c_longlong, ctypes.c_int, _d, _d, _P(ctypes.c_long)], ctypes.c_int),
    "aifmm_server_wait": ([_v, ctypes.c_long, ctypes.c_double, _i, _d, _i], ctypes.c_int),
    "aifmm_server_stats": ([_v, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_launch_counts_split": ([_v, _P(ctypes.c_long), _P(ctypes.c_long)], ctypes.c_int),
    "aifmm_dense_matvec": ([_v, ctypes.c_int, _d, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_total_field": ([_v, ctypes.c_int, _d, _d, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_level_ranks": ([_v, ctypes.c_int, _i, _i], ctypes.c_int),
    "aifmm_box_skeleton": ([_v, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i, ctypes.c_int, _i], ctypes.c_int),
    "aifmm_phase_times": ([_v, _d], ctypes.c_int),
    "aifmm_launch_counts": ([_v, _P(ctypes.c_long), _P(ctypes.c_long)], ctypes.c_int),
    "aifmm_get_stream": ([_v, _P(_v)], ctypes.c_int),
    "aifmm_stats": ([_v, _d, ctypes.c_int], ctypes.c_int),
    "aifmm_kernel_profile": ([_v, ctypes.c_int, ctypes.c_int], ctypes.c_int),
    "aifmm_kernel_profile_read": ([_v, ctypes.c_int, _P(ctypes.c_long), _d, _d], ctypes.c_int),
}


def lib_path():
    return _LIB


def load():
    """Load libaifmm_b200.so (building it first if the sources are newer)."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            from . import build as _b
            _b.build()
        lib = ctypes.CDLL(_LIB)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(_d)


def _ip(a):
    return a.ctypes.data_as(_i)


def _c2r(a):
    """complex128 array -> contiguous interleaved float64 view"""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    return a.view(np.float64)


class LSKernel:
    """The Lippmann-Schwinger user kernel on one GPU (kernel.hpp userkernel + LS2DTree)."""

    def __init__(self, n_cheb=6, kappa=10.0, degree=6, L=1.0, depth=5, tol_pow=8, q_kind="gaussian160",
                 q_amp=1.5, q_width=32.0, q_radius=0.5, device=0):
        lib = load()
        k = Q_KINDS[q_kind] if isinstance(q_kind, str) else int(q_kind)
        self.desc = Desc(n_cheb, float(kappa), degree, float(L), depth, tol_pow, k, float(q_amp),
                         float(q_width), float(q_radius))
        h = _v()
        st = lib.aifmm_problem_create(ctypes.byref(self.desc), device, ctypes.byref(h))
        if st != 0:
            raise AifmmError(st, lib.aifmm_status_string(st).decode())
        self.h = h
        n = ctypes.c_int()
        lib.aifmm_num_points(self.h, ctypes.byref(n))
        self.N = n.value
        self.rank = n_cheb * n_cheb
        self.nLevelsResolve = depth

    def _ck(self, st):
        if st != 0:
            raise AifmmError(st, load().aifmm_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            load().aifmm_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- precomputation (LS/LS_Assembly.hpp:270-276)
    def tables_compute(self, round6=True):
        self._ck(load().aifmm_tables_compute(self.h, 1 if round6 else 0))

    def tables_set(self, M, near):
        """M: 121 x rank complex; near: 9 x rank x rank complex (dir, i, j)."""
        Mi = _c2r(np.asfortranarray(M).ravel(order="F"))
        Ni = _c2r(np.concatenate([np.asarray(t).ravel(order="F") for t in near]))
        self._ck(load().aifmm_tables_set(self.h, _dp(Mi), _dp(Ni)))

    def tables_get(self):
        r = self.rank
        M = np.zeros(121 * r, dtype=np.complex128)
        Nt = np.zeros(9 * r * r, dtype=np.complex128)
        self._ck(load().aifmm_tables_get(self.h, _dp(M.view(np.float64)), _dp(Nt.view(np.float64))))
        return M.reshape(121, r, order="F"), np.stack([Nt[d * r * r:(d + 1) * r * r].reshape(r, r, order="F")
                                                       for d in range(9)])

    # -- userkernel surface (kernel.hpp:49-86, 102-125)
    @property
    def gridPoints(self):
        xy = np.zeros((self.N, 2))
        self._ck(load().aifmm_grid_points(self.h, _dp(xy)))
        return xy

    def rhs_plane_wave(self, thetas):
        th = np.ascontiguousarray(np.atleast_1d(thetas), dtype=np.float64)
        b = np.zeros((len(th), self.N), dtype=np.complex128)
        self._ck(load().aifmm_rhs_plane_wave(self.h, len(th), _dp(th), _dp(b.view(np.float64)), PTR_HOST))
        return b

    def entries(self, I, J):
        I = np.ascontiguousarray(I, dtype=np.int32)
        J = np.ascontiguousarray(J, dtype=np.int32)
        out = np.zeros(len(I), dtype=np.complex128)
        self._ck(load().aifmm_entries(self.h, len(I), _ip(I), _ip(J), _dp(out.view(np.float64)), PTR_HOST))
        return out

    def getMatrixEntry(self, i, j):
        return self.entries([i], [j])[0]

    def getMatrix(self, rows, cols):
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        cols = np.ascontiguousarray(cols, dtype=np.int32)
        out = np.zeros(len(rows) * len(cols), dtype=np.complex128)
        self._ck(load().aifmm_get_matrix(self.h, len(rows), _ip(rows), len(cols), _ip(cols),
                                         _dp(out.view(np.float64)), PTR_HOST))
        return out.reshape(len(rows), len(cols), order="F")

    def getRow(self, j, cols):
        return self.getMatrix([j], cols)[0]

    def getCol(self, k, rows):
        return self.getMatrix(rows, [k])[:, 0]

    def autotune(self):
        """time both GEMM tile widths on this problem's shapes; returns (timings ms, chosen widths)"""
        ms = np.zeros(4)
        tc = np.zeros(2, dtype=np.int32)
        self._ck(load().aifmm_autotune(self.h, _dp(ms), _ip(tc)))
        return ms, tc

    def zgemm(self, A, B, C=None, alpha=1.0, beta=0.0, opA=0, opB=0):
        """C = alpha op(A) op(B) + beta C with the solver's batched GEMM kernel (op 1 = conjugate transpose)."""
        A = np.asfortranarray(A, dtype=np.complex128)
        B = np.asfortranarray(B, dtype=np.complex128)
        m = A.shape[1] if opA else A.shape[0]
        k = A.shape[0] if opA else A.shape[1]
        n = B.shape[0] if opB else B.shape[1]
        C = np.zeros((m, n), np.complex128, order="F") if C is None else np.asfortranarray(C, dtype=np.complex128).copy(order="F")
        al = np.array([complex(alpha)], np.complex128).view(np.float64)
        be = np.array([complex(beta)], np.complex128).view(np.float64)
        self._ck(load().aifmm_zgemm(self.h, opA, opB, m, n, k, _dp(al), _dp(A.ravel(order="F").view(np.float64)),
                                    max(1, A.shape[0]), _dp(B.ravel(order="F").view(np.float64)), max(1, B.shape[0]),
                                    _dp(be), _dp(C.ravel(order="K").view(np.float64)), max(1, m), PTR_HOST))
        return C

    def dense_matvec(self, x):
        """y = A x with exact entries (the find_error fixture product); x: (nrhs, N)."""
        x = np.atleast_2d(np.asarray(x, dtype=np.complex128))
        xi = np.ascontiguousarray(x)
        y = np.zeros_like(xi)
        self._ck(load().aifmm_dense_matvec(self.h, x.shape[0], _dp(xi.view(np.float64)), _dp(y.view(np.float64)),
                                           PTR_HOST))
        return y

    def total_field(self, theta, phi):
        """u = u_inc + G phi (hybrid.cpp:263-281): the incident plane wave at each angle
        plus the scattered field of the solution phi, with G the findPhi = false
        operator (LS/LS_Assembly.hpp:474-541).  theta: (nrhs,), phi: (nrhs, N)."""
        th = np.ascontiguousarray(np.atleast_1d(theta), dtype=np.float64)
        phi = np.ascontiguousarray(np.atleast_2d(np.asarray(phi, dtype=np.complex128)))
        if phi.shape[0] != th.size:
            raise ValueError("one angle per right-hand side")
        u = np.zeros_like(phi)
        self._ck(load().aifmm_total_field(self.h, th.size, _dp(th), _dp(phi.view(np.float64)),
                                          _dp(u.view(np.float64)), PTR_HOST))
        return u


class FMM2DTree:
    """FMM2DTree<userkernel> (FMM2DTree_find_error.hpp) over an ``LSKernel``.

    Method names follow the reference driver (testFMM2D_find_error.cpp:127-171).
    """

    def __init__(self, K, properties=None):
        self.K = K
        self.properties = None if properties is None else np.atleast_2d(np.asarray(properties, np.complex128))
        self.x = None

    def _ck(self, st):
        self.K._ck(st)

    # createTree + assign_Tree_Interactions (F:127-1070)
    def createTree(self):
        self._ck(load().aifmm_build_tree(self.K.h))

    def assign_Tree_Interactions(self):
        pass  # part of createTree on the device side

    # assignLeafChargeLocations .. initialise_P2P_Leaf_Level (F:1072-1741)
    def assemble(self):
        self._ck(load().aifmm_assemble(self.K.h))

    # eliminate_phase_efficient + back_substitution_phase with the rhs carried (F:2407-2532)
    def solve(self, b=None, keep_assembly=False):
        b = self.properties if b is None else np.atleast_2d(np.asarray(b, np.complex128))
        if b is None:
            raise ValueError("no right-hand side")
        bi = np.ascontiguousarray(b)
        x = np.zeros_like(bi)
        flags = PTR_HOST | (KEEP_ASSEMBLY if keep_assembly else 0)
        self._ck(load().aifmm_factorize_solve(self.K.h, b.shape[0], _dp(bi.view(np.float64)),
                                              _dp(x.view(np.float64)), flags))
        self.x = x
        return x

    # eliminate_phase_efficient + the base-level factorisation, right-hand side not carried (F:2407-2485)
    def factorize(self, keep_assembly=False, precision=PRECISION_FP64):
        """eliminate_phase_efficient without a right-hand side; precision PRECISION_C64 runs
        the elimination and later solves in complex64 (refine with solve_refined)"""
        self._ck(load().aifmm_factorize(self.K.h, precision, KEEP_ASSEMBLY if keep_assembly else 0))

    def set_factor_tolerance(self, tol_pow):
        """recompression tolerance 10^-tol_pow of the next factorisations (0: the problem's)"""
        self._ck(load().aifmm_set_factor_tolerance(self.K.h, tol_pow))

    def compressed_matvec(self, x):
        """y = A_c x with the kept pre-elimination assembly (factorize(keep_assembly=True) first)"""
        x = np.ascontiguousarray(np.atleast_2d(np.asarray(x, np.complex128)))
        y = np.zeros_like(x)
        N = self.K.N
        self._ck(load().aifmm_compressed_matvec(self.K.h, x.shape[0], _dp(x.view(np.float64)), N,
                                                _dp(y.view(np.float64)), N, PTR_HOST))
        return y

    def solve_refined(self, b, rtol=1e-10, maxit=60):
        """GMRES on A_c x = b preconditioned by the kept factors; returns (x, iterations, relres)"""
        b = np.ascontiguousarray(np.atleast_2d(np.asarray(b, np.complex128)))
        x = np.zeros_like(b)
        N = self.K.N
        it = ctypes.c_int()
        rr = ctypes.c_double()
        self._ck(load().aifmm_solve_refined(self.K.h, b.shape[0], _dp(b.view(np.float64)), N, _dp(x.view(np.float64)),
                                            N, float(rtol), int(maxit), ctypes.byref(it), ctypes.byref(rr), PTR_HOST))
        self.x = x
        return x, it.value, rr.value

    # the right-hand-side half with kept factors (F:1968-2001, 2252-2293, 2453-2532)
    def solve_factored(self, b, graph=False):
        """x for right-hand sides b (nrhs, N) with the kept factors; graph=True replays the
        CUDA graph of this right-hand-side count (recorded by the first such solve)."""
        b = np.ascontiguousarray(np.atleast_2d(np.asarray(b, np.complex128)))
        x = np.zeros_like(b)
        N = self.K.N
        self._ck(load().aifmm_solve(self.K.h, b.shape[0], _dp(b.view(np.float64)), N, _dp(x.view(np.float64)), N,
                                    None, PTR_HOST | (SOLVE_GRAPH if graph else 0)))
        self.x = x
        return x

    def error_check(self, x_true):
        """relative forward error ||x - x_true|| / ||x_true|| (F:2534-2581), through the C ABI"""
        x_true = np.ascontiguousarray(np.atleast_2d(np.asarray(x_true, np.complex128)))
        x = np.ascontiguousarray(self.x)
        if x.shape != x_true.shape:
            raise ValueError("solution and reference have different shapes")
        rel = ctypes.c_double()
        N = self.K.N
        self._ck(load().aifmm_find_error(self.K.h, x.shape[0], _dp(x.view(np.float64)), N,
                                         _dp(x_true.view(np.float64)), N, ctypes.byref(rel), PTR_HOST))
        return rel.value

    def level_ranks(self, level):
        n = 4 ** level
        ri = np.zeros(n, dtype=np.int32)
        ro = np.zeros(n, dtype=np.int32)
        self._ck(load().aifmm_level_ranks(self.K.h, level, _ip(ri), _ip(ro)))
        return ri, ro

    def box_skeleton(self, level, box, which):
        cap = 8192
        out = np.zeros(cap, dtype=np.int32)
        cnt = ctypes.c_int()
        self._ck(load().aifmm_box_skeleton(self.K.h, level, box, which, _ip(out), cap, ctypes.byref(cnt)))
        return out[:cnt.value].copy()

    def phase_times(self):
        ms = np.zeros(6)
        self._ck(load().aifmm_phase_times(self.K.h, _dp(ms)))
        return ms

    def stats(self):
        v = np.zeros(15)
        self._ck(load().aifmm_stats(self.K.h, _dp(v), 15))
        keys = ["sync_ms", "syncs", "pending_ms", "elim_ms", "back_ms", "compressions", "total_ms", "launches",
                "asm_lists_ms", "asm_aca_ms", "asm_lu_ms", "asm_blocks_ms", "asm_aca_gpu_ms", "pool_bytes",
                "workspace_bytes"]
        return dict(zip(keys, v.tolist()))

    def kernel_profile(self, kind, enable=True):
        self._ck(load().aifmm_kernel_profile(self.K.h, kind, 1 if enable else 0))

    def kernel_profile_read(self, kind):
        n = ctypes.c_long()
        ms = ctypes.c_double()
        fl = ctypes.c_double()
        self._ck(load().aifmm_kernel_profile_read(self.K.h, kind, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(fl)))
        return n.value, ms.value, fl.value

    def launch_counts_split(self):
        a = ctypes.c_long()
        b = ctypes.c_long()
        self._ck(load().aifmm_launch_counts_split(self.K.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def launch_counts(self):
        a = ctypes.c_long()
        b = ctypes.c_long()
        self._ck(load().aifmm_launch_counts(self.K.h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value


class Server:
    """The serving loop of the C ABI (aifmm_server_*): factorisations kept on the
    device under keys, continuous batching of solve requests, admission by device
    memory with LRU eviction.  Requests return ids; ``wait`` returns the result."""

    STAT_KEYS = ["solve_p50_ms", "solve_p99_ms", "factorize_p50_ms", "factorize_p99_ms", "solves", "factorizations",
                 "evictions", "batches", "mean_batch_rhs", "bytes_in_use", "resident", "failed",
                 "mean_gmres_iterations", "promoted_to_fp64"]

    def __init__(self, device=0, hbm_budget_bytes=0.0, workers=2, max_batch_rhs=64, factor_workers=None,
                 precision=PRECISION_FP64, rtol=1e-8):
        """precision PRECISION_C64: the mixed form (complex64 factors, every solve refined
        by FP64 GMRES to relative residual rtol)"""
        h = _v()
        st = load().aifmm_server_create(device, float(hbm_budget_bytes), workers, max_batch_rhs, ctypes.byref(h))
        if st != 0:
            raise AifmmError(st, load().aifmm_status_string(st).decode())
        self.h = h
        self._bufs = {}
        if factor_workers is not None:
            load().aifmm_server_set_factor_workers(self.h, int(factor_workers))
        if precision != PRECISION_FP64:
            st = load().aifmm_server_set_form(self.h, int(precision), float(rtol))
            if st != 0:
                self.close()
                raise AifmmError(st, "invalid serving form")

    def close(self):
        if getattr(self, "h", None):
            load().aifmm_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def factorize(self, key, n_cheb=6, kappa=10.0, degree=6, L=1.0, depth=5, tol_pow=8, q_kind="gaussian160",
                  q_amp=1.5, q_width=32.0, q_radius=0.5):
        k = Q_KINDS[q_kind] if isinstance(q_kind, str) else int(q_kind)
        d = Desc(n_cheb, float(kappa), degree, float(L), depth, tol_pow, k, float(q_amp), float(q_width),
                 float(q_radius))
        rid = ctypes.c_long()
        st = load().aifmm_server_factorize(self.h, key, ctypes.byref(d), ctypes.byref(rid))
        if st != 0:
            raise AifmmError(st, "factorize request refused")
        return rid.value

    def solve(self, key, b):
        """b: (nrhs, N) complex; returns the request id (the solution comes from wait)."""
        b = np.ascontiguousarray(np.atleast_2d(np.asarray(b, np.complex128)))
        x = np.zeros_like(b)
        rid = ctypes.c_long()
        st = load().aifmm_server_solve(self.h, key, b.shape[0], _dp(b.view(np.float64)), _dp(x.view(np.float64)),
                                       ctypes.byref(rid))
        if st != 0:
            raise AifmmError(st, "solve request refused")
        self._bufs[rid.value] = (b, x)  # kept alive until wait()
        return rid.value

    def wait(self, rid, timeout=600.0):
        """Returns (status, latency_ms, batch_rhs, x or None)."""
        res = ctypes.c_int()
        lat = ctypes.c_double()
        br = ctypes.c_int()
        st = load().aifmm_server_wait(self.h, rid, float(timeout), ctypes.byref(res), ctypes.byref(lat),
                                      ctypes.byref(br))
        if st != 0:
            raise AifmmError(st, "request %d not finished or unknown" % rid)
        bufs = self._bufs.pop(rid, None)
        return res.value, lat.value, br.value, (bufs[1] if bufs is not None else None)

    def stats(self):
        v = np.zeros(len(self.STAT_KEYS))
        load().aifmm_server_stats(self.h, _dp(v), len(self.STAT_KEYS))
        return dict(zip(self.STAT_KEYS, v.tolist()))
