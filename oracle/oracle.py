"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle restates the reference AIFMM-LS solver on the CPU.  It is the
checker for the CUDA product path: only the tests, the smoke check and the
CPU-baseline leg of the benchmark load it.  See aifmm_oracle.cpp for the
reference files each routine follows.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "liboracle.so")
_lib = None

Q_KINDS = {"gaussian160": 0, "multi_gauss": 1, "plasma": 2, "flatbump": 3,
           "cavity": 4, "lens": 5, "gauss_aw": 10, "disk": 11}


class OrcParams(ctypes.Structure):
    _fields_ = [("n_cheb", ctypes.c_int), ("kappa", ctypes.c_double),
                ("degree", ctypes.c_int), ("L", ctypes.c_double),
                ("depth", ctypes.c_int), ("tol_pow", ctypes.c_int),
                ("q_kind", ctypes.c_int), ("q_amp", ctypes.c_double),
                ("q_width", ctypes.c_double), ("q_radius", ctypes.c_double)]


def build():
    """Compile the oracle library (make -C oracle)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        P = ctypes.POINTER
        d = P(ctypes.c_double)
        i = P(ctypes.c_int)
        v = ctypes.c_void_p
        _lib.orc_gauss_legendre.argtypes = [ctypes.c_int, d, d]
        _lib.orc_bessel_jy.argtypes = [ctypes.c_int, ctypes.c_double, d, d]
        _lib.orc_tables.argtypes = [P(OrcParams), ctypes.c_int, d, d, d]
        _lib.orc_create.argtypes = [P(OrcParams), d, d]
        _lib.orc_create.restype = v
        _lib.orc_destroy.argtypes = [v]
        _lib.orc_num_points.argtypes = [v]
        _lib.orc_grid_points.argtypes = [v, d]
        _lib.orc_contrast.argtypes = [v, d]
        _lib.orc_rhs_plane_wave.argtypes = [v, ctypes.c_int, d, d]
        _lib.orc_entries.argtypes = [v, ctypes.c_long, i, i, d]
        _lib.orc_dense_matvec.argtypes = [v, ctypes.c_int, d, d]
        _lib.orc_total_field.argtypes = [v, ctypes.c_int, d, d, d]
        _lib.orc_solve.argtypes = [v, ctypes.c_int, d, d, d]
        _lib.orc_solve_again.argtypes = [v, ctypes.c_int, d, d]
        _lib.orc_set_variant.argtypes = [v, ctypes.c_int]
        _lib.orc_set_schedule.argtypes = [v, ctypes.c_int]
        _lib.orc_compressions.argtypes = [v]
        _lib.orc_compressions.restype = ctypes.c_long
        _lib.orc_set_perturbation.argtypes = [v, ctypes.c_double]
        _lib.orc_compressed_dense.argtypes = [P(OrcParams), d, d, d]
        _lib.orc_level_ranks.argtypes = [v, ctypes.c_int, i, i]
        _lib.orc_box_lists.argtypes = [v, ctypes.c_int, ctypes.c_int, i]
        _lib.orc_box_skeleton.argtypes = [v, ctypes.c_int, ctypes.c_int, ctypes.c_int, i, ctypes.c_int]
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def params(n_cheb=6, kappa=10.0, degree=6, L=1.0, depth=5, tol_pow=8,
           q_kind="gaussian160", q_amp=1.5, q_width=32.0, q_radius=0.5):
    k = Q_KINDS[q_kind] if isinstance(q_kind, str) else int(q_kind)
    return OrcParams(n_cheb, kappa, degree, L, depth, tol_pow, k, q_amp, q_width, q_radius)


def gauss_legendre(n):
    x = np.zeros(n)
    w = np.zeros(n)
    lib().orc_gauss_legendre(n, _dp(x), _dp(w))
    return x, w


def bessel_jy(nmax, x):
    J = np.zeros(nmax + 1)
    Y = np.zeros(nmax + 1)
    lib().orc_bessel_jy(nmax, float(x), _dp(J), _dp(Y))
    return J, Y


def tables(p, round6=True):
    rank = p.n_cheb * p.n_cheb
    nb = p.degree * (p.degree + 1) // 2
    M = np.zeros((rank, 121, 2))          # column-major 121 x rank
    near = np.zeros((9, rank, rank, 2))   # per table column-major rank x rank
    qp = np.zeros((rank, nb))
    lib().orc_tables(ctypes.byref(p), 1 if round6 else 0, _dp(M), _dp(near), _dp(qp))
    Mc = (M[..., 0] + 1j * M[..., 1]).T                       # 121 x rank
    nearc = np.transpose(near[..., 0] + 1j * near[..., 1], (0, 2, 1))  # dir, i, j
    return Mc, nearc, qp.T


class Problem:
    """One oracle problem instance built from explicit leaf tables."""

    def __init__(self, p, M, near):
        self.p = p
        Mi = np.ascontiguousarray(np.stack([M.T.real, M.T.imag], -1))
        Ni = np.ascontiguousarray(np.stack([np.transpose(near, (0, 2, 1)).real,
                                            np.transpose(near, (0, 2, 1)).imag], -1))
        self._keep = (Mi, Ni)
        self.h = lib().orc_create(ctypes.byref(p), _dp(Mi), _dp(Ni))
        self.N = lib().orc_num_points(self.h)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_variant(self, full_compress):
        lib().orc_set_variant(self.h, 1 if full_compress else 0)

    def set_schedule(self, flags):
        """Test-only reorderings used by the GPU solver: 1 waves in the back
        substitution, 2 the P2P[k][k] factorisation before the step's
        recompressions, 4 the L2M_f factorisation before the x-phase fill-ins."""
        lib().orc_set_schedule(self.h, int(flags))

    def compressions(self):
        return int(lib().orc_compressions(self.h))

    def set_perturbation(self, rel):
        lib().orc_set_perturbation(self.h, float(rel))

    def compressed_dense(self):
        """Dense matrix implied by the pre-elimination compressed representation."""
        N = self.N
        out = np.zeros((N, N, 2), order="F")
        Mi, Ni = self._keep
        lib().orc_compressed_dense(ctypes.byref(self.p), _dp(Mi), _dp(Ni), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        flat = np.frombuffer(out.tobytes(order="F"), dtype=np.float64)
        c = flat[0::2] + 1j * flat[1::2]
        return c.reshape(N, N, order="F")

    def grid_points(self):
        xy = np.zeros((self.N, 2))
        lib().orc_grid_points(self.h, _dp(xy))
        return xy

    def contrast(self):
        q = np.zeros(self.N)
        lib().orc_contrast(self.h, _dp(q))
        return q

    def rhs_plane_wave(self, thetas):
        th = np.ascontiguousarray(np.asarray(thetas, dtype=np.float64))
        b = np.zeros((len(th), self.N, 2))
        lib().orc_rhs_plane_wave(self.h, len(th), _dp(th), _dp(b))
        return b[..., 0] + 1j * b[..., 1]

    def entries(self, I, J):
        I = np.ascontiguousarray(I, dtype=np.int32)
        J = np.ascontiguousarray(J, dtype=np.int32)
        out = np.zeros((len(I), 2))
        lib().orc_entries(self.h, len(I), _ip(I), _ip(J), _dp(out))
        return out[:, 0] + 1j * out[:, 1]

    def dense(self):
        N = self.N
        I, J = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
        return self.entries(I.ravel(), J.ravel()).reshape(N, N)

    def dense_matvec(self, x):
        x = np.atleast_2d(x)
        xi = np.ascontiguousarray(np.stack([x.real, x.imag], -1))
        y = np.zeros_like(xi)
        lib().orc_dense_matvec(self.h, x.shape[0], _dp(xi), _dp(y))
        return y[..., 0] + 1j * y[..., 1]

    def total_field(self, thetas, phi):
        """u = u_inc + G phi (hybrid.cpp:263-281), phi: (nrhs, N) complex."""
        th = np.ascontiguousarray(np.atleast_1d(thetas), dtype=np.float64)
        phi = np.atleast_2d(phi)
        pi = np.ascontiguousarray(np.stack([phi.real, phi.imag], -1))
        u = np.zeros_like(pi)
        lib().orc_total_field(self.h, len(th), _dp(th), _dp(pi), _dp(u))
        return u[..., 0] + 1j * u[..., 1]

    def solve(self, b):
        """b: (nrhs, N) complex.  Returns x (nrhs, N) and phase times."""
        b = np.atleast_2d(b)
        bi = np.ascontiguousarray(np.stack([b.real, b.imag], -1))
        x = np.zeros_like(bi)
        t = np.zeros(4)
        lib().orc_solve(self.h, b.shape[0], _dp(bi), _dp(x), _dp(t))
        return x[..., 0] + 1j * x[..., 1], t

    def solve_again(self, b):
        """b: (nrhs, N) complex, against the factors of the last solve()."""
        b = np.atleast_2d(b)
        bi = np.ascontiguousarray(np.stack([b.real, b.imag], -1))
        x = np.zeros_like(bi)
        lib().orc_solve_again(self.h, b.shape[0], _dp(bi), _dp(x))
        return x[..., 0] + 1j * x[..., 1]

    def level_ranks(self, level):
        n = 4 ** level
        ri = np.zeros(n, dtype=np.int32)
        ro = np.zeros(n, dtype=np.int32)
        lib().orc_level_ranks(self.h, level, _ip(ri), _ip(ro))
        return ri, ro

    def box_lists(self, level, box):
        out = np.zeros(48, dtype=np.int32)
        lib().orc_box_lists(self.h, level, box, _ip(out))
        return out[:8], out[8:24], out[24:48]

    def box_skeleton(self, level, box, which):
        cap = 4096
        out = np.zeros(cap, dtype=np.int32)
        n = lib().orc_box_skeleton(self.h, level, box, which, _ip(out), cap)
        return out[:n].copy()
