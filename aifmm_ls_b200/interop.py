"""Exchange files with a build of the reference solver.

Two on-disk formats of the reference are read and written here:

* the precomputed tables under ``precomputations/`` (LS/LS_Assembly.hpp:1166-1228 for
  the far-field moments M, :1328-1420 for the neighbour tables).  Each file holds one
  matrix printed by Eigen's ``operator<<``: complex coefficients as ``(re,im)`` at
  the stream's default 6 significant digits, all coefficients right-aligned to the
  widest one, separated by one space, rows separated by newlines, and a final
  newline from the writer's ``endl``.  The reader of the reference
  (``ReadFromTextFile``, :1187-1214) takes the row count from the newlines and the
  column count from the number of whitespace-separated tokens.  The 6-digit print is
  what makes the reference factorise rounded tables.
* the right-hand side and solution vectors under ``rhs_x/`` (FMM2DTree_gen_rhs_x.hpp:17-37,
  testFMM2D_find_error.cpp:80-84): cereal's portable binary archive of a
  ``std::vector<double>`` -- one byte that is 1 when the data are little-endian, the
  element count as a little-endian uint64 (cereal's size type), then the doubles.
  Real and imaginary parts go to separate files.

A uniform tree of depth D uses the leaf level only: M of level D
(``M_<nCheb>_<D>``) and the nine colleague tables of level D
(``colleagueNeighborInteraction_<D>_<n>``, n in the reference's neighbour order
with 8 = the box itself), which is the layout ``LSKernel.tables_set`` takes.
Reading a reference build's files therefore reproduces its system matrix exactly;
writing produces only the leaf-level files, which a reference build would need
for every level before it could read them.
"""
import os
import struct

import numpy as np

SERIES_TERMS = 121  # 2 * 60 + 1 (LS/FarFieldInteraction.hpp: seriesLength = 60)


# ---------------------------------------------------------------- Eigen text
def _g6(v):
    """A double as an iostream with default flags and precision 6 prints it (%g)."""
    return "%.6g" % v


def format_eigen(A):
    """The text Eigen's ``operator<<`` produces for matrix A (without the final
    newline the reference's writer adds with ``endl``)."""
    A = np.atleast_2d(np.asarray(A))
    cplx = np.iscomplexobj(A)
    cells = [["(%s,%s)" % (_g6(v.real), _g6(v.imag)) if cplx else _g6(v) for v in row] for row in A]
    width = max((len(c) for row in cells for c in row), default=0)
    return "\n".join(" ".join(c.rjust(width) for c in row) for row in cells)


def write_eigen_text(path, A):
    with open(path, "w") as f:
        f.write(format_eigen(A) + "\n")


def _token(t):
    if t.startswith("("):
        re_, im_ = t[1:-1].split(",")
        return complex(float(re_), float(im_))
    return complex(float(t), 0.0)


def read_eigen_text(path):
    """A matrix file as the reference reads it: rows = newline count, columns =
    tokens / rows; raises ValueError where the reference would exit."""
    with open(path) as f:
        text = f.read()
    rows = text.count("\n")
    tokens = text.split()
    if rows == 0 or len(tokens) % rows != 0:
        raise ValueError("%s cannot form a matrix" % path)
    cols = len(tokens) // rows
    return np.array([_token(t) for t in tokens], dtype=np.complex128).reshape(rows, cols)


# ---------------------------------------------------------------- tables
def _table_dirs(root, n_cheb, kappa, degree):
    tag = "%d_%d_%d" % (n_cheb, int(kappa), degree)
    pre = os.path.join(root, "precomputations")
    return os.path.join(pre, "M", "M_" + tag), os.path.join(pre, "Neighbor", "Neighbor_" + tag)


def read_reference_tables(root, n_cheb, kappa, degree, depth):
    """The leaf-level tables a reference build wrote under ``root``: M
    (121 x nCheb^2) and near (9 x nCheb^2 x nCheb^2), ready for ``LSKernel.tables_set``."""
    mdir, ndir = _table_dirs(root, n_cheb, kappa, degree)
    rank = n_cheb * n_cheb
    M = read_eigen_text(os.path.join(mdir, "M_%d_%d" % (n_cheb, depth)))
    if M.shape != (SERIES_TERMS, rank):
        raise ValueError("M table has shape %s, expected %s" % (M.shape, (SERIES_TERMS, rank)))
    near = []
    for n in range(9):
        t = read_eigen_text(os.path.join(ndir, "colleagueNeighborInteraction_%d_%d" % (depth, n)))
        if t.shape != (rank, rank):
            raise ValueError("colleague table %d has shape %s" % (n, t.shape))
        near.append(t)
    return M, np.stack(near)


def write_reference_tables(root, n_cheb, kappa, degree, depth, M, near):
    """Write the leaf-level tables in the reference's layout and text format."""
    mdir, ndir = _table_dirs(root, n_cheb, kappa, degree)
    os.makedirs(mdir, exist_ok=True)
    os.makedirs(ndir, exist_ok=True)
    write_eigen_text(os.path.join(mdir, "M_%d_%d" % (n_cheb, depth)), M)
    for n in range(9):
        write_eigen_text(os.path.join(ndir, "colleagueNeighborInteraction_%d_%d" % (depth, n)), near[n])


# ---------------------------------------------------------------- cereal vectors
def write_cereal_vector(path, values):
    """A std::vector<double> in cereal's portable binary archive (little-endian)."""
    v = np.ascontiguousarray(values, dtype="<f8").ravel()
    with open(path, "wb") as f:
        f.write(struct.pack("<BQ", 1, v.size))
        f.write(v.tobytes())


def read_cereal_vector(path):
    with open(path, "rb") as f:
        data = f.read()
    if len(data) < 9:
        raise ValueError("%s: not a cereal portable binary vector" % path)
    little = data[0] == 1
    (n,) = struct.unpack("<Q" if little else ">Q", data[1:9])
    if len(data) != 9 + 8 * n:
        raise ValueError("%s: %d bytes for %d doubles" % (path, len(data), n))
    return np.frombuffer(data[9:], dtype="<f8" if little else ">f8").astype(np.float64)


def _rhs_x_name(root, kind, qchoice, kappa, N):
    return os.path.join(root, "rhs_x", "%s_%%s_%d_%d_%d.bin" % (kind, int(qchoice), int(kappa), int(N)))


def write_rhs_x(root, kind, qchoice, kappa, values):
    """Write a complex vector as the reference's ``rhs_x/<kind>_real|imag_<Q>_<kappa>_<N>.bin``
    pair (kind "rhs" or "x")."""
    v = np.asarray(values, dtype=np.complex128).ravel()
    os.makedirs(os.path.join(root, "rhs_x"), exist_ok=True)
    name = _rhs_x_name(root, kind, qchoice, kappa, v.size)
    write_cereal_vector(name % "real", v.real)
    write_cereal_vector(name % "imag", v.imag)


def read_rhs_x(root, kind, qchoice, kappa, N):
    name = _rhs_x_name(root, kind, qchoice, kappa, N)
    re_, im_ = read_cereal_vector(name % "real"), read_cereal_vector(name % "imag")
    if re_.size != N or im_.size != N:
        raise ValueError("%s: %d / %d values, expected %d" % (name, re_.size, im_.size, N))
    return re_ + 1j * im_
