"""The reference's on-disk formats (precomputations/ tables, rhs_x/ vectors)."""
import os
import struct

import numpy as np


def test_eigen_text_layout():
    from aifmm_ls_b200 import interop
    A = np.array([[1 + 2j, -0.5], [1e-7, 3.14159265]])
    # widest coefficient "(3.14159,0)" (11 characters); every coefficient is
    # right-aligned to it, one space between coefficients, newline between rows
    assert interop.format_eigen(A) == "      (1,2)    (-0.5,0)\n  (1e-07,0) (3.14159,0)"


def test_table_files_reproduce_the_reference_rounding(oracle_mod, tmp_path):
    """Writing unrounded tables in the reference's format and reading them back is
    the 6-digit round trip the reference's tables go through (LS_Assembly.hpp:1166-1228,
    1328-1459); it matches the oracle's emulation of it bit for bit."""
    from aifmm_ls_b200 import interop
    p = oracle_mod.params(depth=3, kappa=10.0)
    M0, N0, _ = oracle_mod.tables(p, round6=False)
    M6, N6, _ = oracle_mod.tables(p, round6=True)
    interop.write_reference_tables(str(tmp_path), p.n_cheb, p.kappa, p.degree, p.depth, M0, N0)
    assert os.path.exists(tmp_path / "precomputations" / "M" / "M_6_10_6" / "M_6_3")
    assert os.path.exists(tmp_path / "precomputations" / "Neighbor" / "Neighbor_6_10_6" / "colleagueNeighborInteraction_3_8")
    M, N = interop.read_reference_tables(str(tmp_path), p.n_cheb, p.kappa, p.degree, p.depth)
    assert M.shape == (121, 36) and N.shape == (9, 36, 36)
    assert np.array_equal(M, M6)
    assert np.array_equal(N, N6)


def test_cereal_vector_layout(tmp_path):
    from aifmm_ls_b200 import interop
    path = str(tmp_path / "v.bin")
    interop.write_cereal_vector(path, [1.5, -2.0])
    with open(path, "rb") as f:
        data = f.read()
    assert data == b"\x01" + struct.pack("<Q", 2) + struct.pack("<2d", 1.5, -2.0)
    assert np.array_equal(interop.read_cereal_vector(path), [1.5, -2.0])
    # an archive written on a big-endian machine carries the flag 0
    big = str(tmp_path / "b.bin")
    with open(big, "wb") as f:
        f.write(b"\x00" + struct.pack(">Q", 3) + struct.pack(">3d", 1.0, 2.5, -7.0))
    assert np.array_equal(interop.read_cereal_vector(big), [1.0, 2.5, -7.0])


def test_rhs_x_files(tmp_path):
    from aifmm_ls_b200 import interop
    rng = np.random.default_rng(3)
    v = rng.standard_normal(576) + 1j * rng.standard_normal(576)
    interop.write_rhs_x(str(tmp_path), "rhs", 0, 10.0, v)
    assert os.path.exists(tmp_path / "rhs_x" / "rhs_real_0_10_576.bin")
    assert os.path.exists(tmp_path / "rhs_x" / "rhs_imag_0_10_576.bin")
    assert np.array_equal(interop.read_rhs_x(str(tmp_path), "rhs", 0, 10.0, 576), v)


def test_cpp_reader_matches_python_reader(oracle_mod, tmp_path):
    """include/aifmm_fmm2dtree.hpp reads the reference's table files for C++ users
    (userkernel::readTables); its values and layout equal the Python reader's."""
    import shutil
    import subprocess
    from aifmm_ls_b200 import interop
    cxx = shutil.which("g++")
    if cxx is None:
        import pytest
        pytest.skip("no host C++ compiler")
    p = oracle_mod.params(depth=3, kappa=10.0)
    M0, N0, _ = oracle_mod.tables(p, round6=False)
    interop.write_reference_tables(str(tmp_path), p.n_cheb, p.kappa, p.degree, p.depth, M0, N0)
    src = tmp_path / "read.cpp"
    src.write_text(r'''
#include <cstdio>
#include "aifmm_fmm2dtree.hpp"
int main(int, char** argv) {
  std::vector<double> M, nt;
  aifmm::read_reference_tables(argv[1], 6, 10.0, 6, 3, M, nt);
  FILE* f = std::fopen(argv[2], "wb");
  std::fwrite(M.data(), sizeof(double), M.size(), f);
  std::fwrite(nt.data(), sizeof(double), nt.size(), f);
  std::fclose(f);
  return 0;
}
''')
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = tmp_path / "read"
    subprocess.check_call([cxx, "-std=c++17", "-O1", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)])
    out = tmp_path / "tables.bin"
    subprocess.check_call([str(exe), str(tmp_path), str(out)])
    raw = np.fromfile(str(out), dtype=np.float64).view(np.complex128)
    M, N = interop.read_reference_tables(str(tmp_path), p.n_cheb, p.kappa, p.degree, p.depth)
    r = p.n_cheb ** 2
    assert np.array_equal(raw[:121 * r], M.ravel(order="F"))
    assert np.array_equal(raw[121 * r:], np.concatenate([t.ravel(order="F") for t in N]))
