"""CPU checks of the product library: it builds for sm_100a, loads, exports every
entry point declared in include/aifmm_b200.h, and refuses to run without a GPU
(there is no CPU fallback)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    src = open(os.path.join(ROOT, "include", "aifmm_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(aifmm_\w+)\s*\(", src, re.M)))


def test_header_declares_the_abi():
    syms = _declared_symbols()
    assert "aifmm_problem_create" in syms and "aifmm_factorize_solve" in syms
    assert len(syms) >= 20


def test_library_builds_and_exports_every_declared_symbol():
    import aifmm_ls_b200 as A
    from aifmm_ls_b200 import build
    path = build.build()
    assert os.path.exists(path)
    lib = ctypes.CDLL(path)
    missing = [s for s in _declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(_declared_symbols()) == set(A.SIGNATURES)


def test_status_strings():
    import aifmm_ls_b200 as A
    lib = A.load()
    for s in range(7):
        assert lib.aifmm_status_string(s)


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import aifmm_ls_b200 as A
    with pytest.raises(A.AifmmError) as e:
        A.LSKernel(depth=2)
    assert e.value.status in (2, 6)  # CUDA error / no device


def test_invalid_description_is_rejected():
    import aifmm_ls_b200 as A
    lib = A.load()
    d = A.Desc(6, 10.0, 6, 1.0, 1, 8, 0, 1.5, 32.0, 0.5)  # depth 1 is not a valid AIFMM tree
    h = ctypes.c_void_p()
    st = lib.aifmm_problem_create(ctypes.byref(d), 0, ctypes.byref(h))
    assert st != 0


def test_server_refuses_to_start_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import aifmm_ls_b200 as A
    with pytest.raises(A.AifmmError) as e:
        A.Server(workers=1)
    assert e.value.status == 6  # AIFMM_ERR_NODEVICE


def test_entry_points_reject_null_handles():
    """Argument checks that need no device: every handle-taking entry point of the
    factor / solve / mixed-form / serving surface answers AIFMM_ERR_ARG (1) for a
    NULL handle instead of touching it."""
    import aifmm_ls_b200 as A
    lib = A.load()
    null = None
    assert lib.aifmm_factorize(null, A.PRECISION_C64, 0) == 1
    assert lib.aifmm_factorize(null, 7, 0) == 1
    assert lib.aifmm_release_workspaces(null) == 1
    assert lib.aifmm_trim(null) == 1
    assert lib.aifmm_set_factor_tolerance(null, 6) == 1
    assert lib.aifmm_server_set_form(null, A.PRECISION_C64, 1e-8) == 1
    assert lib.aifmm_server_set_factor_workers(null, 2) == 1


def test_cpp_shim_compiles_with_the_mixed_form(tmp_path):
    """The C++ drop-in surface (include/aifmm_fmm2dtree.hpp) with the factor
    precision and the refinement compiles against the C ABI header."""
    import shutil
    import subprocess
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "shim.cpp"
    src.write_text(
        '#include "aifmm_fmm2dtree.hpp"\\n'
        "int main() {\\n"
        "  aifmm::FMM2DTree<aifmm::userkernel>* T = nullptr;\\n"
        "  if (T) {\\n"
        "    T->eliminate_phase_efficient(AIFMM_PRECISION_C64, true);\\n"
        "    T->back_substitution_phase();\\n"
        "    double r = 0;\\n"
        "    T->refine(1e-10, 60, &r);\\n"
        "  }\\n"
        "  return 0;\\n"
        "}\\n")
    out = subprocess.run([cxx, "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "include"), str(src)],
                         capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
