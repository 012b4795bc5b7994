"""Build the CUDA library libaifmm_b200.so in-tree for sm_100a.

    python -m aifmm_ls_b200.build          # or aifmm_ls_b200.build.build()

The library is the product: hand-written sm_100a kernels plus the C++ host
orchestration behind the C ABI declared in include/aifmm_b200.h.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libaifmm_b200.so")
SOURCES = ["k_geom.cu", "k_tables.cu", "k_entries.cu", "k_aca.cu", "k_dense.cu", "solver.cu", "server.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _host_cxx():
    # the system g++ carries the runtime pieces nvcc's host pass expects
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def build(verbose=False, jobs=None):
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "aifmm_b200.h"))
    headers.append(os.path.join(ROOT, "include", "aifmm_fmm2dtree.hpp"))
    headers.append(os.path.join(HERE, "cli", "testFMM2D_find_error.cpp"))
    newest_dep = max(os.path.getmtime(p) for p in srcs + headers)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest_dep:
        return LIB
    flags = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", _host_cxx(),
                    "-diag-suppress", "39,550"]
    procs = []
    objs = []
    for s in srcs:
        o = os.path.join(objdir, os.path.splitext(os.path.basename(s))[0] + ".o")
        objs.append(o)
        cmd = [nvcc()] + flags + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, pr in procs:
        out, _ = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError("nvcc failed: %s\n%s" % (" ".join(cmd), out.decode(errors="replace")))
        if verbose and out:
            print(out.decode(errors="replace"))
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-ccbin", _host_cxx(), "-o", tmp] + objs + ["-lcudart", "-lpthread"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    # the reference driver's command line, on the C++ surface of include/aifmm_fmm2dtree.hpp
    cli = os.path.join(HERE, "cli", "testFMM2D_find_error.cpp")
    subprocess.check_call([_host_cxx(), "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), cli,
                           "-L", LIBDIR, "-laifmm_b200", "-Wl,-rpath,$ORIGIN", "-o",
                           os.path.join(LIBDIR, "testFMM2D_find_error")])
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
