"""In-tree build of the native parts (no JIT cache: the .so files travel with the tree).

* ``libsns_b200.so``      CUDA kernels + C ABI (nvcc, sm_100a only)
* ``libsns_b200_check.so`` the same with -DSNS_BOUNDS_CHECK: every index of the TMA /
                          tensor-memory pass kernels checked against its buffer (tests only)
* ``libspectral_b200.so`` C++ drop-in classes (B200Fft3D, SpectralNavierStokes,
                          TaylorGreenSolver, run_taylor_green) over the C ABI
* ``bin/taylor_green_b200`` the reference's CLI (same flags and CSV)
* ``bin/spectral_ns_tests_b200`` the reference's C++ tests compiled against B200Fft3D

Rebuilds only what is older than its sources.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
INC = os.path.join(ROOT, "include")
BIN = os.path.join(PKG, "bin")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(os.path.realpath(NVCC)))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-Xptxas", "-O3"]

LIB = os.path.join(PKG, "libsns_b200.so")
CHECK_LIB = os.path.join(PKG, "libsns_b200_check.so")
HOSTLIB = os.path.join(PKG, "libspectral_b200.so")


def _sources(d, exts):
    if not os.path.isdir(d):
        return []
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(exts))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)


def build_cuda(verbose=False, ptxas_verbose=False, check=False):
    lib = CHECK_LIB if check else LIB
    cus = _sources(CSRC, (".cu",))
    deps = cus + _sources(CSRC, (".cuh", ".h")) + _sources(INC, (".h",))
    if not _stale(lib, deps) and not ptxas_verbose:
        return lib
    objdir = os.path.join(PKG, "_build", "check" if check else "")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    defs = ["-DSNS_BOUNDS_CHECK"] if check else []
    for cu in cus:
        obj = os.path.join(objdir, os.path.basename(cu) + ".o")
        extra = ["-Xptxas", "-v"] if ptxas_verbose else []
        if _stale(obj, [cu] + _sources(CSRC, (".cuh", ".h")) + _sources(INC, (".h",))) or ptxas_verbose:
            _run([NVCC, *ARCH, *NVFLAGS, *defs, *extra, "-I", INC, "-c", cu, "-o", obj], verbose or ptxas_verbose)
        objs.append(obj)
    _run([NVCC, *ARCH, "-shared", "-o", lib, *objs, "-lcudart"], verbose)
    return lib


def build_host(verbose=False):
    """C++ drop-in classes and executables (g++, linked against libsns_b200.so)."""
    srcs = _sources(HOST, (".cpp",))
    if not srcs:
        return None
    hdrs = _sources(INC, (".h", ".hpp")) + _sources(os.path.join(INC, "spectral"), (".hpp", ".h"))
    lib_srcs = [s for s in srcs if not os.path.basename(s).startswith(("main_", "test_"))]
    cxx = os.environ.get("CXX", "g++")
    flags = ["-O2", "-std=c++17", "-fPIC", "-Wall", "-Wextra", "-I", INC]
    rpath = "-Wl,-rpath,$ORIGIN"
    if _stale(HOSTLIB, lib_srcs + hdrs + [LIB]):
        _run([cxx, *flags, "-shared", "-o", HOSTLIB, *lib_srcs, "-L", PKG, "-lsns_b200", rpath], verbose)
    os.makedirs(BIN, exist_ok=True)
    for s in srcs:
        b = os.path.basename(s)
        if not b.startswith(("main_", "test_")):
            continue
        exe = os.path.join(BIN, b.split("_", 1)[1].rsplit(".", 1)[0] + "_b200")
        if _stale(exe, [s, HOSTLIB] + hdrs):
            _run([cxx, *flags, "-o", exe, s, "-L", PKG, "-lspectral_b200", "-lsns_b200",
                  "-Wl,-rpath,$ORIGIN/.."], verbose)
    return HOSTLIB


def build(verbose=False):
    build_cuda(verbose)
    build_host(verbose)
    build_cuda(verbose, check=True)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    if "--ptxas" in sys.argv:
        build_cuda(verbose=True, ptxas_verbose=True)
