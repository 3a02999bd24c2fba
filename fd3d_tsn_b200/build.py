"""Build the in-tree shared libraries.

* ``fd3d_tsn_b200/libfd3d_gpu.so``: the product, CUDA for sm_100a behind the C ABI
  of ``include/fd3d_gpu.h``.
* ``oracle/liboracle_fd3d.so``: the CPU oracle (test infrastructure only).

Both are written in-tree so they travel with the repository snapshot.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libfd3d_gpu.so")
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "liboracle_fd3d.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: every multiply and add is its own IEEE operation, the same
# arithmetic as the reference's Fortran loops (the sweeps are HBM bound, so the
# unfused flops cost no time).
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC,-O2",
           "-Xptxas", "-O3"]


def _sources():
    srcs = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cpp")):
            srcs.append(os.path.join(CSRC, name))
    return srcs


def _deps():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for name in os.listdir(d):
            out.append(os.path.join(d, name))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_gpu(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale(LIB, _deps()):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in _sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *NVFLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC, "-x", "cu", *ARCH, *NVFLAGS, "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-ldl"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


def build_oracle(force: bool = False) -> str:
    deps = [os.path.join(ORACLE_DIR, "fd3d_oracle.cpp"), os.path.join(ROOT, "include", "fd3d_gpu.h")]
    if not force and not _stale(ORACLE_LIB, deps):
        return ORACLE_LIB
    subprocess.run(["make", "-s", "-C", ORACLE_DIR, "-B"], check=True)
    return ORACLE_LIB


def build_all(force: bool = False, verbose: bool = False):
    build_oracle(force)
    build_gpu(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
