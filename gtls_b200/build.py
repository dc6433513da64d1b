"""Build the CUDA library ``gtls_b200/libgtls_b200.so`` for sm_100a.

Run as ``python -m gtls_b200.build``.  Each ``csrc/*.cu`` is compiled with
nvcc for ``compute_100a``/``sm_100a`` and the objects are linked into one
shared library in the package directory (in-tree, so it ships with the
sources).  Rebuilds only when a source or header is newer than the library.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libgtls_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + os.path.join(ROOT, "include")]


def _sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _deps():
    return _sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(ROOT, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for src in _sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
