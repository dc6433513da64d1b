"""Summation orders of the chi2 kernel's correlations, checked on the CPU.

The correlation helpers (gtls_b200/csrc/chi2_core.cuh) build for the host as
well; tests/csrc/chi2_orders.cu runs them on random tiles and template rows
and checks that the overlapped-rounds form of the split path gives bitwise
the sums of the per-offset form, and that the clamped and unclamped forms
agree where no read passes the tile.  These equalities are what make a
start's chi2 independent of which path and tile the kernel sends it through.
"""
import os
import subprocess
import tempfile

import pytest

from conftest import ROOT

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def test_correlation_orders_are_bitwise_equal():
    if not os.path.exists(NVCC):
        pytest.skip("nvcc not available")
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "chi2_orders")
        subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
                        "-I", os.path.join(ROOT, "gtls_b200", "csrc"), "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "csrc", "chi2_orders.cu"), "-o", exe], check=True)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout
    assert r.stdout.startswith("ok "), r.stdout
