"""The FP64 Tip5 MDS of the GPU kernels is exact: its split convolution
(tip5.cuh, t5_mds_half), built for the host, reproduces the integer circulant
product of every 32-bit half on extreme and random inputs.  The GPU tests check
the same code through whole permutations against the oracle."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "mds_exact.cu")
BIN = os.path.join(ROOT, "tests", "cpp", "_bin", "mds_exact")


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="nvcc not on PATH")
def test_mds_half_product_exact():
    os.makedirs(os.path.dirname(BIN), exist_ok=True)
    r = subprocess.run(["nvcc", "-O2", "-std=c++20", "-o", BIN, SRC], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and " 0 wrong outputs" in r.stdout, r.stdout + r.stderr
