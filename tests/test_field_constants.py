"""Constants the CUDA kernels hard-code, checked against their definitions:
the in-register NTT networks apply their twiddles as powers of two from the
forward 32-point root w_32 = 7^((p-1)/32) = 2^78 (ntt.cu, GL_W32_LOG2), with
2 of multiplicative order 192 (2^96 = -1)."""
import re
import os

from conftest import ROOT

P = 2**64 - 2**32 + 1


def test_w32_is_a_power_of_two():
    src = open(os.path.join(ROOT, "triton-vm-prover_b200", "csrc", "ntt.cu")).read()
    e = int(re.search(r"constexpr int GL_W32_LOG2 = (\d+);", src).group(1))
    w32 = pow(7, (P - 1) // 32, P)
    assert pow(2, e, P) == w32
    assert pow(2, 96, P) == P - 1 and pow(2, 192, P) == 1
    # every root of order 2^m <= 32 used by the networks, forward and inverse
    for m in range(1, 6):
        w = pow(7, (P - 1) >> m, P)
        assert pow(2, e * (1 << (5 - m)) % 192, P) == w
        assert pow(2, (192 - e * (1 << (5 - m)) % 192) % 192, P) == pow(w, P - 2, P)
