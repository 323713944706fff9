"""NTT::evaluate_on_coset on the GPU (tvmc_evaluate_on_coset_gpu / _host) vs
the oracle, bit-exact: coefficient vectors of 2^10 .. 2^20 evaluated on
domains 1, 2, 4 and 8 times longer, several offsets, batched columns, and the
reference's truncation when there are more coefficients than domain points
(src/ntt/ntt.cpp:94-117)."""
import numpy as np
import pytest

from conftest import P, dev_empty, from_dev, rand_u64, to_dev

pytestmark = pytest.mark.gpu


def _coset_gpu(tv, coeffs, L, offset):
    cols, n = coeffs.shape
    d_in = to_dev(coeffs) if n else dev_empty(1)
    d_out = dev_empty(cols * L)
    lib = tv.lib()
    assert lib.tvmc_evaluate_on_coset_gpu(d_in.data_ptr(), n, cols, d_out.data_ptr(), L, offset, None) == 0, \
        lib.tvmc_last_error()
    return from_dev(d_out).reshape(cols, L)


@pytest.mark.parametrize("log_n", [10, 14, 17, 20])
@pytest.mark.parametrize("ratio", [1, 2, 4, 8])
def test_evaluate_on_coset_sizes(tv, oracle, log_n, ratio):
    n, L = 1 << log_n, (1 << log_n) * ratio
    cols = 2 if log_n <= 17 else 1
    c = rand_u64(log_n * 16 + ratio, (cols, n))
    got = _coset_gpu(tv, c, L, 7)
    for k in range(cols):
        assert (got[k] == oracle.evaluate_on_coset(c[k], L, 7)).all(), k


@pytest.mark.parametrize("offset", [1, 3, P - 1, 0x1234567890ABCDEF])
def test_evaluate_on_coset_offsets(tv, oracle, offset):
    c = rand_u64(offset % 1000, (3, 1 << 12))
    got = _coset_gpu(tv, c, 1 << 14, offset)
    for k in range(3):
        assert (got[k] == oracle.evaluate_on_coset(c[k], 1 << 14, offset)).all()


@pytest.mark.parametrize("n,L", [(0, 16), (1, 1), (3, 8), (100, 32), (5000, 1 << 12), (1 << 13, 1 << 11)])
def test_evaluate_on_coset_ragged_and_truncated(tv, oracle, n, L):
    c = rand_u64(n + 7 * L, (2, n), hi=2**64 - 1)  # inputs above p are read mod p
    got = _coset_gpu(tv, c, L, 7)
    for k in range(2):
        assert (got[k] == oracle.evaluate_on_coset(c[k], L, 7)).all(), (n, L)


def test_evaluate_on_coset_host_form(tv, oracle):
    c = rand_u64(55, (4, 1 << 9))
    out = np.empty((4, 1 << 11), np.uint64)
    lib = tv.lib()
    assert lib.tvmc_evaluate_on_coset_host(c.ctypes.data_as(tv._u64p), 1 << 9, 4, out.ctypes.data_as(tv._u64p),
                                           1 << 11, 7) == 0, lib.tvmc_last_error()
    for k in range(4):
        assert (out[k] == oracle.evaluate_on_coset(c[k], 1 << 11, 7)).all()


def test_evaluate_on_coset_rejects_bad_domains(tv):
    lib = tv.lib()
    d = dev_empty(8)
    assert lib.tvmc_evaluate_on_coset_gpu(d.data_ptr(), 4, 1, d.data_ptr(), 12, 7, None) == tv.ERR_INVALID
    assert b"power of 2" in lib.tvmc_last_error()
    assert lib.tvmc_evaluate_on_coset_gpu(d.data_ptr(), 4, 1, d.data_ptr(), 1 << 25, 7, None) == tv.ERR_UNSUPPORTED
