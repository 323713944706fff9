"""Tip5 on the GPU (through the C ABI) vs the oracle and the golden vectors."""
import numpy as np
import pytest

from conftest import EDGE_VALUES, P, dev_empty, from_dev, golden, rand_u64, to_dev

pytestmark = pytest.mark.gpu


def test_permutation_golden(tv):
    g = golden("tip5.npz")
    assert (tv.tip5_permutations(g["states"]) == g["perms"]).all()


def test_permutation_random_and_edges(tv, oracle):
    st = rand_u64(1, (3000, 16), hi=2**64 - 1)
    st[:16] = EDGE_VALUES[np.arange(256).reshape(16, 16) % 16]
    st[16] = EDGE_VALUES
    got = tv.tip5_permutations(st)
    for i in list(range(40)) + list(range(2990, 3000)):
        assert (got[i] == oracle.permutation(st[i])).all(), i
    assert (got < P).all()


def test_hash_varlen_golden_lengths(tv):
    g = golden("tip5.npz")
    off = 0
    for n, exp in enumerate(g["varlen_out"]):
        got = tv.hash_varlen_rows(g["varlen_in"][off:off + n].reshape(1, n))
        assert (got[0] == exp).all(), n
        off += n


@pytest.mark.parametrize("width", [1, 9, 10, 11, 20, 264, 379])
def test_hash_rows_vs_oracle(tv, oracle, width):
    t = rand_u64(width, (300, width))
    got = tv.hash_varlen_rows(t)
    exp = oracle.hash_rows_rm(t)
    assert (got == exp).all()


def test_hash_rows_noncanonical_inputs(tv, oracle):
    t = rand_u64(4, (64, 23), hi=2**64 - 1)
    t[:, 0] = P + np.arange(64, dtype=np.uint64)  # values >= p read mod p
    assert (tv.hash_varlen_rows(t) == oracle.hash_rows_rm(t)).all()


def test_hash_pairs_golden(tv):
    g = golden("tip5.npz")
    assert (tv.hash_pairs(g["pairs_l"], g["pairs_r"]) == g["pairs"]).all()


def test_device_hash_rows_colmajor(tv, oracle):
    rows, w = 1000, 379
    t = rand_u64(8, (w, rows))
    d_t, d_o = to_dev(t), dev_empty(rows * 5)
    tv.hash_rows_gpu(d_t.data_ptr(), rows, w, d_o.data_ptr())
    got = from_dev(d_o).reshape(rows, 5)
    assert (got == oracle.hash_rows_cm(t)).all()


def test_device_hash_xfield_rows(tv, oracle):
    rows, xw = 256, 88
    t = rand_u64(9, (3 * xw, rows))  # (xfe_col*3 + comp) major
    d_t, d_o = to_dev(t), dev_empty(rows * 5)
    tv.hash_xfield_rows_gpu(d_t.data_ptr(), rows, xw, d_o.data_ptr())
    got = from_dev(d_o).reshape(rows, 5)
    assert (got == oracle.hash_rows_cm(t)).all()
