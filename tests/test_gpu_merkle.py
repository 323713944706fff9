"""Merkle trees on the GPU vs the oracle: heap layout (CPU MerkleTree) and the
flat layout of the reference's merkle_tree_gpu."""
import numpy as np
import pytest

from conftest import dev_empty, from_dev, rand_u64, to_dev

pytestmark = pytest.mark.gpu


def flat_index(h, n):
    pm = 1 << (int(h).bit_length() - 1)
    return 2 * n + h - 3 * pm


@pytest.mark.parametrize("logn", [0, 1, 2, 5, 7, 8, 9, 12, 16])
def test_heap_tree(tv, oracle, logn):
    n = 1 << logn
    lv = rand_u64(logn, (n, 5))
    assert (tv.merkle_heap(lv)[1:] == oracle.merkle(lv)[1:]).all()


@pytest.mark.parametrize("logn", [0, 3, 10, 15])
def test_flat_tree_and_root(tv, oracle, logn):
    n = 1 << logn
    lv = rand_u64(100 + logn, (n, 5))
    heap = oracle.merkle(lv)
    d_l, d_t, d_r = to_dev(lv), dev_empty((2 * n - 1) * 5), dev_empty(5)
    tv.merkle_tree_gpu(d_l.data_ptr(), d_t.data_ptr(), n)
    flat = from_dev(d_t).reshape(2 * n - 1, 5)
    for h in range(1, 2 * n):
        assert (flat[flat_index(h, n)] == heap[h]).all(), h
    assert (flat[2 * n - 2] == heap[1]).all()
    tv.merkle_root_gpu(d_l.data_ptr(), d_r.data_ptr(), n)
    assert (from_dev(d_r) == heap[1]).all()


def test_noncanonical_leaves(tv, oracle):
    lv = rand_u64(3, (64, 5), hi=2**64 - 1)
    assert (tv.merkle_heap(lv)[1:] == oracle.merkle(lv)[1:]).all()


def test_bad_leaf_count(tv):
    with pytest.raises(tv.InvalidArgument):
        tv.merkle_heap(np.zeros((12, 5), np.uint64))
