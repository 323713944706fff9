"""Fiat-Shamir absorption on the device vs the oracle's Tip5 permutation
(pad-and-absorb: data, 1, zeros to a multiple of 10; overwrite rate, permute)."""
import numpy as np
import pytest

from conftest import P, rand_u64

pytestmark = pytest.mark.gpu


def oracle_absorb(oracle, state, data):
    s = np.array(state, dtype=np.uint64)
    padded = list(data) + [1]
    while len(padded) % 10:
        padded.append(0)
    for c0 in range(0, len(padded), 10):
        s[:10] = np.array(padded[c0:c0 + 10], dtype=np.uint64) % np.uint64(P)
        s = oracle.permutation(s)
    return s


@pytest.mark.parametrize("length", [0, 1, 6, 9, 10, 11, 19, 20, 37])
def test_sponge_absorb(tv, oracle, length):
    import torch
    state0 = rand_u64(length, 16)
    data = rand_u64(length + 100, max(length, 1))[:length]
    d_state = torch.from_numpy(state0.view(np.int64)).cuda()
    d_data = torch.from_numpy(np.ascontiguousarray(data).view(np.int64)).cuda() if length else None
    tv.sponge_absorb_gpu(d_state.data_ptr(), d_data.data_ptr() if length else 0, length)
    got = d_state.cpu().numpy().view(np.uint64)
    assert (got == oracle_absorb(oracle, state0, data)).all()


def test_commitment_absorb_root(tv, oracle):
    """A chain of two commitments absorbed as MerkleRoot items, root never on the host."""
    import torch
    tables = [rand_u64(31 + i, (23, 1 << 8)) for i in range(2)]
    d_state = torch.zeros(16, dtype=torch.int64, device="cuda")
    exp = np.zeros(16, dtype=np.uint64)
    for t in tables:
        with tv.Commitment(t) as c:
            c.absorb_root(d_state.data_ptr())
            root = oracle.merkle(oracle.hash_rows_cm(oracle.lde(t)))[1]
            exp = oracle_absorb(oracle, exp, [0] + [int(x) for x in root])
            torch.cuda.synchronize()
    assert (d_state.cpu().numpy().view(np.uint64) == exp).all()
