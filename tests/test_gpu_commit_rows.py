"""Commitments to already-evaluated rows (quotient segments) and to given
leaves (FRI round trees: XFieldElement codeword elements padded to digests),
vs the oracle and the reference's Merkle goldens."""
import numpy as np
import pytest

from conftest import P, golden, rand_u64

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,width", [(1, 3), (8, 12), (1 << 10, 12), (1 << 12, 3), (256, 0)])
def test_commit_rows_vs_oracle(tv, oracle, rows, width):
    t = rand_u64(rows * 7 + width, (width, rows))
    exp = oracle.merkle(oracle.hash_rows_cm(t) if width else np.stack([oracle.hash_varlen([])] * rows))
    with tv.Commitment.from_rows(t) as c:
        assert (c.nodes()[1:] == exp[1:]).all()
        if width:
            idx = [0, rows - 1, rows // 2]
            assert (c.read_rows(idx) == t[:, idx].T).all()
            if rows > 1:
                assert (c.auth_paths(idx) == np.stack([oracle.auth_path(exp, i) for i in idx])).all()
    with tv.Commitment.from_rows(np.ascontiguousarray(t.T), row_major=True, discard=True) as r:
        assert (r.root() == exp[1]).all()


def test_commit_rows_device_forms(tv, oracle):
    import torch
    t = rand_u64(99, (15, 1 << 9))
    exp = oracle.merkle(oracle.hash_rows_cm(t))
    d_cm = torch.from_numpy(t.view(np.int64)).cuda()
    d_rm = torch.from_numpy(np.ascontiguousarray(t.T).view(np.int64)).cuda()
    for ptr, rm, disc in [(d_cm, False, False), (d_cm, False, True), (d_rm, True, False)]:
        with tv.Commitment.from_rows(ptr.data_ptr(), width=15, rows=1 << 9, device_ptr=True, row_major=rm,
                                     discard=disc) as c:
            assert (c.nodes()[1:] == exp[1:]).all()
    torch.cuda.synchronize()


def test_commit_digests_equals_reference_tree(tv):
    """Leaves given as digests: every node equals the reference's MerkleTree (golden)."""
    g = golden("commit_w23_n64.npz")
    with tv.Commitment.from_digests(g["leaves"]) as c:
        assert (c.nodes()[1:] == g["nodes"][1:]).all()
        assert (c.auth_paths(g["path_idx"]) == g["paths"]).all()
        assert (c.auth_structure(g["struct_idx"]) == g["struct"]).all()


@pytest.mark.parametrize("n", [1, 2, 1 << 10, 1 << 17])
def test_commit_xfe_codeword_leaves(tv, oracle, n):
    """FRI round tree: codeword element i (c0, c1, c2) is leaf (c0, c1, c2, 0, 0), unhashed."""
    cw = rand_u64(n + 5, (n, 3))
    cw[0, 0] = P + 3  # a non-canonical input is read mod p
    leaves = np.zeros((n, 5), np.uint64)
    leaves[:, :3] = cw % np.uint64(P)
    exp = oracle.merkle(leaves)
    with tv.Commitment.from_digests(cw, xfe=True) as c:
        assert (c.nodes()[1:] == exp[1:]).all()
    import torch
    d = torch.from_numpy(cw.view(np.int64)).cuda()
    with tv.Commitment.from_digests(d.data_ptr(), xfe=True, count=n, device_ptr=True) as c:
        assert (c.root() == exp[1]).all()
    torch.cuda.synchronize()


def test_commit_rows_errors(tv):
    with pytest.raises(tv.InvalidArgument):
        tv.Commitment.from_rows(rand_u64(1, (3, 12)))
    with pytest.raises(tv.InvalidArgument):
        tv.Commitment.from_digests(rand_u64(1, (6, 5)))
