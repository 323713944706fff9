"""Randomized (zero-knowledge) LDE and commitment on the GPU vs the reference's
RandomizedLDE / LDETable outputs (golden fixtures) and the oracle."""
import numpy as np
import pytest

from conftest import P, golden, rand_u64

pytestmark = pytest.mark.gpu


def test_lde_randomized_golden(tv):
    g = golden("lde_randomized.npz")
    for k in [k for k in g.files if k.endswith("_meta")]:
        p = k[:-5]
        if p.startswith("b"):
            n, R, E, t, o = (int(v) for v in g[k])
            got = tv.lde_randomized(g[p + "_trace"], g[p + "_rnd"], E, o, t)
        else:  # XFE columns: three limb columns, truncating variant
            n, R, E, t, o, xr = (int(v) for v in g[k])
            tr, rnd = g[p + "_trace"], g[p + "_rnd"]
            w = tr.shape[0]
            limbs = np.ascontiguousarray(tr.transpose(0, 2, 1).reshape(3 * w, n))
            if xr:
                rl = np.ascontiguousarray(rnd.transpose(0, 2, 1).reshape(3 * w, R))
            else:
                rl = np.zeros((w, 3, R), np.uint64)
                rl[:, 0, :] = rnd
                rl = rl.reshape(3 * w, R)
            out = tv.lde_randomized(limbs, rl, E, o, t, truncate=True)
            got = out.reshape(w, 3, n * E).transpose(0, 2, 1)
        assert (got == g[p + "_out"]).all(), p


def test_commit_randomized_table_root(tv):
    """LDETable::compute_lde_and_merkle (row-major table, 98 randomizers per column)."""
    g = golden("lde_randomized.npz")
    with tv.Commitment(g["table_rows"], row_major=True, randomizers=g["table_rnd"]) as c:
        assert (c.root() == g["table_root"]).all()


@pytest.mark.parametrize("logn", [0, 1, 3, 5, 6, 7, 9, 11, 12, 13, 14, 15])
@pytest.mark.parametrize("R,E,t", [(98, 4, 1), (5, 2, 3), (0, 4, 11), (1, 8, 1)])
def test_lde_randomized_vs_oracle(tv, oracle, logn, R, E, t):
    n = 1 << logn
    w = 3
    tr = rand_u64(logn * 131 + R, (w, n))
    rnd = rand_u64(logn * 17 + R + 1, (w, R))
    got = tv.lde_randomized(tr, rnd, E, 7, t)
    exp = oracle.lde_randomized(tr, rnd, E, 7, t)
    assert (got == exp).all()


@pytest.mark.parametrize("logn,R,E", [(2, 40, 2), (3, 100, 4), (0, 9, 2), (4, 16, 1), (5, 70, 2)])
@pytest.mark.parametrize("truncate", [False, True])
def test_lde_randomized_long_polynomials(tv, oracle, logn, R, E, truncate):
    """R >= N or N + R > L: chunked (exact) or truncated evaluation."""
    n = 1 << logn
    tr = rand_u64(900 + R, (4, n))
    rnd = rand_u64(901 + R, (4, R))
    got = tv.lde_randomized(tr, rnd, E, 7, 5, truncate=truncate)
    assert (got == oracle.lde_randomized(tr, rnd, E, 7, 5, truncate=truncate)).all()


def test_lde_randomized_zero_randomizer_is_plain_lde(tv):
    tr = rand_u64(4, (5, 1 << 10))
    assert (tv.lde_randomized(tr, np.zeros((5, 0), np.uint64)) == tv.lde(tr)).all()
    assert (tv.lde_randomized(tr, np.zeros((5, 3), np.uint64)) == tv.lde(tr)).all()


@pytest.mark.parametrize("logn", [16, 20])
def test_lde_randomized_large_sampled(tv, oracle, logn):
    """2^16 and 2^20 rows (the four-step LDE kernels), 98 randomizers, vs the oracle."""
    n = 1 << logn
    tr = rand_u64(logn, (2, n))
    rnd = rand_u64(logn + 1, (2, 98))
    got = tv.lde_randomized(tr, rnd, 4, 7, 1)
    assert (got == oracle.lde_randomized(tr, rnd, 4, 7, 1)).all()


def test_commit_randomized_forms_agree(tv, oracle):
    """Host / device / row-major / frugal randomized commitments: identical trees,
    equal to the oracle's."""
    import torch
    n, w, R = 1 << 9, 37, 98
    tr = rand_u64(77, (w, n))
    rnd = rand_u64(78, (w, R))
    exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde_randomized(tr, rnd, 4, 7, 3)))
    with tv.Commitment(tr, randomizers=rnd, trace_offset=3) as a:
        assert (a.nodes()[1:] == exp[1:]).all()
        assert (a.lde() == oracle.lde_randomized(tr, rnd, 4, 7, 3)).all()
    with tv.Commitment(np.ascontiguousarray(tr.T), row_major=True, randomizers=rnd, trace_offset=3) as b:
        assert (b.nodes()[1:] == exp[1:]).all()
    with tv.Commitment(tr, randomizers=rnd, trace_offset=3, frugal=True) as f:
        assert (f.nodes()[1:] == exp[1:]).all()
    dt = torch.from_numpy(tr.view(np.int64)).cuda()
    dr = torch.from_numpy(rnd.view(np.int64)).cuda()
    with tv.Commitment(dt.data_ptr(), width=w, trace_len=n, device_ptr=True, randomizers=(dr.data_ptr(), R),
                       trace_offset=3) as d:
        assert (d.nodes()[1:] == exp[1:]).all()
    torch.cuda.synchronize()


def test_randomized_errors(tv):
    tr = rand_u64(1, (2, 16))
    with pytest.raises(tv.InvalidArgument):
        tv.lde_randomized(tr, rand_u64(2, (2, 3)), trace_offset=0)
    with pytest.raises(tv.InvalidArgument):
        tv.lde_randomized(tr, rand_u64(2, (2, 3)), trace_offset=P)
    with pytest.raises(tv.InvalidArgument):
        tv.Commitment(tr, randomizers=rand_u64(2, (2, 3)), trace_offset=0)
