"""The whole table commitment (LDE -> Tip5 row hash -> Merkle) through the C ABI
vs the oracle: every LDE cell, every tree node, the root, auth paths."""
import numpy as np
import pytest

from conftest import P, from_dev, golden, rand_u64, to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["commit_w23_n64", "commit_w379_n4", "commit_w264_n8", "commit_w1_n1"])
def test_commit_golden(tv, name):
    g = golden(f"{name}.npz")
    with tv.Commitment(g["trace"]) as c:
        assert (c.root() == g["root"]).all()
        assert (c.lde() == g["lde"]).all()
        assert (c.leaves() == g["leaves"]).all()
        assert (c.nodes()[1:] == g["nodes"][1:]).all()
        if c.height:
            assert (c.auth_paths(g["path_idx"]) == g["paths"]).all()
        assert (c.auth_structure(g["struct_idx"]) == g["struct"]).all()


def test_commit_main_table_2p10_x379(tv, oracle):
    """2^10 rows x 379 columns, expansion 4, offset 7: every cell and node."""
    n, w = 1 << 10, 379
    t = rand_u64(0x7E5EED01, (w, n))
    with tv.Commitment(t) as c:
        lde = c.lde()
        exp_lde = oracle.lde(t)
        assert (lde == exp_lde).all()
        nodes = c.nodes()
        exp_nodes = oracle.merkle(oracle.hash_rows_cm(exp_lde))
        assert (nodes[1:] == exp_nodes[1:]).all()
        idx = np.random.default_rng(1).integers(0, 4 * n, 16)
        paths = c.auth_paths(idx)
        for i, p in zip(idx, paths):
            assert (p == oracle.auth_path(exp_nodes, int(i))).all()
            assert oracle.verify(exp_nodes[1], int(i), exp_nodes[4 * n + int(i)], p)
        rows = c.read_rows(idx)
        assert (rows == exp_lde[:, idx].T).all()


def test_commit_row_major_equals_column_major(tv):
    t = rand_u64(12, (37, 256))
    with tv.Commitment(t) as a, tv.Commitment(np.ascontiguousarray(t.T), row_major=True) as b:
        assert (a.root() == b.root()).all()
        assert (a.lde() == b.lde()).all()
        assert (a.lde(row_major=True) == b.lde().T).all()


def test_commit_aux_xfe_table(tv, oracle):
    """88 XFieldElement columns = 264 base limbs (c0, c1, c2 per column)."""
    n = 1 << 8
    xfe = rand_u64(88, (n, 88, 3))                 # row-major XFE table
    flat_rm = xfe.reshape(n, 264)                 # hash order x0.c0, x0.c1, x0.c2, x1.c0, ...
    with tv.Commitment(flat_rm, row_major=True) as c:
        exp_lde = oracle.lde(np.ascontiguousarray(flat_rm.T))
        assert (c.lde() == exp_lde).all()
        assert (c.root() == oracle.merkle(oracle.hash_rows_cm(exp_lde))[1]).all()


def test_commit_device_trace_and_discard(tv, oracle):
    t = rand_u64(13, (11, 512))
    d = to_dev(t)
    with tv.Commitment(d.data_ptr(), width=11, trace_len=512, device_ptr=True, discard_lde=True) as c:
        exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde(t)))
        assert (c.root() == exp[1]).all()
        with pytest.raises(tv.InvalidArgument):
            c.read_rows([0])


def test_commit_expansion_8(tv, oracle):
    t = rand_u64(14, (19, 1 << 12))
    with tv.Commitment(t, expansion=8) as c:
        exp = oracle.lde(t, expansion=8)
        assert (c.lde() == exp).all()
        assert (c.root() == oracle.merkle(oracle.hash_rows_cm(exp))[1]).all()


def test_commit_errors(tv):
    t = rand_u64(15, (3, 16))
    with tv.Commitment(t) as c:
        with pytest.raises(tv.OutOfRange):
            c.auth_paths([64])
        with pytest.raises(tv.OutOfRange):
            c.read_rows([64])
        with pytest.raises(tv.OutOfRange):
            c.auth_structure([1, 99])
    with pytest.raises(tv.InvalidArgument):
        tv.Commitment(rand_u64(1, (3, 24)))


def test_commit_full_size_properties(tv, oracle):
    """2^20 x 379 -> 2^22 rows: two full columns vs the oracle, sampled rows'
    leaf digests, and sampled auth paths verified against the root."""
    n, w = 1 << 20, 379
    import torch
    g = torch.Generator(device="cuda").manual_seed(5)
    d = torch.randint(0, 2**62, (w, n), dtype=torch.int64, device="cuda", generator=g)
    with tv.Commitment(d.data_ptr(), width=w, trace_len=n, device_ptr=True) as c:
        root = c.root()
        cols = c.read_columns(0, 1)[0], c.read_columns(378, 1)[0]
        for col, got in zip((0, 378), cols):
            exp = oracle.lde(from_dev(d[col]).reshape(1, n))[0]
            assert (got == exp).all()
        idx = np.random.default_rng(3).integers(0, 4 * n, 64)
        rows = c.read_rows(idx)
        leaves = oracle.hash_rows_rm(rows)
        paths = c.auth_paths(idx)
        for i, lf, p in zip(idx, leaves, paths):
            assert oracle.verify(root, int(i), lf, p)
        assert (root < P).all()


@pytest.mark.parametrize("knob,value", [("hash_unfused_tree", 1), ("lde_mid_ctas", 3)])
@pytest.mark.parametrize("logn", [4, 12, 14])
def test_tuning_knobs_do_not_change_results(tv, oracle, knob, value, logn):
    """Scheduling knobs change no bit: plain and frugal commits vs the default."""
    t = rand_u64(0xC0FFEE + logn, (23, 1 << logn))
    with tv.Commitment(t) as ref:
        exp = ref.nodes()
    try:
        tv.set_tuning(knob, value)
        with tv.Commitment(t) as a, tv.Commitment(t, frugal=True) as b:
            assert (a.nodes()[1:] == exp[1:]).all()
            assert (b.nodes()[1:] == exp[1:]).all()
    finally:
        tv.set_tuning(knob, 0)
    if logn == 4:
        assert (exp[1:] == oracle.merkle(oracle.hash_rows_cm(oracle.lde(t)))[1:]).all()


def test_back_to_back_host_commits_share_staging_safely(tv):
    """Host-trace commits issued back to back on one stream reuse its upload
    staging buffers, the next upload overlapping the previous commit's row hash.
    2^17 x 379 traces upload in several chunks; every root must equal the
    device-input commit's (which uses no staging)."""
    import torch
    tables = [rand_u64(0x5EED00 + i, (379, 1 << 17)) for i in range(3)]
    stream = torch.cuda.Stream()
    commits = [tv.Commitment(t, stream=stream.cuda_stream, discard_lde=True) for t in tables]
    roots = [c.root() for c in commits]
    for c in commits:
        c.free()
    for t, r in zip(tables, roots):
        d = torch.from_numpy(t.view(np.int64)).cuda()
        with tv.Commitment(d.data_ptr(), width=t.shape[0], trace_len=t.shape[1], device_ptr=True) as ref:
            assert (r == ref.root()).all()
    torch.cuda.synchronize()


def test_forget_stream_then_reuse(tv):
    """tvmc_forget_stream frees a stream's cached buffers; later commits on the
    same stream (or a new one) rebuild them and give the same root."""
    import torch
    t = rand_u64(0x0F0F, (64, 1 << 12))
    s = torch.cuda.Stream()
    with tv.Commitment(t, stream=s.cuda_stream, discard_lde=True) as a:
        ra = a.root()
    tv.forget_stream(s.cuda_stream)
    with tv.Commitment(t, stream=s.cuda_stream, discard_lde=True) as b:
        assert (b.root() == ra).all()
    tv.forget_stream(s.cuda_stream)
    tv.release_cached_memory()
    with tv.Commitment(t) as c:
        assert (c.root() == ra).all()
