"""The commitment serving loop (tvmc_server_*): every request's root, tree
openings and rows are bit-identical to committing that table alone, whatever
else is in flight; admission respects the HBM budget; errors and timeouts are
reported per request."""
import threading

import numpy as np
import pytest

from conftest import rand_u64

pytestmark = pytest.mark.gpu


def _mix(seed, count, logs=(4, 6, 8, 10, 12, 14), widths=(379, 264, 23)):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = 1 << int(rng.choice(logs))
        w = int(rng.choice(widths))
        out.append(rand_u64(seed * 1000 + i, (w, n)))
    return out


@pytest.mark.parametrize("streams,budget", [(4, 0), (1, 0), (8, 600 << 20)])
def test_server_results_equal_alone(tv, streams, budget):
    """A mix of sizes submitted at once (a tight budget forces queueing):
    roots and 80 openings per request equal each table committed alone."""
    tables = _mix(7 + streams, 14)
    rng = np.random.default_rng(3)
    with tv.Server(hbm_budget_bytes=budget, streams=streams) as srv:
        ids = [srv.submit(t) for t in tables]
        for rid, t in zip(ids, tables):
            root = srv.wait(rid)
            L = 4 * t.shape[1]
            idx = rng.integers(0, L, 80)
            with tv.Commitment(t) as alone:
                assert (root == alone.root()).all()
                assert (srv.open(rid, idx) == alone.auth_paths(idx)).all()
            srv.release(rid)
        st = srv.stats()
        assert st["completed"] == len(tables) and st["failed"] == 0 and st["bytes_in_use"] == 0
        if budget:
            assert st["bytes_peak"] <= budget


@pytest.mark.parametrize("group_small", [True, False])
def test_server_mix_up_to_2p20_rows_equals_alone(tv, group_small):
    """The serving stream's whole size range in one mix: tables of 2^18 .. 2^20
    rows (large, on the dedicated stream) among bursts of small ones (committed
    together as multi-table groups, or one by one): each root and a set of
    openings equal the table committed alone."""
    tables = _mix(31, 18, logs=(10, 11, 12, 13, 14), widths=(379, 264, 23))
    tables.insert(3, rand_u64(3101, (379, 1 << 20)))
    tables.insert(9, rand_u64(3102, (264, 1 << 19)))
    tables.insert(15, rand_u64(3103, (23, 1 << 18)))
    rng = np.random.default_rng(4)
    with tv.Server(streams=4, group_small=group_small) as srv:
        ids = [srv.submit(t) for t in tables]
        for rid, t in zip(ids, tables):
            root = srv.wait(rid)
            idx = rng.integers(0, 4 * t.shape[1], 8)
            with tv.Commitment(t, discard_lde=True) as alone:
                assert (root == alone.root()).all()
                assert (srv.open(rid, idx) == alone.auth_paths(idx)).all()
            srv.release(rid)
        st = srv.stats()
        assert st["completed"] == len(tables) and st["failed"] == 0 and st["bytes_in_use"] == 0


def test_server_groups_a_burst_of_small_requests(tv, oracle):
    """64 small requests submitted at once while a large one runs: they are
    committed in multi-table groups and every tree equals the oracle's."""
    small = [rand_u64(3200 + i, (int(w), 1 << int(l)))
             for i, (l, w) in enumerate(zip(np.random.default_rng(5).integers(0, 9, 64),
                                            np.random.default_rng(6).choice([1, 9, 23, 379], 64)))]
    big = rand_u64(3199, (379, 1 << 18))
    with tv.Server(streams=2, group_small=True) as srv:
        rb = srv.submit(big)
        ids = [srv.submit(t) for t in small]
        for rid, t in zip(ids, small):
            exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde(t)))
            assert (srv.wait(rid) == exp[1]).all()
            assert (srv.open(rid, [0, 4 * t.shape[1] - 1]) ==
                    np.stack([oracle.auth_path(exp, 0), oracle.auth_path(exp, 4 * t.shape[1] - 1)])).all()
            srv.release(rid)
        with tv.Commitment(big, discard_lde=True) as alone:
            assert (srv.wait(rb) == alone.root()).all()
        srv.release(rb)


def test_server_keep_lde_rows_and_layouts(tv):
    t = rand_u64(11, (37, 1 << 9))
    with tv.Server(keep_lde=True) as srv:
        a = srv.submit(t)
        b = srv.submit(np.ascontiguousarray(t.T), row_major=True)
        c = srv.submit(t, frugal=True)
        with tv.Commitment(t) as alone:
            for rid in (a, b, c):
                assert (srv.wait(rid) == alone.root()).all()
            idx = [0, 5, 2047, 1000]
            paths, rows = srv.open(a, idx, rows=True)
            assert (paths == alone.auth_paths(idx)).all()
            assert (rows == alone.read_rows(idx)).all()
        with pytest.raises(tv.InvalidArgument):  # frugal requests keep no LDE
            srv.open(c, idx, rows=True)
        with pytest.raises(tv.OutOfRange):
            srv.open(a, [4 * 512])


def test_server_concurrent_submitters(tv):
    """Four host threads submitting and waiting at once."""
    tables = _mix(21, 16, logs=(6, 8, 10))
    results = {}
    with tv.Server(streams=4) as srv:
        def worker(k):
            for i in range(k, len(tables), 4):
                rid = srv.submit(tables[i])
                results[i] = srv.wait(rid)
                srv.release(rid)
        th = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for x in th:
            x.start()
        for x in th:
            x.join()
    for i, t in enumerate(tables):
        with tv.Commitment(t) as alone:
            assert (results[i] == alone.root()).all()


def test_server_budget_and_errors(tv):
    big = rand_u64(5, (64, 1 << 12))
    small = rand_u64(6, (8, 1 << 6))
    with tv.Server(hbm_budget_bytes=1 << 20) as srv:  # 1 MiB: the big table cannot fit
        rb = srv.submit(big)
        rs = srv.submit(small)
        with pytest.raises(tv.OutOfMemory):
            srv.wait(rb)
        with tv.Commitment(small) as alone:
            assert (srv.wait(rs) == alone.root()).all()
        srv.release(rb)  # failed requests can be released
        srv.release(rs)
        with pytest.raises(tv.InvalidArgument):
            srv.release(rs)
        with pytest.raises(tv.InvalidArgument):
            srv.submit(rand_u64(1, (3, 12)))  # not a power of two
        assert srv.stats()["failed"] == 1


def test_server_wait_timeout_and_times(tv):
    t = rand_u64(9, (379, 1 << 14))
    with tv.Server() as srv:
        rid = srv.submit(t)
        try:
            srv.wait(rid, timeout_ms=0)
        except tv.Timeout:
            pass  # still running: the bounded wait returned without blocking
        srv.wait(rid)
        sub, start, done = srv.times(rid)
        assert 0 < sub <= start <= done
        with pytest.raises(tv.InvalidArgument):
            srv.wait(rid + 1000)


def test_server_randomized_requests(tv, oracle):
    """Randomized (zero-knowledge) requests mixed with plain ones: each equals
    tvmc_commit_randomized alone (and the oracle's tree for a small one)."""
    specs = [(1 << 6, 23, 98, 3), (1 << 10, 64, 7, 1), (1 << 12, 379, 98, 5), (1 << 8, 10, 0, 1)]
    tables = [(rand_u64(70 + i, (w, n)), rand_u64(80 + i, (w, R)), t) for i, (n, w, R, t) in enumerate(specs)]
    with tv.Server(streams=3) as srv:
        ids = [srv.submit(tr, randomizers=rnd, trace_offset=t) for tr, rnd, t in tables]
        plain = srv.submit(tables[1][0])
        for rid, (tr, rnd, t) in zip(ids, tables):
            with tv.Commitment(tr, randomizers=rnd, trace_offset=t) as alone:
                assert (srv.wait(rid) == alone.root()).all()
                idx = [0, 3, 4 * tr.shape[1] - 1]
                assert (srv.open(rid, idx) == alone.auth_paths(idx)).all()
        with tv.Commitment(tables[1][0]) as alone:
            assert (srv.wait(plain) == alone.root()).all()
    tr, rnd, t = tables[0]
    exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde_randomized(tr, rnd, 4, 7, t)))
    with tv.Commitment(tr, randomizers=rnd, trace_offset=t) as alone:
        assert (alone.root() == exp[1]).all()
