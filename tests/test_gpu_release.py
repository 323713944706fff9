"""tvmc_release_cached_memory frees the per-stream scratch and the cached
twiddle / coset-scale tables (one set per size, expansion and offset ever
used), which the next commit rebuilds; a live batch keeps the tables its graph
refers to.  Results before and after a release are identical."""
import numpy as np
import pytest

from conftest import memcpy_h2d, rand_u64

pytestmark = pytest.mark.gpu


def test_release_then_recommit_with_many_offsets(tv, oracle):
    t = rand_u64(9500, (5, 1 << 12))
    rnd = rand_u64(9501, (5, 3))
    roots = {}
    for to in (1, 3, 5, 11, 13):  # distinct trace offsets: distinct coset-scale tables
        with tv.Commitment(t, randomizers=rnd, trace_offset=to) as c:
            roots[to] = c.root()
    tv.release_cached_memory()
    for to in (1, 3, 5, 11, 13):
        with tv.Commitment(t, randomizers=rnd, trace_offset=to) as c:
            assert (c.root() == roots[to]).all()
    exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde_randomized(t, rnd, 4, 7, 5)))[1]
    assert (roots[5] == exp).all()


def test_release_keeps_tables_of_a_live_batch(tv):
    shapes = [(1 << 10, 23), (1 << 12, 9)]
    traces = [rand_u64(9600 + i, (w, n)) for i, (n, w) in enumerate(shapes)]
    with tv.Batch(shapes) as b:
        for i, t in enumerate(traces):
            memcpy_h2d(b.input_ptr(i), t)
        b.run()
        before = b.roots()
        tv.release_cached_memory()
        b.run()
        assert (b.roots() == before).all()
    for t, r in zip(traces, before):
        with tv.Commitment(t) as c:
            assert (c.root() == r).all()
