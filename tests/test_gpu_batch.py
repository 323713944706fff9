"""Batched commitment of uneven tables in one CUDA-graph launch: every root
(and sampled auth paths) must equal the table committed alone."""
import numpy as np
import pytest

from conftest import memcpy_h2d, rand_u64

pytestmark = pytest.mark.gpu


def uneven_shapes(seed, count, lo=12, hi=18):
    rng = np.random.default_rng(seed)
    logs = rng.integers(lo, hi + 1, count)
    widths = np.where(rng.random(count) < 0.5, 379, 264)
    return [(1 << int(l), int(w)) for l, w in zip(logs, widths)]


def fill(tv, batch, tables):
    """Copy host tables into the batch-owned device input buffers."""
    for i, t in enumerate(tables):
        t = np.ascontiguousarray(t, dtype=np.uint64)
        if t.size:
            memcpy_h2d(batch.input_ptr(i), t)


def test_small_batch_vs_oracle(tv, oracle):
    shapes = [(16, 23), (64, 11), (8, 264), (256, 10), (1, 5)]
    tables = [rand_u64(40 + i, (w, n)) for i, (n, w) in enumerate(shapes)]
    with tv.Batch(shapes) as b:
        fill(tv, b, tables)
        b.run()
        for t, c in zip(tables, b.tables):
            exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde(t)))
            assert (c.nodes()[1:] == exp[1:]).all()
            assert (c.lde() == oracle.lde(t)).all()


@pytest.mark.parametrize("streams", [1, 8])
def test_uneven_32_tables_equal_alone(tv, streams):
    """32 tables, heights log-uniform in 2^12..2^18, widths 379 / 264 (50/50)."""
    tv.set_tuning("batch_streams", streams)
    try:
        shapes = uneven_shapes(2026, 32)
        tables = [rand_u64(500 + i, (w, n)) for i, (n, w) in enumerate(shapes)]
        alone = []
        for t in tables:
            with tv.Commitment(t) as c:
                alone.append(c.root())
        with tv.Batch(shapes) as b:
            fill(tv, b, tables)
            for _ in range(2):  # the graph replays
                b.run()
                roots = b.roots()
                for i in range(32):
                    assert (roots[i] == alone[i]).all(), i
            idx = [0, 5, 77]
            with tv.Commitment(tables[3]) as c:
                assert (b.tables[3].auth_paths(idx) == c.auth_paths(idx)).all()
    finally:
        tv.set_tuning("batch_streams", 0)


def test_batch_refills_between_runs(tv):
    shapes = [(1 << 12, 379), (1 << 13, 264)]
    with tv.Batch(shapes) as b:
        for seed in (1, 2):
            tables = [rand_u64(seed * 10 + i, (w, n)) for i, (n, w) in enumerate(shapes)]
            fill(tv, b, tables)
            b.run()
            for t, c in zip(tables, b.tables):
                with tv.Commitment(t) as a:
                    assert (c.root() == a.root()).all()


def test_batch_handles_are_not_freed_individually(tv):
    with tv.Batch([(16, 3)]) as b:
        fill(tv, b, [rand_u64(1, (3, 16))])
        b.run()
        rc = tv.lib().tvmc_commitment_free(b.tables[0].h)
        assert rc == tv.ERR_INVALID
