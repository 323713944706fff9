"""tvmc_commit_multi: many plain commitments with one multi-table row-hash
launch.  Every table's tree equals its lone commitment and the oracle, bit for
bit, across heights (1 row .. 2^16 rows), widths, expansions and offsets, with
host and device traces, more tables than one launch takes, and tree tops both
in the multi-table kernel and in the single-tree kernels."""
import numpy as np
import pytest

from conftest import rand_u64, to_dev

pytestmark = pytest.mark.gpu


def _shapes(seed, count, max_log):
    rng = np.random.default_rng(seed)
    return [(1 << int(rng.integers(0, max_log + 1)), int(rng.choice([1, 9, 10, 23, 264, 379]))) for _ in range(count)]


def test_multi_commit_matches_oracle_small_mix(tv, oracle):
    shapes = _shapes(8100, 12, 9)
    traces = [rand_u64(8101 + i, (w, n)) for i, (n, w) in enumerate(shapes)]
    cs = tv.commit_multi(traces)
    try:
        for t, c in zip(traces, cs):
            exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde(t)))
            assert (c.nodes()[1:] == exp[1:]).all()
            assert (c.lde() == oracle.lde(t)).all()
    finally:
        for c in cs:
            c.free()


@pytest.mark.parametrize("discard", [False, True])
def test_multi_commit_equals_lone_commits(tv, discard):
    shapes = _shapes(8200, 40, 14) + [(1 << 16, 23), (1 << 15, 264)]  # the last two: tree tops > 1024 nodes
    traces = [rand_u64(8201 + i, (w, n)) for i, (n, w) in enumerate(shapes)]
    cs = tv.commit_multi(traces, discard_lde=discard)
    try:
        for t, c in zip(traces, cs):
            with tv.Commitment(t, discard_lde=True) as lone:
                assert (c.root() == lone.root()).all()
                assert (c.nodes()[1:] == lone.nodes()[1:]).all()
    finally:
        for c in cs:
            c.free()


def test_multi_commit_more_tables_than_one_launch_device_traces(tv):
    shapes = [(1 << (i % 7), 1 + (i * 37) % 50) for i in range(150)]  # 150 tables > 64 per launch
    traces = [rand_u64(8300 + i, (w, n)) for i, (n, w) in enumerate(shapes)]
    devs = [to_dev(t) for t in traces]
    cs = tv.commit_multi([d.data_ptr() for d in devs], device_ptr=True, shapes=shapes, expansion=2, offset=3,
                         sync=True)
    try:
        for t, c in zip(traces, cs):
            with tv.Commitment(t, expansion=2, offset=3, discard_lde=True) as lone:
                assert (c.root() == lone.root()).all()
    finally:
        for c in cs:
            c.free()


def test_multi_commit_openings(tv, oracle):
    t = rand_u64(8400, (37, 1 << 8))
    (c,) = tv.commit_multi([t])
    try:
        nodes = oracle.merkle(oracle.hash_rows_cm(oracle.lde(t)))
        for leaf in (0, 5, 1023):
            assert (c.auth_paths([leaf])[0] == oracle.auth_path(nodes, leaf)).all()
    finally:
        c.free()


def test_multi_commit_rejects_bad_tables(tv):
    good = rand_u64(8500, (3, 16))
    with pytest.raises(tv.InvalidArgument):
        tv.commit_multi([good, rand_u64(8501, (3, 12))])  # 12 rows: not a power of 2
    with pytest.raises(tv.InvalidArgument):
        tv.commit_multi([good], expansion=3)
    assert tv.commit_multi([]) == []
