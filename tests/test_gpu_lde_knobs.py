"""The LDE's scheduling knobs change how the work is split and staged, never
the result: every combination of the fused middle kernel's variant and
occupancy, the four-step split and the tile size gives the oracle's LDE bit for
bit, for the plain and the randomized (zero-knowledge) LDE.  Knobs are process
wide; each test restores the defaults."""
import itertools

import numpy as np
import pytest

from conftest import dev_empty, from_dev, rand_u64, to_dev

pytestmark = pytest.mark.gpu

KNOBS = ("lde_mid_variant", "lde_mid_ctas", "lde_split_l1", "ntt_tile_log")


@pytest.fixture
def knobs(tv):
    saved = {k: tv.get_tuning(k) for k in KNOBS}
    yield tv
    for k, v in saved.items():
        tv.set_tuning(k, v)


def _set(tv, variant, ctas, split, tile):
    tv.set_tuning("lde_mid_variant", variant)
    tv.set_tuning("lde_mid_ctas", ctas)
    tv.set_tuning("lde_split_l1", split)
    tv.set_tuning("ntt_tile_log", tile)


@pytest.mark.parametrize("logn,expansion", [(12, 4), (14, 2), (16, 16), (18, 4)])
def test_lde_every_knob_combination_equals_oracle(knobs, oracle, logn, expansion):
    tv = knobs
    t = rand_u64(7000 + logn, (3, 1 << logn))
    exp = oracle.lde(t, expansion=expansion)
    splits = sorted({0, logn // 2 - 1, logn // 2 + 1, max(1, logn - 12)})
    for variant, ctas, split, tile in itertools.product((1, 2), (2, 3), splits, (12, 13, 14)):
        _set(tv, variant, ctas, split, tile)
        got = tv.lde(t, expansion=expansion)
        assert (got == exp).all(), (variant, ctas, split, tile)


def test_lde_largest_trace_at_expansion_16(tv, oracle):
    """2^22 rows x 16: the split moves work to K2 so that K3's tile of all 16
    cosets fits in shared memory.  Checked against the oracle's interpolation
    and coset evaluation (LDE::extend_column's two steps)."""
    n, E = 1 << 22, 16
    t = rand_u64(7300, (1, n))
    d_t = to_dev(t)
    d_o = dev_empty(E * n)
    tv.lde_gpu(d_t.data_ptr(), 1, n, d_o.data_ptr(), E * n)
    exp = oracle.evaluate_on_coset(oracle.ntt(t[0], inverse=True), E * n, 7)
    assert (from_dev(d_o) == exp).all()


def test_lde_knobs_full_size_column(knobs, oracle):
    tv = knobs
    n = 1 << 20
    t = rand_u64(7100, (2, n))
    exp = oracle.lde(t)
    d_t = to_dev(t)
    d_o = dev_empty(2 * 4 * n)
    for variant, ctas, split, tile in ((2, 3, 0, 13), (2, 2, 8, 13), (1, 3, 8, 14), (2, 3, 12, 12)):
        _set(tv, variant, ctas, split, tile)
        tv.lde_gpu(d_t.data_ptr(), 2, n, d_o.data_ptr(), 4 * n)
        assert (from_dev(d_o).reshape(2, 4 * n) == exp).all(), (variant, ctas, split, tile)


@pytest.mark.parametrize("variant", [1, 2])
def test_randomized_lde_with_each_mid_variant(knobs, oracle, variant):
    tv = knobs
    tv.set_tuning("lde_mid_variant", variant)
    t = rand_u64(7200, (3, 1 << 14))
    rnd = rand_u64(7201, (3, 40))
    exp = oracle.lde_randomized(t, rnd, 4, 7, 3)
    with tv.Commitment(t, randomizers=rnd, trace_offset=3) as c:
        assert (c.lde() == exp).all()


def test_knob_values_are_validated(knobs):
    tv = knobs
    for key, bad in (("lde_mid_variant", 3), ("lde_split_l1", 13), ("ntt_tile_log", 9)):
        with pytest.raises(tv.InvalidArgument):
            tv.set_tuning(key, bad)
