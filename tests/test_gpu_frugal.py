"""Frugal streaming commitment (TVMC_FRUGAL): the LDE is produced in
10-column-aligned stripes that are absorbed at once into resident sponge
states, so the full LDE never exists.  Every node of the tree must equal the
materialised commitment's (and the oracle's)."""
import numpy as np
import pytest

from conftest import rand_u64

pytestmark = pytest.mark.gpu


@pytest.fixture
def stripe_knob(tv):
    yield lambda v: tv.set_tuning("frugal_stripe_cols", v)
    tv.set_tuning("frugal_stripe_cols", 0)


@pytest.mark.parametrize("width", [0, 1, 9, 10, 11, 20, 25, 264, 379])
def test_frugal_equals_oracle(tv, oracle, stripe_knob, width):
    stripe_knob(10)
    n = 1 << 8
    t = rand_u64(300 + width, (width, n))
    with tv.Commitment(t, frugal=True) as c:
        nodes = c.nodes()
    exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde(t))) if width else None
    if width:
        assert (nodes[1:] == exp[1:]).all()
    else:
        with tv.Commitment(t) as p:
            assert (nodes[1:] == p.nodes()[1:]).all()


@pytest.mark.parametrize("stripe", [10, 20, 30, 380, 0])
def test_frugal_stripe_widths_equal_plain(tv, stripe_knob, stripe):
    stripe_knob(stripe)
    t = rand_u64(7, (379, 1 << 12))
    with tv.Commitment(t) as plain, tv.Commitment(t, frugal=True) as fr:
        assert (fr.nodes()[1:] == plain.nodes()[1:]).all()
        with pytest.raises(tv.InvalidArgument):
            fr.read_rows([0])


def test_frugal_row_major_and_device_inputs(tv, stripe_knob):
    import torch
    from conftest import to_dev
    stripe_knob(20)
    t = rand_u64(8, (264, 1 << 10))
    with tv.Commitment(t) as plain:
        ref = plain.root()
    with tv.Commitment(np.ascontiguousarray(t.T), row_major=True, frugal=True) as a:
        assert (a.root() == ref).all()
    d = to_dev(t)
    with tv.Commitment(d.data_ptr(), width=264, trace_len=1 << 10, device_ptr=True, frugal=True) as b:
        assert (b.root() == ref).all()
    torch.cuda.synchronize()


def test_frugal_2p22_x379_root_and_auth_paths(tv):
    """Padded height 2^22 x 379 -> 2^24-row LDE (50.9 GB if materialised):
    the frugal root and 64 sampled auth paths equal the materialised commit's."""
    import torch
    n, w = 1 << 22, 379
    g = torch.Generator(device="cuda").manual_seed(22)
    d = torch.randint(0, 2**62, (w, n), dtype=torch.int64, device="cuda", generator=g)
    idx = np.random.default_rng(4).integers(0, 4 * n, 64)
    with tv.Commitment(d.data_ptr(), width=w, trace_len=n, device_ptr=True, frugal=True) as fr:
        root_f = fr.root()
        paths_f = fr.auth_paths(idx)
    with tv.Commitment(d.data_ptr(), width=w, trace_len=n, device_ptr=True) as full:
        assert (full.root() == root_f).all()
        assert (full.auth_paths(idx) == paths_f).all()
    del d
    torch.cuda.empty_cache()
