"""Batched NTT and LDE on the GPU vs the oracle (bit-exact)."""
import numpy as np
import pytest

from conftest import dev_empty, from_dev, golden, rand_u64, to_dev

pytestmark = pytest.mark.gpu


def test_ntt_golden(tv):
    g = golden("ntt.npz")
    for k in range(10):
        assert (tv.ntt(g[f"in{k}"]) == g[f"fwd{k}"]).all(), k
        assert (tv.ntt(g[f"in{k}"], inverse=True) == g[f"inv{k}"]).all(), k


@pytest.mark.parametrize("logn", [10, 11, 12, 13, 14, 15, 16, 17])
def test_ntt_sizes_vs_oracle(tv, oracle, logn):
    cols = 3
    a = rand_u64(logn, (cols, 1 << logn))
    f = tv.ntt(a)
    i = tv.ntt(a, inverse=True)
    for c in range(cols):
        assert (f[c] == oracle.ntt(a[c])).all()
        assert (i[c] == oracle.ntt(a[c], inverse=True)).all()


@pytest.mark.parametrize("logn", [20, 24])
def test_ntt_large(tv, oracle, logn):
    a = rand_u64(logn, 1 << logn)
    d = to_dev(a)
    tv.ntt_gpu(d.data_ptr(), 1 << logn, 1)
    f = from_dev(d)
    assert (f == oracle.ntt(a)).all()
    tv.ntt_gpu(d.data_ptr(), 1 << logn, 1, inverse=True)
    assert (from_dev(d) == a).all()


def test_ntt_many_columns_device(tv, oracle):
    n, cols = 1 << 13, 70
    a = rand_u64(77, (cols, n))
    d = to_dev(a)
    tv.ntt_gpu(d.data_ptr(), n, cols)
    f = from_dev(d).reshape(cols, n)
    for c in (0, 1, 35, 69):
        assert (f[c] == oracle.ntt(a[c])).all()


def test_ntt_rejects_bad_sizes(tv):
    with pytest.raises(tv.InvalidArgument):
        tv.ntt(np.zeros(12, np.uint64))
    with pytest.raises(tv.TvmcError):
        d = dev_empty(1)
        tv.ntt_gpu(d.data_ptr(), 1 << 25, 1)


@pytest.mark.parametrize("logn", list(range(0, 15)))
def test_lde_sizes_vs_oracle(tv, oracle, logn):
    w = 5 if logn < 12 else 2
    t = rand_u64(1000 + logn, (w, 1 << logn))
    assert (tv.lde(t) == oracle.lde(t)).all()


@pytest.mark.parametrize("expansion", [1, 2, 8, 16])
@pytest.mark.parametrize("logn", [3, 11, 13])
def test_lde_expansions(tv, oracle, logn, expansion):
    t = rand_u64(logn * 31 + expansion, (3, 1 << logn))
    assert (tv.lde(t, expansion=expansion) == oracle.lde(t, expansion=expansion)).all()


def test_lde_other_offset(tv, oracle):
    t = rand_u64(5, (4, 1 << 12))
    assert (tv.lde(t, offset=3) == oracle.lde(t, offset=3)).all()
    assert (tv.lde(t, offset=1) == oracle.lde(t, offset=1)).all()


def test_lde_golden(tv):
    for name in ("commit_w23_n64", "commit_w379_n4", "commit_w264_n8", "commit_w1_n1"):
        g = golden(f"{name}.npz")
        assert (tv.lde(g["trace"]) == g["lde"]).all(), name


@pytest.mark.parametrize("logn", [16, 20, 22])
def test_lde_large_column(tv, oracle, logn):
    t = rand_u64(logn, (1, 1 << logn))
    d_t = to_dev(t)
    d_o = dev_empty(4 << logn)
    tv.lde_gpu(d_t.data_ptr(), 1, 1 << logn, d_o.data_ptr(), 4 << logn)
    assert (from_dev(d_o) == oracle.lde(t)[0]).all()


def test_lde_noncanonical_input(tv, oracle):
    t = rand_u64(6, (2, 1 << 13), hi=2**64 - 1)
    assert (tv.lde(t) == oracle.lde(t)).all()


def test_lde_unsupported_sizes(tv):
    with pytest.raises(tv.TvmcError) as e:
        d = dev_empty(1)
        tv.lde_gpu(d.data_ptr(), 1, 1 << 23, d.data_ptr(), 1 << 25)
    assert e.value.status == tv.ERR_UNSUPPORTED
