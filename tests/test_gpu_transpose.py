"""Row-major -> column-major on the device (tvmc_rowmajor_to_colmajor_gpu, the
replacement of qzc_rowmajor_to_colmajor_bfe): the TMA tile path (even widths
and heights) and the shared-memory tile path give numpy's transpose for full
tiles, edge tiles and tiny tables, and a row-major commit through either path
equals the oracle."""
import numpy as np
import pytest

from conftest import dev_empty, from_dev, rand_u64, to_dev

pytestmark = pytest.mark.gpu


@pytest.fixture
def tma(tv):
    saved = tv.get_tuning("transpose_tma")
    yield tv
    tv.set_tuning("transpose_tma", saved)


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("rows,cols", [(1 << 20, 264), (1 << 12, 10), (64, 2), (2, 16), (32, 18), (96, 34),
                                       (1 << 10, 379), (1 << 16, 1), (3, 5), (1 << 22, 3), (1 << 22, 2)])
def test_transpose_equals_numpy(tma, rows, cols, mode):
    tv = tma
    tv.set_tuning("transpose_tma", mode)
    a = rand_u64(rows * 7 + cols, (rows, cols), hi=2**64 - 1)
    d_in, d_out = to_dev(a), dev_empty(rows * cols)
    lib = tv.lib()
    assert lib.tvmc_rowmajor_to_colmajor_gpu(d_in.data_ptr(), rows, cols, d_out.data_ptr(), None) == 0, \
        lib.tvmc_last_error()
    assert (from_dev(d_out).reshape(cols, rows) == a.T).all()
    assert tv.get_tuning("tma_timeouts") == 0


@pytest.mark.parametrize("mode", [1, 2])
def test_row_major_commit_through_each_transpose(tma, oracle, mode):
    tv = tma
    tv.set_tuning("transpose_tma", mode)
    t = rand_u64(9900, (264, 1 << 10))
    with tv.Commitment(np.ascontiguousarray(t.T), row_major=True) as c:
        assert (c.root() == oracle.merkle(oracle.hash_rows_cm(oracle.lde(t)))[1]).all()


def test_transpose_rejects_in_place(tv):
    d = dev_empty(16)
    assert tv.lib().tvmc_rowmajor_to_colmajor_gpu(d.data_ptr(), 4, 4, d.data_ptr(), None) == tv.ERR_INVALID
