"""The scratch-free LDE entry point, tvmc_lde_batch_noalloc_gpu.

Some callers of this library cannot allocate device memory at the moment they
need an LDE: a prover whose GPU memory was reserved up front by another
framework or memory manager, or a latency-critical proving loop that must not
hit cudaMalloc/cudaFree and the synchronisation they can imply.  For them the
library offers the same LDE with its intermediates and twiddle tables in one
static device array.  This file checks, through the C ABI, that it returns
exactly what the allocating entry point (tvmc_lde_batch_gpu) returns -- the
path is integer arithmetic mod p, so the tolerance is zero -- on two calls in a
row that share the static array, and that sizes beyond the array are refused.

The file name makes pytest collect it last.
"""
import numpy as np
import pytest

from conftest import dev_empty, from_dev, rand_u64, to_dev

pytestmark = pytest.mark.gpu


def _both(tv, trace, expansion, offset):
    import torch
    w, n = trace.shape
    L = n * expansion
    d_trace = to_dev(trace)
    d_ref, d_new = dev_empty(w * L), dev_empty(w * L)
    lib = tv.lib()
    assert lib.tvmc_lde_batch_gpu(d_trace.data_ptr(), w, n, d_ref.data_ptr(), L, 1, offset, None) == 0, \
        lib.tvmc_last_error()
    assert lib.tvmc_lde_batch_noalloc_gpu(d_trace.data_ptr(), w, n, d_new.data_ptr(), L, 1, offset, None) == 0, \
        lib.tvmc_last_error()
    torch.cuda.synchronize()
    return from_dev(d_ref).reshape(w, L), from_dev(d_new).reshape(w, L)


def test_noalloc_lde_equals_allocating_lde_on_two_consecutive_calls(tv):
    # 1st call: 2^20 rows x 3 columns, x4 onto the coset 7*<w> -- one column per
    # pass through the static array, so the array is reused three times.
    ref, new = _both(tv, rand_u64(101, (3, 1 << 20)), 4, 7)
    assert (new == ref).all()
    # 2nd call right after: another size, expansion and offset, so the tables
    # and intermediates left by the first call must all be overwritten.
    ref, new = _both(tv, rand_u64(102, (5, 1 << 13)), 8, 3)
    assert (new == ref).all()


@pytest.mark.parametrize("width,log_n,expansion,offset", [
    (7, 6, 4, 7),    # small-LDE kernel (whole columns per CTA)
    (2, 0, 2, 7),    # one-row traces
    (1, 16, 1, 7),   # expansion 1
    (1, 18, 16, 5),  # expansion 16: the largest coset-scale tables
])
def test_noalloc_lde_equals_allocating_lde_across_kernel_paths(tv, width, log_n, expansion, offset):
    ref, new = _both(tv, rand_u64(200 + log_n, (width, 1 << log_n)), expansion, offset)
    assert (new == ref).all()


def test_noalloc_lde_repeated_and_changed_parameters(tv):
    # the same size and offset twice (the second call reuses the tables already
    # in the array), then a different offset at the same size, then back again
    for seed, offset in ((300, 7), (301, 7), (302, 3), (303, 7)):
        ref, new = _both(tv, rand_u64(seed, (3, 1 << 12)), 4, offset)
        assert (new == ref).all(), offset


def test_noalloc_lde_refuses_sizes_beyond_the_static_array(tv):
    lib = tv.lib()
    d = dev_empty(8)
    # 2^21 rows at expansion 4 need 2^21 * 5 words per column > the array
    rc = lib.tvmc_lde_batch_noalloc_gpu(d.data_ptr(), 1, 1 << 21, d.data_ptr(), 1 << 23, 1, 7, None)
    assert rc == tv.ERR_UNSUPPORTED
    assert b"static scratch" in lib.tvmc_last_error()
    # the size rules are the allocating entry point's own
    rc = lib.tvmc_lde_batch_noalloc_gpu(d.data_ptr(), 1, 12, d.data_ptr(), 48, 1, 7, None)
    assert rc == tv.ERR_INVALID and b"power of 2" in lib.tvmc_last_error()
