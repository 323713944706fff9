"""Out-of-memory paths, by host-side fault injection (tuning key
"fail_alloc_after"): the k-th device allocation the library requests fails as
out-of-memory without reaching the driver, so the GPU sees no fault.  Every
allocation a commit makes is failed in turn; each failure must surface as
TVMC_ERR_NOMEM (tvmc.OutOfMemory) from the call that made it, return the device
memory the attempt had taken (the stream-ordered pool's used bytes come back
to where they were), and leave the library usable: the next commit equals the
oracle.  The reference checks free memory up front instead
(check_gpu_memory, src/gpu/gpu_stark.cu:1588-1730) and throws."""
import numpy as np
import pytest

from conftest import rand_u64

pytestmark = pytest.mark.gpu


def _expected_root(oracle, trace):
    return oracle.merkle(oracle.hash_rows_cm(oracle.lde(trace)))[1]


def _each_allocation_fails_once(tv, make, expect_root, max_allocs=64):
    import torch
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream
    with make(sp) as c:  # warm the stream's cached scratch, so later attempts allocate the same set
        assert (c.root() == expect_root).all()
    torch.cuda.synchronize()
    base = tv.get_tuning("pool_used_bytes")
    failures = 0
    try:
        for k in range(1, max_allocs + 1):
            tv.set_tuning("fail_alloc_after", k)
            try:
                with make(sp) as c:
                    root = c.root()
                tv.set_tuning("fail_alloc_after", 0)
                assert (root == expect_root).all()
                break  # the commit made fewer than k allocations
            except tv.OutOfMemory:
                failures += 1
            torch.cuda.synchronize()
            assert tv.get_tuning("pool_used_bytes") == base, f"allocation {k}: memory not returned"
        else:
            pytest.fail(f"commit still failing after {max_allocs} injected failures")
    finally:
        tv.set_tuning("fail_alloc_after", 0)
    assert failures >= 1
    with make(sp) as c:  # usable afterwards
        assert (c.root() == expect_root).all()
    torch.cuda.synchronize()
    return failures


def test_commit_from_host_each_allocation_fails_cleanly(tv, oracle):
    trace = rand_u64(4101, (23, 1 << 12))
    exp = _expected_root(oracle, trace)
    _each_allocation_fails_once(tv, lambda sp: tv.Commitment(trace, stream=sp), exp)


def test_commit_from_device_discarding_lde_each_allocation_fails_cleanly(tv, oracle):
    from conftest import to_dev
    trace = rand_u64(4102, (11, 1 << 13))
    d = to_dev(trace)
    exp = _expected_root(oracle, trace)
    _each_allocation_fails_once(
        tv, lambda sp: tv.Commitment(d.data_ptr(), width=11, trace_len=1 << 13, device_ptr=True, stream=sp,
                                     discard_lde=True), exp)


def test_randomized_and_row_major_commit_allocation_failures(tv, oracle):
    trace = rand_u64(4103, (1 << 10, 9))  # row-major
    rnd = rand_u64(4104, (9, 5))
    exp = oracle.merkle(oracle.hash_rows_cm(oracle.lde_randomized(np.ascontiguousarray(trace.T), rnd, 4, 7, 3)))[1]
    _each_allocation_fails_once(
        tv, lambda sp: tv.Commitment(trace, row_major=True, stream=sp, randomizers=rnd, trace_offset=3), exp)


def test_server_reports_an_allocation_failure_and_keeps_serving(tv, oracle):
    a, b = rand_u64(4105, (7, 1 << 10)), rand_u64(4106, (5, 1 << 11))
    with tv.Server(streams=2) as srv:
        tv.set_tuning("fail_alloc_after", 1)
        try:
            bad = srv.submit(a)
            with pytest.raises(tv.OutOfMemory):
                srv.wait(bad)
        finally:
            tv.set_tuning("fail_alloc_after", 0)
        good = srv.submit(b)
        assert (srv.wait(good) == _expected_root(oracle, b)).all()
        srv.release(good)
        st = srv.stats()
        assert st["failed"] >= 1 and st["completed"] >= 1


def test_injection_knob_roundtrip_needs_no_device(tv):
    tv.set_tuning("fail_alloc_after", 3)
    assert tv.get_tuning("fail_alloc_after") == 3
    tv.set_tuning("fail_alloc_after", 0)
    assert tv.get_tuning("fail_alloc_after") == 0
