"""The C ABI library loads, exports every symbol include/tvmc.h declares, and its
host-side logic (argument checks, auth-structure indices) behaves like the
reference -- all without touching a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "tvmc.h")


def declared_symbols(path):
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tvmc_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    import tvmc
    L = tvmc.lib()
    names = declared_symbols(HEADER)
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers all of them
    assert set(names) <= set(tvmc.SIGNATURES), set(names) - set(tvmc.SIGNATURES)


def test_library_fails_loudly_when_missing(tmp_path, monkeypatch):
    import tvmc
    monkeypatch.setattr(tvmc, "_lib", None)
    monkeypatch.setattr(tvmc, "LIB_PATH", str(tmp_path / "libtvmc.so"))
    with pytest.raises(FileNotFoundError):
        tvmc.lib()


def test_status_strings_and_version():
    import tvmc
    L = tvmc.lib()
    assert L.tvmc_version() >= 1
    assert L.tvmc_status_string(0) == b"ok"
    assert L.tvmc_status_string(2) == b"index out of range"
    assert L.tvmc_device_count() >= 0


def test_size_checks_need_no_gpu():
    import tvmc
    with pytest.raises(tvmc.InvalidArgument, match="power of 2"):
        tvmc.ntt(np.zeros(6, np.uint64))
    with pytest.raises(tvmc.InvalidArgument, match="power of 2"):
        tvmc.lde(np.zeros((2, 12), np.uint64))
    with pytest.raises(tvmc.InvalidArgument, match="power of 2"):
        tvmc.merkle_heap(np.zeros((3, 5), np.uint64))
    with pytest.raises(tvmc.TvmcError) as e:
        tvmc.lde(np.zeros((1, 4), np.uint64), expansion=32)
    assert e.value.status == tvmc.ERR_UNSUPPORTED
    with pytest.raises(tvmc.InvalidArgument):
        tvmc.Commitment(np.zeros((2, 8), np.uint64), expansion=3)


def test_auth_structure_indices_match_oracle(oracle):
    import tvmc
    rng = np.random.default_rng(11)
    for n in (1, 2, 8, 64, 1024):
        for m in (1, 2, 5, 16):
            idx = rng.integers(0, n, m)
            got = tvmc.auth_structure_indices(n, idx)
            exp = oracle.auth_structure_indices(n, idx)
            assert (got == exp).all(), (n, idx)
    with pytest.raises(tvmc.OutOfRange):
        tvmc.auth_structure_indices(8, [8])
    with pytest.raises(tvmc.InvalidArgument):
        tvmc.auth_structure_indices(6, [1])


def test_tip5_parameters_match_oracle(oracle):
    """The Tip5 tables the library exports (for the C++ Tip5 statics) equal the
    oracle's, whose permutation is pinned by the upstream known-answer tests."""
    import tvmc
    lk, mds, rc = tvmc.tip5_parameters()
    olk = np.zeros(256, np.uint8)
    omds = np.zeros(16, np.uint64)
    orc = np.zeros(80, np.uint64)
    oracle.L.tvmo_tip5_parameters(olk.ctypes.data_as(ctypes.c_void_p), omds.ctypes.data_as(ctypes.c_void_p),
                                  orc.ctypes.data_as(ctypes.c_void_p))
    assert (lk == olk).all() and (mds == omds).all() and (rc == orc).all()
    assert sorted(lk.tolist()) == list(range(256))  # a permutation of the bytes
