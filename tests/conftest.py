"""Shared pytest configuration: the `gpu` marker, import paths, fixtures."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "triton-vm-prover_b200")
for p in (os.path.join(ROOT, "oracle"), PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")
P = 0xFFFFFFFF00000001


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def tv():
    """The tvmc binding; GPU tests require the CUDA library and a device."""
    import tvmc
    tvmc.lib()
    if tvmc.lib().tvmc_device_count() < 1:
        pytest.fail("no CUDA device visible to libtvmc.so")
    return tvmc


def golden(name):
    return np.load(os.path.join(GOLDEN, name))


def rand_u64(seed, shape, hi=P):
    rng = np.random.default_rng(seed)
    return rng.integers(0, hi, size=shape, dtype=np.uint64)


EDGE_VALUES = np.array([0, 1, 2, P - 1, P - 2, 2**32 - 1, 2**32, 2**32 + 1, 2**63, 7, 0xFFFFFFFE00000001,
                        P // 2, P // 2 + 1, 0xFFFFFFFF, 0x100000000FFFFFFFF % 2**64, 12345678901234567],
                       dtype=np.uint64)


def to_dev(a):
    """numpy uint64 -> CUDA int64 tensor with the same bits."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64)).cuda()


def from_dev(t):
    return t.cpu().numpy().view(np.uint64)


def dev_empty(*shape):
    import torch
    return torch.empty(*shape, dtype=torch.int64, device="cuda")


def _cudart():
    """The CUDA runtime libtvmc.so itself links (loaded with it)."""
    import ctypes
    import tvmc
    tvmc.lib()
    rt = ctypes.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    return rt


def memcpy_h2d(dst_ptr, host):
    """Synchronous host -> device copy into a raw device pointer."""
    host = np.ascontiguousarray(host)
    rc = _cudart().cudaMemcpy(dst_ptr, host.ctypes.data, host.nbytes, 1)  # cudaMemcpyHostToDevice
    assert rc == 0, rc
