"""Python binding of the tvmc C ABI (include/tvmc.h) via ctypes.

This is a thin host-side mirror of the reference's operator interfaces for the
table-commitment path (NTT / LDE / Tip5 / MerkleTree / table commitment).  It
loads the in-tree libtvmc.so and raises if it is missing: there is no CPU
fallback.  Host-buffer functions take numpy arrays; the *_gpu functions take
device pointers (ints), e.g. torch.Tensor.data_ptr().
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtvmc.so")
P = 0xFFFFFFFF00000001

OK, ERR_INVALID, ERR_RANGE, ERR_NOMEM, ERR_CUDA, ERR_TIMEOUT, ERR_UNSUPPORTED = range(7)

TRACE_DEVICE = 0x1
TRACE_ROW_MAJOR = 0x2
DISCARD_LDE = 0x4
SYNC = 0x8
PROFILE = 0x10
FRUGAL = 0x20
RAND_TRUNCATE = 0x40
LEAVES_XFE = 0x80

_u64p = ctypes.POINTER(ctypes.c_uint64)
_szp = ctypes.POINTER(ctypes.c_size_t)
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t


class TvmcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"tvmc status {status}: {msg}")
        self.status = status


class InvalidArgument(TvmcError, ValueError):
    pass


class OutOfRange(TvmcError, IndexError):
    pass


class Timeout(TvmcError, TimeoutError):
    pass


class OutOfMemory(TvmcError, MemoryError):
    pass


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


# Every exported symbol and its (restype, argtypes).
SIGNATURES = {
    "tvmc_last_error": (ctypes.c_char_p, []),
    "tvmc_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "tvmc_version": (ctypes.c_int, []),
    "tvmc_device_count": (ctypes.c_int, []),
    "tvmc_ntt_forward_batched_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp]),
    "tvmc_ntt_inverse_batched_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp]),
    "tvmc_ntt_host": (ctypes.c_int, [_u64p, _sz, _sz, ctypes.c_int]),
    "tvmc_lde_batch_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp, _sz, ctypes.c_uint64, ctypes.c_uint64, _vp]),
    "tvmc_lde_host": (ctypes.c_int, [_u64p, _sz, _sz, _u64p, _sz, ctypes.c_uint64]),
    "tvmc_lde_randomized_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp, _sz, _vp, _sz, ctypes.c_uint64,
                                               ctypes.c_uint64, ctypes.c_uint32, _vp]),
    "tvmc_lde_randomized_host": (ctypes.c_int, [_u64p, _sz, _sz, _u64p, _sz, _u64p, _sz, ctypes.c_uint64,
                                                ctypes.c_uint64, ctypes.c_uint32]),
    "tvmc_lde_batch_noalloc_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp, _sz, ctypes.c_uint64, ctypes.c_uint64,
                                                  _vp]),
    "tvmc_hash_bfield_rows_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "tvmc_hash_xfield_rows_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "tvmc_hash_varlen_host": (ctypes.c_int, [_u64p, _sz, _sz, _u64p]),
    "tvmc_hash_pairs_gpu": (ctypes.c_int, [_vp, _vp, _vp, _sz, _vp]),
    "tvmc_hash_pairs_host": (ctypes.c_int, [_u64p, _u64p, _u64p, _sz]),
    "tvmc_tip5_permutation_batch_gpu": (ctypes.c_int, [_vp, _sz, _vp]),
    "tvmc_tip5_permutation_batch_host": (ctypes.c_int, [_u64p, _sz]),
    "tvmc_tip5_rounds_host": (ctypes.c_int, [_u64p, _sz, ctypes.c_uint32, ctypes.c_uint32, _u64p]),
    "tvmc_tip5_parameters": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint8), _u64p, _u64p]),
    "tvmc_evaluate_on_coset_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp, _sz, ctypes.c_uint64, _vp]),
    "tvmc_evaluate_on_coset_host": (ctypes.c_int, [_u64p, _sz, _sz, _u64p, _sz, ctypes.c_uint64]),
    "tvmc_merkle_root_from_paths_gpu": (ctypes.c_int, [_vp, _vp, _vp, _sz, _sz, _vp, _vp]),
    "tvmc_merkle_root_from_paths_host": (ctypes.c_int, [_szp, _u64p, _u64p, _sz, _sz, _u64p]),
    "tvmc_merkle_tree_gpu": (ctypes.c_int, [_vp, _vp, _sz, _vp]),
    "tvmc_merkle_root_gpu": (ctypes.c_int, [_vp, _vp, _sz, _vp]),
    "tvmc_merkle_tree_heap_host": (ctypes.c_int, [_u64p, _sz, _u64p]),
    "tvmc_commit": (ctypes.c_int, [_vp, _sz, _sz, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32, _vp,
                                   ctypes.POINTER(_vp)]),
    "tvmc_commit_randomized": (ctypes.c_int, [_vp, _sz, _sz, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                                              _vp, _sz, ctypes.c_uint32, _vp, ctypes.POINTER(_vp)]),
    "tvmc_commit_rows": (ctypes.c_int, [_vp, _sz, _sz, ctypes.c_uint32, _vp, ctypes.POINTER(_vp)]),
    "tvmc_commit_digests": (ctypes.c_int, [_vp, _sz, ctypes.c_uint32, _vp, ctypes.POINTER(_vp)]),
    "tvmc_sponge_absorb_gpu": (ctypes.c_int, [_vp, _vp, _sz, _vp]),
    "tvmc_commitment_absorb_root": (ctypes.c_int, [_vp, _vp, _vp]),
    "tvmc_commitment_root": (ctypes.c_int, [_vp, _u64p]),
    "tvmc_commitment_sync": (ctypes.c_int, [_vp]),
    "tvmc_commitment_shape": (ctypes.c_int, [_vp, _szp, _szp]),
    "tvmc_commitment_device_lde": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "tvmc_commitment_device_tree": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "tvmc_commitment_auth_paths": (ctypes.c_int, [_vp, _szp, _sz, _u64p]),
    "tvmc_commitment_auth_structure": (ctypes.c_int, [_vp, _szp, _sz, _u64p, _sz, _szp]),
    "tvmc_auth_structure_indices": (ctypes.c_int, [_sz, _szp, _sz, _u64p, _sz, _szp]),
    "tvmc_commitment_read_rows": (ctypes.c_int, [_vp, _szp, _sz, _u64p]),
    "tvmc_commitment_read_columns": (ctypes.c_int, [_vp, _sz, _sz, _u64p]),
    "tvmc_commitment_read_lde": (ctypes.c_int, [_vp, _u64p, ctypes.c_int]),
    "tvmc_commitment_read_leaves": (ctypes.c_int, [_vp, _u64p]),
    "tvmc_commitment_read_nodes": (ctypes.c_int, [_vp, _u64p]),
    "tvmc_commitment_free": (ctypes.c_int, [_vp]),
    "tvmc_commitment_phase_ms": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_float)]),
    "tvmc_launch_count": (ctypes.c_ulonglong, []),
    "tvmc_batch_create": (ctypes.c_int, [_vp, _sz, ctypes.POINTER(_vp)]),
    "tvmc_batch_input": (ctypes.c_int, [_vp, _sz, ctypes.POINTER(_vp)]),
    "tvmc_batch_run": (ctypes.c_int, [_vp, _vp]),
    "tvmc_batch_commitment": (ctypes.c_int, [_vp, _sz, ctypes.POINTER(_vp)]),
    "tvmc_batch_free": (ctypes.c_int, [_vp]),
    "tvmc_release_cached_memory": (ctypes.c_int, []),
    "tvmc_forget_stream": (ctypes.c_int, [_vp]),
    "tvmc_server_create": (ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    "tvmc_server_submit": (ctypes.c_int, [_vp, _vp, _sz, _sz, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32,
                                          ctypes.POINTER(ctypes.c_uint64)]),
    "tvmc_server_submit_randomized": (ctypes.c_int, [_vp, _vp, _sz, _sz, ctypes.c_uint32, ctypes.c_uint64,
                                                     ctypes.c_uint64, _vp, _sz, ctypes.c_uint32,
                                                     ctypes.POINTER(ctypes.c_uint64)]),
    "tvmc_server_wait": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_int64, _u64p]),
    "tvmc_server_open": (ctypes.c_int, [_vp, ctypes.c_uint64, _szp, _sz, _u64p, _u64p]),
    "tvmc_server_times": (ctypes.c_int, [_vp, ctypes.c_uint64, _u64p, _u64p, _u64p]),
    "tvmc_server_release": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "tvmc_server_get_stats": (ctypes.c_int, [_vp, _vp]),
    "tvmc_server_destroy": (ctypes.c_int, [_vp]),
    "tvmc_commit_multi": (ctypes.c_int, [_vp, _sz, ctypes.c_uint32, _vp, _vp]),
    "tvmc_rowmajor_to_colmajor_gpu": (ctypes.c_int, [_vp, _sz, _sz, _vp, _vp]),
    "tvmc_set_tuning": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_longlong]),
    "tvmc_get_tuning": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_longlong)]),
}

_lib = None


def lib():
    """Load libtvmc.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build the CUDA extension first (make -C {HERE})")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status: int) -> None:
    if status == OK:
        return
    msg = lib().tvmc_last_error().decode(errors="replace")
    if status == ERR_INVALID:
        raise InvalidArgument(status, msg)
    if status == ERR_RANGE:
        raise OutOfRange(status, msg)
    if status == ERR_TIMEOUT:
        raise Timeout(status, msg)
    if status == ERR_NOMEM:
        raise OutOfMemory(status, msg)
    raise TvmcError(status, msg)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_u64p)


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint64)


# ---------------------------------------------------------------- host API

def ntt(data, inverse: bool = False) -> np.ndarray:
    """NTT::forward / NTT::inverse of each row of a (cols, n) array (or a 1-D array)."""
    a = _u64(data).copy()
    cols, n = (1, a.size) if a.ndim == 1 else a.shape
    _check(lib().tvmc_ntt_host(_p(a), n, cols, int(inverse)))
    return a


def lde_randomized(trace_cm, randomizers, expansion: int = 4, offset: int = 7, trace_offset: int = 1,
                   truncate: bool = False) -> np.ndarray:
    """RandomizedLDE::extend_column_with_randomizer on each row of (width, n);
    randomizers is (width, R).  truncate selects the XFieldElement variants' truncation."""
    t = _u64(trace_cm)
    w, n = t.shape
    r = _u64(randomizers).reshape(w, -1)
    out = np.empty((w, n * expansion), dtype=np.uint64)
    _check(lib().tvmc_lde_randomized_host(_p(t), w, n, _p(r) if r.size else None, r.shape[1], _p(out),
                                          n * expansion, trace_offset, offset, RAND_TRUNCATE if truncate else 0))
    return out


def evaluate_on_coset(coeffs, domain_len: int, offset: int) -> np.ndarray:
    """NTT::evaluate_on_coset of each row of a (cols, n) array (or a 1-D array)."""
    a = _u64(coeffs)
    one = a.ndim == 1
    a2 = a.reshape(1, -1) if one else a
    cols, n = a2.shape
    out = np.empty((cols, domain_len), dtype=np.uint64)
    _check(lib().tvmc_evaluate_on_coset_host(_p(a2) if a2.size else None, n, cols, _p(out), domain_len, offset))
    return out[0] if one else out


def tip5_rounds(states, first_round: int, num_rounds: int, trace: bool = False):
    """Tip5 rounds on (count, 16) states; with trace, also (count, num_rounds, 16)."""
    s = _u64(states).reshape(-1, 16).copy()
    tr = np.zeros((s.shape[0], num_rounds, 16), dtype=np.uint64) if trace else None
    _check(lib().tvmc_tip5_rounds_host(_p(s), s.shape[0], first_round, num_rounds,
                                       _p(tr) if trace and tr.size else None))
    return (s, tr) if trace else s


def tip5_parameters():
    """(lookup table (256,) u8, MDS first column (16,), round constants (80,))."""
    lk = np.zeros(256, dtype=np.uint8)
    mds = np.zeros(16, dtype=np.uint64)
    rc = np.zeros(80, dtype=np.uint64)
    _check(lib().tvmc_tip5_parameters(lk.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), _p(mds), _p(rc)))
    return lk, mds, rc


def merkle_roots_from_paths(leaf_idx, leaves, paths) -> np.ndarray:
    """Root implied by each (index, leaf digest, path (len, 5)) triple."""
    ix = np.ascontiguousarray(leaf_idx, dtype=np.uintp)
    lv = _u64(leaves).reshape(-1, 5)
    pp = _u64(paths).reshape(ix.size, -1, 5)
    out = np.zeros((ix.size, 5), dtype=np.uint64)
    _check(lib().tvmc_merkle_root_from_paths_host(ix.ctypes.data_as(_szp), _p(lv), _p(pp) if pp.size else None,
                                                  ix.size, pp.shape[1], _p(out)))
    return out


def lde(trace_cm, expansion: int = 4, offset: int = 7) -> np.ndarray:
    """LDE::extend_table on column-major (width, n) data -> (width, n*expansion)."""
    t = _u64(trace_cm)
    w, n = t.shape
    out = np.empty((w, n * expansion), dtype=np.uint64)
    _check(lib().tvmc_lde_host(_p(t), w, n, _p(out), n * expansion, offset))
    return out


def hash_varlen_rows(rows_rm) -> np.ndarray:
    """Tip5::hash_varlen of every row of a row-major (rows, len) array -> (rows, 5)."""
    t = _u64(rows_rm)
    r, w = t.shape
    out = np.zeros((r, 5), dtype=np.uint64)
    _check(lib().tvmc_hash_varlen_host(_p(t) if t.size else _p(np.zeros(1, np.uint64)), r, w, _p(out)))
    return out


def hash_pairs(left, right) -> np.ndarray:
    l, r = _u64(left).reshape(-1, 5), _u64(right).reshape(-1, 5)
    out = np.zeros_like(l)
    _check(lib().tvmc_hash_pairs_host(_p(l), _p(r), _p(out), l.shape[0]))
    return out


def tip5_permutations(states) -> np.ndarray:
    s = _u64(states).reshape(-1, 16).copy()
    _check(lib().tvmc_tip5_permutation_batch_host(_p(s), s.shape[0]))
    return s


def merkle_heap(leaves) -> np.ndarray:
    lv = _u64(leaves).reshape(-1, 5)
    n = lv.shape[0]
    nodes = np.zeros((2 * n, 5), dtype=np.uint64)
    _check(lib().tvmc_merkle_tree_heap_host(_p(lv), n, _p(nodes)))
    return nodes


def set_tuning(key: str, value: int) -> None:
    _check(lib().tvmc_set_tuning(key.encode(), int(value)))


def release_cached_memory() -> None:
    """Free the per-stream scratch and trim the device pool (synchronizes)."""
    _check(lib().tvmc_release_cached_memory())


def forget_stream(stream) -> None:
    """Free the library's cached buffers for a stream about to be destroyed."""
    _check(lib().tvmc_forget_stream(_stream(stream)))


def get_tuning(key: str) -> int:
    v = ctypes.c_longlong(0)
    _check(lib().tvmc_get_tuning(key.encode(), ctypes.byref(v)))
    return v.value


def auth_structure_indices(num_leaves: int, leaves) -> np.ndarray:
    """Heap indices of MerkleTree::authentication_structure, descending (host only)."""
    ix = np.ascontiguousarray(leaves, dtype=np.uintp)
    cap = max(1, ix.size * 64)
    out = np.zeros(cap, dtype=np.uint64)
    cnt = ctypes.c_size_t(0)
    _check(lib().tvmc_auth_structure_indices(num_leaves, ix.ctypes.data_as(_szp), ix.size, _p(out), cap,
                                             ctypes.byref(cnt)))
    return out[: cnt.value]


# ---------------------------------------------------------------- device API

def _stream(stream) -> int | None:
    if stream is None:
        return None
    return int(getattr(stream, "cuda_stream", stream))


def ntt_gpu(d_data: int, n: int, cols: int, inverse: bool = False, stream=None) -> None:
    f = lib().tvmc_ntt_inverse_batched_gpu if inverse else lib().tvmc_ntt_forward_batched_gpu
    _check(f(d_data, n, cols, _stream(stream)))


def lde_gpu(d_trace: int, cols: int, n: int, d_out: int, L: int, offset: int = 7, stream=None) -> None:
    _check(lib().tvmc_lde_batch_gpu(d_trace, cols, n, d_out, L, 1, offset, _stream(stream)))


def lde_randomized_gpu(d_trace: int, cols: int, n: int, d_rnd: int, R: int, d_out: int, L: int, offset: int = 7,
                       trace_offset: int = 1, truncate: bool = False, stream=None) -> None:
    _check(lib().tvmc_lde_randomized_gpu(d_trace, cols, n, d_rnd or None, R, d_out, L, trace_offset, offset,
                                         RAND_TRUNCATE if truncate else 0, _stream(stream)))


def sponge_absorb_gpu(d_state: int, d_data: int, length: int, stream=None) -> None:
    _check(lib().tvmc_sponge_absorb_gpu(d_state, d_data or None, length, _stream(stream)))


def hash_rows_gpu(d_table: int, rows: int, cols: int, d_digests: int, stream=None) -> None:
    _check(lib().tvmc_hash_bfield_rows_gpu(d_table, rows, cols, d_digests, _stream(stream)))


def hash_xfield_rows_gpu(d_table: int, rows: int, xfe_cols: int, d_digests: int, stream=None) -> None:
    _check(lib().tvmc_hash_xfield_rows_gpu(d_table, rows, xfe_cols, d_digests, _stream(stream)))


def hash_pairs_gpu(d_left: int, d_right: int, d_out: int, count: int, stream=None) -> None:
    _check(lib().tvmc_hash_pairs_gpu(d_left, d_right, d_out, count, _stream(stream)))


def tip5_permutations_gpu(d_states: int, count: int, stream=None) -> None:
    _check(lib().tvmc_tip5_permutation_batch_gpu(d_states, count, _stream(stream)))


def merkle_tree_gpu(d_leaves: int, d_tree: int, n: int, stream=None) -> None:
    _check(lib().tvmc_merkle_tree_gpu(d_leaves, d_tree, n, _stream(stream)))


def merkle_root_gpu(d_leaves: int, d_root: int, n: int, stream=None) -> None:
    _check(lib().tvmc_merkle_root_gpu(d_leaves, d_root, n, _stream(stream)))


# ---------------------------------------------------------------- commitment

class MultiTable(ctypes.Structure):
    _fields_ = [("trace", ctypes.c_void_p), ("trace_len", ctypes.c_size_t), ("width", ctypes.c_size_t),
                ("expansion", ctypes.c_uint32), ("offset", ctypes.c_uint64)]


def commit_multi(traces, expansion: int = 4, offset: int = 7, device_ptr: bool = False, shapes=None,
                 discard_lde: bool = False, stream=None, sync: bool = False) -> list:
    """tvmc_commit_multi: several plain commitments with one multi-table row
    hash.  traces: host (width, n) arrays, or with device_ptr=True device
    pointers with shapes = [(n, width), ...]."""
    descs, keep = [], []
    for i, t in enumerate(traces):
        if device_ptr:
            n, w = shapes[i]
            ptr = int(t)
        else:
            a = _u64(t)
            w, n = a.shape
            keep.append(a)
            ptr = a.ctypes.data if a.size else None
        descs.append(MultiTable(ptr, n, w, expansion, offset))
    arr = (MultiTable * max(1, len(descs)))(*descs)
    hs = (_vp * max(1, len(descs)))()
    flags = (TRACE_DEVICE if device_ptr else 0) | (DISCARD_LDE if discard_lde else 0) | (SYNC if sync else 0)
    _check(lib().tvmc_commit_multi(ctypes.cast(arr, _vp), len(descs), flags, _stream(stream), ctypes.cast(hs, _vp)))
    out = []
    for d, h in zip(descs, hs[:len(descs)]):
        c = Commitment._wrap(_vp(h), d.width, d.trace_len * expansion, keep)
        c.trace_len = d.trace_len
        out.append(c)
    return out


class Commitment:
    """A committed table: device-resident LDE (column-major) and heap tree.

    Mirrors the reference's TableCommitment / MerkleTree accessors
    (include/table/table_commitment.hpp, include/merkle/merkle_tree.hpp)."""

    def __init__(self, trace, width: int | None = None, trace_len: int | None = None, expansion: int = 4,
                 offset: int = 7, row_major: bool = False, device_ptr: bool = False, discard_lde: bool = False,
                 stream=None, sync: bool = False, profile: bool = False, frugal: bool = False,
                 randomizers=None, trace_offset: int = 1, truncate: bool = False):
        """randomizers: host (width, R) array, or with device_ptr=True a device
        pointer to width*R words given as (pointer, R)."""
        flags = (PROFILE if profile else 0) | (FRUGAL if frugal else 0) | (RAND_TRUNCATE if truncate else 0)
        if device_ptr:
            flags |= TRACE_DEVICE
            ptr = int(trace)
            self._keep = None
            assert width is not None and trace_len is not None
        else:
            t = _u64(trace)
            if row_major:
                trace_len, width = t.shape
            else:
                width, trace_len = t.shape
            self._keep = t  # the host buffer must live until the upload is done
            ptr = t.ctypes.data if t.size else None
        if row_major:
            flags |= TRACE_ROW_MAJOR
        if discard_lde:
            flags |= DISCARD_LDE
        if sync:
            flags |= SYNC
        rptr, R = None, 0
        if randomizers is not None:
            if device_ptr:
                rptr, R = int(randomizers[0]), int(randomizers[1])
            else:
                r = _u64(randomizers).reshape(width, -1)
                self._keep_r = r
                rptr, R = (r.ctypes.data if r.size else None), r.shape[1]
        h = _vp()
        _check(lib().tvmc_commit_randomized(ptr, trace_len, width, expansion, trace_offset, offset, rptr, R, flags,
                                            _stream(stream), ctypes.byref(h)))
        self.h = h
        self.width = width
        self.trace_len = trace_len
        self.lde_len = trace_len * expansion

    @classmethod
    def _wrap(cls, h, width, rows, keep=None):
        obj = cls.__new__(cls)
        obj.h, obj.width, obj.trace_len, obj.lde_len, obj._keep = h, width, rows, rows, keep
        return obj

    @classmethod
    def from_rows(cls, table, row_major: bool = False, width: int | None = None, rows: int | None = None,
                  device_ptr: bool = False, discard: bool = False, stream=None, sync: bool = False):
        """tvmc_commit_rows: leaves = Tip5 hash of each row of an already evaluated
        table (numpy (width, rows), or (rows, width) with row_major), no LDE."""
        flags = (TRACE_ROW_MAJOR if row_major else 0) | (DISCARD_LDE if discard else 0) | (SYNC if sync else 0)
        if device_ptr:
            flags |= TRACE_DEVICE
            ptr, keep = int(table), None
        else:
            t = _u64(table)
            rows, width = t.shape if row_major else t.shape[::-1]
            ptr, keep = (t.ctypes.data if t.size else None), t
        h = _vp()
        _check(lib().tvmc_commit_rows(ptr, rows, width, flags, _stream(stream), ctypes.byref(h)))
        return cls._wrap(h, width, rows, keep)

    @classmethod
    def from_digests(cls, leaves, xfe: bool = False, count: int | None = None, device_ptr: bool = False,
                     stream=None, sync: bool = False):
        """tvmc_commit_digests: a tree over (n, 5) leaf digests, or with xfe=True over an
        (n, 3) XFieldElement codeword (leaf = (c0, c1, c2, 0, 0))."""
        flags = (LEAVES_XFE if xfe else 0) | (SYNC if sync else 0)
        if device_ptr:
            flags |= TRACE_DEVICE
            ptr, keep = int(leaves), None
        else:
            lv = _u64(leaves).reshape(-1, 3 if xfe else 5)
            count, ptr, keep = lv.shape[0], lv.ctypes.data, lv
        h = _vp()
        _check(lib().tvmc_commit_digests(ptr, count, flags, _stream(stream), ctypes.byref(h)))
        return cls._wrap(h, 0, count, keep)

    def _h(self):
        if self.h is None:
            raise ValueError("commitment already freed")
        return self.h

    def absorb_root(self, d_state: int, stream=None) -> None:
        """Absorb the root (as proof item MerkleRoot) into a device sponge state."""
        _check(lib().tvmc_commitment_absorb_root(self._h(), d_state, _stream(stream)))

    def sync(self) -> None:
        _check(lib().tvmc_commitment_sync(self._h()))
        self._keep = None

    def root(self) -> np.ndarray:
        out = np.zeros(5, dtype=np.uint64)
        _check(lib().tvmc_commitment_root(self._h(), _p(out)))
        self._keep = None
        return out

    @property
    def height(self) -> int:
        return self.lde_len.bit_length() - 1

    def auth_paths(self, leaves) -> np.ndarray:
        ix = np.ascontiguousarray(leaves, dtype=np.uintp)
        out = np.zeros((ix.size, self.height, 5), dtype=np.uint64)
        _check(lib().tvmc_commitment_auth_paths(self._h(), ix.ctypes.data_as(_szp), ix.size,
                                                _p(out) if out.size else None))
        return out

    def auth_structure(self, leaves) -> np.ndarray:
        ix = np.ascontiguousarray(leaves, dtype=np.uintp)
        cap = max(1, ix.size * max(1, self.height))
        out = np.zeros((cap, 5), dtype=np.uint64)
        cnt = ctypes.c_size_t(0)
        _check(lib().tvmc_commitment_auth_structure(self._h(), ix.ctypes.data_as(_szp), ix.size, _p(out), cap,
                                                    ctypes.byref(cnt)))
        return out[: cnt.value]

    def read_rows(self, rows) -> np.ndarray:
        ix = np.ascontiguousarray(rows, dtype=np.uintp)
        out = np.zeros((ix.size, self.width), dtype=np.uint64)
        _check(lib().tvmc_commitment_read_rows(self._h(), ix.ctypes.data_as(_szp), ix.size,
                                               _p(out) if out.size else None))
        return out

    def read_columns(self, col0: int, ncols: int) -> np.ndarray:
        out = np.zeros((ncols, self.lde_len), dtype=np.uint64)
        _check(lib().tvmc_commitment_read_columns(self._h(), col0, ncols, _p(out) if out.size else None))
        return out

    def lde(self, row_major: bool = False) -> np.ndarray:
        shape = (self.lde_len, self.width) if row_major else (self.width, self.lde_len)
        out = np.zeros(shape, dtype=np.uint64)
        _check(lib().tvmc_commitment_read_lde(self._h(), _p(out) if out.size else None, int(row_major)))
        return out

    def leaves(self) -> np.ndarray:
        out = np.zeros((self.lde_len, 5), dtype=np.uint64)
        _check(lib().tvmc_commitment_read_leaves(self._h(), _p(out)))
        return out

    def nodes(self) -> np.ndarray:
        out = np.zeros((2 * self.lde_len, 5), dtype=np.uint64)
        _check(lib().tvmc_commitment_read_nodes(self._h(), _p(out)))
        return out

    def phase_ms(self) -> tuple[float, float, float]:
        """(upload, LDE, row hash + tree) device milliseconds of a profiled commit."""
        ms = (ctypes.c_float * 3)()
        _check(lib().tvmc_commitment_phase_ms(self._h(), ms))
        return ms[0], ms[1], ms[2]

    def device_lde(self) -> int:
        p = _vp()
        _check(lib().tvmc_commitment_device_lde(self._h(), ctypes.byref(p)))
        return p.value or 0

    def device_tree(self) -> int:
        p = _vp()
        _check(lib().tvmc_commitment_device_tree(self._h(), ctypes.byref(p)))
        return p.value or 0

    def free(self) -> None:
        if self.h is not None:
            lib().tvmc_commitment_free(self.h)
            self.h = None
            self._keep = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()


class TableShape(ctypes.Structure):
    """tvmc_table_shape."""
    _fields_ = [("trace_len", ctypes.c_size_t), ("width", ctypes.c_size_t), ("expansion", ctypes.c_uint32),
                ("offset", ctypes.c_uint64)]


class _BatchTable(Commitment):
    """A batch-owned commitment handle: accessors only, freed with its batch."""

    def __init__(self, h, width, trace_len, expansion):  # noqa: D401 - no commit here
        self.h = h
        self.width = width
        self.trace_len = trace_len
        self.lde_len = trace_len * expansion
        self._keep = None

    def free(self) -> None:
        self.h = None


class Batch:
    """Many tables of uneven heights/widths committed by one CUDA-graph launch.

    shapes: list of (trace_len, width[, expansion=4[, offset=7]])."""

    def __init__(self, shapes):
        norm = [tuple(s) + (4, 7)[len(s) - 2:] for s in shapes]
        arr = (TableShape * len(norm))(*[TableShape(n, w, e, o) for n, w, e, o in norm])
        h = _vp()
        _check(lib().tvmc_batch_create(ctypes.cast(arr, _vp), len(norm), ctypes.byref(h)))
        self.h = h
        self.shapes = norm
        self.tables = []
        for i, (n, w, e, _o) in enumerate(norm):
            c = _vp()
            _check(lib().tvmc_batch_commitment(self.h, i, ctypes.byref(c)))
            self.tables.append(_BatchTable(c, w, n, e))

    def input_ptr(self, i: int) -> int:
        p = _vp()
        _check(lib().tvmc_batch_input(self.h, i, ctypes.byref(p)))
        return p.value or 0

    def run(self, stream=None) -> None:
        _check(lib().tvmc_batch_run(self.h, _stream(stream)))

    def roots(self) -> np.ndarray:
        return np.stack([t.root() for t in self.tables])

    def free(self) -> None:
        if self.h is not None:
            for t in self.tables:
                t.free()
            lib().tvmc_batch_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.free()


SERVER_KEEP_LDE = 0x1
SERVER_GROUP_SMALL = 0x2


class ServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_size_t), ("num_streams", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("max_large_inflight", ctypes.c_uint32)]


class ServerStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in ("submitted", "completed", "failed", "released", "queued",
                                                "running")] + \
               [(k, ctypes.c_size_t) for k in ("bytes_in_use", "bytes_peak", "budget")]


class Server:
    """Commitment serving loop (tvmc_server_*): HBM-budget admission, requests
    dispatched over worker streams as they arrive, trees kept on the device
    for openings until release."""

    def __init__(self, hbm_budget_bytes: int = 0, streams: int = 4, keep_lde: bool = False, max_large: int = 0,
                 group_small: bool = False):
        flags = (SERVER_KEEP_LDE if keep_lde else 0) | (SERVER_GROUP_SMALL if group_small else 0)
        cfg = ServerConfig(hbm_budget_bytes, streams, flags, max_large)
        h = _vp()
        _check(lib().tvmc_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.h = h
        self.keep_lde = keep_lde
        self._meta = {}  # id -> (height, width, trace buffer kept alive until committed)

    def submit(self, trace, expansion: int = 4, offset: int = 7, row_major: bool = False, frugal: bool = False,
               width: int | None = None, trace_len: int | None = None, device_ptr: bool = False,
               randomizers=None, trace_offset: int = 1, truncate: bool = False) -> int:
        """randomizers: host (width, R) array, or with device_ptr=True (pointer, R)."""
        flags = (TRACE_ROW_MAJOR if row_major else 0) | (FRUGAL if frugal else 0) | \
            (RAND_TRUNCATE if truncate else 0)
        if device_ptr:
            flags |= TRACE_DEVICE
            ptr, keep = int(trace), None
        else:
            t = _u64(trace)
            trace_len, width = t.shape if row_major else t.shape[::-1]
            ptr, keep = (t.ctypes.data if t.size else None), t
        rptr, R = None, 0
        if randomizers is not None:
            if device_ptr:
                rptr, R = int(randomizers[0]), int(randomizers[1])
            else:
                r = _u64(randomizers).reshape(width, -1)
                rptr, R = (r.ctypes.data if r.size else None), r.shape[1]
                keep = (keep, r)
        rid = ctypes.c_uint64(0)
        _check(lib().tvmc_server_submit_randomized(self.h, ptr, trace_len, width, expansion, trace_offset, offset,
                                                   rptr, R, flags, ctypes.byref(rid)))
        self._meta[rid.value] = ((trace_len * expansion).bit_length() - 1, width, keep)
        return rid.value

    def wait(self, rid: int, timeout_ms: int = -1) -> np.ndarray:
        root = np.zeros(5, dtype=np.uint64)
        _check(lib().tvmc_server_wait(self.h, rid, timeout_ms, _p(root)))
        h, w, _ = self._meta[rid]
        self._meta[rid] = (h, w, None)
        return root

    def open(self, rid: int, leaves, rows: bool = False):
        h, w, _ = self._meta[rid]
        ix = np.ascontiguousarray(leaves, dtype=np.uintp)
        paths = np.zeros((ix.size, h, 5), dtype=np.uint64)
        rr = np.zeros((ix.size, w), dtype=np.uint64) if rows else None
        _check(lib().tvmc_server_open(self.h, rid, ix.ctypes.data_as(_szp), ix.size,
                                      _p(paths) if paths.size else None,
                                      _p(rr) if rows and rr.size else None))
        return (paths, rr) if rows else paths

    def times(self, rid: int):
        """(submit, start, done) in time.monotonic_ns() nanoseconds."""
        a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        _check(lib().tvmc_server_times(self.h, rid, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def release(self, rid: int) -> None:
        _check(lib().tvmc_server_release(self.h, rid))
        self._meta.pop(rid, None)

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().tvmc_server_get_stats(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self) -> None:
        if self.h is not None:
            lib().tvmc_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
