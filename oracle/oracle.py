"""ctypes wrappers for the CPU checkers (TEST INFRASTRUCTURE ONLY).

`Oracle` wraps liboracle.so, the plain-C restatement of the reference's CPU
path (tvm_oracle.c).  `RefLib` wraps _ref/libtvm_ref.so, the reference's own
C++ sources compiled unchanged (built only where the reference tree exists; it
then travels as a prebuilt file).  Only tests, the smoke check and the
benchmark's CPU-baseline leg may use this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
P = 0xFFFFFFFF00000001
# The reference source tree: environment variable REF (the Makefiles under
# oracle/, tests/cpp/ and triton-vm-prover_b200/cpp/ read the same variable).
# Only present on the development host; the GPU host uses the prebuilt files.
REF_DIR = os.environ.get("REF", "/root/reference")

_u64p = ctypes.POINTER(ctypes.c_uint64)
_szp = ctypes.POINTER(ctypes.c_size_t)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_u64p)


def build(ref: bool = True) -> None:
    """Compile liboracle.so (always) and _ref/libtvm_ref.so (when the
    reference sources are present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if ref and os.path.isdir(os.path.join(REF_DIR, "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_DIR}"], check=True)


class Oracle:
    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = ctypes.CDLL(path)
        self.L = L
        for name in ("tvmo_add", "tvmo_sub", "tvmo_mul", "tvmo_pow"):
            f = getattr(L, name)
            f.restype = ctypes.c_uint64
            f.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.tvmo_inverse.restype = ctypes.c_uint64
        L.tvmo_inverse.argtypes = [ctypes.c_uint64]
        L.tvmo_primitive_root.restype = ctypes.c_uint64
        L.tvmo_primitive_root.argtypes = [ctypes.c_uint32]
        L.tvmo_ntt_forward.argtypes = [_u64p, ctypes.c_size_t]
        L.tvmo_ntt_inverse.argtypes = [_u64p, ctypes.c_size_t]
        L.tvmo_lde_table.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, _u64p, ctypes.c_size_t,
                                     ctypes.c_uint64]
        L.tvmo_evaluate_on_coset.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, ctypes.c_uint64]
        L.tvmo_tip5_permutation.argtypes = [_u64p]
        L.tvmo_hash_varlen.argtypes = [_u64p, ctypes.c_size_t, _u64p]
        L.tvmo_hash_10.argtypes = [_u64p, _u64p]
        L.tvmo_hash_pair.argtypes = [_u64p, _u64p, _u64p]
        L.tvmo_hash_rows.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                                     ctypes.c_size_t, _u64p]
        L.tvmo_merkle_build.argtypes = [_u64p, ctypes.c_size_t, _u64p]
        L.tvmo_auth_path.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, _u64p]
        L.tvmo_auth_structure_indices.restype = ctypes.c_long
        L.tvmo_auth_structure_indices.argtypes = [ctypes.c_size_t, _szp, ctypes.c_size_t, _szp,
                                                  ctypes.c_size_t]
        L.tvmo_merkle_verify.argtypes = [_u64p, ctypes.c_size_t, _u64p, _u64p, ctypes.c_size_t]
        L.tvmo_lde_randomized_column.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, _u64p,
                                                 ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64,
                                                 ctypes.c_int]

    # field
    def mul(self, a, b): return self.L.tvmo_mul(a, b)
    def add(self, a, b): return self.L.tvmo_add(a, b)
    def pow(self, a, e): return self.L.tvmo_pow(a, e)
    def inverse(self, a): return self.L.tvmo_inverse(a)
    def primitive_root(self, k): return self.L.tvmo_primitive_root(k)

    def ntt(self, a, inverse=False) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        fn = self.L.tvmo_ntt_inverse if inverse else self.L.tvmo_ntt_forward
        if fn(_ptr(a), a.size) != 0:
            raise ValueError("NTT size must be a power of 2")
        return a

    def evaluate_on_coset(self, coeffs, domain_len: int, offset: int) -> np.ndarray:
        """NTT::evaluate_on_coset of one coefficient vector (any length)."""
        c = np.ascontiguousarray(coeffs, dtype=np.uint64)
        out = np.empty(domain_len, dtype=np.uint64)
        cc = c if c.size else np.zeros(1, np.uint64)
        if self.L.tvmo_evaluate_on_coset(_ptr(cc), c.size, _ptr(out), domain_len, offset) != 0:
            raise ValueError("NTT size must be a power of 2")
        return out

    def lde(self, trace_cm: np.ndarray, expansion: int = 4, offset: int = 7) -> np.ndarray:
        """Column-major (width, n) -> column-major (width, expansion*n)."""
        t = np.ascontiguousarray(trace_cm, dtype=np.uint64)
        w, n = t.shape
        out = np.empty((w, n * expansion), dtype=np.uint64)
        if self.L.tvmo_lde_table(_ptr(t), n, w, _ptr(out), n * expansion, offset) != 0:
            raise ValueError("bad LDE size")
        return out

    def lde_randomized(self, trace_cm, rnd_cm, expansion: int = 4, offset: int = 7, trace_offset: int = 1,
                       truncate: bool = False) -> np.ndarray:
        """Randomized LDE of column-major (width, n) with randomizers (width, R)."""
        t = np.ascontiguousarray(trace_cm, dtype=np.uint64)
        w, n = t.shape
        r = np.ascontiguousarray(rnd_cm, dtype=np.uint64).reshape(w, -1)
        R = r.shape[1]
        rr = r if R else np.zeros((w, 1), dtype=np.uint64)
        out = np.empty((w, n * expansion), dtype=np.uint64)
        for c in range(w):
            if self.L.tvmo_lde_randomized_column(_ptr(t[c]), n, _ptr(rr[c]), R, _ptr(out[c]), n * expansion,
                                                 trace_offset, offset, int(truncate)) != 0:
                raise ValueError("bad LDE size")
        return out

    def permutation(self, state) -> np.ndarray:
        s = np.ascontiguousarray(state, dtype=np.uint64).copy()
        self.L.tvmo_tip5_permutation(_ptr(s))
        return s

    def hash_varlen(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.uint64)
        out = np.zeros(5, dtype=np.uint64)
        self.L.tvmo_hash_varlen(_ptr(x) if x.size else _ptr(np.zeros(1, np.uint64)), x.size, _ptr(out))
        return out

    def hash_10(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.uint64)
        out = np.zeros(5, dtype=np.uint64)
        self.L.tvmo_hash_10(_ptr(x), _ptr(out))
        return out

    def hash_pair(self, l, r) -> np.ndarray:
        l = np.ascontiguousarray(l, dtype=np.uint64)
        r = np.ascontiguousarray(r, dtype=np.uint64)
        out = np.zeros(5, dtype=np.uint64)
        self.L.tvmo_hash_pair(_ptr(l), _ptr(r), _ptr(out))
        return out

    def hash_rows_cm(self, table_cm: np.ndarray) -> np.ndarray:
        """Leaf digest of each row of a column-major (width, rows) table."""
        t = np.ascontiguousarray(table_cm, dtype=np.uint64)
        w, rows = t.shape
        out = np.zeros((rows, 5), dtype=np.uint64)
        self.L.tvmo_hash_rows(_ptr(t), rows, w, 1, rows, _ptr(out))
        return out

    def hash_rows_rm(self, table_rm: np.ndarray) -> np.ndarray:
        t = np.ascontiguousarray(table_rm, dtype=np.uint64)
        rows, w = t.shape
        out = np.zeros((rows, 5), dtype=np.uint64)
        self.L.tvmo_hash_rows(_ptr(t), rows, w, w, 1, _ptr(out))
        return out

    def merkle(self, leaves: np.ndarray) -> np.ndarray:
        """Heap-layout tree: (2n, 5); node 1 is the root, leaves at [n, 2n)."""
        lv = np.ascontiguousarray(leaves, dtype=np.uint64)
        n = lv.shape[0]
        nodes = np.zeros((2 * n, 5), dtype=np.uint64)
        if self.L.tvmo_merkle_build(_ptr(lv), n, _ptr(nodes)) != 0:
            raise ValueError("Number of leaves must be a power of 2")
        return nodes

    def auth_path(self, nodes: np.ndarray, leaf: int) -> np.ndarray:
        n = nodes.shape[0] // 2
        out = np.zeros((64, 5), dtype=np.uint64)
        k = self.L.tvmo_auth_path(_ptr(np.ascontiguousarray(nodes)), n, leaf, _ptr(out))
        if k < 0:
            raise IndexError("Leaf index out of range")
        return out[:k]

    def auth_structure_indices(self, n: int, leaves) -> np.ndarray:
        lv = np.ascontiguousarray(leaves, dtype=np.uintp)
        cap = max(1, 64 * max(1, lv.size))
        out = np.zeros(cap, dtype=np.uintp)
        k = self.L.tvmo_auth_structure_indices(n, lv.ctypes.data_as(_szp), lv.size,
                                               out.ctypes.data_as(_szp), cap)
        if k < 0:
            raise IndexError("Leaf index out of range")
        return out[:k].astype(np.uint64)

    def verify(self, root, leaf_index, leaf, path) -> bool:
        root = np.ascontiguousarray(root, dtype=np.uint64)
        leaf = np.ascontiguousarray(leaf, dtype=np.uint64)
        path = np.ascontiguousarray(path, dtype=np.uint64).reshape(-1, 5)
        pp = _ptr(path) if path.size else _ptr(np.zeros(5, np.uint64))
        return bool(self.L.tvmo_merkle_verify(_ptr(root), leaf_index, _ptr(leaf), pp, path.shape[0]))


class RefLib:
    """The reference's own CPU functions (compiled unchanged) behind a C ABI."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "_ref", "libtvm_ref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        self.L = L
        L.tvmr_primitive_root.restype = ctypes.c_uint64
        L.tvmr_primitive_root.argtypes = [ctypes.c_uint32]
        L.tvmr_tip5_permutation.argtypes = [_u64p]
        L.tvmr_hash_varlen.argtypes = [_u64p, ctypes.c_size_t, _u64p]
        L.tvmr_hash_pair.argtypes = [_u64p, _u64p, _u64p]
        L.tvmr_ntt.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_int]
        L.tvmr_lde_table.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, _u64p, ctypes.c_size_t,
                                     ctypes.c_uint64]
        L.tvmr_evaluate_on_coset.argtypes = [_u64p, ctypes.c_size_t, _u64p, ctypes.c_size_t, ctypes.c_uint64]
        L.tvmr_hash_rows.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                                     ctypes.c_size_t, _u64p]
        L.tvmr_merkle.argtypes = [_u64p, ctypes.c_size_t, _u64p]
        L.tvmr_auth_path.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, _u64p]
        L.tvmr_auth_structure.restype = ctypes.c_long
        L.tvmr_auth_structure.argtypes = [_u64p, ctypes.c_size_t, _szp, ctypes.c_size_t, _u64p,
                                          ctypes.c_size_t]
        L.tvmr_commit.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                                  ctypes.c_uint64, _u64p, _u64p]
        L.tvmr_lde_randomized.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, _u64p, ctypes.c_size_t,
                                          _u64p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64]
        L.tvmr_lde_randomized_xfe.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, _u64p,
                                              ctypes.c_size_t, ctypes.c_int, _u64p, ctypes.c_size_t,
                                              ctypes.c_uint64, ctypes.c_uint64]
        L.tvmr_lde_table_root.argtypes = [_u64p, ctypes.c_size_t, ctypes.c_size_t, _u64p, ctypes.c_size_t,
                                          ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64, _u64p]
        L.tvmr_max_threads.restype = ctypes.c_int
        L.tvmr_set_threads.argtypes = [ctypes.c_int]

    def max_threads(self) -> int:
        return self.L.tvmr_max_threads()

    def set_threads(self, n: int) -> None:
        self.L.tvmr_set_threads(n)

    def primitive_root(self, k): return self.L.tvmr_primitive_root(k)

    def permutation(self, state):
        s = np.ascontiguousarray(state, dtype=np.uint64).copy()
        self.L.tvmr_tip5_permutation(_ptr(s))
        return s

    def hash_varlen(self, x):
        x = np.ascontiguousarray(x, dtype=np.uint64)
        out = np.zeros(5, dtype=np.uint64)
        self.L.tvmr_hash_varlen(_ptr(x) if x.size else _ptr(np.zeros(1, np.uint64)), x.size, _ptr(out))
        return out

    def hash_pair(self, l, r):
        out = np.zeros(5, dtype=np.uint64)
        self.L.tvmr_hash_pair(_ptr(np.ascontiguousarray(l, dtype=np.uint64)),
                              _ptr(np.ascontiguousarray(r, dtype=np.uint64)), _ptr(out))
        return out

    def ntt(self, a, inverse=False):
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        self.L.tvmr_ntt(_ptr(a), a.size, int(inverse))
        return a

    def evaluate_on_coset(self, coeffs, domain_len, offset):
        c = np.ascontiguousarray(coeffs, dtype=np.uint64)
        out = np.empty(domain_len, dtype=np.uint64)
        cc = c if c.size else np.zeros(1, np.uint64)
        self.L.tvmr_evaluate_on_coset(_ptr(cc), c.size, _ptr(out), domain_len, offset)
        return out

    def lde(self, trace_cm, expansion=4, offset=7):
        t = np.ascontiguousarray(trace_cm, dtype=np.uint64)
        w, n = t.shape
        out = np.empty((w, n * expansion), dtype=np.uint64)
        self.L.tvmr_lde_table(_ptr(t), n, w, _ptr(out), n * expansion, offset)
        return out

    def lde_randomized(self, trace_cm, rnd_cm, expansion=4, offset=7, trace_offset=1):
        t = np.ascontiguousarray(trace_cm, dtype=np.uint64)
        w, n = t.shape
        r = np.ascontiguousarray(rnd_cm, dtype=np.uint64).reshape(w, -1)
        rr = r if r.size else np.zeros((w, 1), dtype=np.uint64)
        out = np.empty((w, n * expansion), dtype=np.uint64)
        self.L.tvmr_lde_randomized(_ptr(t), n, w, _ptr(rr), r.shape[1], _ptr(out), n * expansion,
                                   trace_offset, offset)
        return out

    def lde_randomized_xfe(self, trace_x, rnd, expansion=4, offset=7, trace_offset=1):
        """XFE columns (width, n, 3); rnd (width, R) base-field or (width, R, 3) XFE randomizers."""
        t = np.ascontiguousarray(trace_x, dtype=np.uint64)
        w, n, _ = t.shape
        r = np.ascontiguousarray(rnd, dtype=np.uint64)
        xr = int(r.ndim == 3)
        R = r.shape[1]
        rr = r if r.size else np.zeros(3, dtype=np.uint64)
        out = np.empty((w, n * expansion, 3), dtype=np.uint64)
        self.L.tvmr_lde_randomized_xfe(_ptr(t), n, w, _ptr(rr), R, xr, _ptr(out), n * expansion,
                                       trace_offset, offset)
        return out

    def lde_table_root(self, rows_rm, rnd_cm, expansion=4, offset=7, trace_offset=1):
        """LDETable::compute_lde_and_merkle of a row-major (n, width) table."""
        t = np.ascontiguousarray(rows_rm, dtype=np.uint64)
        n, w = t.shape
        r = np.ascontiguousarray(rnd_cm, dtype=np.uint64).reshape(w, -1)
        rr = r if r.size else np.zeros(1, dtype=np.uint64)
        root = np.zeros(5, dtype=np.uint64)
        if self.L.tvmr_lde_table_root(_ptr(t), n, w, _ptr(rr), r.shape[1], n * expansion, trace_offset,
                                      offset, _ptr(root)) != 0:
            raise ValueError("LDETable::compute_lde_and_merkle threw")
        return root

    def hash_rows_cm(self, table_cm, r0=0, r1=None):
        t = np.ascontiguousarray(table_cm, dtype=np.uint64)
        w, rows = t.shape
        r1 = rows if r1 is None else r1
        out = np.zeros((r1 - r0, 5), dtype=np.uint64)
        self.L.tvmr_hash_rows(_ptr(t), rows, w, r0, r1, _ptr(out))
        return out

    def merkle(self, leaves):
        lv = np.ascontiguousarray(leaves, dtype=np.uint64)
        n = lv.shape[0]
        nodes = np.zeros((2 * n, 5), dtype=np.uint64)
        if self.L.tvmr_merkle(_ptr(lv), n, _ptr(nodes)) != 0:
            raise ValueError("bad leaf count")
        return nodes

    def auth_path(self, leaves, leaf):
        lv = np.ascontiguousarray(leaves, dtype=np.uint64)
        out = np.zeros((64, 5), dtype=np.uint64)
        k = self.L.tvmr_auth_path(_ptr(lv), lv.shape[0], leaf, _ptr(out))
        if k < 0:
            raise IndexError("Leaf index out of range")
        return out[:k]

    def auth_structure(self, leaves, idx):
        lv = np.ascontiguousarray(leaves, dtype=np.uint64)
        ix = np.ascontiguousarray(idx, dtype=np.uintp)
        cap = 64 * max(1, ix.size)
        out = np.zeros((cap, 5), dtype=np.uint64)
        k = self.L.tvmr_auth_structure(_ptr(lv), lv.shape[0], ix.ctypes.data_as(_szp), ix.size,
                                       _ptr(out), cap)
        if k < 0:
            raise IndexError("Leaf index out of range")
        return out[:k]

    def commit(self, trace_cm, expansion=4, offset=7, lde_buf=None):
        """The reference's CPU commit of one column-major table; returns
        (LDE, root).  lde_buf: an optional flat uint64 buffer of at least
        width * n * expansion words to hold the LDE (reused across calls)."""
        t = np.ascontiguousarray(trace_cm, dtype=np.uint64)
        w, n = t.shape
        if lde_buf is None:
            lde = np.empty((w, n * expansion), dtype=np.uint64)
        else:
            lde = lde_buf[: w * n * expansion].reshape(w, n * expansion)
        root = np.zeros(5, dtype=np.uint64)
        if self.L.tvmr_commit(_ptr(t), n, w, n * expansion, offset, _ptr(lde), _ptr(root)) != 0:
            raise ValueError("commit failed")
        return lde, root


def random_table(seed: int, width: int, n: int) -> np.ndarray:
    """Seeded column-major (width, n) table, entries uniform in [0, p)."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, P, size=(width, n), dtype=np.uint64)
