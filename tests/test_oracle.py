"""The CPU oracle is pinned before it is trusted: upstream Tip5 known-answer
tests, the upstream primitive-root table, the golden fixtures produced by the
reference's own compiled code, and (where it was built) that code itself."""
import os

import numpy as np
import pytest

from conftest import EDGE_VALUES, P, golden, rand_u64

# twenty-first 0.50.0, src/math/b_field_element.rs:42-77 (PRIMITIVE_ROOTS)
ROOTS = {0: 1, 1: 18446744069414584320, 2: 281474976710656, 3: 18446744069397807105,
         4: 17293822564807737345, 5: 70368744161280, 6: 549755813888, 7: 17870292113338400769,
         8: 13797081185216407910, 9: 1803076106186727246, 10: 11353340290879379826,
         11: 455906449640507599, 12: 17492915097719143606, 16: 6115771955107415310,
         20: 3511170319078647661, 22: 5416168637041100469, 24: 9713644485405565297,
         32: 1753635133440165772}


def test_primitive_roots(oracle):
    for k, w in ROOTS.items():
        assert oracle.primitive_root(k) == w


def test_hash10_kat(oracle):
    # twenty-first src/tip5/mod.rs:1130-1163
    pre = np.zeros(10, dtype=np.uint64)
    for i in range(6):
        pre[i:i + 5] = oracle.hash_10(pre)
    d = oracle.hash_10(pre)
    assert list(map(int, d)) == [10869784347448351760, 1853783032222938415, 6856460589287344822,
                                 17178399545409290325, 7650660984651717733]


def test_hash_varlen_kat(oracle):
    # twenty-first src/tip5/mod.rs:1166-1200
    s = [0] * 5
    for i in range(20):
        d = oracle.hash_varlen(np.arange(i, dtype=np.uint64))
        s = [(a + int(b)) % P for a, b in zip(s, d)]
    assert s == [7610004073009036015, 5725198067541094245, 4721320565792709122, 1732504843634706218,
                 259800783350288362]


def test_tip5_golden(oracle):
    g = golden("tip5.npz")
    for st, pe in zip(g["states"], g["perms"]):
        assert (oracle.permutation(st) == pe).all()
    off = 0
    for n, exp in enumerate(g["varlen_out"]):
        assert (oracle.hash_varlen(g["varlen_in"][off:off + n]) == exp).all()
        off += n
    for a, b, exp in zip(g["pairs_l"], g["pairs_r"], g["pairs"]):
        assert (oracle.hash_pair(a, b) == exp).all()


def test_ntt_golden(oracle):
    g = golden("ntt.npz")
    for k in range(10):
        assert (oracle.ntt(g[f"in{k}"]) == g[f"fwd{k}"]).all()
        assert (oracle.ntt(g[f"in{k}"], inverse=True) == g[f"inv{k}"]).all()


@pytest.mark.parametrize("name", ["commit_w23_n64", "commit_w379_n4", "commit_w264_n8", "commit_w1_n1"])
def test_commit_golden(oracle, name):
    g = golden(f"{name}.npz")
    lde = oracle.lde(g["trace"])
    assert (lde == g["lde"]).all()
    leaves = oracle.hash_rows_cm(lde)
    assert (leaves == g["leaves"]).all()
    nodes = oracle.merkle(leaves)
    assert (nodes[1:] == g["nodes"][1:]).all()
    for i, p in zip(g["path_idx"], g["paths"]):
        assert (oracle.auth_path(nodes, int(i)) == p).all()
        assert oracle.verify(g["root"], int(i), leaves[int(i)], p)
    sidx = oracle.auth_structure_indices(lde.shape[1], g["struct_idx"])
    assert (nodes[sidx.astype(np.int64)] == g["struct"]).all()


def test_ntt_properties(oracle):
    a = rand_u64(3, 64)
    assert (oracle.ntt(oracle.ntt(a), inverse=True) == a).all()
    with pytest.raises(ValueError):
        oracle.ntt(np.zeros(6, np.uint64))


def test_lde_is_coset_evaluation(oracle):
    # LDE[j] = f(7 * w_L^j) where f interpolates the trace on <w_n>.
    n, L = 8, 32
    t = rand_u64(5, (1, n))
    coef = oracle.ntt(t[0], inverse=True)
    out = oracle.lde(t)[0]
    wL = oracle.primitive_root(5)
    for j in (0, 1, 7, 31):
        x = oracle.mul(7, oracle.pow(wL, j))
        acc, xp = 0, 1
        for c in coef:
            acc = oracle.add(acc, oracle.mul(int(c), xp))
            xp = oracle.mul(xp, x)
        assert int(out[j]) == acc


def test_noncanonical_inputs_read_mod_p(oracle):
    st = EDGE_VALUES.copy()
    st2 = np.array([int(v) % P for v in st], dtype=np.uint64)
    assert (oracle.permutation(st) == oracle.permutation(st2)).all()


def _ref_available():
    return os.path.exists(os.path.join(os.path.dirname(os.path.dirname(__file__)), "oracle", "_ref",
                                       "libtvm_ref.so"))


@pytest.mark.skipif(not _ref_available(), reason="reference build oracle/_ref not present")
def test_oracle_matches_reference_build(oracle):
    from oracle import RefLib
    r = RefLib()
    for s in range(20):
        st = rand_u64(100 + s, 16, hi=2**64 - 1)
        assert (oracle.permutation(st) == r.permutation(st)).all()
    for n in (0, 1, 9, 10, 11, 264, 379):
        x = rand_u64(n, n)
        assert (oracle.hash_varlen(x) == r.hash_varlen(x)).all()
    t = rand_u64(9, (7, 128))
    lde = oracle.lde(t, expansion=8)
    assert (lde == r.lde(t, expansion=8)).all()
    leaves = oracle.hash_rows_cm(lde)
    assert (leaves == r.hash_rows_cm(lde)).all()
    assert (oracle.merkle(leaves)[1:] == r.merkle(leaves)[1:]).all()


@pytest.mark.skipif(not _ref_available(), reason="reference build oracle/_ref not present")
def test_oracle_evaluate_on_coset_matches_reference_build(oracle):
    """NTT::evaluate_on_coset: zero-extension (n < L), equal sizes and the
    reference's truncation of coefficients beyond the domain (n > L)."""
    from oracle import RefLib
    r = RefLib()
    for n, L, off in ((0, 8, 7), (1, 1, 7), (5, 16, 7), (64, 64, 3), (100, 32, 7), (1 << 10, 1 << 13, 7),
                      (1 << 12, 1 << 12, 0xFFFFFFFF00000000)):
        c = rand_u64(n + L, n)
        assert (oracle.evaluate_on_coset(c, L, off) == r.evaluate_on_coset(c, L, off)).all(), (n, L)


def test_lde_randomized_golden(oracle):
    """The oracle's randomized LDE equals the reference's RandomizedLDE outputs."""
    g = golden("lde_randomized.npz")
    for k in [k for k in g.files if k.endswith("_meta")]:
        p = k[:-5]
        if p.startswith("b"):
            n, R, E, t, o = (int(v) for v in g[k])
            got = oracle.lde_randomized(g[p + "_trace"], g[p + "_rnd"], E, o, t)
        else:
            n, R, E, t, o, xr = (int(v) for v in g[k])
            tr, rnd = g[p + "_trace"], g[p + "_rnd"]
            limbs = []
            for l in range(3):
                rl = rnd[:, :, l] if xr else (rnd if l == 0 else np.zeros_like(rnd))
                limbs.append(oracle.lde_randomized(tr[:, :, l], rl, E, o, t, truncate=True))
            got = np.stack(limbs, -1)
        assert (got == g[p + "_out"]).all(), p
    # LDETable::compute_lde_and_merkle root
    rows, rnd = g["table_rows"], g["table_rnd"]
    lde = oracle.lde_randomized(np.ascontiguousarray(rows.T), rnd, 4, 7, 1)
    assert (oracle.merkle(oracle.hash_rows_cm(lde))[1] == g["table_root"]).all()
