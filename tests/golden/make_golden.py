"""Writes the golden fixtures in this directory from the reference's OWN code.

Run where the reference tree exists (it compiles oracle/_ref/libtvm_ref.so
from the reference's unchanged C++ sources first):

    python tests/golden/make_golden.py

Every array written here is an output of the reference prover's CPU functions
(NTT::forward/inverse, LDE::extend_column, Tip5::permutation/hash_varlen/
hash_pair, MerkleTree and its authentication paths/structure, the randomized
LDE of RandomizedLDE and LDETable::compute_lde_and_merkle) on seeded inputs.  Tests compare both the CPU oracle and the CUDA path against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import RefLib, build  # noqa: E402

P = 0xFFFFFFFF00000001


def main():
    build(ref=True)
    r = RefLib()
    rng = np.random.default_rng(20261203)

    # Tip5 permutation on edge and random states; hash_varlen of lengths 0..45.
    edge = np.array([0, 1, 2, P - 1, P - 2, 2**32 - 1, 2**32, 2**32 + 1, 2**63, 7, 0xFFFFFFFE00000001,
                     P // 2, P // 2 + 1, 0xFFFFFFFF, P, 2**64 - 1], dtype=np.uint64)
    states = [edge, edge[::-1].copy(), np.zeros(16, np.uint64), np.full(16, P - 1, np.uint64)]
    states += [rng.integers(0, 2**64 - 1, 16, dtype=np.uint64, endpoint=True) for _ in range(28)]
    states = np.stack(states)
    perms = np.stack([r.permutation(s) for s in states])
    vl_in = rng.integers(0, P, 45 * 46 // 2, dtype=np.uint64)
    vl_out, off = [], 0
    for n in range(46):
        vl_out.append(r.hash_varlen(vl_in[off:off + n]))
        off += n
    pairs_l = rng.integers(0, P, (16, 5), dtype=np.uint64)
    pairs_r = rng.integers(0, P, (16, 5), dtype=np.uint64)
    pairs = np.stack([r.hash_pair(a, b) for a, b in zip(pairs_l, pairs_r)])
    np.savez(os.path.join(HERE, "tip5.npz"), states=states, perms=perms, varlen_in=vl_in,
             varlen_out=np.stack(vl_out), pairs_l=pairs_l, pairs_r=pairs_r, pairs=pairs)

    # NTT forward / inverse for every size 1..2^9.
    ntt = {}
    for k in range(10):
        a = rng.integers(0, P, 1 << k, dtype=np.uint64)
        ntt[f"in{k}"] = a
        ntt[f"fwd{k}"] = r.ntt(a)
        ntt[f"inv{k}"] = r.ntt(a, inverse=True)
    np.savez(os.path.join(HERE, "ntt.npz"), **ntt)

    # Table commitments: LDE (expansion 4, offset 7), every tree node, auth data.
    for name, (w, n) in {"commit_w23_n64": (23, 64), "commit_w379_n4": (379, 4),
                         "commit_w264_n8": (264, 8), "commit_w1_n1": (1, 1)}.items():
        trace = rng.integers(0, P, (w, n), dtype=np.uint64)
        lde = r.lde(trace)
        leaves = r.hash_rows_cm(lde)
        nodes = r.merkle(leaves)
        L = 4 * n
        idx = rng.integers(0, L, 4)
        paths = np.stack([r.auth_path(leaves, int(i)) for i in idx]) if L > 1 else np.zeros((4, 0, 5), np.uint64)
        sidx = np.unique(rng.integers(0, L, 3))
        struct = r.auth_structure(leaves, sidx)
        np.savez(os.path.join(HERE, f"{name}.npz"), trace=trace, lde=lde, leaves=leaves, nodes=nodes,
                 root=nodes[1], path_idx=idx, paths=paths, struct_idx=sidx, struct=struct)

    # Randomized (zero-knowledge) LDE: base-field columns, XFE columns with base
    # or XFE randomizers, and the LDETable root.  Cases cover R = 0, N = 1, a
    # trace offset != 1, polynomials longer than the LDE (chunked evaluation for
    # base columns, truncation for XFE columns) and R = 98, the reference's
    # default number of trace randomizers (src/stark.cpp:440-446).
    rl = {}
    for i, (n, R, E, t, o) in enumerate([(1, 0, 4, 1, 7), (1, 5, 4, 1, 7), (2, 3, 2, 3, 7), (4, 20, 2, 11, 7),
                                         (8, 3, 4, 5, 7), (16, 0, 4, 3, 7), (64, 98, 4, 1, 7),
                                         (256, 98, 8, 1, 7), (32, 98, 4, 1, 7), (128, 7, 2, 13, 5)]):
        trace = rng.integers(0, P, (3, n), dtype=np.uint64)
        rnd = rng.integers(0, P, (3, R), dtype=np.uint64)
        rl[f"b{i}_meta"] = np.array([n, R, E, t, o], dtype=np.uint64)
        rl[f"b{i}_trace"], rl[f"b{i}_rnd"] = trace, rnd
        rl[f"b{i}_out"] = r.lde_randomized(trace, rnd, E, o, t)
    for i, (n, R, E, t, xr) in enumerate([(4, 9, 2, 1, 0), (4, 9, 2, 1, 1), (32, 98, 4, 1, 0), (16, 5, 4, 3, 1)]):
        trace = rng.integers(0, P, (2, n, 3), dtype=np.uint64)
        rnd = rng.integers(0, P, (2, R, 3) if xr else (2, R), dtype=np.uint64)
        rl[f"x{i}_meta"] = np.array([n, R, E, t, 7, xr], dtype=np.uint64)
        rl[f"x{i}_trace"], rl[f"x{i}_rnd"] = trace, rnd
        rl[f"x{i}_out"] = r.lde_randomized_xfe(trace, rnd, E, 7, t)
    rows = rng.integers(0, P, (64, 23), dtype=np.uint64)
    rnd = rng.integers(0, P, (23, 98), dtype=np.uint64)
    rl["table_rows"], rl["table_rnd"] = rows, rnd
    rl["table_root"] = r.lde_table_root(rows, rnd, 4, 7, 1)
    np.savez(os.path.join(HERE, "lde_randomized.npz"), **rl)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
