"""The Montgomery-form arithmetic of the CUDA kernels, restated limb by limb.

field.cuh's gl_redc reduces a 128-bit product T by 2^64 with nine 32-bit
instructions (p^-1 = 1 + 2^32 mod 2^64), gl_to_mont multiplies by 2^64 with
seven, and tip5.cuh's t5_recombine joins the two biased FP64 MDS halves from
their unmasked high words, the constant that adds being taken out of the round
constants (T5_RECOMBINE_EXCESS).  These tests restate each carry chain with
explicit 32-bit limbs, carries and borrows, check the results against exact
integer arithmetic on edge and random inputs, and check the constants the
sources hard-code.  The GPU tests check the same code through whole LDEs and
permutations against the oracle."""
import os
import random
import re
import struct

from conftest import ROOT

P = 2**64 - 2**32 + 1
M32 = 2**32
CSRC = os.path.join(ROOT, "triton-vm-prover_b200", "csrc")


def _src(name):
    return open(os.path.join(CSRC, name)).read()


def redc(r0, r1, r2, r3):
    """gl_redc: add.cc a1 = r1 + r0; addc t = a1 + carry; b = (a1:r0) - t;
    x = (r3:r2) - b; a borrow subtracts 2^32 - 1 (adds p)."""
    s = r1 + r0
    a1, cf = s % M32, s >> 32
    t = a1 + cf
    assert t < M32  # a carry leaves a1 <= 2^32 - 2
    d = r0 - t
    b0, br = d % M32, int(d < 0)
    b1 = (a1 - br) % M32
    d = r2 - b0
    x0, br = d % M32, int(d < 0)
    d = r3 - b1 - br
    x1, br = d % M32, int(d < 0)
    c = (-br) % M32
    d = x0 - c
    y0, br = d % M32, int(d < 0)
    y1 = (x1 - br) % M32
    return y0 | (y1 << 32)


def to_mont(x):
    """gl_to_mont: x0 * (2^32 - 1) - x1 as (x0 : -x0) - x1, plus p on a borrow."""
    x0, x1 = x % M32, x >> 32
    d = 0 - x0
    t0, br = d % M32, int(d < 0)
    t1 = (x0 - br) % M32
    d = t0 - x1
    m0, br = d % M32, int(d < 0)
    d = t1 - br
    m1, br = d % M32, int(d < 0)
    k = (-br) % M32
    d = m0 - k
    r0, br = d % M32, int(d < 0)
    r1 = (m1 - br) % M32
    return r0 | (r1 << 32)


def recombine(l0, l1, h0, h1):
    """t5_recombine on limbs as given: L0 - H1 + (H0 + L1 + H1) * 2^32 with the
    net carry c in {-1, 0, 1} folded back as c * (2^32 - 1)."""
    a = (l1 + h1) % M32
    s = h0 + a
    x1, c = s % M32, s >> 32
    d = l0 - h1
    x0, b = d % M32, int(d < 0)
    d = x1 - b
    x1, b2 = d % M32, int(d < 0)
    c -= b2
    e0, e1 = (-c) % M32, (M32 - 1 if c < 0 else 0)
    s = x0 + e0
    x0, cy = s % M32, s >> 32
    x1 = (x1 + e1 + cy) % M32
    return x0 | (x1 << 32)


def _edge64():
    return [0, 1, 2, P - 1, P - 2, P, P + 1, 2**64 - 1, 2**64 - 2**32, 2**63, 2**32 - 1, 2**32]


def test_inverse_of_p_mod_2_64():
    assert (P * (1 + 2**32)) % 2**64 == 1


def test_redc_matches_montgomery_reduction():
    rinv = pow(2, -64, P)
    rng = random.Random(0x5EED)
    cases = [(x, y) for x in _edge64() for y in _edge64()]
    cases += [(rng.randrange(2**64), rng.randrange(2**64)) for _ in range(20000)]
    cases += [(rng.randrange(2**64), rng.randrange(P)) for _ in range(20000)]
    for x, y in cases:
        t = x * y
        r = redc(t % M32, (t >> 32) % M32, (t >> 64) % M32, t >> 96)
        assert r < 2**64 and r % P == (t * rinv) % P, (x, y)
        if t < P * 2**64:  # one factor below p: canonical
            assert r < P, (x, y)


def test_to_mont_multiplies_by_2_64():
    rng = random.Random(7)
    for x in _edge64() + [rng.randrange(2**64) for _ in range(20000)]:
        r = to_mont(x)
        assert r == (x * 2**64) % P, x


def test_recombine_with_unmasked_high_words():
    k = 0x43300000
    excess = (2 * k * 2**32 - k) % P
    rng = random.Random(11)
    for _ in range(20000):
        lo, hi = rng.randrange(2**52), rng.randrange(2**52)
        if rng.random() < 0.1:
            lo, hi = 2**52 - 1 - rng.randrange(64), 2**52 - 1 - rng.randrange(64)
        # the words of the doubles 2^52 + lo and 2^52 + hi, as t5_recombine reads them
        wl = struct.unpack("<II", struct.pack("<d", 2.0**52 + lo))
        wh = struct.unpack("<II", struct.pack("<d", 2.0**52 + hi))
        assert wl == (lo % M32, k + (lo >> 32)) and wh == (hi % M32, k + (hi >> 32))
        r = recombine(wl[0], wl[1], wh[0], wh[1])
        assert r < 2**64 and (r - excess) % P == (lo + hi * 2**32) % P, (lo, hi)


def test_constants_in_the_sources():
    tip5 = _src("tip5.cuh")
    assert "constexpr uint64_t T5_MONT_ONE = 0xFFFFFFFFull;" in tip5
    assert 0xFFFFFFFF == 2**64 % P
    m = re.search(r"T5_RECOMBINE_EXCESS = 2ull \* 0x43300000ull \* 0x100000000ull - 0x43300000ull;", tip5)
    assert m is not None
    field = _src("field.cuh")
    for fn in ("gl_redc", "gl_mont_mul", "gl_to_mont", "gl_from_mont"):
        assert f"uint64_t {fn}(" in field, fn
