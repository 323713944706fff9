// Goldilocks field arithmetic for sm_100a: p = 2^64 - 2^32 + 1.
//
// Values inside kernels are kept "partially reduced": any 64-bit word is a
// valid representative of its residue mod p.  Functions named *_c return the
// canonical residue in [0, p), which is the representation the reference's
// BFieldElement stores (include/types/b_field_element.hpp:28-104) and what
// every output buffer holds.  Reduction of a 128-bit product uses
// 2^64 = 2^32 - 1 and 2^96 = -1 (mod p).
#pragma once
#include <cstdint>

namespace tvmc {

constexpr uint64_t GL_P = 0xFFFFFFFF00000001ull;
constexpr uint64_t GL_EPS = 0xFFFFFFFFull;  // 2^64 mod p

// The add/sub/canonicalisation helpers below are 32-bit carry chains: a >= p
// exactly when a + (2^32 - 1) carries out of 64 bits, so the comparison is the
// carry of the correction itself (no separate compares), and a borrow becomes
// an all-ones mask that subtracts 2^32 - 1 (adds p) directly.

// Canonical representative of any 64-bit value.
__device__ __forceinline__ uint64_t gl_canon(uint64_t a) {
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 t0, t1, c;\n\t"
        ".reg .pred q;\n\t"
        "add.cc.u32 t0, %2, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 t1, %3, 0;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "setp.ne.u32 q, c, 0;\n\t"
        "selp.b32 %0, t0, %2, q;\n\t"
        "selp.b32 %1, t1, %3, q;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}

// 64x64 -> 128-bit product as four 32-bit limbs (r3:r2:r1:r0), one carry
// chain of 32-bit multiply-adds.
__device__ __forceinline__ void gl_mul128(uint64_t a, uint64_t b, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                          uint32_t& r3) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    asm("{\n\t"
        "mul.lo.u32 %0, %4, %6;\n\t"
        "mul.hi.u32 %1, %4, %6;\n\t"
        "mad.lo.cc.u32 %1, %4, %7, %1;\n\t"
        "madc.hi.u32 %2, %4, %7, 0;\n\t"
        "mad.lo.cc.u32 %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "madc.hi.u32 %3, %5, %7, 0;\n\t"
        "mad.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "addc.u32 %3, %3, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
}

// a^2 as four 32-bit limbs with three partial products: the cross term a0*a1
// is formed once and doubled on the ALU (into 65 bits), which saves one 32-bit
// multiply and one high multiply against gl_mul128(a, a).
__device__ __forceinline__ void gl_sqr128(uint64_t a, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32);
    asm("{\n\t"
        ".reg .u32 t1, m0, m1, d2;\n\t"
        "mul.lo.u32 %0, %4, %4;\n\t"
        "mul.hi.u32 t1, %4, %4;\n\t"
        "mul.lo.u32 m0, %4, %5;\n\t"
        "mul.hi.u32 m1, %4, %5;\n\t"
        "add.cc.u32 m0, m0, m0;\n\t"
        "addc.cc.u32 m1, m1, m1;\n\t"
        "addc.u32 d2, 0, 0;\n\t"
        "add.cc.u32 %1, t1, m0;\n\t"
        "madc.lo.cc.u32 %2, %5, %5, m1;\n\t"
        "madc.hi.u32 %3, %5, %5, d2;\n\t"
        "}"
        : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
        : "r"(a0), "r"(a1));
}

// (r3:r2:r1:r0) -> (r1:r0) + r2*(2^32-1) - r3 (mod p) as a 64-bit
// representative (2^64 = 2^32 - 1 and 2^96 = -1 mod p).  The first sum is two
// multiply-adds (on the FMA pipe) with carry c in {0, 1}; subtracting r3 leaves
// c in {-1, 0, 1}; c*2^64 is folded back as c*(2^32 - 1), which cannot wrap:
// for c = 1 the low 64 bits are at most 2^64 - 2^33, for c = -1 at least
// 2^64 - 2^32 + 1.
__device__ __forceinline__ uint64_t gl_reduce_limbs(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
    uint32_t x0, x1;
    asm("{\n\t"
        ".reg .u32 c, e0, e1;\n\t"
        "mad.lo.cc.u32 %0, %4, 0xFFFFFFFF, %2;\n\t"
        "madc.hi.cc.u32 %1, %4, 0xFFFFFFFF, %3;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, %5;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32 c, c, 0;\n\t"
        "neg.s32 e0, c;\n\t"             // c*(2^32 - 1) as a signed 64-bit (e1:e0):
        "shr.s32 e1, c, 31;\n\t"         // (0, 2^32 - 1), (0, 0) or (2^32 - 1, 1)
        "add.cc.u32 %0, %0, e0;\n\t"
        "addc.u32 %1, %1, e1;\n\t"
        "}"
        : "=r"(x0), "=r"(x1)
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
    return ((uint64_t)x1 << 32) | x0;
}

// a * b for any 64-bit representatives; partial result.
__device__ __forceinline__ uint64_t gl_mul(uint64_t a, uint64_t b) {
    uint32_t r0, r1, r2, r3;
    gl_mul128(a, b, r0, r1, r2, r3);
    return gl_reduce_limbs(r0, r1, r2, r3);
}
// a * b, canonical.
__device__ __forceinline__ uint64_t gl_mul_c(uint64_t a, uint64_t b) { return gl_canon(gl_mul(a, b)); }

__device__ __forceinline__ uint64_t gl_sqr(uint64_t a) { return gl_mul(a, a); }

// a + b where b < p (a any representative); partial result.  A carry out of
// 64 bits means the sum exceeds 2^64 by less than p, so adding 2^32 - 1 (i.e.
// subtracting p modulo 2^64) cannot carry again.
__device__ __forceinline__ uint64_t gl_add_pc(uint64_t a, uint64_t b) {
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 s0, s1, m;\n\t"
        "add.cc.u32 s0, %2, %4;\n\t"
        "addc.cc.u32 s1, %3, %5;\n\t"
        "addc.u32 m, 0, 0;\n\t"
        "neg.s32 m, m;\n\t"
        "add.cc.u32 %0, s0, m;\n\t"
        "addc.u32 %1, s1, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}

// Canonical add of canonical operands as a subtraction: a + b = a - (p - b),
// where p - b lies in [1, p]; a borrow adds p back (subtracts 2^32 - 1 modulo
// 2^64), which cannot borrow again because the wrapped difference is at least
// 2^64 - p = 2^32 - 1.  Seven instructions against nine for the add-then-
// compare form.
__device__ __forceinline__ uint64_t gl_add_c(uint64_t a, uint64_t b) {
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 n0, n1, s0, s1, m;\n\t"
        "sub.cc.u32 n0, 1, %4;\n\t"
        "subc.u32 n1, 0xFFFFFFFF, %5;\n\t"
        "sub.cc.u32 s0, %2, n0;\n\t"
        "subc.cc.u32 s1, %3, n1;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, s0, m;\n\t"
        "subc.u32 %1, s1, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}

// Canonical sub of canonical operands: on a borrow the wrapped difference is at
// least 2^32, so subtracting 2^32 - 1 (adding p modulo 2^64) cannot borrow again.
__device__ __forceinline__ uint64_t gl_sub_c(uint64_t a, uint64_t b) {
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 s0, s1, m;\n\t"
        "sub.cc.u32 s0, %2, %4;\n\t"
        "subc.cc.u32 s1, %3, %5;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, s0, m;\n\t"
        "subc.u32 %1, s1, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"((uint32_t)a), "r"((uint32_t)(a >> 32)), "r"((uint32_t)b), "r"((uint32_t)(b >> 32)));
    return ((uint64_t)r1 << 32) | r0;
}

// ---- Montgomery products ---------------------------------------------------
// With R = 2^64, the Montgomery reduction of a 128-bit T = (r3:r2:r1:r0) is
// T * R^-1 (mod p) = (T - m p) / 2^64 for m = T * p^-1 (mod 2^64), and
// p^-1 = 1 + 2^32 (mod 2^64) makes m = a = lo + (lo << 32) (mod 2^64), lo =
// (r1:r0), with carry e; then (m p) >> 64 = a - (a >> 32) - e =: b, and the
// result is hi - b, plus p on a borrow.  For T < p * 2^64 (one factor below p)
// the result is canonical; for any T it is a 64-bit representative.  Nine
// instructions: a's high limb plus its carry, t = a1 + e, cannot wrap (a carry
// leaves a1 <= 2^32 - 2), so b = (a1 : r0) - t is one two-limb subtraction.
__device__ __forceinline__ uint64_t gl_redc(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
    uint32_t x0, x1;
    asm("{\n\t"
        ".reg .u32 a1, t, b0, b1, c;\n\t"
        "add.cc.u32 a1, %3, %2;\n\t"
        "addc.u32 t, a1, 0;\n\t"
        "sub.cc.u32 b0, %2, t;\n\t"
        "subc.u32 b1, a1, 0;\n\t"
        "sub.cc.u32 %0, %4, b0;\n\t"
        "subc.cc.u32 %1, %5, b1;\n\t"
        "subc.u32 c, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, c;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(x0), "=r"(x1)
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
    return ((uint64_t)x1 << 32) | x0;
}

// x * w for any 64-bit x and a factor given in Montgomery form wm = w * 2^64
// (mod p), wm < p; canonical.
__device__ __forceinline__ uint64_t gl_mont_mul(uint64_t x, uint64_t wm) {
    uint32_t r0, r1, r2, r3;
    gl_mul128(x, wm, r0, r1, r2, r3);
    return gl_redc(r0, r1, r2, r3);
}

// x * 2^-64 (mod p), canonical, for any 64-bit x (the reduction of T = x < p * 2^64).
__device__ __forceinline__ uint64_t gl_from_mont(uint64_t x) {
    return gl_redc((uint32_t)x, (uint32_t)(x >> 32), 0u, 0u);
}

// x * 2^64 (mod p), canonical, for any 64-bit x = x1 * 2^32 + x0: 2^64 = 2^32 - 1
// and 2^96 = -1 give x0 * (2^32 - 1) - x1, whose positive part is below p; a
// borrow adds p (subtracts 2^32 - 1 modulo 2^64) and cannot recur.
__device__ __forceinline__ uint64_t gl_to_mont(uint64_t x) {
    uint32_t m0, m1;
    asm("{\n\t"
        ".reg .u32 t0, t1, k;\n\t"
        "sub.cc.u32 t0, 0, %2;\n\t"
        "subc.u32 t1, %2, 0;\n\t"
        "sub.cc.u32 %0, t0, %3;\n\t"
        "subc.cc.u32 %1, t1, 0;\n\t"
        "subc.u32 k, 0, 0;\n\t"
        "sub.cc.u32 %0, %0, k;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(m0), "=r"(m1)
        : "r"((uint32_t)x), "r"((uint32_t)(x >> 32)));
    return ((uint64_t)m1 << 32) | m0;
}

// ---- multiplication by powers of two -------------------------------------
// 2 has order 192 mod p (2^96 = -1), so every root of unity of order <= 64 is
// +-2^s with s < 96: a shift and a short reduction instead of a multiply.  The
// shift amounts below must be constants after inlining and unrolling (the
// branches on them then fold away).

// x * 2^s for 0 < s <= 32 and any 64-bit x: lo + hi*(2^32 - 1) with hi < 2^32
// (carry c in {0, 1}, folded as c*(2^32 - 1) without a second carry); partial.
__device__ __forceinline__ uint64_t gl_shl_le32(uint64_t x, int s) {
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    const uint32_t lo0 = s == 32 ? 0u : x0 << s;
    const uint32_t lo1 = s == 32 ? x0 : __funnelshift_l(x0, x1, s);
    const uint32_t hi = s == 32 ? x1 : x1 >> (32 - s);
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 c;\n\t"
        "mad.lo.cc.u32 %0, %4, 0xFFFFFFFF, %2;\n\t"
        "madc.hi.cc.u32 %1, %4, 0xFFFFFFFF, %3;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "neg.s32 c, c;\n\t"
        "add.cc.u32 %0, %0, c;\n\t"
        "addc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"(lo0), "r"(lo1), "r"(hi));
    return ((uint64_t)r1 << 32) | r0;
}

// x * 2^s for 32 < s < 64: the 128-bit shift reduced by gl_reduce_limbs; partial.
__device__ __forceinline__ uint64_t gl_shl_gt32(uint64_t x, int s) {
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    return gl_reduce_limbs(0u, x0 << (s - 32), __funnelshift_r(x0, x1, 64 - s), x1 >> (64 - s));
}

// x * 2^-k for 0 < k <= 32 and canonical x, canonical: with x = q*2^k + r,
// x * 2^-k = q + r*2^(32-k) * 2^-32 and 2^-32 = 1 - 2^32 (mod p), so the
// result is u - t*2^32 with t = r*2^(32-k) < 2^32 and u = q + t < 2^63 + 2^32;
// a borrow adds p back (subtracts 2^32 - 1 modulo 2^64) and cannot recur.
__device__ __forceinline__ uint64_t gl_shr_c(uint64_t x, int k) {
    const uint32_t x0 = (uint32_t)x, x1 = (uint32_t)(x >> 32);
    const uint32_t q0 = k == 32 ? x1 : __funnelshift_r(x0, x1, k);
    const uint32_t q1 = k == 32 ? 0u : x1 >> k;
    const uint32_t t = k == 32 ? x0 : x0 << (32 - k);
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 u0, u1, m;\n\t"
        "add.cc.u32 u0, %2, %4;\n\t"
        "addc.u32 u1, %3, 0;\n\t"
        "sub.cc.u32 %1, u1, %4;\n\t"
        "subc.u32 m, 0, 0;\n\t"
        "sub.cc.u32 %0, u0, m;\n\t"
        "subc.u32 %1, %1, 0;\n\t"
        "}"
        : "=r"(r0), "=r"(r1)
        : "r"(q0), "r"(q1), "r"(t));
    return ((uint64_t)r1 << 32) | r0;
}

// (a - c) * 2^e for canonical a, c and 0 <= e < 192; canonical.  A negative
// factor (2^e = -2^(e-96), and 2^s = -2^-(96-s)) swaps the subtraction.  For
// 32 < s < 64 the factor is applied as -2^-32 * 2^-(64-s): two right shifts
// (20 instructions with the subtraction) instead of a 128-bit left shift and
// its reduction (24).
__device__ __forceinline__ uint64_t gl_sub_mul_pow2_c(uint64_t a, uint64_t c, int e) {
    bool neg = e >= 96;
    const int s = neg ? e - 96 : e;
    if (s > 32) neg = !neg;
    const uint64_t d = neg ? gl_sub_c(c, a) : gl_sub_c(a, c);
    if (s == 0) return d;
    if (s <= 32) return gl_canon(gl_shl_le32(d, s));
    if (s < 64) return gl_shr_c(gl_shr_c(d, 32), 64 - s);
    return gl_shr_c(d, 96 - s);
}

__device__ __forceinline__ uint64_t gl_pow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    while (e) {
        if (e & 1) r = gl_mul(r, b);
        b = gl_mul(b, b);
        e >>= 1;
    }
    return gl_canon(r);
}

}  // namespace tvmc
