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

// (r3:r2:r1:r0) -> (r1:r0) - r3 + r2*(2^32-1) (mod p) as a 64-bit representative.
__device__ __forceinline__ uint64_t gl_reduce_limbs(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
    uint32_t x0, x1;
    asm("{\n\t"
        ".reg .u32 z, t0, t1, bm, u0, u1, cm;\n\t"
        "mov.u32 z, 0;\n\t"
        "sub.cc.u32 t0, %2, %5;\n\t"    // t = (r1:r0) - r3
        "subc.cc.u32 t1, %3, z;\n\t"
        "subc.u32 bm, z, z;\n\t"        // borrow mask
        "sub.cc.u32 t0, t0, bm;\n\t"    // borrow: t -= 2^32 - 1 (i.e. + p)
        "subc.u32 t1, t1, z;\n\t"
        "sub.cc.u32 u0, z, %4;\n\t"     // u = r2*(2^32 - 1) = (r2 << 32) - r2
        "subc.u32 u1, %4, z;\n\t"
        "add.cc.u32 %0, t0, u0;\n\t"    // x = t + u
        "addc.cc.u32 %1, t1, u1;\n\t"
        "addc.u32 cm, z, z;\n\t"        // carry out
        "neg.s32 cm, cm;\n\t"           // carry: + (2^32 - 1); cannot wrap again
        "add.cc.u32 %0, %0, cm;\n\t"
        "addc.u32 %1, %1, z;\n\t"
        "}"
        : "=r"(x0), "=r"(x1)
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
    return ((uint64_t)x1 << 32) | x0;
}

// Canonical form of (r3:r2:r1:r0) mod p.  With t = (r1:r0) - r3 (+p on a
// borrow) and u = r2*(2^32-1), x = t + u is below 2^65 - 2^33: if it carries,
// x - 2^64 + (2^32 - 1) is already canonical (and does not carry); if not, x is
// canonical unless x + (2^32 - 1) carries.  So one "add 2^32 - 1, keep it on
// any carry" step both folds the carry and canonicalises.
__device__ __forceinline__ uint64_t gl_reduce_limbs_c(uint32_t r0, uint32_t r1, uint32_t r2, uint32_t r3) {
    uint32_t y0, y1;
    asm("{\n\t"
        ".reg .u32 t0, t1, bm, u0, u1, x0, x1, z0, z1, c;\n\t"
        ".reg .pred q;\n\t"
        "sub.cc.u32 t0, %2, %5;\n\t"    // t = (r1:r0) - r3
        "subc.cc.u32 t1, %3, 0;\n\t"
        "subc.u32 bm, 0, 0;\n\t"        // borrow mask
        "sub.cc.u32 t0, t0, bm;\n\t"    // borrow: t -= 2^32 - 1 (i.e. + p)
        "subc.u32 t1, t1, 0;\n\t"
        "sub.cc.u32 u0, 0, %4;\n\t"     // u = (r2 << 32) - r2
        "subc.u32 u1, %4, 0;\n\t"
        "add.cc.u32 x0, t0, u0;\n\t"    // x = t + u, carry c
        "addc.cc.u32 x1, t1, u1;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "add.cc.u32 z0, x0, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 z1, x1, 0;\n\t"
        "addc.u32 c, c, 0;\n\t"
        "setp.ne.u32 q, c, 0;\n\t"
        "selp.b32 %0, z0, x0, q;\n\t"
        "selp.b32 %1, z1, x1, q;\n\t"
        "}"
        : "=r"(y0), "=r"(y1)
        : "r"(r0), "r"(r1), "r"(r2), "r"(r3));
    return ((uint64_t)y1 << 32) | y0;
}

// a * b for any 64-bit representatives; partial result.
__device__ __forceinline__ uint64_t gl_mul(uint64_t a, uint64_t b) {
    uint32_t r0, r1, r2, r3;
    gl_mul128(a, b, r0, r1, r2, r3);
    return gl_reduce_limbs(r0, r1, r2, r3);
}
// a * b, canonical.
__device__ __forceinline__ uint64_t gl_mul_c(uint64_t a, uint64_t b) {
    uint32_t r0, r1, r2, r3;
    gl_mul128(a, b, r0, r1, r2, r3);
    return gl_reduce_limbs_c(r0, r1, r2, r3);
}

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

// Canonical add of canonical operands: s = a + b (65 bits); s - p is s + 2^32 - 1
// modulo 2^64, taken when either addition carries.
__device__ __forceinline__ uint64_t gl_add_c(uint64_t a, uint64_t b) {
    uint32_t r0, r1;
    asm("{\n\t"
        ".reg .u32 s0, s1, t0, t1, c;\n\t"
        ".reg .pred q;\n\t"
        "add.cc.u32 s0, %2, %4;\n\t"
        "addc.cc.u32 s1, %3, %5;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "add.cc.u32 t0, s0, 0xFFFFFFFF;\n\t"
        "addc.cc.u32 t1, s1, 0;\n\t"
        "addc.u32 c, c, 0;\n\t"
        "setp.ne.u32 q, c, 0;\n\t"
        "selp.b32 %0, t0, s0, q;\n\t"
        "selp.b32 %1, t1, s1, q;\n\t"
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
