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

__device__ __forceinline__ uint64_t gl_canon(uint64_t a) { return a >= GL_P ? a - GL_P : a; }

// (hi:lo) -> a 64-bit representative (not necessarily < p) of the residue.
__device__ __forceinline__ uint64_t gl_reduce128(uint64_t lo, uint64_t hi) {
    uint64_t hh = hi >> 32;
    uint64_t hl = hi & GL_EPS;
    uint64_t t = lo - hh;
    if (lo < hh) t -= GL_EPS;            // borrow: + p
    uint64_t u = (hl << 32) - hl;        // hl * (2^32 - 1), no overflow
    uint64_t r = t + u;
    if (r < u) r += GL_EPS;              // carry: - p
    return r;
}

// a * b for any 64-bit representatives; partial result.
__device__ __forceinline__ uint64_t gl_mul(uint64_t a, uint64_t b) {
    return gl_reduce128(a * b, __umul64hi(a, b));
}
__device__ __forceinline__ uint64_t gl_mul_c(uint64_t a, uint64_t b) { return gl_canon(gl_mul(a, b)); }

__device__ __forceinline__ uint64_t gl_sqr(uint64_t a) { return gl_mul(a, a); }

// a + b where b < p (a any representative); partial result.
__device__ __forceinline__ uint64_t gl_add_pc(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    if (s < b) s += GL_EPS;
    return s;
}

// Canonical add / sub of canonical operands.
__device__ __forceinline__ uint64_t gl_add_c(uint64_t a, uint64_t b) {
    uint64_t s = a + b;
    if (s < a || s >= GL_P) s -= GL_P;
    return s;
}
__device__ __forceinline__ uint64_t gl_sub_c(uint64_t a, uint64_t b) {
    uint64_t d = a - b;
    if (a < b) d += GL_P;
    return d;
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
