// Tip5 permutation for sm_100a, one sponge state per thread held in registers.
//
// Semantics follow the reference's Tip5 (src/hash/tip5.cpp:92-203): 16-word
// state, 5 rounds of [S-box -> MDS -> round constants].  The S-box applies
// split-and-lookup to words 0-3 (a byte-wise table on the Montgomery
// representation) and x^7 to words 4-15; the MDS is the circulant matrix whose
// first column is given below.  The byte table is the offset Fermat cube map
// x -> (x+1)^3 - 1 over F_257, generated here rather than tabulated.
//
// B200 layout choices (measured on sm_100a: 32-bit IMAD and DFMA are
// half-rate, IMAD.HI quarter-rate, IMAD.WIDE takes two issue slots):
//   * the hashing kernels keep the state in Montgomery form (w * 2^64 mod p,
//     the representation the reference's BFieldElement holds), converting at
//     absorb and squeeze only: the byte lookups then need no conversion, and
//     every x^7 product reduces by a nine-instruction Montgomery reduction
//     (gl_redc) instead of a two-step reduction and canonicalisation;
//   * the byte table lives in shared memory as 256 words x 32 lanes, one
//     entry per word and every lane owning its own bank, so the 8 lookups per
//     word never conflict and the looked-up bytes are assembled by byte
//     permutes with constant selectors;
//   * the MDS runs exactly on the FP64 pipe (t5_mds), in parallel with the
//     integer S-box work on the ALU/FMA pipes; being linear with integer
//     entries it commutes with the Montgomery form, and its round constants
//     are stored in that form;
//   * x^7 runs unrolled over the twelve words.
#pragma once
#include <cstdint>
#include "field.cuh"
#include "tip5_params.h"

namespace tvmc {

constexpr int T5_STATE = 16;
constexpr int T5_RATE = 10;
constexpr int T5_ROUNDS = 5;

// The MDS first column is inlined in t5_mds_half as FP64 literals.  The round
// constants (tip5_params.h) enter the MDS's last FMA (t5_mds): the biases
// below carry each constant's 32-bit halves.
constexpr double t5_mds_column_sum() {
    const double m[T5_STATE] = {TVMC_T5_MDS_FIRST_COLUMN};
    double acc = 0.0;
    for (int k = 0; k < T5_STATE; k++) acc += m[k];
    return acc;
}
// 2^52 + 2^31 * sum(M): the output bias of a centred half-product (t5_mds_half).
constexpr double T5_MDS_BIAS = 4503599627370496.0 + 2147483648.0 * t5_mds_column_sum();

// x * 2^64 (mod p) at compile time: x0 * (2^32 - 1) - x1 for x = x1 * 2^32 + x0.
constexpr uint64_t t5_to_mont_const(uint64_t x) {
    const uint64_t v = (x & 0xFFFFFFFFull) * 0xFFFFFFFFull, x1 = x >> 32;
    return v >= x1 ? v - x1 : GL_P - (x1 - v);
}
// t5_recombine takes the high words of the biased MDS halves as they are,
// exponent bits included: each is L1 + K (H1 + K) with K = 0x43300000, which
// adds 2K * 2^32 - K to every result; the round constants carry its negative.
constexpr uint64_t T5_RECOMBINE_EXCESS = 2ull * 0x43300000ull * 0x100000000ull - 0x43300000ull;
// The round constants enter in Montgomery form, like the state (t5_permutation_m).
struct T5RoundBias {
    double lo[T5_ROUNDS * T5_STATE];  // T5_MDS_BIAS + (rc * 2^64 mod p) & (2^32 - 1)
    double hi[T5_ROUNDS * T5_STATE];  // T5_MDS_BIAS + (rc * 2^64 mod p) >> 32
};
constexpr T5RoundBias t5_round_bias() {
    const uint64_t rc[T5_ROUNDS * T5_STATE] = {TVMC_T5_ROUND_CONSTANTS};
    T5RoundBias b{};
    for (int i = 0; i < T5_ROUNDS * T5_STATE; i++) {
        // less the constant that t5_recombine's unmasked high limbs add
        const uint64_t m0 = t5_to_mont_const(rc[i]);
        const uint64_t m = m0 >= T5_RECOMBINE_EXCESS ? m0 - T5_RECOMBINE_EXCESS : m0 + (GL_P - T5_RECOMBINE_EXCESS);
        b.lo[i] = T5_MDS_BIAS + (double)(uint32_t)m;
        b.hi[i] = T5_MDS_BIAS + (double)(uint32_t)(m >> 32);
    }
    return b;
}
// 1 in Montgomery form (2^64 mod p): the capacity of hash_pair and the padding 1.
constexpr uint64_t T5_MONT_ONE = 0xFFFFFFFFull;
__device__ __constant__ T5RoundBias c_t5_bias = t5_round_bias();

// Shared-memory S-box table (32 KB): word v*32 + l holds the table byte for
// input byte v, in lane l's private column.
constexpr int T5_SBOX_WORDS = 256 * 32;

// The byte table itself, generated at compile time: v -> (v + 1)^3 - 1 over F_257.
struct T5Sbox {
    uint32_t v[256];
};
constexpr T5Sbox t5_sbox_bytes() {
    T5Sbox t{};
    for (int v = 0; v < 256; v++) {
        const int x = v + 1;
        t.v[v] = (uint32_t)(((x * x % 257) * x % 257 + 256) % 257);
    }
    return t;
}
__device__ __constant__ T5Sbox c_t5_sbox = t5_sbox_bytes();

// Fill the lane-replicated byte table from the constant bank (all 32 lanes of
// a warp read the same entry); call from all threads, then sync.
__device__ __forceinline__ void t5_sbox_init(uint32_t* tbl) {
    for (int i = threadIdx.x; i < T5_SBOX_WORDS; i += blockDim.x) tbl[i] = c_t5_sbox.v[i >> 5];
}

// Byte-wise S-box of a 32-bit word through the lane's private table column:
// each index byte is extracted by one byte permute (selector 0x444k: byte k,
// zero-extended), each lookup returns its byte in bits 0-7, so the assembly is
// three byte permutes with constant selectors.
__device__ __forceinline__ uint32_t t5_lookup32(uint32_t m, const uint32_t* lane_tbl) {
    const uint32_t w0 = lane_tbl[__byte_perm(m, 0, 0x4440) << 5];
    const uint32_t w1 = lane_tbl[__byte_perm(m, 0, 0x4441) << 5];
    const uint32_t w2 = lane_tbl[__byte_perm(m, 0, 0x4442) << 5];
    const uint32_t w3 = lane_tbl[__byte_perm(m, 0, 0x4443) << 5];
    return __byte_perm(__byte_perm(w0, w1, 0x0040), __byte_perm(w2, w3, 0x0040), 0x5410);
}

// split_and_lookup on a state word held in Montgomery form (t5_permutation_m):
// the reference applies the byte table to the canonical Montgomery
// representation and keeps the result as the new Montgomery representation
// (src/hash/tip5.cpp:119-145), so only a canonicalisation precedes the lookups.
__device__ __forceinline__ uint64_t t5_split_lookup_m(uint64_t x, const uint32_t* lane_tbl) {
    const uint64_t y = gl_canon(x);
    const uint32_t y0 = t5_lookup32((uint32_t)y, lane_tbl);
    const uint32_t y1 = t5_lookup32((uint32_t)(y >> 32), lane_tbl);
    return ((uint64_t)y1 << 32) | y0;
}

// x^7 of a Montgomery-form word: four Montgomery products (gl_redc, nine ALU
// instructions each); any 64-bit representative in and out.
__device__ __forceinline__ uint64_t t5_pow7_m(uint64_t x) {
    uint32_t r0, r1, r2, r3;
    gl_sqr128(x, r0, r1, r2, r3);
    const uint64_t x2 = gl_redc(r0, r1, r2, r3);
    gl_mul128(x, x2, r0, r1, r2, r3);
    const uint64_t x3 = gl_redc(r0, r1, r2, r3);
    gl_sqr128(x2, r0, r1, r2, r3);
    const uint64_t x4 = gl_redc(r0, r1, r2, r3);
    gl_mul128(x3, x4, r0, r1, r2, r3);
    return gl_redc(r0, r1, r2, r3);
}

// Circulant MDS: out[r] = sum_c M[(r - c) mod 16] * s[c] (mod p), i.e. the
// cyclic convolution m(x) s(x) mod x^16 - 1.  Each word is split into 32-bit
// halves and each half is convolved exactly on the FP64 pipe, through the
// factorisation x^16 - 1 = (x^4 - 1)(x^4 + 1)(x^8 + 1): the half is reduced
// modulo each factor (additions), multiplied there by the matching reduction of
// m (a cyclic 4-point, a negacyclic 4-point and a negacyclic 8-point product:
// 96 DFMAs instead of the 256 of the direct product), and recombined by the
// inverse of the same butterflies.  The halves are centred (v - 2^31), so
// every intermediate is an integer of magnitude at most 524757 * 2^33 < 2^53
// (524757 = sum of the column, an upper bound on the l1 norm of every reduced
// column), hence exact; the last FMA scales by 1/4 and adds bias[r] =
// T5_MDS_BIAS + a[r] (2^52 + 2^31 * 524757 undoes the centring; a[r] < 2^32 is
// the round constant's half), leaving y + a + 2^52 with y + a < 2^52 exact.
// The halves are then recombined as lo + hi*2^32 with one 128-bit reduction per
// word.  Moving this work off the integer pipes leaves them to the S-box.
// Inputs x[c] = 2^52 + v_c (t5_half_biased); the first butterflies centre them
// for free: x_j - x_{j+8} = v_j - v_{j+8}, and (x_j - 2*(2^52 + 2^31)) + x_{j+8}
// = (v_j - 2^31) + (v_{j+8} - 2^31), both exact (every operand and sum is an
// integer below 2^53 in magnitude).
constexpr double T5_HALF_BIAS = 4503599627370496.0 + 2147483648.0;  // 2^52 + 2^31
__host__ __device__ __forceinline__ void t5_mds_half(double x[T5_STATE], const double* bias) {
    const double M[T5_STATE] = {TVMC_T5_MDS_FIRST_COLUMN};
    // reductions of the half modulo x^8 - 1 (a), x^8 + 1 (d), x^4 - 1 (e), x^4 + 1 (f)
    double a[8], d[8], e[4], f[4];
#pragma unroll
    for (int j = 0; j < 8; j++) {
        a[j] = (x[j] - 2.0 * T5_HALF_BIAS) + x[j + 8];
        d[j] = x[j] - x[j + 8];
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        e[j] = a[j] + a[j + 4];
        f[j] = a[j] - a[j + 4];
    }
    // the same reductions of m: cyclic-4 c4, negacyclic-4 n4, negacyclic-8 n8
    double P[4], Q[4], V[8];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        double p = 0.0, q = 0.0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int i = (r - k) & 3;
            const double c4 = M[i] + M[i + 4] + M[i + 8] + M[i + 12];
            const double n4 = (M[i] + M[i + 8]) - (M[i + 4] + M[i + 12]);
            p = fma(c4, e[k], p);
            q = fma(k > r ? -n4 : n4, f[k], q);
        }
        P[r] = p;
        Q[r] = q;
    }
#pragma unroll
    for (int r = 0; r < 8; r++) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int i = (r - k) & 7;
            const double n8 = M[i] - M[i + 8];
            v = fma(k > r ? -n8 : n8, d[k], v);
        }
        V[r] = v;
    }
    // inverse butterflies: 2u_r = P + Q, 2u_{r+4} = P - Q (u = result mod x^8 - 1),
    // 4y_r = 2u_r + 2V_r, 4y_{r+8} = 2u_r - 2V_r
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const double s = P[r] + Q[r], t = P[r] - Q[r];
        x[r] = fma(fma(V[r], 2.0, s), 0.25, bias[r]);
        x[r + 8] = fma(fma(V[r], -2.0, s), 0.25, bias[r + 8]);
        x[r + 4] = fma(fma(V[r + 4], 2.0, t), 0.25, bias[r + 4]);
        x[r + 12] = fma(fma(V[r + 4], -2.0, t), 0.25, bias[r + 12]);
    }
}

// A 32-bit half v as the double 2^52 + v (the bits 0x43300000:v).
__device__ __forceinline__ double t5_half_biased(uint32_t v) {
    return __hiloint2double(0x43300000, (int)v);
}

// lo + hi*2^32 (mod p) from the two biased MDS halves 2^52 + lo and 2^52 + hi
// (lo, hi < 2^52), as 32-bit limbs: with lo = L1*2^32 + L0 and hi = H1*2^32 + H0
// (L1, H1 < 2^20), lo + hi*2^32 = L0 + (L1 + H0)*2^32 + H1*2^64, and
// 2^64 = 2^32 - 1 (mod p) turns it into L0 - H1 + (H0 + L1 + H1)*2^32.  The
// carry c of the high sum and the borrows of the subtraction net to c in
// {-1, 0, 1}, folded back as c*(2^32 - 1): for c = 1 the high limb is at most
// 2^32 - 2, for c = -1 it is 2^32 - 1, so the fold cannot wrap.  The low limbs of
// the doubles are L0 and H0 as they are; the high limbs enter unmasked, as
// L1 + K and H1 + K (K = 0x43300000, the exponent bits; 2K + L1 + H1 < 2^32),
// and the constant this adds is taken out of the round constants
// (T5_RECOMBINE_EXCESS).
__device__ __forceinline__ uint64_t t5_recombine(double dlo, double dhi) {
    const uint32_t l0 = (uint32_t)__double2loint(dlo), l1 = (uint32_t)__double2hiint(dlo);
    const uint32_t h0 = (uint32_t)__double2loint(dhi), h1 = (uint32_t)__double2hiint(dhi);
    uint32_t x0, x1;
    asm("{\n\t"
        ".reg .u32 a, c, e0, e1;\n\t"
        "add.u32 a, %3, %5;\n\t"
        "add.cc.u32 %1, %4, a;\n\t"
        "addc.u32 c, 0, 0;\n\t"
        "sub.cc.u32 %0, %2, %5;\n\t"
        "subc.cc.u32 %1, %1, 0;\n\t"
        "subc.u32 c, c, 0;\n\t"
        "neg.s32 e0, c;\n\t"
        "shr.s32 e1, c, 31;\n\t"
        "add.cc.u32 %0, %0, e0;\n\t"
        "addc.u32 %1, %1, e1;\n\t"
        "}"
        : "=r"(x0), "=r"(x1)
        : "r"(l0), "r"(l1), "r"(h0), "r"(h1));
    return ((uint64_t)x1 << 32) | x0;
}

// MDS of the state plus the round constants of round rnd.
__device__ __forceinline__ void t5_mds(uint64_t s[T5_STATE], int rnd) {
    double dl[T5_STATE], dh[T5_STATE];
#pragma unroll
    for (int c = 0; c < T5_STATE; c++) {
        dl[c] = t5_half_biased((uint32_t)s[c]);
        dh[c] = t5_half_biased((uint32_t)(s[c] >> 32));
    }
    t5_mds_half(dl, c_t5_bias.lo + rnd * T5_STATE);
    t5_mds_half(dh, c_t5_bias.hi + rnd * T5_STATE);
#pragma unroll
    for (int r = 0; r < T5_STATE; r++) s[r] = t5_recombine(dl[r], dh[r]);
}

// x^7 on words 4..15, written as two groups of six that the compiler unrolls
// (the rotation between the groups becomes register renaming).  With the
// Montgomery-form products the unrolled round body is small enough for the
// instruction cache: unrolled measured 3.1% faster than the rolled loop (with
// the earlier plain-form products it had measured 3.4% slower).
__device__ __forceinline__ void t5_pow7_layer_m(uint64_t s[T5_STATE]) {
#pragma unroll
    for (int g = 0; g < 2; g++) {
#pragma unroll
        for (int i = 4; i < 10; i++) s[i] = t5_pow7_m(s[i]);
        uint64_t t[6];
#pragma unroll
        for (int i = 0; i < 6; i++) t[i] = s[4 + i];
#pragma unroll
        for (int i = 4; i < 10; i++) s[i] = s[i + 6];
#pragma unroll
        for (int i = 0; i < 6; i++) s[10 + i] = t[i];
    }
}

// The permutation on a state held in Montgomery form (every word w * 2^64 mod
// p, any 64-bit representative): the form the reference's BFieldElement keeps
// internally.  The byte lookups then need no conversion, the x^7 products
// reduce by gl_redc, and the MDS, being linear with integer entries, commutes
// with the form; its round constants are stored in Montgomery form.
__device__ __forceinline__ void t5_permutation_m(uint64_t s[T5_STATE], const uint32_t* lane_tbl) {
#pragma unroll 1
    for (int rnd = 0; rnd < T5_ROUNDS; rnd++) {
#pragma unroll
        for (int i = 0; i < 4; i++) s[i] = t5_split_lookup_m(s[i], lane_tbl);
        t5_pow7_layer_m(s);
        t5_mds(s, rnd);  // and the round constants
    }
}

// The permutation on a plain state (any representatives in, canonical out).
__device__ __forceinline__ void t5_permutation(uint64_t s[T5_STATE], const uint32_t* lane_tbl) {
#pragma unroll
    for (int i = 0; i < T5_STATE; i++) s[i] = gl_to_mont(s[i]);
    t5_permutation_m(s, lane_tbl);
#pragma unroll
    for (int i = 0; i < T5_STATE; i++) s[i] = gl_from_mont(s[i]);
}

// One round (Tip5::round, src/hash/tip5.cpp:114-118) on a plain state, for the
// off-path single-round and trace entry points.
__device__ __forceinline__ void t5_round(uint64_t s[T5_STATE], const uint32_t* lane_tbl, int rnd) {
#pragma unroll
    for (int i = 0; i < T5_STATE; i++) s[i] = gl_to_mont(s[i]);
#pragma unroll
    for (int i = 0; i < 4; i++) s[i] = t5_split_lookup_m(s[i], lane_tbl);
    t5_pow7_layer_m(s);
    t5_mds(s, rnd);
#pragma unroll
    for (int i = 0; i < T5_STATE; i++) s[i] = gl_from_mont(s[i]);
}

// Tip5::hash_pair / hash_10: rate = left || right, capacity = 1s; plain digests
// in, canonical digest out.
__device__ __forceinline__ void t5_hash_pair(const uint64_t l[5], const uint64_t r[5], uint64_t out[5],
                                             const uint32_t* lane_tbl) {
    uint64_t s[T5_STATE];
#pragma unroll
    for (int i = 0; i < 5; i++) { s[i] = gl_to_mont(l[i]); s[5 + i] = gl_to_mont(r[i]); }
#pragma unroll
    for (int i = T5_RATE; i < T5_STATE; i++) s[i] = T5_MONT_ONE;
    t5_permutation_m(s, lane_tbl);
#pragma unroll
    for (int i = 0; i < 5; i++) out[i] = gl_from_mont(s[i]);
}

}  // namespace tvmc
