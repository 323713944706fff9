/*
 * CPU oracle for the table-commitment path (TEST INFRASTRUCTURE ONLY).
 *
 * This file is a plain-C restatement of the reference prover's CPU algorithms
 * for the low-degree extension (LDE), the Tip5 row hash and the Tip5 Merkle
 * tree.  It exists so that tests, the smoke check and the CPU-baseline leg of
 * the benchmark can check the CUDA product path bit-exactly.  No product code
 * may link or call it.
 *
 * Reference functions restated here (paths inside the reference project):
 *   Goldilocks field        src/types/b_field_element.cpp:11-192
 *   NTT forward / inverse   src/ntt/ntt.cpp:8-86   (radix-2 DIT after bit reversal)
 *   evaluate_on_coset       src/ntt/ntt.cpp:94-117
 *   LDE::extend_column      src/ntt/ntt.cpp:121-131
 *   RandomizedLDE           src/lde/lde_randomized.cpp:10-68 (zerofier * randomizer),
 *                           :71-154 (extend_column_with_randomizer, incl. chunked
 *                           evaluation), :178-277 (XFE variants: truncation to L)
 *   Tip5 permutation        src/hash/tip5.cpp:92-203
 *   Tip5::hash_varlen       src/hash/tip5.cpp:246-282
 *   Tip5::hash_10/hash_pair src/hash/tip5.cpp:224-297
 *   MerkleTree              src/merkle/merkle_tree.cpp:12-113 (heap layout, root at 1)
 *   authentication_structure_node_indices  src/merkle/merkle_tree.cpp:228-262
 *
 * Pinned by: the Tip5 known-answer tests of the upstream twenty-first crate
 * (triton-vm/twenty-first-local/twenty-first/src/tip5/mod.rs:1130-1200), the
 * primitive-root table of the same crate (src/math/b_field_element.rs:42-77),
 * and golden vectors produced by the reference's own C++ sources compiled
 * unchanged (oracle/_ref, see oracle/Makefile and tests/golden/make_golden.py).
 */
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

#define GL_P 0xFFFFFFFF00000001ULL
#define GL_EPS 0xFFFFFFFFULL /* 2^64 mod p */

/* ---------------------------------------------------------------- field -- */

static inline uint64_t gl_canon(uint64_t a) { return a >= GL_P ? a - GL_P : a; }

/* 128-bit -> canonical residue, using 2^64 = 2^32-1 and 2^96 = -1 (mod p). */
static inline uint64_t gl_reduce128(u128 x) {
    uint64_t lo = (uint64_t)x;
    uint64_t hi = (uint64_t)(x >> 64);
    uint64_t hh = hi >> 32, hl = hi & 0xFFFFFFFFULL;
    uint64_t t = lo - hh;
    if (lo < hh) t -= GL_EPS;
    uint64_t u = (hl << 32) - hl;
    uint64_t r = t + u;
    if (r < u) r += GL_EPS;
    return gl_canon(r);
}

uint64_t tvmo_add(uint64_t a, uint64_t b) {
    a = gl_canon(a); b = gl_canon(b);
    uint64_t s = a + b;
    if (s < a || s >= GL_P) s -= GL_P;
    return s;
}
uint64_t tvmo_sub(uint64_t a, uint64_t b) {
    a = gl_canon(a); b = gl_canon(b);
    return a >= b ? a - b : a + (GL_P - b);
}
uint64_t tvmo_mul(uint64_t a, uint64_t b) { return gl_reduce128((u128)a * b); }

uint64_t tvmo_pow(uint64_t base, uint64_t e) {
    uint64_t r = 1, b = gl_canon(base);
    while (e) {
        if (e & 1) r = tvmo_mul(r, b);
        b = tvmo_mul(b, b);
        e >>= 1;
    }
    return r;
}
uint64_t tvmo_inverse(uint64_t a) { return tvmo_pow(a, GL_P - 2); }

/* omega_k = 7^((p-1) >> k), k <= 32 (src/types/b_field_element.cpp:179-192). */
uint64_t tvmo_primitive_root(uint32_t log2_order) {
    if (log2_order > 32) return 0;
    return tvmo_pow(7, (GL_P - 1) >> log2_order);
}

/* ------------------------------------------------------------------ NTT -- */

static int ilog2_exact(size_t n) {
    if (n == 0 || (n & (n - 1))) return -1;
    int k = 0;
    while (((size_t)1 << k) < n) k++;
    return k;
}

static void bitrev_permute(uint64_t* a, size_t n, int logn) {
    for (size_t i = 0; i < n; i++) {
        size_t r = 0;
        for (int j = 0; j < logn; j++)
            if (i & ((size_t)1 << j)) r |= (size_t)1 << (logn - 1 - j);
        if (i < r) { uint64_t t = a[i]; a[i] = a[r]; a[r] = t; }
    }
}

/* In-place DIT NTT after bit-reversal; natural order in and out. */
static void ntt_core(uint64_t* a, size_t n, uint64_t omega, int inverse) {
    int logn = ilog2_exact(n);
    bitrev_permute(a, n, logn);
    for (size_t len = 2; len <= n; len <<= 1) {
        uint64_t wl = tvmo_pow(omega, n / len);
        size_t half = len >> 1;
        for (size_t i = 0; i < n; i += len) {
            uint64_t w = 1;
            for (size_t j = 0; j < half; j++) {
                uint64_t u = a[i + j];
                uint64_t v = tvmo_mul(a[i + j + half], w);
                a[i + j] = tvmo_add(u, v);
                a[i + j + half] = tvmo_sub(u, v);
                w = tvmo_mul(w, wl);
            }
        }
    }
    if (inverse) {
        uint64_t ninv = tvmo_inverse((uint64_t)n % GL_P);
        for (size_t i = 0; i < n; i++) a[i] = tvmo_mul(a[i], ninv);
    }
}

/* Returns 0 on success, -1 if n is not a power of two (ntt.cpp:61-63). */
int tvmo_ntt_forward(uint64_t* a, size_t n) {
    int logn = ilog2_exact(n);
    if (logn < 0) return -1;
    for (size_t i = 0; i < n; i++) a[i] = gl_canon(a[i]);
    ntt_core(a, n, tvmo_primitive_root((uint32_t)logn), 0);
    return 0;
}

int tvmo_ntt_inverse(uint64_t* a, size_t n) {
    int logn = ilog2_exact(n);
    if (logn < 0) return -1;
    for (size_t i = 0; i < n; i++) a[i] = gl_canon(a[i]);
    ntt_core(a, n, tvmo_inverse(tvmo_primitive_root((uint32_t)logn)), 1);
    return 0;
}

/* Zero-extend to L, scale c_i by offset^i, forward NTT of length L. */
int tvmo_evaluate_on_coset(const uint64_t* coeffs, size_t n, uint64_t* out, size_t L,
                           uint64_t offset) {
    if (ilog2_exact(L) < 0) return -1;
    uint64_t s = 1;
    for (size_t i = 0; i < L; i++) {
        uint64_t c = i < n ? gl_canon(coeffs[i]) : 0;
        out[i] = tvmo_mul(c, s);
        s = tvmo_mul(s, offset);
    }
    return tvmo_ntt_forward(out, L);
}

/* LDE::extend_column: interpolate on the size-n subgroup (trace offset is
 * ignored, as in the reference), then evaluate on offset * <omega_L>. */
int tvmo_lde_column(const uint64_t* trace, size_t n, uint64_t* out, size_t L, uint64_t offset) {
    if (ilog2_exact(n) < 0 || ilog2_exact(L) < 0) return -1;
    uint64_t* c = (uint64_t*)malloc(n * sizeof(uint64_t));
    if (!c) return -2;
    memcpy(c, trace, n * sizeof(uint64_t));
    tvmo_ntt_inverse(c, n);
    int rc = tvmo_evaluate_on_coset(c, n, out, L, offset);
    free(c);
    return rc;
}

/* Column-major table LDE: trace[c*n + r] -> out[c*L + r]. */
int tvmo_lde_table(const uint64_t* trace, size_t n, size_t width, uint64_t* out, size_t L,
                   uint64_t offset) {
    for (size_t c = 0; c < width; c++) {
        int rc = tvmo_lde_column(trace + c * n, n, out + c * L, L, offset);
        if (rc) return rc;
    }
    return 0;
}

/* RandomizedLDE::extend_column_with_randomizer: interpolant on the trace coset
 * t * <omega_n> (inverse NTT, then c_i * t^-i), plus the zerofier times the
 * randomizer, (x^n - t^n) * r(x), evaluated on o * <omega_L>.  A polynomial
 * longer than L is evaluated chunk by chunk, chunk k scaled by o^(kL), as the
 * reference does (truncate = 0); truncate = 1 drops every coefficient of
 * degree >= L first, as the reference's XFieldElement variants do. */
int tvmo_lde_randomized_column(const uint64_t* trace, size_t n, const uint64_t* r, size_t R, uint64_t* out,
                               size_t L, uint64_t t, uint64_t o, int truncate) {
    if (ilog2_exact(n) < 0 || ilog2_exact(L) < 0) return -1;
    size_t len = R ? n + R : n;
    uint64_t* p = (uint64_t*)calloc(len, sizeof(uint64_t));
    uint64_t* ev = (uint64_t*)malloc(L * sizeof(uint64_t));
    if (!p || !ev) {
        free(p), free(ev);
        return -2;
    }
    memcpy(p, trace, n * sizeof(uint64_t));
    tvmo_ntt_inverse(p, n);
    uint64_t ti = tvmo_inverse(gl_canon(t)), s = 1;
    for (size_t i = 0; i < n; i++) {
        p[i] = tvmo_mul(p[i], s);
        s = tvmo_mul(s, ti);
    }
    uint64_t tn = tvmo_pow(gl_canon(t), n);
    for (size_t k = 0; k < R; k++) {
        uint64_t rk = gl_canon(r[k]);
        p[k] = tvmo_sub(p[k], tvmo_mul(tn, rk));
        p[n + k] = tvmo_add(p[n + k], rk);
    }
    if (truncate && len > L) len = L;
    memset(out, 0, L * sizeof(uint64_t));
    for (size_t c0 = 0; c0 < len; c0 += L) {
        size_t m = len - c0 < L ? len - c0 : L;
        tvmo_evaluate_on_coset(p + c0, m, ev, L, o);
        uint64_t sc = tvmo_pow(gl_canon(o), c0);
        for (size_t j = 0; j < L; j++) out[j] = tvmo_add(out[j], tvmo_mul(ev[j], sc));
    }
    free(p), free(ev);
    return 0;
}

/* ----------------------------------------------------------------- Tip5 -- */

#define T5_STATE 16
#define T5_RATE 10
#define T5_ROUNDS 5

static uint8_t t5_lookup[256];
static int t5_ready = 0;

/* S-box byte map: the offset Fermat cube map x -> (x+1)^3 - 1 over F_257,
 * which is what the reference's 256-entry table tabulates (tip5.cpp:7-24). */
static void t5_init(void) {
    if (t5_ready) return;
    for (int x = 0; x < 256; x++) {
        int y = x + 1;
        int c = (y * y % 257) * y % 257;
        t5_lookup[x] = (uint8_t)((c + 256) % 257);
    }
    t5_ready = 1;
}

static const uint64_t t5_mds_col[T5_STATE] = {
    61402, 1108, 28750, 33823, 7454, 43244, 53865, 12034,
    56951, 27521, 41351, 40901, 12021, 59689, 26798, 17845};

static const uint64_t t5_rc[T5_ROUNDS * T5_STATE] = {
    0xBD2A3DEB61AB60DEULL, 0xEA7DF21AD9547ED2ULL, 0x900B3677A1DE063FULL, 0x1B46887E876C8677ULL,
    0xD364D977889CFB97ULL, 0xDC8DFAC843699F02ULL, 0x375C405D7190DB58ULL, 0x27924006D2B0D4B1ULL,
    0x78DD1172D483CD38ULL, 0x3346C66244882A56ULL, 0xB0249B279F498AA5ULL, 0x94CD51BE79338D4DULL,
    0xB0E0DC7052C5B218ULL, 0xF8DCC4D248ADAD95ULL, 0x68E3C635FEC868B7ULL, 0xD7D06B3FFB6B0D8CULL,
    0xF3500DEA20EF032AULL, 0x4865BF175BBA5803ULL, 0xD5F7FE3027287A27ULL, 0xA57333F44E193412ULL,
    0x8726E153A977EAE2ULL, 0x3014A98463FC191BULL, 0xBA145461AF39B212ULL, 0x03AB70105933202FULL,
    0x3D90B7EEBFCF71E5ULL, 0x386322B1CC520BFDULL, 0x27C2C8DAF774F675ULL, 0x4FCB83F50309BC6AULL,
    0x5E6D5CE8275F3CB3ULL, 0xECC2F6592C8F905CULL, 0x837F532461E609B4ULL, 0xB2B1F6B95C92C93CULL,
    0xC0027AF556411DC1ULL, 0x16E18C885FC2A26CULL, 0x8880EF183D9F2BF3ULL, 0xB2930BDB5CA88C45ULL,
    0x9C2EC8322E1C1553ULL, 0xE5B05EAF3220A674ULL, 0xA49CC6AE4B861C4EULL, 0x11708E0AEB86EBD7ULL,
    0xC09DE92BBC3902E0ULL, 0x929B3C79516BCBC1ULL, 0xE006E5BF738F27D1ULL, 0x2D9E1EC0EAC8EA38ULL,
    0x0984D8D94BF937C5ULL, 0x4959273C220E6747ULL, 0xFE1D934207E796FAULL, 0x2B9B9298F2F6DD73ULL,
    0x07A1F5A67D6E3A41ULL, 0x4407593EE73743D9ULL, 0x9F054720EF802E59ULL, 0x78D4B711336E6AA6ULL,
    0xADC638AEF3C8B228ULL, 0xA4D6D3E86AFB2114ULL, 0x9D4808E725531968ULL, 0x369804DF3866D0EFULL,
    0xE6DBD9A9D2215024ULL, 0x8ED22CA212EE85B2ULL, 0x397BB882FCD23EB6ULL, 0xEB8F8786D7277531ULL,
    0x9999D4CDAFF543B5ULL, 0xF382A61217F192D6ULL, 0x49C37260B026ADC1ULL, 0x3FF8918CE35C1019ULL,
    0x2E7DF8B76080BD07ULL, 0xF5DBAC250B8A28B9ULL, 0x853C3727AE9DA4CCULL, 0xB2F1F5F3D9E5A26DULL,
    0x3FCE22012D337847ULL, 0x6B5A3E6DB7EEE347ULL, 0x171582CD59DDE50DULL, 0xC0C0B3095EE62A8AULL,
    0x665B25C6F6A203D2ULL, 0x3099AED93B6AE69FULL, 0x801DF6092BE69C38ULL, 0x8066AD0CDFFF43CDULL,
    0x8AF9D44A5F4FDC6BULL, 0xD80219CD97C0D762ULL, 0x10C9CEBA14148EBBULL, 0x539BD4C3F2F24474ULL};

/* Montgomery reduction (hi:lo) * 2^-64 mod p, exactly as tip5.cpp:99-117. */
static uint64_t t5_montyred(uint64_t hi, uint64_t lo) {
    uint64_t sh = lo << 32;
    uint64_t a = lo + sh;
    int ovf = a < lo;
    uint64_t b = a - (a >> 32) - (uint64_t)ovf;
    uint64_t r = hi - b;
    if (hi < b) r -= GL_EPS;
    return r;
}

/* The parameter tables above, for checking a product's exported copies. */
void tvmo_tip5_parameters(uint8_t lookup[256], uint64_t mds[16], uint64_t rc[80]) {
    t5_init();
    memcpy(lookup, t5_lookup, 256);
    memcpy(mds, t5_mds_col, sizeof t5_mds_col);
    memcpy(rc, t5_rc, sizeof t5_rc);
}

/* split_and_lookup (tip5.cpp:119-145): to Montgomery form, byte-wise S-box,
 * back from Montgomery form; the result is reduced mod p. */
static uint64_t t5_split_lookup(uint64_t v) {
    const uint64_t R2 = 0xFFFFFFFE00000001ULL;
    u128 prod = (u128)gl_canon(v) * R2;
    uint64_t m = t5_montyred((uint64_t)(prod >> 64), (uint64_t)prod);
    uint64_t o = 0;
    for (int i = 0; i < 8; i++) o |= (uint64_t)t5_lookup[(m >> (8 * i)) & 0xFF] << (8 * i);
    return gl_canon(t5_montyred(0, o));
}

void tvmo_tip5_permutation(uint64_t st[T5_STATE]) {
    t5_init();
    for (int i = 0; i < T5_STATE; i++) st[i] = gl_canon(st[i]);
    for (int r = 0; r < T5_ROUNDS; r++) {
        for (int i = 0; i < 4; i++) st[i] = t5_split_lookup(st[i]);
        for (int i = 4; i < T5_STATE; i++) {
            uint64_t x2 = tvmo_mul(st[i], st[i]);
            uint64_t x4 = tvmo_mul(x2, x2);
            st[i] = tvmo_mul(tvmo_mul(st[i], x2), x4);
        }
        uint64_t ns[T5_STATE];
        for (int row = 0; row < T5_STATE; row++) {
            u128 acc = 0;
            for (int col = 0; col < T5_STATE; col++)
                acc += (u128)t5_mds_col[(row - col) & 15] * st[col];
            ns[row] = gl_reduce128(acc);
        }
        for (int i = 0; i < T5_STATE; i++) st[i] = tvmo_add(ns[i], t5_rc[r * T5_STATE + i]);
    }
}

/* hash_varlen over n elements read at in[i*stride]: zero state, overwrite the
 * rate with each full chunk and permute; last chunk = rest, 1, zeros. */
void tvmo_hash_varlen_strided(const uint64_t* in, size_t n, size_t stride, uint64_t out[5]) {
    uint64_t st[T5_STATE] = {0};
    size_t done = 0;
    while (done + T5_RATE <= n) {
        for (int i = 0; i < T5_RATE; i++) st[i] = in[(done + i) * stride];
        tvmo_tip5_permutation(st);
        done += T5_RATE;
    }
    size_t rem = n - done;
    for (size_t i = 0; i < T5_RATE; i++) st[i] = i < rem ? in[(done + i) * stride] : (i == rem);
    tvmo_tip5_permutation(st);
    for (int i = 0; i < 5; i++) out[i] = st[i];
}

void tvmo_hash_varlen(const uint64_t* in, size_t n, uint64_t out[5]) {
    tvmo_hash_varlen_strided(in, n, 1, out);
}

void tvmo_hash_10(const uint64_t in[10], uint64_t out[5]) {
    uint64_t st[T5_STATE];
    for (int i = 0; i < T5_RATE; i++) st[i] = in[i];
    for (int i = T5_RATE; i < T5_STATE; i++) st[i] = 1;
    tvmo_tip5_permutation(st);
    for (int i = 0; i < 5; i++) out[i] = st[i];
}

void tvmo_hash_pair(const uint64_t l[5], const uint64_t r[5], uint64_t out[5]) {
    uint64_t in[10];
    for (int i = 0; i < 5; i++) { in[i] = l[i]; in[5 + i] = r[i]; }
    tvmo_hash_10(in, out);
}

/* Digest of every row: element (r, c) is at table[r*row_stride + c*col_stride]. */
void tvmo_hash_rows(const uint64_t* table, size_t rows, size_t cols, size_t row_stride,
                    size_t col_stride, uint64_t* digests) {
    for (size_t r = 0; r < rows; r++)
        tvmo_hash_varlen_strided(table + r * row_stride, cols, col_stride, digests + 5 * r);
}

/* --------------------------------------------------------------- Merkle -- */

/* nodes: 2*n digests (5 words each), heap layout; leaves at [n, 2n), root at 1,
 * node 0 unused (written as zeros). Returns -1 if n is not a power of two. */
int tvmo_merkle_build(const uint64_t* leaves, size_t n, uint64_t* nodes) {
    if (ilog2_exact(n) < 0) return -1;
    memset(nodes, 0, 5 * sizeof(uint64_t));
    memcpy(nodes + 5 * n, leaves, 5 * n * sizeof(uint64_t));
    for (size_t i = n - 1; i >= 1; i--) tvmo_hash_pair(nodes + 10 * i, nodes + 10 * i + 5, nodes + 5 * i);
    return 0;
}

/* Sibling digests from the leaf up to (excluding) the root: log2(n) digests. */
int tvmo_auth_path(const uint64_t* nodes, size_t n, size_t leaf, uint64_t* out) {
    if (leaf >= n) return -1;
    size_t k = 0;
    for (size_t i = n + leaf; i > 1; i >>= 1, k++) memcpy(out + 5 * k, nodes + 5 * (i ^ 1), 40);
    return (int)k;
}

static int cmp_desc(const void* a, const void* b) {
    size_t x = *(const size_t*)a, y = *(const size_t*)b;
    return x < y ? 1 : (x > y ? -1 : 0);
}

/* Heap indices of the authentication structure: siblings of every node on a
 * leaf-to-root path that are not themselves on one, sorted descending
 * (merkle_tree.cpp:228-262). Writes at most max_out indices; returns count or
 * -1 on bad input. */
long tvmo_auth_structure_indices(size_t n, const size_t* leaves, size_t m, size_t* out, size_t max_out) {
    if (ilog2_exact(n) < 0) return -1;
    unsigned char* mark = (unsigned char*)calloc(2 * n, 1); /* bit0 on-path, bit1 needed */
    if (!mark) return -1;
    for (size_t j = 0; j < m; j++) {
        if (leaves[j] >= n) { free(mark); return -1; }
        for (size_t i = n + leaves[j]; i > 1; i >>= 1) { mark[i] |= 1; mark[i ^ 1] |= 2; }
    }
    size_t cnt = 0;
    for (size_t i = 2 * n - 1; i >= 1; i--)
        if (mark[i] == 2) { if (cnt < max_out) out[cnt] = i; cnt++; }
    free(mark);
    qsort(out, cnt < max_out ? cnt : max_out, sizeof(size_t), cmp_desc);
    return (long)cnt;
}

int tvmo_merkle_verify(const uint64_t root[5], size_t leaf, const uint64_t d[5], const uint64_t* path,
                       size_t len) {
    uint64_t cur[5], nxt[5];
    memcpy(cur, d, 40);
    for (size_t k = 0; k < len; k++, leaf >>= 1) {
        if (leaf & 1) tvmo_hash_pair(path + 5 * k, cur, nxt);
        else tvmo_hash_pair(cur, path + 5 * k, nxt);
        memcpy(cur, nxt, 40);
    }
    return memcmp(cur, root, 40) == 0;
}

/* Whole commit on the CPU: column-major trace (n x width) -> column-major LDE
 * (L x width), leaf digests and the heap tree (2L digests). */
int tvmo_commit(const uint64_t* trace, size_t n, size_t width, size_t L, uint64_t offset,
                uint64_t* lde, uint64_t* nodes) {
    int rc = tvmo_lde_table(trace, n, width, lde, L, offset);
    if (rc) return rc;
    uint64_t* leaves = (uint64_t*)malloc(L * 40);
    if (!leaves) return -2;
    tvmo_hash_rows(lde, L, width, 1, L, leaves);
    rc = tvmo_merkle_build(leaves, L, nodes);
    free(leaves);
    return rc;
}
