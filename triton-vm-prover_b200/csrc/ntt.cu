// Batched Goldilocks NTT and fused low-degree extension (sm_100a).
//
// Every transform here is the DFT X[k] = sum_i x[i] w^(ik) with natural-order
// input and output, w = 7^((p-1)/n) (src/types/b_field_element.cpp:179-192);
// the inverse uses w^-1 and scales by n^-1 (src/ntt/ntt.cpp:59-86).  Results
// are canonical, so they equal the reference's radix-2 DIT bit for bit.
//
// Sizes up to 2^11 run in one pass per column (whole column in shared memory).
// Larger sizes use the four-step split n = n1*n2, i = i1 + n1*i2,
// k = n2*k1 + k2:
//   pass A: for each i1, DFT_n2 over i2 (elements at stride n1), times w^(i1*k2)
//   pass B: for each k2, DFT_n1 over i1 (contiguous rows) -> X[n2*k1 + k2]
// Each CTA moves T sequences at a time so that global accesses come in runs
// of T consecutive words.
//
// LDE (LDE::extend_column, src/ntt/ntt.cpp:121-131; evaluate_on_coset :94-117):
// the E*N-point forward transform of the zero-padded, offset-scaled
// coefficients is evaluated as E cosets of size N, LDE[E*q + c] =
// DFT_N(coef_i * s_c^i)[q] with s_c = offset * w_{EN}^c, because
// w_{EN}^(i(Eq+c)) = w_N^(iq) * w_{EN}^(ic).  The inverse's pass B and the
// forward's pass A touch the same index sets when the forward split is taken
// as (n2, n1), so one kernel does both for all E cosets:
//   K1 (lde_inv_a): inverse pass A, trace -> Y
//   K2 (lde_mid):   inverse pass B, scale by N^-1 s_c^i, forward pass A -> Z_c
//   K3 (lde_fwd_b): forward pass B for all cosets, written interleaved -> LDE
#include "internal.cuh"
#include "field.cuh"

namespace tvmc {

__device__ __forceinline__ uint32_t brev_bits(uint32_t k, int bits) {
    return bits == 0 ? 0u : (__brev(k) >> (32 - bits));
}

__device__ __forceinline__ uint64_t tw2(const uint64_t* __restrict__ lo, const uint64_t* __restrict__ hi,
                                        uint32_t e) {
    return gl_mul(__ldg(lo + (e & 4095)), __ldg(hi + (e >> 12)));
}

// Radix-2 DIF on T interleaved sequences of length 2^ls held in shared memory
// (element k of sequence t at s[k*T + t], T = 2^lT).  On return element k of
// the transform sits at s[brev(k)*T + t].  tw[m] = w^m, m < 2^(ls-1).
__device__ void dif_smem(uint64_t* s, int ls, int lT, const uint64_t* tw) {
    const int T = 1 << lT;
    const int half_total = (1 << (ls - 1)) * T;
    for (int st = 0; st < ls; st++) {
        const int lh = ls - 1 - st;
        const int h = 1 << lh;
        for (int b = threadIdx.x; b < half_total; b += blockDim.x) {
            const int t = b & (T - 1);
            const int q = b >> lT;
            const int j = q & (h - 1);
            const int i0 = ((q >> lh) << (lh + 1)) + j;
            uint64_t* p0 = s + (i0 << lT) + t;
            uint64_t* p1 = p0 + (h << lT);
            uint64_t a = *p0, c = *p1;
            *p0 = gl_add_c(a, c);
            *p1 = gl_mul_c(gl_sub_c(a, c), tw[j << st]);
        }
        __syncthreads();
    }
}

__device__ __forceinline__ void load_tw(uint64_t* tw, const uint64_t* __restrict__ tw12, int ls) {
    const int half = ls > 0 ? (1 << (ls - 1)) : 0;
    for (int m = threadIdx.x; m < half; m += blockDim.x) tw[m] = __ldg(tw12 + (m << (12 - ls)));
}

// ---------------------------------------------------------------- plain NTT

// Whole columns in shared memory: T = 2^lT columns per CTA, size 2^ls <= 2^11.
__global__ void k_ntt_small(uint64_t* data, uint64_t ld, uint64_t cols, int ls, int lT, const uint64_t* tw12,
                            uint64_t scale) {
    extern __shared__ uint64_t sm[];
    const int n = 1 << ls, T = 1 << lT;
    uint64_t* tw = sm;
    uint64_t* s = sm + (n > 1 ? n / 2 : 1);
    load_tw(tw, tw12, ls);
    const uint64_t c0 = (uint64_t)blockIdx.x * T;
    for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
        int t = idx / n, k = idx - t * n;  // coalesced: consecutive k of one column
        uint64_t col = c0 + t;
        s[(k << lT) + t] = col < cols ? gl_canon(data[col * ld + k]) : 0;
    }
    __syncthreads();
    if (ls > 0) dif_smem(s, ls, lT, tw);
    for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
        int t = idx / n, k = idx - t * n;
        uint64_t col = c0 + t;
        if (col < cols) data[col * ld + k] = gl_mul_c(s[(brev_bits(k, ls) << lT) + t], scale);
    }
}

// Pass A: out[i1 + n1*k2] = w^(i1*k2) * DFT_n2(in[i1 + n1*i2])[k2]; in may equal out.
__global__ void k_pass_a(const uint64_t* in, uint64_t ild, uint64_t* out, uint64_t old, int l1, int l2, int lT,
                         const uint64_t* tw12, const uint64_t* wlo, const uint64_t* whi) {
    extern __shared__ uint64_t sm[];
    const int n2 = 1 << l2, T = 1 << lT;
    uint64_t* tw = sm;
    uint64_t* s = sm + n2 / 2;
    load_tw(tw, tw12, l2);
    const uint64_t col = blockIdx.y;
    const uint32_t i10 = blockIdx.x << lT;
    const uint64_t* src = in + col * ild;
    for (int idx = threadIdx.x; idx < (n2 << lT); idx += blockDim.x) {
        int t = idx & (T - 1), i2 = idx >> lT;
        s[idx] = gl_canon(src[i10 + t + ((uint64_t)i2 << l1)]);
    }
    __syncthreads();
    dif_smem(s, l2, lT, tw);
    uint64_t* dst = out + col * old;
    for (int idx = threadIdx.x; idx < (n2 << lT); idx += blockDim.x) {
        int t = idx & (T - 1), k2 = idx >> lT;
        uint64_t v = s[(brev_bits(k2, l2) << lT) + t];
        v = gl_mul_c(v, tw2(wlo, whi, (i10 + t) * (uint32_t)k2));
        dst[i10 + t + ((uint64_t)k2 << l1)] = v;
    }
}

// Pass B: out[n2*k1 + k2] = scale * DFT_n1(in[i1 + n1*k2])[k1]; in != out.
__global__ void k_pass_b(const uint64_t* in, uint64_t ild, uint64_t* out, uint64_t old, int l1, int l2, int lT,
                         const uint64_t* tw12, uint64_t scale) {
    extern __shared__ uint64_t sm[];
    const int n1 = 1 << l1, T = 1 << lT;
    uint64_t* tw = sm;
    uint64_t* s = sm + n1 / 2;
    load_tw(tw, tw12, l1);
    const uint64_t col = blockIdx.y;
    const uint32_t k20 = blockIdx.x << lT;
    const uint64_t* src = in + col * ild + ((uint64_t)k20 << l1);
    for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
        int t = idx >> l1, i1 = idx & (n1 - 1);  // coalesced along a row
        s[(i1 << lT) + t] = src[idx];
    }
    __syncthreads();
    dif_smem(s, l1, lT, tw);
    uint64_t* dst = out + col * old;
    for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
        int t = idx & (T - 1), k1 = idx >> lT;
        uint64_t v = s[(brev_bits(k1, l1) << lT) + t];
        dst[((uint64_t)k1 << l2) + k20 + t] = gl_mul_c(v, scale);
    }
}

// ---------------------------------------------------------------------- LDE

// Small LDE: whole column in shared memory (N <= 2^11), T columns per CTA.
__global__ void k_lde_small(const uint64_t* trace, uint64_t tld, uint64_t* out, uint64_t old, uint64_t cols,
                            int ls, int lT, int le, const uint64_t* tw12_i, const uint64_t* tw12_f,
                            const uint64_t* sc_lo, const uint64_t* sc_hi, int hi_len) {
    extern __shared__ uint64_t sm[];
    const int n = 1 << ls, T = 1 << lT, E = 1 << le;
    const int hw = n > 1 ? n / 2 : 1;
    uint64_t* twi = sm;
    uint64_t* twf = twi + hw;
    uint64_t* s = twf + hw;     // coefficients, T x n
    uint64_t* w = s + n * T;    // work, T x n
    load_tw(twi, tw12_i, ls);
    load_tw(twf, tw12_f, ls);
    const uint64_t c0 = (uint64_t)blockIdx.x * T;
    for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
        int t = idx / n, k = idx - t * n;
        uint64_t col = c0 + t;
        s[(k << lT) + t] = col < cols ? gl_canon(trace[col * tld + k]) : 0;
    }
    __syncthreads();
    if (ls > 0) dif_smem(s, ls, lT, twi);
    for (int c = 0; c < E; c++) {
        const uint64_t* lo = sc_lo + 4096 * c;
        const uint64_t* hi = sc_hi + hi_len * c;
        for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
            int t = idx & (T - 1), i = idx >> lT;
            w[idx] = gl_mul_c(s[(brev_bits(i, ls) << lT) + t], tw2(lo, hi, (uint32_t)i));
        }
        __syncthreads();
        if (ls > 0) dif_smem(w, ls, lT, twf);
        for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
            int t = idx / n, q = idx - t * n;
            uint64_t col = c0 + t;
            if (col < cols) out[col * old + (uint64_t)q * E + c] = w[(brev_bits(q, ls) << lT) + t];
        }
        __syncthreads();
    }
}

// K1: inverse pass A over the trace: Y[i1 + n1*k2] = w^-(i1*k2) DFT^-1_n2(...)[k2].
// (k_pass_a with the inverse tables; separate name only for profiles.)
__global__ void k_lde_inv_a(const uint64_t* trace, uint64_t tld, uint64_t* Y, uint64_t yld, int l1, int l2,
                            int lT, const uint64_t* tw12_i, const uint64_t* wlo, const uint64_t* whi) {
    extern __shared__ uint64_t sm[];
    const int n2 = 1 << l2, T = 1 << lT;
    uint64_t* tw = sm;
    uint64_t* s = sm + n2 / 2;
    load_tw(tw, tw12_i, l2);
    const uint64_t col = blockIdx.y;
    const uint32_t i10 = blockIdx.x << lT;
    const uint64_t* src = trace + col * tld;
    for (int idx = threadIdx.x; idx < (n2 << lT); idx += blockDim.x) {
        int t = idx & (T - 1), i2 = idx >> lT;
        s[idx] = gl_canon(src[i10 + t + ((uint64_t)i2 << l1)]);
    }
    __syncthreads();
    dif_smem(s, l2, lT, tw);
    uint64_t* dst = Y + col * yld;
    for (int idx = threadIdx.x; idx < (n2 << lT); idx += blockDim.x) {
        int t = idx & (T - 1), k2 = idx >> lT;
        uint64_t v = s[(brev_bits(k2, l2) << lT) + t];
        dst[i10 + t + ((uint64_t)k2 << l1)] = gl_mul_c(v, tw2(wlo, whi, (i10 + t) * (uint32_t)k2));
    }
}

// K2: rows k2 in [k20, k20+T) of Y: inverse DFT_n1 -> coefficients c[n2*k1 + k2];
// per coset: a = c * N^-1 s_c^i, forward DFT_n1 over k1, times w_N^(k2*q2),
// Z_c[k2 + n2*q2].  Z holds E planes of N words per column: Z[(col*E + c)*N + .].
__global__ void k_lde_mid(const uint64_t* Y, uint64_t yld, uint64_t* Z, int l1, int l2, int lT, int le,
                          const uint64_t* tw12_i, const uint64_t* tw12_f, const uint64_t* wlo,
                          const uint64_t* whi, const uint64_t* sc_lo, const uint64_t* sc_hi, int hi_len) {
    extern __shared__ uint64_t sm[];
    const int n1 = 1 << l1, T = 1 << lT, E = 1 << le;
    uint64_t* twi = sm;
    uint64_t* twf = twi + n1 / 2;
    uint64_t* s = twf + n1 / 2;
    uint64_t* w = s + (n1 << lT);
    load_tw(twi, tw12_i, l1);
    load_tw(twf, tw12_f, l1);
    const uint64_t col = blockIdx.y;
    const uint32_t k20 = blockIdx.x << lT;
    const uint64_t* src = Y + col * yld + ((uint64_t)k20 << l1);
    for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
        int t = idx >> l1, i1 = idx & (n1 - 1);
        s[(i1 << lT) + t] = src[idx];
    }
    __syncthreads();
    dif_smem(s, l1, lT, twi);
    const uint64_t N = 1ull << (l1 + l2);
    for (int c = 0; c < E; c++) {
        const uint64_t* lo = sc_lo + 4096 * c;
        const uint64_t* hi = sc_hi + hi_len * c;
        for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
            int t = idx & (T - 1), k1 = idx >> lT;
            uint32_t i = ((uint32_t)k1 << l2) + k20 + t;
            w[idx] = gl_mul_c(s[(brev_bits(k1, l1) << lT) + t], tw2(lo, hi, i));
        }
        __syncthreads();
        dif_smem(w, l1, lT, twf);
        uint64_t* dst = Z + (col * E + c) * N;
        for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
            int t = idx & (T - 1), q2 = idx >> lT;
            uint64_t v = w[(brev_bits(q2, l1) << lT) + t];
            v = gl_mul_c(v, tw2(wlo, whi, (k20 + t) * (uint32_t)q2));
            dst[k20 + t + ((uint64_t)q2 << l2)] = v;
        }
        __syncthreads();
    }
}

// K3: for q2 in [q20, q20+T3), all E cosets: DFT_n2 over rows Z_c[i1' + n2*q2];
// E_c[n1*q1 + q2] -> LDE[E*(n1*q1 + q2) + c], written as runs of E*T3 words.
__global__ void k_lde_fwd_b(const uint64_t* Z, uint64_t* out, uint64_t old, int l1, int l2, int lT3, int le,
                            const uint64_t* tw12_f) {
    extern __shared__ uint64_t sm[];
    const int n2 = 1 << l2, T3 = 1 << lT3, E = 1 << le;
    const int lS = lT3 + le;  // sequences per CTA = E*T3, seq u = E*t + c
    uint64_t* tw = sm;
    uint64_t* s = sm + n2 / 2;
    load_tw(tw, tw12_f, l2);
    const uint64_t col = blockIdx.y;
    const uint32_t q20 = blockIdx.x << lT3;
    const uint64_t N = 1ull << (l1 + l2);
    for (int idx = threadIdx.x; idx < (n2 << lS); idx += blockDim.x) {
        int seq = idx >> l2, i1 = idx & (n2 - 1);
        int c = seq >> lT3, t = seq & (T3 - 1);
        uint64_t v = Z[(col * E + c) * N + ((uint64_t)(q20 + t) << l2) + i1];
        s[(i1 << lS) + (t << le) + c] = v;
    }
    __syncthreads();
    dif_smem(s, l2, lS, tw);
    uint64_t* dst = out + col * old;
    const int S = 1 << lS;
    for (int idx = threadIdx.x; idx < (n2 << lS); idx += blockDim.x) {
        int u = idx & (S - 1), q1 = idx >> lS;
        uint64_t v = s[(brev_bits(q1, l2) << lS) + u];
        dst[(((uint64_t)q1 << l1) + q20) * E + u] = v;
    }
}

// ------------------------------------------------------------------ helpers

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static int choose_lT(int ls, int budget_words_log) {
    // T = 2^lT sequences so that T * 2^ls ~ 2^budget, within [1, 8].
    return clampi(budget_words_log - ls, 0, 3);
}

static cudaError_t set_smem(const void* fn, size_t bytes) {
    if (bytes > 48 * 1024)
        return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return cudaSuccess;
}

size_t ntt_scratch_words(int logn, uint64_t cols) { return logn <= 11 ? 0 : (size_t)cols << logn; }

cudaError_t launch_ntt(const LdePlan& pl, int inverse, uint64_t* data, uint64_t ld, uint64_t cols,
                       uint64_t* scratch, cudaStream_t st) {
    const int l = pl.logn;
    const uint64_t* tw12 = inverse ? pl.tw12_i : pl.tw12_f;
    uint64_t scale = 1;
    if (inverse) {
        // n^-1 = p - (p-1)/n  (since n divides p-1)
        scale = l == 0 ? 1 : GL_P - ((GL_P - 1) >> l);
    }
    if (cols == 0) return cudaSuccess;
    if (l <= 11) {
        int lT = choose_lT(l, 11);
        int T = 1 << lT;
        size_t smem = ((l > 0 ? (1u << l) / 2 : 1) + ((size_t)T << l)) * 8;
        cudaError_t e = set_smem((const void*)k_ntt_small, smem);
        if (e != cudaSuccess) return e;
        count_launch();
        k_ntt_small<<<(unsigned)((cols + T - 1) / T), 256, smem, st>>>(data, ld, cols, l, lT, tw12, scale);
        return cudaGetLastError();
    }
    const int l1 = (l + 1) / 2, l2 = l / 2;
    const uint64_t n = 1ull << l;
    const uint64_t* wlo = inverse ? pl.wn_i_lo : pl.wn_f_lo;
    const uint64_t* whi = inverse ? pl.wn_i_hi : pl.wn_f_hi;
    int lTa = choose_lT(l2, 13);
    size_t smem_a = ((1u << l2) / 2 + ((size_t)1 << (l2 + lTa))) * 8;
    int lTb = choose_lT(l1, 13);
    size_t smem_b = ((1u << l1) / 2 + ((size_t)1 << (l1 + lTb))) * 8;
    cudaError_t e = set_smem((const void*)k_pass_a, smem_a);
    if (e == cudaSuccess) e = set_smem((const void*)k_pass_b, smem_b);
    if (e != cudaSuccess) return e;
    // columns in chunks of at most 65535 (grid.y limit)
    for (uint64_t c0 = 0; c0 < cols; c0 += 65535) {
        unsigned nc = (unsigned)((cols - c0) < 65535 ? (cols - c0) : 65535);
        dim3 ga((unsigned)((1u << l1) >> lTa), nc);
        count_launch();
        k_pass_a<<<ga, 256, smem_a, st>>>(data + c0 * ld, ld, scratch, n, l1, l2, lTa, tw12, wlo, whi);
        dim3 gb((unsigned)((1u << l2) >> lTb), nc);
        count_launch();
        k_pass_b<<<gb, 256, smem_b, st>>>(scratch, n, data + c0 * ld, ld, l1, l2, lTb, tw12, scale);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

size_t lde_scratch_words(int logn, int log_exp, uint64_t cols) {
    if (logn <= 11) return 0;
    return (size_t)cols * ((size_t)1 << logn) * (1 + ((size_t)1 << log_exp));
}

cudaError_t launch_lde(const LdePlan& pl, const uint64_t* trace, uint64_t tld, uint64_t* out, uint64_t old,
                       uint64_t cols, uint64_t* scratch, cudaStream_t st) {
    const int l = pl.logn, le = pl.log_exp;
    const int E = 1 << le;
    const int hi_len = l > 12 ? (1 << (l - 12)) : 1;
    if (cols == 0) return cudaSuccess;
    if (l <= 11) {
        int lT = choose_lT(l, 10);
        int T = 1 << lT;
        int hw = l > 0 ? (1 << l) / 2 : 1;
        size_t smem = (2 * (size_t)hw + 2 * ((size_t)T << l)) * 8;
        cudaError_t e = set_smem((const void*)k_lde_small, smem);
        if (e != cudaSuccess) return e;
        count_launch();
        k_lde_small<<<(unsigned)((cols + T - 1) / T), 256, smem, st>>>(trace, tld, out, old, cols, l, lT, le,
                                                                     pl.tw12_i, pl.tw12_f, pl.sc_lo, pl.sc_hi,
                                                                     hi_len);
        return cudaGetLastError();
    }
    const int l1 = (l + 1) / 2, l2 = l / 2;
    const uint64_t N = 1ull << l;
    int lT1 = choose_lT(l2, 13);
    size_t smem1 = ((1u << l2) / 2 + ((size_t)1 << (l2 + lT1))) * 8;
    int lT2 = choose_lT(l1, 12);
    size_t smem2 = ((size_t)(1u << l1) + 2 * ((size_t)1 << (l1 + lT2))) * 8;
    int lT3 = clampi(13 - l2 - le, 0, 1);
    size_t smem3 = ((1u << l2) / 2 + ((size_t)1 << (l2 + lT3 + le))) * 8;
    cudaError_t e = set_smem((const void*)k_lde_inv_a, smem1);
    if (e == cudaSuccess) e = set_smem((const void*)k_lde_mid, smem2);
    if (e == cudaSuccess) e = set_smem((const void*)k_lde_fwd_b, smem3);
    if (e != cudaSuccess) return e;
    uint64_t* Y = scratch;
    for (uint64_t c0 = 0; c0 < cols; c0 += 65535) {
        unsigned nc = (unsigned)((cols - c0) < 65535 ? (cols - c0) : 65535);
        uint64_t* Z = scratch + (size_t)nc * N;
        dim3 g1((unsigned)((1u << l1) >> lT1), nc);
        count_launch();
        k_lde_inv_a<<<g1, 256, smem1, st>>>(trace + c0 * tld, tld, Y, N, l1, l2, lT1, pl.tw12_i, pl.wn_i_lo,
                                           pl.wn_i_hi);
        dim3 g2((unsigned)((1u << l2) >> lT2), nc);
        count_launch();
        k_lde_mid<<<g2, 256, smem2, st>>>(Y, N, Z, l1, l2, lT2, le, pl.tw12_i, pl.tw12_f, pl.wn_f_lo,
                                         pl.wn_f_hi, pl.sc_lo, pl.sc_hi, hi_len);
        dim3 g3((unsigned)((1u << l1) >> lT3), nc);
        count_launch();
        k_lde_fwd_b<<<g3, 256, smem3, st>>>(Z, out + c0 * old, old, l1, l2, lT3, le, pl.tw12_f);
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    (void)E;
    return cudaSuccess;
}

// ---------------------------------------------------------------- transpose

__global__ void k_transpose(const uint64_t* __restrict__ in, uint64_t ild, uint64_t* __restrict__ out,
                            uint64_t old, uint64_t R, uint64_t C) {
    // in: R x C with row stride ild; out: C x R with row stride old.
    __shared__ uint64_t tile[32][33];
    uint64_t r0 = (uint64_t)blockIdx.y * 32, c0 = (uint64_t)blockIdx.x * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        uint64_t r = r0 + k, c = c0 + threadIdx.x;
        if (r < R && c < C) tile[k][threadIdx.x] = in[r * ild + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        uint64_t c = c0 + k, r = r0 + threadIdx.x;
        if (r < R && c < C) out[c * old + r] = tile[threadIdx.x][k];
    }
}

cudaError_t launch_transpose(const uint64_t* in, uint64_t rld, uint64_t* out, uint64_t cld, uint64_t rows,
                             uint64_t cols, cudaStream_t st) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    dim3 g((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
    count_launch();
    k_transpose<<<g, dim3(32, 8), 0, st>>>(in, rld, out, cld, rows, cols);
    return cudaGetLastError();
}

cudaError_t launch_transpose_cm_to_rm(const uint64_t* in, uint64_t cld, uint64_t* out, uint64_t rld,
                                      uint64_t rows, uint64_t cols, cudaStream_t st) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    dim3 g((unsigned)((rows + 31) / 32), (unsigned)((cols + 31) / 32));
    count_launch();
    k_transpose<<<g, dim3(32, 8), 0, st>>>(in, cld, out, rld, cols, rows);
    return cudaGetLastError();
}

}  // namespace tvmc
