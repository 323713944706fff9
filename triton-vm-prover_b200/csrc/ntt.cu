// Batched Goldilocks NTT and fused low-degree extension (sm_100a).
//
// Every transform here is the DFT X[k] = sum_i x[i] w^(ik) with natural-order
// input and output, w = 7^((p-1)/n) (src/types/b_field_element.cpp:179-192);
// the inverse uses w^-1 and scales by n^-1 (src/ntt/ntt.cpp:59-86).  Results
// are canonical, so they equal the reference's radix-2 DIT bit for bit.
//
// Global structure.  Sizes up to 2^11 run in one pass per column (whole column
// in shared memory).  Larger sizes use the four-step split n = n1*n2,
// i = i1 + n1*i2, k = n2*k1 + k2:
//   pass A: for each i1, DFT_n2 over i2 (elements at stride n1), times w^(i1*k2)
//   pass B: for each k2, DFT_n1 over i1 (contiguous rows) -> X[n2*k1 + k2]
// A CTA moves T sequences at a time so that global accesses come in runs of T
// consecutive words.
//
// In-CTA structure (sub_dft).  A sub-transform of size 2^LS <= 2^12 held in
// shared memory is itself split four-step into rounds of radix <= 32; in each
// round a thread loads one line of R elements into registers, runs a radix-2
// DIF network there, applies the inter-round twiddle and writes the line back.
// One __syncthreads per round instead of one per butterfly stage.
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

constexpr int NTT_THREADS = 256;

// ------------------------------------------------------------ sub-transform

// Shared-memory slot of element k (T = 2^lT interleaved sequences); one row of
// padding per 32 elements keeps every round's line accesses bank-conflict free.
__device__ __forceinline__ int spos(int k, int lT) { return (k + (k >> 5)) << lT; }
__host__ __device__ constexpr int spad_words(int n, int lT) { return (n + (n >> 5) + 1) << lT; }

// Round sizes (log2) of a 2^LS transform: one round up to 2^5, two up to 2^10,
// three beyond.  b1 is the last round (contiguous digit).
template <int LS>
struct Plan {
    static constexpr int NR = LS <= 5 ? 1 : (LS <= 10 ? 2 : 3);
    static constexpr int b1 = NR == 1 ? LS : (NR == 2 ? LS - LS / 2 : (LS + 2) / 3);
    static constexpr int b2 = NR == 1 ? 0 : (NR == 2 ? LS / 2 : (LS + 1) / 3);
    static constexpr int b3 = NR == 3 ? LS / 3 : 0;
    static_assert(b1 + b2 + b3 == LS, "round split");
    static_assert(b1 <= 5 && b2 <= 5 && b3 <= 5, "radix <= 32");
};

template <int B>
__device__ __forceinline__ constexpr int brevc(int k) {
    int r = 0;
    for (int i = 0; i < B; i++) r |= ((k >> i) & 1) << (B - 1 - i);
    return r;
}

// Radix-2 DIF network on R = 2^B registers; X[k] ends in v[brev(k)].
// tw[e] = w^e for the 2^LS-point root w, so w_{2h}^j = tw[j * 2^LS / 2h].
template <int LS, int B>
__device__ __forceinline__ void reg_dft(uint64_t (&v)[1 << B], const uint64_t* tw) {
#pragma unroll
    for (int st = 0; st < B; st++) {
        constexpr int R = 1 << B;
        const int h = R >> (st + 1);
#pragma unroll
        for (int blk = 0; blk < R; blk += 2 * h) {
#pragma unroll
            for (int j = 0; j < h; j++) {
                const uint64_t a = v[blk + j], c = v[blk + j + h];
                v[blk + j] = gl_add_c(a, c);
                const uint64_t d = gl_sub_c(a, c);
                v[blk + j + h] = j == 0 ? d : gl_mul_c(d, tw[j << (LS - B + st)]);
            }
        }
    }
}

// One round along the digit of stride S (elements lo + S*j + S*R*hi), for all
// T x S x H lines.  MODE 0: no twiddle; 1: w^((d2*k) << b1) (first of three
// rounds, d2 = lo >> b1); 2: w^(lo * (R3*k + hi)) (middle round).
template <int LS, int B, int MODE>
__device__ __forceinline__ void sub_round(uint64_t* s, int lT, const uint64_t* tw, int lS, int b1, int R3) {
    constexpr int R = 1 << B;
    const int T = 1 << lT;
    const int nlines = (1 << (LS - B)) << lT;
    for (int id = threadIdx.x; id < nlines; id += blockDim.x) {
        const int t = id & (T - 1);
        const int rest = id >> lT;
        const int lo = rest & ((1 << lS) - 1);
        const int hi = rest >> lS;
        const int base = lo + (hi << (lS + B));
        uint64_t v[R];
#pragma unroll
        for (int j = 0; j < R; j++) v[j] = s[spos(base + (j << lS), lT) + t];
        reg_dft<LS, B>(v, tw);
#pragma unroll
        for (int k = 0; k < R; k++) {
            uint64_t x = v[brevc<B>(k)];
            if (MODE == 1) {
                const int e = ((lo >> b1) * k) << b1;
                if (e) x = gl_mul_c(x, tw[e]);
            } else if (MODE == 2) {
                const int e = lo * (R3 * k + hi);
                if (e) x = gl_mul_c(x, tw[e]);
            }
            s[spos(base + (k << lS), lT) + t] = x;
        }
    }
    __syncthreads();
}

// DFT of size 2^LS of T sequences in shared memory, in place; X[k] ends at
// element slot out_pos<LS>(k).  tw: 2^LS entries w^e in shared memory.
template <int LS>
__device__ __forceinline__ void sub_dft(uint64_t* s, int lT, const uint64_t* tw) {
    using PL = Plan<LS>;
    if constexpr (PL::NR == 1) {
        sub_round<LS, PL::b1, 0>(s, lT, tw, 0, 0, 1);
    } else if constexpr (PL::NR == 2) {
        sub_round<LS, PL::b2, 2>(s, lT, tw, PL::b1, PL::b1, 1);
        sub_round<LS, PL::b1, 0>(s, lT, tw, 0, 0, 1);
    } else {
        sub_round<LS, PL::b3, 1>(s, lT, tw, PL::b1 + PL::b2, PL::b1, 1);
        sub_round<LS, PL::b2, 2>(s, lT, tw, PL::b1, PL::b1, 1 << PL::b3);
        sub_round<LS, PL::b1, 0>(s, lT, tw, 0, 0, 1);
    }
}

template <int LS>
__device__ __forceinline__ int out_pos(int k) {
    using PL = Plan<LS>;
    if constexpr (PL::NR == 1) {
        return k;
    } else if constexpr (PL::NR == 2) {
        // X[R2*k1 + k2] sits at k1 + R1*k2
        return (k >> PL::b2) + ((k & ((1 << PL::b2) - 1)) << PL::b1);
    } else {
        // X[M*k1 + R3*k2 + k3] sits at k1 + R1*k2 + R1*R2*k3
        const int k1 = k >> (PL::b2 + PL::b3);
        const int k2 = (k >> PL::b3) & ((1 << PL::b2) - 1);
        const int k3 = k & ((1 << PL::b3) - 1);
        return k1 + (k2 << PL::b1) + (k3 << (PL::b1 + PL::b2));
    }
}

__device__ __forceinline__ uint64_t tw2(const uint64_t* __restrict__ lo, const uint64_t* __restrict__ hi,
                                        uint32_t e) {
    return gl_mul(__ldg(lo + (e & 4095)), __ldg(hi + (e >> 12)));
}

// tw[e] = w_{2^LS}^e, e < 2^LS, from the 4096-entry table of w_4096 powers.
template <int LS>
__device__ __forceinline__ void load_tw(uint64_t* tw, const uint64_t* __restrict__ tw12) {
    for (int m = threadIdx.x; m < (1 << LS); m += blockDim.x) tw[m] = __ldg(tw12 + (m << (12 - LS)));
}

// ---------------------------------------------------------------- plain NTT

// Whole columns in shared memory: T = 2^lT columns per CTA, size 2^LS <= 2^11.
template <int LS>
__global__ void __launch_bounds__(NTT_THREADS) k_ntt_small(uint64_t* data, uint64_t ld, uint64_t cols, int lT,
                                                           const uint64_t* tw12, uint64_t scale) {
    extern __shared__ uint64_t sm[];
    constexpr int n = 1 << LS;
    const int T = 1 << lT;
    uint64_t* tw = sm;
    uint64_t* s = sm + n;
    load_tw<LS>(tw, tw12);
    const uint64_t c0 = (uint64_t)blockIdx.x * T;
    for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
        const int t = idx >> LS, k = idx & (n - 1);  // coalesced along a column
        const uint64_t col = c0 + t;
        s[spos(k, lT) + t] = col < cols ? gl_canon(data[col * ld + k]) : 0;
    }
    __syncthreads();
    sub_dft<LS>(s, lT, tw);
    for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
        const int t = idx >> LS, k = idx & (n - 1);
        const uint64_t col = c0 + t;
        if (col < cols) data[col * ld + k] = gl_mul_c(s[spos(out_pos<LS>(k), lT) + t], scale);
    }
}

// Pass A: out[i1 + n1*k2] = w^(i1*k2) * DFT_n2(in[i1 + n1*i2])[k2]; in may equal out.
template <int L2>
__global__ void __launch_bounds__(NTT_THREADS) k_pass_a(const uint64_t* in, uint64_t ild, uint64_t* out,
                                                        uint64_t old, int l1, int lT, const uint64_t* tw12,
                                                        const uint64_t* wlo, const uint64_t* whi) {
    extern __shared__ uint64_t sm[];
    constexpr int n2 = 1 << L2;
    const int T = 1 << lT;
    uint64_t* tw = sm;
    uint64_t* s = sm + n2;
    load_tw<L2>(tw, tw12);
    const uint64_t col = blockIdx.y;
    const uint32_t i10 = blockIdx.x << lT;
    const uint64_t* src = in + col * ild;
    for (int idx = threadIdx.x; idx < (n2 << lT); idx += blockDim.x) {
        const int t = idx & (T - 1), i2 = idx >> lT;
        s[spos(i2, lT) + t] = gl_canon(src[i10 + t + ((uint64_t)i2 << l1)]);
    }
    __syncthreads();
    sub_dft<L2>(s, lT, tw);
    uint64_t* dst = out + col * old;
    for (int idx = threadIdx.x; idx < (n2 << lT); idx += blockDim.x) {
        const int t = idx & (T - 1), k2 = idx >> lT;
        uint64_t v = s[spos(out_pos<L2>(k2), lT) + t];
        v = gl_mul_c(v, tw2(wlo, whi, (i10 + t) * (uint32_t)k2));
        dst[i10 + t + ((uint64_t)k2 << l1)] = v;
    }
}

// Pass B: out[n2*k1 + k2] = scale * DFT_n1(in[i1 + n1*k2])[k1]; in != out.
template <int L1>
__global__ void __launch_bounds__(NTT_THREADS) k_pass_b(const uint64_t* in, uint64_t ild, uint64_t* out,
                                                        uint64_t old, int l2, int lT, const uint64_t* tw12,
                                                        uint64_t scale) {
    extern __shared__ uint64_t sm[];
    constexpr int n1 = 1 << L1;
    const int T = 1 << lT;
    uint64_t* tw = sm;
    uint64_t* s = sm + n1;
    load_tw<L1>(tw, tw12);
    const uint64_t col = blockIdx.y;
    const uint32_t k20 = blockIdx.x << lT;
    const uint64_t* src = in + col * ild + ((uint64_t)k20 << L1);
    for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
        const int t = idx >> L1, i1 = idx & (n1 - 1);  // coalesced along a row
        s[spos(i1, lT) + t] = src[idx];
    }
    __syncthreads();
    sub_dft<L1>(s, lT, tw);
    uint64_t* dst = out + col * old;
    for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
        const int t = idx & (T - 1), k1 = idx >> lT;
        const uint64_t v = s[spos(out_pos<L1>(k1), lT) + t];
        dst[((uint64_t)k1 << l2) + k20 + t] = gl_mul_c(v, scale);
    }
}

// ---------------------------------------------------------------------- LDE

// Small LDE: whole column in shared memory (N <= 2^11), T columns per CTA.
template <int LS>
__global__ void __launch_bounds__(NTT_THREADS) k_lde_small(const uint64_t* trace, uint64_t tld, uint64_t* out,
                                                           uint64_t old, uint64_t cols, int lT, int le,
                                                           const uint64_t* tw12_i, const uint64_t* tw12_f,
                                                           const uint64_t* sc_lo, const uint64_t* sc_hi,
                                                           int hi_len) {
    extern __shared__ uint64_t sm[];
    constexpr int n = 1 << LS;
    const int T = 1 << lT, E = 1 << le;
    uint64_t* twi = sm;
    uint64_t* twf = twi + n;
    uint64_t* s = twf + n;                 // coefficients
    uint64_t* w = s + spad_words(n, lT);   // work
    load_tw<LS>(twi, tw12_i);
    load_tw<LS>(twf, tw12_f);
    const uint64_t c0 = (uint64_t)blockIdx.x * T;
    for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
        const int t = idx >> LS, k = idx & (n - 1);
        const uint64_t col = c0 + t;
        s[spos(k, lT) + t] = col < cols ? gl_canon(trace[col * tld + k]) : 0;
    }
    __syncthreads();
    sub_dft<LS>(s, lT, twi);
    for (int c = 0; c < E; c++) {
        const uint64_t* lo = sc_lo + 4096 * c;
        const uint64_t* hi = sc_hi + hi_len * c;
        for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
            const int t = idx & (T - 1), i = idx >> lT;
            w[spos(i, lT) + t] = gl_mul_c(s[spos(out_pos<LS>(i), lT) + t], tw2(lo, hi, (uint32_t)i));
        }
        __syncthreads();
        sub_dft<LS>(w, lT, twf);
        for (int idx = threadIdx.x; idx < n * T; idx += blockDim.x) {
            const int t = idx >> LS, q = idx & (n - 1);
            const uint64_t col = c0 + t;
            if (col < cols) out[col * old + (uint64_t)q * E + c] = w[spos(out_pos<LS>(q), lT) + t];
        }
        __syncthreads();
    }
}

// K1: inverse pass A over the trace: Y[i1 + n1*k2] = w^-(i1*k2) DFT^-1_n2(...)[k2].
template <int L2>
__global__ void __launch_bounds__(NTT_THREADS) k_lde_inv_a(const uint64_t* trace, uint64_t tld, uint64_t* Y,
                                                           uint64_t yld, int l1, int lT, const uint64_t* tw12_i,
                                                           const uint64_t* wlo, const uint64_t* whi) {
    extern __shared__ uint64_t sm[];
    constexpr int n2 = 1 << L2;
    const int T = 1 << lT;
    uint64_t* tw = sm;
    uint64_t* s = sm + n2;
    load_tw<L2>(tw, tw12_i);
    const uint64_t col = blockIdx.y;
    const uint32_t i10 = blockIdx.x << lT;
    const uint64_t* src = trace + col * tld;
    for (int idx = threadIdx.x; idx < (n2 << lT); idx += blockDim.x) {
        const int t = idx & (T - 1), i2 = idx >> lT;
        s[spos(i2, lT) + t] = gl_canon(src[i10 + t + ((uint64_t)i2 << l1)]);
    }
    __syncthreads();
    sub_dft<L2>(s, lT, tw);
    uint64_t* dst = Y + col * yld;
    for (int idx = threadIdx.x; idx < (n2 << lT); idx += blockDim.x) {
        const int t = idx & (T - 1), k2 = idx >> lT;
        const uint64_t v = s[spos(out_pos<L2>(k2), lT) + t];
        dst[i10 + t + ((uint64_t)k2 << l1)] = gl_mul_c(v, tw2(wlo, whi, (i10 + t) * (uint32_t)k2));
    }
}

// K2: rows k2 in [k20, k20+T) of Y: inverse DFT_n1 -> coefficients c[n2*k1 + k2];
// per coset: a = c * N^-1 s_c^i, forward DFT_n1 over k1, times w_N^(k2*q2),
// Z_c[k2 + n2*q2].  Z holds E planes of N words per column: Z[(col*E + c)*N + .].
template <int L1>
__global__ void __launch_bounds__(NTT_THREADS) k_lde_mid(const uint64_t* Y, uint64_t yld, uint64_t* Z, int l2,
                                                         int lT, int le, const uint64_t* tw12_i,
                                                         const uint64_t* tw12_f, const uint64_t* wlo,
                                                         const uint64_t* whi, const uint64_t* sc_lo,
                                                         const uint64_t* sc_hi, int hi_len) {
    extern __shared__ uint64_t sm[];
    constexpr int n1 = 1 << L1;
    const int T = 1 << lT, E = 1 << le;
    uint64_t* twi = sm;
    uint64_t* twf = twi + n1;
    uint64_t* s = twf + n1;
    uint64_t* w = s + spad_words(n1, lT);
    load_tw<L1>(twi, tw12_i);
    load_tw<L1>(twf, tw12_f);
    const uint64_t col = blockIdx.y;
    const uint32_t k20 = blockIdx.x << lT;
    const uint64_t* src = Y + col * yld + ((uint64_t)k20 << L1);
    for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
        const int t = idx >> L1, i1 = idx & (n1 - 1);
        s[spos(i1, lT) + t] = src[idx];
    }
    __syncthreads();
    sub_dft<L1>(s, lT, twi);
    const uint64_t N = 1ull << (L1 + l2);
    for (int c = 0; c < E; c++) {
        const uint64_t* lo = sc_lo + 4096 * c;
        const uint64_t* hi = sc_hi + hi_len * c;
        for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
            const int t = idx & (T - 1), k1 = idx >> lT;
            const uint32_t i = ((uint32_t)k1 << l2) + k20 + t;
            w[spos(k1, lT) + t] = gl_mul_c(s[spos(out_pos<L1>(k1), lT) + t], tw2(lo, hi, i));
        }
        __syncthreads();
        sub_dft<L1>(w, lT, twf);
        uint64_t* dst = Z + (col * E + c) * N;
        for (int idx = threadIdx.x; idx < (n1 << lT); idx += blockDim.x) {
            const int t = idx & (T - 1), q2 = idx >> lT;
            uint64_t v = w[spos(out_pos<L1>(q2), lT) + t];
            v = gl_mul_c(v, tw2(wlo, whi, (k20 + t) * (uint32_t)q2));
            dst[k20 + t + ((uint64_t)q2 << l2)] = v;
        }
        __syncthreads();
    }
}

// K3: for q2 in [q20, q20+T3), all E cosets: DFT_n2 over rows Z_c[i1' + n2*q2];
// E_c[n1*q1 + q2] -> LDE[E*(n1*q1 + q2) + c], written as runs of E*T3 words.
template <int L2>
__global__ void __launch_bounds__(NTT_THREADS) k_lde_fwd_b(const uint64_t* Z, uint64_t* out, uint64_t old,
                                                           int l1, int lT3, int le, const uint64_t* tw12_f) {
    extern __shared__ uint64_t sm[];
    constexpr int n2 = 1 << L2;
    const int T3 = 1 << lT3, E = 1 << le;
    const int lS = lT3 + le;  // sequences per CTA = E*T3, seq u = E*t + c
    uint64_t* tw = sm;
    uint64_t* s = sm + n2;
    load_tw<L2>(tw, tw12_f);
    const uint64_t col = blockIdx.y;
    const uint32_t q20 = blockIdx.x << lT3;
    const uint64_t N = 1ull << (l1 + L2);
    for (int idx = threadIdx.x; idx < (n2 << lS); idx += blockDim.x) {
        const int seq = idx >> L2, i1 = idx & (n2 - 1);
        const int c = seq >> lT3, t = seq & (T3 - 1);
        const uint64_t v = Z[(col * E + c) * N + ((uint64_t)(q20 + t) << L2) + i1];
        s[spos(i1, lS) + (t << le) + c] = v;
    }
    __syncthreads();
    sub_dft<L2>(s, lS, tw);
    uint64_t* dst = out + col * old;
    const int S = 1 << lS;
    for (int idx = threadIdx.x; idx < (n2 << lS); idx += blockDim.x) {
        const int u = idx & (S - 1), q1 = idx >> lS;
        dst[(((uint64_t)q1 << l1) + q20) * E + u] = s[spos(out_pos<L2>(q1), lS) + u];
    }
}

// ------------------------------------------------------------------ helpers

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// T = 2^lT sequences so that T * 2^ls ~ 2^budget, within [1, 8].
static int choose_lT(int ls, int budget_words_log) { return clampi(budget_words_log - ls, 0, 3); }

static cudaError_t set_smem(const void* fn, size_t bytes) {
    if (bytes > 48 * 1024)
        return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return cudaSuccess;
}

// Calls F.template operator()<L>() for the runtime L in [1, 12].
template <typename F>
static cudaError_t dispatch_ls(int l, F&& f) {
    switch (l) {
        case 1: return f.template operator()<1>();
        case 2: return f.template operator()<2>();
        case 3: return f.template operator()<3>();
        case 4: return f.template operator()<4>();
        case 5: return f.template operator()<5>();
        case 6: return f.template operator()<6>();
        case 7: return f.template operator()<7>();
        case 8: return f.template operator()<8>();
        case 9: return f.template operator()<9>();
        case 10: return f.template operator()<10>();
        case 11: return f.template operator()<11>();
        case 12: return f.template operator()<12>();
        default: return cudaErrorInvalidValue;
    }
}

static size_t words_bytes(size_t w) { return w * 8; }

size_t ntt_scratch_words(int logn, uint64_t cols) { return logn <= 11 ? 0 : (size_t)cols << logn; }

cudaError_t launch_ntt(const LdePlan& pl, int inverse, uint64_t* data, uint64_t ld, uint64_t cols,
                       uint64_t* scratch, cudaStream_t st) {
    const int l = pl.logn;
    const uint64_t* tw12 = inverse ? pl.tw12_i : pl.tw12_f;
    const uint64_t scale = (inverse && l > 0) ? GL_P - ((GL_P - 1) >> l) : 1;  // n^-1 = p - (p-1)/n
    if (cols == 0 || l == 0) return cudaSuccess;  // size-1 transform is the identity
    if (l <= 11) {
        const int lT = choose_lT(l, 11);
        const int T = 1 << lT;
        const size_t smem = words_bytes((1u << l) + spad_words(1 << l, lT));
        return dispatch_ls(l, [&]<int LS>() -> cudaError_t {
            cudaError_t e = set_smem((const void*)k_ntt_small<LS>, smem);
            if (e != cudaSuccess) return e;
            count_launch();
            k_ntt_small<LS><<<(unsigned)((cols + T - 1) / T), NTT_THREADS, smem, st>>>(data, ld, cols, lT, tw12,
                                                                                      scale);
            return cudaGetLastError();
        });
    }
    const int l1 = (l + 1) / 2, l2 = l / 2;
    const uint64_t n = 1ull << l;
    const uint64_t* wlo = inverse ? pl.wn_i_lo : pl.wn_f_lo;
    const uint64_t* whi = inverse ? pl.wn_i_hi : pl.wn_f_hi;
    const int lTa = choose_lT(l2, 13), lTb = choose_lT(l1, 13);
    const size_t smem_a = words_bytes((1u << l2) + spad_words(1 << l2, lTa));
    const size_t smem_b = words_bytes((1u << l1) + spad_words(1 << l1, lTb));
    for (uint64_t c0 = 0; c0 < cols; c0 += 65535) {
        const unsigned nc = (unsigned)((cols - c0) < 65535 ? (cols - c0) : 65535);
        cudaError_t e = dispatch_ls(l2, [&]<int L2>() -> cudaError_t {
            cudaError_t e2 = set_smem((const void*)k_pass_a<L2>, smem_a);
            if (e2 != cudaSuccess) return e2;
            count_launch();
            k_pass_a<L2><<<dim3((1u << l1) >> lTa, nc), NTT_THREADS, smem_a, st>>>(data + c0 * ld, ld, scratch, n,
                                                                                  l1, lTa, tw12, wlo, whi);
            return cudaGetLastError();
        });
        if (e != cudaSuccess) return e;
        e = dispatch_ls(l1, [&]<int L1>() -> cudaError_t {
            cudaError_t e2 = set_smem((const void*)k_pass_b<L1>, smem_b);
            if (e2 != cudaSuccess) return e2;
            count_launch();
            k_pass_b<L1><<<dim3((1u << l2) >> lTb, nc), NTT_THREADS, smem_b, st>>>(scratch, n, data + c0 * ld, ld,
                                                                                  l2, lTb, tw12, scale);
            return cudaGetLastError();
        });
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
    const int hi_len = l > 12 ? (1 << (l - 12)) : 1;
    if (cols == 0) return cudaSuccess;
    if (l <= 11) {
        if (l == 0) {
            // N = 1: every LDE row equals the single trace value (constant polynomial)
            const int E = 1 << le;
            cudaError_t e = cudaSuccess;
            for (uint64_t c = 0; c < cols && e == cudaSuccess; c++)
                for (int r = 0; r < E && e == cudaSuccess; r++)
                    e = cudaMemcpyAsync(out + c * old + r, trace + c * tld, 8, cudaMemcpyDeviceToDevice, st);
            return e;
        }
        const int lT = choose_lT(l, 10);
        const int T = 1 << lT;
        const size_t smem = words_bytes(2 * (size_t)(1u << l) + 2 * spad_words(1 << l, lT));
        return dispatch_ls(l, [&]<int LS>() -> cudaError_t {
            cudaError_t e = set_smem((const void*)k_lde_small<LS>, smem);
            if (e != cudaSuccess) return e;
            count_launch();
            k_lde_small<LS><<<(unsigned)((cols + T - 1) / T), NTT_THREADS, smem, st>>>(
                trace, tld, out, old, cols, lT, le, pl.tw12_i, pl.tw12_f, pl.sc_lo, pl.sc_hi, hi_len);
            return cudaGetLastError();
        });
    }
    const int l1 = (l + 1) / 2, l2 = l / 2;
    const uint64_t N = 1ull << l;
    const int lT1 = choose_lT(l2, 13);
    const size_t smem1 = words_bytes((1u << l2) + spad_words(1 << l2, lT1));
    const int lT2 = choose_lT(l1, 13);
    const size_t smem2 = words_bytes(2 * (size_t)(1u << l1) + 2 * spad_words(1 << l1, lT2));
    const int lT3 = clampi(13 - l2 - le, 0, 1);
    const size_t smem3 = words_bytes((1u << l2) + spad_words(1 << l2, lT3 + le));
    uint64_t* Y = scratch;
    for (uint64_t c0 = 0; c0 < cols; c0 += 65535) {
        const unsigned nc = (unsigned)((cols - c0) < 65535 ? (cols - c0) : 65535);
        uint64_t* Z = scratch + (size_t)nc * N;
        cudaError_t e = dispatch_ls(l2, [&]<int L2>() -> cudaError_t {
            cudaError_t e2 = set_smem((const void*)k_lde_inv_a<L2>, smem1);
            if (e2 != cudaSuccess) return e2;
            count_launch();
            k_lde_inv_a<L2><<<dim3((1u << l1) >> lT1, nc), NTT_THREADS, smem1, st>>>(
                trace + c0 * tld, tld, Y, N, l1, lT1, pl.tw12_i, pl.wn_i_lo, pl.wn_i_hi);
            return cudaGetLastError();
        });
        if (e != cudaSuccess) return e;
        e = dispatch_ls(l1, [&]<int L1>() -> cudaError_t {
            cudaError_t e2 = set_smem((const void*)k_lde_mid<L1>, smem2);
            if (e2 != cudaSuccess) return e2;
            count_launch();
            k_lde_mid<L1><<<dim3((1u << l2) >> lT2, nc), NTT_THREADS, smem2, st>>>(
                Y, N, Z, l2, lT2, le, pl.tw12_i, pl.tw12_f, pl.wn_f_lo, pl.wn_f_hi, pl.sc_lo, pl.sc_hi, hi_len);
            return cudaGetLastError();
        });
        if (e != cudaSuccess) return e;
        e = dispatch_ls(l2, [&]<int L2>() -> cudaError_t {
            cudaError_t e2 = set_smem((const void*)k_lde_fwd_b<L2>, smem3);
            if (e2 != cudaSuccess) return e2;
            count_launch();
            k_lde_fwd_b<L2><<<dim3((1u << l1) >> lT3, nc), NTT_THREADS, smem3, st>>>(Z, out + c0 * old, old, l1,
                                                                                   lT3, le, pl.tw12_f);
            return cudaGetLastError();
        });
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ---------------------------------------------------------------- transpose

__global__ void k_transpose(const uint64_t* __restrict__ in, uint64_t ild, uint64_t* __restrict__ out,
                            uint64_t old, uint64_t R, uint64_t C) {
    // in: R x C with row stride ild; out: C x R with row stride old.
    __shared__ uint64_t tile[32][33];
    const uint64_t r0 = (uint64_t)blockIdx.y * 32, c0 = (uint64_t)blockIdx.x * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const uint64_t r = r0 + k, c = c0 + threadIdx.x;
        if (r < R && c < C) tile[k][threadIdx.x] = in[r * ild + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const uint64_t c = c0 + k, r = r0 + threadIdx.x;
        if (r < R && c < C) out[c * old + r] = tile[threadIdx.x][k];
    }
}

cudaError_t launch_transpose(const uint64_t* in, uint64_t rld, uint64_t* out, uint64_t cld, uint64_t rows,
                             uint64_t cols, cudaStream_t st) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    const dim3 g((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
    count_launch();
    k_transpose<<<g, dim3(32, 8), 0, st>>>(in, rld, out, cld, rows, cols);
    return cudaGetLastError();
}

cudaError_t launch_transpose_cm_to_rm(const uint64_t* in, uint64_t cld, uint64_t* out, uint64_t rld,
                                      uint64_t rows, uint64_t cols, cudaStream_t st) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    const dim3 g((unsigned)((rows + 31) / 32), (unsigned)((cols + 31) / 32));
    count_launch();
    k_transpose<<<g, dim3(32, 8), 0, st>>>(in, cld, out, rld, cols, rows);
    return cudaGetLastError();
}

}  // namespace tvmc
