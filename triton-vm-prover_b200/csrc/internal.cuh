// Internal launcher declarations shared by the CUDA translation units.
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <cstdint>
#include <cstddef>

namespace tvmc {

// NVTX range around the host-side enqueue of one phase (LDE, row hash, tree,
// frugal stripe, batch, serving commit), so that a timeline profiler groups each
// phase's kernels under its name -- the counterpart of the reference's
// TRITON_VM_PROFILE phase timers (include/common/debug_control.hpp).  Without
// an attached profiler an NVTX push/pop is a no-op call.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

// Number of kernels this library has launched (all devices, all threads).
void count_launch();
// Records `msg` as the calling thread's tvmc_last_error() text; returns code.
int set_error(int code, const char* msg);
// Validates the sizes of an LDE from trace_len to extended_len rows (both
// powers of two, trace_len <= 2^MAX_LOG_LDE_TRACE, expansion <= 16) and returns
// their logs; on failure records the message and returns the status, as every
// LDE entry point reports it.
int check_lde_sizes(size_t trace_len, size_t extended_len, int* logn, int* le);
// Tuning knob "lde_mid_ctas" (2 or 3 resident CTAs per SM for the fused LDE
// middle kernel; default 3).
int tuning_lde_mid_ctas();
// Tuning knob "lde_mid_variant": 1 = k_lde_mid_sym (twiddles from global tables
// per coset), 2 = k_lde_mid_sym2 (inter-pass twiddles shared across cosets in
// shared memory); 0 = the default (2).
int tuning_lde_mid_variant();
// Tuning knob "lde_split_l1": log2 of the four-step factor n1 of the LDE (the
// K2 transform size), 0 = balanced; a split with either factor outside
// [2^6, 2^12] falls back to balanced.
int tuning_lde_split_l1();
// Tuning knob "ntt_tile_log": log2 of the words one NTT/LDE pass CTA moves per
// tile (sequences per CTA = 2^(tile - log2 size), clamped); default 13.
int tuning_ntt_tile_log();
// Merkle levels built inside the row-hash CTA (8 by default; 0 with the tuning
// knob "hash_unfused_tree" = 1); the rest are built by k_merkle_up.
int tuning_hash_fuse_levels();

// Merkle node storage layouts.
//   HEAP: 2n digests, node h at h (root 1, leaves [n, 2n), slot 0 unused) --
//         the reference's CPU MerkleTree (src/merkle/merkle_tree.cpp:12-33).
//   FLAT: 2n-1 digests, [leaves | level 1 | ... | root] -- the reference's
//         GPU merkle_tree_gpu layout (src/gpu/kernels/merkle_kernel.cu:41-105).
enum NodeLayout : int { LAYOUT_HEAP = 0, LAYOUT_FLAT = 1 };

__host__ __device__ inline uint64_t node_slot(uint64_t h, uint64_t n, int layout) {
    if (layout == LAYOUT_HEAP) return h;
    // h lies on the level with 2^m nodes; that level starts at 2n - 2^(m+1) in FLAT.
#ifdef __CUDA_ARCH__
    uint64_t pm = 1ull << (63 - __clzll((long long)h));
#else
    uint64_t pm = 1ull << (63 - __builtin_clzll(h));
#endif
    return 2 * n + h - 3 * pm;
}

// ---- hash.cu -------------------------------------------------------------
// Leaf digests of `rows` rows; element (r, c) at table[r*rstride + c*cstride].
// If `tree` is non-null, rows must be a power of two: leaves are written as
// tree nodes (layout) and the whole tree is completed up to the root.
// Otherwise digests go to `digests` (rows x 5).
cudaError_t launch_hash_rows(const uint64_t* table, uint64_t rstride, uint64_t cstride, uint64_t rows,
                             uint32_t width, uint64_t* digests, uint64_t* tree, int layout,
                             cudaStream_t st);
// Complete a tree whose leaf level (n leaves) is already stored in `tree`.
cudaError_t launch_merkle_from_leaves(uint64_t* tree, uint64_t n, int layout, cudaStream_t st);
// Copy n leaf digests into the tree's leaf slots and complete the tree.  With
// leaf_words = 3 the leaves are XFieldElements, each padded to (c0, c1, c2, 0, 0).
cudaError_t launch_merkle_tree(const uint64_t* leaves, uint64_t* tree, uint64_t n, int layout,
                               cudaStream_t st, int leaf_words = 5);
// Frugal streaming: absorb ncols LDE columns (stride L) into per-row capacity
// state cap[6][L]; `last` pads, finishes the digests as leaves of the heap tree
// (2L digests) and builds the whole tree.
cudaError_t launch_absorb_stripe(const uint64_t* stripe, uint64_t L, uint32_t ncols, uint64_t* cap, int first,
                                 int last, uint64_t* tree, cudaStream_t st);
cudaError_t launch_hash_pairs(const uint64_t* left, const uint64_t* right, uint64_t* out, uint64_t count,
                              cudaStream_t st);

// Multi-table row hash + heap Merkle trees (one launch for up to
// HASH_MULTI_MAX tables, one more for the small tree tops).
struct MultiHashTable {
    const uint64_t* lde;  // column-major, column stride L
    uint64_t* tree;       // heap layout, 2L digests (node 0 unused)
    uint64_t L;           // rows, a power of two
    uint32_t width;
};
constexpr int HASH_MULTI_MAX = 64;
constexpr uint64_t MULTI_TOP_MAX_NODES = 1024;  // larger tree tops use the single-tree kernels
struct HashJob {
    const uint64_t* lde;
    uint64_t* tree;
    uint64_t L;
    uint32_t width;
    uint32_t block0;  // first CTA of this table
};
struct HashJobs {
    HashJob j[HASH_MULTI_MAX];
    int count;
};
struct TopJob {
    uint64_t* tree;
    uint64_t m;  // nodes of the level already in place
};
struct TopJobs {
    TopJob j[HASH_MULTI_MAX];
};
cudaError_t launch_hash_rows_multi(const MultiHashTable* tabs, int count, cudaStream_t st);
cudaError_t launch_tip5_permutations(uint64_t* states, uint64_t count, cudaStream_t st);
// Fiat-Shamir absorb of [lead (if has_lead)] ++ data[0..len) into the 16-word sponge state.
cudaError_t launch_sponge_absorb(uint64_t* state, const uint64_t* data, uint64_t len, int has_lead, uint64_t lead,
                                 cudaStream_t st);
// Tip5 rounds [r0, r0 + nr) of each state; trace (optional) gets the state after each round.
cudaError_t launch_tip5_rounds(uint64_t* states, uint64_t count, int r0, int nr, uint64_t* trace, cudaStream_t st);
// roots[q] = root implied by leaf digest leaves[q] at index idx[q] and its path of len siblings.
cudaError_t launch_root_from_paths(const uint64_t* idx, const uint64_t* leaves, const uint64_t* paths, uint64_t count,
                                   uint64_t len, uint64_t* roots, cudaStream_t st);
// out[q*height + k] = sibling of the k-th ancestor of leaf idx[q] (k = 0 is the leaf's sibling).
cudaError_t launch_gather_auth_paths(const uint64_t* tree, uint64_t n, int layout, const uint64_t* idx,
                                     uint64_t count, uint64_t* out, cudaStream_t st);
cudaError_t launch_gather_nodes(const uint64_t* tree, uint64_t n, int layout, const uint64_t* heap_idx,
                                uint64_t count, uint64_t* out, cudaStream_t st);
// Rows of a column-major table (col stride ld) gathered row-major: out[q*width + c].
cudaError_t launch_gather_rows(const uint64_t* table, uint64_t ld, uint32_t width, const uint64_t* rows,
                               uint64_t count, uint64_t* out, cudaStream_t st);

// ---- ntt.cu --------------------------------------------------------------
struct NttTables;  // device twiddle tables, owned by api.cu's per-device cache

// Twiddle bundle for one transform size / LDE configuration.
struct LdePlan {
    int logn;             // trace length N = 2^logn
    int log_exp;          // expansion E = 2^log_exp
    uint64_t offset;      // coset offset of the evaluation domain
    const uint64_t* tw12_f;   // w_4096^m, m < 4096 (forward sub-DFT twiddles)
    const uint64_t* tw12_i;   // inverse of the above
    const uint64_t* wn_f_lo;  // w_N^(e & 4095)
    const uint64_t* wn_f_hi;  // w_N^((e >> 12) * 4096)
    const uint64_t* wn_i_lo;  // same for w_N^-1
    const uint64_t* wn_i_hi;
    const uint64_t* sc_lo;    // E tables of 4096: s_c^(i & 4095), s_c = offset * w_{EN}^c
    const uint64_t* sc_hi;    // E tables of max(1, N/4096): N^-1 * s_c^((i >> 12) * 4096)
};

// Batched LDE of `cols` column-major columns: trace[c*tld + r] (r < N) ->
// out[c*old + r] (r < E*N).  scratch must hold scratch_words_lde(...) words.
// With rm > 0, add holds the randomizer addends of launch_rand_addend for
// these columns ([col][coset][rm]); the plan's offset is then o / t.
size_t lde_scratch_words(int logn, int log_exp, uint64_t cols);
cudaError_t launch_lde(const LdePlan& pl, const uint64_t* trace, uint64_t tld, uint64_t* out, uint64_t old,
                       uint64_t cols, uint64_t* scratch, cudaStream_t st, const uint64_t* add = nullptr,
                       int rm = 0);
// Interpolant coefficients touched by R randomizer coefficients: min(N, R).
inline int rand_rows(int logn, uint64_t R) {
    return R < (1ull << logn) ? (int)R : (1 << logn);
}
// Randomizer addends for `cols` columns with R coefficients each (r[col*R + k]):
// out[(col*E + c)*rm + i], rm = rand_rows(logn, R).  t = trace offset, tN = t^N,
// oN = o^N for the evaluation offset o, wE = primitive E-th root of unity; the
// product (x^N - t^N) r(x) is truncated to degree < qlen.
cudaError_t launch_rand_addend(const uint64_t* r, uint64_t R, uint64_t cols, int logn, int le, uint64_t t,
                               uint64_t tN, uint64_t oN, uint64_t wE, uint64_t qlen, uint64_t* out, cudaStream_t st);
// Batched NTT in place on column-major data[c*ld + r], r < 2^logn.
size_t ntt_scratch_words(int logn, uint64_t cols);
cudaError_t launch_ntt(const LdePlan& pl, int inverse, uint64_t* data, uint64_t ld, uint64_t cols,
                       uint64_t* scratch, cudaStream_t st);
// out[c*L + i] = in[c*ild + i] * o^i for i < min(n, L), 0 above (the coefficient
// side of NTT::evaluate_on_coset); a forward NTT of length L finishes it.
cudaError_t launch_coset_scale(const uint64_t* in, uint64_t ild, uint64_t n, uint64_t* out, uint64_t L, uint64_t cols,
                               uint64_t o, cudaStream_t st);
// Row-major (rows x cols, row stride rld) -> column-major (col stride cld).
cudaError_t launch_transpose(const uint64_t* in, uint64_t rld, uint64_t* out, uint64_t cld, uint64_t rows,
                             uint64_t cols, cudaStream_t st);
// The same with TMA tile copies (transpose.cu) for packed tables of even width
// and height; cudaErrorNotSupported otherwise (the caller falls back).
cudaError_t launch_transpose_tma(const uint64_t* in, uint64_t* out, uint64_t rows, uint64_t cols, cudaStream_t st);
// TMA transpose tiles skipped because their load never completed (bounded wait).
unsigned int tma_timeouts();
// Tuning knob "transpose_tma": 1 = row-major -> column-major through TMA tiles
// where the shape allows it, 2 = the shared-memory tile kernel always.
bool tuning_transpose_tma();
// Column-major -> row-major.
cudaError_t launch_transpose_cm_to_rm(const uint64_t* in, uint64_t cld, uint64_t* out, uint64_t rld,
                                      uint64_t rows, uint64_t cols, cudaStream_t st);

constexpr int MAX_LOG_NTT = 24;       // plain NTT sizes up to 2^24
constexpr int MAX_LOG_LDE_TRACE = 22; // LDE trace lengths up to 2^22

}  // namespace tvmc
