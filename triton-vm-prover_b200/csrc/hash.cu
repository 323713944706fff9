// Tip5 row hashing and Merkle tree kernels (sm_100a).
//
// Row hash: one LDE row per thread, the 16-word sponge state in registers,
// the next 10-element chunk prefetched into registers while the current one is
// permuted.  Rows are read column-major (a warp reads 32 consecutive rows of
// one column, 256 contiguous bytes).  Semantics: Tip5::hash_varlen
// (src/hash/tip5.cpp:246-282) -- zero state, overwrite the rate with each full
// chunk and permute, last chunk = rest, 1, zeros.
//
// Merkle: parent = hash_pair(left, right) (src/merkle/merkle_tree.cpp:41-61).
// The lowest log2(blockDim) levels are built in shared memory inside the row
// hash kernel itself; the remaining levels take one launch per 8 levels.
#include "internal.cuh"
#include "tip5.cuh"

namespace tvmc {

// Row-hash CTAs: 128 threads, six per SM (24 warps, <= 85 registers a thread,
// a few spilled): measured 2.7% faster than 256 x 2 (16 warps, 120 registers)
// on the 2^22-row commit, the extra warps covering the ALU and multiply-add
// pipe stalls; seven or eight per SM spill too much.
constexpr int HASH_THREADS = 128;
constexpr int HASH_CTAS_PER_SM = 6;
constexpr int UP_THREADS = 128;
// Tree levels with at least this many parents are built one level per launch.
constexpr uint64_t MERKLE_LEVEL_MIN_PARENTS = 1ull << 16;

__device__ __forceinline__ void store_digest(uint64_t* p, const uint64_t d[5]) {
#pragma unroll
    for (int i = 0; i < 5; i++) p[i] = d[i];
}

// Builds `levels` tree levels above the `count` digests held in sd (count <=
// blockDim.x, a power of two), where those digests are heap nodes
// [base, base + count).  Every thread of the CTA must call it.
__device__ __forceinline__ void subtree_levels(uint64_t* sd, uint64_t base, int levels, uint64_t* tree,
                                               uint64_t n, int layout, const uint32_t* lt,
                                               int count = -1) {
    if (count < 0) count = blockDim.x;
    for (int lv = 1; lv <= levels; lv++) {
        count >>= 1;
        base >>= 1;
        uint64_t h[5];
        bool act = threadIdx.x < count;
        if (act) t5_hash_pair(sd + 10 * threadIdx.x, sd + 10 * threadIdx.x + 5, h, lt);
        __syncthreads();
        if (act) {
            store_digest(sd + 5 * threadIdx.x, h);
            store_digest(tree + 5 * node_slot(base + threadIdx.x, n, layout), h);
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(HASH_THREADS, HASH_CTAS_PER_SM) k_hash_rows(
    const uint64_t* __restrict__ tab, uint64_t rstride, uint64_t cstride, uint64_t rows, uint32_t width,
    uint64_t* __restrict__ digests, uint64_t* __restrict__ tree, int layout, int fuse) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    extern __shared__ uint64_t sd[];  // 5 * blockDim words when fuse > 0 (fused tree levels), else none
    t5_sbox_init(sbox);
    __syncthreads();
    const uint32_t* lt = sbox + (threadIdx.x & 31);

    const uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = row < rows;
    const uint64_t* p = tab + (live ? row : 0) * rstride;

    uint64_t s[T5_STATE];
#pragma unroll
    for (int i = 0; i < T5_STATE; i++) s[i] = 0;

    const uint32_t full = width / T5_RATE;
    const uint32_t rem = width - full * T5_RATE;
    // Chunks are loaded just before their permutation: the 24 warps per SM hide
    // the load latency, and the registers a next-chunk prefetch would hold are
    // worth more to the permutation (measured ~2% faster on 2^22 x 379).
    for (uint32_t k = 0; k < full; k++) {
#pragma unroll
        for (int i = 0; i < T5_RATE; i++)
            s[i] = live ? gl_to_mont(__ldg(p + (uint64_t)(k * T5_RATE + i) * cstride)) : 0;
        t5_permutation_m(s, lt);
    }
#pragma unroll
    for (int i = 0; i < T5_RATE; i++)
        s[i] = ((uint32_t)i < rem) ? (live ? gl_to_mont(__ldg(p + (uint64_t)(full * T5_RATE + i) * cstride)) : 0)
                                   : ((uint32_t)i == rem ? T5_MONT_ONE : 0);
    t5_permutation_m(s, lt);

    uint64_t d[5];
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = gl_from_mont(s[i]);

    if (tree == nullptr) {
        if (live) store_digest(digests + 5 * row, d);
        return;
    }
    // rows is a power of two and a multiple of blockDim here
    store_digest(tree + 5 * node_slot(rows + row, rows, layout), d);
    if (fuse > 0) {
        store_digest(sd + 5 * threadIdx.x, d);
        __syncthreads();
        subtree_levels(sd, rows + (uint64_t)blockIdx.x * blockDim.x, fuse, tree, rows, layout, lt);
    }
}

// Frugal streaming: absorb one stripe of `ncols` LDE columns (column-major,
// stride L) into the sponge of every row.  Between stripes only the capacity
// words 10..15 survive (overwrite mode replaces the rate at every absorb), so
// they are all that is stored: cap[w*L + r], w < 6 (coalesced per word).  The
// first stripe starts from the zero state.  Every stripe but the last must
// hold whole 10-column chunks; the last one appends the hash_varlen padding
// (rest, 1, zeros), finishes the digest and writes it as tree leaf n + r,
// building the lowest log2(blockDim) levels in shared memory as k_hash_rows does.
__global__ void __launch_bounds__(HASH_THREADS, HASH_CTAS_PER_SM) k_absorb_stripe(
    const uint64_t* __restrict__ stripe, uint64_t L, uint32_t ncols, uint64_t* __restrict__ cap, int first,
    int last, uint64_t* __restrict__ tree, int fuse) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    extern __shared__ uint64_t sd[];  // 5 * blockDim words when fuse > 0 (fused tree levels), else none
    t5_sbox_init(sbox);
    __syncthreads();
    const uint32_t* lt = sbox + (threadIdx.x & 31);
    const uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;  // L is a multiple of blockDim
    const uint64_t* p = stripe + row;

    uint64_t s[T5_STATE];
#pragma unroll
    for (int i = 0; i < T5_RATE; i++) s[i] = 0;
#pragma unroll
    for (int i = 0; i < T5_STATE - T5_RATE; i++) s[T5_RATE + i] = first ? 0 : cap[(uint64_t)i * L + row];

    const uint32_t full = ncols / T5_RATE;
    const uint32_t rem = ncols - full * T5_RATE;
    for (uint32_t k = 0; k < full; k++) {  // chunks loaded as in k_hash_rows
#pragma unroll
        for (int i = 0; i < T5_RATE; i++) s[i] = gl_to_mont(__ldg(p + (uint64_t)(k * T5_RATE + i) * L));
        t5_permutation_m(s, lt);
    }
    if (!last) {
#pragma unroll
        for (int i = 0; i < T5_STATE - T5_RATE; i++) cap[(uint64_t)i * L + row] = s[T5_RATE + i];
        return;
    }
#pragma unroll
    for (int i = 0; i < T5_RATE; i++)
        s[i] = ((uint32_t)i < rem) ? gl_to_mont(__ldg(p + (uint64_t)(full * T5_RATE + i) * L))
                                   : ((uint32_t)i == rem ? T5_MONT_ONE : 0);
    t5_permutation_m(s, lt);
    uint64_t d[5];
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = gl_from_mont(s[i]);
    store_digest(tree + 5 * (L + row), d);
    if (fuse > 0) {
        store_digest(sd + 5 * threadIdx.x, d);
        __syncthreads();
        subtree_levels(sd, L + (uint64_t)blockIdx.x * blockDim.x, fuse, tree, L, LAYOUT_HEAP, lt);
    }
}

// ---- multi-table commitments ------------------------------------------------
// Small tables (a few thousand rows) leave most of the GPU idle when hashed one
// launch at a time: a 2^12-row LDE is 32 CTAs, and each row is a chain of 38
// permutations.  These kernels take up to HASH_MULTI_MAX tables of any heights
// and widths in one launch, so that many small commitments (the serving loop's
// queued requests, a batch of uneven tables) fill the GPU together.

// Row hash of several tables: CTA b belongs to the job j with
// block0[j] <= b < block0[j + 1]; its rows are hashed as in k_hash_rows and
// the lowest levels of that table's heap tree are built in shared memory.
__global__ void __launch_bounds__(HASH_THREADS, HASH_CTAS_PER_SM) k_hash_rows_multi(const __grid_constant__ HashJobs jobs,
                                                                                  int fuse_max) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    extern __shared__ uint64_t sd[];  // 5 * blockDim words
    t5_sbox_init(sbox);
    int j = 0;
    for (int k = 1; k < jobs.count; k++)
        if (jobs.j[k].block0 <= blockIdx.x) j = k;
    const uint64_t* tab = jobs.j[j].lde;
    uint64_t* tree = jobs.j[j].tree;
    const uint64_t L = jobs.j[j].L;
    const uint32_t width = jobs.j[j].width;
    __syncthreads();
    const uint32_t* lt = sbox + (threadIdx.x & 31);
    const int active = L < blockDim.x ? (int)L : (int)blockDim.x;  // L is a power of two
    const uint64_t row0 = (uint64_t)(blockIdx.x - jobs.j[j].block0) * blockDim.x;
    const uint64_t row = row0 + threadIdx.x;
    const bool live = threadIdx.x < active;
    const uint64_t* p = tab + (live ? row : 0);

    uint64_t s[T5_STATE];
#pragma unroll
    for (int i = 0; i < T5_STATE; i++) s[i] = 0;
    const uint32_t full = width / T5_RATE;
    const uint32_t rem = width - full * T5_RATE;
    for (uint32_t k = 0; k < full; k++) {
#pragma unroll
        for (int i = 0; i < T5_RATE; i++) s[i] = live ? gl_to_mont(__ldg(p + (uint64_t)(k * T5_RATE + i) * L)) : 0;
        t5_permutation_m(s, lt);
    }
#pragma unroll
    for (int i = 0; i < T5_RATE; i++)
        s[i] = ((uint32_t)i < rem) ? (live ? gl_to_mont(__ldg(p + (uint64_t)(full * T5_RATE + i) * L)) : 0)
                                   : ((uint32_t)i == rem ? T5_MONT_ONE : 0);
    t5_permutation_m(s, lt);
    uint64_t d[5];
#pragma unroll
    for (int i = 0; i < 5; i++) d[i] = gl_from_mont(s[i]);
    if (live) {
        store_digest(tree + 5 * (L + row), d);
        store_digest(sd + 5 * threadIdx.x, d);
    }
    __syncthreads();
    const int levels = min(fuse_max, 31 - __clz(active));
    subtree_levels(sd, L + row0, levels, tree, L, LAYOUT_HEAP, lt, active);
}

// The tops of several heap trees, one CTA per tree: tree j has its level of
// m[j] nodes (heap [m, 2m)) in place and gets every level above it.  Each
// level is read from global memory after the barrier that follows its writes.
__global__ void __launch_bounds__(256) k_merkle_tops_multi(const __grid_constant__ TopJobs jobs) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    t5_sbox_init(sbox);
    __syncthreads();
    const uint32_t* lt = sbox + (threadIdx.x & 31);
    uint64_t* tree = jobs.j[blockIdx.x].tree;
    for (uint64_t m = jobs.j[blockIdx.x].m; m > 1; m >>= 1) {
        for (uint64_t par = (m >> 1) + threadIdx.x; par < m; par += blockDim.x) {
            uint64_t a[5], b[5], h[5];
#pragma unroll
            for (int i = 0; i < 5; i++) {
                a[i] = tree[5 * (2 * par) + i];
                b[i] = tree[5 * (2 * par + 1) + i];
            }
            t5_hash_pair(a, b, h, lt);
            store_digest(tree + 5 * par, h);
        }
        __syncthreads();
    }
}

// One launch builds up to `levels` levels above the level of m nodes.
__global__ void __launch_bounds__(UP_THREADS) k_merkle_up(uint64_t* __restrict__ tree, uint64_t n,
                                                          uint64_t m, int layout, int levels) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    __shared__ uint64_t sd[UP_THREADS * 5];
    t5_sbox_init(sbox);
    __syncthreads();
    const uint32_t* lt = sbox + (threadIdx.x & 31);
    // parents of this block: heap nodes [m/2 + blockIdx.x*blockDim.x, +blockDim.x)
    uint64_t par = (m >> 1) + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* l = tree + 5 * node_slot(2 * par, n, layout);
    const uint64_t* r = tree + 5 * node_slot(2 * par + 1, n, layout);
    uint64_t a[5], b[5], h[5];
#pragma unroll
    for (int i = 0; i < 5; i++) { a[i] = l[i]; b[i] = r[i]; }
    t5_hash_pair(a, b, h, lt);
    store_digest(tree + 5 * node_slot(par, n, layout), h);
    if (levels > 1) {
        store_digest(sd + 5 * threadIdx.x, h);
        __syncthreads();
        subtree_levels(sd, par - threadIdx.x, levels - 1, tree, n, layout, lt);
    }
}

// One tree level: parent p in [m/2, m) = hash_pair(node 2p, node 2p + 1), one
// parent per thread.  Used while a level has enough parents to fill the GPU;
// adjacent parents read adjacent child pairs, so loads and stores coalesce.
__global__ void __launch_bounds__(HASH_THREADS) k_merkle_level(uint64_t* __restrict__ tree, uint64_t n, uint64_t m,
                                                               int layout) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    t5_sbox_init(sbox);
    __syncthreads();
    const uint64_t par = (m >> 1) + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (par >= m) return;
    const uint64_t* l = tree + 5 * node_slot(2 * par, n, layout);
    const uint64_t* r = tree + 5 * node_slot(2 * par + 1, n, layout);
    uint64_t a[5], b[5], h[5];
#pragma unroll
    for (int i = 0; i < 5; i++) { a[i] = l[i]; b[i] = r[i]; }
    t5_hash_pair(a, b, h, sbox + (threadIdx.x & 31));
    store_digest(tree + 5 * node_slot(par, n, layout), h);
}

// Leaf i = the in_words words at leaves[in_words*i], zero-padded to a digest:
// in_words = 5 copies digests, 3 turns an XFieldElement into the digest
// (c0, c1, c2, 0, 0), as the reference's FRI trees do (src/fri/fri.cpp:25-43).
__global__ void k_copy_leaves(const uint64_t* __restrict__ leaves, uint64_t* __restrict__ tree, uint64_t n,
                              int layout, int in_words) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t* dst = tree + 5 * node_slot(n + i, n, layout);
#pragma unroll
    for (int k = 0; k < 5; k++) dst[k] = k < in_words ? gl_canon(leaves[(uint64_t)in_words * i + k]) : 0;
}

__global__ void __launch_bounds__(128) k_hash_pairs(const uint64_t* __restrict__ left,
                                                    const uint64_t* __restrict__ right,
                                                    uint64_t* __restrict__ out, uint64_t count) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    t5_sbox_init(sbox);
    __syncthreads();
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint64_t a[5], b[5], h[5];
#pragma unroll
    for (int k = 0; k < 5; k++) { a[k] = left[5 * i + k]; b[k] = right[5 * i + k]; }
    t5_hash_pair(a, b, h, sbox + (threadIdx.x & 31));
    store_digest(out + 5 * i, h);
}

__global__ void __launch_bounds__(128) k_tip5_perm(uint64_t* __restrict__ states, uint64_t count) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    t5_sbox_init(sbox);
    __syncthreads();
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint64_t s[T5_STATE];
#pragma unroll
    for (int k = 0; k < T5_STATE; k++) s[k] = states[16 * i + k];
    t5_permutation(s, sbox + (threadIdx.x & 31));
#pragma unroll
    for (int k = 0; k < T5_STATE; k++) states[16 * i + k] = gl_canon(s[k]);
}

// Rounds [r0, r0 + nr) on each state; with `trace`, the state after each round
// at trace[(i*nr + k)*16 + .].
__global__ void __launch_bounds__(128) k_tip5_rounds(uint64_t* __restrict__ states, uint64_t count, int r0, int nr,
                                                     uint64_t* __restrict__ trace) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    t5_sbox_init(sbox);
    __syncthreads();
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint64_t s[T5_STATE];
#pragma unroll
    for (int k = 0; k < T5_STATE; k++) s[k] = states[16 * i + k];
    for (int k = 0; k < nr; k++) {
        t5_round(s, sbox + (threadIdx.x & 31), r0 + k);
        if (trace) {
#pragma unroll
            for (int j = 0; j < T5_STATE; j++) trace[(i * nr + k) * 16 + j] = gl_canon(s[j]);
        }
    }
#pragma unroll
    for (int k = 0; k < T5_STATE; k++) states[16 * i + k] = gl_canon(s[k]);
}

// Root implied by leaf q and its authentication path (MerkleTree::verify,
// src/merkle/merkle_tree.cpp:343-364): paths[(q*len + k)*5 + .] is the sibling
// at height k; leaf index bit k says which side the running digest is on.
__global__ void __launch_bounds__(128) k_root_from_paths(const uint64_t* __restrict__ idx,
                                                         const uint64_t* __restrict__ leaves,
                                                         const uint64_t* __restrict__ paths, uint64_t count,
                                                         uint64_t len, uint64_t* __restrict__ roots) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    t5_sbox_init(sbox);
    __syncthreads();
    uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    uint64_t cur[5], sib[5];
#pragma unroll
    for (int j = 0; j < 5; j++) cur[j] = gl_canon(leaves[5 * q + j]);
    uint64_t at = idx[q];
    for (uint64_t k = 0; k < len; k++) {
#pragma unroll
        for (int j = 0; j < 5; j++) sib[j] = gl_canon(paths[(q * len + k) * 5 + j]);
        if (at & 1)
            t5_hash_pair(sib, cur, cur, sbox + (threadIdx.x & 31));
        else
            t5_hash_pair(cur, sib, cur, sbox + (threadIdx.x & 31));
        at >>= 1;
    }
#pragma unroll
    for (int j = 0; j < 5; j++) roots[5 * q + j] = cur[j];
}

// Fiat-Shamir absorb into one device sponge state: the elements (an optional
// leading word `lead`, then data[0..len)), then 1, then zeros to a multiple of
// 10; each 10-word chunk overwrites the rate and is followed by a permutation.
// One thread runs the chunks in order; the block only fills the S-box table.
__global__ void __launch_bounds__(32) k_sponge_absorb(uint64_t* __restrict__ state, const uint64_t* __restrict__ data,
                                                      uint64_t len, int has_lead, uint64_t lead) {
    __shared__ uint32_t sbox[T5_SBOX_WORDS];
    t5_sbox_init(sbox);
    __syncthreads();
    if (threadIdx.x != 0) return;
    uint64_t s[T5_STATE];
#pragma unroll
    for (int i = 0; i < T5_STATE; i++) s[i] = state[i];
    const uint64_t total = len + (has_lead ? 1 : 0);
    const uint64_t padded = (total + T5_RATE) / T5_RATE * T5_RATE;  // room for the 1
    for (uint64_t c0 = 0; c0 < padded; c0 += T5_RATE) {
#pragma unroll
        for (int i = 0; i < T5_RATE; i++) {
            const uint64_t j = c0 + i;
            uint64_t v = 0;
            if (j < total) v = has_lead ? (j == 0 ? lead : data[j - 1]) : data[j];
            else if (j == total) v = 1;
            s[i] = gl_canon(v);
        }
        t5_permutation(s, sbox);
    }
#pragma unroll
    for (int i = 0; i < T5_STATE; i++) state[i] = gl_canon(s[i]);
}

__global__ void k_gather_auth(const uint64_t* __restrict__ tree, uint64_t n, int layout, int height,
                              const uint64_t* __restrict__ idx, uint64_t count, uint64_t* __restrict__ out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count * (uint64_t)height) return;
    uint64_t q = t / height;
    int k = (int)(t - q * height);
    uint64_t node = ((n + idx[q]) >> k) ^ 1;
    const uint64_t* src = tree + 5 * node_slot(node, n, layout);
#pragma unroll
    for (int i = 0; i < 5; i++) out[5 * t + i] = src[i];
}

__global__ void k_gather_nodes(const uint64_t* __restrict__ tree, uint64_t n, int layout,
                               const uint64_t* __restrict__ hidx, uint64_t count, uint64_t* __restrict__ out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint64_t* src = tree + 5 * node_slot(hidx[t], n, layout);
#pragma unroll
    for (int i = 0; i < 5; i++) out[5 * t + i] = src[i];
}

__global__ void k_gather_rows(const uint64_t* __restrict__ tab, uint64_t ld, uint32_t width,
                              const uint64_t* __restrict__ rows, uint64_t count, uint64_t* __restrict__ out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count * (uint64_t)width) return;
    uint64_t q = t / width;
    uint64_t c = t - q * width;
    out[t] = tab[c * ld + rows[q]];
}

static inline int ilog2u(uint64_t x) { return 63 - __builtin_clzll(x); }

static inline unsigned grid_for(uint64_t work, unsigned threads) {
    return (unsigned)((work + threads - 1) / threads);
}

// The m nodes of one level (heap indices [m, 2m)) of a tree with n leaves are
// in place: build every level above.  Wide levels go one per launch with every
// thread busy; the rest, 8 levels per launch in shared memory.
static cudaError_t launch_tree_above(uint64_t* tree, uint64_t n, uint64_t m, int layout, cudaStream_t st) {
    while ((m >> 1) >= MERKLE_LEVEL_MIN_PARENTS) {
        count_launch();
        k_merkle_level<<<grid_for(m >> 1, HASH_THREADS), HASH_THREADS, 0, st>>>(tree, n, m, layout);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        m >>= 1;
    }
    while (m > 1) {
        const uint64_t parents = m >> 1;
        const unsigned threads = (unsigned)(parents < UP_THREADS ? parents : UP_THREADS);
        const int levels = ilog2u(threads) + 1;
        count_launch();
        k_merkle_up<<<grid_for(parents, threads), threads, 0, st>>>(tree, n, m, layout, levels);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        m >>= levels;
    }
    return cudaSuccess;
}

cudaError_t launch_merkle_from_leaves(uint64_t* tree, uint64_t n, int layout, cudaStream_t st) {
    return launch_tree_above(tree, n, n, layout, st);  // n leaves already in place
}

cudaError_t launch_hash_rows(const uint64_t* table, uint64_t rstride, uint64_t cstride, uint64_t rows,
                             uint32_t width, uint64_t* digests, uint64_t* tree, int layout,
                             cudaStream_t st) {
    if (rows == 0) return cudaSuccess;
    NvtxRange range("tvmc row hash + Merkle tree");
    if (tree == nullptr) {
        count_launch();
        k_hash_rows<<<grid_for(rows, HASH_THREADS), HASH_THREADS, 0, st>>>(table, rstride, cstride, rows, width,
                                                                           digests, nullptr, layout, 0);
        return cudaGetLastError();
    }
    unsigned threads = (unsigned)(rows < HASH_THREADS ? rows : HASH_THREADS);
    const int fuse = ilog2u(threads) < tuning_hash_fuse_levels() ? ilog2u(threads) : tuning_hash_fuse_levels();
    count_launch();
    k_hash_rows<<<grid_for(rows, threads), threads, fuse > 0 ? 40 * threads : 0, st>>>(
        table, rstride, cstride, rows, width, nullptr, tree, layout, fuse);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    // the block subtrees are complete up to `fuse` levels; continue from there
    return launch_tree_above(tree, rows, rows >> fuse, layout, st);
}

cudaError_t launch_hash_rows_multi(const MultiHashTable* tabs, int count, cudaStream_t st) {
    NvtxRange range("tvmc multi-table row hash + Merkle trees");
    const int fuse = ilog2u(HASH_THREADS);  // every level a CTA's rows span
    for (int c0 = 0; c0 < count; c0 += HASH_MULTI_MAX) {
        const int nj = count - c0 < HASH_MULTI_MAX ? count - c0 : HASH_MULTI_MAX;
        HashJobs hj{};
        TopJobs tj{};
        uint64_t blocks = 0;
        int ntops = 0;
        for (int k = 0; k < nj; k++) {
            const MultiHashTable& t = tabs[c0 + k];
            hj.j[k] = HashJob{t.lde, t.tree, t.L, t.width, (uint32_t)blocks};
            blocks += (t.L + HASH_THREADS - 1) / HASH_THREADS;
        }
        hj.count = nj;
        if (blocks == 0) continue;
        count_launch();
        k_hash_rows_multi<<<(unsigned)blocks, HASH_THREADS, 40 * HASH_THREADS, st>>>(hj, fuse);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        // above the fused levels: small remainders in one multi-tree launch, large
        // ones with the single-tree kernels
        for (int k = 0; k < nj; k++) {
            const MultiHashTable& t = tabs[c0 + k];
            const uint64_t m = t.L > HASH_THREADS ? t.L / HASH_THREADS : 1;
            if (m <= 1) continue;
            if (m <= MULTI_TOP_MAX_NODES) {
                tj.j[ntops++] = TopJob{t.tree, m};
            } else if ((e = launch_tree_above(t.tree, t.L, m, LAYOUT_HEAP, st)) != cudaSuccess) {
                return e;
            }
        }
        if (ntops) {
            count_launch();
            k_merkle_tops_multi<<<(unsigned)ntops, 256, 0, st>>>(tj);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

cudaError_t launch_merkle_tree(const uint64_t* leaves, uint64_t* tree, uint64_t n, int layout,
                               cudaStream_t st, int leaf_words) {
    count_launch();
    k_copy_leaves<<<grid_for(n, 256), 256, 0, st>>>(leaves, tree, n, layout, leaf_words);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_merkle_from_leaves(tree, n, layout, st);
}

cudaError_t launch_hash_pairs(const uint64_t* left, const uint64_t* right, uint64_t* out, uint64_t count,
                              cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    count_launch();
    k_hash_pairs<<<grid_for(count, 128), 128, 0, st>>>(left, right, out, count);
    return cudaGetLastError();
}

cudaError_t launch_tip5_permutations(uint64_t* states, uint64_t count, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    count_launch();
    k_tip5_perm<<<grid_for(count, 128), 128, 0, st>>>(states, count);
    return cudaGetLastError();
}

cudaError_t launch_tip5_rounds(uint64_t* states, uint64_t count, int r0, int nr, uint64_t* trace, cudaStream_t st) {
    if (count == 0 || nr == 0) return cudaSuccess;
    count_launch();
    k_tip5_rounds<<<grid_for(count, 128), 128, 0, st>>>(states, count, r0, nr, trace);
    return cudaGetLastError();
}

cudaError_t launch_root_from_paths(const uint64_t* idx, const uint64_t* leaves, const uint64_t* paths, uint64_t count,
                                   uint64_t len, uint64_t* roots, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    count_launch();
    k_root_from_paths<<<grid_for(count, 128), 128, 0, st>>>(idx, leaves, paths, count, len, roots);
    return cudaGetLastError();
}

cudaError_t launch_sponge_absorb(uint64_t* state, const uint64_t* data, uint64_t len, int has_lead, uint64_t lead,
                                 cudaStream_t st) {
    count_launch();
    k_sponge_absorb<<<1, 32, 0, st>>>(state, data, len, has_lead, lead);
    return cudaGetLastError();
}

cudaError_t launch_gather_auth_paths(const uint64_t* tree, uint64_t n, int layout, const uint64_t* idx,
                                     uint64_t count, uint64_t* out, cudaStream_t st) {
    int height = ilog2u(n);
    if (count == 0 || height == 0) return cudaSuccess;
    count_launch();
    k_gather_auth<<<grid_for(count * height, 256), 256, 0, st>>>(tree, n, layout, height, idx, count, out);
    return cudaGetLastError();
}

cudaError_t launch_gather_nodes(const uint64_t* tree, uint64_t n, int layout, const uint64_t* heap_idx,
                                uint64_t count, uint64_t* out, cudaStream_t st) {
    if (count == 0) return cudaSuccess;
    count_launch();
    k_gather_nodes<<<grid_for(count, 256), 256, 0, st>>>(tree, n, layout, heap_idx, count, out);
    return cudaGetLastError();
}

cudaError_t launch_gather_rows(const uint64_t* table, uint64_t ld, uint32_t width, const uint64_t* rows,
                               uint64_t count, uint64_t* out, cudaStream_t st) {
    if (count == 0 || width == 0) return cudaSuccess;
    count_launch();
    k_gather_rows<<<grid_for(count * width, 256), 256, 0, st>>>(table, ld, width, rows, count, out);
    return cudaGetLastError();
}

cudaError_t launch_absorb_stripe(const uint64_t* stripe, uint64_t L, uint32_t ncols, uint64_t* cap, int first,
                                 int last, uint64_t* tree, cudaStream_t st) {
    NvtxRange range("tvmc frugal stripe absorb");
    const unsigned threads = (unsigned)(L < HASH_THREADS ? L : HASH_THREADS);
    const int lt = 63 - __builtin_clzll(threads);
    const int fuse = last ? (lt < tuning_hash_fuse_levels() ? lt : tuning_hash_fuse_levels()) : 0;
    count_launch();
    k_absorb_stripe<<<(unsigned)(L / threads), threads, fuse > 0 ? 40 * threads : 0, st>>>(stripe, L, ncols, cap,
                                                                                          first, last, tree, fuse);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !last) return e;
    return launch_tree_above(tree, L, L >> fuse, LAYOUT_HEAP, st);  // complete the tree above the block subtrees
}

}  // namespace tvmc
