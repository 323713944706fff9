/*
 * tvmc -- B200 (sm_100a) table-commitment library, C ABI.
 *
 * The table-commitment path of the Triton VM prover: per-column low-degree
 * extension (LDE) over Goldilocks p = 2^64 - 2^32 + 1, the Tip5 hash of every
 * LDE row, and the Tip5 Merkle tree over the row digests.  Every result is
 * bit-identical to the reference prover's CPU path (canonical field elements).
 *
 * Conventions
 *   - Field elements are uint64_t.  Inputs >= p are accepted and read as their
 *     residue mod p (the reference's BFieldElement(uint64_t) constructor does
 *     the same); every output is canonical (< p).
 *   - A digest is 5 consecutive uint64_t.
 *   - "Column-major" table: element (row r, column c) at ptr[c*len + r].
 *     "Row-major": ptr[r*width + c].  An XFieldElement column contributes three
 *     consecutive base columns (c0, c1, c2), the order in which the reference
 *     flattens aux rows for hashing (src/table/table_commitment.cpp:65-77).
 *   - Functions named *_gpu take DEVICE pointers, are stream-ordered and
 *     return after enqueueing work; `stream` is a cudaStream_t (NULL = the
 *     legacy default stream).  Functions named *_host take HOST pointers and
 *     return when the result is in host memory.
 *   - Every function returns a tvmc status; tvmc_last_error() describes the
 *     most recent failure on the calling thread.
 *   - Thread safety: the library is safe to call from several threads; one
 *     commitment handle must not be used from two threads at once.
 *   - The first call on a device builds twiddle tables with synchronous copies;
 *     make one call before capturing work into a CUDA graph.
 *
 * Reference interfaces replaced are cited per entry point (paths inside the
 * reference project).
 */
#ifndef TVMC_H
#define TVMC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define TVMC_OK 0
#define TVMC_ERR_INVALID 1     /* size not a power of two, zero width, bad flag ... */
#define TVMC_ERR_RANGE 2       /* leaf / row index out of range */
#define TVMC_ERR_NOMEM 3       /* device allocation or admission failure */
#define TVMC_ERR_CUDA 4        /* CUDA runtime error (see tvmc_last_error) */
#define TVMC_ERR_TIMEOUT 5     /* a bounded device wait expired */
#define TVMC_ERR_UNSUPPORTED 6 /* size beyond what this build supports */

/* Largest supported sizes (log2). */
#define TVMC_MAX_LOG_NTT 24       /* plain NTT length */
#define TVMC_MAX_LOG_LDE_TRACE 22 /* LDE trace length; LDE length up to 2^26 */

const char* tvmc_last_error(void);
const char* tvmc_status_string(int status);
int tvmc_version(void);
/* Number of CUDA devices visible (0 when no GPU); never fails. */
int tvmc_device_count(void);

/* ---- NTT (include/gpu/kernels/ntt_kernel.cuh:88-106, src/ntt/ntt.cpp:59-86) ---- */

/* In-place forward NTT of num_cols column-major columns of length n
 * (d_data[col*n + row]); natural order in and out; w = 7^((p-1)/n).
 * Replaces triton_vm::gpu::kernels::ntt_forward_batched_gpu. */
int tvmc_ntt_forward_batched_gpu(uint64_t* d_data, size_t n, size_t num_cols, void* stream);
/* In-place inverse NTT (w^-1, scaled by n^-1).
 * Replaces triton_vm::gpu::kernels::ntt_inverse_batched_gpu. */
int tvmc_ntt_inverse_batched_gpu(uint64_t* d_data, size_t n, size_t num_cols, void* stream);
/* Host-buffer form of the two above (NTT::forward / NTT::inverse on each column). */
int tvmc_ntt_host(uint64_t* data, size_t n, size_t num_cols, int inverse);
/* NTT::evaluate_on_coset (src/ntt/ntt.cpp:94-117) of num_cols coefficient
 * columns (d_coeffs[col*num_coeffs + i]): the first min(num_coeffs, domain_len)
 * coefficients, zero-extended to domain_len and scaled by offset^i, forward
 * NTT; d_out[col*domain_len + j] = f(offset * w^j). */
int tvmc_evaluate_on_coset_gpu(const uint64_t* d_coeffs, size_t num_coeffs, size_t num_cols, uint64_t* d_out,
                               size_t domain_len, uint64_t offset, void* stream);
/* Host-buffer form. */
int tvmc_evaluate_on_coset_host(const uint64_t* coeffs, size_t num_coeffs, size_t num_cols, uint64_t* out,
                                size_t domain_len, uint64_t offset);

/* Row-major (the CPU layout vector<vector<BFE>>, d_in[r*cols + c]) to
 * column-major (d_out[c*rows + r]) on the device, out of place.  Replaces
 * qzc_rowmajor_to_colmajor_bfe (src/gpu/gpu_stark.cu:125-180). */
int tvmc_rowmajor_to_colmajor_gpu(const uint64_t* d_in, size_t rows, size_t cols, uint64_t* d_out, void* stream);

/* ---- LDE (include/gpu/kernels/lde_kernel.cuh lde_batch_gpu; src/ntt/ntt.cpp:121-131) ---- */

/* Low-degree extension of num_columns column-major columns: interpolate each
 * column on the size-trace_len subgroup, then evaluate on
 * extended_offset * <w_extended_len>.  trace_offset is ignored, as in the
 * reference's LDE::extend_column and lde_column_gpu.  extended_len must be
 * trace_len * 2^k with 0 <= k <= 4.  Replaces lde_batch_gpu. */
int tvmc_lde_batch_gpu(const uint64_t* d_traces, size_t num_columns, size_t trace_len, uint64_t* d_extended,
                       size_t extended_len, uint64_t trace_offset, uint64_t extended_offset, void* stream);
/* Host-buffer form (LDE::extend_table on column-major data). */
int tvmc_lde_host(const uint64_t* traces, size_t num_columns, size_t trace_len, uint64_t* extended,
                  size_t extended_len, uint64_t extended_offset);

/* Randomized LDE (RandomizedLDE::extend_column_with_randomizer,
 * src/lde/lde_randomized.cpp:71-154; the GPU counterpart is the randomized LDE
 * of src/gpu/gpu_stark.cu:2132-2617): interpolant of each column on
 * trace_offset * <w_trace_len> (the trace offset is honoured here), plus
 * (x^trace_len - trace_offset^trace_len) * r(x) with r's num_randomizers
 * coefficients at d_randomizers[col*num_randomizers + k], evaluated on
 * extended_offset * <w_extended_len>.  flags: 0 or TVMC_RAND_TRUNCATE. */
int tvmc_lde_randomized_gpu(const uint64_t* d_traces, size_t num_columns, size_t trace_len,
                            const uint64_t* d_randomizers, size_t num_randomizers, uint64_t* d_extended,
                            size_t extended_len, uint64_t trace_offset, uint64_t extended_offset, uint32_t flags,
                            void* stream);
/* Host-buffer form. */
int tvmc_lde_randomized_host(const uint64_t* traces, size_t num_columns, size_t trace_len,
                             const uint64_t* randomizers, size_t num_randomizers, uint64_t* extended,
                             size_t extended_len, uint64_t trace_offset, uint64_t extended_offset, uint32_t flags);

/* Words (64 MiB) of the static device array used by tvmc_lde_batch_noalloc_gpu. */
#define TVMC_NOALLOC_SCRATCH_WORDS ((size_t)1 << 23)
/* The same LDE as tvmc_lde_batch_gpu, same arguments and results, but it never
 * allocates device memory: intermediates and twiddle tables live in one static
 * device array of TVMC_NOALLOC_SCRATCH_WORDS words that every GPU loading this
 * library keeps until the process exits.  For callers that may not call the
 * CUDA allocator (a prover running under a pre-reserved or custom memory
 * manager, or a latency-critical loop where cudaMalloc's implicit
 * synchronisation is not acceptable).  Limit: trace_len * (1 + expansion)
 * must fit in the array minus its 100352 table words (e.g. 2^20 rows at
 * expansion 4); larger sizes return TVMC_ERR_UNSUPPORTED.  The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress), so
 * make that first call before capturing any stream.  All calls share the
 * array: calls that overlap on the GPU race, so issue them on one stream.
 * No counterpart in the reference. */
int tvmc_lde_batch_noalloc_gpu(const uint64_t* d_traces, size_t num_columns, size_t trace_len,
                               uint64_t* d_extended, size_t extended_len, uint64_t trace_offset,
                               uint64_t extended_offset, void* stream);

/* ---- Tip5 (include/gpu/kernels/row_hash_kernel.cuh:26-49, src/hash/tip5.cpp) ---- */

/* Tip5::hash_varlen of every row of a column-major table (d_table[col*num_rows + row]).
 * Replaces hash_bfield_rows_gpu. */
int tvmc_hash_bfield_rows_gpu(const uint64_t* d_table, size_t num_rows, size_t num_cols, uint64_t* d_digests,
                              void* stream);
/* Same for an XFieldElement table stored as (xfe_col*3 + component)*num_rows + row.
 * Replaces hash_xfield_rows_gpu. */
int tvmc_hash_xfield_rows_gpu(const uint64_t* d_table, size_t num_rows, size_t num_xfe_cols,
                              uint64_t* d_digests, void* stream);
/* Tip5::hash_varlen of num_rows host rows of row_len elements each (row-major). */
int tvmc_hash_varlen_host(const uint64_t* rows, size_t num_rows, size_t row_len, uint64_t* digests);
/* Tip5::hash_pair on count pairs (Backend::hash_pairs, include/backend/backend.hpp:106-120). */
int tvmc_hash_pairs_gpu(const uint64_t* d_left, const uint64_t* d_right, uint64_t* d_out, size_t count,
                        void* stream);
int tvmc_hash_pairs_host(const uint64_t* left, const uint64_t* right, uint64_t* out, size_t count);
/* Tip5 permutation of num_states 16-word states in place
 * (Backend::tip5_permutation_batch, include/backend/backend.hpp:99-104). */
int tvmc_tip5_permutation_batch_gpu(uint64_t* d_states, size_t num_states, void* stream);
int tvmc_tip5_permutation_batch_host(uint64_t* states, size_t num_states);
/* Tip5::round for rounds [first_round, first_round + num_rounds) of each state
 * (src/hash/tip5.cpp:114-118); with a non-null trace, the state after each
 * round goes to trace[(i*num_rounds + k)*16 + .] (Tip5::trace, :97-112). */
int tvmc_tip5_rounds_host(uint64_t* states, size_t num_states, uint32_t first_round, uint32_t num_rounds,
                          uint64_t* trace);
/* The Tip5 parameters this library computes with: the 256-byte S-box lookup
 * table, the MDS matrix's first column and the 80 round constants
 * (Tip5::LOOKUP_TABLE, MDS_MATRIX_FIRST_COLUMN, ROUND_CONSTANTS,
 * src/hash/tip5.cpp:7-79).  Host only; any pointer may be null. */
int tvmc_tip5_parameters(uint8_t* lookup_table, uint64_t* mds_first_column, uint64_t* round_constants);

/* ---- Merkle (include/gpu/kernels/merkle_kernel.cuh:26-50, src/merkle/merkle_tree.cpp) ---- */

/* Full tree in the reference GPU layout: d_tree holds 2n-1 digests
 * [leaves | level 1 | ... | root], root at index 2n-2.  Replaces merkle_tree_gpu. */
int tvmc_merkle_tree_gpu(const uint64_t* d_leaves, uint64_t* d_tree, size_t num_leaves, void* stream);
/* Root only (5 words to device memory).  Replaces merkle_root_gpu. */
int tvmc_merkle_root_gpu(const uint64_t* d_leaves, uint64_t* d_root, size_t num_leaves, void* stream);
/* Heap layout, as the reference's CPU MerkleTree: nodes holds 2n digests,
 * node 1 is the root, leaves at [n, 2n), node 0 is written as zeros. */
int tvmc_merkle_tree_heap_host(const uint64_t* leaves, size_t num_leaves, uint64_t* nodes);
/* Root implied by each (leaf index, leaf digest, authentication path) triple,
 * as MerkleTree::verify walks it (src/merkle/merkle_tree.cpp:343-364): sibling
 * k of triple q at paths[(q*path_len + k)*5 + .]; roots[q*5 + .].  A path
 * verifies iff its root equals the tree's. */
int tvmc_merkle_root_from_paths_gpu(const size_t* d_leaf_idx, const uint64_t* d_leaves, const uint64_t* d_paths,
                                    size_t count, size_t path_len, uint64_t* d_roots, void* stream);
/* Host-buffer form. */
int tvmc_merkle_root_from_paths_host(const size_t* leaf_idx, const uint64_t* leaves, const uint64_t* paths,
                                     size_t count, size_t path_len, uint64_t* roots);

/* ---- table commitment (the whole path; src/gpu/gpu_stark.cu:2132-2617 step 2/3,
 *      src/stark.cpp:1163-1196, LDETable::compute_lde_and_merkle src/lde/lde_table.cpp:86-101) ---- */

typedef struct tvmc_commitment tvmc_commitment;

#define TVMC_TRACE_DEVICE 0x1u    /* trace is a device pointer (else host) */
#define TVMC_TRACE_ROW_MAJOR 0x2u /* trace is row-major [trace_len][width] (else column-major) */
#define TVMC_DISCARD_LDE 0x4u     /* free the LDE after hashing; keep only the tree */
#define TVMC_SYNC 0x8u            /* return only when the commitment is complete */
#define TVMC_PROFILE 0x10u        /* record CUDA events around the upload, LDE and hash/tree phases */
#define TVMC_FRUGAL 0x20u         /* streaming mode: LDE in 10-column-aligned stripes absorbed into
                                     resident sponge states; the full LDE is never stored (implies
                                     TVMC_DISCARD_LDE); for very tall tables (2^22 rows and up) */
#define TVMC_RAND_TRUNCATE 0x40u  /* randomized LDE: drop coefficients of degree >= the LDE length
                                     before evaluating, as the reference's XFieldElement variants do
                                     (RandomizedLDE::extend_xfield_column_with_randomizer,
                                     src/lde/lde_randomized.cpp:246-251); otherwise a longer
                                     polynomial is evaluated exactly (chunked, :120-153) */

/* Tuning knobs (process-wide; 0 restores the default):
 *   "frugal_stripe_cols"  columns per TVMC_FRUGAL stripe, rounded down to a multiple of 10
 *                         (default: the widest stripe whose LDE fits in 2 GiB, at least 10)
 *   "lde_scratch_bytes"   LDE intermediate budget per call (default 2 GiB); columns are
 *                         processed in chunks that fit
 *   "batch_streams"       worker streams a tvmc_batch spreads its tables over (default 8)
 *   "transpose_tma"       1: row-major traces are transposed with TMA tile copies where the width
 *                         and height are even; 2 (or 0, the default): shared-memory tiles
 *   "batch_multi_hash"    1: a tvmc_batch hashes all its tables with one multi-table launch after
 *                         their LDEs; 2: each worker stream hashes its own tables; default 1
 *   "lde_mid_ctas"        resident CTAs per SM for the fused LDE middle kernel: 2 (no register
 *                         spills) or 3 (a few spills); default 3
 *   "lde_mid_variant"     1: the fused LDE middle kernel reads its twiddles from global tables per
 *                         coset; 2: it forms the inter-pass twiddles once per CTA in shared
 *                         memory for all cosets; default 2
 *   "lde_split_l1"        log2 of the LDE's four-step factor n1 (6 .. 12, with log2(N) - n1 also
 *                         in 6 .. 12, else the balanced split is used); default 0 = balanced
 *   "ntt_tile_log"        log2 of the words an NTT/LDE pass CTA moves per tile (11 .. 15);
 *                         default 0 = 13
 *   "hash_unfused_tree"   1: build every Merkle level in the tree kernel instead of the lowest
 *                         eight inside the row-hash CTAs; default 0
 *   "fail_alloc_after"    fault injection for tests: k > 0 makes the k-th device allocation the
 *                         library requests from now on fail as out-of-memory (once, on the host,
 *                         without reaching the driver); 0 disables
 * Unknown keys return TVMC_ERR_INVALID.  tvmc_get_tuning also reads "pool_used_bytes": the bytes
 * currently allocated from the current device's stream-ordered pool (a leak check). */
int tvmc_set_tuning(const char* key, long long value);
/* The library keeps its LDE/NTT scratch, upload staging and the LDE of
 * TVMC_DISCARD_LDE commitments per (device, stream) once used, and the device's
 * stream-ordered memory pool keeps freed memory, so that repeated commits never
 * wait for the driver to map memory.  This frees
 * that scratch, the cached twiddle and coset-scale tables (unless a tvmc_batch
 * is alive on the device: its graph refers to them) and returns the pool's
 * unused memory on the current device; it synchronizes the device first.  Call
 * it only while no other thread is issuing work to this library on the device. */
int tvmc_release_cached_memory(void);
/* Frees the buffers this library keeps for one stream (and its upload stream),
 * ordered after the work already queued on it.  Call before destroying a
 * stream that was passed to this library, so that its memory is not held. */
int tvmc_forget_stream(void* stream);
int tvmc_get_tuning(const char* key, long long* value);

/* Commit to one table: LDE of every column onto offset * <w_{trace_len*expansion}>
 * (expansion a power of two <= 16), Tip5 hash_varlen of every LDE row, Merkle
 * tree over the row digests.  The LDE (column-major, len trace_len*expansion)
 * and the heap-layout tree stay in device memory, owned by *out, until
 * tvmc_commitment_free.  Work is enqueued on `stream`. */
int tvmc_commit(const uint64_t* trace, size_t trace_len, size_t width, uint32_t expansion, uint64_t offset,
                uint32_t flags, void* stream, tvmc_commitment** out);
/* Several plain commitments at once: per table the same as tvmc_commit (LDE
 * onto offset * <w_{trace_len*expansion}>, Tip5 row hash, heap Merkle tree),
 * but the row hashing and the small tree tops of all tables run as one launch
 * each, so that many small tables fill the GPU together instead of one after
 * another.  out[i] receives table i's commitment (free each with
 * tvmc_commitment_free).  Flags: TVMC_TRACE_DEVICE (every trace is a device
 * pointer), TVMC_DISCARD_LDE, TVMC_SYNC.  On failure no commitment is
 * returned.  No reference counterpart (the reference commits one table at a
 * time, src/stark.cpp:1163-1196). */
typedef struct {
    const uint64_t* trace; /* column-major, width x trace_len */
    size_t trace_len;
    size_t width;
    uint32_t expansion;
    uint64_t offset;
} tvmc_multi_table;
int tvmc_commit_multi(const tvmc_multi_table* tables, size_t count, uint32_t flags, void* stream,
                      tvmc_commitment** out);
/* The same commitment over the randomized (zero-knowledge) LDE of
 * LDETable::extend_table_with_randomizers / RandomizedLDE::extend_column_with_randomizer
 * (src/lde/lde_table.cpp:8-57, src/lde/lde_randomized.cpp:71-154): per column
 * the interpolant on trace_offset * <w_trace_len> plus (x^trace_len - trace_offset^trace_len)
 * times the randomizer polynomial, evaluated on offset * <w_{trace_len*expansion}>.
 * randomizers holds num_randomizers coefficients per column, column after column
 * (randomizers[col*num_randomizers + k]) whatever the trace layout, on the host,
 * or on the device with TVMC_TRACE_DEVICE.  num_randomizers = 0 with trace_offset = 1
 * is tvmc_commit.  TVMC_RAND_TRUNCATE selects the truncating variant. */
int tvmc_commit_randomized(const uint64_t* trace, size_t trace_len, size_t width, uint32_t expansion,
                           uint64_t trace_offset, uint64_t offset, const uint64_t* randomizers,
                           size_t num_randomizers, uint32_t flags, void* stream, tvmc_commitment** out);
/* Commitment to rows that are already evaluated, with no LDE: the quotient
 * segments' table (leaf = hash_xfield_row of each row, src/stark.cpp:759-764 and
 * 1942-1987, TableCommitment::from_digests src/table/table_commitment.cpp) or any
 * other codeword table.  Leaf r = Tip5 hash_varlen of row r; num_rows must be a
 * power of two.  Flags: TVMC_TRACE_DEVICE, TVMC_TRACE_ROW_MAJOR (as for
 * tvmc_commit), TVMC_DISCARD_LDE (keep only the tree; otherwise a column-major
 * copy of the rows is kept for tvmc_commitment_read_rows), TVMC_SYNC.  The
 * handle's "LDE" is the table itself (tvmc_commitment_shape: lde_len = num_rows). */
int tvmc_commit_rows(const uint64_t* table, size_t num_rows, size_t width, uint32_t flags, void* stream,
                     tvmc_commitment** out);

#define TVMC_LEAVES_XFE 0x80u /* tvmc_commit_digests: leaves are XFieldElements (3 words each) */
/* Commitment to given leaves: a Merkle tree over num_leaves digests (5 words
 * each; MerkleTree(leaves), TableCommitment::from_digests), or with
 * TVMC_LEAVES_XFE over an XFieldElement codeword whose element i becomes the leaf
 * (c0, c1, c2, 0, 0) with no hashing -- the FRI round trees (src/fri/fri.cpp:25-43,
 * 715-730).  Host leaves, or device leaves with TVMC_TRACE_DEVICE; TVMC_SYNC. */
int tvmc_commit_digests(const uint64_t* leaves, size_t num_leaves, uint32_t flags, void* stream,
                        tvmc_commitment** out);
/* Fiat-Shamir absorb into a device sponge state (16 words; start from zeros):
 * d_data[0..len) followed by 1 and zeros up to a multiple of 10, each 10-word
 * chunk overwriting the rate, then one Tip5 permutation per chunk -- the
 * reference's fs_absorb_device_gpu (src/gpu/kernels/fiat_shamir_kernel.cu:174-191)
 * and ProofStream's pad-and-absorb, as one launch. */
int tvmc_sponge_absorb_gpu(uint64_t* d_state, const uint64_t* d_data, size_t len, void* stream);
/* Absorbs the commitment's root, encoded as the proof item MerkleRoot
 * (discriminant 0, then the 5 root words), into d_state on `stream`, ordered
 * after the commitment: the root never visits the host (src/gpu/gpu_stark.cu:2577-2585). */
int tvmc_commitment_absorb_root(tvmc_commitment* c, uint64_t* d_state, void* stream);
/* Wait for the commitment and copy its root (5 words) to host memory. */
int tvmc_commitment_root(tvmc_commitment* c, uint64_t* root);
int tvmc_commitment_sync(tvmc_commitment* c);
/* Sizes: LDE length (= number of leaves) and width. */
int tvmc_commitment_shape(const tvmc_commitment* c, size_t* lde_len, size_t* width);
/* Device pointers: column-major LDE (NULL after TVMC_DISCARD_LDE) and heap tree. */
int tvmc_commitment_device_lde(const tvmc_commitment* c, const uint64_t** d_lde);
int tvmc_commitment_device_tree(const tvmc_commitment* c, const uint64_t** d_nodes);
/* Authentication paths (MerkleTree::authentication_path, src/merkle/merkle_tree.cpp:93-113):
 * out holds count * log2(lde_len) digests, path of leaf_idx[q] first-sibling first. */
int tvmc_commitment_auth_paths(tvmc_commitment* c, const size_t* leaf_idx, size_t count, uint64_t* out);
/* Batched authentication structure (MerkleTree::authentication_structure,
 * src/merkle/merkle_tree.cpp:115-226): digests of the needed-but-not-computable
 * nodes in descending heap-index order.  Writes at most max_digests digests and
 * sets *num_digests to the full count. */
int tvmc_commitment_auth_structure(tvmc_commitment* c, const size_t* leaf_idx, size_t count, uint64_t* out,
                                   size_t max_digests, size_t* num_digests);
/* Heap indices of the authentication structure for leaf_idx over a tree of
 * num_leaves leaves, descending (MerkleTree::authentication_structure_node_indices,
 * src/merkle/merkle_tree.cpp:228-262).  Host-only; no device work. */
int tvmc_auth_structure_indices(size_t num_leaves, const size_t* leaf_idx, size_t count, uint64_t* out,
                                size_t max_out, size_t* num_out);
/* Rows of the LDE, row-major: out[q*width + col] = LDE[rows[q]][col]. */
int tvmc_commitment_read_rows(tvmc_commitment* c, const size_t* rows, size_t count, uint64_t* out);
/* Columns [col0, col0 + ncols) of the LDE to host memory, column-major. */
int tvmc_commitment_read_columns(tvmc_commitment* c, size_t col0, size_t ncols, uint64_t* out);
/* The whole LDE to host memory, column-major (or row-major with row_major != 0). */
int tvmc_commitment_read_lde(tvmc_commitment* c, uint64_t* out, int row_major);
/* All leaf digests (lde_len x 5) / all heap nodes (2*lde_len x 5) to host memory. */
int tvmc_commitment_read_leaves(tvmc_commitment* c, uint64_t* out);
int tvmc_commitment_read_nodes(tvmc_commitment* c, uint64_t* out);
int tvmc_commitment_free(tvmc_commitment* c);
/* ---- batched commitment of many tables (one CUDA-graph launch per run) ---- */

typedef struct tvmc_batch tvmc_batch;
typedef struct {
    size_t trace_len;   /* power of two, <= 2^22 */
    size_t width;       /* base columns (3 per XFieldElement column) */
    uint32_t expansion; /* power of two <= 16 */
    uint64_t offset;    /* coset offset of the evaluation domain */
} tvmc_table_shape;

/* Plan a batch of `count` tables of uneven heights and widths: allocate every
 * table's input buffer, LDE, tree and scratch once, and capture the whole
 * commitment of all tables (LDE -> row hash -> Merkle, tables spread over
 * worker streams that overlap on the device) into one instantiated CUDA
 * graph.  Worker-stream count: tuning knob "batch_streams" (default 8). */
int tvmc_batch_create(const tvmc_table_shape* shapes, size_t count, tvmc_batch** out);
/* Device input buffer of table i: column-major [width][trace_len]; fill it
 * (e.g. cudaMemcpyAsync on the run stream) before tvmc_batch_run. */
int tvmc_batch_input(tvmc_batch* b, size_t i, uint64_t** d_trace);
/* Commit every table: one cudaGraphLaunch on `stream`. */
int tvmc_batch_run(tvmc_batch* b, void* stream);
/* Commitment handle of table i (valid until tvmc_batch_free; do not free it):
 * all tvmc_commitment_* accessors work on it and wait for the last run. */
int tvmc_batch_commitment(tvmc_batch* b, size_t i, tvmc_commitment** c);
int tvmc_batch_free(tvmc_batch* b);

/* ---- commitment serving (no reference counterpart: the reference commits one
 *      table at a time in src/stark.cpp:1163-1196) ----
 *
 * A server runs a request loop on the current device: submitted tables queue
 * in arrival order; the head is admitted as soon as its device footprint
 * (tree, LDE, LDE scratch, upload staging) fits the HBM budget beside the
 * running requests and the trees still held, and is issued at once on the
 * least-loaded of its worker streams.  Small tables (LDE up to 128 MB) run
 * concurrently on num_streams high-priority streams and never wait behind
 * large ones; with TVMC_SERVER_GROUP_SMALL, plain small requests queued at
 * the same time are committed together as one tvmc_commit_multi (their row
 * hashes share one launch, so a burst of small tables fills the GPU instead
 * of trickling through it); large tables, each enough to fill the GPU, go in arrival order
 * onto one dedicated stream, with up to max_large_inflight of them issued at
 * once (the next one's upload overlaps the current one's kernels).  Each request's
 * Merkle tree stays on the device for openings until tvmc_server_release;
 * with TVMC_SERVER_KEEP_LDE its LDE stays too (rows can be opened).  Results
 * are bit-identical to tvmc_commit of the same table alone.  The trace buffer
 * must stay valid until tvmc_server_wait has returned for the request.  All
 * functions are thread-safe. */
typedef struct tvmc_server tvmc_server;

#define TVMC_SERVER_KEEP_LDE 0x1u
#define TVMC_SERVER_GROUP_SMALL 0x2u /* commit queued small requests together */

typedef struct tvmc_server_config {
    size_t hbm_budget_bytes; /* 0: 90% of the device memory free at creation */
    uint32_t num_streams;    /* worker streams for small tables, 0: 4 (at most 64) */
    uint32_t flags;          /* TVMC_SERVER_KEEP_LDE, TVMC_SERVER_GROUP_SMALL */
    uint32_t max_large_inflight; /* large tables issued at once, 0: 2 (at most 16) */
} tvmc_server_config;

typedef struct tvmc_server_stats {
    uint64_t submitted, completed, failed, released, queued, running;
    size_t bytes_in_use, bytes_peak, budget; /* admitted footprint bytes */
} tvmc_server_stats;

int tvmc_server_create(const tvmc_server_config* cfg, tvmc_server** out);
/* Queue one table (the arguments of tvmc_commit; flags may hold only
 * TVMC_TRACE_DEVICE, TVMC_TRACE_ROW_MAJOR and TVMC_FRUGAL). */
int tvmc_server_submit(tvmc_server* s, const uint64_t* trace, size_t trace_len, size_t width, uint32_t expansion,
                       uint64_t offset, uint32_t flags, uint64_t* request_id);
/* Queue one randomized commitment (the arguments of tvmc_commit_randomized;
 * flags may also hold TVMC_RAND_TRUNCATE).  The randomizer buffer, like the
 * trace, must stay valid until tvmc_server_wait has returned. */
int tvmc_server_submit_randomized(tvmc_server* s, const uint64_t* trace, size_t trace_len, size_t width,
                                  uint32_t expansion, uint64_t trace_offset, uint64_t offset,
                                  const uint64_t* randomizers, size_t num_randomizers, uint32_t flags,
                                  uint64_t* request_id);
/* Wait until the request is committed (timeout_ms < 0: no limit; expiry returns
 * TVMC_ERR_TIMEOUT) and copy its root; a request whose footprint exceeds the
 * whole budget fails with TVMC_ERR_NOMEM. */
int tvmc_server_wait(tvmc_server* s, uint64_t request_id, int64_t timeout_ms, uint64_t* root);
/* Openings of a committed request from its device-resident tree: auth paths
 * (count x height x 5 words, as tvmc_commitment_auth_paths) and, when the
 * server keeps LDEs and rows is non-null, the opened rows (count x width). */
int tvmc_server_open(tvmc_server* s, uint64_t request_id, const size_t* leaf_idx, size_t count, uint64_t* paths,
                     uint64_t* rows);
/* Submission, dispatch and completion times (CLOCK_MONOTONIC nanoseconds). */
int tvmc_server_times(tvmc_server* s, uint64_t request_id, uint64_t* submit_ns, uint64_t* start_ns,
                      uint64_t* done_ns);
/* Free a finished request's tree (and LDE) and return its bytes to the budget. */
int tvmc_server_release(tvmc_server* s, uint64_t request_id);
int tvmc_server_get_stats(tvmc_server* s, tvmc_server_stats* out);
/* Stops dispatching, waits for running requests and frees everything. */
int tvmc_server_destroy(tvmc_server* s);

/* For a TVMC_PROFILE commitment: device milliseconds of [upload (or transpose),
 * LDE, row hash + Merkle tree]; with a pipelined host upload the upload is
 * counted inside the LDE phase. */
int tvmc_commitment_phase_ms(tvmc_commitment* c, float* ms3);
/* Total kernels launched by this library so far (all threads and devices). */
unsigned long long tvmc_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* TVMC_H */
