// Harness over the reference prover's OWN CUDA kernels (MEASUREMENT ONLY).
//
// Built by `make refgpu` (oracle/Makefile) into oracle/_ref/libtvm_ref_gpu.so
// from the unchanged reference sources src/gpu/kernels/{ntt,randomized_lde,
// row_hash,tip5,merkle}_kernel.cu, compiled with nvcc for sm_100a.  It exposes
// the reference's host launchers for the commitment path behind a C ABI so
// that `bench.py --impl reference --reference-gpu` can time them on the same
// B200 and the same inputs as this library:
//   randomized_lde_batch_gpu_preallocated (src/gpu/kernels/randomized_lde_kernel.cu:956-1256,
//       with no randomizers and trace offset 1: the plain LDE of LDE::extend_column),
//   ntt_{forward,inverse}_batched_gpu (src/gpu/kernels/ntt_kernel.cu:2009-2600),
//   hash_bfield_rows_gpu / hash_xfield_rows_gpu (src/gpu/kernels/row_hash_kernel.cu:358-526),
//   merkle_tree_gpu (src/gpu/kernels/merkle_kernel.cu:41-105).
// Each wrapper returns the CUDA error state after the launcher (the reference's
// launchers return nothing).
#include <cuda_runtime.h>
#include <cstdint>

#include "gpu/kernels/merkle_kernel.cuh"
#include "gpu/kernels/ntt_kernel.cuh"
#include "gpu/kernels/randomized_lde_kernel.cuh"
#include "gpu/kernels/row_hash_kernel.cuh"

using namespace triton_vm::gpu::kernels;

extern "C" {

// Plain LDE of `cols` column-major columns (trace[c*n + r] -> out[c*L + r])
// onto offset * <w_L>; scratch holds cols * n words.
int tvmrg_lde(const uint64_t* d_trace, size_t cols, size_t n, uint64_t* d_out, size_t L, uint64_t offset,
              uint64_t* d_scratch, void* stream) {
    randomized_lde_batch_gpu_preallocated(d_trace, cols, n, nullptr, 0, 1, offset, L, d_out, d_scratch, d_scratch,
                                          static_cast<cudaStream_t>(stream));
    return (int)cudaGetLastError();
}

int tvmrg_ntt(uint64_t* d_data, size_t n, size_t cols, int inverse, void* stream) {
    if (inverse)
        ntt_inverse_batched_gpu(d_data, n, cols, static_cast<cudaStream_t>(stream));
    else
        ntt_forward_batched_gpu(d_data, n, cols, static_cast<cudaStream_t>(stream));
    return (int)cudaGetLastError();
}

int tvmrg_hash_bfield_rows(const uint64_t* d_table, size_t rows, size_t cols, uint64_t* d_digests, void* stream) {
    hash_bfield_rows_gpu(d_table, rows, cols, d_digests, static_cast<cudaStream_t>(stream));
    return (int)cudaGetLastError();
}

int tvmrg_hash_xfield_rows(const uint64_t* d_table, size_t rows, size_t xfe_cols, uint64_t* d_digests,
                           void* stream) {
    hash_xfield_rows_gpu(d_table, rows, xfe_cols, d_digests, static_cast<cudaStream_t>(stream));
    return (int)cudaGetLastError();
}

// Flat tree of 2n - 1 digests: leaves first, root last.
int tvmrg_merkle_tree(const uint64_t* d_leaves, uint64_t* d_tree, size_t n, void* stream) {
    merkle_tree_gpu(d_leaves, d_tree, n, static_cast<cudaStream_t>(stream));
    return (int)cudaGetLastError();
}

}  // extern "C"
