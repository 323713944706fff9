// Row-major -> column-major transpose of a trace with TMA tile copies
// (sm_100a): the replacement of the reference GPU prover's
// qzc_rowmajor_to_colmajor_bfe (src/gpu/gpu_stark.cu:125-180), which turns the
// CPU layout vector<vector<BFE>> ([row][col]) into the column-major layout the
// LDE and the row hash read.
//
// One CTA moves a tile of 32 rows x 16 columns: one thread issues a 2D TMA
// load of the tile (cp.async.bulk.tensor, completion on an mbarrier) into
// shared memory with the 128-byte swizzle, so that reading it column by column
// touches eight different bank groups per eight rows; the threads write the
// transposed tile densely, and one thread stores it with a 2D TMA store into
// the column-major output.  Out-of-range parts of edge tiles are filled with
// zeros on load and clipped on store by the TMA unit.  Tensor maps need 16-byte
// row strides, so this path takes tables whose width and height are even (a
// power-of-two height always is); others use the shared-memory tile kernel.
// Every mbarrier wait is bounded: after TMA_WAIT_LIMIT polls the CTA records a
// timeout in g_tma_timeouts and skips its tile.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>

#include "internal.cuh"

namespace tvmc {

__device__ unsigned int g_tma_timeouts = 0;

constexpr int TT_ROWS = 32, TT_COLS = 16;  // tile: 32 rows x 16 columns of 8-byte words
constexpr int TMA_WAIT_LIMIT = 1 << 22;

__global__ void __launch_bounds__(128) k_transpose_tma(const __grid_constant__ CUtensorMap in_map,
                                                       const __grid_constant__ CUtensorMap out_map) {
    __shared__ alignas(1024) uint64_t tin[TT_ROWS * TT_COLS];   // rows of 128 bytes, 128B-swizzled
    __shared__ alignas(128) uint64_t tout[TT_COLS * TT_ROWS];   // [col][row], dense
    __shared__ alignas(8) uint64_t bar;
    __shared__ int ok;
    const int r0 = blockIdx.x * TT_ROWS, c0 = blockIdx.y * TT_COLS;
    const uint32_t bar_a = (uint32_t)__cvta_generic_to_shared(&bar);
    const uint32_t tin_a = (uint32_t)__cvta_generic_to_shared(tin);
    const uint32_t tout_a = (uint32_t)__cvta_generic_to_shared(tout);
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_a));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_a),
                     "r"((uint32_t)sizeof(tin))
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(tin_a),
            "l"(reinterpret_cast<uint64_t>(&in_map)), "r"(c0), "r"(r0), "r"(bar_a)
            : "memory");
        uint32_t done = 0;
        for (int i = 0; i < TMA_WAIT_LIMIT && !done; i++)
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
                "selp.u32 %0, 1, 0, p;\n\t}"
                : "=r"(done)
                : "r"(bar_a)
                : "memory");
        ok = (int)done;
        if (!done) atomicAdd(&g_tma_timeouts, 1u);
    }
    __syncthreads();
    if (!ok) return;  // the load never completed: skip the tile (counted above)
    // element (r, c) of the swizzled tile: 16-byte granule c/2 of row r sits at granule (c/2) ^ (r & 7)
    const int r = threadIdx.x;  // 32 rows
#pragma unroll
    for (int k = 0; k < TT_COLS / 4; k++) {
        const int c = threadIdx.y + 4 * k;
        const int word = r * TT_COLS + ((((c >> 1) ^ (r & 7)) << 1) | (c & 1));
        tout[c * TT_ROWS + r] = tin[word];
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
        asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                         reinterpret_cast<uint64_t>(&out_map)),
                     "r"(r0), "r"(c0), "r"(tout_a)
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");  // smem must outlive the store's reads
    }
}

namespace {
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

bool encode_2d(CUtensorMap* m, const void* base, uint64_t inner, uint64_t outer, uint32_t box_inner,
               uint32_t box_outer, CUtensorMapSwizzle swz) {
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {inner * 8};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t estr[2] = {1, 1};
    return g_encode(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
}  // namespace

cudaError_t launch_transpose_tma(const uint64_t* in, uint64_t* out, uint64_t rows, uint64_t cols, cudaStream_t st) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    if ((rows & 1) || (cols & 1) || ((uintptr_t)in & 15) || ((uintptr_t)out & 15) || rows >= (1ull << 32) ||
        cols >= (1ull << 32))
        return cudaErrorNotSupported;
    std::call_once(g_encode_once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    });
    if (!g_encode) return cudaErrorNotSupported;
    CUtensorMap in_map, out_map;
    if (!encode_2d(&in_map, in, cols, rows, TT_COLS, TT_ROWS, CU_TENSOR_MAP_SWIZZLE_128B) ||
        !encode_2d(&out_map, out, rows, cols, TT_ROWS, TT_COLS, CU_TENSOR_MAP_SWIZZLE_NONE))
        return cudaErrorNotSupported;
    const dim3 grid((unsigned)((rows + TT_ROWS - 1) / TT_ROWS), (unsigned)((cols + TT_COLS - 1) / TT_COLS));
    if (grid.y > 65535) return cudaErrorNotSupported;
    count_launch();
    k_transpose_tma<<<grid, dim3(32, 4), 0, st>>>(in_map, out_map);
    return cudaGetLastError();
}

unsigned int tma_timeouts() {
    unsigned int v = 0;
    cudaMemcpyFromSymbol(&v, g_tma_timeouts, sizeof v);
    return v;
}

}  // namespace tvmc
