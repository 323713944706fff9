// Integer issue-rate probe: the denominator of the Tip5 roofline.
//
// Tip5 hashing is bound by 32-bit integer instruction issue, for which there
// is no vendor-measured peak on hand.  This kernel runs 16 independent chains
// per thread of an equal mix of IMAD (mad.lo.u32) and ALU (add.u32 / xor.b32)
// instructions, written as volatile PTX so that each counts as exactly one
// instruction, across 8 CTAs x 256 threads per SM.  The returned rate is
// thread-level integer instructions per second.
#include <cuda_runtime.h>
#include <cstdint>

#include "internal.cuh"
#include "tvmc.h"

namespace tvmc {

constexpr int PROBE_ITERS = 4096;
constexpr int PROBE_CHAINS = 16;
constexpr int PROBE_OPS_PER_ITER = PROBE_CHAINS * 4;  // 2 mad + 1 add + 1 xor per chain

__global__ void __launch_bounds__(256) k_int_probe(uint32_t* out, uint32_t seed) {
    uint32_t a[PROBE_CHAINS], b[PROBE_CHAINS];
#pragma unroll
    for (int j = 0; j < PROBE_CHAINS; j++) {
        a[j] = seed + threadIdx.x * 31u + j;
        b[j] = seed ^ (blockIdx.x * 131u + j);
    }
    for (int i = 0; i < PROBE_ITERS; i++) {
#pragma unroll
        for (int j = 0; j < PROBE_CHAINS; j++) {
            asm volatile("mad.lo.u32 %0, %0, 0x9E3779B1, %1;" : "+r"(a[j]) : "r"(b[j]));
            asm volatile("add.u32 %0, %0, %1;" : "+r"(b[j]) : "r"(a[j]));
            asm volatile("mad.lo.u32 %0, %0, 0x85EBCA6B, %1;" : "+r"(b[j]) : "r"(a[j]));
            asm volatile("xor.b32 %0, %0, %1;" : "+r"(a[j]) : "r"(b[j]));
        }
    }
    uint32_t acc = 0;
#pragma unroll
    for (int j = 0; j < PROBE_CHAINS; j++) acc ^= a[j] + b[j];
    if (acc == 0x12345678u) out[0] = acc;  // keeps the chains live
}

}  // namespace tvmc

extern "C" double tvmc_int_peak_probe(void* stream) {
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1.0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1.0;
    uint32_t* out = nullptr;
    if (cudaMallocAsync((void**)&out, 4, st) != cudaSuccess) return -1.0;
    const unsigned blocks = (unsigned)sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    tvmc::count_launch();
    tvmc::k_int_probe<<<blocks, threads, 0, st>>>(out, 1u);  // warm-up
    cudaEventRecord(e0, st);
    tvmc::count_launch();
    tvmc::k_int_probe<<<blocks, threads, 0, st>>>(out, 2u);
    cudaEventRecord(e1, st);
    float ms = 0.f;
    cudaError_t e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(out, st);
    if (e != cudaSuccess || ms <= 0.f) return -1.0;
    double ops = (double)blocks * threads * tvmc::PROBE_ITERS * tvmc::PROBE_OPS_PER_ITER;
    return ops / (ms * 1e-3);
}
