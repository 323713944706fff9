// Low-degree extension without any device allocation.
//
// Who needs this: callers that cannot call cudaMalloc at the point where they
// want an LDE -- code running under a custom allocator that must not be
// bypassed, a host process whose device memory is fully pre-reserved by
// another framework, or a hard-real-time prover loop in which an allocation
// (and the implicit synchronisation cudaMalloc/cudaFree may perform) is not
// allowed.  tvmc_lde_batch_gpu obtains its intermediate buffers and twiddle
// tables from the device allocator; this variant takes both from one
// file-scope static device array instead, so after the first call on a device
// it only launches kernels on the caller's stream.
//
// The array g_noalloc_scratch (TVMC_NOALLOC_SCRATCH_WORDS words = 64 MiB) is
// resident on every GPU that loads the library, until the process exits.
// Its first NOALLOC_TABLE_WORDS words hold the twiddle and coset-scale tables,
// rewritten by a small kernel whenever a call's size, expansion or offset
// differs from the previous call's on that device; the rest holds the
// four-step intermediates.  Nothing in it needs to start at zero: every word a
// call reads was written earlier by the same call.  All calls share the
// array, so calls whose work overlaps on the GPU (different streams, or
// different host threads) race and corrupt each other's results; serialize
// them on one stream.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>

#include "field.cuh"
#include "internal.cuh"
#include "tvmc.h"

namespace tvmc {
namespace {

constexpr size_t NOALLOC_TOTAL_WORDS = TVMC_NOALLOC_SCRATCH_WORDS;
// table layout (words): tw12_f 4096 | tw12_i 4096 | wn_f_lo 4096 | wn_f_hi 1024 |
// wn_i_lo 4096 | wn_i_hi 1024 | sc_lo 16*4096 | sc_hi 16*1024
constexpr size_t T_TW12_F = 0, T_TW12_I = 4096, T_WNF_LO = 8192, T_WNF_HI = 12288, T_WNI_LO = 13312,
                 T_WNI_HI = 17408, T_SC_LO = 18432, T_SC_HI = 18432 + 16 * 4096;
constexpr size_t NOALLOC_TABLE_WORDS = T_SC_HI + 16 * 1024;  // 100352
constexpr size_t NOALLOC_WORK_WORDS = NOALLOC_TOTAL_WORDS - NOALLOC_TABLE_WORDS;

static __device__ __align__(256) uint64_t g_noalloc_scratch[NOALLOC_TOTAL_WORDS];

// Device address of g_noalloc_scratch, looked up once per device.
constexpr int MAX_DEVICES = 64;
uint64_t* g_base[MAX_DEVICES] = {};
std::mutex g_setup_mu;
// The (logn, le, offset) whose tables the array holds on each device, or
// logn = -1 before the first call.  A call with the same parameters skips the
// table kernel: under the one-stream rule every earlier call's work, its table
// writes included, comes before this call's kernels on the GPU, and the tables
// region is written by the table kernel alone.
struct TableKey {
    int logn = -1, le = -1;
    uint64_t offset = 0;
};
TableKey g_tables[MAX_DEVICES];

// Formats the message into a stack buffer and hands it to tvmc_last_error().
int fail(int code, const char* fmt, ...) {
    char msg[256];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(msg, sizeof msg, fmt, ap);
    va_end(ap);
    return set_error(code, msg);
}

// Fills every table for an LDE of 2^logn rows, expansion 2^le, coset `offset`.
__global__ void k_noalloc_tables(uint64_t* t, int logn, int le, uint64_t offset) {
    const uint64_t pm1 = GL_P - 1;
    const uint64_t N = 1ull << logn;
    const int hi_len = logn > 12 ? 1 << (logn - 12) : 1;
    const int E = 1 << le;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < NOALLOC_TABLE_WORDS;
         i += (size_t)gridDim.x * blockDim.x) {
        uint64_t v = 0;
        if (i < T_WNF_LO) {  // w_4096^(+-m)
            const uint64_t w = gl_pow(7, pm1 >> 12);
            const uint64_t m = i & 4095;
            v = gl_pow(i < T_TW12_I ? w : gl_pow(w, pm1 - 1), m);
        } else if (i < T_SC_LO) {  // w_N^(+-e), lo and hi parts
            const bool inv = i >= T_WNI_LO;
            const size_t j = i - (inv ? T_WNI_LO : T_WNF_LO);
            uint64_t w = gl_pow(7, pm1 >> logn);
            if (inv) w = gl_pow(w, pm1 - 1);
            if (j < 4096) v = gl_pow(w, j);
            else if (j - 4096 < (size_t)hi_len) v = gl_pow(w, 4096 * (j - 4096));
        } else if (i < T_SC_HI) {  // s_c^e, s_c = offset * w_{EN}^c
            const size_t c = (i - T_SC_LO) / 4096, e = (i - T_SC_LO) % 4096;
            if (c < (size_t)E) v = gl_pow(gl_mul_c(offset, gl_pow(gl_pow(7, pm1 >> (logn + le)), c)), e);
        } else {  // N^-1 * s_c^(4096 j)
            const size_t c = (i - T_SC_HI) / hi_len, j = (i - T_SC_HI) % hi_len;
            if (c < (size_t)E) {
                const uint64_t s = gl_mul_c(offset, gl_pow(gl_pow(7, pm1 >> (logn + le)), c));
                v = gl_mul_c(GL_P - (pm1 >> logn), gl_pow(s, 4096 * j));  // N^-1 = p - (p-1)/N
            }
        }
        t[i] = v;
    }
    (void)N;
}

int setup_device(int dev, uint64_t** base) {
    if (dev < 0 || dev >= MAX_DEVICES) return fail(TVMC_ERR_UNSUPPORTED, "device ordinal %d not supported", dev);
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_base[dev]) {
        // On the host, g_noalloc_scratch names a shadow object, not device memory:
        // the kernels must be given the address the runtime reports for this device.
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(TVMC_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_base[dev] = static_cast<uint64_t*>(p);
    }
    *base = g_base[dev];
    return TVMC_OK;
}

}  // namespace
}  // namespace tvmc

extern "C" int tvmc_lde_batch_noalloc_gpu(const uint64_t* d_traces, size_t num_columns, size_t trace_len,
                                          uint64_t* d_extended, size_t extended_len, uint64_t trace_offset,
                                          uint64_t extended_offset, void* stream) {
    using namespace tvmc;
    (void)trace_offset;  // ignored, as in tvmc_lde_batch_gpu and the reference's LDE::extend_column
    int logn = 0, le = 0;
    int rc = check_lde_sizes(trace_len, extended_len, &logn, &le);  // the allocating entry point's rules
    if (rc) return rc;
    const size_t per_col = lde_scratch_words(logn, le, 1);
    if (per_col > NOALLOC_WORK_WORDS)
        return fail(TVMC_ERR_UNSUPPORTED,
                    "one column needs %zu scratch words (trace_len * (1 + expansion)); the static scratch holds "
                    "%zu -- use tvmc_lde_batch_gpu for this size",
                    per_col, NOALLOC_WORK_WORDS);
    if (num_columns == 0) return TVMC_OK;

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(TVMC_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    uint64_t* base = nullptr;
    if ((rc = setup_device(dev, &base))) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);

    const uint64_t off = extended_offset % GL_P;
    {
        std::lock_guard<std::mutex> lk(g_setup_mu);
        TableKey& k = g_tables[dev];
        if (k.logn != logn || k.le != le || k.offset != off) {
            k.logn = -1;  // invalid until the table kernel is enqueued
            count_launch();
            k_noalloc_tables<<<98, 1024, 0, st>>>(base, logn, le, off);
            if ((e = cudaGetLastError()) != cudaSuccess)
                return fail(TVMC_ERR_CUDA, "table kernel: %s", cudaGetErrorString(e));
            k.logn = logn;
            k.le = le;
            k.offset = off;
        }
    }

    LdePlan pl;
    pl.logn = logn;
    pl.log_exp = le;
    pl.offset = extended_offset;
    pl.tw12_f = base + T_TW12_F;
    pl.tw12_i = base + T_TW12_I;
    pl.wn_f_lo = base + T_WNF_LO;
    pl.wn_f_hi = base + T_WNF_HI;
    pl.wn_i_lo = base + T_WNI_LO;
    pl.wn_i_hi = base + T_WNI_HI;
    pl.sc_lo = base + T_SC_LO;
    pl.sc_hi = base + T_SC_HI;
    uint64_t* work = base + NOALLOC_TABLE_WORDS;
    const size_t chunk = per_col ? NOALLOC_WORK_WORDS / per_col : num_columns;
    for (size_t c0 = 0; c0 < num_columns; c0 += chunk) {
        const size_t nc = num_columns - c0 < chunk ? num_columns - c0 : chunk;
        e = launch_lde(pl, d_traces + c0 * trace_len, trace_len, d_extended + c0 * extended_len, extended_len, nc,
                       work, st);
        if (e != cudaSuccess) return fail(TVMC_ERR_CUDA, "launch_lde: %s", cudaGetErrorString(e));
    }
    return TVMC_OK;
}
