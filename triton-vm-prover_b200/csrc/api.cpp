// C ABI of the table-commitment library (declared in include/tvmc.h).
//
// Host side: argument checking with the reference's error semantics, the
// per-device twiddle-table cache, stream-ordered scratch (cudaMallocAsync from
// the device's default pool), and the commitment handle that keeps the LDE and
// the Merkle tree resident for later openings.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "internal.cuh"
#include "tip5_params.h"
#include "tvmc.h"

using namespace tvmc;

namespace {
std::atomic<unsigned long long> g_launches{0};
}

void tvmc::count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char* where) {
    if (e == cudaErrorMemoryAllocation) return fail(TVMC_ERR_NOMEM, "%s: %s", where, cudaGetErrorString(e));
    return fail(TVMC_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

#define CK(expr)                                            \
    do {                                                    \
        cudaError_t e_ = (expr);                            \
        if (e_ != cudaSuccess) return cuda_fail(e_, #expr); \
    } while (0)

// Allocation-failure injection (tuning key "fail_alloc_after" = k > 0): the
// k-th device allocation this library requests from then on fails with
// cudaErrorMemoryAllocation without reaching the driver, once.  A host-side
// fault for tests of the out-of-memory paths (the counterpart of the
// reference's pre-flight check_gpu_memory, src/gpu/gpu_stark.cu:1588-1730);
// the GPU itself sees nothing.
std::atomic<long long> g_fail_alloc_after{0};

bool injected_alloc_failure() {
    long long k = g_fail_alloc_after.load();
    while (k > 0) {
        if (g_fail_alloc_after.compare_exchange_weak(k, k - 1)) return k == 1;
    }
    return false;
}

// Every device allocation of this file goes through these two.
template <class T>
cudaError_t dev_malloc(T** p, size_t bytes) {
    if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
    return cudaMalloc((void**)p, bytes);
}
template <class T>
cudaError_t dev_malloc_async(T** p, size_t bytes, cudaStream_t st) {
    if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
    return cudaMallocAsync((void**)p, bytes, st);
}

bool is_pow2(size_t n) { return n != 0 && (n & (n - 1)) == 0; }
int log2u(size_t n) {
    int k = 0;
    while ((size_t(1) << k) < n) k++;
    return k;
}

// ---- host Goldilocks (table construction only) ----
constexpr uint64_t P = 0xFFFFFFFF00000001ull;
uint64_t hmul(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) % P); }
uint64_t hpow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    b %= P;
    while (e) {
        if (e & 1) r = hmul(r, b);
        b = hmul(b, b);
        e >>= 1;
    }
    return r;
}
uint64_t hinv(uint64_t a) { return hpow(a, P - 2); }
uint64_t root_of_unity(int k) { return hpow(7, (P - 1) >> k); }

// ---- per-device table cache ----
struct DevTables {
    uint64_t* tw12_f = nullptr;
    uint64_t* tw12_i = nullptr;
    std::map<int, std::pair<uint64_t*, uint64_t*>> wn_f, wn_i;                  // logn -> (lo, hi)
    std::map<std::tuple<int, int, uint64_t>, std::pair<uint64_t*, uint64_t*>> sc;  // (logn, le, offset)
    bool pool_set = false;
    int live_batches = 0;  // batches hold plan pointers in their graphs: tables stay while any is alive
};
std::mutex g_mu;
std::map<int, DevTables> g_dev;

cudaError_t upload(const std::vector<uint64_t>& h, uint64_t** d) {
    cudaError_t e = dev_malloc(d, h.size() * 8);
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*d, h.data(), h.size() * 8, cudaMemcpyHostToDevice);
}

int current_device(int* dev) {
    CK(cudaGetDevice(dev));
    return TVMC_OK;
}

// Builds (once per device) the tables needed for size 2^logn and, if le >= 0,
// the LDE coset scales for expansion 2^le and `offset`.
int get_plan(int logn, int le, uint64_t offset, LdePlan* pl) {
    int dev;
    int rc = current_device(&dev);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_mu);
    DevTables& T = g_dev[dev];
    if (!T.pool_set) {
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        T.pool_set = true;
    }
    if (!T.tw12_f) {
        std::vector<uint64_t> f(4096), i(4096);
        uint64_t w = root_of_unity(12), wi = hinv(w), x = 1, y = 1;
        for (int m = 0; m < 4096; m++) {
            f[m] = x;
            i[m] = y;
            x = hmul(x, w);
            y = hmul(y, wi);
        }
        CK(upload(f, &T.tw12_f));
        CK(upload(i, &T.tw12_i));
    }
    auto make_wn = [&](bool inv, std::pair<uint64_t*, uint64_t*>* out) -> int {
        uint64_t w = root_of_unity(logn);
        if (inv) w = hinv(w);
        size_t hi_len = logn > 12 ? (size_t(1) << (logn - 12)) : 1;
        std::vector<uint64_t> lo(4096), hi(hi_len);
        uint64_t x = 1;
        for (int e = 0; e < 4096; e++) { lo[e] = x; x = hmul(x, w); }
        uint64_t w4096 = hpow(w, 4096);
        x = 1;
        for (size_t j = 0; j < hi_len; j++) { hi[j] = x; x = hmul(x, w4096); }
        CK(upload(lo, &out->first));
        CK(upload(hi, &out->second));
        return TVMC_OK;
    };
    if (!T.wn_f.count(logn)) {
        std::pair<uint64_t*, uint64_t*> a{}, b{};
        if ((rc = make_wn(false, &a))) return rc;
        if ((rc = make_wn(true, &b))) return rc;
        T.wn_f[logn] = a;
        T.wn_i[logn] = b;
    }
    pl->logn = logn;
    pl->log_exp = le < 0 ? 0 : le;
    pl->offset = offset;
    pl->tw12_f = T.tw12_f;
    pl->tw12_i = T.tw12_i;
    pl->wn_f_lo = T.wn_f[logn].first;
    pl->wn_f_hi = T.wn_f[logn].second;
    pl->wn_i_lo = T.wn_i[logn].first;
    pl->wn_i_hi = T.wn_i[logn].second;
    pl->sc_lo = pl->sc_hi = nullptr;
    if (le >= 0) {
        auto key = std::make_tuple(logn, le, offset % P);
        if (!T.sc.count(key)) {
            int E = 1 << le;
            size_t N = size_t(1) << logn;
            size_t hi_len = logn > 12 ? (size_t(1) << (logn - 12)) : 1;
            uint64_t wEN = root_of_unity(logn + le);
            uint64_t ninv = hinv(N % P);
            std::vector<uint64_t> lo(4096 * (size_t)E), hi(hi_len * (size_t)E);
            for (int c = 0; c < E; c++) {
                uint64_t s = hmul(offset % P, hpow(wEN, (uint64_t)c));
                uint64_t x = 1;
                for (int e = 0; e < 4096; e++) { lo[4096 * c + e] = x; x = hmul(x, s); }
                uint64_t s4096 = hpow(s, 4096);
                x = ninv;
                for (size_t j = 0; j < hi_len; j++) { hi[hi_len * c + j] = x; x = hmul(x, s4096); }
            }
            std::pair<uint64_t*, uint64_t*> pr{};
            CK(upload(lo, &pr.first));
            CK(upload(hi, &pr.second));
            T.sc[key] = pr;
        }
        pl->sc_lo = T.sc[key].first;
        pl->sc_hi = T.sc[key].second;
    }
    return TVMC_OK;
}

cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Process-wide tuning knobs (tvmc_set_tuning); 0 = default.
std::atomic<long long> g_tune_stripe_cols{0};
std::atomic<long long> g_tune_scratch_bytes{0};

size_t scratch_budget() {
    const long long b = g_tune_scratch_bytes.load();
    return b > 0 ? (size_t)b : (size_t(2) << 30);
}

// Column chunk so that LDE scratch stays within the budget.
size_t lde_chunk_cols(int logn, int le, size_t width) {
    size_t per = lde_scratch_words(logn, le, 1) * 8;
    if (per == 0) return width ? width : 1;
    size_t lim = scratch_budget() / per;
    if (lim < 1) lim = 1;
    return std::min(width ? width : size_t(1), lim);
}

// Randomizer addends of one table on the device, [col][coset][rm] (launch_rand_addend).
struct RandAdd {
    const uint64_t* add = nullptr;
    int rm = 0;
    int le = 0;
    const uint64_t* cols(size_t c0) const { return rm ? add + c0 * ((size_t)rm << le) : nullptr; }
};

// Enqueues the addends of `width` columns of R randomizer coefficients each
// (device r[col*R + k]) on st; *buf (pool memory on st) is the caller's to free.
int build_rand_add(const uint64_t* d_r, size_t R, size_t width, int logn, int le, uint64_t t, uint64_t o,
                   bool truncate, cudaStream_t st, uint64_t** buf, RandAdd* ra) {
    *buf = nullptr;
    *ra = RandAdd{};
    if (R == 0 || width == 0) return TVMC_OK;
    const int rm = rand_rows(logn, R);
    const size_t N = size_t(1) << logn, L = N << le;
    CK(dev_malloc_async((void**)buf, width * ((size_t)rm << le) * 8, st));
    const uint64_t tc = t % P, oc = o % P;
    const uint64_t qlen = truncate ? std::min<uint64_t>(N + R, L) : N + R;
    cudaError_t e = launch_rand_addend(d_r, R, width, logn, le, tc, hpow(tc, N), hpow(oc, N), root_of_unity(le),
                                       qlen, *buf, st);
    if (e != cudaSuccess) {
        cudaFreeAsync(*buf, st);
        *buf = nullptr;
        return cuda_fail(e, "randomizer addends");
    }
    ra->add = *buf;
    ra->rm = rm;
    ra->le = le;
    return TVMC_OK;
}

// Coset offset of the LDE plan for trace offset t and evaluation offset o: o / t.
uint64_t plan_offset(uint64_t t, uint64_t o) { return hmul(o % P, hinv(t % P)); }

// LDE/NTT scratch kept per (device, stream) and grown on demand.  Work issued
// on one stream runs in order on the GPU, so commits on a stream can share it,
// and repeated commits allocate no scratch at all: a fresh allocation that had
// to grow the memory pool would stall the host (and the stream behind it)
// while the driver maps memory.  tvmc_release_cached_memory frees them.
struct ScratchSlot {
    uint64_t* p = nullptr;
    size_t words = 0;
    // staging slots: completes when the last kernel reading the buffer is done
    // (the next upload into it waits for this, not for the whole stream)
    cudaEvent_t last_use = nullptr;
};
// kind: 0 = LDE/NTT intermediates, 1 and 2 = the first two upload staging
// buffers (UPLOAD_STAGES in all: stage_kind), 3 = the LDE of commits that
// discard it after hashing, 4 = the multi-table staging buffer.
std::map<std::tuple<int, cudaStream_t, int>, ScratchSlot> g_scratch;  // guarded by g_mu

// *grown (optional) is set when the buffer was (re)allocated by this call, i.e.
// it becomes usable only in stream order on st.
int stream_scratch(cudaStream_t st, size_t words, uint64_t** out, int kind = 0, bool* grown = nullptr) {
    *out = nullptr;
    if (grown) *grown = false;
    if (words == 0) return TVMC_OK;
    int dev;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_mu);
    ScratchSlot& slot = g_scratch[{dev, st, kind}];
    if (slot.words < words) {
        if (slot.p) cudaFreeAsync(slot.p, st);  // ordered after the work that used it
        if (slot.last_use) cudaEventDestroy(slot.last_use);
        slot = ScratchSlot{};
        CK(dev_malloc_async((void**)&slot.p, words * 8, st));
        slot.words = words;
        if (grown) *grown = true;
    }
    *out = slot.p;
    return TVMC_OK;
}

// Commits enqueueing uploads on one stream take turns (the staging buffers and
// their last-use events are per stream); other streams are not held up.
std::map<std::pair<int, cudaStream_t>, std::unique_ptr<std::mutex>> g_upload_mu;  // guarded by g_mu

std::mutex& upload_mutex(cudaStream_t st) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    auto& m = g_upload_mu[{dev, st}];
    if (!m) m = std::make_unique<std::mutex>();
    return *m;
}

// The last-use event of a staging slot: take it (the caller now owns it, or
// gets null) or hand a new one over (the slot then owns it).
cudaEvent_t take_slot_event(cudaStream_t st, int kind) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_scratch.find({dev, st, kind});
    if (it == g_scratch.end()) return nullptr;
    cudaEvent_t ev = it->second.last_use;
    it->second.last_use = nullptr;
    return ev;
}

void give_slot_event(cudaStream_t st, int kind, cudaEvent_t ev) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_scratch.find({dev, st, kind});
    if (it == g_scratch.end()) {
        cudaEventDestroy(ev);
        return;
    }
    if (it->second.last_use) cudaEventDestroy(it->second.last_use);
    it->second.last_use = ev;
}

int run_lde(const LdePlan& pl, const uint64_t* d_tr, uint64_t tld, uint64_t* d_out, uint64_t old, size_t width,
            cudaStream_t st, const RandAdd& ra = RandAdd{}) {
    size_t chunk = lde_chunk_cols(pl.logn, pl.log_exp, width);
    uint64_t* scratch = nullptr;
    int rc = stream_scratch(st, lde_scratch_words(pl.logn, pl.log_exp, chunk), &scratch);
    if (rc) return rc;
    for (size_t c0 = 0; c0 < width; c0 += chunk) {
        size_t nc = std::min(chunk, width - c0);
        cudaError_t e =
            launch_lde(pl, d_tr + c0 * tld, tld, d_out + c0 * old, old, nc, scratch, st, ra.cols(c0), ra.rm);
        if (e != cudaSuccess) return cuda_fail(e, "launch_lde");
    }
    return TVMC_OK;
}

// Per-device non-blocking stream for host->device uploads.
// One non-blocking upload stream per (device, compute stream): the uploads of
// a commit wait on its own compute stream's progress, so commits issued on
// different streams never queue behind each other's uploads.
std::map<std::pair<int, cudaStream_t>, cudaStream_t> g_copy_streams;

int copy_stream(cudaStream_t compute, cudaStream_t* out) {
    int dev;
    int rc = current_device(&dev);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_mu);
    auto key = std::make_pair(dev, compute);
    auto it = g_copy_streams.find(key);
    if (it == g_copy_streams.end()) {
        cudaStream_t s;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        it = g_copy_streams.emplace(key, s).first;
    }
    *out = it->second;
    return TVMC_OK;
}

// Host column-major trace -> device LDE.  Column chunks of about 256 MB are
// staged through UPLOAD_STAGES device buffers per stream: the copy stream uploads
// ahead while `st` runs the LDE of an earlier chunk, and a commit's first
// UPLOAD_STAGES chunks wait only for the previous commit's LDE kernels that read
// those buffers, so they upload during that commit's row hash.  Returns after
// enqueueing; `st` is ordered after every copy.
constexpr int UPLOAD_STAGES = 4;
constexpr int stage_kind(int b) { return b < 2 ? 1 + b : 16 + b; }
int upload_lde_pipelined(const LdePlan& pl, const uint64_t* h_trace, size_t n, size_t width, uint64_t* d_out,
                         size_t L, cudaStream_t st, const RandAdd& ra = RandAdd{}) {
    cudaStream_t cs = nullptr;
    int rc = copy_stream(st, &cs);
    if (rc) return rc;
    size_t chunk = lde_chunk_cols(pl.logn, pl.log_exp, width);
    // keep staging chunks near 256 MB so the first upload is short
    size_t stage_cols = std::max<size_t>(1, (size_t(256) << 20) / (n * 8));
    chunk = std::min(chunk, stage_cols);
    const size_t nchunks = (width + chunk - 1) / chunk;
    std::lock_guard<std::mutex> turn(upload_mutex(st));
    const int nst = (int)std::min<size_t>(UPLOAD_STAGES, nchunks);
    uint64_t *scratch = nullptr, *stage[UPLOAD_STAGES] = {};
    cudaEvent_t ready[UPLOAD_STAGES] = {}, freed[UPLOAD_STAGES] = {}, prev[UPLOAD_STAGES] = {};
    bool used[UPLOAD_STAGES] = {};
    if ((rc = stream_scratch(st, lde_scratch_words(pl.logn, pl.log_exp, chunk), &scratch))) return rc;
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < nst && e == cudaSuccess; b++) {
        bool grown = false;
        if (stream_scratch(st, chunk * n, &stage[b], stage_kind(b), &grown)) e = cudaErrorMemoryAllocation;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&freed[b], cudaEventDisableTiming);
        // The first copy into stage[b] waits for the last kernel that read it (the
        // previous commit's on this stream), so it can overlap that commit's row
        // hash; a freshly allocated buffer is ordered on st instead.
        if (e == cudaSuccess && !grown) prev[b] = take_slot_event(st, stage_kind(b));
        if (e == cudaSuccess && !prev[b]) e = cudaEventRecord(freed[b], st);
    }
    for (size_t k = 0; k < nchunks && e == cudaSuccess; k++) {
        const int b = (int)(k % (size_t)nst);
        const size_t c0 = k * chunk, nc = std::min(chunk, width - c0);
        e = cudaStreamWaitEvent(cs, (!used[b] && prev[b]) ? prev[b] : freed[b], 0);
        used[b] = true;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(stage[b], h_trace + c0 * n, nc * n * 8, cudaMemcpyHostToDevice, cs);
        if (e == cudaSuccess) e = cudaEventRecord(ready[b], cs);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ready[b], 0);
        if (e == cudaSuccess) e = launch_lde(pl, stage[b], n, d_out + c0 * L, L, nc, scratch, st, ra.cols(c0), ra.rm);
        if (e == cudaSuccess) e = cudaEventRecord(freed[b], st);
    }
    for (int b = 0; b < nst; b++) {
        if (ready[b]) cudaEventDestroy(ready[b]);  // destruction is deferred until the event completes
        if (e == cudaSuccess && used[b]) {
            give_slot_event(st, stage_kind(b), freed[b]);  // recorded after the last kernel reading stage[b]
            if (prev[b]) cudaEventDestroy(prev[b]);
        } else {
            if (freed[b]) cudaEventDestroy(freed[b]);
            if (prev[b]) give_slot_event(st, stage_kind(b), prev[b]);  // still the guard for that buffer
        }
    }
    if (e != cudaSuccess) return cuda_fail(e, "pipelined upload/LDE");
    return TVMC_OK;
}

int ntt_impl(uint64_t* d, size_t n, size_t cols, int inverse, cudaStream_t st) {
    if (!is_pow2(n)) return fail(TVMC_ERR_INVALID, "NTT size must be a power of 2 (got %zu)", n);
    int l = log2u(n);
    if (l > MAX_LOG_NTT) return fail(TVMC_ERR_UNSUPPORTED, "NTT size 2^%d exceeds 2^%d", l, MAX_LOG_NTT);
    if (cols == 0) return TVMC_OK;
    LdePlan pl;
    int rc = get_plan(l, -1, 0, &pl);
    if (rc) return rc;
    uint64_t* scratch = nullptr;
    if ((rc = stream_scratch(st, ntt_scratch_words(l, cols), &scratch))) return rc;
    cudaError_t e = launch_ntt(pl, inverse, d, n, cols, scratch, st);
    if (e != cudaSuccess) return cuda_fail(e, "launch_ntt");
    return TVMC_OK;
}

// RAII device buffer for host-API calls.
struct DBuf {
    uint64_t* p = nullptr;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t words) { return dev_malloc((void**)&p, words ? words * 8 : 8); }
};

// Per-thread, per-device device buffer reused by the host-buffer entry points,
// so frequent small calls (one permutation, one path) pay no cudaMalloc/cudaFree.
// Requests above 2^24 words get a buffer of their own instead.
struct HostScratch {
    std::map<int, std::pair<uint64_t*, size_t>> buf;
    ~HostScratch() {
        for (auto& kv : buf)
            if (kv.second.first) cudaFree(kv.second.first);
    }
};
thread_local HostScratch t_scratch;

struct HostBuf {
    uint64_t* p = nullptr;
    DBuf own;
};

int host_buf(size_t words, HostBuf* hb) {
    if (words > (size_t(1) << 24)) {
        CK(hb->own.alloc(words));
        hb->p = hb->own.p;
        return TVMC_OK;
    }
    int dev;
    CK(cudaGetDevice(&dev));
    auto& b = t_scratch.buf[dev];
    if (b.second < words) {
        if (b.first) cudaFree(b.first);
        b = {nullptr, 0};
        const size_t cap = std::max(words, size_t(1) << 16);
        CK(dev_malloc((void**)&b.first, cap * 8));
        b.second = cap;
    }
    hb->p = b.first;
    return TVMC_OK;
}

// Per-thread, per-device non-blocking stream for the small synchronous reads
// (openings): they neither queue behind other streams' commits nor, having no
// cudaFree, stall the device.
struct AccStreams {
    std::map<int, cudaStream_t> s;
    ~AccStreams() {
        for (auto& kv : s) cudaStreamDestroy(kv.second);
    }
};
thread_local AccStreams t_acc;

int acc_stream(cudaStream_t* out) {
    int dev;
    CK(cudaGetDevice(&dev));
    auto it = t_acc.s.find(dev);
    if (it == t_acc.s.end()) {
        // the greatest priority: an opening's small gather kernel is dispatched
        // ahead of the remaining CTAs of the commits filling the GPU
        int lo = 0, hi = 0;
        CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        cudaStream_t st;
        CK(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, hi));
        it = t_acc.s.emplace(dev, st).first;
    }
    *out = it->second;
    return TVMC_OK;
}

// TVMC_FRUGAL commit: the LDE is produced stripe by stripe (10-column aligned)
// and each stripe is absorbed at once into the per-row sponge capacity state,
// so only one stripe of LDE (plus 48 bytes of state per row) is ever resident.
// Leaves go straight into the heap tree `nodes`, which the last stripe completes.
int commit_frugal(const LdePlan& pl, const uint64_t* trace, bool dev, bool rm, size_t n, size_t width, size_t L,
                  uint64_t* nodes, cudaStream_t st, cudaEvent_t* prof, const RandAdd& ra) {
    const size_t NW = n * width;
    const uint64_t* src = trace;
    uint64_t *up = nullptr, *cm = nullptr, *cap = nullptr, *stripe = nullptr, *scratch = nullptr;
    cudaError_t e = cudaSuccess;
    if (width && !dev) {
        e = dev_malloc_async((void**)&up, NW * 8, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(up, trace, NW * 8, cudaMemcpyHostToDevice, st);
        src = up;
    }
    if (e == cudaSuccess && width && rm) {
        e = dev_malloc_async((void**)&cm, NW * 8, st);
        if (e == cudaSuccess) e = launch_transpose(src, width, cm, n, n, width, st);
        src = cm;
    }
    if (prof) cudaEventRecord(prof[1], st);
    // stripe width: a multiple of 10 columns whose LDE fits the knob or 2 GiB
    size_t sc = g_tune_stripe_cols.load() > 0 ? (size_t)g_tune_stripe_cols.load()
                                                : ((size_t(2) << 30) / (L * 8)) / 10 * 10;
    sc = std::max<size_t>(10, sc / 10 * 10);
    const size_t stripe_cols = std::min(sc, std::max<size_t>(width, 1));
    const size_t chunk = std::min(lde_chunk_cols(pl.logn, pl.log_exp, stripe_cols), stripe_cols);
    if (e == cudaSuccess) e = dev_malloc_async((void**)&cap, 6 * L * 8, st);
    if (e == cudaSuccess && width) e = dev_malloc_async((void**)&stripe, stripe_cols * L * 8, st);
    if (e == cudaSuccess && stream_scratch(st, lde_scratch_words(pl.logn, pl.log_exp, chunk), &scratch))
        e = cudaErrorMemoryAllocation;
    size_t c0 = 0;
    bool first = true;
    while (e == cudaSuccess) {
        const size_t nc = std::min(sc, width - c0);
        const bool last = c0 + nc == width;
        for (size_t k = 0; k < nc && e == cudaSuccess; k += chunk) {
            const size_t kc = std::min(chunk, nc - k);
            e = launch_lde(pl, src + (c0 + k) * n, n, stripe + k * L, L, kc, scratch, st, ra.cols(c0 + k), ra.rm);
        }
        if (e == cudaSuccess) e = launch_absorb_stripe(stripe, L, (uint32_t)nc, cap, first, last, nodes, st);
        first = false;
        c0 += nc;
        if (last) break;
    }
    for (uint64_t* p : {up, cm, cap, stripe})
        if (p) cudaFreeAsync(p, st);
    if (prof) cudaEventRecord(prof[2], st);
    if (e != cudaSuccess) return cuda_fail(e, "frugal commit");
    return TVMC_OK;
}

// Needed-minus-computable node set of a batch of leaf paths, descending.
int auth_structure_nodes(size_t n, const size_t* leaf_idx, size_t count, std::vector<uint64_t>* res) {
    std::vector<uint64_t> path, need;
    for (size_t q = 0; q < count; q++) {
        if (leaf_idx[q] >= n) return fail(TVMC_ERR_RANGE, "Leaf index %zu out of range", leaf_idx[q]);
        for (uint64_t i = n + leaf_idx[q]; i > 1; i >>= 1) {
            path.push_back(i);
            need.push_back(i ^ 1);
        }
    }
    std::sort(path.begin(), path.end());
    path.erase(std::unique(path.begin(), path.end()), path.end());
    std::sort(need.begin(), need.end());
    need.erase(std::unique(need.begin(), need.end()), need.end());
    res->clear();
    std::set_difference(need.begin(), need.end(), path.begin(), path.end(), std::back_inserter(*res));
    std::reverse(res->begin(), res->end());
    return TVMC_OK;
}

}  // namespace

int tvmc::check_lde_sizes(size_t trace_len, size_t extended_len, int* logn, int* le) {
    if (!is_pow2(trace_len)) return fail(TVMC_ERR_INVALID, "trace length %zu is not a power of 2", trace_len);
    if (!is_pow2(extended_len) || extended_len < trace_len)
        return fail(TVMC_ERR_INVALID, "extended length %zu is not a power of 2 >= trace length", extended_len);
    *logn = log2u(trace_len);
    *le = log2u(extended_len) - *logn;
    if (*logn > MAX_LOG_LDE_TRACE)
        return fail(TVMC_ERR_UNSUPPORTED, "LDE trace length 2^%d exceeds 2^%d", *logn, MAX_LOG_LDE_TRACE);
    if (*le > 4) return fail(TVMC_ERR_UNSUPPORTED, "expansion factor 2^%d exceeds 16", *le);
    return TVMC_OK;
}

int tvmc::set_error(int code, const char* msg) {
    g_err = msg;
    return code;
}

struct tvmc_commitment {
    int device = 0;
    cudaStream_t stream = nullptr;
    size_t n = 0, width = 0, L = 0;
    uint64_t* d_lde = nullptr;
    uint64_t* d_nodes = nullptr;
    cudaEvent_t done = nullptr;
    // TVMC_PROFILE: events at start / after upload / after LDE / after hash+tree
    cudaEvent_t prof[4] = {nullptr, nullptr, nullptr, nullptr};
    bool batch_owned = false;  // freed by tvmc_batch_free only
    bool pooled = false;       // buffers from cudaMallocAsync on `stream`
    bool lde_borrowed = false; // d_lde is the stream's cached buffer (TVMC_DISCARD_LDE), not owned
};

namespace {
void destroy_commitment(tvmc_commitment* c) {
    if (c->pooled) {
        // ordered after the commitment's own work on its stream; the host does not wait
        if (c->d_lde && !c->lde_borrowed) cudaFreeAsync(c->d_lde, c->stream);
        if (c->d_nodes) cudaFreeAsync(c->d_nodes, c->stream);
        if (c->done) cudaEventDestroy(c->done);
    } else {
        if (c->done) {
            cudaEventSynchronize(c->done);
            cudaEventDestroy(c->done);
        } else {
            cudaStreamSynchronize(c->stream);
        }
        if (c->d_lde) cudaFree(c->d_lde);
        if (c->d_nodes) cudaFree(c->d_nodes);
    }
    for (auto ev : c->prof)
        if (ev) cudaEventDestroy(ev);
    delete c;
}
std::atomic<long long> g_tune_batch_streams{0};
std::atomic<long long> g_tune_batch_multi{0};  // 0 / 1: multi-table hash; 2: per-table hash
std::atomic<long long> g_tune_mid_ctas{0};
std::atomic<long long> g_tune_unfused_tree{0};
}  // namespace

std::atomic<long long> g_tune_mid_variant{0};
// Defaults from an A/B of every combination on 64 columns of 2^20 rows (B200):
// the table-sharing variant at 3 CTAs/SM was fastest (7.56 ms against 7.71 ms
// for the per-coset variant and 8.19 ms at 2 CTAs/SM).
int tvmc::tuning_lde_mid_ctas() { return g_tune_mid_ctas.load() == 2 ? 2 : 3; }
int tvmc::tuning_lde_mid_variant() { return g_tune_mid_variant.load() == 1 ? 1 : 2; }
std::atomic<long long> g_tune_transpose_tma{0};
bool tvmc::tuning_transpose_tma() { return g_tune_transpose_tma.load() == 1; }
std::atomic<long long> g_tune_split_l1{0};
std::atomic<long long> g_tune_tile_log{0};
int tvmc::tuning_lde_split_l1() { return (int)g_tune_split_l1.load(); }
int tvmc::tuning_ntt_tile_log() {
    const long long v = g_tune_tile_log.load();
    return v >= 11 && v <= 15 ? (int)v : 13;
}
int tvmc::tuning_hash_fuse_levels() { return g_tune_unfused_tree.load() ? 0 : 8; }

struct tvmc_batch {
    int device = 0;
    std::vector<tvmc_table_shape> shapes;
    std::vector<tvmc_commitment*> tables;  // batch-owned handles (LDE + tree)
    std::vector<uint64_t*> inputs;         // per-table device trace buffers
    std::vector<uint64_t*> scratch;        // per-worker LDE scratch
    std::vector<cudaStream_t> workers;
    std::vector<cudaEvent_t> events;       // fork + one join per worker
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long kernels_per_run = 0;
    bool counted = false;  // holds a DevTables::live_batches count
};

namespace {
// Index list -> device, a gather kernel, result -> host, all on the calling
// thread's accessor stream after the commitment's completion event; per_item
// output words per index.
template <typename Gather>
int gather_sync(const tvmc_commitment* c, const void* idx, size_t count, size_t per_item, uint64_t* out,
                Gather gather) {
    static_assert(sizeof(size_t) == 8, "64-bit indices");
    cudaStream_t st;
    int rc = acc_stream(&st);
    if (rc) return rc;
    HostBuf hb;
    if ((rc = host_buf(count * (1 + per_item), &hb))) return rc;
    uint64_t *di = hb.p, *dout = hb.p + count;
    CK(cudaStreamWaitEvent(st, c->done, 0));
    CK(cudaMemcpyAsync(di, idx, count * 8, cudaMemcpyHostToDevice, st));
    CK(gather(di, dout, st));
    CK(cudaMemcpyAsync(out, dout, count * per_item * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return TVMC_OK;
}

// Device words -> host after the commitment's completion, on the accessor stream.
int read_sync(const tvmc_commitment* c, const uint64_t* src, size_t words, uint64_t* out) {
    cudaStream_t st;
    int rc = acc_stream(&st);
    if (rc) return rc;
    CK(cudaStreamWaitEvent(st, c->done, 0));
    CK(cudaMemcpyAsync(out, src, words * 8, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return TVMC_OK;
}
}  // namespace

extern "C" {

const char* tvmc_last_error(void) { return g_err.c_str(); }

const char* tvmc_status_string(int s) {
    switch (s) {
        case TVMC_OK: return "ok";
        case TVMC_ERR_INVALID: return "invalid argument";
        case TVMC_ERR_RANGE: return "index out of range";
        case TVMC_ERR_NOMEM: return "out of device memory";
        case TVMC_ERR_CUDA: return "CUDA error";
        case TVMC_ERR_TIMEOUT: return "device wait timed out";
        case TVMC_ERR_UNSUPPORTED: return "unsupported size";
        default: return "unknown status";
    }
}

int tvmc_version(void) { return 1; }

unsigned long long tvmc_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int tvmc_forget_stream(void* stream) {
    cudaStream_t st = as_stream(stream);
    int dev;
    CK(cudaGetDevice(&dev));
    cudaStream_t cs = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (auto it = g_scratch.begin(); it != g_scratch.end();) {
            if (std::get<0>(it->first) == dev && std::get<1>(it->first) == st) {
                if (it->second.p) cudaFreeAsync(it->second.p, st);  // after the stream's queued work
                if (it->second.last_use) cudaEventDestroy(it->second.last_use);
                it = g_scratch.erase(it);
            } else {
                ++it;
            }
        }
        auto c = g_copy_streams.find({dev, st});
        if (c != g_copy_streams.end()) {
            cs = c->second;
            g_copy_streams.erase(c);
        }
        g_upload_mu.erase({dev, st});
    }
    if (cs) {
        CK(cudaStreamSynchronize(cs));
        CK(cudaStreamDestroy(cs));
    }
    return TVMC_OK;
}

int tvmc_release_cached_memory(void) {
    int dev;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceSynchronize());
    {
        std::lock_guard<std::mutex> lk(g_mu);
        for (auto it = g_scratch.begin(); it != g_scratch.end();) {
            if (std::get<0>(it->first) == dev) {
                if (it->second.p) cudaFree(it->second.p);
                if (it->second.last_use) cudaEventDestroy(it->second.last_use);
                it = g_scratch.erase(it);
            } else {
                ++it;
            }
        }
        // The twiddle and coset-scale tables: one set per (size, expansion, offset)
        // ever used, so randomized LDEs with many distinct offsets would otherwise
        // keep growing them.  They are rebuilt on the next use.
        auto t = g_dev.find(dev);
        if (t != g_dev.end() && t->second.live_batches == 0) {
            DevTables& T = t->second;
            for (auto* m : {&T.wn_f, &T.wn_i})
                for (auto& kv : *m) {
                    cudaFree(kv.second.first);
                    cudaFree(kv.second.second);
                }
            for (auto& kv : T.sc) {
                cudaFree(kv.second.first);
                cudaFree(kv.second.second);
            }
            T.wn_f.clear();
            T.wn_i.clear();
            T.sc.clear();
        }
    }
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, dev));
    CK(cudaMemPoolTrimTo(pool, 0));
    return TVMC_OK;
}

int tvmc_set_tuning(const char* key, long long value) {
    if (!key) return fail(TVMC_ERR_INVALID, "null tuning key");
    if (value < 0) return fail(TVMC_ERR_INVALID, "tuning value must be >= 0");
    if (!strcmp(key, "frugal_stripe_cols")) g_tune_stripe_cols = value;
    else if (!strcmp(key, "lde_scratch_bytes")) g_tune_scratch_bytes = value;
    else if (!strcmp(key, "batch_streams")) g_tune_batch_streams = value;
    else if (!strcmp(key, "lde_mid_ctas")) {
        if (value != 0 && value != 2 && value != 3) return fail(TVMC_ERR_INVALID, "lde_mid_ctas must be 0, 2 or 3");
        g_tune_mid_ctas = value;
    } else if (!strcmp(key, "lde_mid_variant")) {
        if (value > 2) return fail(TVMC_ERR_INVALID, "lde_mid_variant must be 0, 1 or 2");
        g_tune_mid_variant = value;
    } else if (!strcmp(key, "transpose_tma")) {
        if (value > 2) return fail(TVMC_ERR_INVALID, "transpose_tma must be 0, 1 or 2");
        g_tune_transpose_tma = value;
    } else if (!strcmp(key, "batch_multi_hash")) {
        if (value > 2) return fail(TVMC_ERR_INVALID, "batch_multi_hash must be 0, 1 or 2");
        g_tune_batch_multi = value;
    } else if (!strcmp(key, "lde_split_l1")) {
        if (value > 12) return fail(TVMC_ERR_INVALID, "lde_split_l1 must be 0 .. 12");
        g_tune_split_l1 = value;
    } else if (!strcmp(key, "ntt_tile_log")) {
        if (value != 0 && (value < 11 || value > 15)) return fail(TVMC_ERR_INVALID, "ntt_tile_log must be 0 or 11 .. 15");
        g_tune_tile_log = value;
    } else if (!strcmp(key, "hash_unfused_tree")) g_tune_unfused_tree = value ? 1 : 0;
    else if (!strcmp(key, "fail_alloc_after")) g_fail_alloc_after = value;
    else return fail(TVMC_ERR_INVALID, "unknown tuning key '%s'", key);
    return TVMC_OK;
}

int tvmc_get_tuning(const char* key, long long* value) {
    if (!key || !value) return fail(TVMC_ERR_INVALID, "null argument");
    if (!strcmp(key, "frugal_stripe_cols")) *value = g_tune_stripe_cols;
    else if (!strcmp(key, "lde_scratch_bytes")) *value = g_tune_scratch_bytes;
    else if (!strcmp(key, "batch_streams")) *value = g_tune_batch_streams;
    else if (!strcmp(key, "lde_mid_ctas")) *value = g_tune_mid_ctas;
    else if (!strcmp(key, "hash_unfused_tree")) *value = g_tune_unfused_tree;
    else if (!strcmp(key, "lde_mid_variant")) *value = g_tune_mid_variant;
    else if (!strcmp(key, "lde_split_l1")) *value = g_tune_split_l1;
    else if (!strcmp(key, "batch_multi_hash")) *value = g_tune_batch_multi;
    else if (!strcmp(key, "transpose_tma")) *value = g_tune_transpose_tma;
    else if (!strcmp(key, "tma_timeouts")) *value = (long long)tma_timeouts();
    else if (!strcmp(key, "ntt_tile_log")) *value = g_tune_tile_log;
    else if (!strcmp(key, "fail_alloc_after")) *value = g_fail_alloc_after;
    else if (!strcmp(key, "pool_used_bytes")) {
        int dev;
        cudaMemPool_t pool;
        size_t used = 0;
        CK(cudaGetDevice(&dev));
        CK(cudaDeviceGetDefaultMemPool(&pool, dev));
        CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
        *value = (long long)used;
    } else return fail(TVMC_ERR_INVALID, "unknown tuning key '%s'", key);
    return TVMC_OK;
}

int tvmc_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

// ---------------------------------------------------------------- NTT

int tvmc_ntt_forward_batched_gpu(uint64_t* d_data, size_t n, size_t num_cols, void* stream) {
    return ntt_impl(d_data, n, num_cols, 0, as_stream(stream));
}
int tvmc_ntt_inverse_batched_gpu(uint64_t* d_data, size_t n, size_t num_cols, void* stream) {
    return ntt_impl(d_data, n, num_cols, 1, as_stream(stream));
}

int tvmc_ntt_host(uint64_t* data, size_t n, size_t num_cols, int inverse) {
    if (!is_pow2(n)) return fail(TVMC_ERR_INVALID, "NTT size must be a power of 2 (got %zu)", n);
    DBuf d;
    CK(d.alloc(n * num_cols));
    CK(cudaMemcpy(d.p, data, n * num_cols * 8, cudaMemcpyHostToDevice));
    int rc = ntt_impl(d.p, n, num_cols, inverse, nullptr);
    if (rc) return rc;
    CK(cudaMemcpy(data, d.p, n * num_cols * 8, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_evaluate_on_coset_gpu(const uint64_t* d_coeffs, size_t num_coeffs, size_t num_cols, uint64_t* d_out,
                               size_t domain_len, uint64_t offset, void* stream) {
    if (!is_pow2(domain_len)) return fail(TVMC_ERR_INVALID, "NTT size must be a power of 2 (got %zu)", domain_len);
    if (log2u(domain_len) > MAX_LOG_NTT)
        return fail(TVMC_ERR_UNSUPPORTED, "NTT size 2^%d exceeds 2^%d", log2u(domain_len), MAX_LOG_NTT);
    if (num_cols == 0) return TVMC_OK;
    cudaStream_t st = as_stream(stream);
    CK(launch_coset_scale(d_coeffs, num_coeffs, num_coeffs, d_out, domain_len, num_cols, offset, st));
    return ntt_impl(d_out, domain_len, num_cols, 0, st);
}

int tvmc_evaluate_on_coset_host(const uint64_t* coeffs, size_t num_coeffs, size_t num_cols, uint64_t* out,
                                size_t domain_len, uint64_t offset) {
    if (!is_pow2(domain_len)) return fail(TVMC_ERR_INVALID, "NTT size must be a power of 2 (got %zu)", domain_len);
    if (num_cols == 0) return TVMC_OK;
    HostBuf hb;
    int rc = host_buf(num_cols * (num_coeffs + domain_len), &hb);
    if (rc) return rc;
    uint64_t *a = hb.p, *b = a + num_cols * num_coeffs;
    if (num_coeffs) CK(cudaMemcpy(a, coeffs, 8 * num_cols * num_coeffs, cudaMemcpyHostToDevice));
    if ((rc = tvmc_evaluate_on_coset_gpu(a, num_coeffs, num_cols, b, domain_len, offset, nullptr))) return rc;
    CK(cudaMemcpy(out, b, 8 * num_cols * domain_len, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_rowmajor_to_colmajor_gpu(const uint64_t* d_in, size_t rows, size_t cols, uint64_t* d_out, void* stream) {
    if ((rows && cols) && (!d_in || !d_out)) return fail(TVMC_ERR_INVALID, "null argument");
    if (d_in == d_out && rows && cols) return fail(TVMC_ERR_INVALID, "the transpose is out of place");
    CK(launch_transpose(d_in, cols, d_out, rows, rows, cols, as_stream(stream)));
    return TVMC_OK;
}

// ---------------------------------------------------------------- LDE

int tvmc_lde_batch_gpu(const uint64_t* d_traces, size_t num_columns, size_t trace_len, uint64_t* d_extended,
                       size_t extended_len, uint64_t trace_offset, uint64_t extended_offset, void* stream) {
    (void)trace_offset;
    int logn, le;
    int rc = check_lde_sizes(trace_len, extended_len, &logn, &le);
    if (rc) return rc;
    if (num_columns == 0) return TVMC_OK;
    LdePlan pl;
    if ((rc = get_plan(logn, le, extended_offset, &pl))) return rc;
    return run_lde(pl, d_traces, trace_len, d_extended, extended_len, num_columns, as_stream(stream));
}

int tvmc_lde_host(const uint64_t* traces, size_t num_columns, size_t trace_len, uint64_t* extended,
                  size_t extended_len, uint64_t extended_offset) {
    int logn, le;
    int rc = check_lde_sizes(trace_len, extended_len, &logn, &le);
    if (rc) return rc;
    if (num_columns == 0) return TVMC_OK;
    DBuf a, b;
    CK(a.alloc(trace_len * num_columns));
    CK(b.alloc(extended_len * num_columns));
    CK(cudaMemcpy(a.p, traces, trace_len * num_columns * 8, cudaMemcpyHostToDevice));
    if ((rc = tvmc_lde_batch_gpu(a.p, num_columns, trace_len, b.p, extended_len, 1, extended_offset, nullptr)))
        return rc;
    CK(cudaMemcpy(extended, b.p, extended_len * num_columns * 8, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_lde_randomized_gpu(const uint64_t* d_traces, size_t num_columns, size_t trace_len,
                            const uint64_t* d_randomizers, size_t num_randomizers, uint64_t* d_extended,
                            size_t extended_len, uint64_t trace_offset, uint64_t extended_offset, uint32_t flags,
                            void* stream) {
    int logn, le;
    int rc = check_lde_sizes(trace_len, extended_len, &logn, &le);
    if (rc) return rc;
    if (flags & ~(uint32_t)TVMC_RAND_TRUNCATE) return fail(TVMC_ERR_INVALID, "unknown flag bits 0x%x", flags);
    if (trace_offset % P == 0) return fail(TVMC_ERR_INVALID, "trace offset must be nonzero mod p");
    if (num_columns == 0) return TVMC_OK;
    if (num_randomizers && !d_randomizers) return fail(TVMC_ERR_INVALID, "null randomizers");
    cudaStream_t st = as_stream(stream);
    LdePlan pl;
    if ((rc = get_plan(logn, le, plan_offset(trace_offset, extended_offset), &pl))) return rc;
    uint64_t* d_add = nullptr;
    RandAdd ra;
    rc = build_rand_add(d_randomizers, num_randomizers, num_columns, logn, le, trace_offset, extended_offset,
                        flags & TVMC_RAND_TRUNCATE, st, &d_add, &ra);
    if (rc) return rc;
    rc = run_lde(pl, d_traces, trace_len, d_extended, extended_len, num_columns, st, ra);
    if (d_add) cudaFreeAsync(d_add, st);
    return rc;
}

int tvmc_lde_randomized_host(const uint64_t* traces, size_t num_columns, size_t trace_len,
                             const uint64_t* randomizers, size_t num_randomizers, uint64_t* extended,
                             size_t extended_len, uint64_t trace_offset, uint64_t extended_offset, uint32_t flags) {
    int logn, le;
    int rc = check_lde_sizes(trace_len, extended_len, &logn, &le);
    if (rc) return rc;
    if (num_columns == 0) return TVMC_OK;
    if (num_randomizers && !randomizers) return fail(TVMC_ERR_INVALID, "null randomizers");
    DBuf a, b, r;
    CK(a.alloc(trace_len * num_columns));
    CK(b.alloc(extended_len * num_columns));
    CK(r.alloc(num_randomizers * num_columns));
    CK(cudaMemcpy(a.p, traces, trace_len * num_columns * 8, cudaMemcpyHostToDevice));
    if (num_randomizers) CK(cudaMemcpy(r.p, randomizers, num_randomizers * num_columns * 8, cudaMemcpyHostToDevice));
    rc = tvmc_lde_randomized_gpu(a.p, num_columns, trace_len, r.p, num_randomizers, b.p, extended_len, trace_offset,
                                 extended_offset, flags, nullptr);
    if (rc) return rc;
    CK(cudaMemcpy(extended, b.p, extended_len * num_columns * 8, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

// ---------------------------------------------------------------- Tip5

int tvmc_hash_bfield_rows_gpu(const uint64_t* d_table, size_t num_rows, size_t num_cols, uint64_t* d_digests,
                              void* stream) {
    CK(launch_hash_rows(d_table, 1, num_rows, num_rows, (uint32_t)num_cols, d_digests, nullptr, LAYOUT_HEAP,
                        as_stream(stream)));
    return TVMC_OK;
}

int tvmc_hash_xfield_rows_gpu(const uint64_t* d_table, size_t num_rows, size_t num_xfe_cols,
                              uint64_t* d_digests, void* stream) {
    return tvmc_hash_bfield_rows_gpu(d_table, num_rows, 3 * num_xfe_cols, d_digests, stream);
}

int tvmc_hash_varlen_host(const uint64_t* rows, size_t num_rows, size_t row_len, uint64_t* digests) {
    if (num_rows == 0) return TVMC_OK;
    DBuf a, b;
    CK(a.alloc(num_rows * row_len));
    CK(b.alloc(num_rows * 5));
    if (row_len) CK(cudaMemcpy(a.p, rows, num_rows * row_len * 8, cudaMemcpyHostToDevice));
    CK(launch_hash_rows(a.p, row_len, 1, num_rows, (uint32_t)row_len, b.p, nullptr, LAYOUT_HEAP, nullptr));
    CK(cudaMemcpy(digests, b.p, num_rows * 40, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_hash_pairs_gpu(const uint64_t* d_left, const uint64_t* d_right, uint64_t* d_out, size_t count,
                        void* stream) {
    CK(launch_hash_pairs(d_left, d_right, d_out, count, as_stream(stream)));
    return TVMC_OK;
}

int tvmc_hash_pairs_host(const uint64_t* left, const uint64_t* right, uint64_t* out, size_t count) {
    if (count == 0) return TVMC_OK;
    HostBuf hb;
    int rc = host_buf(15 * count, &hb);
    if (rc) return rc;
    uint64_t *a = hb.p, *b = a + 5 * count, *c = b + 5 * count;
    CK(cudaMemcpy(a, left, 40 * count, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b, right, 40 * count, cudaMemcpyHostToDevice));
    CK(launch_hash_pairs(a, b, c, count, nullptr));
    CK(cudaMemcpy(out, c, 40 * count, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_tip5_permutation_batch_gpu(uint64_t* d_states, size_t num_states, void* stream) {
    CK(launch_tip5_permutations(d_states, num_states, as_stream(stream)));
    return TVMC_OK;
}

int tvmc_tip5_permutation_batch_host(uint64_t* states, size_t num_states) {
    if (num_states == 0) return TVMC_OK;
    HostBuf a;
    int rc = host_buf(16 * num_states, &a);
    if (rc) return rc;
    CK(cudaMemcpy(a.p, states, 128 * num_states, cudaMemcpyHostToDevice));
    CK(launch_tip5_permutations(a.p, num_states, nullptr));
    CK(cudaMemcpy(states, a.p, 128 * num_states, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_tip5_rounds_host(uint64_t* states, size_t num_states, uint32_t first_round, uint32_t num_rounds,
                          uint64_t* trace) {
    if (first_round > 5 || num_rounds > 5 - first_round)
        return fail(TVMC_ERR_INVALID, "rounds [%u, %u) outside [0, 5)", first_round, first_round + num_rounds);
    if (num_states == 0 || num_rounds == 0) return TVMC_OK;
    HostBuf a;
    int rc = host_buf(16 * num_states * (1 + (trace ? num_rounds : 0)), &a);
    if (rc) return rc;
    uint64_t* d_trace = trace ? a.p + 16 * num_states : nullptr;
    CK(cudaMemcpy(a.p, states, 128 * num_states, cudaMemcpyHostToDevice));
    CK(launch_tip5_rounds(a.p, num_states, (int)first_round, (int)num_rounds, d_trace, nullptr));
    CK(cudaMemcpy(states, a.p, 128 * num_states, cudaMemcpyDeviceToHost));
    if (trace) CK(cudaMemcpy(trace, d_trace, 128 * num_states * num_rounds, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_tip5_parameters(uint8_t* lookup_table, uint64_t* mds_first_column, uint64_t* round_constants) {
    static const uint64_t rc[80] = {TVMC_T5_ROUND_CONSTANTS};
    static const uint64_t mds[16] = {TVMC_T5_MDS_FIRST_COLUMN};
    if (lookup_table)
        for (uint32_t i = 0; i < 256; i++) {
            const uint32_t x = i + 1;  // offset Fermat cube map: (i + 1)^3 - 1 mod 257
            lookup_table[i] = (uint8_t)((x * x % 257 * x % 257 + 256) % 257);
        }
    if (mds_first_column) std::memcpy(mds_first_column, mds, sizeof mds);
    if (round_constants) std::memcpy(round_constants, rc, sizeof rc);
    return TVMC_OK;
}

// ---------------------------------------------------------------- Merkle

int tvmc_merkle_tree_gpu(const uint64_t* d_leaves, uint64_t* d_tree, size_t num_leaves, void* stream) {
    if (!is_pow2(num_leaves))
        return fail(TVMC_ERR_INVALID, "Number of leaves must be a power of 2 (got %zu)", num_leaves);
    CK(launch_merkle_tree(d_leaves, d_tree, num_leaves, LAYOUT_FLAT, as_stream(stream)));
    return TVMC_OK;
}

int tvmc_merkle_root_gpu(const uint64_t* d_leaves, uint64_t* d_root, size_t num_leaves, void* stream) {
    if (!is_pow2(num_leaves))
        return fail(TVMC_ERR_INVALID, "Number of leaves must be a power of 2 (got %zu)", num_leaves);
    cudaStream_t st = as_stream(stream);
    uint64_t* tree = nullptr;
    CK(dev_malloc_async((void**)&tree, (2 * num_leaves - 1) * 40, st));
    cudaError_t e = launch_merkle_tree(d_leaves, tree, num_leaves, LAYOUT_FLAT, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_root, tree + 5 * (2 * num_leaves - 2), 40, cudaMemcpyDeviceToDevice, st);
    cudaFreeAsync(tree, st);
    if (e != cudaSuccess) return cuda_fail(e, "merkle_root");
    return TVMC_OK;
}

int tvmc_merkle_root_from_paths_gpu(const size_t* d_leaf_idx, const uint64_t* d_leaves, const uint64_t* d_paths,
                                    size_t count, size_t path_len, uint64_t* d_roots, void* stream) {
    static_assert(sizeof(size_t) == sizeof(uint64_t), "64-bit size_t");
    CK(launch_root_from_paths(reinterpret_cast<const uint64_t*>(d_leaf_idx), d_leaves, d_paths, count, path_len,
                              d_roots, as_stream(stream)));
    return TVMC_OK;
}

int tvmc_merkle_root_from_paths_host(const size_t* leaf_idx, const uint64_t* leaves, const uint64_t* paths,
                                     size_t count, size_t path_len, uint64_t* roots) {
    if (count == 0) return TVMC_OK;
    HostBuf hb;
    int rc = host_buf(count * (11 + 5 * path_len), &hb);
    if (rc) return rc;
    uint64_t *ix = hb.p, *lv = ix + count, *pp = lv + 5 * count, *rt = pp + 5 * count * path_len;
    CK(cudaMemcpy(ix, leaf_idx, 8 * count, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(lv, leaves, 40 * count, cudaMemcpyHostToDevice));
    if (path_len) CK(cudaMemcpy(pp, paths, 40 * count * path_len, cudaMemcpyHostToDevice));
    CK(launch_root_from_paths(ix, lv, pp, count, path_len, rt, nullptr));
    CK(cudaMemcpy(roots, rt, 40 * count, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_merkle_tree_heap_host(const uint64_t* leaves, size_t num_leaves, uint64_t* nodes) {
    if (!is_pow2(num_leaves))
        return fail(TVMC_ERR_INVALID, "Number of leaves must be a power of 2 (got %zu)", num_leaves);
    DBuf a, t;
    CK(a.alloc(5 * num_leaves));
    CK(t.alloc(10 * num_leaves));
    CK(cudaMemcpy(a.p, leaves, 40 * num_leaves, cudaMemcpyHostToDevice));
    CK(cudaMemset(t.p, 0, 40));
    CK(launch_merkle_tree(a.p, t.p, num_leaves, LAYOUT_HEAP, nullptr));
    CK(cudaMemcpy(nodes, t.p, 80 * num_leaves, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

// ---------------------------------------------------------------- commitment

int tvmc_commit(const uint64_t* trace, size_t trace_len, size_t width, uint32_t expansion, uint64_t offset,
                uint32_t flags, void* stream, tvmc_commitment** out) {
    return tvmc_commit_randomized(trace, trace_len, width, expansion, 1, offset, nullptr, 0, flags, stream, out);
}

int tvmc_commit_randomized(const uint64_t* trace, size_t trace_len, size_t width, uint32_t expansion,
                           uint64_t trace_offset, uint64_t offset, const uint64_t* randomizers,
                           size_t num_randomizers, uint32_t flags, void* stream, tvmc_commitment** out) {
    if (!out) return fail(TVMC_ERR_INVALID, "null output handle");
    *out = nullptr;
    if (!is_pow2(expansion) || expansion > 16)
        return fail(TVMC_ERR_INVALID, "expansion factor %u is not a power of 2 <= 16", expansion);
    if (flags & ~(TVMC_TRACE_DEVICE | TVMC_TRACE_ROW_MAJOR | TVMC_DISCARD_LDE | TVMC_SYNC | TVMC_PROFILE |
                  TVMC_FRUGAL | TVMC_RAND_TRUNCATE))
        return fail(TVMC_ERR_INVALID, "unknown flag bits 0x%x", flags);
    int logn, le;
    int rc = check_lde_sizes(trace_len, trace_len * expansion, &logn, &le);
    if (rc) return rc;
    if (width && !trace) return fail(TVMC_ERR_INVALID, "null trace");
    if (trace_offset % P == 0) return fail(TVMC_ERR_INVALID, "trace offset must be nonzero mod p");
    if (width && num_randomizers && !randomizers) return fail(TVMC_ERR_INVALID, "null randomizers");
    cudaStream_t st = as_stream(stream);
    LdePlan pl;
    if ((rc = get_plan(logn, le, plan_offset(trace_offset, offset), &pl))) return rc;

    tvmc_commitment* c = new tvmc_commitment();
    CK(cudaGetDevice(&c->device));
    c->stream = st;
    c->n = trace_len;
    c->width = width;
    c->L = trace_len * expansion;
    auto bail = [&](int code) {
        tvmc_commitment_free(c);
        return code;
    };
    const size_t NW = trace_len * width;
    const bool frugal = flags & TVMC_FRUGAL;
    // stream-ordered pool memory: repeated commits reuse it without page mapping,
    // and freeing a commitment never stalls the device
    c->pooled = true;
    // An LDE that is discarded after hashing lives in the stream's cached buffer
    // (kind 3), so a run of commits of varying sizes does not fragment the pool
    // with multi-GB blocks (a later, larger one would then grow the pool, and the
    // host would stall while the driver maps memory).  Work on the stream runs in
    // order, so the next commit reuses it only after this one's hash.
    c->lde_borrowed = width && !frugal && (flags & TVMC_DISCARD_LDE);
    if (dev_malloc_async((void**)&c->d_nodes, 2 * c->L * 40, st) != cudaSuccess ||
        (width && !frugal &&
         (c->lde_borrowed ? stream_scratch(st, c->L * width, &c->d_lde, 3) != TVMC_OK
                          : dev_malloc_async((void**)&c->d_lde, c->L * width * 8, st) != cudaSuccess))) {
        cudaGetLastError();
        if (c->lde_borrowed) c->d_lde = nullptr;
        return bail(fail(TVMC_ERR_NOMEM, "cannot allocate LDE (%zu x %zu) and tree", c->L, width));
    }
    if (cudaError_t e = cudaMemsetAsync(c->d_nodes, 0, 40, st); e != cudaSuccess) return bail(cuda_fail(e, "memset"));

    // randomizer addends (column-major [col][k], on the trace's side of the bus)
    const size_t R = width ? num_randomizers : 0;
    uint64_t *d_rnd = nullptr, *d_add = nullptr;
    RandAdd ra;
    if (R) {
        const uint64_t* src_r = randomizers;
        if (!(flags & TVMC_TRACE_DEVICE)) {
            cudaError_t e = dev_malloc_async((void**)&d_rnd, width * R * 8, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(d_rnd, randomizers, width * R * 8, cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) {
                if (d_rnd) cudaFreeAsync(d_rnd, st);
                return bail(cuda_fail(e, "randomizer upload"));
            }
            src_r = d_rnd;
        }
        rc = build_rand_add(src_r, R, width, logn, le, trace_offset, offset, flags & TVMC_RAND_TRUNCATE, st, &d_add,
                            &ra);
        if (d_rnd) cudaFreeAsync(d_rnd, st);
        if (rc) return bail(rc);
    }
    // frees the addends (stream-ordered) on every exit from here on
    struct AddGuard {
        uint64_t* p;
        cudaStream_t s;
        ~AddGuard() {
            if (p) cudaFreeAsync(p, s);
        }
    } add_guard{d_add, st};

    const bool prof = flags & TVMC_PROFILE;
    if (prof) {
        for (auto& ev : c->prof)
            if (cudaError_t e = cudaEventCreate(&ev); e != cudaSuccess) return bail(cuda_fail(e, "event"));
        cudaEventRecord(c->prof[0], st);
    }
    const bool dev = flags & TVMC_TRACE_DEVICE, rm = flags & TVMC_TRACE_ROW_MAJOR;
    if (frugal) {
        rc = commit_frugal(pl, trace, dev, rm, trace_len, width, c->L, c->d_nodes, st, prof ? c->prof : nullptr,
                           ra);
        if (rc) return bail(rc);
    } else if (width && !dev && !rm) {
        // host column-major trace: upload column chunks on a copy stream,
        // overlapping the LDE of the previous chunk
        if (prof) cudaEventRecord(c->prof[1], st);
        rc = upload_lde_pipelined(pl, trace, trace_len, width, c->d_lde, c->L, st, ra);
        if (rc) return bail(rc);
    } else if (width) {
        const uint64_t* d_src = trace;
        uint64_t* d_up = nullptr;
        uint64_t* d_cm = nullptr;
        cudaError_t e = cudaSuccess;
        if (!dev) {
            e = dev_malloc_async((void**)&d_up, NW * 8, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(d_up, trace, NW * 8, cudaMemcpyHostToDevice, st);
            d_src = d_up;
        }
        if (e == cudaSuccess && rm) {
            e = dev_malloc_async((void**)&d_cm, NW * 8, st);
            if (e == cudaSuccess) e = launch_transpose(d_src, width, d_cm, trace_len, trace_len, width, st);
            d_src = d_cm;
        }
        if (e != cudaSuccess) {
            if (d_up) cudaFreeAsync(d_up, st);
            if (d_cm) cudaFreeAsync(d_cm, st);
            return bail(cuda_fail(e, "trace upload"));
        }
        if (prof) cudaEventRecord(c->prof[1], st);
        rc = run_lde(pl, d_src, trace_len, c->d_lde, c->L, width, st, ra);
        if (d_up) cudaFreeAsync(d_up, st);
        if (d_cm) cudaFreeAsync(d_cm, st);
        if (rc) return bail(rc);
    } else if (prof) {
        cudaEventRecord(c->prof[1], st);
    }
    if (prof && !frugal) cudaEventRecord(c->prof[2], st);
    if (!frugal) {  // (the frugal stripes already hashed every row and built the tree)
        cudaError_t e =
            launch_hash_rows(c->d_lde, 1, c->L, c->L, (uint32_t)width, nullptr, c->d_nodes, LAYOUT_HEAP, st);
        if (e != cudaSuccess) return bail(cuda_fail(e, "hash/merkle"));
    }
    if (prof) cudaEventRecord(c->prof[3], st);
    if ((flags & TVMC_DISCARD_LDE) && c->d_lde) {
        if (!c->lde_borrowed) cudaFreeAsync(c->d_lde, st);  // stream-ordered after the hash kernel
        c->d_lde = nullptr;
    }
    {
        cudaError_t e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(c->done, st);
        if (e != cudaSuccess) return bail(cuda_fail(e, "event"));
    }
    if (flags & TVMC_SYNC) {
        if (cudaError_t e = cudaEventSynchronize(c->done); e != cudaSuccess) return bail(cuda_fail(e, "sync"));
    }
    *out = c;
    return TVMC_OK;
}

int tvmc_commit_multi(const tvmc_multi_table* tables, size_t count, uint32_t flags, void* stream,
                      tvmc_commitment** out) {
    if (!out || (count && !tables)) return fail(TVMC_ERR_INVALID, "null argument");
    for (size_t i = 0; i < count; i++) out[i] = nullptr;
    if (flags & ~(TVMC_TRACE_DEVICE | TVMC_DISCARD_LDE | TVMC_SYNC))
        return fail(TVMC_ERR_INVALID, "tvmc_commit_multi takes TVMC_TRACE_DEVICE, TVMC_DISCARD_LDE and TVMC_SYNC");
    if (count == 0) return TVMC_OK;
    const bool dev = flags & TVMC_TRACE_DEVICE, discard = flags & TVMC_DISCARD_LDE;
    cudaStream_t st = as_stream(stream);
    std::vector<LdePlan> plans(count);
    size_t stage_words = 0, lde_words = 0;
    for (size_t i = 0; i < count; i++) {
        const tvmc_multi_table& t = tables[i];
        if (!is_pow2(t.expansion) || t.expansion > 16)
            return fail(TVMC_ERR_INVALID, "table %zu: expansion factor %u is not a power of 2 <= 16", i, t.expansion);
        int logn, le;
        int rc = check_lde_sizes(t.trace_len, t.trace_len * t.expansion, &logn, &le);
        if (rc) return rc;
        if (t.width && !t.trace) return fail(TVMC_ERR_INVALID, "table %zu: null trace", i);
        if ((rc = get_plan(logn, le, t.offset, &plans[i]))) return rc;
        stage_words += dev ? 0 : t.trace_len * t.width;
        lde_words += t.trace_len * t.expansion * t.width;
    }
    NvtxRange range("tvmc multi-table commit");
    std::vector<tvmc_commitment*> cs(count, nullptr);
    auto bail = [&](int code) {
        for (auto* c : cs)
            if (c) destroy_commitment(c);
        return code;
    };
    uint64_t *stage = nullptr, *lde_all = nullptr;
    int rc = stream_scratch(st, stage_words, &stage, 4);
    if (!rc && discard) rc = stream_scratch(st, lde_words, &lde_all, 3);
    if (rc) return rc;
    std::vector<MultiHashTable> hjobs;
    size_t so = 0, lo = 0;
    for (size_t i = 0; i < count; i++) {
        const tvmc_multi_table& t = tables[i];
        tvmc_commitment* c = cs[i] = new tvmc_commitment();
        c->device = -1;
        CK(cudaGetDevice(&c->device));
        c->stream = st;
        c->n = t.trace_len;
        c->width = t.width;
        c->L = t.trace_len * t.expansion;
        c->pooled = true;
        if (dev_malloc_async(&c->d_nodes, 2 * c->L * 40, st) != cudaSuccess)
            return bail(fail(TVMC_ERR_NOMEM, "table %zu: cannot allocate the tree of %zu leaves", i, c->L));
        if (cudaError_t e = cudaMemsetAsync(c->d_nodes, 0, 40, st); e != cudaSuccess) return bail(cuda_fail(e, "memset"));
        uint64_t* lde = nullptr;
        if (t.width) {
            if (discard) {
                lde = lde_all + lo;
                lo += c->L * t.width;
            } else {
                if (dev_malloc_async(&c->d_lde, c->L * t.width * 8, st) != cudaSuccess)
                    return bail(fail(TVMC_ERR_NOMEM, "table %zu: cannot allocate its LDE", i));
                lde = c->d_lde;
            }
            const uint64_t* src = t.trace;
            if (!dev) {
                uint64_t* d = stage + so;
                so += t.trace_len * t.width;
                if (cudaError_t e = cudaMemcpyAsync(d, t.trace, t.trace_len * t.width * 8, cudaMemcpyHostToDevice, st);
                    e != cudaSuccess)
                    return bail(cuda_fail(e, "trace upload"));
                src = d;
            }
            if ((rc = run_lde(plans[i], src, t.trace_len, lde, c->L, t.width, st))) return bail(rc);
        }
        hjobs.push_back(MultiHashTable{lde, c->d_nodes, c->L, (uint32_t)t.width});
    }
    if (cudaError_t e = launch_hash_rows_multi(hjobs.data(), (int)hjobs.size(), st); e != cudaSuccess)
        return bail(cuda_fail(e, "multi-table hash/merkle"));
    for (size_t i = 0; i < count; i++) {
        cudaError_t e = cudaEventCreateWithFlags(&cs[i]->done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(cs[i]->done, st);
        if (e != cudaSuccess) return bail(cuda_fail(e, "event"));
    }
    if (flags & TVMC_SYNC) {
        if (cudaError_t e = cudaEventSynchronize(cs[count - 1]->done); e != cudaSuccess) return bail(cuda_fail(e, "sync"));
    }
    for (size_t i = 0; i < count; i++) out[i] = cs[i];
    return TVMC_OK;
}

// Shared tail of the rows/digests commitments: completion event, optional sync.
static int finish_commitment(tvmc_commitment* c, uint32_t flags, tvmc_commitment** out) {
    cudaError_t e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(c->done, c->stream);
    if (e != cudaSuccess) {
        const int rc = cuda_fail(e, "event");
        tvmc_commitment_free(c);
        return rc;
    }
    if ((flags & TVMC_SYNC) && (e = cudaEventSynchronize(c->done)) != cudaSuccess) {
        const int rc = cuda_fail(e, "sync");
        tvmc_commitment_free(c);
        return rc;
    }
    *out = c;
    return TVMC_OK;
}

int tvmc_commit_rows(const uint64_t* table, size_t num_rows, size_t width, uint32_t flags, void* stream,
                     tvmc_commitment** out) {
    if (!out) return fail(TVMC_ERR_INVALID, "null output handle");
    *out = nullptr;
    if (flags & ~(TVMC_TRACE_DEVICE | TVMC_TRACE_ROW_MAJOR | TVMC_DISCARD_LDE | TVMC_SYNC))
        return fail(TVMC_ERR_INVALID, "unknown flag bits 0x%x", flags);
    if (!is_pow2(num_rows)) return fail(TVMC_ERR_INVALID, "Number of leaves must be a power of 2 (got %zu)", num_rows);
    if (width && !table) return fail(TVMC_ERR_INVALID, "null table");
    cudaStream_t st = as_stream(stream);
    const bool dev = flags & TVMC_TRACE_DEVICE, rm = flags & TVMC_TRACE_ROW_MAJOR,
               discard = flags & TVMC_DISCARD_LDE;
    tvmc_commitment* c = new tvmc_commitment();
    CK(cudaGetDevice(&c->device));
    c->stream = st;
    c->n = c->L = num_rows;
    c->width = width;
    c->pooled = true;
    auto bail = [&](int code) {
        tvmc_commitment_free(c);
        return code;
    };
    const size_t NW = num_rows * width;
    if (dev_malloc_async((void**)&c->d_nodes, 2 * num_rows * 40, st) != cudaSuccess ||
        cudaMemsetAsync(c->d_nodes, 0, 40, st) != cudaSuccess) {
        cudaGetLastError();
        return bail(fail(TVMC_ERR_NOMEM, "cannot allocate the tree of %zu leaves", num_rows));
    }
    // rows to hash, column-major: the caller's device table itself when it can be
    // used as is and is not kept, else a copy the handle owns
    const uint64_t* src = table;
    if (width && !(dev && !rm && discard)) {
        uint64_t* up = nullptr;
        cudaError_t e = dev_malloc_async((void**)&c->d_lde, NW * 8, st);
        if (e == cudaSuccess && !dev && rm) {
            e = dev_malloc_async((void**)&up, NW * 8, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(up, table, NW * 8, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = launch_transpose(up, width, c->d_lde, num_rows, num_rows, width, st);
        } else if (e == cudaSuccess && rm) {
            e = launch_transpose(table, width, c->d_lde, num_rows, num_rows, width, st);
        } else if (e == cudaSuccess) {
            e = cudaMemcpyAsync(c->d_lde, table, NW * 8, dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
        }
        if (up) cudaFreeAsync(up, st);
        if (e != cudaSuccess) return bail(cuda_fail(e, "row upload"));
        src = c->d_lde;
    }
    cudaError_t e = launch_hash_rows(src, 1, num_rows, num_rows, (uint32_t)width, nullptr, c->d_nodes, LAYOUT_HEAP, st);
    if (e != cudaSuccess) return bail(cuda_fail(e, "hash/merkle"));
    if (discard && c->d_lde) {
        cudaFreeAsync(c->d_lde, st);
        c->d_lde = nullptr;
    }
    return finish_commitment(c, flags, out);
}

int tvmc_commit_digests(const uint64_t* leaves, size_t num_leaves, uint32_t flags, void* stream,
                        tvmc_commitment** out) {
    if (!out) return fail(TVMC_ERR_INVALID, "null output handle");
    *out = nullptr;
    if (flags & ~(TVMC_TRACE_DEVICE | TVMC_LEAVES_XFE | TVMC_SYNC))
        return fail(TVMC_ERR_INVALID, "unknown flag bits 0x%x", flags);
    if (!is_pow2(num_leaves))
        return fail(TVMC_ERR_INVALID, "Number of leaves must be a power of 2 (got %zu)", num_leaves);
    if (!leaves) return fail(TVMC_ERR_INVALID, "null leaves");
    cudaStream_t st = as_stream(stream);
    const int words = (flags & TVMC_LEAVES_XFE) ? 3 : 5;
    tvmc_commitment* c = new tvmc_commitment();
    CK(cudaGetDevice(&c->device));
    c->stream = st;
    c->n = c->L = num_leaves;
    c->width = 0;
    c->pooled = true;
    auto bail = [&](int code) {
        tvmc_commitment_free(c);
        return code;
    };
    if (dev_malloc_async((void**)&c->d_nodes, 2 * num_leaves * 40, st) != cudaSuccess ||
        cudaMemsetAsync(c->d_nodes, 0, 40, st) != cudaSuccess) {
        cudaGetLastError();
        return bail(fail(TVMC_ERR_NOMEM, "cannot allocate the tree of %zu leaves", num_leaves));
    }
    const uint64_t* src = leaves;
    uint64_t* up = nullptr;
    cudaError_t e = cudaSuccess;
    if (!(flags & TVMC_TRACE_DEVICE)) {
        e = dev_malloc_async((void**)&up, num_leaves * words * 8, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(up, leaves, num_leaves * words * 8, cudaMemcpyHostToDevice, st);
        src = up;
    }
    if (e == cudaSuccess) e = launch_merkle_tree(src, c->d_nodes, num_leaves, LAYOUT_HEAP, st, words);
    if (up) cudaFreeAsync(up, st);
    if (e != cudaSuccess) return bail(cuda_fail(e, "merkle"));
    return finish_commitment(c, flags, out);
}

int tvmc_sponge_absorb_gpu(uint64_t* d_state, const uint64_t* d_data, size_t len, void* stream) {
    if (!d_state || (len && !d_data)) return fail(TVMC_ERR_INVALID, "null argument");
    CK(launch_sponge_absorb(d_state, d_data, len, 0, 0, as_stream(stream)));
    return TVMC_OK;
}

int tvmc_commitment_absorb_root(tvmc_commitment* c, uint64_t* d_state, void* stream) {
    if (!c || !d_state) return fail(TVMC_ERR_INVALID, "null argument");
    cudaStream_t st = as_stream(stream);
    CK(cudaStreamWaitEvent(st, c->done, 0));
    // the proof item MerkleRoot: discriminant 0, then the root (heap node 1)
    CK(launch_sponge_absorb(d_state, c->d_nodes + 5, 5, 1, 0, st));
    if (st != c->stream) {  // a later free of the tree (on the commitment's stream) waits for this read
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaError_t e = cudaEventRecord(ev, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(c->stream, ev, 0);
        cudaEventDestroy(ev);
        CK(e);
    }
    return TVMC_OK;
}

int tvmc_commitment_sync(tvmc_commitment* c) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    CK(cudaEventSynchronize(c->done));
    return TVMC_OK;
}

int tvmc_commitment_root(tvmc_commitment* c, uint64_t* root) {
    if (!c || !root) return fail(TVMC_ERR_INVALID, "null argument");
    return read_sync(c, c->d_nodes + 5, 5, root);
}

int tvmc_commitment_shape(const tvmc_commitment* c, size_t* lde_len, size_t* width) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    if (lde_len) *lde_len = c->L;
    if (width) *width = c->width;
    return TVMC_OK;
}

int tvmc_commitment_device_lde(const tvmc_commitment* c, const uint64_t** d_lde) {
    if (!c || !d_lde) return fail(TVMC_ERR_INVALID, "null argument");
    *d_lde = c->d_lde;
    return TVMC_OK;
}

int tvmc_commitment_device_tree(const tvmc_commitment* c, const uint64_t** d_nodes) {
    if (!c || !d_nodes) return fail(TVMC_ERR_INVALID, "null argument");
    *d_nodes = c->d_nodes;
    return TVMC_OK;
}

int tvmc_commitment_auth_paths(tvmc_commitment* c, const size_t* leaf_idx, size_t count, uint64_t* out) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    if (count == 0) return TVMC_OK;
    for (size_t q = 0; q < count; q++)
        if (leaf_idx[q] >= c->L) return fail(TVMC_ERR_RANGE, "Leaf index %zu out of range", leaf_idx[q]);
    int h = log2u(c->L);
    if (h == 0) return TVMC_OK;
    return gather_sync(c, leaf_idx, count, (size_t)h * 5, out, [&](const uint64_t* di, uint64_t* dout, cudaStream_t st) {
        return launch_gather_auth_paths(c->d_nodes, c->L, LAYOUT_HEAP, di, count, dout, st);
    });
}

int tvmc_auth_structure_indices(size_t num_leaves, const size_t* leaf_idx, size_t count, uint64_t* out,
                                size_t max_out, size_t* num_out) {
    if (!is_pow2(num_leaves)) return fail(TVMC_ERR_INVALID, "num_leaves must be a power of 2 (got %zu)", num_leaves);
    std::vector<uint64_t> res;
    int rc = auth_structure_nodes(num_leaves, leaf_idx, count, &res);
    if (rc) return rc;
    if (num_out) *num_out = res.size();
    for (size_t i = 0; i < res.size() && i < max_out; i++) out[i] = res[i];
    return TVMC_OK;
}

int tvmc_commitment_auth_structure(tvmc_commitment* c, const size_t* leaf_idx, size_t count, uint64_t* out,
                                   size_t max_digests, size_t* num_digests) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    const size_t n = c->L;
    std::vector<uint64_t> res;
    int rc = auth_structure_nodes(n, leaf_idx, count, &res);
    if (rc) return rc;
    if (num_digests) *num_digests = res.size();
    size_t m = std::min(res.size(), max_digests);
    if (m == 0) return TVMC_OK;
    return gather_sync(c, res.data(), m, 5, out, [&](const uint64_t* di, uint64_t* dout, cudaStream_t st) {
        return launch_gather_nodes(c->d_nodes, n, LAYOUT_HEAP, di, m, dout, st);
    });
}

int tvmc_commitment_read_rows(tvmc_commitment* c, const size_t* rows, size_t count, uint64_t* out) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    if (!c->d_lde && c->width) return fail(TVMC_ERR_INVALID, "LDE was discarded");
    for (size_t q = 0; q < count; q++)
        if (rows[q] >= c->L) return fail(TVMC_ERR_RANGE, "Row index %zu out of range", rows[q]);
    if (count == 0 || c->width == 0) return TVMC_OK;
    return gather_sync(c, rows, count, c->width, out, [&](const uint64_t* di, uint64_t* dout, cudaStream_t st) {
        return launch_gather_rows(c->d_lde, c->L, (uint32_t)c->width, di, count, dout, st);
    });
}

int tvmc_commitment_read_columns(tvmc_commitment* c, size_t col0, size_t ncols, uint64_t* out) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    if (!c->d_lde && c->width) return fail(TVMC_ERR_INVALID, "LDE was discarded");
    if (col0 > c->width || ncols > c->width - col0)
        return fail(TVMC_ERR_RANGE, "columns [%zu, %zu) out of range", col0, col0 + ncols);
    if (ncols == 0) return TVMC_OK;
    CK(cudaEventSynchronize(c->done));
    CK(cudaMemcpy(out, c->d_lde + col0 * c->L, ncols * c->L * 8, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_commitment_read_lde(tvmc_commitment* c, uint64_t* out, int row_major) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    if (!c->d_lde && c->width) return fail(TVMC_ERR_INVALID, "LDE was discarded");
    if (c->width == 0) return TVMC_OK;
    CK(cudaEventSynchronize(c->done));
    const size_t W = c->L * c->width;
    if (!row_major) {
        CK(cudaMemcpy(out, c->d_lde, W * 8, cudaMemcpyDeviceToHost));
        return TVMC_OK;
    }
    DBuf t;
    CK(t.alloc(W));
    CK(launch_transpose_cm_to_rm(c->d_lde, c->L, t.p, c->width, c->L, c->width, nullptr));
    CK(cudaMemcpy(out, t.p, W * 8, cudaMemcpyDeviceToHost));
    return TVMC_OK;
}

int tvmc_commitment_read_leaves(tvmc_commitment* c, uint64_t* out) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    return read_sync(c, c->d_nodes + 5 * c->L, c->L * 5, out);
}

int tvmc_commitment_read_nodes(tvmc_commitment* c, uint64_t* out) {
    if (!c) return fail(TVMC_ERR_INVALID, "null handle");
    return read_sync(c, c->d_nodes, c->L * 10, out);
}

int tvmc_commitment_free(tvmc_commitment* c) {
    if (!c) return TVMC_OK;
    if (c->batch_owned) return fail(TVMC_ERR_INVALID, "commitment belongs to a batch; free the batch");
    destroy_commitment(c);
    return TVMC_OK;
}

int tvmc_batch_free(tvmc_batch* b) {
    if (!b) return TVMC_OK;
    if (b->counted) {
        std::lock_guard<std::mutex> lk(g_mu);
        g_dev[b->device].live_batches--;
    }
    for (auto* c : b->tables) destroy_commitment(c);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto s : b->workers) cudaStreamDestroy(s);
    if (b->capture) cudaStreamDestroy(b->capture);
    for (auto e : b->events) cudaEventDestroy(e);
    for (auto p : b->inputs) cudaFree(p);
    for (auto p : b->scratch) cudaFree(p);
    delete b;
    return TVMC_OK;
}

int tvmc_batch_create(const tvmc_table_shape* shapes, size_t count, tvmc_batch** out) {
    if (!out || (count && !shapes)) return fail(TVMC_ERR_INVALID, "null argument");
    *out = nullptr;
    if (count == 0) return fail(TVMC_ERR_INVALID, "empty batch");
    std::vector<LdePlan> plans(count);
    for (size_t i = 0; i < count; i++) {
        const tvmc_table_shape& s = shapes[i];
        if (!is_pow2(s.expansion) || s.expansion > 16)
            return fail(TVMC_ERR_INVALID, "table %zu: expansion %u is not a power of 2 <= 16", i, s.expansion);
        int logn, le;
        int rc = check_lde_sizes(s.trace_len, s.trace_len * s.expansion, &logn, &le);
        if (rc) return rc;
        if ((rc = get_plan(logn, le, s.offset, &plans[i]))) return rc;  // tables built before capture
    }
    tvmc_batch* b = new tvmc_batch();
    auto bail = [&](int code) {
        tvmc_batch_free(b);
        return code;
    };
    CK(cudaGetDevice(&b->device));
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_dev[b->device].live_batches++;
        b->counted = true;
    }
    b->shapes.assign(shapes, shapes + count);
    const long long ks = g_tune_batch_streams.load();
    const size_t K = std::min<size_t>(count, ks > 0 ? (size_t)ks : 8);
    // tables, largest first, onto the least-loaded worker
    std::vector<size_t> order(count);
    for (size_t i = 0; i < count; i++) order[i] = i;
    auto work = [&](size_t i) { return (double)shapes[i].trace_len * shapes[i].expansion * (shapes[i].width + 1); };
    std::sort(order.begin(), order.end(), [&](size_t a, size_t c) { return work(a) > work(c); });
    std::vector<std::vector<size_t>> assign(K);
    std::vector<double> load(K, 0.0);
    for (size_t i : order) {
        const size_t w = std::min_element(load.begin(), load.end()) - load.begin();
        assign[w].push_back(i);
        load[w] += work(i);
    }
    // buffers
    const size_t budget = std::max<size_t>(scratch_budget() / K, size_t(64) << 20);
    std::vector<size_t> chunk(count);
    for (size_t i = 0; i < count; i++) {
        const tvmc_table_shape& s = shapes[i];
        tvmc_commitment* c = new tvmc_commitment();
        c->batch_owned = true;
        c->device = b->device;
        c->n = s.trace_len;
        c->width = s.width;
        c->L = s.trace_len * s.expansion;
        b->tables.push_back(c);
        uint64_t* in = nullptr;
        if (dev_malloc((void**)&c->d_nodes, 2 * c->L * 40) != cudaSuccess ||
            (s.width && dev_malloc((void**)&c->d_lde, c->L * s.width * 8) != cudaSuccess) ||
            (s.width && dev_malloc((void**)&in, s.trace_len * s.width * 8) != cudaSuccess)) {
            cudaGetLastError();
            if (in) cudaFree(in);
            return bail(fail(TVMC_ERR_NOMEM, "cannot allocate table %zu of the batch", i));
        }
        b->inputs.push_back(in);
        CK(cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming));
        const size_t per = lde_scratch_words(plans[i].logn, plans[i].log_exp, 1) * 8;
        chunk[i] = per ? std::max<size_t>(1, std::min(s.width, budget / per)) : std::max<size_t>(s.width, 1);
    }
    for (size_t w = 0; w < K; w++) {
        size_t words = 0;
        for (size_t i : assign[w]) words = std::max(words, lde_scratch_words(plans[i].logn, plans[i].log_exp, chunk[i]));
        uint64_t* p = nullptr;
        if (words && dev_malloc((void**)&p, words * 8) != cudaSuccess) {
            cudaGetLastError();
            return bail(fail(TVMC_ERR_NOMEM, "cannot allocate batch scratch"));
        }
        b->scratch.push_back(p);
        cudaStream_t s;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        b->workers.push_back(s);
    }
    for (size_t e = 0; e <= K; e++) {
        cudaEvent_t ev;
        CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        b->events.push_back(ev);
    }
    CK(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking));
    // capture: fork -> per-worker table commits -> join; with knob
    // "batch_multi_hash" (default on) the workers run the LDEs only and one
    // multi-table launch hashes every table after the join
    const bool multi = g_tune_batch_multi.load() != 2;
    const unsigned long long k0 = g_launches.load();
    CK(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeRelaxed));
    cudaError_t e = cudaEventRecord(b->events[0], b->capture);
    for (size_t w = 0; w < K && e == cudaSuccess; w++) {
        cudaStream_t st = b->workers[w];
        e = cudaStreamWaitEvent(st, b->events[0], 0);
        for (size_t t = 0; t < assign[w].size() && e == cudaSuccess; t++) {
            const size_t i = assign[w][t];
            tvmc_commitment* c = b->tables[i];
            const size_t W = shapes[i].width, N = shapes[i].trace_len;
            e = cudaMemsetAsync(c->d_nodes, 0, 40, st);
            for (size_t c0 = 0; c0 < W && e == cudaSuccess; c0 += chunk[i]) {
                const size_t nc = std::min(chunk[i], W - c0);
                e = launch_lde(plans[i], b->inputs[i] + c0 * N, N, c->d_lde + c0 * c->L, c->L, nc, b->scratch[w], st);
            }
            if (e == cudaSuccess && !multi)
                e = launch_hash_rows(c->d_lde, 1, c->L, c->L, (uint32_t)W, nullptr, c->d_nodes, LAYOUT_HEAP, st);
        }
        if (e == cudaSuccess) e = cudaEventRecord(b->events[w + 1], st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->capture, b->events[w + 1], 0);
    }
    if (multi && e == cudaSuccess) {
        // after every LDE: all tables' row hashes as one launch (largest first,
        // so that the small tables' CTAs fill the tail), then the tree tops
        std::vector<MultiHashTable> jobs;
        for (size_t i : order) {
            tvmc_commitment* c = b->tables[i];
            jobs.push_back(MultiHashTable{c->d_lde, c->d_nodes, c->L, (uint32_t)shapes[i].width});
        }
        e = launch_hash_rows_multi(jobs.data(), (int)jobs.size(), b->capture);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(b->capture, &g);
    b->graph = g;
    b->kernels_per_run = g_launches.load() - k0;
    g_launches.fetch_sub(b->kernels_per_run);  // counted again at every run
    if (e != cudaSuccess) return bail(cuda_fail(e, "batch capture"));
    if (e2 != cudaSuccess) return bail(cuda_fail(e2, "batch capture end"));
    CK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    *out = b;
    return TVMC_OK;
}

int tvmc_batch_input(tvmc_batch* b, size_t i, uint64_t** d_trace) {
    if (!b || !d_trace) return fail(TVMC_ERR_INVALID, "null argument");
    if (i >= b->tables.size()) return fail(TVMC_ERR_RANGE, "table %zu out of range", i);
    *d_trace = b->inputs[i];
    return TVMC_OK;
}

int tvmc_batch_run(tvmc_batch* b, void* stream) {
    if (!b) return fail(TVMC_ERR_INVALID, "null batch");
    cudaStream_t st = as_stream(stream);
    NvtxRange range("tvmc batch launch");
    CK(cudaGraphLaunch(b->exec, st));
    g_launches.fetch_add(b->kernels_per_run);
    for (auto* c : b->tables) {
        c->stream = st;
        CK(cudaEventRecord(c->done, st));
    }
    return TVMC_OK;
}

int tvmc_batch_commitment(tvmc_batch* b, size_t i, tvmc_commitment** c) {
    if (!b || !c) return fail(TVMC_ERR_INVALID, "null argument");
    if (i >= b->tables.size()) return fail(TVMC_ERR_RANGE, "table %zu out of range", i);
    *c = b->tables[i];
    return TVMC_OK;
}

int tvmc_commitment_phase_ms(tvmc_commitment* c, float* ms) {
    if (!c || !ms) return fail(TVMC_ERR_INVALID, "null argument");
    if (!c->prof[0]) return fail(TVMC_ERR_INVALID, "commitment was not made with TVMC_PROFILE");
    CK(cudaEventSynchronize(c->done));
    for (int i = 0; i < 3; i++) CK(cudaEventElapsedTime(&ms[i], c->prof[i], c->prof[i + 1]));
    return TVMC_OK;
}

}  // extern "C"
