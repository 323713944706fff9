// Commitment serving runtime (host C++; the GPU work is tvmc_commit's).
//
// A server owns worker streams on one device and a dispatcher thread.
// Submitted requests queue in arrival order, in two classes: large tables
// (LDE above 128 MB, enough work to fill the GPU alone) and small ones.  The
// dispatcher admits a queue head as soon as its device footprint fits the HBM
// budget next to what running requests and resident trees already hold --
// small tables at once, on high-priority worker streams, and large tables up
// to a limit in flight (default 2) on one dedicated stream: two GPU-filling
// commits running side by side were measured slower than one after the other,
// but a second one issued behind the first gets its uploads and launches
// queued while the first computes, and the stream's cached LDE, scratch and
// staging buffers pass from one large commit to the next -- so small requests
// never wait behind large ones and requests of mixed sizes overlap as they
// arrive.  A host callback
// on the stream marks each request done, records its completion time and
// returns its transient memory to the budget; its Merkle tree (and, with
// TVMC_SERVER_KEEP_LDE, its LDE) stays on the device for openings until the
// caller releases it.  The reference has no counterpart: its prover commits
// one table at a time (src/stark.cpp:1163-1196).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.cuh"
#include "tvmc.h"

namespace {

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

enum class State { Queued, Running, Done, Failed };

struct Request {
    uint64_t id = 0;
    const uint64_t* trace = nullptr;
    size_t n = 0, width = 0;
    uint32_t expansion = 4, flags = 0;
    uint64_t offset = 7, trace_offset = 1;
    const uint64_t* randomizers = nullptr;  // width x R, same side of the bus as the trace
    size_t R = 0;
    size_t resident = 0, transient = 0;  // budget bytes held until release / until done
    bool large = false;
    int stream = -1;
    State state = State::Queued;
    int status = TVMC_OK;
    std::string error;
    tvmc_commitment* c = nullptr;
    uint64_t t_submit = 0, t_start = 0, t_done = 0;
};

// Device bytes a request holds: the tree (and a kept LDE) until release; the
// LDE, LDE scratch, upload staging and frugal state until it completes.
void footprint(Request* r, bool keep_lde, size_t scratch_budget) {
    const size_t N = r->n, L = N * r->expansion, W = r->width, NW = N * W * 8;
    const bool frugal = r->flags & TVMC_FRUGAL, dev = r->flags & TVMC_TRACE_DEVICE,
               rm = r->flags & TVMC_TRACE_ROW_MAJOR;
    const size_t tree = 2 * L * 40;
    const size_t lde = frugal ? std::min<size_t>(L * W * 8, size_t(2) << 30) : L * W * 8;
    const size_t scratch = N > 2048 ? std::min(scratch_budget, N * (1 + r->expansion) * 8 * std::max<size_t>(W, 1)) : 0;
    size_t upload = 0;
    if (frugal) upload = (dev ? 0 : NW) + (rm ? NW : 0) + 6 * L * 8;
    else if (!dev && !rm) {
        // host uploads stage column chunks of about 256 MB through up to four
        // buffers per stream (fewer when the table has fewer chunks)
        const size_t stage = std::min<size_t>(NW, size_t(256) << 20);
        upload = std::min<size_t>(4, (NW + stage - 1) / stage) * stage;
    }
    else upload = (dev ? 0 : NW) + (rm ? NW : 0);
    // randomized LDE: randomizer upload and the per-coset addends
    const size_t rrows = r->R < N ? r->R : N;
    const size_t rand = r->R ? (dev ? 0 : W * r->R * 8) + W * r->expansion * rrows * 8 : 0;
    r->resident = tree + (keep_lde && !frugal ? lde : 0);
    r->transient = (keep_lde && !frugal ? 0 : lde) + scratch + upload + rand;
    r->large = L * std::max<size_t>(W, 1) * 8 > (size_t(128) << 20);
}

}  // namespace

struct tvmc_server {
    int device = 0;
    size_t budget = 0;
    bool keep_lde = false;
    size_t scratch_budget = size_t(2) << 30;
    std::vector<cudaStream_t> streams;  // [0, n_small): small tables; the rest: one per large slot
    std::vector<int> inflight;          // per stream
    int n_small = 0;
    std::mutex mu;
    std::condition_variable cv;  // queue changes, completions, releases
    std::deque<Request*> queue_small, queue_large;
    int max_large = 1, large_running = 0;
    bool group_small = false;  // TVMC_SERVER_GROUP_SMALL: queued small requests committed together
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    size_t used = 0, peak = 0;
    uint64_t next_id = 1, submitted = 0, completed = 0, failed = 0, released = 0;
    int running = 0;
    bool stop = false;
    std::thread dispatcher;
};

namespace {

struct DoneCtx {
    tvmc_server* s;
    std::vector<Request*> rs;  // one request, or a group committed together
};

void CUDART_CB on_done(void* p) {
    std::unique_ptr<DoneCtx> ctx(static_cast<DoneCtx*>(p));
    tvmc_server* s = ctx->s;
    std::lock_guard<std::mutex> lk(s->mu);
    const uint64_t t = now_ns();
    for (Request* r : ctx->rs) {
        r->state = State::Done;
        r->t_done = t;
        s->used -= r->transient;
        s->inflight[r->stream]--;
        s->running--;
        if (r->large) s->large_running--;
        s->completed++;
    }
    s->cv.notify_all();
}

// A small request joins a multi-table group (tvmc_commit_multi) when it is a
// plain commitment of a column-major trace.
bool groupable(const Request* r) {
    return !r->large && r->R == 0 && r->trace_offset % 0xFFFFFFFF00000001ull == 1 &&
           !(r->flags & (TVMC_TRACE_ROW_MAJOR | TVMC_FRUGAL | TVMC_RAND_TRUNCATE));
}
constexpr size_t GROUP_MAX_TABLES = 64;
constexpr size_t GROUP_MAX_TRACE_WORDS = size_t(1) << 25;  // 256 MB of traces per group

void fail_request(tvmc_server* s, Request* r, int status, const std::string& msg) {
    r->state = State::Failed;
    r->status = status;
    r->error = msg;
    r->t_done = now_ns();
    s->failed++;
    s->cv.notify_all();
}

// The next request to issue: a small head that fits, else a large head that
// fits under the in-flight limit, else a head that can never fit (to fail it).
Request* pick(tvmc_server* s) {
    auto fits = [&](Request* r) { return s->used + r->resident + r->transient <= s->budget; };
    auto never = [&](Request* r) { return r->resident + r->transient > s->budget; };
    if (!s->queue_small.empty() && (fits(s->queue_small.front()) || never(s->queue_small.front())))
        return s->queue_small.front();
    if (!s->queue_large.empty()) {
        Request* r = s->queue_large.front();
        if (never(r) || (s->large_running < s->max_large && fits(r))) return r;
    }
    return nullptr;
}

// Issues a group of admitted small requests (lock held on entry and exit) as
// one tvmc_commit_multi on the least-loaded small-table stream: their row
// hashes run as one launch, so queued small tables fill the GPU together.
void issue_group(tvmc_server* s, std::vector<Request*>& g, std::unique_lock<std::mutex>& lk) {
    int best = 0;
    for (int i = 0; i < s->n_small; i++)
        if (s->inflight[i] < s->inflight[best]) best = i;
    const uint64_t t0 = now_ns();
    std::vector<tvmc_multi_table> tabs;
    for (Request* r : g) {
        s->used += r->resident + r->transient;
        r->stream = best;
        s->inflight[best]++;
        s->running++;
        r->state = State::Running;
        r->t_start = t0;
        tabs.push_back(tvmc_multi_table{r->trace, r->n, r->width, r->expansion, r->offset});
    }
    s->peak = std::max(s->peak, s->used);
    const uint32_t flags = (g[0]->flags & TVMC_TRACE_DEVICE) | (s->keep_lde ? 0u : (uint32_t)TVMC_DISCARD_LDE);
    cudaStream_t st = s->streams[best];
    lk.unlock();
    std::vector<tvmc_commitment*> cs(g.size(), nullptr);
    int rc = tvmc_commit_multi(tabs.data(), tabs.size(), flags, st, cs.data());
    const std::string err = rc ? tvmc_last_error() : "";
    DoneCtx* ctx = nullptr;
    if (!rc) {
        ctx = new DoneCtx{s, g};
        lk.lock();
        for (size_t i = 0; i < g.size(); i++) g[i]->c = cs[i];  // set before the callback can run
        lk.unlock();
        if (cudaLaunchHostFunc(st, on_done, ctx) != cudaSuccess) {
            delete ctx;
            ctx = nullptr;
            rc = TVMC_ERR_CUDA;
        }
    }
    lk.lock();
    if (!ctx) {
        for (size_t i = 0; i < g.size(); i++) {
            Request* r = g[i];
            s->used -= r->resident + r->transient;
            s->inflight[best]--;
            s->running--;
            r->c = nullptr;
            fail_request(s, r, rc, rc == TVMC_ERR_CUDA && err.empty() ? "cannot queue the completion callback" : err);
        }
        lk.unlock();
        for (auto* c : cs)
            if (c) tvmc_commitment_free(c);
        lk.lock();
    }
}

void dispatch_loop(tvmc_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        Request* r = nullptr;
        s->cv.wait(lk, [&] { return s->stop || (r = pick(s)) != nullptr; });
        if (s->stop) return;
        (r->large ? s->queue_large : s->queue_small).pop_front();
        const size_t need = r->resident + r->transient;
        if (need > s->budget) {
            fail_request(s, r, TVMC_ERR_NOMEM, "request footprint exceeds the server's HBM budget");
            continue;
        }
        if (s->group_small && groupable(r)) {
            // continuous batching: every queued small request that can join, in
            // arrival order, while the budget holds
            std::vector<Request*> g{r};
            size_t words = r->n * r->width, extra = need;
            for (auto it = s->queue_small.begin(); it != s->queue_small.end() && g.size() < GROUP_MAX_TABLES;) {
                Request* q = *it;
                const size_t qn = q->resident + q->transient;
                if (!groupable(q) || (q->flags & TVMC_TRACE_DEVICE) != (r->flags & TVMC_TRACE_DEVICE) ||
                    words + q->n * q->width > GROUP_MAX_TRACE_WORDS || s->used + extra + qn > s->budget) {
                    ++it;
                    continue;
                }
                g.push_back(q);
                words += q->n * q->width;
                extra += qn;
                it = s->queue_small.erase(it);
            }
            issue_group(s, g, lk);
            continue;
        }
        s->used += need;
        s->peak = std::max(s->peak, s->used);
        const int lo = r->large ? s->n_small : 0, hi = r->large ? (int)s->streams.size() : s->n_small;
        int best = lo;
        for (int i = lo; i < hi; i++)
            if (s->inflight[i] < s->inflight[best]) best = i;
        r->stream = best;
        s->inflight[best]++;
        s->running++;
        if (r->large) s->large_running++;
        r->state = State::Running;
        r->t_start = now_ns();
        const uint32_t flags = (r->flags & (TVMC_TRACE_DEVICE | TVMC_TRACE_ROW_MAJOR | TVMC_FRUGAL |
                                            TVMC_RAND_TRUNCATE)) |
                               (s->keep_lde ? 0u : (uint32_t)TVMC_DISCARD_LDE);
        cudaStream_t st = s->streams[best];
        lk.unlock();
        tvmc_commitment* c = nullptr;
        const int rc = tvmc_commit_randomized(r->trace, r->n, r->width, r->expansion, r->trace_offset, r->offset,
                                              r->randomizers, r->R, flags, st, &c);
        const std::string err = rc ? tvmc_last_error() : "";
        lk.lock();
        auto undo = [&] {
            s->used -= need;
            s->inflight[best]--;
            s->running--;
            if (r->large) s->large_running--;
        };
        if (rc) {
            undo();
            fail_request(s, r, rc, err);
            continue;
        }
        r->c = c;  // set before the completion callback can run
        lk.unlock();
        auto* ctx = new DoneCtx{s, {r}};
        const cudaError_t e = cudaLaunchHostFunc(st, on_done, ctx);
        lk.lock();
        if (e != cudaSuccess) {
            delete ctx;
            r->c = nullptr;
            undo();
            fail_request(s, r, TVMC_ERR_CUDA, cudaGetErrorString(e));
            lk.unlock();
            tvmc_commitment_free(c);
            lk.lock();
            continue;
        }
        // the resident part stays charged until release; on_done returns the transient part
    }
}

Request* find(tvmc_server* s, uint64_t id) {
    auto it = s->reqs.find(id);
    return it == s->reqs.end() ? nullptr : it->second.get();
}

}  // namespace

extern "C" {

int tvmc_server_create(const tvmc_server_config* cfg, tvmc_server** out) {
    if (!out) return tvmc::set_error(TVMC_ERR_INVALID, "null output handle");
    *out = nullptr;
    tvmc_server_config c{};
    if (cfg) c = *cfg;
    if (c.flags & ~(uint32_t)(TVMC_SERVER_KEEP_LDE | TVMC_SERVER_GROUP_SMALL))
        return tvmc::set_error(TVMC_ERR_INVALID, "unknown server flags");
    auto s = std::make_unique<tvmc_server>();
    if (cudaGetDevice(&s->device) != cudaSuccess) return tvmc::set_error(TVMC_ERR_CUDA, "no CUDA device");
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return tvmc::set_error(TVMC_ERR_CUDA, "cudaMemGetInfo");
    s->budget = c.hbm_budget_bytes ? c.hbm_budget_bytes : free_b / 10 * 9;
    s->keep_lde = c.flags & TVMC_SERVER_KEEP_LDE;
    s->group_small = c.flags & TVMC_SERVER_GROUP_SMALL;
    s->max_large = c.max_large_inflight ? (int)c.max_large_inflight : 2;
    long long sb = 0;
    if (tvmc_get_tuning("lde_scratch_bytes", &sb) == TVMC_OK && sb > 0) s->scratch_budget = (size_t)sb;
    s->n_small = c.num_streams ? (int)std::min<uint32_t>(c.num_streams, 64) : 4;
    s->max_large = (int)std::min<uint32_t>(s->max_large, 16);
    const int ns = s->n_small + 1;  // small-table streams + the large-table stream
    int lo_prio = 0, hi_prio = 0;
    cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio);
    // small tables one step below the greatest priority, which the openings'
    // accessor streams use; large tables at the lowest
    const int small_prio = hi_prio < lo_prio ? hi_prio + 1 : hi_prio;
    for (int i = 0; i < ns; i++) {
        cudaStream_t st;
        const int prio = i < s->n_small ? small_prio : lo_prio;
        if (cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio) != cudaSuccess) {
            for (auto x : s->streams) cudaStreamDestroy(x);
            return tvmc::set_error(TVMC_ERR_CUDA, "cannot create worker streams");
        }
        s->streams.push_back(st);
    }
    s->inflight.assign(ns, 0);
    tvmc_server* raw = s.release();
    raw->dispatcher = std::thread(dispatch_loop, raw);
    *out = raw;
    return TVMC_OK;
}

int tvmc_server_submit(tvmc_server* s, const uint64_t* trace, size_t trace_len, size_t width, uint32_t expansion,
                       uint64_t offset, uint32_t flags, uint64_t* id) {
    return tvmc_server_submit_randomized(s, trace, trace_len, width, expansion, 1, offset, nullptr, 0, flags, id);
}

int tvmc_server_submit_randomized(tvmc_server* s, const uint64_t* trace, size_t trace_len, size_t width,
                                  uint32_t expansion, uint64_t trace_offset, uint64_t offset,
                                  const uint64_t* randomizers, size_t num_randomizers, uint32_t flags,
                                  uint64_t* id) {
    if (!s || !id) return tvmc::set_error(TVMC_ERR_INVALID, "null argument");
    if (flags & ~(uint32_t)(TVMC_TRACE_DEVICE | TVMC_TRACE_ROW_MAJOR | TVMC_FRUGAL | TVMC_RAND_TRUNCATE))
        return tvmc::set_error(TVMC_ERR_INVALID, "server requests take only trace-layout, frugal and randomizer flags");
    if (trace_offset % 0xFFFFFFFF00000001ull == 0)
        return tvmc::set_error(TVMC_ERR_INVALID, "trace offset must be nonzero mod p");
    if (width && num_randomizers && !randomizers) return tvmc::set_error(TVMC_ERR_INVALID, "null randomizers");
    if (!trace_len || (trace_len & (trace_len - 1)) || trace_len > (size_t(1) << TVMC_MAX_LOG_LDE_TRACE))
        return tvmc::set_error(TVMC_ERR_INVALID, "trace length is not a supported power of 2");
    if (!expansion || (expansion & (expansion - 1)) || expansion > 16)
        return tvmc::set_error(TVMC_ERR_INVALID, "expansion factor is not a power of 2 <= 16");
    if (width && !trace) return tvmc::set_error(TVMC_ERR_INVALID, "null trace");
    auto r = std::make_unique<Request>();
    r->trace = trace;
    r->n = trace_len;
    r->width = width;
    r->expansion = expansion;
    r->offset = offset;
    r->trace_offset = trace_offset;
    r->randomizers = randomizers;
    r->R = width ? num_randomizers : 0;
    r->flags = flags;
    r->t_submit = now_ns();
    std::lock_guard<std::mutex> lk(s->mu);
    footprint(r.get(), s->keep_lde, s->scratch_budget);
    r->id = s->next_id++;
    *id = r->id;
    (r->large ? s->queue_large : s->queue_small).push_back(r.get());
    s->reqs.emplace(r->id, std::move(r));
    s->submitted++;
    s->cv.notify_all();
    return TVMC_OK;
}

int tvmc_server_wait(tvmc_server* s, uint64_t id, int64_t timeout_ms, uint64_t* root) {
    if (!s) return tvmc::set_error(TVMC_ERR_INVALID, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    Request* r = find(s, id);
    if (!r) return tvmc::set_error(TVMC_ERR_INVALID, "unknown request id");
    auto ready = [&] { return r->state == State::Done || r->state == State::Failed; };
    if (timeout_ms < 0)
        s->cv.wait(lk, ready);
    else if (!s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
        return tvmc::set_error(TVMC_ERR_TIMEOUT, "request not complete within the timeout");
    if (r->state == State::Failed) return tvmc::set_error(r->status, r->error.c_str());
    tvmc_commitment* c = r->c;
    lk.unlock();
    if (!c) return tvmc::set_error(TVMC_ERR_CUDA, "request finished without a commitment");
    return root ? tvmc_commitment_root(c, root) : TVMC_OK;
}

int tvmc_server_open(tvmc_server* s, uint64_t id, const size_t* leaf_idx, size_t count, uint64_t* paths,
                     uint64_t* rows) {
    if (!s) return tvmc::set_error(TVMC_ERR_INVALID, "null server");
    tvmc_commitment* c = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        Request* r = find(s, id);
        if (!r) return tvmc::set_error(TVMC_ERR_INVALID, "unknown request id");
        if (r->state != State::Done || !r->c) return tvmc::set_error(TVMC_ERR_INVALID, "request not committed");
        if (rows && !s->keep_lde) return tvmc::set_error(TVMC_ERR_INVALID, "server does not keep LDEs");
        c = r->c;
    }
    int rc = paths ? tvmc_commitment_auth_paths(c, leaf_idx, count, paths) : TVMC_OK;
    if (!rc && rows) rc = tvmc_commitment_read_rows(c, leaf_idx, count, rows);
    return rc;
}

int tvmc_server_times(tvmc_server* s, uint64_t id, uint64_t* submit_ns, uint64_t* start_ns, uint64_t* done_ns) {
    if (!s) return tvmc::set_error(TVMC_ERR_INVALID, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    Request* r = find(s, id);
    if (!r) return tvmc::set_error(TVMC_ERR_INVALID, "unknown request id");
    if (submit_ns) *submit_ns = r->t_submit;
    if (start_ns) *start_ns = r->t_start;
    if (done_ns) *done_ns = r->t_done;
    return TVMC_OK;
}

int tvmc_server_release(tvmc_server* s, uint64_t id) {
    if (!s) return tvmc::set_error(TVMC_ERR_INVALID, "null server");
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) return tvmc::set_error(TVMC_ERR_INVALID, "unknown request id");
        Request* q = it->second.get();
        if (q->state == State::Queued || q->state == State::Running)
            return tvmc::set_error(TVMC_ERR_INVALID, "request still in flight; wait for it first");
        if (q->state == State::Done) s->used -= q->resident;
        r = std::move(it->second);
        s->reqs.erase(it);
        s->released++;
        s->cv.notify_all();
    }
    if (r->c) tvmc_commitment_free(r->c);
    return TVMC_OK;
}

int tvmc_server_get_stats(tvmc_server* s, tvmc_server_stats* out) {
    if (!s || !out) return tvmc::set_error(TVMC_ERR_INVALID, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->failed = s->failed;
    out->released = s->released;
    out->queued = s->queue_small.size() + s->queue_large.size();
    out->running = (uint64_t)s->running;
    out->bytes_in_use = s->used;
    out->bytes_peak = s->peak;
    out->budget = s->budget;
    return TVMC_OK;
}

int tvmc_server_destroy(tvmc_server* s) {
    if (!s) return TVMC_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    s->dispatcher.join();
    for (auto st : s->streams) cudaStreamSynchronize(st);  // every on_done has run
    for (auto& kv : s->reqs)
        if (kv.second->c) tvmc_commitment_free(kv.second->c);
    for (auto st : s->streams) {
        tvmc_forget_stream(st);  // the library's cached buffers for this stream
        cudaStreamDestroy(st);
    }
    delete s;
    return TVMC_OK;
}

}  // extern "C"
