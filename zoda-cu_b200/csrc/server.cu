// Serving loop with continuous batching (zoda_server_* in include/zoda_b200.h).
//
// One native thread owns the device side. Each pass:
//   1. retire: every launch whose completion event has fired marks its
//      requests done (latency stamped) and frees its stream slot;
//   2. admit + launch: while a slot is free and requests wait, take them in
//      arrival order as long as their outputs fit in the arena (the HBM
//      budget) and the launch has room, then encode them with one batched
//      kernel (k_extend_batch) on that slot's stream;
//   3. otherwise sleep on a condition variable until a submit, or briefly
//      while launches are in flight.
// Requests that arrive while others run join the next launch; up to
// max_inflight launches overlap on the GPU. Nothing is allocated per request:
// outputs come from the arena, descriptors from per-slot buffers.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "tma_host.hpp"

namespace zb {
namespace {

using clk = std::chrono::steady_clock;

// First-fit allocator over one device range, offsets aligned to 256 bytes,
// neighbouring free ranges merged on release.
class Arena {
   public:
    void init(uint64_t size) {
        free_.clear();
        free_[0] = size;
    }
    bool alloc(uint64_t size, uint64_t* off) {
        size = (size + 255) & ~255ull;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= size) {
                *off = it->first;
                const uint64_t rest = it->second - size, at = it->first + size;
                free_.erase(it);
                if (rest) free_[at] = rest;
                return true;
            }
        }
        return false;
    }
    void release(uint64_t off, uint64_t size) {
        size = (size + 255) & ~255ull;
        auto it = free_.emplace(off, size).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }

   private:
    std::map<uint64_t, uint64_t> free_;
};

enum class RState { Queued, Launched, Done, Cancelled };

struct Request {
    const uint32_t* d_in = nullptr;
    uint32_t k = 0;
    uint64_t cols = 0;
    uint64_t out_off = 0, out_bytes = 0;
    bool has_out = false;
    RState state = RState::Queued;
    zoda_status status = ZODA_OK;
    clk::time_point t_submit, t_launch, t_done;
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    DevBuf d_sq, d_counter;
    BatchSquare* h_sq = nullptr;  // pinned
    std::vector<uint64_t> reqs;
    bool busy = false;
};

}  // namespace
}  // namespace zb

struct zoda_server {
    zoda_ctx* ctx = nullptr;
    uint64_t budget = 0;
    uint32_t max_inflight = 4, max_batch = 128;
    zb::DevBuf arena_mem, d_tables;
    zb::Arena arena;
    std::vector<zb::Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::unordered_map<uint64_t, zb::Request> reqs;
    std::deque<uint64_t> pending;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread th;
    // statistics
    uint64_t submitted = 0, completed = 0, cancelled = 0, launches = 0, elements = 0;
    std::vector<double> latencies;
    bool any_submit = false;
    zb::clk::time_point first_submit, last_done;
};

namespace zb {
namespace {

double ms_between(clk::time_point a, clk::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Called with the mutex held. Returns true if it changed anything.
bool retire(zoda_server* s) {
    bool any = false;
    for (auto& sl : s->slots) {
        if (!sl.busy) continue;
        const cudaError_t q = cudaEventQuery(sl.done);
        if (q == cudaErrorNotReady) continue;
        const auto now = clk::now();
        for (uint64_t id : sl.reqs) {
            auto it = s->reqs.find(id);
            if (it == s->reqs.end()) continue;
            Request& r = it->second;
            r.state = RState::Done;
            r.t_done = now;
            if (q != cudaSuccess) {
                set_last_error("serving launch", q);
                r.status = ZODA_ERR_CUDA;
            } else {
                s->completed++;
                s->elements += (uint64_t)r.k * r.cols;
                s->latencies.push_back(ms_between(r.t_submit, now));
                s->last_done = now;
            }
        }
        sl.reqs.clear();
        sl.busy = false;
        any = true;
    }
    if (any) s->cv_done.notify_all();
    return any;
}

// Called with the mutex held: fill one free slot from the head of the queue.
bool admit_and_launch(zoda_server* s, Slot& sl) {
    std::vector<uint64_t> take;
    while (!s->pending.empty() && take.size() < s->max_batch) {
        const uint64_t id = s->pending.front();
        Request& r = s->reqs[id];
        if (r.state != RState::Queued) {  // cancelled while queued
            s->pending.pop_front();
            continue;
        }
        uint64_t off;
        if (!s->arena.alloc(r.out_bytes, &off)) break;  // wait for outputs to be released (FIFO order)
        r.out_off = off;
        r.has_out = true;
        s->pending.pop_front();
        take.push_back(id);
    }
    if (take.empty()) return false;
    std::stable_sort(take.begin(), take.end(), [&](uint64_t a, uint64_t b) { return s->reqs[a].k > s->reqs[b].k; });
    uint64_t first = 0;
    uint32_t n = 0;
    int max_log = 0;  // the launch's largest side sets its level radix
    const auto now = clk::now();
    for (uint64_t id : take) {
        Request& r = s->reqs[id];
        zoda_square q{r.d_in, (uint32_t*)((char*)s->arena_mem.p + r.out_off), r.k, 0, r.cols};
        BatchSquare& b = sl.h_sq[n];
        int ls = 0;
        while ((1u << ls) < r.k) ls++;
        const zoda_status st = make_batch_square(q, &b, side_l2_promo(s->ctx, ls));
        r.t_launch = now;
        if (st != ZODA_OK) {
            r.state = RState::Done;
            r.status = st;
            r.t_done = now;
            continue;
        }
        b.first = first;
        first += b.ntiles;
        if (ls > max_log) max_log = ls;
        r.state = RState::Launched;
        sl.reqs.push_back(id);
        n++;
    }
    if (n == 0) {
        s->cv_done.notify_all();
        return true;
    }
    cudaError_t e = cudaMemcpyAsync(sl.d_sq.p, sl.h_sq, n * sizeof(BatchSquare), cudaMemcpyHostToDevice, sl.st);
    if (e == cudaSuccess) e = cudaMemsetAsync(sl.d_counter.p, 0, sizeof(unsigned long long), sl.st);
    zoda_status ls = ZODA_ERR_CUDA;
    if (e == cudaSuccess)
    {
        const int lept = batch_lept(s->ctx, max_log);
        ls = launch_batch_kernel(s->ctx, (const BatchSquare*)sl.d_sq.p, n, first, (unsigned long long*)sl.d_counter.p,
                                 (const SideTables*)s->d_tables.p + (lept == 3 ? 13 : 0), lept, sl.st);
    }
    if (ls == ZODA_OK) e = cudaEventRecord(sl.done, sl.st);
    if (ls != ZODA_OK || e != cudaSuccess) {
        if (e != cudaSuccess) set_last_error("serving launch setup", e);
        for (uint64_t id : sl.reqs) {
            Request& r = s->reqs[id];
            r.state = RState::Done;
            r.status = ZODA_ERR_CUDA;
            r.t_done = clk::now();
        }
        sl.reqs.clear();
        s->cv_done.notify_all();
        return true;
    }
    sl.busy = true;
    s->launches++;
    return true;
}

void server_loop(zoda_server* s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lock(s->mu);
    for (;;) {
        bool changed = retire(s);
        bool inflight = false;
        for (auto& sl : s->slots) {
            if (!sl.busy && !s->pending.empty()) changed |= admit_and_launch(s, sl);
            inflight |= sl.busy;
        }
        if (s->stop && !inflight) break;
        if (changed) continue;
        if (inflight)
            s->cv_work.wait_for(lock, std::chrono::microseconds(20));
        else
            s->cv_work.wait_for(lock, std::chrono::milliseconds(5));
    }
}

}  // namespace
}  // namespace zb

using namespace zb;

extern "C" {

zoda_status zoda_server_create(zoda_ctx* ctx, const zoda_server_config* cfg, zoda_server** out) {
    if (!ctx || !out) return ZODA_ERR_ARG;
    *out = nullptr;
    zoda_server* s = new (std::nothrow) zoda_server();
    if (!s) return ZODA_ERR_NOMEM;
    s->ctx = ctx;
    s->budget = cfg && cfg->hbm_budget_bytes ? cfg->hbm_budget_bytes : (64ull << 30);
    s->max_inflight = cfg && cfg->max_inflight ? cfg->max_inflight : 4;
    s->max_batch = cfg && cfg->max_batch ? cfg->max_batch : 128;
    auto fail = [&](zoda_status st) {
        zoda_server_destroy(s);
        return st;
    };
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
        set_last_error("cudaSetDevice", e);
        return fail(ZODA_ERR_CUDA);
    }
    zoda_status st;
    if ((st = s->arena_mem.ensure(s->budget)) != ZODA_OK) return fail(st);
    s->arena.init(s->budget);
    if ((st = s->d_tables.ensure(26 * sizeof(SideTables))) != ZODA_OK) return fail(st);
    std::vector<SideTables> tabs(26);  // radix 16 at [log_s], radix 8 at [13 + log_s]
    for (int ls = BATCH_MIN_LOG; ls <= BATCH_MAX_LOG; ls++) {
        tabs[ls] = side_tables(ctx, ls, 4);
        tabs[13 + ls] = side_tables(ctx, ls, 3);
    }
    if ((e = cudaMemcpy(s->d_tables.p, tabs.data(), 26 * sizeof(SideTables), cudaMemcpyHostToDevice)) !=
        cudaSuccess) {
        set_last_error("cudaMemcpy(server tables)", e);
        return fail(ZODA_ERR_CUDA);
    }
    if ((st = set_batch_kernel_attributes()) != ZODA_OK) return fail(st);
    s->slots.resize(s->max_inflight);
    for (auto& sl : s->slots) {
        if ((e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaHostAlloc((void**)&sl.h_sq, s->max_batch * sizeof(BatchSquare), cudaHostAllocDefault)) !=
                cudaSuccess) {
            set_last_error("server slot setup", e);
            return fail(ZODA_ERR_CUDA);
        }
        if ((st = sl.d_sq.ensure(s->max_batch * sizeof(BatchSquare))) != ZODA_OK) return fail(st);
        if ((st = sl.d_counter.ensure(sizeof(unsigned long long))) != ZODA_OK) return fail(st);
    }
    try {
        s->th = std::thread(server_loop, s);
    } catch (...) {
        return fail(ZODA_ERR_STATE);
    }
    *out = s;
    return ZODA_OK;
}

zoda_status zoda_server_submit(zoda_server* s, const uint32_t* d_in, uint32_t k, uint64_t cols, uint64_t* ticket) {
    if (!s || !d_in || !ticket || k < 32 || k > 2048 || (k & (k - 1)) || cols % 4 || ((uintptr_t)d_in & 15))
        return ZODA_ERR_ARG;
    const uint64_t out_bytes = 8ull * k * cols;
    if (out_bytes > s->budget) {
        set_last_error_text("request output exceeds the server's HBM budget");
        return ZODA_ERR_BUDGET;
    }
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stop) return ZODA_ERR_STATE;
        const uint64_t id = s->next_id++;
        Request& r = s->reqs[id];
        r.d_in = d_in;
        r.k = k;
        r.cols = cols;
        r.out_bytes = out_bytes;
        r.t_submit = clk::now();
        if (!s->any_submit) {
            s->any_submit = true;
            s->first_submit = r.t_submit;
        }
        s->pending.push_back(id);
        s->submitted++;
        *ticket = id;
    }
    s->cv_work.notify_one();
    return ZODA_OK;
}

zoda_status zoda_server_wait(zoda_server* s, uint64_t ticket, uint32_t timeout_ms, zoda_request_info* info) {
    if (!s) return ZODA_ERR_ARG;
    std::unique_lock<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return ZODA_ERR_ARG;
    auto finished = [&] {
        const RState st = s->reqs[ticket].state;
        return st == RState::Done || st == RState::Cancelled;
    };
    if (!finished() && timeout_ms) s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), finished);
    if (!finished()) return ZODA_ERR_TIMEOUT;
    Request& r = s->reqs[ticket];
    if (r.state == RState::Cancelled) return ZODA_ERR_CANCELLED;
    if (info) {
        info->d_out = (uint32_t*)((char*)s->arena_mem.p + r.out_off);
        info->queue_ms = ms_between(r.t_submit, r.t_launch);
        info->latency_ms = ms_between(r.t_submit, r.t_done);
        info->status = r.status;
        info->reserved = 0;
    }
    return r.status;
}

zoda_status zoda_server_release(zoda_server* s, uint64_t ticket) {
    if (!s) return ZODA_ERR_ARG;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        auto it = s->reqs.find(ticket);
        if (it == s->reqs.end()) return ZODA_ERR_ARG;
        Request& r = it->second;
        if (r.state == RState::Queued || r.state == RState::Launched) return ZODA_ERR_STATE;
        if (r.has_out) s->arena.release(r.out_off, r.out_bytes);
        s->reqs.erase(it);
    }
    s->cv_work.notify_one();  // freed space may admit waiting requests
    return ZODA_OK;
}

zoda_status zoda_server_cancel(zoda_server* s, uint64_t ticket) {
    if (!s) return ZODA_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return ZODA_ERR_ARG;
    if (it->second.state != RState::Queued) return ZODA_ERR_STATE;
    it->second.state = RState::Cancelled;
    s->cancelled++;
    s->cv_done.notify_all();
    return ZODA_OK;
}

zoda_status zoda_server_get_stats(zoda_server* s, zoda_server_stats* out) {
    if (!s || !out) return ZODA_ERR_ARG;
    std::lock_guard<std::mutex> lock(s->mu);
    memset(out, 0, sizeof *out);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->cancelled = s->cancelled;
    out->launches = s->launches;
    out->elements = s->elements;
    if (!s->latencies.empty()) {
        std::vector<double> v = s->latencies;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) { return v[std::min(v.size() - 1, (size_t)(p * (double)(v.size() - 1) + 0.5))]; };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->max_ms = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        out->mean_ms = sum / (double)v.size();
        out->first_submit_to_last_done_ms = ms_between(s->first_submit, s->last_done);
    }
    return ZODA_OK;
}

void zoda_server_destroy(zoda_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stop = true;
        for (uint64_t id : s->pending) {
            Request& r = s->reqs[id];
            if (r.state == RState::Queued) {
                r.state = RState::Cancelled;
                s->cancelled++;
            }
        }
        s->pending.clear();
    }
    s->cv_work.notify_all();
    if (s->th.joinable()) s->th.join();
    if (s->ctx) cudaSetDevice(s->ctx->device);
    for (auto& sl : s->slots) {
        if (sl.st) cudaStreamSynchronize(sl.st);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.st) cudaStreamDestroy(sl.st);
        if (sl.h_sq) cudaFreeHost(sl.h_sq);
        sl.d_sq.release();
        sl.d_counter.release();
    }
    s->arena_mem.release();
    s->d_tables.release();
    delete s;
}

}  // extern "C"
