// Context, twiddle tables, status reporting and the fused-extension entry
// points of the C ABI (include/zoda_b200.h, part 2).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "async.cuh"
#include "internal.hpp"

namespace zb {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const char* where, cudaError_t e) {
    char buf[512];
    snprintf(buf, sizeof buf, "%s: %s (%d)", where, cudaGetErrorString(e), (int)e);
    g_last_error = buf;
}
void set_last_error_text(const std::string& s) { g_last_error = s; }

zoda_status DevBuf::ensure(size_t need) {
    if (need <= bytes) return ZODA_OK;
    release();
    if (need == 0) return ZODA_OK;
    cudaError_t e = cudaMalloc(&p, need);
    if (e != cudaSuccess) {
        set_last_error("cudaMalloc", e);
        p = nullptr;
        return ZODA_ERR_NOMEM;
    }
    bytes = need;
    return ZODA_OK;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

static uint32_t powmod(uint32_t b, uint64_t e) { return powmod_c(b, e); }

// Host-built tables: tw[j] = omega_8192^j; twist[S + i] = omega_2S^i / S.
static void build_tables(std::vector<Tw>& tw, std::vector<Tw>& twist) {
    constexpr int LOG_TW = 13;
    const uint32_t n = 1u << LOG_TW;
    tw.resize(n);
    const uint32_t w = root_of_unity(LOG_TW);
    uint32_t cur = 1;
    for (uint32_t j = 0; j < n; j++) {
        tw[j] = Tw{cur, shoup(cur)};
        cur = mulmod_c(cur, w);
    }
    twist.assign(n, Tw{0, 0});
    for (int ls = 0; ls <= 12; ls++) {
        const uint32_t S = 1u << ls;
        const uint32_t g = root_of_unity(ls + 1);
        const uint32_t s_inv = powmod(S, P - 2);
        uint32_t c = s_inv;
        for (uint32_t i = 0; i < S; i++) {
            twist[S + i] = Tw{c, shoup(c)};
            c = mulmod_c(c, g);
        }
    }
}

// Level tables of the TMA-staged kernel for side 2^ls (layout documented at
// SideTables in extend_tma.cuh). Offsets are entries into `all`.
// Level tables of the TMA kernel for side 2^ls with level radix 2^lept
// (off: INTT levels 0..2, NTT level 0 with the twist, NTT levels 1..2, end).
static void build_side_tables(int ls, int lept, std::vector<Tw>& all, size_t off[8]) {
    const int nlev = (ls + lept - 1) / lept;
    auto lr = [&](int l) { return l < nlev - 1 ? lept : ls - lept * (nlev - 1); };
    auto nlr = [&](int l) { return lr(nlev - 1 - l); };
    const uint32_t S = 1u << ls;
    auto tw_of = [](uint32_t w) { return Tw{w, shoup(w)}; };
    auto pow_root = [](int logn, uint64_t e) { return powmod_c(root_of_unity(logn), e); };
    for (int k = 0; k < 8; k++) off[k] = all.size();
    // INTT levels 0 .. nlev-2: [k2*L + m] = omega_N^(-m*k2)
    int pb = 0;
    for (int l = 0; l < 3; l++) {
        off[l] = all.size();
        if (l < nlev - 1) {
            const int logn = ls - pb, R = 1 << lr(l), L = 1 << (logn - lr(l));
            const uint32_t N = 1u << logn;
            for (int k2 = 0; k2 < R; k2++)
                for (int m = 0; m < L; m++) all.push_back(tw_of(pow_root(logn, (N - (uint64_t)m * k2 % N) % N)));
            pb += lr(l);
        }
    }
    // NTT level 0 with the twist: [k2*NB + b] = g^c0 / S * omega_S^(c0*k2)
    off[3] = all.size();
    {
        const int LR = lr(nlev - 1), R = 1 << LR;
        const uint32_t NB = S >> LR;
        const uint32_t g = root_of_unity(ls + 1);
        const uint32_t s_inv = powmod_c(S, P - 2);
        const std::vector<uint32_t> c0s = SideLevels(ls, lept).last_c0();
        for (int k2 = 0; k2 < R; k2++)
            for (uint32_t b = 0; b < NB; b++) {
                const uint32_t c0 = c0s[b];
                const uint32_t v = mulmod_c(mulmod_c(powmod_c(g, c0), s_inv), pow_root(ls, (uint64_t)c0 * k2 % S));
                all.push_back(tw_of(v));
            }
    }
    // NTT levels 1 .. nlev-2: [k2*L + m] = omega_N^(m*k2)
    int npb = nlr(0);
    for (int l = 1; l < 3; l++) {
        off[3 + l] = all.size();
        if (l <= nlev - 2) {
            const int logn = ls - npb, R = 1 << nlr(l), L = 1 << (logn - nlr(l));
            const uint32_t N = 1u << logn;
            for (int k2 = 0; k2 < R; k2++)
                for (int m = 0; m < L; m++) all.push_back(tw_of(pow_root(logn, (uint64_t)m * k2 % N)));
            npb += nlr(l);
        }
    }
    off[6] = all.size();
}

// Copies columns [0, ncopy) of every input row m to output row 2m on host
// threads (one per ZB_HOST_COPY_DIV hardware threads, 1 … 16), from
// construction until join() (or destruction, on an early error return).
#ifndef ZB_HOST_COPY_DIV
#define ZB_HOST_COPY_DIV 2
#endif
class EvenRowCopy {
   public:
    EvenRowCopy(const uint32_t* in, uint32_t* out, uint32_t k, uint64_t cols, uint64_t ncopy) {
        if (ncopy == 0) return;
        unsigned n = std::thread::hardware_concurrency() / ZB_HOST_COPY_DIV;
        n = n < 1 ? 1 : n > 16 ? 16 : n;
        if (n > k) n = k;
        for (unsigned t = 0; t < n; t++)
            th_.emplace_back([=] {
                for (uint64_t m = (uint64_t)k * t / n; m < (uint64_t)k * (t + 1) / n; m++)
                    memcpy(out + 2 * m * cols, in + m * cols, ncopy * 4);
            });
    }
    void join() {
        for (auto& t : th_)
            if (t.joinable()) t.join();
    }
    ~EvenRowCopy() { join(); }

   private:
    std::vector<std::thread> th_;
};

// Share of the column chunks of a host call whose even output rows return
// over PCIe rather than through the host copy (measured on B200 hosts).
#ifndef ZB_HOST_EVEN_SHARE
#define ZB_HOST_EVEN_SHARE 0.125
#endif
constexpr double HOST_EVEN_DEVICE_SHARE = ZB_HOST_EVEN_SHARE;

// Input bytes per column chunk of a host call (at most MAX_CHUNKS chunks).
#ifndef ZB_HOST_CHUNK_MIB
#define ZB_HOST_CHUNK_MIB 64
#endif

// A wait that nothing completes: the bounded wait gives up and flags it.
__global__ void k_selftest_wait(int* __restrict__ err) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);  // one arrival expected, none ever made
        fence_mbar_init();
    }
    __syncthreads();
    if (!mbar_wait_bounded(&bar, 0) && threadIdx.x == 0) atomicOr(err, 8);
}

static int log2_exact(uint64_t x) {
    if (x == 0 || (x & (x - 1))) return -1;
    int l = 0;
    while ((1ull << l) < x) l++;
    return l;
}

}  // namespace zb

using namespace zb;

extern "C" {

const char* zoda_status_string(zoda_status s) {
    switch (s) {
        case ZODA_OK: return "ok";
        case ZODA_ERR_ARG: return "invalid argument";
        case ZODA_ERR_CUDA: return "CUDA error";
        case ZODA_ERR_NOMEM: return "out of memory";
        case ZODA_ERR_UNSUPPORTED: return "unsupported shape";
        case ZODA_ERR_BUDGET: return "over the admission budget";
        case ZODA_ERR_TIMEOUT: return "timed out";
        case ZODA_ERR_CANCELLED: return "cancelled";
        case ZODA_ERR_STATE: return "invalid state";
    }
    return "unknown status";
}

const char* zoda_last_error(void) { return g_last_error.c_str(); }

uint32_t zoda_max_side(void) { return 1u << LONG_MAX_LOG; }

zoda_status zoda_ctx_create(int device, zoda_ctx** out) {
    if (!out) return ZODA_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    ZB_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return ZODA_ERR_ARG;
    ZB_CUDA(cudaSetDevice(device));
    zoda_ctx* c = new (std::nothrow) zoda_ctx();
    if (!c) return ZODA_ERR_NOMEM;
    c->device = device;
    auto fail = [&](zoda_status s) {
        zoda_ctx_destroy(c);
        return s;
    };
    cudaError_t e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        set_last_error("cudaDeviceGetAttribute", e);
        return fail(ZODA_ERR_CUDA);
    }
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        set_last_error("cudaStreamCreate", e);
        return fail(ZODA_ERR_CUDA);
    }
    for (auto& ev : c->ev) {
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) {
            set_last_error("cudaEventCreate", e);
            return fail(ZODA_ERR_CUDA);
        }
    }
    std::vector<Tw> tw, twist;
    build_tables(tw, twist);
    if ((e = cudaMalloc(&c->tables.tw, tw.size() * sizeof(Tw))) != cudaSuccess ||
        (e = cudaMalloc(&c->tables.twist, twist.size() * sizeof(Tw))) != cudaSuccess) {
        set_last_error("cudaMalloc(tables)", e);
        return fail(ZODA_ERR_NOMEM);
    }
    if ((e = cudaMemcpy(c->tables.tw, tw.data(), tw.size() * sizeof(Tw), cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(c->tables.twist, twist.data(), twist.size() * sizeof(Tw), cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
        set_last_error("cudaMemcpy(tables)", e);
        return fail(ZODA_ERR_CUDA);
    }
    {
        // omega_{2^26}^j for j < 8192: the low half of the two-level root table of the long-column passes
        std::vector<Tw> lo(8192);
        const uint32_t w = root_of_unity(26);
        uint32_t cur = 1;
        for (auto& x : lo) {
            x = Tw{cur, shoup(cur)};
            cur = mulmod_c(cur, w);
        }
        if ((e = cudaMalloc(&c->tables.tw_lo, lo.size() * sizeof(Tw))) != cudaSuccess ||
            (e = cudaMemcpy(c->tables.tw_lo, lo.data(), lo.size() * sizeof(Tw), cudaMemcpyHostToDevice)) !=
                cudaSuccess) {
            set_last_error("cudaMalloc(tw_lo)", e);
            return fail(ZODA_ERR_NOMEM);
        }
    }
    {
        // compact roots of every size up to 8192 points, one size per run of entries
        std::vector<Tw> cmp((size_t)2 << 13, Tw{1, shoup(1)});
        for (int l = 0; l <= 13; l++) {
            const uint32_t w = root_of_unity(l);
            uint32_t cur = 1;
            for (uint32_t j = 0; j < (1u << l); j++) {
                cmp[(1u << l) + j] = Tw{cur, shoup(cur)};
                cur = mulmod_c(cur, w);
            }
        }
        if ((e = cudaMalloc(&c->tables.twc, cmp.size() * sizeof(Tw))) != cudaSuccess ||
            (e = cudaMemcpy(c->tables.twc, cmp.data(), cmp.size() * sizeof(Tw), cudaMemcpyHostToDevice)) !=
                cudaSuccess) {
            set_last_error("cudaMalloc(twc)", e);
            return fail(ZODA_ERR_NOMEM);
        }
    }
    if ((e = cudaMalloc(&c->d_err, sizeof(int))) != cudaSuccess || (e = cudaMemset(c->d_err, 0, sizeof(int))) != cudaSuccess) {
        set_last_error("cudaMalloc(err)", e);
        return fail(ZODA_ERR_NOMEM);
    }
    {
        std::vector<Tw> side;
        for (int ls = 5; ls <= 12; ls++)
            for (int r = 0; r < 2; r++) build_side_tables(ls, r == 0 ? 4 : 3, side, c->tables.side_off[ls][r]);
        if ((e = cudaMalloc(&c->tables.side, side.size() * sizeof(Tw))) != cudaSuccess ||
            (e = cudaMemcpy(c->tables.side, side.data(), side.size() * sizeof(Tw), cudaMemcpyHostToDevice)) !=
                cudaSuccess) {
            set_last_error("cudaMalloc(side tables)", e);
            return fail(ZODA_ERR_NOMEM);
        }
    }
    zoda_status s = extend_init_attributes();
    if (s == ZODA_OK) s = rlc_init_attributes();
    for (int L = FOURSTEP_MIN_LOG; L <= 12 && s == ZODA_OK; L++) s = coset_mid_tables(c, L, L + 1, &c->tables.ext4[L]);
    if (s != ZODA_OK) return fail(s);
    *out = c;
    return ZODA_OK;
}

void zoda_ctx_destroy(zoda_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < zoda_ctx::NHS; i++) {
        if (c->hs[i]) cudaStreamSynchronize(c->hs[i]);
        c->hin[i].release();
        c->hout[i].release();
        if (c->hs[i]) cudaStreamDestroy(c->hs[i]);
    }
    for (auto& row : c->cev)
        for (auto& e : row)
            if (e) cudaEventDestroy(e);
    general_release(c);
    rlc_release(c);
    c->pipe_cnt.release();
    if (c->pipe_done) cudaEventDestroy(c->pipe_done);
    if (c->d_err) cudaFree(c->d_err);
    if (c->tables.tw) cudaFree(c->tables.tw);
    if (c->tables.tw_lo) cudaFree(c->tables.tw_lo);
    if (c->tables.twc) cudaFree(c->tables.twc);
    if (c->tables.twist) cudaFree(c->tables.twist);
    if (c->tables.side) cudaFree(c->tables.side);
    for (auto& ev : c->ev)
        if (ev) cudaEventDestroy(ev);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static zoda_status check_extend_args(const zoda_ctx* ctx, const void* in, const void* out, uint32_t k, uint64_t cols,
                                     int* log_s) {
    if (!ctx || !in || !out) return ZODA_ERR_ARG;
    const int ls = log2_exact(k);
    if (ls < 0) return ZODA_ERR_ARG;
    if (k > zoda_max_side()) return ZODA_ERR_UNSUPPORTED;
    if (cols % 4 != 0) return ZODA_ERR_ARG;
    if (((uintptr_t)in | (uintptr_t)out) & 15) return ZODA_ERR_ARG;
    *log_s = ls;
    return ZODA_OK;
}

zoda_status zoda_extend_device(zoda_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t k, uint64_t cols,
                               void* stream) {
    int ls = 0;
    zoda_status s = check_extend_args(ctx, d_in, d_out, k, cols, &ls);
    if (s != ZODA_OK) return s;
    const uint64_t in_bytes = (uint64_t)k * cols * 4;
    const char* a = (const char*)d_in;
    const char* b = (const char*)d_out;
    if (a < b + 2 * in_bytes && b < a + in_bytes) return ZODA_ERR_ARG;  // overlap
    if (cols == 0) return ZODA_OK;
    ZB_CUDA(cudaSetDevice(ctx->device));
    if (ls > 12) {  // no column fits one pass: three four-step passes
        const uint2* tabs = nullptr;
        {
            std::lock_guard<std::mutex> lock(ctx->mu);  // the context's table map
            if ((s = coset_mid_tables(ctx, ls, ls + 1, &tabs)) != ZODA_OK) return s;
        }
        return long_extend(ctx, ls, tabs, d_in, d_out, cols, (cudaStream_t)stream);
    }
    return launch_extend(ctx, ls, d_in, d_out, cols, (cudaStream_t)stream, ctx->impl);
}

zoda_status zoda_ctx_inject_fault(zoda_ctx* ctx, uint32_t site, uint32_t after) {
    if (!ctx || site > ZODA_FAULT_PIPE_WAIT) return ZODA_ERR_ARG;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ctx->fault_site = site;
    ctx->fault_after = after;
    return ZODA_OK;
}

zoda_status zoda_ctx_set_impl(zoda_ctx* ctx, int impl) {
    if (!ctx || impl < 0 || impl > 3) return ZODA_ERR_ARG;
    ctx->impl = impl;
    return ZODA_OK;
}

zoda_status zoda_selftest_bounded_wait(zoda_ctx* ctx, void* stream) {
    if (!ctx) return ZODA_ERR_ARG;
    ZB_CUDA(cudaSetDevice(ctx->device));
    k_selftest_wait<<<1, 32, 0, (cudaStream_t)stream>>>(ctx->d_err);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

zoda_status zoda_ctx_check(zoda_ctx* ctx) {
    if (!ctx) return ZODA_ERR_ARG;
    ZB_CUDA(cudaSetDevice(ctx->device));
    ZB_CUDA(cudaDeviceSynchronize());
    int flag = 0;
    ZB_CUDA(cudaMemcpy(&flag, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        ZB_CUDA(cudaMemset(ctx->d_err, 0, sizeof(int)));
        set_last_error_text("a kernel gave up a bounded wait");
        return ZODA_ERR_TIMEOUT;
    }
    return ZODA_OK;
}

zoda_status zoda_extend_host(zoda_ctx* ctx, const uint32_t* h_in, uint32_t* h_out, uint32_t k, uint64_t cols,
                             zoda_timing* timing) {
    int ls = 0;
    zoda_status s = check_extend_args(ctx, h_in, h_out, k, cols, &ls);
    if (s != ZODA_OK) return s;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ZB_CUDA(cudaSetDevice(ctx->device));
    if (cols == 0) {
        if (timing) *timing = zoda_timing{0, 0, 0, 0};
        return ZODA_OK;
    }
    const auto t_start = std::chrono::steady_clock::now();
    // Column chunks of ~64 MiB input rotate over NHS streams, so the upload of
    // one chunk, the kernel of another and the download of a third overlap
    // (the two copy directions run on separate engines).
    const uint64_t in_bytes = (uint64_t)k * cols * 4, chunk_bytes = (uint64_t)ZB_HOST_CHUNK_MIB << 20;
    uint64_t nch = (in_bytes + chunk_bytes - 1) / chunk_bytes;
    if (nch > (uint64_t)zoda_ctx::MAX_CHUNKS) nch = zoda_ctx::MAX_CHUNKS;
    if (nch > cols / 4) nch = cols / 4 ? cols / 4 : 1;
    uint64_t cw = (cols + nch - 1) / nch;
    cw = (cw + 3) & ~3ull;
    nch = (cols + cw - 1) / cw;
    // The even output rows are the input rows (the code is systematic): host
    // threads copy them from h_in while the GPU computes the odd rows, which
    // come back compactly. The host copy is the slower of the two (host memory
    // bandwidth; PCIe has time to spare), so the even rows of the last
    // dev_even chunks come back over PCIe instead, from the device's copy of
    // the input: PCIe carries k*cols words up and (1 + dev_even/nch)*k*cols
    // down, instead of k*cols up and 2*k*cols down.
    uint64_t dev_even = (uint64_t)(nch * HOST_EVEN_DEVICE_SHARE + 0.5);
    if (dev_even >= nch) dev_even = nch - 1;
    const uint64_t host_cols = (nch - dev_even) * cw < cols ? (nch - dev_even) * cw : cols;
    EvenRowCopy even(h_in, h_out, k, cols, host_cols);
    uint64_t h2d_bytes = 0, d2h_bytes = 0;
    // Everything that queues copies into the caller's buffers. On a failure the
    // streams are drained before the status is returned, so no copy queued
    // here lands in h_out (or reads h_in) after the call has returned.
    auto pipeline = [&]() -> zoda_status {
        zoda_status r;
        for (int i = 0; i < zoda_ctx::NHS; i++) {
            if (!ctx->hs[i]) ZB_CUDA(cudaStreamCreateWithFlags(&ctx->hs[i], cudaStreamNonBlocking));
            if ((r = ctx->hin[i].ensure((size_t)k * cw * 4)) != ZODA_OK) return r;
            if ((r = ctx->hout[i].ensure((size_t)k * cw * 4)) != ZODA_OK) return r;
        }
        for (uint64_t c = 0; c < nch; c++)
            for (auto& e : ctx->cev[c])
                if (!e) ZB_CUDA(cudaEventCreate(&e));
        const uint2* long_tabs = nullptr;  // sides above 4096: the three-pass extension's factor tables
        if (ls > 12 && (r = coset_mid_tables(ctx, ls, ls + 1, &long_tabs)) != ZODA_OK) return r;
        // all streams start after ev[0]
        ZB_CUDA(cudaEventRecord(ctx->ev[0], ctx->hs[0]));
        for (int i = 1; i < zoda_ctx::NHS; i++) ZB_CUDA(cudaStreamWaitEvent(ctx->hs[i], ctx->ev[0], 0));
        for (uint64_t c = 0; c < nch; c++) {
            const int b = (int)(c % zoda_ctx::NHS);
            cudaStream_t st = ctx->hs[b];
            const uint64_t c0 = c * cw, w = (cols - c0 < cw) ? cols - c0 : cw;
            uint32_t* din = (uint32_t*)ctx->hin[b].p;
            uint32_t* dout = (uint32_t*)ctx->hout[b].p;
            cudaEvent_t* e = ctx->cev[c];
            ZB_CUDA(cudaEventRecord(e[0], st));
            ZB_CUDA(cudaMemcpy2DAsync(din, w * 4, h_in + c0, cols * 4, w * 4, k, cudaMemcpyHostToDevice, st));
            h2d_bytes += (uint64_t)k * w * 4;
            ZB_CUDA(cudaEventRecord(e[1], st));
            if (ctx->fault_site == ZODA_FAULT_HOST_CHUNK && ctx->fault_after-- == 0) {
                ctx->fault_site = 0;
                set_last_error_text("injected fault: zoda_extend_host chunk launch");
                return ZODA_ERR_CUDA;
            }
            r = ls > 12 ? long_extend(ctx, ls, long_tabs, din, dout, w, st, true)
                        : launch_extend(ctx, ls, din, dout, w, st, ctx->impl, true);
            if (r != ZODA_OK) return r;
            ZB_CUDA(cudaEventRecord(e[2], st));
            // odd rows 1, 3, .. of the output: a stride of two output rows
            ZB_CUDA(cudaMemcpy2DAsync(h_out + cols + c0, 2 * cols * 4, dout, w * 4, w * 4, (size_t)k,
                                      cudaMemcpyDeviceToHost, st));
            d2h_bytes += (uint64_t)k * w * 4;
            if (c0 >= host_cols) {  // even rows 0, 2, .. of this chunk: the uploaded input, before the buffer is reused
                ZB_CUDA(cudaMemcpy2DAsync(h_out + c0, 2 * cols * 4, din, w * 4, w * 4, (size_t)k,
                                          cudaMemcpyDeviceToHost, st));
                d2h_bytes += (uint64_t)k * w * 4;
            }
            ZB_CUDA(cudaEventRecord(e[3], st));
        }
        for (int i = 1; i < zoda_ctx::NHS; i++) {
            ZB_CUDA(cudaEventRecord(ctx->ev[1], ctx->hs[i]));
            ZB_CUDA(cudaStreamWaitEvent(ctx->hs[0], ctx->ev[1], 0));
        }
        ZB_CUDA(cudaEventRecord(ctx->ev[3], ctx->hs[0]));
        ZB_CUDA(cudaEventSynchronize(ctx->ev[3]));
        return ZODA_OK;
    };
    s = pipeline();
    if (s != ZODA_OK) {
        for (int i = 0; i < zoda_ctx::NHS; i++)
            if (ctx->hs[i]) cudaStreamSynchronize(ctx->hs[i]);  // drain; the first failure is what is reported
        return s;  // `even` joins its host threads on the way out
    }
    even.join();
    if (timing) {
        float h = 0, kk = 0, d = 0, x = 0;
        for (uint64_t c = 0; c < nch; c++) {
            ZB_CUDA(cudaEventElapsedTime(&x, ctx->cev[c][0], ctx->cev[c][1]));
            h += x;
            ZB_CUDA(cudaEventElapsedTime(&x, ctx->cev[c][1], ctx->cev[c][2]));
            kk += x;
            ZB_CUDA(cudaEventElapsedTime(&x, ctx->cev[c][2], ctx->cev[c][3]));
            d += x;
        }
        timing->h2d_ms = h;
        timing->kernel_ms = kk;
        timing->d2h_ms = d;
        timing->total_ms =
            std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t_start).count();
        timing->h2d_bytes = h2d_bytes;
        timing->d2h_bytes = d2h_bytes;
    }
    return ZODA_OK;
}

}  // extern "C"
