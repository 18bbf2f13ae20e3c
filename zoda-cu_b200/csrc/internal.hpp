// Library-internal declarations shared by the .cu translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/zoda_b200.h"
#include "field.cuh"

namespace zb {

// Per-thread record of the last CUDA failure, returned by zoda_last_error().
void set_last_error(const char* where, cudaError_t e);
void set_last_error_text(const std::string& s);

#define ZB_CUDA(call)                                \
    do {                                             \
        cudaError_t zb_e_ = (call);                  \
        if (zb_e_ != cudaSuccess) {                  \
            ::zb::set_last_error(#call, zb_e_);      \
            return ZODA_ERR_CUDA;                    \
        }                                            \
    } while (0)

// Level structure of the TMA kernels' side 2^ls with level radix 2^lept
// (ExtPlan with schedule 0): full levels of lept bits, the leftover last.
struct SideLevels {
    int nlev, lept, ls;
    SideLevels(int ls_, int lept_) : nlev((ls_ + lept_ - 1) / lept_), lept(lept_), ls(ls_) {}
    int lr(int l) const { return l < nlev - 1 ? lept : ls - lept * (nlev - 1); }
    int last_lr() const { return lr(nlev - 1); }
    // c0 of INTT last-level block b: the digit reversal of slot b * R over the
    // INTT radices, the first coefficient index the block holds
    std::vector<uint32_t> last_c0() const {
        const int LR = last_lr();
        const uint32_t NB = (1u << ls) >> LR;
        std::vector<uint32_t> c0s(NB);
        for (uint32_t b = 0; b < NB; b++) {
            uint32_t slot = b << LR, c0 = 0;
            int sh_in = ls, sh_out = 0;
            for (int l = 0; l < nlev; l++) {
                sh_in -= lr(l);
                c0 |= ((slot >> sh_in) & ((1u << lr(l)) - 1)) << sh_out;
                sh_out += lr(l);
            }
            c0s[b] = c0;
        }
        return c0s;
    }
};

// Grow-only device buffer owned by a context.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    zoda_status ensure(size_t need);
    void release();
};

// Twiddle tables in HBM, built once per context:
//   tw[j]            = omega_8192^j with its Shoup companion, j in [0, 8192)
//   twist[S + i]     = omega_2S^i * S^-1, i in [0, S), for S = 1 .. 4096
struct Tables {
    Tw* tw = nullptr;
    Tw* tw_lo = nullptr;  // omega_{2^26}^j, j in [0, 8192): with tw, every 2^26-th root of unity
    Tw* twc = nullptr;    // compact roots: twc[2^l + j] = omega_{2^l}^j, l = 0 .. 13
    Tw* twist = nullptr;
    // per-side level tables of the TMA-staged kernels (log2 side 5..12), one buffer
    Tw* side = nullptr;
    // factor tables of the four-step extension plan for log2 side 10..12 (in the
    // context's coset table map; built at creation so launches need no lock)
    const uint2* ext4[13] = {};
    // [log_s][radix 16, radix 8][intt0, intt1, intt2, ntt0, ntt1, ntt2, end] entry offsets
    size_t side_off[13][2][8] = {};
};

}  // namespace zb

struct zoda_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    zb::Tables tables;
    int* d_err = nullptr;  // device flag a kernel sets when a bounded wait gives up
    int impl = 0;          // zoda_extend_impl
    zoda_plan plan[13] = {};  // per log2 side, valid where planned[] is set
    bool planned[13] = {};
    // host-call staging: NHS streams, one input and one output buffer each, and
    // 4 timing events per chunk for up to MAX_CHUNKS chunks
#ifndef ZB_HOST_STREAMS
#define ZB_HOST_STREAMS 3
#endif
#ifndef ZB_HOST_MAX_CHUNKS
#define ZB_HOST_MAX_CHUNKS 64
#endif
    static constexpr int NHS = ZB_HOST_STREAMS;
    static constexpr int MAX_CHUNKS = ZB_HOST_MAX_CHUNKS;
    cudaStream_t hs[NHS] = {};
    zb::DevBuf hin[NHS], hout[NHS];
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t cev[MAX_CHUNKS][4] = {};
    std::mutex mu;  // serialises host calls on one context
    // armed fault site (zoda_ctx_inject_fault) and the passes left before it fires
    uint32_t fault_site = 0, fault_after = 0;
    // encode of any (k, n) and erasure decoder (general.cu): two column-chunk
    // scratch matrices, per-pattern tables, coset twist tables keyed by
    // (log2 n_k, log2 n_kn), and an event after each call's last use of them
    zb::DevBuf gen_a, gen_b, gen_tab, gen_small;
    std::map<int, zb::DevBuf> coset_tabs;
    cudaEvent_t gen_done = nullptr;
    // the pipelined four-step launch (fourstep.cu): per-chunk counters, their lock,
    // and an event after the last launch that used them
    zb::DevBuf pipe_cnt;
    std::mutex pipe_mu;
    cudaEvent_t pipe_done = nullptr;
    // RLC consumers (rlc.cu): canonical coefficient table, row
    // accumulators and the check's matrices, under their own lock
    zb::DevBuf rlc_w, rlc_acc, rlc_d, rlc_e, rlc_f, rlc_cnt;
    std::mutex rlc_mu;
};

namespace zb {
// Launches the fused extension kernel for side 2^log_s (0 <= log_s <= 12).
// impl: 0 = the side's plan (tuned, or the default), 1 = direct-load kernel,
// 2 = TMA-staged kernel (sides 32..4096), both with default knobs. With
// odd_only the kernel writes only the odd rows, as a compact [S][cols] out.
// in_rows < S: input rows past it are zeros (never read); out_rows < 2S: rows
// of the interleaved output past it are not written; 0 means S and 2S.
zoda_status launch_extend(const zoda_ctx* ctx, int log_s, const uint32_t* in, uint32_t* out, uint64_t cols,
                          cudaStream_t st, int impl = 0, bool odd_only = false, uint32_t in_rows = 0,
                          uint32_t out_rows = 0);
// The plan a side runs with impl 0 and no tuning.
zoda_plan default_plan(int log_s);
// ZODA_OK when the plan can run for this side.
zoda_status check_plan(int log_s, const zoda_plan& p);
// Launches one explicit plan.
zoda_status launch_plan(const zoda_ctx* ctx, int log_s, const zoda_plan& p, const uint32_t* in, uint32_t* out,
                        uint64_t cols, cudaStream_t st, bool odd_only = false, uint32_t in_rows = 0,
                        uint32_t out_rows = 0);
// The L2 promotion a side's TMA loads use on this context (for the batch maps).
int side_l2_promo(const zoda_ctx* ctx, int log_s);
// Sets the dynamic shared memory attribute of every extension instantiation.
zoda_status extend_init_attributes();
// Frees what the general encode / decoder left in the context.
void general_release(zoda_ctx* ctx);
// Sets the dynamic shared memory attribute of the RLC row kernel.
zoda_status rlc_init_attributes();
// Frees the RLC consumers' scratch.
void rlc_release(zoda_ctx* ctx);

// Long columns (fourstep.cu): transforms of 2^13 .. 2^26 points in four-step passes.
constexpr int LONG_MIN_LOG = 13, LONG_MAX_LOG = 26;
// The decoder's erasure-pattern tables cost O(2k * erasures), so it stops at
// codewords of 2^18 rows (k = 131072).
constexpr int LONG_RECOVER_MAX_LOG = 18;
// Legacy layout: B = [2^L][w4] (polynomials in columns) -> natural-order
// transform in A ([2^L][w4]); B is overwritten; inverse roots and `scale` when inv.
zoda_status long_cols_ntt(const zoda_ctx* ctx, uint32_t* B, uint32_t* A, int L, uint64_t w4, bool inv, Tw scale,
                          cudaStream_t st);
// The coset factor tables of the long encode over 2^ln points with n_k = 2^L (built
// once, kept in ctx->coset_tabs: call it holding ctx->mu).
zoda_status coset_mid_tables(zoda_ctx* ctx, int L, int ln, const uint2** tabs);
// Extension of a 2^L square (10 <= L <= 26) in three passes, the odd output rows as
// scratch; odd_only: out is the compact [S][cols] odd rows (the even rows are the input).
// tabs = coset_mid_tables(ctx, L, L + 1).
// shape: the launch shape of the passes (fourstep.cuh, StepShape). pipelined (L <=
// PIPE_MAX_LOG): one persistent launch runs the passes column chunk by column chunk
// (k_fourstep_pipe) instead of three launches over the whole square.
constexpr int PIPE_MAX_LOG = 14;
zoda_status long_extend(const zoda_ctx* ctx, int L, const uint2* tabs, const uint32_t* in, uint32_t* out,
                        uint64_t cols, cudaStream_t st, bool odd_only = false, int shape = 0,
                        bool pipelined = false);
// The four-step launch shape of a plan's (radix, ctas); staged adds STEP_STAGED (the
// passes copy each next tile in by cp.async while the current one computes).
constexpr int STEP_STAGED = 8;
int fourstep_shape(int radix, int ctas, bool staged = false);
// Smallest side (log2) the four-step plan covers.
constexpr int FOURSTEP_MIN_LOG = 10;
// Cosets c >= 1 of the encode of k data rows with n parity rows, n_k = next_pow2(k)
// in [2^13, 2^26], on the context's scratch (the caller holds ctx->mu and copies coset 0).
zoda_status long_encode(zoda_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t k, uint32_t n, uint64_t cols,
                        cudaStream_t st);
// k-of-2k recovery for 2k = 2^L, LONG_MIN_LOG < L <= LONG_RECOVER_MAX_LOG (the caller holds ctx->mu).
zoda_status long_recover(zoda_ctx* ctx, const uint32_t* d_code, const std::vector<uint32_t>& erased_roots,
                         uint32_t k, uint64_t cols, uint32_t* d_data, unsigned long long* d_cnt, cudaStream_t st);
}  // namespace zb
