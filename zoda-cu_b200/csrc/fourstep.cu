// Long columns: transforms of 2^13 .. 2^26 points as four-step passes
// (fourstep.cuh), behind the legacy transform (legacy.cu), the extension of
// squares above side 4096 (api.cu), the encode of any shape with n_k above
// 4096 and the erasure decoder with 2k above 8192 (general.cu).
//
// Every transform of S = N1 * N2 points (N1 = 2^floor(L/2), N2 = 2^ceil(L/2))
// is a strided pass over N1 points and a block pass over N2 points. Chains of
// transforms fuse the block pass of one with the strided pass of the next
// (k_step2), so
//   * the extension (INTT, twist, NTT) is 3 passes: strided INTT pass A, one
//     block pass (INTT pass B, twist, NTT pass A), strided NTT pass B;
//   * the decoder's four transforms are 5 passes.
// Passes read and write whole columns of a matrix view, so they run on column
// chunks with a scratch matrix, or in place: a square's extension keeps its
// intermediate results in the output's odd rows (the rows the last pass
// fills), so it needs no memory beyond the input and the output.
#include <algorithm>
#include <vector>

#include "fourstep.cuh"
#include "internal.hpp"

namespace zb {
namespace {

// Grid of a pass: one round of tiles over the resident CTAs, at most.
inline unsigned pass_grid(const zoda_ctx* ctx, uint64_t ntiles, int minb) {
    const uint64_t cap = (uint64_t)ctx->sm_count * minb;
    return (unsigned)(ntiles < cap ? ntiles : cap);
}

// One pass of any features (F = SF_ALL), or of a feature set the caller fixes.
// Passes compiled with SF_FOLD read their level twiddles from the compact table.
template <int F>
inline const Tw* pass_tw(const zoda_ctx* ctx) {
    return (F & SF_FOLD) ? ctx->tables.twc : ctx->tables.tw;
}

template <int LOG_N, bool INV, int SHAPE, int F = SF_ALL>
zoda_status step_t(const zoda_ctx* ctx, const StepArgs& a, cudaStream_t st) {
    using SH = StepShape<LOG_N, SHAPE>;
    using PL = typename SH::PL;
    const uint64_t ntiles = (a.nquads + PL::Q4 - 1) / PL::Q4;
    if (ntiles == 0) return ZODA_OK;
    if (PL::SMEM > 0)
        ZB_CUDA(cudaFuncSetAttribute(k_step<LOG_N, INV, SHAPE, F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)PL::SMEM));
    k_step<LOG_N, INV, SHAPE, F><<<pass_grid(ctx, ntiles, SH::MINB), PL::THREADS, PL::SMEM, st>>>(
        a, ntiles, pass_tw<F>(ctx), ctx->tables.tw_lo);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

template <int LOG_N, bool INV1, int SHAPE, int F = SF_ALL>
zoda_status step2_t(const zoda_ctx* ctx, const StepArgs& a, cudaStream_t st) {
    using SH = StepShape<LOG_N, SHAPE>;
    using PL = typename SH::PL;
    const uint64_t ntiles = (a.nquads + PL::Q4 - 1) / PL::Q4;
    if (ntiles == 0) return ZODA_OK;
    if (PL::SMEM > 0)
        ZB_CUDA(cudaFuncSetAttribute(k_step2<LOG_N, INV1, !INV1, SHAPE, F>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::SMEM));
    k_step2<LOG_N, INV1, !INV1, SHAPE, F><<<pass_grid(ctx, ntiles, SH::MINB), PL::THREADS, PL::SMEM, st>>>(
        a, ntiles, pass_tw<F>(ctx), ctx->tables.tw_lo);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

// The staged pass (k_step_st): two tiles of shared memory, the next one arriving
// by cp.async while the current one computes.
template <int LOG_N, bool INV, bool TWO, int SHAPE, int F>
zoda_status step_st_t(const zoda_ctx* ctx, const StepArgs& a, cudaStream_t st) {
    using SH = StepShape<LOG_N, SHAPE>;
    using PL = typename SH::PL;
    static_assert(SH::MINB_ST >= 1, "two tiles fit one SM");
    const uint64_t ntiles = (a.nquads + PL::Q4 - 1) / PL::Q4;
    if (ntiles == 0) return ZODA_OK;
    constexpr size_t smem = 2 * PL::SMEM;
    ZB_CUDA(cudaFuncSetAttribute(k_step_st<LOG_N, INV, TWO, SHAPE, F>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    k_step_st<LOG_N, INV, TWO, SHAPE, F><<<pass_grid(ctx, ntiles, SH::MINB_ST), PL::THREADS, smem, st>>>(
        a, ntiles, pass_tw<F>(ctx), ctx->tables.tw_lo);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

// One transform (two = false) or two fused transforms (two: INTT then NTT when
// inv, else NTT then INTT) of 2^log_n points (5 <= log_n <= 13) per virtual
// quad, every feature available, one CTA per SM.
zoda_status run_pass(const zoda_ctx* ctx, int log_n, bool two, bool inv, const StepArgs& a, cudaStream_t st) {
    switch (log_n) {
#define ZB_CASE(L)                                                                                     \
    case L:                                                                                            \
        if (two) return inv ? step2_t<L, true, 0>(ctx, a, st) : step2_t<L, false, 0>(ctx, a, st);     \
        return inv ? step_t<L, true, 0>(ctx, a, st) : step_t<L, false, 0>(ctx, a, st);
        ZB_CASE(5) ZB_CASE(6) ZB_CASE(7) ZB_CASE(8) ZB_CASE(9) ZB_CASE(10) ZB_CASE(11) ZB_CASE(12) ZB_CASE(13)
#undef ZB_CASE
        default: return ZODA_ERR_UNSUPPORTED;
    }
}
zoda_status run_step(const zoda_ctx* ctx, int log_n, bool inv, const StepArgs& a, cudaStream_t st) {
    return run_pass(ctx, log_n, false, inv, a, st);
}
zoda_status run_step2(const zoda_ctx* ctx, int log_n, bool inv1, const StepArgs& a, cudaStream_t st) {
    return run_pass(ctx, log_n, true, inv1, a, st);
}

// The passes of a square's extension (long_extend, sides up to 2^PIPE_MAX_LOG), with
// only the features each one uses: PASS 0 = the strided INTT pass (twiddle, even-row
// copy), 1 = the block pass (middle factors, twiddle), 2 = the strided NTT pass.
// shape: 0..3 (fourstep.cuh StepShape), plus STEP_STAGED for the staged form.
template <int LOG_N, int PASS, int SHAPE>
zoda_status ext_pass_t(const zoda_ctx* ctx, bool staged, const StepArgs& a, cudaStream_t st) {
    constexpr int F = PASS == 0 ? SF_EXT_A : PASS == 1 ? SF_EXT_M : SF_EXT_B;
    constexpr bool INV = PASS < 2;
    if constexpr (SHAPE >= 1) {
        if (staged) return step_st_t<LOG_N, INV, PASS == 1, SHAPE, F>(ctx, a, st);
    }
    if (staged) return ZODA_ERR_UNSUPPORTED;
    if constexpr (PASS == 1) return step2_t<LOG_N, true, SHAPE, F | SF_PASS_GROUPS>(ctx, a, st);
    else return step_t<LOG_N, INV, SHAPE, F | SF_PASS_GROUPS>(ctx, a, st);
}
template <int LOG_N, int PASS>
zoda_status ext_pass_shape(const zoda_ctx* ctx, int shape, const StepArgs& a, cudaStream_t st) {
    const bool staged = shape & STEP_STAGED;
    switch (shape & ~STEP_STAGED) {
        case 1: return ext_pass_t<LOG_N, PASS, 1>(ctx, staged, a, st);
        case 2: return ext_pass_t<LOG_N, PASS, 2>(ctx, staged, a, st);
        case 3: return ext_pass_t<LOG_N, PASS, 3>(ctx, staged, a, st);
        case 4: return ext_pass_t<LOG_N, PASS, 4>(ctx, staged, a, st);
        default: return ext_pass_t<LOG_N, PASS, 0>(ctx, staged, a, st);
    }
}
template <int PASS>
zoda_status ext_pass(const zoda_ctx* ctx, int log_n, int shape, const StepArgs& a, cudaStream_t st) {
    switch (log_n) {
        case 5: return ext_pass_shape<5, PASS>(ctx, shape, a, st);
        case 6: return ext_pass_shape<6, PASS>(ctx, shape, a, st);
        case 7: return ext_pass_shape<7, PASS>(ctx, shape, a, st);
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

constexpr uint64_t NO_LIMIT = ~0ull;

// Arguments with no limits, factors or twiddles.
StepArgs plain_args(View in, View out, uint32_t qpc, uint64_t nquads) {
    StepArgs a{};
    a.in = in;
    a.out = out;
    a.qpc = qpc;
    a.nquads = nquads;
    a.qlim = ~0u;
    a.in_limit = NO_LIMIT;
    a.out_limit = NO_LIMIT;
    a.scale = Tw{1u, shoup(1u)};
    return a;
}

inline uint2 shoup_pair(uint32_t w) { return make_uint2(w, shoup(w)); }

// Device copy of a host table, kept in the context under `key`.
zoda_status upload_table(zoda_ctx* ctx, int key, const std::vector<uint2>& h, const uint2** out) {
    DevBuf& b = ctx->coset_tabs[key];
    if (!b.p) {
        zoda_status s = b.ensure(std::max<size_t>(1, h.size()) * sizeof(uint2));
        if (s != ZODA_OK) return s;
        ZB_CUDA(cudaMemcpy(b.p, h.data(), h.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    }
    *out = (const uint2*)b.p;
    return ZODA_OK;
}

}  // namespace

// Factor tables of the block passes that turn INTT coefficients into the NTT
// inputs of the encode over 2^ln points with n_k = 2^L: for coset c in
// [1, 2^(ln - L)), coefficient i = k1 + N1*k2 is multiplied by base^i / n_k,
// base = omega_{2^ln}^c, split into [k1: base^k1 / n_k] (N1 entries) and
// [k2: base^(N1*k2)] (N2 entries). Coset c's two tables sit at
// *tabs + (c - 1) * (N1 + N2); built once per (L, ln). The extension is
// ln = L + 1, c = 1 (base = g = omega_2S); for it (L <= PIPE_MAX_LOG) three
// tables of 2^L entries follow at *tabs + N1 + N2: the product table [k2][k1],
// and the post-factor tables of the extension's INTT pass A ([i2][k1]) and of
// its block pass ([k1][m1]).
zoda_status coset_mid_tables(zoda_ctx* ctx, int L, int ln, const uint2** tabs) {
    const int L1 = L / 2, L2 = L - L1;
    const uint32_t N1 = 1u << L1, N2 = 1u << L2;
    const uint64_t cosets = (1ull << (ln - L)) - 1;
    DevBuf& b = ctx->coset_tabs[-(300000000 + L * 32 + (ln - L))];  // disjoint from the other keys
    if (!b.p) {
        std::vector<uint2> h;
        h.reserve(cosets * (N1 + N2));
        const uint32_t sinv = powmod_c(1u << L, P - 2), wn = root_of_unity(ln);
        for (uint64_t c = 1, base = wn; c <= cosets; c++, base = mulmod_c((uint32_t)base, wn)) {
            for (uint32_t k1 = 0, x = sinv; k1 < N1; k1++, x = mulmod_c(x, (uint32_t)base)) h.push_back(shoup_pair(x));
            const uint32_t step = powmod_c((uint32_t)base, N1);
            for (uint32_t k2 = 0, x = 1; k2 < N2; k2++, x = mulmod_c(x, step)) h.push_back(shoup_pair(x));
        }
        if (ln == L + 1 && L <= PIPE_MAX_LOG) {
            // the extension's two factors as one table [k2][k1] = f1[k1] * f2[k2]:
            // one product per coefficient in its block pass instead of two
            const size_t f2 = N1;
            for (uint32_t k2 = 0; k2 < N2; k2++)
                for (uint32_t k1 = 0; k1 < N1; k1++) h.push_back(shoup_pair(mulmod_c(h[k1].x, h[f2 + k2].x)));
            // the output twiddles of its two transforms' first passes as post-factor
            // tables: INTT pass A, [i2][k1] = omega_S^-(i2 * k1) (i2 < N2, k1 < N1);
            // NTT pass A in the block pass, [k1][m1] = omega_S^(k1 * m1) (k1 < N1, m1 < N2)
            const uint32_t wS = root_of_unity(L), wSi = powmod_c(wS, P - 2);
            for (uint32_t i2 = 0; i2 < N2; i2++)
                for (uint32_t k1 = 0, x = 1, st = powmod_c(wSi, i2); k1 < N1; k1++, x = mulmod_c(x, st))
                    h.push_back(shoup_pair(x));
            for (uint32_t k1 = 0; k1 < N1; k1++)
                for (uint32_t m1 = 0, x = 1, st = powmod_c(wS, k1); m1 < N2; m1++, x = mulmod_c(x, st))
                    h.push_back(shoup_pair(x));
        }
        zoda_status s = b.ensure(h.size() * sizeof(uint2));
        if (s != ZODA_OK) return s;
        ZB_CUDA(cudaMemcpy(b.p, h.data(), h.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    }
    *tabs = (const uint2*)b.p;
    return ZODA_OK;
}

// Legacy layout: B holds [n][w4] (polynomials in columns), n = 2^L. Leaves the
// natural-order transform in A ([n][w4]); B is overwritten. Inverse roots and
// the scale when inv.
zoda_status long_cols_ntt(const zoda_ctx* ctx, uint32_t* B, uint32_t* A, int L, uint64_t w4, bool inv, Tw scale,
                          cudaStream_t st) {
    if (L < LONG_MIN_LOG || L > LONG_MAX_LOG || w4 % 4) return ZODA_ERR_UNSUPPORTED;
    const int L1 = L / 2, L2 = L - L1;
    const uint64_t N1 = 1ull << L1, N2 = 1ull << L2;
    const uint32_t qpc = (uint32_t)(w4 / 4);
    // pass A, in place: wide rows i1 (N2 rows apart), column block i2
    StepArgs pa = plain_args(View{B, N2 * w4, w4}, View{B, N2 * w4, w4}, qpc, N2 * qpc);
    pa.tw_log = L;
    pa.tw_inv = inv;
    zoda_status s = run_step(ctx, L1, inv, pa, st);
    if (s != ZODA_OK) return s;
    // pass B: block k1 (N2 consecutive rows) -> rows k1 + N1*k2 of A
    StepArgs pb = plain_args(View{B, w4, N2 * w4}, View{A, N1 * w4, w4}, qpc, N1 * qpc);
    pb.use_scale = inv;
    pb.scale = scale;
    return run_step(ctx, L2, inv, pb, st);
}

// The same three passes in one persistent launch, column chunk by column chunk
// (k_fourstep_pipe), so each chunk's intermediate stays in L2 between its passes.
// The most tiles one work item of the pipelined launch covers, and the pipeline
// depth in units of the items the CTAs hold (measured at side 4096, CUDA events,
// on one box each: 1 tile and depth 2 12.96 ms, 4 and 2 12.82, 8 and 2 12.72-12.82,
// 8 and 1 12.96-13.03, 1 and 1 13.05, 2 and 1 12.71).
#ifndef ZB_PIPE_TILES
#define ZB_PIPE_TILES 2
#endif
static_assert(ZB_PIPE_TILES >= 1 && ZB_PIPE_TILES <= 32 && (ZB_PIPE_TILES & (ZB_PIPE_TILES - 1)) == 0,
              "tiles per work item: a power of two that divides every pass's tile count");
#ifndef ZB_PIPE_DEPTH_HELD
#define ZB_PIPE_DEPTH_HELD 1
#endif

template <int L1, int L2, int SHAPE, bool STAGE>
zoda_status pipe_t(const zoda_ctx* ctx, const StepArgs pass[3], uint64_t cols, cudaStream_t st) {
    using PS = PipeShape<L1, L2, SHAPE>;
    using PA = typename PS::A::PL;
    using PM = typename PS::M::PL;
    const uint64_t quads = cols / 4;
    const uint64_t nch = (quads + PS::CQ - 1) / PS::CQ;
    PipeArgs pa{};
    for (int i = 0; i < 3; i++) pa.pass[i] = pass[i];
    const uint64_t NB2 = 1ull << L2, NB1 = 1ull << L1;  // column blocks of the strided / block passes
    pa.pass[0].qpc = pa.pass[2].qpc = pa.pass[1].qpc = PS::CQ;
    pa.pass[0].nquads = pa.pass[2].nquads = NB2 * PS::CQ;
    pa.pass[1].nquads = NB1 * PS::CQ;
    // tiles per work item: more tiles per item spread the item's fixed costs (the
    // completion fence and count, the dependency wait) over more work, as long as
    // the launch keeps at least 16 items per resident CTA (small squares would
    // otherwise leave CTAs idle at the end); every pass has a power-of-two tile
    // count of at least 32 per chunk
    const uint64_t tiles_a = NB2 * PS::CQ / PA::Q4, tiles_m = NB1 * PS::CQ / PM::Q4;
    const uint64_t resident = (uint64_t)ctx->sm_count * (STAGE ? PS::MINB_ST : PS::MINB);
    uint32_t tpi = 1;
    while (!STAGE && tpi < (uint32_t)ZB_PIPE_TILES &&
           nch * (2 * tiles_a + tiles_m) / (2 * tpi) >= 16 * resident)
        tpi *= 2;
    pa.tpi = tpi;
    pa.tiles[0] = pa.tiles[2] = (uint32_t)(tiles_a / tpi);
    pa.tiles[1] = (uint32_t)(tiles_m / tpi);
    pa.chunk_u32 = 4ull * PS::CQ;
    pa.nchunks = (uint32_t)nch;
    pa.last_qlim = (uint32_t)(quads - (nch - 1) * PS::CQ);
    constexpr int minb = STAGE ? PS::MINB_ST : PS::MINB;
    static_assert(minb >= 1, "the CTA's buffers fit one SM");
    constexpr size_t smem = (STAGE ? 2 : 1) * PS::SMEM;
    const uint64_t grid = (uint64_t)ctx->sm_count * minb;
    const uint64_t per_round = (uint64_t)pa.tiles[0] + pa.tiles[1] + pa.tiles[2];
    // depth: enough rounds between a chunk's passes that its earlier tiles are
    // mostly done before the later ones are dealt, measured in the items the CTAs
    // hold at once (the current one and the two drawn ahead): ZB_PIPE_DEPTH_HELD
    // times that many items. A deeper pipeline waits less but keeps more chunks'
    // intermediates in flight, and those stay in L2 only while they fit.
    uint64_t depth = ((uint64_t)ZB_PIPE_DEPTH_HELD * 3 * grid + per_round - 1) / per_round;
    if (depth < 1) depth = 1;
    pa.depth = (uint32_t)depth;
    if (nch > (1u << 30) || (nch + 2 * depth) * per_round + 3 * grid >= (1ull << 31)) return ZODA_ERR_UNSUPPORTED;
    zoda_ctx* mc = const_cast<zoda_ctx*>(ctx);  // the pipeline's counters and ordering event
    std::lock_guard<std::mutex> lock(mc->pipe_mu);
    const size_t cbytes = (size_t)(1 + 2 * nch) * sizeof(uint32_t);
    // a larger square replaces the counters: the launch before, on whatever
    // stream, finishes with the old ones first
    if (mc->pipe_done && cbytes > mc->pipe_cnt.bytes) ZB_CUDA(cudaEventSynchronize(mc->pipe_done));
    zoda_status s = mc->pipe_cnt.ensure(cbytes);
    if (s != ZODA_OK) return s;
    if (!mc->pipe_done) ZB_CUDA(cudaEventCreateWithFlags(&mc->pipe_done, cudaEventDisableTiming));
    pa.counters = (uint32_t*)mc->pipe_cnt.p;
    pa.err = ctx->d_err;
    if (mc->fault_site == ZODA_FAULT_PIPE_WAIT && mc->fault_after-- == 0) {
        mc->fault_site = 0;
        pa.wait_extra = 1;  // a count no chunk reaches: every dependency wait runs out
    }
    // launches on other streams share the counters: each waits for the one before
    ZB_CUDA(cudaStreamWaitEvent(st, mc->pipe_done, 0));
    ZB_CUDA(cudaMemsetAsync(pa.counters, 0, cbytes, st));
    ZB_CUDA(cudaFuncSetAttribute(k_fourstep_pipe<L1, L2, SHAPE, STAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    k_fourstep_pipe<L1, L2, SHAPE, STAGE><<<(unsigned)grid, PS::THREADS, smem, st>>>(pa, ctx->tables.twc,
                                                                                    ctx->tables.tw_lo);
    ZB_CUDA(cudaGetLastError());
    ZB_CUDA(cudaEventRecord(mc->pipe_done, st));
    return ZODA_OK;
}

template <int L1, int L2>
zoda_status pipe_shape(const zoda_ctx* ctx, int shape, const StepArgs pass[3], uint64_t cols, cudaStream_t st) {
    const bool staged = shape & STEP_STAGED;
    switch (shape & ~STEP_STAGED) {
        case 1: return staged ? pipe_t<L1, L2, 1, true>(ctx, pass, cols, st) : pipe_t<L1, L2, 1, false>(ctx, pass, cols, st);
        case 2: return staged ? pipe_t<L1, L2, 2, true>(ctx, pass, cols, st) : pipe_t<L1, L2, 2, false>(ctx, pass, cols, st);
        case 3: return staged ? pipe_t<L1, L2, 3, true>(ctx, pass, cols, st) : pipe_t<L1, L2, 3, false>(ctx, pass, cols, st);
        case 4: return staged ? pipe_t<L1, L2, 4, true>(ctx, pass, cols, st) : pipe_t<L1, L2, 4, false>(ctx, pass, cols, st);
        default: return staged ? ZODA_ERR_UNSUPPORTED : pipe_t<L1, L2, 0, false>(ctx, pass, cols, st);
    }
}

// Extension of a square of side S = 2^L in three passes, 10 <= L <= 26 (above
// 4096 no column fits one pass; from 1024 to 4096 it is an alternative plan): in
// [S][cols] -> out [2S][cols]. The first pass writes the even rows (the input)
// as it loads them; the odd rows hold the intermediate matrices. `tabs` =
// coset_mid_tables(ctx, L, L + 1).
int fourstep_shape(int radix, int ctas, bool staged) {
    if (ctas <= 1) return 0;
    const int shape = radix == 16 ? 1 : radix == 4 ? 4 : ctas == 2 ? 2 : 3;
    return shape | (staged ? STEP_STAGED : 0);
}

zoda_status long_extend(const zoda_ctx* ctx, int L, const uint2* tabs, const uint32_t* in, uint32_t* out,
                        uint64_t cols, cudaStream_t st, bool odd_only, int shape, bool pipelined) {
    if (L < FOURSTEP_MIN_LOG || L > LONG_MAX_LOG || cols % 4) return ZODA_ERR_UNSUPPORTED;
    if (pipelined && L > PIPE_MAX_LOG) return ZODA_ERR_UNSUPPORTED;
    if (cols == 0) return ZODA_OK;
    const int L1 = L / 2, L2 = L - L1;
    const uint64_t N1 = 1ull << L1, N2 = 1ull << L2;
    const uint32_t qpc = (uint32_t)(cols / 4);
    zoda_status s;
    const uint2 *cbtab = tabs, *ktab = tabs + N1;
    // odd rows: row r at odd + r * op (interleaved [2S][cols], or compact [S][cols] with odd_only)
    uint32_t* odd = odd_only ? out : out + cols;
    const uint64_t op = odd_only ? cols : 2 * cols;
    StepArgs pass[3];
    // pass A (INTT over i1): input rows N2*i1 + i2 -> odd row N2*k1 + i2; the
    // loaded rows also go to the even rows
    StepArgs& pa = pass[0];
    pa = plain_args(View{const_cast<uint32_t*>(in), N2 * cols, cols}, View{odd, N2 * op, op}, qpc, N2 * qpc);
    const uint64_t S = 1ull << L;
    if (L <= PIPE_MAX_LOG) {
        pa.post = FTab{tabs + N1 + N2 + S, 1, (uint32_t)N1};  // omega_S^-(i2 * k1) at [i2][k1]
    } else {
        pa.tw_log = L;
        pa.tw_inv = 1;
    }
    if (!odd_only) pa.copy = View{out, 2 * N2 * cols, 2 * cols};
    // block pass, in place: INTT pass B over i2 in block k1, the twist g^i / S
    // (g = omega_2S), NTT pass A over the block's coefficients (decomposition
    // (N2, N1)), its twiddle omega_S^(k1 * m1)
    StepArgs& pm = pass[1];
    pm = plain_args(View{odd, op, N2 * op}, View{odd, op, N2 * op}, qpc, N1 * qpc);
    if (L <= PIPE_MAX_LOG) {
        pm.mid1 = FTab{tabs + N1 + N2, (uint32_t)N1, 1};      // [k2][k1] products
        pm.post = FTab{tabs + N1 + N2 + 2 * S, 1, (uint32_t)N2};  // omega_S^(k1 * m1) at [k1][m1]
    } else {
        pm.mid1 = FTab{cbtab, 0, 1};
        pm.mid2 = FTab{ktab, 1, 0};
        pm.tw_log = L;
    }
    // pass B of the NTT, in place: wide rows j2 of column block m1 -> odd row m1 + N2*m2
    StepArgs& pb = pass[2];
    pb = plain_args(View{odd, N2 * op, op}, View{odd, N2 * op, op}, qpc, N2 * qpc);
    if (pipelined) {
        switch (L) {
            case 10: return pipe_shape<5, 5>(ctx, shape, pass, cols, st);
            case 11: return pipe_shape<5, 6>(ctx, shape, pass, cols, st);
            case 12: return pipe_shape<6, 6>(ctx, shape, pass, cols, st);
            case 13: return pipe_shape<6, 7>(ctx, shape, pass, cols, st);
            case 14: return pipe_shape<7, 7>(ctx, shape, pass, cols, st);
            default: return ZODA_ERR_UNSUPPORTED;
        }
    }
    if (L <= PIPE_MAX_LOG) {
        if ((s = ext_pass<0>(ctx, L1, shape, pa, st)) != ZODA_OK) return s;
        if ((s = ext_pass<1>(ctx, L2, shape, pm, st)) != ZODA_OK) return s;
        return ext_pass<2>(ctx, L1, shape, pb, st);
    }
    if ((s = run_step(ctx, L1, true, pa, st)) != ZODA_OK) return s;
    if ((s = run_step2(ctx, L2, true, pm, st)) != ZODA_OK) return s;
    return run_step(ctx, L1, false, pb, st);
}

// Cosets c >= 1 of the encode for n_k = 2^lp > 4096 (general.cu copies coset 0,
// the data): per column chunk, the INTT's strided pass into the scratch, then
// per coset a block pass (INTT pass B, the coset twist, NTT pass A) and the
// NTT's strided pass into output rows R*m + c.
zoda_status long_encode(zoda_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t k, uint32_t n, uint64_t cols,
                        cudaStream_t st) {
    uint64_t P_ = 1, N = 1;
    while (P_ < k) P_ <<= 1;
    while (N < (uint64_t)k + n) N <<= 1;
    int lp = 0, ln = 0;
    while ((1ull << lp) < P_) lp++;
    while ((1ull << ln) < N) ln++;
    if (lp < LONG_MIN_LOG || lp > LONG_MAX_LOG) return ZODA_ERR_UNSUPPORTED;
    const uint64_t R = N / P_, rows_out = (uint64_t)k + n;
    if (R == 1 || cols == 0) return ZODA_OK;
    const int L1 = lp / 2, L2 = lp - L1;
    const uint64_t N1 = 1ull << L1, N2 = 1ull << L2;
    // column chunk: one scratch matrix of P_ rows (two when R > 2: the INTT's
    // first pass is kept for every coset), at most 256 MiB each
    uint64_t w0 = ((64ull << 20) / P_) & ~3ull;
    if (w0 < 4) w0 = 4;
    if (w0 > cols) w0 = cols;
    zoda_status s;
    if ((s = ctx->gen_a.ensure(P_ * w0 * 4)) != ZODA_OK) return s;
    if (R > 2 && (s = ctx->gen_b.ensure(P_ * w0 * 4)) != ZODA_OK) return s;
    uint32_t* A = (uint32_t*)ctx->gen_a.p;
    uint32_t* Bm = R > 2 ? (uint32_t*)ctx->gen_b.p : A;
    const uint2* tabs = nullptr;
    if ((s = coset_mid_tables(ctx, lp, ln, &tabs)) != ZODA_OK) return s;
    for (uint64_t c0 = 0; c0 < cols; c0 += w0) {
        const uint64_t w = std::min(w0, cols - c0);
        const uint32_t qpc = (uint32_t)(w / 4);
        // INTT pass A over i1; data rows N2*i1 + i2 >= k are zeros
        StepArgs pa = plain_args(View{const_cast<uint32_t*>(in) + c0, N2 * cols, cols}, View{A, N2 * w, w}, qpc,
                                 N2 * qpc);
        pa.in_lim_rm = (uint32_t)N2;
        pa.in_lim_cm = 1;
        pa.in_limit = k;
        pa.tw_log = lp;
        pa.tw_inv = 1;
        if ((s = run_step(ctx, L1, true, pa, st)) != ZODA_OK) return s;
        for (uint64_t c = 1; c < R && c < rows_out; c++) {
            const uint64_t mc = std::min<uint64_t>(P_, (rows_out - c + R - 1) / R);
            const uint2* cbtab = tabs + (c - 1) * (N1 + N2);
            const uint2* ktab = cbtab + N1;
            StepArgs pm = plain_args(View{A, w, N2 * w}, View{Bm, w, N2 * w}, qpc, N1 * qpc);
            pm.mid1 = FTab{cbtab, 0, 1};
            pm.mid2 = FTab{ktab, 1, 0};
            pm.tw_log = lp;
            if ((s = run_step2(ctx, L2, true, pm, st)) != ZODA_OK) return s;
            // NTT pass B: wide rows j2 of block m1 -> output row R*(m1 + N2*m2) + c
            StepArgs pb = plain_args(View{Bm, N2 * w, w}, View{out + c * cols + c0, R * N2 * cols, R * cols}, qpc,
                                     N2 * qpc);
            pb.out_lim_rm = (uint32_t)N2;
            pb.out_lim_cm = 1;
            pb.out_limit = mc;
            if ((s = run_step(ctx, L1, false, pb, st)) != ZODA_OK) return s;
        }
    }
    return ZODA_OK;
}

// zk[j] = Z(omega_N^j) and izh[j] = 1 / Z(h * omega_N^j) for N = 2^log_n up to
// 2^26, Z the vanishing polynomial of the erased points (roots given), h = 31.
__global__ void k_erasure_tables_long(const uint32_t* __restrict__ erased_roots, uint32_t ne, int log_n,
                                      const Tw* __restrict__ tw_hi, const Tw* __restrict__ tw_lo,
                                      uint2* __restrict__ zk, uint2* __restrict__ izh) {
    const uint32_t N = 1u << log_n;
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    const uint32_t E = (j << (LOG_TWM - log_n)) & TWM_MASK;
    const uint32_t x = mul_slow(tw_hi[E >> 13].w, tw_lo[E & 8191u].w);  // omega_N^j
    const uint32_t y = mul_slow(GENERATOR, x);
    uint32_t zx = 1, zy = 1;
    for (uint32_t i = 0; i < ne; i++) {
        const uint32_t r = erased_roots[i];
        zx = mul_slow(zx, x >= r ? x - r : x + P - r);
        zy = mul_slow(zy, y >= r ? y - r : y + P - r);
    }
    uint32_t inv = 1, b = zy, e = P - 2;
    while (e) {
        if (e & 1) inv = mul_slow(inv, b);
        b = mul_slow(b, b);
        e >>= 1;
    }
    zk[j] = make_uint2(zx, (uint32_t)(((uint64_t)zx << 32) / P));
    izh[j] = make_uint2(inv, (uint32_t)(((uint64_t)inv << 32) / P));
}

// k-of-2k recovery for N = 2k = 2^L points, L > 13: the decoder's four
// transforms (general.cu) as five passes on column chunks of the scratch:
//   P1 strided: INTT pass A of y * Z                      (pre-factor zk)
//   P2 block:   INTT pass B, h^i / N, NTT pass A
//   P3 strided: NTT pass B, 1 / Z(h w^j), INTT pass A
//   P4 block:   INTT pass B, h^-i / N [i < k] (optionally counting the nonzero
//               coefficients i >= k), NTT pass A
//   P5 strided: NTT pass B of the even outputs only: data row m = output 2m.
zoda_status long_recover(zoda_ctx* ctx, const uint32_t* d_code, const std::vector<uint32_t>& erased_roots,
                         uint32_t k, uint64_t cols, uint32_t* d_data, unsigned long long* d_cnt, cudaStream_t st) {
    int L = 0;
    while ((1ull << L) < 2ull * k) L++;
    if (L <= LONG_MIN_LOG || L > LONG_RECOVER_MAX_LOG) return ZODA_ERR_UNSUPPORTED;
    const uint64_t N = 1ull << L;
    const int L1 = L / 2, L2 = L - L1;
    const uint64_t N1 = 1ull << L1, N2 = 1ull << L2;
    zoda_status s;
    // pattern tables: zk | izh, then the erased roots
    if ((s = ctx->gen_tab.ensure((size_t)2 * N * sizeof(uint2))) != ZODA_OK) return s;
    if ((s = ctx->gen_small.ensure(std::max<size_t>(1, erased_roots.size()) * 4 + 64)) != ZODA_OK) return s;
    uint2* zk = (uint2*)ctx->gen_tab.p;
    uint2* izh = zk + N;
    uint32_t* d_er = (uint32_t*)ctx->gen_small.p;
    if (!erased_roots.empty())
        ZB_CUDA(cudaMemcpyAsync(d_er, erased_roots.data(), erased_roots.size() * 4, cudaMemcpyHostToDevice, st));
    k_erasure_tables_long<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(d_er, (uint32_t)erased_roots.size(), L,
                                                                       ctx->tables.tw, ctx->tables.tw_lo, zk, izh);
    ZB_CUDA(cudaGetLastError());
    // pattern-independent factors: [k1: h^(+-k1) / N] and [k2: h^(+-N1 k2)], the
    // second direction's k2 table zeroing k2 >= N2 / 2 (coefficients i >= k)
    const uint2* mtab = nullptr;
    {
        std::vector<uint2> h;
        const uint32_t hinv = powmod_c(GENERATOR, P - 2), ninv = powmod_c((uint32_t)N, P - 2);
        for (int dir = 0; dir < 2; dir++) {
            const uint32_t base = dir == 0 ? GENERATOR : hinv;
            for (uint32_t k1 = 0, x = ninv; k1 < N1; k1++, x = mulmod_c(x, base)) h.push_back(shoup_pair(x));
            const uint32_t step = powmod_c(base, N1);
            for (uint32_t k2 = 0, x = 1; k2 < N2; k2++, x = mulmod_c(x, step))
                h.push_back(dir == 1 && k2 >= N2 / 2 ? make_uint2(0u, 0u) : shoup_pair(x));
        }
        if ((s = upload_table(ctx, -(400000000 + L), h, &mtab)) != ZODA_OK) return s;
    }
    const uint2 *cb_a = mtab, *k_a = mtab + N1, *cb_b = mtab + N1 + N2, *k_b = mtab + 2 * N1 + N2;
    uint64_t w0 = ((64ull << 20) / N) & ~3ull;
    if (w0 < 4) w0 = 4;
    if (w0 > cols) w0 = cols;
    if ((s = ctx->gen_a.ensure(N * w0 * 4)) != ZODA_OK) return s;
    uint32_t* A = (uint32_t*)ctx->gen_a.p;
    for (uint64_t c0 = 0; c0 < cols; c0 += w0) {
        const uint64_t w = std::min(w0, cols - c0);
        const uint32_t qpc = (uint32_t)(w / 4);
        const View strided{A, N2 * w, w}, block{A, w, N2 * w};
        // P1: code rows N2*i1 + i2 times zk (erased rows are not read)
        StepArgs p1 = plain_args(View{const_cast<uint32_t*>(d_code) + c0, N2 * cols, cols}, strided, qpc, N2 * qpc);
        p1.pre = FTab{zk, (uint32_t)N2, 1};
        p1.tw_log = L;
        p1.tw_inv = 1;
        if ((s = run_step(ctx, L1, true, p1, st)) != ZODA_OK) return s;
        StepArgs p2 = plain_args(block, block, qpc, N1 * qpc);
        p2.mid1 = FTab{cb_a, 0, 1};
        p2.mid2 = FTab{k_a, 1, 0};
        p2.tw_log = L;
        if ((s = run_step2(ctx, L2, true, p2, st)) != ZODA_OK) return s;
        StepArgs p3 = plain_args(strided, strided, qpc, N2 * qpc);
        p3.mid1 = FTab{izh, (uint32_t)N2, 1};  // NTT output j = m1 + N2 * m2
        p3.tw_log = L;
        p3.tw_inv = 1;
        if ((s = run_step2(ctx, L1, false, p3, st)) != ZODA_OK) return s;
        StepArgs p4 = plain_args(block, block, qpc, N1 * qpc);
        p4.mid1 = FTab{cb_b, 0, 1};
        p4.mid2 = FTab{k_b, 1, 0};
        p4.tw_log = L;
        if (d_cnt) {
            p4.counter = d_cnt;
            p4.count_from = (uint32_t)(N2 / 2);  // i = k1 + N1*k2 >= k  <=>  k2 >= N2 / 2
        }
        if ((s = run_step2(ctx, L2, true, p4, st)) != ZODA_OK) return s;
        // P5: only the even outputs m = m1 + N2*m2 (m1 even): column blocks m1 = 2*b,
        // data row m / 2 = b + (N2/2) * m2
        StepArgs p5 = plain_args(View{A, N2 * w, 2 * w}, View{d_data + c0, (N2 / 2) * cols, cols}, qpc,
                                 (N2 / 2) * qpc);
        if ((s = run_step(ctx, L1, false, p5, st)) != ZODA_OK) return s;
    }
    return ZODA_OK;
}

}  // namespace zb
