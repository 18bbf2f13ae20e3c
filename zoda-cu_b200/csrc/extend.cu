// Instantiations and launchers of the fused extension kernels (extend.cuh,
// extend_tma.cuh).
#include "extend.cuh"
#include "tma_host.hpp"

namespace zb {

namespace {
// S = 1: NTT_2 of (v, 0) is (v, v); with odd_only just the odd row.
__global__ void k_extend_side1(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint64_t cols,
                               bool odd_only) {
    for (uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) * 4; c < cols;
         c += (uint64_t)gridDim.x * blockDim.x * 4) {
        V4 x = ld_v4(in + c);
        st_v4(out + c, x);
        if (!odd_only) st_v4(out + cols + c, x);
    }
}

template <int LOG_S, int SCHED, int LEPT = 4>
zoda_status launch_t(const zoda_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t cols, uint32_t flags,
                     uint32_t in_rows, uint32_t out_rows, cudaStream_t st) {
    using PL = ExtPlan<LOG_S, SCHED, LEPT, LEPT == 3 ? 1024 : 512>;
    const uint64_t ntiles = (cols + PL::C - 1) / PL::C;
    if (ntiles == 0) return ZODA_OK;
    const uint64_t grid = ntiles < (uint64_t)ctx->sm_count ? ntiles : (uint64_t)ctx->sm_count;
    k_extend<LOG_S, SCHED, LEPT><<<(unsigned)grid, PL::THREADS, PL::SMEM, st>>>(in, out, cols, ntiles,
                                                                                ctx->tables.tw, ctx->tables.twist,
                                                                                flags, in_rows, out_rows);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

template <int LOG_S, int LEPT>
zoda_status launch_tma_t(const zoda_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t cols, int promo,
                         uint32_t flags, uint32_t in_rows, uint32_t out_rows, cudaStream_t st) {
    using TP = TPlan<LOG_S, LEPT>;
    const uint64_t ntiles = (cols + TP::C - 1) / TP::C;
    if (ntiles == 0) return ZODA_OK;
    CUtensorMap m_in, m_even;
    zoda_status s = make_tile_maps<TP>(&m_in, &m_even, in, out, cols, promo, in_rows, (out_rows + 1) / 2);
    if (s != ZODA_OK) return s;
    const uint64_t grid = ntiles < (uint64_t)ctx->sm_count ? ntiles : (uint64_t)ctx->sm_count;
    const SideTables tb = side_tables(ctx, LOG_S, LEPT);
    k_extend_tma<LOG_S, LEPT><<<(unsigned)grid, TP::THREADS, TP::SMEM, st>>>(m_in, m_even, out, cols, ntiles, tb,
                                                                            ctx->d_err, flags, out_rows);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

// The leftover radix differs from 16 (so schedule 1 is a distinct kernel) for
// these sides only; the same for radix 8.
constexpr bool has_sched1(int ls) { return ls >= 5 && ls % 4 != 0; }
constexpr bool has_sched1_r8(int ls) { return ls >= 6 && ls % 3 != 0; }
// Sides with a radix-8 direct kernel.
constexpr bool has_direct_r8(int ls) { return ls >= 6; }

template <int LOG_S>
zoda_status set_attr_t() {
    using PL = ExtPlan<LOG_S>;
    if (PL::SMEM > 0) {
        ZB_CUDA(cudaFuncSetAttribute(k_extend<LOG_S, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::SMEM));
        if constexpr (has_sched1(LOG_S))
            ZB_CUDA(cudaFuncSetAttribute(k_extend<LOG_S, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ExtPlan<LOG_S, 1>::SMEM));
    }
    if constexpr (has_direct_r8(LOG_S)) {
        ZB_CUDA(cudaFuncSetAttribute(k_extend<LOG_S, 0, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ExtPlan<LOG_S, 0, 3, 1024>::SMEM));
        if constexpr (has_sched1_r8(LOG_S))
            ZB_CUDA(cudaFuncSetAttribute(k_extend<LOG_S, 1, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ExtPlan<LOG_S, 1, 3, 1024>::SMEM));
    }
    if constexpr (LOG_S >= 5) {
        ZB_CUDA(cudaFuncSetAttribute(k_extend_tma<LOG_S, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)TPlan<LOG_S, 4>::SMEM));
        ZB_CUDA(cudaFuncSetAttribute(k_extend_tma<LOG_S, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)TPlan<LOG_S, 3>::SMEM));
    }
    return ZODA_OK;
}

template <int LOG_S>
zoda_status launch_direct(const zoda_ctx* ctx, int sched, int radix, const uint32_t* in, uint32_t* out,
                          uint64_t cols, uint32_t flags, uint32_t in_rows, uint32_t out_rows, cudaStream_t st) {
    if constexpr (has_direct_r8(LOG_S)) {
        if (radix == 8) {
            if constexpr (has_sched1_r8(LOG_S))
                if (sched == 1) return launch_t<LOG_S, 1, 3>(ctx, in, out, cols, flags, in_rows, out_rows, st);
            return launch_t<LOG_S, 0, 3>(ctx, in, out, cols, flags, in_rows, out_rows, st);
        }
    }
    if constexpr (has_sched1(LOG_S))
        if (sched == 1) return launch_t<LOG_S, 1>(ctx, in, out, cols, flags, in_rows, out_rows, st);
    return launch_t<LOG_S, 0>(ctx, in, out, cols, flags, in_rows, out_rows, st);
}
}  // namespace

zoda_status extend_init_attributes() {
    zoda_status s = ZODA_OK;
#define ZB_ATTR(L) \
    if (s == ZODA_OK) s = set_attr_t<L>();
    ZB_ATTR(1) ZB_ATTR(2) ZB_ATTR(3) ZB_ATTR(4) ZB_ATTR(5) ZB_ATTR(6)
    ZB_ATTR(7) ZB_ATTR(8) ZB_ATTR(9) ZB_ATTR(10) ZB_ATTR(11) ZB_ATTR(12)
#undef ZB_ATTR
    return s;
}

zoda_plan default_plan(int log_s) {
    // the TMA-staged kernel from side 128 up to 2048; at side 4096 its
    // 8-column tiles split 32-byte sectors between the two warp-groups, and the
    // direct-load kernel is faster
    zoda_plan p{};
    p.impl = (log_s >= 7 && log_s <= 11) ? ZODA_IMPL_TMA : ZODA_IMPL_DIRECT;
    p.sched = 0;
    p.l2_promo = 3;
    p.blocked = 0;
    p.stagger = 1;
    p.radix = 16;
    p.ms = 0.f;
    return p;
}

zoda_status check_plan(int log_s, const zoda_plan& p) {
    if (log_s < 0 || log_s > 12) return ZODA_ERR_UNSUPPORTED;
    if (p.impl != ZODA_IMPL_DIRECT && p.impl != ZODA_IMPL_TMA && p.impl != ZODA_IMPL_FOURSTEP) return ZODA_ERR_ARG;
    if (p.impl == ZODA_IMPL_TMA && log_s < 5) return ZODA_ERR_UNSUPPORTED;
    if (p.impl == ZODA_IMPL_FOURSTEP) {
        if (log_s < FOURSTEP_MIN_LOG) return ZODA_ERR_UNSUPPORTED;
        // (radix, CTAs per SM): (16, 1), (16, 2), (8, 2), (8, 4), (4, 5); ctas 0 counts as 1
        const int c = p.ctas == 0 ? 1 : p.ctas;
        const bool shape_ok = (p.radix == 16 && (c == 1 || c == 2)) || (p.radix == 8 && (c == 2 || c == 4)) ||
                              (p.radix == 4 && c == 5);
        if (!shape_ok) return ZODA_ERR_ARG;
        // sched 1: staged passes, which exist for the shapes of 2 and 4 CTAs per SM
        if (p.sched == 1 && p.ctas <= 1) return ZODA_ERR_ARG;
    }
    if (p.sched < 0 || p.sched > 1 || p.l2_promo < 0 || p.l2_promo > 3 || p.blocked < 0 || p.blocked > 1 ||
        p.stagger < 0 || p.stagger > 3 || (p.radix != 16 && p.radix != 8 && !(p.radix == 4 && p.impl == ZODA_IMPL_FOURSTEP)))
        return ZODA_ERR_ARG;
    if (p.radix == 8 && p.impl == ZODA_IMPL_DIRECT && log_s < 6) return ZODA_ERR_UNSUPPORTED;
    return ZODA_OK;
}

int side_l2_promo(const zoda_ctx* ctx, int log_s) {
    if (log_s >= 0 && log_s <= 12 && ctx->planned[log_s] && ctx->plan[log_s].impl == ZODA_IMPL_TMA)
        return ctx->plan[log_s].l2_promo;
    return 3;
}

zoda_status launch_plan(const zoda_ctx* ctx, int log_s, const zoda_plan& p, const uint32_t* in, uint32_t* out,
                        uint64_t cols, cudaStream_t st, bool odd_only, uint32_t in_rows, uint32_t out_rows) {
    zoda_status s = check_plan(log_s, p);
    if (s != ZODA_OK) return s;
    const uint32_t S = 1u << log_s;
    if (in_rows == 0) in_rows = S;
    if (out_rows == 0) out_rows = 2 * S;
    if (in_rows > S || out_rows > 2 * S || (log_s == 0 && (in_rows != 1 || out_rows != 2))) return ZODA_ERR_ARG;
    if (p.impl == ZODA_IMPL_FOURSTEP) {
        // three four-step passes; they keep their intermediate matrices in the odd
        // output rows, so an output cut short (an encode of fewer rows) takes the
        // side's default plan instead
        if (in_rows == S && out_rows == 2 * S)
            return long_extend(ctx, log_s, ctx->tables.ext4[log_s], in, out, cols, st, odd_only,
                               fourstep_shape(p.radix, p.ctas, p.sched != 0), p.blocked != 0);
        return launch_plan(ctx, log_s, default_plan(log_s), in, out, cols, st, odd_only, in_rows, out_rows);
    }
    // stagger 1: release after all INTT levels but the last; 2: after the first; 3: right away
    const uint32_t at_code = p.stagger == 2 ? 2u : p.stagger == 3 ? 1u : 0u;
    const uint32_t flags = (p.blocked ? 1u : 0u) | (p.stagger ? 0u : 2u) | (at_code << 2) | (odd_only ? 16u : 0u);
    if (p.impl == ZODA_IMPL_TMA) {
        switch (log_s) {
#define ZB_CASE(L)                                                                  \
    case L:                                                                         \
        return p.radix == 8 ? launch_tma_t<L, 3>(ctx, in, out, cols, p.l2_promo, flags, in_rows, out_rows, st) \
                            : launch_tma_t<L, 4>(ctx, in, out, cols, p.l2_promo, flags, in_rows, out_rows, st);
            ZB_CASE(5) ZB_CASE(6) ZB_CASE(7) ZB_CASE(8) ZB_CASE(9) ZB_CASE(10) ZB_CASE(11) ZB_CASE(12)
#undef ZB_CASE
            default: return ZODA_ERR_UNSUPPORTED;
        }
    }
    switch (log_s) {
        case 0: {
            const uint64_t quads = cols / 4;
            const unsigned grid = (unsigned)((quads + 255) / 256 < 4096 ? (quads + 255) / 256 : 4096);
            if (grid) k_extend_side1<<<grid, 256, 0, st>>>(in, out, cols, odd_only);
            ZB_CUDA(cudaGetLastError());
            return ZODA_OK;
        }
#define ZB_CASE(L) \
    case L: return launch_direct<L>(ctx, p.sched, p.radix, in, out, cols, flags, in_rows, out_rows, st);
        ZB_CASE(1) ZB_CASE(2) ZB_CASE(3) ZB_CASE(4) ZB_CASE(5) ZB_CASE(6)
        ZB_CASE(7) ZB_CASE(8) ZB_CASE(9) ZB_CASE(10) ZB_CASE(11) ZB_CASE(12)
#undef ZB_CASE
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

zoda_status launch_extend(const zoda_ctx* ctx, int log_s, const uint32_t* in, uint32_t* out, uint64_t cols,
                          cudaStream_t st, int impl, bool odd_only, uint32_t in_rows, uint32_t out_rows) {
    if (log_s < 0 || log_s > 12) return ZODA_ERR_UNSUPPORTED;
    zoda_plan p = default_plan(log_s);
    if (impl == ZODA_IMPL_AUTO && ctx->planned[log_s]) p = ctx->plan[log_s];
    else if (impl == ZODA_IMPL_DIRECT) p.impl = ZODA_IMPL_DIRECT;
    else if (impl == ZODA_IMPL_TMA) p.impl = ZODA_IMPL_TMA;
    else if (impl == ZODA_IMPL_FOURSTEP && log_s >= FOURSTEP_MIN_LOG) p.impl = ZODA_IMPL_FOURSTEP;
    return launch_plan(ctx, log_s, p, in, out, cols, st, odd_only, in_rows, out_rows);
}

}  // namespace zb
