// Instantiations and launchers of the fused extension kernels (extend.cuh,
// extend_tma.cuh).
#include "extend.cuh"
#include "tma_host.hpp"

namespace zb {

namespace {
// S = 1: NTT_2 of (v, 0) is (v, v).
__global__ void k_extend_side1(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint64_t cols) {
    for (uint64_t c = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) * 4; c < cols;
         c += (uint64_t)gridDim.x * blockDim.x * 4) {
        V4 x = ld_v4(in + c);
        st_v4(out + c, x);
        st_v4(out + cols + c, x);
    }
}

template <int LOG_S>
zoda_status launch_t(const zoda_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t cols, cudaStream_t st) {
    using PL = ExtPlan<LOG_S>;
    const uint64_t ntiles = (cols + PL::C - 1) / PL::C;
    if (ntiles == 0) return ZODA_OK;
    const uint64_t grid = ntiles < (uint64_t)ctx->sm_count ? ntiles : (uint64_t)ctx->sm_count;
    k_extend<LOG_S><<<(unsigned)grid, PL::THREADS, PL::SMEM, st>>>(in, out, cols, ntiles, ctx->tables.tw,
                                                                   ctx->tables.twist);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

template <int LOG_S>
zoda_status launch_tma_t(const zoda_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t cols, cudaStream_t st) {
    using TP = TPlan<LOG_S>;
    const uint64_t ntiles = (cols + TP::C - 1) / TP::C;
    if (ntiles == 0) return ZODA_OK;
    CUtensorMap m_in, m_even;
    zoda_status s = make_tile_maps<TP>(&m_in, &m_even, in, out, cols);
    if (s != ZODA_OK) return s;
    const uint64_t grid = ntiles < (uint64_t)ctx->sm_count ? ntiles : (uint64_t)ctx->sm_count;
    const SideTables tb = side_tables(ctx, LOG_S);
    k_extend_tma<LOG_S><<<(unsigned)grid, 512, TP::SMEM, st>>>(m_in, m_even, out, cols, ntiles, tb, ctx->d_err);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

template <int LOG_S>
zoda_status set_attr_t() {
    using PL = ExtPlan<LOG_S>;
    if (PL::SMEM > 0)
        ZB_CUDA(cudaFuncSetAttribute(k_extend<LOG_S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::SMEM));
    if constexpr (LOG_S >= 5)
        ZB_CUDA(cudaFuncSetAttribute(k_extend_tma<LOG_S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)TPlan<LOG_S>::SMEM));
    return ZODA_OK;
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

zoda_status launch_extend(const zoda_ctx* ctx, int log_s, const uint32_t* in, uint32_t* out, uint64_t cols,
                          cudaStream_t st, int impl) {
    // AUTO: the TMA-staged kernel from side 128 up to 2048; at side 4096 its
    // 8-column tiles split 32-byte sectors between the two warp-groups, and the
    // direct-load kernel is faster.
    const bool tma = (impl == 2) || (impl == 0 && log_s >= 7 && log_s <= 11);
    if (impl == 2 && (log_s < 5 || log_s > 12)) return ZODA_ERR_UNSUPPORTED;
    if (tma) {
        switch (log_s) {
            case 5: return launch_tma_t<5>(ctx, in, out, cols, st);
            case 6: return launch_tma_t<6>(ctx, in, out, cols, st);
            case 7: return launch_tma_t<7>(ctx, in, out, cols, st);
            case 8: return launch_tma_t<8>(ctx, in, out, cols, st);
            case 9: return launch_tma_t<9>(ctx, in, out, cols, st);
            case 10: return launch_tma_t<10>(ctx, in, out, cols, st);
            case 11: return launch_tma_t<11>(ctx, in, out, cols, st);
            case 12: return launch_tma_t<12>(ctx, in, out, cols, st);
            default: return ZODA_ERR_UNSUPPORTED;
        }
    }
    switch (log_s) {
        case 0: {
            const uint64_t quads = cols / 4;
            const unsigned grid = (unsigned)((quads + 255) / 256 < 4096 ? (quads + 255) / 256 : 4096);
            if (grid) k_extend_side1<<<grid, 256, 0, st>>>(in, out, cols);
            ZB_CUDA(cudaGetLastError());
            return ZODA_OK;
        }
        case 1: return launch_t<1>(ctx, in, out, cols, st);
        case 2: return launch_t<2>(ctx, in, out, cols, st);
        case 3: return launch_t<3>(ctx, in, out, cols, st);
        case 4: return launch_t<4>(ctx, in, out, cols, st);
        case 5: return launch_t<5>(ctx, in, out, cols, st);
        case 6: return launch_t<6>(ctx, in, out, cols, st);
        case 7: return launch_t<7>(ctx, in, out, cols, st);
        case 8: return launch_t<8>(ctx, in, out, cols, st);
        case 9: return launch_t<9>(ctx, in, out, cols, st);
        case 10: return launch_t<10>(ctx, in, out, cols, st);
        case 11: return launch_t<11>(ctx, in, out, cols, st);
        case 12: return launch_t<12>(ctx, in, out, cols, st);
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

}  // namespace zb
