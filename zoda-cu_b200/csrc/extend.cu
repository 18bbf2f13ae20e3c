// Instantiations and launcher of the fused extension kernel (extend.cuh).
#include "extend.cuh"
#include "internal.hpp"

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
zoda_status set_attr_t() {
    using PL = ExtPlan<LOG_S>;
    if (PL::SMEM > 0)
        ZB_CUDA(cudaFuncSetAttribute(k_extend<LOG_S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::SMEM));
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
                          cudaStream_t st) {
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
