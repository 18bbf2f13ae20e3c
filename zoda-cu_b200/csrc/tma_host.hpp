// Host-side helpers of the TMA-staged kernels: tensor maps and per-side tables.
#pragma once
#include <cudaTypedefs.h>

#include <mutex>
#include <string>

#include "extend_tma.cuh"
#include "internal.hpp"

namespace zb {

inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// 2-D u32 tensor map: `rows` rows of `cols` elements, rows `row_bytes` apart,
// boxes of box_r rows x box_c columns, zero fill out of bounds.
inline zoda_status make_map(CUtensorMap* m, const void* base, uint64_t cols, uint64_t rows, uint64_t row_bytes,
                            uint32_t box_c, uint32_t box_r, CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_NONE,
                            int promo = 3) {
    auto fn = encode_fn();
    if (!fn) {
        set_last_error_text("cuTensorMapEncodeTiled unavailable");
        return ZODA_ERR_CUDA;
    }
    const cuuint64_t dims[2] = {cols, rows};
    const cuuint64_t strides[1] = {row_bytes};
    const cuuint32_t box[2] = {box_c, box_r};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, swz, (CUtensorMapL2promotion)promo,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_last_error_text("cuTensorMapEncodeTiled failed with CUresult " + std::to_string((int)r));
        return ZODA_ERR_CUDA;
    }
    return ZODA_OK;
}

// The input map and the even-output-row map of one square for side plan TP.
// promo: L2 promotion of the input loads (0 none, 1 64 B, 2 128 B, 3 256 B).
// in_rows / even_rows bound the maps (TMA reads zeros past in_rows and clips
// stores past even_rows); 0 means S.
template <class TP>
constexpr CUtensorMapSwizzle tile_swizzle() {
    return TP::SWZ_MASK == 7   ? CU_TENSOR_MAP_SWIZZLE_128B
           : TP::SWZ_MASK == 3 ? CU_TENSOR_MAP_SWIZZLE_64B
           : TP::SWZ_MASK == 1 ? CU_TENSOR_MAP_SWIZZLE_32B
                               : CU_TENSOR_MAP_SWIZZLE_NONE;
}

template <class TP>
zoda_status make_tile_maps(CUtensorMap* m_in, CUtensorMap* m_even, const uint32_t* in, uint32_t* out,
                           uint64_t cols, int promo = 3, uint32_t in_rows = 0, uint32_t even_rows = 0) {
    const CUtensorMapSwizzle swz = tile_swizzle<TP>();
    zoda_status s = make_map(m_in, in, cols, in_rows ? in_rows : TP::S, cols * 4, TP::BOX_C, TP::BOX_R, swz, promo);
    if (s != ZODA_OK) return s;
    return make_map(m_even, out, cols, even_rows ? even_rows : TP::S, cols * 8, TP::BOX_C, TP::BOX_R, swz);
}

// Device pointers of the side's level tables (built in zoda_ctx_create) for
// level radix 2^lept (4 or 3).
inline SideTables side_tables(const zoda_ctx* ctx, int log_s, int lept = 4) {
    SideTables tb;
    const size_t* off = ctx->tables.side_off[log_s][lept == 3 ? 1 : 0];
    const uint2* base = reinterpret_cast<const uint2*>(ctx->tables.side);
    for (int l = 0; l < 3; l++) tb.intt[l] = base + off[l];
    tb.ntt0 = base + off[3];
    tb.ntt[0] = nullptr;  // NTT level 0 reads ntt0
    tb.ntt[1] = base + off[4];
    tb.ntt[2] = base + off[5];
    return tb;
}

}  // namespace zb

namespace zb {
// Batch building blocks shared by zoda_batch_* and the serving loop (batch.cu).
// Descriptor of one square; ZODA_ERR_UNSUPPORTED outside sides 32..2048.
zoda_status make_batch_square(const zoda_square& q, BatchSquare* out, int promo = 3);
// One launch of k_extend_batch over d_sq[0..nsq) (sorted by first), with
// *d_counter already zero on `st`; d_tables[log_s] must hold the level tables
// of radix 2^lept (4 or 3).
zoda_status launch_batch_kernel(const zoda_ctx* ctx, const BatchSquare* d_sq, uint32_t nsq, uint64_t total_tiles,
                                unsigned long long* d_counter, const SideTables* d_tables, int lept, cudaStream_t st);
zoda_status set_batch_kernel_attributes();
// The level radix a batch whose largest square has side 2^max_log uses: that
// side's planned radix (it carries most of the bytes), else 16.
int batch_lept(const zoda_ctx* ctx, int max_log);
}  // namespace zb
