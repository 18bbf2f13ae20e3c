// Batched extension of many squares in one persistent launch (the
// zoda_batch_* entry points of include/zoda_b200.h).
//
// Host side of k_extend_batch (extend_tma.cuh): one BatchSquare descriptor per
// square (two TMA maps, output pointer, shape, first global tile index),
// squares ordered by decreasing side, a device counter the CTAs draw tiles
// from, and a CUDA graph holding the counter reset and the launch.
#include <algorithm>
#include <new>
#include <vector>

#include "tma_host.hpp"

struct zoda_batch {
    zoda_ctx* ctx = nullptr;
    uint32_t nsq = 0;
    uint64_t total_tiles = 0;
    uint64_t elements = 0;
    zb::DevBuf squares;  // BatchSquare[nsq]
    zb::DevBuf counter;  // unsigned long long
    zb::DevBuf tables;   // SideTables[26]: radix 16 at [log_s], radix 8 at [13 + log_s]
    int lept = 4;        // level radix 2^lept of this batch's launch
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace zb {
namespace {

template <int LOG_S>
zoda_status fill_square(BatchSquare* b, const zoda_square& q, int promo) {
    using TP = TPlan<LOG_S>;
    zoda_status s = make_tile_maps<TP>(&b->in_map, &b->even_map, q.d_in, q.d_out, q.cols, promo);
    if (s != ZODA_OK) return s;
    b->out = q.d_out;
    b->cols = q.cols;
    b->log_s = LOG_S;
    b->ntiles = (uint32_t)((q.cols + TP::C - 1) / TP::C);
    return ZODA_OK;
}

int log2_side(uint32_t k) {
    if (k == 0 || (k & (k - 1))) return -1;
    int l = 0;
    while ((1u << l) < k) l++;
    return l;
}

}  // namespace

zoda_status make_batch_square(const zoda_square& q, BatchSquare* b, int promo) {
    const int ls = log2_side(q.k);
    if (!q.d_in || !q.d_out || ls < 0 || q.cols % 4 || (((uintptr_t)q.d_in | (uintptr_t)q.d_out) & 15))
        return ZODA_ERR_ARG;
    if (ls < BATCH_MIN_LOG || ls > BATCH_MAX_LOG) {
        set_last_error_text("batched sides are 32 .. 2048");
        return ZODA_ERR_UNSUPPORTED;
    }
    memset(b, 0, sizeof *b);
    switch (ls) {
        case 5: return fill_square<5>(b, q, promo);
        case 6: return fill_square<6>(b, q, promo);
        case 7: return fill_square<7>(b, q, promo);
        case 8: return fill_square<8>(b, q, promo);
        case 9: return fill_square<9>(b, q, promo);
        case 10: return fill_square<10>(b, q, promo);
        default: return fill_square<11>(b, q, promo);
    }
}

zoda_status launch_batch_kernel(const zoda_ctx* ctx, const BatchSquare* d_sq, uint32_t nsq, uint64_t total_tiles,
                                unsigned long long* d_counter, const SideTables* d_tables, int lept, cudaStream_t st) {
    if (total_tiles == 0) return ZODA_OK;
    const uint64_t grid = total_tiles < (uint64_t)ctx->sm_count ? total_tiles : (uint64_t)ctx->sm_count;
    if (lept == 3)
        k_extend_batch<3><<<(unsigned)grid, BatchGeom<3>::THREADS, BatchGeom<3>::SMEM, st>>>(
            d_sq, nsq, total_tiles, d_counter, d_tables, ctx->d_err);
    else
        k_extend_batch<4><<<(unsigned)grid, BatchGeom<4>::THREADS, BatchGeom<4>::SMEM, st>>>(
            d_sq, nsq, total_tiles, d_counter, d_tables, ctx->d_err);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

zoda_status set_batch_kernel_attributes() {
    ZB_CUDA(cudaFuncSetAttribute(k_extend_batch<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)BatchGeom<4>::SMEM));
    ZB_CUDA(cudaFuncSetAttribute(k_extend_batch<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)BatchGeom<3>::SMEM));
    return ZODA_OK;
}

int batch_lept(const zoda_ctx* ctx, int max_log) {
    if (max_log >= 0 && max_log <= 12 && ctx->planned[max_log] && ctx->plan[max_log].impl == ZODA_IMPL_TMA &&
        ctx->plan[max_log].radix == 8)
        return 3;
    return 4;
}

}  // namespace zb

using namespace zb;

extern "C" {

zoda_status zoda_batch_create(zoda_ctx* ctx, const zoda_square* squares, uint32_t n, zoda_batch** out) {
    if (!ctx || !out || (n && !squares)) return ZODA_ERR_ARG;
    *out = nullptr;
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return squares[a].k > squares[b].k; });
    std::vector<BatchSquare> host(n);
    uint64_t first = 0, elements = 0;
    for (uint32_t j = 0; j < n; j++) {
        const zoda_square& q = squares[order[j]];
        BatchSquare& b = host[j];
        const zoda_status s = make_batch_square(q, &b, side_l2_promo(ctx, log2_side(q.k)));
        if (s != ZODA_OK) return s;
        b.first = first;
        first += b.ntiles;
        elements += (uint64_t)q.k * q.cols;
    }
    zoda_batch* bt = new (std::nothrow) zoda_batch();
    if (!bt) return ZODA_ERR_NOMEM;
    bt->ctx = ctx;
    bt->nsq = n;
    bt->total_tiles = first;
    bt->elements = elements;
    auto fail = [&](zoda_status s) {
        zoda_batch_destroy(bt);
        return s;
    };
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) {
        set_last_error("cudaSetDevice", e);
        return fail(ZODA_ERR_CUDA);
    }
    zoda_status s;
    if ((s = bt->squares.ensure(std::max<size_t>(1, n) * sizeof(BatchSquare))) != ZODA_OK) return fail(s);
    if ((s = bt->counter.ensure(sizeof(unsigned long long))) != ZODA_OK) return fail(s);
    if ((s = bt->tables.ensure(26 * sizeof(SideTables))) != ZODA_OK) return fail(s);
    std::vector<SideTables> tabs(26);
    for (int ls = BATCH_MIN_LOG; ls <= BATCH_MAX_LOG; ls++) {
        tabs[ls] = side_tables(ctx, ls, 4);
        tabs[13 + ls] = side_tables(ctx, ls, 3);
    }
    bt->lept = batch_lept(ctx, n ? log2_side(squares[order[0]].k) : 0);
    if (n && (e = cudaMemcpy(bt->squares.p, host.data(), n * sizeof(BatchSquare), cudaMemcpyHostToDevice)) !=
                 cudaSuccess) {
        set_last_error("cudaMemcpy(batch squares)", e);
        return fail(ZODA_ERR_CUDA);
    }
    if ((e = cudaMemcpy(bt->tables.p, tabs.data(), 26 * sizeof(SideTables), cudaMemcpyHostToDevice)) != cudaSuccess) {
        set_last_error("cudaMemcpy(batch tables)", e);
        return fail(ZODA_ERR_CUDA);
    }
    if ((s = set_batch_kernel_attributes()) != ZODA_OK) return fail(s);
    *out = bt;
    return ZODA_OK;
}

zoda_status zoda_batch_run(zoda_batch* bt, void* stream) {
    if (!bt) return ZODA_ERR_ARG;
    if (bt->total_tiles == 0) return ZODA_OK;
    zoda_ctx* ctx = bt->ctx;
    ZB_CUDA(cudaSetDevice(ctx->device));
    if (!bt->exec) {
        // capture: counter = 0, then the persistent kernel, one CTA per SM
        ZB_CUDA(cudaStreamCreateWithFlags(&bt->cap, cudaStreamNonBlocking));
        ZB_CUDA(cudaStreamBeginCapture(bt->cap, cudaStreamCaptureModeThreadLocal));
        cudaMemsetAsync(bt->counter.p, 0, sizeof(unsigned long long), bt->cap);
        const zoda_status ls = launch_batch_kernel(
            ctx, (const BatchSquare*)bt->squares.p, bt->nsq, bt->total_tiles, (unsigned long long*)bt->counter.p,
            (const SideTables*)bt->tables.p + (bt->lept == 3 ? 13 : 0), bt->lept, bt->cap);
        cudaError_t e = cudaStreamEndCapture(bt->cap, &bt->graph);
        if (ls != ZODA_OK) return ls;
        if (e != cudaSuccess) {
            set_last_error("cudaStreamEndCapture", e);
            return ZODA_ERR_CUDA;
        }
        ZB_CUDA(cudaGraphInstantiate(&bt->exec, bt->graph, 0));
    }
    ZB_CUDA(cudaGraphLaunch(bt->exec, (cudaStream_t)stream));
    return ZODA_OK;
}

uint64_t zoda_batch_elements(const zoda_batch* bt) { return bt ? bt->elements : 0; }

void zoda_batch_destroy(zoda_batch* bt) {
    if (!bt) return;
    if (bt->ctx) cudaSetDevice(bt->ctx->device);
    cudaDeviceSynchronize();  // a replay may still be running on the caller's stream
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    if (bt->graph) cudaGraphDestroy(bt->graph);
    if (bt->cap) cudaStreamDestroy(bt->cap);
    bt->squares.release();
    bt->counter.release();
    bt->tables.release();
    delete bt;
}

}  // extern "C"
