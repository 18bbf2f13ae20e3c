// zoda_ntt_device_noalloc: the batched NTT / INTT of cuda_ntt and cuda_intt
// on device buffers, with every byte of device memory it needs besides the
// caller's input and output held in file-scope __device__ arrays.
//
// Who needs it: callers that may not allocate device memory while they run.
// A host whose device memory is owned by a pool allocator (a framework that
// hands out every byte itself and forbids raw cudaMalloc), or a latency-bound
// path where cudaMalloc / cudaFree would synchronise the device and stall
// other streams, can still transform polynomials with this call: it performs
// no cudaMalloc, no cudaFree and calls no allocating library routine.
//
// Cost of that: the scratch array (16 MiB) and the twiddle table (64 KiB)
// below are part of the library image, so every GPU that loads the library
// holds them until the process exits, and all calls share them (see the
// header for the concurrency rule).
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "extend.cuh"
#include "internal.hpp"

namespace zb {
namespace {

// Largest n * round_up(polys, 4) the entry point accepts, in u32 elements.
constexpr size_t NOALLOC_MAX_ELEMS = (size_t)4 << 20;  // 16 MiB

// The polynomials transposed into columns ([n][round_up(polys, 4)] u32) while
// they are transformed; and omega_8192^j with Shoup companions.
static __device__ __align__(256) uint32_t g_noalloc_scratch[NOALLOC_MAX_ELEMS];
static __device__ __align__(256) Tw g_noalloc_tw[TW_N];

struct NoallocDevice {
    uint32_t* scratch = nullptr;  // device address of g_noalloc_scratch
    Tw* tw = nullptr;             // device address of g_noalloc_tw
    int sm_count = 0;
};
std::mutex g_noalloc_mu;
std::map<int, NoallocDevice> g_noalloc_dev;

// out[c * ld_out + r] = in[r * ld_in + c] for r < R, c < Cn. Row tiles are
// walked with a grid stride in y: R reaches 2^21 polynomials at n = 2, more
// 32-row tiles than gridDim.y may hold (65535).
__global__ void k_noalloc_transpose(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t R,
                                    uint32_t Cn, uint64_t ld_in, uint64_t ld_out) {
    __shared__ uint32_t tile[32][33];
    const uint32_t c0 = blockIdx.x * 32;
    for (uint32_t r0 = blockIdx.y * 32; r0 < R; r0 += gridDim.y * 32) {
        for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
            const uint32_t r = r0 + i, c = c0 + threadIdx.x;
            if (r < R && c < Cn) tile[i][threadIdx.x] = in[r * ld_in + c];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
            const uint32_t c = c0 + i, r = r0 + threadIdx.x;
            if (r < R && c < Cn) out[c * ld_out + r] = tile[threadIdx.x][i];
        }
        __syncthreads();  // the next row tile reuses the tile buffer
    }
}

// Grid of a k_noalloc_transpose launch over R x Cn: Cn on x, R on y (capped).
dim3 noalloc_transpose_grid(uint32_t R, uint32_t Cn) {
    const uint32_t gy = (R + 31) / 32;
    return dim3((Cn + 31) / 32, gy < 65535u ? gy : 65535u);
}

template <int LOG_N, bool INV>
zoda_status noalloc_attr() {
    using PL = ExtPlan<LOG_N>;
    if (PL::SMEM > 0)
        ZB_CUDA(cudaFuncSetAttribute(k_colntt<LOG_N, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::SMEM));
    return ZODA_OK;
}

// Once per device, with that device current: the device addresses of the two
// arrays (a __device__ symbol's host-side name is not a device address), the
// twiddle table contents, and the kernels' shared-memory limits.
zoda_status noalloc_setup(int dev, NoallocDevice* out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    auto it = g_noalloc_dev.find(dev);
    if (it != g_noalloc_dev.end()) {
        *out = it->second;
        return ZODA_OK;
    }
    NoallocDevice d;
    void* p = nullptr;
    ZB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    d.scratch = static_cast<uint32_t*>(p);
    ZB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_tw));
    d.tw = static_cast<Tw*>(p);
    std::vector<Tw> tw(TW_N);
    const uint32_t w = root_of_unity(LOG_TW);
    uint32_t cur = 1;
    for (int j = 0; j < TW_N; j++) {
        tw[j] = Tw{cur, shoup(cur)};
        cur = mulmod_c(cur, w);
    }
    ZB_CUDA(cudaMemcpyToSymbol(g_noalloc_tw, tw.data(), TW_N * sizeof(Tw)));
    ZB_CUDA(cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount, dev));
    zoda_status s = ZODA_OK;
#define ZB_NA_ATTR(L)                                   \
    if (s == ZODA_OK) s = noalloc_attr<L, false>();     \
    if (s == ZODA_OK) s = noalloc_attr<L, true>();
    ZB_NA_ATTR(1) ZB_NA_ATTR(2) ZB_NA_ATTR(3) ZB_NA_ATTR(4) ZB_NA_ATTR(5) ZB_NA_ATTR(6)
    ZB_NA_ATTR(7) ZB_NA_ATTR(8) ZB_NA_ATTR(9) ZB_NA_ATTR(10) ZB_NA_ATTR(11) ZB_NA_ATTR(12)
#undef ZB_NA_ATTR
    if (s != ZODA_OK) return s;
    g_noalloc_dev[dev] = d;
    *out = d;
    return ZODA_OK;
}

template <int LOG_N, bool INV>
zoda_status noalloc_colntt_t(const NoallocDevice& d, uint32_t* buf, uint64_t cols, Tw scale, cudaStream_t st) {
    using PL = ExtPlan<LOG_N>;
    const uint64_t ntiles = (cols + PL::C - 1) / PL::C;
    const uint64_t grid = ntiles < (uint64_t)d.sm_count ? ntiles : (uint64_t)d.sm_count;
    // in place: every CTA reads all rows of its tile's columns before it writes them
    k_colntt<LOG_N, INV><<<(unsigned)grid, PL::THREADS, PL::SMEM, st>>>(buf, buf, cols, ntiles, d.tw, scale, 1u);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

template <bool INV>
zoda_status noalloc_colntt(const NoallocDevice& d, int log_n, uint32_t* buf, uint64_t cols, Tw scale,
                           cudaStream_t st) {
    switch (log_n) {
#define ZB_NA_CASE(L) \
    case L: return noalloc_colntt_t<L, INV>(d, buf, cols, scale, st);
        ZB_NA_CASE(1) ZB_NA_CASE(2) ZB_NA_CASE(3) ZB_NA_CASE(4) ZB_NA_CASE(5) ZB_NA_CASE(6)
        ZB_NA_CASE(7) ZB_NA_CASE(8) ZB_NA_CASE(9) ZB_NA_CASE(10) ZB_NA_CASE(11) ZB_NA_CASE(12)
#undef ZB_NA_CASE
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

}  // namespace
}  // namespace zb

using namespace zb;

extern "C" zoda_status zoda_ntt_device_noalloc(const uint32_t* d_in, uint32_t* d_out, uint32_t n, uint32_t polys,
                                               int inverse, void* stream) {
    if (!d_in || !d_out || n == 0 || (n & (n - 1))) {
        set_last_error_text("zoda_ntt_device_noalloc: null buffer or n not a power of two");
        return ZODA_ERR_ARG;
    }
    int log_n = 0;
    while ((1u << log_n) < n) log_n++;
    if (log_n > 12) {
        set_last_error_text("zoda_ntt_device_noalloc: n = " + std::to_string(n) + " exceeds the largest n, 4096");
        return ZODA_ERR_UNSUPPORTED;
    }
    const uint64_t polys4 = ((uint64_t)polys + 3) & ~3ull;
    if ((uint64_t)n * polys4 > NOALLOC_MAX_ELEMS) {
        set_last_error_text("zoda_ntt_device_noalloc: n * round_up(polys, 4) = " +
                            std::to_string((uint64_t)n * polys4) + " u32 exceeds the " +
                            std::to_string(NOALLOC_MAX_ELEMS) + "-element scratch array");
        return ZODA_ERR_UNSUPPORTED;
    }
    if (polys == 0) return ZODA_OK;
    int dev = 0;
    ZB_CUDA(cudaGetDevice(&dev));
    NoallocDevice d;
    zoda_status s = noalloc_setup(dev, &d);
    if (s != ZODA_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const uint64_t bytes = (uint64_t)n * polys * 4;
    if (n == 1) {  // a length-1 transform (and its 1^-1 scale) is the identity
        if (d_out != d_in) ZB_CUDA(cudaMemcpyAsync(d_out, d_in, bytes, cudaMemcpyDeviceToDevice, st));
        return ZODA_OK;
    }
    const uint32_t n_inv = inverse ? powmod_c(n, P - 2) : 1u;
    const Tw scale{n_inv, shoup(n_inv)};
    // polynomials (rows of d_in) -> columns of the scratch, transform the
    // columns in place, columns -> rows of d_out. The scratch's padding
    // columns (polys .. polys4) hold whatever an earlier call left; their
    // results are never copied out, so nothing needs clearing.
    dim3 block(32, 8);
    k_noalloc_transpose<<<noalloc_transpose_grid(polys, n), block, 0, st>>>(d_in, d.scratch, polys, n, n, polys4);
    ZB_CUDA(cudaGetLastError());
    s = inverse ? noalloc_colntt<true>(d, log_n, d.scratch, polys4, scale, st)
                : noalloc_colntt<false>(d, log_n, d.scratch, polys4, scale, st);
    if (s != ZODA_OK) return s;
    k_noalloc_transpose<<<noalloc_transpose_grid(n, polys), block, 0, st>>>(d.scratch, d_out, n, polys, polys4, n);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}
