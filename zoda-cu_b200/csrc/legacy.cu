// The reference's four FFI symbols (cuda/ntt_kernel.cu:184-208, bound by
// src/ntt/cuda.rs:15-22), reimplemented on the library's device kernels.
//
// Semantics kept: host buffer in, host buffer out, in place; `polys`
// polynomials `stride` u32 apart, only the first n of each transformed, the
// rest untouched; canonical values; natural order; synchronous; returns a
// cudaError_t value (0 = success).
//
// What changes: the reference uploads its roots and converts them to
// Montgomery form on every call, creates three streams and three chunk
// buffers per call, and runs log2(n) + 3 device passes per chunk. Here a
// per-device context keeps the twiddle tables and the chunk buffers alive
// across calls, and the device work per chunk is one transpose in, one
// single-pass transform, one transpose out.
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "extend.cuh"
#include "internal.hpp"

namespace zb {

namespace {

// out[c][r] = in[g(r)][c] for an R x Cn u32 matrix (both dense), where
// g(r) = r, or (r * gmul) mod R when gmul != 1 (R a power of two: the output
// permutation of a caller's root table). The row tiles are walked with a grid
// stride in y, so any R fits the 65535-block limit of gridDim.y (R reaches
// 2^24 polynomials per chunk at n = 2).
__global__ void k_transpose(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t R, uint32_t Cn,
                            uint32_t gmul) {
    __shared__ uint32_t tile[32][33];
    const uint32_t c0 = blockIdx.x * 32;
    for (uint32_t r0 = blockIdx.y * 32; r0 < R; r0 += gridDim.y * 32) {
        for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
            const uint32_t r = r0 + i, c = c0 + threadIdx.x;
            const uint32_t g = gmul == 1 ? r : (r * gmul) & (R - 1);
            if (r < R && c < Cn) tile[i][threadIdx.x] = in[(size_t)g * Cn + c];
        }
        __syncthreads();
        for (uint32_t i = threadIdx.y; i < 32; i += blockDim.y) {
            const uint32_t c = c0 + i, r = r0 + threadIdx.x;
            if (r < R && c < Cn) out[(size_t)c * R + r] = tile[threadIdx.x][i];
        }
        __syncthreads();  // the tile is rewritten by the next row tile
    }
}

zoda_status transpose(const uint32_t* in, uint32_t* out, uint32_t R, uint32_t Cn, cudaStream_t st,
                      uint32_t gmul = 1) {
    const uint32_t gy = (R + 31) / 32;
    dim3 grid((Cn + 31) / 32, gy < 65535u ? gy : 65535u), block(32, 8);
    k_transpose<<<grid, block, 0, st>>>(in, out, R, Cn, gmul);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

template <int LOG_N, bool INV>
zoda_status colntt_t(const zoda_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t cols, Tw scale, uint32_t a,
                     cudaStream_t st) {
    using PL = ExtPlan<LOG_N>;
    // per call: the attribute belongs to the current device, and calls may come on any device
    if (PL::SMEM > 0)
        ZB_CUDA(cudaFuncSetAttribute(k_colntt<LOG_N, INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PL::SMEM));
    const uint64_t ntiles = (cols + PL::C - 1) / PL::C;
    const uint64_t grid = ntiles < (uint64_t)ctx->sm_count ? ntiles : (uint64_t)ctx->sm_count;
    k_colntt<LOG_N, INV><<<(unsigned)grid, PL::THREADS, PL::SMEM, st>>>(in, out, cols, ntiles, ctx->tables.tw, scale, a);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

template <bool INV>
zoda_status colntt(const zoda_ctx* ctx, int log_n, const uint32_t* in, uint32_t* out, uint64_t cols, Tw scale,
                   uint32_t a, cudaStream_t st) {
    switch (log_n) {
#define ZB_CASE(L) \
    case L: return colntt_t<L, INV>(ctx, in, out, cols, scale, a, st);
        ZB_CASE(1) ZB_CASE(2) ZB_CASE(3) ZB_CASE(4) ZB_CASE(5) ZB_CASE(6)
        ZB_CASE(7) ZB_CASE(8) ZB_CASE(9) ZB_CASE(10) ZB_CASE(11) ZB_CASE(12)
#undef ZB_CASE
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

struct LegacyState {
    zoda_ctx* ctx = nullptr;
    DevBuf a, b;
    std::map<uint32_t, std::vector<uint32_t>> roots_seen;  // n -> last validated table
    std::map<uint32_t, uint32_t> perm;                      // n -> a^-1 mod n
};

std::mutex g_mu;
std::map<int, LegacyState> g_state;  // per CUDA device

int log2_u32(uint32_t n) {
    int l = 0;
    while ((1u << l) < n) l++;
    return l;
}

// Checks that roots = [w^0 .. w^(n-1)] for a primitive n-th root w and returns,
// through perm_out, a^-1 mod n where w = omega_n^a (omega_n the library's root).
bool check_roots(LegacyState& S, const uint32_t* roots, uint32_t n, uint32_t* perm_out) {
    auto it = S.roots_seen.find(n);
    if (it != S.roots_seen.end() && memcmp(it->second.data(), roots, n * sizeof(uint32_t)) == 0) {
        *perm_out = S.perm[n];
        return true;
    }
    if (roots[0] != 1) return false;
    const int L = log2_u32(n);
    if (n == 1) {
        S.roots_seen[n].assign(roots, roots + 1);
        S.perm[n] = 0;
        *perm_out = 0;
        return true;
    }
    const uint32_t w = roots[1];
    for (uint32_t i = 1; i < n; i++)
        if (roots[i] >= P || roots[i] != mulmod_c(roots[i - 1], w)) return false;
    if (mulmod_c(roots[n - 1], w) != 1 || powmod_c(w, n / 2) != P - 1) return false;  // order exactly n
    // discrete log of w to base omega_n, bit by bit (cyclic group of order 2^L)
    const uint32_t om = root_of_unity(L);
    uint32_t a = 0;
    for (int i = 0; i < L; i++) {
        const uint32_t cur = mulmod_c(w, powmod_c(om, (uint64_t)n - a));  // w * omega^-a
        if (powmod_c(cur, (uint64_t)1 << (L - 1 - i)) != 1) a |= 1u << i;
    }
    // a is odd; invert mod 2^L by Newton iteration
    uint32_t inv = a;
    for (int i = 0; i < 5; i++) inv *= 2u - a * inv;
    inv &= n - 1;
    S.roots_seen[n].assign(roots, roots + n);
    S.perm[n] = inv;
    *perm_out = inv;
    return true;
}

int to_cuda_error(zoda_status s) {
    switch (s) {
        case ZODA_OK: return (int)cudaSuccess;
        case ZODA_ERR_ARG: return (int)cudaErrorInvalidValue;
        case ZODA_ERR_NOMEM: return (int)cudaErrorMemoryAllocation;
        case ZODA_ERR_UNSUPPORTED: return (int)cudaErrorNotSupported;
        default: return (int)cudaErrorUnknown;
    }
}

zoda_status legacy_run(uint32_t* values, const uint32_t* roots, uint32_t n, uint32_t polys, uint32_t stride,
                       bool inverse) {
    if (polys == 0) return ZODA_OK;
    if (!values || !roots || n == 0 || (n & (n - 1)) || stride < n) return ZODA_ERR_ARG;
    const int L = log2_u32(n);
    int dev = 0;
    ZB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(g_mu);
    LegacyState& S = g_state[dev];
    uint32_t a_inv = 0;
    if (!check_roots(S, roots, n, &a_inv)) return ZODA_ERR_ARG;
    if (n == 1) return ZODA_OK;  // a length-1 transform (and its 1^-1 scale) is the identity
    if (L > LONG_MAX_LOG) {
        set_last_error_text("cuda_ntt/cuda_intt: n above 2^26 is not supported");
        return ZODA_ERR_UNSUPPORTED;
    }
    // above 4096 points: four-step passes in natural order, and the caller's
    // root w = omega^a applied when transposing back: X_w[j] = X_omega[a * j]
    const bool long_n = L > 12;
    uint32_t a_fwd = a_inv;  // a = (a^-1)^-1 mod n, by Newton's iteration mod 2^32
    for (int i = 0; i < 5; i++) a_fwd *= 2u - a_inv * a_fwd;
    a_fwd &= n - 1;
    if (!S.ctx) {
        zoda_status s = zoda_ctx_create(dev, &S.ctx);
        if (s != ZODA_OK) return s;
    }
    zoda_ctx* ctx = S.ctx;
    cudaStream_t st = ctx->stream;
    const uint32_t n_inv = inverse ? powmod_c(n, P - 2) : 1u;
    const Tw scale{n_inv, shoup(n_inv)};
    // chunk of polynomials per device round trip (~128 MiB each way)
    const uint64_t per_poly = (uint64_t)n * 4;
    uint64_t chunk = ((uint64_t)128 << 20) / per_poly;
    if (chunk < 4) chunk = 4;
    if (chunk > polys) chunk = polys;
    const uint64_t chunk4 = (chunk + 3) & ~3ull;
    zoda_status s;
    if ((s = S.a.ensure(chunk4 * per_poly)) != ZODA_OK) return s;
    if ((s = S.b.ensure(chunk4 * per_poly)) != ZODA_OK) return s;
    uint32_t* A = (uint32_t*)S.a.p;
    uint32_t* B = (uint32_t*)S.b.p;
    for (uint64_t p0 = 0; p0 < polys; p0 += chunk) {
        const uint64_t w = (polys - p0 < chunk) ? polys - p0 : chunk;
        const uint64_t w4 = (w + 3) & ~3ull;
        uint32_t* host = values + p0 * stride;
        ZB_CUDA(cudaMemcpy2DAsync(A, per_poly, host, (size_t)stride * 4, per_poly, w, cudaMemcpyHostToDevice, st));
        if (w4 != w) ZB_CUDA(cudaMemsetAsync(A + w * n, 0, (w4 - w) * per_poly, st));
        if ((s = transpose(A, B, (uint32_t)w4, n, st)) != ZODA_OK) return s;  // B = [n][w4]
        if (long_n) {
            if ((s = long_cols_ntt(ctx, B, A, L, w4, inverse, scale, st)) != ZODA_OK) return s;
            if ((s = transpose(A, B, n, (uint32_t)w4, st, a_fwd)) != ZODA_OK) return s;  // B = [w4][n], permuted
        } else {
            s = inverse ? colntt<true>(ctx, L, B, A, w4, scale, a_inv, st)
                        : colntt<false>(ctx, L, B, A, w4, scale, a_inv, st);
            if (s != ZODA_OK) return s;
            if ((s = transpose(A, B, n, (uint32_t)w4, st)) != ZODA_OK) return s;  // B = [w4][n]
        }
        ZB_CUDA(cudaMemcpy2DAsync(host, (size_t)stride * 4, B, per_poly, per_poly, w, cudaMemcpyDeviceToHost, st));
    }
    ZB_CUDA(cudaStreamSynchronize(st));
    return ZODA_OK;
}

}  // namespace

}  // namespace zb

extern "C" {

uint32_t* cuda_host_alloc(size_t count) {
    void* p = nullptr;
    return cudaHostAlloc(&p, count * sizeof(uint32_t), cudaHostAllocDefault) == cudaSuccess ? (uint32_t*)p : nullptr;
}

void cuda_host_free(uint32_t* p) {
    if (p) cudaFreeHost(p);
}

int cuda_ntt(uint32_t* values, const uint32_t* roots, uint32_t n, uint32_t polys, uint32_t stride) {
    return zb::to_cuda_error(zb::legacy_run(values, roots, n, polys, stride, false));
}

int cuda_intt(uint32_t* values, const uint32_t* roots, uint32_t n, uint32_t polys, uint32_t stride) {
    return zb::to_cuda_error(zb::legacy_run(values, roots, n, polys, stride, true));
}

}  // extern "C"
