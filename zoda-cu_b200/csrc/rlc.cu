// Row-side consumers of the encoding: data root, RLC coefficients, per-row
// random linear combinations and the RLC check (include/zoda_b200.h, part 2).
//
//   data root      SHA-256 over every encoded row's little-endian u32 bytes,
//                  lowercase hex (src/benchmarks/utils.rs:51-59); sequential,
//                  so it runs on the host as in the reference.
//   coefficients   column i: SHA-256(root_hex || u64_le(i)), four limbs from
//                  the digest's big-endian 8-byte windows, each reduced mod p
//                  (src/zoda/rlc.rs:48-65); one device thread per column, the
//                  root's whole 64-byte blocks compressed once on the host.
//   rows           rlc[r][l] = sum_c x[r][c] * coeff[c][l] mod p
//                  (src/zoda/rlc.rs:32-40) as a device reduction over the
//                  row-major matrix: one HBM read of it, Shoup products with
//                  the coefficients' companions, 64-bit lazy sums.
//   check          RLC(encoded row j) == extension of the data rows' RLC at j,
//                  limb for limb, for EVERY row (the reference samples 64:
//                  utils.rs:225-272); the extension of the k x 4 RLC matrix is
//                  the library's own encode with cols = 4.
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.hpp"
#include "sha256.hpp"

namespace zb {
namespace sha {

namespace {
using u128 = unsigned __int128;
uint64_t isqrt128(u128 v) {  // floor(sqrt(v)) for v < 2^100
    uint64_t lo = 0, hi = 1ull << 50;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo + 1) / 2;
        if ((u128)mid * mid <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
uint64_t icbrt128(u128 v) {  // floor(cbrt(v)) for v < 2^120
    uint64_t lo = 0, hi = 1ull << 40;
    while (lo < hi) {
        const uint64_t mid = lo + (hi - lo + 1) / 2;
        if ((u128)mid * mid * mid <= v) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}
}  // namespace

const Consts& consts() {
    static Consts c = [] {
        Consts r{};
        int found = 0;
        for (uint64_t n = 2; found < 64; n++) {
            bool prime = true;
            for (uint64_t d = 2; d * d <= n; d++)
                if (n % d == 0) {
                    prime = false;
                    break;
                }
            if (!prime) continue;
            r.k[found] = (uint32_t)icbrt128((u128)n << 96);  // low 32 bits: the fraction
            if (found < 8) r.h0[found] = (uint32_t)isqrt128((u128)n << 64);
            found++;
        }
        return r;
    }();
    return c;
}

Hasher::Hasher() { memcpy(h_, consts().h0, sizeof h_); }

void Hasher::update(const void* data, size_t len) {
    const uint8_t* p = (const uint8_t*)data;
    len_ += len;
    const uint32_t* k = consts().k;
    uint32_t w[16];
    auto block = [&](const uint8_t* b) {
        for (int i = 0; i < 16; i++)
            w[i] = (uint32_t)b[4 * i] << 24 | (uint32_t)b[4 * i + 1] << 16 | (uint32_t)b[4 * i + 2] << 8 | b[4 * i + 3];
        compress(h_, w, k);
    };
    if (n_) {
        const size_t t = len < 64 - n_ ? len : 64 - n_;
        memcpy(buf_ + n_, p, t);
        n_ += t;
        p += t;
        len -= t;
        if (n_ < 64) return;
        block(buf_);
        n_ = 0;
    }
    for (; len >= 64; p += 64, len -= 64) block(p);
    memcpy(buf_, p, len);
    n_ = len;
}

void Hasher::final(uint8_t out[32]) {
    const uint64_t bits = len_ * 8;
    const uint8_t pad = 0x80;
    update(&pad, 1);
    const uint8_t zero[64] = {};
    update(zero, n_ <= 56 ? 56 - n_ : 120 - n_);
    uint8_t L[8];
    for (int i = 0; i < 8; i++) L[i] = (uint8_t)(bits >> (56 - 8 * i));
    update(L, 8);
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 4; j++) out[4 * i + j] = (uint8_t)(h_[i] >> (24 - 8 * j));
}

}  // namespace sha

namespace {

__constant__ uint32_t c_sha_k[64];

struct CoeffJob {
    uint32_t mid[8];     // state after the root's whole 64-byte blocks
    uint8_t tail[64];    // the root's remaining bytes
    uint32_t tail_len;   // < 64
    uint64_t total_len;  // root length + 8
};

// coeff[i][l] = be64(digest[8l .. 8l+8)) mod p, digest = SHA-256(root || u64_le(i))
__global__ void k_rlc_coeff(const CoeffJob job, uint64_t ncols, uint32_t* __restrict__ coeff) {
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= ncols) return;
    uint8_t m[128];
    uint32_t n = 0;
    for (uint32_t j = 0; j < job.tail_len; j++) m[n++] = job.tail[j];
    for (int j = 0; j < 8; j++) m[n++] = (uint8_t)(i >> (8 * j));
    m[n++] = 0x80;
    const uint32_t nblk = n + 8 <= 64 ? 1 : 2;
    while (n < nblk * 64 - 8) m[n++] = 0;
    const uint64_t bits = job.total_len * 8;
    for (int j = 0; j < 8; j++) m[n++] = (uint8_t)(bits >> (56 - 8 * j));
    uint32_t h[8];
    for (int j = 0; j < 8; j++) h[j] = job.mid[j];
    uint32_t w[16];
    for (uint32_t b = 0; b < nblk; b++) {
        for (int j = 0; j < 16; j++) {
            const uint8_t* q = m + 64 * b + 4 * j;
            w[j] = (uint32_t)q[0] << 24 | (uint32_t)q[1] << 16 | (uint32_t)q[2] << 8 | q[3];
        }
        sha::compress(h, w, c_sha_k);
    }
    for (int l = 0; l < 4; l++) {
        const uint64_t v = (uint64_t)h[2 * l] << 32 | h[2 * l + 1];
        coeff[i * 4 + l] = (uint32_t)(v % P);
    }
}

// Shoup companions of the coefficient limbs, one uint4 pair per column.
__global__ void k_rlc_prep(const uint4* __restrict__ coeff, uint64_t ncols, uint4* __restrict__ w,
                           uint4* __restrict__ ws) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < ncols;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint4 c = coeff[i];
        c.x %= P;  // canonical limbs (a caller's table may hold any u32)
        c.y %= P;
        c.z %= P;
        c.w %= P;
        w[i] = c;
        ws[i] = make_uint4(shoup(c.x), shoup(c.y), shoup(c.z), shoup(c.w));
    }
}

// 4 rows per CTA: 16 lazy 64-bit sums per thread keep the kernel at two
// 256-thread CTAs per SM (measured 1.5x faster than 8 rows at one CTA).
constexpr int RB = 4;  // rows per CTA

// acc[r][l] += (sum over this CTA's columns of x[r][c] * coeff[c][l]) mod p
__global__ void __launch_bounds__(256, 2) k_rlc_rows(const uint32_t* __restrict__ x, uint64_t pitch,
                                                               uint32_t rows, uint64_t quads,
                                                               const uint4* __restrict__ cw,
                                                               const uint4* __restrict__ cws,
                                                               unsigned long long* __restrict__ acc) {
    const uint32_t r0 = blockIdx.y * RB;
    uint64_t s[RB][4];
#pragma unroll
    for (int r = 0; r < RB; r++)
#pragma unroll
        for (int l = 0; l < 4; l++) s[r][l] = 0;
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < quads; q += (uint64_t)gridDim.x * blockDim.x) {
        uint4 w[4], ws[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            w[j] = __ldg(cw + 4 * q + j);
            ws[j] = __ldg(cws + 4 * q + j);
        }
#pragma unroll
        for (int r = 0; r < RB; r++) {
            if (r0 + r >= rows) break;
            const uint4 v = __ldcs(reinterpret_cast<const uint4*>(x + (uint64_t)(r0 + r) * pitch) + q);
            const uint32_t xv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int j = 0; j < 4; j++) {
                s[r][0] += mul_lazy(xv[j], w[j].x, ws[j].x);
                s[r][1] += mul_lazy(xv[j], w[j].y, ws[j].y);
                s[r][2] += mul_lazy(xv[j], w[j].z, ws[j].z);
                s[r][3] += mul_lazy(xv[j], w[j].w, ws[j].w);
            }
        }
    }
    __shared__ unsigned long long red[8][RB * 4];
    static_assert(RB * 4 <= 256, "one thread per (row, limb) in the final step");
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int r = 0; r < RB; r++)
#pragma unroll
        for (int l = 0; l < 4; l++) {
            uint64_t v = s[r][l] % P;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
            if (lane == 0) red[wid][r * 4 + l] = v;
        }
    __syncthreads();
    if (threadIdx.x < RB * 4) {
        const int r = threadIdx.x / 4;
        if (r0 + r < rows) {
            uint64_t v = 0;
            for (int w2 = 0; w2 < (int)(blockDim.x / 32); w2++) v += red[w2][threadIdx.x];
            atomicAdd(acc + (uint64_t)(r0 + r) * 4 + (threadIdx.x & 3), (unsigned long long)(v % P));
        }
    }
}

__global__ void k_rlc_final(const unsigned long long* __restrict__ acc, uint64_t n, uint32_t* __restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)(acc[i] % P);
}

__global__ void k_count_diff(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b, uint64_t n,
                             unsigned long long* __restrict__ cnt) {
    unsigned long long c = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        c += a[i] != b[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, c);
}

unsigned grid1(const zoda_ctx* ctx, uint64_t n) {
    const uint64_t g = (n + 255) / 256, cap = (uint64_t)ctx->sm_count * 8;
    return (unsigned)(g < 1 ? 1 : g > cap ? cap : g);
}

// rlc of rows [rows][cols] (pitch cols) into out [rows][4]; tables w/ws prepared.
zoda_status rlc_rows(const zoda_ctx* ctx, const uint32_t* x, uint32_t rows, uint64_t cols, const uint4* w,
                     const uint4* ws, unsigned long long* acc, uint32_t* out, cudaStream_t st) {
    ZB_CUDA(cudaMemsetAsync(acc, 0, (size_t)rows * 4 * sizeof(unsigned long long), st));
    const uint64_t quads = cols / 4;
    const uint32_t gy = (rows + RB - 1) / RB;
    uint64_t gx = (quads + 256 * 8 - 1) / (256 * 8) * (8 / RB);  // ~RB column quads per thread
    if (gx < 1) gx = 1;
    if (gy > 65535) {
        set_last_error_text("rlc: more than 262140 rows");
        return ZODA_ERR_UNSUPPORTED;
    }
    if (quads) {
        k_rlc_rows<<<dim3((unsigned)gx, gy), 256, 0, st>>>(x, cols, rows, quads, w, ws, acc);
        ZB_CUDA(cudaGetLastError());
    }
    k_rlc_final<<<grid1(ctx, (uint64_t)rows * 4), 256, 0, st>>>(acc, (uint64_t)rows * 4, out);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

zoda_status prep_tables(zoda_ctx* ctx, const uint32_t* d_coeff, uint64_t cols, cudaStream_t st) {
    zoda_status s;
    if ((s = ctx->rlc_w.ensure(cols * 16 + 16)) != ZODA_OK) return s;
    if ((s = ctx->rlc_ws.ensure(cols * 16 + 16)) != ZODA_OK) return s;
    k_rlc_prep<<<grid1(ctx, cols), 256, 0, st>>>((const uint4*)d_coeff, cols, (uint4*)ctx->rlc_w.p,
                                                 (uint4*)ctx->rlc_ws.p);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

}  // namespace

void rlc_release(zoda_ctx* ctx) {
    for (DevBuf* b : {&ctx->rlc_w, &ctx->rlc_ws, &ctx->rlc_acc, &ctx->rlc_d, &ctx->rlc_e, &ctx->rlc_f, &ctx->rlc_cnt})
        b->release();
}

}  // namespace zb

using namespace zb;

extern "C" {

zoda_status zoda_data_root_host(const uint32_t* rows, uint64_t nrows, uint64_t cols, char out_hex[65]) {
    if ((!rows && nrows * cols) || !out_hex) return ZODA_ERR_ARG;
    sha::Hasher h;
    // the rows' u32 values as little-endian bytes, row after row
    std::vector<uint8_t> buf;
    const uint64_t n = nrows * cols;
    const uint64_t chunk = 1 << 20;
    buf.resize(chunk * 4);
    for (uint64_t i = 0; i < n; i += chunk) {
        const uint64_t m = n - i < chunk ? n - i : chunk;
        for (uint64_t j = 0; j < m; j++) {
            const uint32_t v = rows[i + j];
            buf[4 * j] = (uint8_t)v;
            buf[4 * j + 1] = (uint8_t)(v >> 8);
            buf[4 * j + 2] = (uint8_t)(v >> 16);
            buf[4 * j + 3] = (uint8_t)(v >> 24);
        }
        h.update(buf.data(), m * 4);
    }
    uint8_t d[32];
    h.final(d);
    for (int i = 0; i < 32; i++) snprintf(out_hex + 2 * i, 3, "%02x", d[i]);
    out_hex[64] = 0;
    return ZODA_OK;
}

zoda_status zoda_rlc_coefficients_device(zoda_ctx* ctx, const char* root, size_t root_len, uint64_t ncols,
                                         uint32_t* d_coeff, void* stream) {
    if (!ctx || (!root && root_len) || !d_coeff) return ZODA_ERR_ARG;
    if (ncols == 0) return ZODA_OK;
    ZB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    sha::Hasher h;
    const size_t whole = root_len / 64 * 64;
    h.update(root, whole);
    CoeffJob job{};
    memcpy(job.mid, h.state(), sizeof job.mid);
    job.tail_len = (uint32_t)(root_len - whole);
    memcpy(job.tail, root + whole, job.tail_len);
    job.total_len = (uint64_t)root_len + 8;
    ZB_CUDA(cudaMemcpyToSymbolAsync(c_sha_k, sha::consts().k, sizeof(uint32_t) * 64, 0, cudaMemcpyHostToDevice, st));
    k_rlc_coeff<<<(unsigned)((ncols + 127) / 128), 128, 0, st>>>(job, ncols, d_coeff);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

zoda_status zoda_rlc_rows_device(zoda_ctx* ctx, const uint32_t* d_rows, uint32_t rows, uint64_t cols,
                                 const uint32_t* d_coeff, uint32_t* d_out, void* stream) {
    if (!ctx || !d_rows || !d_coeff || !d_out || cols % 4 != 0) return ZODA_ERR_ARG;
    if (((uintptr_t)d_rows | (uintptr_t)d_coeff) & 15) return ZODA_ERR_ARG;
    if (rows == 0) return ZODA_OK;
    ZB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    std::lock_guard<std::mutex> lock(ctx->rlc_mu);
    zoda_status s = prep_tables(ctx, d_coeff, cols, st);
    if (s != ZODA_OK) return s;
    if ((s = ctx->rlc_acc.ensure((size_t)rows * 4 * 8)) != ZODA_OK) return s;
    return rlc_rows(ctx, d_rows, rows, cols, (const uint4*)ctx->rlc_w.p, (const uint4*)ctx->rlc_ws.p,
                    (unsigned long long*)ctx->rlc_acc.p, d_out, st);
}

zoda_status zoda_rlc_check_device(zoda_ctx* ctx, const uint32_t* d_data, const uint32_t* d_code, uint32_t k,
                                  uint32_t n, uint64_t cols, const uint32_t* d_coeff, uint64_t* mismatches,
                                  void* stream) {
    if (!ctx || !d_data || !d_code || !d_coeff || !mismatches || k == 0 || cols % 4 != 0) return ZODA_ERR_ARG;
    if (((uintptr_t)d_data | (uintptr_t)d_code | (uintptr_t)d_coeff) & 15) return ZODA_ERR_ARG;
    ZB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t rows = k + n;
    std::lock_guard<std::mutex> lock(ctx->rlc_mu);
    zoda_status s = prep_tables(ctx, d_coeff, cols, st);
    if (s != ZODA_OK) return s;
    if ((s = ctx->rlc_acc.ensure((size_t)rows * 4 * 8)) != ZODA_OK) return s;
    if ((s = ctx->rlc_d.ensure((size_t)k * 16)) != ZODA_OK) return s;
    if ((s = ctx->rlc_e.ensure((size_t)rows * 16)) != ZODA_OK) return s;
    if ((s = ctx->rlc_f.ensure((size_t)rows * 16)) != ZODA_OK) return s;
    if ((s = ctx->rlc_cnt.ensure(8)) != ZODA_OK) return s;
    const uint4* w = (const uint4*)ctx->rlc_w.p;
    const uint4* ws = (const uint4*)ctx->rlc_ws.p;
    unsigned long long* acc = (unsigned long long*)ctx->rlc_acc.p;
    uint32_t *D = (uint32_t*)ctx->rlc_d.p, *E = (uint32_t*)ctx->rlc_e.p, *F = (uint32_t*)ctx->rlc_f.p;
    if ((s = rlc_rows(ctx, d_data, k, cols, w, ws, acc, D, st)) != ZODA_OK) return s;
    // the RLC and the extension commute (both F_p-linear): extend the k x 4 RLC matrix
    if ((s = zoda_encode_device(ctx, D, F, k, n, 4, st)) != ZODA_OK) return s;
    if ((s = rlc_rows(ctx, d_code, rows, cols, w, ws, acc, E, st)) != ZODA_OK) return s;
    ZB_CUDA(cudaMemsetAsync(ctx->rlc_cnt.p, 0, 8, st));
    k_count_diff<<<grid1(ctx, (uint64_t)rows * 4), 256, 0, st>>>(E, F, (uint64_t)rows * 4,
                                                                (unsigned long long*)ctx->rlc_cnt.p);
    ZB_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    ZB_CUDA(cudaMemcpyAsync(&h, ctx->rlc_cnt.p, 8, cudaMemcpyDeviceToHost, st));
    ZB_CUDA(cudaStreamSynchronize(st));
    *mismatches = h;
    return ZODA_OK;
}

}  // extern "C"
