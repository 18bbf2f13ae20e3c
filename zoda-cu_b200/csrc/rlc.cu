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
//                  row-major matrix: one HBM read of it through a bulk-copy
//                  ring, centered residues, signed 64-bit sums of wide
//                  products with one shift-and-add fold per eight.
//   check          RLC(encoded row j) == extension of the data rows' RLC at j,
//                  limb for limb, for EVERY row (the reference samples 64:
//                  utils.rs:225-272); the extension of the k x 4 RLC matrix is
//                  the library's own encode with cols = 4.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "async.cuh"
#include "internal.hpp"
#include "sha256.hpp"
#include "tma_host.hpp"

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

// ---- per-row RLC --------------------------------------------------------------
// Residues are handled in centered form, r - p for r > (p-1)/2, so |x|, |c| <=
// (p-1)/2 and a product is below 2^60 in magnitude: eight of them on top of a
// folded sum stay inside a signed 64-bit word (0.95 * 2^63 at worst), and a
// product is one signed wide multiply-add. 2^32 = 2p + (2^28 - 2) gives the
// fold h*2^32 + lo == h*(2^28 - 2) + lo (mod p), done with shifts and adds so
// that the multiply pipe only carries the products; its result lies in
// (-2^59, 2^59 + 2^32).
constexpr uint32_t HALF_P = (P - 1) / 2;
constexpr uint32_t TWO32_MOD_P = 268435454u;
static_assert((uint64_t)TWO32_MOD_P == (1ull << 32) - 2ull * P && TWO32_MOD_P == (1u << 28) - 2, "2^32 mod p");
// p * 2^29 exceeds every folded magnitude: adding it makes a folded sum a
// non-negative value below 2^62 with the same residue.
constexpr uint64_t P_SHIFT29 = (uint64_t)P << 29;

__host__ __device__ __forceinline__ int32_t centered(uint32_t r) {  // r in [0, p + 2^28)
    return (int32_t)(r > HALF_P ? r - P : r);
}
// any u32 -> its centered residue: one subtract-min leaves [0, 2^32 - p) =
// [0, p + 2^28 - 2), whose part past p is already below (p-1)/2 after - p
__device__ __forceinline__ int32_t centered_any(uint32_t v) { return centered(reduce_2p(v)); }
__device__ __forceinline__ int64_t sfold(int64_t a) {
    // h*2^28 - 2h + lo on the integer ALU: funnel shifts build the 64-bit terms,
    // carry-chained adds combine them, so the fold leaves the multiply pipe to
    // the products (4% faster row kernel on B200 than the same fold written as
    // 64-bit shifts, which can become a wide multiply)
    const uint32_t lo = (uint32_t)a, h = (uint32_t)(a >> 32);
    const uint32_t t_lo = __funnelshift_l(0u, h, 28), t_hi = (uint32_t)((int32_t)h >> 4);
    const uint32_t d_lo = __funnelshift_l(0u, h, 1), d_hi = (uint32_t)((int32_t)h >> 31);
    uint32_t r_lo, r_hi;
    asm("add.cc.u32 %0, %2, %3;\n\t"
        "addc.u32 %1, %4, 0;\n\t"
        "sub.cc.u32 %0, %0, %5;\n\t"
        "subc.u32 %1, %1, %6;"
        : "=&r"(r_lo), "=&r"(r_hi)
        : "r"(t_lo), "r"(lo), "r"(t_hi), "r"(d_lo), "r"(d_hi));
    return (int64_t)(((uint64_t)r_hi << 32) | r_lo);
}
// unsigned fold for the final reduction: a < 2^64 -> a' == a (mod p), a' < 2^60
__device__ __forceinline__ uint64_t fold32(uint64_t a) {
    return (uint64_t)(uint32_t)(a >> 32) * TWO32_MOD_P + (uint32_t)a;
}

// Centered copies of the coefficient limbs (a caller's table may hold any u32):
//   planar  four planes, plane j holding for every column quad q the limbs of
//           column 4q + j, so one plane of a column chunk is one contiguous copy
//           (the few-rows kernel);
//   rowwise [column][limb] padded with zero columns to npad, a multiple of the
//           row kernel's 32-column chunk.
// A null table pointer skips that layout.
__global__ void k_rlc_prep(const uint4* __restrict__ coeff, uint64_t quads, uint64_t npad, int4* __restrict__ planar,
                           int4* __restrict__ rowwise) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < npad;
         i += (uint64_t)gridDim.x * blockDim.x) {
        int4 w = make_int4(0, 0, 0, 0);
        if (i < 4 * quads) {
            const uint4 c = coeff[i];
            w = make_int4(centered(c.x % P), centered(c.y % P), centered(c.z % P), centered(c.w % P));
            if (planar) planar[(i & 3) * quads + (i >> 2)] = w;
        }
        if (rowwise) rowwise[i] = w;
    }
}

__device__ __forceinline__ int32_t limb(const int4& v, int l) {
    return l == 0 ? v.x : l == 1 ? v.y : l == 2 ? v.z : v.w;
}

// Warp sum of NV values per lane (NV = 16 or 32) that halves the set at each
// exchange: at offset o a lane keeps one half, sends the other and adds what
// its partner sent for the kept half. NV - 1 64-bit shuffles (plus one for
// NV = 16) instead of 5 * NV. Afterwards v[0] holds the warp's total of value
// lane >> 1 (NV = 16) or lane (NV = 32).
template <int NV>
__device__ __forceinline__ void warp_sum_split(uint64_t (&v)[NV], int lane) {
#pragma unroll
    for (int h = NV / 2; h >= 1; h >>= 1) {
        const int o = h * 32 / NV;
        const bool up = lane & o;
#pragma unroll
        for (int i = 0; i < h; i++) {
            const uint64_t send = up ? v[i] : v[i + h];
            const uint64_t keep = up ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xFFFFFFFFu, send, o);
        }
    }
    if (NV == 16) v[0] += __shfl_xor_sync(0xFFFFFFFFu, v[0], 1);
}

// The work is the sequence of units (row block rb, column chunk ch), row block
// major: u = rb * nch + ch. CTA b of G takes units [b*U/G, (b+1)*U/G), so every
// CTA gets the same share to one unit. A unit is UROWS rows x CHQ column quads
// of the matrix plus the chunk's four coefficient planes; the producer warp
// brings it into one of NST shared-memory stages with 1D bulk copies, one copy
// per lane, and CG groups of 256 consumer threads (RPT rows each, QPU quads per
// thread) fold it into their sums. The sums are flushed (reduced, then added to
// acc) when the row block changes and at the end of the range.
namespace rlcb {
constexpr int CG = 2;
constexpr int RPT = 4;
constexpr int UROWS = CG * RPT;
constexpr int QPU = 2;  // quads per consumer thread per unit: 4 * QPU <= 8 products per fold
constexpr int CHQ = 256 * QPU;
constexpr int NST = 2;
constexpr int X_BYTES = UROWS * CHQ * 16;
constexpr int STAGE_BYTES = X_BYTES + 4 * CHQ * 16;
constexpr int OFF_RED = NST * STAGE_BYTES;
constexpr int NV = RPT * 4;
constexpr int OFF_BAR = OFF_RED + CG * 8 * NV * 8;
constexpr int SMEM = OFF_BAR + 2 * NST * 8;
constexpr int THREADS = CG * 256 + 32;
static_assert(QPU >= 1 && QPU <= 2, "at most eight centered products between folds");
static_assert(NV == 16 || NV == 32, "warp_sum_split takes 16 or 32 values");
static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
static_assert(UROWS + 4 <= 32, "one producer lane per copy");
}  // namespace rlcb

// acc[r][l] += (sum over the CTA's columns of x[r][c] * coeff[c][l]) mod p;
// x may hold any u32 (reduced on load), cw is the centered planar table.
__global__ void __launch_bounds__(rlcb::THREADS, 1) k_rlc_rows(const uint32_t* __restrict__ x, uint64_t pitch,
                                                               uint32_t rows, uint64_t quads,
                                                               const int4* __restrict__ cw,
                                                               unsigned long long* __restrict__ acc,
                                                               int* __restrict__ err) {
    using namespace rlcb;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + OFF_BAR);  // stage landed (bulk tx)
    uint64_t* empty = full + NST;                                   // every consumer warp is done with it
    const int tid = threadIdx.x;
    const uint64_t nch = (quads + CHQ - 1) / CHQ;
    const uint64_t U = nch * ((rows + UROWS - 1) / UROWS);
    const uint64_t u0 = U * blockIdx.x / gridDim.x, u1 = U * (blockIdx.x + 1) / gridDim.x;
    if (tid == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CG * 8);
        }
        fence_mbar_init();
    }
    __syncthreads();
    // the unit's position is carried along (no division per unit): row block rb,
    // chunk ch, stage s and that stage's phase parity ph
    const uint32_t rb0 = (uint32_t)(u0 / nch);
    const uint64_t ch0 = u0 % nch;
    if (tid >= CG * 256) {  // producer warp
        const int pl = tid - CG * 256;
        uint32_t rb = rb0, ph = 0;
        uint64_t ch = ch0;
        int s = 0;
        bool reuse = false;  // from the second pass over the stages on
        for (uint64_t u = u0; u < u1; u++) {
            if (reuse) {
                bool ok = true;
                if (pl == 0) ok = mbar_wait_bounded(&empty[s], ph ^ 1);
                if (!__shfl_sync(0xFFFFFFFFu, ok, 0)) {
                    if (pl == 0) atomicOr(err, 4);  // the consumers then time out on `full` and leave
                    return;
                }
                fence_proxy_async();
            }
            const uint32_t r0 = rb * UROWS;
            const uint64_t q0 = ch * CHQ;
            const uint32_t bytes = (uint32_t)min((uint64_t)CHQ, quads - q0) * 16;
            const uint32_t nr = min((uint32_t)UROWS, rows - r0);
            unsigned char* st = smem + s * STAGE_BYTES;
            if (pl == 0) mbar_expect_tx(&full[s], bytes * (nr + 4));
            __syncwarp();
            if (pl < (int)nr)
                bulk_load_1d(st + pl * CHQ * 16, x + (uint64_t)(r0 + pl) * pitch + q0 * 4, bytes, &full[s]);
            else if (pl >= UROWS && pl < UROWS + 4)
                bulk_load_1d(st + X_BYTES + (pl - UROWS) * CHQ * 16, cw + (pl - UROWS) * quads + q0, bytes, &full[s]);
            if (++s == NST) {
                s = 0;
                ph ^= 1;
                reuse = true;
            }
            if (++ch == nch) {
                ch = 0;
                rb++;
            }
        }
        return;
    }
    const int g = tid >> 8, t = tid & 255, lane = tid & 31;
    const int bar = 1 + g;
    int64_t sum[NV];
#pragma unroll
    for (int i = 0; i < NV; i++) sum[i] = 0;
    unsigned long long* red = reinterpret_cast<unsigned long long*>(smem + OFF_RED) + g * 8 * NV;
    uint32_t rb = rb0, ph = 0;
    uint64_t ch = ch0;
    int s = 0;
    // A warp whose wait gives up flags the error and from then on only keeps
    // step: it arrives on `empty` and joins the flushes, so no barrier is left
    // short and every other warp finishes its units.
    bool dead = false;
    for (uint64_t u = u0; u < u1; u++) {
        if (!dead && !__all_sync(0xFFFFFFFFu, mbar_wait_bounded(&full[s], ph))) {
            dead = true;
            if (lane == 0) atomicOr(err, 1);
        }
        const uint32_t rg = rb * UROWS + g * RPT;  // this group's first row
        const uint64_t qb = ch * CHQ;
        const uint4* sx = reinterpret_cast<const uint4*>(smem + s * STAGE_BYTES);
        const int4* sc = reinterpret_cast<const int4*>(smem + s * STAGE_BYTES + X_BYTES);
#pragma unroll
        for (int k = 0; k < QPU; k++) {
            const int qi = k * 256 + t;
            if (dead || qb + qi >= quads) break;
            int4 w[4];
#pragma unroll
            for (int j = 0; j < 4; j++) w[j] = sc[j * CHQ + qi];
#pragma unroll
            for (int r = 0; r < RPT; r++) {
                if (rg + r >= rows) break;
                const uint4 v = sx[(g * RPT + r) * CHQ + qi];
                const int32_t xv[4] = {centered_any(v.x), centered_any(v.y), centered_any(v.z), centered_any(v.w)};
#pragma unroll
                for (int l = 0; l < 4; l++)
#pragma unroll
                    for (int j = 0; j < 4; j++) sum[r * 4 + l] += (int64_t)xv[j] * limb(w[j], l);
            }
        }
#pragma unroll
        for (int k = 0; k < NV; k++) sum[k] = sfold(sum[k]);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (u + 1 == u1 || ch + 1 == nch) {
            // flush: + p*2^29 makes the folded sums non-negative below 2^62, one fold
            // brings them below 2^57 (32 lanes < 2^62), the warp totals fold again
            // (8 warps < 2^62)
            uint64_t v[NV];
#pragma unroll
            for (int k = 0; k < NV; k++) v[k] = fold32((uint64_t)(sum[k] + (int64_t)P_SHIFT29));
            warp_sum_split<NV>(v, lane);
            if (NV == 32 || !(lane & 1)) red[(t >> 5) * NV + (NV == 32 ? lane : lane >> 1)] = fold32(v[0]);
            group_bar(bar, 256);
            if (t < NV && rg + t / 4 < rows) {
                uint64_t r = 0;
#pragma unroll
                for (int w2 = 0; w2 < 8; w2++) r += red[w2 * NV + t];
                atomicAdd(acc + (uint64_t)(rg + t / 4) * 4 + (t & 3), (unsigned long long)(r % P));
            }
            group_bar(bar, 256);  // red is free for the next flush
#pragma unroll
            for (int k = 0; k < NV; k++) sum[k] = 0;
        }
        if (++s == NST) {
            s = 0;
            ph ^= 1;
        }
        if (++ch == nch) {
            ch = 0;
            rb++;
        }
    }
}

// ---- row kernel: one consumer thread per row ------------------------------------
// For tall matrices. A unit is UROWS = 512 rows x 32 columns, two TMA boxes of
// 256 rows x 128 bytes with the 128-byte swizzle (a row's 16-byte chunk j sits
// at chunk j ^ (row & 7) of its 128-byte line, so the 8 rows a quarter-warp
// reads fall in 8 distinct bank groups), plus the 32 columns' coefficients
// (512 bytes, read by every thread at the same address: broadcasts). Thread t
// owns rows t + CT k of the unit and sums each over the unit's columns in
// registers, so no cross-thread reduction exists: a flush is 4 atomics per row.
// Rows and columns past the matrix arrive as TMA zero fill and the coefficient
// table is zero-padded, so the last unit needs no special case. Units are
// dealt as in the few-rows kernel (row block major, an equal share per CTA).
namespace rlct {
constexpr int BOX_C = 32;
constexpr int BOX_R = 256;
constexpr int CT = 512;  // consumer threads
constexpr int UROWS = 2 * BOX_R;
constexpr int RPT = UROWS / CT;
constexpr int NST = 3;
constexpr int X_BYTES = UROWS * BOX_C * 4;
constexpr int C_BYTES = BOX_C * 16;
constexpr int STAGE_BYTES = X_BYTES + 1024;  // coefficients after the boxes; keeps stages 1024-byte aligned
constexpr int OFF_BAR = NST * STAGE_BYTES;
constexpr int SMEM = OFF_BAR + 2 * NST * 8;
constexpr int THREADS = CT + 32;
static_assert(C_BYTES <= 1024, "coefficients fit the stage's tail");
static_assert(SMEM <= 227 * 1024, "shared memory per CTA");
static_assert(UROWS % CT == 0 && BOX_C % 8 == 0, "geometry");
}  // namespace rlct

__global__ void __launch_bounds__(rlct::THREADS, 1) k_rlc_rows_t(const __grid_constant__ CUtensorMap tm_x,
                                                                 uint32_t rows, uint64_t cols,
                                                                 const int4* __restrict__ cw,
                                                                 unsigned long long* __restrict__ acc,
                                                                 int* __restrict__ err) {
    using namespace rlct;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + OFF_BAR);
    uint64_t* empty = full + NST;
    const int tid = threadIdx.x;
    const uint64_t nch = (cols + BOX_C - 1) / BOX_C;
    const uint64_t U = nch * ((rows + UROWS - 1) / UROWS);
    const uint64_t u0 = U * blockIdx.x / gridDim.x, u1 = U * (blockIdx.x + 1) / gridDim.x;
    if (tid == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CT / 32);
        }
        fence_mbar_init();
    }
    __syncthreads();
    const uint32_t rb0 = (uint32_t)(u0 / nch);
    const uint64_t ch0 = u0 % nch;
    if (tid >= CT) {  // producer warp, lane 0
        if (tid != CT) return;
        uint32_t rb = rb0, ph = 0;
        uint64_t ch = ch0;
        int s = 0;
        bool reuse = false;
        for (uint64_t u = u0; u < u1; u++) {
            if (reuse) {
                if (!mbar_wait_bounded(&empty[s], ph ^ 1)) {
                    atomicOr(err, 4);
                    return;
                }
                fence_proxy_async();
            }
            unsigned char* st = smem + s * STAGE_BYTES;
            mbar_expect_tx(&full[s], X_BYTES + C_BYTES);
            for (int b = 0; b < UROWS / BOX_R; b++)
                tma_load_2d(st + b * BOX_R * BOX_C * 4, &tm_x, (int)(ch * BOX_C), (int)(rb * UROWS + b * BOX_R),
                            &full[s]);
            bulk_load_1d(st + X_BYTES, cw + ch * BOX_C, C_BYTES, &full[s]);
            if (++s == NST) {
                s = 0;
                ph ^= 1;
                reuse = true;
            }
            if (++ch == nch) {
                ch = 0;
                rb++;
            }
        }
        return;
    }
    const int lane = tid & 31;
    int64_t sum[RPT][4];
#pragma unroll
    for (int k = 0; k < RPT; k++)
#pragma unroll
        for (int l = 0; l < 4; l++) sum[k][l] = 0;
    // this thread's rows in a unit: t + CT k, each in box (t + CT k) / BOX_R at line (t + CT k) % BOX_R
    uint32_t line_off[RPT];
#pragma unroll
    for (int k = 0; k < RPT; k++) {
        const int r = tid + CT * k;
        line_off[k] = (uint32_t)((r / BOX_R) * BOX_R * BOX_C * 4 + (r % BOX_R) * BOX_C * 4);
    }
    const int swz = tid & 7;  // (row & 7) is the same for all of this thread's rows: CT and BOX_R are multiples of 8
    uint32_t rb = rb0, ph = 0;
    uint64_t ch = ch0;
    int s = 0;
    bool dead = false;  // as in the few-rows kernel: a warp that gave up a wait only keeps step
    for (uint64_t u = u0; u < u1; u++) {
        if (!dead && !__all_sync(0xFFFFFFFFu, mbar_wait_bounded(&full[s], ph))) {
            dead = true;
            if (lane == 0) atomicOr(err, 1);
        }
        if (!dead) {
            const unsigned char* st = smem + s * STAGE_BYTES;
            const int4* sc = reinterpret_cast<const int4*>(st + X_BYTES);
#pragma unroll
            for (int q = 0; q < BOX_C / 4; q++) {
                int4 w[4];
#pragma unroll
                for (int j = 0; j < 4; j++) w[j] = sc[4 * q + j];
#pragma unroll
                for (int k = 0; k < RPT; k++) {
                    const uint4 v = *reinterpret_cast<const uint4*>(st + line_off[k] + ((q ^ swz) << 4));
                    const int32_t xv[4] = {centered_any(v.x), centered_any(v.y), centered_any(v.z),
                                           centered_any(v.w)};
#pragma unroll
                    for (int l = 0; l < 4; l++)
#pragma unroll
                        for (int j = 0; j < 4; j++) sum[k][l] += (int64_t)xv[j] * limb(w[j], l);
                }
                if (q & 1) {  // eight products per sum since the last fold
#pragma unroll
                    for (int k = 0; k < RPT; k++)
#pragma unroll
                        for (int l = 0; l < 4; l++) sum[k][l] = sfold(sum[k][l]);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (u + 1 == u1 || ch + 1 == nch) {
#pragma unroll
            for (int k = 0; k < RPT; k++) {
                const uint32_t row = rb * UROWS + tid + CT * k;
                if (row < rows) {
#pragma unroll
                    for (int l = 0; l < 4; l++)
                        atomicAdd(acc + (uint64_t)row * 4 + l,
                                  (unsigned long long)((uint64_t)(sum[k][l] + (int64_t)P_SHIFT29) % P));
                }
#pragma unroll
                for (int l = 0; l < 4; l++) sum[k][l] = 0;
            }
        }
        if (++s == NST) {
            s = 0;
            ph ^= 1;
        }
        if (++ch == nch) {
            ch = 0;
            rb++;
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

// From this many rows on, the row kernel (a thread per row) runs; below, the
// few-rows kernel (a thread per column quad).
constexpr uint32_t RLC_ROW_KERNEL_MIN_ROWS = 256;

// Byte offset of the row-wise table in ctx->rlc_w, after the planar one.
inline uint64_t rowwise_offset(uint64_t cols) { return (cols * 16 + 255) / 256 * 256; }
inline uint64_t rowwise_cols(uint64_t cols) { return (cols + rlct::BOX_C - 1) / rlct::BOX_C * rlct::BOX_C; }

// rlc of rows [rows][cols] (pitch cols) into out [rows][4]; tables prepared.
zoda_status rlc_rows(const zoda_ctx* ctx, const uint32_t* x, uint32_t rows, uint64_t cols, unsigned long long* acc,
                     uint32_t* out, cudaStream_t st) {
    ZB_CUDA(cudaMemsetAsync(acc, 0, (size_t)rows * 4 * sizeof(unsigned long long), st));
    const uint64_t quads = cols / 4;
    if (rows > 262140) {
        set_last_error_text("rlc: more than 262140 rows");
        return ZODA_ERR_UNSUPPORTED;
    }
    const unsigned char* tabs = (const unsigned char*)ctx->rlc_w.p;
    if (quads && rows >= RLC_ROW_KERNEL_MIN_ROWS) {
        CUtensorMap tm;
        zoda_status s = make_map(&tm, x, cols, rows, cols * 4, rlct::BOX_C, rlct::BOX_R, CU_TENSOR_MAP_SWIZZLE_128B);
        if (s != ZODA_OK) return s;
        const uint64_t units = (cols + rlct::BOX_C - 1) / rlct::BOX_C * ((rows + rlct::UROWS - 1) / rlct::UROWS);
        const unsigned g = (unsigned)std::min<uint64_t>(units, (uint64_t)ctx->sm_count);
        k_rlc_rows_t<<<g, rlct::THREADS, rlct::SMEM, st>>>(
            tm, rows, cols, (const int4*)(tabs + rowwise_offset(cols)), acc, ctx->d_err);
        ZB_CUDA(cudaGetLastError());
    } else if (quads) {
        const uint64_t units = (quads + rlcb::CHQ - 1) / rlcb::CHQ * ((rows + rlcb::UROWS - 1) / rlcb::UROWS);
        const unsigned g = (unsigned)std::min<uint64_t>(units, (uint64_t)ctx->sm_count);
        k_rlc_rows<<<g, rlcb::THREADS, rlcb::SMEM, st>>>(x, cols, rows, quads, (const int4*)tabs, acc, ctx->d_err);
        ZB_CUDA(cudaGetLastError());
    }
    k_rlc_final<<<grid1(ctx, (uint64_t)rows * 4), 256, 0, st>>>(acc, (uint64_t)rows * 4, out);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

// Coefficient tables for RLCs of `rows_a` and `rows_b` rows (0: none): only the
// layouts the kernels for those row counts read.
zoda_status prep_tables(zoda_ctx* ctx, const uint32_t* d_coeff, uint64_t cols, uint32_t rows_a, uint32_t rows_b,
                        cudaStream_t st) {
    zoda_status s;
    const uint64_t npad = rowwise_cols(cols);
    if ((s = ctx->rlc_w.ensure(rowwise_offset(cols) + npad * 16)) != ZODA_OK) return s;
    unsigned char* tabs = (unsigned char*)ctx->rlc_w.p;
    auto row_kernel = [](uint32_t r) { return r >= RLC_ROW_KERNEL_MIN_ROWS; };
    const bool planar = (rows_a && !row_kernel(rows_a)) || (rows_b && !row_kernel(rows_b));
    const bool rowwise = row_kernel(rows_a) || row_kernel(rows_b);
    k_rlc_prep<<<grid1(ctx, npad), 256, 0, st>>>((const uint4*)d_coeff, cols / 4, rowwise ? npad : cols,
                                                 planar ? (int4*)tabs : nullptr,
                                                 rowwise ? (int4*)(tabs + rowwise_offset(cols)) : nullptr);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

}  // namespace

zoda_status rlc_init_attributes() {
    ZB_CUDA(cudaFuncSetAttribute(k_rlc_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, rlcb::SMEM));
    ZB_CUDA(cudaFuncSetAttribute(k_rlc_rows_t, cudaFuncAttributeMaxDynamicSharedMemorySize, rlct::SMEM));
    return ZODA_OK;
}

void rlc_release(zoda_ctx* ctx) {
    for (DevBuf* b : {&ctx->rlc_w, &ctx->rlc_acc, &ctx->rlc_d, &ctx->rlc_e, &ctx->rlc_f, &ctx->rlc_cnt})
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
    zoda_status s = prep_tables(ctx, d_coeff, cols, rows, 0, st);
    if (s != ZODA_OK) return s;
    if ((s = ctx->rlc_acc.ensure((size_t)rows * 4 * 8)) != ZODA_OK) return s;
    return rlc_rows(ctx, d_rows, rows, cols, (unsigned long long*)ctx->rlc_acc.p, d_out, st);
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
    zoda_status s = prep_tables(ctx, d_coeff, cols, k, rows, st);
    if (s != ZODA_OK) return s;
    if ((s = ctx->rlc_acc.ensure((size_t)rows * 4 * 8)) != ZODA_OK) return s;
    if ((s = ctx->rlc_d.ensure((size_t)k * 16)) != ZODA_OK) return s;
    if ((s = ctx->rlc_e.ensure((size_t)rows * 16)) != ZODA_OK) return s;
    if ((s = ctx->rlc_f.ensure((size_t)rows * 16)) != ZODA_OK) return s;
    if ((s = ctx->rlc_cnt.ensure(8)) != ZODA_OK) return s;
    unsigned long long* acc = (unsigned long long*)ctx->rlc_acc.p;
    uint32_t *D = (uint32_t*)ctx->rlc_d.p, *E = (uint32_t*)ctx->rlc_e.p, *F = (uint32_t*)ctx->rlc_f.p;
    if ((s = rlc_rows(ctx, d_data, k, cols, acc, D, st)) != ZODA_OK) return s;
    // the RLC and the extension commute (both F_p-linear): extend the k x 4 RLC matrix
    if ((s = zoda_encode_device(ctx, D, F, k, n, 4, st)) != ZODA_OK) return s;
    if ((s = rlc_rows(ctx, d_code, rows, cols, acc, E, st)) != ZODA_OK) return s;
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
