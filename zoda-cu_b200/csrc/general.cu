// Encode of any shape (k data rows, n parity rows) and the k-of-2k erasure
// decoder, both built on the general column transform (coltx.cuh).
//
// Encode, as the reference defines it (src/benchmarks/utils.rs:42-48,100-146,
// src/zoda/babybear.rs:137-152): n_k = next_pow2(k), n_kn = next_pow2(k + n);
// the k rows are zero-padded to n_k, interpolated (INTT over n_k), zero-padded
// to n_kn coefficients and evaluated (NTT over n_kn); the encoding is output
// rows 0 .. k+n-1 in natural order. With R = n_kn / n_k, output row R*m + c is
//   c = 0:  the padded data row m (a copy),
//   c > 0:  NTT_{n_k}(omega_{n_kn}^(c*i) * coef_i)[m], one transform per coset.
// R = 2 (every square, and any n <= 2 n_k - k) runs on the fused extension
// kernels, which read zeros past row k and stop writing after row k+n. For
// R >= 4 with 128 <= n_k <= 4096 each coset c is one fused TMA-staged pass
// NTT(omega_{n_kn}^(c i) / n_k * INTT(data)) (enc_coset_pass); other n_k take
// one interpolation and a per-coset evaluation on the direct-load shape.
//
// Decoder: f of degree < k is known at a set K of the 2k points omega_2k^j.
// With Z(x) = prod over the erased points of (x - omega^e), g = f * Z has
// degree < 2k and is known everywhere (zero at the erased points), so
//   G   = INTT_2k(y_j * Z(omega^j))                    coefficients of g
//   g~  = NTT_2k(G_i * h^i)                            g on the coset h*omega^j
//   F~  = INTT_2k(g~_j / Z(h * omega^j))               coefficients of f(h x)
//   row = NTT_k(F~_i * h^-i), i < k                     f at omega_k^m = data row m
// with h = 31 (a generator of F_p^*, never a 2k-th root of unity, so Z(h w) != 0).
// F~_i must vanish for i >= k when the known rows are one codeword; the
// optional check counts the entries that do not. The four transforms run as two
// fused passes, each an INTT and an NTT with the pointwise factor between them
// applied in registers: pass A gives g~, pass B gives the data rows as the even
// outputs of NTT_2k(F~_i * h^-i, zero for i >= k), which is NTT_k of the first
// k coefficients at omega_2k^(2m) = omega_k^m. From 128 to 4096 points the
// passes run on the TMA-staged pipeline (k_dec_tma, extend_tma.cuh), elsewhere
// on the direct-load shape (k_coltx2, coltx.cuh).
#include <algorithm>
#include <vector>

#include "coltx.cuh"
#include "internal.hpp"
#include "tma_host.hpp"

namespace zb {
namespace {

constexpr uint64_t SCRATCH_ELEMS = 64ull << 20;  // u32 per scratch matrix (256 MiB)

int log2_exact64(uint64_t x) {
    if (x == 0 || (x & (x - 1))) return -1;
    int l = 0;
    while ((1ull << l) < x) l++;
    return l;
}
uint64_t next_pow2_64(uint64_t x) {
    uint64_t r = 1;
    while (r < x) r <<= 1;
    return r;
}
inline uint2 shoup_pair(uint32_t w) { return make_uint2(w, shoup(w)); }

// From 512 points the radix-8, 1024-thread shape (twice the warps) runs the
// decoder's and the coset path's transforms 14-21% faster than radix 16.
template <int LOG_N, bool INV>
zoda_status coltx_t(const zoda_ctx* ctx, const ColTx& a, cudaStream_t st) {
    constexpr int LEPT = LOG_N >= 9 ? 3 : 4;
    using PL = ExtPlan<LOG_N, 0, LEPT, LEPT == 3 ? 1024 : 512>;
    const uint64_t ntiles = (a.cols + PL::C - 1) / PL::C;
    if (ntiles == 0 || a.out_rows == 0) return ZODA_OK;
    if (PL::SMEM > 0)
        ZB_CUDA(cudaFuncSetAttribute(k_coltx<LOG_N, INV, LEPT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)PL::SMEM));
    const uint64_t grid = ntiles < (uint64_t)ctx->sm_count ? ntiles : (uint64_t)ctx->sm_count;
    k_coltx<LOG_N, INV, LEPT><<<(unsigned)grid, PL::THREADS, PL::SMEM, st>>>(a, ntiles, ctx->tables.tw);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

// Column transform of size 2^log_n (1 <= log_n <= 13).
zoda_status coltx(const zoda_ctx* ctx, int log_n, bool inv, const ColTx& a, cudaStream_t st) {
    switch (log_n) {
#define ZB_CASE(L) \
    case L: return inv ? coltx_t<L, true>(ctx, a, st) : coltx_t<L, false>(ctx, a, st);
        ZB_CASE(1) ZB_CASE(2) ZB_CASE(3) ZB_CASE(4) ZB_CASE(5) ZB_CASE(6)
        ZB_CASE(7) ZB_CASE(8) ZB_CASE(9) ZB_CASE(10) ZB_CASE(11) ZB_CASE(12) ZB_CASE(13)
#undef ZB_CASE
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

template <int LOG_N, int OSH, bool COUNT>
zoda_status coltx2_t(const zoda_ctx* ctx, const ColTx2& a, cudaStream_t st) {
    constexpr int LEPT = LOG_N >= 9 ? 3 : 4;
    using PL = ExtPlan<LOG_N, 0, LEPT, LEPT == 3 ? 1024 : 512>;
    const uint64_t ntiles = (a.cols + PL::C - 1) / PL::C;
    if (ntiles == 0 || a.out_rows == 0) return ZODA_OK;
    if (PL::SMEM > 0)
        ZB_CUDA(cudaFuncSetAttribute(k_coltx2<LOG_N, LEPT, OSH, COUNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)PL::SMEM));
    const uint64_t grid = ntiles < (uint64_t)ctx->sm_count ? ntiles : (uint64_t)ctx->sm_count;
    k_coltx2<LOG_N, LEPT, OSH, COUNT><<<(unsigned)grid, PL::THREADS, PL::SMEM, st>>>(a, ntiles, ctx->tables.tw);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

// INTT -> mid -> NTT of size 2^log_n (1 <= log_n <= 13) in one pass; even_out
// stores only the even outputs (row r / 2); a.counter selects the counting form.
zoda_status coltx2(const zoda_ctx* ctx, int log_n, bool even_out, const ColTx2& a, cudaStream_t st) {
    switch (log_n) {
#define ZB_CASE(L)                                                                       \
    case L:                                                                              \
        if (!even_out) return coltx2_t<L, 0, false>(ctx, a, st);                         \
        return a.counter ? coltx2_t<L, 1, true>(ctx, a, st) : coltx2_t<L, 1, false>(ctx, a, st);
        ZB_CASE(1) ZB_CASE(2) ZB_CASE(3) ZB_CASE(4) ZB_CASE(5) ZB_CASE(6)
        ZB_CASE(7) ZB_CASE(8) ZB_CASE(9) ZB_CASE(10) ZB_CASE(11) ZB_CASE(12) ZB_CASE(13)
#undef ZB_CASE
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

// ---- the decoder's passes on the TMA-staged shape (k_dec_tma) ------------------
// Sides 2^7 .. 2^12 (the TMA-staged range, a whole tile per CTA). Level radix
// 8 at 512 and 2048 points, 16 at the others: the faster shape of each for the
// decoder on B200 (interleaved runs on one box: 3-4% apart at 512 and 4096
// points, equal at 1024 and 2048).
constexpr int DEC_TMA_MIN_LOG = 7, DEC_TMA_MAX_LOG = 12;
constexpr int dec_lept(int ls) { return ls == 9 || ls == 11 ? 3 : 4; }

// Pattern-independent tables of the two passes for side S = 2^ls, built once:
//   ntt0_a, ntt0_b  NTT level 0 as in SideTables, with the block factor
//                   h^(+c0)/S resp. h^(-c0)/S in place of g^c0/S (S entries each)
//   ktw_a[k2]  = h^((S/R) k2)
//   ktw_b[k2]  = h^(-(S/R) k2) for k2 < R/2, else 0 (drops coefficients >= S/2)
//   ktw_bc[k2] = h^(-(S/R) k2) (the checking form zeroes them after counting)
// so that mid(c0 + (S/R) k2) = block(c0) * ktw[k2] is h^(+-i)/S, resp. that
// times [i < S/2]. R = 2^lr(last INTT level).
struct DecTables {
    const uint2 *ntt0_a, *ntt0_b, *ktw_a, *ktw_b, *ktw_bc;
};
zoda_status dec_tables(zoda_ctx* ctx, int ls, DecTables* out) {
    const SideLevels sl(ls, dec_lept(ls));
    DevBuf& b = ctx->coset_tabs[-1 - ls];  // coset keys are >= 0
    const uint32_t S = 1u << ls;
    const int LR = sl.last_lr();
    const uint32_t R = 1u << LR, NB = S >> LR, step = S / R;
    if (!b.p) {
        std::vector<uint2> h;
        const uint32_t hinv = powmod_c(GENERATOR, P - 2), sinv = powmod_c(S, P - 2);
        const std::vector<uint32_t> c0s = sl.last_c0();
        for (int dir = 0; dir < 2; dir++) {
            const uint32_t base = dir == 0 ? GENERATOR : hinv;
            for (uint32_t k2 = 0; k2 < R; k2++)
                for (uint32_t bb = 0; bb < NB; bb++) {
                    const uint32_t c0 = c0s[bb];
                    const uint32_t v = mulmod_c(mulmod_c(powmod_c(base, c0), sinv),
                                                powmod_c(root_of_unity(ls), (uint64_t)c0 * k2 % S));
                    h.push_back(shoup_pair(v));
                }
        }
        for (uint32_t k2 = 0; k2 < R; k2++) h.push_back(shoup_pair(powmod_c(GENERATOR, (uint64_t)step * k2)));
        for (uint32_t k2 = 0; k2 < R; k2++)
            h.push_back(k2 < R / 2 ? shoup_pair(powmod_c(hinv, (uint64_t)step * k2)) : make_uint2(0u, 0u));
        for (uint32_t k2 = 0; k2 < R; k2++) h.push_back(shoup_pair(powmod_c(hinv, (uint64_t)step * k2)));
        zoda_status s = b.ensure(h.size() * sizeof(uint2));
        if (s != ZODA_OK) return s;
        ZB_CUDA(cudaMemcpy(b.p, h.data(), h.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    }
    const uint2* t = (const uint2*)b.p;
    *out = DecTables{t, t + S, t + 2 * S, t + 2 * S + R, t + 2 * S + 2 * R};
    return ZODA_OK;
}

// One k_dec_tma launch over w columns; input rows >= in_rows (0: S) read as zeros.
template <int LS, int OSH, int TWM, bool PRE = true>
zoda_status dec_pass_t(const zoda_ctx* ctx, const uint32_t* in, uint64_t in_pitch, const uint2* pre,
                       const uint2* ntt0, const uint2* ktw, uint32_t* out, uint64_t out_pitch, uint32_t out_rows,
                       uint64_t w, unsigned long long* counter, cudaStream_t st, uint32_t in_rows = 0) {
    constexpr int LEPT = dec_lept(LS);
    using TP = TPlan<LS, LEPT>;
    const uint64_t ntiles = (w + TP::C - 1) / TP::C;
    if (ntiles == 0) return ZODA_OK;
    // L2 promotion, tile order and stagger of the side's plan (tuned or default)
    const zoda_plan p = ctx->planned[LS] ? ctx->plan[LS] : default_plan(LS);
    const uint32_t at_code = p.stagger == 2 ? 2u : p.stagger == 3 ? 1u : 0u;
    const uint32_t flags = (p.blocked ? 1u : 0u) | (p.stagger ? 0u : 2u) | (at_code << 2);
    CUtensorMap m;
    zoda_status s = make_map(&m, in, w, in_rows ? in_rows : TP::S, in_pitch * 4, TP::BOX_C, TP::BOX_R,
                             tile_swizzle<TP>(), p.impl == ZODA_IMPL_TMA ? p.l2_promo : 3);
    if (s != ZODA_OK) return s;
    SideTables tb = side_tables(ctx, LS, LEPT);
    tb.ntt0 = ntt0;
    ZB_CUDA(cudaFuncSetAttribute(k_dec_tma<LS, LEPT, OSH, TWM, PRE>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TP::SMEM));
    const uint64_t grid = ntiles < (uint64_t)ctx->sm_count ? ntiles : (uint64_t)ctx->sm_count;
    k_dec_tma<LS, LEPT, OSH, TWM, PRE><<<(unsigned)grid, TP::THREADS, TP::SMEM, st>>>(
        m, out, out_pitch, out_rows, w, ntiles, tb, pre, ktw, counter, ctx->d_err, flags);
    ZB_CUDA(cudaGetLastError());
    return ZODA_OK;
}

// Pass A (second = false) or B of the decoder on side 2^ls, DEC_TMA_MIN_LOG <= ls <= DEC_TMA_MAX_LOG.
zoda_status dec_pass(const zoda_ctx* ctx, int ls, bool second, const DecTables& t, const uint32_t* in,
                     uint64_t in_pitch, const uint2* pre, uint32_t* out, uint64_t out_pitch, uint64_t w,
                     unsigned long long* counter, cudaStream_t st) {
    const uint32_t S = 1u << ls;
    switch (ls) {
#define ZB_CASE(L)                                                                                             \
    case L:                                                                                                    \
        if (!second) return dec_pass_t<L, 0, 1>(ctx, in, in_pitch, pre, t.ntt0_a, t.ktw_a, out, out_pitch, S, w, \
                                                nullptr, st);                                                  \
        if (counter) return dec_pass_t<L, 1, 2>(ctx, in, in_pitch, pre, t.ntt0_b, t.ktw_bc, out, out_pitch, S, w, \
                                                counter, st);                                                  \
        return dec_pass_t<L, 1, 1>(ctx, in, in_pitch, pre, t.ntt0_b, t.ktw_b, out, out_pitch, S, w, nullptr, st);
        ZB_CASE(7) ZB_CASE(8) ZB_CASE(9) ZB_CASE(10) ZB_CASE(11) ZB_CASE(12)
#undef ZB_CASE
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

// Coset passes of the any-shape encode on the TMA-staged shape, for n_k = 2^lp
// in the decoder's TMA range: coset c of n_kn = 2^ln is
//   NTT_{n_k}(omega_{n_kn}^(c i) / n_k * INTT_{n_k}(data))
// in one pass (k_dec_tma without pre-factors; rows >= k arrive as zeros). The
// twist splits as the extension's does: block factor omega_{n_kn}^(c c0) / n_k
// in NTT level 0's table, digit factor omega_{n_kn}^(c (S/R) k2) in the INTT's
// last stage. Tables for every coset c in [1, R), built once per shape:
// coset c's [ntt0 (S entries) | ktw (R entries)] at (c - 1) * (S + R).
zoda_status enc_tables(zoda_ctx* ctx, int lp, int ln, const uint2** out, uint32_t* stride) {
    const SideLevels sl(lp, dec_lept(lp));
    DevBuf& b = ctx->coset_tabs[-(100000 + lp * 64 + ln)];  // disjoint from the other keys
    const uint32_t S = 1u << lp;
    const int LR = sl.last_lr();
    const uint32_t R = 1u << LR, NB = S >> LR, step = S / R;
    const uint64_t cosets = (1ull << (ln - lp)) - 1;
    if (!b.p) {
        // c0 of every INTT last-level block, and omega_S^e: each entry is then two products
        const std::vector<uint32_t> c0s = sl.last_c0();
        std::vector<uint32_t> ws(S);
        const uint32_t wS = root_of_unity(lp);
        for (uint32_t e = 0, x = 1; e < S; e++, x = mulmod_c(x, wS)) ws[e] = x;
        std::vector<uint2> h;
        h.reserve(cosets * (S + R));
        std::vector<uint32_t> pw(NB);  // base^i / S for i < NB (every c0 is below S / R = NB)
        const uint32_t sinv = powmod_c(S, P - 2), wn = root_of_unity(ln);
        for (uint64_t c = 1, base = wn; c <= cosets; c++, base = mulmod_c((uint32_t)base, wn)) {
            for (uint32_t i = 0, x = sinv; i < NB; i++, x = mulmod_c(x, (uint32_t)base)) pw[i] = x;
            for (uint32_t k2 = 0; k2 < R; k2++)
                for (uint32_t bb = 0; bb < NB; bb++)
                    h.push_back(shoup_pair(mulmod_c(pw[c0s[bb]], ws[(uint64_t)c0s[bb] * k2 % S])));
            const uint32_t g = powmod_c((uint32_t)base, step);
            for (uint32_t k2 = 0, x = 1; k2 < R; k2++, x = mulmod_c(x, g)) h.push_back(shoup_pair(x));
        }
        zoda_status s = b.ensure(h.size() * sizeof(uint2));
        if (s != ZODA_OK) return s;
        ZB_CUDA(cudaMemcpy(b.p, h.data(), h.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    }
    *out = (const uint2*)b.p;
    *stride = S + R;
    return ZODA_OK;
}

// Coset c's pass: output rows R*m + c (m < mc) of out, pitch out_pitch.
zoda_status enc_coset_pass(const zoda_ctx* ctx, int lp, const uint2* tab, const uint32_t* in, uint32_t k,
                           uint64_t cols, uint32_t* out, uint64_t out_pitch, uint32_t mc, cudaStream_t st) {
    const uint2* ntt0 = tab;
    const uint2* ktw = tab + (1u << lp);
    switch (lp) {
#define ZB_CASE(L) \
    case L: return dec_pass_t<L, 0, 1, false>(ctx, in, cols, nullptr, ntt0, ktw, out, out_pitch, mc, cols, nullptr, st, k);
        ZB_CASE(7) ZB_CASE(8) ZB_CASE(9) ZB_CASE(10) ZB_CASE(11) ZB_CASE(12)
#undef ZB_CASE
        default: return ZODA_ERR_UNSUPPORTED;
    }
}

// out[r * pitch + c] = in[c] for r in [0, rows), c in [0, cols).
__global__ void k_bcast_rows(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint64_t pitch,
                             uint32_t rows, uint64_t cols) {
    const uint64_t n = (uint64_t)rows * cols;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = i / cols, c = i - r * cols;
        out[r * pitch + c] = in[c];
    }
}

__device__ __forceinline__ uint32_t pow_slow(uint32_t b, uint32_t e) {
    uint32_t r = 1;
    while (e) {
        if (e & 1) r = mul_slow(r, b);
        b = mul_slow(b, b);
        e >>= 1;
    }
    return r;
}
__device__ __forceinline__ uint2 shoup_pair_dev(uint32_t w) {
    return make_uint2(w, (uint32_t)(((uint64_t)w << 32) / P));
}

// Decoder tables for one erasure pattern over N = 2^log_n points (see the top
// of this file); roots[e] = omega_N^e for the erased e:
//   zk[j]    = Z(omega^j)          (0 at erased j)
//   izh[j]   = 1 / Z(h * omega^j)
//   mid_a[i] = h^i / N
//   mid_b[i] = h^-i / N for i < k, else 0
__global__ void k_erasure_tables(const uint32_t* __restrict__ erased_roots, uint32_t ne, int log_n,
                                 const Tw* __restrict__ tw, uint32_t k, uint32_t ninv, uint2* __restrict__ zk,
                                 uint2* __restrict__ izh, uint2* __restrict__ mid_a, uint2* __restrict__ mid_b) {
    const uint32_t N = 1u << log_n;
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= N) return;
    const uint32_t x = tw[(size_t)j << (LOG_TW - log_n)].w;  // omega_N^j
    const uint32_t y = mul_slow(GENERATOR, x);
    uint32_t zx = 1, zy = 1;
    for (uint32_t i = 0; i < ne; i++) {
        const uint32_t r = erased_roots[i];
        zx = mul_slow(zx, x >= r ? x - r : x + P - r);
        zy = mul_slow(zy, y >= r ? y - r : y + P - r);
    }
    zk[j] = shoup_pair_dev(zx);
    izh[j] = shoup_pair_dev(pow_slow(zy, P - 2));
    // the coset shift g^j and its inverse, with the INTTs' 1/N; coefficients
    // j >= k of the quotient are dropped (zero) before the last NTT
    const uint32_t hj = pow_slow(GENERATOR, j);
    mid_a[j] = shoup_pair_dev(mul_slow(hj, ninv));
    mid_b[j] = j < k ? shoup_pair_dev(mul_slow(pow_slow(hj, P - 2), ninv)) : make_uint2(0u, 0u);
}

unsigned grid_for(const zoda_ctx* ctx, uint64_t n) {
    const uint64_t g = (n + 255) / 256;
    const uint64_t cap = (uint64_t)ctx->sm_count * 8;
    return (unsigned)(g < 1 ? 1 : g > cap ? cap : g);
}

// Scratch of one chunk: w columns of `rows` rows per matrix.
uint64_t chunk_cols(uint64_t cols, uint64_t rows) {
    uint64_t w = SCRATCH_ELEMS / rows;
    w &= ~3ull;
    if (w < 4) w = 4;
    return w < cols ? w : cols;
}

// Orders this call's use of the context scratch after the previous call's,
// whichever streams the two calls used.
zoda_status gen_begin(zoda_ctx* ctx, cudaStream_t st) {
    if (!ctx->gen_done) {
        ZB_CUDA(cudaEventCreateWithFlags(&ctx->gen_done, cudaEventDisableTiming));
        return ZODA_OK;
    }
    ZB_CUDA(cudaStreamWaitEvent(st, ctx->gen_done, 0));
    return ZODA_OK;
}
zoda_status gen_end(zoda_ctx* ctx, cudaStream_t st) {
    ZB_CUDA(cudaEventRecord(ctx->gen_done, st));
    return ZODA_OK;
}

// omega_{n_kn}^(c*i) for c in [0, R), i in [0, n_k), row c at c * n_k; built once per shape.
zoda_status coset_table(zoda_ctx* ctx, int lp, int ln, const uint2** out) {
    const int key = lp * 64 + ln;
    DevBuf& b = ctx->coset_tabs[key];
    const uint64_t P_ = 1ull << lp, R = 1ull << (ln - lp);
    if (!b.p) {
        std::vector<uint2> h(R * P_);
        const uint32_t wn = root_of_unity(ln);
        for (uint64_t c = 0; c < R; c++) {
            const uint32_t step = powmod_c(wn, c);
            uint32_t x = 1;
            for (uint64_t i = 0; i < P_; i++) {
                h[c * P_ + i] = shoup_pair(x);
                x = mulmod_c(x, step);
            }
        }
        zoda_status s = b.ensure(h.size() * sizeof(uint2));
        if (s != ZODA_OK) return s;
        ZB_CUDA(cudaMemcpy(b.p, h.data(), h.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    }
    *out = (const uint2*)b.p;
    return ZODA_OK;
}

zoda_status encode_general(zoda_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t k, uint32_t n, uint64_t cols,
                           cudaStream_t st) {
    const uint64_t P_ = next_pow2_64(k), N = next_pow2_64((uint64_t)k + n), rows_out = (uint64_t)k + n;
    const int lp = log2_exact64(P_), ln = log2_exact64(N);
    const uint64_t R = N / P_;
    const uint64_t rb = cols * 4;  // row bytes
    // c = 0 rows: R*m for m < ceil(rows_out / R); data rows first, then zero rows
    const uint64_t m0 = (rows_out + R - 1) / R;
    const uint64_t mdata = std::min<uint64_t>(k, m0);
    ZB_CUDA(cudaMemcpy2DAsync(out, R * rb, in, rb, rb, mdata, cudaMemcpyDeviceToDevice, st));
    if (m0 > mdata) ZB_CUDA(cudaMemset2DAsync(out + R * mdata * cols, R * rb, 0, rb, m0 - mdata, st));
    if (R == 1) return ZODA_OK;
    if (lp > 12) return long_encode(ctx, in, out, k, n, cols, st);  // no column fits one pass
    if (P_ == 1) {  // every coset row is the single data row
        for (uint64_t c = 1; c < R && c < rows_out; c++) {
            const uint32_t mc = (uint32_t)((rows_out - c + R - 1) / R);
            k_bcast_rows<<<grid_for(ctx, (uint64_t)mc * cols), 256, 0, st>>>(in, out + c * cols, R * cols, mc, cols);
            ZB_CUDA(cudaGetLastError());
        }
        return ZODA_OK;
    }
    zoda_status s;
    if (lp >= DEC_TMA_MIN_LOG && lp <= DEC_TMA_MAX_LOG) {  // one fused TMA-staged pass per coset, no scratch
        const uint2* et = nullptr;
        uint32_t es = 0;
        if ((s = enc_tables(ctx, lp, ln, &et, &es)) != ZODA_OK) return s;
        for (uint64_t c = 1; c < R && c < rows_out; c++) {
            const uint32_t mc = (uint32_t)std::min<uint64_t>(P_, (rows_out - c + R - 1) / R);
            if ((s = enc_coset_pass(ctx, lp, et + (c - 1) * es, in, k, cols, out + c * cols, R * cols, mc, st)) !=
                ZODA_OK)
                return s;
        }
        return ZODA_OK;
    }
    const uint2* tabs = nullptr;
    if ((s = coset_table(ctx, lp, ln, &tabs)) != ZODA_OK) return s;
    const uint64_t w0 = chunk_cols(cols, P_);
    if ((s = ctx->gen_a.ensure(P_ * w0 * 4)) != ZODA_OK) return s;
    uint32_t* A = (uint32_t*)ctx->gen_a.p;
    const uint32_t pinv = powmod_c((uint32_t)P_, P - 2);
    for (uint64_t c0 = 0; c0 < cols; c0 += w0) {
        const uint64_t w = std::min(w0, cols - c0);
        // coefficients of the zero-padded data: INTT over n_k, scaled by n_k^-1
        ColTx a{in + c0, cols, k, nullptr, A, w, (uint32_t)P_, nullptr, Tw{pinv, shoup(pinv)}, w};
        if ((s = coltx(ctx, lp, true, a, st)) != ZODA_OK) return s;
        for (uint64_t c = 1; c < R && c < rows_out; c++) {
            const uint64_t mc = std::min<uint64_t>(P_, (rows_out - c + R - 1) / R);
            ColTx b{A, w, (uint32_t)P_, tabs + c * P_, out + c * cols + c0, R * cols, (uint32_t)mc, nullptr,
                    Tw{1u, shoup(1u)}, w};
            if ((s = coltx(ctx, lp, false, b, st)) != ZODA_OK) return s;
        }
    }
    return ZODA_OK;
}

}  // namespace

void general_release(zoda_ctx* ctx) {
    ctx->gen_a.release();
    ctx->gen_b.release();
    ctx->gen_tab.release();
    ctx->gen_small.release();
    for (auto& kv : ctx->coset_tabs) kv.second.release();
    ctx->coset_tabs.clear();
    if (ctx->gen_done) cudaEventDestroy(ctx->gen_done);
    ctx->gen_done = nullptr;
}

}  // namespace zb

using namespace zb;

extern "C" {

zoda_status zoda_encode_device(zoda_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t k, uint32_t n,
                               uint64_t cols, void* stream) {
    if (!ctx || !d_in || !d_out || k == 0 || cols % 4 != 0) return ZODA_ERR_ARG;
    if (((uintptr_t)d_in | (uintptr_t)d_out) & 15) return ZODA_ERR_ARG;
    const uint64_t rows_out = (uint64_t)k + n;
    const char* a = (const char*)d_in;
    const char* b = (const char*)d_out;
    if (cols && a < b + rows_out * cols * 4 && b < a + (uint64_t)k * cols * 4) return ZODA_ERR_ARG;  // overlap
    if (next_pow2_64(k) > zoda_max_side() || rows_out > (1ull << 27)) {
        set_last_error_text("encode supports next_pow2(k) <= 2^26 and k + n <= 2^27");
        return ZODA_ERR_UNSUPPORTED;
    }
    if (n == k && log2_exact64(k) >= 0) return zoda_extend_device(ctx, d_in, d_out, k, cols, stream);
    if (cols == 0) return ZODA_OK;
    const uint64_t P_ = next_pow2_64(k), N = next_pow2_64(rows_out);
    if (N == 2 * P_ && P_ >= 2 && P_ <= 4096) {
        // n_kn = 2 n_k: the fused kernels, reading zeros past row k and cutting
        // the output after row k+n
        ZB_CUDA(cudaSetDevice(ctx->device));
        return launch_extend(ctx, log2_exact64(P_), d_in, d_out, cols, (cudaStream_t)stream, ctx->impl, false, k,
                             (uint32_t)rows_out);
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    ZB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    zoda_status s = gen_begin(ctx, st);
    if (s != ZODA_OK) return s;
    s = encode_general(ctx, d_in, d_out, k, n, cols, st);
    zoda_status e = gen_end(ctx, st);
    return s != ZODA_OK ? s : e;
}

zoda_status zoda_recover_device(zoda_ctx* ctx, const uint32_t* d_code, const uint32_t* known_rows, uint32_t nknown,
                                uint32_t k, uint64_t cols, uint32_t* d_data, uint64_t* mismatch, void* stream) {
    if (!ctx || !d_code || !d_data || !known_rows || cols % 4 != 0) return ZODA_ERR_ARG;
    if (((uintptr_t)d_code | (uintptr_t)d_data) & 15) return ZODA_ERR_ARG;
    const int lk = log2_exact64(k);
    if (lk < 0) return ZODA_ERR_ARG;
    if (lk + 1 > LONG_RECOVER_MAX_LOG) {
        set_last_error_text("the decoder covers k <= 131072 (codewords of up to 2^18 rows)");
        return ZODA_ERR_UNSUPPORTED;
    }
    const uint32_t N = 2 * k;
    const int ln = lk + 1;
    std::vector<uint8_t> have(N, 0);
    for (uint32_t i = 0; i < nknown; i++) {
        if (known_rows[i] >= N) return ZODA_ERR_ARG;
        have[known_rows[i]] = 1;
    }
    uint32_t nk = 0;
    for (uint8_t h : have) nk += h;
    if (nk < k) {
        set_last_error_text("fewer than k distinct known rows");
        return ZODA_ERR_ARG;
    }
    const char* a = (const char*)d_code;
    const char* b = (const char*)d_data;
    if (cols && a < b + (uint64_t)k * cols * 4 && b < a + (uint64_t)N * cols * 4) return ZODA_ERR_ARG;  // overlap
    if (mismatch) *mismatch = 0;
    if (cols == 0) return ZODA_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    ZB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    zoda_status s = gen_begin(ctx, st);
    if (s != ZODA_OK) return s;
    auto finish = [&](zoda_status r) {
        zoda_status e = gen_end(ctx, st);
        return r != ZODA_OK ? r : e;
    };
    bool evens = true;
    for (uint32_t m = 0; m < k; m++) evens = evens && have[2 * m];
    const uint64_t rb = cols * 4;
    if (evens && !mismatch) {  // the data rows are all there
        ZB_CUDA(cudaMemcpy2DAsync(d_data, rb, d_code, 2 * rb, rb, k, cudaMemcpyDeviceToDevice, st));
        return finish(ZODA_OK);
    }
    // pattern tables: roots of the erased points, then zk | izh | mid_a | mid_b
    std::vector<uint32_t> er;
    const uint32_t wn = root_of_unity(ln);
    for (uint32_t j = 0, x = 1; j < N; j++, x = mulmod_c(x, wn))
        if (!have[j]) er.push_back(x);
    // gen_small: the erased roots, then the mismatch counter
    if ((s = ctx->gen_small.ensure(std::max<size_t>(1, er.size()) * 4 + 64)) != ZODA_OK) return finish(s);
    uint32_t* d_er = (uint32_t*)ctx->gen_small.p;
    unsigned long long* d_cnt = (unsigned long long*)((char*)ctx->gen_small.p + ((er.size() * 4 + 15) / 16) * 16);
    if (mismatch) ZB_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), st));
    if (ln > 13) {  // above 8192 points: the four transforms as five four-step passes (fourstep.cu)
        if ((s = long_recover(ctx, d_code, er, k, cols, d_data, mismatch ? d_cnt : nullptr, st)) != ZODA_OK)
            return finish(s);
        if (mismatch) {
            unsigned long long h = 0;
            ZB_CUDA(cudaMemcpyAsync(&h, d_cnt, sizeof h, cudaMemcpyDeviceToHost, st));
            ZB_CUDA(cudaStreamSynchronize(st));
            *mismatch = h;
        }
        return finish(ZODA_OK);
    }
    if ((s = ctx->gen_tab.ensure((size_t)4 * N * sizeof(uint2))) != ZODA_OK) return finish(s);
    uint2* T = (uint2*)ctx->gen_tab.p;
    uint2 *zk = T, *izh = T + N, *mid_a = T + 2 * N, *mid_b = T + 3 * N;
    if (!er.empty())
        ZB_CUDA(cudaMemcpyAsync(d_er, er.data(), er.size() * 4, cudaMemcpyHostToDevice, st));
    const uint32_t ninv = powmod_c(N, P - 2);
    k_erasure_tables<<<(N + 127) / 128, 128, 0, st>>>(d_er, (uint32_t)er.size(), ln, ctx->tables.tw, k, ninv, zk,
                                                      izh, mid_a, mid_b);
    ZB_CUDA(cudaGetLastError());
    const uint64_t w0 = chunk_cols(cols, N);
    if ((s = ctx->gen_a.ensure((uint64_t)N * w0 * 4)) != ZODA_OK) return finish(s);
    uint32_t* A = (uint32_t*)ctx->gen_a.p;
    const bool tma = ln >= DEC_TMA_MIN_LOG && ln <= DEC_TMA_MAX_LOG;
    DecTables dt{};
    if (tma && (s = dec_tables(ctx, ln, &dt)) != ZODA_OK) return finish(s);
    for (uint64_t c0 = 0; c0 < cols; c0 += w0) {
        const uint64_t w = std::min(w0, cols - c0);
        unsigned long long* cnt = mismatch ? d_cnt : nullptr;
        if (tma) {  // the same two passes on the TMA-staged shape
            if ((s = dec_pass(ctx, ln, false, dt, d_code + c0, cols, zk, A, w, w, nullptr, st)) != ZODA_OK)
                return finish(s);
            if ((s = dec_pass(ctx, ln, true, dt, A, w, izh, d_data + c0, cols, w, cnt, st)) != ZODA_OK)
                return finish(s);
            continue;
        }
        // pass A: g~ = NTT(h^i / N * INTT(y * Z)) into the scratch
        const ColTx2 pa{d_code + c0, cols, N, zk, (const Tw*)mid_a, A, w, N, w, 0, nullptr};
        // pass B: data row m = even output 2m of NTT(h^-i / N [i < k] * INTT(g~ / Z(h w)))
        const ColTx2 pb{A, w, N, izh, (const Tw*)mid_b, d_data + c0, cols, N, w, k, cnt};
        if ((s = coltx2(ctx, ln, false, pa, st)) != ZODA_OK) return finish(s);
        if ((s = coltx2(ctx, ln, true, pb, st)) != ZODA_OK) return finish(s);
    }
    if (mismatch) {
        unsigned long long h = 0;
        ZB_CUDA(cudaMemcpyAsync(&h, d_cnt, sizeof h, cudaMemcpyDeviceToHost, st));
        ZB_CUDA(cudaStreamSynchronize(st));
        *mismatch = h;
    }
    return finish(ZODA_OK);
}

}  // extern "C"
