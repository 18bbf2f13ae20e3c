// General column transform on row-major matrices, the building block of the
// encode for any (k, n) and of the erasure decoder.
//
// For every column c in [0, cols) and output row r < out_rows:
//   out[r * out_pitch + c] = post(r) * sum_{i < N} pre(i) * in[i * in_pitch + c] * omega_N^(+-i*r)
// with N = 2^LOG_N, in[i] = 0 for i >= in_rows (those rows are never read),
// pre(i) = 1 when no pre table is given, post(r) = post[r] when a post table is
// given and `scale` otherwise; rows whose pre-factor is 0 are not read. Tables
// hold (w, floor(w * 2^32 / p)) pairs, the Shoup form every product here uses.
//
// Same register-resident DIF levels as the extension kernels (extend.cuh): the
// thread's quad of 4 adjacent columns, radix-16 levels exchanged through shared
// memory, natural-order output by digit reversal. Row pre-factors are applied
// as the rows are loaded, so a pointwise scaling never costs its own HBM pass.
#pragma once
#include "extend.cuh"

namespace zb {

struct ColTx {
    const uint32_t* in;
    uint64_t in_pitch;  // u32 elements between input rows
    uint32_t in_rows;   // rows >= in_rows are zero
    const uint2* pre;   // per input row, or nullptr
    uint32_t* out;
    uint64_t out_pitch;  // u32 elements between output rows
    uint32_t out_rows;   // output rows >= out_rows are not written
    const uint2* post;   // per output row, or nullptr (then `scale`)
    Tw scale;
    uint64_t cols;  // multiple of 4
};

// LEPT 4: radix-16 levels, 512 threads; 3: radix-8 levels, 1024 threads.
template <int LOG_N, bool INV, int LEPT = 4>
__global__ void __launch_bounds__(LEPT == 3 ? 1024 : 512, 1)
    k_coltx(const ColTx a, uint64_t ntiles, const Tw* __restrict__ tw) {
    using PL = ExtPlan<LOG_N, 0, LEPT, LEPT == 3 ? 1024 : 512>;
    extern __shared__ uint4 sm[];
    const int tid = threadIdx.x;
    const int q = tid % PL::Q4;
    const int t = tid / PL::Q4;
    V4 v[PL::EPT];
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t col = tile * PL::C + 4 * (uint64_t)q;
        const bool active = col < a.cols;
        constexpr int R0 = 1 << PL::lr(0);
        constexpr int L0 = PL::S / R0;
#pragma unroll
        for (int j = 0; j < R0; j++) {
            const uint32_t row = (uint32_t)t + (uint32_t)L0 * j;
            // a zero pre-factor (an erased row) skips the load
            const uint2 u = a.pre && row < a.in_rows ? __ldg(a.pre + row) : make_uint2(1u, 0u);
            if (active && row < a.in_rows && u.x != 0) {
                v[j] = ldg_stream_v4(a.in + (uint64_t)row * a.in_pitch + col);
                if (a.pre) mul4(v[j], Tw{u.x, u.y});
            } else {
                v[j] = V4{{0, 0, 0, 0}};
            }
        }
        dif_levels<PL, 0, INV>(v, sm, t, q, tw);
        using LV = Level<PL, PL::lr(PL::NLEV - 1), PL::pre(PL::NLEV - 1)>;
#pragma unroll
        for (int g = 0; g < LV::G; g++) {
            const uint32_t blk = LV::gid(g, t);
#pragma unroll
            for (int r = 0; r < LV::R; r++) {
                const uint32_t k = digit_rev<PL, false>((blk << PL::lr(PL::NLEV - 1)) +
                                                        (uint32_t)bitrev(r, PL::lr(PL::NLEV - 1)));
                if (active && k < a.out_rows) {
                    V4 x = v[g * LV::R + r];
                    if (a.post) {
                        const uint2 u = __ldg(a.post + k);
                        mul4(x, Tw{u.x, u.y});
                    } else {
                        mul4(x, a.scale);
                    }
                    stg_stream_v4(a.out + (uint64_t)k * a.out_pitch + col, x);
                }
            }
        }
    }
}

// Two transforms in one pass, the decoder's building block:
//   out[r] = NTT_N( mid(i) * INTT_N( pre(j) * in[j] )(i) )(r)
// with the INTT unscaled (mid carries any 1/N), rows j >= in_rows or with a
// zero pre-factor never read, and the product staying in registers between
// the transforms (the fused extension's INTT -> twist -> NTT with tables in
// place of g^i / S). OSH = 1 stores only the even outputs r = 2m, at row m:
// the k-point NTT of coefficients zero-padded to N = 2k. With `counter`, the
// INTT coefficients i >= count_from that are nonzero are counted (before mid).
struct ColTx2 {
    const uint32_t* in;
    uint64_t in_pitch;
    uint32_t in_rows;
    const uint2* pre;  // per input row
    const Tw* mid;     // per coefficient index, N entries
    uint32_t* out;
    uint64_t out_pitch;
    uint32_t out_rows;  // outputs r >= out_rows are not stored
    uint64_t cols;      // multiple of 4
    uint32_t count_from;
    unsigned long long* counter;  // or nullptr
};

template <int LOG_N, int LEPT, int OSH, bool COUNT>
__global__ void __launch_bounds__(LEPT == 3 ? 1024 : 512, 1)
    k_coltx2(const ColTx2 a, uint64_t ntiles, const Tw* __restrict__ tw) {
    using PL = ExtPlan<LOG_N, 0, LEPT, LEPT == 3 ? 1024 : 512>;
    extern __shared__ uint4 sm[];
    const int tid = threadIdx.x;
    const int q = tid % PL::Q4;
    const int t = tid / PL::Q4;
    const OddOut oo{a.out, a.out_pitch, a.out_rows};
    unsigned long long cnt = 0;
    V4 v[PL::EPT];
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t col = tile * PL::C + 4 * (uint64_t)q;
        const bool active = col < a.cols;
        constexpr int R0 = 1 << PL::lr(0);
        constexpr int G0 = PL::EPT / R0;
        constexpr int L0 = PL::S / R0;
#pragma unroll
        for (int g = 0; g < G0; g++)
#pragma unroll
            for (int j = 0; j < R0; j++) {
                const uint32_t row = (uint32_t)(g * PL::TPQ + t) + (uint32_t)L0 * j;
                const uint2 u = row < a.in_rows ? __ldg(a.pre + row) : make_uint2(0u, 0u);
                if (active && u.x != 0) {
                    v[g * R0 + j] = ldg_stream_v4(a.in + (uint64_t)row * a.in_pitch + col);
                    mul4(v[g * R0 + j], Tw{u.x, u.y});
                } else {
                    v[g * R0 + j] = V4{{0, 0, 0, 0}};
                }
            }
        dif_levels<PL, 0, true>(v, sm, t, q, tw);
        if constexpr (COUNT) {
            // the INTT's last level: group g holds coefficients c0 + (S/R) j at v[g R + bitrev(j)]
            constexpr int LR = PL::lr(PL::NLEV - 1);
            constexpr int R = 1 << LR;
            constexpr int SH = PL::LOG_S - LR;
#pragma unroll
            for (int g = 0; g < PL::EPT / R; g++) {
                const uint32_t c0 = digit_rev<PL, false>((uint32_t)(g * PL::TPQ + t) << LR);
#pragma unroll
                for (int j = 0; j < R; j++) {
                    const V4& x = v[g * R + bitrev(j, LR)];
                    if (active && c0 + ((uint32_t)j << SH) >= a.count_from)
#pragma unroll
                        for (int e = 0; e < 4; e++) cnt += x.c[e] % P != 0;
                }
            }
        }
        twist_and_first_ntt<PL, OSH>(v, sm, t, q, tw, a.mid, oo, col, active);
    }
    if constexpr (COUNT) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, o);
        if ((tid & 31) == 0 && cnt) atomicAdd(a.counter, cnt);
    }
}

}  // namespace zb
