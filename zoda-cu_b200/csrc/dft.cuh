// Register-resident DFT building blocks shared by every kernel in the library.
//
// A thread holds a small group of field elements per column in registers,
// always for four adjacent columns at once (a "quad", one 16-byte vector), so
// every twiddle it loads or computes is reused four times.
//
// dft_dif<LOG_R, INV> runs the radix-2^LOG_R Gentleman-Sande network on the
// register group: natural-order input, bit-reversed output (register r holds
// output index bitrev(r)). Its internal twiddles are compile-time constants,
// so they become immediate operands.
#pragma once
#include <cstdint>
#include <utility>

#include "field.cuh"

namespace zb {

struct V4 {
    uint32_t c[4];
};

__device__ __forceinline__ V4 ld_v4(const uint32_t* p) {
    uint4 u = *reinterpret_cast<const uint4*>(p);
    return V4{{u.x, u.y, u.z, u.w}};
}
__device__ __forceinline__ void st_v4(uint32_t* p, const V4& v) {
    *reinterpret_cast<uint4*>(p) = make_uint4(v.c[0], v.c[1], v.c[2], v.c[3]);
}
// streaming (evict-first) variants for data touched once
__device__ __forceinline__ V4 ldg_stream_v4(const uint32_t* p) {
    uint4 u = __ldcs(reinterpret_cast<const uint4*>(p));
    return V4{{u.x, u.y, u.z, u.w}};
}
__device__ __forceinline__ void stg_stream_v4(uint32_t* p, const V4& v) {
    __stcs(reinterpret_cast<uint4*>(p), make_uint4(v.c[0], v.c[1], v.c[2], v.c[3]));
}

__host__ __device__ constexpr int bitrev(int x, int bits) {
    int r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
}

__device__ __forceinline__ void bfly4(V4& a, V4& b, uint32_t w, uint32_t ws) {
#pragma unroll
    for (int c = 0; c < 4; c++) dif_bfly(a.c[c], b.c[c], w, ws);
}
// FM: bit s set = the twiddle-free butterflies of stages with span 2^s use IMAD
template <int LH = 0, int FM = ZB_FREE_IMAD_MASK>
__device__ __forceinline__ void bfly4_1(V4& a, V4& b) {
#pragma unroll
    for (int c = 0; c < 4; c++) dif_bfly1<((FM >> LH) & 1) != 0>(a.c[c], b.c[c]);
}
__device__ __forceinline__ void mul4(V4& a, const Tw t) {
#pragma unroll
    for (int c = 0; c < 4; c++) a.c[c] = mul_tw(a.c[c], t.w, t.ws);
}

namespace detail {
template <bool INV, int LH, int J, int FM>
__device__ __forceinline__ void bfly_at(V4* x) {
    constexpr int h = 1 << LH;
    if constexpr ((J & h) == 0) {
        constexpr int e = J & (h - 1);
        if constexpr (e == 0) {
            bfly4_1<LH, FM>(x[J], x[J + h]);
        } else {
            constexpr uint32_t w = root_pow(LH + 1, (uint32_t)e, INV);
            constexpr uint32_t ws = shoup(w);
            bfly4(x[J], x[J + h], w, ws);
        }
    }
}
template <bool INV, int LH, int FM, int... Js>
__device__ __forceinline__ void stage(V4* x, std::integer_sequence<int, Js...>) {
    (bfly_at<INV, LH, Js, FM>(x), ...);
}
// stages with span 2^LH down to 2^LOW
template <bool INV, int LOG_R, int LH, int LOW = 0, int FM = ZB_FREE_IMAD_MASK>
__device__ __forceinline__ void stages(V4* x) {
    if constexpr (LH >= LOW) {
        stage<INV, LH, FM>(x, std::make_integer_sequence<int, (1 << LOG_R)>{});
        stages<INV, LOG_R, LH - 1, LOW, FM>(x);
    }
}
}  // namespace detail

// In-register DIF DFT of size 2^LOG_R over x[0..2^LOG_R), four columns at once.
// INV selects omega^-1 (the transform src/ntt/cpu.rs:48-60 runs before its n^-1 scale).
template <int LOG_R, bool INV, int FM = ZB_FREE_IMAD_MASK>
__device__ __forceinline__ void dft_dif(V4* x) {
    detail::stages<INV, LOG_R, LOG_R - 1, 0, FM>(x);
}

namespace detail {
template <int LR, bool SKIP0, int I, class TwF>
__device__ __forceinline__ void pair_twout(V4* x, const TwF& twf) {
    constexpr int ka = bitrev(I, LR), kb = bitrev(I + 1, LR);
    const Tw tb = twf.template get<kb>();
    if constexpr (SKIP0 && ka == 0) {
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const uint32_t a = x[I].c[c], b = x[I + 1].c[c];
            x[I].c[c] = add_mod(a, b);
            x[I + 1].c[c] = mul_tw(a - b + P, tb.w, tb.ws);
        }
    } else {
        const Tw ta = twf.template get<ka>();
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const uint32_t a = x[I].c[c], b = x[I + 1].c[c];
            x[I].c[c] = mul_tw(a + b, ta.w, ta.ws);
            x[I + 1].c[c] = mul_tw(a - b + P, tb.w, tb.ws);
        }
    }
}
template <int LR, bool SKIP0, class TwF, int... Is>
__device__ __forceinline__ void last_stage_twout(V4* x, const TwF& twf, std::integer_sequence<int, Is...>) {
    (pair_twout<LR, SKIP0, 2 * Is>(x, twf), ...);
}
}  // namespace detail

// DIF DFT of size 2^LR whose last (twiddle-free) stage also multiplies output
// k2 = bitrev(r) by twf.get<k2>(); a + b and a - b + p lie in [0, 2p), valid
// Shoup inputs, so those sums are never reduced on their own. With SKIP0 the
// output k2 = 0 has factor 1 and is only reduced.
template <int LR, bool INV, bool SKIP0, int FM = ZB_FREE_IMAD_MASK, class TwF>
__device__ __forceinline__ void dft_dif_twout(V4* x, const TwF& twf) {
    if constexpr (LR > 1) detail::stages<INV, LR, LR - 1, 1, FM>(x);
    detail::last_stage_twout<LR, SKIP0>(x, twf, std::make_integer_sequence<int, (1 << LR) / 2>{});
}

}  // namespace zb
