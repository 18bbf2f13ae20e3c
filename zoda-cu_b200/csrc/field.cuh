// BabyBear field core for sm_100a: p = 2^31 - 2^27 + 1.
//
// Values stay canonical in [0, p) in memory and across the C ABI, exactly as
// the reference keeps them on the host (src/field/babybear.rs:11-23); there is
// no Montgomery domain, so no to/from conversion pass exists.
//
// Products by a known twiddle w use Shoup's method: with ws = floor(w * 2^32 / p),
// q = hi32(x * ws) and r = x*w - q*p (mod 2^32) lies in [0, 2p) for ANY 32-bit x.
// That tolerance lets butterfly outputs that feed a multiplication skip their
// reduction. One subtraction-min brings r back to [0, p).
//
// Measured on B200: IMAD runs at 64/clk/SM, IMAD.HI at 32/clk/SM and the ALU
// pipe (IADD3, IMNMX) at 64/clk/SM, so a Shoup product costs 4 FMA-pipe slots
// and each modular add 2 ALU slots; the NTT is bound by these pipes.
#pragma once
#include <cstdint>

namespace zb {

constexpr uint32_t P = 2013265921u;      // 2^31 - 2^27 + 1
constexpr uint32_t GENERATOR = 31u;      // smallest generator of F_p^*
constexpr int TWO_ADICITY = 27;          // p - 1 = 15 * 2^27

// ---- host/device constexpr number theory ----------------------------------
__host__ __device__ constexpr uint32_t mulmod_c(uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * b) % P);
}
__host__ __device__ constexpr uint32_t powmod_c(uint32_t b, uint64_t e) {
    uint32_t r = 1;
    while (e) {
        if (e & 1) r = mulmod_c(r, b);
        b = mulmod_c(b, b);
        e >>= 1;
    }
    return r;
}
// Primitive 2^log_n-th root of unity, the same one src/ntt/cpu.rs:96-110
// produces: 31^((p-1)/n).
__host__ __device__ constexpr uint32_t root_of_unity(int log_n) {
    return powmod_c(GENERATOR, (uint64_t)(P - 1) >> log_n);
}
__host__ __device__ constexpr uint32_t shoup(uint32_t w) {
    return (uint32_t)(((uint64_t)w << 32) / P);
}
// omega_{2^log_n}^e, inverse root when inv.
__host__ __device__ constexpr uint32_t root_pow(int log_n, uint32_t e, bool inv) {
    uint32_t n = 1u << log_n;
    e &= n - 1;
    if (inv) e = (n - e) & (n - 1);
    return powmod_c(root_of_unity(log_n), e);
}

// ---- device arithmetic -----------------------------------------------------
// The reductions use the DPX instruction VIADDMNMX (min(a + b, c) in one issue
// slot, native on sm_100a): a modular add is IADD3 + VIADDMNMX, a reduction
// from [0, 2p) a single VIADDMNMX.
__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b) {  // a, b in [0, p)
    return __viaddmin_u32(a, b, a + b - P);
}
__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b) {  // a, b in [0, p)
    const uint32_t d = a - b;
    return __viaddmin_u32(d, P, d);
}
__device__ __forceinline__ uint32_t reduce_2p(uint32_t r) {  // r in [0, 2p) -> [0, p)
    return __viaddmin_u32(r, 0u - P, r);
}
// x any u32 -> x*w mod p, in [0, 2p)
__device__ __forceinline__ uint32_t mul_lazy(uint32_t x, uint32_t w, uint32_t ws) {
    const uint32_t q = __umulhi(x, ws);
    return x * w - q * P;
}
__device__ __forceinline__ uint32_t mul_tw(uint32_t x, uint32_t w, uint32_t ws) {
    return reduce_2p(mul_lazy(x, w, ws));
}
// Generic modular product of two canonical values (64-bit remainder); used only
// off the hot path (tables, tests).
__device__ __forceinline__ uint32_t mul_slow(uint32_t a, uint32_t b) {
    return (uint32_t)(((uint64_t)a * b) % P);
}

// Gentleman-Sande (DIF) butterfly: (a, b) -> (a + b, (a - b) * w), inputs and
// outputs in [0, p). a - b + p lies in (0, 2p), a valid Shoup input, so the
// difference is never reduced on its own.
__device__ __forceinline__ void dif_bfly(uint32_t& a, uint32_t& b, uint32_t w, uint32_t ws) {
    uint32_t x = add_mod(a, b);
    uint32_t y = mul_tw(a - b + P, w, ws);
    a = x;
    b = y;
}
// Twiddle-free DIF butterfly: (a, b) -> (a + b, a - b). Two forms of the
// unreduced sum and difference: IADD3 adds on the ALU pipe, or IMAD
// (x*1 + y, x*(2^32-1) + y), which moves that work to the FMA pipe (the
// multipliers 1 and 2^32-1 live in constant memory, which the assembler cannot
// see through, so it keeps the IMADs instead of rewriting them as adds). Each
// kernel family picks the form per DIF stage with a mask: bit s set = the
// butterflies of stages with span 2^s use IMAD. ZB_FREE_IMAD_MASK is the
// default (the four-step passes); the TMA-staged kernels pass their own.
#ifndef ZB_FREE_IMAD_MASK
#define ZB_FREE_IMAD_MASK 0xFF
#endif
__constant__ uint32_t c_imad_one = 1u;
__constant__ uint32_t c_imad_neg1 = 0xFFFFFFFFu;
template <bool IMAD = true>
__device__ __forceinline__ void dif_bfly1(uint32_t& a, uint32_t& b) {
    uint32_t u, d;
    if constexpr (IMAD) {
        u = a * c_imad_one + b;     // a + b, IMAD
        d = b * c_imad_neg1 + a;    // a - b (mod 2^32), IMAD
    } else {
        u = a + b;
        d = a - b;
    }
    a = __viaddmin_u32(u, 0u - P, u);             // min(u - p, u)
    b = __viaddmin_u32(d, P, d);                  // min(d + p, d)
}

struct Tw {  // twiddle and its Shoup companion
    uint32_t w, ws;
};

}  // namespace zb
