// Fused column-wise Reed-Solomon extension, one HBM pass.
//
// For a data square stored row-major as in[k][cols] (k = S = 2^LOG_S rows), the
// reference (src/benchmarks/utils.rs:100-146, src/zoda/babybear.rs:34-46)
// transposes to column-major, zero-pads every column to 2S, runs INTT_S on the
// first S values and NTT_2S on all of them. With g = omega_2S (so omega_S = g^2):
//   out[2m]   = in[m]                                (the data, unchanged)
//   out[2m+1] = NTT_S( g^i / S * INTT_S'(in col) )[m] (INTT_S' = unscaled inverse DFT)
// This kernel computes exactly that, per column, reading in[] once and writing
// out[2S][cols] once, both row-major with 16-byte vectors.
//
// Work split: a CTA owns C = 4*Q4 adjacent columns of the whole square (a
// tile). Each thread owns one 16-byte column quad and EPT = 16 positions of it.
// The INTT runs as DIF levels of radix 16 (the last level takes the leftover
// bits), the twist multiplies by g^i / S, and the NTT runs the levels in the
// mirrored order, so the INTT's last level and the NTT's first level share
// their register groups and need no exchange. Between the other levels the
// tile is exchanged through shared memory (in place, slot-major).
#pragma once
#include <cstdint>

#include "dft.cuh"

namespace zb {

constexpr int LOG_TW = 13;  // global twiddle table: omega_8192^j, covers 2S up to 8192
constexpr int TW_N = 1 << LOG_TW;

// SCHED picks where the leftover radix goes when LOG_S is not a multiple of 4:
// 0 = the INTT's last level (and the NTT's first), 1 = the INTT's first level
// (and the NTT's last). The autotuner chooses per side.
// LEPT_ is the log2 of the level radix and of the positions a thread holds
// per column (4: radix 16; 3: radix 8 with half the registers, so twice the
// threads fit), THREADS_ the CTA size.
template <int LOG_S_, int SCHED_ = 0, int LEPT_ = 4, int THREADS_ = 512>
struct ExtPlan {
    static constexpr int LOG_S = LOG_S_;
    static constexpr int SCHED = SCHED_;
    static constexpr int LEPT = LEPT_;
    static constexpr int S = 1 << LOG_S;
    static constexpr int NLEV = (LOG_S + LEPT - 1) / LEPT;  // INTT levels (= NTT levels)
    static constexpr int EPT = LOG_S >= LEPT ? 1 << LEPT : S;
    static constexpr int TPQ = S / EPT;  // threads per column quad
    static constexpr int THREADS = THREADS_;
    static constexpr int Q4 = THREADS / TPQ;  // column quads per tile
    static constexpr int C = 4 * Q4;          // columns per tile
    static constexpr size_t SMEM = NLEV > 1 ? (size_t)S * Q4 * 16 : 0;
    static constexpr int LEFT = LOG_S - LEPT * (NLEV - 1);  // the leftover level's log2 radix
    // log2 radix of INTT level l; the NTT runs them in reverse order
    __host__ __device__ static constexpr int lr(int l) {
        return SCHED == 0 ? (l < NLEV - 1 ? LEPT : LEFT) : (l == 0 ? LEFT : LEPT);
    }
    __host__ __device__ static constexpr int nlr(int l) { return lr(NLEV - 1 - l); }
    __host__ __device__ static constexpr int pre(int l) {
        int s = 0;
        for (int i = 0; i < l; i++) s += lr(i);
        return s;
    }
    __host__ __device__ static constexpr int npre(int l) {
        int s = 0;
        for (int i = 0; i < l; i++) s += nlr(i);
        return s;
    }
};

// Output index of a DIF slot: the slot's digits, most significant first, with
// widths a_0..a_{m-1} (the level radices), read back least significant first.
template <class PL, bool NTT_SEQ>
__device__ __forceinline__ uint32_t digit_rev(uint32_t slot) {
    uint32_t out = 0;
    int sh_in = PL::LOG_S, sh_out = 0;
#pragma unroll
    for (int l = 0; l < PL::NLEV; l++) {
        const int a = NTT_SEQ ? PL::nlr(l) : PL::lr(l);
        sh_in -= a;
        out |= ((slot >> sh_in) & ((1u << a) - 1)) << sh_out;
        sh_out += a;
    }
    return out;
}

// omega_{2^logn}^e (INV: omega^-e) from the global table.
template <bool INV>
__device__ __forceinline__ Tw tw_at(const Tw* __restrict__ tw, uint32_t e, int logn) {
    uint32_t idx = e << (LOG_TW - logn);
    if (INV) idx = (TW_N - idx) & (TW_N - 1);
    uint2 u = __ldg(reinterpret_cast<const uint2*>(tw) + idx);
    return Tw{u.x, u.y};
}

// ---- one DIF level over the thread's register groups -----------------------
// Level geometry: 2^PB blocks of N = 2^LOGN slots; each block splits as
// n1 + L*n2 (L = 2^LOGL); a group is (block, n1) and holds R = 2^LR slots.
template <class PL, int LR, int PB>
struct Level {
    static constexpr int LRADIX = LR;
    static constexpr int R = 1 << LR;
    static constexpr int G = PL::EPT / R;
    static constexpr int LOGN = PL::LOG_S - PB;
    static constexpr int LOGL = LOGN - LR;
    __device__ static __forceinline__ uint32_t gid(int g, int t) { return (uint32_t)(g * PL::TPQ + t); }
    __device__ static __forceinline__ uint32_t base(uint32_t gid) {
        return ((gid >> LOGL) << LOGN) + (gid & ((1u << LOGL) - 1));
    }
    __device__ static __forceinline__ uint32_t n1(uint32_t gid) { return gid & ((1u << LOGL) - 1); }

    __device__ static __forceinline__ void read(V4* v, const uint4* sm, int t, int q) {
#pragma unroll
        for (int g = 0; g < G; g++) {
            const uint32_t b = base(gid(g, t));
#pragma unroll
            for (int j = 0; j < R; j++) {
                uint4 u = sm[(size_t)(b + ((uint32_t)j << LOGL)) * PL::Q4 + q];
                v[g * R + j] = V4{{u.x, u.y, u.z, u.w}};
            }
        }
    }
    // multiply output k2 = bitrev(r) of group (.., n1) by omega_N^(+-n1*k2) and
    // store it at slot base + L*k2
    template <bool INV>
    __device__ static __forceinline__ void twiddle_write(V4* v, uint4* sm, int t, int q, const Tw* tw) {
#pragma unroll
        for (int g = 0; g < G; g++) {
            const uint32_t id = gid(g, t);
            const uint32_t b = base(id), m = n1(id);
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int k2 = bitrev(r, LR);
                V4 x = v[g * R + r];
                if (k2 != 0) mul4(x, tw_at<INV>(tw, m * (uint32_t)k2, LOGN));
                sm[(size_t)(b + ((uint32_t)k2 << LOGL)) * PL::Q4 + q] = make_uint4(x.c[0], x.c[1], x.c[2], x.c[3]);
            }
        }
    }
    // store output k2 = bitrev(r) of each group at slot base + L*k2 (its twiddle
    // already applied)
    __device__ static __forceinline__ void write(const V4* v, uint4* sm, int t, int q) {
#pragma unroll
        for (int g = 0; g < G; g++) {
            const uint32_t b = base(gid(g, t));
#pragma unroll
            for (int r = 0; r < R; r++) {
                const V4& x = v[g * R + r];
                sm[(size_t)(b + ((uint32_t)bitrev(r, LR) << LOGL)) * PL::Q4 + q] =
                    make_uint4(x.c[0], x.c[1], x.c[2], x.c[3]);
            }
        }
    }
    template <bool INV>
    __device__ static __forceinline__ void dft(V4* v) {
#pragma unroll
        for (int g = 0; g < G; g++) dft_dif<LR, INV>(v + g * R);
    }
};

// DIF levels l..NLEV-1 with radices lr(); level 0's input is already in v.
// On return v holds the last level's outputs (register r of group g = block
// g*TPQ+t, slot block*R + bitrev(r)); the last level writes nothing.
template <class PL, int l, bool INV>
__device__ __forceinline__ void dif_levels(V4* v, uint4* sm, int t, int q, const Tw* tw) {
    if constexpr (l < PL::NLEV) {
        using LV = Level<PL, PL::lr(l), PL::pre(l)>;
        if constexpr (l > 0) LV::read(v, sm, t, q);
        LV::template dft<INV>(v);
        if constexpr (l < PL::NLEV - 1) {
            if constexpr (l == 0) __syncthreads();  // previous tile's last reads are done
            LV::template twiddle_write<INV>(v, sm, t, q, tw);
            __syncthreads();
            dif_levels<PL, l + 1, INV>(v, sm, t, q, tw);
        }
    }
}

// Where the odd output rows go: row k (k < rows) at p + k * stride, with
// (out + cols, 2 * cols) for the interleaved [2S][cols] layout and (out, cols)
// for the odd rows only; rows < S when the output is cut short (an encoding
// with fewer parity rows than data rows).
struct OddOut {
    uint32_t* p;
    uint64_t stride;
    uint32_t rows;
};

// OSH > 0 (the decoder's last pass): only outputs k with k % 2^OSH == 0 are
// stored, at row k >> OSH.
template <class PL, int l, int OSH = 0>
__device__ __forceinline__ void ntt_levels(V4* v, uint4* sm, int t, int q, const Tw* tw,
                                           const OddOut& oo, uint64_t col, bool active) {
    using LV = Level<PL, PL::nlr(l), PL::npre(l)>;
    if constexpr (l > 0) LV::read(v, sm, t, q);
    LV::template dft<false>(v);
    if constexpr (l < PL::NLEV - 1) {
        LV::template twiddle_write<false>(v, sm, t, q, tw);
        __syncthreads();
        ntt_levels<PL, l + 1, OSH>(v, sm, t, q, tw, oo, col, active);
    } else {
        // last level: L = 1, slot = block*R + k2 -> output index by digit reversal
#pragma unroll
        for (int g = 0; g < LV::G; g++) {
            const uint32_t blk = LV::gid(g, t);
#pragma unroll
            for (int r = 0; r < LV::R; r++) {
                const uint32_t k = digit_rev<PL, true>((blk << PL::nlr(l)) + (uint32_t)bitrev(r, PL::nlr(l)));
                if (active && k < oo.rows && (k & ((1u << OSH) - 1)) == 0)
                    stg_stream_v4(oo.p + (uint64_t)(k >> OSH) * oo.stride + col, v[g * LV::R + r]);
            }
        }
    }
}

// Twist between the INTT's last level and the NTT's first level. The INTT's
// last level has L = 1: group g of thread t is block b = g*TPQ + t holding
// slots b*R + k2, i.e. coefficients c0 + (S/R)*k2 with c0 = digit_rev(b*R).
// The NTT's first level (radix R over stride S/R) needs exactly those
// coefficients, in natural k2 order, as group n1 = c0.
template <class PL, int OSH = 0>
__device__ __forceinline__ void twist_and_first_ntt(V4* v, uint4* sm, int t, int q, const Tw* tw,
                                                    const Tw* __restrict__ twist, const OddOut& oo, uint64_t col,
                                                    bool active) {
    constexpr int LR = PL::lr(PL::NLEV - 1);
    constexpr int R = 1 << LR;
    constexpr int G = PL::EPT / R;
    constexpr int SH = PL::LOG_S - LR;  // log2(S/R)
    uint32_t c0[G];
#pragma unroll
    for (int g = 0; g < G; g++) {
        const uint32_t b = (uint32_t)(g * PL::TPQ + t);
        c0[g] = digit_rev<PL, false>(b << LR);
        V4 y[R];
#pragma unroll
        for (int j = 0; j < R; j++) {
            y[j] = v[g * R + bitrev(j, LR)];
            const uint2 u = __ldg(reinterpret_cast<const uint2*>(twist) + c0[g] + ((uint32_t)j << SH));
            mul4(y[j], Tw{u.x, u.y});
        }
#pragma unroll
        for (int j = 0; j < R; j++) v[g * R + j] = y[j];
    }
    // NTT level 0: radix R over stride S/R, one block; group n1 = c0
#pragma unroll
    for (int g = 0; g < G; g++) dft_dif<LR, false>(v + g * R);
    if constexpr (PL::NLEV > 1) {
        __syncthreads();  // every thread finished reading the INTT's last level
#pragma unroll
        for (int g = 0; g < G; g++) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int k2 = bitrev(r, LR);
                V4 x = v[g * R + r];
                if (k2 != 0) mul4(x, tw_at<false>(tw, c0[g] * (uint32_t)k2, PL::LOG_S));
                sm[(size_t)(c0[g] + ((uint32_t)k2 << SH)) * PL::Q4 + q] = make_uint4(x.c[0], x.c[1], x.c[2], x.c[3]);
            }
        }
        __syncthreads();
        ntt_levels<PL, 1, OSH>(v, sm, t, q, tw, oo, col, active);
    } else {
        // single level: output index k2 = bitrev(r)
#pragma unroll
        for (int r = 0; r < R; r++) {
            const uint32_t k = (uint32_t)bitrev(r, LR);
            if (active && k < oo.rows && (k & ((1u << OSH) - 1)) == 0)
                stg_stream_v4(oo.p + (uint64_t)(k >> OSH) * oo.stride + col, v[r]);
        }
    }
}

// in: [S][cols] row-major, out: [2S][cols] row-major. cols % 4 == 0, 16-byte
// aligned rows. Tiles of C columns are dealt to CTAs round-robin.
// Tiles a CTA visits: interleaved (tile = blockIdx.x + i * gridDim.x), or with
// `blocked` one contiguous run of ceil(ntiles / gridDim.x) tiles per CTA.
struct TileRange {
    uint64_t first, last, step;
    __device__ __forceinline__ TileRange(uint64_t ntiles, bool blocked) {
        if (blocked) {
            const uint64_t per = (ntiles + gridDim.x - 1) / gridDim.x;
            first = blockIdx.x * per;
            last = first + per < ntiles ? first + per : ntiles;
            step = 1;
        } else {
            first = blockIdx.x;
            last = ntiles;
            step = gridDim.x;
        }
    }
};

// LEPT 4: radix-16 levels, 512 threads; 3: radix-8 levels, 1024 threads.
template <int LOG_S, int SCHED = 0, int LEPT = 4>
__global__ void __launch_bounds__(LEPT == 3 ? 1024 : 512, 1)
    k_extend(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint64_t cols, uint64_t ntiles,
             const Tw* __restrict__ tw, const Tw* __restrict__ twist_all, uint32_t flags, uint32_t in_rows,
             uint32_t out_rows) {
    using PL = ExtPlan<LOG_S, SCHED, LEPT, LEPT == 3 ? 1024 : 512>;
    extern __shared__ uint4 sm[];
    const int tid = threadIdx.x;
    const int q = tid % PL::Q4;
    const int t = tid / PL::Q4;
    const Tw* twist = twist_all + PL::S;  // g^i / S for this side, i in [0, S)
    V4 v[PL::EPT];
    // flags bit 4: write only the odd rows, compactly (out is then [S][cols]).
    // Input rows >= in_rows are zeros (never read); rows >= out_rows of the
    // interleaved output are not written (an encoding of k < S data rows and
    // fewer than 2S rows); out_rows = 2S writes everything.
    const bool odd_only = flags & 16;
    const OddOut oo{odd_only ? out : out + cols, odd_only ? cols : 2 * cols, out_rows / 2};
    const TileRange tr(ntiles, flags & 1);
    for (uint64_t tile = tr.first; tile < tr.last; tile += tr.step) {
        const uint64_t col = tile * PL::C + 4 * (uint64_t)q;
        const bool active = col < cols;
        // INTT level 0 gathers, for each of its G0 groups g, rows
        // g*TPQ + t + L0*j (L0 = S / R0) straight from HBM and writes them to
        // the even output rows on the way.
        constexpr int R0 = 1 << PL::lr(0);
        constexpr int G0 = PL::EPT / R0;
        constexpr int L0 = PL::S / R0;
#pragma unroll
        for (int g = 0; g < G0; g++)
#pragma unroll
            for (int j = 0; j < R0; j++) {
                const uint64_t row = (uint64_t)(g * PL::TPQ + t) + (uint64_t)L0 * j;
                v[g * R0 + j] = active && row < in_rows ? ldg_stream_v4(in + row * cols + col) : V4{{0, 0, 0, 0}};
                // even rows: the (zero-padded) data
                if (active && !odd_only && 2 * row < out_rows) stg_stream_v4(out + 2 * row * cols + col, v[g * R0 + j]);
            }
        dif_levels<PL, 0, true>(v, sm, t, q, tw);
        twist_and_first_ntt<PL>(v, sm, t, q, tw, twist, oo, col, active);
    }
}

// Plain batched transform of every column of in[N][cols] (row-major, N =
// 2^LOG_S): out[k][col] = scale * sum_i in[i][col] * omega_N^(+-i*a*k) written
// at row k, natural order. a (odd) selects the primitive root omega^a that a
// caller's roots table holds; scale is 1 or N^-1. This is the device half of
// the reference's cuda_ntt / cuda_intt (cuda/ntt_kernel.cu:106-180).
template <int LOG_S, bool INV>
__global__ void __launch_bounds__(512, 1)
    k_colntt(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint64_t cols, uint64_t ntiles,
             const Tw* __restrict__ tw, Tw scale, uint32_t a) {
    using PL = ExtPlan<LOG_S>;
    extern __shared__ uint4 sm[];
    const int tid = threadIdx.x;
    const int q = tid % PL::Q4;
    const int t = tid / PL::Q4;
    V4 v[PL::EPT];
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint64_t col = tile * PL::C + 4 * (uint64_t)q;
        const bool active = col < cols;
        constexpr int R0 = 1 << PL::lr(0);
        constexpr int L0 = PL::S / R0;
#pragma unroll
        for (int j = 0; j < R0; j++) {
            const uint64_t row = (uint64_t)t + (uint64_t)L0 * j;
            v[j] = active ? ldg_stream_v4(in + row * cols + col) : V4{{0, 0, 0, 0}};
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
                const uint32_t row = (k * a) & (PL::S - 1);
                V4 x = v[g * LV::R + r];
                mul4(x, scale);
                if (active) stg_stream_v4(out + (uint64_t)row * cols + col, x);
            }
        }
    }
}

}  // namespace zb
