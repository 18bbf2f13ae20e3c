// Fused extension, TMA-staged variant for sides 32..4096, one square per launch
// or many squares of mixed sides in one persistent launch.
//
// Same math and level structure as extend.cuh (INTT DIF levels, twist, NTT DIF
// levels in mirrored order), organised for latency hiding:
//   * the CTA's input tile [S rows][C cols] arrives in shared memory by TMA
//     (cp.async.bulk.tensor, boxes of 256 rows x C columns, C*4 >= 32 bytes of
//     contiguous row segment per box row); the next tile's load is issued as
//     soon as every thread has copied the current one into registers, so it
//     overlaps the whole butterfly phase;
//   * the even output rows (a copy of the input) leave by TMA store straight
//     from the staging buffer; the odd rows leave by 16-byte streaming stores;
//   * the CTA is split into two warp-groups of 256 threads, each owning half of
//     the tile's column quads with its own exchange buffer and named barrier,
//     so one group computes while the other waits at a barrier;
//   * the exchange between levels goes through shared memory in two halves
//     (columns 0-1, then 2-3 of every quad), which keeps staging + exchange +
//     twiddle tables inside 227 KB;
//   * the inter-level twiddles and the twist are folded into each level's last
//     butterfly stage: a + b and a - b + p lie in [0, 2p), valid Shoup inputs,
//     so those sums are never reduced on their own.
#pragma once
#include <cuda.h>

#include "async.cuh"
#include "extend.cuh"

namespace zb {

// The TMA-staged kernels build their twiddle-free butterflies with IADD3 adds on
// the ALU pipe (mask 0) rather than the IMAD form: 3% faster at side 1024 and 2%
// on the full 2048 square (radix 8) in A/B runs on one box.
#ifndef ZB_TMA_FREE_MASK
#define ZB_TMA_FREE_MASK 0
#endif
constexpr int TMA_FREE_MASK = ZB_TMA_FREE_MASK;

// ---- geometry ------------------------------------------------------------------
// Shared-memory layouts are chosen so that every warp access is bank-conflict
// free (checked with a bank model of all access patterns):
//   * staging: TMA swizzle (128B / 64B / 32B mode for 128 / 64 / 32-byte rows),
//     16-byte chunk index XOR-ed with row bits, undone when reading; the two
//     warp-groups own alternating column quads;
//   * exchange: word(slot, q) = slot*GQ + q + sum PW*(slot >> PS), a padding that
//     stays additive in the register index, so addresses keep immediate offsets;
//   * twiddle tables live in HBM/L1 in [k2][index] order (see SideTables).
// Exchange padding word(slot) += PW1*(slot >> PS1) + PW2*(slot >> PS2) and
// the lane map's basis images PB0..PB2, per side and level radix, found with a
// bank model of every staging read and exchange access (conflict free except
// a 2-way case in one radix-16 exchange at side 512 and a few radix-8 ones at
// side 4096).
template <int LOG_S, int LEPT>
struct XPad;
template <int LOG_S>
struct XPad<LOG_S, 4> {
    static constexpr int PS1 = LOG_S == 9 ? 1 : LOG_S == 10 ? 3 : LOG_S == 11 ? 3 : LOG_S == 12 ? 4 : 0;
    static constexpr int PW1 = LOG_S == 9 ? 1 : LOG_S == 10 ? 8 : LOG_S == 11 ? 2 : LOG_S == 12 ? 1 : 0;
    static constexpr int PS2 = LOG_S == 10 ? 4 : LOG_S == 11 ? 6 : 0;
    static constexpr int PW2 = LOG_S == 10 ? 4 : LOG_S == 11 ? 2 : 0;
    static constexpr int PB0 = LOG_S == 10 ? 5 : 1;
    static constexpr int PB1 = LOG_S == 10 ? 2 : LOG_S == 11 ? 4 : 2;
    static constexpr int PB2 = LOG_S == 10 ? 1 : LOG_S == 11 ? 2 : 4;
};
template <int LOG_S>
struct XPad<LOG_S, 3> {  // radix 8, 1024 threads (side 4096 keeps a few 2-way conflicts)
    static constexpr int PS1 = LOG_S == 9 ? 1 : LOG_S == 10 ? 3 : LOG_S == 11 ? 3 : LOG_S == 12 ? 4 : 0;
    static constexpr int PW1 = LOG_S == 9 ? 1 : LOG_S == 10 ? 4 : LOG_S == 11 ? 2 : LOG_S == 12 ? 2 : 0;
    static constexpr int PS2 = LOG_S == 9 ? 2 : LOG_S == 10 ? 6 : LOG_S == 11 ? 6 : LOG_S == 12 ? 7 : 0;
    static constexpr int PW2 = LOG_S == 9 ? 2 : LOG_S == 10 ? 4 : LOG_S == 11 ? 2 : LOG_S == 12 ? 1 : 0;
    static constexpr int PB0 = LOG_S == 10 ? 5 : 1;
    static constexpr int PB1 = LOG_S == 10 ? 3 : LOG_S == 11 ? 4 : 2;
    static constexpr int PB2 = LOG_S == 10 ? 1 : LOG_S == 11 ? 2 : 4;
};

// LEPT_ 4: radix-16 levels, 512 threads; 3: radix-8 levels, 1024 threads.
template <int LOG_S_, int LEPT_ = 4>
struct TPlan {
    using PL = ExtPlan<LOG_S_, 0, LEPT_, LEPT_ == 3 ? 1024 : 512>;  // whole-CTA view: Q4 quads, C columns
    static constexpr int LOG_S = LOG_S_;
    static constexpr int LEPT = LEPT_;
    static constexpr int S = PL::S, C = PL::C, Q4 = PL::Q4, TPQ = PL::TPQ, EPT = PL::EPT;
    static constexpr int NLEV = PL::NLEV;
    static constexpr int THREADS = PL::THREADS;
    static constexpr int GS = THREADS / 2;  // threads per warp-group
    static constexpr int GQ = Q4 / 2;       // quads per warp-group
    // TMA boxes: at most 256 rows x 256 columns; sides below 128 have tiles wider
    // than 256 columns and stage them as NBOXC column boxes side by side.
    static constexpr int BOX_R = S < 256 ? S : 256;
    static constexpr int BOX_C = C < 256 ? C : 256;
    static constexpr int NBOXR = S / BOX_R, NBOXC = C / BOX_C;
    static constexpr int NBOX = NBOXR * NBOXC;
    static constexpr uint32_t TILE_BYTES = (uint32_t)S * C * 4;
    // staging swizzle: box rows of BOX_C*4 bytes; 0 = none, else the XOR mask on (offset >> 7)
    static constexpr int ROW_BYTES = BOX_C * 4;
    static constexpr uint32_t SWZ_MASK = ROW_BYTES == 128 ? 7 : ROW_BYTES == 64 ? 3 : ROW_BYTES == 32 ? 1 : 0;
    static constexpr int QB = BOX_C / 4;  // quads per box row
    using XP = XPad<LOG_S, LEPT_>;
    // Lane map inside a warp: quad ql = lane % GQ, row group t = TW*warp + perm(lane / GQ),
    // perm a bit-linear map (images of the basis vectors) chosen, together with the
    // exchange padding, so staging reads and every exchange access are conflict free.
    static constexpr int TW = GQ < 32 ? 32 / GQ : 1;
    static constexpr int PB0 = XP::PB0, PB1 = XP::PB1, PB2 = XP::PB2;
    __device__ static __forceinline__ int lane_t(int x) {  // x = lane / GQ in [0, TW)
        int y = x & ~7;
        if (x & 1) y ^= PB0;
        if (x & 2) y ^= PB1;
        if (x & 4) y ^= PB2;
        return y;
    }
    static constexpr size_t X_WORDS = (size_t)S * GQ + (size_t)XP::PW1 * (S >> XP::PS1) +
                                      (size_t)XP::PW2 * (XP::PW2 ? (S >> XP::PS2) : 0) + GQ;
    static constexpr size_t X_BYTES = X_WORDS * 8;  // one group's half-exchange buffer
    static constexpr size_t OFF_X = TILE_BYTES;
    static constexpr size_t OFF_BAR = (OFF_X + 2 * X_BYTES + 15) / 16 * 16;
    static constexpr size_t SMEM = OFF_BAR + 32;
    static_assert(LOG_S >= 5 && LOG_S <= 12, "TMA path covers sides 32..4096");
    static_assert(NLEV <= 4, "level tables cover four levels");
    static_assert(GQ >= 1, "two warp-groups");
    static_assert(NLEV >= 2, "at least one exchange");
    static_assert(SMEM <= 232448, "shared memory budget");
    static_assert(SWZ_MASK == 0 || (S / 16) * ROW_BYTES % (128 * (SWZ_MASK + 1)) == 0,
                  "staging row offsets j*L0 must keep the swizzle phase");
    __host__ __device__ static constexpr int lr(int l) { return PL::lr(l); }
    __host__ __device__ static constexpr int nlr(int l) { return PL::nlr(l); }
    __host__ __device__ static constexpr int pre(int l) { return PL::pre(l); }
    __host__ __device__ static constexpr int npre(int l) { return PL::npre(l); }
    // padded exchange word offset of a slot (additive over disjoint bit fields)
    __host__ __device__ static constexpr uint32_t xoff(uint32_t slot) {
        return slot * GQ + XP::PW1 * (slot >> XP::PS1) + (XP::PW2 ? XP::PW2 * (slot >> XP::PS2) : 0);
    }
    __device__ static __forceinline__ uint32_t xword(uint32_t slot, int ql) { return xoff(slot) + (uint32_t)ql; }
    // staging byte offset of (row, quad): column box bc sits at bc * S box rows
    __device__ static __forceinline__ uint32_t stage_off(uint32_t row, int q) {
        const uint32_t bc = (uint32_t)q / QB, qi = (uint32_t)q % QB;
        const uint32_t o = (bc * S + row) * ROW_BYTES + 16u * qi;
        if constexpr (SWZ_MASK) return o ^ (((o >> 7) & SWZ_MASK) << 4);
        return o;
    }
    // TMA box b = bc * NBOXR + br: smem element offset and global (x, y) in a tile
    __device__ static __forceinline__ uint32_t box_smem(int b) { return (uint32_t)b * BOX_R * BOX_C; }
    __device__ static __forceinline__ int box_x(uint64_t tile, int b) { return (int)(tile * C) + (b / NBOXR) * BOX_C; }
    __device__ static __forceinline__ int box_y(int b) { return (b % NBOXR) * BOX_R; }
};

// Per-side twiddle tables in HBM (read through L1), laid out [k2][index] so a
// warp's lanes (consecutive group index) read consecutive 8-byte entries:
//   intt[l][k2*L + m] = omega_N^(-m*k2)      INTT levels 0..NLEV-2
//   ntt0[k2*NB + b]   = g^c0(b)/S * omega_S^(c0(b)*k2)   NTT level 0 with the twist
//   ntt[l][k2*L + m]  = omega_N^(m*k2)       NTT levels 1..NLEV-2
// where level geometry (N, L, R) is that of ExtPlan, b the INTT last-level
// block, c0(b) its first coefficient index.
struct SideTables {
    const uint2* intt[3];
    const uint2* ntt0;
    const uint2* ntt[3];
};

// Twiddle functors: get<K>() returns the factor for output k2 = K.
template <int L>
struct TabTw {
    const uint2* p;  // &table[index]
    template <int K>
    __device__ __forceinline__ Tw get() const {
        const uint2 u = __ldg(p + K * L);
        return Tw{u.x, u.y};
    }
};
template <int LOG_M, bool INV>
struct ConstTw {  // omega_{2^LOG_M}^(+-K), an immediate
    template <int K>
    __device__ __forceinline__ Tw get() const {
        constexpr uint32_t w = root_pow(LOG_M, (uint32_t)K, INV);
        constexpr uint32_t ws = shoup(w);
        return Tw{w, ws};
    }
};

struct KTw {  // a per-k2 table: factor for output k2 = K is p[K]
    const uint2* p;
    template <int K>
    __device__ __forceinline__ Tw get() const {
        const uint2 u = __ldg(p + K);
        return Tw{u.x, u.y};
    }
};

// Level geometry (as ExtPlan): 2^PB blocks of N = 2^LOGN slots, slot = block*N |
// n1 | (j << LOGL); the thread's group g is gid = g*TPQ + t.
template <class TP, int LR, int PB>
struct LvlGeom {
    static constexpr int R = 1 << LR;
    static constexpr int G = TP::EPT / R;
    static constexpr int LOGN = TP::LOG_S - PB;
    static constexpr int LOGL = LOGN - LR;
    static constexpr int L = 1 << LOGL;
    __device__ static __forceinline__ uint32_t gid(int g, int t) { return (uint32_t)(g * TP::TPQ + t); }
    __device__ static __forceinline__ uint32_t base(uint32_t id) {
        return ((id >> LOGL) << LOGN) | (id & ((1u << LOGL) - 1));
    }
    __device__ static __forceinline__ uint32_t n1(uint32_t id) { return id & ((1u << LOGL) - 1); }
};

// Exchange through one group's half buffer. The writer's output register
// g*RW + r (DFT output k2 = bitrev(r)) sits at slot wbase(g) | (k2 << WSH); the
// reader's input register g*RR + j at slot rbase(g) | (j << RSH). The base and
// the shifted index occupy disjoint bits, so each padded word address is a
// per-group base plus a compile-time offset. Columns 0-1 go first, then 2-3.
template <class TP, int RW, int WSH, int RR, int RSH, class WB, class RBs>
__device__ __forceinline__ void exchange(V4* v, uint2* xg, int ql, int bar, const WB& wbase, const RBs& rbase) {
    constexpr int GW = TP::EPT / RW, GR = TP::EPT / RR;
    constexpr int LRW = RW == 1 ? 0 : RW == 2 ? 1 : RW == 4 ? 2 : RW == 8 ? 3 : 4;
    uint32_t wb[GW], rb[GR];
#pragma unroll
    for (int g = 0; g < GW; g++) wb[g] = TP::xword(wbase(g), ql);
#pragma unroll
    for (int g = 0; g < GR; g++) rb[g] = TP::xword(rbase(g), ql);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        group_bar(bar, TP::GS);
#pragma unroll
        for (int g = 0; g < GW; g++)
#pragma unroll
            for (int r = 0; r < RW; r++)
                xg[wb[g] + TP::xoff((uint32_t)bitrev(r, LRW) << WSH)] =
                    make_uint2(v[g * RW + r].c[2 * h], v[g * RW + r].c[2 * h + 1]);
        group_bar(bar, TP::GS);
#pragma unroll
        for (int g = 0; g < GR; g++)
#pragma unroll
            for (int j = 0; j < RR; j++) {
                const uint2 u = xg[rb[g] + TP::xoff((uint32_t)j << RSH)];
                v[g * RR + j].c[2 * h] = u.x;
                v[g * RR + j].c[2 * h + 1] = u.y;
            }
    }
}

// INTT levels l .. NLEV-2 (each followed by an exchange); the last INTT level is
// run by the kernel body.
// With stagger_pending set, group 0 releases group 1 (named barrier 3) as it
// starts INTT level `stagger_at`.
template <int THREADS>
__device__ __forceinline__ void stagger_release(bool& stagger_pending) {
    if (stagger_pending) {
        asm volatile("bar.arrive 3, %0;" ::"n"(THREADS) : "memory");
        stagger_pending = false;
    }
}
template <class TP, int l>
__device__ __forceinline__ void intt_upto_last(V4* v, uint2* xg, int t, int ql, int bar, const SideTables& tb,
                                               bool& stagger_pending, int stagger_at) {
    if constexpr (l < TP::NLEV - 1) {
        if (l == stagger_at) stagger_release<TP::THREADS>(stagger_pending);
        using W = LvlGeom<TP, TP::lr(l), TP::pre(l)>;
        using Rd = LvlGeom<TP, TP::lr(l + 1), TP::pre(l + 1)>;
#pragma unroll
        for (int g = 0; g < W::G; g++) {
            const TabTw<W::L> twf{tb.intt[l] + W::n1(W::gid(g, t))};
            dft_dif_twout<TP::lr(l), true, true, TMA_FREE_MASK>(v + g * W::R, twf);
        }
        exchange<TP, W::R, W::LOGL, Rd::R, Rd::LOGL>(
            v, xg, ql, bar, [&](int g) { return W::base(W::gid(g, t)); },
            [&](int g) { return Rd::base(Rd::gid(g, t)); });
        intt_upto_last<TP, l + 1>(v, xg, t, ql, bar, tb, stagger_pending, stagger_at);
    }
}

// NTT levels l .. NLEV-1 (level 0 runs in the kernel body); the last one stores
// the odd output rows (OSH > 0: only outputs k % 2^OSH == 0, at row k >> OSH).
template <class TP, int l, int OSH = 0>
__device__ __forceinline__ void ntt_from(V4* v, uint2* xg, int t, int ql, int bar, const SideTables& tb,
                                         const OddOut& oo, uint64_t col, bool active) {
    using LV = LvlGeom<TP, TP::nlr(l), TP::npre(l)>;
    if constexpr (l < TP::NLEV - 1) {
        using Rd = LvlGeom<TP, TP::nlr(l + 1), TP::npre(l + 1)>;
#pragma unroll
        for (int g = 0; g < LV::G; g++) {
            const TabTw<LV::L> twf{tb.ntt[l] + LV::n1(LV::gid(g, t))};
            dft_dif_twout<TP::nlr(l), false, true, TMA_FREE_MASK>(v + g * LV::R, twf);
        }
        exchange<TP, LV::R, LV::LOGL, Rd::R, Rd::LOGL>(
            v, xg, ql, bar, [&](int g) { return LV::base(LV::gid(g, t)); },
            [&](int g) { return Rd::base(Rd::gid(g, t)); });
        ntt_from<TP, l + 1, OSH>(v, xg, t, ql, bar, tb, oo, col, active);
    } else {
#pragma unroll
        for (int g = 0; g < LV::G; g++) dft_dif<TP::nlr(l), false, TMA_FREE_MASK>(v + g * LV::R);
#pragma unroll
        for (int g = 0; g < LV::G; g++) {
            const uint32_t blk = LV::gid(g, t);
#pragma unroll
            for (int r = 0; r < LV::R; r++) {
                const uint32_t k =
                    digit_rev<typename TP::PL, true>((blk << TP::nlr(l)) | (uint32_t)bitrev(r, TP::nlr(l)));
                if (active && k < oo.rows && (k & ((1u << OSH) - 1)) == 0)
                    stg_stream_v4(oo.p + (uint64_t)(k >> OSH) * oo.stride + col, v[g * LV::R + r]);
            }
        }
    }
}

// ---- per-tile pieces shared by the single-square and the batched kernels -------

// Thread coordinates inside its warp-group (see the lane map in TPlan).
template <class TP>
struct Coords {
    int ql, t, q;
    __device__ __forceinline__ Coords(int ltid, int grp) {
        const int lane = ltid & 31, wg = ltid >> 5;
        ql = TP::GQ < 32 ? lane % TP::GQ : ltid % TP::GQ;
        t = TP::GQ < 32 ? wg * TP::TW + TP::lane_t(lane / TP::GQ) : ltid / TP::GQ;
        q = grp * TP::GQ + ql;
    }
};

template <class TP>
__device__ __forceinline__ void tma_load_tile(uint32_t* stage, const CUtensorMap* map, uint64_t tile,
                                              uint64_t* full) {
    mbar_expect_tx(full, TP::TILE_BYTES);
#pragma unroll
    for (int b = 0; b < TP::NBOX; b++)
        tma_load_2d(stage + TP::box_smem(b), map, TP::box_x(tile, b), TP::box_y(b), full);
}
template <class TP>
__device__ __forceinline__ void tma_store_even(const uint32_t* stage, const CUtensorMap* map, uint64_t tile) {
#pragma unroll
    for (int b = 0; b < TP::NBOX; b++) tma_store_2d(map, TP::box_x(tile, b), TP::box_y(b), stage + TP::box_smem(b));
    bulk_commit();
}

// INTT level 0 gathers rows t + L0*j of the thread's quad from staging.
template <class TP>
__device__ __forceinline__ void stage_read(V4* v, const unsigned char* smem, const Coords<TP>& c) {
    constexpr int R0 = 1 << TP::lr(0);
    constexpr int L0 = TP::S / R0;
    const unsigned char* sb = smem + TP::stage_off((uint32_t)c.t, c.q);
#pragma unroll
    for (int j = 0; j < R0; j++) {
        const uint4 u = *reinterpret_cast<const uint4*>(sb + (size_t)j * L0 * TP::ROW_BYTES);
        v[j] = V4{{u.x, u.y, u.z, u.w}};
    }
}

// Everything after the tile is in registers: INTT, twist, NTT, odd-row stores
// (see OddOut).
// With stagger_pending set, group 0 releases group 1 (named barrier 3) when it
// starts INTT level stagger_at (NLEV-1: after all INTT levels but the last).
// TWM (the decoder's passes): 0 = the extension's twist (immediates in the last
// INTT stage); 1 = per-k2 factors ktw[k2] instead; 2 = the same, then the
// coefficients of the upper half (k2 >= R/2, i.e. index >= S/2) are counted into
// *cnt where nonzero and set to zero. OSH as in ntt_from.
template <class TP, int OSH = 0, int TWM = 0>
__device__ __forceinline__ void tile_compute(V4* v, uint2* xg, const Coords<TP>& c, int bar, const SideTables& tb,
                                             const OddOut& oo, uint64_t col, bool active,
                                             bool& stagger_pending, int stagger_at = TP::NLEV - 1,
                                             const uint2* ktw = nullptr, unsigned long long* cnt = nullptr) {
    const int t = c.t, ql = c.ql;
    // ---- INTT levels 0 .. NLEV-2
    intt_upto_last<TP, 0>(v, xg, t, ql, bar, tb, stagger_pending, stagger_at);
    stagger_release<TP::THREADS>(stagger_pending);
    {
        // ---- INTT last level (L = 1). Its outputs need the twist g^c / S with
        // c = c0 + k2*S/R; g^(k2*S/R) = omega_2R^k2 is an immediate folded into the
        // last butterfly stage, and g^c0 / S is folded into NTT level 0's table.
        constexpr int LR = TP::lr(TP::NLEV - 1);
        constexpr int R = 1 << LR;
        constexpr int G = TP::EPT / R;
        constexpr int NB = TP::S / R;  // INTT last-level blocks
        constexpr int SH = TP::LOG_S - LR;
        using LV = LvlGeom<TP, LR, TP::pre(TP::NLEV - 1)>;
        using Rd = LvlGeom<TP, TP::nlr(1), TP::npre(1)>;
#pragma unroll
        for (int g = 0; g < G; g++) {
            if constexpr (TWM == 0) dft_dif_twout<LR, true, true, TMA_FREE_MASK>(v + g * R, ConstTw<LR + 1, false>{});
            else dft_dif_twout<LR, true, true, TMA_FREE_MASK>(v + g * R, KTw{ktw});
            // NTT level 0 wants coefficient c0 + (S/R)*j in register j
            V4 y[R];
#pragma unroll
            for (int j = 0; j < R; j++) y[j] = v[g * R + bitrev(j, LR)];
#pragma unroll
            for (int j = 0; j < R; j++) v[g * R + j] = y[j];
            if constexpr (TWM == 2) {
#pragma unroll
                for (int j = R / 2; j < R; j++) {
                    if (active)
#pragma unroll
                        for (int e = 0; e < 4; e++) *cnt += v[g * R + j].c[e] % P != 0;
                    v[g * R + j] = V4{{0, 0, 0, 0}};
                }
            }
            // ---- NTT level 0: radix R over stride S/R, then g^c0/S * omega_S^(c0*k2)
            const TabTw<NB> twf{tb.ntt0 + LV::gid(g, t)};
            dft_dif_twout<LR, false, false, TMA_FREE_MASK>(v + g * R, twf);
        }
        exchange<TP, R, SH, Rd::R, Rd::LOGL>(
            v, xg, ql, bar, [&](int g) { return digit_rev<typename TP::PL, false>(LV::gid(g, t) << LR); },
            [&](int g) { return Rd::base(Rd::gid(g, t)); });
    }
    // ---- NTT levels 1 .. NLEV-1, the last one stores the odd rows
    ntt_from<TP, 1, OSH>(v, xg, t, ql, bar, tb, oo, col, active);
}

// Re-derive a value from an opaque copy so the compiler rebuilds per-tile
// addresses inside the loop instead of keeping them all live across it.
__device__ __forceinline__ int opaque(int x) {
    int y;
    asm volatile("mov.u32 %0, %1;" : "=r"(y) : "r"(x));
    return y;
}

// ---- one square ------------------------------------------------------------------
// flags: bit 0 = blocked tile order (TileRange), bit 1 = no stagger between the
// warp-groups, bits 2-3 = the INTT level at which group 0 releases group 1,
// plus one (0: the default, after all INTT levels but the last), bit 4 = write
// only the odd rows, compactly ([S][cols]; the even rows are the input).
template <int LOG_S, int LEPT = 4>
__global__ void __launch_bounds__(TPlan<LOG_S, LEPT>::THREADS, 1)
    k_extend_tma(const __grid_constant__ CUtensorMap tm_in, const __grid_constant__ CUtensorMap tm_even,
                 uint32_t* __restrict__ out, uint64_t cols, uint64_t ntiles, const SideTables tb,
                 int* __restrict__ err, uint32_t flags, uint32_t out_rows) {
    using TP = TPlan<LOG_S, LEPT>;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint32_t* stage = reinterpret_cast<uint32_t*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TP::OFF_BAR);   // tile landed (TMA tx)
    uint64_t* empty = full + 1;                                          // both groups copied it out
    const int tid = threadIdx.x;
    const int grp = tid / TP::GS;
    const int bar = 1 + grp;
    // The first thread of group 1 (the group that reads the staging buffer
    // last) is the producer: it issues every TMA load and even-row store.
    const bool producer = tid == TP::GS;
    if (tid == 0) {
        mbar_init(full, 1);
        mbar_init(empty, 2);
        fence_mbar_init();
    }
    __syncthreads();
    const TileRange tr(ntiles, flags & 1);
    const bool stagger = !(flags & 2);
    // bit 4: only the odd rows, compactly (out is then [S][cols]); rows >= out_rows
    // of the interleaved output are not written (the even-row map is cut there too)
    const bool odd_only = flags & 16;
    const OddOut oo{odd_only ? out : out + cols, odd_only ? cols : 2 * cols, out_rows / 2};
    const int stagger_at = (flags >> 2) & 3 ? (int)((flags >> 2) & 3) - 1 : TP::NLEV - 1;
    uint64_t tile = tr.first;
    if (producer && tile < tr.last) tma_load_tile<TP>(stage, &tm_in, tile, full);
    // Group 1 starts half a tile after group 0 so the two groups' barriers and
    // butterfly phases interleave; group 0 signals from the middle of its first tile.
    if (stagger && grp == 1 && tile < tr.last) asm volatile("bar.sync 3, %0;" ::"n"(TP::THREADS) : "memory");
    bool stagger_pending = stagger && grp == 0 && tile < tr.last;
    V4 v[TP::EPT];
    uint32_t parity = 0;
    for (; tile < tr.last; tile += tr.step, parity ^= 1) {
        const int tid_l = opaque(tid);
        const Coords<TP> c(tid_l % TP::GS, grp);
        uint2* xg = reinterpret_cast<uint2*>(smem + TP::OFF_X + (tid_l / TP::GS) * TP::X_BYTES);
        const bool ok = mbar_wait_bounded(full, parity);
        if (group_vote_or(bar, !ok, TP::GS)) {
            if (tid % TP::GS == 0) atomicOr(err, 1);
            stagger_release<TP::THREADS>(stagger_pending);
            if (producer) bulk_wait0();
            return;
        }
        if (producer && !odd_only) tma_store_even<TP>(stage, &tm_even, tile);  // even output rows = the input tile
        const uint64_t col = tile * TP::C + 4 * (uint64_t)c.q;
        const bool active = col < cols;
        stage_read<TP>(v, smem, c);
        group_bar(bar, TP::GS);  // this group has copied the staging buffer out
        if (tid % TP::GS == 0) mbar_arrive(empty);
        const uint64_t next = tile + tr.step;
        if (producer && next < tr.last) {
            const bool e_ok = mbar_wait_bounded(empty, parity);  // the other group is done too
            bulk_wait_read0();  // the even-row store has finished reading staging
            fence_proxy_async();
            if (e_ok) tma_load_tile<TP>(stage, &tm_in, next, full);
            else atomicOr(err, 2);  // both groups then time out on `full` and leave
        }
        tile_compute<TP>(v, xg, c, bar, tb, oo, col, active, stagger_pending, stagger_at);
    }
    stagger_release<TP::THREADS>(stagger_pending);
    if (producer) bulk_wait0();
}

// ---- one pass of the erasure decoder on the TMA-staged shape ---------------------
// out[r] = NTT_S(mid(i) * INTT_S(pre(j) * in[j])(i))(r) over [S][cols] tiles, with
// mid(c0 + (S/R) k2) = (block factor of c0, in tb.ntt0) * ktw[k2]: the two
// passes of zoda_recover_device (general.cu). Rows with pre = 0 are loaded and
// zeroed (they may hold anything); with PRE = false there are no pre-factors
// (the any-shape encode's coset passes). TWM and OSH as in tile_compute;
// *counter receives the upper-half count with TWM = 2. Same pipeline as
// k_extend_tma without the even-row stores.
template <int LOG_S, int LEPT, int OSH, int TWM, bool PRE = true>
__global__ void __launch_bounds__(TPlan<LOG_S, LEPT>::THREADS, 1)
    k_dec_tma(const __grid_constant__ CUtensorMap tm_in, uint32_t* __restrict__ out, uint64_t out_pitch,
              uint32_t out_rows, uint64_t cols, uint64_t ntiles, const SideTables tb, const uint2* __restrict__ pre,
              const uint2* __restrict__ ktw, unsigned long long* __restrict__ counter, int* __restrict__ err,
              uint32_t flags) {
    using TP = TPlan<LOG_S, LEPT>;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint32_t* stage = reinterpret_cast<uint32_t*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + TP::OFF_BAR);
    uint64_t* empty = full + 1;
    const int tid = threadIdx.x;
    const int grp = tid / TP::GS;
    const int bar = 1 + grp;
    const bool producer = tid == TP::GS;
    if (tid == 0) {
        mbar_init(full, 1);
        mbar_init(empty, 2);
        fence_mbar_init();
    }
    __syncthreads();
    const TileRange tr(ntiles, flags & 1);
    const bool stagger = !(flags & 2);
    const OddOut oo{out, out_pitch, out_rows};
    const int stagger_at = (flags >> 2) & 3 ? (int)((flags >> 2) & 3) - 1 : TP::NLEV - 1;
    unsigned long long cnt = 0;
    uint64_t tile = tr.first;
    if (producer && tile < tr.last) tma_load_tile<TP>(stage, &tm_in, tile, full);
    if (stagger && grp == 1 && tile < tr.last) asm volatile("bar.sync 3, %0;" ::"n"(TP::THREADS) : "memory");
    bool stagger_pending = stagger && grp == 0 && tile < tr.last;
    V4 v[TP::EPT];
    uint32_t parity = 0;
    for (; tile < tr.last; tile += tr.step, parity ^= 1) {
        const int tid_l = opaque(tid);
        const Coords<TP> c(tid_l % TP::GS, grp);
        uint2* xg = reinterpret_cast<uint2*>(smem + TP::OFF_X + (tid_l / TP::GS) * TP::X_BYTES);
        const bool ok = mbar_wait_bounded(full, parity);
        if (group_vote_or(bar, !ok, TP::GS)) {
            if (tid % TP::GS == 0) atomicOr(err, 1);
            stagger_release<TP::THREADS>(stagger_pending);
            return;
        }
        const uint64_t col = tile * TP::C + 4 * (uint64_t)c.q;
        const bool active = col < cols;
        stage_read<TP>(v, smem, c);
        group_bar(bar, TP::GS);  // this group has copied the staging buffer out
        if (tid % TP::GS == 0) mbar_arrive(empty);
        const uint64_t next = tile + tr.step;
        if (producer && next < tr.last) {
            const bool e_ok = mbar_wait_bounded(empty, parity);  // the other group is done too
            fence_proxy_async();
            if (e_ok) tma_load_tile<TP>(stage, &tm_in, next, full);
            else atomicOr(err, 2);  // both groups then time out on `full` and leave
        }
        if constexpr (PRE) {  // row pre-factors: stage_read gave register j row t + L0*j
            constexpr int R0 = 1 << TP::lr(0);
            constexpr int L0 = TP::S / R0;
#pragma unroll
            for (int j = 0; j < R0; j++) {
                const uint2 u = __ldg(pre + (uint32_t)c.t + (uint32_t)L0 * j);
                mul4(v[j], Tw{u.x, u.y});
            }
        }
        tile_compute<TP, OSH, TWM>(v, xg, c, bar, tb, oo, col, active, stagger_pending, stagger_at, ktw, &cnt);
    }
    stagger_release<TP::THREADS>(stagger_pending);
    if constexpr (TWM == 2) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, o);
        if ((tid & 31) == 0 && cnt) atomicAdd(counter, cnt);
    }
}

// ---- many squares of mixed sides in one persistent launch ---------------------------
// Work items are (square, column tile) pairs; squares come sorted by decreasing
// side, and a global counter deals tiles to CTAs in that order, so big squares
// start first and small ones fill the tail. The producer thread takes the next
// item, writes its descriptor next to the staging buffer and starts its TMA
// load; the consumers read the descriptor once the tile has landed.
struct BatchSquare {
    CUtensorMap in_map;    // [k][cols] input, boxes of the side's TPlan
    CUtensorMap even_map;  // even output rows
    uint32_t* out;
    uint64_t cols;
    uint64_t first;        // global index of the square's first tile
    uint32_t log_s, ntiles;
    uint32_t pad_[8];
};
static_assert(sizeof(BatchSquare) % 64 == 0, "tensor maps stay 64-byte aligned");

constexpr int BATCH_MIN_LOG = 5, BATCH_MAX_LOG = 11;
constexpr size_t cmax(size_t a, size_t b) { return a > b ? a : b; }
template <int L, int H, int LEPT>
struct BatchLayout {
    static constexpr size_t X = cmax(TPlan<L, LEPT>::X_BYTES, BatchLayout<L + 1, H, LEPT>::X);
};
template <int H, int LEPT>
struct BatchLayout<H, H, LEPT> {
    static constexpr size_t X = TPlan<H, LEPT>::X_BYTES;
};
// Shared-memory layout of the batched kernel with level radix 2^LEPT:
// 128 KB staging, the two groups' exchange buffers, barriers and the slot.
template <int LEPT>
struct BatchGeom {
    static constexpr int THREADS = LEPT == 3 ? 1024 : 512;
    static constexpr size_t X_BYTES = BatchLayout<BATCH_MIN_LOG, BATCH_MAX_LOG, LEPT>::X;
    static constexpr size_t OFF_X = 128 * 1024;
    static constexpr size_t OFF_BAR = (OFF_X + 2 * X_BYTES + 15) / 16 * 16;
    static constexpr size_t SMEM = OFF_BAR + 64;
    static_assert(SMEM <= 232448, "shared memory budget");
};

struct BatchSlot {  // descriptor of the tile in staging, written by the producer
    uint32_t sq;     // square index, or BATCH_END when the queue is drained
    uint32_t log_s;
    uint64_t tile;
};
constexpr uint32_t BATCH_END = 0xFFFFFFFFu;

#define ZB_BATCH_SWITCH(LS, CALL) \
    switch (LS) {                 \
        case 5: CALL(5); break;   \
        case 6: CALL(6); break;   \
        case 7: CALL(7); break;   \
        case 8: CALL(8); break;   \
        case 9: CALL(9); break;   \
        case 10: CALL(10); break; \
        default: CALL(11); break; \
    }

// sq[0..nsq) sorted by first; total_tiles = sum of ntiles; *counter = 0 at
// launch; tables[log_s] holds the level tables of radix 2^LEPT.
template <int LEPT = 4>
__global__ void __launch_bounds__(BatchGeom<LEPT>::THREADS, 1)
    k_extend_batch(const BatchSquare* __restrict__ sq, uint32_t nsq, uint64_t total_tiles,
                   unsigned long long* __restrict__ counter, const SideTables* __restrict__ tables,
                   int* __restrict__ err) {
    using BG = BatchGeom<LEPT>;
    constexpr int GS = BG::THREADS / 2;
    extern __shared__ __align__(1024) unsigned char smem[];
    uint32_t* stage = reinterpret_cast<uint32_t*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + BG::OFF_BAR);
    uint64_t* empty = full + 1;
    BatchSlot* slot = reinterpret_cast<BatchSlot*>(smem + BG::OFF_BAR + 16);
    uint32_t* sq_hint = reinterpret_cast<uint32_t*>(smem + BG::OFF_BAR + 32);
    const int tid = threadIdx.x;
    const int grp = tid / GS;
    const int bar = 1 + grp;
    const bool producer = tid == GS;
    if (tid == 0) {
        mbar_init(full, 1);
        mbar_init(empty, 2);
        fence_mbar_init();
        *sq_hint = 0;
    }
    __syncthreads();
    // producer: take the next tile from the queue and start its load
    auto fetch = [&]() {
        const unsigned long long g = atomicAdd(counter, 1ull);
        BatchSlot s{BATCH_END, 0, 0};
        if (g < total_tiles) {
            uint32_t i = *sq_hint;  // a CTA's items come in increasing order: short scans
            while (i + 1 < nsq && sq[i + 1].first <= g) i++;
            while (i > 0 && sq[i].first > g) i--;
            *sq_hint = i;
            s.sq = i;
            s.log_s = sq[i].log_s;
            s.tile = g - sq[i].first;
        }
        *slot = s;
        if (s.sq == BATCH_END) {
            mbar_arrive(full);  // completes the phase with no bytes: consumers see the end mark
        } else {
            const BatchSquare& b = sq[s.sq];
#define ZB_LOAD(L) tma_load_tile<TPlan<L, LEPT>>(stage, &b.in_map, s.tile, full)
            ZB_BATCH_SWITCH(s.log_s, ZB_LOAD)
#undef ZB_LOAD
        }
    };
    if (producer) fetch();
    if (grp == 1) asm volatile("bar.sync 3, %0;" ::"n"(BG::THREADS) : "memory");
    bool stagger_pending = grp == 0;
    V4 v[1 << LEPT];
    uint32_t parity = 0;
    for (;; parity ^= 1) {
        const int tid_l = opaque(tid);
        const bool ok = mbar_wait_bounded(full, parity);
        if (group_vote_or(bar, !ok, GS)) {
            if (tid % GS == 0) atomicOr(err, 1);
            break;
        }
        const BatchSlot s = *slot;
        if (s.sq == BATCH_END) break;
        const BatchSquare& b = sq[s.sq];
        if (producer) {
#define ZB_STORE(L) tma_store_even<TPlan<L, LEPT>>(stage, &b.even_map, s.tile)
            ZB_BATCH_SWITCH(s.log_s, ZB_STORE)
#undef ZB_STORE
        }
        const SideTables& tb = tables[s.log_s];
        uint32_t* const out = b.out;
        const uint64_t cols = b.cols;
        // consumers copy the tile out (arriving on `empty`), then the producer
        // refills staging while everybody computes
#define ZB_TILE(L)                                                                               \
    {                                                                                            \
        using TP = TPlan<L, LEPT>;                                                               \
        const Coords<TP> c(tid_l % GS, grp);                                                     \
        uint2* xg = reinterpret_cast<uint2*>(smem + BG::OFF_X + (tid_l / GS) * BG::X_BYTES);     \
        stage_read<TP>(v, smem, c);                                                              \
        group_bar(bar, GS);                                                                      \
        if (tid % GS == 0) mbar_arrive(empty);                                                   \
        if (producer) {                                                                          \
            const bool e_ok = mbar_wait_bounded(empty, parity);                                  \
            bulk_wait_read0();                                                                   \
            fence_proxy_async();                                                                 \
            if (e_ok) fetch();                                                                   \
            else atomicOr(err, 2);                                                               \
        }                                                                                        \
        const uint64_t col = s.tile * TP::C + 4 * (uint64_t)c.q;                                 \
        tile_compute<TP>(v, xg, c, bar, tb, OddOut{out + cols, 2 * cols, (uint32_t)TP::S}, col, col < cols,   \
                         stagger_pending);                                                       \
    }
        ZB_BATCH_SWITCH(s.log_s, ZB_TILE)
#undef ZB_TILE
    }
    stagger_release<BG::THREADS>(stagger_pending);
    if (producer) bulk_wait0();
}

}  // namespace zb
