// Long-column transforms: the four-step decomposition of a column NTT of length
// S = N1 * N2 (S up to 2^26) into passes of N1 or N2 points, each on the same
// register-resident DIF levels as the single-pass kernels (extend.cuh).
//
// With input index i = N2*i1 + i2 and output index k = k1 + N1*k2,
//   X[k1 + N1*k2] = sum_{i2} w_N2^(i2*k2) * [ w_S^(i2*k1) * sum_{i1} x[N2*i1 + i2] * w_N1^(i1*k1) ]
// so pass A transforms over i1 (rows N2 apart: a "wide" matrix whose row i1 is
// the N2 consecutive rows N2*i1 .. N2*i1 + N2-1) and multiplies output k1 of
// wide column i2 by w_S^(i2*k1); pass B transforms over i2 inside block k1 (the
// N2 consecutive rows N2*k1 + i2) and writes row k1 + N1*k2 in natural order.
//
// Every pass reads and writes matrices through a View: element (row r, virtual
// quad v) sits at base + (v / qpc) * cb_pitch + (v % qpc) * 4 + r * row_pitch,
// i.e. quads (4 adjacent u32 columns, one 16-byte vector) are grouped into
// column blocks of qpc quads. Pass A's column block is i2 (row pitch N2*cols,
// block pitch cols); pass B's is k1 (row pitch cols, block pitch N2*cols).
//
// Fused passes run two transforms of the same length with a pointwise factor
// between them in registers:
//   * k_step2<.., INV1 = true, INV2 = false>: pass B of an INTT, the factor,
//     pass A of the following NTT (whose decomposition is (N2, N1), so its
//     wide column is the INTT's block): a "block" pass;
//   * k_step2<.., false, true>: pass B of an NTT, the factor, pass A of the
//     following INTT with the same decomposition: a "strided" pass.
#pragma once
#include "async.cuh"
#include "extend.cuh"

namespace zb {

constexpr int LOG_TWM = 26;  // master root omega_{2^26}: w_S^e = w_M^(e * M / S)
constexpr uint32_t TWM_MASK = (1u << LOG_TWM) - 1;

struct View {
    uint32_t* base;
    uint64_t row_pitch;  // u32 between rows
    uint64_t cb_pitch;   // u32 between column blocks
};

// Factor f(r, cb) = tab[r * rm + cb * cm], a Shoup pair; tab == nullptr: 1.
struct FTab {
    const uint2* tab;
    uint32_t rm, cm;
};

struct StepArgs {
    View in, out;
    View copy;        // base != nullptr: every loaded input row is also stored here, unchanged
    uint32_t qpc;     // quads per column block
    uint64_t nquads;  // virtual quads of the pass
    uint32_t qlim;    // quads at or past this index inside a column block are not real (a ragged chunk)
    // an input row whose index r * lim_rm + cb * lim_cm (its row in the
    // original matrix) is >= in_limit is zero and not read
    uint32_t in_lim_rm, in_lim_cm;
    uint64_t in_limit;
    // an output whose index k * out_lim_rm + cb * out_lim_cm is >= out_limit
    // is not stored
    uint32_t out_lim_rm, out_lim_cm;
    uint64_t out_limit;
    FTab pre;         // per input row (k_step): a zero factor skips the load
    FTab mid1, mid2;  // k_step2: factors on the first transform's output k
    FTab post;        // per output
    int tw_log;       // > 0: output (k, cb) times omega_{2^tw_log}^(+-cb * k), sign - when tw_inv
    int tw_inv;
    int use_scale;  // output times `scale`
    Tw scale;
    uint32_t count_from;          // k_step2 with counter: count nonzero first-transform outputs k >= count_from
    unsigned long long* counter;  // or nullptr
};

// Whether the extension's folded passes that load straight from memory split the
// CTA into two barrier groups (SF_GROUPS).
#ifndef ZB_PASS_GROUPS
#define ZB_PASS_GROUPS 1
#endif

// Features a pass may use, as compile-time flags: a pass instantiated without a
// flag drops that feature's code and its runtime test (SF_ALL keeps every test).
enum : int {
    SF_PRE = 1,       // row pre-factors
    SF_LIM_IN = 2,    // input row limit
    SF_LIM_OUT = 4,   // output cut
    SF_POST = 8,      // output factors
    SF_TW = 16,       // output twiddle omega^(+-cb*k)
    SF_SCALE = 64,    // output scale
    SF_COPY = 128,    // copy of the loaded rows
    SF_MID = 256,     // factors between the two transforms
    SF_CNT = 512,     // count of nonzero high coefficients
    SF_ALL = 1023,
    // SF_FOLD: every twiddle and factor that follows a DFT level is folded into the
    // level's last butterfly stage (dft_dif_twout), whose sums then skip their own
    // reduction. The pass then reads its level twiddles from the compact table
    // (tw_at_c) passed in place of the omega_8192 table, takes its output twiddle
    // as post-factors (no SF_TW), mid1 alone (mid2 unused), and no SF_CNT.
    SF_FOLD = 1024,
    // SF_NOPREBAR: the caller has already ordered the previous tile's last reads of
    // shared memory before this tile (the pipelined launch's per-item barrier), so
    // the first exchange write needs no barrier of its own (direct loads only: a
    // staged tile's buffer is still being read by other threads)
    SF_NOPREBAR = 2048,
    // SF_GROUPS (with SF_FOLD, loads straight from memory): the CTA's threads form
    // two halves, each owning half of the tile's column quads and their exchange
    // slots, with its own named barrier, so one half's exchange waits do not hold
    // the other half
    SF_GROUPS = 4096,
    SF_PASS_GROUPS = ZB_PASS_GROUPS ? SF_GROUPS : 0,  // the extension's direct-load passes
    // the extension's passes (long_extend): strided INTT with its output twiddle
    // (a post-factor table) and the even-row copy; block pass with the middle
    // factor and its output twiddle; strided NTT
    SF_EXT_A = SF_POST | SF_COPY | SF_FOLD,
    SF_EXT_M = SF_MID | SF_POST | SF_FOLD,
    SF_EXT_B = SF_FOLD,
};

__device__ __forceinline__ Tw ftab_at(const FTab& f, uint32_t r, uint32_t cb) {
    const uint2 u = __ldg(f.tab + (r * f.rm + cb * f.cm));
    return Tw{u.x, u.y};
}

// x times omega_{2^tw_log}^(+-e) for e < 2^tw_log, from the two-level table:
// E = e * 2^(26 - tw_log); w_M^E = tw_hi[E >> 13] * tw_lo[E & 8191], where
// tw_hi = omega_8192^j (the context's table) and tw_lo = omega_{2^26}^j.
__device__ __forceinline__ void mul_tw2d(V4& x, uint32_t e, int tw_log, bool inv, const Tw* __restrict__ tw_hi,
                                         const Tw* __restrict__ tw_lo) {
    uint32_t E = (e << (LOG_TWM - tw_log)) & TWM_MASK;
    if (inv) E = (0u - E) & TWM_MASK;
    const uint32_t hi = E >> 13, lo = E & 8191u;
    if (hi) {
        const uint2 u = __ldg(reinterpret_cast<const uint2*>(tw_hi) + hi);
        mul4(x, Tw{u.x, u.y});
    }
    if (lo) {
        const uint2 u = __ldg(reinterpret_cast<const uint2*>(tw_lo) + lo);
        mul4(x, Tw{u.x, u.y});
    }
}

// Quad v's column block and the offset of its 4 columns inside the block.
struct QuadPos {
    uint32_t cb, qi;
    bool active;
    __device__ __forceinline__ QuadPos(uint64_t v, const StepArgs& a) {
        active = v < a.nquads;
        const uint32_t vv = active ? (uint32_t)v : 0u;
        cb = vv / a.qpc;
        qi = vv - cb * a.qpc;
        active = active && qi < a.qlim;
    }
};

// Memory policies of a pass. Loads: streaming (evict-first, the default) or
// through L2 only (LD_L2), for matrices another CTA of the same launch wrote, which
// an SM's L1 may hold a stale copy of. Stores: streaming (the default) or kept
// (ST_KEEP, the normal L2 policy) for intermediates the next pass reads soon.
__device__ __forceinline__ V4 ldg_l2_v4(const uint32_t* p) {
    uint4 u = __ldcg(reinterpret_cast<const uint4*>(p));
    return V4{{u.x, u.y, u.z, u.w}};
}
template <bool LD_L2>
__device__ __forceinline__ V4 step_ld(const uint32_t* p) {
    if constexpr (LD_L2) return ldg_l2_v4(p);
    return ldg_stream_v4(p);
}
template <bool ST_KEEP>
__device__ __forceinline__ void step_st(uint32_t* p, const V4& v) {
    if constexpr (ST_KEEP) st_v4(p, v);
    else stg_stream_v4(p, v);
}

// Input row `row` of the quad exists (the quad is real and the row is inside the limit).
template <int F = SF_ALL>
__device__ __forceinline__ bool row_in(const StepArgs& a, const QuadPos& p, uint32_t row) {
    if constexpr (F & SF_LIM_IN)
        return p.active && (uint64_t)row * a.in_lim_rm + (uint64_t)p.cb * a.in_lim_cm < a.in_limit;
    return p.active;
}

// Level 0 input: rows t + L0*j of the thread's quad, pre-factors applied, rows
// past the limit (or with a zero factor) as zeros.
template <class PL, bool LD_L2 = false, int F = SF_ALL>
__device__ __forceinline__ void step_load(V4* v, const StepArgs& a, const QuadPos& p, int t) {
    constexpr int R0 = 1 << PL::lr(0);
    constexpr int L0 = PL::S / R0;
    const uint32_t* src = a.in.base + (uint64_t)p.cb * a.in.cb_pitch + 4ull * p.qi;
#pragma unroll
    for (int j = 0; j < R0; j++) {
        const uint32_t row = (uint32_t)t + (uint32_t)L0 * j;
        bool ld = row_in<F>(a, p, row);
        Tw f{1u, 0u};
        if ((F & SF_PRE) && a.pre.tab && ld) {
            f = ftab_at(a.pre, row, p.cb);
            ld = f.w != 0;
        }
        if (ld) {
            v[j] = step_ld<LD_L2>(src + (uint64_t)row * a.in.row_pitch);
            if ((F & SF_COPY) && a.copy.base)
                stg_stream_v4(a.copy.base + (uint64_t)p.cb * a.copy.cb_pitch + 4ull * p.qi +
                                  (uint64_t)row * a.copy.row_pitch,
                              v[j]);
            if ((F & SF_PRE) && a.pre.tab) mul4(v[j], f);
        } else {
            v[j] = V4{{0, 0, 0, 0}};
        }
    }
}

// Output k of the thread's quad: post factors, then the store (if in range).
template <bool ST_KEEP = false, int F = SF_ALL>
__device__ __forceinline__ void step_store(V4 x, const StepArgs& a, const QuadPos& p, uint32_t k,
                                           const Tw* __restrict__ tw, const Tw* __restrict__ tw_lo) {
    if (!p.active) return;
    if constexpr (F & SF_LIM_OUT)
        if ((uint64_t)k * a.out_lim_rm + (uint64_t)p.cb * a.out_lim_cm >= a.out_limit) return;
    if ((F & SF_POST) && a.post.tab) mul4(x, ftab_at(a.post, k, p.cb));
    if ((F & SF_TW) && a.tw_log) mul_tw2d(x, p.cb * k, a.tw_log, a.tw_inv, tw, tw_lo);
    if ((F & SF_SCALE) && a.use_scale) mul4(x, a.scale);
    step_st<ST_KEEP>(a.out.base + (uint64_t)p.cb * a.out.cb_pitch + 4ull * p.qi + (uint64_t)k * a.out.row_pitch,
                     x);
}

// ---- staged loads: a tile's level-0 rows arrive by cp.async ---------------------
// Each thread copies exactly the 16-byte slots it reads back later (rows t + L0*j
// of its quad), so a thread's own cp.async.wait_group is the only wait the staged
// data needs. cp.async.cg goes through L2 only, never a stale L1 line. Rows that
// do not exist are zero-filled (source size 0) from a valid address.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
                 "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Start the copies of tile `tile`'s level-0 rows into `stage` ([S][Q4] uint4 slots).
template <class PL, int F = SF_ALL>
__device__ __forceinline__ void step_prefetch(uint4* stage, const StepArgs& a, uint64_t tile, int q, int t) {
    constexpr int R0 = 1 << PL::lr(0);
    constexpr int L0 = PL::S / R0;
    const QuadPos p(tile * PL::Q4 + q, a);
    const uint32_t* src = a.in.base + (uint64_t)p.cb * a.in.cb_pitch + 4ull * p.qi;
#pragma unroll
    for (int j = 0; j < R0; j++) {
        const uint32_t row = (uint32_t)t + (uint32_t)L0 * j;
        const bool ld = row_in<F>(a, p, row);
        cp_async16(stage + (size_t)row * PL::Q4 + q, ld ? src + (uint64_t)row * a.in.row_pitch : a.in.base, ld);
    }
}

// Level 0 input from the stage: the copy of the loaded rows and the pre-factors as
// step_load (a row with a zero pre-factor is loaded and multiplied to zero).
template <class PL, int F = SF_ALL>
__device__ __forceinline__ void step_consume(V4* v, const uint4* stage, const StepArgs& a, const QuadPos& p, int q,
                                             int t) {
    constexpr int R0 = 1 << PL::lr(0);
    constexpr int L0 = PL::S / R0;
#pragma unroll
    for (int j = 0; j < R0; j++) {
        const uint32_t row = (uint32_t)t + (uint32_t)L0 * j;
        const uint4 u = stage[(size_t)row * PL::Q4 + q];
        v[j] = V4{{u.x, u.y, u.z, u.w}};
        if (((F & SF_COPY) && a.copy.base) || ((F & SF_PRE) && a.pre.tab)) {
            const bool ld = row_in<F>(a, p, row);
            if ((F & SF_COPY) && ld && a.copy.base)
                stg_stream_v4(a.copy.base + (uint64_t)p.cb * a.copy.cb_pitch + 4ull * p.qi +
                                  (uint64_t)row * a.copy.row_pitch,
                              v[j]);
            if ((F & SF_PRE) && ld && a.pre.tab) mul4(v[j], ftab_at(a.pre, row, p.cb));
        }
    }
}

// Launch shapes of the passes: level radix 2^LEPT, THREADS per CTA, MINB CTAs
// resident per SM (MINB > 1 lets one CTA load its tile while another computes,
// which the single-CTA shape cannot do: its loads go straight to registers).
//   0: radix 16 / 512 threads (radix 8 / 1024 from 512 points), one CTA per SM
//   1: radix 16, 256 threads, 2 per SM      2: radix 8, 512 threads, 2 per SM
//   3: radix 8, 256 threads, 4 per SM       4: radix 4, 256 threads, 5 per SM
//   (1..4: the extension's passes, 32..128 points)
template <int LOG_N, int SHAPE>
struct StepShape {
    static constexpr int LEPT = SHAPE == 0 ? (LOG_N >= 9 ? 3 : 4) : SHAPE == 1 ? 4 : SHAPE == 4 ? 2 : 3;
    static constexpr int THREADS = SHAPE == 0 ? (LOG_N >= 9 ? 1024 : 512) : SHAPE == 2 ? 512 : 256;
    static constexpr int MINB = SHAPE == 0 ? 1 : SHAPE == 3 ? 4 : SHAPE == 4 ? 5 : 2;
    using PL = ExtPlan<LOG_N, 0, LEPT, THREADS>;
    // staged passes hold two tiles (the next one arriving, the current one, which
    // also serves as the exchange buffer): CTAs per SM that fit 227 KB
    static constexpr int MINB_ST_FIT = (int)(232448 / (2 * (PL::SMEM > 0 ? PL::SMEM : 1)));
    static constexpr int MINB_ST = MINB_ST_FIT < MINB ? MINB_ST_FIT : MINB;
};

// ---- levels with folded twiddles (SF_FOLD) --------------------------------------
// Level l of the forward (MIR false) or mirrored (MIR true, the second transform
// of a fused pass) radix sequence.
template <class PL, int l, bool MIR>
using LvlOf = Level<PL, MIR ? PL::nlr(l) : PL::lr(l), MIR ? PL::npre(l) : PL::pre(l)>;

// omega_{2^logn}^(+-e) from the compact table: twc[2^logn + j] = omega_{2^logn}^j
// for logn = 0 .. 13, so the roots of one size sit in consecutive lines.
template <bool INV>
__device__ __forceinline__ Tw tw_at_c(const Tw* __restrict__ twc, uint32_t e, int logn) {
    const uint32_t mask = (1u << logn) - 1u;
    const uint32_t idx = (1u << logn) | ((INV ? 0u - e : e) & mask);
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(twc) + idx);
    return Tw{u.x, u.y};
}

// dft_dif_twout factor functors. LvlTw: a level's twiddle omega_{2^LOGN}^(+-m*k2)
// from the compact table.
template <bool INV, int LOGN>
struct LvlTw {
    const Tw* twc;
    uint32_t m;
    template <int K>
    __device__ __forceinline__ Tw get() const {
        return tw_at_c<INV>(twc, m * (uint32_t)K, LOGN);
    }
};
// FacTw: a factor table's entry for output k = kb + (K << SH) of quad block cb
// (the middle factor of the block pass, a pass's post-factors).
template <int SH>
struct FacTw {
    FTab f;
    uint32_t kb, cb;
    template <int K>
    __device__ __forceinline__ Tw get() const {
        return ftab_at(f, kb + ((uint32_t)K << SH), cb);
    }
};

// A thread's quad q (of the tile's Q4) and row group t; with SF_GROUPS, half g of
// the CTA (threads g*T/2 .. ) owns quads g*Q4/2 .. (g+1)*Q4/2 - 1, each half a
// whole number of warps.
#ifndef ZB_PASS_NGROUPS
#define ZB_PASS_NGROUPS 2
#endif
template <class PL, int F>
struct PassThread {
    static constexpr bool GROUPS = (F & SF_GROUPS) != 0;
    static constexpr int NG = GROUPS ? ZB_PASS_NGROUPS : 1;
    static constexpr int GS = PL::THREADS / NG;  // threads of a barrier group
    static constexpr int GQ = PL::Q4 / NG;       // quads of a group
    static_assert(!GROUPS || (GS % 32 == 0 && GQ >= 1 && GS % GQ == 0), "halves of whole warps and quads");
    int q, t, grp;
    __device__ __forceinline__ explicit PassThread(int tid) {
        grp = GROUPS ? tid / GS : 0;
        const int l = tid - grp * GS;
        q = grp * GQ + l % GQ;
        t = l / GQ;
    }
    // the barrier between exchange writes and reads: the group's named barrier
    // (ids 1 .. NG), or the whole CTA's
    __device__ __forceinline__ void bar() const {
        if constexpr (GROUPS) group_bar(1 + grp, GS);
        else __syncthreads();
    }
};

// Levels l .. NLEV-2 of one transform, each level's twiddles folded into its last
// butterfly stage; returns with the last level's input in v. The write of level 0
// waits for the previous tile's last exchange reads.
template <class PL, int l, bool INV, bool MIR, bool PREBAR = true, class PT>
__device__ __forceinline__ void fs_levels(V4* v, uint4* sm, const PT& pt, const Tw* twc) {
    using LV = LvlOf<PL, l, MIR>;
    if constexpr (l > 0) LV::read(v, sm, pt.t, pt.q);
    if constexpr (l < PL::NLEV - 1) {
#pragma unroll
        for (int g = 0; g < LV::G; g++)
            dft_dif_twout<LV::LRADIX, INV, true>(v + g * LV::R,
                                                 LvlTw<INV, LV::LOGN>{twc, LV::n1(LV::gid(g, pt.t))});
        if constexpr (l == 0 && PREBAR) pt.bar();
        LV::write(v, sm, pt.t, pt.q);
        pt.bar();
        fs_levels<PL, l + 1, INV, MIR, true, PT>(v, sm, pt, twc);
    }
}

// The last level of a transform and the stores of its outputs, the post-factors
// (SF_POST) folded into the level's last butterfly stage.
template <class PL, bool INV, bool MIR, bool ST_KEEP, int F>
__device__ __forceinline__ void fs_last_store(V4* v, int t, const StepArgs& a, const QuadPos& p) {
    static_assert(!(F & SF_TW), "folded passes take their output twiddle as post-factors");
    using LV = LvlOf<PL, PL::NLEV - 1, MIR>;
    constexpr int LR = LV::LRADIX;
    constexpr int SH = PL::LOG_S - LR;
#pragma unroll
    for (int g = 0; g < LV::G; g++) {
        const uint32_t kb = digit_rev<PL, MIR>(LV::gid(g, t) << LR);
        if constexpr (F & SF_POST) dft_dif_twout<LR, INV, false>(v + g * LV::R, FacTw<SH>{a.post, kb, p.cb});
        else dft_dif<LR, INV>(v + g * LV::R);
#pragma unroll
        for (int r = 0; r < LV::R; r++)
            step_store<ST_KEEP, F & ~SF_POST>(v[g * LV::R + r], a, p, kb + ((uint32_t)bitrev(r, LR) << SH), nullptr,
                                              nullptr);
    }
}

// One tile of a one-transform pass: N = 2^LOG_N points per virtual quad (INV:
// inverse roots, unscaled) for the Q4 consecutive quads of tile `tile`.
// STAGED: the level-0 rows are already in sm (step_prefetch), which then also
// serves as the exchange buffer.
template <int LOG_N, bool INV, int SHAPE, bool LD_L2 = false, bool ST_KEEP = false, bool STAGED = false,
          int F = SF_ALL>
__device__ __forceinline__ void step_tile(const StepArgs& a, uint64_t tile, uint4* sm, int tid,
                                          const Tw* __restrict__ tw, const Tw* __restrict__ tw_lo) {
    using PL = typename StepShape<LOG_N, SHAPE>::PL;
    static_assert(!(F & SF_GROUPS) || ((F & SF_FOLD) && !STAGED), "groups: folded passes loading from memory");
    const PassThread<PL, F> pt(tid);
    const int q = pt.q;
    const int t = pt.t;
    V4 v[PL::EPT];
    const QuadPos p(tile * PL::Q4 + q, a);
    if constexpr (STAGED) step_consume<PL, F>(v, sm, a, p, q, t);
    else step_load<PL, LD_L2, F>(v, a, p, t);
    if constexpr (F & SF_FOLD) {
        static_assert(!(STAGED && (F & SF_NOPREBAR)), "a staged tile's buffer needs the barrier");
        fs_levels<PL, 0, INV, false, !(F & SF_NOPREBAR)>(v, sm, pt, tw);  // tw: the compact table
        fs_last_store<PL, INV, false, ST_KEEP, F>(v, t, a, p);
        return;
    }
    dif_levels<PL, 0, INV>(v, sm, t, q, tw);
    using LV = Level<PL, PL::lr(PL::NLEV - 1), PL::pre(PL::NLEV - 1)>;
#pragma unroll
    for (int g = 0; g < LV::G; g++) {
        const uint32_t blk = LV::gid(g, t);
#pragma unroll
        for (int r = 0; r < LV::R; r++) {
            const uint32_t k =
                digit_rev<PL, false>((blk << PL::lr(PL::NLEV - 1)) + (uint32_t)bitrev(r, PL::lr(PL::NLEV - 1)));
            step_store<ST_KEEP, F>(v[g * LV::R + r], a, p, k, tw, tw_lo);
        }
    }
}

// One transform of N = 2^LOG_N points per virtual quad (INV: inverse roots,
// unscaled), tiles of Q4 consecutive quads dealt round-robin.
template <int LOG_N, bool INV, int SHAPE, int F = SF_ALL>
__global__ void __launch_bounds__(StepShape<LOG_N, SHAPE>::THREADS, StepShape<LOG_N, SHAPE>::MINB)
    k_step(const StepArgs a, uint64_t ntiles, const Tw* __restrict__ tw, const Tw* __restrict__ tw_lo) {
    extern __shared__ uint4 sm[];
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
        step_tile<LOG_N, INV, SHAPE, false, false, false, F>(a, tile, sm, threadIdx.x, tw, tw_lo);
}

// The second transform's levels 1 .. NLEV-1 (mirrored radices, as ntt_levels in
// extend.cuh, with either root direction); the last level stores every output.
template <class PL, int l, bool INV2, bool ST_KEEP = false, int F = SF_ALL>
__device__ __forceinline__ void step2_levels(V4* v, uint4* sm, int t, int q, const Tw* tw, const Tw* tw_lo,
                                             const StepArgs& a, const QuadPos& p) {
    using LV = Level<PL, PL::nlr(l), PL::npre(l)>;
    if constexpr (l > 0) LV::read(v, sm, t, q);
    LV::template dft<INV2>(v);
    if constexpr (l < PL::NLEV - 1) {
        LV::template twiddle_write<INV2>(v, sm, t, q, tw);
        __syncthreads();
        step2_levels<PL, l + 1, INV2, ST_KEEP, F>(v, sm, t, q, tw, tw_lo, a, p);
    } else {
#pragma unroll
        for (int g = 0; g < LV::G; g++) {
            const uint32_t blk = LV::gid(g, t);
#pragma unroll
            for (int r = 0; r < LV::R; r++) {
                const uint32_t k = digit_rev<PL, true>((blk << PL::nlr(l)) + (uint32_t)bitrev(r, PL::nlr(l)));
                step_store<ST_KEEP, F>(v[g * LV::R + r], a, p, k, tw, tw_lo);
            }
        }
    }
}

// One tile of a two-transform pass: out = T2( mid(k) * T1(pre * in)(k) ) over
// N = 2^LOG_N points per virtual quad, T1 with roots w^-1 when INV1, T2 with w^-1
// when INV2, both unscaled. mid(k, cb) = mid1(k, cb) * mid2(k, cb). With a
// counter, the nonzero outputs k >= count_from of T1 (before mid) are added to
// cnt (the decoder's consistency check).
template <int LOG_N, bool INV1, bool INV2, int SHAPE, bool LD_L2 = false, bool ST_KEEP = false,
          bool STAGED = false, int F = SF_ALL>
__device__ __forceinline__ void step2_tile(const StepArgs& a, uint64_t tile, uint4* sm, int tid,
                                           const Tw* __restrict__ tw, const Tw* __restrict__ tw_lo,
                                           unsigned long long& cnt) {
    using PL = typename StepShape<LOG_N, SHAPE>::PL;
    static_assert(!(F & SF_GROUPS) || ((F & SF_FOLD) && !STAGED), "groups: folded passes loading from memory");
    const PassThread<PL, F> pt(tid);
    const int q = pt.q;
    const int t = pt.t;
    V4 v[PL::EPT];
    const QuadPos p(tile * PL::Q4 + q, a);
    if constexpr (STAGED) step_consume<PL, F>(v, sm, a, p, q, t);
    else step_load<PL, LD_L2, F>(v, a, p, t);
    if constexpr (F & SF_FOLD) {
        static_assert(!(F & SF_CNT), "the count reads T1's outputs before the middle factor");
        static_assert(PL::NLEV > 1, "T2 exchanges after its first level");
        static_assert(!(STAGED && (F & SF_NOPREBAR)), "a staged tile's buffer needs the barrier");
        fs_levels<PL, 0, INV1, false, !(F & SF_NOPREBAR)>(v, sm, pt, tw);
        constexpr int LR = PL::lr(PL::NLEV - 1);
        constexpr int R = 1 << LR;
        constexpr int G = PL::EPT / R;
        constexpr int SH = PL::LOG_S - LR;
        uint32_t c0[G];
#pragma unroll
        for (int g = 0; g < G; g++) {
            c0[g] = digit_rev<PL, false>((uint32_t)(g * PL::TPQ + t) << LR);
            // T1's last level with the middle factor of output c0 + (S/R) k2 folded in
            if constexpr (F & SF_MID) dft_dif_twout<LR, INV1, false>(v + g * R, FacTw<SH>{a.mid1, c0[g], p.cb});
            else dft_dif<LR, INV1>(v + g * R);
            V4 y[R];
#pragma unroll
            for (int j = 0; j < R; j++) y[j] = v[g * R + bitrev(j, LR)];
            // T2 level 0 (radix R over stride S/R, group n1 = c0) with its twiddles
            dft_dif_twout<LR, INV2, true>(y, LvlTw<INV2, PL::LOG_S>{tw, c0[g]});  // tw: compact
#pragma unroll
            for (int j = 0; j < R; j++) v[g * R + j] = y[j];
        }
        pt.bar();  // every thread (of the group) finished reading T1's last level
#pragma unroll
        for (int g = 0; g < G; g++)
#pragma unroll
            for (int r = 0; r < R; r++) {
                const V4& x = v[g * R + r];
                sm[(size_t)(c0[g] + ((uint32_t)bitrev(r, LR) << SH)) * PL::Q4 + q] =
                    make_uint4(x.c[0], x.c[1], x.c[2], x.c[3]);
            }
        pt.bar();
        fs_levels<PL, 1, INV2, true, true>(v, sm, pt, tw);
        fs_last_store<PL, INV2, true, ST_KEEP, F>(v, t, a, p);
        return;
    }
    dif_levels<PL, 0, INV1>(v, sm, t, q, tw);
    // T1's last level: group g (block b = g*TPQ + t) holds outputs c0 + (S/R)*j at
    // v[g*R + bitrev(j)]; T2's first level (radix R over stride S/R) wants them in
    // natural j order as its group n1 = c0, so no exchange sits between the two.
    constexpr int LR = PL::lr(PL::NLEV - 1);
    constexpr int R = 1 << LR;
    constexpr int G = PL::EPT / R;
    constexpr int SH = PL::LOG_S - LR;
    uint32_t c0[G];
#pragma unroll
    for (int g = 0; g < G; g++) {
        const uint32_t b = (uint32_t)(g * PL::TPQ + t);
        c0[g] = digit_rev<PL, false>(b << LR);
        V4 y[R];
#pragma unroll
        for (int j = 0; j < R; j++) {
            y[j] = v[g * R + bitrev(j, LR)];
            const uint32_t k = c0[g] + ((uint32_t)j << SH);
            if ((F & SF_CNT) && a.counter && p.active && k >= a.count_from)
#pragma unroll
                for (int e = 0; e < 4; e++) cnt += y[j].c[e] != 0;
            if ((F & SF_MID) && a.mid1.tab) mul4(y[j], ftab_at(a.mid1, k, p.cb));
            if ((F & SF_MID) && a.mid2.tab) mul4(y[j], ftab_at(a.mid2, k, p.cb));
        }
#pragma unroll
        for (int j = 0; j < R; j++) v[g * R + j] = y[j];
    }
    // T2 level 0: radix R over stride S/R, one block; group n1 = c0
#pragma unroll
    for (int g = 0; g < G; g++) dft_dif<LR, INV2>(v + g * R);
    if constexpr (PL::NLEV > 1) {
        __syncthreads();  // every thread finished reading T1's last level
#pragma unroll
        for (int g = 0; g < G; g++) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int k2 = bitrev(r, LR);
                V4 x = v[g * R + r];
                if (k2 != 0) mul4(x, tw_at<INV2>(tw, c0[g] * (uint32_t)k2, PL::LOG_S));
                sm[(size_t)(c0[g] + ((uint32_t)k2 << SH)) * PL::Q4 + q] =
                    make_uint4(x.c[0], x.c[1], x.c[2], x.c[3]);
            }
        }
        __syncthreads();
        step2_levels<PL, 1, INV2, ST_KEEP, F>(v, sm, t, q, tw, tw_lo, a, p);
    } else {
#pragma unroll
        for (int r = 0; r < R; r++) step_store<ST_KEEP, F>(v[r], a, p, (uint32_t)bitrev(r, LR), tw, tw_lo);
    }
}

// Two transforms per virtual quad with a factor between them (step2_tile), tiles
// of Q4 consecutive quads dealt round-robin.
template <int LOG_N, bool INV1, bool INV2, int SHAPE, int F = SF_ALL>
__global__ void __launch_bounds__(StepShape<LOG_N, SHAPE>::THREADS, StepShape<LOG_N, SHAPE>::MINB)
    k_step2(const StepArgs a, uint64_t ntiles, const Tw* __restrict__ tw, const Tw* __restrict__ tw_lo) {
    extern __shared__ uint4 sm[];
    const int tid = threadIdx.x;
    unsigned long long cnt = 0;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
        step2_tile<LOG_N, INV1, INV2, SHAPE, false, false, false, F>(a, tile, sm, tid, tw, tw_lo, cnt);
    if ((F & SF_CNT) && a.counter) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, o);
        if ((tid & 31) == 0 && cnt) atomicAdd(a.counter, cnt);
    }
}

// One pass (TWO: two transforms, T1 inverse when INV, T2 the other direction; else
// one transform) with the next tile's rows copied in by cp.async while the
// current tile computes. Shared memory holds two tiles; the current one is also
// the exchange buffer, so a barrier at the top of each tile keeps the copies into
// the other stage behind the previous tile's last exchange reads.
template <int LOG_N, bool INV, bool TWO, int SHAPE, int F = SF_ALL>
__global__ void __launch_bounds__(StepShape<LOG_N, SHAPE>::THREADS, StepShape<LOG_N, SHAPE>::MINB_ST)
    k_step_st(const StepArgs a, uint64_t ntiles, const Tw* __restrict__ tw, const Tw* __restrict__ tw_lo) {
    using PL = typename StepShape<LOG_N, SHAPE>::PL;
    static_assert(PL::SMEM > 0, "staged passes exchange through the stage");
    extern __shared__ uint4 sm[];
    constexpr size_t STG = PL::SMEM / sizeof(uint4);
    const int tid = threadIdx.x;
    const int q = tid % PL::Q4;
    const int t = tid / PL::Q4;
    unsigned long long cnt = 0;
    uint64_t tile = blockIdx.x;
    if (tile < ntiles) step_prefetch<PL, F>(sm, a, tile, q, t);
    cp_async_commit();
    for (int i = 0; tile < ntiles; tile += gridDim.x, i ^= 1) {
        __syncthreads();  // the previous tile's exchange reads of the other stage are done
        const uint64_t next = tile + gridDim.x;
        if (next < ntiles) step_prefetch<PL, F>(sm + (i ^ 1) * STG, a, next, q, t);
        cp_async_commit();
        cp_async_wait<1>();  // this thread's rows of the current tile have landed
        uint4* cur = sm + i * STG;
        if constexpr (TWO)
            step2_tile<LOG_N, INV, !INV, SHAPE, false, false, true, F>(a, tile, cur, tid, tw, tw_lo, cnt);
        else
            step_tile<LOG_N, INV, SHAPE, false, false, true, F>(a, tile, cur, tid, tw, tw_lo);
    }
    cp_async_wait<0>();
    if (TWO && (F & SF_CNT) && a.counter) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xFFFFFFFFu, cnt, o);
        if ((tid & 31) == 0 && cnt) atomicAdd(a.counter, cnt);
    }
}

// ---- the extension's three passes in one persistent launch, chunk by chunk ----
// The three passes of a square's extension (strided INTT pass A, block pass,
// strided NTT pass B) each read and write a whole matrix. Run one after the
// other over the square, every intermediate goes to HBM and back: 56 bytes per
// input element at side 4096 against the 12 the extension must move. Here the
// columns are cut into chunks of CQ quads, and one persistent launch runs the
// passes chunk by chunk, a few chunks apart, so a chunk's intermediate (its odd
// output rows) is still in L2 when the next pass reads it.
//
// Work items are the tiles of (chunk, pass). Round r holds, in this order, the
// tiles of pass A of chunk r, of the block pass of chunk r - depth and of pass B
// of chunk r - 2*depth (chunks out of range are empty items); a global counter
// deals items in that order. The block pass of a chunk waits until all its pass-A
// tiles are done (a per-chunk counter), pass B until all its block tiles are. An
// item waits only on items dealt before it, to CTAs that are running them, so
// the launch cannot deadlock whatever the number of resident CTAs. Each wait is
// bounded; on expiry the CTA flags the error (bit 4) and leaves.
//
// Matrices a pass reads after another CTA of the launch wrote them are loaded
// through L2 only (an SM's L1 may hold a stale copy of a line); intermediates
// are stored with the normal L2 policy, streamed data (the input, the even rows,
// the final odd rows) with evict-first.
struct PipeArgs {
    StepArgs pass[3];    // chunk 0's views; qpc = CQ, nquads = blocks * CQ
    uint64_t chunk_u32;  // u32 from one chunk's first column to the next chunk's
    uint32_t nchunks;
    uint32_t last_qlim;  // real quads in the last chunk
    uint32_t tiles[3];   // work items per chunk of each pass
    uint32_t tpi;        // tiles per work item (1 in the staged form)
    uint32_t wait_extra; // added to every dependency count a work item waits for (fault injection: 1)
    uint32_t depth;      // rounds between a chunk's passes
    uint32_t* counters;  // [0] item counter; [1 + c] pass-A tiles done; [1 + nchunks + c] block tiles done
    int* err;
};

constexpr uint32_t PIPE_WAIT_POLLS = 1u << 21;  // about a second of polling

__device__ __forceinline__ bool pipe_wait_count(const uint32_t* p, uint32_t need) {
    for (uint32_t i = 0; i < PIPE_WAIT_POLLS; i++) {
        uint32_t v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= need) return true;
        __nanosleep(64);
    }
    return false;
}

// Chunk c's view of pass PH.
template <int PH>
__device__ __forceinline__ StepArgs pipe_args(const PipeArgs& pa, uint32_t c) {
    StepArgs x = pa.pass[PH];
    const uint64_t off = (uint64_t)c * pa.chunk_u32;
    x.in.base += off;
    x.out.base += off;
    if (x.copy.base) x.copy.base += off;
    if (c + 1 == pa.nchunks) x.qlim = pa.last_qlim;
    return x;
}

// STAGED0: pass-A tiles arrive staged in sm (step_prefetch); the other passes read
// what this launch wrote straight from L2.
template <int PH, int L1, int L2, int SHAPE, bool STAGED0>
__device__ __forceinline__ void pipe_pass(const PipeArgs& pa, uint32_t c, uint32_t tile, uint4* sm, int tid,
                                          const Tw* __restrict__ tw, const Tw* __restrict__ tw_lo) {
    const StepArgs x = pipe_args<PH>(pa, c);
    if constexpr (PH == 0) {
        step_tile<L1, true, SHAPE, false, true, STAGED0,
                  STAGED0 ? SF_EXT_A : (SF_EXT_A | SF_NOPREBAR | SF_PASS_GROUPS)>(x, tile, sm, tid, tw, tw_lo);
    } else if constexpr (PH == 1) {
        unsigned long long cnt = 0;
        step2_tile<L2, true, false, SHAPE, true, true, false, SF_EXT_M | SF_NOPREBAR | SF_PASS_GROUPS>(
            x, tile, sm, tid, tw, tw_lo, cnt);
    } else {
        step_tile<L1, false, SHAPE, true, false, false, SF_EXT_B | SF_NOPREBAR | SF_PASS_GROUPS>(x, tile, sm, tid,
                                                                                              tw, tw_lo);
    }
}

template <int L1, int L2, int SHAPE>
struct PipeShape {
    using A = StepShape<L1, SHAPE>;
    using M = StepShape<L2, SHAPE>;
    static_assert(A::THREADS == M::THREADS && A::MINB == M::MINB, "one CTA shape for all passes");
    static constexpr int THREADS = A::THREADS, MINB = A::MINB;
    static constexpr size_t SMEM = A::PL::SMEM > M::PL::SMEM ? A::PL::SMEM : M::PL::SMEM;
    static constexpr uint32_t CQ = A::PL::Q4 > M::PL::Q4 ? A::PL::Q4 : M::PL::Q4;  // quads per chunk
    // staged: two tile buffers
    static constexpr int MINB_ST_FIT = (int)(232448 / (2 * SMEM));
    static constexpr int MINB_ST = MINB_ST_FIT < MINB ? MINB_ST_FIT : MINB;
};

// An item's pass, chunk (-1 or past the last: an empty item) and tile in the chunk.
struct PipeItem {
    int ph;
    int64_t c;
    uint32_t j;
};
__device__ __forceinline__ PipeItem pipe_decode(const PipeArgs& pa, uint32_t item, uint32_t per_round) {
    const uint32_t r = item / per_round;
    uint32_t j = item - r * per_round;
    if (j < pa.tiles[0]) return PipeItem{0, (int64_t)r, j};
    j -= pa.tiles[0];
    if (j < pa.tiles[1]) return PipeItem{1, (int64_t)r - pa.depth, j};
    return PipeItem{2, (int64_t)r - 2 * (int64_t)pa.depth, j - pa.tiles[1]};
}

// STAGE: two tile buffers; every CTA knows its next item one tile ahead, and when
// that item is a pass-A tile (no dependencies) its rows are copied in by cp.async
// while the current item computes. Items alternate buffers; the barrier at the top
// of each item keeps the copies behind the previous item's last reads.
template <int L1, int L2, int SHAPE, bool STAGE>
__global__ void __launch_bounds__(PipeShape<L1, L2, SHAPE>::THREADS,
                                  STAGE ? PipeShape<L1, L2, SHAPE>::MINB_ST : PipeShape<L1, L2, SHAPE>::MINB)
    k_fourstep_pipe(const __grid_constant__ PipeArgs pa, const Tw* __restrict__ tw, const Tw* __restrict__ tw_lo) {
    using PS = PipeShape<L1, L2, SHAPE>;
    using PLA = typename PS::A::PL;
    constexpr size_t BUF = PS::SMEM / sizeof(uint4);
    extern __shared__ uint4 sm[];
    __shared__ uint32_t s_item, s_next[2];  // s_next: a ring, so one barrier per item covers its reads
    __shared__ int s_fail;
    const int tid = threadIdx.x;
    const uint32_t per_round = pa.tiles[0] + pa.tiles[1] + pa.tiles[2];
    const uint32_t total = (pa.nchunks + 2 * pa.depth) * per_round;  // the host keeps this below 2^31
    auto prefetch_a = [&](uint32_t it, uint4* buf) {  // the rows of a pass-A item, if it is one
        if (it >= total) return;
        const PipeItem pi = pipe_decode(pa, it, per_round);
        if (pi.ph == 0 && pi.c < (int64_t)pa.nchunks)
            step_prefetch<PLA, SF_EXT_A>(buf, pipe_args<0>(pa, (uint32_t)pi.c), pi.j, tid % PLA::Q4, tid / PLA::Q4);
    };
    if (tid == 0) {
        s_item = atomicAdd(pa.counters, 1u);
        s_next[0] = atomicAdd(pa.counters, 1u);
        s_fail = 0;
    }
    __syncthreads();
    uint32_t item = s_item, next = s_next[0];
    int b = 0;
    if constexpr (STAGE) {
        prefetch_a(item, sm);
        cp_async_commit();
    }
    // Every item ends with one barrier: the item's tile is stored (and, before a
    // pass-A or block tile is counted, fenced by thread 0: the fence is cumulative
    // over the stores the barrier ordered before it), its shared memory reads are
    // done, and s_next is published. The next item's first shared-memory write,
    // or a copy into the other buffer, comes after that barrier.
    for (uint32_t it = 0; item < total; it++) {
        uint32_t nn = 0;
        if (tid == 0) nn = atomicAdd(pa.counters, 1u);  // the item after next, used after this tile
        uint4* buf = sm;
        if constexpr (STAGE) {
            buf = sm + b * BUF;
            prefetch_a(next, sm + (b ^ 1) * BUF);
            cp_async_commit();
        }
        const PipeItem pi = pipe_decode(pa, item, per_round);
        if (pi.c >= 0 && pi.c < (int64_t)pa.nchunks) {
            const uint32_t cc = (uint32_t)pi.c;
            if (pi.ph > 0) {
                if (tid == 0) {
                    const uint32_t* done = pa.counters + 1 + (pi.ph == 1 ? 0u : pa.nchunks) + cc;
                    if (!pipe_wait_count(done, pa.tiles[pi.ph - 1] + pa.wait_extra)) {
                        s_fail = 1;
                        atomicOr(pa.err, 4);
                    }
                    __threadfence();
                }
                __syncthreads();
                if (s_fail) {
                    if constexpr (STAGE) cp_async_wait<0>();
                    return;
                }
            }
            // the item's tiles in turn; a barrier between two of them orders the first
            // one's last exchange reads before the next one's first exchange write
            for (uint32_t u = 0; u < pa.tpi; u++) {
                const uint32_t tile = pi.j * pa.tpi + u;
                if (u) __syncthreads();
                if (pi.ph == 0) {
                    if constexpr (STAGE) cp_async_wait<1>();  // this item's rows (the newest group is the next item's)
                    pipe_pass<0, L1, L2, SHAPE, STAGE>(pa, cc, tile, buf, tid, tw, tw_lo);
                } else if (pi.ph == 1) {
                    pipe_pass<1, L1, L2, SHAPE, STAGE>(pa, cc, tile, buf, tid, tw, tw_lo);
                } else {
                    pipe_pass<2, L1, L2, SHAPE, STAGE>(pa, cc, tile, buf, tid, tw, tw_lo);
                }
            }
        }
        if (tid == 0) s_next[(it + 1) & 1] = nn;
        __syncthreads();
        if (tid == 0 && pi.ph < 2 && pi.c >= 0 && pi.c < (int64_t)pa.nchunks) {
            __threadfence();  // every thread's stores of the tile (ordered by the barrier), before the count
            atomicAdd(pa.counters + 1 + (pi.ph == 0 ? 0u : pa.nchunks) + (uint32_t)pi.c, 1u);
        }
        item = next;
        next = s_next[(it + 1) & 1];
        b ^= 1;
    }
    if constexpr (STAGE) cp_async_wait<0>();
}

}  // namespace zb
