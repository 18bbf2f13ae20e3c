"""CPU restatements of the arithmetic the device kernels rely on, checked with
exact Python integers: the RLC kernels' centered residues, signed 64-bit sums
and folds (csrc/rlc.cu), the identities behind the decoder's two fused passes
(csrc/general.cu, k_coltx2 in csrc/coltx.cuh), and the split of the TMA-staged
passes' middle factor into block and digit tables (k_dec_tma in
csrc/extend_tma.cuh, the tables in csrc/general.cu). No GPU needed."""
import numpy as np
import pytest

import oracle as O

P = O.P
H = (P - 1) // 2
TWO32_MOD_P = (1 << 32) - 2 * P  # 2^28 - 2
P_SHIFT29 = P << 29
I64_MIN, I64_MAX = -(1 << 63), (1 << 63) - 1


def reduce_2p(v: int) -> int:
    """min(v - p, v) over u32 (one subtract-min)."""
    return min((v - P) & 0xFFFFFFFF, v)


def centered_any(v: int) -> int:
    r = reduce_2p(v)
    return r - P if r > H else r


def sfold(a: int) -> int:
    h = a >> 32  # floor
    return (h << 28) - (h << 1) + (a & 0xFFFFFFFF)


def fold32(a: int) -> int:
    return (a >> 32) * TWO32_MOD_P + (a & 0xFFFFFFFF)


def test_fold_constants():
    assert TWO32_MOD_P == (1 << 28) - 2 == (1 << 32) % P
    assert P_SHIFT29 % P == 0


@pytest.mark.parametrize("v", [0, 1, H, H + 1, P - 1, P, P + H, P + H + 1, 2 * P - 1, 2 * P, (1 << 32) - 1])
def test_centered_any_edges(v):
    c = centered_any(v)
    assert (c - v) % P == 0 and -H <= c <= H


def test_centered_any_random():
    rng = np.random.default_rng(5)
    for v in rng.integers(0, 1 << 32, size=20000, dtype=np.uint64):
        c = centered_any(int(v))
        assert (c - int(v)) % P == 0 and -H <= c <= H


def test_sfold_range_and_residue():
    rng = np.random.default_rng(6)
    samples = [I64_MIN, I64_MAX, 0, -1, 1 << 62, -(1 << 62)] + [int(x) for x in rng.integers(I64_MIN, I64_MAX, 5000)]
    for a in samples:
        f = sfold(a)
        assert (f - a) % P == 0
        assert -(1 << 59) < f < (1 << 59) + (1 << 32)


def emulate_row_sum(xs, cs, products_per_fold=8):
    """One limb of one row as the kernels sum it: centered products added to a
    signed sum, folded after every `products_per_fold` products; asserts the
    signed 64-bit range at every step. Returns the residue the flush produces."""
    s = 0
    for i, (x, c) in enumerate(zip(xs, cs)):
        s += centered_any(x) * c
        assert I64_MIN <= s <= I64_MAX
        if (i + 1) % products_per_fold == 0:
            s = sfold(s)
    s = sfold(s)
    u = s + P_SHIFT29
    assert 0 <= u < (1 << 64)
    return u % P


@pytest.mark.parametrize("xv,cv", [(H, H), (H + 1, H + 1), (H, H + 1), (P - 1, P - 1), ((1 << 32) - 1, H + 1)])
def test_row_sum_worst_cases(xv, cv):
    """Every value and coefficient at the extremes of the centered range: the
    partial sums run at their bound for 4096 columns."""
    n = 4096
    c = centered_any(cv % P)
    got = emulate_row_sum([xv] * n, [c] * n)
    assert got == n * (xv % P) * (cv % P) % P


def test_row_sum_random_matches_oracle():
    rng = np.random.default_rng(7)
    n = 2000
    xs = [int(v) for v in rng.integers(0, 1 << 32, size=n, dtype=np.uint64)]
    coeff = rng.integers(0, P, size=(n, 4), dtype=np.uint64)
    want = O.rlc_rows(np.array(xs, dtype=np.uint64)[None, :], coeff)[0]
    for limb in range(4):
        cs = [centered_any(int(c)) for c in coeff[:, limb]]
        assert emulate_row_sum(xs, cs) == int(want[limb])


def test_nine_products_could_overflow():
    """Eight products per fold is the most the signed word allows."""
    worst = (1 << 59) + (1 << 32) + 8 * H * H
    assert worst <= I64_MAX
    assert (1 << 59) + 9 * H * H > I64_MAX


def test_warp_reduction_bounds():
    """The few-rows kernel's reduction: a folded sum + p*2^29 folded once is
    below 2^57, so 32 lanes sum below 2^62; a warp total folded again keeps
    8 warps below 2^62."""
    top = (1 << 59) + (1 << 32) + P_SHIFT29
    lane = fold32(top)
    assert lane < (1 << 57) and 32 * lane < (1 << 62)
    warp = fold32(32 * ((1 << 57) - 1))
    assert 8 * warp < (1 << 62)


# ---- decoder identities ---------------------------------------------------------

def modpow(b, e):
    return pow(int(b), int(e), P)


def test_k_point_ntt_is_even_outputs_of_padded_2k():
    rng = np.random.default_rng(8)
    for k in (1, 2, 8, 64):
        a = rng.integers(0, P, size=k, dtype=np.uint64).astype(np.uint32)
        padded = np.concatenate([a, np.zeros(k, dtype=np.uint32)])
        assert np.array_equal(O.ntt(a) if k > 1 else a, O.ntt(padded)[0::2])


def decoder_fused_passes(rows: np.ndarray, known, k: int):
    """The two fused passes on one column, with the kernel's tables: the INTT is
    unscaled and the middle tables carry 1/N."""
    N = 2 * k
    w = int(O.roots_of_unity(N)[1])
    hgen = 31
    pts = [modpow(w, j) for j in range(N)]
    erased = [j for j in range(N) if j not in set(known)]
    zk = [0] * N
    izh = [0] * N
    for j in range(N):
        z = 1
        zh = 1
        for e in erased:
            z = z * (pts[j] - pts[e]) % P
            zh = zh * (hgen * pts[j] - pts[e]) % P
        zk[j] = z if j in set(known) else 0
        izh[j] = modpow(zh, P - 2)
    ninv = modpow(N, P - 2)
    mid_a = [modpow(hgen, i) * ninv % P for i in range(N)]
    mid_b = [modpow(modpow(hgen, i), P - 2) * ninv % P if i < k else 0 for i in range(N)]

    def unscaled_intt(v):
        return (O.intt(np.array(v, dtype=np.uint32)).astype(np.uint64) * N % P).astype(np.uint32)

    y = [int(rows[j]) if j in set(known) else 0 for j in range(N)]
    a1 = unscaled_intt([y[j] * zk[j] % P for j in range(N)])
    b = O.ntt(np.array([int(a1[i]) * mid_a[i] % P for i in range(N)], dtype=np.uint32))
    a2 = unscaled_intt([int(b[j]) * izh[j] % P for j in range(N)])
    high_nonzero = int(np.count_nonzero(a2[k:]))
    out = O.ntt(np.array([int(a2[i]) * mid_b[i] % P for i in range(N)], dtype=np.uint32))
    return out[0::2][:k], high_nonzero


@pytest.mark.parametrize("k", [2, 4, 16])
def test_decoder_fused_passes_recover_the_data(k):
    rng = np.random.default_rng(10 + k)
    data = rng.integers(0, P, size=(k, 1), dtype=np.uint64).astype(np.uint32)
    code = O.encode_rowmajor(data)  # [2k][1], interleaved
    known = sorted(rng.choice(2 * k, size=k, replace=False).tolist())
    got, high = decoder_fused_passes(code[:, 0], known, k)
    assert np.array_equal(got, data[:, 0])
    assert high == 0  # (with exactly k known rows any values are one codeword)


@pytest.mark.parametrize("k", [4, 16])
def test_decoder_check_catches_a_corrupted_row(k):
    rng = np.random.default_rng(20 + k)
    data = rng.integers(0, P, size=(k, 1), dtype=np.uint64).astype(np.uint32)
    code = O.encode_rowmajor(data)
    known = sorted(rng.choice(2 * k, size=k + 2, replace=False).tolist())  # redundancy to detect with
    bad = code[:, 0].copy()
    bad[known[1]] = (int(bad[known[1]]) + 12345) % P
    _, high = decoder_fused_passes(bad, known, k)
    assert high > 0
    _, high_ok = decoder_fused_passes(code[:, 0], known, k)
    assert high_ok == 0


# ---- the TMA-staged passes' factor split --------------------------------------------

def last_c0(ls: int, lept: int):
    """c0 of every INTT last-level block (SideLevels::last_c0 in internal.hpp)."""
    nlev = (ls + lept - 1) // lept
    lr = lambda l: lept if l < nlev - 1 else ls - lept * (nlev - 1)
    LR = lr(nlev - 1)
    out = []
    for b in range((1 << ls) >> LR):
        slot, c0, sh_in, sh_out = b << LR, 0, ls, 0
        for l in range(nlev):
            sh_in -= lr(l)
            c0 |= ((slot >> sh_in) & ((1 << lr(l)) - 1)) << sh_out
            sh_out += lr(l)
        out.append(c0)
    return out, 1 << LR


def dec_lept(ls: int) -> int:  # the radix rule of general.cu
    return 3 if ls in (9, 11) else 4


@pytest.mark.parametrize("ls", [7, 8, 9, 10, 11, 12])
def test_middle_factor_splits_into_block_and_digit_parts(ls):
    """mid(c0 + (S/R) k2) = block(c0) * digit(k2) for the decoder's two passes and
    for an encode coset, over every coefficient index exactly once."""
    S = 1 << ls
    c0s, R = last_c0(ls, dec_lept(ls))
    step = S // R
    idx = sorted(c0 + step * k2 for c0 in c0s for k2 in range(R))
    assert idx == list(range(S)) and max(c0s) < S // R
    sinv = modpow(S, P - 2)
    h, hinv = 31, modpow(31, P - 2)
    w = int(O.roots_of_unity(4 * S)[1])  # coset c = 1 of n_kn = 4 n_k
    for c0 in c0s[:: max(1, len(c0s) // 64)]:
        for k2 in range(R):
            i = c0 + step * k2
            # pass A: h^i / S
            assert modpow(h, c0) * sinv * modpow(h, step * k2) % P == modpow(h, i) * sinv % P
            # pass B: h^-i / S for i < S/2, else 0 (the digit factor is 0 for k2 >= R/2)
            digit_b = modpow(hinv, step * k2) if k2 < R // 2 else 0
            want_b = modpow(hinv, i) * sinv % P if i < S // 2 else 0
            assert modpow(hinv, c0) * sinv * digit_b % P == want_b
            # encode coset: omega_{4S}^i / S
            assert modpow(w, c0) * sinv * modpow(w, step * k2) % P == modpow(w, i) * sinv % P
