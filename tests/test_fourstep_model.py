"""CPU model of the long-column (four-step) passes, checked against the oracle.

The model restates what every k_step / k_step2 launch of csrc/fourstep.cu does
to memory, with the same matrix views (row pitch, column-block pitch, quads
per block), factor tables (f(r, cb) = tab[r*rm + cb*cm]), two-dimensional
twiddles omega_S^(+-cb*k), input limits and output cuts, and the same pass
sequences and table formulas as long_cols_ntt, long_extend, long_encode and
long_recover. Each transform in the model is the oracle's NTT (the reference's
src/ntt/cpu.rs restated), so a wrong view, table, twiddle sign or pass order
shows here, on the CPU, before the kernels run on a GPU."""
import numpy as np
import pytest

import oracle as O

P = O.P


def powtab(w: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint64)
    x = 1
    for i in range(n):
        out[i] = x
        x = x * w % P
    return out


def root(log_n: int) -> int:
    return pow(31, (P - 1) >> log_n, P)


class View:
    def __init__(self, buf: np.ndarray, base: int, row_pitch: int, cb_pitch: int):
        self.buf, self.base, self.rp, self.cp = buf, base, row_pitch, cb_pitch


def addr(view: View, rows, cb, ci):
    return view.base + cb * view.cp + ci + rows * view.rp


def dft_cols(x: np.ndarray, inv: bool) -> np.ndarray:
    """Unscaled DFT of every column of x [N][V] (natural order in and out)."""
    n, v = x.shape
    flat = np.ascontiguousarray(x.T.astype(np.uint32)).ravel()
    y = O.ntt_polys(flat, n, n, inverse=inv).reshape(v, n).T.astype(np.uint64)
    return y * n % P if inv else y


def model_pass(a: dict):
    """One k_step (a['two'] False) or k_step2 launch. Keys: N (points), inv (T1), in, out
    (Views), qpc, nquads, pre / mid1 / mid2 / post ((tab, rm, cm) or None), tw ((log, inv) or
    None), scale, in_lim / out_lim ((rm, cm, limit) or None), copy (View or None),
    count_from (int or None; returns the count)."""
    N, qpc, nq = a["N"], a["qpc"], a["nquads"]
    # a["quads"] = (q0, q1): only virtual quads q0 .. q1-1 (one tile); a["qlim"]: quads
    # at or past it inside a column block are not real (the pipeline's ragged last chunk)
    q0, q1 = a.get("quads", (0, nq))
    v = np.arange(q0 * 4, min(q1, nq) * 4)
    cb, ci = (v // 4) // qpc, (v // 4) % qpc * 4 + v % 4
    if a.get("qlim") is not None:
        keep = (v // 4) % qpc < a["qlim"]
        v, cb, ci = v[keep], cb[keep], ci[keep]
    r = np.arange(N)[:, None]
    ia = addr(a["in"], r, cb[None, :], ci[None, :])
    ld = np.ones((N, len(v)), dtype=bool)
    if a.get("in_lim"):
        rm, cm, lim = a["in_lim"]
        ld &= (r * rm + cb[None, :] * cm) < lim
    x = np.zeros((N, len(v)), dtype=np.uint64)
    x[ld] = a["in"].buf[ia[ld]]
    if a.get("copy") is not None:
        ca = addr(a["copy"], r, cb[None, :], ci[None, :])
        a["copy"].buf[ca[ld]] = x[ld]
    if a.get("pre"):
        tab, rm, cm = a["pre"]
        x = x * tab[r * rm + cb[None, :] * cm] % P
    x = dft_cols(x, a["inv"])
    cnt = 0
    if a.get("two"):
        k = np.arange(N)[:, None]
        if a.get("count_from") is not None:
            cnt = int(np.count_nonzero(x[a["count_from"]:]))
        for key in ("mid1", "mid2"):
            if a.get(key):
                tab, rm, cm = a[key]
                x = x * tab[k * rm + cb[None, :] * cm] % P
        x = dft_cols(x, not a["inv"])
    k = np.arange(N)[:, None]
    st = np.ones((N, len(v)), dtype=bool)
    if a.get("out_lim"):
        rm, cm, lim = a["out_lim"]
        st &= (k * rm + cb[None, :] * cm) < lim
    if a.get("post"):
        tab, rm, cm = a["post"]
        x = x * tab[k * rm + cb[None, :] * cm] % P
    if a.get("tw"):
        log, tinv = a["tw"]
        S = 1 << log
        e = (cb[None, :] * k) % S
        if tinv:
            e = (S - e) % S
        x = x * powtab(root(log), S)[e] % P
    if a.get("scale") is not None:
        x = x * a["scale"] % P
    oa = addr(a["out"], k, cb[None, :], ci[None, :])
    a["out"].buf[oa[st]] = x[st]
    return cnt


def split(L):
    L1 = L // 2
    return L1, L - L1, 1 << L1, 1 << (L - L1)


def coset_mid_tables(L, ln):
    """fourstep.cu coset_mid_tables: per coset c >= 1, [k1: base^k1 / n_k] then [k2: base^(N1 k2)]."""
    L1, L2, N1, N2 = split(L)
    sinv, wn = pow(1 << L, P - 2, P), root(ln)
    out = []
    for c in range(1, 1 << (ln - L)):
        base = pow(wn, c, P)
        out.append((powtab(base, N1) * sinv % P, powtab(pow(base, N1, P), N2)))
    return out


def model_extend(data: np.ndarray) -> np.ndarray:
    """long_extend: in [S][cols] -> out [2S][cols], odd rows as the scratch."""
    S, cols = data.shape
    L = S.bit_length() - 1
    L1, L2, N1, N2 = split(L)
    qpc = cols // 4
    inp = data.astype(np.uint64).ravel()
    out = np.full(2 * S * cols, 12345, dtype=np.uint64)  # garbage the passes must overwrite
    cbt, kt = coset_mid_tables(L, L + 1)[0]
    model_pass(dict(N=N1, inv=True, **{"in": View(inp, 0, N2 * cols, cols)},
                    out=View(out, cols, 2 * N2 * cols, 2 * cols), qpc=qpc, nquads=N2 * qpc, tw=(L, 1),
                    copy=View(out, 0, 2 * N2 * cols, 2 * cols)))
    blk = View(out, cols, 2 * cols, 2 * N2 * cols)
    model_pass(dict(N=N2, inv=True, two=True, **{"in": blk}, out=blk, qpc=qpc, nquads=N1 * qpc,
                    mid1=(cbt, 0, 1), mid2=(kt, 1, 0), tw=(L, 0)))
    strd = View(out, cols, 2 * N2 * cols, 2 * cols)
    model_pass(dict(N=N1, inv=False, **{"in": strd}, out=strd, qpc=qpc, nquads=N2 * qpc))
    return out.reshape(2 * S, cols).astype(np.uint32)


def pipe_geometry(L: int, q4a: int, q4m: int, grid: int, cols: int, tpi: int = 1) -> dict:
    """fourstep.cu pipe_t: chunk quads, work items (of tpi tiles) per chunk and pass, chunks, depth."""
    L1, L2, N1, N2 = split(L)
    cq = max(q4a, q4m)
    quads = cols // 4
    nch = -(-quads // cq)
    tiles = [N2 * cq // q4a // tpi, N1 * cq // q4m // tpi, N2 * cq // q4a // tpi]
    per_round = sum(tiles)
    depth = max(1, -(-(2 * 3 * grid) // per_round))
    return dict(cq=cq, nch=nch, tiles=tiles, per_round=per_round, depth=depth, tpi=tpi,
                last_qlim=quads - (nch - 1) * cq, total=(nch + 2 * depth) * per_round)


def pipe_decode(item: int, g: dict):
    """k_fourstep_pipe's item -> (pass, chunk, tile); chunk None for an empty item."""
    r, j = divmod(item, g["per_round"])
    t = g["tiles"]
    if j < t[0]:
        ph, c = 0, r
    elif j < t[0] + t[1]:
        ph, c, j = 1, r - g["depth"], j - t[0]
    else:
        ph, c, j = 2, r - 2 * g["depth"], j - t[0] - t[1]
    return ph, (c if 0 <= c < g["nch"] else None), j


def model_extend_pipelined(data: np.ndarray, q4a: int, q4m: int, grid: int, seed: int, tpi: int = 1) -> np.ndarray:
    """k_fourstep_pipe: the passes of long_extend as tiles of (chunk, pass), dealt in the
    kernel's order to `grid` CTAs that each hold one item and the two drawn after it, and
    finished in a random order among those whose dependencies are met (a pass-B or block
    tile waits for every tile of the chunk's previous pass). Fails on a deadlock, a tile
    run twice or missed, or a tile run before its dependencies."""
    S, cols = data.shape
    L = S.bit_length() - 1
    L1, L2, N1, N2 = split(L)
    g = pipe_geometry(L, q4a, q4m, grid, cols, tpi)
    cq = g["cq"]
    inp = data.astype(np.uint64).ravel()
    out = np.full(2 * S * cols, 12345, dtype=np.uint64)
    cbt, kt = coset_mid_tables(L, L + 1)[0]
    nq = {0: N2 * cq, 1: N1 * cq, 2: N2 * cq}

    def args(ph, c):
        off = c * 4 * cq
        qlim = g["last_qlim"] if c == g["nch"] - 1 else cq
        if ph == 0:
            return dict(N=N1, inv=True, **{"in": View(inp, off, N2 * cols, cols)},
                        out=View(out, cols + off, 2 * N2 * cols, 2 * cols), qpc=cq, nquads=nq[0], tw=(L, 1),
                        copy=View(out, off, 2 * N2 * cols, 2 * cols), qlim=qlim), q4a
        if ph == 1:
            blk = View(out, cols + off, 2 * cols, 2 * N2 * cols)
            return dict(N=N2, inv=True, two=True, **{"in": blk}, out=blk, qpc=cq, nquads=nq[1],
                        mid1=(cbt, 0, 1), mid2=(kt, 1, 0), tw=(L, 0), qlim=qlim), q4m
        strd = View(out, cols + off, 2 * N2 * cols, 2 * cols)
        return dict(N=N1, inv=False, **{"in": strd}, out=strd, qpc=cq, nquads=nq[2], qlim=qlim), q4a

    rng = np.random.default_rng(seed)
    counter = 0
    done = {0: np.zeros(g["nch"], int), 1: np.zeros(g["nch"], int)}
    ran = set()

    def draw():
        nonlocal counter
        counter += 1
        return counter - 1

    # [current, next, the one after]: the kernel draws two items up front and, at the top
    # of every item, the one after next (before it waits on the current one's dependencies)
    ctas = [[draw(), draw()] for _ in range(grid)]
    for cta in ctas:
        cta.append(draw())
    while True:
        live = [k for k, cta in enumerate(ctas) if cta[0] < g["total"]]
        if not live:
            break
        ready = []
        for k in live:
            ph, c, _ = pipe_decode(ctas[k][0], g)
            if c is None or ph == 0 or done[ph - 1][c] >= g["tiles"][ph - 1]:
                ready.append(k)
        assert ready, "deadlock: every CTA waits"
        k = ready[rng.integers(len(ready))]
        item, nxt, after = ctas[k]
        ph, c, j = pipe_decode(item, g)
        if c is not None:
            assert (ph, c, j) not in ran
            ran.add((ph, c, j))
            for u in range(tpi):  # the item's tiles in turn
                a, q4 = args(ph, c)
                t = j * tpi + u
                a["quads"] = (t * q4, t * q4 + q4)
                model_pass(a)
            if ph < 2:
                done[ph][c] += 1
        ctas[k] = [nxt, after, draw()]
    assert len(ran) == g["nch"] * sum(g["tiles"])
    return out.reshape(2 * S, cols).astype(np.uint32)


def model_cols_ntt(B: np.ndarray, L: int, inv: bool) -> np.ndarray:
    """long_cols_ntt on the legacy layout B = [n][w4] (flat), returns A = [n][w4]."""
    n = 1 << L
    w4 = B.size // n
    L1, L2, N1, N2 = split(L)
    qpc = w4 // 4
    B = B.astype(np.uint64).copy()
    A = np.zeros_like(B)
    model_pass(dict(N=N1, inv=inv, **{"in": View(B, 0, N2 * w4, w4)}, out=View(B, 0, N2 * w4, w4), qpc=qpc,
                    nquads=N2 * qpc, tw=(L, int(inv))))
    model_pass(dict(N=N2, inv=inv, **{"in": View(B, 0, w4, N2 * w4)}, out=View(A, 0, N1 * w4, w4), qpc=qpc,
                    nquads=N1 * qpc, scale=pow(n, P - 2, P) if inv else None))
    return A


def model_encode(data: np.ndarray, n: int, w0: int) -> np.ndarray:
    """general.cu's coset-0 copy plus long_encode (column chunks of w0)."""
    k, cols = data.shape
    P_, N = O.next_pow2(k), O.next_pow2(k + n)
    lp, ln = P_.bit_length() - 1, N.bit_length() - 1
    R, rows_out = N // P_, k + n
    L1, L2, N1, N2 = split(lp)
    out = np.full((rows_out, cols), 777, dtype=np.uint64)
    m0 = (rows_out + R - 1) // R
    md = min(k, m0)
    out[0:R * md:R] = data[:md]
    out[R * md::R][:m0 - md] = 0
    out = out.ravel()
    inp = data.astype(np.uint64).ravel()
    tabs = coset_mid_tables(lp, ln)
    for c0 in range(0, cols, w0):
        w = min(w0, cols - c0)
        qpc = w // 4
        A = np.zeros(P_ * w, dtype=np.uint64)
        Bm = np.zeros(P_ * w, dtype=np.uint64) if R > 2 else A
        model_pass(dict(N=N1, inv=True, **{"in": View(inp, c0, N2 * cols, cols)}, out=View(A, 0, N2 * w, w),
                        qpc=qpc, nquads=N2 * qpc, in_lim=(N2, 1, k), tw=(lp, 1)))
        for c in range(1, min(R, rows_out)):
            mc = min(P_, (rows_out - c + R - 1) // R)
            cbt, kt = tabs[c - 1]
            model_pass(dict(N=N2, inv=True, two=True, **{"in": View(A, 0, w, N2 * w)}, out=View(Bm, 0, w, N2 * w),
                            qpc=qpc, nquads=N1 * qpc, mid1=(cbt, 0, 1), mid2=(kt, 1, 0), tw=(lp, 0)))
            model_pass(dict(N=N1, inv=False, **{"in": View(Bm, 0, N2 * w, w)},
                            out=View(out, c * cols + c0, R * N2 * cols, R * cols), qpc=qpc, nquads=N2 * qpc,
                            out_lim=(N2, 1, mc)))
    return out.reshape(rows_out, cols).astype(np.uint32)


def model_recover(code: np.ndarray, known, k: int, check: bool = False):
    """long_recover: the five passes, with the pattern tables of k_erasure_tables_long."""
    N2k, cols = code.shape
    L = N2k.bit_length() - 1
    L1, L2, N1, N2 = split(L)
    have = np.zeros(N2k, dtype=bool)
    have[list(known)] = True
    wts = powtab(root(L), N2k)
    er = wts[~have]
    x, y = wts, wts * 31 % P
    zx, zy = np.ones(N2k, dtype=np.uint64), np.ones(N2k, dtype=np.uint64)
    for rr in er:
        zx = zx * ((x + P - rr) % P) % P
        zy = zy * ((y + P - rr) % P) % P
    zk = zx
    izh = np.array([pow(int(z), P - 2, P) for z in zy], dtype=np.uint64)
    hinv, ninv = pow(31, P - 2, P), pow(N2k, P - 2, P)
    cb_a, k_a = powtab(31, N1) * ninv % P, powtab(pow(31, N1, P), N2)
    cb_b, k_b = powtab(hinv, N1) * ninv % P, powtab(pow(hinv, N1, P), N2)
    k_b[N2 // 2:] = 0
    A = np.zeros(N2k * cols, dtype=np.uint64)
    src = code.astype(np.uint64).ravel()
    data = np.full(k * cols, 99, dtype=np.uint64)
    qpc = cols // 4
    strided, block = View(A, 0, N2 * cols, cols), View(A, 0, cols, N2 * cols)
    model_pass(dict(N=N1, inv=True, **{"in": View(src, 0, N2 * cols, cols)}, out=strided, qpc=qpc,
                    nquads=N2 * qpc, pre=(zk, N2, 1), tw=(L, 1)))
    model_pass(dict(N=N2, inv=True, two=True, **{"in": block}, out=block, qpc=qpc, nquads=N1 * qpc,
                    mid1=(cb_a, 0, 1), mid2=(k_a, 1, 0), tw=(L, 0)))
    model_pass(dict(N=N1, inv=False, two=True, **{"in": strided}, out=strided, qpc=qpc, nquads=N2 * qpc,
                    mid1=(izh, N2, 1), tw=(L, 1)))
    cnt = model_pass(dict(N=N2, inv=True, two=True, **{"in": block}, out=block, qpc=qpc, nquads=N1 * qpc,
                          mid1=(cb_b, 0, 1), mid2=(k_b, 1, 0), tw=(L, 0), count_from=N2 // 2 if check else None))
    model_pass(dict(N=N1, inv=False, **{"in": View(A, 0, N2 * cols, 2 * cols)},
                    out=View(data, 0, (N2 // 2) * cols, cols), qpc=qpc, nquads=(N2 // 2) * qpc))
    return data.reshape(k, cols).astype(np.uint32), cnt


@pytest.mark.parametrize("L", [12, 13, 14])
def test_model_extension_matches_oracle(L):
    S, cols = 1 << L, 8
    data = O.seeded_input(S, cols, seed=L)
    assert np.array_equal(model_extend(data), O.encode_rowmajor(data))


@pytest.mark.parametrize("L,inv", [(13, False), (13, True), (14, False), (15, True)])
def test_model_legacy_transform_matches_oracle(L, inv):
    n, polys = 1 << L, 5
    vals = O.seeded_input(1, n * polys, seed=L + 3)[0]
    B = vals.reshape(polys, n).T.copy()  # [n][polys]
    B = np.concatenate([B, np.zeros((n, 3), dtype=np.uint32)], axis=1)  # w4 = 8
    A = model_cols_ntt(B.ravel(), L, inv).reshape(n, 8)
    want = O.ntt_polys(vals, n, n, inv).reshape(polys, n).T
    assert np.array_equal(A[:, :polys].astype(np.uint32), want)


def test_model_legacy_permuted_root():
    # a caller's root w = omega^a: legacy.cu gathers rows (j * a) mod n when transposing back
    L, n = 13, 1 << 13
    a = 5
    w = pow(root(L), a, P)
    roots = powtab(w, n).astype(np.uint32)
    vals = O.seeded_input(1, n, seed=9)[0]
    B = np.concatenate([vals[:, None], np.zeros((n, 3), dtype=np.uint32)], axis=1)
    A = model_cols_ntt(B.ravel(), L, False).reshape(n, 4)
    got = A[(np.arange(n) * a) % n, 0].astype(np.uint32)
    assert np.array_equal(got, O.ntt(vals, roots))


@pytest.mark.parametrize("k,n,w0", [(5000, 3000, 8), (8192, 100, 4), (5000, 20000, 8), (4097, 4000, 12)])
def test_model_encode_matches_oracle(k, n, w0):
    cols = 12
    data = O.seeded_input(k, cols, seed=k + n)
    assert np.array_equal(model_encode(data, n, w0), O.encode_rowmajor(data, n))


def test_model_recover():
    k, cols = 8192, 4
    data = O.seeded_input(k, cols, seed=77)
    code = O.encode_rowmajor(data)
    rng = np.random.default_rng(5)
    known = np.sort(rng.choice(2 * k, size=k + 16, replace=False))  # more than k rows: checkable
    erased = np.setdiff1d(np.arange(2 * k), known)
    garbage = code.copy()
    garbage[erased] = rng.integers(0, P, (len(erased), cols), dtype=np.uint32)
    got, cnt = model_recover(garbage, known, k, check=True)
    assert cnt == 0
    assert np.array_equal(got, data)
    # one wrong known value makes the known rows inconsistent: the count is nonzero
    garbage[known[3], 1] = (int(garbage[known[3], 1]) + 1) % P
    _, cnt = model_recover(garbage, known, k, check=True)
    assert cnt > 0


# (L, Q4 of the strided passes, Q4 of the block pass, grid, columns): the kernel's tile
# widths per launch shape (Q4 = threads / (N / positions per thread)), small grids so
# that chunks overlap, ragged column counts so the last chunk is partial
@pytest.mark.parametrize("L,q4a,q4m,grid,cols", [(10, 256, 256, 3, 4 * 256 * 3 + 8), (11, 256, 128, 5, 4 * 256 * 4 + 12),
                                                 (12, 128, 128, 7, 4 * 128 * 5 + 4), (12, 32, 32, 16, 4 * 32 * 9 + 20),
                                                 (13, 128, 64, 4, 4 * 128 * 3 + 16)])
@pytest.mark.parametrize("tpi", [1, 2, 4])
def test_model_pipelined_extension_matches_oracle(L, q4a, q4m, grid, cols, tpi):
    S = 1 << L
    data = O.seeded_input(S, cols, seed=L + cols)
    assert np.array_equal(model_extend_pipelined(data, q4a, q4m, grid, seed=L + tpi, tpi=tpi),
                          O.encode_rowmajor(data))


def test_pipe_geometry_limits():
    # the kernel's item counter is 32-bit: the host keeps every draw below 2^31
    for L, q4a, q4m in ((10, 256, 256), (12, 128, 128), (12, 32, 32), (14, 64, 64)):
        g = pipe_geometry(L, q4a, q4m, 592, 1 << 26)
        assert g["total"] + 3 * 592 < 1 << 31
        assert all(t * q for t, q in zip(g["tiles"], (q4a, q4m, q4a)))
