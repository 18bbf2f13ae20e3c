"""CPU oracle for zoda-cu's column-wise Reed-Solomon extension over BabyBear.

TEST INFRASTRUCTURE ONLY. The tests, the smoke check and the bench's CPU
baseline use this module as the checker; the product path (the CUDA library
in zoda-cu_b200/) never imports it.

Three layers, each citing the reference function it restates:
  * ``liboracle.so`` (zoda_oracle.c): the reference's CPU NTT, INTT and
    extension (src/ntt/cpu.rs, src/zoda/babybear.rs:34-46), column-parallel.
  * pure-Python NTT/INTT (``py_ntt``/``py_intt``) for tiny cases, used to
    cross-check the C restatement line by line.
  * the validation side of the reference: RLC coefficients and rows
    (src/zoda/rlc.rs:32-65), the data root (src/benchmarks/utils.rs:51-59),
    the two-phase validation (utils.rs:174-278), and a k-of-2k erasure
    decoder (no reference counterpart; it is checked against the original).
"""
from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess

import numpy as np

P = 2013265921  # src/field/babybear.rs:9
RLC_LIMBS = 4  # src/zoda/rlc.rs:18
HERE = os.path.dirname(os.path.abspath(__file__))

_lib = None


def lib():
    """Load liboracle.so, building it with the Makefile beside it if absent."""
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        L = ctypes.CDLL(path)
        u32p = ctypes.POINTER(ctypes.c_uint32)
        L.zo_pow_mod.restype = ctypes.c_uint32
        L.zo_pow_mod.argtypes = [ctypes.c_uint32] * 3
        L.zo_find_generator.restype = ctypes.c_uint32
        L.zo_find_generator.argtypes = [ctypes.c_uint32]
        L.zo_roots_of_unity.argtypes = [ctypes.c_uint32, ctypes.c_uint32, u32p]
        L.zo_ntt.argtypes = [u32p, u32p, ctypes.c_size_t, ctypes.c_uint32]
        L.zo_intt.argtypes = [u32p, u32p, ctypes.c_size_t, ctypes.c_uint32]
        L.zo_ntt_babybear.argtypes = [u32p, ctypes.c_size_t]
        L.zo_intt_babybear.argtypes = [u32p, ctypes.c_size_t]
        L.zo_extend_colmajor.argtypes = [u32p, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_int]
        L.zo_encode_rowmajor.argtypes = [u32p, u32p] + [ctypes.c_size_t] * 5 + [ctypes.c_int]
        L.zo_ntt_polys.argtypes = [u32p, u32p] + [ctypes.c_uint32] * 3 + [ctypes.c_int]
        for name in ("zo_bb_new",):
            getattr(L, name).restype = ctypes.c_uint32
            getattr(L, name).argtypes = [ctypes.c_uint64]
        for name in ("zo_bb_add", "zo_bb_sub", "zo_bb_mul"):
            getattr(L, name).restype = ctypes.c_uint32
            getattr(L, name).argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))


def num_threads() -> int:
    return int(lib().zo_num_threads())


# ---- number theory and transforms (src/ntt/cpu.rs) --------------------------

def pow_mod(b: int, e: int, p: int = P) -> int:
    return int(lib().zo_pow_mod(b, e, p))


def find_generator(p: int = P) -> int:
    return int(lib().zo_find_generator(p))


def roots_of_unity(n: int, p: int = P) -> np.ndarray:
    """src/ntt/cpu.rs:96-110."""
    out = np.empty(n, dtype=np.uint32)
    if lib().zo_roots_of_unity(n, p, _ptr(out)) != 0:
        raise ValueError("n must divide p - 1")
    return out


def ntt(values, roots=None, p: int = P) -> np.ndarray:
    """src/ntt/cpu.rs:1-32 (roots default to roots_of_unity(n, p))."""
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    r = roots_of_unity(len(v), p) if roots is None else np.ascontiguousarray(roots, dtype=np.uint32)
    lib().zo_ntt(_ptr(v), _ptr(r), len(v), p)
    return v


def intt(values, roots=None, p: int = P) -> np.ndarray:
    """src/ntt/cpu.rs:48-60."""
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    r = roots_of_unity(len(v), p) if roots is None else np.ascontiguousarray(roots, dtype=np.uint32)
    lib().zo_intt(_ptr(v), _ptr(r), len(v), p)
    return v


def ntt_polys(values: np.ndarray, n: int, stride: int, inverse: bool) -> np.ndarray:
    """What cuda_ntt / cuda_intt must return (cuda/ntt_kernel.cu:190-208):
    the first n of every stride-long polynomial transformed, the rest untouched."""
    v = np.ascontiguousarray(values, dtype=np.uint32).copy()
    polys = v.size // stride
    r = roots_of_unity(n)
    if lib().zo_ntt_polys(_ptr(v), _ptr(r), n, polys, stride, int(inverse)) != 0:
        raise ValueError("bad arguments")
    return v


# pure-Python restatement for tiny inputs (src/ntt/cpu.rs:1-60), used to pin the C code

def _py_reverse(values):
    if len(values) <= 1:
        return list(values)
    return _py_reverse(values[0::2]) + _py_reverse(values[1::2])


def py_ntt(values, roots, p):
    coeffs = _py_reverse([int(x) for x in values])
    n = len(coeffs)
    length = 2
    while length <= n:
        half, stride = length // 2, n // length
        for blk in range(0, n, length):
            for j in range(half):
                w = int(roots[j * stride])
                a = coeffs[blk + j]
                b = coeffs[blk + half + j] * w % p
                coeffs[blk + j] = (a + b) % p
                coeffs[blk + half + j] = (a + p - b) % p
        length *= 2
    return coeffs


def py_intt(values, roots, p):
    n = len(values)
    inv_roots = [int(roots[0])] + [int(x) for x in roots[1:][::-1]]
    c = py_ntt(values, inv_roots, p)
    n_inv = pow(n, p - 2, p)
    return [x * n_inv % p for x in c]


def py_roots_of_unity(n, p):
    m, q, fac = p - 1, 2, []
    while q * q <= m:
        if m % q == 0:
            fac.append(q)
            while m % q == 0:
                m //= q
        q += 1
    if m > 1:
        fac.append(m)
    g = next(g for g in range(2, p) if all(pow(g, (p - 1) // f, p) != 1 for f in fac))
    w = pow(g, (p - 1) // n, p)
    return [pow(w, i, p) for i in range(n)]


# ---- ZODA extension --------------------------------------------------------

def next_pow2(x: int) -> int:
    r = 1
    while r < x:
        r <<= 1
    return r


def extend_colmajor(square: np.ndarray, n_k: int, n_kn: int, threads: int = 0) -> np.ndarray:
    """src/zoda/babybear.rs:40-45 on a column-major [cols][n_kn] buffer."""
    sq = np.ascontiguousarray(square, dtype=np.uint32).copy()
    cols = sq.size // n_kn
    if lib().zo_extend_colmajor(_ptr(sq), n_k, n_kn, cols, threads) != 0:
        raise ValueError("bad extend arguments")
    return sq


def encode_rowmajor(data: np.ndarray, n: int | None = None, col0: int = 0, ncols: int | None = None,
                    threads: int = 0) -> np.ndarray:
    """Row-major [k][cols] -> row-major [k+n][cols] (src/benchmarks/utils.rs:100-146 with CPU
    transforms): INTT over next_pow2(k) rows, zero pad, NTT over next_pow2(k+n) rows.
    col0/ncols restrict the work to a window of columns."""
    data = np.ascontiguousarray(data, dtype=np.uint32)
    k, cols = data.shape
    n = k if n is None else n
    ncols = cols - col0 if ncols is None else ncols
    out = np.empty((k + n, ncols), dtype=np.uint32)
    if lib().zo_encode_rowmajor(_ptr(data), _ptr(out), k, n, cols, col0, ncols, threads) != 0:
        raise ValueError("bad encode arguments")
    return out


# ---- inputs ------------------------------------------------------------------

def reference_input(k: int, cols: int) -> np.ndarray:
    """src/benchmarks/utils.rs:81-84: element (row, col) = (row*cols + col) mod p."""
    return (np.arange(k * cols, dtype=np.uint64) % P).astype(np.uint32).reshape(k, cols)


def seeded_input(k: int, cols: int, seed: int) -> np.ndarray:
    """Seeded uniform canonical values in [0, p)."""
    rng = np.random.default_rng(seed)
    return rng.integers(0, P, size=(k, cols), dtype=np.uint32)


# ---- validation side (src/zoda/rlc.rs, src/benchmarks/utils.rs) ------------

def compute_data_root(rows: np.ndarray) -> str:
    """src/benchmarks/utils.rs:51-59: SHA-256 over the rows' little-endian u32 bytes, lowercase hex."""
    return hashlib.sha256(np.ascontiguousarray(rows, dtype="<u4").tobytes()).hexdigest()


def coefficients(data_root: str, num_columns: int) -> np.ndarray:
    """src/zoda/rlc.rs:48-65: coeff[col][l] = BE_u64(SHA256(root_hex || col as u64 LE)[8l:8l+8]) mod p."""
    out = np.empty((num_columns, RLC_LIMBS), dtype=np.uint64)
    root = data_root.encode()
    for i in range(num_columns):
        d = hashlib.sha256(root + int(i).to_bytes(8, "little")).digest()
        for limb in range(RLC_LIMBS):
            out[i, limb] = int.from_bytes(d[8 * limb:8 * limb + 8], "big") % P
    return out


def rlc_rows(rows: np.ndarray, coeff: np.ndarray) -> np.ndarray:
    """src/zoda/rlc.rs:32-40 for many rows at once: out[r][l] = sum_c rows[r][c]*coeff[c][l] mod p.
    Products are < 2^62, so each is reduced before summing in chunks."""
    rows = np.asarray(rows, dtype=np.uint64)
    if rows.ndim == 1:
        rows = rows[None, :]
    acc = np.zeros((rows.shape[0], RLC_LIMBS), dtype=np.uint64)
    chunk = 1 << 20
    for c0 in range(0, rows.shape[1], chunk):
        r = rows[:, c0:c0 + chunk]
        for limb in range(RLC_LIMBS):
            prod = (r * coeff[c0:c0 + chunk, limb][None, :]) % P
            # at most 2^20 terms of < 2^31 each: the sum stays below 2^51
            acc[:, limb] = (acc[:, limb] + prod.sum(axis=1)) % P
    return acc


def validate_encoding(data: np.ndarray, encoded: np.ndarray, n: int | None = None,
                      sample_rows: int = 64, sample_cols: int = 64) -> tuple[bool, str]:
    """src/benchmarks/utils.rs:174-278: phase 1 re-encodes evenly spaced columns on the CPU and
    compares all k+n rows; phase 2 derives RLC coefficients from the data root of the encoded rows,
    extends the RLC of the original rows limb by limb and compares evenly spaced encoded rows."""
    k, cols = data.shape
    n = k if n is None else n
    n_k, n_kn = next_pow2(k), next_pow2(k + n)
    ncheck = min(sample_cols, cols)
    for i in range(ncheck):
        c = i * cols // ncheck
        ref = encode_rowmajor(data, n, col0=c, ncols=1)[:, 0]
        if not np.array_equal(ref, encoded[:k + n, c]):
            return False, f"column {c} differs from the CPU re-encode"
    root = compute_data_root(encoded[:k + n])
    coeff = coefficients(root, cols)
    y = rlc_rows(data, coeff)  # [k][limbs]
    limb_polys = np.zeros((n_kn, RLC_LIMBS), dtype=np.uint32)
    for limb in range(RLC_LIMBS):
        v = np.zeros(n_k, dtype=np.uint32)
        v[:k] = y[:, limb]
        c = intt(v)
        pad = np.zeros(n_kn, dtype=np.uint32)
        pad[:n_k] = c
        limb_polys[:, limb] = ntt(pad)
    nrlc = min(sample_rows, k + n)
    idx = [i * (k + n) // nrlc for i in range(nrlc)]
    got = rlc_rows(encoded[idx], coeff)
    if not np.array_equal(got.astype(np.uint32), limb_polys[idx]):
        return False, "RLC of an encoded row differs from the extended RLC vector"
    return True, "ok"


# ---- erasure recovery (no reference counterpart) -----------------------------

def _inv(x):
    return pow(int(x), P - 2, P)


def _prod_mod_rows(a: np.ndarray) -> np.ndarray:
    """Product mod p along axis 1 of a uint64 matrix with entries < p (pairwise tree)."""
    a = a % P
    while a.shape[1] > 1:
        if a.shape[1] & 1:
            a = np.concatenate([a, np.ones((a.shape[0], 1), dtype=np.uint64)], axis=1)
        a = (a[:, 0::2] * a[:, 1::2]) % P
    return a[:, 0]


def recover_rows(known_rows: np.ndarray, known_idx, want_idx, n_kn: int) -> np.ndarray:
    """Given codeword rows at indices known_idx (evaluations at w^j, w the primitive n_kn-th
    root of unity of src/ntt/cpu.rs:96-110), with len(known_idx) equal to the degree bound,
    evaluate the interpolant at rows want_idx by Lagrange interpolation.
    Returns [len(want_idx)][cols]."""
    known_idx = [int(j) for j in known_idx]
    w = int(roots_of_unity(n_kn)[1])
    xs = np.array([pow(w, j, P) for j in known_idx], dtype=np.uint64)
    m = len(xs)
    diff = (xs[:, None] + P - xs[None, :]) % P
    np.fill_diagonal(diff, 1)
    bw = np.array([_inv(v) for v in _prod_mod_rows(diff)], dtype=np.uint64)  # barycentric weights
    known = np.asarray(known_rows, dtype=np.uint64)
    pos = {j: t for t, j in enumerate(known_idx)}
    out = np.zeros((len(want_idx), known.shape[1]), dtype=np.uint64)
    for t, r in enumerate(want_idx):
        r = int(r)
        if r in pos:
            out[t] = known[pos[r]]
            continue
        y = pow(w, r, P)
        yd = (y + P - xs) % P  # y - x_j, never 0 here
        full = int(_prod_mod_rows(yd[None, :])[0])
        lj = np.array([full * int(b) % P * _inv(d) % P for b, d in zip(bw, yd)], dtype=np.uint64)
        terms = (known * lj[:, None]) % P  # each < p, at most 2^27 of them per column
        out[t] = terms.sum(axis=0) % P
    return out.astype(np.uint32)
