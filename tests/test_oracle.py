"""Pins the CPU oracle against the reference's own CPU tests (src/field/babybear.rs:80-106,
src/ntt/cpu.rs:112-187, src/zoda/babybear.rs:116-215) and against a pure-Python line-by-line
restatement of src/ntt/cpu.rs."""
import numpy as np
import pytest

import oracle as O

P = O.P


# ---- src/field/babybear.rs:84-105 -------------------------------------------------

def test_field_basic_arithmetic():
    L = O.lib()
    a, b = L.zo_bb_new(100), L.zo_bb_new(200)
    assert L.zo_bb_add(a, b) == 300
    assert L.zo_bb_sub(b, a) == 100
    assert L.zo_bb_sub(a, b) == P - 100
    assert L.zo_bb_mul(a, b) == 20000


def test_field_modular_reduction():
    L = O.lib()
    assert L.zo_bb_new(P + 5) == 5
    assert L.zo_bb_add(L.zo_bb_new(P - 1), 1) == 0


def test_field_mul_wraps():
    L = O.lib()
    m1 = L.zo_bb_new(P - 1)
    assert L.zo_bb_mul(m1, m1) == 1


# ---- src/ntt/cpu.rs ---------------------------------------------------------------

def test_generator_is_31():
    # smallest generator of F_p for BabyBear; it fixes every root table
    assert O.find_generator(P) == 31
    assert O.find_generator(257) == 3


def test_roundtrip_p257():
    # src/ntt/cpu.rs:112-121
    poly = np.array([1, 3, 4, 5, 6, 7, 9, 10], dtype=np.uint32)
    roots = O.roots_of_unity(8, 257)
    out = O.intt(O.ntt(poly, roots, 257), roots, 257)
    assert np.array_equal(out, poly)


@pytest.mark.parametrize("log_n", [0, 1, 4, 8, 12])
def test_babybear_roundtrip(log_n):
    # src/ntt/cpu.rs:158-168, input 7i+3
    n = 1 << log_n
    v = (np.arange(n, dtype=np.uint64) * 7 + 3).astype(np.uint32)
    assert np.array_equal(O.intt(O.ntt(v)), v)


def test_ntt_matches_naive_evaluation():
    # src/ntt/cpu.rs:170-187: NTT output k equals the polynomial evaluated at roots[k]
    n = 8
    roots = O.roots_of_unity(n)
    c = [13 * i + 5 for i in range(n)]
    evals = O.ntt(np.array(c, dtype=np.uint32))
    for k in range(n):
        x = int(roots[k])
        assert int(evals[k]) == sum(ci * pow(x, i, P) for i, ci in enumerate(c)) % P


@pytest.mark.parametrize("n", [1, 2, 4, 8, 32, 64])
def test_c_matches_pure_python(n):
    rng = np.random.default_rng(n)
    v = rng.integers(0, P, n, dtype=np.uint32)
    roots = O.py_roots_of_unity(n, P)
    assert np.array_equal(O.roots_of_unity(n), np.array(roots, dtype=np.uint32))
    assert [int(x) for x in O.ntt(v)] == O.py_ntt(v, roots, P)
    assert [int(x) for x in O.intt(v)] == O.py_intt(v, roots, P)


# ---- src/zoda/babybear.rs:116-215 (CPU branch) -------------------------------------

@pytest.mark.parametrize("size", [4, 8, 16, 32])
def test_zoda_cpu_self_check(size):
    rng = np.random.default_rng(1000 + size)
    data = rng.integers(1, 256, size=(size, size), dtype=np.uint32)  # rows x cols
    k, cols = data.shape
    n_k, n_kn = O.next_pow2(k), O.next_pow2(2 * k)
    square = np.zeros((cols, n_kn), dtype=np.uint32)
    square[:, :k] = data.T
    ext = O.extend_colmajor(square.reshape(-1), n_k, n_kn).reshape(cols, n_kn)
    # the RLC of the original rows, extended limb by limb, matches the RLC of extended rows
    cells = ext.T  # [n_kn][cols]
    coeff = O.coefficients(O.compute_data_root(cells), cols)
    y = O.rlc_rows(data, coeff)
    for limb in range(O.RLC_LIMBS):
        v = np.zeros(n_k, dtype=np.uint32)
        v[:k] = y[:, limb]
        pad = np.zeros(n_kn, dtype=np.uint32)
        pad[:n_k] = O.intt(v)
        yl = O.ntt(pad)
        for row in rng.integers(0, n_kn, 64):
            assert O.rlc_rows(cells[row], coeff)[0, limb] == yl[row]
    # data at every (n_kn/n_k)-th row, and every column is a codeword of degree < n_k
    stride = n_kn // n_k
    assert np.array_equal(ext[:, ::stride][:, :k], data.T)
    for c in range(cols):
        assert not O.intt(ext[c])[n_k:].any()


def test_encode_rowmajor_matches_colmajor_extend():
    data = O.seeded_input(16, 40, seed=3)
    out = O.encode_rowmajor(data)
    sq = np.zeros((40, 32), dtype=np.uint32)
    sq[:, :16] = data.T
    ext = O.extend_colmajor(sq.reshape(-1), 16, 32).reshape(40, 32)
    assert np.array_equal(out, ext.T)
    # column window
    win = O.encode_rowmajor(data, col0=7, ncols=5)
    assert np.array_equal(win, out[:, 7:12])


def test_validate_encoding_side64_reference_input():
    # src/benchmarks/utils.rs:174-278 on the 64x64 square (8192 columns), input (row*cols+col) mod p
    data = O.reference_input(64, 64 * 128)
    enc = O.encode_rowmajor(data)
    ok, why = O.validate_encoding(data, enc)
    assert ok, why
    bad = enc.copy()
    bad[78, 4000] ^= 1  # a wrong value in a sampled row outside the sampled columns fails the RLC phase
    assert not O.validate_encoding(data, bad)[0]


def test_erasure_recovery_random_k_of_2k():
    rng = np.random.default_rng(9)
    data = O.seeded_input(64, 24, seed=11)
    enc = O.encode_rowmajor(data)
    keep = np.sort(rng.choice(128, size=64, replace=False))
    rec = O.recover_rows(enc[keep], keep, list(range(0, 128, 2)), 128)
    assert np.array_equal(rec, data)
