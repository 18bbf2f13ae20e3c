"""Encode of any (k, n) shape and the k-of-2k erasure decoder, through the C ABI.

Encode parity: bit-exact against the oracle's restatement of the reference's
encode for general shapes (src/benchmarks/utils.rs:42-48,100-146: pad k to
n_k = next_pow2(k), INTT over n_k, NTT over n_kn = next_pow2(k + n), keep rows
0..k+n-1).

Decoder parity: the recovered data equals the original square bit for bit, for
random erasure patterns, and agrees with the oracle's Lagrange interpolation
of the same known rows."""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = O.P


@pytest.fixture(scope="module")
def ctx():
    import zoda_b200
    c = zoda_b200.Context(0)
    yield c
    c.close()


@pytest.fixture(autouse=True)
def no_wait_gave_up(ctx):
    """After every test: no kernel's bounded wait ran out (zoda_ctx_check)."""
    yield
    ctx.check()


def to_dev(a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def from_dev(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


SHAPES = [
    (100, 100),   # non-power-of-two k, rate 1/2: n_k 128, n_kn 256
    (64, 192),    # rate 1/4: three cosets
    (5, 3),       # tiny, n_kn 8 over n_k 8: R = 1 (data and zero rows only)
    (6, 3),       # n_kn 16 over n_k 8
    (1, 1),       # n_k = 1, a single data row
    (1, 6),       # n_k = 1, n_kn = 8
    (128, 64),    # fewer parity rows than data rows, n_kn = 256
    (96, 0),      # no parity: the padded data
    (1000, 24),   # n_kn 1024 = n_k: R = 1
    (1000, 1000), # n_k 1024, n_kn 2048
    (3, 125),     # rate 1/32
    (2048, 100),  # n_k 2048, n_kn 4096
    (3, 3),       # n_k 4, n_kn 8, fused kernels with rows cut
    (2, 1),       # n_k 2, n_kn 4
    (33, 31),     # n_k 64, fused, 64 output rows
    (300, 212),   # n_k 512, fused, n_kn 1024 exactly filled
    (1500, 1000), # n_k 2048, fused with the tuned side-2048 plan
    (3000, 3000), # n_k 4096, fused (direct kernel)
    # n_kn >= 4 n_k with n_k 128 .. 2048: one fused TMA-staged pass per coset
    (100, 300),   # n_k 128, R = 4
    (129, 900),   # n_k 256 (k just past a power of two), n_kn 2048: R = 8
    (200, 1800),  # n_k 256, R = 8
    (500, 7500),  # n_k 512, R = 16
    (1000, 3000), # n_k 1024, R = 4
    (2000, 6000), # n_k 2048, R = 4
]


@pytest.mark.parametrize("k,n", SHAPES, ids=[f"k{k}-n{n}" for k, n in SHAPES])
def test_encode_any_shape_matches_oracle(ctx, k, n):
    cols = 36 if k >= 1000 else 2 * 2048 + 20
    if (k, n) in ((33, 31), (300, 212)):
        cols = 3 * 32768 // 64 + 12 if k == 33 else 3 * 64 + 12  # several tiles, ragged
    data = O.seeded_input(k, cols, seed=7 * k + n)
    want = O.encode_rowmajor(data, n)
    d_in = to_dev(data)
    d_out = torch.full((k + n, cols), -1, dtype=torch.int32, device="cuda")
    ctx.encode(d_in, d_out, k, n, cols)
    torch.cuda.synchronize()
    got = from_dev(d_out)
    assert got.shape == want.shape
    assert np.array_equal(got, want)


def test_encode_square_power_of_two_is_the_extension(ctx):
    k, cols = 256, 4096
    data = O.seeded_input(k, cols, seed=3)
    d_in = to_dev(data)
    a = torch.empty((2 * k, cols), dtype=torch.int32, device="cuda")
    b = torch.empty_like(a)
    ctx.encode(d_in, a, k, k, cols)
    ctx.extend(d_in, b, k, cols)
    torch.cuda.synchronize()
    assert torch.equal(a, b)
    assert np.array_equal(from_dev(a)[:, :64], O.encode_rowmajor(data[:, :64]))


def test_encode_many_column_chunks(ctx):
    # n_k = 4096, n_kn = 16384 (the interpolation + per-coset path), with more columns than one
    # 256 MiB scratch chunk holds (16384)
    k, n, cols = 3000, 9000, 16384 + 64
    data = O.seeded_input(k, cols, seed=11)
    d_in = to_dev(data)
    d_out = torch.empty((k + n, cols), dtype=torch.int32, device="cuda")
    ctx.encode(d_in, d_out, k, n, cols)
    torch.cuda.synchronize()
    for c0 in (0, 16380, cols - 8):
        got = from_dev(d_out[:, c0:c0 + 8].contiguous())
        assert np.array_equal(got, O.encode_rowmajor(data[:, c0:c0 + 8], n)), c0


def test_encode_bad_args(ctx):
    import zoda_b200
    d = torch.zeros((8, 8), dtype=torch.int32, device="cuda")
    o = torch.zeros((16, 8), dtype=torch.int32, device="cuda")
    with pytest.raises(zoda_b200.ZodaError):
        ctx.encode(d, o, 0, 8, 8)       # k = 0
    with pytest.raises(zoda_b200.ZodaError):
        ctx.encode(d, o, 8, 8, 6)       # cols not a multiple of 4
    big = torch.zeros((4, 8), dtype=torch.int32, device="cuda")
    with pytest.raises(zoda_b200.ZodaError):
        ctx.encode(big, o, (1 << 26) + 1, 1, 8)  # next_pow2(k) > 2^26


# ---- decoder -------------------------------------------------------------------

def encoded(ctx, data):
    k, cols = data.shape
    d_in = to_dev(data)
    code = torch.empty((2 * k, cols), dtype=torch.int32, device="cuda")
    ctx.extend(d_in, code, k, cols)
    return code


def recover(ctx, code, known, k, cols, check=False):
    out = torch.full((k, cols), -1, dtype=torch.int32, device="cuda")
    mm = ctx.recover(code, known, k, cols, out, check=check)
    torch.cuda.synchronize()
    return from_dev(out), mm


@pytest.mark.parametrize("k", [1, 2, 4, 16, 64, 256, 1024, 2048, 4096])
def test_recover_random_k_of_2k(ctx, k):
    cols = 4096 + 36 if k <= 256 else {1024: 260, 2048: 132, 4096: 20}[k]
    data = O.seeded_input(k, cols, seed=500 + k)
    code = encoded(ctx, data)
    rng = np.random.default_rng(k)
    for trial in range(3):
        known = np.sort(rng.choice(2 * k, size=k, replace=False))
        # the unknown rows hold garbage: the decoder must not read them
        garbage = torch.from_numpy(rng.integers(0, 2**31, size=(2 * k, cols), dtype=np.int64).astype(np.int32)).cuda()
        mask = torch.ones(2 * k, dtype=torch.bool, device="cuda")
        mask[torch.from_numpy(known).cuda()] = False
        noisy = torch.where(mask[:, None], garbage, code)
        got, mm = recover(ctx, noisy, known, k, cols, check=True)
        assert mm == 0
        assert np.array_equal(got, data), (k, trial)


def test_recover_matches_lagrange_oracle(ctx):
    k, cols = 32, 64
    data = O.seeded_input(k, cols, seed=9)
    code = encoded(ctx, data)
    code_h = from_dev(code)
    known = list(range(1, 2 * k, 2))  # the odd rows only: every data row is erased
    got, _ = recover(ctx, code, known, k, cols)
    want = O.recover_rows(code_h[known], known, [2 * m for m in range(k)], 2 * k)
    assert np.array_equal(got, want)
    assert np.array_equal(got, data)


def test_recover_more_than_k_rows_and_fast_path(ctx):
    k, cols = 128, 2048
    data = O.seeded_input(k, cols, seed=21)
    code = encoded(ctx, data)
    rng = np.random.default_rng(5)
    known = np.sort(rng.choice(2 * k, size=k + 37, replace=False))
    got, mm = recover(ctx, code, known, k, cols, check=True)
    assert mm == 0 and np.array_equal(got, data)
    got, _ = recover(ctx, code, range(0, 2 * k, 2), k, cols)  # all data rows known: a copy
    assert np.array_equal(got, data)


def test_recover_flags_inconsistent_rows(ctx):
    k, cols = 64, 1024
    data = O.seeded_input(k, cols, seed=77)
    code = encoded(ctx, data)
    known = list(range(2 * k))  # all rows, one of them corrupted in 3 columns
    code[5, 100] = (int(code[5, 100]) + 1) % P
    code[5, 101] = (int(code[5, 101]) + 7) % P
    code[9, 900] = (int(code[9, 900]) + 3) % P
    _, mm = recover(ctx, code, known, k, cols, check=True)
    assert mm > 0


def test_recover_many_column_chunks(ctx):
    # 2k = 4096 rows: one scratch chunk holds 16384 columns
    k, cols = 2048, 16384 + 32
    data = O.seeded_input(k, cols, seed=8)
    code = encoded(ctx, data)
    rng = np.random.default_rng(1)
    known = np.sort(rng.choice(2 * k, size=k, replace=False))
    got, mm = recover(ctx, code, known, k, cols, check=True)
    assert mm == 0
    assert np.array_equal(got, data)


def test_recover_bad_args(ctx):
    import zoda_b200
    k, cols = 16, 64
    code = torch.zeros((2 * k, cols), dtype=torch.int32, device="cuda")
    out = torch.zeros((k, cols), dtype=torch.int32, device="cuda")
    with pytest.raises(zoda_b200.ZodaError):
        ctx.recover(code, range(k - 1), k, cols, out)           # too few rows
    with pytest.raises(zoda_b200.ZodaError):
        ctx.recover(code, list(range(k - 1)) + [2 * k], k, cols, out)  # index out of range
    with pytest.raises(zoda_b200.ZodaError):
        ctx.recover(code, range(k), 12, cols, out)              # k not a power of two
    big = torch.zeros((8, 8), dtype=torch.int32, device="cuda")
    with pytest.raises(zoda_b200.ZodaError):
        ctx.recover(big, range(8), 1 << 27, 8, big)             # beyond the largest k
