"""Row-side consumers on the device, through the C ABI: RLC coefficients
(src/zoda/rlc.rs:48-65), per-row RLC (rlc.rs:32-40) and the RLC check of every
encoded row (src/benchmarks/utils.rs:225-272), bit-exact against the oracle."""
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
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


def from_dev(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("root_len", [0, 1, 47, 48, 55, 56, 63, 64, 100, 111, 112, 130])
def test_coefficients_match_oracle(ctx, root_len):
    root = ("0123456789abcdef" * 9)[:root_len]
    ncols = 1000
    d = torch.empty((ncols, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_coefficients(root, ncols, d)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(d).astype(np.uint64), O.coefficients(root, ncols))


def test_coefficients_of_a_data_root(ctx):
    data = O.seeded_input(64, 8192, seed=5)
    root = O.compute_data_root(O.encode_rowmajor(data))
    d = torch.empty((8192, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_coefficients(root, 8192, d)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(d).astype(np.uint64), O.coefficients(root, 8192))


# shapes on both kernels: a thread per column quad below 256 rows, a thread per
# row from 256 on (ragged row blocks of 512, ragged and narrow 32-column chunks)
@pytest.mark.parametrize("rows,cols", [(1, 4), (37, 4100), (8, 131072), (255, 1028), (256, 4), (300, 512),
                                       (300, 36), (513, 4100), (1000, 20), (1536, 8192)])
def test_rlc_rows_match_oracle(ctx, rows, cols):
    m = O.seeded_input(rows, cols, seed=rows + cols)
    rng = np.random.default_rng(3)
    coeff = rng.integers(0, P, size=(cols, 4), dtype=np.uint64)
    out = torch.empty((rows, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_rows(to_dev(m), rows, cols, to_dev(coeff.astype(np.uint32)), out)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(out).astype(np.uint64), O.rlc_rows(m, coeff))


def test_rlc_rows_extreme_values(ctx):
    rows, cols = 9, 2048
    m = np.full((rows, cols), P - 1, dtype=np.uint32)
    coeff = np.full((cols, 4), P - 1, dtype=np.uint64)
    out = torch.empty((rows, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_rows(to_dev(m), rows, cols, to_dev(coeff.astype(np.uint32)), out)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(out).astype(np.uint64), O.rlc_rows(m, coeff))


@pytest.mark.parametrize("rows", [13, 300])
def test_rlc_rows_any_u32(ctx, rows):
    """Row values and coefficients over the whole u32 range (p, 2p, 2^32 - 1 among
    them): the sums are those of the values' residues."""
    cols = 8200
    rng = np.random.default_rng(17)
    m = rng.integers(0, 1 << 32, size=(rows, cols), dtype=np.uint64)
    m[0, :6] = [P, 2 * P, 2 * P - 1, (1 << 32) - 1, P - 1, 0]
    m[1] = (1 << 32) - 1
    coeff = rng.integers(0, 1 << 32, size=(cols, 4), dtype=np.uint64)
    out = torch.empty((rows, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_rows(to_dev(m.astype(np.uint32)), rows, cols, to_dev(coeff.astype(np.uint32)), out)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(out).astype(np.uint64), O.rlc_rows(m, coeff))


def test_rlc_rows_wide_and_short(ctx):
    rows, cols = 3, 1 << 20
    m = O.seeded_input(rows, cols, seed=23)
    coeff = np.random.default_rng(29).integers(0, P, size=(cols, 4), dtype=np.uint64)
    out = torch.empty((rows, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_rows(to_dev(m), rows, cols, to_dev(coeff.astype(np.uint32)), out)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(out).astype(np.uint64), O.rlc_rows(m, coeff))


HALF = (P - 1) // 2


@pytest.mark.parametrize("xv,cv", [(P - 1, P - 1), (HALF + 1, HALF + 1), (HALF, HALF + 1), (HALF, HALF),
                                   ((1 << 32) - 1, HALF + 1)])
def test_rlc_rows_full_size_worst_case(ctx, xv, cv):
    """The 1024 square's 2048 x 131072 code matrix with one value everywhere and
    one coefficient in every limb: residues at +-(p-1)/2 give the largest product
    magnitudes of either sign (p - 1 the largest canonical value), so every
    partial sum runs at its bound. Every limb is cols * x * c mod p."""
    rows, cols = 2048, 131072
    to_i32 = lambda v: v - (1 << 32) if v >= 1 << 31 else v
    x = torch.full((rows, cols), to_i32(xv), dtype=torch.int32, device="cuda")
    coeff = torch.full((cols, 4), to_i32(cv), dtype=torch.int32, device="cuda")
    out = torch.empty((rows, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_rows(x, rows, cols, coeff, out)
    torch.cuda.synchronize()
    assert bool((out == cols * (xv % P) * cv % P).all())


def test_rlc_rows_full_size_sampled(ctx):
    """Random 2048 x 131072 matrix: sampled rows against the oracle."""
    rows, cols = 2048, 131072
    gen = torch.Generator(device="cuda").manual_seed(31)
    x = torch.randint(0, P, (rows, cols), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    coeff = torch.randint(0, P, (cols, 4), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    out = torch.empty((rows, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_rows(x, rows, cols, coeff, out)
    torch.cuda.synchronize()
    pick = [0, 1, 3, 4, 5, 1023, 1024, 2046, 2047] + list(np.random.default_rng(37).integers(0, rows, 7))
    want = O.rlc_rows(from_dev(x[pick]).astype(np.uint64), from_dev(coeff).astype(np.uint64))
    assert np.array_equal(from_dev(out)[pick].astype(np.uint64), want)


def reference_flow(ctx, data, n):
    """encode -> data root (host) -> coefficients (device) -> RLC check of every row."""
    import zoda_b200
    k, cols = data.shape
    d_in = to_dev(data)
    code = torch.empty((k + n, cols), dtype=torch.int32, device="cuda")
    ctx.encode(d_in, code, k, n, cols)
    torch.cuda.synchronize()
    root = zoda_b200.data_root(from_dev(code))
    coeff = torch.empty((cols, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_coefficients(root, cols, coeff)
    return d_in, code, coeff


@pytest.mark.parametrize("k,n", [(64, 64), (256, 256), (1024, 1024), (100, 50), (3, 13)])
def test_rlc_check_passes_on_valid_encodings(ctx, k, n):
    cols = 8192 if k <= 256 else 1024
    data = O.reference_input(k, cols) if k == 64 else O.seeded_input(k, cols, seed=k + n)
    d_in, code, coeff = reference_flow(ctx, data, n)
    assert ctx.rlc_check(d_in, code, k, n, cols, coeff) == 0


def test_rlc_check_catches_a_corrupted_share(ctx):
    k, cols = 128, 4096
    data = O.seeded_input(k, cols, seed=1)
    d_in, code, coeff = reference_flow(ctx, data, k)
    code[77, 1234] = (int(code[77, 1234]) + 1) % P  # one element of one parity row
    assert ctx.rlc_check(d_in, code, k, k, cols, coeff) == 4  # every limb of row 77
    code[77, 1234] = (int(code[77, 1234]) + P - 1) % P
    assert ctx.rlc_check(d_in, code, k, k, cols, coeff) == 0


def test_rlc_check_matches_reference_validation(ctx):
    # the reference's own validation path (utils.rs:170-272) in the oracle agrees
    k, cols = 64, 8192
    data = O.reference_input(k, cols)
    d_in, code, coeff = reference_flow(ctx, data, k)
    ok = O.validate_encoding(data, from_dev(code))
    assert ok[0] if isinstance(ok, tuple) else ok
    assert ctx.rlc_check(d_in, code, k, k, cols, coeff) == 0
