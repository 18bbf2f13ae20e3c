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


@pytest.mark.parametrize("rows,cols", [(1, 4), (37, 4100), (8, 131072), (300, 512)])
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
