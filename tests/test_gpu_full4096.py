"""The 4096 x 4096 square at full size (8 GiB in, 16 GiB out, resident in HBM),
validated the way its workload asks: the RLC check of every one of the 8192
encoded rows (src/benchmarks/utils.rs:225-272, on the device) and a random
k-of-2k erasure recovery (k = 4096) on a window of columns, plus a CPU
re-encode of sampled columns (utils.rs:185-218) by the oracle."""
import hashlib

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = O.P
K = 4096
COLS = K * 128


def data_root_streamed(rows) -> str:
    """compute_data_root (utils.rs:51-59) of a device matrix: SHA-256 over the little-endian
    row bytes, streamed to the host in slabs of 32 rows."""
    h = hashlib.sha256()
    buf = torch.empty((32, rows.shape[1]), dtype=torch.int32).pin_memory()
    for r0 in range(0, rows.shape[0], 32):
        n = min(32, rows.shape[0] - r0)
        buf[:n].copy_(rows[r0:r0 + n])
        h.update(buf[:n].numpy())
    return h.hexdigest()


@pytest.fixture(scope="module")
def square():
    import zoda_b200
    ctx = zoda_b200.Context(0)
    gen = torch.Generator(device="cuda").manual_seed(4096)
    d_in = torch.empty((K, COLS), dtype=torch.int32, device="cuda")
    for r0 in range(0, K, 512):  # seeded uniform in [0, p), generated in slabs to bound the int64 temporary
        d_in[r0:r0 + 512] = torch.randint(0, P, (512, COLS), dtype=torch.int64, device="cuda",
                                          generator=gen).to(torch.int32)
    d_out = torch.empty((2 * K, COLS), dtype=torch.int32, device="cuda")
    ctx.extend(d_in, d_out, K, COLS)
    torch.cuda.synchronize()
    ctx.check()
    yield ctx, d_in, d_out
    del d_in, d_out
    torch.cuda.empty_cache()
    ctx.close()


def test_even_rows_are_the_data(square):
    _, d_in, d_out = square
    assert torch.equal(d_out[0::2], d_in)


def test_sampled_columns_match_cpu_reencode(square):
    _, d_in, d_out = square
    for c0 in (0, 262144, COLS - 4):
        data = d_in[:, c0:c0 + 4].contiguous().cpu().numpy().view(np.uint32)
        got = d_out[:, c0:c0 + 4].contiguous().cpu().numpy().view(np.uint32)
        assert np.array_equal(got, O.encode_rowmajor(data)), c0


def test_rlc_check_of_every_row(square):
    ctx, d_in, d_out = square
    coeff = torch.empty((COLS, 4), dtype=torch.int32, device="cuda")
    # coefficients from the data root of the encoded rows, as the reference derives them
    ctx.rlc_coefficients(data_root_streamed(d_out), COLS, coeff)
    assert ctx.rlc_check(d_in, d_out, K, K, COLS, coeff) == 0
    # one wrong share in one row is caught (all four limbs of that row)
    d_out[5001, 77] = (int(d_out[5001, 77]) + 1) % P
    assert ctx.rlc_check(d_in, d_out, K, K, COLS, coeff) == 4
    d_out[5001, 77] = (int(d_out[5001, 77]) + P - 1) % P


def test_random_half_erasure_recovery(square):
    ctx, d_in, d_out = square
    rng = np.random.default_rng(4096)
    for c0 in (0, 300000):
        code = d_out[:, c0:c0 + 64].contiguous()
        known = np.sort(rng.choice(2 * K, size=K, replace=False))
        out = torch.empty((K, 64), dtype=torch.int32, device="cuda")
        assert ctx.recover(code, known, K, 64, out, check=True) == 0
        assert torch.equal(out, d_in[:, c0:c0 + 64])
