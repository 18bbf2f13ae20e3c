"""Parity of the fused extension kernel (zoda_extend_device / zoda_extend_host)
against the CPU oracle, bit-exact, through the C ABI.

The oracle is the reference's encode (src/benchmarks/utils.rs:100-146 with
src/ntt/cpu.rs transforms): INTT over k rows, zero pad, NTT over 2k rows,
rows gathered in natural order."""
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
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def from_dev(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


def run_extend(ctx, data: np.ndarray) -> np.ndarray:
    k, cols = data.shape
    d_in = to_dev(data)
    d_out = torch.empty((2 * k, cols), dtype=torch.int32, device="cuda")
    ctx.extend(d_in, d_out, k, cols)
    torch.cuda.synchronize()
    return from_dev(d_out)


def tile_cols(side: int) -> int:
    """Columns per CTA tile of the kernel for this side (used to size ragged cases)."""
    return 2048 if side <= 16 else 32768 // side


SIDES = [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]
IMPLS = [(s, 1) for s in SIDES] + [(s, 2) for s in SIDES if s >= 32]


@pytest.mark.parametrize("side,impl", IMPLS, ids=[f"side{s}-{'direct' if i == 1 else 'tma'}" for s, i in IMPLS])
def test_extend_matches_oracle_all_sides(ctx, side, impl):
    # both kernel variants; two full tiles plus a ragged third (still a multiple of 4 columns)
    cols = 2 * tile_cols(side) + 12 if side > 1 else 36
    data = O.seeded_input(side, cols, seed=100 + side)
    ctx.set_impl(impl)
    try:
        got = run_extend(ctx, data)
        ctx.check()
    finally:
        ctx.set_impl(0)
    want = O.encode_rowmajor(data)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("side", [128, 1024, 2048])
def test_extend_many_tiles_per_cta(ctx, side):
    # more tiles than SMs, so every CTA loops and reuses its staging buffer
    cols = 148 * 3 * tile_cols(side) + 40
    data = O.seeded_input(side, cols, seed=300 + side)
    got = run_extend(ctx, data)
    ctx.check()
    idx = np.r_[0:64, cols // 2:cols // 2 + 64, cols - 64:cols]
    want = O.encode_rowmajor(data[:, idx])
    assert np.array_equal(got[:, idx], want)


def test_extend_config_side64_full(ctx):
    # 64x64 square of 512-byte shares: [64][8192] -> [128][8192], seeded uniform in [0, p)
    data = O.seeded_input(64, 64 * 128, seed=1)
    assert np.array_equal(run_extend(ctx, data), O.encode_rowmajor(data))


def test_extend_reference_input_validates(ctx):
    # src/benchmarks/utils.rs:174-278 on the reference's own input at side 256
    data = O.reference_input(256, 256 * 128)
    enc = run_extend(ctx, data)
    ok, why = O.validate_encoding(data, enc)
    assert ok, why


def test_extend_edge_values(ctx):
    # all zeros, all p-1, and alternating extremes
    side, cols = 128, 512
    for fill in (0, P - 1):
        data = np.full((side, cols), fill, dtype=np.uint32)
        assert np.array_equal(run_extend(ctx, data), O.encode_rowmajor(data))
    data = np.zeros((side, cols), dtype=np.uint32)
    data[::2] = P - 1
    assert np.array_equal(run_extend(ctx, data), O.encode_rowmajor(data))


def test_extend_outputs_canonical_and_systematic(ctx):
    data = O.seeded_input(512, 1024, seed=5)
    enc = run_extend(ctx, data)
    assert enc.max() < P
    assert np.array_equal(enc[0::2], data)


def test_extend_side1024_full_size_properties(ctx):
    # 1024x1024 square ([1024][131072] u32, 512 MiB in, 1 GiB out): even rows are the
    # data, sampled columns match the CPU re-encode, sampled rows pass the RLC check
    side, cols = 1024, 1024 * 128
    gen = torch.Generator(device="cuda").manual_seed(7)
    d_in = torch.randint(0, P, (side, cols), dtype=torch.int64, device="cuda", generator=gen).to(torch.int32)
    d_out = torch.empty((2 * side, cols), dtype=torch.int32, device="cuda")
    ctx.extend(d_in, d_out, side, cols)
    torch.cuda.synchronize()
    assert torch.equal(d_out[0::2], d_in)
    data = from_dev(d_in)
    enc = from_dev(d_out)
    ok, why = O.validate_encoding(data, enc, sample_rows=64, sample_cols=32)
    assert ok, why


def test_extend_erasure_recovery(ctx):
    # any k of the 2k extended rows determine the square (k-of-2k recovery)
    side, cols = 256, 64
    data = O.seeded_input(side, cols, seed=21)
    enc = run_extend(ctx, data)
    rng = np.random.default_rng(3)
    keep = np.sort(rng.choice(2 * side, size=side, replace=False))
    want = list(range(0, 2 * side, 2))
    rec = O.recover_rows(enc[keep], keep, want, 2 * side)
    assert np.array_equal(rec, data)


@pytest.mark.parametrize("side,cols", [(1, 64), (2, 128), (16, 2048 + 4), (256, 4096), (512, 512 * 128 + 4 * 37),
                                       (2048, 4096), (4096, 256)])
def test_extend_host_matches_device(ctx, side, cols):
    # (512, ...) moves ~134 MB in three column chunks over three streams, the last one ragged;
    # only the odd rows come back over PCIe, the even rows are copied on the host
    data = O.seeded_input(side, cols, seed=9)
    h_in = torch.from_numpy(data.view(np.int32)).pin_memory()
    h_out = torch.full((2 * side, cols), -1, dtype=torch.int32).pin_memory()
    t = ctx.extend_host(h_in, h_out, side, cols)
    assert t.kernel_ms > 0 and t.total_ms >= t.kernel_ms
    assert np.array_equal(h_out.numpy().view(np.uint32), run_extend(ctx, data))


def test_extend_host_pageable_buffers(ctx):
    side, cols = 128, 128 * 128
    data = O.seeded_input(side, cols, seed=13)
    h_in = torch.from_numpy(data.view(np.int32).copy())  # not pinned
    h_out = torch.full((2 * side, cols), -1, dtype=torch.int32)
    ctx.extend_host(h_in, h_out, side, cols)
    assert np.array_equal(h_out.numpy().view(np.uint32), O.encode_rowmajor(data))


def test_extend_rejects_bad_arguments(ctx):
    import zoda_b200
    a = torch.zeros((4, 64), dtype=torch.int32, device="cuda")
    b = torch.zeros((8, 64), dtype=torch.int32, device="cuda")
    with pytest.raises(zoda_b200.ZodaError) as e:
        ctx.extend(a, b, 3, 64)  # k not a power of two
    assert e.value.status == 1
    with pytest.raises(zoda_b200.ZodaError) as e:
        ctx.extend(a, b, 4, 62)  # cols not a multiple of 4
    assert e.value.status == 1
    with pytest.raises(zoda_b200.ZodaError) as e:
        ctx.extend(a, b, 1 << 27, 4)  # beyond the largest side (2^26)
    assert e.value.status == 4
    with pytest.raises(zoda_b200.ZodaError):
        ctx.extend(a, a, 2, 64)  # output overlaps input
