"""The batched extension (zoda_batch_*): many squares of mixed sides in one
persistent, graph-captured launch. Every square's output must equal the
single-square call's output (and the CPU oracle's), bit-exact."""
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


def tile_cols(side):
    return 32768 // side


def make_squares(sides, seed, ragged=True):
    rng = np.random.default_rng(seed)
    out = []
    for i, s in enumerate(sides):
        cols = tile_cols(s) * int(rng.integers(1, 4)) + (4 * int(rng.integers(0, 8)) if ragged else 0)
        data = rng.integers(0, P, size=(s, cols), dtype=np.uint32)
        d_in = torch.from_numpy(data.view(np.int32)).cuda()
        d_out = torch.full((2 * s, cols), -1, dtype=torch.int32, device="cuda")
        out.append((data, d_in, d_out))
    return out


def test_batch_mixed_sides_match_single_calls(ctx):
    import zoda_b200
    sides = [32, 2048, 64, 128, 1024, 256, 512, 32, 2048, 128, 64, 512]
    sq = make_squares(sides, seed=1)
    batch = zoda_b200.Batch(ctx, [(a, b, s, a.shape[1]) for (_, a, b), s in zip(sq, sides)])
    assert batch.elements == sum(s * a.shape[1] for (_, a, _), s in zip(sq, sides))
    batch.run()
    torch.cuda.synchronize()
    ctx.check()
    for (data, d_in, d_out), s in zip(sq, sides):
        single = torch.empty_like(d_out)
        ctx.extend(d_in, single, s, d_in.shape[1])
        torch.cuda.synchronize()
        assert torch.equal(d_out, single), f"side {s}"
    # a few against the CPU oracle directly
    for (data, _, d_out), s in list(zip(sq, sides))[:4]:
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), O.encode_rowmajor(data))
    batch.close()


def test_batch_replay_sees_new_inputs(ctx):
    import zoda_b200
    sides = [1024, 64, 256]
    sq = make_squares(sides, seed=2)
    batch = zoda_b200.Batch(ctx, [(a, b, s, a.shape[1]) for (_, a, b), s in zip(sq, sides)])
    batch.run()
    rng = np.random.default_rng(3)
    fresh = []
    for (_, d_in, _), s in zip(sq, sides):
        new = rng.integers(0, P, size=tuple(d_in.shape), dtype=np.uint32)
        d_in.copy_(torch.from_numpy(new.view(np.int32)))
        fresh.append(new)
    batch.run()  # graph replay with the same buffers, new contents
    torch.cuda.synchronize()
    ctx.check()
    for new, (_, _, d_out) in zip(fresh, sq):
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), O.encode_rowmajor(new))
    batch.close()


def test_batch_single_tile_squares_and_empty(ctx):
    import zoda_b200
    sides = [32] * 7 + [64] * 5
    sq = make_squares(sides, seed=4, ragged=False)
    batch = zoda_b200.Batch(ctx, [(a, b, s, a.shape[1]) for (_, a, b), s in zip(sq, sides)])
    batch.run()
    torch.cuda.synchronize()
    for (data, _, d_out), s in zip(sq, sides):
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), O.encode_rowmajor(data))
    batch.close()
    empty = zoda_b200.Batch(ctx, [])
    empty.run()
    empty.close()


def test_batch_rejects_unsupported_sides(ctx):
    import zoda_b200
    a = torch.zeros((16, 64), dtype=torch.int32, device="cuda")
    b = torch.zeros((32, 64), dtype=torch.int32, device="cuda")
    with pytest.raises(zoda_b200.ZodaError) as e:
        zoda_b200.Batch(ctx, [(a, b, 16, 64)])
    assert e.value.status == 4
    with pytest.raises(zoda_b200.ZodaError) as e:
        zoda_b200.Batch(ctx, [(a, b, 12, 64)])
    assert e.value.status == 1
