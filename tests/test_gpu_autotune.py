"""Launch plans and the autotuner (zoda_autotune, zoda_plan_*), through the C ABI.

Every plan the tuner can choose must give the same bits as the oracle (the
reference's encode, src/benchmarks/utils.rs:100-146 with src/ntt/cpu.rs
transforms): each candidate is installed by hand and checked, at sizes where a
CTA gets several tiles so that both tile orders are exercised."""
import functools
import json

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import zoda_b200
    c = zoda_b200.Context(0)
    yield c
    c.close()


def to_dev(a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def tile_cols(side: int) -> int:
    return 2048 if side <= 16 else 32768 // side


def shape(side: int):
    c = tile_cols(side)
    return side, (c * 300 + 12 if side >= 16 else c * 150 + 12)


@functools.lru_cache(maxsize=None)
def case(side: int):
    k, cols = shape(side)
    data = O.seeded_input(k, cols, seed=1000 + side)
    return data, O.encode_rowmajor(data)


def plans_for(side: int):
    ls = side.bit_length() - 1
    out = []
    for blocked in (0, 1):
        for sched in ((0, 1) if ls >= 5 and ls % 4 else (0,)):
            out.append(dict(impl=1, sched=sched, l2_promo=3, blocked=blocked, stagger=1))
        if ls >= 6:
            for sched in ((0, 1) if ls % 3 else (0,)):
                out.append(dict(impl=1, sched=sched, l2_promo=3, blocked=blocked, stagger=1, radix=8))
        if ls >= 5:
            for radix in (16, 8):
                for promo in (3, 2, 0):
                    for stagger in (1, 2, 3, 0):
                        out.append(dict(impl=2, sched=0, l2_promo=promo, blocked=blocked, stagger=stagger,
                                        radix=radix))
    return out


CASES = [(s, i, p) for s in (1, 2, 16, 32, 64, 128, 512, 1024, 2048, 4096) for i, p in enumerate(plans_for(s))]


@pytest.mark.parametrize("side,i,plan", CASES, ids=[f"side{s}-{i}" for s, i, _ in CASES])
def test_every_plan_is_bit_exact(ctx, side, i, plan):
    data, want = case(side)
    k, cols = data.shape
    ctx.plan_set(side, plan)
    try:
        d_in = to_dev(data)
        d_out = torch.full((2 * k, cols), -1, dtype=torch.int32, device="cuda")
        ctx.extend(d_in, d_out, k, cols)
        torch.cuda.synchronize()
        ctx.check()
        got = d_out.cpu().numpy().view(np.uint32)
        assert np.array_equal(got, want), plan
    finally:
        ctx.plan_clear()


def test_autotune_installs_bit_exact_plans(ctx, tmp_path):
    plans = ctx.autotune(32, 256, cols=8192, reps=2)
    assert sorted(plans) == [32, 64, 128, 256]
    for side, p in plans.items():
        assert p["impl"] in (1, 2) and p["ms"] > 0
        got = ctx.plan_get(side)
        assert {k: v for k, v in got.items() if k != "ms"} == {k: v for k, v in p.items() if k != "ms"}
        data, want = case(side) if side >= 128 else (None, None)
        if data is not None:
            k, cols = data.shape
            d_out = torch.empty((2 * k, cols), dtype=torch.int32, device="cuda")
            ctx.extend(to_dev(data), d_out, k, cols)
            torch.cuda.synchronize()
            assert np.array_equal(d_out.cpu().numpy().view(np.uint32), want)
    path = tmp_path / "plans.json"
    ctx.save_plans(str(path))
    saved = json.loads(path.read_text())
    assert sorted(int(s) for s in saved) == [32, 64, 128, 256]
    ctx.plan_clear()
    assert ctx.plan_get(64) is None
    ctx.load_plans(str(path))
    assert ctx.plan_get(64)["impl"] == plans[64]["impl"]
    ctx.plan_clear()


def test_plan_errors(ctx):
    import zoda_b200
    with pytest.raises(zoda_b200.ZodaError):
        ctx.plan_set(16, dict(impl=2, sched=0, l2_promo=3, blocked=0, stagger=1))  # TMA needs side >= 32
    with pytest.raises(zoda_b200.ZodaError):
        ctx.plan_set(64, dict(impl=3, sched=0, l2_promo=3, blocked=0, stagger=1))
    with pytest.raises(zoda_b200.ZodaError):
        ctx.plan_set(64, dict(impl=2, sched=0, l2_promo=4, blocked=0, stagger=1))
    with pytest.raises(zoda_b200.ZodaError):
        ctx.plan_set(48, dict(impl=1, sched=0, l2_promo=3, blocked=0, stagger=1))  # not a power of two
    with pytest.raises(zoda_b200.ZodaError):
        ctx.plan_set(64, dict(impl=2, sched=0, l2_promo=3, blocked=0, stagger=1, radix=4))
    with pytest.raises(zoda_b200.ZodaError):
        ctx.plan_set(32, dict(impl=1, sched=0, l2_promo=3, blocked=0, stagger=1, radix=8))  # direct radix 8 from 64
    with pytest.raises(zoda_b200.ZodaError):
        ctx.autotune(64, 32)
    assert ctx.plan_get(1024) is None


def test_batch_follows_the_side_promotion(ctx):
    import zoda_b200
    sides = [64, 256, 64, 128]
    datas = [O.seeded_input(s, 4 * tile_cols(s) + 4, seed=70 + i) for i, s in enumerate(sides)]
    ins = [to_dev(d) for d in datas]
    outs = [torch.empty((2 * d.shape[0], d.shape[1]), dtype=torch.int32, device="cuda") for d in datas]
    for s in (64, 128, 256):
        ctx.plan_set(s, dict(impl=2, sched=0, l2_promo=0, blocked=0, stagger=1))
    try:
        b = zoda_b200.Batch(ctx, [(i, o, d.shape[0], d.shape[1]) for i, o, d in zip(ins, outs, datas)])
        b.run()
        torch.cuda.synchronize()
        b.close()
        for d, o in zip(datas, outs):
            assert np.array_equal(o.cpu().numpy().view(np.uint32), O.encode_rowmajor(d))
    finally:
        ctx.plan_clear()


@pytest.mark.parametrize("radix", [16, 8])
def test_batch_runs_the_largest_sides_radix(ctx, radix):
    import zoda_b200
    sides = [32, 2048, 64, 512, 128, 1024, 256]
    datas = [O.seeded_input(s, 3 * tile_cols(s) + 4, seed=90 + i) for i, s in enumerate(sides)]
    ins = [to_dev(d) for d in datas]
    outs = [torch.empty((2 * d.shape[0], d.shape[1]), dtype=torch.int32, device="cuda") for d in datas]
    ctx.plan_set(2048, dict(impl=2, sched=0, l2_promo=3, blocked=0, stagger=1, radix=radix))
    try:
        b = zoda_b200.Batch(ctx, [(i, o, d.shape[0], d.shape[1]) for i, o, d in zip(ins, outs, datas)])
        b.run()
        torch.cuda.synchronize()
        ctx.check()
        b.close()
        for d, o in zip(datas, outs):
            assert np.array_equal(o.cpu().numpy().view(np.uint32), O.encode_rowmajor(d)), d.shape
    finally:
        ctx.plan_clear()
