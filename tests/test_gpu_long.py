"""Columns longer than 4096 rows: the four-step passes (csrc/fourstep.cu) behind the
C ABI, bit-exact against the oracle (the reference's src/ntt/cpu.rs restated) and
against the reference's own CUDA kernel built from its source.

* cuda_ntt / cuda_intt at n = 8192 .. 131072 (the reference has no size cap,
  cuda/ntt_kernel.cu:106-160), strided, with a non-standard root;
* zoda_extend_device above side 4096, and the four-step plan at sides 1024 ..
  4096 in every launch shape (also through the host-buffer call);
* the reference's validated configurations (src/benchmarks/zoda_validated.rs:
  105-126): k = n = 32768 and k = n = 65536 on a 1024-column window
  (row_size 4096 B), every encoded row RLC-checked on the device and sampled
  columns re-encoded by the oracle; and uneven (k, n) with n_k > 4096;
* zoda_recover_device for k = 8192 and 32768 with a random half erased."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = O.P
REF_SO = os.path.join(os.path.dirname(O.__file__), "_ref", "libntt_cuda_ref.so")


@pytest.fixture(scope="module")
def zb():
    import zoda_b200
    zoda_b200.load()
    return zoda_b200


@pytest.fixture(scope="module")
def ctx(zb):
    c = zb.Context(0)
    yield c
    c.close()


@pytest.fixture(autouse=True)
def no_wait_gave_up(request):
    """After every test that used the context: no bounded wait ran out."""
    yield
    if "ctx" in request.fixturenames:
        request.getfixturevalue("ctx").check()


def to_dev(a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32)).cuda()


def from_dev(t) -> np.ndarray:
    return t.cpu().numpy().view(np.uint32)


def rand_dev(rows: int, cols: int, seed: int):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    out = torch.empty((rows, cols), dtype=torch.int32, device="cuda")
    for r0 in range(0, rows, 8192):
        r1 = min(rows, r0 + 8192)
        out[r0:r1] = torch.randint(0, P, (r1 - r0, cols), dtype=torch.int64, device="cuda",
                                   generator=gen).to(torch.int32)
    return out


# ---- the reference's FFI above 4096 points ------------------------------------

@pytest.mark.parametrize("log_n", [13, 15, 17])
@pytest.mark.parametrize("inverse", [False, True])
def test_long_legacy_matches_oracle(zb, log_n, inverse):
    n, polys = 1 << log_n, 3
    stride = n + 8  # rows n .. stride of every polynomial must stay untouched
    vals = np.random.default_rng(log_n * 2 + inverse).integers(0, P, polys * stride, dtype=np.uint32)
    got = vals.copy()
    (zb.intt_cuda if inverse else zb.ntt_cuda)(got, n, stride)
    assert np.array_equal(got, O.ntt_polys(vals, n, stride, inverse))


def test_long_legacy_non_standard_root(zb):
    n = 1 << 14
    w = pow(int(O.roots_of_unity(n)[1]), 3, P)
    roots = np.array([pow(w, i, P) for i in range(n)], dtype=np.uint32)
    v = O.seeded_input(1, n, seed=12)[0]
    got = v.copy()
    zb.ntt_cuda(got, n, n, roots=roots)
    assert np.array_equal(got, O.ntt(v, roots))
    got2 = v.copy()
    zb.intt_cuda(got2, n, n, roots=roots)
    assert np.array_equal(got2, O.intt(v, roots))


def test_long_legacy_many_polys(zb):
    # more polynomials than one 128 MiB device chunk holds at n = 16384 (2048 per chunk)
    n, polys = 1 << 14, 2500
    vals = np.random.default_rng(3).integers(0, P, polys * n, dtype=np.uint32)
    got = vals.copy()
    zb.ntt_cuda(got, n, n)
    assert np.array_equal(got, O.ntt_polys(vals, n, n, False))


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference CUDA build not present")
@pytest.mark.parametrize("log_n", [14, 17])
@pytest.mark.parametrize("inverse", [False, True])
def test_long_legacy_matches_reference_cuda_kernel(zb, log_n, inverse):
    ref = ctypes.CDLL(REF_SO)
    ref.cuda_ntt.argtypes = ref.cuda_intt.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_uint32] * 3
    n, polys = 1 << log_n, 6
    vals = O.seeded_input(1, polys * n, seed=log_n + 90)[0]
    roots = O.roots_of_unity(n)
    a, b = vals.copy(), vals.copy()
    fn = ref.cuda_intt if inverse else ref.cuda_ntt
    assert fn(a.ctypes.data, roots.ctypes.data, n, polys, n) == 0
    (zb.intt_cuda if inverse else zb.ntt_cuda)(b, n, n)
    assert np.array_equal(a, b)


# ---- the extension above side 4096, and the four-step plan ----------------------

@pytest.mark.parametrize("side,cols", [(8192, 64), (16384, 36), (65536, 4)])
def test_long_extension_matches_oracle(ctx, side, cols):
    data = O.seeded_input(side, cols, seed=side + cols)
    d_out = torch.full((2 * side, cols), -1, dtype=torch.int32, device="cuda")
    ctx.extend(to_dev(data), d_out, side, cols)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(d_out), O.encode_rowmajor(data))


FOURSTEP_SHAPES = [(16, 1), (16, 2), (8, 2), (8, 4), (4, 5)]


# plan forms: (sched, blocked) = three launches, three staged launches (cp.async
# prefetch of each next tile), one pipelined launch, one pipelined launch with the
# next pass-A tile staged
FORMS = {"three-launches": (0, 0), "staged": (1, 0), "pipelined": (0, 1), "staged-pipelined": (1, 1)}
FOURSTEP_PLANS = [(f, r, c) for f in FORMS for r, c in FOURSTEP_SHAPES if not (FORMS[f][0] == 1 and c == 1)]


@pytest.mark.parametrize("side", [1024, 2048, 4096])
@pytest.mark.parametrize("form,radix,ctas", FOURSTEP_PLANS)
def test_fourstep_plan_matches_oracle(ctx, side, form, radix, ctas):
    sched, blocked = FORMS[form]
    plan = {"impl": 3, "sched": sched, "l2_promo": 3, "blocked": blocked, "stagger": 1, "radix": radix,
            "ctas": ctas}
    cols = 1024 + 36  # ragged: not a whole number of tiles (the pipeline's last chunk is partial)
    data = O.seeded_input(side, cols, seed=side + radix + ctas + 3 * sched + blocked)
    ctx.plan_set(side, plan)
    try:
        d_out = torch.full((2 * side, cols), -1, dtype=torch.int32, device="cuda")
        ctx.extend(to_dev(data), d_out, side, cols)
        torch.cuda.synchronize()
        got = from_dev(d_out)
    finally:
        ctx.plan_clear()
    assert np.array_equal(got, O.encode_rowmajor(data))


@pytest.mark.parametrize("side", [1024, 2048, 4096])
@pytest.mark.parametrize("form,radix,ctas", [p for p in FOURSTEP_PLANS if p[0] != "three-launches"])
def test_fourstep_many_tiles(ctx, side, form, radix, ctas):
    # the pipelined launch over hundreds of column chunks (many rounds of its work
    # queue, chunks' passes overlapping), and the staged passes over many tiles per
    # CTA, against the single-pass default plan, which the tests above pin to the oracle
    sched, blocked = FORMS[form]
    cols = 65536 + 36
    d_in = rand_dev(side, cols, seed=side + 7 * radix + ctas)
    want = torch.empty((2 * side, cols), dtype=torch.int32, device="cuda")
    ctx.extend(d_in, want, side, cols)
    ctx.plan_set(side, {"impl": 3, "sched": sched, "l2_promo": 3, "blocked": blocked, "stagger": 1, "radix": radix,
                        "ctas": ctas})
    try:
        for _ in range(2):  # twice: the second launch starts from counters the first one left
            got = torch.full((2 * side, cols), -1, dtype=torch.int32, device="cuda")
            ctx.extend(d_in, got, side, cols)
            torch.cuda.synchronize()
            assert torch.equal(got, want)
    finally:
        ctx.plan_clear()


@pytest.mark.parametrize("form", list(FORMS))
def test_fourstep_plan_host_call(ctx, form):
    # the host-buffer call runs the plan on odd rows only (the even rows are copied on the host)
    side, cols = 4096, 512
    sched, blocked = FORMS[form]
    ctx.plan_set(side, {"impl": 3, "sched": sched, "l2_promo": 3, "blocked": blocked, "stagger": 1, "radix": 8,
                        "ctas": 2})
    try:
        data = O.seeded_input(side, cols, seed=31)
        h_in = torch.from_numpy(data.view(np.int32)).pin_memory()
        h_out = torch.full((2 * side, cols), -1, dtype=torch.int32).pin_memory()
        ctx.extend_host(h_in, h_out, side, cols)
    finally:
        ctx.plan_clear()
    assert np.array_equal(h_out.numpy().view(np.uint32), O.encode_rowmajor(data))


def test_long_extension_host_call(ctx):
    side, cols = 8192, 256
    data = O.seeded_input(side, cols, seed=41)
    h_in = torch.from_numpy(data.view(np.int32)).pin_memory()
    h_out = torch.full((2 * side, cols), -1, dtype=torch.int32).pin_memory()
    ctx.extend_host(h_in, h_out, side, cols)
    assert np.array_equal(h_out.numpy().view(np.uint32), O.encode_rowmajor(data))


def test_fourstep_encode_with_cut_rows_takes_default_plan(ctx):
    # an encode of fewer rows than 2 n_k cannot use the odd rows as scratch: the
    # four-step plan falls back to the side's default kernel, same bits
    k, n, cols = 3000, 3000, 72
    ctx.plan_set(4096, {"impl": 3, "sched": 0, "l2_promo": 3, "blocked": 0, "stagger": 1, "radix": 16, "ctas": 2})
    try:
        data = O.seeded_input(k, cols, seed=51)
        d_out = torch.empty((k + n, cols), dtype=torch.int32, device="cuda")
        ctx.encode(to_dev(data), d_out, k, n, cols)
        torch.cuda.synchronize()
    finally:
        ctx.plan_clear()
    assert np.array_equal(from_dev(d_out), O.encode_rowmajor(data, n))


# ---- the reference's validated configurations ------------------------------------

@pytest.mark.parametrize("k", [32768, 65536])
def test_validated_config_row_size_4096(ctx, k):
    """src/benchmarks/zoda_validated.rs:105-126: k = n (32768 and 65536), row_size 4096 B = 1024
    columns. Every encoded row passes the device RLC check, the even rows are the data, and
    sampled columns equal the oracle's re-encode."""
    cols = 1024
    d_in = rand_dev(k, cols, seed=k)
    d_out = torch.empty((2 * k, cols), dtype=torch.int32, device="cuda")
    ctx.encode(d_in, d_out, k, k, cols)
    torch.cuda.synchronize()
    assert torch.equal(d_out[0::2], d_in)
    coeff = torch.empty((cols, 4), dtype=torch.int32, device="cuda")
    ctx.rlc_coefficients(f"validated-{k}", cols, coeff)
    assert ctx.rlc_check(d_in, d_out, k, k, cols, coeff) == 0
    for c0 in (0, 508, cols - 4):
        data = d_in[:, c0:c0 + 4].contiguous().cpu().numpy().view(np.uint32)
        got = d_out[:, c0:c0 + 4].contiguous().cpu().numpy().view(np.uint32)
        assert np.array_equal(got, O.encode_rowmajor(data)), c0
    # one wrong value in one row is caught by the check
    d_out[2 * k - 3, 100] = (int(d_out[2 * k - 3, 100]) + 1) % P
    assert ctx.rlc_check(d_in, d_out, k, k, cols, coeff) == 4


LONG_SHAPES = [
    (5000, 3000),   # n_k 8192, n_kn 16384: one coset
    (8192, 100),    # n_kn 16384, rows cut right after the data
    (5000, 20000),  # n_kn 32768: three cosets
    (4097, 4000),   # k just past 4096
    (9000, 9000),   # n_k 16384, n_kn 32768
    (8191, 1),      # n_kn = n_k: the data and one zero row
]


@pytest.mark.parametrize("k,n", LONG_SHAPES, ids=[f"k{k}-n{n}" for k, n in LONG_SHAPES])
def test_long_encode_any_shape(ctx, k, n):
    cols = 36
    data = O.seeded_input(k, cols, seed=k * 3 + n)
    d_out = torch.full((k + n, cols), -1, dtype=torch.int32, device="cuda")
    ctx.encode(to_dev(data), d_out, k, n, cols)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(d_out), O.encode_rowmajor(data, n))


def test_long_encode_column_chunks(ctx):
    # n_k = 8192: a 256 MiB scratch chunk holds 8192 columns, so 8228 columns take two chunks
    k, n, cols = 6000, 5000, 8192 + 36
    data = O.seeded_input(k, cols, seed=61)
    d_out = torch.empty((k + n, cols), dtype=torch.int32, device="cuda")
    ctx.encode(to_dev(data), d_out, k, n, cols)
    torch.cuda.synchronize()
    got = from_dev(d_out)
    idx = np.r_[0:8, 8184:8200, cols - 8:cols]
    assert np.array_equal(got[:, idx], O.encode_rowmajor(np.ascontiguousarray(data[:, idx]), n))


# ---- the decoder above k = 4096 ------------------------------------------------------

@pytest.mark.parametrize("k,cols", [(8192, 64), (32768, 8)])
def test_long_recover_random_half(ctx, k, cols):
    data = O.seeded_input(k, cols, seed=k + 5)
    code = O.encode_rowmajor(data)
    rng = np.random.default_rng(k)
    known = np.sort(rng.choice(2 * k, size=k, replace=False))
    erased = np.setdiff1d(np.arange(2 * k), known)
    code[erased] = rng.integers(0, P, (len(erased), cols), dtype=np.uint32)  # garbage in the erased rows
    d_code = to_dev(code)
    out = torch.empty((k, cols), dtype=torch.int32, device="cuda")
    assert ctx.recover(d_code, known, k, cols, out, check=True) == 0
    assert np.array_equal(from_dev(out), data)


def test_long_recover_detects_inconsistent_rows(ctx):
    k, cols = 8192, 16
    data = O.seeded_input(k, cols, seed=71)
    code = O.encode_rowmajor(data)
    rng = np.random.default_rng(71)
    known = np.sort(rng.choice(2 * k, size=k + 32, replace=False))
    out = torch.empty((k, cols), dtype=torch.int32, device="cuda")
    assert ctx.recover(to_dev(code), known, k, cols, out, check=True) == 0
    assert np.array_equal(from_dev(out), data)
    code[known[7], 3] = (int(code[known[7], 3]) + 1) % P
    assert ctx.recover(to_dev(code), known, k, cols, out, check=True) > 0


def test_pipelined_plan_on_concurrent_streams(ctx):
    # Pipelined launches on different streams share the context's work-queue
    # counters; each waits for the one before (an event), so launches queued on
    # four streams at once, on four different squares, all come out right.
    side, cols = 2048, 8192 + 36
    ctx.plan_set(side, {"impl": 3, "sched": 0, "l2_promo": 3, "blocked": 1, "stagger": 1, "radix": 8, "ctas": 4})
    try:
        ins = [rand_dev(side, cols, seed=100 + i) for i in range(4)]
        wants = []
        for d_in in ins:  # the single-pass TMA plan, pinned to the oracle by the tests above
            w = torch.empty((2 * side, cols), dtype=torch.int32, device="cuda")
            ctx.set_impl(2)
            ctx.extend(d_in, w, side, cols)
            wants.append(w)
        ctx.set_impl(0)
        outs = [torch.full((2 * side, cols), -1, dtype=torch.int32, device="cuda") for _ in ins]
        streams = [torch.cuda.Stream() for _ in ins]
        torch.cuda.synchronize()  # inputs, references and filled outputs are ready before the other streams run
        for st, d_in, d_out in zip(streams, ins, outs):
            ctx.extend(d_in, d_out, side, cols, stream=st)
        torch.cuda.synchronize()
        for d_out, w in zip(outs, wants):
            assert torch.equal(d_out, w)
    finally:
        ctx.set_impl(0)
        ctx.plan_clear()
