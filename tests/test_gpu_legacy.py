"""The reference's FFI (cuda_ntt / cuda_intt / cuda_host_alloc / cuda_host_free)
through the C ABI: the reference's own GPU-vs-CPU tests (src/ntt/cuda.rs:133-237)
restated, plus a cross-check against the reference's CUDA kernel built from its
source (oracle/_ref/libntt_cuda_ref.so) when that build is present."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O

pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = O.P
REF_SO = os.path.join(os.path.dirname(O.__file__), "_ref", "libntt_cuda_ref.so")


@pytest.fixture(scope="module")
def zb():
    import zoda_b200
    zoda_b200.load()
    return zoda_b200


def sample(n):  # src/ntt/cuda.rs:138-140
    return (np.arange(n, dtype=np.uint64) * 7 + 3).astype(np.uint32)


def one_poly(zb, values):
    sq = zb.PinnedSquare(len(values), 1)
    sq.array[:] = values
    return sq


@pytest.mark.parametrize("log_n", [1, 4, 8, 12])
def test_cuda_ntt_vs_cpu(zb, log_n):
    # src/ntt/cuda.rs:150-164
    n = 1 << log_n
    sq = one_poly(zb, sample(n))
    zb.ntt_cuda(sq, n, n)
    assert np.array_equal(sq.array, O.ntt(sample(n)))


@pytest.mark.parametrize("log_n", [1, 4, 8, 12])
def test_cuda_intt_vs_cpu(zb, log_n):
    # src/ntt/cuda.rs:166-180
    n = 1 << log_n
    sq = one_poly(zb, sample(n))
    zb.intt_cuda(sq, n, n)
    assert np.array_equal(sq.array, O.intt(sample(n)))


def test_cuda_roundtrip(zb):
    # src/ntt/cuda.rs:182-192
    n = 1 << 10
    sq = one_poly(zb, sample(n))
    zb.ntt_cuda(sq, n, n)
    zb.intt_cuda(sq, n, n)
    assert np.array_equal(sq.array, sample(n))


def test_cuda_many_columns_vs_cpu(zb):
    # src/ntt/cuda.rs:194-214: 37 columns of n = 256, value row*31 + col*7 + 1
    n, cols = 1 << 8, 37
    sq = zb.PinnedSquare(n, cols)
    for col in range(cols):
        sq.column(col)[:] = np.arange(n, dtype=np.uint32) * 31 + col * 7 + 1
    before = sq.array.copy()
    zb.ntt_cuda(sq, n, n)
    for col in range(cols):
        assert np.array_equal(sq.column(col), O.ntt(before[col * n:(col + 1) * n]))


def test_cuda_strided_vs_cpu(zb):
    # src/ntt/cuda.rs:216-237: n = 64 inside stride = 256, rows >= n untouched
    n, stride, cols = 1 << 6, 1 << 8, 5
    sq = zb.PinnedSquare(stride, cols)
    for col in range(cols):
        sq.column(col)[:] = np.arange(stride, dtype=np.uint32) * 13 + col * 3 + 2
    before = sq.array.copy()
    zb.ntt_cuda(sq, n, stride)
    assert np.array_equal(sq.array, O.ntt_polys(before, n, stride, inverse=False))
    for col in range(cols):
        assert np.array_equal(sq.column(col)[n:], before[col * stride + n:(col + 1) * stride])


@pytest.mark.parametrize("log_n", [0, 2, 3, 5, 7, 9, 11])
@pytest.mark.parametrize("inverse", [False, True])
def test_legacy_seeded_many_polys(zb, log_n, inverse):
    n = 1 << log_n
    polys, stride = 203, n + 3
    rng = np.random.default_rng(log_n)
    vals = rng.integers(0, P, polys * stride, dtype=np.uint32)
    got = vals.copy()
    (zb.intt_cuda if inverse else zb.ntt_cuda)(got, n, stride)
    assert np.array_equal(got, O.ntt_polys(vals, n, stride, inverse))


@pytest.mark.parametrize("log_n,polys", [(1, (1 << 21) + 5), (2, (1 << 22) + 3)])
def test_legacy_many_short_polys(zb, log_n, polys):
    # more than 65535 32-polynomial tiles in one device chunk (the transposes walk them with a grid stride)
    n = 1 << log_n
    rng = np.random.default_rng(polys)
    vals = rng.integers(0, P, polys * n, dtype=np.uint32)
    for inverse in (False, True):
        got = vals.copy()
        (zb.intt_cuda if inverse else zb.ntt_cuda)(got, n, n)
        assert np.array_equal(got, O.ntt_polys(vals, n, n, inverse))


def test_legacy_zoda_extend_two_calls(zb):
    # src/zoda/babybear.rs:34-39 GPU branch: intt over n_k inside n_kn-tall columns, then ntt over n_kn
    k, cols = 32, 40
    n_kn = 2 * k
    data = O.seeded_input(k, cols, seed=4)
    sq = zb.PinnedSquare(n_kn, cols)
    for c in range(cols):
        sq.column(c)[:k] = data[:, c]
    zb.intt_cuda(sq, k, n_kn)
    zb.ntt_cuda(sq, n_kn, n_kn)
    want = O.encode_rowmajor(data)
    got = sq.array.reshape(cols, n_kn).T
    assert np.array_equal(got, want)


def test_legacy_non_standard_root(zb):
    # any primitive n-th root works: w = omega^3
    n = 256
    w = pow(int(O.roots_of_unity(n)[1]), 3, P)
    roots = np.array([pow(w, i, P) for i in range(n)], dtype=np.uint32)
    v = O.seeded_input(1, n, seed=2)[0]
    got = v.copy()
    zb.ntt_cuda(got, n, n, roots=roots)
    assert np.array_equal(got, O.ntt(v, roots))
    got2 = v.copy()
    zb.intt_cuda(got2, n, n, roots=roots)
    assert np.array_equal(got2, O.intt(v, roots))


def test_legacy_bad_arguments(zb):
    lib = zb.load()
    v = np.zeros(64, dtype=np.uint32)
    roots = O.roots_of_unity(64)
    assert lib.cuda_ntt(v.ctypes.data, roots.ctypes.data, 48, 1, 64) == 1      # n not a power of two
    assert lib.cuda_ntt(v.ctypes.data, roots.ctypes.data, 64, 1, 32) == 1      # stride < n
    bad = roots.copy()
    bad[5] ^= 1
    assert lib.cuda_ntt(v.ctypes.data, bad.ctypes.data, 64, 1, 64) == 1       # not a root table
    assert lib.cuda_ntt(v.ctypes.data, roots.ctypes.data, 64, 0, 64) == 0      # nothing to do


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference CUDA build not present")
@pytest.mark.parametrize("log_n", [3, 8, 11])
@pytest.mark.parametrize("inverse", [False, True])
def test_legacy_matches_reference_cuda_kernel(zb, log_n, inverse):
    ref = ctypes.CDLL(REF_SO)
    ref.cuda_ntt.argtypes = ref.cuda_intt.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_uint32] * 3
    n, polys = 1 << log_n, 1500
    stride = 2 * n
    vals = O.seeded_input(1, polys * stride, seed=log_n + 50)[0]
    roots = O.roots_of_unity(n)
    a = vals.copy()
    b = vals.copy()
    fn = ref.cuda_intt if inverse else ref.cuda_ntt
    assert fn(a.ctypes.data, roots.ctypes.data, n, polys, stride) == 0
    (zb.intt_cuda if inverse else zb.ntt_cuda)(b, n, stride)
    assert np.array_equal(a, b)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference CUDA build not present")
@pytest.mark.parametrize("side,cols", [(64, 8192), (1024, 2048)])
def test_fused_extension_matches_reference_cuda_encode(zb, side, cols):
    """The reference's GPU encode window (src/benchmarks/utils.rs:114-140: column-major
    square, zero rows k..2k, intt_cuda over k rows, ntt_cuda over 2k) run by the reference's
    own CUDA kernel, against the fused extension kernel, on the same seeded input."""
    import torch
    ref = ctypes.CDLL(REF_SO)
    ref.cuda_ntt.argtypes = ref.cuda_intt.argtypes = [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_uint32] * 3
    data = O.seeded_input(side, cols, seed=side + 7)
    square = np.zeros((cols, 2 * side), dtype=np.uint32)  # column c at square[c]
    square[:, :side] = data.T
    assert ref.cuda_intt(square.ctypes.data, O.roots_of_unity(side).ctypes.data, side, cols, 2 * side) == 0
    assert ref.cuda_ntt(square.ctypes.data, O.roots_of_unity(2 * side).ctypes.data, 2 * side, cols, 2 * side) == 0
    ctx = zb.Context(0)
    d_in = torch.from_numpy(data.view(np.int32)).cuda()
    d_out = torch.empty((2 * side, cols), dtype=torch.int32, device="cuda")
    ctx.extend(d_in, d_out, side, cols)
    torch.cuda.synchronize()
    ctx.close()
    assert np.array_equal(d_out.cpu().numpy().view(np.uint32), square.T)
