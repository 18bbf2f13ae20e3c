"""zoda_ntt_device_noalloc: the transform for callers that cannot allocate
device memory (a pool allocator owns it, or cudaMalloc's device-wide
synchronisation is not allowed on their path). It keeps its working copy in a
fixed array inside the library instead of allocating.

Checked through the C ABI against the existing entry points cuda_ntt /
cuda_intt on the same inputs, bit-exact, over two calls in a row (the array
keeps the previous call's contents, so the second call must not see them),
and directly against the CPU oracle's restatement of the reference's
transform (src/ntt/cpu.rs:1-60), including the largest accepted request at
n = 2 (2^21 polynomials, more 32-row tiles than a grid's y dimension holds).
This file is collected last so that a run stopping at its first failure has
run every other test first; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = 2013265921
MAX_ELEMS = 4 << 20  # the library's fixed scratch, in u32


@pytest.fixture(scope="module")
def zb():
    import zoda_b200
    zoda_b200.load()
    return zoda_b200


def reference_entry(zb, values: np.ndarray, n: int, inverse: bool) -> np.ndarray:
    """The existing entry point (host buffer, stride = n) on a copy."""
    out = np.ascontiguousarray(values, dtype=np.uint32).copy()
    (zb.intt_cuda if inverse else zb.ntt_cuda)(out, n, n)
    return out


def noalloc(zb, values: np.ndarray, n: int, polys: int, inverse: bool, in_place: bool = False) -> np.ndarray:
    d_in = torch.from_numpy(values.view(np.int32)).cuda()
    d_out = d_in if in_place else torch.empty_like(d_in)
    rc = zb.load().zoda_ntt_device_noalloc(d_in.data_ptr(), d_out.data_ptr(), n, polys, int(inverse), None)
    assert rc == 0, zb.load().zoda_last_error().decode()
    torch.cuda.synchronize()
    return d_out.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("n,polys", [(2, 37), (16, 101), (256, 1000), (4096, 1024), (1024, 4093)])
@pytest.mark.parametrize("inverse", [False, True])
def test_noalloc_matches_existing_entry_two_calls(zb, n, polys, inverse):
    assert n * ((polys + 3) // 4 * 4) <= MAX_ELEMS
    rng = np.random.default_rng(n * 7 + polys + int(inverse))
    for call in range(2):  # two calls in a row, different data
        vals = rng.integers(0, P, n * polys, dtype=np.uint32)
        got = noalloc(zb, vals, n, polys, inverse, in_place=(call == 1))
        want = reference_entry(zb, vals, n, inverse)
        assert np.array_equal(got, want), f"call {call}"


@pytest.mark.parametrize("n,polys", [(2, 2097152), (2, 2097149), (4, 1048573), (8, 1000), (4096, 1021)])
@pytest.mark.parametrize("inverse", [False, True])
def test_noalloc_matches_oracle(zb, n, polys, inverse):
    # the CPU oracle (src/ntt/cpu.rs restated), up to the array's limit: n * round_up(polys, 4) = 4 Mi u32
    assert n * ((polys + 3) // 4 * 4) <= MAX_ELEMS
    rng = np.random.default_rng(n + polys + 11 * int(inverse))
    for call in range(2):
        vals = rng.integers(0, P, n * polys, dtype=np.uint32)
        got = noalloc(zb, vals, n, polys, inverse)
        assert np.array_equal(got, O.ntt_polys(vals, n, n, inverse)), f"call {call}"


def test_noalloc_rejects_requests_beyond_its_array(zb):
    lib = zb.load()
    d = torch.empty(8, dtype=torch.int32, device="cuda")
    # 4096 * 1028 u32 is more than the 4194304-element array
    assert lib.zoda_ntt_device_noalloc(d.data_ptr(), d.data_ptr(), 4096, 1025, 0, None) == 4
    assert b"exceeds" in lib.zoda_last_error()
    # one polynomial past the limit at n = 2
    assert lib.zoda_ntt_device_noalloc(d.data_ptr(), d.data_ptr(), 2, 2097153, 0, None) == 4
    assert lib.zoda_ntt_device_noalloc(d.data_ptr(), d.data_ptr(), 8192, 1, 0, None) == 4
    assert lib.zoda_ntt_device_noalloc(d.data_ptr(), d.data_ptr(), 48, 1, 0, None) == 1
