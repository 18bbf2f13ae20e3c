"""Failure detection on the GPU without a fault: a kernel's bounded barrier wait
runs out (nothing completes the barrier), the kernel flags it and returns, the
context reports ZODA_ERR_TIMEOUT once and stays usable."""
import numpy as np
import pytest

import oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ZODA_ERR_TIMEOUT = 6


def test_bounded_wait_is_reported_and_the_context_survives():
    import zoda_b200
    c = zoda_b200.Context(0)
    try:
        c.check()  # clean start
        c.selftest_bounded_wait()
        with pytest.raises(zoda_b200.ZodaError) as e:
            c.check()
        assert e.value.status == ZODA_ERR_TIMEOUT
        c.check()  # the flag was cleared
        # the context still works: a small extension, bit-exact against the oracle
        data = O.seeded_input(64, 512, seed=3)
        d_in = torch.from_numpy(data.view(np.int32)).cuda()
        d_out = torch.empty((128, 512), dtype=torch.int32, device="cuda")
        c.extend(d_in, d_out, 64, 512)
        torch.cuda.synchronize()
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), O.encode_rowmajor(data))
        c.check()
    finally:
        c.close()


def test_host_call_error_returns_with_no_copy_outstanding():
    """A column chunk of zoda_extend_host fails mid-call (injected after two chunks
    have queued their copies): the call reports the failure only once every copy it
    queued has finished, so nothing lands in the caller's output after it returns;
    the next call on the same context is bit-exact."""
    import time

    import zoda_b200
    side, cols = 64, 1 << 20  # 256 MiB of input: four 64 MiB column chunks
    c = zoda_b200.Context(0)
    try:
        data = O.seeded_input(side, 4096, seed=8)
        h_in = torch.from_numpy(np.tile(data, (1, cols // 4096)).view(np.int32)).pin_memory()
        h_out = torch.zeros((2 * side, cols), dtype=torch.int32).pin_memory()
        c.inject_fault(1, after=2)
        with pytest.raises(zoda_b200.ZodaError) as e:
            c.extend_host(h_in, h_out, side, cols)
        assert e.value.status == 2 and "injected" in str(e.value)
        h_out.fill_(-7)  # after the return nothing may write here any more
        time.sleep(0.3)
        assert bool((h_out == -7).all())
        t = c.extend_host(h_in, h_out, side, cols)  # the fault disarmed itself
        want = O.encode_rowmajor(data)
        got = h_out.numpy().view(np.uint32)
        for c0 in (0, cols // 2, cols - 4096):
            assert np.array_equal(got[:, c0:c0 + 4096], want)
        assert t.h2d_bytes == side * cols * 4 and t.d2h_bytes >= side * cols * 4
    finally:
        c.close()


def test_pipelined_fourstep_wait_runs_out_and_the_context_survives():
    """The pipelined four-step launch (one persistent launch whose block-pass and
    pass-B tiles wait on per-chunk counts of finished tiles) is told to wait for one
    tile more than a chunk has (ZODA_FAULT_PIPE_WAIT): every wait runs out after
    about a second, each CTA flags the error and leaves, the context reports
    ZODA_ERR_TIMEOUT once, and the next launch is bit-exact again. No GPU fault:
    the waits are bounded polls of a counter in device memory."""
    import time

    import zoda_b200
    c = zoda_b200.Context(0)
    side, cols = 1024, 4096
    try:
        c.plan_set(side, {"impl": 3, "sched": 0, "l2_promo": 3, "blocked": 1, "stagger": 1, "radix": 8,
                          "ctas": 4})
        data = O.seeded_input(side, cols, seed=17)
        d_in = torch.from_numpy(data.view(np.int32)).cuda()
        d_out = torch.empty((2 * side, cols), dtype=torch.int32, device="cuda")
        c.check()
        c.inject_fault(2)
        t0 = time.perf_counter()
        c.extend(d_in, d_out, side, cols)
        torch.cuda.synchronize()
        elapsed = time.perf_counter() - t0
        with pytest.raises(zoda_b200.ZodaError) as e:
            c.check()
        assert e.value.status == ZODA_ERR_TIMEOUT
        assert elapsed < 30.0  # bounded: about a second of polling per CTA, the CTAs in parallel
        c.check()  # the flag was cleared
        c.extend(d_in, d_out, side, cols)  # the fault disarmed itself
        torch.cuda.synchronize()
        c.check()
        assert np.array_equal(d_out.cpu().numpy().view(np.uint32), O.encode_rowmajor(data))
    finally:
        c.plan_clear()
        c.close()
