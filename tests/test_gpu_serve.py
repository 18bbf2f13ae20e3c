"""The serving loop (zoda_server_*): requests submitted while others run are
batched together and overlap on the GPU; each result must be bit-exact with the
same square encoded alone (zoda_extend_device)."""
import threading
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

P = 2013265921


@pytest.fixture(scope="module")
def ctx():
    import zoda_b200
    c = zoda_b200.Context(0)
    yield c
    c.close()


def as_u32(t):
    return t.cpu().numpy().view(np.uint32)


def test_results_same_alone_and_in_the_mix(ctx):
    import zoda_b200
    rng = np.random.default_rng(11)
    # three large squares first (about 1.4 ms of GPU work each) fill the server's
    # three launch slots, so the burst behind them waits and is batched whatever
    # the host's speed; then 48 squares of random sides
    sides = [2048] * 3 + [int(2 ** rng.integers(5, 12)) for _ in range(48)]
    inputs = []
    for i, s in enumerate(sides):
        cols = 131072 if i < 3 else 4 * int(rng.integers(1, 1 + 262144 // (4 * s)))
        inputs.append(torch.randint(0, P, (s, cols), dtype=torch.int64, device="cuda").to(torch.int32))
    torch.cuda.synchronize()
    srv = zoda_b200.Server(ctx, budget_bytes=8 << 30, max_inflight=3, max_batch=16)
    tickets = [None] * len(sides)

    def producer():  # a burst (more requests than streams), then Poisson-like arrivals
        for i, (s, a) in enumerate(zip(sides, inputs)):
            tickets[i] = srv.submit(a, s, a.shape[1])
            if i >= 27:
                time.sleep(float(rng.exponential(0.0005)))

    th = threading.Thread(target=producer)
    th.start()
    th.join()
    for i, (s, a) in enumerate(zip(sides, inputs)):
        info = srv.wait(tickets[i])
        assert info.status == 0 and info.latency_ms >= info.queue_ms >= 0
        served = torch.empty((2 * s, a.shape[1]), dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        zoda_b200.device_copy(served, info.d_out, served.numel() * 4)  # out of the arena
        srv.release(tickets[i])
        alone = torch.empty_like(served)
        ctx.extend(a, alone, s, a.shape[1])  # the same square encoded alone
        torch.cuda.synchronize()
        assert torch.equal(served, alone), f"request {i} side {s}"
    st = srv.stats()
    assert st.completed == len(sides) and st.launches >= 1
    assert st.launches < len(sides)  # requests were batched
    assert 0 < st.p50_ms <= st.p99_ms <= st.max_ms
    srv.close()


def test_budget_admission_and_cancel(ctx):
    import zoda_b200
    srv = zoda_b200.Server(ctx, budget_bytes=48 << 20, max_inflight=1, max_batch=4)
    big = torch.zeros((1024, 8192), dtype=torch.int32, device="cuda")
    with pytest.raises(zoda_b200.ZodaError) as e:
        srv.submit(big, 1024, 8192)  # its 64 MiB output can never fit the 48 MiB budget
    assert e.value.status == 5
    a = torch.zeros((256, 8192), dtype=torch.int32, device="cuda")  # 16 MiB output each
    tk = [srv.submit(a, 256, 8192) for _ in range(12)]
    # at most 3 outputs fit the budget at once; the last request is normally still queued
    try:
        srv.cancel(tk[-1])
        cancelled = True
    except zoda_b200.ZodaError as err:
        assert err.status == 8
        cancelled = False
    for t in tk[:-1]:
        srv.wait(t)
        srv.release(t)
    if cancelled:
        with pytest.raises(zoda_b200.ZodaError) as e:
            srv.wait(tk[-1])
        assert e.value.status == 7
    st = srv.stats()
    assert st.completed >= 11
    srv.close()


def test_server_rejects_bad_requests(ctx):
    import zoda_b200
    srv = zoda_b200.Server(ctx, budget_bytes=16 << 20)
    a = torch.zeros((16, 64), dtype=torch.int32, device="cuda")
    for k, cols in ((16, 64), (48, 64), (32, 62), (4096, 64)):
        with pytest.raises(zoda_b200.ZodaError) as e:
            srv.submit(a, k, cols)
        assert e.value.status == 1
    srv.close()
