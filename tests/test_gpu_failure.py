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
