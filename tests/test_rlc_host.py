"""The library's host SHA-256 data root (zoda_data_root_host) against the
oracle's compute_data_root (src/benchmarks/utils.rs:51-59, hashlib). Runs on
CPU: the call touches no GPU."""
import numpy as np
import pytest

import oracle as O


@pytest.mark.parametrize("shape", [(1, 1), (1, 13), (1, 14), (1, 16), (1, 15), (3, 5), (64, 8192), (1100, 1024),
                                   (2, 524289)])
def test_data_root_matches_oracle(lib, shape):
    import zoda_b200
    a = O.seeded_input(*shape, seed=shape[0] * 31 + shape[1])
    assert zoda_b200.data_root(a) == O.compute_data_root(a)


def test_data_root_of_nothing(lib):
    import hashlib
    import zoda_b200
    assert zoda_b200.data_root(np.zeros((0, 4), dtype=np.uint32)) == hashlib.sha256(b"").hexdigest()


def test_data_root_of_the_reference_input(lib):
    import zoda_b200
    a = O.reference_input(64, 8192)
    enc = O.encode_rowmajor(a)
    assert zoda_b200.data_root(enc) == O.compute_data_root(enc)
