"""Error reporting across the C ABI (backend.rs:13-22, ComputeError).

An allocation the device cannot satisfy (a cached FP64 matrix of
dim = 300,000: 1.44 TB) returns LUM_ERR_OOM with the requested and free
byte counts (lum_last_oom), mapped to OutOfMemory { requested, available };
the context stays usable afterwards.  Nothing here faults the GPU: the
failing call is a cudaMalloc that returns an error.
"""
import pytest

import lumina_b200 as lb
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def test_oom_reports_requested_and_available(backend, rng):
    dim = 300000
    with pytest.raises(lb.OutOfMemory) as e:
        backend.create_session(dim, "fp64")
    ld = (dim + 15) // 16 * 16
    assert e.value.requested == 16 * ld * dim
    assert 0 < e.value.available < e.value.requested
    # the context is still usable
    A = rng.standard_normal((96, 96)) + 1j * rng.standard_normal((96, 96))
    x = rng.standard_normal(96) + 1j * rng.standard_normal(96)
    with backend.create_session(96, "fp64") as s:
        s.upload_matrix(A)
        assert rel_err(s.matvec(x, "fp64"), A @ x) < 1e-13
