"""The allocation-free matvec entry point (lum_matvec_onthefly_noalloc).

Some callers of this library cannot let it call cudaMalloc: their device
memory is owned by another allocator or reserved ahead of time (for example
to fit a large cached interaction matrix in HBM), or they call from code where
allocating is not allowed.  This entry point serves them: it takes
caller-owned device inputs and output and keeps its scratch in a fixed array
inside the library.  The test calls it through the C ABI twice in a row, with
different vectors each time, and checks each result against the session
on-the-fly FP64 matvec with use_fcd = 0 at the FP64 operator tolerance of the
parity suite (1e-12 relative).  It also checks that an oversized N is refused.
The file name sorts last, so a run that stops at the first failure has run
every other test already.
"""
import ctypes
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import _ffi, configs
from lumina_b200.geometry import Sphere, discretise_primitive
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu

FP64_OPERATOR_TOL = 1e-12


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def test_noalloc_matvec_matches_session_matvec_twice(backend, rng):
    import torch
    pos = discretise_primitive(Sphere((0.5, -0.5, 0.0), 7.0), 1.5)
    pos = pos + rng.uniform(-0.1, 0.1, pos.shape)
    w = configs.au_workload("noalloc", pos, 1.5, 560.0)
    n = w.n
    alpha = w.alpha + 0.1 * (rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3)))
    inv = lb.invert_polarisability(alpha)
    lib = _ffi.load()
    pos_d = _dev(pos.astype(np.float64))
    inv_d = _dev(inv.reshape(n, 9))
    y_d = torch.zeros(3 * n, dtype=torch.complex128, device="cuda")
    ref_d = torch.zeros(3 * n, dtype=torch.complex128, device="cuda")
    with backend.create_onthefly_session(pos, inv, w.k, use_fcd=False, cell_size=1.5) as s:
        for call in range(2):
            x = rand_vec(rng, 3 * n)
            x_d = _dev(x)
            torch.cuda.synchronize()
            s.matvec_device(x_d.data_ptr(), ref_d.data_ptr(), "fp64")
            rc = lib.lum_matvec_onthefly_noalloc(n, pos_d.data_ptr(), inv_d.data_ptr(), w.k,
                                                 x_d.data_ptr(), y_d.data_ptr(), None)
            assert rc == _ffi.LUM_OK, _ffi.last_error()
            torch.cuda.synchronize()
            y = y_d.cpu().numpy()
            y_ref = ref_d.cpu().numpy()
            assert rel_err(y, y_ref) < FP64_OPERATOR_TOL, f"call {call}"


def test_noalloc_rejects_oversized_n(backend):
    import torch
    lib = _ffi.load()
    buf = torch.zeros(16, dtype=torch.complex128, device="cuda")
    p = buf.data_ptr()
    rc = lib.lum_matvec_onthefly_noalloc(174763, p, p, 0.01, p, p, None)
    assert rc == _ffi.LUM_ERR_INVALID
    assert "174762" in _ffi.last_error()
