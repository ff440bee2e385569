"""The allocation-free matvec entry point (lum_matvec_onthefly_noalloc).

Some callers of this library cannot let it call cudaMalloc: their device
memory is owned by another allocator or reserved ahead of time (for example
to fit a large cached interaction matrix in HBM), or they call from code where
allocating is not allowed.  This entry point serves them: it takes
caller-owned device inputs and output and keeps its scratch in a fixed array
inside the library.  The test calls it through the C ABI twice in a row, with
different vectors each time, and checks each result against the session
on-the-fly FP64 matvec with use_fcd = 0 and against the oracle's
matvec_on_the_fly (assembly.rs:209-318, use_fcd = false) at the FP64 operator
tolerance of the parity suite (1e-12 relative).  The device's free memory is
the same after the second call as after the first (the first call on a
device may load the library's device code, which holds the fixed array).  It
also checks that an oversized N is refused.  The file name sorts last, so a
run that stops at the first failure has run every other test already.
"""
import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import _ffi, configs
from lumina_b200.geometry import Sphere, discretise_primitive
from oracle import oracle as orc
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu

FP64_OPERATOR_TOL = 1e-12


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def test_noalloc_matvec_matches_session_and_oracle_twice(backend, rng):
    import torch
    pos = discretise_primitive(Sphere((0.5, -0.5, 0.0), 7.0), 1.5)
    pos = pos + rng.uniform(-0.1, 0.1, pos.shape)
    w = configs.au_workload("noalloc", pos, 1.5, 560.0)
    n = w.n
    alpha = w.alpha + 0.1 * (rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3)))
    inv = lb.invert_polarisability(alpha)
    lib = _ffi.load()
    xs = [rand_vec(rng, 3 * n) for _ in range(2)]
    # every device buffer and both session references exist before the calls
    pos_d = _dev(pos.astype(np.float64))
    inv_d = _dev(inv.reshape(n, 9))
    x_d = [_dev(x) for x in xs]
    y_d = [torch.zeros(3 * n, dtype=torch.complex128, device="cuda") for _ in xs]
    ref_d = [torch.zeros(3 * n, dtype=torch.complex128, device="cuda") for _ in xs]
    with backend.create_onthefly_session(pos, inv, w.k, use_fcd=False, cell_size=1.5) as s:
        for c in range(2):
            s.matvec_device(x_d[c].data_ptr(), ref_d[c].data_ptr(), "fp64")
        torch.cuda.synchronize()
        free_after = []
        for c in range(2):
            rc = lib.lum_matvec_onthefly_noalloc(n, pos_d.data_ptr(), inv_d.data_ptr(), w.k,
                                                 x_d[c].data_ptr(), y_d[c].data_ptr(), None)
            assert rc == _ffi.LUM_OK, _ffi.last_error()
            torch.cuda.synchronize()
            free_after.append(torch.cuda.mem_get_info()[0])
    assert free_after[1] == free_after[0]
    for c in range(2):
        y = y_d[c].cpu().numpy()
        assert rel_err(y, ref_d[c].cpu().numpy()) < FP64_OPERATOR_TOL, f"call {c} vs session"
        y_orc = orc.matvec_onthefly(pos, alpha, xs[c], w.k, use_fcd=False)
        assert rel_err(y, y_orc) < FP64_OPERATOR_TOL, f"call {c} vs oracle"


def test_noalloc_rejects_oversized_n(backend):
    import torch
    lib = _ffi.load()
    buf = torch.zeros(16, dtype=torch.complex128, device="cuda")
    p = buf.data_ptr()
    rc = lib.lum_matvec_onthefly_noalloc(174763, p, p, 0.01, p, p, None)
    assert rc == _ffi.LUM_ERR_INVALID
    assert "174762" in _ffi.last_error()
