"""C ABI surface checks that need no GPU: the library loads, every function
include/*.h declares is exported, the ctypes table matches the header, and
the product path fails loudly (Unavailable) when no device is present."""
import ctypes
import glob
import os
import re

import pytest

from lumina_b200 import _ffi
from tests.conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"LUM_API\s+[\w\s\*]+?\b(lum_\w+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = _declared()
    assert "lum_session_create_onthefly" in names and "lum_solve_gmres" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_ffi.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_ctypes_table_covers_header():
    assert _declared() == set(_ffi.SIGNATURES)


def test_constants_match_header():
    """Every LUM_* enumerator of the header that the ctypes mirror defines
    has the header's value (status codes, precisions, solve modes, the
    symmetric storage flag)."""
    text = "".join(open(h).read() for h in glob.glob(os.path.join(ROOT, "include", "*.h")))
    values = {n: int(v, 0) for n, v in re.findall(r"\b(LUM_[A-Z0-9_]+)\s*=\s*(0x[0-9a-fA-F]+|\d+)",
                                                   text)}
    checked = [n for n in values if hasattr(_ffi, n)]
    assert "LUM_STORAGE_SYMMETRIC" in checked and "LUM_ERR_TIMEOUT" in checked
    for n in checked:
        assert getattr(_ffi, n) == values[n], n


def test_no_device_means_unavailable():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import lumina_b200 as lb
    with pytest.raises(lb.Unavailable):
        lb.CudaBackend(0)


def test_host_helpers_without_device():
    import numpy as np
    import lumina_b200 as lb
    from oracle import oracle as orc
    rng = np.random.default_rng(5)
    alpha = np.eye(3)[None] * (2 + 1j) + 0.2 * (rng.standard_normal((4, 3, 3))
                                                + 1j * rng.standard_normal((4, 3, 3)))
    inv = lb.invert_polarisability(alpha)
    for i in range(4):
        assert np.allclose(inv[i], orc.invert_3x3(alpha[i]), rtol=1e-13, atol=1e-15)
    pos = rng.uniform(-5, 5, (4, 3))
    k = 2 * np.pi / 530.0
    assert np.allclose(lb.incident_field(pos, k, lb.IncidentField()), orc.incident_field(pos, k),
                       rtol=0, atol=1e-15)
    m = rng.standard_normal(12) + 1j * rng.standard_normal(12)
    cs = lb.cross_sections(pos, inv, m, k, lb.IncidentField())
    ref = orc.cross_sections(pos, alpha, m, k)
    assert np.allclose(cs, ref, rtol=1e-12, atol=0)
    with pytest.raises(lb.InvalidGeometry):
        lb.invert_polarisability(np.zeros((1, 3, 3)))


def test_cdasolver_storage_choice_without_device():
    """CdaSolver's dispatch (cda/mod.rs:271-391) keeps the reference's branch
    choice and picks symmetric tiles only for free-space cached systems."""
    import numpy as np

    import lumina_b200 as lb
    from lumina_b200.lattice import LatticeSpec, SubstrateRuntime
    pos = np.stack(np.meshgrid(*[np.arange(6.0)] * 3, indexing="ij"), -1).reshape(-1, 3) * 2.0
    pos = pos + 0.1 * np.sin(np.arange(pos.size)).reshape(pos.shape)  # off the lattice: no FFT
    ds = lb.DipoleSet(pos, np.tile(np.eye(3, dtype=complex), (pos.shape[0], 1, 1)))
    free = lb.SimulationParams()
    sub = lb.SimulationParams(substrate_runtime=SubstrateRuntime(-5.0, complex(0.2)))

    def plan(params, direct=False, **kw):
        s = lb.CdaSolver(backend=object(), cell_size=2.0, **kw)
        branch, storage, _ = s._plan(ds, params, direct)
        return branch, storage

    assert plan(free, direct=True) == ("cached", "fp64+sym")
    assert plan(free) == ("cached", "fp64+sym")
    assert plan(free, precision="fp32_refine") == ("cached", "fp32+sym")
    assert plan(free, symmetric_storage=False) == ("cached", "fp64")
    assert plan(sub) == ("cached", "fp64")
    lat = LatticeSpec.planar((400.0, 0.0, 0.0), (0.0, 400.0, 0.0))
    assert plan(free, lattice=lat) == ("cached", "fp64")
    assert plan(free, matrix_memory_budget=0) == ("onthefly", None)
