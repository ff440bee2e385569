"""Golden fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py
from an independent numpy restatement solved with LAPACK LU).

CPU: the C++ oracle reproduces every fixture's A x (1e-12) and moments (1e-10).
GPU: the CUDA operators reproduce A x (FP64 1e-12, FP32 2e-5), and the
device GMRES reproduces the moments (1e-8) and C_ext (1e-9) at tol 1e-11.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as orc
from tests.conftest import ROOT, rel_err

FIXTURES = sorted(glob.glob(os.path.join(ROOT, "tests", "golden", "*.npz")))


def load(path):
    d = np.load(path)
    sub = d["substrate"]
    substrate = None
    if not np.isnan(sub[0].real):
        from lumina_b200.lattice import SubstrateRuntime
        substrate = SubstrateRuntime(sub[0].real, complex(sub[1]))
    return (d["positions"], d["alpha"], float(d["k"]), bool(d["use_fcd"]), float(d["cell"]),
            substrate, d["x"], d["y"], d["moments"], d["cross"])


def ids():
    return [os.path.basename(p)[:-4] for p in FIXTURES]


def test_fixtures_present():
    assert len(FIXTURES) >= 4


@pytest.mark.parametrize("path", FIXTURES, ids=ids())
def test_oracle_matches_fixture(path):
    pos, alpha, k, fcd, cell, sub, x, y, mom, cross = load(path)
    y_o = orc.matvec_onthefly(pos, alpha, x, k, fcd, cell, substrate=sub)
    assert rel_err(y_o, y) < 1e-12
    A = orc.assemble(pos, alpha, k, fcd, cell, substrate=sub)
    b = orc.incident_field(pos, k)
    p = orc.lu_solve(A, b)
    assert rel_err(p, mom) < 1e-10
    cs = orc.cross_sections(pos, alpha, p, k)
    assert np.max(np.abs(cs - cross) / np.abs(cross)) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=ids())
def test_gpu_matches_fixture(backend, path):
    import lumina_b200 as lb
    pos, alpha, k, fcd, cell, sub, x, y, mom, cross = load(path)
    inv = lb.invert_polarisability(alpha)
    with backend.create_onthefly_session(pos, inv, k, fcd, cell, substrate=sub) as s:
        assert rel_err(s.matvec(x, "fp64"), y) < 1e-12
        assert rel_err(s.matvec(x, "fp32"), y) < 2e-5
        b = lb.incident_field(pos, k, lb.IncidentField())
        p, info = s.solve(b, 1e-11, 5000, 30, "fp64")
        assert info["converged"] and rel_err(p, mom) < 1e-8
        cs = lb.cross_sections(pos, inv, p, k, lb.IncidentField())
        assert abs(cs[0] - cross[0]) / abs(cross[0]) < 1e-9
        p32, info32 = s.solve(b, 1e-10, 5000, 30, "fp32_refine")
        cs32 = lb.cross_sections(pos, inv, p32, k, lb.IncidentField())
        assert info32["converged"] and abs(cs32[0] - cross[0]) / abs(cross[0]) < 1e-8
