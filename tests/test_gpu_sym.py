"""GPU parity of the symmetric FP32 pair scheme (each unordered pair
evaluated once, pairs_f32_sym.cuh), forced with LUMINA_F32_SYM=2 (or 3,
the three-CTA-per-SM build) so that it
runs at sizes the oracle handles; tolerance the FP32 bar 2e-5."""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from oracle import oracle as orc
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture
def force_sym(monkeypatch):
    monkeypatch.setenv("LUMINA_F32_SYM", "2")
    yield
    monkeypatch.delenv("LUMINA_F32_SYM", raising=False)


def _cases(rng):
    # N below, at and across superblock boundaries (512), jittered (lo != 0)
    # and exact lattices (lo == 0), FCD on and off
    out = []
    for r, spacing in ((4.0, 2.0), (9.0, 2.0), (11.0, 2.0)):
        pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), r), spacing)
        out.append(("sphere%d" % pos.shape[0], pos, True, spacing))
    base = discretise_primitive(Sphere((0.3, -0.2, 0.1), 10.0), 1.9)
    out.append(("jitter", base + rng.uniform(-0.15, 0.15, base.shape), False, 1.9))
    return out


def test_sym_matvec_matches_oracle(backend, rng, force_sym):
    for name, pos, fcd, cell in _cases(rng):
        n = pos.shape[0]
        alpha = (np.eye(3) * (2.0 + 1.0j))[None] + 0.2 * (rng.standard_normal((n, 3, 3)) +
                                                        1j * rng.standard_normal((n, 3, 3)))
        k = 2 * math.pi / 540.0
        x = rand_vec(rng, 3 * n)
        y_ref = orc.matvec_onthefly(pos, alpha, x, k, fcd, cell)
        with backend.create_onthefly_session(pos, lb.invert_polarisability(alpha), k, fcd,
                                             cell) as s:
            assert s.kernel_config()["f32_sym"] == 2, name
            y = s.matvec(x, "fp32")
        assert rel_err(y, y_ref) < 2e-5, name


def test_sym_solve_meets_gate(backend, force_sym):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 10.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 520.0)
    inv = lb.invert_polarisability(w.alpha)
    b = orc.incident_field(w.positions, w.k)
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    cs_ref = orc.cross_sections(w.positions, w.alpha, orc.lu_solve(A, b), w.k)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, 2.0) as s:
        x, info = s.solve(b, 1e-10, 3000, 30, "fp32_refine")
    cs = lb.cross_sections(w.positions, inv, x, w.k, lb.IncidentField())
    assert info["converged"] == 1
    assert abs(cs[0] - cs_ref[0]) / abs(cs_ref[0]) < 1e-6


def test_sym_equals_split_scheme(backend, rng, monkeypatch):
    """The same session geometry under both FP32 schemes: the products agree
    to FP32 accuracy (different summation order)."""
    pos = configs.cell_centred_cuboid((14.0, 12.0, 8.0), 1.0)  # N = 1344: 3 superblocks
    w = configs.au_workload("c", pos, 1.0, 650.0)
    inv = lb.invert_polarisability(w.alpha)
    x = rand_vec(rng, 3 * w.n)
    out = {}
    for flag in ("2", "3", "0"):
        monkeypatch.setenv("LUMINA_F32_SYM", flag)
        with backend.create_onthefly_session(w.positions, inv, w.k, True, 1.0) as s:
            assert s.kernel_config()["f32_sym"] == int(flag)
            out[flag] = s.matvec(x, "fp32")
            y64 = s.matvec(x, "fp64")
    for flag in ("2", "3"):
        assert rel_err(out[flag], y64) < 2e-5
        assert rel_err(out[flag], out["0"]) < 2e-5
