"""Several right-hand sides per session (lum_solve_gmres_multi): two GMRES runs
in lockstep share every operator application (the two-vector pair kernels).

Each right-hand side must get what its own single-vector solve gives:
FP64 plain solves agree to 1e-12 (the two-vector FP64 kernel repeats the
single-vector arithmetic for each vector), FP32+refine solves reach the same
C_ext within 1e-8 (the FP32 two-vector kernel has its own split and rounding;
both meet the 1e-10 tolerance of the FP64 residual), and the iteration
counts match within two steps.
"""
import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def rhs_set(w, pols):
    return [lb.incident_field(w.positions, w.k, lb.IncidentField((0.0, 0.0, 1.0), p, 1.0))
            for p in pols]


@pytest.mark.parametrize("mode", ["fp64", "fp32_refine"])
def test_multi_rhs_equals_single_solves(backend, mode):
    w = configs.cuboid_au((14.0, 12.0, 10.0), 1.0, 600.0)
    inv = lb.invert_polarisability(w.alpha)
    pols = [(1.0, 0.0, 0.0), (0.0, 1.0, 0.0), (0.6, 0.8, 0.0)]
    B = np.stack(rhs_set(w, pols))
    with backend.create_onthefly_session(w.positions, inv, w.k, True, w.cell_size) as s:
        X, infos = s.solve_multi(B, 1e-10, 4000, 30, mode)
        for r, p in enumerate(pols):
            x1, i1 = s.solve(B[r], 1e-10, 4000, 30, mode)
            inc = lb.IncidentField((0.0, 0.0, 1.0), p, 1.0)
            c1 = lb.cross_sections(w.positions, inv, x1, w.k, inc)[0]
            cm = lb.cross_sections(w.positions, inv, X[r], w.k, inc)[0]
            assert infos[r]["converged"] == 1
            assert abs(infos[r]["iterations"] - i1["iterations"]) <= 2, (r, infos[r], i1)
            if mode == "fp64":
                assert rel_err(X[r], x1) < 1e-12
            else:
                assert rel_err(X[r], x1) < 1e-8
            assert abs(cm - c1) <= 1e-8 * abs(c1)


def test_multi_rhs_uneven_convergence(backend):
    """A zero right-hand side and a hard one: the finished run drops out."""
    w = configs.cuboid_au((10.0, 8.0, 6.0), 1.0, 650.0)
    inv = lb.invert_polarisability(w.alpha)
    b = rhs_set(w, [(1.0, 0.0, 0.0)])[0]
    B = np.stack([np.zeros_like(b), b, 1e-3 * b])
    with backend.create_onthefly_session(w.positions, inv, w.k, True, w.cell_size) as s:
        X, infos = s.solve_multi(B, 1e-10, 4000, 30, "fp32_refine")
        x1, _ = s.solve(b, 1e-10, 4000, 30, "fp32_refine")
    assert infos[0]["converged"] == 1 and infos[0]["iterations"] == 0
    assert np.all(X[0] == 0)
    assert rel_err(X[1], x1) < 1e-8
    assert rel_err(X[2], 1e-3 * x1) < 1e-8


def test_multi_rhs_with_substrate(backend):
    """Image-dipole pass with two vectors (no lattice)."""
    from lumina_b200.lattice import SubstrateRuntime, fresnel_reflection_amplitude
    w = configs.cuboid_au((8.0, 8.0, 6.0), 2.0, 620.0)
    pos = w.positions + np.array([0.0, 0.0, 6.0])
    inv = lb.invert_polarisability(w.alpha)
    sub = SubstrateRuntime(0.0, fresnel_reflection_amplitude(1.45 ** 2, 1.0))
    B = np.stack(rhs_set(w, [(1.0, 0.0, 0.0), (0.0, 1.0, 0.0)]))
    with backend.create_onthefly_session(pos, inv, w.k, True, w.cell_size, substrate=sub) as s:
        # the image pass contracts each vector with its own instruction
        # stream, so FP64 agrees to rounding rather than bit for bit here
        for mode, tol in (("fp64", 1e-9), ("fp32_refine", 1e-8)):
            X, _ = s.solve_multi(B, 1e-10, 4000, 30, mode)
            for r in range(2):
                x1, _ = s.solve(B[r], 1e-10, 4000, 30, mode)
                assert rel_err(X[r], x1) < tol, (mode, r)
