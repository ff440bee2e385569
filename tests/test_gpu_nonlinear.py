"""GPU parity of the SHG / THG response (nonlinear.rs) against the oracle:
device sources 1e-13, the harmonic solve against the oracle's dense LU at
the harmonic wave number 1e-8 (moments, GMRES tol 1e-10), and the
reference's own end-to-end tests (zero tensor -> zero intensity, E^4 / E^6
scaling, harmonic wavelengths)."""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs, nonlinear
from lumina_b200.geometry import Sphere, discretise_primitive
from oracle import oracle as orc
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _linear(backend, lam=800.0):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 6.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, lam)
    solver = lb.CdaSolver(backend=backend, iterative_threshold=0, use_fcd=True, cell_size=2.0)
    params = lb.SimulationParams(solver_tolerance=1e-10, max_iterations=5000)
    resp = solver.solve_dipoles(lb.DipoleSet(w.positions, w.alpha), lam, params)
    return pos, solver, params, resp


def test_sources_match_oracle(backend, rng):
    e = rng.standard_normal((50, 3)) + 1j * rng.standard_normal((50, 3))
    c2 = rng.standard_normal((50, 27)) + 1j * rng.standard_normal((50, 27))
    c3 = rng.standard_normal(81) + 1j * rng.standard_normal(81)
    assert rel_err(nonlinear.harmonic_sources(backend, 2, e, list(c2)),
                   orc.harmonic_sources(2, e, c2)) < 1e-13
    assert rel_err(nonlinear.harmonic_sources(backend, 3, e, [c3]),
                   orc.harmonic_sources(3, e, c3)) < 1e-13


@pytest.mark.parametrize("order", [2, 3])
def test_harmonic_response_matches_lu(backend, order):
    pos, solver, params, resp = _linear(backend)
    lam_h = 800.0 / order
    wh = configs.au_workload("h", pos, 2.0, lam_h)
    dh = lb.DipoleSet(wh.positions, wh.alpha)
    tensor = (nonlinear.Chi2Tensor.isotropic_surface(1.0 + 0.2j, 0.4) if order == 2
              else nonlinear.Chi3Tensor.isotropic_bulk(1.0, 0.3 - 0.1j))
    fn = nonlinear.compute_shg_response if order == 2 else nonlinear.compute_thg_response
    res = fn(solver, resp, dh, [tensor], params, calc_far_field=True)
    assert res.harmonic_nm == pytest.approx(lam_h)
    src = orc.harmonic_sources(order, resp.local_fields, tensor.components)
    assert rel_err(res.source_moments, src) < 1e-13
    k_h = 2 * math.pi / lam_h
    A = orc.assemble(wh.positions, wh.alpha, k_h, True, 2.0)
    p = orc.lu_solve(A, src.reshape(-1)).reshape(-1, 3)
    assert rel_err(res.driven_moments, p) < 1e-8
    assert res.intensity == pytest.approx(float(np.sum(np.abs(p) ** 2)), rel=1e-8)
    _, _, ff = orc.far_field(wh.positions, p, k_h, 36, 72)
    assert rel_err(res.far_field.intensity, ff) < 1e-7


def test_reference_end_to_end_cases(backend):
    """nonlinear.rs tests: zero tensors give zero intensity; intensity scales
    as E^4 (SHG) and E^6 (THG); harmonic wavelengths 300 / 200 nm."""
    solver = lb.CdaSolver(backend=backend, use_fcd=False)
    params = lb.SimulationParams()
    d = lb.DipoleSet(np.zeros((1, 3)), np.array([1.0 + 0j]))

    def resp(e):
        e = np.asarray(e, complex).reshape(1, 3)
        return lb.DipoleResponse(600.0, 1.0, np.zeros((1, 3), complex), e)

    r = nonlinear.compute_shg_response(solver, resp([3.0, 1.0, 0.5]), d,
                                       [nonlinear.Chi2Tensor.zero()], params)
    assert r.intensity < 1e-20 and r.fundamental_nm == 600.0 and r.harmonic_nm == 300.0
    r = nonlinear.compute_thg_response(solver, resp([3.0, 1.0, 0.5]), d,
                                       [nonlinear.Chi3Tensor.zero()], params)
    assert r.intensity < 1e-20 and abs(r.harmonic_nm - 200.0) < 1e-10
    t2 = nonlinear.Chi2Tensor.zero()
    t2.components[0] = 1.0
    r1 = nonlinear.compute_shg_response(solver, resp([1.0, 0, 0]), d, [t2], params)
    r2 = nonlinear.compute_shg_response(solver, resp([2.0, 0, 0]), d, [t2], params)
    assert abs(r2.intensity / r1.intensity - 16.0) < 1e-8
    t3 = nonlinear.Chi3Tensor.zero()
    t3.components[0] = 1.0
    r1 = nonlinear.compute_thg_response(solver, resp([1.0, 0, 0]), d, [t3], params)
    r2 = nonlinear.compute_thg_response(solver, resp([2.0, 0, 0]), d, [t3], params)
    assert abs(r2.intensity / r1.intensity - 64.0) < 1e-6
