"""GPU parity of the field kernels (fields.rs) against the FP64 oracle.

Tolerance: 1e-12 relative to max |reference| (FP64 throughout; the device
contracts G with the moments instead of forming the 3x3 tensor)."""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs, fields
from lumina_b200.geometry import Sphere, discretise_primitive
from oracle import oracle as orc
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _dipoles(rng, n_extra=0):
    pos = discretise_primitive(Sphere((0.5, -0.3, 0.2), 6.0), 2.0)
    mom = rng.standard_normal((pos.shape[0], 3)) + 1j * rng.standard_normal((pos.shape[0], 3))
    return pos, mom


def test_near_field_matches_oracle(backend, rng):
    pos, mom = _dipoles(rng)
    k = 2 * math.pi / 520.0
    obs = np.vstack([rng.uniform(-20, 20, (700, 3)), pos[:3]])  # 3 points on dipoles
    inc = lb.IncidentField((0.0, 0.6, 0.8), (1.0, 0.0, 0.0), 1.7)
    e = fields.field_at_points(backend, pos, mom, k, obs, inc)
    ref = orc.field_at_points(pos, mom, k, obs, inc.direction, inc.polarisation, inc.amplitude)
    assert rel_err(e, ref) < 1e-12


def test_near_field_map_matches_oracle(backend, rng):
    pos, mom = _dipoles(rng)
    k = 2 * math.pi / 600.0
    plane = fields.NearFieldPlane((0.0, 0.0, 9.0), (0.2, 0.1, 1.0), 25.0, 15.0, 37, 23)
    nf = fields.compute_near_field_map(backend, pos, mom, plane, k, lb.IncidentField())
    P, E = orc.near_field_plane(plane.centre, plane.normal, plane.half_width, plane.half_height,
                                plane.nx, plane.ny)
    assert np.array_equal(nf.positions, P) and np.array_equal(nf.extent, E)
    ref = orc.field_at_points(pos, mom, k, P)
    inten = np.sum(np.abs(ref) ** 2, axis=1)
    assert rel_err(nf.field_intensity, inten) < 1e-12
    assert nf.nx == 37 and nf.ny == 23


def test_far_field_matches_oracle(backend, rng):
    pos, mom = _dipoles(rng)
    k = 2 * math.pi / 480.0
    resp = lb.DipoleResponse(480.0, 1.0, mom, mom)
    ff = fields.compute_far_field(backend, pos, resp, k, 19, 36)
    th, ph, it = orc.far_field(pos, mom, k, 19, 36)
    assert np.allclose(ff.theta, th, rtol=0, atol=1e-15)
    assert np.allclose(ff.phi, ph, rtol=0, atol=1e-15)
    assert rel_err(ff.intensity, it) < 1e-12


def test_field_edge_cases(backend, rng):
    k = 0.01
    obs = np.array([[0.0, 0.0, 5.0], [1.0, 1.0, 1.0]])
    # no dipoles: the incident field alone
    e = fields.field_at_points(backend, np.zeros((0, 3)), np.zeros((0, 3)), k, obs)
    assert np.allclose(e[:, 0], np.exp(1j * k * obs[:, 2]), rtol=0, atol=1e-15)
    # no observation points / an empty grid
    assert fields.field_at_points(backend, [[0, 0, 0]], [[1, 0, 0]], k,
                                  np.zeros((0, 3))).shape == (0, 3)
    ff = fields.compute_far_field(backend, [[0, 0, 0]], lb.DipoleResponse(1, 1, np.array([[0, 0, 1]]),
                                                                          None), k, 0, 4)
    assert ff.intensity.size == 0
    # one theta sample: theta = 0 (the reference's (n-1).max(1) step)
    ff = fields.compute_far_field(backend, [[0, 0, 0]], lb.DipoleResponse(1, 1, np.array([[1, 0, 0]]),
                                                                          None), k, 1, 3)
    assert np.allclose(ff.theta, 0.0) and np.allclose(ff.intensity, 1.0)
    with pytest.raises(lb.SolverError):
        fields.field_at_points(backend, [[0, 0, 0]], [[1, 0, 0]], -1.0, obs)


def test_solver_field_hooks_end_to_end(backend):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 6.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 520.0)
    solver = lb.CdaSolver(backend=backend, iterative_threshold=0, use_fcd=True, cell_size=2.0)
    params = lb.SimulationParams(solver_tolerance=1e-10, max_iterations=2000)
    ds = lb.DipoleSet(w.positions, w.alpha)
    resp = solver.solve_dipoles(ds, 520.0, params)
    plane = fields.NearFieldPlane((0.0, 0.0, 10.0), (0.0, 0.0, 1.0), 12.0, 12.0, 16, 16)
    nf = solver.compute_near_field(ds, resp, plane)
    ff = solver.compute_far_field(ds, resp, 9, 12)
    k = lb.wavenumber(520.0, 1.0)
    P, _ = orc.near_field_plane(plane.centre, plane.normal, 12.0, 12.0, 16, 16)
    ref = np.sum(np.abs(orc.field_at_points(w.positions, resp.moments, k, P)) ** 2, axis=1)
    assert rel_err(nf.field_intensity, ref) < 1e-12
    _, _, it = orc.far_field(w.positions, resp.moments, k, 9, 12)
    assert rel_err(ff.intensity, it) < 1e-12
