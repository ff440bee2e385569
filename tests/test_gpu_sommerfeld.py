"""GPU parity of the Sommerfeld substrate (sommerfeld.rs, assembly.rs:157-166,
:296-303) against the oracle.

Tolerances (max |error| / max |reference|):
  reflected tensor per pair (FP64 quadrature)          1e-11
  FP64 operator (on-the-fly table or assembled matrix)  1e-12
  FP32 operator / FP32-stored matrix                    2e-5
  solves: C_ext against LU on the oracle matrix         1e-6
"""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from lumina_b200.lattice import LatticeSpec, SommerfeldRuntime
from lumina_b200.sommerfeld import SommerfeldGreens
from oracle import oracle as orc
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu

SUBSTRATES = [
    (600.0, 2.25 + 0.0j, 1.0),        # glass in air: three quadrature segments
    (520.0, -4.7 + 2.4j, 1.0),        # Au-like: no middle segment
    (700.0, 12.0 + 0.1j, 1.77),       # high index under water
]


def _pairs(rng, m, z0=0.0):
    ri = rng.uniform(-40, 40, (m, 3))
    rj = rng.uniform(-40, 40, (m, 3))
    ri[:, 2] = z0 + rng.uniform(0.3, 60, m)
    rj[:, 2] = z0 + rng.uniform(0.3, 60, m)
    # edge cases: rho = 0, i == j, below the interface, far above it
    rj[0, :2] = ri[0, :2]
    rj[1] = ri[1]
    ri[2, 2] = z0 - 5.0
    rj[2, 2] = z0 + 1.0
    ri[3, 2], rj[3, 2] = z0 + 2500.0, z0 + 2490.0
    return ri, rj


@pytest.mark.parametrize("wl,eps_sub,eps_env", SUBSTRATES)
def test_reflected_tensor_matches_oracle(backend, rng, wl, eps_sub, eps_env):
    somm = SommerfeldRuntime(1.5, wl, eps_sub, eps_env)
    ri, rj = _pairs(rng, 400, 1.5)
    g = backend.sommerfeld_tensor(somm, ri, rj)
    g_ref = orc.sommerfeld_tensor(somm, ri, rj)
    for q in range(len(ri)):
        scale = np.abs(g_ref[q]).max()
        if scale == 0.0:
            assert np.abs(g[q]).max() == 0.0
        else:
            assert np.abs(g[q] - g_ref[q]).max() <= 1e-11 * scale, q


def test_reference_unit_cases_on_device(backend):
    """The reference's own tensor tests (sommerfeld.rs:477-555) on the device."""
    sg = SommerfeldGreens(500.0, 2.25, 2.25, backend=backend)
    assert np.abs(sg.evaluate([0.0, 0.0, 10.0], [3.0, 0.0, 8.0], 0.0)).max() < 1e-10
    sg = SommerfeldGreens(600.0, 2.25, 1.0, backend=backend)
    g = sg.evaluate([5.0, 3.0, 12.0], [2.0, 1.0, 8.0], 0.0)
    assert abs(g[0, 1] - g[1, 0]) < 1e-10 and abs(g[0, 2] - g[2, 0]) < 1e-10
    g = sg.evaluate([0.0, 0.0, 12.0], [0.0, 0.0, 8.0], 0.0)
    assert abs(g[0, 2]) < 1e-8 and abs(g[1, 2]) < 1e-8 and abs(g[0, 1]) < 1e-8
    assert abs(g[0, 0] - g[1, 1]) < 1e-8 * abs(g[0, 0])
    g = SommerfeldGreens(500.0, 2.25, 1.0, backend=backend).evaluate(
        [0.0, 0.0, 2502.5], [0.0, 0.0, 2497.5], 0.0)
    assert np.isfinite(g).all()


def _particle(spacing=2.0, radius=6.0, lift=1.0, wl=600.0):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), radius), spacing)
    pos = pos.copy()
    pos[:, 2] += radius + lift        # sphere resting above z = 0
    w = configs.au_workload("s", pos, spacing, wl)
    return w, lb.invert_polarisability(w.alpha)


@pytest.mark.parametrize("layout", ["lattice_keys", "pairs"])
@pytest.mark.parametrize("wl,eps_sub,eps_env", SUBSTRATES)
def test_onthefly_operator_matches_oracle(backend, rng, wl, eps_sub, eps_env, layout):
    """Dipoles on the cubic lattice use the (rho, z-sum) key table; a jitter
    of 1e-3 nm takes them off it and onto the per-pair table."""
    w, inv = _particle(wl=wl)
    pos = w.positions.copy()
    if layout == "pairs":
        pos += rng.uniform(-1e-3, 1e-3, pos.shape)
    somm = SommerfeldRuntime(0.0, wl, eps_sub, eps_env)
    x = rng.standard_normal(3 * w.n) + 1j * rng.standard_normal(3 * w.n)
    y_ref = orc.matvec_sommerfeld(pos, w.alpha, x, w.k, somm, True, 2.0)
    with backend.create_onthefly_session(pos, inv, w.k, True, 2.0, substrate=somm) as s:
        assert s.kernel_config()["sommerfeld"] == layout
        assert rel_err(s.matvec(x, "fp64"), y_ref) < 1e-12
        assert rel_err(s.matvec(x, "fp32"), y_ref) < 2e-5


@pytest.mark.parametrize("storage,tol", [("fp64", 1e-12), ("fp32", 2e-5)])
def test_assembled_matrix_matches_oracle(backend, rng, storage, tol):
    wl, eps_sub, eps_env = SUBSTRATES[0]
    w, inv = _particle(wl=wl)
    somm = SommerfeldRuntime(0.0, wl, eps_sub, eps_env)
    A_ref = orc.assemble_sommerfeld(w.positions, w.alpha, w.k, somm, True, 2.0)
    X = rng.standard_normal((3 * w.n, 5)) + 1j * rng.standard_normal((3 * w.n, 5))
    with backend.assemble_and_create_session(w.positions, w.k, inv, True, 2.0, substrate=somm,
                                             precision=storage) as s:
        for r in range(X.shape[1]):
            assert rel_err(s.matvec(X[:, r], storage), A_ref @ X[:, r]) < tol
        if storage == "fp32":
            assert rel_err(s.matmul(X, "tensor"), A_ref @ X) < tol
            # the FP64 residual operator of an FP32-stored session
            assert rel_err(s.matvec(X[:, 0], "fp64"), A_ref @ X[:, 0]) < 1e-12


@pytest.mark.parametrize("kind,mode", [("onthefly", "fp64"), ("onthefly", "fp32_refine"),
                                       ("cached", "fp32_refine")])
def test_solve_matches_lu(backend, kind, mode):
    wl, eps_sub, eps_env = SUBSTRATES[1]
    w, inv = _particle(wl=wl)
    somm = SommerfeldRuntime(0.0, wl, eps_sub, eps_env)
    A = orc.assemble_sommerfeld(w.positions, w.alpha, w.k, somm, True, 2.0)
    b = orc.incident_field(w.positions, w.k)
    ref = orc.cross_sections(w.positions, w.alpha, orc.lu_solve(A, b), w.k)
    if kind == "onthefly":
        sess = backend.create_onthefly_session(w.positions, inv, w.k, True, 2.0, substrate=somm)
    else:
        sess = backend.assemble_and_create_session(w.positions, w.k, inv, True, 2.0,
                                                   substrate=somm, precision="fp32")
    with sess as s:
        x, info = s.solve(b, 1e-10, 5000, 30, mode)
    cs = lb.cross_sections(w.positions, inv, x, w.k, lb.IncidentField())
    assert info["converged"]
    assert abs(cs[0] - ref[0]) / abs(ref[0]) < 1e-6


def test_set_wavelength_marks_table_stale_then_rebuilds(backend, rng):
    w, inv = _particle(wl=600.0)
    w2, inv2 = _particle(wl=650.0)
    s1 = SommerfeldRuntime(0.0, 600.0, 2.25, 1.0)
    s2 = SommerfeldRuntime(0.0, 650.0, 2.2, 1.0)
    x = rng.standard_normal(3 * w.n) + 1j * rng.standard_normal(3 * w.n)
    y_ref = orc.matvec_sommerfeld(w2.positions, w2.alpha, x, w2.k, s2, True, 2.0)
    for kind in ("onthefly", "cached"):
        if kind == "onthefly":
            sess = backend.create_onthefly_session(w.positions, inv, w.k, True, 2.0, substrate=s1)
        else:
            sess = backend.assemble_and_create_session(w.positions, w.k, inv, True, 2.0,
                                                       substrate=s1, precision="fp64")
        with sess as s:
            # the Fresnel re-target alone leaves the Sommerfeld table stale
            s._lib.lum_session_set_wavelength(s._h, float(w2.k),
                                              lb.backend._dp(np.ascontiguousarray(inv2).view(np.float64)),
                                              None)
            with pytest.raises(lb.SolverError):
                s.matvec(x, "fp64")
            if kind == "cached":  # nor may the multi-vector product use the old matrix
                with pytest.raises(lb.SolverError):
                    s.matmul(np.stack([x, x], axis=1), "cuda_cores")
            s.set_wavelength(w2.k, inv2, substrate=s2)
            assert rel_err(s.matvec(x, "fp64"), y_ref) < 1e-12


def test_lattice_with_sommerfeld(backend, rng):
    """Ewald direct term plus the (non-periodic) Sommerfeld term
    (assembly.rs:39-41)."""
    wl = 600.0
    pos = np.array([[0.0, 0.0, 6.0], [3.0, 0.0, 6.0], [0.0, 3.0, 9.0], [3.0, 3.0, 9.0]])
    w = configs.au_workload("s", pos, 3.0, wl)
    inv = lb.invert_polarisability(w.alpha)
    lat = LatticeSpec.planar((60.0, 0.0, 0.0), (0.0, 60.0, 0.0))
    somm = SommerfeldRuntime(0.0, wl, 2.25, 1.0)
    A_ref = orc.assemble_sommerfeld(w.positions, w.alpha, w.k, somm, False, 3.0, lattice=lat)
    x = rng.standard_normal(3 * w.n) + 1j * rng.standard_normal(3 * w.n)
    with backend.assemble_and_create_session(w.positions, w.k, inv, False, 3.0, lattice=lat,
                                             substrate=somm, precision="fp64") as s:
        assert rel_err(s.matvec(x, "fp64"), A_ref @ x) < 1e-10
    y_ref = orc.matvec_sommerfeld(w.positions, w.alpha, x, w.k, somm, False, 3.0, lattice=lat)
    with backend.create_onthefly_session(w.positions, inv, w.k, False, 3.0, lattice=lat,
                                         substrate=somm) as s:
        assert rel_err(s.matvec(x, "fp64"), y_ref) < 1e-10


def test_invalid_sommerfeld_arguments(backend):
    pos = np.array([[0.0, 0.0, 5.0], [2.0, 0.0, 5.0]])
    w = configs.au_workload("s", pos, 2.0, 600.0)
    inv = lb.invert_polarisability(w.alpha)
    with pytest.raises(lb.SolverError):
        backend.create_onthefly_session(pos, inv, w.k, True, 2.0,
                                        substrate=SommerfeldRuntime(0.0, -1.0, 2.25, 1.0))
    with pytest.raises(lb.SolverError):
        backend.sommerfeld_tensor(SommerfeldRuntime(0.0, 600.0, 2.25, 0.0), pos[0], pos[1])


@pytest.mark.parametrize("kind", ["onthefly", "cached", "fft"])
def test_single_dipole_self_image(backend, rng, kind):
    """N = 1: only the self block, G_refl(r, r) at rho = 0 (assembly.rs:157-166
    runs for i == j), in each session kind."""
    pos = np.array([[1.0, -2.0, 4.0]])
    w = configs.au_workload("one", pos, 2.0, 600.0)
    inv = lb.invert_polarisability(w.alpha)
    somm = SommerfeldRuntime(0.0, 600.0, 2.25 + 0.3j, 1.0)
    x = rng.standard_normal(3) + 1j * rng.standard_normal(3)
    y_ref = orc.matvec_sommerfeld(pos, w.alpha, x, w.k, somm, True, 2.0)
    if kind == "onthefly":
        s = backend.create_onthefly_session(pos, inv, w.k, True, 2.0, substrate=somm)
    elif kind == "cached":
        s = backend.assemble_and_create_session(pos, w.k, inv, True, 2.0, substrate=somm,
                                                precision="fp64")
    else:
        s = backend.create_fft_session(pos, inv, w.k, True, 2.0, substrate=somm)
    with s:
        assert rel_err(s.matvec(x, "fp64"), y_ref) < 1e-12


def test_dipoles_below_interface_have_no_reflected_term(backend, rng):
    """dz <= 0 gives a zero tensor (sommerfeld.rs:263-266): with the
    interface above every dipole the operator is the free-space one."""
    w, inv = _particle(wl=600.0)
    somm = SommerfeldRuntime(float(w.positions[:, 2].max()) + 50.0, 600.0, 2.25, 1.0)
    x = rng.standard_normal(3 * w.n) + 1j * rng.standard_normal(3 * w.n)
    y_free = orc.matvec_onthefly(w.positions, w.alpha, x, w.k, True, 2.0)
    for layout_jitter in (0.0, 1e-3):
        pos = w.positions + rng.uniform(-layout_jitter, layout_jitter, w.positions.shape)
        y_ref = orc.matvec_onthefly(pos, w.alpha, x, w.k, True, 2.0) if layout_jitter else y_free
        with backend.create_onthefly_session(pos, inv, w.k, True, 2.0, substrate=somm) as s:
            assert rel_err(s.matvec(x, "fp64"), y_ref) < 1e-12
