"""GPU parity of the block-Toeplitz (3D FFT) operator.

The reference's FFT matvec is checked against its on-the-fly matvec
(fft_matvec.rs:430-527, < 1e-10); here the FP64 FFT product is held to the
oracle's on-the-fly product at 1e-12 (max-norm relative), with and without
FCD, on full boxes and on partially occupied lattices; the FP32 product to
the FP32 bar 2e-5; FP32+refine solves to the C_ext gate 1e-6."""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from oracle import oracle as orc
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu


def _box(nx, ny, nz, s, origin=(-3.25, 1.5, 0.75)):
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1)
    return np.asarray(origin) + s * g.reshape(-1, 3).astype(float)


def _aniso_alpha(rng, n):
    return (np.eye(3) * (3.0 + 1.5j))[None] + 0.3 * (rng.standard_normal((n, 3, 3)) +
                                                     1j * rng.standard_normal((n, 3, 3)))


CASES = [
    ("box_point", False),
    ("box_fcd", True),
    ("sphere_fcd", True),
    ("slab_fcd", True),
]


def _geometry(kind, rng):
    if kind.startswith("box"):
        pos = _box(7, 5, 4, 1.5)
    elif kind.startswith("sphere"):
        pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 6.0), 2.0)
    else:  # a single layer: one node along z
        pos = _box(9, 6, 1, 2.0)
    s = 1.5 if kind.startswith("box") else 2.0
    return pos, s


@pytest.mark.parametrize("kind,fcd", CASES)
def test_fft_matvec_matches_oracle(backend, rng, kind, fcd):
    pos, s = _geometry(kind, rng)
    n = pos.shape[0]
    alpha = _aniso_alpha(rng, n)
    k = 2 * math.pi / 520.0
    x = rand_vec(rng, 3 * n)
    y_ref = orc.matvec_onthefly(pos, alpha, x, k, fcd, s)
    inv = lb.invert_polarisability(alpha)
    with backend.create_fft_session(pos, inv, k, fcd, s) as S:
        y64 = S.matvec(x, "fp64")
        y32 = S.matvec(x, "fp32")
    assert rel_err(y64, y_ref) < 1e-12
    assert rel_err(y32, y_ref) < 2e-5


def test_fft_equals_onthefly_session(backend, rng):
    pos = configs.cell_centred_cuboid((12.0, 10.0, 6.0), 1.0)
    w = configs.au_workload("c", pos, 1.0, 600.0)
    inv = lb.invert_polarisability(w.alpha)
    x = rand_vec(rng, 3 * w.n)
    with backend.create_fft_session(w.positions, inv, w.k, True, 1.0) as F, \
            backend.create_onthefly_session(w.positions, inv, w.k, True, 1.0) as O:
        assert rel_err(F.matvec(x, "fp64"), O.matvec(x, "fp64")) < 1e-12
        assert rel_err(F.matvec(x, "fp32"), O.matvec(x, "fp64")) < 2e-5


def test_fft_solve_meets_gate(backend):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 8.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 520.0)
    inv = lb.invert_polarisability(w.alpha)
    b = orc.incident_field(w.positions, w.k)
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    cs_ref = orc.cross_sections(w.positions, w.alpha, orc.lu_solve(A, b), w.k)
    with backend.create_fft_session(w.positions, inv, w.k, True, 2.0) as S:
        for mode in ("fp64", "fp32_refine"):
            x, info = S.solve(b, 1e-10, 3000, 30, mode)
            cs = lb.cross_sections(w.positions, inv, x, w.k, lb.IncidentField())
            assert info["converged"] == 1
            assert abs(cs[0] - cs_ref[0]) / abs(cs_ref[0]) < 1e-6
            assert abs(cs[1] - cs_ref[1]) / abs(cs_ref[1]) < 1e-6


def test_fft_set_wavelength_matches_fresh(backend, rng):
    pos = _box(6, 6, 3, 2.0)
    n = pos.shape[0]
    a1, a2 = _aniso_alpha(rng, n), _aniso_alpha(rng, n)
    k1, k2 = 2 * math.pi / 500.0, 2 * math.pi / 750.0
    x = rand_vec(rng, 3 * n)
    with backend.create_fft_session(pos, lb.invert_polarisability(a1), k1, True, 2.0) as S:
        S.set_wavelength(k2, lb.invert_polarisability(a2))
        y = S.matvec(x, "fp64")
    assert rel_err(y, orc.matvec_onthefly(pos, a2, x, k2, True, 2.0)) < 1e-12


def test_fft_rejects_off_lattice_and_duplicates(backend, rng):
    pos = _box(3, 3, 3, 1.0)
    inv = lb.invert_polarisability(_aniso_alpha(rng, pos.shape[0]))
    bad = pos.copy()
    bad[5, 0] += 0.3
    with pytest.raises(lb.SolverError):
        backend.create_fft_session(bad, inv, 0.01, True, 1.0)
    dup = pos.copy()
    dup[4] = dup[3]
    with pytest.raises(lb.SolverError):
        backend.create_fft_session(dup, inv, 0.01, True, 1.0)
    # a lattice pitch different from the FCD cell
    two = _box(4, 3, 3, 2.0)
    inv2 = lb.invert_polarisability(_aniso_alpha(rng, two.shape[0]))
    x = rand_vec(rng, 3 * two.shape[0])
    alpha2 = np.linalg.inv(inv2.reshape(-1, 3, 3))
    with backend.create_fft_session(two, inv2, 0.012, True, 1.0, spacing=2.0) as S:
        assert rel_err(S.matvec(x, "fp64"),
                       orc.matvec_onthefly(two, alpha2, x, 0.012, True, 1.0)) < 1e-11


# --- planar substrate through the z-mirrored convolution ---------------------
from lumina_b200.lattice import SommerfeldRuntime, SubstrateRuntime  # noqa: E402

SUB_CASES = ["fresnel_box", "fresnel_sphere", "sommerfeld_box", "sommerfeld_sphere",
             "sommerfeld_layer"]


def _sub_geometry(kind):
    if kind.endswith("sphere"):
        pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 6.0), 2.0).copy()
        pos[:, 2] += 8.0
        return pos, 2.0
    if kind.endswith("layer"):
        return _box(9, 6, 1, 2.0, origin=(-3.0, 1.0, 3.0)), 2.0
    return _box(7, 5, 4, 1.5, origin=(-3.25, 1.5, 2.0)), 1.5


@pytest.mark.parametrize("kind", SUB_CASES)
def test_fft_substrate_matches_oracle(backend, rng, kind):
    """The reflected term as a second convolution in the z-mirrored
    coordinate equals the on-the-fly substrate term (assembly.rs:274-303)."""
    pos, s = _sub_geometry(kind)
    n = pos.shape[0]
    alpha = _aniso_alpha(rng, n)
    lam = 600.0
    k = 2 * math.pi / lam
    x = rand_vec(rng, 3 * n)
    inv = lb.invert_polarisability(alpha)
    if kind.startswith("fresnel"):
        sub = SubstrateRuntime(0.5, 0.2 + 0.05j)
        y_ref = orc.matvec_onthefly(pos, alpha, x, k, True, s, substrate=sub)
    else:
        sub = SommerfeldRuntime(0.5, lam, 2.25 + 0.1j, 1.0)
        y_ref = orc.matvec_sommerfeld(pos, alpha, x, k, sub, True, s)
    with backend.create_fft_session(pos, inv, k, True, s, substrate=sub) as S:
        assert rel_err(S.matvec(x, "fp64"), y_ref) < 1e-12
        assert rel_err(S.matvec(x, "fp32"), y_ref) < 2e-5


def test_fft_sommerfeld_solve_and_wavelength_change(backend, rng):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 6.0), 2.0).copy()
    pos[:, 2] += 9.0
    w1 = configs.au_workload("s", pos, 2.0, 520.0)
    w2 = configs.au_workload("s", pos, 2.0, 640.0)
    s1 = SommerfeldRuntime(0.0, 520.0, 2.25, 1.0)
    s2 = SommerfeldRuntime(0.0, 640.0, 2.2, 1.0)
    inv1, inv2 = lb.invert_polarisability(w1.alpha), lb.invert_polarisability(w2.alpha)
    A = orc.assemble_sommerfeld(w1.positions, w1.alpha, w1.k, s1, True, 2.0)
    b = orc.incident_field(w1.positions, w1.k)
    ref = orc.cross_sections(w1.positions, w1.alpha, orc.lu_solve(A, b), w1.k)
    x2 = rand_vec(rng, 3 * w1.n)
    with backend.create_fft_session(w1.positions, inv1, w1.k, True, 2.0, substrate=s1) as S:
        x, info = S.solve(b, 1e-10, 5000, 30, "fp32_refine")
        cs = lb.cross_sections(w1.positions, inv1, x, w1.k, lb.IncidentField())
        assert info["converged"] and abs(cs[0] - ref[0]) / abs(ref[0]) < 1e-6
        # the Fresnel-free re-target leaves the Sommerfeld spectra stale
        S._lib.lum_session_set_wavelength(S._h, float(w2.k),
                                          lb.backend._dp(np.ascontiguousarray(inv2).view(np.float64)),
                                          None)
        with pytest.raises(lb.SolverError):
            S.matvec(x2, "fp64")
        S.set_wavelength(w2.k, inv2, substrate=s2)
        y = S.matvec(x2, "fp64")
    assert rel_err(y, orc.matvec_sommerfeld(w2.positions, w2.alpha, x2, w2.k, s2, True, 2.0)) < 1e-12
