"""The oracle pinned against the reference's own known-answer tests.

Each test restates one assertion of the reference's test suite for this path
(file:line in the test name's docstring) and runs it against the C++ FP64
oracle, or against the package's host-side input code where the reference
test covers an input (geometry, materials, Fresnel factors).  The reference
itself cannot be built here (Rust, no toolchain), so these are the pins.
"""
import math

import numpy as np
import pytest

from lumina_b200 import geometry, lattice, materials, types
from lumina_b200.lattice import LatticeSpec
from oracle import oracle as orc

PI = math.pi


def near_c(a, b, tol):
    return abs(complex(a) - complex(b)) < tol


# --- greens.rs:169-262 --------------------------------------------------------

def test_greens_reciprocity():
    """greens.rs:174-190: G(r,r') = G(r',r)^T to 1e-12."""
    k = 2 * PI / 500.0
    g12 = orc.greens([0, 0, 0], [10, 5, 3], k)
    g21 = orc.greens([10, 5, 3], [0, 0, 0], k)
    assert np.max(np.abs(g12 - g21.T)) < 1e-12


def test_greens_self_interaction_rejected():
    """greens.rs:192-199: coincident points are rejected."""
    with pytest.raises(ValueError):
        orc.greens([1, 2, 3], [1, 2, 3], 0.01)


def test_fcd_equals_point_at_distance():
    """greens.rs:201-218: FCD == point G at 10 cells (1e-10)."""
    k = 2 * PI / 500.0
    gp = orc.greens([0, 0, 0], [30, 0, 0], k)
    gf = orc.greens_filtered([0, 0, 0], [30, 0, 0], k, 3.0)
    assert np.max(np.abs(gp - gf)) < 1e-10


def test_fcd_finite_and_different_at_one_cell():
    """greens.rs:220-261: FCD finite at R = d and differs from point G by > 1e-8."""
    k = 2 * PI / 500.0
    gf = orc.greens_filtered([0, 0, 0], [3, 0, 0], k, 3.0)
    gp = orc.greens([0, 0, 0], [3, 0, 0], k)
    assert np.all(np.isfinite(gf.view(np.float64)))
    assert np.max(np.abs(gf - gp)) > 1e-8


# --- assembly.rs:365-393 ----------------------------------------------------

def test_invert_identity_and_isotropic():
    inv = orc.invert_3x3(np.eye(3, dtype=complex))
    assert np.max(np.abs(inv - np.eye(3))) < 1e-12
    a = complex(2.0, 0.5)
    inv = orc.invert_3x3(np.eye(3) * a)
    assert max(abs(inv[i, i] - 1 / a) for i in range(3)) < 1e-12


# --- iterative.rs:208-323 ----------------------------------------------------

def test_gmres_identity_system():
    n = 6
    rhs = np.array([complex(i + 1.0, 0.5 * i) for i in range(n)])
    r = orc.gmres_dense(np.eye(n, dtype=complex), rhs, 1e-10, 100)
    assert r.converged and np.max(np.abs(r.x - rhs)) < 1e-8


def test_gmres_complex_3x3():
    A = np.array([[4 + 1j, -1 + .5j, 0], [-1 - .5j, 4, -1 + .2j], [0, -1 - .2j, 4 - 1j]])
    b = np.array([1, 1j, -1 + .5j])
    r = orc.gmres_dense(A, b, 1e-12, 100)
    assert np.linalg.norm(b - A @ r.x) / np.linalg.norm(b) < 1e-10


def test_gmres_known_solution():
    n = 9
    diag = np.array([complex(2.0 + i, 0.3 * i) for i in range(n)])
    rhs = diag * complex(1.0, -0.5)
    r = orc.gmres_dense(np.diag(diag), rhs, 1e-12, 100)
    assert np.max(np.abs(r.x - complex(1.0, -0.5))) < 1e-8


def test_gmres_convergence_failure():
    r = orc.gmres_dense(np.zeros((3, 3), complex), np.array([1, 1j, 1 + 1j]), 1e-10, 50)
    assert not r.converged


# --- direct.rs:62-117 ------------------------------------------------------------

def test_lu_identity_and_2x2():
    b = np.arange(6, dtype=complex)
    assert np.max(np.abs(orc.lu_solve(np.eye(6, dtype=complex), b) - b)) < 1e-12
    A = np.array([[1 + 1j, 2], [1j, 3 - 1j]])
    b = np.array([5 + 1j, 4 + 2j])
    assert np.max(np.abs(A @ orc.lu_solve(A, b) - b)) < 1e-10


# --- ewald.rs:806-1197 -----------------------------------------------------------

def test_erfc_basic():
    assert abs(orc.erfc(0.0) - 1.0) < 1e-7
    assert orc.erfc(10.0) < 1e-40
    assert abs(orc.erfc(1.5) + orc.erfc(-1.5) - 2.0) < 1e-6


def test_csqrt_positive_imag():
    s = orc.csqrt_positive_imag(complex(-4.0, 0.0))
    assert s.imag > 0 and abs(s.imag - 2.0) < 1e-12
    s = orc.csqrt_positive_imag(complex(9.0, 0.0))
    assert abs(s.real - 3.0) < 1e-12 and abs(s.imag) < 1e-12


SQ100 = LatticeSpec.planar((100.0, 0.0, 0.0), (0.0, 100.0, 0.0))


def test_ewald_self_image_finite():
    g = orc.ewald(SQ100, [0, 0, 0], [0, 0, 0], 2 * PI / 600.0)
    assert np.all(np.isfinite(g.view(np.float64)))


def test_ewald_evaluate_splits():
    lat = LatticeSpec.planar((80.0, 0.0, 0.0), (0.0, 80.0, 0.0))
    k = 2 * PI / 500.0
    r = [10.0, 5.0, 2.0]
    full = orc.ewald(lat, r, [0, 0, 0], k)
    parts = orc.ewald(lat, r, [0, 0, 0], k, "real") + orc.ewald(lat, r, [0, 0, 0], k, "recip")
    assert np.max(np.abs(full - parts)) < 1e-20


def test_ewald_gamma_reciprocity():
    k = 2 * PI / 600.0
    r = np.array([15.0, 8.0, 3.0])
    g = orc.ewald(SQ100, r, [0, 0, 0], k)
    gn = orc.ewald(SQ100, -r, [0, 0, 0], k)
    assert np.max(np.abs(g - gn.T)) < 1e-8


def test_ewald_square_self_image_symmetry():
    g = orc.ewald(SQ100, [0, 0, 0], [0, 0, 0], 2 * PI / 600.0)
    assert near_c(g[0, 0], g[1, 1], 1e-8)
    assert abs(g[0, 1]) < 1e-8


def test_ewald_1d_chain_finite_nonzero_reciprocal():
    chain = LatticeSpec.chain((80.0, 0.0, 0.0))
    k = 2 * PI / 500.0
    g = orc.ewald(chain, [10.0, 5.0, 0.0], [0, 0, 0], k)
    assert np.all(np.isfinite(g.view(np.float64))) and np.max(np.abs(g)) > 1e-12
    k = 2 * PI / 600.0
    r = np.array([10.0, 5.0, 0.0])
    assert np.max(np.abs(orc.ewald(chain, r, [0, 0, 0], k)
                         - orc.ewald(chain, -r, [0, 0, 0], k).T)) < 1e-6


def test_ewald_shell_convergence():
    k = 2 * PI / 600.0
    r = [15.0, 8.0, 3.0]
    g5 = orc.ewald(LatticeSpec((100.0, 0, 0), (0, 100.0, 0), truncation_real=5), r, [0, 0, 0], k)
    g10 = orc.ewald(LatticeSpec((100.0, 0, 0), (0, 100.0, 0), truncation_real=10), r, [0, 0, 0], k)
    assert np.max(np.abs(g5 - g10)) < 0.05 * np.max(np.abs(g5))


def test_ewald_2d_recip_finite():
    g = orc.ewald(SQ100, [10.0, 5.0, 20.0], [0, 0, 0], 2 * PI / 600.0, "recip")
    assert np.all(np.isfinite(g.view(np.float64)))


def test_bessel_table_values():
    assert abs(orc.bessel("k0", 1.0) - 0.4210244382) < 1e-6
    assert abs(orc.bessel("k0", 2.0) - 0.1138938727) < 1e-4
    assert abs(orc.bessel("k0", 5.0) - 0.003691) < 1e-6
    assert abs(orc.bessel("k1", 1.0) - 0.6019072302) < 1e-6
    assert abs(orc.bessel("k1", 2.0) - 0.1399358445) < 1e-4
    assert abs(orc.bessel("y0", 1.0) - 0.08826) < 1e-4
    assert abs(orc.bessel("y0", 2.0) - 0.51038) < 1e-4
    assert abs(orc.bessel("y1", 1.0) + 0.7812) < 1e-4
    assert abs(orc.bessel("y1", 2.0) + 0.1070) < 1e-4
    assert abs(orc.bessel("y1", 0.1) + 6.4590) < 1e-2
    assert abs(orc.bessel("y1", 0.5) + 1.4715) < 1e-3


def test_bessel_k_imaginary_identities():
    for a in (1.0, 2.0, 3.0):
        k0 = orc.bessel_kc(0, complex(0, a))
        assert abs(k0.real + (PI / 2) * orc.bessel("y0", a)) < 1e-5
        assert abs(k0.imag - (PI / 2) * orc.bessel("j0", a)) < 1e-5
        k1 = orc.bessel_kc(1, complex(0, a))
        assert abs(k1.real + (PI / 2) * orc.bessel("j1", a)) < 1e-5
        assert abs(k1.imag + (PI / 2) * orc.bessel("y1", a)) < 1e-5


CH10 = LatticeSpec.chain((10.0, 0.0, 0.0))


def test_1d_recip_reciprocity_nonzero_and_rho_guard():
    k = 0.01
    r = np.array([3.0, 5.0, 0.0])
    g1 = orc.ewald(CH10, r, [0, 0, 0], k, "recip")
    g2 = orc.ewald(CH10, -r, [0, 0, 0], k, "recip")
    assert np.max(np.abs(g1 - g2.T)) < 1e-10
    assert np.sum(np.abs(g1)) > 1e-12
    g0 = orc.ewald(CH10, [3.0, 0.0, 0.0], [0, 0, 0], k, "recip")
    assert np.max(np.abs(g0)) < 1e-30


def test_1d_recip_tensor_elements():
    """ewald.rs:1132-1196: xx, yy, xy against the direct spectral formula."""
    k, a1, dx, rho = 0.01, 10.0, 5.0, 3.0
    g = orc.ewald(CH10, [dx, rho, 0.0], [0, 0, 0], k, "recip")
    two_pi_a = 2 * PI / a1
    norm = 1.0 / (2 * PI * a1)
    gxx = gyy = gxy = 0j
    for m in range(-50, 51):
        gm = m * two_pi_a
        kap = orc.csqrt_positive_imag(complex(gm * gm - k * k, 0.0))
        k0 = orc.bessel_kc(0, kap * rho)
        k1 = orc.bessel_kc(1, kap * rho)
        k1r = kap * k1 / rho
        ph = complex(math.cos(gm * dx), math.sin(gm * dx))
        gxx += ph * (k * k - gm * gm) * k0
        gyy += ph * (gm * gm * k0 + k1r)
        gxy += ph * complex(0, -gm) * k1r
    assert abs(g[0, 0] - gxx * norm) < 1e-8
    assert abs(g[1, 1] - gyy * norm) < 1e-8
    assert abs(g[0, 1] - gxy * norm) < 1e-8
    assert abs(g[0, 1] - g[1, 0]) < 1e-12


# --- lattice.rs:236-302 ----------------------------------------------------------

def test_lattice_area_eta():
    assert abs(SQ100.cell_measure() - 10000.0) < 1e-10
    assert abs(SQ100.eta() - math.sqrt(PI / 10000.0)) < 1e-10
    assert abs(orc.lattice_eta(SQ100) - SQ100.eta()) < 1e-15


# --- substrate.rs:199-335 --------------------------------------------------------

def test_fresnel_factors():
    assert abs(orc.fresnel(2.25, 1.0, False) - 1.25 / 3.25) < 1e-10
    assert abs(orc.fresnel(2.0, 2.0, False)) < 1e-12
    assert abs(orc.fresnel(complex(-100, 5), 1.0, False)) > 0.95
    assert abs(orc.fresnel(2.25, 1.0, True) - 0.2) < 1e-10
    assert abs(orc.fresnel(2.25, 2.25, True)) < 1e-12
    for e in (2.25, complex(-10, 1.5), complex(2.1025, 0.0)):
        assert abs(orc.fresnel(e, 1.0, True) - lattice.fresnel_reflection_amplitude(e, 1.0)) < 1e-14
        assert abs(orc.fresnel(e, 1.0, False) - lattice.fresnel_delta_eps(e, 1.0)) < 1e-14


# --- spline.rs:93-114, johnson_christy.rs:258-279 -------------------------------

def test_spline_through_points_and_package_agrees():
    xs, ys = [1.0, 2.0, 3.0, 4.0, 5.0], [2.0, 3.0, 5.0, 4.0, 1.0]
    ev = orc.spline(xs, ys)
    sp = materials.CubicSpline(xs, ys)
    for x, y in zip(xs, ys):
        assert abs(ev(x) - y) < 1e-10
    for x in np.linspace(0.5, 5.5, 23):
        assert abs(ev(x) - sp.evaluate(x)) < 1e-14


def test_gold_range_and_out_of_range():
    au = materials.JohnsonChristyMaterial.gold()
    lo, hi = au.wavelength_range()
    assert abs(lo - 187.9) < 1e-9 and abs(hi - 892.0) < 1e-9
    with pytest.raises(materials.OutOfRange):
        au.dielectric_function(900.0)
    e = au.dielectric_function(520.0)
    assert e.real < 0 and e.imag > 0


# --- polarisability (types.rs:243-317) -------------------------------------------

def test_rrcm_matches_oracle():
    k = 2 * PI / 520.0
    eps = complex(-3.88, 2.61)
    a_pkg = types.radiative_correction(types.clausius_mossotti(8.0, eps, 1.0), k)
    assert abs(a_pkg - orc.rrcm(8.0, eps, 1.0, k)) < 1e-13 * abs(a_pkg)
    R = geometry.rotation_zyx(20.0, -35.0, 50.0)
    dep = geometry.ellipsoid_depol_factors([10.0, 5.0, 3.0])
    t_pkg = types.ellipsoid_polarisability_tensor(3.375, dep, eps, 1.0, k, R.ravel())
    t_orc = orc.ellipsoid_tensor(3.375, dep, eps, 1.0, k, R.ravel())
    assert np.max(np.abs(t_pkg - t_orc)) < 1e-13 * np.max(np.abs(t_orc))


# --- ellipsoid.rs:120-181 --------------------------------------------------------

def test_depolarisation_factors():
    assert max(abs(v - 1 / 3) for v in geometry.ellipsoid_depol_factors([10, 10, 10])) < 1e-12
    for axes in ([10.0, 5.0, 3.0], [20.0, 20.0, 5.0], [4.0, 8.0, 16.0], [8.0, 8.0, 8.0]):
        assert abs(sum(geometry.ellipsoid_depol_factors(axes)) - 1.0) < 1e-6
    a, b = 20.0, 10.0
    e2 = 1 - (b / a) ** 2
    e = math.sqrt(e2)
    la = (1 - e2) / e2 * (0.5 * math.log((1 + e) / (1 - e)) / e - 1)
    assert abs(geometry.ellipsoid_depol_factors([a, b, b])[0] - la) < 1e-8


# --- geometry (discretise.rs, mie_validation.rs:370-416) ------------------------

def test_discretisation_counts():
    assert len(geometry.discretise_primitive(geometry.Sphere((0, 0, 0), 12.0), 2.0)) == 925
    cyl = geometry.Cylinder((0, 0, 0), (0, 0, 1), 20.0, 5.0)
    pts = geometry.discretise_primitive(cyl, 2.0)
    assert 100 < len(pts) < 400 and np.all(cyl.contains(pts))
    hel = geometry.Helix((0, 0, 0), (0, 0, 1), 10.0, 10.0, 2.0, 3.0)
    pts = geometry.discretise_primitive(hel, 2.0)
    assert len(pts) > 10 and np.all(hel.contains(pts))
    assert geometry.cell_centred_cuboid((60.0, 50.0, 10.0), 1.0).shape == (30000, 3)


# --- solver-level tests (cda_diagnostic.rs, v012_v013_features.rs, mie_validation.rs)

def _solve_lu(pos, alpha, k, fcd, cell, pol=(1, 0, 0)):
    A = orc.assemble(pos, alpha, k, fcd, cell)
    b = orc.incident_field(pos, k, polarisation=pol)
    return orc.lu_solve(A, b)


def test_single_dipole_rayleigh():
    """cda_diagnostic.rs:121-166: one dipole, C_ext = k Im(alpha) within 1 %."""
    k = 2 * PI / 600.0
    vol = 4.0 / 3.0 * PI * 1000.0
    a = orc.rrcm(vol, complex(-10.0, 1.5), 1.0, k)
    alpha = np.eye(3)[None] * a
    pos = np.zeros((1, 3))
    x = _solve_lu(pos, alpha, k, True, 3.0)
    cext = orc.cross_sections(pos, alpha, x, k)[0]
    assert abs(cext - k * a.imag) / (k * a.imag) < 0.01


def _gold_sphere(radius, spacing, wl):
    pos = geometry.discretise_primitive(geometry.Sphere((0, 0, 0), radius), spacing)
    eps = materials.JohnsonChristyMaterial.gold().dielectric_function(wl)
    k = 2 * PI / wl
    a = orc.rrcm(spacing ** 3, eps, 1.0, k)
    return pos, np.broadcast_to(np.eye(3) * a, (len(pos), 3, 3)).copy(), k


def test_cd_zero_for_isotropic_sphere():
    """v012_v013_features.rs:471-498."""
    pos, alpha, k = _gold_sphere(8.0, 2.0, 500.0)
    px = _solve_lu(pos, alpha, k, True, 2.0, (1, 0, 0))
    py = _solve_lu(pos, alpha, k, True, 2.0, (0, 1, 0))
    assert abs(orc.circular_dichroism(px, py, k)) < 1e-6


def test_cext_same_for_x_and_y_pol():
    """v012_v013_features.rs:561-578 (relative 1e-8)."""
    pos, alpha, k = _gold_sphere(8.0, 2.0, 520.0)
    cx = orc.cross_sections(pos, alpha, _solve_lu(pos, alpha, k, True, 2.0, (1, 0, 0)), k)
    cy = orc.cross_sections(pos, alpha, _solve_lu(pos, alpha, k, True, 2.0, (0, 1, 0)), k,
                            polarisation=(0, 1, 0))
    assert abs(cx[0] - cy[0]) < 1e-8 * abs(cx[0]) and abs(cx[1] - cy[1]) < 1e-8 * abs(cx[1])


def test_gmres_agrees_with_direct():
    """mie_validation.rs:305-367: C_ext GMRES vs LU < 1e-4 (here far tighter)."""
    pos = geometry.discretise_primitive(geometry.Sphere((0, 0, 0), 10.0), 3.0)
    k = 2 * PI / 500.0
    a = orc.rrcm(27.0, complex(4.0, 0.5), 1.0, k)
    alpha = np.broadcast_to(np.eye(3) * a, (len(pos), 3, 3)).copy()
    A = orc.assemble(pos, alpha, k, False, 3.0)
    b = orc.incident_field(pos, k)
    x_lu = orc.lu_solve(A, b)
    g = orc.gmres_onthefly(pos, alpha, b, k, False, 3.0, tol=1e-8, max_iter=2000)
    c_lu = orc.cross_sections(pos, alpha, x_lu, k)[0]
    c_gm = orc.cross_sections(pos, alpha, g.x, k)[0]
    assert g.converged and abs(c_gm - c_lu) / c_lu < 1e-6


def test_oracle_lu_matches_numpy():
    pos, alpha, k = _gold_sphere(6.0, 2.0, 520.0)
    A = orc.assemble(pos, alpha, k, True, 2.0)
    b = orc.incident_field(pos, k)
    assert np.max(np.abs(orc.lu_solve(A, b) - np.linalg.solve(A, b))) < 1e-11 * np.max(np.abs(np.linalg.solve(A, b)))


def test_onthefly_equals_assembled_with_all_terms():
    pos, alpha, k = _gold_sphere(5.0, 2.0, 560.0)
    pos = pos + np.array([0.0, 0.0, 10.0])
    sub = lattice.SubstrateRuntime(0.0, complex(0.2, 0.01))
    x = np.random.default_rng(3).standard_normal(3 * len(pos)) * (1 + 0.5j)
    for kw in ({"use_fcd": True, "cell_size": 2.0}, {"use_fcd": True, "cell_size": 2.0, "substrate": sub},
               {"lattice": SQ100, "k_bloch": (0.001, 0, 0)}):
        y = orc.matvec_onthefly(pos, alpha, x, k, **kw)
        A = orc.assemble(pos, alpha, k, **kw)
        assert np.max(np.abs(A @ x - y)) < 1e-13 * np.max(np.abs(y))
