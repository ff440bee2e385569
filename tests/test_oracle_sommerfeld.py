"""The oracle's Sommerfeld reflected tensor (sommerfeld.rs) against the
reference's own unit tests (sommerfeld.rs:424-556, substrate.rs:319-334)
and against an independent numpy restatement of the integrand, which guards
the C transcription (constants, segment limits, term order).
"""
import math

import numpy as np
import pytest

from lumina_b200.lattice import SommerfeldRuntime, SubstrateRuntime, SubstrateSpec
from oracle import oracle as orc

TOL = 1e-6  # sommerfeld.rs:428


def _somm(wl, eps_sub, eps_env, z0=0.0):
    return SommerfeldRuntime(z0, wl, complex(eps_sub), eps_env)


# --- the reference's Bessel tests (sommerfeld.rs:432-473) --------------------
def test_j0_at_zero():
    assert abs(orc.somm_bessel(0, 0.0) - 1.0) < TOL


def test_j0_first_root():
    assert abs(orc.somm_bessel(0, 2.404825557)) < 1e-5


def test_j1_at_zero():
    assert abs(orc.somm_bessel(1, 0.0)) < TOL


def test_j1_first_root():
    assert abs(orc.somm_bessel(1, 3.83170597)) < 1e-5


def test_j2_at_zero():
    assert abs(orc.somm_bessel(2, 0.0)) < TOL


def test_j2_recurrence():
    x = 3.0
    assert abs(orc.somm_bessel(2, x) - ((2.0 / x) * orc.somm_bessel(1, x) - orc.somm_bessel(0, x))) < TOL


def test_bessel_coefficients_are_the_modules_own():
    """Below x = 8 J0 follows the rational approximation (~1e-8 of the exact
    function); from x = 8 on, sommerfeld.rs's asymptotic coefficients differ
    from the exact expansion, so its J0 / J1 are off by ~1e-3 there.  The
    oracle keeps them: the reflected tensor is defined by them."""
    from scipy.special import j0, j1
    for x in (0.3, 1.7, 4.2, 6.9):
        assert abs(orc.somm_bessel(0, x) - j0(x)) < 1e-8
    assert abs(orc.somm_bessel(0, 8.0) - j0(8.0)) > 1e-3
    assert abs(orc.somm_bessel(1, 10.0) - j1(10.0)) > 1e-4


# --- the reference's tensor tests (sommerfeld.rs:477-555) --------------------
def test_no_substrate_zero_tensor():
    g = orc.sommerfeld_tensor(_somm(500.0, 2.25, 2.25), [0.0, 0.0, 10.0], [3.0, 0.0, 8.0])
    assert np.abs(g).max() < 1e-10


def test_tensor_symmetry_reciprocity():
    g = orc.sommerfeld_tensor(_somm(600.0, 2.25, 1.0), [5.0, 3.0, 12.0], [2.0, 1.0, 8.0])
    assert abs(g[0, 1] - g[1, 0]) < 1e-10
    assert abs(g[0, 2] - g[2, 0]) < 1e-10
    assert abs(g[1, 2] - g[2, 1]) < 1e-10


def test_xz_zero_for_zero_rho():
    g = orc.sommerfeld_tensor(_somm(600.0, 2.25, 1.0), [0.0, 0.0, 12.0], [0.0, 0.0, 8.0])
    assert abs(g[0, 2]) < 1e-8 and abs(g[1, 2]) < 1e-8 and abs(g[0, 1]) < 1e-8


def test_far_field_decay():
    g = orc.sommerfeld_tensor(_somm(500.0, 2.25, 1.0), [0.0, 0.0, 2502.5], [0.0, 0.0, 2497.5])
    assert np.isfinite(g).all()


def test_sommerfeld_matches_fresnel_on_axis_large_dz():
    lam = 600.0
    dz = 2.0 * lam
    g = orc.sommerfeld_tensor(_somm(lam, 2.25, 1.0), [0.0, 0.0, 0.6 * dz], [0.0, 0.0, 0.4 * dz])
    assert abs(g[0, 0] - g[1, 1]) < 1e-8 * max(abs(g[0, 0]), 1e-20)
    assert np.isfinite(g).all()


def test_substrate_runtime_sommerfeld():
    """substrate.rs:319-334."""
    spec = SubstrateSpec(z_interface=5.0, material="SiO2_Palik", use_retarded=True,
                         use_sommerfeld=True)
    rt = SubstrateRuntime.from_spec(spec, 2.25, 1.0, 600.0)
    assert isinstance(rt, SommerfeldRuntime)
    assert rt.z_interface == 5.0
    assert not SubstrateSpec().use_sommerfeld


def test_below_interface_gives_zero():
    g = orc.sommerfeld_tensor(_somm(600.0, 2.25, 1.0, z0=10.0), [0.0, 0.0, 4.0], [1.0, 0.0, 6.0])
    assert np.abs(g).max() == 0.0


# --- independent numpy restatement -------------------------------------------
_GX = np.array([-0.991455371120813, -0.949107912342758, -0.864864423359769,
                -0.741531185599394, -0.586087235467691, -0.405845151377397,
                -0.207784955007898, 0.0, 0.207784955007898, 0.405845151377397,
                0.586087235467691, 0.741531185599394, 0.864864423359769, 0.949107912342758,
                0.991455371120813])
_GW = np.array([0.022935322010529, 0.063092092629979, 0.104790010322250, 0.140653259715525,
                0.169004726639267, 0.190350578064785, 0.204432940075298, 0.209482141084728,
                0.204432940075298, 0.190350578064785, 0.169004726639267, 0.140653259715525,
                0.104790010322250, 0.063092092629979, 0.022935322010529])


def _sqrt_pos_im(z):
    s = np.sqrt(np.asarray(z, np.complex128))
    return np.where(s.imag < 0, -s, s)


def _np_tensor(wl, eps_sub, eps_env, ri, rj, z0=0.0):
    k0 = 2 * math.pi / wl
    k = k0 * math.sqrt(eps_env)
    k_sub = _sqrt_pos_im(eps_sub * k0 * k0)
    dz = (ri[2] - z0) + (rj[2] - z0)
    if dz <= 0:
        return np.zeros((3, 3), complex)
    dx, dy = ri[0] - rj[0], ri[1] - rj[1]
    rho = math.hypot(dx, dy)
    phi = math.atan2(dy, dx)
    kmax = max(10 * math.log(10) / dz, 5 * k) if dz > 1e-6 else 20 * k
    segs = [(0.0, k)]
    seg2 = k_sub.real > 1.001 * k
    if seg2:
        segs.append((k, k_sub.real))
    lo = max(k_sub.real, k) if seg2 else k
    if kmax > 1.001 * lo:
        segs.append((lo, kmax))
    I = np.zeros(5, complex)
    for a, b in segs:
        kp = 0.5 * (a + b) + 0.5 * (b - a) * _GX
        w = _GW * 0.5 * (b - a)
        kz = _sqrt_pos_im(k * k - kp * kp + 0j)
        kzs = _sqrt_pos_im(eps_sub * k * k / eps_env - kp * kp)
        rs = (kz - kzs) / (kz + kzs)
        rp = (eps_sub * kz - eps_env * kzs) / (eps_sub * kz + eps_env * kzs)
        ph = np.exp(1j * kz * dz)
        x = kp * rho
        J0 = np.array([orc.somm_bessel(0, v) for v in x])
        J1 = np.array([orc.somm_bessel(1, v) for v in x])
        J2 = np.array([orc.somm_bessel(2, v) for v in x])
        f = kp / kz
        I += [np.sum(w * rs * J0 * ph * f), np.sum(w * rp * kz * kz / k ** 2 * J0 * ph * f),
              np.sum(w * rp * kp * kp / k ** 2 * J0 * ph * f),
              np.sum(w * rp * kp / k * kz / k * J1 * ph),
              np.sum(w * rp * kz * kz / k ** 2 * J2 * ph * f)]
    pre = 1j / (8 * math.pi)
    c, s = math.cos(phi), math.sin(phi)
    c2, s2 = 2 * c * c - 1, 2 * s * c
    g = np.empty((3, 3), complex)
    g[0, 0] = pre * (I[0] + I[1] - I[4] * c2)
    g[1, 1] = pre * (I[0] + I[1] + I[4] * c2)
    g[2, 2] = -pre * I[2]
    g[0, 1] = g[1, 0] = -pre * I[4] * s2
    g[0, 2] = g[2, 0] = pre * I[3] * c
    g[1, 2] = g[2, 1] = pre * I[3] * s
    return g


@pytest.mark.parametrize("wl,eps_sub,eps_env", [
    (600.0, 2.25, 1.0),              # glass in air: three segments
    (520.0, -4.7 + 2.4j, 1.0),       # Au-like: Re k_sub < k_env, no middle segment
    (700.0, 12.0 + 0.1j, 1.77),      # high index under water
])
def test_oracle_matches_numpy_restatement(wl, eps_sub, eps_env):
    rng = np.random.default_rng(7)
    for _ in range(6):
        ri = rng.uniform(-30, 30, 3)
        rj = rng.uniform(-30, 30, 3)
        ri[2], rj[2] = rng.uniform(0.5, 40), rng.uniform(0.5, 40)
        g_ref = _np_tensor(wl, eps_sub, eps_env, ri, rj)
        g = orc.sommerfeld_tensor(_somm(wl, eps_sub, eps_env), ri, rj)
        assert np.abs(g - g_ref).max() <= 1e-11 * np.abs(g_ref).max()


def test_assembly_and_matvec_add_the_reflected_blocks():
    """assembly.rs:157-166 and :296-303: every block (i, j), i == j included,
    gets -G_refl; the on-the-fly matvec equals the assembled product."""
    rng = np.random.default_rng(3)
    n = 7
    pos = rng.uniform(-8, 8, (n, 3))
    pos[:, 2] = rng.uniform(2, 12, n)
    alpha = np.tile((50.0 + 10.0j) * np.eye(3, dtype=complex), (n, 1, 1))
    k = 2 * math.pi / 600.0
    somm = _somm(600.0, 2.25, 1.0)
    A0 = orc.assemble(pos, alpha, k, False, 3.0)
    A = orc.assemble_sommerfeld(pos, alpha, k, somm, False, 3.0)
    for i in range(n):
        for j in range(n):
            g = orc.sommerfeld_tensor(somm, pos[i], pos[j])
            blk = A[3 * i:3 * i + 3, 3 * j:3 * j + 3] - A0[3 * i:3 * i + 3, 3 * j:3 * j + 3]
            assert np.abs(blk + g).max() <= 1e-15 * max(np.abs(g).max(), 1e-300) + 1e-18
    x = rng.standard_normal(3 * n) + 1j * rng.standard_normal(3 * n)
    y = orc.matvec_sommerfeld(pos, alpha, x, k, somm, False, 3.0)
    assert np.abs(y - A @ x).max() <= 1e-12 * np.abs(y).max()
