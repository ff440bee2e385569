"""The oracle's field functions (fields.rs) against known answers and an
independent numpy restatement; CPU only."""
import math

import numpy as np

from oracle import oracle as orc


def _greens_np(r1, r2, k):
    """greens.rs:34-71 written out in numpy (independent of the oracle)."""
    d = np.asarray(r1, float) - np.asarray(r2, float)
    r = np.linalg.norm(d)
    kr = k * r
    pref = np.exp(1j * kr) * k * k / (4 * math.pi * r)
    a = 1 + (1j * kr - 1) / kr ** 2
    b = (3 - 3j * kr - kr ** 2) / kr ** 2
    n = d / r
    return pref * (a * np.eye(3) + b * np.outer(n, n))


def test_far_field_single_dipole_pattern():
    # |(I - rr) p|^2 = sin^2(theta) for p = z, wherever the dipole sits
    for pos in ([0, 0, 0], [3.0, -2.0, 5.0]):
        th, ph, inten = orc.far_field([pos], [0, 0, 1], 0.0121, 13, 8)
        assert np.allclose(inten, np.sin(th) ** 2, rtol=0, atol=1e-14)
        assert np.allclose(th.reshape(13, 8)[:, 0], np.linspace(0, math.pi, 13))
        assert np.allclose(ph.reshape(13, 8)[0], 2 * math.pi * np.arange(8) / 8)


def test_far_field_matches_numpy():
    rng = np.random.default_rng(5)
    pos = rng.uniform(-10, 10, (9, 3))
    mom = rng.standard_normal((9, 3)) + 1j * rng.standard_normal((9, 3))
    k = 2 * math.pi / 600
    th, ph, inten = orc.far_field(pos, mom, k, 7, 6)
    for q in range(th.size):
        rh = np.array([math.sin(th[q]) * math.cos(ph[q]), math.sin(th[q]) * math.sin(ph[q]),
                       math.cos(th[q])])
        f = (mom * np.exp(-1j * k * (pos @ rh))[:, None]).sum(0)
        ft = f - (rh @ f) * rh
        assert abs(inten[q] - np.sum(np.abs(ft) ** 2)) <= 1e-12 * max(1.0, inten[q])


def test_near_field_plane_basis_and_grid():
    P, E = orc.near_field_plane([1.0, 2.0, 3.0], [0, 0, 2.0], 10.0, 5.0, 3, 2)
    # normal z: u = x, v = z x x = y; iy outer, ix inner
    expect = [[1 + u, 2 + v, 3.0] for v in (-5.0, 5.0) for u in (-10.0, 0.0, 10.0)]
    assert np.allclose(P, expect, rtol=0, atol=1e-14)
    assert np.allclose(E, [-9.0, 11.0, -3.0, 7.0])
    # normal x: seed y, u = y, v = x X y = z
    P, _ = orc.near_field_plane([0, 0, 0], [1.0, 0, 0], 1.0, 1.0, 2, 2)
    assert np.allclose(P[1], [0.0, 1.0, -1.0]) and np.allclose(P[2], [0.0, -1.0, 1.0])
    # nx = ny = 1: the step is 0, so the single point is the (-hw, -hh) corner,
    # not the centre (fields.rs:71-80)
    n = np.array([0.3, -0.2, 0.9]) / np.linalg.norm([0.3, -0.2, 0.9])
    u = np.array([1.0, 0, 0]) - n[0] * n
    u /= np.linalg.norm(u)
    v = np.cross(n, u)
    P, _ = orc.near_field_plane([4.0, 5.0, 6.0], [0.3, -0.2, 0.9], 7.0, 8.0, 1, 1)
    assert np.allclose(P[0], np.array([4.0, 5.0, 6.0]) - 7.0 * u - 8.0 * v, atol=1e-13)


def test_field_at_points_matches_numpy_and_skips_coincident():
    rng = np.random.default_rng(9)
    pos = rng.uniform(-6, 6, (7, 3))
    mom = rng.standard_normal((7, 3)) + 1j * rng.standard_normal((7, 3))
    k = 2 * math.pi / 520
    obs = np.vstack([rng.uniform(-15, 15, (5, 3)), pos[3]])  # the last point is dipole 3
    e = orc.field_at_points(pos, mom, k, obs, direction=(0, 0, 1), polarisation=(1, 0, 0))
    for q, o in enumerate(obs):
        ref = np.exp(1j * k * o[2]) * np.array([1.0, 0, 0], complex)
        for i in range(7):
            if np.sum((o - pos[i]) ** 2) < 1e-20:
                continue
            ref = ref + _greens_np(o, pos[i], k) @ mom[i]
        assert np.max(np.abs(e[q] - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_field_with_no_dipoles_is_incident():
    obs = np.array([[0.0, 0.0, 10.0], [1.0, 2.0, -3.0]])
    k = 0.01
    e = orc.field_at_points(np.zeros((0, 3)), np.zeros(0), k, obs, direction=(0, 0, 1),
                            polarisation=(0, 1, 0), amplitude=2.0)
    assert np.allclose(e[:, 1], 2.0 * np.exp(1j * k * obs[:, 2]))
    assert np.allclose(e[:, [0, 2]], 0.0)
