"""The oracle's adjoint gradient of C_ext against central finite differences of
its own C_ext (dense LU).  The reference has no gradient code, so this is
what pins the oracle gradient (parity with the reference is unpinned here).

Steps: 1e-4 nm in position, 1e-6 in eps.  Jittered positions keep every
pair away from the FCD near/far switch at 2*cell, where C_ext has a step.
"""
import numpy as np
import pytest

from lumina_b200.types import rrcm_array, wavenumber
from oracle import oracle as orc


def jittered_cluster(n_side=3, spacing=2.0, jitter=0.15, seed=4):
    g = np.arange(n_side) * spacing
    X, Y, Z = np.meshgrid(g, g, g[:2], indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    pos = pos + np.random.default_rng(seed).uniform(-jitter, jitter, pos.shape)
    return np.ascontiguousarray(pos)


def rrcm_alpha(eps, vol, k):
    a = rrcm_array(vol, np.asarray(eps), 1.0, k)
    return np.einsum("i,ab->iab", a, np.eye(3)).astype(np.complex128)


def dinv_deps(eps, vol):
    d = -1.0 / (vol * (np.asarray(eps) - 1.0) ** 2)  # d(1/alpha)/d eps for RRCM, eps_m = 1
    return np.einsum("i,ab->iab", d, np.eye(3)).astype(np.complex128)


@pytest.mark.parametrize("pol", [(1, 0, 0), (1 / np.sqrt(2), 1j / np.sqrt(2), 0)],
                         ids=["linear", "circular"])
@pytest.mark.parametrize("use_fcd", [True, False])
def test_oracle_gradient_matches_finite_differences(pol, use_fcd):
    pos = jittered_cluster()
    n = pos.shape[0]
    spacing = 2.0
    vol = spacing ** 3
    k = wavenumber(650.0, 1.0)
    eps = np.full(n, -13.6 + 1.05j) + np.linspace(0, 0.5, n)
    alpha = rrcm_alpha(eps, vol, k)
    direction = (0.3, -0.2, np.sqrt(1 - 0.13))
    c0, gr, ge, _ = orc.grad_cext(pos, alpha, k, use_fcd, spacing, direction, pol, 1.0,
                                  dinv_deps(eps, vol))
    assert c0 > 0
    h = 1e-4
    for i, c in [(0, 0), (3, 1), (7, 2), (n - 1, 0)]:
        pp, pm = pos.copy(), pos.copy()
        pp[i, c] += h
        pm[i, c] -= h
        cp = orc.grad_cext(pp, alpha, k, use_fcd, spacing, direction, pol)[0]
        cm = orc.grad_cext(pm, alpha, k, use_fcd, spacing, direction, pol)[0]
        fd = (cp - cm) / (2 * h)
        assert abs(fd - gr[i, c]) <= 1e-6 * np.max(np.abs(gr)) + 1e-6 * abs(fd), (i, c, fd, gr[i, c])
    he = 1e-6
    for i in (0, 5, n - 1):
        for part, step in ((0, he), (1, 1j * he)):
            ep, em = eps.copy(), eps.copy()
            ep[i] += step
            em[i] -= step
            cp = orc.grad_cext(pos, rrcm_alpha(ep, vol, k), k, use_fcd, spacing, direction, pol)[0]
            cm = orc.grad_cext(pos, rrcm_alpha(em, vol, k), k, use_fcd, spacing, direction, pol)[0]
            fd = (cp - cm) / (2 * he)
            assert abs(fd - ge[i, part]) <= 1e-5 * np.max(np.abs(ge)) + 1e-5 * abs(fd), \
                (i, part, fd, ge[i, part])


def test_oracle_gradient_cext_equals_cross_sections():
    """The C_ext the gradient routine returns is the reference's C_ext
    (cda/mod.rs:175-236) for a real polarisation."""
    pos = jittered_cluster(seed=9)
    n = pos.shape[0]
    k = wavenumber(600.0, 1.0)
    alpha = rrcm_alpha(np.full(n, -10 + 1.2j), 8.0, k)
    c0, _, _, mom = orc.grad_cext(pos, alpha, k, True, 2.0, (0, 0, 1), (0, 1, 0))
    cs = orc.cross_sections(pos, alpha, mom, k, (0, 0, 1), (0, 1, 0))
    assert abs(c0 - cs[0]) <= 1e-12 * abs(cs[0])
