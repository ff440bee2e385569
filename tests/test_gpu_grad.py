"""Adjoint gradients of C_ext on the GPU (lum_grad_cext).

The reference has no gradient code: the GPU gradient is checked against the
oracle's FP64 gradient (dense LU, its own tensor-derivative restatement,
itself pinned by finite differences in test_oracle_grad.py) and against
central finite differences of GPU forward solves (1e-4 nm in position, 1e-6
in eps).  Tolerances: FP64 solves at tol 1e-12 give gradients within 1e-8
(max-norm relative) of the oracle; FP32+refine within 1e-6; FD within 1e-5.
"""
import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from lumina_b200.types import rrcm_array, wavenumber
from oracle import oracle as orc
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def jittered_block(nx=6, ny=5, nz=4, spacing=2.0, jitter=0.2, seed=2):
    g = [np.arange(m) * spacing for m in (nx, ny, nz)]
    X, Y, Z = np.meshgrid(*g, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    return np.ascontiguousarray(pos + np.random.default_rng(seed).uniform(-jitter, jitter, pos.shape))


def rrcm_setup(pos, spacing, wl, eps):
    k = wavenumber(wl, 1.0)
    vol = spacing ** 3
    a = rrcm_array(vol, eps, 1.0, k)
    alpha = np.einsum("i,ab->iab", a, np.eye(3)).astype(np.complex128)
    dinv = np.einsum("i,ab->iab", -1.0 / (vol * (eps - 1.0) ** 2), np.eye(3)).astype(np.complex128)
    return k, alpha, dinv


@pytest.mark.parametrize("pol", [(1, 0, 0), (1 / np.sqrt(2), 1j / np.sqrt(2), 0)],
                         ids=["linear", "circular"])
def test_gradient_matches_oracle(backend, pol):
    pos = jittered_block()
    n = pos.shape[0]
    eps = np.full(n, -12.5 + 1.1j) + np.linspace(0.0, 0.8, n)
    k, alpha, dinv = rrcm_setup(pos, 2.0, 640.0, eps)
    direction = (0.2, 0.1, np.sqrt(0.95))
    c_ref, gr_ref, ge_ref, _ = orc.grad_cext(pos, alpha, k, True, 2.0, direction, pol, 1.0, dinv)
    inv = lb.invert_polarisability(alpha)
    with backend.create_onthefly_session(pos, inv, k, True, 2.0) as s:
        r64 = s.grad_cext(direction, pol, 1.0, dinv, tol=1e-12, max_iter=5000, mode="fp64")
        r32 = s.grad_cext(direction, pol, 1.0, dinv, tol=1e-10, max_iter=5000, mode="fp32_refine")
    assert abs(r64["c_ext"] - c_ref) <= 1e-10 * abs(c_ref)
    assert rel_err(r64["grad_r"], gr_ref) < 1e-8
    assert rel_err(r64["grad_eps"], ge_ref) < 1e-8
    assert rel_err(r32["grad_r"], gr_ref) < 1e-6
    assert rel_err(r32["grad_eps"], ge_ref) < 1e-6
    # the adjoint solve is as hard as the forward one (A^T = A)
    assert abs(r64["info_adjoint"]["iterations"] - r64["info_forward"]["iterations"]) <= 2


def test_gradient_central_differences(backend):
    """GPU gradient against central differences of GPU forward solves."""
    pos = jittered_block(5, 4, 3, seed=8)
    n = pos.shape[0]
    eps = np.full(n, -10.0 + 0.9j)
    k, alpha, dinv = rrcm_setup(pos, 2.0, 600.0, eps)
    direction, pol = (0.0, 0.0, 1.0), (0.0, 1.0, 0.0)
    inv = lb.invert_polarisability(alpha)

    def c_ext(p, inv_a):
        with backend.create_onthefly_session(p, inv_a, k, True, 2.0) as s:
            return s.grad_cext(direction, pol, 1.0, None, tol=1e-13, max_iter=5000,
                               want_eps=False)["c_ext"]

    with backend.create_onthefly_session(pos, inv, k, True, 2.0) as s:
        r = s.grad_cext(direction, pol, 1.0, dinv, tol=1e-13, max_iter=5000)
    h = 1e-4
    scale_r = np.max(np.abs(r["grad_r"]))
    for i, c in [(0, 0), (11, 1), (n - 1, 2)]:
        pp, pm = pos.copy(), pos.copy()
        pp[i, c] += h
        pm[i, c] -= h
        fd = (c_ext(pp, inv) - c_ext(pm, inv)) / (2 * h)
        assert abs(fd - r["grad_r"][i, c]) <= 1e-5 * scale_r, (i, c, fd, r["grad_r"][i, c])
    he = 1e-6
    scale_e = np.max(np.abs(r["grad_eps"]))
    for i in (3, n // 2):
        for part, step in ((0, he), (1, 1j * he)):
            ep, em = eps.copy(), eps.copy()
            ep[i] += step
            em[i] -= step
            ip = lb.invert_polarisability(rrcm_setup(pos, 2.0, 600.0, ep)[1])
            im = lb.invert_polarisability(rrcm_setup(pos, 2.0, 600.0, em)[1])
            fd = (c_ext(pos, ip) - c_ext(pos, im)) / (2 * he)
            assert abs(fd - r["grad_eps"][i, part]) <= 1e-5 * scale_e, (i, part, fd)


def test_circular_dichroism_gradient_helix_dimer(backend):
    """Left-handed helix dimer (4 nm lattice, FCD off so no pair sits on the
    near/far step): dCD/dr and dCD/d eps against the oracle."""
    d = configs.helix_dimer(spacing=4.0)
    w = d.workload
    inv = lb.invert_polarisability(w.alpha)
    dinv = d.dinv_alpha_deps()
    out = {}
    with backend.create_onthefly_session(w.positions, inv, w.k, False, w.cell_size) as s:
        for name, pol in (("L", d.lcp), ("R", d.rcp)):
            out[name] = s.grad_cext(d.direction, pol, 1.0, dinv, tol=1e-12, max_iter=5000)
    ref = {name: orc.grad_cext(w.positions, w.alpha, w.k, False, w.cell_size, d.direction, pol,
                               1.0, dinv)
           for name, pol in (("L", d.lcp), ("R", d.rcp))}
    cd = out["L"]["c_ext"] - out["R"]["c_ext"]
    cd_ref = ref["L"][0] - ref["R"][0]
    assert abs(cd - cd_ref) <= 1e-9 * abs(ref["L"][0])
    g = out["L"]["grad_r"] - out["R"]["grad_r"]
    g_ref = ref["L"][1] - ref["R"][1]
    assert rel_err(g, g_ref) < 1e-7
    ge = out["L"]["grad_eps"] - out["R"]["grad_eps"]
    assert rel_err(ge, ref["L"][2] - ref["R"][2]) < 1e-7


def test_gradient_rejects_periodic_session(backend):
    pw = configs.metasurface(spacing=8.0, diameter=24.0, height=8.0, period=120.0)
    w = pw.workload
    with backend.create_onthefly_session(w.positions, lb.invert_polarisability(w.alpha), w.k,
                                         True, w.cell_size, lattice=pw.lattice,
                                         k_bloch=pw.k_bloch) as s:
        with pytest.raises(lb.InvalidGeometry):
            s.grad_cext((0, 0, 1), (1, 0, 0))
