"""Periodic metasurface on a substrate (the Ewald + Fresnel-image path) on the
GPU against the oracle's per-pair Ewald evaluation (ewald.rs:91-338,
assembly.rs:87-170), at reduced size.

On a dipole lattice the library tabulates the periodic tensors once per
wavelength (table.cu); jittered positions force the per-pair Ewald kernel.
Tolerances: FP64 1e-10 (both sides sum 242 lattice terms per pair in a
different order), FP32 2e-5, FP32+refine C_ext vs LU 1e-6.
"""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from oracle import oracle as orc
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu


def small_metasurface(jitter=0.0, wl=620.0, seed=0):
    pw = configs.metasurface(spacing=2.0, wavelength_nm=wl, diameter=12.0, height=6.0, period=120.0)
    w = pw.workload
    pos = w.positions
    if jitter:
        pos = pos + np.random.default_rng(seed).uniform(-jitter, jitter, pos.shape)
    return pw, pos, w.alpha, w.k


@pytest.mark.parametrize("jitter", [0.0, 0.05], ids=["lattice_table", "per_pair"])
def test_periodic_matvec_matches_oracle(backend, rng, jitter):
    pw, pos, alpha, k = small_metasurface(jitter)
    inv = lb.invert_polarisability(alpha)
    x = rand_vec(rng, 3 * len(pos))
    y_ref = orc.matvec_onthefly(pos, alpha, x, k, True, 2.0, lattice=pw.lattice,
                                k_bloch=pw.k_bloch, substrate=pw.substrate)
    with backend.create_onthefly_session(pos, inv, k, True, 2.0, lattice=pw.lattice,
                                         k_bloch=pw.k_bloch, substrate=pw.substrate) as s:
        assert rel_err(s.matvec(x, "fp64"), y_ref) < 1e-10
        assert rel_err(s.matvec(x, "fp32"), y_ref) < 2e-5
        cfg = s.kernel_config()
    A = orc.assemble(pos, alpha, k, True, 2.0, lattice=pw.lattice, k_bloch=pw.k_bloch,
                     substrate=pw.substrate)
    for prec, tol in (("fp64", 1e-10), ("fp32", 2e-5)):
        with backend.assemble_and_create_session(pos, k, inv, use_fcd=True, cell_size=2.0,
                                                 lattice=pw.lattice, k_bloch=pw.k_bloch,
                                                 substrate=pw.substrate, precision=prec) as s:
            assert rel_err(s.matvec(x, prec), A @ x) < tol


def test_periodic_solve_fp32_refine_gate(backend):
    pw, pos, alpha, k = small_metasurface()
    inv = lb.invert_polarisability(alpha)
    A = orc.assemble(pos, alpha, k, True, 2.0, lattice=pw.lattice, k_bloch=pw.k_bloch,
                     substrate=pw.substrate)
    inc = pw.incident
    b = orc.incident_field(pos, k, inc.direction, inc.polarisation)
    x_lu = orc.lu_solve(A, b)
    cs_lu = orc.cross_sections(pos, alpha, x_lu, k, inc.direction, inc.polarisation)
    with backend.create_onthefly_session(pos, inv, k, True, 2.0, lattice=pw.lattice,
                                         k_bloch=pw.k_bloch, substrate=pw.substrate) as s:
        for mode in ("fp64", "fp32_refine"):
            x, info = s.solve(b, 1e-10, 5000, 30, mode)
            cs = lb.cross_sections(pos, inv, x, k, inc)
            assert info["converged"] == 1
            assert abs(cs[0] - cs_lu[0]) / abs(cs_lu[0]) < 1e-6, mode
            assert abs(cs[1] - cs_lu[1]) / abs(cs_lu[1]) < 1e-6, mode


def test_periodic_set_wavelength_rebuilds_tables(backend, rng):
    pw1, pos, alpha1, k1 = small_metasurface(wl=620.0)
    pw2, _, alpha2, k2 = small_metasurface(wl=700.0)
    x = rand_vec(rng, 3 * len(pos))
    inv1, inv2 = lb.invert_polarisability(alpha1), lb.invert_polarisability(alpha2)
    with backend.create_onthefly_session(pos, inv1, k1, True, 2.0, lattice=pw1.lattice,
                                         k_bloch=pw1.k_bloch, substrate=pw1.substrate) as s:
        s.set_wavelength(k2, inv2, pw2.substrate)
        y = s.matvec(x, "fp64")
    # the Bloch vector is part of the session's geometry: keep pw1's
    y_ref = orc.matvec_onthefly(pos, alpha2, x, k2, True, 2.0, lattice=pw1.lattice,
                                k_bloch=pw1.k_bloch, substrate=pw2.substrate)
    assert rel_err(y, y_ref) < 1e-10
