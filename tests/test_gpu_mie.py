"""CDA against Mie theory through the device solver (the reference's
tests/mie_validation.rs:30-230, 30 % bar): CdaSolver with its defaults
(FCD, cell 3 nm, the direct-size branch solved by device GMRES to 1e-12),
and the device result against the oracle's LU at 1e-9."""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200.geometry import Sphere, discretise_primitive
from lumina_b200.materials import JohnsonChristyMaterial
from lumina_b200.types import clausius_mossotti, radiative_correction
from oracle import oracle as orc
from oracle.mie import mie_cross_sections

pytestmark = pytest.mark.gpu


def _solve(backend, eps, wl, radius=10.0, spacing=3.0):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), radius), spacing)
    k = 2.0 * math.pi / wl
    a = radiative_correction(clausius_mossotti(spacing ** 3, eps, 1.0), k)
    ds = lb.DipoleSet(pos, np.full(pos.shape[0], a))
    cs = lb.CdaSolver(backend=backend).compute_cross_sections(ds, wl, lb.SimulationParams())
    A = orc.assemble(pos, ds.polarisability, k, True, 3.0)
    ref = orc.cross_sections(pos, ds.polarisability, orc.lu_solve(A, orc.incident_field(pos, k)), k)
    assert abs(cs.extinction - ref[0]) / abs(ref[0]) < 1e-9
    return cs


@pytest.mark.parametrize("wl", [420.0, 450.0, 480.0, 510.0])
def test_gold_sphere_vs_mie(backend, wl):
    eps = JohnsonChristyMaterial.gold().dielectric_function(wl)
    cs = _solve(backend, eps, wl)
    mie = mie_cross_sections(10.0, wl, eps)[0]
    assert abs(cs.extinction - mie) / mie < 0.30
    assert cs.extinction > 0 and cs.absorption > 0


@pytest.mark.parametrize("eps", [4.0 + 0.0j, 4.0 + 0.5j, 6.0 + 1.0j, -1.0 + 3.0j])
def test_dielectric_sphere_vs_mie(backend, eps):
    for wl in (500.0, 600.0, 700.0):
        cs = _solve(backend, eps, wl)
        mie = mie_cross_sections(10.0, wl, eps)[0]
        assert abs(cs.extinction - mie) / mie < 0.30, (eps, wl)


def test_finer_discretisation_does_not_degrade(backend):
    wl, eps = 550.0, 4.0 + 0.5j
    mie = mie_cross_sections(8.0, wl, eps)[0]
    prev = math.inf
    for spacing in (4.0, 3.0, 2.5, 2.0):
        err = abs(_solve(backend, eps, wl, 8.0, spacing).extinction - mie) / mie
        assert err < prev * 3.0
        prev = err
