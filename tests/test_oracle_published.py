"""The oracle against absolute numbers the reference itself published.

docs/src/theory/validation.md:112-118 tabulates the FCD extinction error
against Mie theory for the gold sphere of R = 10 nm at d = 2 nm (N = 515,
the run of tests/mie_validation.rs:235-302: CdaSolver::with_fcd(1000, true,
2.0), RRCM Johnson & Christy gold, vacuum; N <= 1000 so the direct LU
branch), with the J&C permittivity at each wavelength.  The oracle (assembly,
LU, cross sections) and the Mie restatement (oracle/mie.py) reproduce every
row: the published errors are given as "~16 %" etc., so they are checked to
within 1.5 percentage points, the permittivities to the table's two
decimals.
"""
import math

import numpy as np
import pytest

from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from oracle import oracle as orc
from oracle.mie import mie_cross_sections

# wavelength (nm): (eps_1, eps_2, published FCD error in %)
PUBLISHED_FCD = {
    420.0: (-1.70, 5.71, 16.0),
    480.0: (-1.78, 4.55, 13.0),
    510.0: (-3.15, 3.06, 24.0),
    550.0: (-5.93, 2.10, 81.0),
    600.0: (-9.42, 1.50, 112.0),
}


@pytest.fixture(scope="module")
def sphere_r10_d2():
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 10.0), 2.0)
    return pos


def test_sphere_r10_d2_count(sphere_r10_d2):
    # "N ~ 515 dipoles" (validation.md:110)
    assert sphere_r10_d2.shape[0] == 515


@pytest.mark.parametrize("wl", sorted(PUBLISHED_FCD))
def test_fcd_error_table_reproduced(sphere_r10_d2, wl):
    e1, e2, err_pub = PUBLISHED_FCD[wl]
    eps = configs.gold_eps(wl)
    assert round(eps.real, 2) == pytest.approx(e1, abs=1e-9)
    assert round(eps.imag, 2) == pytest.approx(e2, abs=1e-9)
    w = configs.au_workload("sphere_r10_d2", sphere_r10_d2, 2.0, wl)
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    p = orc.lu_solve(A, orc.incident_field(w.positions, w.k))
    c_ext = orc.cross_sections(w.positions, w.alpha, p, w.k)[0]
    mie_ext = mie_cross_sections(10.0, wl, eps, 1.0)[0]
    err = 100.0 * abs(c_ext - mie_ext) / mie_ext
    assert abs(err - err_pub) < 1.5, f"{wl} nm: oracle FCD error {err:.1f} % vs published ~{err_pub} %"


# The table's point-dipole column (v0.1.0, before FCD) matches the point CDA
# of the R = 10 nm sphere on the 3 nm lattice of tests/mie_validation.rs:
# 30-98 in the interband rows.  Its Drude rows (~50 % at 550 nm, > 100 % at
# 600 nm) are not reproduced (the oracle gives 63.7 % and 95.7 %) and are not
# checked.
PUBLISHED_POINT_INTERBAND = {420.0: 25.0, 480.0: 22.0, 510.0: 28.0}


@pytest.mark.parametrize("wl", sorted(PUBLISHED_POINT_INTERBAND))
def test_point_cda_interband_rows_reproduced(wl):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 10.0), 3.0)
    w = configs.au_workload("sphere_r10_d3", pos, 3.0, wl)
    A = orc.assemble(w.positions, w.alpha, w.k, False, 3.0)
    p = orc.lu_solve(A, orc.incident_field(w.positions, w.k))
    c_ext = orc.cross_sections(w.positions, w.alpha, p, w.k)[0]
    mie_ext = mie_cross_sections(10.0, wl, configs.gold_eps(wl), 1.0)[0]
    err = 100.0 * abs(c_ext - mie_ext) / mie_ext
    assert abs(err - PUBLISHED_POINT_INTERBAND[wl]) < 1.5, f"{wl} nm: {err:.1f} %"


def test_fcd_improves_on_point_cda_in_interband(sphere_r10_d2):
    """validation.md:112-116: FCD beats the point-dipole CDA at 420-510 nm."""
    for wl in (420.0, 480.0, 510.0):
        w = configs.au_workload("s", sphere_r10_d2, 2.0, wl)
        mie_ext = mie_cross_sections(10.0, wl, configs.gold_eps(wl), 1.0)[0]
        errs = []
        for fcd in (False, True):
            A = orc.assemble(w.positions, w.alpha, w.k, fcd, 2.0)
            p = orc.lu_solve(A, orc.incident_field(w.positions, w.k))
            errs.append(abs(orc.cross_sections(w.positions, w.alpha, p, w.k)[0] - mie_ext))
        assert errs[1] < errs[0], wl
