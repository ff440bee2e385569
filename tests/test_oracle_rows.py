"""The oracle's row-range matvecs (bounded samples of matvec_on_the_fly,
assembly.rs:209-318, used to check the device operators at full size) equal
the corresponding rows of the full oracle matvec bit for bit: free space with
FCD, and the periodic metasurface cell with the Ewald lattice, Bloch vector
and Fresnel image."""
import numpy as np

from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from oracle import oracle as orc


def test_rows_equal_full_matvec_free_space():
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 7.0), 1.5)
    w = configs.au_workload("s", pos, 1.5, 540.0)
    rng = np.random.default_rng(3)
    x = rng.standard_normal(3 * w.n) + 1j * rng.standard_normal(3 * w.n)
    y = orc.matvec_onthefly(w.positions, w.alpha, x, w.k, True, 1.5)
    for r0, r1 in ((0, 7), (50, 90), (w.n - 5, w.n)):
        assert np.array_equal(orc.matvec_onthefly_rows(w.positions, w.alpha, x, w.k, True, 1.5,
                                                       r0, r1), y[3 * r0:3 * r1])
        assert np.array_equal(orc.matvec_onthefly_rows_ex(w.positions, w.alpha, x, w.k, True,
                                                          1.5, r0, r1), y[3 * r0:3 * r1])


def test_rows_equal_full_matvec_periodic_substrate():
    pw = configs.metasurface(spacing=8.0, wavelength_nm=600.0)
    w = pw.workload
    rng = np.random.default_rng(4)
    x = rng.standard_normal(3 * w.n) + 1j * rng.standard_normal(3 * w.n)
    kw = dict(lattice=pw.lattice, k_bloch=pw.k_bloch, substrate=pw.substrate)
    y = orc.matvec_onthefly(w.positions, w.alpha, x, w.k, True, w.cell_size, **kw)
    for r0, r1 in ((0, 9), (300, 333), (w.n - 4, w.n)):
        yr = orc.matvec_onthefly_rows_ex(w.positions, w.alpha, x, w.k, True, w.cell_size, r0, r1,
                                         **kw)
        assert np.array_equal(yr, y[3 * r0:3 * r1])
