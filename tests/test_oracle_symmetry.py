"""The symmetry that the symmetric tile storage of a cached matrix relies on,
checked on the oracle's assemble_interaction_matrix (assembly.rs:45-175).

Free space: A = A^T to rounding, with the point tensor and with the FCD
cell average (greens.rs:34-167), for isotropic and for anisotropic but
symmetric polarisabilities.  The Fresnel image term (assembly.rs:129-156)
keeps A symmetric as well (reciprocity), although the device tile storage
does not take substrates.  The reference's periodic sum (ewald.rs:91-106,
its full spectral sum) does not: there A stays in dense rows."""
import math

import numpy as np
import pytest

from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from lumina_b200.lattice import LatticeSpec, SubstrateRuntime
from oracle import oracle as orc


def _asym(A):
    return float(np.max(np.abs(A - A.T)) / np.max(np.abs(A)))


@pytest.fixture(scope="module")
def sphere():
    pos = discretise_primitive(Sphere((0.0, 0.0, 12.0), 6.0), 2.0)
    return configs.au_workload("s", pos, 2.0, 560.0)


@pytest.mark.parametrize("fcd", [True, False])
def test_free_space_matrix_is_complex_symmetric(sphere, fcd):
    A = orc.assemble(sphere.positions, sphere.alpha, sphere.k, fcd, 2.0)
    assert _asym(A) < 1e-14


def test_symmetric_anisotropic_alpha_keeps_symmetry(sphere):
    rng = np.random.default_rng(5)
    n = sphere.n
    m = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    alpha = (np.eye(3) * (3.0 + 1.5j))[None] + 0.2 * (m + np.transpose(m, (0, 2, 1)))
    A = orc.assemble(sphere.positions, alpha, 2 * math.pi / 480.0, True, 2.0)
    assert _asym(A) < 1e-14


def test_fresnel_image_keeps_symmetry(sphere):
    sub = SubstrateRuntime(0.0, complex(0.45 / 2.45, 0.05))
    A = orc.assemble(sphere.positions, sphere.alpha, sphere.k, True, 2.0, substrate=sub)
    assert _asym(A) < 1e-14


def test_periodic_sum_is_not_symmetric():
    pos = discretise_primitive(Sphere((0.0, 0.0, 12.0), 4.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 560.0)
    L = LatticeSpec.planar((100.0, 0.0, 0.0), (0.0, 100.0, 0.0))
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0, lattice=L)
    assert _asym(A) > 1e-3
