"""The oracle's nonlinear sources against the reference's own known answers
(nonlinear.rs tests) and the tensor constructors of the host mirror; CPU."""
import numpy as np

from lumina_b200.nonlinear import Chi2Tensor, Chi3Tensor
from oracle import oracle as orc


def test_zero_tensors_give_zero_sources():
    e = np.array([[1.0, 0.5, 0.2]] * 4, complex)
    assert np.all(orc.harmonic_sources(2, e, Chi2Tensor.zero().components) == 0)
    assert np.all(orc.harmonic_sources(3, e, Chi3Tensor.zero().components) == 0)


def test_xxx_and_xxxx_contractions():
    t2 = Chi2Tensor.zero()
    t2.components[0] = 1.0
    p = orc.harmonic_sources(2, [[2.5, 0, 0]], t2.components)
    assert abs(p[0, 0] - 6.25) < 1e-12 and np.all(np.abs(p[0, 1:]) < 1e-12)
    t3 = Chi3Tensor.zero()
    t3.components[0] = 1.0
    p = orc.harmonic_sources(3, [[2.0, 0, 0]], t3.components)
    assert abs(p[0, 0] - 8.0) < 1e-12 and np.all(np.abs(p[0, 1:]) < 1e-12)


def test_tensor_structures():
    t = Chi2Tensor.isotropic_surface(1.0, 0.5)
    for idx, v in ((26, 1.0), (18, 0.5), (22, 0.5), (2, 0.5), (6, 0.5), (14, 0.5), (16, 0.5)):
        assert abs(t.components[idx] - v) < 1e-14
    assert np.count_nonzero(np.abs(t.components) > 1e-14) == 7
    b = Chi3Tensor.isotropic_bulk(1.0, 0.25)
    assert abs(b.components[0] - 1.0) < 1e-14
    for idx in (4, 10, 12):
        assert abs(b.components[idx] - 0.25) < 1e-14


def test_sources_match_numpy_einsum():
    rng = np.random.default_rng(2)
    e = rng.standard_normal((6, 3)) + 1j * rng.standard_normal((6, 3))
    c2 = rng.standard_normal((6, 27)) + 1j * rng.standard_normal((6, 27))
    c3 = rng.standard_normal((6, 81)) + 1j * rng.standard_normal((6, 81))
    p2 = np.einsum("nabc,nb,nc->na", c2.reshape(6, 3, 3, 3), e, e)
    p3 = np.einsum("nabcd,nb,nc,nd->na", c3.reshape(6, 3, 3, 3, 3), e, e, e)
    assert np.max(np.abs(orc.harmonic_sources(2, e, c2) - p2)) < 1e-12 * np.max(np.abs(p2))
    assert np.max(np.abs(orc.harmonic_sources(3, e, c3) - p3)) < 1e-12 * np.max(np.abs(p3))
