"""GPU parity of the symmetric tile storage of a device-assembled matrix.

A free-space system (no lattice sum, no substrate) has a complex-symmetric
matrix: G(d) = G(d)^T = G(-d) (greens.rs:34-71) and the FCD cell average is
symmetric in its two dipoles (greens.rs:94-167).  lum_session_assemble with
LUM_STORAGE_SYMMETRIC keeps only the upper-triangle tiles (192 x 192 entries,
64 dipoles a side) and applies each off-diagonal tile twice, as A_IJ x_J and
A_IJ^T x_I.  Its products are compared with the oracle's assembled matrix
(assemble_interaction_matrix, assembly.rs:45-175) at the suite's bars:
FP64 storage 1e-12, FP32 storage 2e-5 (max |error| / max |reference|), and
with the dense-row storage of the same session kind.  Sizes cross the tile
edges: 1, 2, 63, 64, 65, 128 and 129 dipoles, and spheres of a few hundred.
"""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from lumina_b200.backend import InvalidGeometry
from lumina_b200.geometry import Sphere, discretise_primitive
from lumina_b200.lattice import LatticeSpec, SubstrateRuntime
from oracle import oracle as orc
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu

BARS = {"fp64": 1e-12, "fp32": 2e-5}


def _jittered(rng, n, spacing=2.0):
    """n dipoles of a jittered cubic lattice (FCD cell = spacing)."""
    side = max(1, math.ceil(n ** (1.0 / 3.0)))
    g = np.stack(np.meshgrid(*[np.arange(side)] * 3, indexing="ij"), -1).reshape(-1, 3)
    pos = spacing * g[:n].astype(np.float64) + rng.uniform(-0.15, 0.15, (n, 3))
    return configs.au_workload("jit", pos, spacing, 560.0)


def _sphere(wl=520.0, radius=6.0):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), radius), 2.0)
    return configs.au_workload("s", pos, 2.0, wl)


@pytest.mark.parametrize("n", [1, 2, 63, 64, 65, 128, 129])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_sym_tiles_match_oracle_across_tile_edges(backend, rng, n, precision):
    w = _jittered(rng, n)
    inv = lb.invert_polarisability(w.alpha)
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    x = rand_vec(rng, 3 * n)
    with backend.assemble_and_create_session(w.positions, w.k, inv, use_fcd=True, cell_size=2.0,
                                             precision=precision, symmetric=True) as s:
        y = s.matvec(x, precision)
    assert rel_err(y, A @ x) < BARS[precision]


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("fcd", [True, False])
def test_sym_tiles_match_dense_rows(backend, rng, precision, fcd):
    """A sphere of 1,791 dipoles (29 tiles a side): the tile product equals the
    dense-row product of the same assembly (FP64 to rounding; FP32 within the
    FP32 bar, as the two sum in different orders)."""
    w = _sphere(600.0, 15.0)
    inv = lb.invert_polarisability(w.alpha)
    x = rand_vec(rng, 3 * w.n)
    with backend.assemble_and_create_session(w.positions, w.k, inv, use_fcd=fcd, cell_size=2.0,
                                             precision=precision) as d, \
            backend.assemble_and_create_session(w.positions, w.k, inv, use_fcd=fcd,
                                                cell_size=2.0, precision=precision,
                                                symmetric=True) as s:
        yd = d.matvec(x, precision)
        ys = s.matvec(x, precision)
        ys2 = s.matvec(x, precision)
    assert rel_err(ys, yd) < (1e-13 if precision == "fp64" else 2e-6)
    assert np.array_equal(ys, ys2)  # no atomics: products are reproducible bit for bit
    y_ref = orc.matvec_onthefly(w.positions, w.alpha, x, w.k, fcd, 2.0)
    assert rel_err(ys, y_ref) < BARS[precision]


def test_sym_tiles_anisotropic_alpha(backend, rng):
    """Anisotropic, non-symmetric alpha^-1 sits in the diagonal tiles, which
    are stored whole."""
    base = discretise_primitive(Sphere((1.0, -2.0, 0.5), 7.0), 1.5)
    pos = base + rng.uniform(-0.2, 0.2, base.shape)
    n = pos.shape[0]
    alpha = (np.eye(3) * (3.0 + 1.5j))[None] + 0.3 * (rng.standard_normal((n, 3, 3))
                                                      + 1j * rng.standard_normal((n, 3, 3)))
    k = 2 * math.pi / 480.0
    inv = lb.invert_polarisability(alpha)
    A = orc.assemble(pos, alpha, k, True, 1.5)
    x = rand_vec(rng, 3 * n)
    with backend.assemble_and_create_session(pos, k, inv, use_fcd=True, cell_size=1.5,
                                             precision="fp64", symmetric=True) as s:
        y = s.matvec(x, "fp64")
    assert n > 64
    assert rel_err(y, A @ x) < 1e-12


def test_sym_tiles_set_wavelength(backend, rng):
    w1, w2 = _sphere(520.0), _sphere(640.0)
    inv1, inv2 = lb.invert_polarisability(w1.alpha), lb.invert_polarisability(w2.alpha)
    x = rand_vec(rng, 3 * w1.n)
    with backend.assemble_and_create_session(w1.positions, w1.k, inv1, use_fcd=True,
                                             cell_size=2.0, precision="fp64",
                                             symmetric=True) as s:
        s.set_wavelength(w2.k, inv2)
        y = s.matvec(x, "fp64")
        with pytest.raises(InvalidGeometry):
            s.set_wavelength(w2.k, inv2, SubstrateRuntime(0.0, complex(0.45 / 2.45)))
    y_ref = orc.matvec_onthefly(w2.positions, w2.alpha, x, w2.k, True, 2.0)
    assert rel_err(y, y_ref) < 1e-12


@pytest.mark.parametrize("storage", ["fp32", "fp64"])
def test_sym_tiles_solve_meets_gate(backend, storage):
    """FP32+refine GMRES on the tile product (FP64 restart residuals from the
    on-the-fly FP64 operator for FP32 storage): C_ext within 1e-6 of LU."""
    w = _sphere(520.0, 8.0)
    inv = lb.invert_polarisability(w.alpha)
    b = orc.incident_field(w.positions, w.k)
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    ref = orc.cross_sections(w.positions, w.alpha, orc.lu_solve(A, b), w.k)
    with backend.assemble_and_create_session(w.positions, w.k, inv, use_fcd=True, cell_size=2.0,
                                             precision=storage, symmetric=True) as s:
        x, info = s.solve(b, 1e-10, 5000, 30, "fp32_refine")
    cs = lb.cross_sections(w.positions, inv, x, w.k, lb.IncidentField())
    assert info["converged"] == 1
    assert abs(cs[0] - ref[0]) / abs(ref[0]) < 1e-6


def test_sym_tiles_vectors_and_rhs_batch(backend, rng):
    """Multi-vector products run one tile product per vector (the tensor-core
    product needs dense rows); a right-hand-side batch over the session agrees
    with single solves."""
    w = _sphere(600.0)
    inv = lb.invert_polarisability(w.alpha)
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    X = rng.standard_normal((3 * w.n, 5)) + 1j * rng.standard_normal((3 * w.n, 5))
    rhs = [orc.incident_field(w.positions, w.k, d, e)
           for d, e in (((0, 0, 1), (1, 0, 0)), ((0, 0, 1), (0, 1, 0)), ((1, 0, 0), (0, 0, 1)))]
    with backend.assemble_and_create_session(w.positions, w.k, inv, use_fcd=True, cell_size=2.0,
                                             precision="fp64", symmetric=True) as s:
        Y = s.matmul(X, "cuda_cores")
        Ya = s.matmul(X, "auto")
        with pytest.raises(InvalidGeometry):
            s.matmul(X, "tensor")
        with pytest.raises(InvalidGeometry):  # dense rows cannot be uploaded into tiles
            s.upload_matrix(A)
        B = s.rhs_batch(len(rhs))
        xb, info = B.solve(np.concatenate(rhs), 1e-10, 5000, 30, "fp64")
        B.close()
        singles = [s.solve(r, 1e-10, 5000, 30, "fp64")[0] for r in rhs]
    assert rel_err(Y, A @ X) < 1e-12 and np.array_equal(Y, Ya)
    for q in range(len(rhs)):
        assert info[q]["converged"] == 1
        assert rel_err(xb[3 * w.n * q:3 * w.n * (q + 1)], singles[q]) < 1e-7


def test_sym_tiles_reject_lattice_and_substrate(backend):
    w = _sphere()
    inv = lb.invert_polarisability(w.alpha)
    with pytest.raises(InvalidGeometry):
        backend.assemble_and_create_session(w.positions, w.k, inv, True, 2.0,
                                            substrate=SubstrateRuntime(0.0, complex(0.2)),
                                            symmetric=True)
    lat = LatticeSpec.planar((400.0, 0.0, 0.0), (0.0, 400.0, 0.0))
    with pytest.raises(InvalidGeometry):
        backend.assemble_and_create_session(w.positions, w.k, inv, True, 2.0, lattice=lat,
                                            symmetric=True)


@pytest.mark.parametrize("precision", ["fp64", "fp32_refine"])
def test_cdasolver_cached_branch_keeps_symmetric_tiles(backend, precision):
    """CdaSolver's cached branch (cda/mod.rs:346-374) keeps a free-space
    matrix as symmetric tiles; cross sections equal those over dense rows,
    and a substrate system on the same solver falls back to dense rows."""
    from lumina_b200.lattice import SubstrateRuntime as Sub
    w = configs.sphere_au_925()
    kw = dict(iterative_threshold=0, cell_size=2.0, matrix_memory_budget=2 << 30,
              precision=precision)
    sym = lb.CdaSolver(backend=backend, **kw)
    dense = lb.CdaSolver(backend=backend, symmetric_storage=False, **kw)
    ds = lb.DipoleSet(w.positions, w.alpha)
    params = lb.SimulationParams(solver_tolerance=1e-10, max_iterations=20000)
    a = sym.compute_cross_sections(ds, 520.0, params)
    assert sym._kept[0][0] == "cached" and sym._kept[0][1].endswith("+sym")
    b = dense.compute_cross_sections(ds, 520.0, params)
    assert not dense._kept[0][1].endswith("+sym")
    assert abs(a.extinction - b.extinction) <= 1e-8 * abs(b.extinction)
    assert abs(a.absorption - b.absorption) <= 1e-8 * abs(b.absorption)
    pos = w.positions + np.array([0.0, 0.0, 20.0])
    ds2 = lb.DipoleSet(pos, w.alpha)
    p2 = lb.SimulationParams(solver_tolerance=1e-10, max_iterations=20000,
                             substrate_runtime=Sub(0.0, complex(0.45 / 2.45)))
    c = sym.compute_cross_sections(ds2, 520.0, p2)
    assert sym._kept[0][1] in ("fp64", "fp32") and c.extinction > 0
    sym.close()
    dense.close()
