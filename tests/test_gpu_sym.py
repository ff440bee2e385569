"""GPU parity of the symmetric pair schemes (each unordered pair evaluated
once): every FP32 build of pairs_f32_sym.cuh, forced with LUMINA_F32_SYM=v
(1: 2 rows per thread, 2 CTAs/SM; 2: 2 rows, 3 CTAs/SM; 3: 4 rows, 4 CTAs/SM;
4: 4 rows, 3 CTAs/SM; 5, 6: builds 1 and 4 with the step loop unrolled by two;
7, 8: 8 rows, 4 and 5 CTAs/SM; 9, 10, 11: 4 rows at 4 CTAs/SM unrolled by two,
4 rows at 3 CTAs/SM unrolled by four, 8 rows at 4 CTAs/SM unrolled by two; 12, 13:
4 rows at 4 CTAs/SM unrolled by four, 4 rows at 3 CTAs/SM unrolled by eight),
their two-vector builds, and the FP64 scheme of
pairs_f64_sym.cuh, forced with LUMINA_F64_SYM=1, so that they run at sizes
the oracle handles.  Tolerances: the FP32 bar 2e-5, the FP64 bar 1e-12."""
import math

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from lumina_b200.lattice import SubstrateRuntime
from oracle import oracle as orc
from tests.conftest import rand_vec, rel_err

pytestmark = pytest.mark.gpu

SYM_VARIANTS = ("1", "2", "3", "4", "5", "6", "7", "8", "9", "10", "11", "12", "13")
SYM2_VARIANTS = ("1", "2", "3", "4")


def _cases(rng):
    # N below, at and across superblock boundaries (512), jittered (lo != 0)
    # and exact lattices (lo == 0), FCD on and off
    out = []
    for r, spacing in ((4.0, 2.0), (9.0, 2.0), (11.0, 2.0)):
        pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), r), spacing)
        out.append(("sphere%d" % pos.shape[0], pos, True, spacing))
    base = discretise_primitive(Sphere((0.3, -0.2, 0.1), 10.0), 1.9)
    out.append(("jitter", base + rng.uniform(-0.15, 0.15, base.shape), False, 1.9))
    return out


def _alpha(rng, n):
    return (np.eye(3) * (2.0 + 1.0j))[None] + 0.2 * (rng.standard_normal((n, 3, 3)) +
                                                     1j * rng.standard_normal((n, 3, 3)))


@pytest.mark.parametrize("variant", SYM_VARIANTS)
def test_sym_matvec_matches_oracle(backend, rng, monkeypatch, variant):
    monkeypatch.setenv("LUMINA_F32_SYM", variant)
    for name, pos, fcd, cell in _cases(rng):
        n = pos.shape[0]
        alpha = _alpha(rng, n)
        k = 2 * math.pi / 540.0
        x = rand_vec(rng, 3 * n)
        y_ref = orc.matvec_onthefly(pos, alpha, x, k, fcd, cell)
        with backend.create_onthefly_session(pos, lb.invert_polarisability(alpha), k, fcd,
                                             cell) as s:
            cfg = s.kernel_config()
            assert cfg["f32_sym"] == int(variant), name
            assert cfg["sym_variant"].startswith("sym_rows"), name
            y = s.matvec(x, "fp32")
        assert rel_err(y, y_ref) < 2e-5, (name, variant)


def test_sym64_matvec_matches_oracle(backend, rng, monkeypatch):
    monkeypatch.setenv("LUMINA_F64_SYM", "1")
    for name, pos, fcd, cell in _cases(rng):
        n = pos.shape[0]
        alpha = _alpha(rng, n)
        k = 2 * math.pi / 540.0
        x = rand_vec(rng, 3 * n)
        y_ref = orc.matvec_onthefly(pos, alpha, x, k, fcd, cell)
        with backend.create_onthefly_session(pos, lb.invert_polarisability(alpha), k, fcd,
                                             cell) as s:
            assert s.kernel_config()["f64_sym"] == 1, name
            y = s.matvec(x, "fp64")
        assert rel_err(y, y_ref) < 1e-12, name


def test_sym64_excluded_with_substrate(backend, rng, monkeypatch):
    """The image term is not symmetric in (i, j): a substrate session keeps
    the split FP64 kernel even when the symmetric one is asked for."""
    monkeypatch.setenv("LUMINA_F64_SYM", "1")
    pos = discretise_primitive(Sphere((0.0, 0.0, 8.0), 5.0), 2.0)
    n = pos.shape[0]
    alpha = _alpha(rng, n)
    k = 2 * math.pi / 560.0
    sub = SubstrateRuntime(0.0, complex(0.45 / 2.45))
    with backend.create_onthefly_session(pos, lb.invert_polarisability(alpha), k, True, 2.0,
                                         substrate=sub) as s:
        assert s.kernel_config()["f64_sym"] == 0


@pytest.mark.parametrize("variant", ("1", "3"))
def test_sym_solve_meets_gate(backend, monkeypatch, variant):
    monkeypatch.setenv("LUMINA_F32_SYM", variant)
    monkeypatch.setenv("LUMINA_F64_SYM", "1")
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 10.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 520.0)
    inv = lb.invert_polarisability(w.alpha)
    b = orc.incident_field(w.positions, w.k)
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    cs_ref = orc.cross_sections(w.positions, w.alpha, orc.lu_solve(A, b), w.k)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, 2.0) as s:
        x, info = s.solve(b, 1e-10, 3000, 30, "fp32_refine")
        x64, info64 = s.solve(b, 1e-10, 3000, 30, "fp64")
    for sol, inf in ((x, info), (x64, info64)):
        cs = lb.cross_sections(w.positions, inv, sol, w.k, lb.IncidentField())
        assert inf["converged"] == 1
        assert abs(cs[0] - cs_ref[0]) / abs(cs_ref[0]) < 1e-6


def test_sym_equals_split_scheme(backend, rng, monkeypatch):
    """The same session geometry under every FP32 scheme, and both FP64
    schemes: the products agree to FP32 accuracy (FP64: 1e-13; different
    summation order)."""
    pos = configs.cell_centred_cuboid((14.0, 12.0, 8.0), 1.0)  # N = 1344: 3 superblocks
    w = configs.au_workload("c", pos, 1.0, 650.0)
    inv = lb.invert_polarisability(w.alpha)
    x = rand_vec(rng, 3 * w.n)
    out = {}
    y64 = {}
    for flag in SYM_VARIANTS + ("0",):
        monkeypatch.setenv("LUMINA_F32_SYM", flag)
        monkeypatch.setenv("LUMINA_F64_SYM", "1" if flag == "1" else "0")
        with backend.create_onthefly_session(w.positions, inv, w.k, True, 1.0) as s:
            assert s.kernel_config()["f32_sym"] == int(flag)
            out[flag] = s.matvec(x, "fp32")
            y64[flag] = s.matvec(x, "fp64")
    for flag in SYM_VARIANTS:
        assert rel_err(out[flag], y64["0"]) < 2e-5
        assert rel_err(out[flag], out["0"]) < 2e-5
    assert rel_err(y64["1"], y64["0"]) < 1e-13


def test_sym_deterministic(backend, rng, monkeypatch):
    """Fixed-order slots: two applications of each scheme are bitwise equal."""
    monkeypatch.setenv("LUMINA_F32_SYM", "3")
    monkeypatch.setenv("LUMINA_F64_SYM", "1")
    pos = configs.cell_centred_cuboid((12.0, 10.0, 9.0), 1.0)  # N = 1080
    w = configs.au_workload("c", pos, 1.0, 600.0)
    x = rand_vec(rng, 3 * w.n)
    with backend.create_onthefly_session(w.positions, lb.invert_polarisability(w.alpha), w.k,
                                         True, 1.0) as s:
        a32, b32 = s.matvec(x, "fp32"), s.matvec(x, "fp32")
        a64, b64 = s.matvec(x, "fp64"), s.matvec(x, "fp64")
    assert np.array_equal(a32, b32)
    assert np.array_equal(a64, b64)


@pytest.mark.parametrize("variant", SYM2_VARIANTS)
def test_sym2_two_vector_product_matches_oracle(backend, rng, monkeypatch, variant):
    """The two-vector symmetric builds (FP32 forced with LUMINA_F32_SYM=v,
    FP64 with LUMINA_F64_SYM=1) through a right-hand-side batch's operator
    (two vectors per launch, the path of lockstep forward + adjoint solves):
    each vector against the oracle, an odd count so the last vector takes the
    single-vector scheme."""
    monkeypatch.setenv("LUMINA_F32_SYM", variant)
    monkeypatch.setenv("LUMINA_F64_SYM", "1")
    for name, pos, fcd, cell in _cases(rng):
        n = pos.shape[0]
        alpha = _alpha(rng, n)
        k = 2 * math.pi / 600.0
        xs = [rand_vec(rng, 3 * n) for _ in range(3)]
        with backend.create_onthefly_session(pos, lb.invert_polarisability(alpha), k, fcd,
                                             cell) as s:
            B = s.rhs_batch(3)
            y = B.matvec(np.concatenate(xs), "fp32")
            y64 = B.matvec(np.concatenate(xs), "fp64")
            cfg = s.kernel_config()
            B.close()
        assert cfg["f32x2_sym"] == int(variant) and cfg["f64_sym"] == 1, name
        for q in range(3):
            y_ref = orc.matvec_onthefly(pos, alpha, xs[q], k, fcd, cell)
            sl = slice(3 * n * q, 3 * n * (q + 1))
            assert rel_err(y[sl], y_ref) < 2e-5, (name, variant, q)
            assert rel_err(y64[sl], y_ref) < 1e-12, (name, variant, q)


def test_sym2_lockstep_solves_match_single(backend, monkeypatch):
    """Lockstep solves of two polarisations over the symmetric two-vector
    builds reach the C_ext of the single solves."""
    monkeypatch.setenv("LUMINA_F32_SYM", "1")
    monkeypatch.setenv("LUMINA_F64_SYM", "1")
    w = configs.cuboid_au((14.0, 12.0, 10.0), 1.0, 600.0)
    inv = lb.invert_polarisability(w.alpha)
    pols = [(1.0, 0.0, 0.0), (0.0, 1.0, 0.0)]
    B = np.stack([lb.incident_field(w.positions, w.k, lb.IncidentField((0.0, 0.0, 1.0), p, 1.0))
                  for p in pols])
    with backend.create_onthefly_session(w.positions, inv, w.k, True, w.cell_size) as s:
        X, infos = s.solve_multi(B, 1e-10, 4000, 30, "fp32_refine")
        assert s.kernel_config()["f32x2_sym"] == 1
        for r, p in enumerate(pols):
            x1, _ = s.solve(B[r], 1e-10, 4000, 30, "fp32_refine")
            inc = lb.IncidentField((0.0, 0.0, 1.0), p, 1.0)
            c1 = lb.cross_sections(w.positions, inv, x1, w.k, inc)[0]
            cm = lb.cross_sections(w.positions, inv, X[r], w.k, inc)[0]
            assert infos[r]["converged"] == 1
            assert abs(cm - c1) <= 1e-8 * abs(c1)
