"""Parity at the headline size: the Au cuboid 60 x 50 x 10 nm on the
cell-centred 1 nm lattice (N = 30,000), FCD cell 1 nm, RRCM gold.

* Operator rows: the tuned FP32 operator (and the symmetric FP32 builds
  forced one by one) and the FP64 operator against the oracle's rows of
  matvec_on_the_fly (assembly.rs:209-318) on 320 sampled rows -- the first
  superblock, a superblock boundary, the middle, and the last (partial)
  superblock -- at the suite's tolerances, 2e-5 (FP32) and 1e-12 (FP64).
* Solves: FP32+refine and plain FP64 GMRES(30) to tol 1e-8 against the full
  FP64 oracle solves stored in tests/golden/cuboid30k_oracle.json
  (make_cuboid30k_oracle.py): C_ext within 1e-6 (the precision gate) and the
  stored moments of 514 dipoles within 1e-6 of their largest magnitude.
"""
import json
import os

import numpy as np
import pytest

import lumina_b200 as lb
from lumina_b200 import configs
from oracle import oracle as orc
from tests.conftest import rand_vec

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "cuboid30k_oracle.json")
N = 30000
ROW_RANGES = ((0, 64), (512 * 29 - 32, 512 * 29 + 32), (15000, 15064), (29640, 29704),
              (N - 64, N))


@pytest.fixture(scope="module")
def cuboid():
    w = configs.cuboid_au_30k(520.0)
    assert w.n == N
    rng = np.random.default_rng(30000)
    x = rand_vec(rng, 3 * N)
    ref = {r: orc.matvec_onthefly_rows(w.positions, w.alpha, x, w.k, True, 1.0, r[0], r[1])
           for r in ROW_RANGES}
    return w, x, ref


def _rows(y):
    return np.concatenate([y[3 * a:3 * b] for a, b in ROW_RANGES])


def _ref_rows(ref):
    return np.concatenate([ref[r] for r in ROW_RANGES])


def _err(y, yref):
    return float(np.max(np.abs(y - yref)) / np.max(np.abs(yref)))


def test_cuboid30k_tuned_operator_rows_match_oracle(backend, cuboid, monkeypatch):
    monkeypatch.delenv("LUMINA_F32_SYM", raising=False)
    monkeypatch.delenv("LUMINA_F64_SYM", raising=False)
    w, x, ref = cuboid
    inv = lb.invert_polarisability(w.alpha)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, 1.0) as s:
        y32 = s.matvec(x, "fp32")
        y64 = s.matvec(x, "fp64")
    yref = _ref_rows(ref)
    assert _err(_rows(y32), yref) < 2e-5
    assert _err(_rows(y64), yref) < 1e-12


@pytest.mark.parametrize("variant", ("1", "3", "6", "7"))
def test_cuboid30k_symmetric_builds_match_oracle(backend, cuboid, monkeypatch, variant):
    monkeypatch.setenv("LUMINA_F32_SYM", variant)
    monkeypatch.setenv("LUMINA_F64_SYM", "1")
    w, x, ref = cuboid
    inv = lb.invert_polarisability(w.alpha)
    with backend.create_onthefly_session(w.positions, inv, w.k, True, 1.0) as s:
        cfg = s.kernel_config()
        assert cfg["f32_sym"] == int(variant) and cfg["f64_sym"] == 1
        assert cfg["sym_superblocks"] == (N + 511) // 512
        y32 = s.matvec(x, "fp32")
        y64 = s.matvec(x, "fp64")
    yref = _ref_rows(ref)
    assert _err(_rows(y32), yref) < 2e-5
    assert _err(_rows(y64), yref) < 1e-12


def test_cuboid30k_solves_match_oracle_solve(backend, monkeypatch):
    monkeypatch.delenv("LUMINA_F32_SYM", raising=False)
    monkeypatch.delenv("LUMINA_F64_SYM", raising=False)
    with open(FIXTURE) as f:
        data = json.load(f)
    assert data["solves"]
    for rec in data["solves"]:
        w = configs.cuboid_au_30k(rec["wavelength_nm"])
        assert abs(w.k - rec["k"]) < 1e-15 * rec["k"]
        inv = lb.invert_polarisability(w.alpha)
        b = lb.incident_field(w.positions, w.k, lb.IncidentField())
        idx = np.asarray(rec["sample_dipoles"])
        p_ref = (np.asarray(rec["sample_moments_re"]) +
                 1j * np.asarray(rec["sample_moments_im"])).reshape(-1, 3)
        with backend.create_onthefly_session(w.positions, inv, w.k, True, 1.0) as s:
            for mode in ("fp32_refine", "fp64"):
                x, info = s.solve(b, rec["tol"], 5000, 30, mode)
                assert info["converged"] == 1, mode
                cs = lb.cross_sections(w.positions, inv, x, w.k, lb.IncidentField())
                assert abs(cs[0] - rec["c_ext"]) / abs(rec["c_ext"]) <= 1e-6, mode
                assert abs(cs[1] - rec["c_abs"]) / abs(rec["c_abs"]) <= 1e-6, mode
                p = x.reshape(-1, 3)[idx]
                assert np.max(np.abs(p - p_ref)) / np.max(np.abs(p_ref)) <= 1e-6, mode
