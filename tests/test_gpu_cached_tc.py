"""GPU parity of the multi-right-hand-side cached product Y = A X.

The tensor-core method (tcgen05, TF32 operands split hi + lo, three products
per operand pair, FP32 accumulation) is compared with the exact FP64 product
of the FP32-stored matrix, and with the CUDA-core method.  Tolerances
(max |error| / max |reference| over the block):
  tensor cores vs exact product of the stored matrix   1e-5
  FP32-stored physics matrix vs the FP64 oracle matrix  2e-5 (the FP32 bar)
"""
import math

import numpy as np
import pytest
import torch

import lumina_b200 as lb
from lumina_b200 import configs
from lumina_b200.geometry import Sphere, discretise_primitive
from oracle import oracle as orc
from tests.conftest import rel_err

pytestmark = pytest.mark.gpu


def _rand_matrix(rng, dim):
    return rng.standard_normal((dim, dim)) + 1j * rng.standard_normal((dim, dim))


def _rand_block(rng, dim, nrhs):
    return rng.standard_normal((dim, nrhs)) + 1j * rng.standard_normal((dim, nrhs))


@pytest.mark.parametrize("dim", [48, 999, 1536])
@pytest.mark.parametrize("nrhs", [1, 3, 8, 17, 64, 130, 300])
def test_tensor_product_matches_stored_matrix(backend, rng, dim, nrhs):
    A = _rand_matrix(rng, dim)
    X = _rand_block(rng, dim, nrhs)
    A32 = A.astype(np.complex64).astype(np.complex128)
    Y_ref = A32 @ X
    with backend.create_session(dim, "fp32") as s:
        s.upload_matrix(A)
        Y = s.matmul(X, "tensor")
        Yc = s.matmul(X, "cuda_cores")
    assert Y.shape == (dim, nrhs)
    assert rel_err(Y, Y_ref) < 1e-5
    assert rel_err(Yc, Y_ref) < 1e-12
    # every column on its own, so a wrong column mapping cannot hide
    for r in range(nrhs):
        assert rel_err(Y[:, r], Y_ref[:, r]) < 1e-5


def test_tensor_product_repeated_calls_and_auto(backend, rng):
    dim, nrhs = 600, 12
    A = _rand_matrix(rng, dim)
    A32 = A.astype(np.complex64).astype(np.complex128)
    with backend.create_session(dim, "fp32") as s:
        s.upload_matrix(A)
        for _ in range(3):
            X = _rand_block(rng, dim, nrhs)
            Y = s.matmul(X, "auto")
            assert rel_err(Y, A32 @ X) < 1e-5
        # fewer columns after more: the workspace is reused, not re-sized down
        X = _rand_block(rng, dim, 2)
        assert rel_err(s.matmul(X, "tensor"), A32 @ X) < 1e-5


def test_assembled_physics_matrix(backend, rng):
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 8.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 520.0)
    inv = lb.invert_polarisability(w.alpha)
    dim = 3 * w.n
    A_ref = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    X = _rand_block(rng, dim, 24)
    with backend.assemble_and_create_session(w.positions, w.k, inv, True, 2.0,
                                             precision="fp32") as s:
        Y = s.matmul(X, "tensor")
        y0 = s.matvec(X[:, 0], "fp32")
    Y_ref = A_ref @ X
    assert rel_err(Y, Y_ref) < 2e-5
    # the single-vector GEMV of the same stored matrix agrees with column 0
    assert rel_err(Y[:, 0], y0) < 1e-5


def test_long_accumulation_chain_accuracy(backend, rng):
    """N = 1000 Au cuboid (K = 6000 real terms per output): the tensor-core
    accumulation is cut into short chains summed on the CUDA cores, so the
    product keeps FP32-operator accuracy against the FP64 oracle matrix
    (one long TMEM chain gave ~1e-5 here and ~1e-4 at N = 6000)."""
    w = configs.cuboid_au((10.0, 10.0, 10.0), 1.0, 520.0)
    inv = lb.invert_polarisability(w.alpha)
    A_ref = orc.assemble(w.positions, w.alpha, w.k, True, 1.0)
    X = _rand_block(rng, 3 * w.n, 16)
    with backend.assemble_and_create_session(w.positions, w.k, inv, True, 1.0,
                                             precision="fp32") as s:
        Y = s.matmul(X, "tensor")
    assert rel_err(Y, A_ref @ X) < 5e-6


def test_row_major_device_entry(backend, rng):
    dim, nrhs = 513, 9
    A = _rand_matrix(rng, dim)
    A32 = A.astype(np.complex64).astype(np.complex128)
    X = _rand_block(rng, dim, nrhs)
    Xd = torch.from_numpy(np.ascontiguousarray(X)).to("cuda")  # row-major dim x nrhs
    Yd = torch.zeros_like(Xd)
    with backend.create_session(dim, "fp32") as s:
        s.upload_matrix(A)
        s.matmul_device(Xd.data_ptr(), Yd.data_ptr(), nrhs)
        torch.cuda.synchronize()
    assert rel_err(Yd.cpu().numpy(), A32 @ X) < 1e-5


def test_vectors_device_entry(backend, rng):
    dim, nrhs = 390, 5
    A = _rand_matrix(rng, dim)
    A32 = A.astype(np.complex64).astype(np.complex128)
    X = _rand_block(rng, dim, nrhs)
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).to("cuda")  # vectors back to back
    Yd = torch.zeros_like(Xd)
    with backend.create_session(dim, "fp32") as s:
        s.upload_matrix(A)
        s.matmul_vectors_device(Xd.data_ptr(), Yd.data_ptr(), nrhs, "tensor")
        torch.cuda.synchronize()
    assert rel_err(Yd.cpu().numpy().T, A32 @ X) < 1e-5


def test_tensor_method_needs_fp32_storage(backend, rng):
    dim = 64
    with backend.create_session(dim, "fp64") as s:
        s.upload_matrix(_rand_matrix(rng, dim))
        X = _rand_block(rng, dim, 4)
        with pytest.raises(lb.SolverError):
            s.matmul(X, "tensor")
        # the CUDA-core method serves FP64 storage exactly
        A = _rand_matrix(rng, dim)
        s.upload_matrix(A)
        assert rel_err(s.matmul(X, "auto"), A @ X) < 1e-13


def _directions(m):
    """m incidence directions on a cone around +z with polarisations
    perpendicular to them (real, unit)."""
    out = []
    for q in range(m):
        th = 0.3 + 0.5 * q / max(m - 1, 1)
        ph = 2 * math.pi * q / m
        d = np.array([math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)])
        e = np.cross(d, [0.0, 0.0, 1.0])
        e /= np.linalg.norm(e)
        out.append((d, e))
    return out


@pytest.mark.parametrize("storage", ["fp32", "fp64"])
def test_rhs_batch_solve_matches_lu(backend, storage):
    """Many incidence directions of one cached matrix solved together: every
    FP32 step is one tensor-core product over all right-hand sides; C_ext of
    each direction meets the 1e-6 gate against the LU oracle."""
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 6.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 520.0)
    inv = lb.invert_polarisability(w.alpha)
    dirs = _directions(9)
    A = orc.assemble(w.positions, w.alpha, w.k, True, 2.0)
    rhs = [orc.incident_field(w.positions, w.k, d, e) for d, e in dirs]
    with backend.assemble_and_create_session(w.positions, w.k, inv, True, 2.0,
                                             precision=storage) as S:
        B = S.rhs_batch(len(dirs))
        x, info = B.solve(np.concatenate(rhs), 1e-10, 5000, 30, "fp32_refine")
        B.close()
    for q, (d, e) in enumerate(dirs):
        xq = x[3 * w.n * q:3 * w.n * (q + 1)]
        inc = lb.IncidentField(tuple(d), tuple(e))
        cs = lb.cross_sections(w.positions, inv, xq, w.k, inc)
        ref = orc.cross_sections(w.positions, w.alpha, orc.lu_solve(A, rhs[q]), w.k, d, e)
        assert info[q]["converged"] == 1
        assert abs(cs[0] - ref[0]) / abs(ref[0]) < 1e-6


def test_rhs_batch_on_the_fly_session(backend):
    """The same right-hand-side batch over an on-the-fly session (two vectors
    per pair-kernel launch) agrees with single solves."""
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 6.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 600.0)
    inv = lb.invert_polarisability(w.alpha)
    dirs = _directions(5)
    rhs = [orc.incident_field(w.positions, w.k, d, e) for d, e in dirs]
    with backend.create_onthefly_session(w.positions, inv, w.k, True, 2.0) as S:
        B = S.rhs_batch(len(dirs))
        x, info = B.solve(np.concatenate(rhs), 1e-10, 5000, 30, "fp64")
        B.close()
        for q in range(len(dirs)):
            x1, _ = S.solve(rhs[q], 1e-10, 5000, 30, "fp64")
            assert rel_err(x[3 * w.n * q:3 * w.n * (q + 1)], x1) < 1e-7


def test_tensor_wait_limit_reports_timeout_and_context_recovers(backend, rng, monkeypatch):
    """A pipeline wait that never completes (the first CTA's split warps
    withhold one arrival, LUMINA_TC_WITHHOLD_SPLIT=1) gives up after the
    launch's wait limit (LUMINA_TC_WAIT_CYCLES, here ~10 ms of SM clocks):
    the product returns TIMEOUT, and the next product on the same session is
    exact again."""
    dim, nrhs = 999, 8
    A = _rand_matrix(rng, dim)
    X = _rand_block(rng, dim, nrhs)
    Y_ref = A.astype(np.complex64).astype(np.complex128) @ X
    with backend.create_session(dim, "fp32") as s:
        s.upload_matrix(A)
        monkeypatch.setenv("LUMINA_TC_WAIT_CYCLES", "20000000")
        monkeypatch.setenv("LUMINA_TC_WITHHOLD_SPLIT", "1")
        with pytest.raises(lb.DeviceTimeout):
            s.matmul(X, "tensor")
        monkeypatch.delenv("LUMINA_TC_WITHHOLD_SPLIT")
        Y = s.matmul(X, "tensor")  # short limit kept: a healthy product meets it
        monkeypatch.delenv("LUMINA_TC_WAIT_CYCLES")
        Y2 = s.matmul(X, "tensor")
    assert rel_err(Y, Y_ref) < 1e-5
    assert rel_err(Y2, Y_ref) < 1e-5


def test_rhs_batch_reports_tensor_timeout(backend, monkeypatch):
    """The right-hand-side batch on FP32 cached storage reads the tensor-core
    status after every restart cycle: a product that gave up a wait ends the
    solve with TIMEOUT instead of a wrong solution, and a later solve on the
    same session converges."""
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 6.0), 2.0)
    w = configs.au_workload("s", pos, 2.0, 520.0)
    inv = lb.invert_polarisability(w.alpha)
    dirs = _directions(4)
    rhs = np.concatenate([orc.incident_field(w.positions, w.k, d, e) for d, e in dirs])
    with backend.assemble_and_create_session(w.positions, w.k, inv, True, 2.0,
                                             precision="fp32") as S:
        B = S.rhs_batch(len(dirs))
        monkeypatch.setenv("LUMINA_TC_WAIT_CYCLES", "20000000")
        monkeypatch.setenv("LUMINA_TC_WITHHOLD_SPLIT", "1")
        with pytest.raises(lb.DeviceTimeout):
            B.solve(rhs, 1e-10, 5000, 30, "fp32_refine")
        monkeypatch.delenv("LUMINA_TC_WITHHOLD_SPLIT")
        monkeypatch.delenv("LUMINA_TC_WAIT_CYCLES")
        x, info = B.solve(rhs, 1e-10, 5000, 30, "fp32_refine")
        B.close()
    assert all(i["converged"] == 1 for i in info)
    assert np.all(np.isfinite(x))
