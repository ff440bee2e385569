"""GPU parity of the multi-right-hand-side cached product Y = A X.

The tensor-core method (tcgen05, TF32 operands split hi + lo, three products
per operand pair, FP32 accumulation) is compared with the exact FP64 product
of the FP32-stored matrix, and with the CUDA-core method.  Tolerances
(max |error| / max |reference| over the block):
  tensor cores vs exact product of the stored matrix   1e-5
  FP32-stored physics matrix vs the FP64 oracle matrix  2e-5 (the FP32 bar)
"""
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
