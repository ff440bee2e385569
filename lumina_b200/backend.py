"""CUDA compute backend: the B200 drop-in for the reference's ComputeBackend.

``CudaBackend`` mirrors the trait in crates/lumina-compute/src/backend.rs:62-134
(``device_info``, ``create_session``, ``matvec``,
``assemble_and_create_session``, ``dense_solve``) plus the two hooks the
reference's on-the-fly path lacks (``create_onthefly_session`` and
``solve``).  ``CudaSession`` mirrors ``MatvecSession`` (backend.rs:47-55).
Errors mirror ``ComputeError`` (backend.rs:13-22) and ``SolverError``
(solver/mod.rs:18-30).  Every call goes through liblumina_b200.so.
"""
from __future__ import annotations

import ctypes
from ctypes import byref, c_double, c_int, c_longlong, c_size_t, c_void_p
from dataclasses import dataclass
from typing import Optional

import numpy as np

from . import _ffi
from ._ffi import LumLattice, LumSolveInfo, LumSommerfeld, LumSubstrate


class ComputeError(Exception):
    """Backend failure (backend.rs:13-22)."""


class Unavailable(ComputeError):
    pass


class DeviceError(ComputeError):
    pass


class DeviceTimeout(DeviceError):
    """A bounded device-side wait gave up (LUM_ERR_TIMEOUT): the kernel
    returned without finishing its result; the context stays usable."""


class OutOfMemory(ComputeError):
    """ComputeError::OutOfMemory { requested, available } (backend.rs:13-22)."""

    def __init__(self, msg: str, requested: int = 0, available: int = 0):
        super().__init__(msg)
        self.requested = requested
        self.available = available


class SolverError(Exception):
    """Solver failure (solver/mod.rs:18-30)."""


class ConvergenceFailure(SolverError):
    def __init__(self, max_iter: int, residual: float, info: Optional[dict] = None):
        super().__init__(f"Solver failed to converge after {max_iter} iterations "
                         f"(residual: {residual:.2e})")
        self.max_iter = max_iter
        self.residual = residual
        self.info = info or {}


class InvalidGeometry(SolverError):
    pass


class LinAlgError(SolverError):
    pass


def _raise(rc: int, what: str = ""):
    if rc == _ffi.LUM_OK:
        return
    msg = f"{what}: {_ffi.last_error()}" if what else _ffi.last_error()
    if rc == _ffi.LUM_ERR_UNAVAILABLE:
        raise Unavailable(msg)
    if rc == _ffi.LUM_ERR_OOM:
        req, avail = ctypes.c_size_t(0), ctypes.c_size_t(0)
        _ffi.load().lum_last_oom(ctypes.byref(req), ctypes.byref(avail))
        raise OutOfMemory(msg, req.value, avail.value)
    if rc == _ffi.LUM_ERR_INVALID:
        raise InvalidGeometry(msg)
    if rc == _ffi.LUM_ERR_TIMEOUT:
        raise DeviceTimeout(msg)
    raise DeviceError(msg)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(c_double))


def _c128(a, n=None) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a, np.complex128))
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} complex entries, got {a.size}")
    return a


def _prec(p) -> int:
    if p in (_ffi.LUM_FP32, "fp32", "f32", np.float32):
        return _ffi.LUM_FP32
    if p in (_ffi.LUM_FP64, "fp64", "f64", np.float64):
        return _ffi.LUM_FP64
    raise ValueError(f"unknown precision {p!r}")


def _mode(m) -> int:
    if m in (_ffi.LUM_SOLVE_FP64, "fp64"):
        return _ffi.LUM_SOLVE_FP64
    if m in (_ffi.LUM_SOLVE_FP32_REFINE, "fp32_refine", "fp32+refine"):
        return _ffi.LUM_SOLVE_FP32_REFINE
    raise ValueError(f"unknown solve mode {m!r}")


def lattice_struct(lattice) -> Optional[LumLattice]:
    if lattice is None:
        return None
    s = LumLattice()
    s.a1[:] = [float(v) for v in lattice.a1]
    s.a2[:] = [float(v) for v in (lattice.a2 if lattice.a2 is not None else (0.0, 0.0, 0.0))]
    s.is_2d = 1 if lattice.a2 is not None else 0
    s.has_eta = 1 if lattice.ewald_eta is not None else 0
    s.eta = float(lattice.ewald_eta or 0.0)
    s.truncation_real = int(lattice.truncation_real)
    s.truncation_recip = int(lattice.truncation_recip)
    return s


def _is_sommerfeld(substrate) -> bool:
    return substrate is not None and hasattr(substrate, "wavelength_nm")


def sommerfeld_struct(somm) -> LumSommerfeld:
    e = complex(somm.eps_sub)
    return LumSommerfeld(float(somm.z_interface), float(somm.wavelength_nm), e.real, e.imag,
                         float(somm.eps_env))


def substrate_struct(substrate) -> Optional[LumSubstrate]:
    if substrate is None:
        return None
    r = complex(substrate.delta_eps)
    return LumSubstrate(float(substrate.z_interface), r.real, r.imag)


def _ref(s):
    return byref(s) if s is not None else None


def invert_polarisability(alpha: np.ndarray) -> np.ndarray:
    """alpha^-1 per dipole (compute_diagonal_blocks, assembly.rs:325-363)."""
    a = _c128(alpha).reshape(-1, 9)
    out = np.empty_like(a)
    _raise(_ffi.load().lum_invert_polarisability(a.shape[0], _dp(a.view(np.float64)),
                                                 _dp(out.view(np.float64))), "invert")
    return out.reshape(-1, 3, 3)


def incident_field(positions: np.ndarray, k: float, incident) -> np.ndarray:
    """E_inc at every dipole, length 3N (assembly.rs:178-194)."""
    pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
    n = pos.shape[0]
    rhs = np.empty(3 * n, np.complex128)
    d = np.asarray(incident.direction, np.float64)
    p = np.asarray(incident.polarisation, np.float64)
    _raise(_ffi.load().lum_incident_field(n, _dp(pos), _dp(d), _dp(p), float(incident.amplitude),
                                          float(k), _dp(rhs.view(np.float64))), "incident")
    return rhs


def cross_sections(positions, inv_alpha, moments, k, incident) -> np.ndarray:
    """(C_ext, C_abs, C_sca) from solved moments (cda/mod.rs:175-236)."""
    pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
    n = pos.shape[0]
    ia = _c128(inv_alpha, 9 * n)
    m = _c128(moments, 3 * n)
    out = np.zeros(3)
    d = np.asarray(incident.direction, np.float64)
    p = np.asarray(incident.polarisation, np.float64)
    _raise(_ffi.load().lum_cross_sections(n, _dp(pos), _dp(ia.view(np.float64)),
                                          _dp(m.view(np.float64)), float(k), _dp(d), _dp(p),
                                          float(incident.amplitude), _dp(out)), "cross sections")
    return out


@dataclass
class DeviceInfo:
    name: str
    backend_type: str
    memory_bytes: Optional[int]
    compute_units: Optional[int]


class CudaSession:
    """A device session: a cached matrix or a matrix-free geometry."""

    def __init__(self, handle: c_void_p, dim: int, kind: str, owner=None):
        self._h = handle
        self.dim = dim
        self.kind = kind
        self._owner = owner  # keeps the context alive while the session lives
        self._lib = _ffi.load()

    # -- MatvecSession ---------------------------------------------------
    def upload_matrix(self, matrix: np.ndarray) -> None:
        A = _c128(matrix)
        if A.shape != (self.dim, self.dim):
            raise DeviceError(f"Session expects {self.dim}x{self.dim} matrix, got {A.shape}")
        _raise(self._lib.lum_session_upload_matrix(self._h, _dp(A.view(np.float64))), "upload")

    def matvec(self, x: np.ndarray, precision="fp64") -> np.ndarray:
        xv = _c128(x)
        if xv.size != self.dim:
            raise DeviceError(f"Session dim={self.dim}, got vector len={xv.size}")
        y = np.empty(self.dim, np.complex128)
        _raise(self._lib.lum_session_matvec(self._h, _prec(precision), _dp(xv.view(np.float64)),
                                            _dp(y.view(np.float64))), "matvec")
        return y

    # -- device-pointer variants --------------------------------------------
    def matvec_device(self, x_ptr: int, y_ptr: int, precision="fp64", stream: int = 0) -> None:
        _raise(self._lib.lum_session_matvec_device(self._h, _prec(precision), c_void_p(x_ptr),
                                                   c_void_p(y_ptr), c_void_p(stream or None)),
               "matvec_device")

    def matmul_device(self, X_ptr: int, Y_ptr: int, nrhs: int, stream: int = 0) -> None:
        _raise(self._lib.lum_session_matmul_device(self._h, c_void_p(X_ptr), c_void_p(Y_ptr),
                                                   nrhs, c_void_p(stream or None)), "matmul")

    def rhs_batch(self, nrhs: int) -> "CudaBatch":
        """A batch of ``nrhs`` right-hand sides of this session's operator
        (lum_batch_create_rhs): solve with CudaBatch.solve on vectors stored
        back to back.  For an FP32-storage cached session every FP32 operator
        application is one tensor-core product over all vectors."""
        h = c_void_p()
        _raise(self._lib.lum_batch_create_rhs(self._h, int(nrhs), byref(h)), "rhs_batch")
        return CudaBatch(h, [self.dim // 3] * int(nrhs), self)

    _METHODS = {"auto": 0, "tensor": 1, "cuda_cores": 2}

    def matmul(self, X: np.ndarray, method="auto") -> np.ndarray:
        """Y = A X for the columns of X (dim x nrhs) of a cached session: the
        tensor cores (3xTF32) for FP32 storage, or the CUDA cores."""
        Xc = _c128(X)
        if Xc.ndim != 2 or Xc.shape[0] != self.dim:
            raise DeviceError(f"Session dim={self.dim}, got X of shape {Xc.shape}")
        nrhs = Xc.shape[1]
        Xv = np.ascontiguousarray(Xc.T)  # vectors back to back
        Yv = np.empty_like(Xv)
        _raise(self._lib.lum_session_matmul_vectors(self._h, _dp(Xv.view(np.float64)),
                                                    _dp(Yv.view(np.float64)), nrhs,
                                                    self._METHODS[method]), "matmul")
        return Yv.T

    def matmul_vectors_device(self, X_ptr: int, Y_ptr: int, nrhs: int, method="auto",
                              stream: int = 0) -> None:
        """Y = A X for nrhs device vectors stored back to back (no synchronisation)."""
        _raise(self._lib.lum_session_matmul_vectors_device(self._h, c_void_p(X_ptr),
                                                           c_void_p(Y_ptr), nrhs,
                                                           self._METHODS[method],
                                                           c_void_p(stream or None)), "matmul")

    def set_stream(self, stream: int) -> None:
        _raise(self._lib.lum_session_set_stream(self._h, c_void_p(stream or None)), "set_stream")

    def set_wavelength(self, k: float, inv_alpha: np.ndarray, substrate=None) -> None:
        """Re-targets the session (runner.rs:150-183); a SommerfeldRuntime
        substrate rebuilds the session's reflected-tensor table."""
        ia = _c128(inv_alpha, 9 * (self.dim // 3))
        somm = _is_sommerfeld(substrate)
        sub = None if somm else substrate_struct(substrate)
        _raise(self._lib.lum_session_set_wavelength(self._h, float(k), _dp(ia.view(np.float64)),
                                                    _ref(sub)), "set_wavelength")
        if somm:
            self.set_sommerfeld(substrate)

    def set_sommerfeld(self, somm) -> None:
        """Rebuilds the Sommerfeld reflected-tensor table (and an assembled
        matrix) for ``somm`` (a SommerfeldRuntime)."""
        st = sommerfeld_struct(somm)
        _raise(self._lib.lum_session_set_sommerfeld(self._h, byref(st)), "set_sommerfeld")

    # -- solve --------------------------------------------------------------
    def solve(self, rhs: np.ndarray, tol: float = 1e-6, max_iter: int = 1000, restart: int = 30,
              mode="fp64", raise_on_failure: bool = True):
        b = _c128(rhs)
        if b.size != self.dim:
            raise DeviceError(f"Session dim={self.dim}, got rhs len={b.size}")
        x = np.zeros(self.dim, np.complex128)
        info = LumSolveInfo()
        rc = self._lib.lum_solve_gmres(self._h, _dp(b.view(np.float64)), float(tol),
                                       int(max_iter), int(restart), _mode(mode),
                                       _dp(x.view(np.float64)), byref(info))
        d = info.as_dict()
        if rc == _ffi.LUM_ERR_NOT_CONVERGED:
            if raise_on_failure:
                raise ConvergenceFailure(max_iter, info.rel_residual, d)
            return x, d
        _raise(rc, "solve")
        return x, d

    def solve_multi(self, rhs, tol: float = 1e-6, max_iter: int = 1000, restart: int = 30,
                    mode="fp64", raise_on_failure: bool = True):
        """Several right-hand sides (rows of ``rhs``), two per operator
        application; returns (x with the same shape, [info per rhs])."""
        B = np.ascontiguousarray(np.asarray(rhs, np.complex128).reshape(-1, self.dim))
        nrhs = B.shape[0]
        X = np.zeros_like(B)
        infos = (LumSolveInfo * nrhs)()
        rc = self._lib.lum_solve_gmres_multi(self._h, nrhs, _dp(B.view(np.float64)), float(tol),
                                             int(max_iter), int(restart), _mode(mode),
                                             _dp(X.view(np.float64)), infos)
        d = [infos[r].as_dict() for r in range(nrhs)]
        if rc == _ffi.LUM_ERR_NOT_CONVERGED:
            if raise_on_failure:
                raise ConvergenceFailure(max_iter, max(i["rel_residual"] for i in d),
                                         {"rhs": d})
            return X, d
        _raise(rc, "solve_multi")
        return X, d

    def solve_multi_device(self, nrhs: int, b_ptr: int, x_ptr: int, tol: float, max_iter: int,
                           restart: int = 30, mode="fp64", stream: int = 0):
        infos = (LumSolveInfo * nrhs)()
        rc = self._lib.lum_solve_gmres_multi_device(self._h, int(nrhs), c_void_p(b_ptr),
                                                    c_void_p(x_ptr), float(tol), int(max_iter),
                                                    int(restart), _mode(mode), infos,
                                                    c_void_p(stream or None))
        d = [infos[r].as_dict() for r in range(nrhs)]
        if rc == _ffi.LUM_ERR_NOT_CONVERGED:
            raise ConvergenceFailure(max_iter, max(i["rel_residual"] for i in d), {"rhs": d})
        _raise(rc, "solve_multi_device")
        return d

    def solve_device(self, b_ptr: int, x_ptr: int, tol: float, max_iter: int, restart: int = 30,
                     mode="fp64", stream: int = 0) -> dict:
        info = LumSolveInfo()
        rc = self._lib.lum_solve_gmres_device(self._h, c_void_p(b_ptr), c_void_p(x_ptr),
                                              float(tol), int(max_iter), int(restart),
                                              _mode(mode), byref(info), c_void_p(stream or None))
        d = info.as_dict()
        if rc == _ffi.LUM_ERR_NOT_CONVERGED:
            raise ConvergenceFailure(max_iter, info.rel_residual, d)
        _raise(rc, "solve_device")
        return d

    # -- adjoint gradients ----------------------------------------------------
    def grad_cext(self, direction, polarisation, amplitude: float = 1.0, dinv_alpha_deps=None,
                  tol: float = 1e-8, max_iter: int = 1000, restart: int = 30, mode="fp64",
                  want_eps: bool = True) -> dict:
        """C_ext and its adjoint gradients for a plane wave with a (possibly
        complex) polarisation: forward solve, adjoint solve with conj(E),
        device gradient kernels.  Returns c_ext, grad_r (N,3), grad_eps (N,2:
        d/dRe eps, d/dIm eps; zero without ``dinv_alpha_deps``), moments and
        both solves' info."""
        n = self.dim // 3
        d = np.ascontiguousarray(np.asarray(direction, np.float64).reshape(3))
        pol = np.asarray(polarisation, np.complex128).reshape(3)
        pol6 = np.ascontiguousarray(np.stack([pol.real, pol.imag], axis=1).ravel())
        dinv = None if dinv_alpha_deps is None else _c128(dinv_alpha_deps, 9 * n)
        c_ext = c_double(0.0)
        mom = np.zeros(3 * n, np.complex128)
        gr = np.zeros(3 * n)
        ge = np.zeros(2 * n) if want_eps else None
        fi, ai = LumSolveInfo(), LumSolveInfo()
        rc = self._lib.lum_grad_cext(self._h, _dp(d), _dp(pol6), float(amplitude),
                                     None if dinv is None else dinv.ctypes.data, float(tol),
                                     int(max_iter), int(restart), _mode(mode), byref(c_ext),
                                     mom.ctypes.data, _dp(gr),
                                     None if ge is None else ge.ctypes.data, byref(fi),
                                     byref(ai))
        if rc == _ffi.LUM_ERR_NOT_CONVERGED:
            raise ConvergenceFailure(max_iter, max(fi.rel_residual, ai.rel_residual),
                                     {"forward": fi.as_dict(), "adjoint": ai.as_dict()})
        _raise(rc, "grad_cext")
        return {"c_ext": c_ext.value, "grad_r": gr.reshape(n, 3),
                "grad_eps": None if ge is None else ge.reshape(n, 2), "moments": mom,
                "info_forward": fi.as_dict(), "info_adjoint": ai.as_dict()}

    # -- measurement --------------------------------------------------------
    def profile(self, enable: bool = True) -> None:
        _raise(self._lib.lum_session_profile(self._h, int(enable)), "profile")

    def kernel_time(self, precision="fp32"):
        """(launches, total ms) of the dominant kernel at ``precision`` ("fp32",
        "fp64", or "fp32x2" / "fp64x2" for the two-vector kernels) since
        ``profile()`` was last called."""
        n, ms = c_int(0), c_double(0.0)
        # "fp32x2" / "fp64x2": the two-vector pair kernels (recorded under precision + 2)
        code = _prec(precision[:-2]) + 2 if str(precision).endswith("x2") else _prec(precision)
        _raise(self._lib.lum_session_kernel_time(self._h, code, byref(n), byref(ms)),
               "kernel_time")
        return n.value, ms.value

    def stats(self) -> dict:
        npairs, w, s32, s64 = c_longlong(0), c_int(0), c_int(0), c_int(0)
        _raise(self._lib.lum_session_stats(self._h, byref(npairs), byref(w), byref(s32),
                                           byref(s64)), "stats")
        return {"near_pairs": npairs.value, "ell_width": w.value, "nsplit32": s32.value,
                "nsplit64": s64.value}

    def kernel_config(self) -> dict:
        """Autotuned kernel choices of this session."""
        buf = ctypes.create_string_buffer(1024)
        _raise(self._lib.lum_session_kernel_config(self._h, buf, 1024), "kernel_config")
        out = {}
        for tok in buf.value.decode().split():
            key, _, val = tok.partition("=")
            try:
                out[key] = int(val)
            except ValueError:
                try:
                    out[key] = float(val)
                except ValueError:
                    out[key] = val
        return out

    def close(self) -> None:
        if self._h:
            self._lib.lum_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class CudaBatch:
    """K independent isolated systems solved together (lum_batch_*).

    Vectors are the concatenation of the systems' 3N_s complex vectors in
    system order; ``split`` cuts one back into per-system pieces."""

    def __init__(self, handle: c_void_p, sizes, owner=None):
        self._h = handle
        self.sizes = [int(n) for n in sizes]
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.dim = 3 * int(self.offsets[-1])
        self._owner = owner
        self._lib = _ffi.load()

    def split(self, v: np.ndarray):
        v = np.asarray(v)
        return [v[3 * self.offsets[s]:3 * self.offsets[s + 1]] for s in range(len(self.sizes))]

    def matvec(self, x: np.ndarray, precision="fp64") -> np.ndarray:
        xv = _c128(x)
        if xv.size != self.dim:
            raise DeviceError(f"Batch dim={self.dim}, got vector len={xv.size}")
        y = np.empty(self.dim, np.complex128)
        _raise(self._lib.lum_batch_matvec(self._h, _prec(precision), _dp(xv.view(np.float64)),
                                          _dp(y.view(np.float64))), "batch matvec")
        return y

    def matvec_device(self, x_ptr: int, y_ptr: int, precision="fp64") -> None:
        _raise(self._lib.lum_batch_matvec_device(self._h, _prec(precision), c_void_p(x_ptr),
                                                 c_void_p(y_ptr)), "batch matvec_device")

    def set_stream(self, stream: int) -> None:
        _raise(self._lib.lum_batch_set_stream(self._h, c_void_p(stream or None)), "set_stream")

    def _infos(self, arr):
        return [arr[s].as_dict() for s in range(len(self.sizes))]

    def solve(self, rhs: np.ndarray, tol: float = 1e-6, max_iter: int = 1000, restart: int = 30,
              mode="fp64", raise_on_failure: bool = True):
        """(x, [info per system]); x is the concatenated solution."""
        b = _c128(rhs)
        if b.size != self.dim:
            raise DeviceError(f"Batch dim={self.dim}, got rhs len={b.size}")
        x = np.zeros(self.dim, np.complex128)
        infos = (LumSolveInfo * len(self.sizes))()
        rc = self._lib.lum_batch_solve(self._h, _dp(b.view(np.float64)), float(tol),
                                       int(max_iter), int(restart), _mode(mode),
                                       _dp(x.view(np.float64)), infos)
        d = self._infos(infos)
        if rc == _ffi.LUM_ERR_NOT_CONVERGED:
            if raise_on_failure:
                worst = max(i["rel_residual"] for i in d)
                raise ConvergenceFailure(max_iter, worst, {"systems": d})
            return x, d
        _raise(rc, "batch solve")
        return x, d

    def solve_device(self, b_ptr: int, x_ptr: int, tol: float, max_iter: int, restart: int = 30,
                     mode="fp64"):
        infos = (LumSolveInfo * len(self.sizes))()
        rc = self._lib.lum_batch_solve_device(self._h, c_void_p(b_ptr), c_void_p(x_ptr),
                                              float(tol), int(max_iter), int(restart),
                                              _mode(mode), infos)
        d = self._infos(infos)
        if rc == _ffi.LUM_ERR_NOT_CONVERGED:
            raise ConvergenceFailure(max_iter, max(i["rel_residual"] for i in d), {"systems": d})
        _raise(rc, "batch solve_device")
        return d

    def kernel_config(self) -> dict:
        """The FP32 pair scheme this batch chose and its work-list sizes."""
        buf = ctypes.create_string_buffer(512)
        _raise(self._lib.lum_batch_kernel_config(self._h, buf, 512), "batch kernel_config")
        out = {}
        for tok in buf.value.decode().split():
            key, _, val = tok.partition("=")
            try:
                out[key] = int(val)
            except ValueError:
                out[key] = val
        return out

    def info(self) -> dict:
        vals = [c_int(0) for _ in range(9)]
        _raise(self._lib.lum_batch_info(self._h, *[byref(v) for v in vals]), "batch info")
        keys = ("systems", "dipoles", "ell_width", "cluster", "elems_per_thread", "items32",
                "grid32", "items64", "grid64")
        return {k: v.value for k, v in zip(keys, vals)}

    def close(self) -> None:
        if self._h:
            self._lib.lum_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class CudaBackend:
    """ComputeBackend on one B200 (backend.rs:62-134)."""

    def __init__(self, device: int = 0):
        self._lib = _ffi.load()
        h = c_void_p()
        _raise(self._lib.lum_ctx_create(int(device), byref(h)), "context")
        self._h = h
        self.device = device

    def device_info(self) -> DeviceInfo:
        buf = ctypes.create_string_buffer(256)
        mem, sms = c_size_t(0), c_int(0)
        _raise(self._lib.lum_device_info(self._h, buf, 256, byref(mem), byref(sms)), "info")
        return DeviceInfo(buf.value.decode(), "Gpu", mem.value, sms.value)

    def create_session(self, n: int, precision="fp32") -> CudaSession:
        """A cached-matrix session for ``n`` unknowns (backend.rs:70)."""
        h = c_void_p()
        _raise(self._lib.lum_session_create_cached(self._h, int(n), _prec(precision), byref(h)),
               "create_session")
        return CudaSession(h, int(n), "cached", self)

    def matvec(self, matrix: np.ndarray, vector: np.ndarray, precision="fp64") -> np.ndarray:
        """One-off y = A x (backend.rs:89-93)."""
        A = _c128(matrix)
        if A.ndim != 2 or A.shape[0] != A.shape[1] or A.shape[0] != np.asarray(vector).size:
            raise DeviceError(f"Dimension mismatch: matrix {A.shape}, vector {np.asarray(vector).size}")
        with self.create_session(A.shape[0], precision) as s:
            s.upload_matrix(A)
            return s.matvec(vector, precision)

    def assemble_and_create_session(self, positions, k: float, diagonal_blocks, use_fcd=False,
                                    cell_size=3.0, lattice=None, k_bloch=(0.0, 0.0, 0.0),
                                    substrate=None, precision="fp32",
                                    symmetric=False) -> CudaSession:
        """Device-assembled dense session (backend.rs:109-117, widened).

        symmetric=True keeps only the upper-triangle tiles of the matrix
        (LUM_STORAGE_SYMMETRIC): free-space systems only (no lattice, no
        substrate), half the memory and half the bytes per product; products
        run one vector at a time (no tensor-core path)."""
        pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
        n = pos.shape[0]
        ia = _c128(diagonal_blocks, 9 * n)
        kb = np.asarray(k_bloch, np.float64)
        h = c_void_p()
        if _is_sommerfeld(substrate):
            st = sommerfeld_struct(substrate)
            _raise(self._lib.lum_session_assemble_sommerfeld(
                self._h, n, _dp(pos), _dp(ia.view(np.float64)), float(k), int(bool(use_fcd)),
                float(cell_size), _ref(lattice_struct(lattice)), _dp(kb), byref(st),
                _prec(precision), byref(h)), "assemble")
            return CudaSession(h, 3 * n, "cached", self)
        lat, sub = lattice_struct(lattice), substrate_struct(substrate)
        storage = _prec(precision) | (_ffi.LUM_STORAGE_SYMMETRIC if symmetric else 0)
        _raise(self._lib.lum_session_assemble(self._h, n, _dp(pos), _dp(ia.view(np.float64)),
                                              float(k), int(bool(use_fcd)), float(cell_size),
                                              _ref(lat), _dp(kb), _ref(sub), storage,
                                              byref(h)), "assemble")
        return CudaSession(h, 3 * n, "cached", self)

    def create_fft_session(self, positions, inv_alpha, k: float, use_fcd=True,
                           cell_size=3.0, spacing=0.0, substrate=None) -> CudaSession:
        """Block-Toeplitz session through 3D FFTs (fft_matvec.rs:77-258, widened
        to FCD, to any set of cubic-lattice nodes and to a planar substrate --
        a SubstrateRuntime (Fresnel image) or a SommerfeldRuntime)."""
        pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
        n = pos.shape[0]
        ia = _c128(inv_alpha, 9 * n)
        h = c_void_p()
        _raise(self._lib.lum_session_create_fft(self._h, n, _dp(pos), _dp(ia.view(np.float64)),
                                                float(k), int(bool(use_fcd)), float(cell_size),
                                                float(spacing), byref(h)), "create_fft_session")
        sess = CudaSession(h, 3 * n, "fft", self)
        if substrate is not None:
            try:
                if _is_sommerfeld(substrate):
                    sess.set_sommerfeld(substrate)
                else:
                    sess.set_wavelength(k, ia, substrate)
            except Exception:
                sess.close()
                raise
        return sess

    def create_onthefly_session(self, positions, inv_alpha, k: float, use_fcd=True,
                                cell_size=3.0, lattice=None, k_bloch=(0.0, 0.0, 0.0),
                                substrate=None) -> CudaSession:
        """Matrix-free session (matvec_on_the_fly, assembly.rs:209-318)."""
        pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
        n = pos.shape[0]
        ia = _c128(inv_alpha, 9 * n)
        kb = np.asarray(k_bloch, np.float64)
        h = c_void_p()
        if _is_sommerfeld(substrate):
            st = sommerfeld_struct(substrate)
            _raise(self._lib.lum_session_create_onthefly_sommerfeld(
                self._h, n, _dp(pos), _dp(ia.view(np.float64)), float(k), int(bool(use_fcd)),
                float(cell_size), _ref(lattice_struct(lattice)), _dp(kb), byref(st), byref(h)),
                "create_onthefly")
            return CudaSession(h, 3 * n, "onthefly", self)
        lat, sub = lattice_struct(lattice), substrate_struct(substrate)
        _raise(self._lib.lum_session_create_onthefly(self._h, n, _dp(pos),
                                                     _dp(ia.view(np.float64)), float(k),
                                                     int(bool(use_fcd)), float(cell_size),
                                                     _ref(lat), _dp(kb), _ref(sub), byref(h)),
               "create_onthefly")
        return CudaSession(h, 3 * n, "onthefly", self)

    def create_batch(self, systems, use_fcd=True) -> CudaBatch:
        """Batch of isolated systems; ``systems`` is a sequence of
        (positions (N,3), inv_alpha (N,3,3) or 9N complex, k, cell_size)."""
        sizes, pos, ia, ks, cells = [], [], [], [], []
        for p, inv, k, cell in systems:
            p = np.asarray(p, np.float64).reshape(-1, 3)
            sizes.append(p.shape[0])
            pos.append(p)
            ia.append(_c128(inv, 9 * p.shape[0]))
            ks.append(float(k))
            cells.append(float(cell))
        if not sizes:
            raise InvalidGeometry("a batch needs at least one system")
        n_arr = np.asarray(sizes, np.int32)
        P = np.ascontiguousarray(np.concatenate(pos))
        IA = np.ascontiguousarray(np.concatenate(ia))
        K = np.asarray(ks, np.float64)
        C = np.asarray(cells, np.float64)
        h = c_void_p()
        _raise(self._lib.lum_batch_create(self._h, len(sizes),
                                          n_arr.ctypes.data_as(ctypes.POINTER(c_int)), _dp(P),
                                          _dp(IA.view(np.float64)), _dp(K), _dp(C),
                                          int(bool(use_fcd)), byref(h)), "create_batch")
        return CudaBatch(h, sizes, self)

    def sommerfeld_tensor(self, somm, ri, rj) -> np.ndarray:
        """SommerfeldGreens::evaluate (sommerfeld.rs:254-300) on the device for
        point pairs (ri, rj: (P, 3) or (3,)); returns (P, 3, 3) or (3, 3)."""
        a = np.ascontiguousarray(np.asarray(ri, np.float64).reshape(-1, 3))
        b = np.ascontiguousarray(np.asarray(rj, np.float64).reshape(-1, 3))
        if a.shape != b.shape:
            raise InvalidGeometry(f"pair arrays differ: {a.shape} vs {b.shape}")
        g = np.zeros((a.shape[0], 3, 3), np.complex128)
        st = sommerfeld_struct(somm)
        _raise(self._lib.lum_sommerfeld_tensor(self._h, byref(st), a.shape[0], _dp(a), _dp(b),
                                               _dp(g.view(np.float64))), "sommerfeld_tensor")
        return g if np.ndim(ri) > 1 else g[0]

    def dense_solve(self, matrix, rhs):
        """The reference's default (backend.rs:123-133): no dense LU here;
        use ``solve`` on a session."""
        raise Unavailable("Dense solve not implemented for this backend")

    def solve(self, session: CudaSession, rhs, tol=1e-6, max_iter=1000, restart=30, mode="fp64"):
        return session.solve(rhs, tol, max_iter, restart, mode)

    def measure_fma_peak(self):
        """(FP32, FP64) CUDA-core GFLOP/s measured by an FMA-chain kernel."""
        f32, f64 = c_double(0.0), c_double(0.0)
        _raise(self._lib.lum_measure_fma_peak(self._h, byref(f32), byref(f64)), "fma peak")
        return f32.value, f64.value

    def measure_fma2_peak(self):
        """FP32 GFLOP/s of packed f32x2 FMA chains."""
        g = c_double(0.0)
        _raise(self._lib.lum_measure_fma2_peak(self._h, byref(g)), "fma2 peak")
        return g.value

    def measure_l2_peak(self):
        """L2 read bandwidth (GB/s) measured by a 16-byte-load kernel."""
        g = c_double(0.0)
        _raise(self._lib.lum_measure_l2_peak(self._h, byref(g)), "l2 peak")
        return g.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.lum_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
