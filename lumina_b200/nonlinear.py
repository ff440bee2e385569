"""Second- and third-harmonic response (the reference's nonlinear.rs).

p_NL from the linear local fields and chi(2) / chi(3) on the device
(lum_harmonic_sources), then A(k_h) p = p_NL at the harmonic wave number
through the solver's own session dispatch (the same direct / cached /
on-the-fly choice as CdaSolver.solve_dipoles), no incident field at the
harmonic (nonlinear.rs:108-240, :282-412).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _ffi
from .backend import _dp, _raise
from .fields import FarFieldMap, compute_far_field
from .types import DipoleResponse, DipoleSet, SimulationParams


class Chi2Tensor:
    """types.rs:331-393: 27 complex components, (a, b, c) at a*9 + b*3 + c."""

    def __init__(self, components=None):
        self.components = (np.zeros(27, np.complex128) if components is None
                           else np.asarray(components, np.complex128).reshape(27).copy())

    @staticmethod
    def zero() -> "Chi2Tensor":
        return Chi2Tensor()

    @staticmethod
    def from_components(components) -> "Chi2Tensor":
        return Chi2Tensor(components)

    @staticmethod
    def isotropic_surface(chi_zzz: complex, chi_zxx: complex) -> "Chi2Tensor":
        """C_inf_v surface tensor (types.rs:378-392)."""
        t = Chi2Tensor()
        t.components[2 * 9 + 2 * 3 + 2] = chi_zzz
        for a, b, c in ((2, 0, 0), (2, 1, 1), (0, 0, 2), (0, 2, 0), (1, 1, 2), (1, 2, 1)):
            t.components[a * 9 + b * 3 + c] = chi_zxx
        return t


class Chi3Tensor:
    """types.rs:436-522: 81 complex components, (a, b, c, d) at a*27+b*9+c*3+d."""

    def __init__(self, components=None):
        self.components = (np.zeros(81, np.complex128) if components is None
                           else np.asarray(components, np.complex128).reshape(81).copy())

    @staticmethod
    def zero() -> "Chi3Tensor":
        return Chi3Tensor()

    @staticmethod
    def from_components(components) -> "Chi3Tensor":
        return Chi3Tensor(components)

    @staticmethod
    def isotropic_bulk(chi_xxxx: complex, chi_xxyy: complex) -> "Chi3Tensor":
        """Isotropic bulk tensor (types.rs:492-522)."""
        t = Chi3Tensor()
        extra = complex(chi_xxxx) - 3.0 * complex(chi_xxyy)
        for a in range(3):
            for b in range(3):
                for c in range(3):
                    for d in range(3):
                        v = 0j
                        if a == b and c == d:
                            v += chi_xxyy
                        if a == c and b == d:
                            v += chi_xxyy
                        if a == d and b == c:
                            v += chi_xxyy
                        if a == b == c == d:
                            v += extra
                        t.components[a * 27 + b * 9 + c * 3 + d] = v
        return t


@dataclass
class HarmonicResult:
    """ShgResult / ThgResult (types.rs:399-422, :529-552)."""
    fundamental_nm: float
    harmonic_nm: float
    source_moments: np.ndarray      # (N, 3)
    driven_moments: np.ndarray      # (N, 3)
    intensity: float                # sum |p|^2 (shg_intensity / thg_intensity)
    far_field: Optional[FarFieldMap]
    solve_info: dict


def harmonic_sources(backend, order: int, local_fields, tensors) -> np.ndarray:
    """compute_shg_sources (order 2) / compute_thg_sources (order 3) on the
    device: (N, 3) complex."""
    e = np.ascontiguousarray(np.asarray(local_fields, np.complex128).reshape(-1))
    n = e.size // 3
    nc = 27 if order == 2 else 81
    if isinstance(tensors, (Chi2Tensor, Chi3Tensor)):
        tensors = [tensors]
    chi = np.ascontiguousarray(np.stack([np.asarray(t.components if hasattr(t, "components") else t,
                                                    np.complex128).reshape(nc)
                                         for t in tensors]))
    if chi.shape[0] not in (1, n):
        raise ValueError(f"{chi.shape[0]} tensors for {n} dipoles")
    out = np.zeros(3 * n, np.complex128)
    lib = _ffi.load()
    _raise(lib.lum_harmonic_sources(backend._h, int(order), n, _dp(e.view(np.float64)),
                                    chi.shape[0], _dp(chi.view(np.float64)),
                                    _dp(out.view(np.float64))), "harmonic_sources")
    return out.reshape(-1, 3)


def _harmonic_response(order, solver, omega_response: DipoleResponse, dipoles_h: DipoleSet,
                       tensors, params_h: SimulationParams, calc_far_field: bool):
    from . import backend as be
    n = dipoles_h.n
    if n == 0:
        raise be.InvalidGeometry("No dipoles provided")
    if omega_response.moments.shape[0] != n:
        raise ValueError("harmonic dipoles must match the linear response's dipole count")
    fundamental = float(omega_response.wavelength_nm)
    harmonic = fundamental / order
    k_h = 2.0 * math.pi * params_h.environment_n / harmonic
    sources = harmonic_sources(solver.backend, order, omega_response.local_fields, tensors)
    rhs = sources.reshape(-1)
    inv_alpha = be.invert_polarisability(dipoles_h.polarisability)
    direct = n <= solver.iterative_threshold
    sess = solver._session(dipoles_h, inv_alpha, k_h, params_h, direct)
    try:
        if not np.any(rhs):
            x, info = np.zeros_like(rhs), {"iterations": 0, "converged": 1}
        elif direct:
            x, info = sess.solve(rhs, solver.direct_tolerance, max(params_h.max_iterations, 10000),
                                 solver.restart, "fp64")
        else:
            x, info = sess.solve(rhs, params_h.solver_tolerance, params_h.max_iterations,
                                 solver.restart, solver.precision)
    finally:
        solver._release(sess)
    driven = x.reshape(-1, 3)
    intensity = float(np.sum(np.abs(driven) ** 2))
    ff = None
    if calc_far_field:
        resp = DipoleResponse(harmonic, params_h.environment_n, driven, np.zeros_like(driven))
        ff = compute_far_field(solver.backend, dipoles_h.positions, resp, k_h, 36, 72)
    return HarmonicResult(fundamental, harmonic, sources, driven, intensity, ff, info)


def compute_shg_response(solver, omega_response: DipoleResponse, dipoles_2omega: DipoleSet,
                         chi2_tensors: Sequence[Chi2Tensor], params_2omega: SimulationParams,
                         calc_far_field: bool = False) -> HarmonicResult:
    """nonlinear.rs:108-240."""
    return _harmonic_response(2, solver, omega_response, dipoles_2omega, chi2_tensors,
                              params_2omega, calc_far_field)


def compute_thg_response(solver, omega_response: DipoleResponse, dipoles_3omega: DipoleSet,
                         chi3_tensors: Sequence[Chi3Tensor], params_3omega: SimulationParams,
                         calc_far_field: bool = False) -> HarmonicResult:
    """nonlinear.rs:282-412."""
    return _harmonic_response(3, solver, omega_response, dipoles_3omega, chi3_tensors,
                              params_3omega, calc_far_field)
