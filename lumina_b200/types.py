"""Core input/output types of the coupled-dipole solve.

Mirrors crates/lumina-core/src/types.rs: ``Dipole`` (:12-33),
``IncidentField`` (:36-74), ``SimulationParams`` (:77-115), ``CrossSections``
(:118-131), ``DipoleResponse`` (:191-204) and the polarisability
prescriptions (:243-317).  Dipole sets are held as arrays -- positions (N, 3)
float64 and polarisabilities (N, 3, 3) complex128 -- because the device
library consumes them that way.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np


def _cdiv(a: complex, b: complex) -> complex:
    """Complex division through |b|^2 (num-complex's formula)."""
    n = b.real * b.real + b.imag * b.imag
    return complex((a.real * b.real + a.imag * b.imag) / n, (a.imag * b.real - a.real * b.imag) / n)


def wavenumber(wavelength_nm: float, n_medium: float) -> float:
    """k = 2 pi n / lambda (cda/mod.rs:169-171)."""
    return 2.0 * math.pi * n_medium / wavelength_nm


@dataclass
class Dipole:
    """One point dipole: position (nm) and 3x3 complex polarisability."""
    position: Sequence[float]
    polarisability: np.ndarray

    @staticmethod
    def isotropic(position, alpha: complex) -> "Dipole":
        return Dipole(tuple(float(v) for v in position), np.eye(3, dtype=np.complex128) * alpha)


@dataclass
class DipoleSet:
    """N dipoles as arrays: positions (N, 3) and polarisabilities (N, 3, 3)."""
    positions: np.ndarray
    polarisability: np.ndarray

    def __post_init__(self):
        self.positions = np.ascontiguousarray(np.asarray(self.positions, np.float64).reshape(-1, 3))
        pol = np.asarray(self.polarisability, np.complex128)
        if pol.ndim == 1:  # isotropic scalars
            pol = pol[:, None, None] * np.eye(3)[None]
        self.polarisability = np.ascontiguousarray(pol.reshape(-1, 3, 3))
        if self.polarisability.shape[0] != self.positions.shape[0]:
            raise ValueError("positions and polarisabilities differ in length")

    @property
    def n(self) -> int:
        return self.positions.shape[0]

    @staticmethod
    def from_dipoles(dipoles: Sequence[Dipole]) -> "DipoleSet":
        pos = np.array([d.position for d in dipoles], np.float64).reshape(-1, 3)
        pol = np.array([np.asarray(d.polarisability, np.complex128).reshape(3, 3) for d in dipoles])
        return DipoleSet(pos, pol.reshape(-1, 3, 3))

    @staticmethod
    def isotropic(positions, alpha) -> "DipoleSet":
        pos = np.asarray(positions, np.float64).reshape(-1, 3)
        a = np.broadcast_to(np.asarray(alpha, np.complex128), (pos.shape[0],))
        return DipoleSet(pos, a[:, None, None] * np.eye(3)[None])


@dataclass
class IncidentField:
    """Plane wave E0 e exp(i k d.r) with a real polarisation vector."""
    direction: Sequence[float] = (0.0, 0.0, 1.0)
    polarisation: Sequence[float] = (1.0, 0.0, 0.0)
    amplitude: float = 1.0


@dataclass
class SimulationParams:
    wavelength_range: Sequence[float] = (400.0, 900.0)
    num_wavelengths: int = 100
    environment_n: float = 1.0
    solver_tolerance: float = 1e-6
    max_iterations: int = 1000
    k_bloch: Sequence[float] = (0.0, 0.0, 0.0)
    substrate_runtime: Optional[object] = None


@dataclass
class CrossSections:
    wavelength_nm: float
    extinction: float
    absorption: float
    scattering: float
    circular_dichroism: Optional[float] = None


@dataclass
class DipoleResponse:
    wavelength_nm: float
    environment_n: float
    moments: np.ndarray          # (N, 3) complex
    local_fields: np.ndarray     # (N, 3) complex
    solve_info: dict = field(default_factory=dict)


def clausius_mossotti(volume_nm3: float, epsilon: complex, epsilon_m: float) -> complex:
    """alpha_CM = 3 V (eps - eps_m)/(eps + 2 eps_m)  (types.rs:243-246)."""
    eps = complex(epsilon)
    num = (eps - epsilon_m) * (3.0 * volume_nm3)
    return _cdiv(num, eps + 2.0 * epsilon_m)


def radiative_correction(alpha_cm: complex, k: float) -> complex:
    """alpha / (1 - i k^3/(6 pi) alpha)  (types.rs:256-259)."""
    corr = complex(0.0, k ** 3 / (6.0 * math.pi))
    return _cdiv(complex(alpha_cm), 1.0 - corr * complex(alpha_cm))


def ellipsoid_polarisability_tensor(volume_nm3: float, depol: Sequence[float], epsilon: complex,
                                    epsilon_m: float, k: float, rot: Sequence[float]) -> np.ndarray:
    """R diag(alpha_x, alpha_y, alpha_z) R^T with per-axis CM + RRCM
    (types.rs:286-317); rot is row-major 3x3."""
    eps = complex(epsilon)
    d_eps = eps - epsilon_m
    alphas = []
    for L in depol:
        denom = epsilon_m + L * d_eps
        alphas.append(radiative_correction(_cdiv(d_eps * volume_nm3, denom), k))
    R = np.asarray(rot, np.float64).reshape(3, 3)
    return (R * np.array(alphas)[None, :]) @ R.T


def rrcm_array(volume_nm3: float, epsilon, epsilon_m: float, k: float) -> np.ndarray:
    """Vectorised isotropic RRCM polarisabilities for an array of eps values."""
    eps = np.asarray(epsilon, np.complex128)
    a_cm = 3.0 * volume_nm3 * (eps - epsilon_m) / (eps + 2.0 * epsilon_m)
    return a_cm / (1.0 - 1j * (k ** 3 / (6.0 * math.pi)) * a_cm)
