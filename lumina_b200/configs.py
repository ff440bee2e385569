"""Synthetic workloads of the coupled-dipole solve (seeded, no datasets).

sphere_au_925      Au sphere R = 12 nm on the reference's centred 2 nm
                   lattice (discretise.rs inclusive rule: N = 925), 520 nm,
                   vacuum, RRCM, FCD with cell = 2 nm, +z x-polarised.
cuboid_au_30k      Au cuboid 60 x 50 x 10 nm, cell-centred 1 nm lattice
                   (N = 30,000), vacuum, RRCM, FCD with cell = 1 nm; the
                   51-point 400-900 nm sweep (J&C gold ends at 892 nm: the
                   last point uses the spline's boundary polynomial).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .geometry import Sphere, cell_centred_cuboid, discretise_primitive
from .materials import JohnsonChristyMaterial
from .types import rrcm_array, wavenumber


@dataclass
class Workload:
    name: str
    positions: np.ndarray       # (N, 3)
    alpha: np.ndarray           # (N, 3, 3) complex
    wavelength_nm: float
    k: float
    cell_size: float
    use_fcd: bool = True
    environment_n: float = 1.0

    @property
    def n(self):
        return self.positions.shape[0]


def _isotropic(alpha_scalar: complex, n: int) -> np.ndarray:
    return np.broadcast_to(np.eye(3, dtype=np.complex128) * alpha_scalar, (n, 3, 3)).copy()


def gold_eps(wavelength_nm: float) -> complex:
    return JohnsonChristyMaterial.gold().dielectric_function(wavelength_nm, extrapolate=True)


def au_workload(name, positions, spacing, wavelength_nm, n_env=1.0) -> Workload:
    eps = gold_eps(wavelength_nm)
    k = wavenumber(wavelength_nm, n_env)
    a = complex(rrcm_array(spacing ** 3, eps, n_env * n_env, k))
    return Workload(name, positions, _isotropic(a, positions.shape[0]), wavelength_nm, k, spacing,
                    True, n_env)


def sphere_au_925(wavelength_nm: float = 520.0) -> Workload:
    pos = discretise_primitive(Sphere((0.0, 0.0, 0.0), 12.0), 2.0)
    return au_workload("sphere_au_R12_d2", pos, 2.0, wavelength_nm)


def cuboid_au_30k(wavelength_nm: float = 520.0) -> Workload:
    pos = cell_centred_cuboid((60.0, 50.0, 10.0), 1.0)
    return au_workload("cuboid_au_60x50x10_d1", pos, 1.0, wavelength_nm)


def cuboid_au(size, spacing, wavelength_nm=520.0) -> Workload:
    pos = cell_centred_cuboid(size, spacing)
    return au_workload(f"cuboid_au_{size[0]:g}x{size[1]:g}x{size[2]:g}_d{spacing:g}", pos, spacing,
                       wavelength_nm)


def sweep_wavelengths(lo=400.0, hi=900.0, count=51):
    return list(np.linspace(lo, hi, count))
