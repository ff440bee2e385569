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


@dataclass
class PeriodicWorkload:
    workload: Workload
    lattice: object
    substrate: object
    k_bloch: tuple
    incident: object


def metasurface(spacing=4.0, wavelength_nm=600.0, diameter=100.0, height=40.0, period=400.0,
                angle_deg=10.0, n_substrate=1.45, gap=None):
    """Square array (period 400 nm) of Au cylinders (d 100, h 40 nm) on an
    n = 1.45 substrate (retarded Fresnel image, interface z = 0); plane wave
    incident at ``angle_deg`` in the xz plane (p-polarised), Bloch vector
    k sin(angle) x.  At 4 nm the cylinder holds ~5.4k dipoles, at 2 nm ~41k."""
    from .geometry import Cylinder
    from .lattice import LatticeSpec, SubstrateRuntime, fresnel_reflection_amplitude
    from .types import IncidentField
    gap = spacing / 2.0 if gap is None else gap
    cyl = Cylinder((0.0, 0.0, gap), (0.0, 0.0, 1.0), height, diameter / 2.0)
    pos = discretise_primitive(cyl, spacing)
    w = au_workload(f"metasurface_d{diameter:g}_h{height:g}_s{spacing:g}", pos, spacing,
                    wavelength_nm)
    th = math.radians(angle_deg)
    lat = LatticeSpec.planar((period, 0.0, 0.0), (0.0, period, 0.0))
    sub = SubstrateRuntime(0.0, fresnel_reflection_amplitude(n_substrate ** 2, 1.0))
    inc = IncidentField((math.sin(th), 0.0, math.cos(th)), (math.cos(th), 0.0, -math.sin(th)), 1.0)
    return PeriodicWorkload(w, lat, sub, (w.k * math.sin(th), 0.0, 0.0), inc)
