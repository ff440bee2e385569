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


# ---------------------------------------------------------------------------
# Batched clusters
# ---------------------------------------------------------------------------
_M64 = (1 << 64) - 1


class SplitMix64:
    """Vigna's splitmix64 generator (seeded, platform-independent)."""

    def __init__(self, seed: int):
        self.state = seed & _M64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _M64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
        return z ^ (z >> 31)

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))


@dataclass
class Cluster:
    positions: np.ndarray       # (N, 3)
    alpha: np.ndarray           # (N, 3, 3) complex, anisotropic (ellipsoid route)
    semi_axes: tuple
    euler_deg: tuple
    eps: complex


@dataclass
class BatchWorkload:
    name: str
    clusters: list
    wavelength_nm: float
    k: float
    cell_size: float
    polarisations: tuple        # real unit vectors, incidence along +z

    def systems(self):
        """(positions, alpha, k, cell, IncidentField) per (cluster, polarisation),
        clusters outer."""
        from .types import IncidentField
        out = []
        for c in self.clusters:
            for pol in self.polarisations:
                out.append((c.positions, c.alpha, self.k, self.cell_size,
                            IncidentField((0.0, 0.0, 1.0), pol, 1.0)))
        return out

    @property
    def n_dipoles(self):
        return sum(c.positions.shape[0] for c in self.clusters) * len(self.polarisations)


def batch_clusters(count=256, seed=0, spacing=1.5, wavelength_nm=600.0, n_range=(200, 5000),
                   axes_range=(4.0, 20.0), polarisations=((1.0, 0.0, 0.0), (0.0, 1.0, 0.0))):
    """``count`` Drude ellipsoids on a ``spacing`` lattice (splitmix64 ``seed``).

    Per cluster: a target size N ~ U[n_range]; semi-axes ~ U[axes_range]
    redrawn until, scaled to the volume N*spacing^3, all three stay inside
    axes_range; Euler angles ~ U[0, 360) deg; Drude eps_inf ~ U[1, 10],
    omega_p ~ U[8, 9.5] eV, gamma ~ U[0.05, 0.2] eV.  The ellipsoid is
    discretised in its own frame on the centred lattice (discretise.rs:27-58)
    and rotated, and every dipole gets the reference's anisotropic
    ellipsoid tensor (scene.rs:507-517, types.rs:286-317): per-axis CM with
    the ellipsoid's depolarisation factors, RRCM, R diag R^T."""
    from .geometry import Ellipsoid, ellipsoid_depol_factors, rotation_zyx
    from .materials import DrudeLorentz
    from .types import ellipsoid_polarisability_tensor
    rng = SplitMix64(seed)
    k = wavenumber(wavelength_nm, 1.0)
    vol = spacing ** 3
    lo_a, hi_a = axes_range
    clusters = []
    for _ in range(count):
        n_target = rng.uniform(*n_range)
        v_target = n_target * vol
        for _attempt in range(1000):
            ax = [rng.uniform(lo_a, hi_a) for _ in range(3)]
            scale = (3.0 * v_target / (4.0 * math.pi * ax[0] * ax[1] * ax[2])) ** (1.0 / 3.0)
            ax = [a * scale for a in ax]
            if all(lo_a <= a <= hi_a for a in ax):
                break
        euler = tuple(rng.uniform(0.0, 360.0) for _ in range(3))
        drude = DrudeLorentz(rng.uniform(1.0, 10.0), rng.uniform(8.0, 9.5), rng.uniform(0.05, 0.2))
        eps = drude.dielectric_function(wavelength_nm)
        local = discretise_primitive(Ellipsoid((0.0, 0.0, 0.0), ax), spacing)
        R = rotation_zyx(*euler)
        pos = np.ascontiguousarray(local @ R.T)
        L = ellipsoid_depol_factors(ax)
        a = ellipsoid_polarisability_tensor(vol, L, eps, 1.0, k, R.ravel())
        alpha = np.broadcast_to(a, (pos.shape[0], 3, 3)).copy()
        clusters.append(Cluster(pos, alpha, tuple(ax), euler, eps))
    return BatchWorkload(f"clusters{count}_seed{seed}_d{spacing:g}", clusters, wavelength_nm, k,
                         spacing, tuple(polarisations))


# ---------------------------------------------------------------------------
# Chiral dimer (adjoint gradients)
# ---------------------------------------------------------------------------
@dataclass
class DimerWorkload:
    workload: Workload
    eps: complex
    lcp: tuple                  # complex polarisation (x + i y)/sqrt(2)
    rcp: tuple                  # (x - i y)/sqrt(2)
    direction: tuple = (0.0, 0.0, 1.0)

    def dinv_alpha_deps(self):
        """d(alpha^-1)/d eps per dipole for isotropic RRCM in vacuum:
        alpha^-1 = 1/alpha_CM - i k^3/(6 pi) (types.rs:243-259) gives
        -eps_m / (V (eps - eps_m)^2) on the diagonal."""
        w = self.workload
        v = w.cell_size ** 3
        d = -1.0 / (v * (self.eps - 1.0) ** 2)
        return np.broadcast_to(np.eye(3, dtype=np.complex128) * d, (w.n, 3, 3)).copy()


def helix_dimer(spacing=1.0, wavelength_nm=650.0, pitch=40.0, radius=15.0, wire=5.0, turns=2.0,
                gap=20.0):
    """Two left-handed Au helices (axis z) side by side along x with ``gap`` nm
    between their outer surfaces.  The reference's Helix primitive is
    right-handed only (primitives.rs:126-211, v = axis x u), so each helix is
    discretised right-handed and mirrored (x -> -x).  Au J&C, RRCM, FCD with
    cell = spacing, vacuum."""
    from .geometry import Helix
    h = Helix((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), radius, pitch, turns, wire)
    one = discretise_primitive(h, spacing)
    one = one * np.array([-1.0, 1.0, 1.0])[None, :]
    shift = 2.0 * (radius + wire) + gap
    pos = np.ascontiguousarray(np.concatenate([one, one + np.array([shift, 0.0, 0.0])[None, :]]))
    w = au_workload(f"helix_dimer_p{pitch:g}_R{radius:g}_w{wire:g}_d{spacing:g}", pos, spacing,
                    wavelength_nm)
    s = 1.0 / math.sqrt(2.0)
    return DimerWorkload(w, gold_eps(wavelength_nm), (s, 1j * s, 0.0), (s, -1j * s, 0.0))
