"""Periodic lattice and substrate specifications.

``LatticeSpec`` mirrors crates/lumina-geometry/src/lattice.rs:29-102;
``SubstrateSpec`` / ``SubstrateRuntime`` and the Fresnel factors mirror
crates/lumina-core/src/solver/substrate.rs:61-197 (the image-dipole variant;
the Sommerfeld variant is not part of this library).
"""
from __future__ import annotations

import cmath
import math
from dataclasses import dataclass
from typing import Optional, Sequence


@dataclass
class LatticeSpec:
    a1: Sequence[float]
    a2: Optional[Sequence[float]] = None
    ewald_eta: Optional[float] = None
    truncation_real: int = 5
    truncation_recip: int = 5

    @staticmethod
    def chain(a1) -> "LatticeSpec":
        return LatticeSpec(tuple(a1))

    @staticmethod
    def planar(a1, a2) -> "LatticeSpec":
        return LatticeSpec(tuple(a1), tuple(a2))

    def is_2d(self) -> bool:
        return self.a2 is not None

    def cell_measure(self) -> float:
        a1 = self.a1
        if self.a2 is not None:
            a2 = self.a2
            cx = a1[1] * a2[2] - a1[2] * a2[1]
            cy = a1[2] * a2[0] - a1[0] * a2[2]
            cz = a1[0] * a2[1] - a1[1] * a2[0]
            return math.sqrt(cx * cx + cy * cy + cz * cz)
        return math.sqrt(a1[0] ** 2 + a1[1] ** 2 + a1[2] ** 2)

    def eta(self) -> float:
        if self.ewald_eta is not None:
            return self.ewald_eta
        return math.sqrt(math.pi / self.cell_measure())


def fresnel_delta_eps(eps_sub: complex, eps_env: float) -> complex:
    """Quasi-static (eps_s - eps_e)/(eps_s + eps_e)."""
    return (eps_sub - eps_env) / (eps_sub + eps_env)


def fresnel_reflection_amplitude(eps_sub: complex, eps_env: float) -> complex:
    """Retarded normal-incidence r = (n_s - n_e)/(n_s + n_e), principal sqrt."""
    n_sub = cmath.sqrt(complex(eps_sub))
    n_env = math.sqrt(eps_env)
    return (n_sub - n_env) / (n_sub + n_env)


def substrate_reflection_factor(eps_sub: complex, eps_env: float, use_retarded: bool) -> complex:
    if use_retarded:
        return fresnel_reflection_amplitude(eps_sub, eps_env)
    return fresnel_delta_eps(eps_sub, eps_env)


@dataclass
class SubstrateSpec:
    """SubstrateSpec (solver/substrate.rs:56-83); ``use_sommerfeld`` selects
    the full Sommerfeld-integral reflected tensor and overrides
    ``use_retarded``."""
    z_interface: float = 0.0
    material: str = ""
    use_retarded: bool = True
    use_sommerfeld: bool = False


@dataclass
class SommerfeldRuntime:
    """SubstrateRuntime::Sommerfeld (solver/substrate.rs:109-113): the
    interface plane and the SommerfeldGreens parameters (sommerfeld.rs:
    236-241), evaluated on the device by the sessions."""
    z_interface: float
    wavelength_nm: float
    eps_sub: complex
    eps_env: float


@dataclass
class SubstrateRuntime:
    """The Fresnel image-dipole runtime: interface plane and scalar factor."""
    z_interface: float
    delta_eps: complex

    @staticmethod
    def from_spec(spec: SubstrateSpec, eps_sub: complex, eps_env: float,
                  wavelength_nm: Optional[float] = None):
        """SubstrateRuntime::from_spec (substrate.rs:125-137): the Fresnel
        runtime, or a SommerfeldRuntime when ``spec.use_sommerfeld``."""
        if spec.use_sommerfeld:
            if wavelength_nm is None:
                raise ValueError("the Sommerfeld substrate needs the wavelength")
            return SommerfeldRuntime(float(spec.z_interface), float(wavelength_nm),
                                     complex(eps_sub), float(eps_env))
        return SubstrateRuntime(spec.z_interface,
                                substrate_reflection_factor(eps_sub, eps_env, spec.use_retarded))
