"""SommerfeldGreens (crates/lumina-core/src/solver/sommerfeld.rs) on the device.

The reflected Green's dyadic of a planar substrate by the Sommerfeld integral
over k_par: five integrals (15-node Kronrod rule on [0, k_env],
[k_env, Re k_sub] and [max(k_env, Re k_sub), k_max]) combined into the 3x3
tensor of sommerfeld.rs:254-300.  ``evaluate`` runs on the B200
(``lum_sommerfeld_tensor``); the sessions fold the same tensor into their
operator through ``SommerfeldRuntime`` (lattice.py).
"""
from __future__ import annotations

import cmath
import math
from typing import Optional

import numpy as np

from .backend import CudaBackend
from .lattice import SommerfeldRuntime


def _csqrt_pos_im(z: complex) -> complex:
    s = cmath.sqrt(z)
    return -s if s.imag < 0.0 else s


class SommerfeldGreens:
    """SommerfeldGreens::new(wavelength_nm, eps_sub, eps_env)
    (sommerfeld.rs:236-241): k_env = k0 sqrt(eps_env),
    k_sub = sqrt(eps_sub k0^2) with Im >= 0."""

    def __init__(self, wavelength_nm: float, eps_sub: complex, eps_env: float,
                 backend: Optional[CudaBackend] = None):
        k0 = 2.0 * math.pi / wavelength_nm
        self.wavelength_nm = float(wavelength_nm)
        self.eps_sub = complex(eps_sub)
        self.eps_env = float(eps_env)
        self.k_env = k0 * math.sqrt(eps_env)
        self.k_sub = _csqrt_pos_im(self.eps_sub * k0 * k0)
        self.n_subdiv = 1
        self._backend = backend

    def runtime(self, z_interface: float) -> SommerfeldRuntime:
        return SommerfeldRuntime(float(z_interface), self.wavelength_nm, self.eps_sub,
                                 self.eps_env)

    def evaluate(self, ri, rj, z_interface: float) -> np.ndarray:
        """G_refl(r_i, r_j) (sommerfeld.rs:254-300); ri / rj may be (P, 3)
        arrays of pairs, giving (P, 3, 3)."""
        if self._backend is None:
            self._backend = CudaBackend(0)
        return self._backend.sommerfeld_tensor(self.runtime(z_interface), ri, rj)
