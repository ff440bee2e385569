"""TEST INFRASTRUCTURE ONLY -- Mie extinction of a homogeneous sphere.

The published Lorenz-Mie series (Bohren & Huffman, "Absorption and
Scattering of Light by Small Particles", 1983, ch. 4): with size parameter
x = k a, relative index m = sqrt(eps) / n_med, psi_n(z) = z j_n(z) and
xi_n(z) = z h_n^(1)(z),

  a_n = [m psi_n(mx) psi_n'(x) - psi_n(x) psi_n'(mx)] /
        [m psi_n(mx) xi_n'(x)  - xi_n(x)  psi_n'(mx)]
  b_n = [psi_n(mx) psi_n'(x) - m psi_n(x) psi_n'(mx)] /
        [psi_n(mx) xi_n'(x)  - m xi_n(x)  psi_n'(mx)]

  C_ext = (2 pi / k^2) sum_n (2n + 1) Re(a_n + b_n)
  C_sca = (2 pi / k^2) sum_n (2n + 1) (|a_n|^2 + |b_n|^2)

summed to n_max = x + 4 x^(1/3) + 2.  It is the analytic comparison of the
reference's CDA-vs-Mie integration tests (tests/mie_validation.rs); the
reference's own Mie module is not restated here.  Used by tests only.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import spherical_jn, spherical_yn


def _psi(n, z):
    j = spherical_jn(n, z)
    dj = spherical_jn(n, z, derivative=True)
    return z * j, j + z * dj


def _xi(n, x):
    h = spherical_jn(n, x) + 1j * spherical_yn(n, x)
    dh = (spherical_jn(n, x, derivative=True) + 1j * spherical_yn(n, x, derivative=True))
    return x * h, h + x * dh


def mie_cross_sections(radius_nm: float, wavelength_nm: float, epsilon: complex,
                       n_medium: float = 1.0):
    """(C_ext, C_sca, C_abs) in nm^2."""
    k = 2.0 * math.pi * n_medium / wavelength_nm
    x = k * radius_nm
    m = np.sqrt(complex(epsilon)) / n_medium
    nmax = int(math.ceil(x + 4.0 * x ** (1.0 / 3.0) + 2.0))
    n = np.arange(1, nmax + 1)
    px, dpx = _psi(n, x)
    pm, dpm = _psi(n, m * x)
    xx, dxx = _xi(n, x)
    a = (m * pm * dpx - px * dpm) / (m * pm * dxx - xx * dpm)
    b = (pm * dpx - m * px * dpm) / (pm * dxx - m * xx * dpm)
    w = 2.0 * n + 1.0
    c_ext = 2.0 * math.pi / k ** 2 * float(np.sum(w * (a + b).real))
    c_sca = 2.0 * math.pi / k ** 2 * float(np.sum(w * (np.abs(a) ** 2 + np.abs(b) ** 2)))
    return c_ext, c_sca, c_ext - c_sca
