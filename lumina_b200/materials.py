"""Dielectric functions: tabulated gold (Johnson & Christy 1972) through a
natural cubic spline, and a Drude-Lorentz model for synthetic particles.

Mirrors crates/lumina-materials/src/spline.rs:32-90 and
johnson_christy.rs:51-117, 258-279.  The gold table ships in
``data/johnson_christy_au.csv`` (extracted from the reference by
``data/extract_jc_table.py``).
"""
from __future__ import annotations

import math
import os

import numpy as np

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")

HBAR_EV_NM = 1239.8419843320026  # h c in eV nm: E[eV] = HBAR_EV_NM / lambda[nm]


class MaterialError(ValueError):
    pass


class OutOfRange(MaterialError):
    def __init__(self, wavelength_nm, lo, hi):
        super().__init__(f"wavelength {wavelength_nm} nm outside [{lo}, {hi}] nm")
        self.wavelength_nm, self.min, self.max = wavelength_nm, lo, hi


class CubicSpline:
    """Natural cubic spline (second derivatives zero at both ends)."""

    def __init__(self, xs, ys):
        xs = [float(v) for v in xs]
        ys = [float(v) for v in ys]
        if len(xs) != len(ys) or len(xs) < 2:
            raise ValueError("need >= 2 points of equal length")
        for i in range(1, len(xs)):
            if not xs[i] > xs[i - 1]:
                raise ValueError(f"xs must be strictly increasing at index {i}")
        n = len(xs)
        y2 = [0.0] * n
        u = [0.0] * (n - 1)
        for i in range(1, n - 1):
            sig = (xs[i] - xs[i - 1]) / (xs[i + 1] - xs[i - 1])
            p = sig * y2[i - 1] + 2.0
            y2[i] = (sig - 1.0) / p
            u[i] = (ys[i + 1] - ys[i]) / (xs[i + 1] - xs[i]) - (ys[i] - ys[i - 1]) / (xs[i] - xs[i - 1])
            u[i] = (6.0 * u[i] / (xs[i + 1] - xs[i - 1]) - sig * u[i - 1]) / p
        for k in range(n - 3, -1, -1):
            y2[k + 1] = y2[k + 1] * y2[k + 2] + u[k + 1]
        self.xs, self.ys, self.y2s = xs, ys, y2

    def evaluate(self, x: float) -> float:
        xs, ys, y2 = self.xs, self.ys, self.y2s
        lo, hi = 0, len(xs) - 1
        while hi - lo > 1:
            mid = (lo + hi) // 2
            if xs[mid] > x:
                hi = mid
            else:
                lo = mid
        h = xs[hi] - xs[lo]
        a = (xs[hi] - x) / h
        b = (x - xs[lo]) / h
        return a * ys[lo] + b * ys[hi] + ((a * a * a - a) * y2[lo] + (b * b * b - b) * y2[hi]) * h * h / 6.0


class JohnsonChristyMaterial:
    """Spline-interpolated tabulated dielectric function."""

    def __init__(self, name, wavelengths_nm, eps_real, eps_imag):
        self.name = name
        self.wavelengths_nm = list(wavelengths_nm)
        self.spline_real = CubicSpline(wavelengths_nm, eps_real)
        self.spline_imag = CubicSpline(wavelengths_nm, eps_imag)

    @staticmethod
    def gold() -> "JohnsonChristyMaterial":
        wl, er, ei = [], [], []
        with open(os.path.join(_DATA, "johnson_christy_au.csv")) as f:
            for line in f:
                if line.startswith("#") or not line.strip():
                    continue
                w_um, n, k = (float(v) for v in line.split(","))
                wl.append(w_um * 1000.0)
                er.append(n * n - k * k)
                ei.append(2.0 * n * k)
        return JohnsonChristyMaterial("Au (Johnson & Christy)", wl, er, ei)

    def wavelength_range(self):
        return self.wavelengths_nm[0], self.wavelengths_nm[-1]

    def dielectric_function(self, wavelength_nm: float, extrapolate: bool = False) -> complex:
        """eps(lambda); outside the table raises OutOfRange unless
        ``extrapolate`` asks for the spline's boundary polynomial."""
        lo, hi = self.wavelength_range()
        if not extrapolate and (wavelength_nm < lo or wavelength_nm > hi):
            raise OutOfRange(wavelength_nm, lo, hi)
        return complex(self.spline_real.evaluate(wavelength_nm), self.spline_imag.evaluate(wavelength_nm))


class DrudeLorentz:
    """eps(omega) = eps_inf - omega_p^2 / (omega^2 + i gamma omega), energies in eV."""

    def __init__(self, eps_inf: float, omega_p_ev: float, gamma_ev: float):
        self.eps_inf, self.omega_p, self.gamma = eps_inf, omega_p_ev, gamma_ev

    def dielectric_function(self, wavelength_nm: float) -> complex:
        w = HBAR_EV_NM / wavelength_nm
        return self.eps_inf - self.omega_p ** 2 / complex(w * w, self.gamma * w)
