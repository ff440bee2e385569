"""Fields from solved dipole moments on the device (the reference's fields.rs).

Mirror of crates/lumina-core/src/fields.rs and the OpticalSolver hooks
compute_near_field / compute_far_field (solver/mod.rs:56-76); the work runs in
lum_near_field / lum_near_field_map / lum_far_field (csrc/fields.cu).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _ffi
from .backend import CudaBackend, _dp, _raise
from .types import DipoleResponse, IncidentField


@dataclass
class NearFieldPlane:
    """solver/mod.rs:81-96."""
    centre: Sequence[float] = (0.0, 0.0, 0.0)
    normal: Sequence[float] = (0.0, 0.0, 1.0)
    half_width: float = 50.0
    half_height: float = 50.0
    nx: int = 64
    ny: int = 64


@dataclass
class NearFieldMap:
    """types.rs:206-219: positions (nx*ny, 3), |E|^2 (nx*ny,), extent."""
    positions: np.ndarray
    field_intensity: np.ndarray
    nx: int
    ny: int
    extent: np.ndarray


@dataclass
class FarFieldMap:
    """types.rs:172-187."""
    wavelength_nm: float
    theta: np.ndarray
    phi: np.ndarray
    intensity: np.ndarray
    n_theta: int
    n_phi: int


def _v3(v) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(v, np.float64).reshape(3))


def _pos_mom(positions, moments):
    pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
    mom = np.ascontiguousarray(np.asarray(moments, np.complex128).reshape(-1))
    if mom.size != 3 * pos.shape[0]:
        raise ValueError(f"{pos.shape[0]} dipoles but {mom.size} moment entries")
    return pos, mom


def field_at_points(backend: CudaBackend, positions, moments, k: float, obs,
                    incident: IncidentField = IncidentField()) -> np.ndarray:
    """E at every row of ``obs`` (fields.rs:18-49): (M, 3) complex."""
    pos, mom = _pos_mom(positions, moments)
    o = np.ascontiguousarray(np.asarray(obs, np.float64).reshape(-1, 3))
    out = np.zeros(3 * o.shape[0], np.complex128)
    lib = _ffi.load()
    _raise(lib.lum_near_field(backend._h, pos.shape[0], _dp(pos), _dp(mom.view(np.float64)),
                              float(k), _dp(_v3(incident.direction)),
                              _dp(_v3(incident.polarisation)), float(incident.amplitude),
                              o.shape[0], _dp(o), out.ctypes.data, None), "near_field")
    return out.reshape(-1, 3)


def compute_near_field_map(backend: CudaBackend, positions, moments, plane: NearFieldPlane,
                           k: float, incident: IncidentField = IncidentField()) -> NearFieldMap:
    """fields.rs:52-105."""
    pos, mom = _pos_mom(positions, moments)
    m = int(plane.nx) * int(plane.ny)
    grid = np.zeros(3 * m)
    inten = np.zeros(m)
    ext = np.zeros(4)
    lib = _ffi.load()
    _raise(lib.lum_near_field_map(backend._h, pos.shape[0], _dp(pos), _dp(mom.view(np.float64)),
                                  float(k), _dp(_v3(incident.direction)),
                                  _dp(_v3(incident.polarisation)), float(incident.amplitude),
                                  _dp(_v3(plane.centre)), _dp(_v3(plane.normal)),
                                  float(plane.half_width), float(plane.half_height),
                                  int(plane.nx), int(plane.ny), grid.ctypes.data, _dp(inten),
                                  _dp(ext)), "near_field_map")
    return NearFieldMap(grid.reshape(-1, 3), inten, int(plane.nx), int(plane.ny), ext)


def compute_far_field(backend: CudaBackend, positions, response: DipoleResponse, k: float,
                      n_theta: int, n_phi: int) -> FarFieldMap:
    """fields.rs:147-221."""
    pos, mom = _pos_mom(positions, response.moments)
    m = int(n_theta) * int(n_phi)
    th, ph, it = np.zeros(m), np.zeros(m), np.zeros(m)
    lib = _ffi.load()
    _raise(lib.lum_far_field(backend._h, pos.shape[0], _dp(pos), _dp(mom.view(np.float64)),
                             float(k), int(n_theta), int(n_phi), _dp(th), _dp(ph), _dp(it)),
           "far_field")
    return FarFieldMap(response.wavelength_nm, th, ph, it, int(n_theta), int(n_phi))
