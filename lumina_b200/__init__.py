"""lumina_b200 -- B200-native (sm_100a) coupled-dipole (CDA) solve.

The compute path is liblumina_b200.so (hand-written CUDA, C ABI in
include/lumina_b200.h); this package is its host-side mirror of the
reference's ComputeBackend / MatvecSession / CdaSolver interfaces plus the
input types (dipoles, materials, lattices, geometry).
"""
from . import _ffi
from .backend import (ComputeError, ConvergenceFailure, CudaBackend, CudaBatch, CudaSession,
                      DeviceError, DeviceTimeout,
                      InvalidGeometry, OutOfMemory, SolverError, Unavailable, cross_sections,
                      incident_field, invert_polarisability)
from .lattice import LatticeSpec, SommerfeldRuntime, SubstrateRuntime, SubstrateSpec
from .solver import CdaSolver, circular_dichroism
from .types import (CrossSections, Dipole, DipoleResponse, DipoleSet, IncidentField,
                    SimulationParams, clausius_mossotti, ellipsoid_polarisability_tensor,
                    radiative_correction, wavenumber)

__all__ = [
    "CudaBackend", "CudaSession", "CudaBatch", "CdaSolver", "ComputeError", "Unavailable", "DeviceError",
    "DeviceTimeout",
    "OutOfMemory", "SolverError", "ConvergenceFailure", "InvalidGeometry", "LatticeSpec",
    "SubstrateSpec", "SubstrateRuntime", "SommerfeldRuntime", "Dipole", "DipoleSet", "IncidentField",
    "SimulationParams", "CrossSections", "DipoleResponse", "clausius_mossotti",
    "radiative_correction", "ellipsoid_polarisability_tensor", "wavenumber",
    "invert_polarisability", "incident_field", "cross_sections", "circular_dichroism",
]


def build(verbose: bool = False) -> str:
    """Compile liblumina_b200.so in-tree for sm_100a (nvcc)."""
    import os
    import subprocess
    csrc = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc")
    subprocess.run(["make", "-s", "-C", csrc, "-j4"], check=True,
                   stdout=None if verbose else subprocess.DEVNULL)
    return _ffi.LIB_PATH
