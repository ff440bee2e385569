"""ctypes binding of ``liblumina_b200.so`` (the C ABI in include/lumina_b200.h).

The library is loaded from ``lumina_b200/lib/`` inside the package tree.  If
it is missing the import fails loudly: there is no CPU fallback for any
entry point.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_longlong, c_size_t, c_uint64, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "liblumina_b200.so")
HEADER_PATH = os.path.join(os.path.dirname(_HERE), "include", "lumina_b200.h")

LUM_OK = 0
LUM_ERR_UNAVAILABLE = 1
LUM_ERR_DEVICE = 2
LUM_ERR_OOM = 3
LUM_ERR_NOT_CONVERGED = 4
LUM_ERR_TIMEOUT = 5
LUM_ERR_INVALID = 6

LUM_FP64 = 0
LUM_FP32 = 1
LUM_STORAGE_SYMMETRIC = 0x10
LUM_SOLVE_FP64 = 0
LUM_SOLVE_FP32_REFINE = 1

_dp = POINTER(c_double)


class LumLattice(ctypes.Structure):
    _fields_ = [
        ("a1", c_double * 3),
        ("a2", c_double * 3),
        ("is_2d", c_int),
        ("has_eta", c_int),
        ("eta", c_double),
        ("truncation_real", c_int),
        ("truncation_recip", c_int),
    ]


class LumSubstrate(ctypes.Structure):
    _fields_ = [("z_interface", c_double), ("refl_re", c_double), ("refl_im", c_double)]


class LumSommerfeld(ctypes.Structure):
    _fields_ = [("z_interface", c_double), ("wavelength_nm", c_double), ("eps_sub_re", c_double),
                ("eps_sub_im", c_double), ("eps_env", c_double)]


class LumSolveInfo(ctypes.Structure):
    _fields_ = [
        ("iterations", c_int),
        ("restarts", c_int),
        ("matvecs_fp64", c_int),
        ("matvecs_fp32", c_int),
        ("matvecs_reference", c_int),
        ("converged", c_int),
        ("rel_residual", c_double),
        ("seconds", c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# name -> (restype, argtypes); every symbol the header declares.
SIGNATURES = {
    "lum_ctx_create": (c_int, [c_int, POINTER(c_void_p)]),
    "lum_ctx_destroy": (c_int, [c_void_p]),
    "lum_device_info": (c_int, [c_void_p, c_char_p, c_size_t, POINTER(c_size_t), POINTER(c_int)]),
    "lum_last_error": (c_char_p, []),
    "lum_last_oom": (c_int, [POINTER(c_size_t), POINTER(c_size_t)]),
    "lum_launch_count": (c_uint64, []),
    "lum_invert_polarisability": (c_int, [c_int, _dp, _dp]),
    "lum_incident_field": (c_int, [c_int, _dp, _dp, _dp, c_double, c_double, _dp]),
    "lum_cross_sections": (c_int, [c_int, _dp, _dp, _dp, c_double, _dp, _dp, c_double, _dp]),
    "lum_session_create_cached": (c_int, [c_void_p, c_int, c_int, POINTER(c_void_p)]),
    "lum_session_upload_matrix": (c_int, [c_void_p, _dp]),
    "lum_session_assemble": (c_int, [c_void_p, c_int, _dp, _dp, c_double, c_int, c_double,
                                     c_void_p, _dp, c_void_p, c_int, POINTER(c_void_p)]),
    "lum_session_create_onthefly": (c_int, [c_void_p, c_int, _dp, _dp, c_double, c_int,
                                            c_double, c_void_p, _dp, c_void_p,
                                            POINTER(c_void_p)]),
    "lum_session_set_wavelength": (c_int, [c_void_p, c_double, _dp, c_void_p]),
    "lum_session_assemble_sommerfeld": (c_int, [c_void_p, c_int, _dp, _dp, c_double, c_int,
                                                c_double, c_void_p, _dp, c_void_p, c_int,
                                                POINTER(c_void_p)]),
    "lum_session_create_onthefly_sommerfeld": (c_int, [c_void_p, c_int, _dp, _dp, c_double,
                                                       c_int, c_double, c_void_p, _dp, c_void_p,
                                                       POINTER(c_void_p)]),
    "lum_session_set_sommerfeld": (c_int, [c_void_p, c_void_p]),
    "lum_sommerfeld_tensor": (c_int, [c_void_p, c_void_p, c_int, _dp, _dp, _dp]),
    "lum_session_create_fft": (c_int, [c_void_p, c_int, _dp, _dp, c_double, c_int, c_double,
                                       c_double, POINTER(c_void_p)]),
    "lum_session_matvec": (c_int, [c_void_p, c_int, _dp, _dp]),
    "lum_session_matvec_device": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "lum_session_matmul_device": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "lum_session_matmul_vectors_device": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int,
                                                  c_void_p]),
    "lum_session_matmul_vectors": (c_int, [c_void_p, _dp, _dp, c_int, c_int]),
    "lum_session_set_stream": (c_int, [c_void_p, c_void_p]),
    "lum_session_destroy": (c_int, [c_void_p]),
    "lum_solve_gmres": (c_int, [c_void_p, _dp, c_double, c_int, c_int, c_int, _dp,
                                POINTER(LumSolveInfo)]),
    "lum_solve_gmres_device": (c_int, [c_void_p, c_void_p, c_void_p, c_double, c_int, c_int,
                                       c_int, POINTER(LumSolveInfo), c_void_p]),
    "lum_session_profile": (c_int, [c_void_p, c_int]),
    "lum_session_kernel_time": (c_int, [c_void_p, c_int, POINTER(c_int), POINTER(c_double)]),
    "lum_session_stats": (c_int, [c_void_p, POINTER(c_longlong), POINTER(c_int), POINTER(c_int),
                                  POINTER(c_int)]),
    "lum_session_kernel_config": (c_int, [c_void_p, c_char_p, c_size_t]),
    "lum_measure_fma_peak": (c_int, [c_void_p, POINTER(c_double), POINTER(c_double)]),
    "lum_measure_l2_peak": (c_int, [c_void_p, POINTER(c_double)]),
    "lum_measure_fma2_peak": (c_int, [c_void_p, POINTER(c_double)]),
    "lum_near_field": (c_int, [c_void_p, c_int, _dp, _dp, c_double, _dp, _dp, c_double, c_int,
                               _dp, c_void_p, c_void_p]),
    "lum_near_field_map": (c_int, [c_void_p, c_int, _dp, _dp, c_double, _dp, _dp, c_double,
                                   _dp, _dp, c_double, c_double, c_int, c_int, c_void_p, _dp,
                                   _dp]),
    "lum_far_field": (c_int, [c_void_p, c_int, _dp, _dp, c_double, c_int, c_int, _dp, _dp,
                              _dp]),
    "lum_harmonic_sources": (c_int, [c_void_p, c_int, c_int, _dp, c_int, _dp, _dp]),
    "lum_matvec_onthefly_noalloc": (c_int, [c_int, c_void_p, c_void_p, c_double, c_void_p,
                                            c_void_p, c_void_p]),
    "lum_batch_create": (c_int, [c_void_p, c_int, POINTER(c_int), _dp, _dp, _dp, _dp, c_int,
                                 POINTER(c_void_p)]),
    "lum_batch_matvec": (c_int, [c_void_p, c_int, _dp, _dp]),
    "lum_batch_matvec_device": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
    "lum_batch_solve": (c_int, [c_void_p, _dp, c_double, c_int, c_int, c_int, _dp,
                                POINTER(LumSolveInfo)]),
    "lum_batch_solve_device": (c_int, [c_void_p, c_void_p, c_void_p, c_double, c_int, c_int,
                                       c_int, POINTER(LumSolveInfo)]),
    "lum_batch_set_stream": (c_int, [c_void_p, c_void_p]),
    "lum_batch_kernel_config": (c_int, [c_void_p, c_char_p, c_size_t]),
    "lum_batch_create_rhs": (c_int, [c_void_p, c_int, POINTER(c_void_p)]),
    "lum_batch_info": (c_int, [c_void_p] + [POINTER(c_int)] * 9),
    "lum_batch_destroy": (c_int, [c_void_p]),
    "lum_solve_gmres_multi": (c_int, [c_void_p, c_int, _dp, c_double, c_int, c_int, c_int, _dp,
                                      POINTER(LumSolveInfo)]),
    "lum_solve_gmres_multi_device": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_double,
                                             c_int, c_int, c_int, POINTER(LumSolveInfo),
                                             c_void_p]),
    "lum_grad_cext": (c_int, [c_void_p, _dp, _dp, c_double, c_void_p, c_double, c_int, c_int,
                              c_int, _dp, c_void_p, _dp, c_void_p, POINTER(LumSolveInfo),
                              POINTER(LumSolveInfo)]),
}

_lib = None


def load():
    """Load the CUDA library; raises ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"lumina_b200: native library not found at {LIB_PATH}; build it with "
            "`make -C lumina_b200/csrc` (there is no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    msg = load().lum_last_error()
    return msg.decode() if msg else ""


def launch_count() -> int:
    return int(load().lum_launch_count())
