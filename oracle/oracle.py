"""TEST INFRASTRUCTURE ONLY -- ctypes wrapper of the CPU FP64 oracle.

The oracle (``cda_oracle.cpp``) is a C++ FP64 restatement of the reference's
coupled-dipole solve path (greens.rs, assembly.rs, iterative.rs, ewald.rs,
substrate.rs, types.rs, spline.rs, cda/mod.rs).  It is the checker for the
CUDA library and the timed host-CPU baseline; the product package never
imports this module.

Complex arrays are numpy complex128 (interleaved re/im doubles in memory).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liblumina_oracle.so")

_dp = POINTER(c_double)
_ip = POINTER(c_int)


class OrcLattice(ctypes.Structure):
    _fields_ = [
        ("a1", c_double * 3),
        ("a2", c_double * 3),
        ("is_2d", c_int),
        ("has_eta", c_int),
        ("eta", c_double),
        ("truncation_real", c_int),
        ("truncation_recip", c_int),
    ]


class OrcSubstrate(ctypes.Structure):
    _fields_ = [("z_interface", c_double), ("refl_re", c_double), ("refl_im", c_double)]


class OrcSommerfeld(ctypes.Structure):
    _fields_ = [("z_interface", c_double), ("wavelength_nm", c_double), ("eps_sub_re", c_double),
                ("eps_sub_im", c_double), ("eps_env", c_double)]


def build() -> str:
    """Compile the oracle library in place (g++, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def _load():
    if not os.path.exists(_LIB_PATH):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    sig = {
        "orc_greens": (c_int, [_dp, _dp, c_double, _dp]),
        "orc_greens_filtered": (c_int, [_dp, _dp, c_double, c_double, _dp]),
        "orc_invert_3x3": (c_int, [_dp, _dp]),
        "orc_incident_field": (None, [c_int, _dp, _dp, _dp, c_double, c_double, _dp]),
        "orc_field_at_points": (None, [c_int, _dp, _dp, c_double, _dp, _dp, c_double, c_int,
                                       _dp, _dp]),
        "orc_near_field_plane": (None, [_dp, _dp, c_double, c_double, c_int, c_int, _dp, _dp]),
        "orc_far_field": (None, [c_int, _dp, _dp, c_double, c_int, c_int, _dp, _dp, _dp]),
        "orc_harmonic_sources": (None, [c_int, c_int, _dp, c_int, _dp, _dp]),
        "orc_ewald_evaluate": (None, [ctypes.c_void_p, _dp, _dp, c_double, c_int, _dp]),
        "orc_lattice_eta": (c_double, [ctypes.c_void_p]),
        "orc_erfc": (c_double, [c_double]),
        "orc_csqrt_pos_imag": (None, [c_double, c_double, _dp]),
        "orc_bessel": (c_double, [c_int, c_double]),
        "orc_bessel_kc": (None, [c_int, c_double, c_double, _dp]),
        "orc_assemble": (c_int, [c_int, _dp, _dp, c_double, c_int, c_double, ctypes.c_void_p,
                                 _dp, ctypes.c_void_p, _dp, c_int]),
        "orc_matvec_onthefly": (c_int, [c_int, _dp, _dp, _dp, c_double, c_int, c_double,
                                        ctypes.c_void_p, _dp, ctypes.c_void_p, _dp, c_int]),
        "orc_matvec_onthefly_rows": (c_int, [c_int, _dp, _dp, _dp, c_double, c_int, c_double,
                                             c_int, c_int, _dp, c_int]),
        "orc_matvec_onthefly_rows_ex": (c_int, [c_int, _dp, _dp, _dp, c_double, c_int,
                                                c_double, ctypes.c_void_p, _dp,
                                                ctypes.c_void_p, c_int, c_int, _dp, c_int]),
        "orc_gmres_dense": (c_int, [c_int, _dp, _dp, c_double, c_int, c_int, _dp, _ip, _ip,
                                    _dp, c_int]),
        "orc_gmres_onthefly": (c_int, [c_int, _dp, _dp, _dp, c_double, c_int, c_double,
                                       ctypes.c_void_p, _dp, ctypes.c_void_p, c_double, c_int,
                                       _dp, _ip, _ip, _dp, c_int]),
        "orc_lu_solve": (c_int, [c_int, _dp, _dp, _dp]),
        "orc_cross_sections": (c_int, [c_int, _dp, _dp, _dp, c_double, _dp, _dp, c_double, _dp]),
        "orc_rrcm": (None, [c_double, c_double, c_double, c_double, c_double, c_int, _dp]),
        "orc_ellipsoid_tensor": (None, [c_double, _dp, c_double, c_double, c_double, c_double,
                                        _dp, _dp]),
        "orc_fresnel": (None, [c_double, c_double, c_double, c_int, _dp]),
        "orc_spline_build": (None, [c_int, _dp, _dp, _dp]),
        "orc_spline_eval": (c_double, [c_int, _dp, _dp, _dp, c_double]),
        "orc_circular_dichroism": (c_double, [c_int, _dp, _dp, c_double]),
        "orc_wgsl_assemble_f32": (None, [c_int, _dp, _dp, c_double, POINTER(c_float)]),
        "orc_wgsl_matvec_f32": (None, [c_int, POINTER(c_float), POINTER(c_float),
                                       POINTER(c_float)]),
        "orc_grad_cext": (c_int, [c_int, _dp, _dp, c_double, c_int, c_double, _dp, _dp,
                                  c_double, ctypes.c_void_p, _dp, _dp, _dp, _dp, c_int]),
        "orc_max_threads": (c_int, []),
        "orc_somm_bessel": (c_double, [c_int, c_double]),
        "orc_sommerfeld_tensor": (None, [ctypes.c_void_p, c_int, _dp, _dp, _dp, c_int]),
        "orc_assemble_sommerfeld": (c_int, [c_int, _dp, _dp, c_double, c_int, c_double,
                                            ctypes.c_void_p, _dp, ctypes.c_void_p, _dp, c_int]),
        "orc_matvec_sommerfeld": (c_int, [c_int, _dp, _dp, _dp, c_double, c_int, c_double,
                                          ctypes.c_void_p, _dp, ctypes.c_void_p, _dp, c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _vec(a, dtype=np.float64):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def _lat(lattice):
    if lattice is None:
        return None
    s = OrcLattice()
    s.a1[:] = list(lattice.a1)
    a2 = lattice.a2 if lattice.a2 is not None else (0.0, 0.0, 0.0)
    s.a2[:] = list(a2)
    s.is_2d = 1 if lattice.a2 is not None else 0
    s.has_eta = 1 if lattice.ewald_eta is not None else 0
    s.eta = float(lattice.ewald_eta or 0.0)
    s.truncation_real = int(lattice.truncation_real)
    s.truncation_recip = int(lattice.truncation_recip)
    return s


def _sub(substrate):
    if substrate is None:
        return None
    r = complex(substrate.delta_eps)
    return OrcSubstrate(float(substrate.z_interface), r.real, r.imag)


def _somm(somm):
    e = complex(somm.eps_sub)
    return OrcSommerfeld(float(somm.z_interface), float(somm.wavelength_nm), e.real, e.imag,
                         float(somm.eps_env))


def _ref(struct):
    return ctypes.byref(struct) if struct is not None else None


def greens(r1, r2, k):
    out = np.zeros(9, np.complex128)
    if lib().orc_greens(_p(_vec(r1)), _p(_vec(r2)), k, _p(out.view(np.float64))) != 0:
        raise ValueError("Self-interaction: r1 and r2 must not coincide")
    return out.reshape(3, 3)


def greens_filtered(r1, r2, k, cell):
    out = np.zeros(9, np.complex128)
    lib().orc_greens_filtered(_p(_vec(r1)), _p(_vec(r2)), k, cell, _p(out.view(np.float64)))
    return out.reshape(3, 3)


def invert_3x3(m):
    m = np.ascontiguousarray(np.asarray(m, np.complex128).reshape(9))
    out = np.zeros(9, np.complex128)
    if lib().orc_invert_3x3(_p(m.view(np.float64)), _p(out.view(np.float64))) != 0:
        raise ValueError("Singular polarisability tensor")
    return out.reshape(3, 3)


def incident_field(pos, k, direction=(0, 0, 1), polarisation=(1, 0, 0), amplitude=1.0):
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    out = np.zeros(3 * n, np.complex128)
    lib().orc_incident_field(n, _p(pos), _p(_vec(direction)), _p(_vec(polarisation)),
                             amplitude, k, _p(out.view(np.float64)))
    return out


def ewald(lattice, r, kb, k, part="full"):
    s = _lat(lattice)
    out = np.zeros(9, np.complex128)
    lib().orc_ewald_evaluate(ctypes.byref(s), _p(_vec(r)), _p(_vec(kb)), k,
                             {"full": 0, "real": 1, "recip": 2}[part], _p(out.view(np.float64)))
    return out.reshape(3, 3)


def lattice_eta(lattice):
    return lib().orc_lattice_eta(ctypes.byref(_lat(lattice)))


def erfc(x):
    return lib().orc_erfc(float(x))


def csqrt_positive_imag(z):
    out = np.zeros(2)
    lib().orc_csqrt_pos_imag(complex(z).real, complex(z).imag, _p(out))
    return complex(out[0], out[1])


_BESSEL = {"j0": 0, "j1": 1, "y0": 2, "y1": 3, "i0": 4, "i1": 5, "k0": 6, "k1": 7}


def bessel(name, x):
    return lib().orc_bessel(_BESSEL[name], float(x))


def bessel_kc(order, z):
    out = np.zeros(2)
    lib().orc_bessel_kc(order, complex(z).real, complex(z).imag, _p(out))
    return complex(out[0], out[1])


def _alpha_arr(alpha, n):
    a = np.ascontiguousarray(np.asarray(alpha, np.complex128).reshape(n, 9))
    return a


def assemble(pos, alpha, k, use_fcd=False, cell_size=3.0, lattice=None, k_bloch=(0, 0, 0),
             substrate=None, nthreads=0):
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    A = np.zeros((3 * n, 3 * n), np.complex128)
    ls, ss = _lat(lattice), _sub(substrate)
    rc = lib().orc_assemble(n, _p(pos), _p(a.view(np.float64)), k, int(use_fcd), cell_size,
                            _ref(ls), _p(_vec(k_bloch)), _ref(ss), _p(A.view(np.float64)),
                            nthreads)
    if rc != 0:
        raise ValueError("singular polarisability")
    return A


def matvec_onthefly(pos, alpha, x, k, use_fcd=False, cell_size=3.0, lattice=None,
                    k_bloch=(0, 0, 0), substrate=None, nthreads=0):
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    x = np.ascontiguousarray(np.asarray(x, np.complex128))
    y = np.zeros(3 * n, np.complex128)
    ls, ss = _lat(lattice), _sub(substrate)
    rc = lib().orc_matvec_onthefly(n, _p(pos), _p(a.view(np.float64)), _p(x.view(np.float64)),
                                   k, int(use_fcd), cell_size, _ref(ls), _p(_vec(k_bloch)),
                                   _ref(ss), _p(y.view(np.float64)), nthreads)
    if rc != 0:
        raise ValueError("singular polarisability")
    return y


def matvec_onthefly_rows_ex(pos, alpha, x, k, use_fcd, cell_size, row0, row1, lattice=None,
                            k_bloch=(0, 0, 0), substrate=None, nthreads=0):
    """Rows [row0, row1) of matvec_onthefly with the lattice / substrate terms."""
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    x = np.ascontiguousarray(np.asarray(x, np.complex128))
    y = np.zeros(3 * (row1 - row0), np.complex128)
    ls, ss = _lat(lattice), _sub(substrate)
    rc = lib().orc_matvec_onthefly_rows_ex(n, _p(pos), _p(a.view(np.float64)),
                                           _p(x.view(np.float64)), k, int(use_fcd), cell_size,
                                           _ref(ls), _p(_vec(k_bloch)), _ref(ss), row0, row1,
                                           _p(y.view(np.float64)), nthreads)
    if rc != 0:
        raise ValueError("singular polarisability")
    return y


def matvec_onthefly_rows(pos, alpha, x, k, use_fcd, cell_size, row0, row1, nthreads=0):
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    x = np.ascontiguousarray(np.asarray(x, np.complex128))
    y = np.zeros(3 * (row1 - row0), np.complex128)
    lib().orc_matvec_onthefly_rows(n, _p(pos), _p(a.view(np.float64)), _p(x.view(np.float64)),
                                   k, int(use_fcd), cell_size, row0, row1,
                                   _p(y.view(np.float64)), nthreads)
    return y


class GmresResult:
    def __init__(self, x, status, iterations, matvecs, rel_residual):
        self.x = x
        self.status = status
        self.iterations = iterations
        self.matvecs = matvecs
        self.rel_residual = rel_residual

    @property
    def converged(self):
        return self.status == 0


def gmres_dense(A, b, tol, max_iter, restart=30, nthreads=0):
    A = np.ascontiguousarray(np.asarray(A, np.complex128))
    b = np.ascontiguousarray(np.asarray(b, np.complex128))
    n = b.shape[0]
    x = np.zeros(n, np.complex128)
    it, mv, rr = c_int(0), c_int(0), c_double(0)
    st = lib().orc_gmres_dense(n, _p(A.view(np.float64)), _p(b.view(np.float64)), tol, max_iter,
                               restart, _p(x.view(np.float64)), ctypes.byref(it),
                               ctypes.byref(mv), ctypes.byref(rr), nthreads)
    return GmresResult(x, st, it.value, mv.value, rr.value)


def gmres_onthefly(pos, alpha, b, k, use_fcd=False, cell_size=3.0, lattice=None,
                   k_bloch=(0, 0, 0), substrate=None, tol=1e-6, max_iter=1000, nthreads=0):
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    b = np.ascontiguousarray(np.asarray(b, np.complex128))
    x = np.zeros(3 * n, np.complex128)
    it, mv, rr = c_int(0), c_int(0), c_double(0)
    ls, ss = _lat(lattice), _sub(substrate)
    st = lib().orc_gmres_onthefly(n, _p(pos), _p(a.view(np.float64)), _p(b.view(np.float64)), k,
                                  int(use_fcd), cell_size, _ref(ls), _p(_vec(k_bloch)), _ref(ss),
                                  tol, max_iter, _p(x.view(np.float64)), ctypes.byref(it),
                                  ctypes.byref(mv), ctypes.byref(rr), nthreads)
    return GmresResult(x, st, it.value, mv.value, rr.value)


def lu_solve(A, b):
    A = np.ascontiguousarray(np.asarray(A, np.complex128))
    b = np.ascontiguousarray(np.asarray(b, np.complex128))
    x = np.zeros_like(b)
    if lib().orc_lu_solve(b.shape[0], _p(A.view(np.float64)), _p(b.view(np.float64)),
                          _p(x.view(np.float64))) != 0:
        raise ValueError("singular matrix")
    return x


def cross_sections(pos, alpha, moments, k, direction=(0, 0, 1), polarisation=(1, 0, 0),
                   amplitude=1.0):
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    m = np.ascontiguousarray(np.asarray(moments, np.complex128).reshape(3 * n))
    out = np.zeros(3)
    lib().orc_cross_sections(n, _p(pos), _p(a.view(np.float64)), _p(m.view(np.float64)), k,
                             _p(_vec(direction)), _p(_vec(polarisation)), amplitude, _p(out))
    return out


def rrcm(volume, eps, eps_m, k, radiative=True):
    out = np.zeros(2)
    eps = complex(eps)
    lib().orc_rrcm(volume, eps.real, eps.imag, eps_m, k, int(radiative), _p(out))
    return complex(out[0], out[1])


def ellipsoid_tensor(volume, depol, eps, eps_m, k, rot):
    out = np.zeros(9, np.complex128)
    eps = complex(eps)
    lib().orc_ellipsoid_tensor(volume, _p(_vec(depol)), eps.real, eps.imag, eps_m, k,
                               _p(_vec(rot)), _p(out.view(np.float64)))
    return out.reshape(3, 3)


def fresnel(eps_sub, eps_env, retarded=True):
    out = np.zeros(2)
    e = complex(eps_sub)
    lib().orc_fresnel(e.real, e.imag, eps_env, int(retarded), _p(out))
    return complex(out[0], out[1])


def spline(xs, ys):
    xs, ys = _vec(xs), _vec(ys)
    y2 = np.zeros_like(xs)
    lib().orc_spline_build(len(xs), _p(xs), _p(ys), _p(y2))

    def ev(x):
        return lib().orc_spline_eval(len(xs), _p(xs), _p(ys), _p(y2), float(x))

    return ev


def field_at_points(pos, moments, k, obs, direction=(0, 0, 1), polarisation=(1, 0, 0),
                    amplitude=1.0):
    """fields.rs:18-49 at every row of obs: (M, 3) complex."""
    pos = _vec(pos).reshape(-1, 3)
    obs = _vec(obs).reshape(-1, 3)
    mom = np.ascontiguousarray(np.asarray(moments, np.complex128).reshape(-1))
    out = np.zeros(3 * obs.shape[0], np.complex128)
    lib().orc_field_at_points(pos.shape[0], _p(pos), _p(mom.view(np.float64)), k,
                              _p(_vec(direction)), _p(_vec(polarisation)), amplitude,
                              obs.shape[0], _p(obs), _p(out.view(np.float64)))
    return out.reshape(-1, 3)


def near_field_plane(centre, normal, half_width, half_height, nx, ny):
    """Grid of compute_near_field_map (fields.rs:52-139): positions (nx*ny, 3), extent."""
    pos = np.zeros(3 * nx * ny)
    ext = np.zeros(4)
    lib().orc_near_field_plane(_p(_vec(centre)), _p(_vec(normal)), half_width, half_height,
                               nx, ny, _p(pos), _p(ext))
    return pos.reshape(-1, 3), ext


def far_field(pos, moments, k, n_theta, n_phi):
    """compute_far_field (fields.rs:147-221): theta, phi, intensity (n_theta*n_phi)."""
    pos = _vec(pos).reshape(-1, 3)
    mom = np.ascontiguousarray(np.asarray(moments, np.complex128).reshape(-1))
    m = n_theta * n_phi
    th, ph, it = np.zeros(m), np.zeros(m), np.zeros(m)
    lib().orc_far_field(pos.shape[0], _p(pos), _p(mom.view(np.float64)), k, n_theta, n_phi,
                        _p(th), _p(ph), _p(it))
    return th, ph, it


def harmonic_sources(order, local_fields, chi):
    """compute_shg_sources / compute_thg_sources (nonlinear.rs): (N, 3) complex.
    chi: one tensor (27 or 81 complex) or N of them."""
    e = np.ascontiguousarray(np.asarray(local_fields, np.complex128).reshape(-1))
    n = e.size // 3
    nc = 27 if order == 2 else 81
    t = np.ascontiguousarray(np.asarray(chi, np.complex128).reshape(-1, nc))
    out = np.zeros(3 * n, np.complex128)
    lib().orc_harmonic_sources(order, n, _p(e.view(np.float64)), int(t.shape[0] > 1),
                               _p(t.view(np.float64)), _p(out.view(np.float64)))
    return out.reshape(-1, 3)


def circular_dichroism(mom_x, mom_y, k):
    mx = np.ascontiguousarray(np.asarray(mom_x, np.complex128).reshape(-1))
    my = np.ascontiguousarray(np.asarray(mom_y, np.complex128).reshape(-1))
    return lib().orc_circular_dichroism(mx.shape[0] // 3, _p(mx.view(np.float64)),
                                        _p(my.view(np.float64)), k)


def wgsl_assemble_f32(pos, inv_alpha, k):
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    ia = np.ascontiguousarray(np.asarray(inv_alpha, np.complex128).reshape(n, 9))
    A = np.zeros((3 * n, 3 * n), np.complex64)
    lib().orc_wgsl_assemble_f32(n, _p(pos), _p(ia.view(np.float64)), k,
                                A.view(np.float32).ctypes.data_as(POINTER(c_float)))
    return A


def max_threads():
    return lib().orc_max_threads()


def grad_cext(pos, alpha, k, use_fcd=False, cell_size=3.0, direction=(0, 0, 1),
              polarisation=(1, 0, 0), amplitude=1.0, dinv_alpha_deps=None, nthreads=0):
    """(C_ext, dC_ext/dr (N,3), dC_ext/d(Re,Im) eps (N,2), moments) by dense LU and
    the oracle's own tensor-derivative restatement (no reference counterpart)."""
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    pol = np.asarray(polarisation, np.complex128).reshape(3)
    pol6 = np.ascontiguousarray(np.stack([pol.real, pol.imag], axis=1).ravel())
    dinv = None
    if dinv_alpha_deps is not None:
        dinv = _alpha_arr(dinv_alpha_deps, n)
    c_ext = c_double(0.0)
    gr = np.zeros(3 * n)
    ge = np.zeros(2 * n)
    mom = np.zeros(3 * n, np.complex128)
    st = lib().orc_grad_cext(n, _p(pos), _p(a.view(np.float64)), float(k), int(bool(use_fcd)),
                             float(cell_size), _p(_vec(direction)), _p(pol6), float(amplitude),
                             None if dinv is None else dinv.ctypes.data, ctypes.byref(c_ext),
                             _p(gr), _p(ge), _p(mom.view(np.float64)), nthreads)
    if st:
        raise RuntimeError(f"orc_grad_cext failed ({st})")
    return c_ext.value, gr.reshape(n, 3), ge.reshape(n, 2), mom


# --- Sommerfeld reflected Green's tensor (sommerfeld.rs) ---------------------
# `somm` is any object with z_interface, wavelength_nm, eps_sub (complex) and
# eps_env (SubstrateRuntime::Sommerfeld, substrate.rs:109-113).

def somm_bessel(order, x):
    """J0 / J1 / J2 of sommerfeld.rs:103-153 (the module's own coefficients)."""
    return lib().orc_somm_bessel(int(order), float(x))


def sommerfeld_tensor(somm, ri, rj, nthreads=0):
    """SommerfeldGreens::evaluate (sommerfeld.rs:254-300) for pairs of points
    (ri, rj: (P, 3) or (3,)); returns (P, 3, 3) complex (or (3, 3))."""
    ri = _vec(ri).reshape(-1, 3)
    rj = _vec(rj).reshape(-1, 3)
    out = np.zeros((ri.shape[0], 3, 3), np.complex128)
    s = _somm(somm)
    lib().orc_sommerfeld_tensor(ctypes.byref(s), ri.shape[0], _p(ri), _p(rj),
                                _p(out.view(np.float64)), nthreads)
    return out if out.shape[0] != 1 else out[0]


def assemble_sommerfeld(pos, alpha, k, somm, use_fcd=False, cell_size=3.0, lattice=None,
                        k_bloch=(0, 0, 0), nthreads=0):
    """assemble_interaction_matrix with the Sommerfeld substrate runtime."""
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    A = np.zeros((3 * n, 3 * n), np.complex128)
    s = _somm(somm)
    rc = lib().orc_assemble_sommerfeld(n, _p(pos), _p(a.view(np.float64)), k, int(use_fcd),
                                       cell_size, _ref(_lat(lattice)), _p(_vec(k_bloch)),
                                       ctypes.byref(s), _p(A.view(np.float64)), nthreads)
    if rc != 0:
        raise ValueError("singular polarisability")
    return A


def matvec_sommerfeld(pos, alpha, x, k, somm, use_fcd=False, cell_size=3.0, lattice=None,
                      k_bloch=(0, 0, 0), nthreads=0):
    """matvec_on_the_fly with the Sommerfeld substrate runtime."""
    pos = _vec(pos).reshape(-1, 3)
    n = pos.shape[0]
    a = _alpha_arr(alpha, n)
    x = np.ascontiguousarray(np.asarray(x, np.complex128))
    y = np.zeros(3 * n, np.complex128)
    s = _somm(somm)
    rc = lib().orc_matvec_sommerfeld(n, _p(pos), _p(a.view(np.float64)), _p(x.view(np.float64)),
                                     k, int(use_fcd), cell_size, _ref(_lat(lattice)),
                                     _p(_vec(k_bloch)), ctypes.byref(s), _p(y.view(np.float64)),
                                     nthreads)
    if rc != 0:
        raise ValueError("singular polarisability")
    return y
