"""ctypes front end of the C oracle (oracle/_build/libkg_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product never imports it.
The state is exchanged in the reference's Fortran layout
u(1:5, -g:Nx+g, -g:Ny+g, 0:Nz) complex(8), i.e. a flat complex128 array with
the variable index fastest.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libkg_oracle.so")

KERR_SCHILD, SCHW_EF = 0, 1
OUTFLOW, INFLOW = 0, 1


class OracleParams(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int), ("g_pts", C.c_int),
                ("xmin", C.c_double), ("xmax", C.c_double), ("tmin", C.c_double), ("tmax", C.c_double),
                ("CFL", C.c_double), ("a", C.c_double), ("M_bh", C.c_double), ("m", C.c_double),
                ("metric", C.c_int), ("bc_rmax", C.c_int), ("n_det", C.c_int), ("l_max", C.c_int),
                ("dt_override", C.c_double)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        P, D, I, U = C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_uint
        L.kgo_create.restype = P
        L.kgo_create.argtypes = [C.POINTER(OracleParams)]
        L.kgo_destroy.argtypes = [P]
        for name in ("kgo_set_state", "kgo_get_state", "kgo_set_stage", "kgo_get_stage",
                     "kgo_set_stage2", "kgo_get_stage2", "kgo_set_u_p", "kgo_get_scalars",
                     "kgo_get_metric", "kgo_density", "kgo_currents_adm"):
            getattr(L, name).argtypes = [P, D]
        for name in ("kgo_pirk2", "kgo_pirk3", "kgo_rk3", "kgo_rk4"):
            getattr(L, name).argtypes = [P, I]
        L.kgo_rhs.argtypes = [P, D, D, U]
        L.kgo_boundary_faces.argtypes = [P, U]
        L.kgo_set_time.argtypes = [P, C.c_double]
        L.kgo_set_dt.argtypes = [P, C.c_double]
        L.kgo_get_4metric.argtypes = [P, D, D]
        L.kgo_validate_inverse_metric.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.kgo_validate_inverse_metric.restype = I
        L.kgo_mass.argtypes = [P]
        L.kgo_mass.restype = C.c_double
        L.kgo_integrate_real.argtypes = [P, D]
        L.kgo_integrate_real.restype = C.c_double
        L.kgo_currents_detectors.argtypes = [P, D]
        L.kgo_proyector_detectors.argtypes = [P, I, D]
        L.kgo_project_all_shells.argtypes = [P, I, D]
        L.kgo_project_shells.argtypes = [P, I, I, C.POINTER(C.c_int), D]
        L.kgo_set_scheme.argtypes = [P, I, C.c_double]
        L.kgo_set_scheme.restype = I
        L.kgo_boundary_cfg.argtypes = [P]
        L.kgo_sph_jl.argtypes = [I, C.c_double]
        L.kgo_sph_jl.restype = C.c_double
        L.kgo_sph_jl_zeros.argtypes = [I, I, D]
        L.kgo_bessel_basis.argtypes = [P, I, I, D, D]
        L.kgo_sph_ft_radial.argtypes = [P, I, I, D]
        L.kgo_sph_harmonics.argtypes = [P, I, D]
        L.kgo_project_sh.argtypes = [P, D, D, I, D]
        L.kgo_domain_to_sph_shell.argtypes = [P, D, I, D]
        L.kgo_get_detectors.argtypes = [P, D, C.POINTER(C.c_int)]
        L.kgo_set_threads.argtypes = [I]
        L.kgo_max_threads.restype = I
        L.kgo_npts.argtypes = [P]
        L.kgo_npts.restype = C.c_size_t
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """Mirror of the reference `scalar_field` object on the CPU (nproc = 1)."""

    def __init__(self, Nx, Ny, Nz, xmin, xmax, CFL=0.25, m=0.0, a=0.0, M_bh=1.0,
                 metric=KERR_SCHILD, bc_rmax=OUTFLOW, tmin=0.0, tmax=1.0, n_det=5,
                 l_max=10, dt_override=0.0):
        self.p = OracleParams(Nx, Ny, Nz, 2, xmin, xmax, tmin, tmax, CFL, a, M_bh, m,
                              metric, bc_rmax, n_det, l_max, dt_override)
        self.h = lib().kgo_create(C.byref(self.p))
        if not self.h:
            raise ValueError("oracle rejected the grid parameters")
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.NI, self.NJ, self.NK = Nx + 5, Ny + 5, Nz + 1
        self.npts = self.NI * self.NJ * self.NK
        self.n_det = max(2, n_det)

    def close(self):
        if getattr(self, "h", None):
            lib().kgo_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # state in Fortran order: complex128, shape (NK, NJ, NI, 5) in C order
    def shape(self):
        return (self.NK, self.NJ, self.NI, 5)

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.complex128)
        assert u.size == 5 * self.npts
        lib().kgo_set_state(self.h, _dp(u.view(np.float64)))

    def get_state(self):
        out = np.zeros(self.shape(), np.complex128)
        lib().kgo_get_state(self.h, _dp(out.view(np.float64)))
        return out

    def set_stage(self, u):
        u = np.ascontiguousarray(u, dtype=np.complex128)
        lib().kgo_set_stage(self.h, _dp(u.view(np.float64)))

    def get_stage(self):
        out = np.zeros(self.shape(), np.complex128)
        lib().kgo_get_stage(self.h, _dp(out.view(np.float64)))
        return out

    def get_stage2(self):
        out = np.zeros(self.shape(), np.complex128)
        lib().kgo_get_stage2(self.h, _dp(out.view(np.float64)))
        return out

    def set_u_p(self, u):
        u = np.ascontiguousarray(u, dtype=np.complex128)
        lib().kgo_set_u_p(self.h, _dp(u.view(np.float64)))

    def pirk2(self, n=1):
        lib().kgo_pirk2(self.h, n)

    def pirk3(self, n=1):
        lib().kgo_pirk3(self.h, n)

    def rk3(self, n=1):
        lib().kgo_rk3(self.h, n)

    def rk4(self, n=1):
        lib().kgo_rk4(self.h, n)

    def step(self, method, n=1):
        getattr(self, method)(n)

    def rhs(self, vars_, mask=31, rhs_init=None):
        v = np.ascontiguousarray(vars_, dtype=np.complex128)
        out = np.zeros(self.shape(), np.complex128) if rhs_init is None else np.array(rhs_init, np.complex128)
        lib().kgo_rhs(self.h, _dp(v.view(np.float64)), _dp(out.view(np.float64)), mask)
        return out

    def boundary(self, mask=63):
        lib().kgo_boundary_faces(self.h, mask)

    def scalars(self):
        out = np.zeros(8)
        lib().kgo_get_scalars(self.h, _dp(out))
        return dict(dx=out[0], dy=out[1], dz=out[2], dt=out[3], t=out[4], xmin=out[5], xmax=out[6], Nt=int(out[7]))

    def set_time(self, t):
        lib().kgo_set_time(self.h, t)

    def set_dt(self, dt):
        lib().kgo_set_dt(self.h, dt)

    def metric(self):
        out = np.zeros((8, self.NJ, self.NI))
        lib().kgo_get_metric(self.h, _dp(out))
        return out

    def metric4(self):
        gdn = np.zeros((4, 4, self.NJ, self.NI))
        gup = np.zeros((4, 4, self.NJ, self.NI))
        lib().kgo_get_4metric(self.h, _dp(gdn), _dp(gup))
        return gdn, gup

    def validate_inverse_metric(self):
        e4, e3 = C.c_int(0), C.c_int(0)
        lib().kgo_validate_inverse_metric(self.h, C.byref(e4), C.byref(e3))
        return e4.value, e3.value

    def density(self):
        out = np.zeros((self.NK, self.NJ, self.NI))
        lib().kgo_density(self.h, _dp(out))
        return out

    def mass(self):
        return lib().kgo_mass(self.h)

    def currents_detectors(self):
        out = np.zeros((self.n_det, 3))
        lib().kgo_currents_detectors(self.h, _dp(out))
        return out

    def proyector_detectors(self, L):
        out = np.zeros((self.n_det, 2 * L + 1, L + 1), np.complex128)
        lib().kgo_proyector_detectors(self.h, L, _dp(out.view(np.float64)))
        return out

    def project_all_shells(self, L):
        """a_lm on every vertex shell: (Nx, 2L+1, L+1) complex"""
        out = np.zeros((self.Nx, 2 * L + 1, L + 1), np.complex128)
        lib().kgo_project_all_shells(self.h, L, _dp(out.view(np.float64)))
        return out

    def project_shells(self, L, shells):
        """a_lm on the listed vertex shells (1-based), equal to the same rows of
        project_all_shells; for large spheres (no stored Y_lm table, threaded)"""
        iv = np.ascontiguousarray(shells, dtype=np.int32)
        out = np.zeros((len(iv), 2 * L + 1, L + 1), np.complex128)
        lib().kgo_project_shells(self.h, L, len(iv), iv.ctypes.data_as(C.POINTER(C.c_int)),
                                 _dp(out.view(np.float64)))
        return out

    def set_scheme(self, scheme, ko_eps=0.02):
        """0: the reference's second-order method; 1: the configured fourth-order
        method with sixth-order Kreiss-Oliger dissipation and a Sommerfeld outer
        boundary (RK4 only)"""
        if lib().kgo_set_scheme(self.h, int(scheme), float(ko_eps)) != 0:
            raise ValueError("scheme 1 needs the Kerr-Schild metric form")

    def boundary_cfg(self):
        lib().kgo_boundary_cfg(self.h)

    def bessel_basis(self, L, Nk):
        """(k_values (Nk, L+1), j_basis (Nx, Nk, L+1))"""
        k = np.zeros((Nk, L + 1))
        jb = np.zeros((self.Nx, Nk, L + 1))
        lib().kgo_bessel_basis(self.h, L, Nk, _dp(k), _dp(jb))
        return k, jb

    def sph_ft_radial(self, L, Nk):
        """(2L+1, L+1, Nk) complex, [m+L, l, n-1]"""
        out = np.zeros((2 * L + 1, L + 1, Nk), np.complex128)
        lib().kgo_sph_ft_radial(self.h, L, Nk, _dp(out.view(np.float64)))
        return out

    def sph_harmonics(self, L):
        out = np.zeros((self.Nz, self.Ny, 2 * L + 1, L + 1), np.complex128)
        lib().kgo_sph_harmonics(self.h, L, _dp(out.view(np.float64)))
        return out

    def detectors(self):
        r = np.zeros(self.n_det)
        idx = np.zeros(self.n_det, np.int32)
        lib().kgo_get_detectors(self.h, _dp(r), idx.ctypes.data_as(C.POINTER(C.c_int)))
        return r, idx


def sph_jl(l, x):
    return lib().kgo_sph_jl(l, float(x))


def sph_jl_zeros(L, Nk):
    """(L+1, Nk): n-th positive zero of j_l"""
    z = np.zeros((L + 1, Nk))
    lib().kgo_sph_jl_zeros(L, Nk, _dp(z))
    return z


def set_threads(n):
    lib().kgo_set_threads(int(n))


def max_threads():
    return lib().kgo_max_threads()
