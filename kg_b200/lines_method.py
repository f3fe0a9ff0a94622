"""Python mirror of the reference's `lines_method` / `scalar_field` objects
(MoL/lines_method_lib.f90, MoL/diagnostic_lib.f90) over the C ABI.

Method names, argument meaning and call order follow the Fortran type-bound
procedures, so a driver written like main/evolve.f90 reads the same:

    mol = ScalarField(Nx=256, Ny=33, Nz=65, xmin=1.8, xmax=60.0, CFL=0.25, ...)
    mol.u = u0                      # MoL%u = ...
    for l in range(1, mol.Nt + 1):
        mol.pirk2()                 # call MoL%pirk2()
        mol.diagnostic(l)           # call MoL%diagnostic(l)

Every operation runs on the GPU through libkg_b200.so; state arrays cross to
the host only when the `u` / `u_stage` properties are read or written.
Arrays use the reference layout u(1:5, -g:Nx+g, -g:Ny+g, 0:Nz) complex(8),
returned here as numpy complex128 of C shape (Nz+1, Ny+2g+1, Nx+2g+1, 5).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi

_METRICS = {"Kerr_Schild": capi.KG_KERR_SCHILD, "Schw_EF": capi.KG_SCHW_EF}
_BCS = {"outflow": capi.KG_OUTFLOW, "inflow": capi.KG_INFLOW}


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class LinesMethod:
    """lines_method (MoL/lines_method_lib.f90:19-44) on one GPU."""

    nvars = 5

    def __init__(self, Nx, Ny, Nz, xmin, xmax, CFL, tmin=0.0, tmax=1.0, g_pts=2,
                 boundary_type_rmax="outflow", metric="Kerr_Schild", a=0.0, M_bh=1.0, m=0.0,
                 n_det=5, l_max=10, dt=None, save=0.0, device=-1):
        if metric not in _METRICS:
            raise ValueError(f"Metric: {metric} not implemented yet; try with: Kerr_Schild or Schw_EF")
        if boundary_type_rmax not in _BCS:
            raise ValueError("This boundary condition type for r_max is not implemented yet; try with: outflow or inflow")
        self._lib = capi.load()
        self.params = capi.KgParams(Nx, Ny, Nz, g_pts, xmin, xmax, tmin, tmax, CFL, a, M_bh, m,
                                    _METRICS[metric], _BCS[boundary_type_rmax], n_det, l_max,
                                    float(dt) if dt else 0.0, float(save))
        h = C.c_void_p()
        rc = self._lib.kg_create(C.byref(self.params), device, C.byref(h))
        if rc != capi.KG_OK:
            raise capi.KgError(rc, "kg_create failed")
        self._h = h
        self.Nx, self.Ny, self.Nz, self.g_pts = Nx, Ny, Nz, g_pts
        self.metric, self.boundary_type_rmax = metric, boundary_type_rmax
        self.m, self.a, self.M_bh = m, a, M_bh
        self.NI, self.NJ, self.NK = Nx + 2 * g_pts + 1, Ny + 2 * g_pts + 1, Nz + 1
        self.n_det = max(2, n_det)
        self.l_max = l_max

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            self._lib.kg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        capi.check(self._h, rc)

    @property
    def handle(self):
        return self._h

    # -- scalars
    def _scalars(self):
        out = np.zeros(9)
        self._ck(self._lib.kg_get_scalars(self._h, _dp(out)))
        return out

    dx = property(lambda s: s._scalars()[0])
    dy = property(lambda s: s._scalars()[1])
    dz = property(lambda s: s._scalars()[2])
    dt = property(lambda s: s._scalars()[3], lambda s, v: s._ck(s._lib.kg_set_dt(s._h, float(v))))
    t = property(lambda s: s._scalars()[4], lambda s, v: s._ck(s._lib.kg_set_time(s._h, float(v))))
    Nt = property(lambda s: int(s._scalars()[7]))
    r_max = property(lambda s: s._scalars()[8])

    @property
    def device_bytes(self):
        return int(self._lib.kg_device_bytes(self._h))

    # -- state arrays
    def state_shape(self):
        return (self.NK, self.NJ, self.NI, 5)

    def _get(self, which):
        out = np.zeros(self.state_shape(), np.complex128)
        self._ck(self._lib.kg_get_state(self._h, which, _dp(out.view(np.float64))))
        return out

    def _set(self, which, u):
        u = np.ascontiguousarray(u, dtype=np.complex128)
        if u.size != 5 * self.NI * self.NJ * self.NK:
            raise ValueError("state has the wrong size")
        self._ck(self._lib.kg_set_state(self._h, which, _dp(u.view(np.float64))))

    u = property(lambda s: s._get(0), lambda s, v: s._set(0, v))
    u_stage = property(lambda s: s._get(1), lambda s, v: s._set(1, v))
    u_stage_2 = property(lambda s: s._get(2), lambda s, v: s._set(2, v))
    u_p = property(lambda s: s._get(3), lambda s, v: s._set(3, v))

    # -- steppers (MoL/lines_method_lib.f90:211-474)
    def pirk2(self, nsteps=1):
        self._ck(self._lib.kg_pirk2(self._h, nsteps))

    def pirk3(self, nsteps=1):
        self._ck(self._lib.kg_pirk3(self._h, nsteps))

    def rk3(self, rhs=None, nsteps=1):
        """rk3 with the built-in rhs (the type-bound rhs_* applied to u)."""
        if rhs is not None:
            raise NotImplementedError("a host rhs callback cannot run inside the device stepper")
        self._ck(self._lib.kg_rk3(self._h, nsteps))

    def rk4(self, rhs=None, nsteps=1):
        if rhs is not None:
            raise NotImplementedError("a host rhs callback cannot run inside the device stepper")
        self._ck(self._lib.kg_rk4(self._h, nsteps))

    @property
    def precision(self):
        """'fp64' (default) or 'mixed' (rk4: FP32 stencil RHS, FP64 state update)"""
        return "mixed" if self._lib.kg_get_precision(self._h) == 1 else "fp64"

    @precision.setter
    def precision(self, mode):
        if mode not in ("fp64", "mixed"):
            raise ValueError("precision is 'fp64' or 'mixed'")
        self._ck(self._lib.kg_set_precision(self._h, 1 if mode == "mixed" else 0))

    def check_point(self, path):
        """binary checkpoint of u, the stage arrays and the clock (kg_save_checkpoint)"""
        self._ck(self._lib.kg_save_checkpoint(self._h, str(path).encode()))

    def read_from_check_point(self, path):
        """resume from kg_save_checkpoint's file (same grid)"""
        self._ck(self._lib.kg_load_checkpoint(self._h, str(path).encode()))

    def set_scheme(self, scheme, ko_eps=0.02):
        """'reference' (second order, default) or 'configured' (fourth-order
        differences, sixth-order Kreiss-Oliger dissipation of strength ko_eps,
        Sommerfeld outer plane, parity-correct pole ghosts; rk4 only)"""
        if scheme not in ("reference", "configured"):
            raise ValueError("scheme is 'reference' or 'configured'")
        self._ck(self._lib.kg_set_scheme(self._h, 0 if scheme == "reference" else 1, float(ko_eps)))

    def fill_ghosts_configured(self):
        """apply the configured method's ghost fills to u"""
        self._ck(self._lib.kg_fill_ghosts_cfg(self._h))

    def synchronize(self):
        """Wait for the handle's queued device work (steppers return asynchronously)."""
        self._ck(self._lib.kg_synchronize(self._h))

    # -- RHS (MoL/lines_method_lib.f90:671-753)
    def _rhs(self, mask, vars_):
        v = np.ascontiguousarray(vars_, dtype=np.complex128)
        out = np.zeros(self.state_shape(), np.complex128)
        self._ck(self._lib.kg_rhs(self._h, _dp(v.view(np.float64)), _dp(out.view(np.float64)), mask))
        return out

    def rhs_phi(self, vars_):
        return self._rhs(1, vars_)[..., 0]

    def rhs_psi1(self, vars_):
        return self._rhs(2, vars_)[..., 1]

    def rhs_psi2(self, vars_):
        return self._rhs(4, vars_)[..., 2]

    def rhs_psi3(self, vars_):
        return self._rhs(8, vars_)[..., 3]

    def rhs_pi(self, vars_):
        return self._rhs(16, vars_)[..., 4]

    def rhs_all(self, vars_):
        return self._rhs(31, vars_)

    # -- boundaries (MoL/lines_method_lib.f90:475-597)
    def boundary_xL(self):
        self._ck(self._lib.kg_boundary(self._h, 1))

    def boundary_xR(self):
        self._ck(self._lib.kg_boundary(self._h, 2))

    def boundary_yL(self):
        self._ck(self._lib.kg_boundary(self._h, 4))

    def boundary_yR(self):
        self._ck(self._lib.kg_boundary(self._h, 8))

    def boundary_zL(self):
        self._ck(self._lib.kg_boundary(self._h, 16))

    def boundary_zR(self):
        self._ck(self._lib.kg_boundary(self._h, 32))

    def boundary(self):
        self._ck(self._lib.kg_boundary(self._h, 63))

    def send_recv_xL(self):
        self._ck(self._lib.kg_send_recv(self._h))

    send_recv_xR = send_recv_xL

    # -- geometry (MoL/geometry.f90)
    def metric_tables(self):
        out = np.zeros((8, self.NJ, self.NI))
        self._ck(self._lib.kg_get_metric(self._h, _dp(out)))
        return out

    def set_metric_tables(self, tables):
        t = np.ascontiguousarray(tables, dtype=np.float64)
        self._ck(self._lib.kg_set_metric(self._h, _dp(t)))

    def validate_inverse_metric(self):
        e4, e3 = C.c_int(0), C.c_int(0)
        self._ck(self._lib.kg_validate_inverse_metric(self._h, C.byref(e4), C.byref(e3)))
        return e4.value, e3.value


class ScalarField(LinesMethod):
    """scalar_field (MoL/diagnostic_lib.f90:8-32): diagnostics on top of the stepper."""

    def __init__(self, *args, **kw):
        super().__init__(*args, **kw)
        self.Mass_scalar = 0.0
        self.momentum = np.zeros((self.n_det, 3))
        self.alm = np.zeros((self.n_det, 2 * self.l_max + 1, self.l_max + 1), np.complex128)

    def density(self):
        self._ck(self._lib.kg_density(self._h))

    @property
    def rho(self):
        out = np.zeros((self.NK, self.NJ, self.NI))
        self._ck(self._lib.kg_get_density(self._h, _dp(out)))
        return out

    def mass_scalar(self):
        out = C.c_double(0.0)
        self._ck(self._lib.kg_mass_scalar(self._h, C.byref(out)))
        return out.value

    def currents_detectors(self):
        self._ck(self._lib.kg_currents_detectors(self._h, _dp(self.momentum)))
        return self.momentum

    def proyector_detectors(self):
        self._ck(self._lib.kg_proyector_detectors(self._h, _dp(self.alm.view(np.float64))))
        return self.alm

    def diagnostic(self, index):
        out = C.c_double(0.0)
        self._ck(self._lib.kg_diagnostic(self._h, index, C.byref(out)))
        self.Mass_scalar = out.value
        return self.Mass_scalar

    def set_detectors(self, radii):
        r = np.ascontiguousarray(radii, dtype=np.float64)
        self._ck(self._lib.kg_set_detectors(self._h, len(r), _dp(r)))
        self.n_det = len(r)
        self.momentum = np.zeros((self.n_det, 3))
        self.alm = np.zeros((self.n_det, 2 * self.l_max + 1, self.l_max + 1), np.complex128)

    def project_all_shells(self, L, precision=1):
        """a_lm (l <= L) of phi on every vertex shell: array (Nx, 2L+1, L+1) complex.
        precision 1: split-BF16 tensor-core GEMM (FP32 accumulation); 0: FP64."""
        out = np.zeros((self.Nx, 2 * L + 1, L + 1), np.complex128)
        self._ck(self._lib.kg_project_all_shells(self._h, L, precision, _dp(out.view(np.float64))))
        return out

    def bessel_basis(self, L, Nk):
        """(k_values (Nk, L+1), j_basis (Nx, Nk, L+1)): generate_full_bessel_basis"""
        k = np.zeros((Nk, L + 1))
        jb = np.zeros((self.Nx, Nk, L + 1))
        self._ck(self._lib.kg_bessel_basis(self._h, L, Nk, _dp(k), _dp(jb)))
        return k, jb

    def sph_ft_radial(self, L, Nk, precision=0):
        """SphFT_discrete_radial of phi: array (2L+1, L+1, Nk) complex, [m+L, l, n-1]"""
        out = np.zeros((2 * L + 1, L + 1, Nk), np.complex128)
        self._ck(self._lib.kg_sph_ft_radial(self._h, L, Nk, precision, _dp(out.view(np.float64))))
        return out

    def detectors(self):
        r = np.zeros(self.n_det)
        idx = np.zeros(self.n_det, np.int32)
        self._ck(self._lib.kg_get_detectors(self._h, _dp(r), idx.ctypes.data_as(C.POINTER(C.c_int))))
        return r, idx

    def sph_harmonics(self, L=None):
        L = self.l_max if L is None else L
        out = np.zeros((self.Nz, self.Ny, 2 * L + 1, L + 1), np.complex128)
        self._ck(self._lib.kg_sph_harmonics(self._h, L, _dp(out.view(np.float64))))
        return out
