"""Berger-Oliger refinement: radially nested 2:1 levels advanced together.

The reference's mesh_refinement_lib (MoL/mesh_refinement_lib.f90:76-179) builds
one uniform level per rank; this module drives the hierarchy of kg_hier_* (the
transfer kernels are in csrc/kg_refine.cu, the level stepping in kg_capi.cu).

    bo = BergerOliger(Nx, Ny, Nz, xmin, xmax, CFL, r_fine=(20.0, 10.0), m=0.3)
    bo.levels[0].u = u0           # coarse state; finer levels are set the same way
    bo.rk4(100)                   # 100 coarse steps; level l takes 2^l steps each
    bo.levels[2].u                # finest level's state (a ScalarField view)

Level l covers [xmin, ~r_fine[l-1]] with dx_0 / 2^l and dt_0 / 2^l; all levels
share the theta/phi grid and the metric form.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .lines_method import ScalarField, _BCS, _METRICS


class _LevelView(ScalarField):
    """A ScalarField on a level handle owned by the hierarchy (close() is a no-op)."""

    def __init__(self, handle, params, metric, bc, m, a, M_bh, n_det, l_max):
        self._lib = capi.load()
        self._h = handle
        self.params = params
        self.Nx, self.Ny, self.Nz, self.g_pts = params.Nx, params.Ny, params.Nz, params.g_pts
        self.metric, self.boundary_type_rmax = metric, bc
        self.m, self.a, self.M_bh = m, a, M_bh
        self.NI, self.NJ, self.NK = self.Nx + 2 * self.g_pts + 1, self.Ny + 2 * self.g_pts + 1, self.Nz + 1
        self.n_det = max(2, n_det)
        self.l_max = l_max
        self.Mass_scalar = 0.0
        self.momentum = np.zeros((self.n_det, 3))
        self.alm = np.zeros((self.n_det, 2 * self.l_max + 1, self.l_max + 1), np.complex128)

    def close(self):
        self._h = None


class BergerOliger:
    def __init__(self, Nx, Ny, Nz, xmin, xmax, CFL, r_fine=(20.0,), m=0.0, metric="Kerr_Schild", a=0.0,
                 M_bh=1.0, boundary_type_rmax="outflow", n_det=5, l_max=10, dt=None, device=-1):
        self._lib = capi.load()
        base = capi.KgParams(Nx, Ny, Nz, 2, xmin, xmax, 0.0, 1.0, CFL, a, M_bh, m, _METRICS[metric],
                             _BCS[boundary_type_rmax], n_det, l_max, float(dt) if dt else 0.0, 0.0)
        radii = (C.c_double * max(1, len(r_fine)))(*r_fine) if r_fine else (C.c_double * 1)(0.0)
        h = C.c_void_p()
        rc = self._lib.kg_hier_create(C.byref(base), 1 + len(r_fine), radii, device, C.byref(h))
        if rc != capi.KG_OK:
            raise capi.KgError(rc, "kg_hier_create failed")
        self._H = h
        self.levels = []
        n = self._lib.kg_hier_levels(self._H)
        for l in range(n):
            lh = C.c_void_p(self._lib.kg_hier_level(self._H, l))
            sc = (C.c_double * 9)()
            self._lib.kg_get_scalars(lh, sc)
            # the level's own grid integers and radius come from its handle
            p = capi.KgParams(base.Nx, Ny, Nz, 2, xmin, xmax, 0.0, 1.0, CFL, a, M_bh, m, _METRICS[metric],
                              _BCS[boundary_type_rmax], n_det, l_max, 0.0, 0.0)
            if l > 0:
                p.Nx = int(round((sc[6] - sc[5]) / sc[0]))
                p.xmax = sc[6]
            self.levels.append(_LevelView(lh, p, metric, boundary_type_rmax, m, a, M_bh, n_det, l_max))

    def _ck(self, rc):
        if rc != capi.KG_OK:
            raise capi.KgError(rc, self._lib.kg_hier_last_error(self._H).decode())

    def rk4(self, nsteps=1):
        """nsteps coarse RK4 steps (level l takes 2^l steps per coarse step)"""
        self._ck(self._lib.kg_hier_rk4(self._H, int(nsteps)))

    def rk3(self, nsteps=1):
        """nsteps coarse SSP-RK3 steps (level l takes 2^l steps per coarse step)"""
        self._ck(self._lib.kg_hier_rk3(self._H, int(nsteps)))

    def pirk2(self, nsteps=1):
        """nsteps coarse PIRK2 steps (level l takes 2^l steps per coarse step)"""
        self._ck(self._lib.kg_hier_pirk2(self._H, int(nsteps)))

    def pirk3(self, nsteps=1):
        """nsteps coarse PIRK3 steps (level l takes 2^l steps per coarse step)"""
        self._ck(self._lib.kg_hier_pirk3(self._H, int(nsteps)))

    def synchronize(self):
        self._ck(self._lib.kg_hier_synchronize(self._H))

    def close(self):
        if getattr(self, "_H", None):
            for lv in self.levels:
                lv.close()
            self._lib.kg_hier_destroy(self._H)
            self._H = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
