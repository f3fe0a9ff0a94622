"""Whole-array numpy restatement of the KG method-of-lines path.

TEST INFRASTRUCTURE ONLY: imported by tests/ to cross-check the C oracle
(oracle/kg_oracle.c) on small grids.  It is an independent transcription of
the same Fortran statements, written in the array syntax the reference uses
(every operator returns a full temporary), so that a transcription slip in
either restatement shows up as a mismatch.

Reference files (FlavioRosales/KG): tools/finite_differences.f90:17-44,
193-239, 310-338, 767-801; MoL/lines_method_lib.f90:211-597, 671-753;
MoL/geometry.f90:92-406; MoL/mesh_refinement_lib.f90:100-147;
MoL/diagnostic_lib.f90:101-107.

Arrays are indexed [i - iL, j - jL, k] with i = r (iL = -g), j = theta
(jL = -g), k = phi (0..Nz).  Complex-by-real products are numpy's
complex128 x float64, which agree bit for bit with the component-wise
product for finite values.
"""
from __future__ import annotations

import math
import numpy as np


class NumpyKG:
    def __init__(self, Nx, Ny, Nz, xmin, xmax, CFL, m=0.0, a=0.0, M_bh=1.0,
                 metric="Kerr_Schild", bc_rmax="outflow", tmin=0.0, tmax=1.0,
                 g=2, dt_override=0.0):
        self.Nx, self.Ny, self.Nz, self.g = Nx, Ny, Nz, g
        self.m, self.a, self.M, self.metric, self.bc = m, a, M_bh, metric, bc_rmax
        self.iL, self.iR, self.jL, self.jR, self.kL, self.kR = -g, Nx + g, -g, Ny + g, 0, Nz
        self.NI, self.NJ, self.NK = Nx + 2 * g + 1, Ny + 2 * g + 1, Nz + 1
        pi = math.acos(-1.0)
        dxr = (xmax - xmin) / 1.0
        self.xmin = xmin + 0.0 * dxr
        self.xmax = xmin + 1.0 * dxr
        self.xmax_param = xmax
        self.dx = (self.xmax - self.xmin) / float(Nx)
        self.dy = pi / float(Ny - 1)
        self.dz = 2.0 * pi / float(Nz - 1)
        i = np.arange(self.iL, self.iR + 1)
        j = np.arange(self.jL, self.jR + 1)
        self.x = self.xmin + (i + g).astype(np.float64) * self.dx
        self.y = -self.dy / 2.0 + j.astype(np.float64) * self.dy
        dxx = self.x[1] - self.x[0]
        self.dt = CFL * min(dxx, math.exp(xmin) * self.dy, math.exp(xmin) * math.sin(self.dy / 2.0) * self.dz)
        if dt_override > 0:
            self.dt = dt_override
        self.t = tmin
        self._metric()
        shape = (self.NI, self.NJ, self.NK)
        self.u = np.zeros((5,) + shape, np.complex128)
        self.u_p = np.zeros_like(self.u)
        self.u_stage = np.zeros_like(self.u)
        self.u_stage_2 = np.zeros_like(self.u)
        self.rhs_u = np.zeros_like(self.u)

    # ---- metric (MoL/geometry.f90) as 2-D (r, theta) arrays broadcast over phi
    def _metric(self):
        x = self.x[:, None] * np.ones((1, self.NJ))
        y = np.ones((self.NI, 1)) * self.y[None, :]
        M, A = self.M, self.a
        gd = np.zeros((4, 4) + x.shape)
        if self.metric == "Kerr_Schild":
            c2 = np.cos(y) ** 2
            s2 = np.sin(y) ** 2
            gd[0, 0] = -1.0 + 2.0 * M * x / (x ** 2 + A ** 2 * c2)
            gd[0, 1] = (2.0 * M * x / (x ** 2 + A ** 2 * c2))
            gd[0, 3] = -(2.0 * A * M * x * s2 / (x ** 2 + A ** 2 * c2))
            gd[1, 0] = gd[0, 1]
            gd[1, 1] = (1.0 + 2.0 * M * x / (x ** 2 + A ** 2 * c2))
            gd[1, 3] = (-(A * (1.0 + 2.0 * M * x / (x ** 2 + A ** 2 * c2)) * s2))
            gd[2, 2] = (x ** 2 + A ** 2 * c2)
            gd[3, 0] = gd[0, 3]
            gd[3, 1] = gd[1, 3]
            gd[3, 3] = ((A ** 2 + x ** 2) ** 2 - A ** 2 * (-(2.0 * M * x) + A ** 2 + x ** 2) * s2) * s2 / (x ** 2 + A ** 2 * c2)
        else:
            gd[0, 0] = -(1.0 - 2.0 * M / x)
            gd[0, 1] = 2.0 * M / x
            gd[1, 0] = gd[0, 1]
            gd[1, 1] = 1.0 + 2.0 * M / x
            gd[2, 2] = x ** 2
            gd[3, 3] = x ** 2 * np.sin(y) ** 2
        # boundary_theta_dn: last theta row from the one before
        gd[:, :, :, -1] = gd[:, :, :, -2]
        gd[0, 2, :, -1] = -gd[0, 2, :, -2]
        gd[1, 2, :, -1] = -gd[1, 2, :, -2]
        for (p, q) in ((1, 0), (2, 0), (3, 0), (2, 1), (3, 1), (3, 2)):
            gd[p, q] = gd[q, p]
        self.sqrtg = np.sqrt(gd[2, 2] * (gd[1, 1] * gd[3, 3] - gd[1, 3] ** 2))
        g00, g01, g03, g11, g13, g22, g33 = gd[0, 0], gd[0, 1], gd[0, 3], gd[1, 1], gd[1, 3], gd[2, 2], gd[3, 3]
        idetg = 1.0 / (((g33 * g11 - g13 ** 2) * g00 - g33 * g01 ** 2 + 2.0 * g13 * g03 * g01 - g11 * g03 ** 2) * g22)
        gu = np.zeros_like(gd)
        gu[0, 0] = g22 * (g11 * g33 - g13 ** 2) * idetg
        gu[0, 1] = g22 * (g13 * g03 - g01 * g33) * idetg
        gu[0, 3] = g22 * (g13 * g01 - g11 * g03) * idetg
        gu[1, 1] = g22 * (g33 * g00 - g03 ** 2) * idetg
        gu[1, 3] = g22 * (-g13 * g00 + g03 * g01) * idetg
        gu[2, 2] = ((g33 * g11 - g13 ** 2) * g00 - g33 * g01 ** 2 + 2.0 * g13 * g03 * g01 - g11 * g03 ** 2) * idetg
        gu[3, 3] = g22 * (g11 * g00 - g01 ** 2) * idetg
        gu[:, :, :, -1] = gu[:, :, :, -2]
        gu[0, 2, :, -1] = -gu[0, 2, :, -2]
        gu[1, 2, :, -1] = -gu[1, 2, :, -2]
        for (p, q) in ((1, 0), (2, 0), (3, 0), (2, 1), (3, 1), (3, 2)):
            gu[p, q] = gu[q, p]
        self.g_dn, self.g_up = gd, gu
        self.alpha = np.sqrt(-1.0 / gu[0, 0])
        self.beta = np.stack([self.alpha ** 2 * gu[0, i] for i in (1, 2, 3)])
        self.gamma_up = np.zeros((3, 3) + x.shape)
        for i in range(3):
            for j in range(3):
                self.gamma_up[i, j] = gu[i + 1, j + 1] + self.beta[i] * self.beta[j] / self.alpha ** 2
        self.dx_beta = self.dx1(self.beta[0][:, :, None].astype(np.complex128), self.dx).real[:, :, 0]

    def _b(self, t):  # broadcast a 2-D table over phi
        return t[:, :, None]

    @staticmethod
    def cdiv(z, s):
        """Component-wise complex / real quotient (numpy's complex division
        multiplies by a reciprocal, which is not what gfortran emits)."""
        out = np.empty(np.broadcast(z, s).shape, np.complex128)
        out.real = z.real / s
        out.imag = z.imag / s
        return out

    # ---- operators (tools/finite_differences.f90)
    @staticmethod
    def dx1(f, h):
        res = 0.50 / h
        df = np.empty_like(f)
        df[0] = (-3.0 * f[0] + 4.0 * f[1] - f[2]) * res
        df[1:-1] = (-f[:-2] + f[2:]) * res
        df[-1] = (+3.0 * f[-1] - 4.0 * f[-2] + f[-3]) * res
        return df

    def dx2(self, f, h, inpar=False):
        res = 0.50 / h
        df = np.empty_like(f)
        nz = self.kR
        dis = nz // 2
        df[:, 0, :] = (-3.0 * f[:, 0, :] + 4.0 * f[:, 1, :] - f[:, 2, :]) * res
        for k in range(0, nz + 1):
            kt = (k + dis) % (nz - 1)
            if inpar:
                df[:, 0, k] = (f[:, 2, kt] + f[:, 1, k]) * res
            else:
                df[:, 0, k] = (-f[:, 1, k] + f[:, 2, kt]) * res
        df[:, 1:-1, :] = (-f[:, :-2, :] + f[:, 2:, :]) * res
        df[:, -1, :] = (+3.0 * f[:, -1, :] - 4.0 * f[:, -2, :] + f[:, -3, :]) * res
        return df

    @staticmethod
    def dx3(f, h):
        res = 0.50 / h
        df = np.empty_like(f)
        nz = f.shape[2] - 1
        df[:, :, 0] = (-f[:, :, nz - 2] + f[:, :, 1]) * res
        df[:, :, 1:-1] = (-f[:, :, :-2] + f[:, :, 2:]) * res
        df[:, :, nz] = (-f[:, :, 2] + f[:, :, nz - 1]) * res
        return df

    def ad1(self, f, beta, h):
        res = 0.5 / h
        df = np.empty_like(f)
        n = f.shape[0] - 1
        df[0] = (-3.0 * f[0] + 4.0 * f[1] - f[2]) * res
        df[1] = (-3.0 * f[1] + 4.0 * f[2] - f[3]) * res
        fw = (-3.0 * f[2:n - 1] + 4.0 * f[3:n] - f[4:n + 1]) * res
        bw = (3.0 * f[2:n - 1] - 4.0 * f[1:n - 2] + f[0:n - 3]) * res
        ce = (f[3:n] - f[1:n - 2]) * res
        b = np.broadcast_to(beta[2:n - 1], fw.shape)
        df[2:n - 1] = np.where(b > 0.0, fw, np.where(b < 0.0, bw, ce))
        df[n - 1] = (f[n] - f[n - 2]) * res
        df[n] = (3.0 * f[n] - 4.0 * f[n - 1] + f[n - 2]) * res
        return df

    # ---- RHS (MoL/lines_method_lib.f90:671-753)
    def rhs_phi(self, v):
        return self._b(self.alpha) * v[4] + self._b(self.beta[0]) * v[1]

    def rhs_psi1(self, v):
        al, b1 = self._b(self.alpha), self._b(self.beta[0])
        return self.dx1(al * v[4], self.dx) + b1 * self.ad1(v[1], b1, self.dx) + self._b(self.dx_beta) * v[1]

    def rhs_psi2(self, v):
        return self.dx2(self._b(self.alpha) * v[4] + self._b(self.beta[0]) * v[1], self.dy, False)

    def rhs_psi3(self, v):
        return self.dx3(self._b(self.alpha) * v[4] + self._b(self.beta[0]) * v[1], self.dz)

    def rhs_pi(self, v):
        al, sg, b1 = self._b(self.alpha), self._b(self.sqrtg), self._b(self.beta[0])
        g = lambda a, b: self._b(self.gamma_up[a, b])
        if self.metric == "Kerr_Schild":
            return (self.cdiv(self.dx1(al * sg * (g(0, 0) * v[1] + g(0, 2) * v[3]), self.dx), sg)
                    + self.cdiv(self.dx2(al * sg * g(1, 1) * v[2], self.dy, False), sg)
                    + self.cdiv(self.dx3(al * sg * (g(0, 2) * v[1] + g(2, 2) * v[3]), self.dz), sg)
                    + v[4] * self._b(self.dx_beta)
                    + self.cdiv(b1 * self.ad1(v[4] * sg, b1, self.dx), sg)
                    - al * self.m ** 2 * v[0])
        return (self.cdiv(self.dx1(al * sg * g(0, 0) * v[1], self.dx), sg)
                + self.cdiv(self.dx2(al * sg * g(1, 1) * v[2], self.dy, False), sg)
                + self.dx3(al * g(2, 2) * v[3], self.dz)
                + v[4] * self._b(self.dx_beta)
                + self.cdiv(b1 * self.ad1(v[4] * sg, b1, self.dx), sg)
                - al * self.m ** 2 * v[0])

    def rhs_all(self, v):
        return np.stack([self.rhs_phi(v), self.rhs_psi1(v), self.rhs_psi2(v), self.rhs_psi3(v), self.rhs_pi(v)])

    # ---- boundaries (MoL/lines_method_lib.f90:507-597)
    def boundary(self):
        u = self.u
        u[:, 0] = 3.0 * u[:, 1] - 3.0 * u[:, 2] + u[:, 3]
        if self.bc == "outflow":
            u[:, -1] = u[:, -2]
        else:
            u[:, -1] = self.u_p[:, -1]
        nz, ny, g = self.Nz, self.Ny, self.g
        dis = nz // 2
        for k in range(0, nz + 1):
            kt = (k + dis) % (nz - 1)
            for gg in range(g, -1, -1):
                u[:, :, -gg - self.jL, k] = u[:, :, gg + 1 - self.jL, kt]
        for k in range(0, nz + 1):
            kt = (k + dis) % (nz - 1)
            for gg in range(g, -1, -1):
                u[:, :, ny + gg - self.jL, k] = u[:, :, ny - gg - 1 - self.jL, kt]
        u[:, :, :, 0] = u[:, :, :, nz - 1]
        u[:, :, :, nz] = u[:, :, :, 1]

    # ---- steppers (MoL/lines_method_lib.f90:211-474)
    def pirk2(self):
        dt = self.dt
        self.u_p = self.u.copy()
        r = np.stack([self.rhs_phi(self.u), self.rhs_psi1(self.u), self.rhs_psi2(self.u), self.rhs_psi3(self.u)])
        self.u_stage[0:4] = self.u[0:4] + dt * r
        self.u_stage[4] = self.u[4] + dt * self.rhs_pi(self.u_stage)
        self.boundary()
        r = self.rhs_all(self.u_stage)
        self.u = 0.5 * (self.u_p + self.u_stage + dt * r)
        self.boundary()
        self.t += dt

    def pirk3(self):
        dt = self.dt
        self.u_p = self.u.copy()
        r = np.stack([self.rhs_phi(self.u), self.rhs_psi1(self.u), self.rhs_psi2(self.u), self.rhs_psi3(self.u)])
        self.u_stage[0:4] = self.u[0:4] + dt * r
        self.u_stage[4] = self.u[4] + dt * self.rhs_pi(self.u_stage)
        self.boundary()
        r = np.stack([self.rhs_phi(self.u_stage), self.rhs_psi1(self.u_stage), self.rhs_psi2(self.u_stage),
                      self.rhs_psi3(self.u_stage)])
        self.u_stage_2[0:4] = 0.75 * self.u_p[0:4] + 0.25 * (self.u_stage[0:4] + dt * r)
        self.u_stage_2[4] = 0.75 * self.u_p[4] + 0.25 * (self.u_stage[4] + dt * self.rhs_pi(self.u_stage_2))
        self.boundary()
        r = self.rhs_all(self.u_stage_2)
        self.u = (1.0 / 3.0) * self.u_p + (2.0 / 3.0) * (self.u_stage_2 + dt * r)
        self.boundary()
        self.t += dt

    def rk3(self):
        dt = self.dt
        self.u_p = self.u.copy()
        for rk in (1, 2, 3):
            r = self.rhs_all(self.u)
            if rk == 1:
                self.u = self.u_p + r * dt
            elif rk == 2:
                self.u = 0.750 * self.u_p + 0.250 * (self.u + r * dt)
            else:
                self.u = self.cdiv(self.u_p, 3.0) + self.cdiv(2.0 * (self.u + r * dt), 3.0)
            self.boundary()
        self.t += dt

    def rk4(self):
        dt = self.dt
        self.u_p = self.u.copy()
        ks = []
        for rk in (1, 2, 3, 4):
            r = self.rhs_all(self.u)
            kk = r * dt
            ks.append(kk)
            if rk in (1, 2):
                self.u = self.u_p + 0.50 * kk
            elif rk == 3:
                self.u = self.u_p + kk
            else:
                self.u = self.u_p + self.cdiv(ks[0] + 2.0 * ks[1] + 2.0 * ks[2] + ks[3], 6.0)
            self.boundary()
        self.t += dt

    # ---- the configured method: fourth-order differences, sixth-order
    # Kreiss-Oliger dissipation, Sommerfeld outer plane, RK4, Kerr-Schild form.
    # The reference wires only second-order operators; this restates the C
    # oracle's definition of the method (oracle/kg_oracle.c, rhs_cfg,
    # boundary_cfg, rk4_cfg) in array form, with the one-sided closures of
    # first_derivative_x_4 (tools/finite_differences.f90:124-154) on the first
    # and last two r planes.
    def set_scheme_cfg(self, ko_eps=0.02):
        if self.metric != "Kerr_Schild":
            raise ValueError("the configured method is written for the Kerr-Schild form")
        self.ko_eps = ko_eps
        F = self.beta[0]
        res = 1.0 / (12.0 * self.dx)
        n = F.shape[0] - 1
        D = np.empty_like(F)
        D[0] = (-25.0 * F[0] + 48.0 * F[1] - 36.0 * F[2] + 16.0 * F[3] - 3.0 * F[4]) * res
        D[1] = (-3.0 * F[0] - 10.0 * F[1] + 18.0 * F[2] - 6.0 * F[3] + 1.0 * F[4]) * res
        D[2:n - 1] = (F[0:n - 3] - 8.0 * F[1:n - 2] + 8.0 * F[3:n] - F[4:n + 1]) * res
        D[n - 1] = (3.0 * F[n] + 10.0 * F[n - 1] - 18.0 * F[n - 2] + 6.0 * F[n - 3] - 1.0 * F[n - 4]) * res
        D[n] = (25.0 * F[n] - 48.0 * F[n - 1] + 36.0 * F[n - 2] - 16.0 * F[n - 3] + 3.0 * F[n - 4]) * res
        self.dx_beta4 = D

    @staticmethod
    def d4r(F, res):
        """fourth-order r derivative of an array (r first), closures on two planes per end"""
        D = np.empty_like(F)
        n = F.shape[0] - 1
        D[0] = -25.0 * F[0] + 48.0 * F[1] - 36.0 * F[2] + 16.0 * F[3] - 3.0 * F[4]
        D[1] = -3.0 * F[0] - 10.0 * F[1] + 18.0 * F[2] - 6.0 * F[3] + 1.0 * F[4]
        D[2:n - 1] = F[0:n - 3] - 8.0 * F[1:n - 2] + 8.0 * F[3:n] - F[4:n + 1]
        D[n - 1] = 3.0 * F[n] + 10.0 * F[n - 1] - 18.0 * F[n - 2] + 6.0 * F[n - 3] - 1.0 * F[n - 4]
        D[n] = 25.0 * F[n] - 48.0 * F[n - 1] + 36.0 * F[n - 2] - 16.0 * F[n - 3] + 3.0 * F[n - 4]
        return D * res

    @staticmethod
    def d4c(fm2, fm1, fp1, fp2, res):
        return (fm2 - 8.0 * fm1 + 8.0 * fp1 - fp2) * res

    @staticmethod
    def ko6(m3, m2, m1, c0, p1, p2, p3):
        return m3 - 6.0 * m2 + 15.0 * m1 - 20.0 * c0 + 15.0 * p1 - 6.0 * p2 + p3

    def rhs_cfg(self, v):
        NI, NJ, Nz = self.NI, self.NJ, self.Nz
        rr, rt, rp = 1.0 / (12.0 * self.dx), 1.0 / (12.0 * self.dy), 1.0 / (12.0 * self.dz)
        kr, kt, kp = (self.ko_eps / (64.0 * h) for h in (self.dx, self.dy, self.dz))
        b = self._b
        al, b1, sg, dxb = b(self.alpha), b(self.beta[0]), b(self.sqrtg), b(self.dx_beta4)
        asg = b(self.alpha * self.sqrtg)
        gu = self.gamma_up
        n = NI - 1
        I, J, K = slice(0, n), slice(3, NJ - 3), slice(1, Nz)   # points with the full RHS
        ks = np.arange(1, Nz)
        kper = lambda d: ((ks - 1 + d) % (Nz - 1)) + 1
        jsh = lambda d: slice(3 + d, NJ - 3 + d)
        out = np.zeros_like(v)
        # Sommerfeld plane: d_t u = -(d_r u + u / r)
        rN = self.x[-1]
        for w in range(5):
            out[w, n, J, K] = -(self.d4r(v[w], rr)[n, J, K] + self.cdiv(v[w, n, J, K], rN))
        E = al * v[4] + b1 * v[1]
        r = [None] * 5
        r[0] = E[I, J, K]
        r[1] = (self.d4r(al * v[4], rr) + b1 * self.d4r(v[1], rr) + dxb * v[1])[I, J, K]
        r[2] = self.d4c(E[:, jsh(-2)], E[:, jsh(-1)], E[:, jsh(1)], E[:, jsh(2)], rt)[I, :, K]
        r[3] = self.d4c(E[:, :, kper(-2)], E[:, :, kper(-1)], E[:, :, kper(1)], E[:, :, kper(2)], rp)[I, J, :]
        G1 = asg * (b(gu[0, 0]) * v[1] + b(gu[0, 2]) * v[3])
        H = b(self.alpha * self.sqrtg * gu[1, 1]) * v[2]
        H[:, :3] = -H[:, :3]           # the flux takes the sign of sin(theta) on the ghost rows
        H[:, NJ - 3:] = -H[:, NJ - 3:]
        Fp = asg * (b(gu[0, 2]) * v[1] + b(gu[2, 2]) * v[3])
        t1 = self.cdiv(self.d4r(G1, rr), sg)[I, J, K]
        t2 = self.cdiv(self.d4c(H[:, jsh(-2)], H[:, jsh(-1)], H[:, jsh(1)], H[:, jsh(2)], rt), sg[:, J])[I, :, K]
        t3 = self.cdiv(self.d4c(Fp[:, :, kper(-2)], Fp[:, :, kper(-1)], Fp[:, :, kper(1)], Fp[:, :, kper(2)], rp),
                       sg)[I, J, :]
        t4 = (v[4] * dxb)[I, J, K]
        t5 = self.cdiv(b1 * self.d4r(v[4] * sg, rr), sg)[I, J, K]
        t6 = (b(self.alpha * (self.m * self.m)) * v[0])[I, J, K]
        r[4] = t1 + t2 + t3 + t4 + t5 - t6
        for w in range(5):
            u = v[w]
            a = r[w].copy()
            kor = slice(3, n - 2)        # r planes 3 .. n-3 take the r dissipation
            a[kor] = a[kor] + kr * self.ko6(*(u[3 + d:n - 2 + d, J, K] for d in (-3, -2, -1, 0, 1, 2, 3)))
            a = a + kt * self.ko6(*(u[I, jsh(d), K] for d in (-3, -2, -1, 0, 1, 2, 3)))
            a = a + kp * self.ko6(*(u[I, J][:, :, kper(d)] if d else u[I, J, K] for d in (-3, -2, -1, 0, 1, 2, 3)))
            out[w, I, J, K] = a
        return out

    def boundary_cfg(self):
        u, nz = self.u, self.Nz
        u[:, :, :, 0] = u[:, :, :, nz - 1]
        u[:, :, :, nz] = u[:, :, :, 1]
        dis = nz // 2
        sgn = np.array([1.0, 1.0, -1.0, 1.0, 1.0])[:, None]
        for k in range(0, nz + 1):
            kt = (k + dis) % (nz - 1)
            for gg in range(self.g, -1, -1):
                u[:, :, -gg - self.jL, k] = sgn * u[:, :, gg + 1 - self.jL, kt]
                u[:, :, self.Ny + gg - self.jL, k] = sgn * u[:, :, self.Ny - gg - 1 - self.jL, kt]

    def rk4_cfg(self):
        dt = self.dt
        up = self.u.copy()
        ks = []
        for rk in (1, 2, 3, 4):
            kk = self.rhs_cfg(self.u) * dt
            ks.append(kk)
            if rk in (1, 2):
                self.u = up + 0.50 * kk
            elif rk == 3:
                self.u = up + kk
            else:
                self.u = up + self.cdiv(ks[0] + 2.0 * ks[1] + 2.0 * ks[2] + ks[3], 6.0)
            self.boundary_cfg()
        self.t += dt

    # ---- diagnostics (MoL/diagnostic_lib.f90:277-289, tools/integral.f90:220-255, 646-674)
    def density(self):
        """rho = 1/2 (|Pi| + g^rr |psi1|^2 + 2 g^rphi |psi1| psi3 + g^thth |psi2|^2
        + g^phph |psi3|^2 + m^2 |phi|), real part, in the reference's term order"""
        b, gu, u = self._b, self.gamma_up, self.u
        # |z| as the Fortran abs of a complex value (cabs = hypot); numpy's
        # complex abs uses its own algorithm and differs in the last bit
        a1, a2, a3, a4, a5 = (np.hypot(u[w].real, u[w].imag) for w in range(5))
        re = a5 + b(gu[0, 0]) * (a2 * a2)
        re = re + (2.0 * b(gu[0, 2]) * a2) * u[3].real
        re = re + b(gu[1, 1]) * (a3 * a3)
        re = re + b(gu[2, 2]) * (a4 * a4)
        re = re + (self.m * self.m) * a1
        return 0.5 * re

    def integrate_real(self, f):
        """nested trapezium over i in 0..Nx, j in 0..Ny, all k: phi first, then
        theta, then r, each sum accumulated in index order"""
        g = self.g
        f = f[g:g + self.Nx + 1, g:g + self.Ny + 1, :]
        f2 = np.zeros(f.shape[:2])
        for k in range(f.shape[2] - 1):
            f2 = f2 + f[:, :, k] + f[:, :, k + 1]
        f2 = 0.50 * f2 * self.dz
        f1 = np.zeros(f.shape[0])
        for j in range(f.shape[1] - 1):
            f1 = f1 + f2[:, j] + f2[:, j + 1]
        f1 = 0.50 * f1 * self.dy
        f0 = 0.0
        for i in range(f.shape[0] - 1):
            f0 = f0 + f1[i] + f1[i + 1]
        return 0.50 * f0 * self.dx

    def mass(self):
        """Mass_scalar = integrate(rho sqrt(gamma))"""
        return self.integrate_real(self.density() * self._b(self.sqrtg))

    # ---- detectors and their diagnostics (MoL/diagnostic_lib.f90:124-134, 219-274,
    # main/global_numbers.f90:152-164, tools/FFT_sph.f90:247-279, 525-651,
    # tools/integral.f90:330-362); complex products are written out component by
    # component, as the Fortran compiler emits them
    def detectors(self, n_det):
        r = np.zeros(n_det)
        idx = np.zeros(n_det, int)
        r[0] = 1.0 + math.sqrt(1.0 - self.a * self.a)
        r[-1] = self.xmax_param * 0.99
        for d in range(2, n_det):
            r[d - 1] = r[0] + (r[-1] - r[0]) / float(n_det) * float(d - 1)
        for d in range(n_det):
            for i in range(1, self.Nx):
                if self.xmin + float(i - 1) * self.dx <= r[d] <= self.xmin + float(i) * self.dx:
                    idx[d] = i
                    break
        return r, idx

    def _active(self, r, idx):
        return self.xmin <= r < self.xmin + float(self.Nx - 1) * self.dx and idx > 0

    def domain_to_sph_shell(self, f, iv):
        """f (NI, NJ, NK) complex on the evolution grid -> its values on the vertex
        sphere of radius xmin + (iv - 1) dx, (Ny, Nz) [theta, phi]: index search
        in each direction, then trilinear interpolation (phi, theta, r); the
        theta rows outside the cell-centred grid copy the edge row"""
        iL, iR, jL, jR, kL, kR = self.iL, self.iR, self.jL, self.jR, self.kL, self.kR
        RD = lambda i: self.x[i - iL]
        TD = lambda j: self.y[j - jL]
        PD = lambda k: float(k) * self.dz
        rmin, dr = RD(iL), RD(iL + 1) - RD(iL)
        thetamin, dth = TD(jL), abs(TD(jL + 1) - TD(jL))
        phimin, dph = PD(kL), abs(PD(kL + 1) - PD(kL))

        def search(v, vmin, d, lo, hi, at):
            i = int((v - vmin) / d) + lo
            i = max(lo, min(i, hi - 1))
            while i < hi - 1 and v >= at(i + 1):
                i += 1
            while i > lo and v < at(i):
                i -= 1
            return i

        rr = self.xmin + float(iv - 1) * self.dx
        ir = search(rr, rmin, dr, iL, iR, RD)
        out = np.zeros((self.Ny, self.Nz), np.complex128)
        for kv in range(1, self.Nz + 1):
            pp = float(kv - 1) * self.dz
            ip = search(pp, phimin, dph, kL, kR, PD)
            for jv in range(1, self.Ny + 1):
                tt = float(jv - 1) * self.dy
                it = search(tt, thetamin, dth, jL, jR, TD)
                if tt <= thetamin:
                    out[jv - 1, kv - 1] = f[ir - iL, 0, ip]
                    continue
                if tt >= thetamin + dth * float(jR - jL):
                    out[jv - 1, kv - 1] = f[ir - iL, jR - jL, ip]
                    continue
                wr, wt, wp = (rr - RD(ir)) / dr, (tt - TD(it)) / dth, (pp - PD(ip)) / dph
                c = lambda di, dj, dk: f[ir - iL + di, it - jL + dj, ip + dk]

                def lin(w, a, b):
                    return complex((1.0 - w) * a.real + w * b.real, (1.0 - w) * a.imag + w * b.imag)
                f00, f01 = lin(wp, c(0, 0, 0), c(0, 0, 1)), lin(wp, c(0, 1, 0), c(0, 1, 1))
                f10, f11 = lin(wp, c(1, 0, 0), c(1, 0, 1)), lin(wp, c(1, 1, 0), c(1, 1, 1))
                out[jv - 1, kv - 1] = lin(wr, lin(wt, f00, f01), lin(wt, f10, f11))
        return out

    def _trap_weights(self, j, k):
        sel = (1 if j in (1, self.Ny) else 0) + 2 * (1 if k in (1, self.Nz) else 0)
        return None if sel == 0 else (0.25 if sel == 3 else 0.5)

    def project_sh(self, sl, Y, L):
        """a_lm (2L+1, L+1) [m+L, l] of a sphere slice (Ny, Nz) against the Y_lm table
        Y (Nz, Ny, 2L+1, L+1): trapezium of f conj(Y) sin(theta), summed in index order"""
        ire = np.zeros((2 * L + 1, L + 1))
        iim = np.zeros_like(ire)
        for j in range(1, self.Ny + 1):
            st = math.sin(float(j - 1) * self.dy)
            for k in range(1, self.Nz + 1):
                a = sl[j - 1, k - 1]
                y = Y[k - 1, j - 1]
                cre, cim = y.real, -y.imag
                fre = (a.real * cre - a.imag * cim) * st
                fim = (a.real * cim + a.imag * cre) * st
                w = self._trap_weights(j, k)
                if w is None:
                    ire, iim = ire + fre, iim + fim
                else:
                    ire, iim = ire + w * fre, iim + w * fim
        wq = self.dy * self.dz
        out = np.empty(ire.shape, np.complex128)
        out.real, out.imag = wq * ire, wq * iim
        return out

    def trap2d(self, sl):
        re = im = 0.0
        for j in range(1, self.Ny + 1):
            for k in range(1, self.Nz + 1):
                v = sl[j - 1, k - 1]
                w = self._trap_weights(j, k)
                if w is None:
                    re, im = re + v.real, im + v.imag
                else:
                    re, im = re + w * v.real, im + w * v.imag
        wq = self.dy * self.dz
        return complex(wq * re, wq * im)

    def proyector_detectors(self, Y, L, n_det):
        r, idx = self.detectors(n_det)
        out = np.zeros((n_det, 2 * L + 1, L + 1), np.complex128)
        for d in range(n_det):
            if self._active(r[d], idx[d]):
                out[d] = self.project_sh(self.domain_to_sph_shell(self.u[0], idx[d]), Y, L)
        return out

    def currents_detectors(self, n_det):
        """momentum(3, n_det): trapezium over the detector sphere of sqrt(gamma) j_i,
        j_i = -Pi gamma^ij psi_j (currents_ADM), real part"""
        b, gu, u = self._b, self.gamma_up, self.u
        n5r, n5i = -u[4].real, -u[4].imag

        def cx(ar, ai):  # (-Pi) times (ar + i ai), component-wise
            return n5r * ar - n5i * ai, n5r * ai + n5i * ar
        a = b(gu[0, 0]) * u[1] + b(gu[0, 2]) * u[3]
        bb = b(gu[1, 1]) * u[2]
        c = b(gu[0, 2]) * u[1] + b(gu[2, 2]) * u[3]
        r, idx = self.detectors(n_det)
        out = np.zeros((n_det, 3))
        for comp, z in enumerate((a, bb, c)):
            jr, ji = cx(z.real, z.imag)
            g = np.empty(jr.shape, np.complex128)
            g.real, g.imag = jr * b(self.sqrtg), ji * b(self.sqrtg)
            for d in range(n_det):
                if self._active(r[d], idx[d]):
                    out[d, comp] = self.trap2d(self.domain_to_sph_shell(g, idx[d])).real
        return out

    # ---- Fortran-order state helpers: u(5, NI, NJ, NK) complex, var fastest
    def set_state(self, fortran_u):
        self.u = np.ascontiguousarray(np.asarray(fortran_u).reshape(self.NK, self.NJ, self.NI, 5).transpose(3, 2, 1, 0))

    def get_state(self):
        return np.ascontiguousarray(self.u.transpose(3, 2, 1, 0)).reshape(-1)
