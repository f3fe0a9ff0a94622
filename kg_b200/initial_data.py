"""Seeded initial data in the reference's Fortran state layout.

The reference builds its initial data in main/initial_conditions.f90: phi is
set on the whole stored grid, psi_1..3 are the reference's own first-derivative
operators applied to phi (:158-164) and Pi is set from the time derivative.
These helpers produce the same kind of state on the host, as input for both
the device solver and the CPU oracle:

* ``gaussian_y20``   -- phi = A exp(-(r - r0)^2) Y_20(theta), Pi = 0
  (Y_20 in the analytic form of tools/harmonics.f90:63).
* ``shell_ylm``      -- phi = exp(-(r - r0)^2 / sigma^2) sum_{l<=lmax,|m|<=l}
  c_lm Y_lm(theta, phi) with c_lm complex N(0, sd^2) drawn from a numpy seed,
  Pi = 0 (the Gaussian shell form of main/initial_conditions.f90:62,158).

* ``smooth_exact``   -- for the configured fourth-order method: phi =
  amp exp(-((r - r0)/w)^2) times a function that is smooth on the sphere
  (combinations of Re Y_20, Re Y_21, Re Y_22, or Y_20 alone), with psi_1..3 the
  exact derivatives (so the data carry no second-order differencing error),
  Pi = 0.

Arrays returned have C shape (NK, NJ, NI, 5), i.e. the Fortran array
u(1:5, -g:Nx+g, -g:Ny+g, 0:Nz) with the variable index fastest.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.special import sph_harm_y


def grid_axes(Nx, Ny, Nz, xmin, xmax, g=2):
    """Evolution-grid coordinates of MoL/mesh_refinement_lib.f90:100-147 (nproc=1)."""
    pi = math.acos(-1.0)
    dxr = (xmax - xmin) / 1.0
    x0 = xmin + 0.0 * dxr
    x1 = xmin + 1.0 * dxr
    dx = (x1 - x0) / float(Nx)
    dy = pi / float(Ny - 1)
    dz = 2.0 * pi / float(Nz - 1)
    x = x0 + (np.arange(-g, Nx + g + 1) + g).astype(np.float64) * dx
    y = -dy / 2.0 + np.arange(-g, Ny + g + 1).astype(np.float64) * dy
    z = np.arange(0, Nz + 1).astype(np.float64) * dz
    return x, y, z, dx, dy, dz


def _dx1(f, h):
    # first_derivative_x_2_uniform along axis 2 (r) of an (NK, NJ, NI) array
    res = 0.50 / h
    df = np.empty_like(f)
    df[..., 0] = (-3.0 * f[..., 0] + 4.0 * f[..., 1] - f[..., 2]) * res
    df[..., 1:-1] = (-f[..., :-2] + f[..., 2:]) * res
    df[..., -1] = (+3.0 * f[..., -1] - 4.0 * f[..., -2] + f[..., -3]) * res
    return df


def _dx2(f, h, Nz):
    # first_derivative_y_2 with inpar = .false. along axis 1 (theta)
    res = 0.50 / h
    df = np.empty_like(f)
    dis = Nz // 2
    df[:, 1:-1, :] = (-f[:, :-2, :] + f[:, 2:, :]) * res
    df[:, -1, :] = (+3.0 * f[:, -1, :] - 4.0 * f[:, -2, :] + f[:, -3, :]) * res
    for k in range(Nz + 1):
        kt = (k + dis) % (Nz - 1)
        df[k, 0, :] = (-f[k, 1, :] + f[kt, 2, :]) * res
    return df


def _dx3(f, h):
    # first_derivative_z_2 along axis 0 (phi)
    res = 0.50 / h
    df = np.empty_like(f)
    nz = f.shape[0] - 1
    df[0] = (-f[nz - 2] + f[1]) * res
    df[1:-1] = (-f[:-2] + f[2:]) * res
    df[nz] = (-f[2] + f[nz - 1]) * res
    return df


def _assemble(phi, dx, dy, dz, Nz):
    u = np.zeros(phi.shape + (5,), np.complex128)
    u[..., 0] = phi
    u[..., 1] = _dx1(phi, dx)
    u[..., 2] = _dx2(phi, dy, Nz)
    u[..., 3] = _dx3(phi, dz)
    u[..., 4] = 0.0
    return u


def smooth_exact(Nx, Ny, Nz, xmin, xmax, amp=1.0, r0=10.0, width=2.0, angular="mix"):
    """phi = amp exp(-((r-r0)/w)^2) f(theta, phi) with exact psi_1..3 and Pi = 0.
    angular: 'mix' = (3 cos^2 - 1) + 0.5 sin cos cos(phi) + 0.3 sin^2 cos(2 phi);
    'y20' = sqrt(5/(16 pi)) (3 cos^2 - 1)."""
    x, y, z, dx, dy, dz = grid_axes(Nx, Ny, Nz, xmin, xmax)
    T, P = y[None, :, None], z[:, None, None]
    X = x[None, None, :]
    c, sn = np.cos(T), np.sin(T)
    if angular == "y20":
        a = math.sqrt(5.0 / (16.0 * math.pi))
        f = a * (3 * c ** 2 - 1) + 0 * P
        ft = a * (-6 * c * sn) + 0 * P
        fp = 0 * f
    else:
        f = (3 * c ** 2 - 1) + 0.5 * sn * c * np.cos(P) + 0.3 * sn ** 2 * np.cos(2 * P)
        ft = -6 * c * sn + 0.5 * np.cos(2 * T) * np.cos(P) + 0.6 * sn * c * np.cos(2 * P)
        fp = -0.5 * sn * c * np.sin(P) - 0.6 * sn ** 2 * np.sin(2 * P)
    g = amp * np.exp(-((X - r0) / width) ** 2)
    gr = -2.0 * (X - r0) / width ** 2 * g
    u = np.zeros((Nz + 1, Ny + 5, Nx + 5, 5), np.complex128)
    u[..., 0] = f * g
    u[..., 1] = f * gr
    u[..., 2] = ft * g
    u[..., 3] = fp * g
    return u


def gaussian_y20(Nx, Ny, Nz, xmin, xmax, amp=1.0e-3, r0=10.0):
    """phi = amp exp(-(r-r0)^2) Y_20(theta); psi_i by the reference stencils; Pi = 0."""
    x, y, z, dx, dy, dz = grid_axes(Nx, Ny, Nz, xmin, xmax)
    pi = math.acos(-1.0)
    y20 = math.sqrt(5.0 / (16.0 * pi)) * (3.0 * np.cos(y) ** 2 - 1.0)
    radial = amp * np.exp(-(x - r0) ** 2)
    phi = (y20[:, None] * radial[None, :])[None, :, :] * np.ones((Nz + 1, 1, 1))
    return _assemble(phi.astype(np.complex128), dx, dy, dz, Nz)


def shell_ylm(Nx, Ny, Nz, xmin, xmax, seed, lmax=4, sd=1.0e-4, r0=None, sigma=1.5,
              r0_range=(8.0, 15.0)):
    """Gaussian shell times a seeded random Y_lm combination (l <= lmax)."""
    rng = np.random.default_rng(seed)
    if r0 is None:
        r0 = float(rng.uniform(*r0_range))
    x, y, z, dx, dy, dz = grid_axes(Nx, Ny, Nz, xmin, xmax)
    ang = np.zeros((Nz + 1, Ny + 5), np.complex128)
    Y, Z = np.meshgrid(y, z)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            c = complex(rng.normal(0.0, sd), rng.normal(0.0, sd))
            ang += c * sph_harm_y(l, m, Y, Z)
    radial = np.exp(-(x - r0) ** 2 / sigma ** 2)
    phi = ang[:, :, None] * radial[None, None, :]
    return _assemble(phi, dx, dy, dz, Nz), r0


def shell_ylm_device(Nx, Ny, Nz, xmin, xmax, seed, device, lmax=4, sd=1.0e-4, sigma=1.5,
                     r0_range=(8.0, 15.0)):
    """`shell_ylm` assembled on a CUDA device with torch (for grids too large to
    build comfortably on the host).  The seeded coefficients, radial profile and
    angular factor are drawn on the host exactly as in `shell_ylm`; the outer
    product and the three reference derivative stencils run on the device.
    Returns a complex128 tensor of shape (NK, NJ, NI, 5) and r0."""
    import torch
    rng = np.random.default_rng(seed)
    r0 = float(rng.uniform(*r0_range))
    x, y, z, dx, dy, dz = grid_axes(Nx, Ny, Nz, xmin, xmax)
    ang = np.zeros((Nz + 1, Ny + 5), np.complex128)
    Y, Z = np.meshgrid(y, z)
    for l in range(lmax + 1):
        for m in range(-l, l + 1):
            c = complex(rng.normal(0.0, sd), rng.normal(0.0, sd))
            ang += c * sph_harm_y(l, m, Y, Z)
    radial = np.exp(-(x - r0) ** 2 / sigma ** 2)
    a = torch.from_numpy(ang).to(device)
    r = torch.from_numpy(radial.astype(np.complex128)).to(device)
    u = torch.zeros((Nz + 1, Ny + 5, Nx + 5, 5), dtype=torch.complex128, device=device)
    phi = a[:, :, None] * r[None, None, :]
    u[..., 0] = phi
    # psi_1: first_derivative_x_2_uniform along r
    res = 0.50 / dx
    d = u[..., 1]
    d[..., 0] = (-3.0 * phi[..., 0] + 4.0 * phi[..., 1] - phi[..., 2]) * res
    d[..., 1:-1] = (-phi[..., :-2] + phi[..., 2:]) * res
    d[..., -1] = (+3.0 * phi[..., -1] - 4.0 * phi[..., -2] + phi[..., -3]) * res
    # psi_2: first_derivative_y_2 (inpar = .false.) along theta
    res = 0.50 / dy
    d = u[..., 2]
    d[:, 1:-1, :] = (-phi[:, :-2, :] + phi[:, 2:, :]) * res
    d[:, -1, :] = (+3.0 * phi[:, -1, :] - 4.0 * phi[:, -2, :] + phi[:, -3, :]) * res
    kt = torch.tensor([(k + Nz // 2) % (Nz - 1) for k in range(Nz + 1)], device=device)
    d[:, 0, :] = (-phi[:, 1, :] + phi[kt, 2, :]) * res
    # psi_3: first_derivative_z_2 along phi
    res = 0.50 / dz
    d = u[..., 3]
    d[0] = (-phi[Nz - 2] + phi[1]) * res
    d[1:-1] = (-phi[:-2] + phi[2:]) * res
    d[Nz] = (-phi[2] + phi[Nz - 1]) * res
    if u.is_cuda:
        # the solver reads the tensor on its own stream
        torch.cuda.current_stream(u.device).synchronize()
    return u, r0
