"""GPU test of kg_integrate_mass_noalloc, the mass integral for callers that
cannot allocate device memory (a host whose device memory is owned by its own
pool or a fixed budget, or one that must not take the device-wide
synchronisation of cudaMalloc / cudaFree inside its time loop).

The entry point is called through the C ABI on device buffers the test owns,
twice in a row on different densities, and each result is checked against
kg_mass_scalar (the handle-based entry point) at the relative tolerance the
other diagnostic tests use, and against the oracle's trapezium, which it
follows in summation order.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRID = dict(Nx=64, Ny=17, Nz=33, xmin=1.8, xmax=20.0)
RTOL = 1e-12


def _noalloc(lib, rho, sqrtg, sc, out, stream=None):
    g = GRID
    return lib.kg_integrate_mass_noalloc(C.c_void_p(rho.data_ptr()), C.c_void_p(sqrtg.data_ptr()), g["Nx"], g["Ny"],
                                         g["Nz"], sc[0], sc[1], sc[2], C.c_void_p(out.data_ptr()), stream)


def test_mass_noalloc_matches_mass_scalar_twice():
    import torch
    from kg_b200 import ScalarField, capi
    from kg_b200.initial_data import shell_ylm
    from oracle.oracle import Oracle, lib as olib

    g = GRID
    lib = capi.load()
    mol = ScalarField(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=0.3)
    ora = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], CFL=0.25, m=0.3)
    u0, _ = shell_ylm(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], seed=21, r0=8.0, sd=1.0)
    mol.u = u0
    ora.set_state(u0)
    sc = (mol.dx, mol.dy, mol.dz)
    sqrtg = torch.from_numpy(np.ascontiguousarray(mol.metric_tables()[3])).cuda()
    out = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    results = []
    for call in range(2):
        if call == 1:  # a different density for the second call
            mol.pirk2(5)
            ora.pirk2(5)
        mol.density()
        want = mol.mass_scalar()
        rho = torch.from_numpy(np.ascontiguousarray(mol.rho)).cuda()
        out.fill_(np.nan)
        torch.cuda.synchronize()
        rc = _noalloc(lib, rho, sqrtg, sc, out)
        assert rc == capi.KG_OK, lib.kg_last_error(None)
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - want) <= RTOL * abs(want), (call, got, want)
        # same summation order as the oracle's trapezium on the same rho * sqrtg
        f = np.ascontiguousarray(mol.rho * sqrtg.cpu().numpy()[None, :, :])
        exact = olib().kgo_integrate_real(ora.h, f.ctypes.data_as(C.POINTER(C.c_double)))
        assert got == exact, (call, got, exact)
        results.append(got)
    assert results[0] != results[1]


def test_mass_noalloc_rejects_oversized_grid():
    import torch
    from kg_b200 import capi
    lib = capi.load()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    rc = lib.kg_integrate_mass_noalloc(p, p, 4096, 200, 8, 1.0, 1.0, 1.0, p, None)
    assert rc == capi.KG_EINVAL
    assert b"static scratch holds" in lib.kg_last_error(None)


def test_mass_noalloc_wide_theta_grid_and_error_cleared():
    """A grid with more theta rows than a launch's y-dimension allows (Ny + 1 >
    65535) is within the scratch limit and runs; a successful call after a
    rejected one leaves kg_last_error(NULL) empty."""
    import torch
    from kg_b200 import capi
    lib = capi.load()
    bad = torch.zeros(8, dtype=torch.float64, device="cuda")
    pb = C.c_void_p(bad.data_ptr())
    assert lib.kg_integrate_mass_noalloc(pb, pb, 4096, 200, 8, 1.0, 1.0, 1.0, pb, None) == capi.KG_EINVAL
    Nx, Ny, Nz = 1, 100000, 1
    NI, NJ = Nx + 5, Ny + 5
    rho = torch.ones((Nz + 1) * NJ * NI, dtype=torch.float64, device="cuda")
    sqrtg = torch.ones(NJ * NI, dtype=torch.float64, device="cuda")
    out = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    rc = lib.kg_integrate_mass_noalloc(C.c_void_p(rho.data_ptr()), C.c_void_p(sqrtg.data_ptr()), Nx, Ny, Nz,
                                       1.0, 1.0, 1.0, C.c_void_p(out.data_ptr()), None)
    assert rc == capi.KG_OK, lib.kg_last_error(None)
    torch.cuda.synchronize()
    assert lib.kg_last_error(None) == b""
    # trapezium of a constant 1 over [0, Nz] x [0, Ny] x [0, Nx] with unit spacings
    assert float(out.item()) == float(Nx * Ny * Nz)
