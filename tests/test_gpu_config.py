"""GPU tests of the configured method (fourth-order differences, sixth-order
Kreiss-Oliger dissipation, Sommerfeld outer plane, parity-correct pole ghosts;
RK4): against the oracle's restatement, and fourth-order self-convergence
across three resolutions.

The method has no reference arithmetic to reproduce, so its kernels contract
multiply-adds (FMA) while the oracle rounds every product and sum separately.
The two then differ by a few units in the last place per operation; the tests
hold the GPU to the oracle within REL = 1e-13 relative L2 over 10 RK4 steps
(and 1e-12 of max |u| pointwise)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pair(Nx, Ny, Nz, eps=0.02, m=0.2, steps=10):
    from kg_b200 import ScalarField
    from kg_b200.initial_data import smooth_exact
    from oracle.oracle import Oracle
    u0 = smooth_exact(Nx, Ny, Nz, 1.8, 20.0, amp=1e-3)
    dev = ScalarField(Nx, Ny, Nz, 1.8, 20.0, 0.25, m=m)
    dev.set_scheme("configured", eps)
    dev.u = u0
    dev.fill_ghosts_configured()
    ora = Oracle(Nx, Ny, Nz, 1.8, 20.0, CFL=0.25, m=m)
    ora.set_scheme(1, eps)
    ora.set_state(u0)
    ora.boundary_cfg()
    return dev, ora


REL = 1e-13


def _close(a, b):
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    return rel <= REL and np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), rel


@pytest.mark.parametrize("grid", [(24, 17, 33), (37, 13, 25)])
def test_configured_rk4_vs_oracle(grid):
    dev, ora = _pair(*grid)
    assert np.array_equal(dev.u, ora.get_state())   # the ghost fills copy values
    dev.rk4(nsteps=1)
    ora.rk4(1)
    ok, rel = _close(dev.u, ora.get_state())
    assert ok, rel
    dev.rk4(nsteps=9)   # graph replay of step pairs
    ora.rk4(9)
    ok, rel = _close(dev.u, ora.get_state())
    print(f"configured RK4 x10 on {grid}: rel L2 vs oracle {rel:.2e}")
    assert ok, rel


@pytest.mark.parametrize("grid", [(24, 17, 33), (67, 41, 9), (150, 9, 129)])
def test_configured_tiled_equals_per_point(grid):
    """the shared-memory tiled form (default) and the one-thread-per-point form
    (kernel variant 0) give the same bits: partial tiles in r and theta, phi
    chunks of one plane up to the whole range, and the oracle on the first grid"""
    dev, ora = _pair(*grid, steps=3)
    ref, _ = _pair(*grid, steps=3)
    ref._ck(ref._lib.kg_set_kernel_variant(ref.handle, 0))
    dev.rk4(nsteps=3)
    ref.rk4(nsteps=3)
    assert np.array_equal(dev.u, ref.u)
    if grid == (24, 17, 33):
        ora.rk4(3)
        ok, rel = _close(dev.u, ora.get_state())
        assert ok, rel


def test_configured_scheme_guards():
    from kg_b200 import ScalarField, KgError
    s = ScalarField(16, 9, 17, 1.8, 12.0, 0.25)
    s.set_scheme("configured")
    with pytest.raises(KgError):
        s.pirk2(1)
    with pytest.raises(KgError):
        s.precision = "mixed"
    s.set_scheme("reference")
    s.pirk2(1)
    t = ScalarField(16, 9, 17, 1.8, 12.0, 0.25, metric="Schw_EF")
    with pytest.raises(KgError):
        t.set_scheme("configured")


def _run(level, T, dt):
    from kg_b200 import ScalarField
    from kg_b200.initial_data import smooth_exact
    Nx, Nth = 64 * 2 ** level, 16 * 2 ** level
    Ny, Nz = Nth + 1, 2 * Nth + 1
    s = ScalarField(Nx, Ny, Nz, 1.8, 20.0, 0.25, m=0.2, dt=dt)
    s.set_scheme("configured", 0.02)
    s.u = smooth_exact(Nx, Ny, Nz, 1.8, 20.0)
    s.fill_ghosts_configured()
    s.rk4(nsteps=int(round(T / dt)))
    return s.u[..., 0], s.dx


def test_configured_fourth_order_self_convergence():
    """three resolutions (64/128/256 radial, 16/32/64 theta cells), the finest
    grid's time step, t = 0.3; the RMS difference ratio approaches 2^4 = 16"""
    import sys, os
    sys.path.insert(0, os.path.dirname(__file__))
    from test_oracle import cfg_rms_diff
    T = 0.3
    dt = 0.25 * math.exp(1.8) * math.sin(math.pi / 64 / 2) * (2 * math.pi / 128)
    runs = [_run(l, T, dt) for l in range(3)]
    e01 = cfg_rms_diff(runs[1][0], runs[0][0], runs[0][1])
    e12 = cfg_rms_diff(runs[2][0], runs[1][0], runs[1][1])
    factor = e01 / e12
    print(f"configured method: self-convergence factor {factor:.2f}")
    assert 12.0 < factor < 20.0, factor
