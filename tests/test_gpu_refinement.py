"""GPU tests of the Berger-Oliger hierarchy (radially nested 2:1 levels,
csrc/kg_refine.cu).  The reference builds a single uniform level, so there is
no reference output to match; the tests pin the construction by consistency:
a one-level hierarchy is the plain solver bit for bit, restriction copies the
coincident fine values, and a refined level reproduces a uniformly fine solve
inside its region far better than the coarse level does."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

XMIN, XMAX, NY, NZ = 1.8, 30.0, 17, 33


def _ic(level_view):
    from kg_b200.initial_data import smooth_exact
    lv = level_view
    return smooth_exact(lv.Nx, lv.Ny, lv.Nz, XMIN, lv.params.xmax, amp=1e-3, r0=8.0, width=2.0)


@pytest.mark.parametrize("method", ["rk4", "rk3", "pirk2", "pirk3"])
def test_single_level_is_the_plain_solver(method):
    from kg_b200 import ScalarField
    from kg_b200.refinement import BergerOliger
    bo = BergerOliger(48, NY, NZ, XMIN, XMAX, 0.25, r_fine=(), m=0.2)
    s = ScalarField(48, NY, NZ, XMIN, XMAX, 0.25, m=0.2)
    u0 = _ic(bo.levels[0])
    bo.levels[0].u = u0
    s.u = u0
    getattr(bo, method)(5)
    getattr(s, method)(nsteps=5)
    assert np.array_equal(bo.levels[0].u, s.u)
    assert bo.levels[0].t == s.t


def _run_bo(nsteps, r_fine, method="rk4"):
    from kg_b200.refinement import BergerOliger
    bo = BergerOliger(64, NY, NZ, XMIN, XMAX, 0.25, r_fine=r_fine, m=0.2)
    for lv in bo.levels:
        lv.u = _ic(lv)
    getattr(bo, method)(nsteps)
    bo.synchronize()
    return bo


@pytest.mark.parametrize("method", ["rk4", "pirk2"])
def test_restriction_and_level_clocks(method):
    bo = _run_bo(3, (16.0, 9.0), method)
    dt0 = bo.levels[0].dt
    for l, lv in enumerate(bo.levels):
        assert abs(lv.dt - dt0 / 2 ** l) <= 1e-15 * dt0
        assert abs(lv.t - 3 * dt0) <= 1e-12
    c, f = bo.levels[0].u, bo.levels[1].u
    nf = f.shape[2]
    last = nf - 1 - 8
    nc = last // 2 + 1
    assert np.array_equal(c[:, :, :nc], f[:, :, 0:2 * nc:2])
    assert np.all(np.isfinite(bo.levels[2].u))
    bo.close()


@pytest.mark.parametrize("method", ["rk4", "rk3", "pirk2", "pirk3"])
def test_refined_level_tracks_the_uniform_fine_solve(method):
    from kg_b200 import ScalarField
    from kg_b200.initial_data import smooth_exact
    n = 20
    bo = _run_bo(n, (16.0,), method)
    coarse = ScalarField(64, NY, NZ, XMIN, XMAX, 0.25, m=0.2)
    coarse.u = smooth_exact(64, NY, NZ, XMIN, XMAX, amp=1e-3, r0=8.0, width=2.0)
    dt0 = coarse.dt
    getattr(coarse, method)(nsteps=n)
    fine = ScalarField(128, NY, NZ, XMIN, XMAX, 0.25, m=0.2, dt=dt0 / 2)
    fine.u = smooth_exact(128, NY, NZ, XMIN, XMAX, amp=1e-3, r0=8.0, width=2.0)
    getattr(fine, method)(nsteps=2 * n)
    uf, ub, uc = fine.u[..., 0], bo.levels[1].u[..., 0], coarse.u[..., 0]
    dxf = fine.dx
    idx = [i for i in range(0, ub.shape[2], 2) if 4.0 <= XMIN + i * dxf <= 12.0]   # coincident with coarse points
    ref = uf[:, :, idx]
    e_bo = np.linalg.norm(ub[:, :, idx] - ref) / np.linalg.norm(ref)
    e_c = np.linalg.norm(uc[:, :, [i // 2 for i in idx]] - ref) / np.linalg.norm(ref)
    print(f"{method} r in [4, 12]: refined level vs uniform fine {e_bo:.2e}, coarse vs uniform fine {e_c:.2e}")
    assert e_bo < 0.05 * e_c
    bo.close()


@pytest.mark.parametrize("method", ["rk4", "rk3", "pirk2", "pirk3"])
def test_pulse_through_the_interface(method):
    """a pulse that starts next to the coarse-fine interface (r = 16) and runs
    through it: inside the refined level, near the interface, the hierarchy
    stays much closer to the uniformly fine solve than the coarse level does,
    and the interface visibly influences that region (the difference is not 0)"""
    from kg_b200 import ScalarField
    from kg_b200.refinement import BergerOliger
    from kg_b200.initial_data import smooth_exact
    n, r0, w = 40, 13.0, 1.5
    bo = BergerOliger(64, NY, NZ, XMIN, XMAX, 0.25, r_fine=(16.0,), m=0.2)
    for lv in bo.levels:
        lv.u = smooth_exact(lv.Nx, lv.Ny, lv.Nz, XMIN, lv.params.xmax, amp=1e-3, r0=r0, width=w)
    getattr(bo, method)(n)
    bo.synchronize()
    coarse = ScalarField(64, NY, NZ, XMIN, XMAX, 0.25, m=0.2)
    coarse.u = smooth_exact(64, NY, NZ, XMIN, XMAX, amp=1e-3, r0=r0, width=w)
    dt0 = coarse.dt
    getattr(coarse, method)(nsteps=n)
    fine = ScalarField(128, NY, NZ, XMIN, XMAX, 0.25, m=0.2, dt=dt0 / 2)
    fine.u = smooth_exact(128, NY, NZ, XMIN, XMAX, amp=1e-3, r0=r0, width=w)
    getattr(fine, method)(nsteps=2 * n)
    uf, ub, uc = fine.u[..., 0], bo.levels[1].u[..., 0], coarse.u[..., 0]
    dxf = fine.dx
    idx = [i for i in range(0, ub.shape[2], 2) if 10.0 <= XMIN + i * dxf <= 14.5]
    ref = uf[:, :, idx]
    e_bo = np.linalg.norm(ub[:, :, idx] - ref) / np.linalg.norm(ref)
    e_c = np.linalg.norm(uc[:, :, [i // 2 for i in idx]] - ref) / np.linalg.norm(ref)
    print(f"{method} r in [10, 14.5] after the pulse crossed r = 16: refined {e_bo:.2e}, coarse {e_c:.2e}")
    assert 0.0 < e_bo < 1e-3 * e_c
    bo.close()
