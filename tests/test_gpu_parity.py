"""GPU parity tests: the CUDA path through the C ABI against the CPU oracle.

The FP64 solver keeps the reference's operation order and rounding (no fused
multiply-add, component-wise complex-by-real arithmetic), so states after any
number of steps are compared for exact equality.  The parity bound for
the C0 run is 1e-11 relative L2 in phi and Pi after 1000 steps; the test
asserts that bound and, separately, reports bit equality.
Diagnostics that reduce in a different order are compared at 1e-12 relative.
"""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

SMALL = dict(Nx=16, Ny=9, Nz=17, xmin=1.8, xmax=12.0)


def _pair(metric="Kerr_Schild", bc="outflow", m=0.3, grid=SMALL, CFL=0.25, n_det=5, l_max=6):
    from kg_b200 import ScalarField
    from oracle.oracle import Oracle, KERR_SCHILD, SCHW_EF, OUTFLOW, INFLOW
    dev = ScalarField(grid["Nx"], grid["Ny"], grid["Nz"], grid["xmin"], grid["xmax"], CFL, m=m,
                      metric=metric, boundary_type_rmax=bc, n_det=n_det, l_max=l_max)
    ora = Oracle(grid["Nx"], grid["Ny"], grid["Nz"], grid["xmin"], grid["xmax"], CFL=CFL, m=m,
                 metric=KERR_SCHILD if metric == "Kerr_Schild" else SCHW_EF,
                 bc_rmax=OUTFLOW if bc == "outflow" else INFLOW, n_det=n_det, l_max=l_max)
    return dev, ora


def _ic(grid=SMALL, seed=3, r0=6.0):
    from kg_b200.initial_data import shell_ylm
    u, _ = shell_ylm(grid["Nx"], grid["Ny"], grid["Nz"], grid["xmin"], grid["xmax"], seed=seed, r0=r0, sd=1.0)
    return u


def test_metric_tables_match_oracle():
    for metric in ("Kerr_Schild", "Schw_EF"):
        dev, ora = _pair(metric=metric)
        assert np.array_equal(dev.metric_tables(), ora.metric())
        s_dev = (dev.dx, dev.dy, dev.dz, dev.dt)
        s_ora = ora.scalars()
        assert s_dev == (s_ora["dx"], s_ora["dy"], s_ora["dz"], s_ora["dt"])
        assert dev.validate_inverse_metric() == (0, 0)


def test_values_next_to_underflow_per_point_form():
    """A field scaled to ~1e-303, the size a Gaussian tail passes through on its
    way to underflow.  The per-point form (kernel variant 0) divides by
    sqrt(gamma) outright and stays bit-exact with the oracle here.  The tiled
    forms divide by a reciprocal product with one Markstein correction, which
    can differ from IEEE division by one unit in the last place for dividends
    below about 2^-1000, a relative error far inside the parity bound."""
    dev, ora = _pair()
    dev._ck(dev._lib.kg_set_kernel_variant(dev.handle, 0))
    u0 = _ic() * 1e-303
    assert 0 < np.abs(u0).max() < 1e-301
    dev.u = u0
    ora.set_state(u0)
    for method in ("pirk2", "pirk2", "rk4", "pirk3"):
        getattr(dev, method)()
        ora.step(method, 1)
        assert np.array_equal(dev.u, ora.get_state()), method


def test_state_roundtrip():
    dev, _ = _pair()
    u = _ic()
    dev.u = u
    assert np.array_equal(dev.u, u)
    dev.u_stage = u * 2
    assert np.array_equal(dev.u_stage, u * 2)


@pytest.mark.parametrize("metric", ["Kerr_Schild", "Schw_EF"])
def test_rhs_hook_bitexact(metric):
    dev, ora = _pair(metric=metric)
    rng = np.random.default_rng(7)
    shape = dev.state_shape()
    v = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    for mask in (1, 2, 4, 8, 16, 31):
        a = dev._rhs(mask, v)
        b = ora.rhs(v, mask)
        assert np.array_equal(a, b), f"mask {mask}"


@pytest.mark.parametrize("bc", ["outflow", "inflow"])
def test_boundary_faces_bitexact(bc):
    dev, ora = _pair(bc=bc)
    rng = np.random.default_rng(11)
    shape = dev.state_shape()
    for face in range(6):
        u = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        up = rng.normal(size=shape) + 1j * rng.normal(size=shape)
        dev.u = u
        dev.u_p = up
        ora.set_state(u)
        ora.set_u_p(up)
        dev._ck(dev._lib.kg_boundary(dev.handle, 1 << face))
        ora.boundary(1 << face)
        assert np.array_equal(dev.u, ora.get_state()), f"face {face}"


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("method", ["pirk2", "pirk3", "rk3", "rk4"])
@pytest.mark.parametrize("metric,bc", [("Kerr_Schild", "outflow"), ("Schw_EF", "outflow"),
                                       ("Kerr_Schild", "inflow")])
def test_steppers_bitexact(method, metric, bc, variant):
    dev, ora = _pair(metric=metric, bc=bc)
    dev._ck(dev._lib.kg_set_kernel_variant(dev.handle, variant))
    u0 = _ic()
    dev.u = u0
    ora.set_state(u0)
    for _ in range(3):
        getattr(dev, method)(nsteps=4) if method in ("rk3", "rk4") else getattr(dev, method)(4)
        ora.step(method, 4)
        a, b = dev.u, ora.get_state()
        assert np.array_equal(a, b), f"{method} max diff {np.abs(a - b).max()}"
    if method in ("pirk2", "pirk3"):
        assert np.array_equal(dev.u_stage, ora.get_stage())
    if method == "pirk3":
        assert np.array_equal(dev.u_stage_2, ora.get_stage2())
    assert dev.t == ora.scalars()["t"]


@pytest.mark.parametrize("grid", [SMALL, dict(Nx=61, Ny=13, Nz=41, xmin=1.8, xmax=30.0),
                                  dict(Nx=40, Ny=12, Nz=9, xmin=1.8, xmax=20.0),
                                  dict(Nx=4, Ny=5, Nz=5, xmin=1.8, xmax=6.0),
                                  dict(Nx=12, Ny=7, Nz=8, xmin=1.8, xmax=9.0),
                                  dict(Nx=28, Ny=18, Nz=70, xmin=1.8, xmax=15.0),
                                  dict(Nx=92, Ny=20, Nz=9, xmin=1.8, xmax=30.0),
                                  dict(Nx=26, Ny=11, Nz=9, xmin=1.8, xmax=12.0),
                                  dict(Nx=56, Ny=12, Nz=12, xmin=1.8, xmax=20.0)])
@pytest.mark.parametrize("variant", [1, 2, 3])
def test_march_ragged_tiles(grid, variant):
    """Grids whose r, theta and phi extents leave partial tiles and chunks
    (including a last theta tile of one row) stay bit-exact; the smallest grid
    kg_create accepts (Nx = 4, Ny = Nz = 5) and an even Nz, whose pole partner
    plane k + Nz/2 is not a half turn (the reference's index rule), included.
    Nx = 28 and 92 leave a last r tile of a single column in 32-column tiles
    (33 and 97 stored columns); Ny = 20 puts the last theta row alone in a tile
    of 8 rows; Nz = 70 gives two phi chunks of the fused kernel.  The fused
    PIRK stage 1 (form 3) tiles r by 30 columns and moves its last tile back to
    end at the array's last column: Nx = 26 (31 columns) puts column 0 on the
    left halo lane of that tile, Nx = 56 (61 columns) overlaps it with the
    previous tile by 29 columns, Nx = 4 and 12 fit in one tile, and Ny = 11
    and 12 (16 and 17 stored rows) give theta tiles that meet exactly and that
    overlap by 7 rows."""
    dev, ora = _pair(grid=grid)
    dev._ck(dev._lib.kg_set_kernel_variant(dev.handle, variant))
    from kg_b200.initial_data import shell_ylm
    u0, _ = shell_ylm(grid["Nx"], grid["Ny"], grid["Nz"], grid["xmin"], grid["xmax"], seed=2, r0=5.0, sd=1.0)
    dev.u = u0
    ora.set_state(u0)
    for method in ("pirk2", "pirk3", "rk4"):
        getattr(dev, method)()
        ora.step(method, 1)
        assert np.array_equal(dev.u, ora.get_state()), method


@pytest.mark.parametrize("method", ["pirk2", "pirk3", "rk3", "rk4"])
def test_graph_replay_matches_direct(method):
    """Multi-step calls replay a captured two-step CUDA graph; the result and
    the clock equal step-by-step direct launches."""
    dev_g, ora = _pair()
    dev_d, _ = _pair()
    dev_d._ck(dev_d._lib.kg_set_graphs(dev_d.handle, 0))
    u0 = _ic(seed=8)
    dev_g.u = u0
    dev_d.u = u0
    ora.set_state(u0)
    kw = (lambda n: dict(nsteps=n)) if method.startswith("rk") else (lambda n: dict(nsteps=n))
    getattr(dev_g, method)(**kw(7))
    getattr(dev_g, method)(**kw(4))
    for _ in range(11):
        getattr(dev_d, method)(**kw(1))
    ora.step(method, 11)
    assert np.array_equal(dev_g.u, dev_d.u)
    assert np.array_equal(dev_g.u, ora.get_state())
    assert dev_g.t == dev_d.t == ora.scalars()["t"]


def test_mixed_stepper_sequence():
    """Switching steppers on one handle keeps every hidden stage array exact."""
    dev, ora = _pair()
    u0 = _ic(seed=5)
    dev.u = u0
    ora.set_state(u0)
    for method in ("pirk2", "rk4", "pirk3", "pirk2", "rk3", "pirk3"):
        getattr(dev, method)()
        ora.step(method, 1)
    assert np.array_equal(dev.u, ora.get_state())


def test_c0_1000_steps_pirk2():
    """C0 workload (Nx=256, Ny=33, Nz=65 on r in [1.8, 60], Kerr-Schild M=1,
    m=0, outflow, CFL 0.25 reference dt rule), phi = 1e-3 exp(-(r-10)^2) Y20:
    1000 PIRK2 steps, <= 1e-11 relative L2 in phi and Pi."""
    from kg_b200 import ScalarField
    from kg_b200.initial_data import gaussian_y20
    from oracle.oracle import Oracle, set_threads, max_threads
    set_threads(max_threads())
    g = dict(Nx=256, Ny=33, Nz=65, xmin=1.8, xmax=60.0)
    u0 = gaussian_y20(**g)
    dev = ScalarField(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=0.0)
    dev._ck(dev._lib.kg_set_kernel_variant(dev.handle, 2))
    ora = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], CFL=0.25, m=0.0)
    dev.u = u0
    ora.set_state(u0)
    dev.pirk2(1000)
    ora.pirk2(1000)
    a, b = dev.u, ora.get_state()
    assert rel_l2(a[..., 0], b[..., 0]) <= 1e-11
    assert rel_l2(a[..., 4], b[..., 4]) <= 1e-11
    assert np.array_equal(a, b)


# a radial slab of the benchmark grid: the same theta x phi grid (Ny = 129,
# Nz = 257: 134 stored rows, 258 planes), the same dr (r in [1.8, 400] over
# 2048 cells) and the same ragged last r tile (165 = 5 x 32 + 5, as 2053 =
# 64 x 32 + 5), so the default kernels run with the tiling, phi chunking and
# pole partner planes of the benchmarked solve
C1_SLAB = dict(Nx=160, Ny=129, Nz=257, xmin=1.8, xmax=1.8 + 398.2 * 160 / 2048)


@pytest.mark.parametrize("method,variant", [("pirk2", 2), ("pirk3", 2), ("rk3", 2), ("rk4", 2), ("pirk2", 3),
                                            ("pirk3", 3)])
def test_benchmark_sphere_steppers_bitexact(method, variant):
    """TMA kernels on the benchmark's theta x phi grid, 3 steps of each stepper,
    bit-exact against the oracle (threaded): PIRK2 and PIRK3 with stage 1 as two
    launches (variant 2) and fused (variant 3, the default)."""
    from oracle.oracle import set_threads, max_threads
    set_threads(max_threads())
    g = C1_SLAB
    dev, ora = _pair(grid=g, m=0.3)
    dev._ck(dev._lib.kg_set_kernel_variant(dev.handle, variant))
    from kg_b200.initial_data import shell_ylm
    u0, _ = shell_ylm(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], seed=20240601, r0=12.0, sd=1.0)
    dev.u = u0
    ora.set_state(u0)
    for _ in range(3):
        getattr(dev, method)(nsteps=1) if method.startswith("rk") else getattr(dev, method)(1)
        ora.step(method, 1)
    a, b = dev.u, ora.get_state()
    assert np.array_equal(a, b), f"{method} max diff {np.abs(a - b).max()}"
    if method.startswith("pirk"):
        assert np.array_equal(dev.u_stage, ora.get_stage())


def test_diagnostics_match_oracle():
    dev, ora = _pair(m=0.3, l_max=6, n_det=5)
    u0 = _ic(seed=9)
    dev.u = u0
    ora.set_state(u0)
    dev.pirk2(3)
    ora.pirk2(3)
    dev.density()
    rho_d = dev.rho
    rho_o = ora.density()
    assert rel_l2(rho_d, rho_o) <= 1e-14
    assert abs(dev.mass_scalar() - ora.mass()) <= 1e-12 * abs(ora.mass())
    r_d, i_d = dev.detectors()
    r_o, i_o = ora.detectors()
    assert np.array_equal(r_d, r_o) and np.array_equal(i_d, i_o)
    mom_d = dev.currents_detectors()
    mom_o = ora.currents_detectors()
    assert np.allclose(mom_d, mom_o, rtol=1e-12, atol=1e-14 * np.abs(mom_o).max())
    alm_d = dev.proyector_detectors()
    alm_o = ora.proyector_detectors(6)
    assert np.allclose(alm_d, alm_o, rtol=1e-12, atol=1e-13 * np.abs(alm_o).max())


def test_sph_harmonics_table_matches_oracle():
    dev, ora = _pair(l_max=6)
    assert np.array_equal(dev.sph_harmonics(6), ora.sph_harmonics(6))


def test_profile_and_launch_count():
    dev, _ = _pair()
    dev.u = _ic()
    n0 = dev._lib.kg_launch_count(dev.handle)
    dev._lib.kg_profile_enable(dev.handle, 1)
    dev.pirk2(2)
    import ctypes as C
    nk = dev._lib.kg_profile_kinds()
    ms = (C.c_double * nk)()
    cnt = (C.c_longlong * nk)()
    dev._ck(dev._lib.kg_profile_read(dev.handle, ms, cnt))
    # PIRK2 step of the default form: the fused stage 1, stage 2, two ghost-fill launches
    assert dev._lib.kg_launch_count(dev.handle) - n0 == 2 * 4
    assert cnt[2] == 2 and ms[2] > 0.0
    names = [dev._lib.kg_profile_kind_name(i).decode() for i in range(nk)]
    assert cnt[names.index("stage_pirk_s1_fused")] == 2
    # form 2: stage 1 as two launches (psi, Pi)
    dev._ck(dev._lib.kg_set_kernel_variant(dev.handle, 2))
    n0 = dev._lib.kg_launch_count(dev.handle)
    dev.pirk2(2)
    dev._ck(dev._lib.kg_profile_read(dev.handle, ms, cnt))
    assert dev._lib.kg_launch_count(dev.handle) - n0 == 2 * 5
    assert cnt[0] == 2 and cnt[1] == 2 and cnt[names.index("stage_pirk_s1_fused")] == 0


@pytest.mark.parametrize("grid", [SMALL, dict(Nx=61, Ny=13, Nz=41, xmin=1.8, xmax=30.0),
                                  dict(Nx=12, Ny=7, Nz=8, xmin=1.8, xmax=9.0)])
@pytest.mark.parametrize("metric,bc", [("Kerr_Schild", "outflow"), ("Schw_EF", "inflow")])
def test_rk4_tile_rows_4_bitexact(grid, metric, bc):
    """RK4 stage kernels in 32 x 4 tiles (kg_set_tile_rows): the oracle's bits,
    on grids whose theta extent leaves a partial last tile of 4 rows"""
    dev, ora = _pair(grid=grid, metric=metric, bc=bc)
    dev._ck(dev._lib.kg_set_tile_rows(dev.handle, 4))
    assert dev._lib.kg_get_tile_rows(dev.handle) == 4
    assert dev._lib.kg_set_tile_rows(dev.handle, 6) != 0
    from kg_b200.initial_data import shell_ylm
    u0, _ = shell_ylm(grid["Nx"], grid["Ny"], grid["Nz"], grid["xmin"], grid["xmax"], seed=4, r0=5.0, sd=1.0)
    dev.u = u0
    ora.set_state(u0)
    dev.rk4(nsteps=3)
    ora.rk4(3)
    assert np.array_equal(dev.u, ora.get_state())
