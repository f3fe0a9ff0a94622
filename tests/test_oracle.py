"""CPU tests of the oracle: pinned against the reference's own self-checks,
against an independent whole-array restatement, against scipy, and against
the committed golden fixtures."""
import hashlib
import json
import math
import os

import numpy as np
import pytest

from conftest import ROOT, rel_l2

from oracle.oracle import Oracle, KERR_SCHILD, SCHW_EF, OUTFLOW, INFLOW
from oracle.kg_numpy import NumpyKG
from kg_b200.initial_data import shell_ylm, gaussian_y20

GRID = dict(Nx=16, Ny=9, Nz=17, xmin=1.8, xmax=12.0)


def _ic(seed=3, grid=GRID, r0=6.0):
    u, _ = shell_ylm(grid["Nx"], grid["Ny"], grid["Nz"], grid["xmin"], grid["xmax"], seed=seed, r0=r0, sd=1.0)
    return u


@pytest.mark.parametrize("method", ["pirk2", "pirk3", "rk3", "rk4"])
@pytest.mark.parametrize("metric,bc", [("Kerr_Schild", "outflow"), ("Schw_EF", "outflow"), ("Kerr_Schild", "inflow")])
def test_c_oracle_matches_numpy_restatement(method, metric, bc):
    g = GRID
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], CFL=0.25, m=0.3,
               metric=KERR_SCHILD if metric == "Kerr_Schild" else SCHW_EF,
               bc_rmax=OUTFLOW if bc == "outflow" else INFLOW)
    n = NumpyKG(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=0.3, metric=metric, bc_rmax=bc)
    u0 = _ic()
    o.set_state(u0)
    n.set_state(u0.reshape(-1))
    for _ in range(4):
        o.step(method, 1)
        getattr(n, method)()
    assert np.array_equal(o.get_state().reshape(-1), n.get_state())


def test_rhs_matches_numpy_restatement():
    g = GRID
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], m=0.4)
    n = NumpyKG(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=0.4)
    rng = np.random.default_rng(1)
    shape = (g["Nz"] + 1, g["Ny"] + 5, g["Nx"] + 5, 5)
    v = rng.normal(size=shape) + 1j * rng.normal(size=shape)
    n.set_state(v.reshape(-1))
    r_np = n.rhs_all(n.u)
    r_o = o.rhs(v, 31)
    r_np_f = np.ascontiguousarray(r_np.transpose(3, 2, 1, 0)).reshape(shape)
    assert np.array_equal(r_o, r_np_f)


@pytest.mark.parametrize("metric", [KERR_SCHILD, SCHW_EF])
@pytest.mark.parametrize("grid", [GRID, dict(Nx=64, Ny=17, Nz=33, xmin=1.8, xmax=60.0)])
def test_inverse_metric_identity(metric, grid):
    """validate_inverse_metric (MoL/geometry.f90:409-492): zero errors at 1e-10."""
    o = Oracle(grid["Nx"], grid["Ny"], grid["Nz"], grid["xmin"], grid["xmax"], metric=metric)
    assert o.validate_inverse_metric() == (0, 0)


def test_schwarzschild_closed_form():
    """For a = 0 the Kerr-Schild lapse, shift and 3-metric have closed forms."""
    g = GRID
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"])
    mt = o.metric()
    sc = o.scalars()
    x = sc["xmin"] + np.arange(g["Nx"] + 5) * sc["dx"]
    y = -sc["dy"] / 2 + np.arange(-2, g["Ny"] + 3) * sc["dy"]
    y[-1] = y[-2]  # boundary_theta_dn / up copy the last theta row
    X, Yv = np.meshgrid(x, y)
    assert np.allclose(mt[0], 1.0 / np.sqrt(1.0 + 2.0 / X), rtol=1e-14)          # alpha
    assert np.allclose(mt[1], (2.0 / X) / (1.0 + 2.0 / X), rtol=1e-13)            # beta^r
    assert np.allclose(mt[3], X ** 2 * np.abs(np.sin(Yv)) * np.sqrt(1 + 2.0 / X), rtol=1e-13)
    assert np.allclose(mt[4], 1.0 / (1.0 + 2.0 / X), rtol=1e-13)                  # gamma^rr
    assert np.all(mt[5] == 0.0)                                                    # gamma^rphi


def test_ylm_analytic_l2():
    """The analytic l <= 2 harmonics of tools/harmonics.f90:55-65 (Condon-Shortley)."""
    o = Oracle(16, 33, 65, 1.8, 12.0)
    L = 2
    Y = o.sph_harmonics(L)
    sc = o.scalars()
    th = np.arange(33) * sc["dy"]
    ph = np.arange(65) * sc["dz"]
    P, T = np.meshgrid(ph, th, indexing="ij")
    pi = math.acos(-1.0)
    ana = {
        (0, 0): 0.5 / np.sqrt(pi) * np.ones_like(T),
        (1, 1): -np.sqrt(3.0 / (8.0 * pi)) * np.exp(1j * P) * np.sin(T),
        (1, 0): np.sqrt(3.0 / (4.0 * pi)) * np.cos(T),
        (2, 2): np.sqrt(15.0 / (32.0 * pi)) * np.exp(2j * P) * np.sin(T) ** 2,
        (2, 1): -np.sqrt(15.0 / (8.0 * pi)) * np.exp(1j * P) * np.sin(T) * np.cos(T),
        (2, 0): np.sqrt(5.0 / (16.0 * pi)) * (3.0 * np.cos(T) ** 2 - 1.0),
    }
    for (l, m), a in list(ana.items()):
        if m > 0:
            ana[(l, -m)] = (-1.0) ** m * np.conj(a)
    interior = slice(1, -1)  # the reference's pole rule replaces P_lm at theta = 0, pi
    for (l, m), a in ana.items():
        got = Y[:, :, m + L, l]
        assert np.allclose(got[:, interior], a[:, interior], atol=1e-14), (l, m)


def test_ylm_vs_scipy_golden():
    d = np.load(os.path.join(ROOT, "tests", "golden", "ylm_scipy.npz"))
    o = Oracle(16, int(d["Ny"]), int(d["Nz"]), 1.8, 12.0)
    L = int(d["L"])
    Y = o.sph_harmonics(L)
    ref = d["Y"]
    assert np.allclose(Y[:, 1:-1], ref[:, 1:-1], atol=1e-13)
    # pole rows follow the reference's rule: Y_l0 = fact^2, Y_lm = 0 (m != 0)
    pi = math.acos(-1.0)
    for l in range(L + 1):
        fact = math.sqrt((2 * l + 1) / (4 * pi))
        for m in range(-l, l + 1):
            want = fact * fact if m == 0 else 0.0
            assert np.allclose(Y[:, 0, m + L, l], want, atol=1e-15)


def test_ylm_orthonormality():
    """test_orthonormality (tools/FFT_sph.f90:338-406): trapezium inner products
    of Y_lm with l2 <= l1+1 against the identity.

    The reference's tolerance of 1e-5 cannot be met by its own table: the
    theta trapezium is second order, and below dtheta = 0.0141 the pole rule
    (|cos theta| > 0.9999 -> Y_l0 = fact^2, FFT_sph.f90:320-321) reaches
    interior rows.  The check runs on a sphere where the pole rule touches
    only the pole rows (Ny = 201) and pins the normalisation through the
    Euler-Maclaurin error of the rule: for m1 = m2 = 0 the entry is
    delta - (dtheta^2/12) 2 pi [F(0) + F(pi)] with F = Y_l1,0 Y_l2,0, to within
    1e-3 dtheta^2; every other entry is within dtheta^2 / 10 of the identity."""
    Ny, Nz, L = 201, 129, 4
    o = Oracle(4, Ny, Nz, 1.8, 12.0, n_det=2)
    Y = o.sph_harmonics(L)
    sc = o.scalars()
    th = np.arange(Ny) * sc["dy"]
    w = np.ones((Nz, Ny))
    w[:, 0] *= 0.5
    w[:, -1] *= 0.5
    w[0, :] *= 0.5
    w[-1, :] *= 0.5
    w = w * np.sin(th)[None, :] * sc["dy"] * sc["dz"]
    for l1 in range(L + 1):
        for m1 in range(-l1, l1 + 1):
            for l2 in range(0, min(l1 + 1, L) + 1):
                for m2 in range(-l2, l2 + 1):
                    v = abs(np.sum(np.conj(Y[:, :, m1 + L, l1]) * Y[:, :, m2 + L, l2] * w))
                    h2 = sc["dy"] ** 2
                    if m1 == m2 == 0:
                        # T - I = -(h^2/12) 2pi [F(0) + F(pi)], F = Y_l1,0 Y_l2,0
                        c = math.sqrt((2 * l1 + 1) * (2 * l2 + 1)) * (1 + (-1) ** (l1 + l2)) / 2.0
                        pred = (1.0 if l1 == l2 else 0.0) - h2 / 12.0 * c
                        assert abs(v - abs(pred)) <= 1e-3 * h2, (l1, l2, v, pred)
                    else:
                        want = 1.0 if (l1 == l2 and m1 == m2) else 0.0
                        assert abs(v - want) <= h2 / 10, (l1, m1, l2, m2, v)


def test_stencils_exact_on_quadratics():
    """Second-order operators differentiate quadratics exactly (interior and one-sided)."""
    n = NumpyKG(16, 9, 17, 1.8, 12.0, 0.25)
    x = n.x[:, None, None] * np.ones((1, n.NJ, n.NK))
    f = (0.3 * x ** 2 - 1.7 * x + 0.2).astype(np.complex128)
    assert np.allclose(n.dx1(f, n.dx), 0.6 * x - 1.7, atol=1e-11)
    beta = np.ones((n.NI, n.NJ, 1))
    assert np.allclose(n.ad1(f, beta, n.dx), 0.6 * x - 1.7, atol=1e-11)
    z = np.arange(n.NK) * n.dz
    fz = (0.5 * z ** 2 + z)[None, None, :] * np.ones((n.NI, n.NJ, 1))
    d = n.dx3(fz.astype(np.complex128), n.dz)
    assert np.allclose(d[:, :, 1:-1], (z[1:-1] + 1.0)[None, None, :], atol=1e-11)


@pytest.mark.parametrize("case", ["Kerr_Schild/pirk2", "Kerr_Schild/pirk3", "Kerr_Schild/rk3", "Kerr_Schild/rk4",
                                  "Schw_EF/pirk2", "Schw_EF/pirk3", "Schw_EF/rk3", "Schw_EF/rk4"])
def test_oracle_golden(case):
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_small.json")))
    g = d["grid"]
    u0, _ = shell_ylm(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], seed=d["seed"], r0=d["r0"], sd=d["sd"])
    assert hashlib.sha256(np.ascontiguousarray(u0).tobytes()).hexdigest() == d["ic_sha256"]
    metric, method = case.split("/")
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], CFL=d["CFL"], m=d["m"],
               metric=KERR_SCHILD if metric == "Kerr_Schild" else SCHW_EF)
    o.set_state(u0)
    o.step(method, d["steps"])
    u = o.get_state()
    c = d["cases"][case]
    assert hashlib.sha256(np.ascontiguousarray(u).tobytes()).hexdigest() == c["sha256"]
    flat = u.reshape(-1)
    vals = np.array([complex(a, b) for a, b in c["vals"]])
    assert np.array_equal(flat[c["idx"]], vals)


def test_pirk2_uses_previous_stage_pi():
    """rhs_pi of PIRK stage 1 reads u_stage(5) of the previous step
    (MoL/lines_method_lib.f90:288): seeding a different stale stage changes the step."""
    g = GRID
    u0 = _ic()
    a = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], m=0.3)
    b = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], m=0.3)
    a.set_state(u0)
    b.set_state(u0)
    stale = u0.copy()
    stale[..., 4] = u0[..., 0]  # a nonzero stale Pi
    b.set_stage(stale)
    a.pirk2(1)
    b.pirk2(1)
    assert not np.array_equal(a.get_state(), b.get_state())


def test_c0_dt_rule():
    """dt = CFL min(dr, e^xmin dtheta, e^xmin sin(dtheta/2) dphi), MoL/diagnostic_lib.f90:103."""
    o = Oracle(256, 33, 65, 1.8, 60.0, CFL=0.25)
    sc = o.scalars()
    dy, dz = math.pi / 32, 2 * math.pi / 64
    want = 0.25 * min(58.2 / 256, math.exp(1.8) * dy, math.exp(1.8) * math.sin(dy / 2) * dz)
    assert abs(sc["dt"] - want) < 1e-15
    assert abs(sc["dt"] - 0.007285602030047707) < 1e-15


def test_detectors_and_mass():
    g = GRID
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], m=0.3, n_det=5)
    r, idx = o.detectors()
    assert r[0] == 2.0 and abs(r[-1] - 0.99 * 12.0) < 1e-15
    # the vertex grid r(i) = xmin + (i-1) dr ends at r(Nx) < 0.99 xmax here, so the
    # last detector lies outside it and is skipped, as in the reference
    assert np.all(idx[:-1] > 0) and idx[-1] == 0
    o.set_state(_ic())
    m = o.mass()
    assert np.isfinite(m) and m > 0


def test_all_shell_projection_contains_detector_projection():
    """project_all_shells at shell index_det is proyector_detectors at that detector"""
    g = GRID
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], m=0.3, n_det=5)
    o.set_state(_ic())
    _, idx = o.detectors()
    a_det = o.proyector_detectors(6)
    a_all = o.project_all_shells(6)
    assert a_all.shape == (g["Nx"], 13, 7)
    for d, iv in enumerate(idx):
        if iv > 0:
            assert np.array_equal(a_det[d], a_all[iv - 1])


def test_shell_subset_projection_equals_all_shells():
    """project_shells (Y_lm formed per mode, threaded) gives the same bits as
    the rows of project_all_shells (stored Y_lm table)"""
    g = GRID
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], m=0.3)
    o.set_state(_ic())
    a_all = o.project_all_shells(7)
    shells = [1, 3, g["Nx"]]
    a_sub = o.project_shells(7, shells)
    for q, iv in enumerate(shells):
        assert np.array_equal(a_sub[q], a_all[iv - 1])


def test_spherical_bessel_against_scipy():
    """j_l (gsl_sf_bessel_jl in the reference, tools/FFT_sph.f90:29-34) against
    scipy, relative to the function's envelope (|j_l| below l, sqrt(j_l^2 + y_l^2) above)"""
    from scipy.special import spherical_jn, spherical_yn
    from oracle.oracle import sph_jl
    worst = 0.0
    for l in list(range(0, 12)) + [20, 33, 47, 64, 90, 128]:
        for x in np.concatenate([np.geomspace(1e-3, 1.0, 9), np.linspace(1.0, 420.0, 160)]):
            b = spherical_jn(l, x)
            if abs(b) < 1e-250:
                continue
            env = abs(b) if x < l else math.hypot(b, spherical_yn(l, x))
            worst = max(worst, abs(sph_jl(l, x) - b) / env)
    assert worst < 1e-12, worst


def test_spherical_bessel_zeros_against_scipy():
    """zeros of j_l (gsl_sf_bessel_zero_Jnu(l + 1/2, n), tools/FFT_sph.f90:22-27)
    against scipy's brentq on spherical_jn"""
    from scipy.optimize import brentq
    from scipy.special import spherical_jn
    from oracle.oracle import sph_jl_zeros
    z = sph_jl_zeros(64, 100)
    for l in (0, 1, 2, 7, 10, 33, 64):
        for n in (1, 2, 3, 50, 99, 100):
            zz = z[l, n - 1]
            r = brentq(lambda x: spherical_jn(l, x), zz - 0.05, zz + 0.05, xtol=1e-15, rtol=1e-15)
            assert abs(zz - r) <= 4e-15 * r, (l, n, zz, r)
    # strictly increasing in n, interlaced in l
    assert np.all(np.diff(z, axis=1) > 0)
    assert np.all(z[1:, :-1] > z[:-1, :-1]) and np.all(z[1:, :-1] < z[:-1, 1:])


def test_bessel_basis_normalised_and_radial_transform_against_numpy():
    """generate_full_bessel_basis (tools/FFT_sph.f90:13-95): each basis function
    has unit trapezium norm with weight r^2; SphFT_discrete_radial
    (tools/FFT_sph.f90:213-244) equals a numpy trapezium of the oracle's
    all-shell projection against a basis built from scipy's j_l and zeros."""
    from scipy.optimize import brentq
    from scipy.special import spherical_jn
    g = GRID
    L, Nk = 4, 12
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], m=0.3)
    o.set_state(_ic())
    k, jb = o.bessel_basis(L, Nk)
    sc = o.scalars()
    r = g["xmin"] + np.arange(g["Nx"]) * sc["dx"]
    dr = abs(r[1] - r[0])
    w = np.full(g["Nx"], dr)
    w[[0, -1]] *= 0.5
    norms = np.einsum("i,inl,inl->nl", w * r ** 2, jb, jb)
    assert np.allclose(norms, 1.0, rtol=0, atol=1e-13)
    # independent basis
    r_max = g["xmin"] + (g["Nx"] + 4) * sc["dx"]
    jb_s = np.zeros_like(jb)
    for l in range(L + 1):
        zs = []
        x = 0.5
        while len(zs) < Nk:
            if spherical_jn(l, x) * spherical_jn(l, x + 0.05) < 0:
                zs.append(brentq(lambda t: spherical_jn(l, t), x, x + 0.05, xtol=1e-15, rtol=1e-15))
            x += 0.05
        for n, zz in enumerate(zs):
            assert abs(k[n, l] - zz / r_max) <= 1e-14 * k[n, l]
            v = spherical_jn(l, zz / r_max * r)
            jb_s[:, n, l] = v / math.sqrt(np.sum(w * (v * r) ** 2))
    assert np.abs(jb - jb_s).max() <= 1e-11 * np.abs(jb_s).max()
    flm = o.project_all_shells(L)                          # (Nx, 2L+1, L+1)
    ft_np = np.einsum("i,iml,inl->mln", w * r ** 2, flm, jb_s)
    ft = o.sph_ft_radial(L, Nk)
    assert np.abs(ft - ft_np).max() <= 1e-11 * np.abs(ft_np).max()


def _cfg_run(level, T, dt, base=32, tb=8):
    from kg_b200.initial_data import smooth_exact
    Nx, Nth = base * 2 ** level, tb * 2 ** level
    Ny, Nz = Nth + 1, 2 * Nth + 1
    o = Oracle(Nx, Ny, Nz, 1.8, 20.0, CFL=0.25, m=0.2, dt_override=dt)
    o.set_scheme(1, 0.02)
    o.set_state(smooth_exact(Nx, Ny, Nz, 1.8, 20.0))
    o.boundary_cfg()
    o.rk4(int(round(T / dt)))
    sc = o.scalars()
    return o.get_state()[..., 0], sc["dx"]


def cfg_rms_diff(fine, coarse, dx_c):
    """RMS of coarse - fine on common points in 5 <= r <= 15: r and phi nest;
    theta is cell-centred, so the fine rows are interpolated to the coarse
    centre with the fourth-order weights (-1, 9, 9, -1)/16"""
    Kc, Jc, Ic = coarse.shape
    ii = np.arange(Ic)
    sel = (1.8 + ii * dx_c >= 5.0) & (1.8 + ii * dx_c <= 15.0)
    out = []
    for kc in range(1, Kc - 1):
        for jc in range(4, Jc - 4):
            f = (-fine[2 * kc, 2 * jc - 4] + 9 * fine[2 * kc, 2 * jc - 3] + 9 * fine[2 * kc, 2 * jc - 2]
                 - fine[2 * kc, 2 * jc - 1]) / 16
            out.append(coarse[kc, jc, sel] - f[2 * ii[sel]])
    d = np.concatenate(out)
    return float(np.sqrt(np.mean(np.abs(d) ** 2)))


def test_configured_method_converges_faster_than_second_order():
    """The configured fourth-order method (oracle): on three coarse resolutions
    (8, 16, 32 theta cells) the self-convergence factor is about 13, far above
    the second-order 4; the fourth-order 16 is approached on finer grids, which
    the GPU test runs (14.7 there)."""
    T = 0.3
    dt = 0.25 * math.exp(1.8) * math.sin(math.pi / 32 / 2) * (2 * math.pi / 64)
    runs = [_cfg_run(l, T, dt) for l in range(3)]
    e01 = cfg_rms_diff(runs[1][0], runs[0][0], runs[0][1])
    e12 = cfg_rms_diff(runs[2][0], runs[1][0], runs[1][1])
    assert np.all(np.isfinite(runs[2][0]))
    assert e01 / e12 > 11.0, e01 / e12


def test_configured_method_rejects_other_metric_forms():
    g = GRID
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], metric=SCHW_EF)
    with pytest.raises(ValueError):
        o.set_scheme(1)


@pytest.mark.parametrize("grid", [dict(Nx=24, Ny=17, Nz=33), dict(Nx=37, Ny=13, Nz=25), dict(Nx=12, Ny=9, Nz=8)])
def test_configured_method_c_matches_numpy_restatement(grid):
    """The configured fourth-order method has no reference code; its C
    restatement (the GPU's parity target) and an independent whole-array numpy
    restatement of the same definition agree bit for bit over several RK4
    steps, on grids with odd and even Nz."""
    from kg_b200.initial_data import smooth_exact
    Nx, Ny, Nz = grid["Nx"], grid["Ny"], grid["Nz"]
    o = Oracle(Nx, Ny, Nz, 1.8, 20.0, CFL=0.25, m=0.2)
    o.set_scheme(1, 0.02)
    n = NumpyKG(Nx, Ny, Nz, 1.8, 20.0, 0.25, m=0.2)
    n.set_scheme_cfg(0.02)
    u0 = smooth_exact(Nx, Ny, Nz, 1.8, 20.0, amp=1e-3)
    o.set_state(u0)
    o.boundary_cfg()
    n.set_state(u0.reshape(-1))
    n.boundary_cfg()
    assert np.array_equal(o.get_state().reshape(-1), n.get_state())
    for _ in range(3):
        o.rk4(1)
        n.rk4_cfg()
        assert np.array_equal(o.get_state().reshape(-1), n.get_state())
    assert np.abs(n.u).max() > 0


@pytest.mark.parametrize("metric", ["Kerr_Schild", "Schw_EF"])
def test_density_and_mass_c_match_numpy_restatement(metric):
    """The diagnostics the GPU is checked against (density and the nested
    trapezium of rho sqrt(gamma)) agree bit for bit between the C oracle and
    the independent numpy restatement, on an evolved state."""
    g = GRID
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], CFL=0.25, m=0.3,
               metric=KERR_SCHILD if metric == "Kerr_Schild" else SCHW_EF)
    n = NumpyKG(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=0.3, metric=metric)
    u0 = _ic(seed=9)
    o.set_state(u0)
    n.set_state(u0.reshape(-1))
    for _ in range(2):
        o.step("pirk2", 1)
        n.pirk2()
    rho_o = o.density()
    rho_n = n.density().transpose(2, 1, 0)
    assert np.array_equal(rho_o, rho_n)
    assert o.mass() == n.mass()


@pytest.mark.parametrize("metric", ["Kerr_Schild", "Schw_EF"])
def test_detector_diagnostics_c_match_numpy_restatement(metric):
    """domain_to_sph (index search and trilinear interpolation), project_sh and
    the detector currents agree bit for bit between the C oracle and the numpy
    restatement on an evolved state (the Y_lm table is the C oracle's, pinned to
    scipy elsewhere); the last detector lies outside the vertex grid and stays 0."""
    g = GRID
    L, nd = 4, 5
    o = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], CFL=0.25, m=0.3, n_det=nd, l_max=L,
               metric=KERR_SCHILD if metric == "Kerr_Schild" else SCHW_EF)
    n = NumpyKG(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=0.3, metric=metric)
    o.set_state(_ic(seed=11))
    o.step("pirk2", 2)
    n.set_state(o.get_state().reshape(-1))
    r_o, idx_o = o.detectors()
    r_n, idx_n = n.detectors(nd)
    assert np.array_equal(r_o, r_n) and np.array_equal(idx_o, idx_n)
    a_o = o.proyector_detectors(L)
    a_n = n.proyector_detectors(o.sph_harmonics(L), L, nd)
    assert np.array_equal(a_o, a_n)
    assert np.abs(a_n[:-1]).max() > 0 and not np.any(a_n[-1])
    m_o = o.currents_detectors()
    m_n = n.currents_detectors(nd)
    assert np.array_equal(m_o, m_n)
    assert np.abs(m_n[:-1]).max() > 0
