"""GPU test of the reference-format diagnostics writer (kg_b200.output) driven
by a real solve: PIRK2 steps on the device, `diagnostic(l)` after each, and the
files of save_gnuplot (main/save_gnuplot.f90:15-72: Mass_scalar.t.asc and the
detector currents jr/jtheta/jphi_NN.t.asc every save_0d steps) and of savealm
(IO/save_data.f90:54-110: Harmonic_coeficientsNN.lm.asc every `save` steps).
Every row read back from the files is compared with the same quantity from the
oracle, stepped alongside: times exactly, Mass_scalar and currents to 1e-12
relative, a_lm to 1e-12 of the block's largest coefficient.  The reference's
diagnostic integrates rho as it stands (its call to density() is commented
out, MoL/diagnostic_lib.f90:211), so the driver here refreshes rho with
density() before each diagnostic, as the oracle's mass does."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = dict(Nx=48, Ny=17, Nz=33, xmin=1.8, xmax=14.0)


def test_writer_rows_match_the_oracle(tmp_path):
    from kg_b200 import ScalarField
    from kg_b200.initial_data import shell_ylm
    from kg_b200.output import DiagnosticWriter, read_lm
    from oracle.oracle import Oracle
    L = 6
    s = ScalarField(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"], 0.25, m=0.3, n_det=4, l_max=L)
    ora = Oracle(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"], CFL=0.25, m=0.3, n_det=4, l_max=L)
    u0, _ = shell_ylm(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"], seed=31, r0=6.0, sd=1.0)
    s.u = u0
    ora.set_state(u0)
    w = DiagnosticWriter(s, str(tmp_path), save_0d=1, save=2)
    want_mass, want_mom, want_alm, times = [], [], [], []
    nsteps = 6
    for l in range(1, nsteps + 1):
        s.pirk2()
        ora.pirk2(1)
        s.density()
        s.diagnostic(l)
        w.step(l)
        times.append(ora.scalars()["t"])
        ora.density()
        want_mass.append(ora.mass())
        want_mom.append(ora.currents_detectors())
        if l % 2 == 0:
            want_alm.append(ora.proyector_detectors(L))
    m = np.loadtxt(tmp_path / "Mass_scalar.t.asc")
    assert m.shape == (nsteps, 2)
    assert np.array_equal(m[:, 0], np.array(times))
    assert np.allclose(m[:, 1], want_mass, rtol=1e-12, atol=0.0)
    inside = [d for d, _ in w._inside_evolution_grid()]
    assert inside
    for d in inside:
        for c, name in enumerate(("jr_", "jtheta_", "jphi_")):
            rows = np.loadtxt(tmp_path / f"{name}{d + 1:02d}.t.asc")
            assert np.array_equal(rows[:, 0], np.array(times))
            ref = np.array([mm[d, c] for mm in want_mom])
            scale = max(np.abs(np.array(want_mom)).max(), 1e-300)
            assert np.allclose(rows[:, 1], ref, rtol=1e-12, atol=1e-14 * scale), (name, d)
    lm_files = sorted(f for f in os.listdir(tmp_path) if f.startswith("Harmonic_coeficients"))
    assert lm_files
    for f in lm_files:
        d = int(f[len("Harmonic_coeficients"):len("Harmonic_coeficients") + 2]) - 1
        blocks = read_lm(str(tmp_path / f))
        assert len(blocks) == nsteps // 2
        for b, (ll, mm, a) in enumerate(blocks):
            ref = np.array([want_alm[b][d, m + L, l] for l in range(L + 1) for m in range(-l, l + 1)])
            assert list(ll) == [l for l in range(L + 1) for _ in range(-l, l + 1)]
            assert list(mm) == [m for l in range(L + 1) for m in range(-l, l + 1)]
            scale = max(np.abs(ref).max(), 1e-300)
            assert np.abs(a - ref).max() <= 1e-12 * scale, (f, b)
    s.close()
