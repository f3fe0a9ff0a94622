"""CPU tests of the reference-format diagnostics writer (kg_b200.output) with a
stand-in solver: file names, row layout and the detector selection of
save_gnuplot (main/save_gnuplot.f90:15-72) and savealm (IO/save_data.f90:54-110)."""
import os
import types

import numpy as np

from kg_b200.output import DiagnosticWriter, read_lm


class _Fake:
    def __init__(self):
        self.Nx, self.g_pts, self.dx = 16, 2, 0.5
        self.params = types.SimpleNamespace(xmin=1.8)
        self.t, self.Mass_scalar = 0.25, 1.5e-3
        self.r_det = np.array([2.0, 5.0, 30.0])   # the last one is outside
        L = 3
        rng = np.random.default_rng(1)
        self.alm = rng.standard_normal((3, 2 * L + 1, L + 1)) + 1j * rng.standard_normal((3, 2 * L + 1, L + 1))
        self.mom = rng.standard_normal((3, 3))

    def detectors(self):
        return self.r_det, np.array([1, 7, 0])

    def currents_detectors(self):
        return self.mom

    def proyector_detectors(self):
        return self.alm


def test_writer_files_and_rows(tmp_path):
    s = _Fake()
    w = DiagnosticWriter(s, str(tmp_path), save_0d=1, save=2)
    w.step(1)
    s.t = 0.5
    w.step(2)
    names = sorted(os.listdir(tmp_path))
    assert "Mass_scalar.t.asc" in names
    assert "jr_01.t.asc" in names and "jphi_02.t.asc" in names and "jr_03.t.asc" not in names
    assert names.count("Harmonic_coeficients01.lm.asc") == 1 and "Harmonic_coeficients03.lm.asc" not in names
    m = np.loadtxt(tmp_path / "Mass_scalar.t.asc")
    assert m.shape == (2, 2) and m[1, 0] == 0.5 and m[0, 1] == 1.5e-3
    jt = np.loadtxt(tmp_path / "jtheta_02.t.asc")
    assert jt[1, 1] == s.mom[1, 1]
    blocks = read_lm(str(tmp_path / "Harmonic_coeficients02.lm.asc"))
    assert len(blocks) == 1                       # saved at step 2 only
    l, mm, a = blocks[0]
    assert list(l[:4]) == [0, 1, 1, 1] and list(mm[:4]) == [0, -1, 0, 1]
    L = 3
    want = np.array([s.alm[1, m + L, ll] for ll in range(L + 1) for m in range(-ll, ll + 1)])
    assert np.array_equal(a, want)               # 17 significant digits read back exactly
