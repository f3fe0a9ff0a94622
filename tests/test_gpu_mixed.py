"""GPU tests of the mixed-precision RK4 (FP32 stencil RHS on FP32 stage states,
FP64 state update u^n + (k1 + 2k2 + 2k3 + k4)/6, FP64 RHS on the excision planes
and next to the poles).  The FP64 path is bit-exact to the oracle; the mixed
path is held to an error bound against it and must be deterministic, equal
under graph replay and equal alone and in a batch."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [dict(Nx=48, Ny=17, Nz=33, xmin=1.8, xmax=11.4, m=0.3, seed=5),
          dict(Nx=40, Ny=13, Nz=25, xmin=1.8, xmax=9.8, m=0.1, seed=6),
          dict(Nx=33, Ny=9, Nz=17, xmin=1.8, xmax=20.0, m=0.45, seed=7)]


def _solve(sp, precision="fp64", metric="Kerr_Schild", bc="outflow"):
    from kg_b200 import ScalarField
    from kg_b200.initial_data import shell_ylm
    s = ScalarField(sp["Nx"], sp["Ny"], sp["Nz"], sp["xmin"], sp["xmax"], 0.25, m=sp["m"], metric=metric,
                    boundary_type_rmax=bc, l_max=8, n_det=3)
    u0, _ = shell_ylm(sp["Nx"], sp["Ny"], sp["Nz"], sp["xmin"], sp["xmax"], seed=sp["seed"],
                      r0=0.5 * (sp["xmin"] + sp["xmax"]), sd=1.0)
    s.u = u0
    s.precision = precision
    return s


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("metric,bc", [("Kerr_Schild", "outflow"), ("Schw_EF", "outflow"),
                                       ("Kerr_Schild", "inflow")])
def test_mixed_rk4_close_to_fp64(metric, bc):
    sp = SHAPES[0]
    a = _solve(sp, "fp64", metric, bc)
    b = _solve(sp, "mixed", metric, bc)
    assert b.precision == "mixed"
    a.rk4(nsteps=100)
    b.rk4(nsteps=100)
    ua, ub = a.u, b.u
    assert np.all(np.isfinite(ub))
    e_phi, e_pi = _rel(ub[..., 0], ua[..., 0]), _rel(ub[..., 4], ua[..., 4])
    print(f"{metric}/{bc}: 100 mixed RK4 steps, rel L2 error phi {e_phi:.2e}, Pi {e_pi:.2e}")
    assert 0 < e_phi <= 1e-6 and 0 < e_pi <= 1e-6


def test_mixed_rk4_deterministic_and_graph_replay():
    sp = SHAPES[1]
    a = _solve(sp, "mixed")
    b = _solve(sp, "mixed")
    a.rk4(nsteps=9)            # graph replay of step pairs
    for _ in range(9):
        b.rk4(nsteps=1)        # direct launches
    assert np.array_equal(a.u, b.u)
    assert a.t == b.t


def test_mixed_batch_equals_solo():
    from kg_b200.batch import Batch
    batch = Batch(precision="mixed")
    members = [_solve(sp, "fp64") for sp in SHAPES]   # batch precision governs members
    solos = [_solve(sp, "mixed") for sp in SHAPES]
    for m in members:
        batch.add(m)
    batch.rk4(1)
    batch.rk4(6)
    for s in solos:
        s.rk4(nsteps=7)
    for m, s in zip(members, solos):
        assert np.array_equal(m.u, s.u)


def test_mixed_waveform_error_at_detectors():
    """l <= 8 detector waveform of the mixed form against FP64 over 300 steps"""
    sp = SHAPES[0]
    a = _solve(sp, "fp64")
    b = _solve(sp, "mixed")
    wa, wb = [], []
    for _ in range(30):
        a.rk4(nsteps=10)
        b.rk4(nsteps=10)
        wa.append(a.proyector_detectors().copy())
        wb.append(b.proyector_detectors().copy())
    wa, wb = np.array(wa), np.array(wb)
    err = _rel(wb, wa)
    print(f"waveform rel L2 error (300 steps, l<=8, 3 detectors): {err:.2e}")
    assert err <= 1e-6


def test_mixed_tile_rows_same_bits():
    """the mixed stages in 32 x 4 tiles give the bits of the 32 x 8 tiles"""
    out = []
    for rows in (8, 4):
        s = _solve(SHAPES[1], "mixed")
        s._ck(s._lib.kg_set_tile_rows(s.handle, rows))
        s.rk4(nsteps=6)
        out.append(s.u)
    assert np.array_equal(out[0], out[1])
