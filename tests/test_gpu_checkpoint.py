"""GPU tests of checkpoint/resume (kg_save_checkpoint / kg_load_checkpoint, the
complete binary form of check_point / read_from_check_point,
MoL/lines_method_lib.f90:599-667): a run interrupted by save + load into a new
handle continues bit for bit, PIRK stage state included."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

G = dict(Nx=40, Ny=13, Nz=25, xmin=1.8, xmax=9.8)


def _solver():
    from kg_b200 import ScalarField
    from kg_b200.initial_data import shell_ylm
    s = ScalarField(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"], 0.25, m=0.3)
    u0, _ = shell_ylm(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"], seed=4, r0=5.0, sd=1.0)
    s.u = u0
    return s


@pytest.mark.parametrize("method", ["pirk2", "pirk3", "rk4"])
def test_resume_is_bitexact(tmp_path, method):
    from kg_b200 import ScalarField
    step = (lambda s, n: getattr(s, method)(nsteps=n)) if method.startswith("rk") else \
        (lambda s, n: getattr(s, method)(n))
    a = _solver()
    step(a, 3)
    path = tmp_path / "ckpt.bin"
    a.check_point(path)
    step(a, 4)
    b = ScalarField(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"], 0.25, m=0.3)
    b.read_from_check_point(path)
    step(b, 4)
    assert np.array_equal(a.u, b.u)
    assert a.t == b.t


def test_checkpoint_grid_mismatch_is_rejected(tmp_path):
    from kg_b200 import ScalarField, KgError
    a = _solver()
    path = tmp_path / "ckpt.bin"
    a.check_point(path)
    c = ScalarField(G["Nx"] + 8, G["Ny"], G["Nz"], G["xmin"], G["xmax"], 0.25, m=0.3)
    with pytest.raises(KgError):
        c.read_from_check_point(path)
    with pytest.raises(KgError):
        c.read_from_check_point(tmp_path / "missing.bin")


def test_async_snapshots_match_the_state_at_their_step(tmp_path):
    from kg_b200.output import AsyncSnapshots
    a = _solver()
    snaps = AsyncSnapshots(a, str(tmp_path), depth=2)
    want = {}
    for i in range(1, 7):
        a.pirk2(1)
        if i % 2 == 0:
            snaps.snap(i)
            want[i] = (a.u.copy(), a.t)
    snaps.close()
    for i, (u, t) in want.items():
        got = np.load(tmp_path / f"u_{i:08d}.npy")
        assert np.array_equal(got, u)
        assert float(open(tmp_path / f"u_{i:08d}.t").read()) == t


def test_load_without_stage_state_matches_a_fresh_handle(tmp_path):
    """A checkpoint saved before any PIRK step holds no stage arrays; loading it
    into a handle that has already run PIRK must reset the stale Pi slot, so the
    continuation equals the one of a freshly created handle."""
    from kg_b200 import ScalarField
    fresh_src = _solver()
    path = tmp_path / "nostage.bin"
    fresh_src.check_point(path)  # u only: this handle never ran PIRK
    used = _solver()
    used.pirk3(3)  # fills u_stage, u_stage_2 and moves both Pi slots
    used.read_from_check_point(path)
    fresh = ScalarField(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"], 0.25, m=0.3)
    fresh.read_from_check_point(path)
    for s in (used, fresh):
        s.pirk2(2)
        s.pirk3(2)
    assert np.array_equal(used.u, fresh.u)
    assert used.t == fresh.t


def test_checkpoint_parameter_mismatch_is_rejected(tmp_path):
    from kg_b200 import ScalarField, KgError
    a = _solver()
    path = tmp_path / "ckpt.bin"
    a.check_point(path)
    others = [
        dict(metric="Schw_EF"),
        dict(m=0.2),
        dict(boundary_type_rmax="inflow"),
    ]
    for kw in others:
        kw = dict(dict(m=0.3), **kw)
        c = ScalarField(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"], 0.25, **kw)
        with pytest.raises(KgError):
            c.read_from_check_point(path)
    c = ScalarField(G["Nx"], G["Ny"], G["Nz"], G["xmin"], G["xmax"] + 10.0, 0.25, m=0.3)
    with pytest.raises(KgError, match="radial extent"):
        c.read_from_check_point(path)


def test_truncated_checkpoint_leaves_the_handle_untouched(tmp_path):
    from kg_b200 import KgError
    a = _solver()
    a.pirk2(2)
    path = tmp_path / "ckpt.bin"
    a.check_point(path)
    data = path.read_bytes()
    cut = tmp_path / "cut.bin"
    cut.write_bytes(data[: len(data) - 1024])
    b = _solver()
    b.rk4(nsteps=1)
    before, t_before = b.u.copy(), b.t
    with pytest.raises(KgError, match="truncated"):
        b.read_from_check_point(cut)
    assert np.array_equal(b.u, before)
    assert b.t == t_before
