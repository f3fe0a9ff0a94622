"""GPU tests of the batched engine: solves of different grid sizes and field
masses advanced together by one persistent launch per RK4 stage must give,
bit for bit, what each solve gives alone (and what the oracle gives)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [dict(Nx=16, Ny=9, Nz=17, xmin=1.8, xmax=12.0, m=0.3, seed=1),
          dict(Nx=40, Ny=13, Nz=25, xmin=1.8, xmax=9.8, m=0.1, seed=2),
          dict(Nx=33, Ny=17, Nz=9, xmin=1.8, xmax=20.0, m=0.45, seed=3)]


def _solve(sp):
    from kg_b200 import ScalarField
    from kg_b200.initial_data import shell_ylm
    s = ScalarField(sp["Nx"], sp["Ny"], sp["Nz"], sp["xmin"], sp["xmax"], 0.25, m=sp["m"])
    u0, _ = shell_ylm(sp["Nx"], sp["Ny"], sp["Nz"], sp["xmin"], sp["xmax"], seed=sp["seed"],
                      r0=0.5 * (sp["xmin"] + sp["xmax"]), sd=1.0)
    s.u = u0
    return s, u0


def test_batch_matches_solo_and_oracle():
    from kg_b200.batch import Batch
    from oracle.oracle import Oracle
    batch = Batch()
    solos, members, u0s = [], [], []
    for sp in SHAPES:
        m, u0 = _solve(sp)
        s, _ = _solve(sp)
        batch.add(m)
        members.append(m)
        solos.append(s)
        u0s.append(u0)
    batch.rk4(1)
    batch.rk4(6)
    for s in solos:
        s.rk4(nsteps=7)
    for m, s in zip(members, solos):
        assert np.array_equal(m.u, s.u)
        assert m.t == s.t
    sp = SHAPES[1]
    o = Oracle(sp["Nx"], sp["Ny"], sp["Nz"], sp["xmin"], sp["xmax"], CFL=0.25, m=sp["m"])
    o.set_state(u0s[1])
    o.rk4(7)
    assert np.array_equal(members[1].u, o.get_state())


def test_batch_membership_changes_and_tuning():
    from kg_b200.batch import Batch
    batch = Batch()
    a, _ = _solve(SHAPES[0])
    b, _ = _solve(SHAPES[1])
    c, _ = _solve(SHAPES[2])
    ra, _ = _solve(SHAPES[0])
    rb, _ = _solve(SHAPES[1])
    rc, _ = _solve(SHAPES[2])
    batch.add(a)
    batch.add(b)
    batch.rk4(3)
    ra.rk4(nsteps=3)
    rb.rk4(nsteps=3)
    batch.remove(a)
    batch.add(c)
    batch.set_tuning(8, 37)
    batch.rk4(4)
    rb.rk4(nsteps=4)
    rc.rk4(nsteps=4)
    assert np.array_equal(a.u, ra.u)
    assert np.array_equal(b.u, rb.u)
    assert np.array_equal(c.u, rc.u)
    assert len(batch) == 2
    # a member's own diagnostics wait for the batch
    c.density()
    assert np.isfinite(c.mass_scalar())


def test_autotune_returns_a_valid_shape():
    from kg_b200.batch import autotune
    for prec in ("fp64", "mixed"):
        t = autotune([(16, 9, 17), (40, 13, 25)], kchunks=(8, 32), ctas_per_sm=(1, 2), steps=1, precision=prec)
        assert t.blocks > 0 and t.dispatch in (0, 1)
        if t.dispatch == 0:
            assert t.kchunk in (8, 32)
        else:
            assert t.variant in ((2, 1, 0) if prec == "fp64" else (2,))


@pytest.mark.parametrize("variant", [-1, 0, 1, 2])
def test_concurrent_dispatch_matches_solo(variant):
    """dispatch 1: every member's own single-solve kernels on its own stream,
    concurrently; the same bits as each solve stepped alone, in every
    stage-kernel form, and after membership changes"""
    from kg_b200.batch import Batch
    batch = Batch()
    batch.set_tuning(16, 148, 1, variant)
    members, solos = [], []
    for sp in SHAPES:
        m, _ = _solve(sp)
        s, _ = _solve(sp)
        batch.add(m)
        members.append(m)
        solos.append(s)
    batch.rk4(1)
    batch.rk4(4)
    for s in solos:
        s.rk4(nsteps=5)
    batch.remove(members[0])
    batch.rk4(2)
    for s in solos[1:]:
        s.rk4(nsteps=2)
    for m, s in zip(members, solos):
        assert np.array_equal(m.u, s.u)
        assert m.t == s.t
    assert batch.tuning().dispatch == 1


def test_concurrent_dispatch_mixed_matches_persistent():
    from kg_b200.batch import Batch
    out = []
    for tune in ((16, 148, 0, -1), (16, 148, 1, 2)):
        batch = Batch(precision="mixed")
        batch.set_tuning(*tune)
        ms = []
        for sp in SHAPES:
            m, _ = _solve(sp)
            batch.add(m)
            ms.append(m)
        batch.rk4(5)
        batch.synchronize()
        out.append([m.u for m in ms])
    for a, b in zip(*out):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("dispatch", [0, 1])
def test_tile_rows_4_matches_solo(precision, dispatch):
    """32 x 4 tiles in the persistent launch and in the concurrent members'
    kernels: the bits of each solve stepped alone in 32 x 8 tiles"""
    from kg_b200.batch import Batch
    batch = Batch(precision=precision)
    batch.set_tuning(16, 444, dispatch, 2 if dispatch else -1, 4)
    assert batch.tuning().tile_rows == 4
    members, solos = [], []
    for sp in SHAPES:
        m, _ = _solve(sp)
        s, _ = _solve(sp)
        s.precision = precision
        batch.add(m)
        members.append(m)
        solos.append(s)
    batch.rk4(5)
    batch.synchronize()
    for s in solos:
        s.rk4(nsteps=5)
    for m, s in zip(members, solos):
        assert np.array_equal(m.u, s.u)
