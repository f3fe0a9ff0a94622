"""Host logic of the serving loop on the CPU: admission against the HBM budget,
new arrivals prepared while a quantum runs and stepping from the next one,
every waveform sample attributed to its own solve, retirement and clean-up.
The device side (solves and the batched engine) is replaced by fakes that
record what the loop asks of them."""
import numpy as np
import pytest


class FakeSolve:
    def __init__(self, req):
        self.req = req
        self.steps = 0
        self.t = 0.0
        self.closed = False
        self.precision = "fp64"

    def close(self):
        self.closed = True

    # the single-solve path (plain mode)
    def rk4(self, nsteps):
        self.steps += nsteps
        self.t += nsteps * 0.1
        assert self.steps <= self.req.steps

    def proyector_detectors(self):
        return FakeBatch.sample(self)


class FakeBatch:
    instances = []

    def __init__(self, device=-1, precision="fp64"):
        self.members = []
        self.in_flight = set()   # members queued in the running quantum
        self.max_members = 0
        self.closed = False
        FakeBatch.instances.append(self)

    def set_tuning(self, *a):
        pass

    def add(self, s):
        assert s not in self.members
        self.members.append(s)
        self.max_members = max(self.max_members, len(self.members))

    def remove(self, s):
        self.members.remove(s)

    def rk4(self, n):
        self.in_flight = set(id(m) for m in self.members)
        for m in self.members:
            m.steps += n
            m.t += n * 0.1
            assert m.steps <= m.req.steps, "a solve stepped past its request"

    nan_at = {}  # rid -> step count from which the solve's samples are NaN (a state gone bad)

    @staticmethod
    def sample(m):
        # one (n_det, 2L+1, L+1) block; [0, 0, 0] encodes the solve and its step count
        a = np.zeros((2, 3, 2), np.complex128)
        a[0, 0, 0] = m.req.rid + 1j * m.steps
        if m.req.rid in FakeBatch.nan_at and m.steps >= FakeBatch.nan_at[m.req.rid]:
            a[0, 1, 1] = np.nan
        return a

    def proyector_detectors(self):
        return [FakeBatch.sample(m) for m in self.members]

    def close(self):
        self.closed = True


@pytest.fixture
def served(monkeypatch):
    import kg_b200.batch
    import kg_b200.serve as serve
    made = []

    def make(req, l_max, device):
        s = FakeSolve(req)
        made.append(s)
        return s

    FakeBatch.instances.clear()
    FakeBatch.nan_at = {}
    monkeypatch.setattr(serve, "_make_solve", make)
    monkeypatch.setattr(kg_b200.batch, "Batch", FakeBatch)
    return serve, made


def test_batched_loop_attribution_and_cleanup(served):
    serve, made = served
    reqs = serve.draw_requests(seed=3, rate=1e6, count=40, nr=(16, 64), nr_step=16, ntheta=(8, 16),
                               steps=(10, 120), quantum=10)
    budget = 3.5 * max(serve._bytes_estimate(r) for r in reqs)
    out = serve.Server(mode="batched", hbm_budget=budget, save_every=10).run(reqs)
    assert out["completed"] == len(reqs)
    b = FakeBatch.instances[-1]
    assert b.closed and not b.members
    assert all(s.closed for s in made) and len(made) == len(reqs)
    assert out["peak_live"] >= 2               # requests overlapped
    for res, r in zip(out["results"], sorted(reqs, key=lambda x: x.rid)):
        assert res.rid == r.rid
        samples = res.alm[:, 0, 0]
        # one sample per quantum, each from this solve, the first after its first quantum:
        # a solve that joined during a quantum did not take part in it
        assert len(samples) == r.steps // 10
        assert np.all(samples.real == r.rid)
        assert np.array_equal(samples.imag, np.arange(10, r.steps + 1, 10))
        assert np.allclose(res.times, 0.1 * np.arange(10, r.steps + 1, 10))


def test_batched_loop_budget_never_exceeded(served, monkeypatch):
    serve, made = served
    reqs = serve.draw_requests(seed=4, rate=1e6, count=30, nr=(16, 96), nr_step=16, ntheta=(8, 16),
                               steps=(10, 60), quantum=10)
    budget = 2.2 * max(serve._bytes_estimate(r) for r in reqs)
    live_bytes = []
    orig_add = FakeBatch.add

    def add(self, s):
        orig_add(self, s)
        live_bytes.append(sum(serve._bytes_estimate(m.req) for m in self.members))

    monkeypatch.setattr(FakeBatch, "add", add)
    out = serve.Server(mode="batched", hbm_budget=budget, save_every=10).run(reqs)
    assert out["completed"] == len(reqs)
    assert max(live_bytes) <= budget


@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_request_larger_than_budget_is_refused(served, mode):
    """a request that alone exceeds the HBM budget is refused and reported; the
    others are served"""
    serve, made = served
    reqs = serve.draw_requests(seed=5, rate=1e6, count=3, nr=(64, 64), nr_step=16, ntheta=(16,),
                               steps=(10, 10), quantum=10)
    big = serve.Request(rid=99, arrival=0.0, Nr=4096, Ntheta=64, m=0.1, seed=1, steps=10)
    budget = 2 * serve._bytes_estimate(reqs[0])
    assert serve._bytes_estimate(big) > budget
    out = serve.Server(mode=mode, hbm_budget=budget).run(reqs + [big])
    assert out["completed"] == 3
    assert [(r.rid, r.reason) for r in out["failed"]] == [(99, "exceeds the HBM budget alone")]
    assert all(s.req.rid != 99 for s in made)


@pytest.mark.parametrize("mode", ["batched", "plain"])
def test_faults_stay_with_their_request(served, monkeypatch, mode):
    """Host-injected faults, none on the GPU: a malformed request (creation refuses
    its parameters), an allocation failure, a request withdrawn before admission,
    one withdrawn while it runs, and a solve whose state goes non-finite.  Each is
    reported with its reason, its solve (if any) is closed and leaves the batch,
    its memory returns to the budget, and every other request is served in full."""
    import time
    serve, made = served
    reqs = serve.draw_requests(seed=6, rate=1e6, count=12, nr=(16, 48), nr_step=16, ntheta=(8,),
                               steps=(60, 60), quantum=10)
    reqs[1].cancel_at = 0.0                  # withdrawn before admission
    reqs[0].cancel_at = 0.005                # withdrawn after its first quantum (each quantum takes 20 ms)
    FakeBatch.nan_at = {6: 30}               # its state goes bad during its third quantum
    fake_make = serve._make_solve

    def make(req, l_max, device):
        if req.rid == 2:
            raise ValueError("Nx must be at least 4")                   # malformed
        if req.rid == 3:
            raise MemoryError("device allocation of 1e13 bytes failed")  # out of device memory
        return fake_make(req, l_max, device)

    monkeypatch.setattr(serve, "_make_solve", make)
    orig_rk4, orig_srk4 = FakeBatch.rk4, FakeSolve.rk4

    def slow(f):
        def g(self, *a, **k):
            time.sleep(0.02)
            return f(self, *a, **k)
        return g

    monkeypatch.setattr(FakeBatch, "rk4", slow(orig_rk4))
    monkeypatch.setattr(FakeSolve, "rk4", slow(orig_srk4))
    budget = 3.5 * max(serve._bytes_estimate(r) for r in reqs)
    out = serve.Server(mode=mode, hbm_budget=budget, save_every=10).run(reqs)
    failed = {r.rid: r.reason for r in out["failed"]}
    cancelled = {r.rid: r for r in out["cancelled"]}
    assert failed[2].startswith("not created: Nx must be at least 4")
    assert failed[3].startswith("not created: device allocation")
    assert failed[6] == "non-finite waveform after 30 steps"
    assert set(failed) == {2, 3, 6}
    assert cancelled[1].reason == "withdrawn before admission" and len(cancelled[1].alm) == 0
    assert cancelled[0].reason.startswith("withdrawn after") and 0 < len(cancelled[0].alm) < 6
    assert set(cancelled) == {0, 1}
    assert out["completed"] == len(reqs) - 5
    for res in out["results"]:
        assert res.status == "done" and len(res.alm) == 6
    assert all(s.closed for s in made)
    if mode == "batched":
        assert not FakeBatch.instances[-1].members


def test_tuner_candidates_cover_both_dispatches():
    """the batch tuner's search space (host logic): persistent launches over
    (kchunk, CTAs per SM, tile rows) and concurrent single-solve launches over the
    stage-kernel forms, the TMA form in both tile heights; the mixed form has the
    TMA form only"""
    from kg_b200.batch import Tuning, candidates
    c64 = candidates("fp64", kchunks=(16, 32), ctas_per_sm=(1, 2), sms=148)
    assert Tuning(16, 148, 0, -1) in c64 and Tuning(32, 296, 0, -1) in c64
    # 32 x 4 tiles: 1.5x the CTAs per SM of the 32 x 8 candidates
    assert Tuning(16, 148, 0, -1, 4) in c64 and Tuning(32, 444, 0, -1, 4) in c64
    assert {t.variant for t in c64 if t.dispatch == 1} == {0, 1, 2}
    assert {t.tile_rows for t in c64 if t.dispatch == 1 and t.variant == 2} == {8, 4}
    assert {t.tile_rows for t in c64 if t.dispatch == 1 and t.variant != 2} == {8}
    cmx = candidates("mixed", kchunks=(16,), ctas_per_sm=(2,), sms=148)
    assert {(t.variant, t.tile_rows) for t in cmx if t.dispatch == 1} == {(2, 8), (2, 4)}
    assert len(candidates("fp64", kchunks=(16,), ctas_per_sm=(2,), tile_rows=(8,))) == 1 + 3
    t = Tuning(8, 37, 1, 2)
    assert (t.kchunk, t.blocks, t.dispatch, t.variant, t.tile_rows) == (8, 37, 1, 2, 8)
    assert tuple(t) == (8, 37, 1, 2, 8)
