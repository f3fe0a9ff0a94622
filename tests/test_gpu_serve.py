"""GPU test of the serving loop: requests of different grids, masses, initial
data and step counts, arriving while others run, give the same waveform in
the continuous batch as when each is served alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_served_results_equal_solo():
    from kg_b200.serve import Server, draw_requests, waveform_error
    reqs = draw_requests(seed=5, rate=400.0, count=8, nr=(16, 48), nr_step=16, ntheta=(8, 16), steps=(20, 80),
                         mass=(0.0, 0.5), r0=(2.5, 4.0), quantum=10)
    batched = Server(mode="batched", save_every=10, l_max=4).run(reqs)
    plain = Server(mode="plain", save_every=10, l_max=4).run(reqs)
    assert batched["completed"] == plain["completed"] == len(reqs)
    for a, b in zip(batched["results"], plain["results"]):
        assert a.rid == b.rid and a.alm.shape == b.alm.shape
        assert np.array_equal(a.alm, b.alm)
        assert np.array_equal(a.times, b.times)
    assert waveform_error(batched, plain) == 0.0
    assert batched["peak_live"] >= 2   # requests overlapped on the device


def test_served_mixed_equal_solo_and_close_to_fp64():
    """mixed precision: each result is the same in the batch as alone (bit for bit),
    and within 1e-6 relative L2 of the FP64 waveform wherever that waveform is
    above the 1e-10 floor"""
    from kg_b200.serve import Server, draw_requests, waveform_error_detail
    reqs = draw_requests(seed=6, rate=400.0, count=8, nr=(16, 48), nr_step=16, ntheta=(8, 16), steps=(20, 80),
                         mass=(0.0, 0.5), r0=(2.5, 4.0), quantum=10)
    batched = Server(mode="batched", save_every=10, l_max=4, precision="mixed").run(reqs)
    plain = Server(mode="plain", save_every=10, l_max=4, precision="mixed").run(reqs)
    fp64 = Server(mode="plain", save_every=10, l_max=4).run(reqs)
    for a, b in zip(batched["results"], plain["results"]):
        assert np.array_equal(a.alm, b.alm)
    worst, count, _ = waveform_error_detail(batched, fp64)
    print(f"mixed vs FP64 waveform: max rel L2 {worst:.2e} over {count} requests")
    assert count >= 4 and worst <= 1e-6


def test_nan_injected_request_leaves_the_others_untouched(monkeypatch):
    """A request whose host copy of the state carries a NaN (injected after its
    initial data are set and uploaded again) is retired as failed at its first
    waveform sample, in the batch and alone; every other request gives the bits
    it gives when served without it."""
    import kg_b200.serve as serve
    from kg_b200.serve import Server, draw_requests
    reqs = draw_requests(seed=7, rate=400.0, count=6, nr=(16, 48), nr_step=16, ntheta=(8,), steps=(20, 40),
                         mass=(0.0, 0.5), r0=(2.5, 4.0), quantum=10)
    bad = reqs[2].rid
    make = serve._make_solve

    def make_with_nan(req, l_max, device):
        s = make(req, l_max, device)
        if req.rid == bad:
            u = s.u                   # host copy of the state, [k, j, i, variable]
            u[3, :, :, 0] = np.nan    # phi on one phi plane
            s.u = u
        return s

    clean = [r for r in reqs if r.rid != bad]
    alone = Server(mode="plain", save_every=10, l_max=4).run(clean)
    monkeypatch.setattr(serve, "_make_solve", make_with_nan)
    for mode in ("batched", "plain"):
        out = Server(mode=mode, save_every=10, l_max=4).run(reqs)
        assert [(r.rid, r.reason) for r in out["failed"]] == [(bad, "non-finite waveform after 10 steps")]
        assert out["completed"] == len(clean)
        for a, b in zip(out["results"], alone["results"]):
            assert a.rid == b.rid and np.array_equal(a.alm, b.alm)
