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
