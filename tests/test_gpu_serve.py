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
