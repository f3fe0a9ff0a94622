"""GPU tests of failure detection without a GPU fault: a bounded device wait
that runs out is reported as KG_ETIMEOUT and leaves the handle (and its CUDA
context) usable; a solve whose device memory cannot be had is refused at
creation and leaves the device usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRID = dict(Nx=16, Ny=9, Nz=17, xmin=1.8, xmax=12.0)


def _pair():
    from kg_b200 import ScalarField
    from kg_b200.initial_data import shell_ylm
    from oracle.oracle import Oracle
    g = GRID
    dev = ScalarField(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=0.3)
    ora = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], CFL=0.25, m=0.3)
    u0, _ = shell_ylm(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], seed=11, r0=6.0, sd=1.0)
    dev.u = u0
    ora.set_state(u0)
    return dev, ora


def test_bounded_wait_runs_out_and_the_handle_stays_usable():
    from kg_b200 import capi
    dev, ora = _pair()
    lib, h = dev._lib, dev.handle
    dev.pirk2(2)
    ora.pirk2(2)
    assert lib.kg_check_wait_timeout(h, 0) == capi.KG_EINVAL
    assert lib.kg_check_wait_timeout(h, 256) == capi.KG_ETIMEOUT
    assert b"wait ran out" in lib.kg_last_error(h)
    assert lib.kg_synchronize(h) == capi.KG_OK    # the flag was cleared
    dev.pirk2(3)                                  # the context still runs kernels
    ora.pirk2(3)
    assert np.array_equal(dev.u, ora.get_state())


def test_unallocatable_solve_is_refused_and_the_device_stays_usable():
    from kg_b200 import ScalarField, capi
    with pytest.raises(capi.KgError) as e:
        ScalarField(100000, 9, 65537, 1.8, 100.0, 0.25, m=0.3)   # ~7 TB per state copy
    assert e.value.code in (capi.KG_ENOMEM, capi.KG_ECUDA)
    dev, ora = _pair()
    dev.rk4(nsteps=2)
    ora.rk4(2)
    assert np.array_equal(dev.u, ora.get_state())
