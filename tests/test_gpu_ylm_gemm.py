"""GPU tests of the all-shell Y_lm projection (project_sh at every vertex shell,
tools/FFT_sph.f90:247-279 after domain_to_sph, tools/FFT_sph.f90:525-651).

The FP64 form is checked against the oracle to round-off; the tensor-core form
(split-BF16 three-pass GEMM on tcgen05, FP32 accumulation) against the oracle
with a tolerance set by the split: each product keeps ~16 significant bits
beyond BF16: x = hi + lo + e with |e| <= 2^-17 |x|, and the dropped lo.lo term
is below 2^-16 |xy|, so a product carries a relative error below 2^-15.  Summed
with the quadrature weights, the error of a coefficient is then below 2^-15
times sum w sin |f| |Y_lm|, which by Cauchy-Schwarz is at most 2^-15 ||f|| ||Y_lm||
in the quadrature norm (||Y_lm|| = 1 up to the quadrature error).  The tests
allow 2^-14 ||f|| per shell, twice the split bound, for the FP32 accumulation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [dict(Nx=64, Ny=33, Nz=65, L=16, xmin=1.8, xmax=20.0, seed=11),
         dict(Nx=100, Ny=17, Nz=33, L=24, xmin=1.8, xmax=12.0, seed=12),
         dict(Nx=40, Ny=65, Nz=129, L=40, xmin=1.8, xmax=9.8, seed=13)]


def _state(c, noise):
    from kg_b200.initial_data import shell_ylm
    u0, _ = shell_ylm(c["Nx"], c["Ny"], c["Nz"], c["xmin"], c["xmax"], seed=c["seed"],
                      r0=0.5 * (c["xmin"] + c["xmax"]), sd=1.0)
    if noise:
        # white noise in phi puts power in every (l, m) column of the GEMM
        rng = np.random.default_rng(c["seed"] + 100)
        u0[..., 0] += noise * (rng.standard_normal(u0.shape[:3]) + 1j * rng.standard_normal(u0.shape[:3]))
    return u0


def _shell_norms(ora, u0, c):
    """quadrature L2 norm of phi on every vertex shell (the oracle's interpolation)"""
    from oracle.oracle import lib, _dp
    f0 = np.ascontiguousarray(u0[..., 0])
    sc = ora.scalars()
    Ny, Nz = c["Ny"], c["Nz"]
    w = np.ones((Nz, Ny))
    w[:, [0, -1]] *= 0.5
    w[[0, -1], :] *= 0.5
    w *= np.sin(np.arange(Ny) * sc["dy"])[None, :] * sc["dy"] * sc["dz"]
    out = np.zeros(c["Nx"])
    sl = np.zeros((Nz, Ny), np.complex128)
    for iv in range(1, c["Nx"] + 1):
        lib().kgo_domain_to_sph_shell(ora.h, _dp(f0.view(np.float64)), iv, _dp(sl.view(np.float64)))
        out[iv - 1] = np.sqrt(np.sum(w * np.abs(sl) ** 2))
    return out


def _check_split_bound(a_t, a_o, fnorm, label=""):
    err = np.abs(a_t - a_o).reshape(a_t.shape[0], -1).max(axis=1)
    ratio = (err / np.maximum(fnorm, 1e-300)).max()
    print(f"{label} max_shell max_lm |error| / ||f||_shell = {ratio:.3e} (2^-15 = {2.0 ** -15:.3e})")
    assert np.all(err <= 2.0 ** -14 * fnorm + 1e-300)


def _pair(c, noise):
    from kg_b200 import ScalarField
    from oracle.oracle import Oracle
    u0 = _state(c, noise)
    dev = ScalarField(c["Nx"], c["Ny"], c["Nz"], c["xmin"], c["xmax"], 0.25, m=0.2)
    dev.u = u0
    ora = Oracle(c["Nx"], c["Ny"], c["Nz"], c["xmin"], c["xmax"], CFL=0.25, m=0.2)
    ora.set_state(u0)
    return dev, ora


@pytest.mark.parametrize("case", range(len(CASES)))
def test_fp64_all_shells_matches_oracle(case):
    c = CASES[case]
    dev, ora = _pair(c, noise=0.05)
    a_d = dev.project_all_shells(c["L"], precision=0)
    a_o = ora.project_all_shells(c["L"])
    scale = np.abs(a_o).max()
    assert np.abs(a_d - a_o).max() <= 1e-13 * scale


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("noise", [0.0, 0.05])
def test_tensor_core_all_shells_matches_oracle(case, noise):
    c = CASES[case]
    dev, ora = _pair(c, noise)
    a_t = dev.project_all_shells(c["L"], precision=1)
    a_o = ora.project_all_shells(c["L"])
    _check_split_bound(a_t, a_o, _shell_norms(ora, _state(c, noise), c), f"case {case} noise {noise}:")
    # entries outside |m| <= l stay exactly zero
    L = c["L"]
    for l in range(L + 1):
        assert not np.any(a_t[:, : L - l, l]) and not np.any(a_t[:, L + l + 1:, l])


def test_tensor_core_repeat_and_degree_change():
    c = CASES[0]
    dev, ora = _pair(c, noise=0.05)
    a1 = dev.project_all_shells(c["L"], precision=1)
    a2 = dev.project_all_shells(c["L"], precision=1)
    assert np.array_equal(a1, a2)
    a_small = dev.project_all_shells(6, precision=1)
    a_o6 = ora.project_all_shells(6)
    fn = _shell_norms(ora, _state(c, 0.05), c)
    _check_split_bound(a_small, a_o6, fn, "L=6:")
    # after steps, the projection follows the evolved state
    dev.pirk2(2)
    ora.pirk2(2)
    a_t = dev.project_all_shells(c["L"], precision=1)
    a_o = ora.project_all_shells(c["L"])
    _check_split_bound(a_t, a_o, _shell_norms(ora, ora.get_state(), c), "after 2 steps:")


def test_tensor_core_l64_on_the_benchmark_sphere():
    """The precision form's projection: l <= 64 on the 129 x 257 vertex sphere
    of the benchmark grid (K = 33153 sphere points, 2145 modes m >= 0), checked
    on a few shells against the oracle within the split-BF16 bound."""
    from oracle.oracle import set_threads, max_threads
    set_threads(max_threads())
    c = dict(Nx=24, Ny=129, Nz=257, L=64, xmin=1.8, xmax=6.5, seed=14)
    for noise in (0.0, 0.05):
        dev, ora = _pair(c, noise)
        a_t = dev.project_all_shells(c["L"], precision=1)
        shells = [2, 12, 20]
        a_o = ora.project_shells(c["L"], shells)
        fn = _shell_norms(ora, _state(c, noise), c)
        _check_split_bound(a_t[[iv - 1 for iv in shells]], a_o, fn[[iv - 1 for iv in shells]],
                           f"L=64 129x257 noise {noise}:")
        dev.close()


def test_detector_shell_agrees_with_all_shells():
    """the all-shell FP64 projection at a detector's shell is the detector projection"""
    from kg_b200 import ScalarField
    c = CASES[0]
    u0 = _state(c, 0.05)
    dev = ScalarField(c["Nx"], c["Ny"], c["Nz"], c["xmin"], c["xmax"], 0.25, m=0.2, l_max=8, n_det=3)
    dev.u = u0
    _, idx = dev.detectors()
    a_det = dev.proyector_detectors()
    a_all = dev.project_all_shells(8, precision=0)
    for d, iv in enumerate(idx):
        if iv > 0:
            assert np.abs(a_det[d] - a_all[iv - 1]).max() <= 1e-14 * np.abs(a_all).max()


def test_tables_ready_right_after_create_on_a_large_grid():
    """The detector/interpolation tables are uploaded behind the zero fill of
    their buffers: on a grid whose creation queues GB-sized fills, projections
    made right after creation see the tables, not zeros."""
    import ctypes as C
    from kg_b200 import ScalarField
    from kg_b200.initial_data import shell_ylm_device
    Nx, Ny, Nz = 2048, 129, 257
    s = ScalarField(Nx, Ny, Nz, 1.8, 400.0, 0.25, m=0.3, l_max=8, n_det=5)
    u0, _ = shell_ylm_device(Nx, Ny, Nz, 1.8, 400.0, seed=20240601, device="cuda:0")
    s._ck(s._lib.kg_set_state_device(s.handle, 0, C.c_void_p(u0.data_ptr())))
    s.synchronize()
    _, idx = s.detectors()
    assert np.all(idx[:-1] > 0)
    a_all = s.project_all_shells(8, precision=0)
    assert np.abs(a_all).max() > 0
    a_det = s.proyector_detectors()
    for d, iv in enumerate(idx):
        if iv > 0:
            scale = max(np.abs(a_all[iv - 1]).max(), 1e-300)
            assert np.abs(a_det[d] - a_all[iv - 1]).max() <= 1e-13 * scale
    s.close()
