"""GPU tests of the all-shell Y_lm projection (project_sh at every vertex shell,
tools/FFT_sph.f90:247-279 after domain_to_sph, tools/FFT_sph.f90:525-651).

The FP64 form is checked against the oracle to round-off; the tensor-core form
(split-BF16 three-pass GEMM on tcgen05, FP32 accumulation) against the oracle
with a tolerance set by the split: each product keeps ~16 significant bits
beyond BF16, so the error of a coefficient is bounded by ~2^-16 times the
weighted L1 norm of the shell, itself bounded by the shell's L2 norm.  The
tests use 5e-5 of the largest coefficient of the shell set."""
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
    err = np.abs(a_t - a_o).max() / np.abs(a_o).max()
    print(f"case {case} noise {noise}: max error / max |a_lm| = {err:.3e}")
    assert err <= 5e-5
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
    assert np.array_equal(a_small, a1[:, c["L"] - 6: c["L"] + 7, :7]) or \
        np.abs(a_small - a1[:, c["L"] - 6: c["L"] + 7, :7]).max() <= 5e-5 * np.abs(a1).max()
    # after steps, the projection follows the evolved state
    dev.pirk2(2)
    ora.pirk2(2)
    a_t = dev.project_all_shells(c["L"], precision=1)
    a_o = ora.project_all_shells(c["L"])
    assert np.abs(a_t - a_o).max() <= 5e-5 * np.abs(a_o).max()


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
