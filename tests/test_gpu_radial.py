"""GPU tests of the spherical-Bessel radial basis (generate_full_bessel_basis,
tools/FFT_sph.f90:13-95) and the discrete radial transform of the all-shell
Y_lm coefficients (SphFT_discrete_radial, tools/FFT_sph.f90:213-244)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRID = dict(Nx=64, Ny=17, Nz=33, xmin=1.8, xmax=14.6)


def _pair(L=8):
    from kg_b200 import ScalarField
    from kg_b200.initial_data import shell_ylm
    from oracle.oracle import Oracle
    g = GRID
    u0, _ = shell_ylm(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], seed=21, r0=7.0, sd=1.0)
    dev = ScalarField(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=0.2)
    dev.u = u0
    ora = Oracle(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], CFL=0.25, m=0.2)
    ora.set_state(u0)
    return dev, ora


def test_bessel_basis_matches_oracle():
    dev, ora = _pair()
    k_d, jb_d = dev.bessel_basis(10, 30)
    k_o, jb_o = ora.bessel_basis(10, 30)
    assert np.allclose(k_d, k_o, rtol=2e-15, atol=0)
    assert np.abs(jb_d - jb_o).max() <= 1e-12 * np.abs(jb_o).max()


@pytest.mark.parametrize("L,Nk", [(8, 20), (12, 40)])
def test_radial_transform_fp64_matches_oracle(L, Nk):
    dev, ora = _pair()
    ft_d = dev.sph_ft_radial(L, Nk, precision=0)
    ft_o = ora.sph_ft_radial(L, Nk)
    assert np.abs(ft_d - ft_o).max() <= 1e-12 * np.abs(ft_o).max()
    # |m| > l entries are zero
    for l in range(L + 1):
        assert not np.any(ft_d[: L - l, l, :]) and not np.any(ft_d[L + l + 1:, l, :])


def test_radial_transform_tensor_core_projection():
    """with the split-BF16 projection the transform carries the projection's
    error, ~2^-17 of each shell's norm, through a linear map"""
    dev, ora = _pair()
    L, Nk = 8, 20
    ft_t = dev.sph_ft_radial(L, Nk, precision=1)
    ft_o = ora.sph_ft_radial(L, Nk)
    err = np.abs(ft_t - ft_o).max() / np.abs(ft_o).max()
    print(f"tensor-core radial transform: max error / max |ft| = {err:.3e}")
    assert err <= 1e-4
