"""Generate the committed golden fixtures in tests/golden/.

    python tests/golden/make_golden.py

* oracle_small.json -- the CPU oracle's state after 5 steps of each stepper
  (PIRK2, PIRK3, RK3, RK4) on a 16 x 9 x 17 grid, for Kerr_Schild and Schw_EF,
  from the seeded shell initial data: a sha256 of the exact bytes plus a
  strided sample of values.  It pins the oracle (and the device path, which
  must reproduce the same bytes) against regressions.
* ylm_scipy.npz    -- Y_lm for l <= 6 on the reference's vertex grid of a
  Ny = 9, Nz = 17 sphere from scipy.special.sph_harm_y (Condon-Shortley
  phase), an independent check of the Legendre recurrence used for GSL's
  gsl_sf_legendre_Plm.

The reference itself cannot run in this environment (Fortran toolchain,
MPI, HDF5 and GSL are absent), so these fixtures come from the restatement
and from scipy, not from the reference binary.
"""
import hashlib
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kg_b200.initial_data import shell_ylm  # noqa: E402
from oracle.oracle import Oracle, KERR_SCHILD, SCHW_EF  # noqa: E402

GRID = dict(Nx=16, Ny=9, Nz=17, xmin=1.8, xmax=12.0)
STEPS = 5


def state_digest(u):
    b = np.ascontiguousarray(u, dtype=np.complex128).tobytes()
    return hashlib.sha256(b).hexdigest()


def sample(u):
    flat = np.ascontiguousarray(u).reshape(-1)
    idx = np.arange(0, flat.size, 997)
    return idx.tolist(), [[float(z.real), float(z.imag)] for z in flat[idx]]


def main():
    out = {"grid": GRID, "steps": STEPS, "m": 0.3, "CFL": 0.25, "seed": 3, "r0": 6.0, "sd": 1.0, "cases": {}}
    u0, _ = shell_ylm(GRID["Nx"], GRID["Ny"], GRID["Nz"], GRID["xmin"], GRID["xmax"], seed=3, r0=6.0, sd=1.0)
    out["ic_sha256"] = state_digest(u0)
    for mname, mcode in (("Kerr_Schild", KERR_SCHILD), ("Schw_EF", SCHW_EF)):
        for method in ("pirk2", "pirk3", "rk3", "rk4"):
            o = Oracle(GRID["Nx"], GRID["Ny"], GRID["Nz"], GRID["xmin"], GRID["xmax"], CFL=0.25, m=0.3, metric=mcode)
            o.set_state(u0)
            o.step(method, STEPS)
            u = o.get_state()
            idx, vals = sample(u)
            out["cases"][f"{mname}/{method}"] = {"sha256": state_digest(u), "idx": idx, "vals": vals,
                                                 "t": o.scalars()["t"]}
    with open(os.path.join(HERE, "oracle_small.json"), "w") as f:
        json.dump(out, f, indent=1)

    from scipy.special import sph_harm_y
    Ny, Nz, L = 9, 17, 6
    dy = math.acos(-1.0) / (Ny - 1)
    dz = 2.0 * math.acos(-1.0) / (Nz - 1)
    th = np.arange(Ny) * dy
    ph = np.arange(Nz) * dz
    Y = np.zeros((Nz, Ny, 2 * L + 1, L + 1), np.complex128)
    for l in range(L + 1):
        for m in range(-l, l + 1):
            Y[:, :, m + L, l] = sph_harm_y(l, m, th[None, :], ph[:, None])
    np.savez_compressed(os.path.join(HERE, "ylm_scipy.npz"), Y=Y, Ny=Ny, Nz=Nz, L=L)


if __name__ == "__main__":
    main()
