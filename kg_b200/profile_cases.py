"""Small, self-contained runs of each kernel family, for profilers.

    python -m kg_b200.profile_cases pirk       [--grid Nx,Ny,Nz] [--steps K] [--variant V]
    python -m kg_b200.profile_cases mixed      [--grid Nx,Ny,Nz] [--steps K]
    python -m kg_b200.profile_cases proj       [--grid Nx,Ny,Nz] [--steps K] [--lmax L]
    python -m kg_b200.profile_cases configured [--grid Nx,Ny,Nz] [--steps K]
    python -m kg_b200.profile_cases batch      [--solves N] [--precision fp64|mixed] [--mix serving|c3] [--steps K]
    python -m kg_b200.profile_cases refine     [--grid Nx,Ny,Nz] [--steps K]
    python -m kg_b200.profile_cases diag       [--grid Nx,Ny,Nz] [--steps K]
    python -m kg_b200.profile_cases steppers   [--grid Nx,Ny,Nz] [--steps K]

Each case builds seeded synthetic input on the device, runs K steps and exits
0 (or raises); the sizes default to a few GB of device memory, larger than
L2, so a profiler capture of one launch is representative and ends quickly.
  pirk:       PIRK2 of the reference's method on a radial slab of the
              benchmark grid, in the stage-kernel form V (kg_set_kernel_variant)
  mixed:      RK4 with the FP32 stencil RHS and FP64 update (mixed_rk4_* kernels)
  proj:       the all-shell Y_lm projection on the tensor cores, K times
              (split-BF16 tcgen05 GEMM, ylm_gemm_kernel)
  configured: RK4 of the fourth-order method (cfg_stage_kernel)
  batch:      a request mix advanced as one batch (tma_batch_kernel /
              mx_batch_kernel, persistent over a ragged work list): the serving
              mix (Nr 128..512, Ntheta 16/32) or the batching-form mix
              (Nr 128..1024, Ntheta 16/32/64)
  refine:     a two-level Berger-Oliger hierarchy (prolong/restrict kernels)
  diag:       the diagnostics of the evolve loop K times: density, the mass
              integral (warp-shuffle partial sums), the currents and the
              detector projection
  steppers:   PIRK2, PIRK3, SSP-RK3 and RK4 on the benchmark grid (default
              2048 x 129 x 257), K steps each after warm-up, with every kernel
              kind timed by CUDA events; prints one line per stepper with the
              time per launch and the fraction of the measured HBM copy rate
              (MEASURED_PEAKS.json, else 6650 GB/s) its algorithmic bytes reach
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys


def _grid(s, default):
    return tuple(int(v) for v in s.split(",")) if s else default


def _device_ic(s, Nx, Ny, Nz, xmin, xmax, seed=7):
    from .initial_data import shell_ylm_device
    u0, _ = shell_ylm_device(Nx, Ny, Nz, xmin, xmax, seed=seed, device="cuda:0")
    s._ck(s._lib.kg_set_state_device(s.handle, 0, C.c_void_p(u0.data_ptr())))
    s.synchronize()


# algorithmic bytes per stored point of each stage kernel (FP64 complex: 16 B per variable)
STAGE_BYTES = {"stage_pirk_s1_fused": 176, "stage_pirk_s1_psi": 144, "stage_pirk_s1_pi": 112, "stage_pirk2_s2": 240,
               "stage_pirk3_s2_psi": 208, "stage_pirk3_s2_pi": 128, "stage_pirk3_s3": 240,
               "stage_rk3_1": 160, "stage_rk3_2": 240, "stage_rk3_3": 240,
               "stage_rk4_1": 240, "stage_rk4_2": 400, "stage_rk4_3": 400, "stage_rk4_4": 320}


def _steppers(a):
    import json
    import os
    from .lines_method import ScalarField
    Nx, Ny, Nz = _grid(a.grid, (2048, 129, 257))
    xmax = 1.8 + 0.1944 * Nx
    s = ScalarField(Nx, Ny, Nz, 1.8, xmax, 0.25, m=0.3, device=0, n_det=2, l_max=0)
    _device_ic(s, Nx, Ny, Nz, 1.8, xmax)
    lib = s._lib
    nk = lib.kg_profile_kinds()
    names = [lib.kg_profile_kind_name(i).decode() for i in range(nk)]
    pts = (Nx + 5) * (Ny + 5) * (Nz + 1)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    peaks = os.path.join(root, "MEASURED_PEAKS.json")
    peak = float(json.load(open(peaks)).get("hbm_gbs", 6650.0)) if os.path.exists(peaks) else 6650.0
    ms = (C.c_double * nk)()
    cnt = (C.c_longlong * nk)()
    steps = max(a.steps, 2)
    for meth in ("pirk2", "pirk3", "rk3", "rk4"):
        run = getattr(s, meth)
        step = (lambda n: run(nsteps=n)) if meth.startswith("rk") else run
        step(4)  # buffers and the captured graphs of both Pi-slot parities
        s.synchronize()
        lib.kg_profile_enable(s.handle, 1)
        lib.kg_profile_read(s.handle, ms, cnt)
        step(steps)
        s.synchronize()
        lib.kg_profile_read(s.handle, ms, cnt)
        lib.kg_profile_enable(s.handle, 0)
        out = {}
        for i in range(nk):
            if cnt[i]:
                per = ms[i] / cnt[i]
                b = STAGE_BYTES.get(names[i], 0) * pts
                out[names[i]] = {"ms": round(per, 3), "hbm_frac": round(b / (per / 1e3) / 1e9 / peak, 3) if b else None}
        print(meth, json.dumps(out))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["pirk", "mixed", "proj", "configured", "batch", "refine", "diag", "steppers"])
    ap.add_argument("--lmax", type=int, default=64)
    ap.add_argument("--variant", type=int, default=3)
    ap.add_argument("--grid", default=None)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--solves", type=int, default=30)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--mix", default="serving", choices=["serving", "c3"])
    ap.add_argument("--kchunk", type=int, default=64)
    a = ap.parse_args(argv)
    from .lines_method import ScalarField
    if a.case == "pirk":
        Nx, Ny, Nz = _grid(a.grid, (512, 129, 257))
        xmax = 1.8 + 0.1944 * Nx
        s = ScalarField(Nx, Ny, Nz, 1.8, xmax, 0.25, m=0.3, device=0)
        _device_ic(s, Nx, Ny, Nz, 1.8, xmax)
        s._ck(s._lib.kg_set_kernel_variant(s.handle, a.variant))
        for _ in range(a.steps):
            s.pirk2(1)
        s.synchronize()
    elif a.case == "proj":
        Nx, Ny, Nz = _grid(a.grid, (1024, 129, 257))
        xmax = 1.8 + 0.1944 * Nx
        s = ScalarField(Nx, Ny, Nz, 1.8, xmax, 0.25, m=0.3, device=0)
        _device_ic(s, Nx, Ny, Nz, 1.8, xmax)
        for _ in range(a.steps):
            s.project_all_shells(a.lmax, precision=1)
        s.synchronize()
    elif a.case == "mixed":
        Nx, Ny, Nz = _grid(a.grid, (384, 129, 257))
        xmax = 1.8 + 0.1944 * Nx
        s = ScalarField(Nx, Ny, Nz, 1.8, xmax, 0.25, m=0.3, device=0)
        _device_ic(s, Nx, Ny, Nz, 1.8, xmax)
        s.precision = "mixed"
        for _ in range(a.steps):
            s.rk4(nsteps=1)
        s.synchronize()
    elif a.case == "configured":
        from .initial_data import smooth_exact
        Nx, Ny, Nz = _grid(a.grid, (384, 65, 129))
        s = ScalarField(Nx, Ny, Nz, 1.8, 60.0, 0.25, m=0.0, device=0)
        s.set_scheme("configured", 0.02)
        s.u = smooth_exact(Nx, Ny, Nz, 1.8, 60.0, amp=1e-3, r0=10.0, width=1.0, angular="y20")
        s.fill_ghosts_configured()
        for _ in range(a.steps):
            s.rk4(nsteps=1)
        s.synchronize()
    elif a.case == "batch":
        from .batch import Batch
        from .serve import draw_requests, _make_solve
        if a.mix == "serving":
            reqs = draw_requests(seed=20240602, rate=2000.0, count=a.solves, nr=(128, 512), nr_step=64,
                                 ntheta=(16, 32), steps=(100, 1000), quantum=10)
        else:
            reqs = draw_requests(seed=20240603, rate=100.0, count=a.solves, nr=(128, 1024), nr_step=64,
                                 ntheta=(16, 32, 64), steps=(2000, 2000), quantum=10)
        b = Batch(0, precision=a.precision)
        b.set_tuning(a.kchunk, 296)
        solves = [_make_solve(r, 8, 0) for r in reqs]
        for s in solves:
            b.add(s)
        for _ in range(a.steps):
            b.rk4(1)
        b.synchronize()
    elif a.case == "steppers":
        _steppers(a)
    elif a.case == "diag":
        Nx, Ny, Nz = _grid(a.grid, (512, 129, 257))
        xmax = 1.8 + 0.1944 * Nx
        s = ScalarField(Nx, Ny, Nz, 1.8, xmax, 0.25, m=0.3, l_max=8, n_det=5, device=0)
        _device_ic(s, Nx, Ny, Nz, 1.8, xmax)
        for _ in range(a.steps):
            s.density()
            s.mass_scalar()
            s.currents_detectors()
            s.proyector_detectors()
        s.synchronize()
    else:
        from .refinement import BergerOliger
        Nx, Ny, Nz = _grid(a.grid, (512, 65, 129))
        xmax = 1.8 + 0.1944 * Nx
        bo = BergerOliger(Nx, Ny, Nz, 1.8, xmax, 0.25, r_fine=(20.0,), m=0.3, device=0)
        for lv in bo.levels:
            _device_ic(lv, lv.Nx, lv.Ny, lv.Nz, 1.8, lv.params.xmax)
        bo.rk4(a.steps)
        bo.synchronize()
    print("ok", a.case)
    return 0


if __name__ == "__main__":
    sys.exit(main())
