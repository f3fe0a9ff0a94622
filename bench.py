"""Benchmark of the KG method-of-lines hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl kg|reference]

Workload (one "step" = one PIRK2 time step, the stepper of the reference's
evolve loop, main/evolve.f90:25): the single large FP64 solve of the
benchmark description -- Nr = 2048 radial cells on r in [1.8, 400], 128 x 256
theta x phi cells (reference grid integers Nx = 2048, Ny = 129, Nz = 257, two
ghosts), Kerr-Schild M = 1, field mass 0.3, outflow outer boundary, CFL 0.25
with the reference dt rule; seeded Gaussian shell (r0 ~ U[8,15], sigma 1.5)
times sum_{l<=4} c_lm Y_lm, c_lm complex N(0, 1e-4).  Synthetic, seeded data;
the state (5.7 GB per copy) is far larger than L2, so no flush is needed.
The Berger-Oliger refinement levels of that description are not part of this
measurement.

Metric: grid-point-stage updates per second (GPSU/s) = interior points x RK
stages x steps / time.  `value` is device time of K steps with the state
resident in HBM (CUDA events on the solver's stream, max over ranks);
`e2e` goes through the C ABI from pinned host memory: upload of the initial
state, K x (kg_pirk2 + kg_diagnostic with its 8-byte mass read-back), download
of the final state.

With --gpus N (torchrun), every rank runs an independent replica on its own
GPU (the path has no exchange step), `value` sums all ranks, scaling "weak".

--impl reference times the CPU restatement of the reference's own path (the
oracle, all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(Nx=2048, Ny=129, Nz=257, xmin=1.8, xmax=400.0, m=0.3, CFL=0.25, seed=20240601)
METRIC = "RK point-updates/s (FP64 PIRK2, Nr=2048 x Ntheta=128 x Nphi=256)"
UNIT = "GPSU/s"
# algorithmic bytes per stored point of each PIRK2 kernel (complex128 = 16 B per variable)
#   stage_pirk_s1_fused: read u (5 vars), stale u_stage(5); write u_stage(1:5) = 80 + 16 + 80
#   stage_pirk_s1_psi  : read u (5 vars) + write u_stage(1:4)               = 80 + 64   (two-launch form)
#   stage_pirk_s1_pi   : read u_stage(1:4), stale u_stage(5), u(5); write u_stage(5) = 64 + 16 + 16 + 16
#   stage_pirk2_s2     : read u_stage, u_p(=u); write u                     = 80 + 80 + 80
ALG_BYTES = {"stage_pirk_s1_fused": 176, "stage_pirk_s1_psi": 144, "stage_pirk_s1_pi": 112, "stage_pirk2_s2": 240}
PIRK2_MIN_BYTES = 416  # fused minimum per point-step: read u, stale Pi, u_stage, u; write u_stage, u


def workload_config(w):
    full = (w["Nx"], w["Ny"], w["Nz"]) == (2048, 129, 257)
    return {
        "workload": f"FP64 PIRK2 {'large solve' if full else 'reduced grid'}: Nx={w['Nx']} Ny={w['Ny']} "
                    f"Nz={w['Nz']} (Nr={w['Nx']}, Ntheta={w['Ny'] - 1}, Nphi={w['Nz'] - 1}), "
                    f"r in [{w['xmin']:g},{w['xmax']:g}], Kerr-Schild M=1, m={w['m']:g}, outflow, "
                    f"CFL {w['CFL']:g} reference dt rule",
        "grid": [w["Nx"], w["Ny"], w["Nz"]],
        "stepper": "pirk2",
        "refinement": "none (single level)",
        "l2": (("inputs larger than L2 (%.1f GB per state copy)" if 5 * 16 * stored_points(w) > 2 * 126e6 else
                "reduced grid: %.2f GB per state copy, not flushed between steps") % (5 * 16 * stored_points(w) / 1e9)),
        "seed": w["seed"],
    }


def interior_points(w):
    return w["Nx"] * (w["Ny"] - 1) * (w["Nz"] - 1)


def stored_points(w):
    return (w["Nx"] + 5) * (w["Ny"] + 5) * (w["Nz"] + 1)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel):
    """dram bytes per launch from the committed ncu summary, if there is one."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_c1.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.proc = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(gpu_id), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(smax)), "reasons": sorted(reasons),
                "samples": len(sm)}


def oracle_on_workload(w, threads):
    """The oracle (CPU restatement of the reference path) on the workload grid
    itself, loaded with the same seeded initial data as the GPU arm."""
    from oracle.oracle import Oracle, set_threads
    from kg_b200.initial_data import shell_ylm
    set_threads(threads)
    o = Oracle(w["Nx"], w["Ny"], w["Nz"], w["xmin"], w["xmax"], CFL=w["CFL"], m=w["m"])
    u0, _ = shell_ylm(w["Nx"], w["Ny"], w["Nz"], w["xmin"], w["xmax"], seed=w["seed"])
    o.set_state(u0)
    del u0
    return o


def cpu_baseline(w, threads, steps=3):
    """A bounded sample of the same workload on the host cores: `steps` PIRK2
    steps of the oracle on the full workload grid (after one untimed step that
    pages its arrays in)."""
    o = oracle_on_workload(w, threads)
    o.pirk2(1)
    t0 = time.perf_counter()
    o.pirk2(steps)
    dt = time.perf_counter() - t0
    o.close()
    gpsu = interior_points(w) * 2 * steps / dt
    return gpsu, dt, (f"PIRK2 x{steps} on the full workload grid ({w['Nx']}x{w['Ny']}x{w['Nz']}), "
                      f"after one untimed step")


SERVE_DESC = ("scaled serving workload: Poisson arrivals at 2000/s (the offered load exceeds one GPU's "
              "capacity, so solves/s measures sustained throughput), Nr ~ U{128..512 step 64} on r in "
              "[1.8, 1.8+0.1 Nr], Ntheta in {16, 32}, Nphi = 2 Ntheta, m ~ U[0, 0.5], shell r0 ~ U[6, 15], "
              "sigma ~ U[0.8, 2], c_lm (l<=4) N(0, 1e-4), RK4, steps log-uniform [100, 1000] (multiples of 10), "
              "l<=8 waveform at r_ext = 0.8 r_max every 10 steps, 160 GB HBM admission budget; the full serving "
              "description (100 req/s for 120 s, Nr up to 4096, up to 20000 steps) offers several hundred times "
              "one GPU's HBM roofline, so it is scaled down in count, grid and steps")


BATCH_DESC = ("batching form: 512 solves drawn from seed 20240603 (Nr ~ U{128..1024 step 64} on r in "
              "[1.8, 1.8+0.1 Nr], Ntheta in {16, 32, 64}, Nphi = 2 Ntheta, m ~ U[0, 0.5], shell r0 ~ U[6, 15], "
              "sigma ~ U[0.8, 2], c_lm (l<=4) N(0, 1e-4)), RK4; all 512 in FP64 exceed HBM, so they run in "
              "admission waves: the first wave (draw order, 120 GB FP64 budget) is timed over a few steps, plain "
              "FP64 one solve at a time against the same solves batched in FP64 and in the mixed form")


def batch_leg(device, steps=5, budget=120e9, count=512):
    """The batching form on its own solve mix: device time of `steps` RK4 steps of
    the first admission wave, plain FP64 (one solve after another) against one
    persistent launch per stage over all of them (FP64 and mixed)."""
    import torch
    from kg_b200.serve import draw_requests, _bytes_estimate
    from kg_b200.batch import autotune
    reqs = draw_requests(seed=20240603, rate=100.0, count=count, nr=(128, 1024), nr_step=64,
                         ntheta=(16, 32, 64), steps=(2000, 2000), quantum=10)
    waves, cur, used = [], [], 0.0
    for r in reqs:
        b = _bytes_estimate(r, "fp64")
        if cur and used + b > budget:
            waves.append(cur)
            cur, used = [], 0.0
        cur.append(r)
        used += b
    waves.append(cur)
    wave = waves[0]
    shapes = sorted({(r.grid()["Nx"], r.grid()["Ny"], r.grid()["Nz"]) for r in wave})
    sample = shapes[:: max(1, len(shapes) // 6)]
    tune = {p: autotune(sample, device=device, kchunks=(16, 32, 64), steps=2, precision=p) for p in ("fp64", "mixed")}
    torch.cuda.empty_cache()
    eng = engine_leg(wave, device, tune, steps=steps)
    interior = sum(r.Nr * r.Ntheta * 2 * r.Ntheta for r in wave)
    gpsu = lambda ms: interior * 4 * steps / (ms / 1e3)
    return {"workload": BATCH_DESC, "solves_drawn": count, "waves_for_all": len(waves), "wave_solves": len(wave),
            "wave_interior_points": interior, "tuning": {p: _tdesc(t) for p, t in tune.items()},
            "engine_device_time": eng,
            "gpsu": {"plain_fp64": gpsu(eng["plain_fp64_ms"]), "batched_fp64": gpsu(eng["batched_fp64_ms"]),
                     "batched_mixed": gpsu(eng["batched_mixed_ms"])}}


def serve_leg(count, device):
    """plain FP64 (one solve at a time) vs continuous batching, FP64 and mixed, on the same requests"""
    from kg_b200.serve import Server, draw_requests, waveform_error_detail
    from kg_b200.batch import autotune
    reqs = draw_requests(seed=20240602, rate=2000.0, count=count, nr=(128, 512), nr_step=64, ntheta=(16, 32),
                         steps=(100, 1000), quantum=10)
    shapes = sorted({(r.grid()["Nx"], r.grid()["Ny"], r.grid()["Nz"]) for r in reqs})
    sample = shapes[:: max(1, len(shapes) // 6)]
    tune = {p: autotune(sample, device=device, kchunks=(16, 32, 64), steps=2, precision=p) for p in ("fp64", "mixed")}
    plain = Server(mode="plain", device=device).run(reqs)
    batched = Server(mode="batched", device=device, tuning=tune["fp64"]).run(reqs)
    mixed = Server(mode="batched", device=device, tuning=tune["mixed"], precision="mixed").run(reqs)
    strip = lambda d: {k: d[k] for k in ("completed", "wall_s", "solves_per_s", "p50_s", "p99_s") if k in d}
    engine = engine_leg(reqs, device, tune)
    return {"workload": SERVE_DESC, "requests": count, "engine_device_time": engine, "plain_fp64": strip(plain),
            "batched_fp64": dict(strip(batched), peak_live=batched.get("peak_live"), tuning=_tdesc(tune["fp64"])),
            "batched_mixed": dict(strip(mixed), peak_live=mixed.get("peak_live"), tuning=_tdesc(tune["mixed"])),
            "speedup_batched_fp64": batched["solves_per_s"] / plain["solves_per_s"],
            "speedup_batched_mixed": mixed["solves_per_s"] / plain["solves_per_s"],
            "waveform_batched_fp64_vs_plain": _wave(waveform_error_detail(batched, plain)),
            "waveform_batched_mixed_vs_plain_fp64": _wave(waveform_error_detail(mixed, plain))}


def engine_leg(reqs, device, tune, steps=10):
    """Device time (CUDA events, best of 3) of `steps` RK4 steps of every request:
    one after another on its own handle (plain FP64, graph replay) against all of
    them in one batch (FP64 and mixed).  Host-side work of the serving loop
    (request creation, waveform sampling) is outside; the wall-clock serving
    figures above include it."""
    import torch
    from kg_b200.serve import _make_solve
    from kg_b200.batch import Batch
    pts = sum((r.Nr + 5) * (r.Ntheta + 6) * (2 * r.Ntheta + 2) for r in reqs)
    plain_ms = 0.0
    for r in reqs:
        s = _make_solve(r, 8, device)
        s.rk4(nsteps=steps)
        s.synchronize()
        st = torch.cuda.ExternalStream(s._lib.kg_get_stream(s.handle), device=f"cuda:{device}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.rk4(nsteps=steps)
        e1.record(st)
        e1.synchronize()
        plain_ms += e0.elapsed_time(e1)
        s.close()
    out = {"steps": steps, "stored_points": pts, "plain_fp64_ms": plain_ms}
    for prec in ("fp64", "mixed"):
        b = Batch(device, precision=prec)
        b.set_tuning(*tune[prec])
        solves = [_make_solve(r, 8, device) for r in reqs]
        for s in solves:
            b.add(s)
        b.rk4(steps)
        b.synchronize()
        st = torch.cuda.ExternalStream(b.stream, device=f"cuda:{device}")
        best = 1e30
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            b.rk4(steps)
            e1.record(st)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        out[f"batched_{prec}_ms"] = best
        out[f"batched_{prec}_alg_gbs"] = pts * (1360 if prec == "fp64" else 880) * steps / (best / 1e3) / 1e9
        for s in solves:
            b.remove(s)
            s.close()
        b.close()
    out["speedup_batched_fp64"] = plain_ms / out["batched_fp64_ms"]
    out["speedup_batched_mixed"] = plain_ms / out["batched_mixed_ms"]
    return out


def _tdesc(t):
    """a Tuning as the bench line reports it"""
    if t.dispatch == 1:
        form = {0: "one thread per point", 1: "32x8 tiles, register prefetch",
                2: f"32x{t.tile_rows} tiles, TMA ring"}
        return {"dispatch": "concurrent single-solve launches, one stream per solve",
                "stage_kernel_form": form.get(t.variant, t.variant)}
    return {"dispatch": "persistent launch per stage over all solves", "kchunk": t.kchunk, "ctas": t.blocks,
            "tile": f"32x{t.tile_rows}"}


def _wave(d):
    return {"max_rel_l2": d[0], "requests_compared": d[1], "max_abs_l2": d[2],
            "note": "relative error over requests whose FP64 waveform norm exceeds 1e-10; absolute over all"}


def two_shells_device(w, device, Nx=None, xmax=None):
    """The workload's seeded shell (r0 ~ U[8, 15]) plus a second seeded shell
    centred on the extraction radius r = 50 (same form, seed + 1).  Under the
    reference dt rule the workload grid steps dt = 4.5e-4 (the pole term
    e^xmin sin(dtheta/2) dphi binds), so a pulse from r0 <= 15 needs some 8e4
    steps to reach r = 50; the second shell puts signal at the extraction radius
    from the first step of a bounded run."""
    from kg_b200.initial_data import shell_ylm_device
    Nx = Nx or w["Nx"]
    xmax = xmax or w["xmax"]
    u0, _ = shell_ylm_device(Nx, w["Ny"], w["Nz"], w["xmin"], xmax, seed=w["seed"], device=f"cuda:{device}")
    u1, _ = shell_ylm_device(Nx, w["Ny"], w["Nz"], w["xmin"], xmax, seed=w["seed"] + 1, device=f"cuda:{device}",
                             r0_range=(50.0, 50.0))
    u0 += u1
    del u1
    return u0


def precision_leg(w, device, steps=120, every=10, L=64):
    """The precision form on the workload grid: RK4 with the FP32 stencil RHS and
    FP64 state update plus a split-BF16 tensor-core Y_lm projection (l <= L, every
    shell) every `every` steps, against FP64 RK4 with the FP64 projection, from
    the same initial data (two_shells_device).  Device time (CUDA events) of the
    steps and of the projections; errors of phi and Pi, of the l <= 8 detector
    waveforms at r = 12 (inside the first shell) and r = 50 (the extraction
    radius), per mode and in total, and of the last all-shell projection."""
    import torch
    from kg_b200 import ScalarField
    runs = {}
    for prec in ("fp64", "mixed"):
        s = ScalarField(w["Nx"], w["Ny"], w["Nz"], w["xmin"], w["xmax"], w["CFL"], m=w["m"], device=device,
                        l_max=8, n_det=2)
        u0 = two_shells_device(w, device)
        s._ck(s._lib.kg_set_state_device(s.handle, 0, C.c_void_p(u0.data_ptr())))
        s.synchronize()
        del u0
        s.set_detectors([12.0, 50.0])
        s.precision = prec
        lib, h = s._lib, s.handle
        stream = torch.cuda.ExternalStream(lib.kg_get_stream(h), device=f"cuda:{device}")
        alm_p = 1 if prec == "mixed" else 0
        host = np.zeros((w["Nx"], 2 * L + 1, L + 1), np.complex128)
        s.rk4(nsteps=2)  # warm: buffers, graphs
        s._ck(lib.kg_project_all_shells(h, L, alm_p, host.ctypes.data_as(C.POINTER(C.c_double))))
        s.synchronize()
        nk = lib.kg_profile_kinds()
        names = [lib.kg_profile_kind_name(i).decode() for i in range(nk)]
        pms, pcnt = (C.c_double * nk)(), (C.c_longlong * nk)()
        wave = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        step_ms = proj_ms = 0.0
        for q in range(steps // every):
            e0.record(stream)
            s.rk4(nsteps=every)
            e1.record(stream)
            e1.synchronize()
            step_ms += e0.elapsed_time(e1)
            lib.kg_profile_read(h, pms, pcnt)
            lib.kg_profile_enable(h, 1)
            s._ck(lib.kg_project_all_shells(h, L, alm_p, host.ctypes.data_as(C.POINTER(C.c_double))))
            lib.kg_profile_read(h, pms, pcnt)
            lib.kg_profile_enable(h, 0)
            proj_ms += sum(pms[i] for i in range(nk) if names[i].startswith("ylm_all"))
            wave.append(s.proyector_detectors().copy())
        st = torch.empty((w["Nz"] + 1, w["Ny"] + 5, w["Nx"] + 5, 5), dtype=torch.complex128,
                         device=f"cuda:{device}")
        s._ck(lib.kg_get_state_device(h, 0, C.c_void_p(st.data_ptr())))
        s.synchronize()
        runs[prec] = dict(step_ms=step_ms, proj_ms=proj_ms, alm=host.copy(), wave=np.array(wave),
                          phi=st[..., 0].clone(), pi=st[..., 4].clone())
        del st
        s.close()
        torch.cuda.empty_cache()
    pts = interior_points(w) * 4 * steps
    a, b = runs["fp64"], runs["mixed"]
    trel = lambda x, y: float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y))

    def wave_err(d):
        ref, got = a["wave"][:, d], b["wave"][:, d]
        n = np.linalg.norm(ref)
        if n <= 1e-10:
            return {"rel_l2": None, "ref_norm": float(n), "note": "no signal at this radius within the run"}
        per_mode = np.linalg.norm(got - ref, axis=0) / np.maximum(np.linalg.norm(ref, axis=0), 1e-300)
        big = np.linalg.norm(ref, axis=0) > 1e-3 * np.linalg.norm(ref, axis=0).max()
        return {"rel_l2": float(np.linalg.norm(got - ref) / n), "max_per_mode_rel": float(per_mode[big].max()),
                "ref_norm": float(n)}
    return {"workload": f"RK4 on the {w['Nx']}x{w['Ny']}x{w['Nz']} grid, {steps} steps, all-shell Y_lm projection "
                        f"(l<={L}) every {every} steps; detectors at r = 12 and 50; initial data: the workload "
                        f"shell plus a seeded shell at r = 50",
            "steps": steps,
            "fp64_step_gpsu": pts / (a["step_ms"] / 1e3), "mixed_step_gpsu": pts / (b["step_ms"] / 1e3),
            "step_speedup": a["step_ms"] / b["step_ms"],
            "fp64_projection_ms": a["proj_ms"] / (steps // every),
            "tensor_core_projection_ms": b["proj_ms"] / (steps // every),
            "combined_speedup": (a["step_ms"] + a["proj_ms"]) / (b["step_ms"] + b["proj_ms"]),
            "phi_rel_l2_err": trel(b["phi"], a["phi"]), "pi_rel_l2_err": trel(b["pi"], a["pi"]),
            "waveform_r12": wave_err(0), "waveform_r50": wave_err(1),
            "projection_energy_norm_rel_err": float(np.linalg.norm(b["alm"] - a["alm"]) / np.linalg.norm(a["alm"]))}


def c0_leg(device, steps=1000):
    """The plain FP64 test-field description on the configured method: Nr = 256
    on [1.8, 60], 32 x 64 theta x phi cells (Nx=256, Ny=33, Nz=65), Kerr-Schild
    M = 1, m = 0, fourth-order differences, sixth-order Kreiss-Oliger eps = 0.02,
    Sommerfeld outer plane, RK4, 1000 steps, phi = 1e-3 exp(-(r-10)^2) Y_20 with
    exact derivatives, Pi = 0.  dt is the reference rule (CFL 0.25); the
    description's dt = 0.25 dr is run for the same number of steps to record
    whether it stays bounded on this grid (max |u| below 100 x its start)."""
    import torch
    from kg_b200 import ScalarField
    from kg_b200.initial_data import smooth_exact
    Nx, Ny, Nz, xmin, xmax = 256, 33, 65, 1.8, 60.0
    u0 = smooth_exact(Nx, Ny, Nz, xmin, xmax, amp=1e-3, r0=10.0, width=1.0, angular="y20")
    umax0 = float(np.abs(u0).max())

    def run(dt, timed):
        s = ScalarField(Nx, Ny, Nz, xmin, xmax, 0.25, m=0.0, device=device, dt=dt)
        s.set_scheme("configured", 0.02)
        if timed:
            s.u = u0
            s.fill_ghosts_configured()
            s.rk4(nsteps=2)  # warm: buffers, graphs
        s.u = u0
        s.fill_ghosts_configured()
        s.t = 0.0
        stream = torch.cuda.ExternalStream(s._lib.kg_get_stream(s.handle), device=f"cuda:{device}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.rk4(nsteps=steps)
        e1.record(stream)
        e1.synchronize()
        u = s.u
        out = {"dt": s.dt, "t_end": s.t, "ms": e0.elapsed_time(e1), "max_abs_u_end": float(np.abs(u).max())}
        out["bounded"] = bool(np.isfinite(out["max_abs_u_end"]) and out["max_abs_u_end"] < 100 * umax0)
        s.close()
        return out

    ref = run(None, True)
    big = run(0.25 * (xmax - xmin) / Nx, False)
    return {"workload": "Nx=256 Ny=33 Nz=65 on [1.8, 60], configured method (4th-order FD, KO6 0.02, Sommerfeld), "
                        f"RK4 x{steps}, FP64, phi0 = 1e-3 exp(-(r-10)^2) Y20",
            "gpsu": Nx * (Ny - 1) * (Nz - 1) * 4 * steps / (ref["ms"] / 1e3), "ms_per_step": ref["ms"] / steps,
            "dt": ref["dt"], "t_end": ref["t_end"], "max_abs_u_start": umax0,
            "max_abs_u_end": ref["max_abs_u_end"], "bounded": ref["bounded"],
            "dt_0.25dr": {k: big[k] for k in ("dt", "t_end", "max_abs_u_end", "bounded")}}


def refinement_leg(w, device, steps=10, r_fine=(20.0, 15.0, 10.0), wave_steps=16):
    """The workload grid as the coarse level of a Berger-Oliger hierarchy with
    radially nested 2:1 levels inside r < 20, 15, 10 (r_fine); level l takes 2^l
    steps per coarse step.
    * Rates, per stepper (RK4, SSP-RK3, PIRK2, PIRK3): interior points x stages x
      steps summed over levels / device time (CUDA events on the coarse level's
      stream, which every level's work is ordered back into).
    * Waveforms: from the two-shell initial data (two_shells_device), the l <= 8
      detector a_lm at r ~ 12 (on the finest level that covers it) and r ~ 50
      (coarse level), both on a coarse vertex, every coarse step for `wave_steps` steps with RK4 and
      PIRK2, against a uniformly fine solve (the finest level's dr and dt over
      r in [1.8, 60], which holds both radii and is far larger than the signal
      travels in the run) and against the coarse level alone."""
    import torch
    from kg_b200 import ScalarField
    from kg_b200.refinement import BergerOliger

    def load(lv, Nx, xmax):
        u0 = two_shells_device(w, device, Nx=Nx, xmax=xmax)
        lv._ck(lv._lib.kg_set_state_device(lv.handle, 0, C.c_void_p(u0.data_ptr())))
        lv.synchronize()
        del u0

    def make_bo():
        bo = BergerOliger(w["Nx"], w["Ny"], w["Nz"], w["xmin"], w["xmax"], w["CFL"], r_fine=r_fine, m=w["m"],
                          device=device, l_max=8)
        for lv in bo.levels:
            load(lv, lv.Nx, lv.params.xmax)
        return bo

    bo = make_bo()
    l0 = bo.levels[0]
    stream = torch.cuda.ExternalStream(l0._lib.kg_get_stream(l0.handle), device=f"cuda:{device}")
    out = {"workload": f"coarse level = the workload grid; 2:1 levels inside r < {r_fine}, {steps} coarse steps "
                       f"per stepper",
           "levels": [{"Nx": lv.Nx, "r_outer": lv.params.xmax, "dt": lv.dt} for lv in bo.levels]}
    for method, stages in (("rk4", 4), ("rk3", 3), ("pirk2", 2), ("pirk3", 3)):
        getattr(bo, method)(1)
        bo.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        getattr(bo, method)(steps)
        e1.record(stream)
        e1.synchronize()
        bo.synchronize()
        ms = e0.elapsed_time(e1)
        work = sum(lv.Nx * (lv.Ny - 1) * (lv.Nz - 1) * stages * (2 ** l) for l, lv in enumerate(bo.levels)) * steps
        out[method] = {"ms_per_coarse_step": ms / steps, "gpsu": work / (ms / 1e3)}
    finite = True
    for lv in bo.levels:
        lv.density()
        finite = finite and bool(np.isfinite(lv.mass_scalar()))
    out["finite"] = finite
    bo.close()
    torch.cuda.empty_cache()

    # waveforms at r ~ 12 and r ~ 50, on a vertex of the coarse grid, which is a
    # vertex of every finer grid too: the detectors take the vertex at or below
    # their radius without radial interpolation (the reference's index search),
    # so all runs sample the same radius
    dx0 = (w["xmax"] - w["xmin"]) / w["Nx"]
    on_vertex = lambda r: w["xmin"] + round((r - w["xmin"]) / dx0) * dx0 + 1e-6 * dx0
    r_in, r_ext = on_vertex(12.0), on_vertex(50.0)
    nlev = len(r_fine) + 1
    sub = 2 ** (nlev - 1)
    waves = {}
    for method in ("rk4", "pirk2"):
        bo = make_bo()
        dt0 = bo.levels[0].dt
        lin = max(l for l in range(nlev) if l == 0 or r_fine[l - 1] > r_in + 1.0)
        bo.levels[0].set_detectors([r_in, r_ext])
        bo.levels[lin].set_detectors([r_in, r_ext if lin == 0 else r_in])
        hw = []
        for _ in range(wave_steps):
            getattr(bo, method)(1)
            a0 = bo.levels[0].proyector_detectors().copy()
            ai = bo.levels[lin].proyector_detectors().copy()
            hw.append(np.stack([ai[0], a0[1]]))
        finest_dx = bo.levels[-1].dx
        bo.close()
        torch.cuda.empty_cache()
        # the coarse level alone
        cs = ScalarField(w["Nx"], w["Ny"], w["Nz"], w["xmin"], w["xmax"], w["CFL"], m=w["m"], device=device,
                         l_max=8, n_det=2)
        load(cs, w["Nx"], w["xmax"])
        cs.set_detectors([r_in, r_ext])
        cw = []
        for _ in range(wave_steps):
            getattr(cs, method)(nsteps=1)
            cw.append(cs.proyector_detectors().copy())
        cs.close()
        torch.cuda.empty_cache()
        # uniformly fine: the finest level's dr and dt over [1.8, 60]
        nf = int(round((60.0 - w["xmin"]) / finest_dx))
        xf = w["xmin"] + nf * finest_dx
        fsv = ScalarField(nf, w["Ny"], w["Nz"], w["xmin"], xf, w["CFL"], m=w["m"], device=device, l_max=8,
                          n_det=2, dt=dt0 / sub)
        load(fsv, nf, xf)
        fsv.set_detectors([r_in, r_ext])
        fw = []
        for _ in range(wave_steps):
            getattr(fsv, method)(nsteps=sub)
            fw.append(fsv.proyector_detectors().copy())
        fsv.close()
        torch.cuda.empty_cache()
        hw, cw, fw = np.array(hw), np.array(cw), np.array(fw)
        rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
        waves[method] = {
            "radii": [r_in, r_ext],
            "r12": {"hierarchy_vs_uniform_fine": rel(hw[:, 0], fw[:, 0]),
                    "coarse_vs_uniform_fine": rel(cw[:, 0], fw[:, 0]), "level": lin,
                    "ref_norm": float(np.linalg.norm(fw[:, 0]))},
            "r50": {"hierarchy_vs_uniform_fine": rel(hw[:, 1], fw[:, 1]),
                    "coarse_vs_uniform_fine": rel(cw[:, 1], fw[:, 1]),
                    "hierarchy_vs_coarse": rel(hw[:, 1], cw[:, 1]), "level": 0,
                    "ref_norm": float(np.linalg.norm(fw[:, 1]))},
            "uniform_fine": {"Nx": nf, "r": [w["xmin"], xf], "dt": dt0 / sub}}
    out["waveforms"] = dict(waves, steps=wave_steps,
                            note="l <= 8 a_lm at each coarse step, relative L2 over all samples and modes; initial "
                                 "data: the workload shell plus a seeded shell at r = 50")
    return out


def projection_leg(mol, lib, h, L=64, reps=3):
    """All-shell Y_lm projection to l <= L over every radial shell of the solve's
    current state (the precision form's diagnostic): the split-BF16 tcgen05 GEMM
    [2 Nx x K] . [K x 2 Nm] (K = Ny Nz sphere points, Nm = (L+1)(L+2)/2 modes
    with m >= 0) timed per kernel with CUDA events, and its error against the
    FP64 projection of the same state."""
    Nx, Ny, Nz = mol.Nx, mol.Ny, mol.Nz
    K = Ny * Nz
    Nm = (L + 1) * (L + 2) // 2
    pad = lambda v, b: (v + b - 1) // b * b
    Mp, Np, Kp = pad(2 * Nx, 128), pad(2 * Nm, 256), pad(K, 64)
    nk = lib.kg_profile_kinds()
    names = [lib.kg_profile_kind_name(i).decode() for i in range(nk)]
    ms = (C.c_double * nk)()
    cnt = (C.c_longlong * nk)()

    def timed(precision, n):
        out = np.zeros((Nx, 2 * L + 1, L + 1), np.complex128)
        lib.kg_profile_read(h, ms, cnt)
        lib.kg_profile_enable(h, 1)
        for _ in range(n):
            mol._ck(lib.kg_project_all_shells(h, L, precision, out.ctypes.data_as(C.POINTER(C.c_double))))
        lib.kg_profile_read(h, ms, cnt)
        lib.kg_profile_enable(h, 0)
        return out, {names[i]: (ms[i], cnt[i]) for i in range(nk) if cnt[i] > 0}

    timed(1, 1)  # tables, B operand, tensor maps
    a_t, kt = timed(1, reps)
    a_64, k64 = timed(0, 1)
    g_ms, g_n = kt["ylm_all_gemm_bf16x3"]
    p_ms, p_n = kt.get("ylm_all_prepare", (0.0, 1))
    f_ms, _ = k64["ylm_all_fp64"]
    issued = 3 * 2.0 * Mp * Np * Kp
    useful = 2.0 * (2 * Nx) * K * (2 * Nm)
    complex_equiv = 8.0 * Nx * K * (L + 1) ** 2
    gemm_s = g_ms / g_n / 1e3
    d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = float(d.get("bf16_tflops", 1590.0))
    diff = a_t - a_64
    shell_err = np.sqrt(np.sum(np.abs(diff) ** 2, axis=(1, 2)))
    shell_norm = np.sqrt(np.sum(np.abs(a_64) ** 2, axis=(1, 2)))
    # shells where the field is below 1e-6 of its peak shell (the Gaussian tail, down
    # to values FP32 cannot hold) are left out of the per-shell ratios
    live = shell_norm > 1e-6 * shell_norm.max()
    coef_err = np.abs(diff).reshape(Nx, -1).max(axis=1)
    return {
        "workload": f"a_lm for l<={L} on all {Nx} vertex shells of the {Ny}x{Nz} sphere (K={K}), "
                    f"GEMM [{2 * Nx}x{K}].[{K}x{2 * Nm}] padded to {Mp}x{Kp}x{Np}, split-BF16 3 passes",
        "gemm_ms": g_ms / g_n, "prepare_ms_per_call": p_ms / reps, "fp64_ms": f_ms,
        "tensor_roofline": {"bound": "tensor", "achieved": issued / gemm_s / 1e12, "peak": peak,
                            "unit": "TFLOP/s", "frac": issued / gemm_s / 1e12 / peak,
                            "peak_source": "measured bf16 burst" if d else "fallback",
                            "issued_flop_per_launch": issued},
        "useful_real_tflops": useful / gemm_s / 1e12,
        "complex_equiv_tflops": complex_equiv / gemm_s / 1e12,
        "speedup_vs_fp64_projection": f_ms / (g_ms / g_n + p_ms / reps),
        "energy_norm_rel_err_vs_fp64": float(np.linalg.norm(diff) / np.linalg.norm(a_64)),
        "max_shell_energy_rel_err": float((shell_err[live] / shell_norm[live]).max()) if live.any() else None,
        "max_coef_err_over_shell_norm": float((coef_err[live] / shell_norm[live]).max()) if live.any() else None,
        "error_note": "each coefficient carries an absolute error ~2^-17 of its shell's norm (BF16 split); the "
                      "energy-norm error sums it over all (L+1)^2 modes while the field's energy sits in l<=4",
    }


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's PIRK2 path
    (the oracle; the Fortran/MPI reference cannot be built on this image) on
    the same workload grid, initial data, metric and unit as the GPU arm, all
    host threads, one PIRK2 step per step.  Only the oracle's library is
    mapped: the package's solver library stays unloaded."""
    from kg_b200 import capi, replicas
    _, rank, _ = replicas.rank_env()
    if rank != 0:
        return 0
    w = WORKLOAD
    threads = os.cpu_count() or 1
    o = oracle_on_workload(w, threads)
    for _ in range(args.warmup):
        o.pirk2(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.pirk2(1)
    el = time.perf_counter() - t0
    o.close()
    if capi._lib is not None:
        raise RuntimeError("the reference arm mapped libkg_b200.so")
    val = interior_points(w) * 2 * args.steps / el
    sample = (f"PIRK2 on the full workload grid ({w['Nx']}x{w['Ny']}x{w['Nz']}), one step per step, "
              f"{args.warmup} untimed warm-up steps")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic (seeded Gaussian shell x Y_lm, l<=4)",
            "config": dict(workload_config(w), parallelism="host threads"),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def summarize(line, steps):
    """The numbers of every leg in one short object (kept as the line's last key)."""
    g = lambda d, *ks: _dig(d, ks)
    out = {"pirk2_ggpsu": line["value"] / 1e9, "ms_per_step": line["ms_per_step"],
           "roofline_frac": g(line, "roofline", "frac"), "step_hbm_frac": line["step_bandwidth_gbs"] /
           line["roofline"]["peak"] if line.get("roofline") else None,
           "e2e_ggpsu": (line["e2e"]["value"] / 1e9) if line.get("e2e") else None, "e2e_steps": steps,
           "steppers_ggpsu": {k: v / 1e9 for k, v in line.get("steppers_gpsu", {}).items()},
           "cpu_baseline_mgpsu": (g(line, "cpu_baseline", "value") or 0) / 1e6 or None}
    if "projection" in line:
        p = line["projection"]
        out["projection"] = {"gemm_ms": p["gemm_ms"], "tensor_frac": g(p, "tensor_roofline", "frac"),
                             "energy_rel_err": p["energy_norm_rel_err_vs_fp64"]}
    if "precision" in line:
        p = line["precision"]
        out["precision"] = {"step_speedup": p["step_speedup"], "combined_speedup": p["combined_speedup"],
                            "phi_rel_err": p["phi_rel_l2_err"], "pi_rel_err": p["pi_rel_l2_err"],
                            "wave_r12_rel_err": g(p, "waveform_r12", "rel_l2"),
                            "wave_r50_rel_err": g(p, "waveform_r50", "rel_l2"), "steps": p.get("steps")}
    if "refinement" in line:
        r = line["refinement"]
        out["refinement_ggpsu"] = {k: r[k]["gpsu"] / 1e9 for k in ("rk4", "rk3", "pirk2", "pirk3") if k in r}
        if "waveforms" in r:
            out["refinement_waveform_rel_err"] = {
                m: {rad: {k: g(r, "waveforms", m, rad, k) for k in ("hierarchy_vs_uniform_fine",
                                                                     "coarse_vs_uniform_fine")}
                    for rad in ("r12", "r50")} for m in ("rk4", "pirk2")}
    if "c0_configured" in line:
        out["c0_ms_per_step"] = line["c0_configured"]["ms_per_step"]
    if "batching" in line:
        e = line["batching"]["engine_device_time"]
        out["batching_speedup"] = {"fp64": e["speedup_batched_fp64"], "mixed": e["speedup_batched_mixed"]}
    if "serving" in line:
        sv = line["serving"]
        out["serving"] = {"solves_per_s": {k: g(sv, k, "solves_per_s") for k in
                                           ("plain_fp64", "batched_fp64", "batched_mixed")},
                          "speedup_mixed": sv["speedup_batched_mixed"],
                          "device_speedup_mixed": g(sv, "engine_device_time", "speedup_batched_mixed"),
                          "wave_err_mixed": g(sv, "waveform_batched_mixed_vs_plain_fp64", "max_rel_l2")}
    return out


def _dig(d, ks):
    for k in ks:
        if not isinstance(d, dict) or k not in d:
            return None
        d = d[k]
    return d


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=150)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kg", choices=["kg", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default=None,
                    help="Nx,Ny,Nz override (profiling captures of a smaller case); r range scales with Nx")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end and other-stepper legs")
    ap.add_argument("--variant", type=int, default=None, help="stage-kernel form (kg_set_kernel_variant)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving leg")
    ap.add_argument("--serve-count", type=int, default=120)
    ap.add_argument("--no-projection", action="store_true", help="skip the all-shell Y_lm projection leg")
    ap.add_argument("--no-precision", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-refinement", action="store_true", help="skip the Berger-Oliger leg")
    ap.add_argument("--no-c0", action="store_true", help="skip the configured-method test-field leg")
    ap.add_argument("--no-batch", action="store_true", help="skip the batching-form leg")
    args = ap.parse_args()
    if args.grid:
        nx, ny, nz = (int(v) for v in args.grid.split(","))
        WORKLOAD.update(Nx=nx, Ny=ny, Nz=nz,
                        xmax=WORKLOAD["xmin"] + (WORKLOAD["xmax"] - WORKLOAD["xmin"]) * nx / 2048)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    from kg_b200 import ScalarField, replicas
    from kg_b200.initial_data import shell_ylm_device

    world, rank, local = replicas.rank_env()
    torch.cuda.set_device(local)
    replicas.init(world, backend="nccl", timeout_s=120)
    w = WORKLOAD
    mol = ScalarField(w["Nx"], w["Ny"], w["Nz"], w["xmin"], w["xmax"], w["CFL"], m=w["m"], device=local,
                      save=10 * 0.25 * 0.0018, l_max=8)
    lib, h = mol._lib, mol.handle
    if args.variant is not None:
        mol._ck(lib.kg_set_kernel_variant(h, args.variant))
    u0, _ = shell_ylm_device(w["Nx"], w["Ny"], w["Nz"], w["xmin"], w["xmax"],
                             seed=replicas.replica_seed(w["seed"], rank), device=f"cuda:{local}")
    mol._ck(lib.kg_set_state_device(h, 0, C.c_void_p(u0.data_ptr())))
    mol.synchronize()
    stream = torch.cuda.ExternalStream(lib.kg_get_stream(h), device=f"cuda:{local}")

    def barrier():
        replicas.barrier(world)

    # ---- device-resident timing
    for _ in range(args.warmup):
        mol.pirk2(1)
    mol.synchronize()
    nk = lib.kg_profile_kinds()
    ms = (C.c_double * nk)()
    cnt = (C.c_longlong * nk)()
    lib.kg_profile_read(h, ms, cnt)
    lib.kg_profile_enable(h, 1)
    barrier()
    torch.cuda.synchronize()
    gpu_id = torch.cuda.get_device_properties(local).uuid
    clocks = ClockSampler(f"GPU-{gpu_id}" if gpu_id else local)
    launches0 = lib.kg_launch_count(h)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        mol.pirk2(1)
    e1.record(stream)
    e1.synchronize()
    clk = clocks.stop()
    launches = lib.kg_launch_count(h) - launches0
    el_ms = e0.elapsed_time(e1)
    lib.kg_profile_read(h, ms, cnt)
    lib.kg_profile_enable(h, 0)
    el_ms = replicas.max_over_ranks(el_ms, world, device=f"cuda:{local}")
    kinds = {lib.kg_profile_kind_name(i).decode(): (ms[i], cnt[i]) for i in range(nk) if cnt[i] > 0}

    # other steppers, briefly (device-resident, same grid)
    per_stepper = {}
    stages = {"pirk2": 2, "pirk3": 3, "rk3": 3, "rk4": 4}
    for meth in (() if args.no_e2e else ("pirk3", "rk3", "rk4")):
        # warm-up: the buffers, and the captured graphs of both Pi-slot parities
        getattr(mol, meth)(nsteps=4) if meth.startswith("rk") else getattr(mol, meth)(4)
        mol.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n = 5
        a0.record(stream)
        getattr(mol, meth)(nsteps=n) if meth.startswith("rk") else getattr(mol, meth)(n)
        a1.record(stream)
        a1.synchronize()
        per_stepper[meth] = interior_points(w) * stages[meth] * n / (a0.elapsed_time(a1) / 1e3)

    # ---- end to end through the C ABI with pinned host buffers
    state_bytes = 5 * 16 * stored_points(w)
    # one pinned host buffer holds the input and then receives the result: kg_set_state
    # returns after its copy has landed, so the download may overwrite it (5.7 GB of
    # pinned memory per rank instead of 11.4)
    host_u = None
    if not args.no_e2e:
        host_u = torch.empty(u0.numel() * 2, dtype=torch.float64, pin_memory=True)
        host_u.copy_(torch.view_as_real(u0).reshape(-1))
    del u0
    mass = C.c_double(0.0)
    Dp = C.POINTER(C.c_double)
    p_in = p_out = C.cast(C.c_void_p(host_u.data_ptr()), Dp) if host_u is not None else None
    mol.density()
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    if not args.no_e2e:
        mol._ck(lib.kg_set_state(h, 0, p_in))
        for l in range(1, args.steps + 1):
            mol._ck(lib.kg_pirk2(h, 1))
            mol._ck(lib.kg_diagnostic(h, l, C.byref(mass)))
        mol._ck(lib.kg_get_state(h, 0, p_out))
    f1.record(stream)
    f1.synchronize()
    e2e_ms = replicas.max_over_ranks(f0.elapsed_time(f1), world, device=f"cuda:{local}")
    del host_u, p_in, p_out  # pinned host memory, not needed by the legs below

    pts = interior_points(w)
    value = replicas.job_rate(pts * 2 * args.steps, world, el_ms)
    e2e_value = replicas.job_rate(pts * 2 * args.steps, world, e2e_ms)

    # roofline of the dominant kernel
    stage_kinds = {k: v for k, v in kinds.items() if k in ALG_BYTES}
    dom = max(stage_kinds.items(), key=lambda kv: kv[1][0])[0] if stage_kinds else "stage_pirk2_s2"
    dms, dcnt = kinds.get(dom, (0.0, 1))
    peak, peak_kind = measured_peaks()
    alg = ALG_BYTES.get(dom, 0) * stored_points(w)
    achieved = alg / (dms / dcnt / 1e3) / 1e9 if dcnt else 0.0
    tr = profile_traffic(dom)
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": tr,
                "algorithmic_bytes_per_launch": alg, "avg_launch_ms": dms / dcnt if dcnt else None}
    step_bytes = PIRK2_MIN_BYTES * stored_points(w)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": el_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c128", "data": "synthetic (seeded Gaussian shell x Y_lm, l<=4)",
            "config": dict(workload_config(w), parallelism=f"replicas x{world}"),
            "roofline": roofline,
            "step_bandwidth_gbs": step_bytes / (el_ms / args.steps / 1e3) / 1e9,
            "kernels": {k: {"ms": v[0], "launches": v[1]} for k, v in kinds.items()},
            "steppers_gpsu": dict(per_stepper, pirk2=value / world),
            "e2e": None if args.no_e2e else {
                "value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": state_bytes / args.steps,
                "d2h_bytes_per_step": (state_bytes + 8 * args.steps) / args.steps},
            "gpu_launches": int(launches), "clocks": clk}
    if rank == 0 and world == 1 and not args.no_projection:
        line["projection"] = projection_leg(mol, lib, h)
    if rank == 0 and world == 1 and not args.grid and not (args.no_precision and args.no_serve and
                                                            args.no_refinement and args.no_c0 and args.no_batch):
        mol.close()  # the legs below allocate their own solves
        torch.cuda.empty_cache()
        if not args.no_precision:
            line["precision"] = precision_leg(w, local)
        if not args.no_refinement:
            line["refinement"] = refinement_leg(w, local)
        if not args.no_c0:
            line["c0_configured"] = c0_leg(local)
        if not args.no_batch:
            line["batching"] = batch_leg(local)
        if not args.no_serve:
            line["serving"] = serve_leg(args.serve_count, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, secs, sample = cpu_baseline(w, threads)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                                "seconds": secs}
    if rank == 0:
        line["summary"] = summarize(line, args.steps)  # last key: the side legs in a few numbers
        print(json.dumps(line), flush=True)
    mol.close()
    replicas.finish(world)
    return 0


if __name__ == "__main__":
    sys.exit(main())
