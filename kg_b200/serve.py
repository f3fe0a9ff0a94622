"""Serving loop: continuous batching of Klein-Gordon solves on one GPU.

Requests (grid size, field mass, initial data, step count) arrive over time;
the server admits them against an HBM budget as memory frees up, keeps every
live solve's state on the device, advances all live solves together through
the batched engine (one persistent launch per RK4 stage over all of them, a
step replayed from a CUDA graph), samples each solve's l <= l_max waveform
a_lm(t) at r_ext = 0.8 r_max every `save_every` steps, and retires a solve --
returning its waveform -- as soon as it has run its steps.  New arrivals are
set up (host and device) while a quantum runs and step from the next one, so
requests that arrive while others are on the GPU overlap with them.

`mode="plain"` serves the same requests one at a time through the single-solve
path (kg_rk4 on its own handle), the baseline the batched form is compared
with.  `precision="mixed"` runs the batched solves with the FP32 stencil RHS and
the FP64 state update (kg_batch_set_precision).

Failures stay with the request that caused them: a request whose solve cannot
be created (bad parameters, device memory exhausted) is refused and reported,
one withdrawn by its `cancel_at` time leaves at the next quantum boundary with
the waveform it has so far, and a solve whose waveform sample is not finite is
retired as failed; in each case its device memory returns to the admission
budget and the other solves run on.

The reference has no serving layer (one MPI job per solve); the solve itself
is the reference's RK4 path (MoL/lines_method_lib.f90:411-474) and the
waveform is its detector projection (MoL/diagnostic_lib.f90:231-250).
"""
from __future__ import annotations

import ctypes as C
import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    rid: int
    arrival: float       # seconds after the start of the run
    Nr: int              # radial cells
    Ntheta: int          # theta cells (reference Ny = Ntheta + 1, Nz = 2 Ntheta + 1)
    m: float             # field mass
    seed: int            # initial-data seed (shell centre, width, c_lm)
    steps: int
    r0: float = 10.0
    sigma: float = 1.5
    cancel_at: float | None = None  # withdrawn at this time (seconds after the start), if set

    def grid(self):
        return dict(Nx=self.Nr, Ny=self.Ntheta + 1, Nz=2 * self.Ntheta + 1, xmin=1.8, xmax=1.8 + 0.1 * self.Nr)

    def points(self):
        g = self.grid()
        return (g["Nx"] + 5) * (g["Ny"] + 5) * (g["Nz"] + 1)


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    done: float
    steps: int
    times: np.ndarray = field(repr=False)
    alm: np.ndarray = field(repr=False)   # (samples, 2L+1, L+1) complex
    status: str = "done"                  # "done", "cancelled" or "failed"
    reason: str = ""

    @property
    def latency(self):
        return self.done - self.arrival


def draw_requests(seed, rate, count, nr=(128, 1024), nr_step=64, ntheta=(16, 32, 64), steps=(500, 20000),
                  mass=(0.0, 0.5), r0=(6.0, 15.0), sigma=(0.8, 2.0), quantum=10):
    """Poisson arrivals at `rate` per second; parameters drawn as in the batched
    benchmark description (Nr uniform on a grid of nr_step, Ntheta from a set,
    Nphi = 2 Ntheta, log-uniform step counts rounded up to the quantum)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        n_r = int(rng.choice(np.arange(nr[0], nr[1] + 1, nr_step)))
        nt = int(rng.choice(ntheta))
        st = int(math.exp(rng.uniform(math.log(steps[0]), math.log(steps[1]))))
        st = max(quantum, int(math.ceil(st / quantum)) * quantum)
        out.append(Request(rid=i, arrival=t, Nr=n_r, Ntheta=nt, m=float(rng.uniform(*mass)),
                           seed=int(rng.integers(1 << 30)), steps=st, r0=float(rng.uniform(*r0)),
                           sigma=float(rng.uniform(*sigma))))
    return out


def _make_solve(req, l_max, device):
    from .lines_method import ScalarField
    from .initial_data import shell_ylm_device
    g = req.grid()
    s = ScalarField(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], 0.25, m=req.m, l_max=l_max, n_det=2,
                    device=device)
    try:
        u0, _ = shell_ylm_device(g["Nx"], g["Ny"], g["Nz"], g["xmin"], g["xmax"], seed=req.seed,
                                 device=f"cuda:{max(device, 0)}", sigma=req.sigma, r0_range=(req.r0, req.r0))
        s._ck(s._lib.kg_set_state_device(s.handle, 0, C.c_void_p(u0.data_ptr())))
        s.synchronize()
        del u0
        r_max = s.r_max
        s.set_detectors([0.8 * r_max, 0.8 * r_max])
    except BaseException:
        s.close()  # the handle's device memory goes back at once, not at collection
        raise
    return s


# what creating a solve raises when its parameters are refused (KG_EINVAL) or its
# device memory cannot be had
_CREATE_ERRORS = (RuntimeError, ValueError, MemoryError)


def _ended(r, admitted, done, ts, alms, status, reason):
    return Result(r.rid, r.arrival, admitted, done, r.steps, np.array(ts), np.array(alms), status, reason)


def _bytes_estimate(req, precision="fp64"):
    """device bytes of a live solve: u (5 FP64 variables, 80 B per point), the
    RK4 stage buffers and increment sum (15 variables: FP64 240 B, mixed FP32
    120 B per point), staging for the layout conversion (80 B), tables and
    detector data (small)."""
    per_point = 400 if precision == "fp64" else 280
    return req.points() * per_point + (64 << 20)


class Server:
    def __init__(self, mode="batched", hbm_budget=160e9, save_every=10, l_max=8, device=0, tuning=None,
                 max_live=4096, precision="fp64"):
        if mode not in ("batched", "plain"):
            raise ValueError("mode is 'batched' or 'plain'")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision is 'fp64' or 'mixed'")
        self.mode, self.budget, self.q, self.l_max, self.device = mode, hbm_budget, save_every, l_max, device
        self.tuning, self.max_live, self.precision = tuning, max_live, precision

    def _sample(self, s):
        a = s.proyector_detectors()
        return a[0].copy()

    def run(self, requests):
        reqs = sorted(requests, key=lambda r: r.arrival)
        if self.mode == "plain":
            return self._run_plain(reqs)
        return self._run_batched(reqs)

    def _run_plain(self, reqs):
        results = []
        t0 = time.perf_counter()
        for r in reqs:
            now = time.perf_counter() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
            admitted = time.perf_counter() - t0
            if _bytes_estimate(r, self.precision) > self.budget:
                results.append(_ended(r, admitted, admitted, [], [], "failed", "exceeds the HBM budget alone"))
                continue
            if r.cancel_at is not None and r.cancel_at <= admitted:
                results.append(_ended(r, admitted, admitted, [], [], "cancelled", "withdrawn before admission"))
                continue
            try:
                s = _make_solve(r, self.l_max, self.device)
            except _CREATE_ERRORS as e:
                results.append(_ended(r, admitted, admitted, [], [], "failed", f"not created: {e}"))
                continue
            s.precision = self.precision
            ts, alms = [], []
            done_steps = 0
            status, reason = "done", ""
            while done_steps < r.steps:
                if r.cancel_at is not None and time.perf_counter() - t0 >= r.cancel_at:
                    status, reason = "cancelled", f"withdrawn after {done_steps} steps"
                    break
                s.rk4(nsteps=self.q)
                done_steps += self.q
                alms.append(self._sample(s))
                ts.append(s.t)
                if not np.all(np.isfinite(alms[-1])):
                    status, reason = "failed", f"non-finite waveform after {done_steps} steps"
                    break
            done = time.perf_counter() - t0
            results.append(_ended(r, admitted, done, ts, alms, status, reason))
            s.close()
        return self._summary(results, time.perf_counter() - t0)

    def _run_batched(self, reqs):
        from .batch import Batch
        batch = Batch(self.device, precision=self.precision)
        if self.tuning:
            batch.set_tuning(*self.tuning)
        pending = deque()
        live = []  # [req, solve, steps_done, admitted, times, alms]
        used = 0.0
        results = []
        i_next = 0
        t0 = time.perf_counter()
        peak_live = 0
        while i_next < len(reqs) or pending or live:
            now = time.perf_counter() - t0
            while i_next < len(reqs) and reqs[i_next].arrival <= now:
                pending.append(reqs[i_next])
                i_next += 1
            stepping = bool(live)
            if stepping:
                peak_live = max(peak_live, len(live))
                batch.rk4(self.q)  # queued on the device; the host prepares arrivals meanwhile
            # admission against the HBM budget, first come first served: the new
            # solves are created and join the batch while the quantum runs; they
            # are appended after the live members, and step from the next quantum
            joined = []
            while pending and len(live) + len(joined) < self.max_live:
                need = _bytes_estimate(pending[0], self.precision)
                now = time.perf_counter() - t0
                if need > self.budget:
                    r = pending.popleft()
                    results.append(_ended(r, now, now, [], [], "failed", "exceeds the HBM budget alone"))
                    continue
                if used + need > self.budget:
                    break
                r = pending.popleft()
                if r.cancel_at is not None and r.cancel_at <= now:
                    results.append(_ended(r, now, now, [], [], "cancelled", "withdrawn before admission"))
                    continue
                try:
                    s = _make_solve(r, self.l_max, self.device)
                except _CREATE_ERRORS as e:
                    results.append(_ended(r, now, now, [], [], "failed", f"not created: {e}"))
                    continue
                batch.add(s)
                used += _bytes_estimate(r, self.precision)
                joined.append([r, s, 0, time.perf_counter() - t0, [], []])
            still = []
            if stepping:
                # every member's waveform sample from one batched launch sequence;
                # the live solves are the first len(live) members
                samples = batch.proyector_detectors()
                for entry, a in zip(live, samples):
                    r, s = entry[0], entry[1]
                    entry[2] += self.q
                    entry[5].append(a[0].copy())
                    entry[4].append(s.t)
                    now = time.perf_counter() - t0
                    status = None
                    if not np.all(np.isfinite(entry[5][-1])):
                        status, reason = "failed", f"non-finite waveform after {entry[2]} steps"
                    elif entry[2] >= r.steps:
                        status, reason = "done", ""
                    elif r.cancel_at is not None and now >= r.cancel_at:
                        status, reason = "cancelled", f"withdrawn after {entry[2]} steps"
                    if status is None:
                        still.append(entry)
                        continue
                    batch.remove(s)
                    results.append(_ended(r, entry[3], now, entry[4], entry[5], status, reason))
                    used -= _bytes_estimate(r, self.precision)
                    s.close()
            live = still + joined
            # with nothing live and nothing pending, wait for the next arrival (with
            # requests pending, admission ran before this quantum's retirements freed
            # their memory, and the next pass admits them)
            if not live and not pending and i_next < len(reqs):
                time.sleep(max(0.0, reqs[i_next].arrival - (time.perf_counter() - t0)))
        wall = time.perf_counter() - t0
        batch.close()
        out = self._summary(results, wall)
        out["peak_live"] = peak_live
        return out

    @staticmethod
    def _summary(results, wall):
        """rates and latencies over the requests served to the end; the
        cancelled and failed ones are listed with their reasons"""
        ok = [r for r in results if r.status == "done"]
        lat = np.array([r.latency for r in ok])
        return {"results": sorted(ok, key=lambda r: r.rid), "wall_s": wall, "completed": len(ok),
                "solves_per_s": len(ok) / wall if wall > 0 else 0.0,
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "cancelled": sorted((r for r in results if r.status == "cancelled"), key=lambda r: r.rid),
                "failed": sorted((r for r in results if r.status == "failed"), key=lambda r: r.rid)}


def waveform_error(a, b, floor=1e-10):
    """max over requests of the relative L2 difference of two runs' waveforms,
    over the requests whose reference waveform (b) has L2 norm above `floor`.
    Below it the waveform at r_ext is the far tail of the initial shell (values
    down to 1e-150 when the pulse has not reached r_ext); such values are under
    FP32's range and resolution relative to the field, and a relative error of
    them says nothing about the solve."""
    worst = 0.0
    for ra, rb in zip(a["results"], b["results"]):
        n = np.linalg.norm(rb.alm)
        if n > floor:
            worst = max(worst, float(np.linalg.norm(ra.alm - rb.alm) / n))
    return worst


def waveform_error_detail(a, b, floor=1e-10):
    """(max relative L2 over requests above `floor`, number of such requests,
    max absolute L2 difference over all requests)"""
    worst, count, absmax = 0.0, 0, 0.0
    for ra, rb in zip(a["results"], b["results"]):
        n = np.linalg.norm(rb.alm)
        d = float(np.linalg.norm(ra.alm - rb.alm))
        absmax = max(absmax, d)
        if n > floor:
            count += 1
            worst = max(worst, d / n)
    return worst, count, absmax
