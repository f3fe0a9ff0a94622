"""Batched engine and its launch-shape tuner.

`Batch` advances many independent solves (each a `ScalarField` with its own
grid, field mass and state) together by RK4: every stage is one persistent
launch over the ragged work list of all members' tiles plus one batched ghost
fill, and a step is replayed from a CUDA graph (kg_batch_* in
include/kg_capi.h).  Members keep their handles for state exchange and
diagnostics.

`autotune` picks how a batch runs by timing candidates on scratch solves of
the same grid shapes (the live solves are never advanced by the tuning):
  * dispatch 0, one persistent launch per stage over all members: the phi
    planes per work item (kchunk), the number of persistent CTAs and the tile
    height (32 x 8 or 32 x 4 (r, theta) tiles);
  * dispatch 1, every member's own single-solve kernels on its own stream, all
    members concurrently: the stage-kernel form, i.e. the tile shape of the
    stage kernels (32 x 8 or 32 x 4 tiles fed by TMA, 32 x 8 tiles with
    register prefetch, or one thread per point in rows of 128).
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import capi


class Batch:
    """Solves advanced together by RK4 in one persistent launch per stage.
    precision: 'fp64' (default) or 'mixed' (FP32 stencil RHS, FP64 state update)."""

    def __init__(self, device=-1, precision="fp64"):
        self._lib = capi.load()
        h = C.c_void_p()
        rc = self._lib.kg_batch_create(device, C.byref(h))
        if rc != capi.KG_OK:
            raise capi.KgError(rc, "kg_batch_create failed")
        self._b = h
        self.members = []
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision is 'fp64' or 'mixed'")
        if precision == "mixed":
            self._ck(self._lib.kg_batch_set_precision(self._b, 1))
        self.precision = precision

    def _ck(self, rc):
        if rc != capi.KG_OK:
            raise capi.KgError(rc, self._lib.kg_batch_last_error(self._b).decode())

    def close(self):
        if getattr(self, "_b", None):
            self._lib.kg_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, solver):
        self._ck(self._lib.kg_batch_add(self._b, solver.handle))
        self.members.append(solver)

    def remove(self, solver):
        self._ck(self._lib.kg_batch_remove(self._b, solver.handle))
        self.members.remove(solver)

    def __len__(self):
        return self._lib.kg_batch_size(self._b)

    def rk4(self, nsteps=1):
        self._ck(self._lib.kg_batch_rk4(self._b, nsteps))

    def synchronize(self):
        self._ck(self._lib.kg_batch_synchronize(self._b))

    def proyector_detectors(self):
        """every member's detector a_lm (n_det, 2L+1, L+1), in member order, from
        one batched launch sequence and one synchronisation"""
        sizes = [(m.n_det, 2 * m.l_max + 1, m.l_max + 1) for m in self.members]
        out = np.zeros(sum(a * b * c for a, b, c in sizes), np.complex128)
        if self._lib.kg_batch_alm_count(self._b) != out.size:
            raise RuntimeError("batch members' detector tables differ from their Python views")
        if out.size:
            self._ck(self._lib.kg_batch_proyector_detectors(
                self._b, out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double))))
        res, off = [], 0
        for a, b, c in sizes:
            res.append(out[off:off + a * b * c].reshape(a, b, c))
            off += a * b * c
        return res

    def set_tuning(self, kchunk, blocks, dispatch=0, variant=-1, tile_rows=8):
        self._ck(self._lib.kg_batch_set_tuning(self._b, int(kchunk), int(blocks)))
        self._ck(self._lib.kg_batch_set_dispatch(self._b, int(dispatch), int(variant)))
        self._ck(self._lib.kg_batch_set_tile_rows(self._b, int(tile_rows)))

    def tuning(self):
        k, b, d, v, r = C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0), C.c_int(0)
        self._ck(self._lib.kg_batch_get_tuning(self._b, C.byref(k), C.byref(b)))
        self._ck(self._lib.kg_batch_get_dispatch(self._b, C.byref(d), C.byref(v)))
        self._ck(self._lib.kg_batch_get_tile_rows(self._b, C.byref(r)))
        return Tuning(k.value, b.value, d.value, v.value, r.value)

    @property
    def launch_count(self):
        return int(self._lib.kg_batch_launch_count(self._b))

    @property
    def stream(self):
        return self._lib.kg_batch_get_stream(self._b)


class Tuning(tuple):
    """(kchunk, blocks, dispatch, variant, tile_rows): the arguments of Batch.set_tuning"""

    def __new__(cls, kchunk, blocks, dispatch=0, variant=-1, tile_rows=8):
        return super().__new__(cls, (int(kchunk), int(blocks), int(dispatch), int(variant), int(tile_rows)))

    kchunk = property(lambda self: self[0])
    blocks = property(lambda self: self[1])
    dispatch = property(lambda self: self[2])
    variant = property(lambda self: self[3])
    tile_rows = property(lambda self: self[4])


_TUNE_CACHE = {}


def candidates(precision="fp64", kchunks=(16, 24, 32, 48, 64), ctas_per_sm=(1, 2), sms=148,
               variants=(2, 1, 0), tile_rows=(8, 4)):
    """The tuner's search space: persistent launches over (kchunk, CTAs per SM,
    tile rows), and concurrent single-solve launches over the stage-kernel forms
    (the mixed form has the TMA form only), the TMA form in each tile height.
    A 32 x 4 tile holds half the threads and shared memory of a 32 x 8 one, so its
    persistent launches run 1.5x the CTAs per SM."""
    out = []
    for tr in tile_rows:
        per_sm = ctas_per_sm if tr == 8 else tuple(sorted({max(1, (3 * c) // 2) for c in ctas_per_sm}))
        out += [Tuning(kc, cps * sms, 0, -1, tr) for kc in kchunks for cps in per_sm]
    for v in (variants if precision == "fp64" else (2,)):
        for tr in (tile_rows if v == 2 else (8,)):
            out.append(Tuning(kchunks[0], sms, 1, v, tr))
    return out


def autotune(shapes, device=-1, kchunks=(16, 24, 32, 48, 64), ctas_per_sm=(1, 2), steps=3, sms=None,
             precision="fp64", variants=(2, 1, 0), tile_rows=(8, 4)):
    """Choose how a batch of solves with the given grid shapes runs (a Tuning).

    shapes: list of (Nx, Ny, Nz).  Every candidate of `candidates` is timed on
    scratch solves with those shapes (zero state; the kernels' cost does not
    depend on the values), `steps` graph-replayed RK4 steps each after two
    warm-up steps, in the given precision.  Results are cached per sorted
    shape list and precision."""
    from .lines_method import ScalarField
    key = (tuple(sorted(shapes)), precision)
    if key in _TUNE_CACHE:
        return _TUNE_CACHE[key]
    import torch
    if sms is None:
        sms = torch.cuda.get_device_properties(max(device, 0)).multi_processor_count
    scratch = [ScalarField(nx, ny, nz, 1.8, 1.8 + 0.1 * nx, 0.25, device=device, n_det=2, l_max=0)
               for (nx, ny, nz) in shapes]
    best = None
    for cand in candidates(precision, kchunks, ctas_per_sm, sms, variants, tile_rows):
        b = Batch(device, precision=precision)
        for s in scratch:
            b.add(s)
        b.set_tuning(*cand)
        b.rk4(2)  # builds the work list and the graphs
        b.synchronize()
        t0 = time.perf_counter()
        b.rk4(steps)
        b.synchronize()
        dt = (time.perf_counter() - t0) / steps
        if best is None or dt < best[0]:
            best = (dt, cand)
        for s in scratch:
            b.remove(s)
        b.close()
    for s in scratch:
        s.close()
    _TUNE_CACHE[key] = best[1]
    return best[1]
