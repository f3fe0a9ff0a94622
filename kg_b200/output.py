"""The reference's ASCII diagnostics output, written from a solver's results.

save_gnuplot (main/save_gnuplot.f90:15-72) appends, every `save_0d` steps,
  Mass_scalar.t.asc            "t  Mass_scalar"                    (save_t, IO/save_data_lib.f90:9-15)
  jr_NN.t.asc, jtheta_NN.t.asc, jphi_NN.t.asc
                               "t  momentum(c, NN)" for every detector NN inside the grid
and every `save` steps
  Harmonic_coeficientsNN.lm.asc  one block per save: rows "l  m  Re a_lm  Im a_lm  |a_lm|"
                               for l = 0..l_max, m = -l..l, then two blank lines
                               (savealm, IO/save_data.f90:54-110)
for detectors with r(1) <= r_det < r(Nx) on the vertex grid.

The reference writes with Fortran list-directed output; here every value is a
whitespace-separated field with 17 significant digits (integers as integers),
which reads back to the same doubles and parses as the same columns; the
exact column widths of gfortran's list-directed layout are not reproduced.
"""
from __future__ import annotations

import os

import numpy as np


def _fmt(x):
    return f"{x: .17E}"


class DiagnosticWriter:
    def __init__(self, solver, directory=".", save_0d=1, save=1):
        """save_0d, save: the reference's output periods in steps (global_numbers
        save_0d and MoL%save)"""
        self.s = solver
        self.dir = directory
        self.save_0d = int(save_0d)
        self.save = int(save)
        os.makedirs(directory, exist_ok=True)

    def _append(self, name, lines):
        with open(os.path.join(self.dir, name), "a") as f:
            f.write("".join(lines))

    def _inside_evolution_grid(self):
        """detectors with x(-g) <= r_det < x(Nx), save_gnuplot's single-rank test
        r_aux(iL - g) <= r_det < r_aux(iR) on x(i) = xmin + (i + g) dx"""
        r_det, _ = self.s.detectors()
        dx = self.s.dx
        xmin = self.s.params.xmin
        r_lo = xmin
        r_hi = xmin + (self.s.Nx + self.s.g_pts) * dx
        return [(d, r) for d, r in enumerate(r_det) if r_lo <= r < r_hi]

    def _inside_vertex_grid(self):
        r_det, _ = self.s.detectors()
        dx = self.s.dx
        xmin = self.s.params.xmin
        r1, rN = xmin, xmin + (self.s.Nx - 1) * dx
        return [(d, r) for d, r in enumerate(r_det) if r1 <= r < rN]

    def step(self, index):
        """call after step `index` (1-based, as the reference's loop counter),
        after the solver's diagnostic(index) has refreshed Mass_scalar and the
        detector quantities"""
        s = self.s
        t = s.t
        if index % self.save_0d == 0:
            self._append("Mass_scalar.t.asc", [f"{_fmt(t)} {_fmt(s.Mass_scalar)}\n"])
            mom = s.currents_detectors()
            for d, _ in self._inside_evolution_grid():
                nn = f"{d + 1:02d}"
                for c, name in enumerate(("jr_", "jtheta_", "jphi_")):
                    self._append(f"{name}{nn}.t.asc", [f"{_fmt(t)} {_fmt(mom[d, c])}\n"])
        if index % self.save == 0:
            alm = s.proyector_detectors()
            L = alm.shape[2] - 1
            for d, _ in self._inside_vertex_grid():
                rows = []
                for l in range(L + 1):
                    for m in range(-l, l + 1):
                        a = alm[d, m + L, l]
                        rows.append(f"{l:12d}{m:12d} {_fmt(a.real)} {_fmt(a.imag)} {_fmt(abs(a))}\n")
                rows.append("\n\n")
                self._append(f"Harmonic_coeficients{d + 1:02d}.lm.asc", rows)


def read_lm(path):
    """blocks of a Harmonic_coeficientsNN.lm.asc file: list of (l, m, a_lm) arrays"""
    blocks, cur = [], []
    with open(path) as f:
        text = f.read()
    for chunk in text.split("\n\n\n"):
        rows = [r.split() for r in chunk.strip().splitlines() if r.strip()]
        if rows:
            arr = np.array([[float(x) for x in r] for r in rows])
            blocks.append((arr[:, 0].astype(int), arr[:, 1].astype(int), arr[:, 2] + 1j * arr[:, 3]))
    return blocks


class AsyncSnapshots:
    """3-D snapshots of the state while the solve keeps stepping: the reference
    writes HDF5 files of the fields every save_3d steps (hdf5/hdf5_lib.f90, from
    save_gnuplot); here `snap(index)` copies u on the device (kg_get_state_device,
    ordered on the solver's stream) into one of `depth` device buffers and a
    worker thread moves it to pinned host memory and writes
    `<prefix>_<index>.npy` (complex128, shape (Nz+1, Ny+2g+1, Nx+2g+1, 5), the
    reference's u(1:5,-g:Nx+g,-g:Ny+g,0:Nz) memory order) with the time in
    `<prefix>_<index>.t`.  The solver's stream only waits for the device copy."""

    def __init__(self, solver, directory=".", prefix="u", depth=2):
        import queue
        import threading
        import torch
        import ctypes as C
        self.s, self.dir, self.prefix = solver, directory, prefix
        os.makedirs(directory, exist_ok=True)
        dev = f"cuda:{max(torch.cuda.current_device(), 0)}"
        shape = (solver.NK, solver.NJ, solver.NI, 5)
        self._bufs = [torch.empty(shape, dtype=torch.complex128, device=dev) for _ in range(depth)]
        self._free = queue.Queue()
        for i in range(depth):
            self._free.put(i)
        self._work = queue.Queue()
        self._host = torch.empty(shape, dtype=torch.complex128, pin_memory=True)
        self._C = C
        self._err = None
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    def snap(self, index):
        import torch
        i = self._free.get()                       # waits only if `depth` snapshots are in flight
        s = self.s
        s._ck(s._lib.kg_get_state_device(s.handle, 0, self._C.c_void_p(self._bufs[i].data_ptr())))
        stream = torch.cuda.ExternalStream(s._lib.kg_get_stream(s.handle))
        ev = torch.cuda.Event()
        ev.record(stream)
        self._work.put((i, ev, int(index), s.t))

    def _run(self):
        while True:
            item = self._work.get()
            if item is None:
                return
            i, ev, index, t = item
            try:
                ev.synchronize()
                self._host.copy_(self._bufs[i])
                base = os.path.join(self.dir, f"{self.prefix}_{index:08d}")
                np.save(base + ".npy", self._host.numpy())
                with open(base + ".t", "w") as f:
                    f.write(f"{float(t)!r}\n")
            except Exception as e:  # reported by close()
                self._err = e
            finally:
                self._free.put(i)

    def close(self):
        """wait for every snapshot to be on disk"""
        self._work.put(None)
        self._thread.join()
        if self._err is not None:
            raise self._err
