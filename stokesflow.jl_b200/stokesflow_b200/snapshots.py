"""Snapshot output in the reference's .mat layout, written asynchronously.

StokesFlow2D saves, at start-up and after every timestep when `save_to_file`
is set (scripts/StokesFlow2D_multixpu.jl:136-141, 194-198):

* ``viz_out/stats.mat``: ``dims`` (the rank grid) and ``nt`` (saveStats, :242-252);
* ``viz_out/markers_%04d_%04d.mat`` (timestep, rank): ``x_m``, ``y_m``, ``rho_m``
  as Float32 (saveMarkers, :259-268; on one rank the coordinate shift is 0);
* ``viz_out/grid_%04d_%04d.mat``: the coordinate vectors ``x, y, x_p, y_p,
  x_vx, y_vx, x_vy, y_vy`` and ``mu_b, P, Vx, Vy`` as Float32 (saveGrid,
  :275-299), with the coordinates of :117-124.

scripts/viz.jl reads them back with MAT.jl, which reads MATLAB v5 files; these
are written as v5 (scipy.io.savemat), arrays in their Julia shape (column
vectors for the coordinates).

On the GPU the arrays are converted to Float32 on the device and copied into
pinned host buffers on a side stream that waits for the caller's stream, so
the timestep loop does not wait for them; a writer thread waits for the copies
and writes the files.  Two buffer sets alternate, so one snapshot can be in
flight while the next is taken.
"""
from __future__ import annotations

import os
import queue
import threading

import numpy as np
import scipy.io
import torch


def grid_coordinates(Nx: int, Ny: int, dx: float, dy: float) -> dict:
    """The local coordinate vectors of StokesFlow2D_multixpu.jl:117-124 (Float64, Julia index order)."""
    ix, iy = np.arange(1, Nx + 3, dtype=np.float64), np.arange(1, Ny + 3, dtype=np.float64)
    return {"x": (ix[:Nx] - 1) * dx, "y": (iy[:Ny] - 1) * dy,
            "x_p": (ix[:Nx - 1] - 1) * dx + 0.5 * dx, "y_p": (iy[:Ny - 1] - 1) * dy + 0.5 * dy,
            "x_vx": (ix[:Nx + 2] - 2) * dx, "y_vx": (iy[:Ny + 1] - 1) * dy - 0.5 * dy,
            "x_vy": (ix[:Nx + 1] - 1) * dx - 0.5 * dx, "y_vy": (iy[:Ny + 2] - 2) * dy}


class SnapshotWriter:
    """Writes the reference's snapshot files for one StokesFlow2D state (one rank)."""

    FIELDS = ("x_m", "y_m", "rho_m", "mu_b", "P", "Vx", "Vy")

    def __init__(self, out_dir: str, state, rank: int = 0, dims=(1, 1, 1)):
        self.dir = out_dir
        os.makedirs(out_dir, exist_ok=True)
        self.st = state
        self.rank = rank
        self.dims = np.asarray(dims, dtype=np.int64)
        self.coords = {k: v.astype(np.float32) for k, v in
                       grid_coordinates(state.Nx, state.Ny, state.dx, state.dy).items()}
        self.cuda = state.x_m.is_cuda
        src = self._sources()
        # two sets of float32 staging: device (conversion) and pinned host
        self.sets = []
        for _ in range(2):
            host = {k: torch.empty(v.numel(), dtype=torch.float32, pin_memory=self.cuda) for k, v in src.items()}
            dev = {k: torch.empty(v.numel(), dtype=torch.float32, device=v.device) for k, v in src.items()}
            self.sets.append({"host": host, "dev": dev, "done": threading.Event(), "event": None})
            self.sets[-1]["done"].set()
        self.next = 0
        self.stream = torch.cuda.Stream() if self.cuda else None
        self.jobs: queue.Queue = queue.Queue()
        self.error = None
        self.worker = threading.Thread(target=self._run, daemon=True)
        self.worker.start()

    def _sources(self):
        s = self.st
        return {"x_m": s.x_m, "y_m": s.y_m, "rho_m": s.rho_m, "mu_b": s.mu_b, "P": s.P, "Vx": s.Vx, "Vy": s.Vy}

    def snapshot(self, nt: int):
        """Take snapshot `nt` of the state as it is once the work queued so far on the current stream is done."""
        if self.error is not None:
            raise self.error
        b = self.sets[self.next]
        self.next ^= 1
        b["done"].wait()                # this set's previous file is written
        b["done"].clear()
        src = self._sources()
        shapes = {k: tuple(v.shape) for k, v in src.items()}
        if self.cuda:
            cur = torch.cuda.current_stream()
            self.stream.wait_stream(cur)
            with torch.cuda.stream(self.stream):
                for k, v in src.items():
                    # column-major Julia arrays: the transposed view is contiguous, so flatten that
                    flat = v.t().contiguous().view(-1) if v.dim() == 2 else v
                    b["dev"][k].copy_(flat)
                    b["host"][k].copy_(b["dev"][k], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(self.stream)
            for v in src.values():          # keep the sources alive until the side stream has read them
                v.record_stream(self.stream)
            b["event"] = ev
        else:
            for k, v in src.items():
                flat = v.t().contiguous().view(-1) if v.dim() == 2 else v
                b["host"][k].copy_(flat)
            b["event"] = None
        self.jobs.put((nt, b, shapes))

    def _run(self):
        while True:
            job = self.jobs.get()
            if job is None:
                return
            nt, b, shapes = job
            try:
                if b["event"] is not None:
                    b["event"].synchronize()
                self._write(nt, b["host"], shapes)
            except Exception as e:          # surfaced by the next snapshot() or close()
                self.error = e
            finally:
                b["done"].set()

    def _write(self, nt, host, shapes):
        def arr(k):
            t = host[k]
            if len(shapes[k]) == 2:
                nx, ny = shapes[k]
                return np.asfortranarray(t.numpy().reshape(ny, nx).T)
            return t.numpy().copy()
        if self.rank == 0:
            scipy.io.savemat(os.path.join(self.dir, "stats.mat"), {"dims": self.dims, "nt": np.int64(nt)},
                             oned_as="column")
        tag = f"{nt:04d}_{self.rank:04d}"
        scipy.io.savemat(os.path.join(self.dir, f"markers_{tag}.mat"),
                         {"x_m": arr("x_m"), "y_m": arr("y_m"), "rho_m": arr("rho_m")}, oned_as="column")
        c = self.coords
        scipy.io.savemat(os.path.join(self.dir, f"grid_{tag}.mat"),
                         {"x": c["x"], "y": c["y"], "mu_b": arr("mu_b"), "x_p": c["x_p"], "y_p": c["y_p"],
                          "P": arr("P"), "x_vx": c["x_vx"], "y_vx": c["y_vx"], "Vx": arr("Vx"),
                          "x_vy": c["x_vy"], "y_vy": c["y_vy"], "Vy": arr("Vy")}, oned_as="column")

    def flush(self):
        for b in self.sets:
            b["done"].wait()
        if self.error is not None:
            raise self.error

    def close(self):
        self.flush()
        self.jobs.put(None)
        self.worker.join()
