"""Timestep driver: the body of StokesFlow2D (scripts/StokesFlow2D_multixpu.jl:55-235)
on one GPU, without plotting or file output.

Per timestep (:157-218): deposit rho -> rho_vy, mu -> mu_b, mu -> mu_p
(:164-166), solveStokes! (:171-176), moveMarkersRK4! (:181), and the marker
exchange (:186-191), which is the identity on a single domain -- so, unlike
the reference, the markers never leave the device.  Optionally each timestep
also rebins the markers by cell (per-cell counts).

All arrays are allocated once (:89-114) and the solver is warm-started across
timesteps exactly like the reference (P, Vx, Vy, dVxdt, dVydt persist).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

from . import api


# HBM bytes of one FP32 sweep per point: read dVx, dVy, dP, mu_b, mu_p, rho, rdiv, the two damped rates and
# the two momentum residuals, write dVx, dVy, dP and the two rates (11 reads + 5 writes of 4 bytes)
MIXED_BYTES_PER_POINT = 64


def node_origins(dx, dy):
    """First coordinates of the staggered node sets (StokesFlow2D_multixpu.jl:117-126)."""
    return dict(x=0.0, y=0.0, x_p=0.0 * dx + 0.5 * dx, y_p=0.0 * dy + 0.5 * dy, x_vx=(1 - 2) * dx,
                y_vx=0.0 * dy - 0.5 * dy, x_vy=0.0 * dx - 0.5 * dx, y_vy=(1 - 2) * dy, x_rho=0.0 * dx - 0.5 * dx,
                y_rho=(2 - 2) * dy)


@dataclass
class StepTimes:
    deposit_ms: float = 0.0
    solve_ms: float = 0.0
    advect_ms: float = 0.0
    rebin_ms: float = 0.0
    h2d_ms: float = 0.0
    d2h_ms: float = 0.0

    def total(self):
        return self.deposit_ms + self.solve_ms + self.advect_ms + self.rebin_ms + self.h2d_ms + self.d2h_ms


@dataclass
class StokesFlow2D:
    """State of one StokesFlow2D run (single rank).  ``step()`` advances one timestep."""
    Nx: int
    Ny: int
    Lx: float
    Ly: float
    model: api.PlumeModel
    marker_density: int = 5
    stokes_eps: float = 1e-5          # absolute eps, reference keyword stokes_eps
    stokes_rtol: float | None = None  # if set: eps = rtol * mean|g rho_vy| (relative residual)
    jitter: float = 0.0               # 0: RAND_MARKER_POS = false; 1: reference jitter width
    seed: int = 0
    g_y: float = 9.81                 # :72
    maxdisp: float = 0.5              # :71
    iter_max: int = 100000
    rebin: bool = False
    device: str = "cuda"
    keep_work_arrays: bool = True     # allocate tau, divV, dtau, R like the reference
    host_markers: bool = False        # markers start in pinned host memory (end-to-end path)
    solver: str = "fp64"              # "fp64": plain path, bit-identical to the reference; "mixed": FP32 sweeps +
                                      # FP64 defect correction
    mixed_opts: object = None
    snapshot_dir: str | None = None   # save_to_file: the reference's .mat snapshots at start and after every step
    ctx: api.Context | None = None
    history: list = field(default_factory=list)

    def __post_init__(self):
        Nx, Ny = self.Nx, self.Ny
        self.dx = self.Lx / (Nx - 1)      # :76-77
        self.dy = self.Ly / (Ny - 1)
        self.lx = (Nx - 1) * self.dx      # :78-79
        self.ly = (Ny - 1) * self.dy
        self.o = node_origins(self.dx, self.dy)
        z = lambda *s: api.zeros(*s, device=self.device)  # noqa: E731
        self.P = z(Nx - 1, Ny - 1)
        self.Vx = z(Nx + 2, Ny + 1)
        self.Vy = z(Nx + 1, Ny + 2)
        self.rho_vy = z(Nx + 1, Ny)
        self.mu_b = z(Nx, Ny)
        self.mu_p = z(Nx - 1, Ny - 1)
        w = self.keep_work_arrays
        self.txx = z(Nx - 1, Ny - 1) if w else None
        self.tyy = z(Nx - 1, Ny - 1) if w else None
        self.txy = z(Nx, Ny) if w else None
        self.divV = z(Nx - 1, Ny - 1) if w else None
        self.dtPt = z(Nx - 1, Ny - 1) if w else None
        self.Rx = z(Nx - 2, Ny - 1) if w else None
        self.Ry = z(Nx - 1, Ny - 2) if w else None
        self.dtVx = z(Nx - 2, Ny - 1) if w else None
        self.dtVy = z(Nx - 1, Ny - 2) if w else None
        self.dVxdt = z(Nx - 2, Ny - 1)
        self.dVydt = z(Nx - 1, Ny - 2)
        self.Vx_s = z(Nx, Ny + 1)
        self.Vy_s = z(Nx + 1, Ny)
        self.val_wt_sum = z(Nx + 1, Ny) if w else None   # interp_size (:112-114)
        self.wt_sum = z(Nx + 1, Ny) if w else None
        self.ctx = self.ctx or api.default_context()
        if self.host_markers:
            self.x_host, self.y_host = api.initialize_markers_host(self.marker_density, self.lx, self.ly, self.dx,
                                                                   self.dy, Nx, Ny, self.jitter, self.seed)
            self.rho_host, self.mu_host = api.set_initial_marker_properties(self.x_host, self.y_host, self.model)
            self.x_m = torch.empty(self.x_host.numel(), dtype=torch.float64, device=self.device)
            self.y_m = torch.empty_like(self.x_m)
            self.rho_m = torch.empty_like(self.x_m)
            self.mu_m = torch.empty_like(self.x_m)
            for d, h in ((self.x_m, self.x_host), (self.y_m, self.y_host), (self.rho_m, self.rho_host),
                         (self.mu_m, self.mu_host)):
                d.copy_(h, non_blocking=True)
        else:
            self.x_m, self.y_m = api.initialize_markers(self.marker_density, self.lx, self.ly, self.dx, self.dy, Nx,
                                                        Ny, self.jitter, self.seed, device=self.device, ctx=self.ctx)
            if hasattr(self.model, "marker_properties"):   # any other material model (workloads.InclusionModel)
                self.rho_m, self.mu_m = self.model.marker_properties(self.x_m, self.y_m)
            else:
                self.rho_m, self.mu_m = api.set_initial_marker_properties(self.x_m, self.y_m, self.model,
                                                                          ctx=self.ctx)
        self.dt = 0.0
        self.t_tot = 0.0
        self.nt = 0
        self.counts = None
        self._rebin_out = None
        self._ev = [torch.cuda.Event(enable_timing=True) for _ in range(8)]
        self.snapshots = None
        if self.snapshot_dir:   # StokesFlow2D_multixpu.jl:136-141: stats, markers and grid before the first step
            from .snapshots import SnapshotWriter
            self.snapshots = SnapshotWriter(self.snapshot_dir, self)
            self.snapshots.snapshot(0)

    @property
    def n_markers(self):
        return self.x_m.numel()

    # ------------------------------------------------------------------
    def deposit(self):
        # StokesFlow2D_multixpu.jl:164-166, the three bilinearMarkerToGrid! calls in one: rho_vy, mu_b, mu_p
        o = self.o
        api.bilinear_marker_to_grids([(o["x_rho"], o["y_rho"], self.rho_vy, self.rho_m),
                                      (o["x"], o["y"], self.mu_b, self.mu_m),
                                      (o["x_p"], o["y_p"], self.mu_p, self.mu_m)],
                                     self.x_m, self.y_m, self.dx, self.dy, self.val_wt_sum, self.wt_sum, ctx=self.ctx)

    def eps(self):
        if self.stokes_rtol is None:
            return self.stokes_eps
        return self.stokes_rtol * api.residual_scale(self.rho_vy, self.Nx, self.Ny, self.g_y, ctx=self.ctx)

    def mixed_problem(self):
        """This timestep's Stokes problem for the mixed-precision / batched solver."""
        return api.MixedProblem(self.P, self.Vx, self.Vy, self.rho_vy, self.mu_b, self.mu_p, self.Vx_s, self.Vy_s,
                                self.g_y, self.dx, self.dy, self.Nx, self.Ny, self.dt, self.maxdisp,
                                eps=self.stokes_eps, rel_tol=self.stokes_rtol or 0.0, dVxdt=self.dVxdt,
                                dVydt=self.dVydt)

    def solve(self):
        if self.solver == "mixed":
            p = self.mixed_problem()
            r = api.solve_stokes_batch_mixed([p], options=self.mixed_opts, ctx=self.ctx)[0]
            self.dt = r["dt_out"]
            return dict(r, dt=r["dt_out"], iters=r["inner_iters"], loop_ms=r["batch_ms"],
                        bytes_per_iter=float(MIXED_BYTES_PER_POINT * (self.Nx - 1) * (self.Ny - 1)))
        info = api.solve_stokes_info(self.P, self.Vx, self.Vy, self.rho_vy, self.mu_b, self.mu_p, self.txx, self.tyy,
                                     self.txy, self.divV, self.dtPt, self.Rx, self.Ry, self.dVxdt, self.dVydt,
                                     self.dtVx, self.dtVy, self.Vx_s, self.Vy_s, self.g_y, self.dx, self.dy, self.Nx,
                                     self.Ny, self.dt, self.maxdisp, use_free_surface_stabilization=True,
                                     eps=self.eps(), print_info=False, iter_max=self.iter_max, ctx=self.ctx)
        self.dt = info["dt"]
        return info

    def advect(self):
        o = self.o
        api.move_markers_rk4(self.x_m, self.y_m, self.Vx, self.Vy, o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"],
                             self.dt, self.lx, self.ly, self.dx, self.dy, ctx=self.ctx)

    def do_rebin(self):
        # the outputs are allocated once and filled in every timestep
        nm, ncells = self.n_markers, (self.Nx + 1) * (self.Ny + 1)
        if self._rebin_out is None or self._rebin_out[2].numel() < max(nm, 1):
            dev = self.x_m.device
            self._rebin_out = (torch.empty(ncells, dtype=torch.int32, device=dev),
                               torch.empty(ncells + 1, dtype=torch.int32, device=dev),
                               torch.empty(max(nm, 1), dtype=torch.int32, device=dev))
        self.counts, self.cell_offsets, self.cell_perm = api.rebin_markers(
            self.x_m, self.y_m, self.o["x"], self.o["y"], self.dx, self.dy, self.Nx, self.Ny, out=self._rebin_out,
            ctx=self.ctx)

    def step(self, host_io: bool = False) -> dict:
        """One timestep.  host_io: the reference's per-timestep host round trip
        (markers H2D from pinned host buffers before, markers and velocities
        D2H after), for an end-to-end measurement."""
        ev = self._ev
        t = StepTimes()
        s = torch.cuda.current_stream()
        ev[0].record(s)
        if host_io:
            for d, h in ((self.x_m, self.x_host), (self.y_m, self.y_host), (self.rho_m, self.rho_host),
                         (self.mu_m, self.mu_host)):
                d.copy_(h, non_blocking=True)
        ev[1].record(s)
        self.deposit()
        ev[2].record(s)
        info = self.solve()
        ev[3].record(s)
        self.advect()
        ev[4].record(s)
        if self.rebin:
            self.do_rebin()
        ev[5].record(s)
        if host_io:
            self.x_host.copy_(self.x_m, non_blocking=True)
            self.y_host.copy_(self.y_m, non_blocking=True)
            self._vx_host = self.Vx.t().to("cpu", non_blocking=True)
            self._vy_host = self.Vy.t().to("cpu", non_blocking=True)
        ev[6].record(s)
        ev[6].synchronize()
        t.h2d_ms = ev[0].elapsed_time(ev[1])
        t.deposit_ms = ev[1].elapsed_time(ev[2])
        t.solve_ms = ev[2].elapsed_time(ev[3])
        t.advect_ms = ev[3].elapsed_time(ev[4])
        t.rebin_ms = ev[4].elapsed_time(ev[5])
        t.d2h_ms = ev[5].elapsed_time(ev[6])
        self.t_tot += self.dt
        self.nt += 1
        if self.snapshots is not None:   # :194-198, written in the background
            self.snapshots.snapshot(self.nt)
        rec = dict(nt=self.nt, dt=self.dt, t_tot=self.t_tot, times=t, info=info)
        self.history.append(rec)
        return rec

    def close_snapshots(self):
        """Wait for the snapshot files still being written."""
        if self.snapshots is not None:
            self.snapshots.close()
            self.snapshots = None

    # split timestep for a serving loop: the solve runs in a shared engine between the two halves
    def begin_timestep(self) -> api.MixedProblem:
        """Deposit (:164-166) and return this timestep's Stokes problem."""
        self.deposit()
        return self.mixed_problem()

    def end_timestep(self, result: dict):
        """After the solve (:171-176): take its dt, advect (:181), rebin if asked, count the timestep."""
        self.dt = result["dt_out"]
        self.advect()
        if self.rebin:
            self.do_rebin()
        self.t_tot += self.dt
        self.nt += 1

    def device_bytes(self) -> int:
        """Device bytes held by this state (markers and grid arrays)."""
        ts = [self.x_m, self.y_m, self.rho_m, self.mu_m, self.P, self.Vx, self.Vy, self.rho_vy, self.mu_b, self.mu_p,
              self.dVxdt, self.dVydt, self.Vx_s, self.Vy_s]
        ts += [t for t in (self.txx, self.tyy, self.txy, self.divV, self.dtPt, self.Rx, self.Ry, self.dtVx, self.dtVy,
                           self.val_wt_sum, self.wt_sum) if t is not None]
        return int(sum(t.numel() * t.element_size() for t in ts))

    def h2d_bytes_per_step(self):
        return 4 * 8 * self.n_markers

    def d2h_bytes_per_step(self):
        return 2 * 8 * self.n_markers + 8 * (self.Vx.numel() + self.Vy.numel())

    # ------------------------------------------------------------------
    def velocities_host(self):
        """(Vx_pad, Vy_pad) as Fortran-ordered numpy arrays with the Julia shape."""
        return _host(self.Vx), _host(self.Vy)


def _host(a: torch.Tensor) -> np.ndarray:
    return np.asfortranarray(a.t().contiguous().cpu().numpy().T)


def stokes_flow_2d(Nt, Nx, Ny, Lx, Ly, model: api.PlumeModel, *, marker_density=5, stokes_eps=1e-5,
                   stokes_rtol=None, jitter=0.0, seed=0, g_y=9.81, maxdisp=0.5, iter_max=100000, rebin=False,
                   save_to_file=False, out_dir="viz_out", return_state=False):
    """StokesFlow2D (StokesFlow2D_multixpu.jl:55-235) on one GPU.
    Returns (Vx_glob, Vy_glob, t_tot) as host arrays (Julia shape, Fortran order)
    and, with return_state, the StokesFlow2D state object.  save_to_file writes the reference's .mat
    snapshots into out_dir (stats.mat, markers_%04d_0000.mat, grid_%04d_0000.mat)."""
    st = StokesFlow2D(Nx, Ny, float(Lx), float(Ly), model, marker_density=marker_density, stokes_eps=stokes_eps,
                      stokes_rtol=stokes_rtol, jitter=jitter, seed=seed, g_y=g_y, maxdisp=maxdisp,
                      iter_max=iter_max, rebin=rebin, snapshot_dir=out_dir if save_to_file else None)
    for _ in range(Nt):
        st.step()
    st.close_snapshots()
    Vx, Vy = st.velocities_host()
    if return_state:
        return Vx, Vy, st.t_tot, st
    return Vx, Vy, st.t_tot


def plume_model_unit_square():
    """The benchmark material model: unit square, gravity along +y, free slip;
    air (rho = mu = 1e-3) for y < 0.1, plume (rho = 0.9, mu = 0.1) of radius
    0.1 at (0.5, 0.75), matrix rho = mu = 1."""
    return api.PlumeModel(air_height=0.1, plume_x=0.5, plume_y=0.75, plume_r=0.1, rho_air=1e-3, rho_matrix=1.0,
                          rho_plume=0.9, mu_air=1e-3, mu_matrix=1.0, mu_plume=0.1)


def plume_model_test_flow():
    """Material model of test/test_StokesFlow2D.jl:208-230 (Lx = Ly = 10)."""
    return api.PlumeModel(air_height=0.2 * 10, plume_x=10 / 2, plume_y=10 / 2, plume_r=min(10, 10) / 5, rho_air=1e-2,
                          rho_matrix=3.3, rho_plume=3.2, mu_air=1e-1, mu_matrix=1e0, mu_plume=5e-1)


def marker_density_for(markers_per_cell: int) -> int:
    md = int(round(math.sqrt(markers_per_cell)))
    if md * md != markers_per_cell:
        raise ValueError("markers per cell must be a square (md x md sub-grid)")
    return md
