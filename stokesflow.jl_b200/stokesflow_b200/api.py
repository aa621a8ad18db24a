"""Python mirror of the reference's hot-path functions on CUDA tensors.

Each function keeps the name (snake_case), argument order, meaning and
in-place behaviour of its Julia counterpart and calls straight into
libstokesflow_b200.so:

=========================================  =====================================================
reference (dastrm/StokesFlow.jl)           here
=========================================  =====================================================
bilinearMarkerToGrid!  MarkerToGrid.jl:18  :func:`bilinear_marker_to_grid`
solveStokes!  StokesSolver_multixpu.jl:14  :func:`solve_stokes` (returns ``(dt, T_eff, runtime)``)
moveMarkersRK4!  MoveMarkers.jl:15         :func:`move_markers_rk4`
initializeMarkersCPU  common.jl:40         :func:`initialize_markers`
setInitialMarkerProperties!  common.jl:104 :func:`set_initial_marker_properties`
exchangeMarkers  MarkerExchange.jl:8       identity on a single domain (not needed)
=========================================  =====================================================

Grid arrays are float64 CUDA tensors with the Julia shape ``(nx, ny)`` in
column-major storage (strides ``(1, nx)``), so ``A[ix-1, iy-1]`` is Julia's
``A[ix, iy]``; :func:`zeros` makes them.  Marker arrays are 1-D contiguous
float64 CUDA tensors.  Work is queued on the current torch CUDA stream; the
solve synchronises it (its stopping test reads the residual on the host).
The MPI ``comm`` / ImplicitGlobalGrid ``grid`` arguments are accepted and
ignored: the domain is a single rank.
"""
from __future__ import annotations

import ctypes as C
import threading

import torch

from . import _lib
from ._lib import check, lib

__all__ = ["Context", "default_context", "zeros", "bilinear_marker_to_grid", "solve_stokes", "solve_stokes_info",
           "residual_scale", "move_markers_rk4", "rebin_markers", "marker_count", "initialize_markers",
           "initialize_markers_host", "set_initial_marker_properties", "get_warnings", "PlumeModel", "MixedProblem",
           "mixed_options", "batch_stats", "solve_stokes_batch_mixed", "Engine", "bilinear_marker_to_grid_noalloc"]


class Context:
    """Owns an sf_ctx (device scratch) on one CUDA device."""

    def __init__(self, device: int | None = None):
        if device is None:
            device = torch.cuda.current_device()
        self.device = int(device)
        h = C.c_void_p()
        check(lib().sf_ctx_create(self.device, C.byref(h)), "sf_ctx_create")
        self.handle = h

    def close(self):
        if self.handle:
            lib().sf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launch_count(self) -> int:
        """Kernels launched through this context so far."""
        n = C.c_int64()
        check(lib().sf_ctx_launch_count(self.handle, C.byref(n)))
        return n.value

    def scratch_bytes(self) -> int:
        b = C.c_int64()
        check(lib().sf_ctx_scratch_bytes(self.handle, C.byref(b)))
        return b.value


_ctx_lock = threading.Lock()
_contexts: dict[int, Context] = {}


def default_context(device: int | None = None) -> Context:
    if device is None:
        device = torch.cuda.current_device()
    with _ctx_lock:
        ctx = _contexts.get(int(device))
        if ctx is None:
            ctx = _contexts[int(device)] = Context(device)
        return ctx


def zeros(*shape, device="cuda") -> torch.Tensor:
    """Julia ``@zeros(nx, ny)``: float64, column-major, Julia shape."""
    if len(shape) == 1 and isinstance(shape[0], (tuple, list)):
        shape = tuple(shape[0])
    if len(shape) == 1:
        return torch.zeros(shape[0], dtype=torch.float64, device=device)
    nx, ny = shape
    return torch.zeros((ny, nx), dtype=torch.float64, device=device).t()


def _grid(a: torch.Tensor, name: str, shape=None) -> int:
    if a.dtype != torch.float64 or not a.is_cuda:
        raise TypeError(f"{name}: need a float64 CUDA tensor")
    if a.dim() != 2 or a.stride() != (1, a.shape[0]):
        raise ValueError(f"{name}: need a column-major (nx, ny) tensor (strides (1, nx)); got strides {a.stride()}")
    if shape is not None and tuple(a.shape) != tuple(shape):
        raise ValueError(f"{name}: shape {tuple(a.shape)} != expected {tuple(shape)}")
    return a.data_ptr()


def _opt_grid(a, name, shape):
    return None if a is None else _grid(a, name, shape)


def _vec(a: torch.Tensor, name: str) -> int:
    if a.dtype != torch.float64 or not a.is_cuda or a.dim() != 1 or not a.is_contiguous():
        raise TypeError(f"{name}: need a contiguous 1-D float64 CUDA tensor")
    return a.data_ptr()


def _stream(stream=None) -> int:
    if stream is None:
        stream = torch.cuda.current_stream()
    return stream.cuda_stream


def _ctx(ctx: Context | None) -> Context:
    return ctx if ctx is not None else default_context()


def _one_device(*tensors) -> torch.device:
    """The CUDA device all the given tensors (None skipped) live on; ValueError if they are on several."""
    devs = {t.device for t in tensors if t is not None}
    if len(devs) != 1:
        raise ValueError(f"the arrays must be on one CUDA device, got {sorted(str(d) for d in devs)}")
    return devs.pop()


def _ctx_on(ctx: Context | None, device: torch.device) -> Context:
    """ctx (or the default context of `device`), checked to run on the device the arrays are on."""
    c = ctx if ctx is not None else default_context(device.index)
    if c.device != device.index:
        raise ValueError(f"the context runs on cuda:{c.device}, the arrays are on {device}")
    return c


# ---------------------------------------------------------------------------
def selftest_bounded_wait(arrive: bool, budget_ns: int, *, ctx: Context | None = None) -> bool:
    """Runs the kernels' bounded wait on a barrier that is completed first (arrive) or that nothing completes;
    returns True if the wait gave up after budget_ns.  The context stays usable either way."""
    out = C.c_int32(0)
    check(lib().sf_selftest_bounded_wait(_ctx(ctx).handle, int(bool(arrive)), int(budget_ns), C.byref(out)),
          "selftest_bounded_wait")
    return bool(out.value)


def bilinear_marker_to_grid(x_grid_min, y_grid_min, val_grid, x_m, y_m, val_m, dx, dy, val_wt_sum=None,
                            wt_sum=None, grid=None, *, ctx: Context | None = None, stream=None):
    """bilinearMarkerToGrid! (MarkerToGrid.jl:18-38): deposit val_m onto val_grid in place."""
    nx, ny = val_grid.shape
    pg = _grid(val_grid, "val_grid")
    nm = x_m.numel()
    px, py, pv = _vec(x_m, "x_m"), _vec(y_m, "y_m"), _vec(val_m, "val_m")
    if y_m.numel() != nm or val_m.numel() != nm:
        raise ValueError("x_m, y_m, val_m must have the same length")  # MarkerToGrid.jl:22
    if (val_wt_sum is None) != (wt_sum is None):
        raise ValueError("give both val_wt_sum and wt_sum or neither")
    ps = pw = None
    ld = n_sum = 0
    if wt_sum is not None:
        ps = _grid(val_wt_sum, "val_wt_sum")
        pw = _grid(wt_sum, "wt_sum", val_wt_sum.shape)
        ld, n_sum = wt_sum.shape[0], wt_sum.numel()
    dev = _one_device(val_grid, x_m, y_m, val_m, val_wt_sum, wt_sum)
    c = _ctx_on(ctx, dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    check(lib().sf_bilinear_marker_to_grid(c.handle, float(x_grid_min), float(y_grid_min), pg, nx, ny, px, py, pv,
                                           nm, float(dx), float(dy), ps, pw, ld, n_sum, _stream(st)),
          "bilinear_marker_to_grid")


def bilinear_marker_to_grids(grids, x_m, y_m, dx, dy, val_wt_sum=None, wt_sum=None, *, ctx: Context | None = None,
                             stream=None):
    """The deposits of one timestep in one call: ``grids`` is a sequence of (x_grid_min, y_grid_min, val_grid,
    val_m), at most SF_MAX_GRIDS (4), over the same markers.  Same result, bit for bit, as
    :func:`bilinear_marker_to_grid` once per grid in order (val_wt_sum / wt_sum, when given, end with the last
    grid's sums); the markers' positions are read once for all grids' cell assignments."""
    grids = list(grids)
    if not 1 <= len(grids) <= 4:
        raise ValueError("1 to 4 grids")
    nm = x_m.numel()
    px, py = _vec(x_m, "x_m"), _vec(y_m, "y_m")
    if y_m.numel() != nm:
        raise ValueError("x_m, y_m, val_m must have the same length")  # MarkerToGrid.jl:22
    arr = (_lib.DepositGrid * len(grids))()
    tensors = [x_m, y_m]
    for k, (x0, y0, val_grid, val_m) in enumerate(grids):
        if val_m.numel() != nm:
            raise ValueError("x_m, y_m, val_m must have the same length")
        nx, ny = val_grid.shape
        arr[k] = _lib.DepositGrid(float(x0), float(y0), _grid(val_grid, f"grids[{k}].val_grid"), nx, ny,
                                  _vec(val_m, f"grids[{k}].val_m"))
        tensors += [val_grid, val_m]
    if (val_wt_sum is None) != (wt_sum is None):
        raise ValueError("give both val_wt_sum and wt_sum or neither")
    ps = pw = None
    ld = n_sum = 0
    if wt_sum is not None:
        ps = _grid(val_wt_sum, "val_wt_sum")
        pw = _grid(wt_sum, "wt_sum", val_wt_sum.shape)
        ld, n_sum = wt_sum.shape[0], wt_sum.numel()
        tensors += [val_wt_sum, wt_sum]
    dev = _one_device(*tensors)
    c = _ctx_on(ctx, dev)
    st = stream if stream is not None else torch.cuda.current_stream(dev)
    check(lib().sf_bilinear_marker_to_grids(c.handle, arr, len(grids), px, py, nm, float(dx), float(dy), ps, pw, ld,
                                            n_sum, _stream(st)), "bilinear_marker_to_grids")


def bilinear_marker_to_grid_noalloc(x_grid_min, y_grid_min, val_grid, x_m, y_m, val_m, dx, dy, *, stream=None):
    """The deposit of :func:`bilinear_marker_to_grid` without any device allocation, for callers that
    cannot let a library allocate GPU memory (a runtime that owns the memory through its own pool, a
    stream loop that cudaMalloc's device-wide synchronisation would stall, a fixed memory budget).
    Scratch is a fixed array inside the library, so at most SF_NOALLOC_MAX_MARKERS markers and
    (nx+1)*(ny+1) <= SF_NOALLOC_MAX_CELLS; calls that overlap on the GPU race (they share that array).
    Runs on the device the arrays are on (all four must share it), on that device's current stream unless
    `stream` is given; no context is used."""
    nx, ny = val_grid.shape
    nm = x_m.numel()
    if y_m.numel() != nm or val_m.numel() != nm:
        raise ValueError("x_m, y_m, val_m must have the same length")
    dev = _one_device(val_grid, x_m, y_m, val_m)
    pg, px, py, pv = _grid(val_grid, "val_grid"), _vec(x_m, "x_m"), _vec(y_m, "y_m"), _vec(val_m, "val_m")
    with torch.cuda.device(dev):
        st = stream if stream is not None else torch.cuda.current_stream(dev)
        check(lib().sf_bilinear_marker_to_grid_noalloc(float(x_grid_min), float(y_grid_min), pg, nx, ny, px, py, pv,
                                                       nm, float(dx), float(dy), _stream(st)),
              "bilinear_marker_to_grid_noalloc")


def solve_stokes_info(P, Vx_pad, Vy_pad, rho_vy, mu_b, mu_p, txx, tyy, txy, divV, dtPt, Rx, Ry, dVxdt, dVydt, dtVx,
                      dtVy, Vx_s, Vy_s, g_y, dx, dy, Nx, Ny, dt, maxdisp, comm=None, *,
                      use_free_surface_stabilization=True, eps=1e-8, print_info=False, iter_max=100000,
                      ctx: Context | None = None, stream=None) -> dict:
    """solveStokes! (StokesSolver_multixpu.jl:14-96); returns the full sf_solve_info as a dict.
    The work arrays txx ... dtVy may be None."""
    Nx, Ny = int(Nx), int(Ny)
    ptrs = [
        _grid(P, "P", (Nx - 1, Ny - 1)), _grid(Vx_pad, "Vx_pad", (Nx + 2, Ny + 1)),
        _grid(Vy_pad, "Vy_pad", (Nx + 1, Ny + 2)), _grid(rho_vy, "rho_vy", (Nx + 1, Ny)),
        _grid(mu_b, "mu_b", (Nx, Ny)), _grid(mu_p, "mu_p", (Nx - 1, Ny - 1)),
        _opt_grid(txx, "txx", (Nx - 1, Ny - 1)), _opt_grid(tyy, "tyy", (Nx - 1, Ny - 1)),
        _opt_grid(txy, "txy", (Nx, Ny)), _opt_grid(divV, "divV", (Nx - 1, Ny - 1)),
        _opt_grid(dtPt, "dtPt", (Nx - 1, Ny - 1)), _opt_grid(Rx, "Rx", (Nx - 2, Ny - 1)),
        _opt_grid(Ry, "Ry", (Nx - 1, Ny - 2)), _grid(dVxdt, "dVxdt", (Nx - 2, Ny - 1)),
        _grid(dVydt, "dVydt", (Nx - 1, Ny - 2)), _opt_grid(dtVx, "dtVx", (Nx - 2, Ny - 1)),
        _opt_grid(dtVy, "dtVy", (Nx - 1, Ny - 2)), _grid(Vx_s, "Vx_s", (Nx, Ny + 1)),
        _grid(Vy_s, "Vy_s", (Nx + 1, Ny)),
    ]
    info = _lib.SolveInfo()
    c = _ctx(ctx)
    check(lib().sf_solve_stokes(c.handle, *ptrs, float(g_y), float(dx), float(dy), Nx, Ny, float(dt), float(maxdisp),
                                int(bool(use_free_surface_stabilization)), float(eps), int(bool(print_info)),
                                int(iter_max), _stream(stream), C.byref(info)), "solve_stokes")
    return info.as_dict()


def solve_stokes(P, Vx_pad, Vy_pad, rho_vy, mu_b, mu_p, txx, tyy, txy, divV, dtPt, Rx, Ry, dVxdt, dVydt, dtVx, dtVy,
                 Vx_s, Vy_s, g_y, dx, dy, Nx, Ny, dt, maxdisp, comm=None, *, use_free_surface_stabilization=True,
                 eps=1e-8, print_info=True, iter_max=100000, ctx: Context | None = None, stream=None):
    """solveStokes! (StokesSolver_multixpu.jl:14-96) -> (dt, T_eff, runtime)."""
    r = solve_stokes_info(P, Vx_pad, Vy_pad, rho_vy, mu_b, mu_p, txx, tyy, txy, divV, dtPt, Rx, Ry, dVxdt, dVydt,
                          dtVx, dtVy, Vx_s, Vy_s, g_y, dx, dy, Nx, Ny, dt, maxdisp, comm,
                          use_free_surface_stabilization=use_free_surface_stabilization, eps=eps,
                          print_info=print_info, iter_max=iter_max, ctx=ctx, stream=stream)
    return r["dt"], r["T_eff"], r["runtime"]


class MixedProblem:
    """One Stokes problem for the mixed-precision / batched solver: the caller arrays of
    :func:`solve_stokes` (state in/out) and its scalars.  ``eps`` is absolute; ``rel_tol`` > 0
    replaces it by rel_tol * mean|g_y rho_vy|.  ``dVxdt``, ``dVydt`` (optional, in/out) are the damped
    rates that solveStokes! keeps from one call to the next; without them the solve starts them at zero.
    After a solve, ``result`` holds dt_out, err, inner/outer iteration counts and the convergence flag."""

    def __init__(self, P, Vx_pad, Vy_pad, rho_vy, mu_b, mu_p, Vx_s, Vy_s, g_y, dx, dy, Nx, Ny, dt, maxdisp,
                 eps=1e-8, rel_tol=0.0, use_free_surface_stabilization=True, dVxdt=None, dVydt=None):
        Nx, Ny = int(Nx), int(Ny)
        self.arrays = dict(P=P, Vx_pad=Vx_pad, Vy_pad=Vy_pad, rho_vy=rho_vy, mu_b=mu_b, mu_p=mu_p, Vx_s=Vx_s,
                           Vy_s=Vy_s)
        shapes = dict(P=(Nx - 1, Ny - 1), Vx_pad=(Nx + 2, Ny + 1), Vy_pad=(Nx + 1, Ny + 2), rho_vy=(Nx + 1, Ny),
                      mu_b=(Nx, Ny), mu_p=(Nx - 1, Ny - 1), Vx_s=(Nx, Ny + 1), Vy_s=(Nx + 1, Ny))
        c = _lib.BatchInstance()
        for k, a in self.arrays.items():
            setattr(c, k, _grid(a, k, shapes[k]))
        c.dVxdt = _opt_grid(dVxdt, "dVxdt", (Nx - 2, Ny - 1))
        c.dVydt = _opt_grid(dVydt, "dVydt", (Nx - 1, Ny - 2))
        if dVxdt is not None:
            self.arrays["dVxdt"] = dVxdt
        if dVydt is not None:
            self.arrays["dVydt"] = dVydt
        c.Nx, c.Ny = Nx, Ny
        c.g_y, c.dx, c.dy, c.dt, c.maxdisp = float(g_y), float(dx), float(dy), float(dt), float(maxdisp)
        c.eps, c.rel_tol = float(eps), float(rel_tol)
        c.use_free_surface_stabilization = int(bool(use_free_surface_stabilization))
        self.c = c
        self.result = None


def mixed_options(max_sweeps=4_000_000, fold_every=400, use_graphs=True, dtau_local_max=False,
                  retry_local_max=True, tile_rows=0, tile_schedule=None, overlap_launches=False):
    """Options of the mixed-precision / batched solver (sf_mixed_options).  dtau_local_max: pseudo-time
    steps from the stencil's largest viscosity instead of the reference's average (faster on soft
    inclusions); the converged solution is the same.  retry_local_max: an instance that diverges restarts
    from its inputs with the stencil-maximum step.  tile_rows: 8, 16 or 32 rows per sweep tile, or 0 for
    the autotuner's choice of rows, schedule and launch mode (every choice gives the same bits);
    tile_schedule ("strided" or "chunked") and overlap_launches (sweeps launched under programmatic dependent
    launch) go with a fixed tile_rows."""
    sched = {None: 0, "strided": 1, "chunked": 2}[tile_schedule]
    return _lib.MixedOptions(int(max_sweeps), int(fold_every), int(bool(use_graphs)), int(bool(dtau_local_max)),
                             int(bool(retry_local_max)), int(tile_rows), sched, int(bool(overlap_launches)), 0)


def batch_stats(ctx: Context | None = None) -> dict:
    """Stats of the engine behind the context's last batched / mixed solve (sf_ctx_batch_stats): the sweep
    tile rows and schedule in use, the tuner's state and its measured ns per point-sweep of each candidate
    ((rows, schedule) -> ns)."""
    s = _lib.EngineStats()
    check(lib().sf_ctx_batch_stats(_ctx(ctx).handle, C.byref(s)), "sf_ctx_batch_stats")
    return s.as_dict()


def solve_stokes_batch_mixed(problems, *, options=None, ctx: Context | None = None, stream=None):
    """Solve a list of :class:`MixedProblem` (independent, any grid sizes) with FP64 defect correction
    around FP32 PT sweeps, all instances sharing each sweep launch.  Returns the per-instance results."""
    arr = (_lib.BatchInstance * len(problems))(*[p.c for p in problems])
    opt = options if options is not None else mixed_options()
    c = _ctx(ctx)
    check(lib().sf_solve_stokes_batch_mixed(c.handle, arr, len(problems), C.byref(opt), _stream(stream)),
          "solve_stokes_batch_mixed")
    out = []
    for p, r in zip(problems, arr):
        p.c = r
        p.result = r.results()
        out.append(p.result)
    return out


class Engine:
    """Resident solve engine (sf_engine) for continuous batching: :class:`MixedProblem` instances join with
    :meth:`submit` whenever the arena has room (``None`` when it has not: admission by HBM budget) and
    leave, written back to their arrays, from the :meth:`step` that sees them converge.  Each instance's
    result is bit-identical to solving it alone with :func:`solve_stokes_batch_mixed`."""

    def __init__(self, arena_bytes: int, max_instances: int = 1024, *, options=None, ctx: Context | None = None):
        self._ctx = _ctx(ctx)
        opt = options if options is not None else mixed_options()
        h = C.c_void_p()
        check(lib().sf_engine_create(self._ctx.handle, int(arena_bytes), int(max_instances), C.byref(opt),
                                     C.byref(h)), "sf_engine_create")
        self.handle = h.value
        self._live = {}  # ticket -> MixedProblem; keeps each submitted struct alive at a fixed address
        self._fin = (C.c_int64 * int(max_instances))()

    @staticmethod
    def instance_bytes(Nx: int, Ny: int) -> int:
        b = C.c_int64()
        check(lib().sf_engine_instance_bytes(int(Nx), int(Ny), C.byref(b)), "sf_engine_instance_bytes")
        return b.value

    def submit(self, problem: MixedProblem, *, stream=None):
        """Admit ``problem``; its inputs are read after the work queued on ``stream``.  Returns its ticket,
        or None when the arena or the instance table is full right now."""
        t = C.c_int64(-1)
        st = lib().sf_engine_submit(self.handle, C.byref(problem.c), _stream(stream), C.byref(t))
        if st == _lib.SF_ERR_BUSY:
            return None
        check(st, "sf_engine_submit")
        self._live[t.value] = problem
        problem.result = None
        return t.value

    def step(self, *, stream=None):
        """One round; returns the problems that finished in it (their arrays written back, ordered on
        ``stream``; ``problem.result`` set)."""
        nf, na = C.c_int32(0), C.c_int32(0)
        # room for every admitted instance: nothing stays pending between calls
        check(lib().sf_engine_step(self.handle, _stream(stream), self._fin, len(self._fin), C.byref(nf),
                                   C.byref(na)), "sf_engine_step")
        done = []
        for k in range(nf.value):
            p = self._live.pop(self._fin[k])
            p.result = p.c.results()
            done.append(p)
        return done

    @property
    def active(self) -> int:
        return len(self._live)

    def stats(self) -> dict:
        s = _lib.EngineStats()
        check(lib().sf_engine_get_stats(self.handle, C.byref(s)), "sf_engine_get_stats")
        return s.as_dict()

    def close(self):
        if self.handle:
            lib().sf_engine_destroy(self.handle)
            self.handle = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def residual_scale(rho_vy, Nx, Ny, g_y, *, ctx: Context | None = None, stream=None) -> float:
    """mean |g_y rho_vy| over the Ry interior: eps = rtol * residual_scale(...) is a relative stopping test."""
    out = C.c_double()
    c = _ctx(ctx)
    check(lib().sf_stokes_residual_scale(c.handle, _grid(rho_vy, "rho_vy", (Nx + 1, Ny)), int(Nx), int(Ny),
                                         float(g_y), _stream(stream), C.byref(out)), "residual_scale")
    return out.value


def move_markers_rk4(x_m, y_m, Vx, Vy, x_vx_min, y_vx_min, x_vy_min, y_vy_min, dt, lx, ly, dx, dy, *,
                     ctx: Context | None = None, stream=None):
    """moveMarkersRK4! (MoveMarkers.jl:15-23): advect x_m, y_m in place."""
    nm = x_m.numel()
    if y_m.numel() != nm:
        raise ValueError("x and y Marker coords have not same length")  # MoveMarkers.jl:18
    c = _ctx(ctx)
    check(lib().sf_move_markers_rk4(c.handle, _vec(x_m, "x_m"), _vec(y_m, "y_m"), nm, _grid(Vx, "Vx"), Vx.shape[0],
                                    Vx.shape[1], _grid(Vy, "Vy"), Vy.shape[0], Vy.shape[1], float(x_vx_min),
                                    float(y_vx_min), float(x_vy_min), float(y_vy_min), float(dt), float(lx),
                                    float(ly), float(dx), float(dy), _stream(stream)), "move_markers_rk4")


def rebin_markers(x_m, y_m, x_grid_min, y_grid_min, dx, dy, nx, ny, *, out=None, ctx: Context | None = None,
                  stream=None):
    """Stable counting sort of the markers by cell of an (nx, ny)-node grid.
    Returns int32 CUDA tensors (counts[(nx+1)*(ny+1)], offsets[+1], perm[nm]); `out` may give those three
    tensors (sizes as above, perm at least max(nm, 1)) to be filled instead of new ones."""
    nm = x_m.numel()
    ncells = (nx + 1) * (ny + 1)
    dev = x_m.device
    if out is not None:
        counts, offsets, perm = out
        ok = all(t.dtype == torch.int32 and t.device == dev and t.is_contiguous() for t in out)
        if not ok or counts.numel() != ncells or offsets.numel() != ncells + 1 or perm.numel() < max(nm, 1):
            raise ValueError("rebin_markers: out must be int32 tensors on the markers' device of sizes "
                             f"{ncells}, {ncells + 1} and >= {max(nm, 1)}")
    else:
        counts = torch.empty(ncells, dtype=torch.int32, device=dev)
        offsets = torch.empty(ncells + 1, dtype=torch.int32, device=dev)
        perm = torch.empty(max(nm, 1), dtype=torch.int32, device=dev)
    c = _ctx(ctx)
    check(lib().sf_rebin_markers(c.handle, _vec(x_m, "x_m"), _vec(y_m, "y_m"), nm, float(x_grid_min),
                                 float(y_grid_min), float(dx), float(dy), int(nx), int(ny), counts.data_ptr(),
                                 offsets.data_ptr(), perm.data_ptr(), _stream(stream)), "rebin_markers")
    return counts, offsets, perm[:nm]


def get_warnings(reset: bool = False, *, ctx: Context | None = None) -> dict:
    w = _lib.Warnings()
    c = _ctx(ctx)
    check(lib().sf_get_warnings(c.handle, C.byref(w), int(bool(reset))), "get_warnings")
    return w.as_dict()


# ---------------------------------------------------------------------------
# markers (common.jl:40-110)
# ---------------------------------------------------------------------------
def marker_count(marker_density, nx, ny):
    a, b = C.c_int64(), C.c_int64()
    check(lib().sf_marker_count(int(marker_density), int(nx), int(ny), C.byref(a), C.byref(b)), "marker_count")
    return a.value, b.value


def initialize_markers(marker_density, lx, ly, dx, dy, nx, ny, jitter=0.0, seed=0, *, device="cuda",
                       ctx: Context | None = None, stream=None):
    """initializeMarkersCPU (common.jl:40-90, one rank), generated on the device.
    jitter: width of the uniform jitter in marker sub-spacings (reference: 1.0, RAND_MARKER_POS=false: 0.0)."""
    nmx, nmy = marker_count(marker_density, nx, ny)
    x = torch.empty(nmx * nmy, dtype=torch.float64, device=device)
    y = torch.empty_like(x)
    c = _ctx(ctx)
    check(lib().sf_init_markers(c.handle, int(marker_density), float(lx), float(ly), float(dx), float(dy), int(nx),
                                int(ny), float(jitter), int(seed), x.data_ptr(), y.data_ptr(), _stream(stream)),
          "initialize_markers")
    return x, y


def initialize_markers_host(marker_density, lx, ly, dx, dy, nx, ny, jitter=0.0, seed=0):
    """Same as :func:`initialize_markers` into pinned host tensors (for the end-to-end path)."""
    nmx, nmy = marker_count(marker_density, nx, ny)
    x = torch.empty(nmx * nmy, dtype=torch.float64, pin_memory=torch.cuda.is_available())
    y = torch.empty_like(x)
    check(lib().sf_init_markers_host(int(marker_density), float(lx), float(ly), float(dx), float(dy), int(nx),
                                     int(ny), float(jitter), int(seed), C.c_void_p(x.data_ptr()),
                                     C.c_void_p(y.data_ptr())), "initialize_markers_host")
    return x, y


class PlumeModel:
    """Layered 'sticky air' + circular plume + matrix material model
    (StokesFlow2D_multixpu.jl:382-404): y < air_height -> air, else inside the
    plume circle -> plume, else matrix."""

    FIELDS = ("air_height", "plume_x", "plume_y", "plume_r", "rho_air", "rho_matrix", "rho_plume", "mu_air",
              "mu_matrix", "mu_plume")

    def __init__(self, **kw):
        for f in self.FIELDS:
            setattr(self, f, float(kw[f]))

    def c(self):
        return _lib.PlumeModelC(*[getattr(self, f) for f in self.FIELDS])

    def __repr__(self):
        return "PlumeModel(" + ", ".join(f"{f}={getattr(self, f)!r}" for f in self.FIELDS) + ")"


def set_initial_marker_properties(x_m, y_m, model: PlumeModel, x0=0.0, y0=0.0, *, ctx: Context | None = None,
                                  stream=None):
    """setInitialMarkerProperties! (common.jl:104-110) -> (rho_m, mu_m) on the markers' device."""
    nm = x_m.numel()
    rho = torch.empty_like(x_m)
    mu = torch.empty_like(x_m)
    cm = model.c()
    if x_m.is_cuda:
        c = _ctx(ctx)
        check(lib().sf_set_marker_properties(c.handle, C.byref(cm), _vec(x_m, "x_m"), _vec(y_m, "y_m"), nm,
                                             float(x0), float(y0), rho.data_ptr(), mu.data_ptr(), _stream(stream)),
              "set_initial_marker_properties")
    else:
        assert x_m.dtype == torch.float64 and x_m.is_contiguous() and y_m.is_contiguous()
        check(lib().sf_set_marker_properties_host(C.byref(cm), C.c_void_p(x_m.data_ptr()), C.c_void_p(y_m.data_ptr()),
                                                  nm, float(x0), float(y0), C.c_void_p(rho.data_ptr()),
                                                  C.c_void_p(mu.data_ptr())), "set_initial_marker_properties")
    return rho, mu
