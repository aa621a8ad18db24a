"""Domain decomposition of one Stokes solve over a grid of ranks, as the reference's ImplicitGlobalGrid
set-up does it (init_global_grid with overlaps 2: StokesFlow2D_multixpu.jl:61, StokesSolver_multixpu.jl).

Every rank holds a local grid of Nx x Ny points; neighbouring ranks overlap by 2 points, so the global grid
has ``nx_g = dims_x * (Nx - 2) + 2`` points in x (``nx_g()``), and the local point i of the rank at
coordinate cx is the global point ``cx * (Nx - 2) + i``.  A staggered array that is ``s`` entries larger than
the grid in a dimension (Vx_s: Nx in x, Ny + 1 in y) has its local entries at the same offsets, ``N + s`` of
them.  :func:`solve_stokes_decomposed` runs all ranks from this process (one GPU per rank, or several
ranks on one GPU) through ``sf_solve_stokes_decomposed``.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import check, lib

# the arrays of a rank: name -> (extra entries in x, in y) relative to the local grid
ARRAYS = {"P": (-1, -1), "Vx_pad": (2, 1), "Vy_pad": (1, 2), "rho_vy": (1, 0), "mu_b": (0, 0), "mu_p": (-1, -1),
          "dVxdt": (-2, -1), "dVydt": (-1, -2), "Vx_s": (0, 1), "Vy_s": (1, 0)}


def global_size(dims: int, n_local: int) -> int:
    """nx_g() / ny_g(): points of the global grid along a dimension of `dims` ranks."""
    return dims * (n_local - 2) + 2


def local_size(dims: int, n_global: int) -> int:
    """Points per rank that tile a global grid of n_global points with `dims` ranks (exact division needed)."""
    if (n_global - 2) % dims:
        raise ValueError(f"{n_global} points do not split into {dims} ranks with overlap 2")
    return (n_global - 2) // dims + 2


def local_slices(name: str, coord, Nx: int, Ny: int):
    """(x slice, y slice) of a rank's array `name` in the global array."""
    sx, sy = ARRAYS[name]
    x0, y0 = coord[0] * (Nx - 2), coord[1] * (Ny - 2)
    return slice(x0, x0 + Nx + sx), slice(y0, y0 + Ny + sy)


def split(global_arrays: dict, dims, Nx: int, Ny: int) -> dict:
    """{(cx, cy): {name: local column-major copy}} of the given global (column-major) tensors."""
    out = {}
    for cy in range(dims[1]):
        for cx in range(dims[0]):
            loc = {}
            for name, a in global_arrays.items():
                xs, ys = local_slices(name, (cx, cy), Nx, Ny)
                v = a[xs, ys]
                # always a copy (a whole-array slice of a 1-rank split would otherwise share storage),
                # column-major like the library's arrays
                loc[name] = v.t().clone().t()
            out[(cx, cy)] = loc
    return out


def gather(ranks: dict, name: str, dims, Nx: int, Ny: int) -> torch.Tensor:
    """The global array `name` from the ranks' local ones, as gather_V_grid / create_grid_view assemble it
    (GlobalGather.jl:59-114): along each dimension the overlap o = 2 + s (s: extra entries of the array)
    splits at every rank boundary, o//2 entries dropped from the lower rank and the rest from the upper."""
    sx, sy = ARRAYS[name]
    some = next(iter(ranks.values()))[name]
    out = torch.empty((global_size(dims[0], Nx) + sx, global_size(dims[1], Ny) + sy), dtype=some.dtype,
                      device=some.device)

    def kept(c, dimsn, n_loc, s):
        o = 2 + s
        nl = o // 2
        nr = o - nl
        lo = nr if c > 0 else 0
        hi = n_loc + s - nl if c < dimsn - 1 else n_loc + s
        return lo, hi, c * (n_loc - 2)

    for (cx, cy), loc in ranks.items():
        x_lo, x_hi, x0 = kept(cx, dims[0], Nx, sx)
        y_lo, y_hi, y0 = kept(cy, dims[1], Ny, sy)
        out[x0 + x_lo:x0 + x_hi, y0 + y_lo:y0 + y_hi] = loc[name][x_lo:x_hi, y_lo:y_hi]
    return out


def gather_markers(ranks_markers: dict, dims, lx_loc: float, ly_loc: float, dx: float, dy: float):
    """gather_markers! (GlobalGather.jl:10-48): the ranks' markers concatenated in MPI rank order of the
    Cartesian communicator (x coordinate slowest), each shifted from local to global coordinates by
    (coord_x (lx_loc - dx), coord_y (ly_loc - dy)).  ranks_markers: {(cx, cy): (x_m, y_m, rho_m, mu_m)}."""
    xs, ys, rs, ms = [], [], [], []
    for cx in range(dims[0]):
        for cy in range(dims[1]):
            x, y, r, m = ranks_markers[(cx, cy)]
            xs.append(x + cx * (lx_loc - dx))
            ys.append(y + cy * (ly_loc - dy))
            rs.append(r)
            ms.append(m)
    return torch.cat(xs), torch.cat(ys), torch.cat(rs), torch.cat(ms)


def _ordered(d: dict):
    return sorted(d.items(), key=lambda kv: (kv[0][1], kv[0][0]))


def sum_overlapping_values(arrays: dict, dims, Nx: int, Ny: int, contexts: dict):
    """sumOverlappingValues! (MarkerToGrid.jl:183-269) over all ranks: arrays {(cx, cy): column-major CUDA
    tensor}, all of one shape; contexts {(cx, cy): api.Context}, one per rank."""
    from .api import _grid
    arr = (_lib.RankArray * len(arrays))()
    shape = None
    for k, (coord, a) in enumerate(_ordered(arrays)):
        shape = tuple(a.shape)
        arr[k].ctx = contexts[coord].handle
        arr[k].a = _grid(a, "array", shape)
        arr[k].coord_x, arr[k].coord_y = int(coord[0]), int(coord[1])
    check(lib().sf_sum_overlapping_values(arr, int(dims[0]), int(dims[1]), int(Nx), int(Ny), shape[0], shape[1]),
          "sum_overlapping_values")


def deposit_decomposed(x_grid_min, y_grid_min, val_grids: dict, markers: dict, dx, dy, dims, Nx: int, Ny: int,
                       contexts: dict, sums: dict | None = None):
    """bilinearMarkerToGrid! on every rank (MarkerToGrid.jl:18-38): each rank's markers summed onto its own
    grid, the weight and value sums added across the overlaps (sumOverlappingValues! on the (Nx+1, Ny)
    interpolation arrays, StokesFlow2D_multixpu.jl:112-114), then safeDivision.  val_grids {(cx, cy): grid},
    markers {(cx, cy): (x_m, y_m, val_m)} in local coordinates; sums: reusable {(cx, cy): (val_wt_sum,
    wt_sum)} of shape (Nx+1, Ny)."""
    from . import api
    if sums is None:
        sums = {c: (api.zeros(Nx + 1, Ny, device=g.device), api.zeros(Nx + 1, Ny, device=g.device))
                for c, g in val_grids.items()}
    for coord, g in val_grids.items():
        x, y, v = markers[coord]
        vws, ws = sums[coord]
        api.bilinear_marker_to_grid(x_grid_min, y_grid_min, g, x, y, v, dx, dy, vws, ws, ctx=contexts[coord])
    sum_overlapping_values({c: s[1] for c, s in sums.items()}, dims, Nx, Ny, contexts)
    sum_overlapping_values({c: s[0] for c, s in sums.items()}, dims, Nx, Ny, contexts)
    for coord, g in val_grids.items():
        vws, ws = sums[coord]
        check(lib().sf_safe_division(contexts[coord].handle, api._grid(g, "val_grid"), g.shape[0], g.shape[1],
                                     vws.data_ptr(), ws.data_ptr(), vws.shape[0], api._stream(None)),
              "safe_division")
    return sums


def exchange_markers(markers: dict, dims, lx, ly, dx, dy, contexts: dict) -> dict:
    """exchangeMarkers (MarkerExchange.jl:8-163) for all ranks: markers {(cx, cy): (x, y, rho, mu)} in local
    coordinates -> the same after the exchange (new tensors): kept markers in order, then the received ones
    by neighbour index 1..8."""
    ranks = _ordered(markers)
    arr = (_lib.MarkerRank * len(ranks))()
    outs = {}

    def fill(cap_of):
        for k, (coord, (x, y, r, m)) in enumerate(ranks):
            cap = cap_of(coord, x.numel())
            o = [torch.empty(max(cap, 1), dtype=torch.float64, device=x.device) for _ in range(4)]
            outs[coord] = o
            d = arr[k]
            d.ctx = contexts[coord].handle
            d.x, d.y, d.rho, d.mu = x.data_ptr(), y.data_ptr(), r.data_ptr(), m.data_ptr()
            d.n = x.numel()
            d.x_out, d.y_out, d.rho_out, d.mu_out = (t.data_ptr() for t in o)
            d.capacity = cap
            d.coord_x, d.coord_y = int(coord[0]), int(coord[1])

    torch.cuda.synchronize()
    fill(lambda coord, n: n + n // 8 + 1024)
    st = lib().sf_exchange_markers(arr, int(dims[0]), int(dims[1]), float(lx), float(ly), float(dx), float(dy))
    if st == _lib.SF_ERR_TOO_LARGE:   # more arrived than the first guess holds: size exactly and redo
        need = {coord: arr[k].n_out for k, (coord, _) in enumerate(ranks)}
        fill(lambda coord, n: need[coord])
        st = lib().sf_exchange_markers(arr, int(dims[0]), int(dims[1]), float(lx), float(ly), float(dx), float(dy))
    check(st, "exchange_markers")
    return {coord: tuple(t[:arr[k].n_out] for t in outs[coord]) for k, (coord, _) in enumerate(ranks)}


def marker_count_rank(marker_density: int, Nx: int, Ny: int, coord, dims):
    """Markers in x / y on the rank at ``coord`` (common.jl:43-66): a side that faces a neighbour loses
    floor(md/2) (low side) or ceil(md/2) (high side) marker columns, so the ranks' markers tile the global
    layout."""
    a, b = C.c_int64(), C.c_int64()
    check(lib().sf_marker_count_rank(int(marker_density), int(Nx), int(Ny), int(coord[0]), int(coord[1]),
                                     int(dims[0]), int(dims[1]), C.byref(a), C.byref(b)), "marker_count_rank")
    return a.value, b.value


def rank_seed(seed: int, coord, dims) -> int:
    """The jitter seed of a rank: ``seed`` plus its MPI rank in the Cartesian communicator (x slowest), so
    that one rank draws what the one-domain ``initialize_markers`` draws with ``seed``."""
    return int(seed) + coord[0] * dims[1] + coord[1]


def initialize_markers_decomposed(dims, Nx: int, Ny: int, Lx: float, Ly: float, model, marker_density: int,
                                  contexts: dict, *, jitter: float = 0.0, seed: int = 0) -> dict:
    """initializeMarkersCPU then setInitialMarkerProperties! on every rank (StokesFlow2D_multixpu.jl:135-136,
    common.jl:40-110), generated on each rank's device.  Each rank lays out its own part of the global marker
    lattice in local coordinates; with jitter and an odd density the markers that jittered across a rank
    boundary move to the neighbour through :func:`exchange_markers` with zero properties (common.jl:93-97),
    and then the properties are set from the model at the global position ``x0 + x_m`` with
    ``x0 = coord_x (Nx - 2) dx`` (StokesFlow2D_multixpu.jl:80-81).  ``model`` is an ``api.PlumeModel`` or any
    object with ``marker_properties(x, y)``.  Returns {(cx, cy): (x_m, y_m, rho_m, mu_m)}."""
    from . import api
    dx = Lx / (global_size(dims[0], Nx) - 1)
    dy = Ly / (global_size(dims[1], Ny) - 1)
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    out = {}
    for coord, ctx in _ordered(contexts):
        nmx, nmy = marker_count_rank(marker_density, Nx, Ny, coord, dims)
        dev = f"cuda:{ctx.device}"
        x = torch.empty(nmx * nmy, dtype=torch.float64, device=dev)
        y = torch.empty_like(x)
        with torch.cuda.device(ctx.device):
            check(lib().sf_init_markers_rank(ctx.handle, int(marker_density), float(lx), float(ly), float(dx),
                                             float(dy), int(Nx), int(Ny), int(coord[0]), int(coord[1]),
                                             int(dims[0]), int(dims[1]), float(jitter),
                                             rank_seed(seed, coord, dims), x.data_ptr(), y.data_ptr(),
                                             api._stream(None)), "initialize_markers_decomposed")
        out[coord] = (x, y, torch.zeros_like(x), torch.zeros_like(x))
    if jitter != 0.0 and marker_density % 2 == 1:
        out = exchange_markers(out, dims, lx, ly, dx, dy, contexts)
    for coord, (x, y, _, _) in out.items():
        x0, y0 = coord[0] * (Nx - 2) * dx, coord[1] * (Ny - 2) * dy
        with torch.cuda.device(contexts[coord].device):
            if hasattr(model, "marker_properties"):
                rho, mu = model.marker_properties(x0 + x, y0 + y)
            else:
                rho, mu = api.set_initial_marker_properties(x, y, model, x0, y0, ctx=contexts[coord])
        out[coord] = (x, y, rho, mu)
    return out


def rank_devices(dims, n_devices: int) -> dict:
    """Devices for a dims[0] x dims[1] grid of ranks on n_devices GPUs: {(cx, cy): device index}.  The ranks
    are taken in MPI rank order of the Cartesian communicator (x slowest, rank = cx * dims[1] + cy) and cut
    into n_devices contiguous runs of near-equal length (sizes differ by at most one), so that the ranks
    sharing a GPU are y-neighbours and a halo update crosses between GPUs only at the runs' ends.  With more
    devices than ranks every rank has a GPU of its own."""
    if n_devices < 1:
        raise ValueError("rank_devices: need at least one device")
    n = dims[0] * dims[1]
    return {(cx, cy): (cx * dims[1] + cy) * n_devices // n for cx in range(dims[0]) for cy in range(dims[1])}


class DecomposedStokesFlow2D:
    """The StokesFlow2D timestep loop (StokesFlow2D_multixpu.jl:157-191) on dims[0] x dims[1] ranks driven from
    this process: per timestep the three deposits with overlap sums, the decomposed solve, RK4 advection of
    each rank's markers on its local domain, and the marker exchange.  Nx, Ny: local grid points of a rank;
    Lx, Ly: the global domain.  markers {(cx, cy): (x_m, y_m, rho_m, mu_m)} in local coordinates (the ranks'
    initial markers), or None to lay them out from ``model`` with :func:`initialize_markers_decomposed`;
    devices {(cx, cy): CUDA device index}, or "auto" for :func:`rank_devices` over every visible GPU (default:
    the current device for all).  Halo planes and overlap blocks between ranks on different GPUs are read
    directly from the neighbour's memory where the two GPUs are peers (NVLink), else copied by the runtime."""

    def __init__(self, dims, Nx: int, Ny: int, Lx: float, Ly: float, markers: dict | None = None, *, model=None,
                 marker_density: int = 4, jitter: float = 0.0, seed: int = 0, eps=1e-5, iter_max=100000,
                 g_y=9.81, maxdisp=0.5, devices: dict | None = None):
        from . import api
        from .driver import node_origins
        self.dims, self.Nx, self.Ny = tuple(dims), Nx, Ny
        self.dx = Lx / (global_size(dims[0], Nx) - 1)    # :76-77 with nx_g()
        self.dy = Ly / (global_size(dims[1], Ny) - 1)
        self.lx, self.ly = (Nx - 1) * self.dx, (Ny - 1) * self.dy
        self.o = node_origins(self.dx, self.dy)
        self.eps, self.iter_max, self.g_y, self.maxdisp = eps, iter_max, g_y, maxdisp
        self.dt, self.t_tot, self.nt = 0.0, 0.0, 0
        self.ctx, self.ranks, self.sums = {}, {}, {}
        coords = [(cx, cy) for cy in range(dims[1]) for cx in range(dims[0])]
        if devices == "auto":
            devices = rank_devices(dims, torch.cuda.device_count())
        for c in coords:
            dev = (devices or {}).get(c, torch.cuda.current_device())
            with torch.cuda.device(dev):
                self.ctx[c] = api.Context(dev)
                z = lambda *s: api.zeros(*s, device=f"cuda:{dev}")  # noqa: E731
                self.ranks[c] = {n: z(Nx + sx, Ny + sy) for n, (sx, sy) in ARRAYS.items()}
                self.sums[c] = (z(Nx + 1, Ny), z(Nx + 1, Ny))   # interp_size (:112-114)
        if markers is None:
            if model is None:
                raise ValueError("DecomposedStokesFlow2D: give markers or a model")
            markers = initialize_markers_decomposed(dims, Nx, Ny, Lx, Ly, model, marker_density, self.ctx,
                                                    jitter=jitter, seed=seed)
        self.markers = {c: tuple(t.to(f"cuda:{self.ranks[c]['P'].device.index}") for t in markers[c]) for c in coords}

    def step(self) -> dict:
        from . import api
        d, o = self.dims, self.o
        Nx, Ny = self.Nx, self.Ny
        for name, (xo, yo), q in (("rho_vy", ("x_rho", "y_rho"), 2), ("mu_b", ("x", "y"), 3),
                                  ("mu_p", ("x_p", "y_p"), 3)):          # :164-166
            grids = {c: r[name] for c, r in self.ranks.items()}
            mk = {c: (m[0], m[1], m[q]) for c, m in self.markers.items()}
            deposit_decomposed(o[xo], o[yo], grids, mk, self.dx, self.dy, d, Nx, Ny, self.ctx, self.sums)
        info = solve_stokes_decomposed(self.ranks, d, Nx, Ny, self.g_y, self.dx, self.dy, self.dt, self.maxdisp,
                                       eps=self.eps, iter_max=self.iter_max, contexts=self.ctx)   # :171-176
        self.dt = info["dt"]
        for c, r in self.ranks.items():                                   # :181, on the local domain
            x, y = self.markers[c][0], self.markers[c][1]
            api.move_markers_rk4(x, y, r["Vx_pad"], r["Vy_pad"], o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"],
                                 self.dt, self.lx, self.ly, self.dx, self.dy, ctx=self.ctx[c])
        self.markers = exchange_markers(self.markers, d, self.lx, self.ly, self.dx, self.dy, self.ctx)   # :186-191
        self.t_tot += self.dt
        self.nt += 1
        return dict(nt=self.nt, dt=self.dt, t_tot=self.t_tot, info=info)

    def velocities(self):
        """(Vx_glob, Vy_glob) as gather_V_grid hands them back (StokesFlow2D_multixpu.jl:232)."""
        return (gather(self.ranks, "Vx_pad", self.dims, self.Nx, self.Ny),
                gather(self.ranks, "Vy_pad", self.dims, self.Nx, self.Ny))


def solve_stokes_decomposed(ranks: dict, dims, Nx: int, Ny: int, g_y, dx, dy, dt, maxdisp, *, eps=1e-8,
                            iter_max=100000, use_free_surface_stabilization=True, contexts=None) -> dict:
    """solveStokes! on dims[0] x dims[1] ranks (StokesSolver_multixpu.jl:14-96 with update_halo! and the
    Allreduce reductions).  ranks: {(cx, cy): {array name: local CUDA tensor}}; contexts: {(cx, cy):
    api.Context} (one per rank; default: a new context on each tensor's device).  Returns the global
    results of sf_solve_info."""
    from .api import Context, _grid
    n = len(ranks)
    arr = (_lib.Domain * n)()
    ctxs = {}
    for k, (coord, loc) in enumerate(sorted(ranks.items(), key=lambda kv: (kv[0][1], kv[0][0]))):
        ctx = (contexts or {}).get(coord) or Context(loc["P"].device.index)
        ctxs[coord] = ctx
        d = arr[k]
        d.ctx = ctx.handle
        for name, (sx, sy) in ARRAYS.items():
            setattr(d, name, _grid(loc[name], name, (Nx + sx, Ny + sy)))
        d.coord_x, d.coord_y = int(coord[0]), int(coord[1])
    info = _lib.SolveInfo()
    check(lib().sf_solve_stokes_decomposed(arr, int(dims[0]), int(dims[1]), int(Nx), int(Ny), float(g_y), float(dx),
                                           float(dy), float(dt), float(maxdisp),
                                           int(bool(use_free_surface_stabilization)), float(eps), int(iter_max),
                                           C.byref(info)), "solve_stokes_decomposed")
    for c in ctxs.values():
        torch.cuda.synchronize(torch.device("cuda", c.device))
    return info.as_dict()
