"""CPU oracle for the StokesFlow.jl per-timestep hot path.

TEST INFRASTRUCTURE ONLY.  This package is the checker for the CUDA path and
the timed CPU baseline of ``bench.py``.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py`` (its CPU-baseline and reference
legs) may import it; the product package never does.

It wraps ``liboracle.so`` (built from ``sf_oracle.c`` by ``oracle/Makefile``),
a plain-C restatement of the Julia reference (dastrm/StokesFlow.jl) with the
reference's floating-point expression order:

* ``scripts/common.jl:22-110``           marker layout, properties, topleftIndexRelDist
* ``scripts/MarkerToGrid.jl:18-172``     bilinearMarkerToGrid! (serial, marker order)
* ``scripts/StokesSolver_multixpu.jl``   solveStokes! (pseudo-transient iteration)
* ``scripts/MoveMarkers.jl:15-187``      moveMarkersRK4!, interpolateV

plus numpy restatements of the pieces that cross ranks (``sumOverlappingValues!``,
``exchangeMarkers``) and a composition of the decomposed timestep from them.

Pinned against every known-answer test the reference holds for this path, at
the reference's own tolerances: test_StokesSolver.jl, test_MarkerToGrid.jl,
test_MoveMarkers.jl, test_InitialMarkerCoords.jl, the three
test_MarkerExchange_*.jl and test_StokesFlow2D.jl, the last four also on the
rank grids the reference runs them on (tests/test_oracle_golden.py,
tests/test_oracle_exchange_reference.py, tests/test_domains*.py).

Grid arrays are numpy arrays in Fortran order with the Julia shape, so
``A[ix-1, iy-1]`` is Julia's ``A[ix, iy]`` and ``A.ravel(order="F")`` is
Julia's linear indexing.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_d = C.c_double
_i64 = C.c_int64
_pd = C.POINTER(C.c_double)
_pi64 = C.POINTER(C.c_int64)


def build() -> str:
    """Compile liboracle.so with oracle/Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class _SolveResult(C.Structure):
    _fields_ = [("dt_out", _d), ("err", _d), ("iters", _i64), ("n_checks", _i64), ("runtime_s", _d)]


class _PlumeModel(C.Structure):
    _fields_ = [(n, _d) for n in (
        "air_height", "plume_x", "plume_y", "plume_r",
        "rho_air", "rho_matrix", "rho_plume", "mu_air", "mu_matrix", "mu_plume")]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.orc_topleft_index_rel_dist.argtypes = [_d, _d, _d, _d, _d, _d, _pi64, _pi64, _pd, _pd]
        L.orc_uniform.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_uniform.restype = _d
        L.orc_marker_counts.argtypes = [_i64, _i64, _i64, _pi64, _pi64]
        L.orc_init_markers.argtypes = [_i64, _d, _d, _d, _d, _i64, _i64, _d, C.c_uint64, _pd, _pd]
        L.orc_marker_counts_rank.argtypes = [_i64, _i64, _i64, C.c_int, C.c_int, C.c_int, C.c_int, _pi64, _pi64]
        L.orc_init_markers_rank.argtypes = [_i64, _d, _d, _d, _d, _i64, _i64, C.c_int, C.c_int, C.c_int, C.c_int,
                                            _d, C.c_uint64, _pd, _pd]
        L.orc_set_marker_properties.argtypes = [C.POINTER(_PlumeModel), _pd, _pd, _i64, _d, _d, _pd, _pd]
        L.orc_bilinear_marker_to_grid.argtypes = [_d, _d, _pd, _i64, _i64, _pd, _pd, _pd, _i64, _d, _d,
                                                  _pd, _pd, _i64, _i64, _pi64, _pi64]
        L.orc_solve_stokes.argtypes = [_pd] * 19 + [_d, _d, _d, _i64, _i64, _d, _d, C.c_int, _d, _i64,
                                                    C.c_int, C.POINTER(_SolveResult)]
        L.orc_compute_dt.argtypes = [_pd, _i64, _pd, _i64, _d, _d, _d]
        L.orc_compute_dt.restype = _d
        L.orc_interpolate_v.argtypes = [_d, _d, _pd, _i64, _i64, _pd, _i64, _i64, _d, _d, _d, _d, _d, _d,
                                        _pd, _pd, _pi64]
        L.orc_move_markers_rk4.argtypes = [_pd, _pd, _i64, _pd, _i64, _i64, _pd, _i64, _i64, _d, _d, _d, _d,
                                           _d, _d, _d, _d, _d, C.c_int, _pi64]
        L.orc_cell_counts.argtypes = [_pd, _pd, _i64, _d, _d, _d, _d, _i64, _i64, C.POINTER(C.c_int32)]
        L.orc_cell_counts.restype = _i64
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1), "need float64 column-major"
    return a.ctypes.data_as(_pd)


def zeros(*shape) -> np.ndarray:
    """Julia @zeros(shape...): Float64, column-major."""
    return np.zeros(shape, dtype=np.float64, order="F")


# --------------------------------------------------------------------------
# common.jl
# --------------------------------------------------------------------------
def topleft_index_rel_dist(x_grid_min, y_grid_min, x, y, dx, dy):
    """common.jl:22-33 -> (ix, iy, dxij, dyij), ix/iy 1-based."""
    ix, iy, a, b = _i64(), _i64(), _d(), _d()
    lib().orc_topleft_index_rel_dist(x_grid_min, y_grid_min, x, y, dx, dy,
                                     C.byref(ix), C.byref(iy), C.byref(a), C.byref(b))
    return ix.value, iy.value, a.value, b.value


def uniform(seed: int, counter: int) -> float:
    return lib().orc_uniform(seed, counter)


def marker_counts(marker_density, nx, ny):
    a, b = _i64(), _i64()
    lib().orc_marker_counts(marker_density, nx, ny, C.byref(a), C.byref(b))
    return a.value, b.value


def initialize_markers(marker_density, lx, ly, dx, dy, nx, ny, jitter=0.0, seed=0):
    """common.jl:40-90 on one rank; jitter = width of the uniform jitter in sub-spacings."""
    nmx, nmy = marker_counts(marker_density, nx, ny)
    x = np.empty(nmx * nmy)
    y = np.empty(nmx * nmy)
    lib().orc_init_markers(marker_density, lx, ly, dx, dy, nx, ny, jitter, seed, _p(x), _p(y))
    return x, y


def marker_counts_rank(marker_density, nx, ny, coords, dims):
    """common.jl:43-66: markers in x / y on the rank at ``coords`` of a ``dims`` grid."""
    a, b = _i64(), _i64()
    lib().orc_marker_counts_rank(marker_density, nx, ny, coords[0], coords[1], dims[0], dims[1],
                                 C.byref(a), C.byref(b))
    return a.value, b.value


def initialize_markers_rank(marker_density, lx, ly, dx, dy, nx, ny, coords, dims, jitter=0.0, seed=0):
    """common.jl:40-94 on the rank at ``coords``; lx, ly, nx, ny are the rank's local sizes."""
    nmx, nmy = marker_counts_rank(marker_density, nx, ny, coords, dims)
    x = np.empty(nmx * nmy)
    y = np.empty(nmx * nmy)
    lib().orc_init_markers_rank(marker_density, lx, ly, dx, dy, nx, ny, coords[0], coords[1], dims[0], dims[1],
                                jitter, seed, _p(x), _p(y))
    return x, y


@dataclass
class PlumeModel:
    air_height: float
    plume_x: float
    plume_y: float
    plume_r: float
    rho_air: float
    rho_matrix: float
    rho_plume: float
    mu_air: float
    mu_matrix: float
    mu_plume: float

    def _c(self):
        return _PlumeModel(*[float(getattr(self, f[0])) for f in _PlumeModel._fields_])


def set_marker_properties(model: PlumeModel, x_m, y_m, x0=0.0, y0=0.0):
    """common.jl:104-110."""
    rho = np.empty_like(x_m)
    mu = np.empty_like(x_m)
    cm = model._c()
    lib().orc_set_marker_properties(C.byref(cm), _p(x_m), _p(y_m), x_m.size, x0, y0, _p(rho), _p(mu))
    return rho, mu


# --------------------------------------------------------------------------
# MarkerToGrid.jl
# --------------------------------------------------------------------------
def bilinear_marker_to_grid(x_grid_min, y_grid_min, val_grid, x_m, y_m, val_m, dx, dy,
                            val_wt_sum, wt_sum):
    """MarkerToGrid.jl:18-38 (single rank).  Mutates val_grid, val_wt_sum, wt_sum.
    Returns (n_bad_markers, n_empty_nodes)."""
    nx, ny = val_grid.shape
    assert val_wt_sum.shape == wt_sum.shape
    nb, ne = _i64(), _i64()
    lib().orc_bilinear_marker_to_grid(x_grid_min, y_grid_min, _p(val_grid), nx, ny, _p(x_m), _p(y_m),
                                      _p(val_m), x_m.size, dx, dy, _p(val_wt_sum), _p(wt_sum),
                                      wt_sum.shape[0], wt_sum.size, C.byref(nb), C.byref(ne))
    return nb.value, ne.value


def cell_counts(x_m, y_m, x_grid_min, y_grid_min, dx, dy, nx, ny):
    """Markers per cell of an (nx, ny)-node grid, keys (ix, iy) in 0..nx x 0..ny
    (0-based array index = 1-based topleftIndexRelDist index).  Returns
    (counts[(nx+1)*(ny+1)] as int32, n_outside)."""
    counts = np.zeros((nx + 1) * (ny + 1), dtype=np.int32)
    nout = lib().orc_cell_counts(_p(x_m), _p(y_m), x_m.size, x_grid_min, y_grid_min, dx, dy, nx, ny,
                                 counts.ctypes.data_as(C.POINTER(C.c_int32)))
    return counts, nout


# --------------------------------------------------------------------------
# StokesSolver_multixpu.jl
# --------------------------------------------------------------------------
@dataclass
class SolveResult:
    dt: float
    err: float
    iters: int
    n_checks: int
    runtime_s: float


def stokes_arrays(Nx, Ny):
    """All arrays of StokesFlow2D_multixpu.jl:89-109, zero-initialised."""
    return dict(
        P=zeros(Nx - 1, Ny - 1), Vx=zeros(Nx + 2, Ny + 1), Vy=zeros(Nx + 1, Ny + 2),
        rho_vy=zeros(Nx + 1, Ny), mu_b=zeros(Nx, Ny), mu_p=zeros(Nx - 1, Ny - 1),
        txx=zeros(Nx - 1, Ny - 1), tyy=zeros(Nx - 1, Ny - 1), txy=zeros(Nx, Ny),
        divV=zeros(Nx - 1, Ny - 1), dtPt=zeros(Nx - 1, Ny - 1), Rx=zeros(Nx - 2, Ny - 1),
        Ry=zeros(Nx - 1, Ny - 2), dVxdt=zeros(Nx - 2, Ny - 1), dVydt=zeros(Nx - 1, Ny - 2),
        dtVx=zeros(Nx - 2, Ny - 1), dtVy=zeros(Nx - 1, Ny - 2), Vx_s=zeros(Nx, Ny + 1),
        Vy_s=zeros(Nx + 1, Ny))


_SOLVE_ORDER = ["P", "Vx", "Vy", "rho_vy", "mu_b", "mu_p", "txx", "tyy", "txy", "divV", "dtPt", "Rx", "Ry",
                "dVxdt", "dVydt", "dtVx", "dtVy", "Vx_s", "Vy_s"]


def solve_stokes(a: dict, g_y, dx, dy, Nx, Ny, dt, maxdisp, use_free_surface_stabilization=True,
                 eps=1e-8, iter_max=100000, nthreads=1) -> SolveResult:
    """StokesSolver_multixpu.jl:14-96 on the arrays of ``stokes_arrays``."""
    for k in _SOLVE_ORDER:
        assert a[k].flags.f_contiguous and a[k].dtype == np.float64, k
    r = _SolveResult()
    lib().orc_solve_stokes(*[_p(a[k]) for k in _SOLVE_ORDER], g_y, dx, dy, Nx, Ny, dt, maxdisp,
                           int(bool(use_free_surface_stabilization)), eps, iter_max, nthreads, C.byref(r))
    return SolveResult(r.dt_out, r.err, r.iters, r.n_checks, r.runtime_s)


def compute_dt(Vx, Vy, maxdisp, dx, dy):
    """StokesSolver_multixpu.jl:118-121 (single rank)."""
    return lib().orc_compute_dt(_p(Vx), Vx.size, _p(Vy), Vy.size, maxdisp, dx, dy)


# --------------------------------------------------------------------------
# MoveMarkers.jl
# --------------------------------------------------------------------------
def interpolate_v(x, y, Vx, Vy, x_vx_min, y_vx_min, x_vy_min, y_vy_min, dx, dy):
    """MoveMarkers.jl:76-174 -> (vx, vy, n_failsafe)."""
    vx, vy, nf = _d(), _d(), _i64(0)
    lib().orc_interpolate_v(x, y, _p(Vx), Vx.shape[0], Vx.shape[1], _p(Vy), Vy.shape[0], Vy.shape[1],
                            x_vx_min, y_vx_min, x_vy_min, y_vy_min, dx, dy,
                            C.byref(vx), C.byref(vy), C.byref(nf))
    return vx.value, vy.value, nf.value


def move_markers_rk4(x_m, y_m, Vx, Vy, x_vx_min, y_vx_min, x_vy_min, y_vy_min, dt, lx, ly, dx, dy,
                     nthreads=1) -> int:
    """MoveMarkers.jl:15-69; mutates x_m, y_m; returns the failsafe count."""
    nf = _i64(0)
    lib().orc_move_markers_rk4(_p(x_m), _p(y_m), x_m.size, _p(Vx), Vx.shape[0], Vx.shape[1], _p(Vy),
                               Vy.shape[0], Vy.shape[1], x_vx_min, y_vx_min, x_vy_min, y_vy_min, dt, lx,
                               ly, dx, dy, nthreads, C.byref(nf))
    return nf.value


# --------------------------------------------------------------------------
# StokesFlow2D_multixpu.jl driver (single rank, no I/O)
# --------------------------------------------------------------------------
def node_origins(dx, dy):
    """First coordinates of the staggered node sets, StokesFlow2D_multixpu.jl:117-126."""
    return dict(
        x=0.0, y=0.0,                      # basic nodes  x[1], y[1]
        x_p=0.0 * dx + 0.5 * dx, y_p=0.0 * dy + 0.5 * dy,
        x_vx=(1 - 2) * dx, y_vx=0.0 * dy - 0.5 * dy,
        x_vy=0.0 * dx - 0.5 * dx, y_vy=(1 - 2) * dy,
        x_rho=0.0 * dx - 0.5 * dx, y_rho=(2 - 2) * dy)


def stokes_flow_2d(Nt, Nx, Ny, Lx, Ly, model: PlumeModel, marker_density=5, stokes_eps=1e-5,
                   jitter=0.0, seed=0, g_y=9.81, maxdisp=0.5, iter_max=100000, nthreads=1,
                   return_state=False):
    """StokesFlow2D_multixpu.jl:55-235 on one rank without plotting or saving.
    Returns (Vx_pad, Vy_pad, t_tot[, state])."""
    dx = Lx / (Nx - 1)
    dy = Ly / (Ny - 1)
    lx = (Nx - 1) * dx
    ly = (Ny - 1) * dy
    a = stokes_arrays(Nx, Ny)
    interp = (max(Nx + 1, Nx, Nx - 1), max(Ny, Ny, Ny - 1))
    val_wt_sum = zeros(*interp)
    wt_sum = zeros(*interp)
    o = node_origins(dx, dy)
    x_m, y_m = initialize_markers(marker_density, lx, ly, dx, dy, Nx, Ny, jitter, seed)
    rho_m, mu_m = set_marker_properties(model, x_m, y_m)
    dt = 0.0
    t_tot = 0.0
    iters = []
    for _ in range(Nt):
        bilinear_marker_to_grid(o["x_rho"], o["y_rho"], a["rho_vy"], x_m, y_m, rho_m, dx, dy, val_wt_sum, wt_sum)
        bilinear_marker_to_grid(o["x"], o["y"], a["mu_b"], x_m, y_m, mu_m, dx, dy, val_wt_sum, wt_sum)
        bilinear_marker_to_grid(o["x_p"], o["y_p"], a["mu_p"], x_m, y_m, mu_m, dx, dy, val_wt_sum, wt_sum)
        r = solve_stokes(a, g_y, dx, dy, Nx, Ny, dt, maxdisp, True, stokes_eps, iter_max, nthreads)
        dt = r.dt
        iters.append(r.iters)
        move_markers_rk4(x_m, y_m, a["Vx"], a["Vy"], o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, lx, ly,
                         dx, dy, nthreads)
        t_tot += dt
    if return_state:
        return a["Vx"], a["Vy"], t_tot, dict(arrays=a, x_m=x_m, y_m=y_m, rho_m=rho_m, mu_m=mu_m, iters=iters)
    return a["Vx"], a["Vy"], t_tot


# --------------------------------------------------------------------------
# decomposed run: the pieces that cross ranks (numpy restatements)
# --------------------------------------------------------------------------
def sum_overlapping_values(arrays: dict, dims, Nx: int, Ny: int) -> None:
    """sumOverlappingValues!(A, grid) (scripts/MarkerToGrid.jl:183-269) on numpy arrays in the Julia shape,
    keyed by rank coordinates (cx, cy): the x exchange first (:223-246), then y (:249-266); every received
    block holds the neighbour's values from before that pass, added as own + received (A .+= recv)."""
    nx, ny = next(iter(arrays.values())).shape
    ox, oy = 2 + nx - Nx, 2 + ny - Ny
    assert 2 * ox <= nx and 2 * oy <= ny                                   # :199
    if ox > 0:
        recv = {}
        for (cx, cy) in arrays:
            left, right = arrays.get((cx - 1, cy)), arrays.get((cx + 1, cy))
            recv[(cx, cy)] = (None if left is None else left[nx - ox:, :].copy(),
                              None if right is None else right[:ox, :].copy())
        for c, A in arrays.items():
            lr, rl = recv[c]
            if lr is not None:
                A[:ox, :] += lr
            if rl is not None:
                A[nx - ox:, :] += rl
    if oy > 0:
        recv = {}
        for (cx, cy) in arrays:
            above, below = arrays.get((cx, cy - 1)), arrays.get((cx, cy + 1))   # nb[1,2] / nb[2,2]
            recv[(cx, cy)] = (None if above is None else above[:, ny - oy:].copy(),
                              None if below is None else below[:, :oy].copy())
        for c, A in arrays.items():
            down, up = recv[c]
            if down is not None:
                A[:, :oy] += down
            if up is not None:
                A[:, ny - oy:] += up


_SHIFT = {1: (-1, -1), 2: (0, -1), 3: (1, -1), 4: (1, 0), 5: (1, 1), 6: (0, 1), 7: (-1, 1), 8: (-1, 0)}


def _pos_to_neighbour_idx(x, y, lx, ly, hx, hy, cx, cy, dimx, dimy):
    """posToNeighbourIdx (scripts/MarkerExchange.jl:204-222), vectorised; the conditions in its order."""
    d = np.zeros(x.shape, dtype=np.int64)
    lo_y, hi_y = (y < hy) & (cy != 0), (y > ly - hy) & (cy != dimy - 1)
    lo_x, hi_x = (x < hx) & (cx != 0), (x > lx - hx) & (cx != dimx - 1)
    d = np.where(lo_y, np.where(lo_x, 1, np.where(hi_x, 3, 2)),
                 np.where(hi_y, np.where(lo_x, 7, np.where(hi_x, 5, 6)),
                          np.where(lo_x, 8, np.where(hi_x, 4, 0))))
    return d


def exchange_markers(markers: dict, dims, lx, ly, dx, dy) -> dict:
    """exchangeMarkers (scripts/MarkerExchange.jl:8-163) for every rank: markers {(cx, cy): (x, y, rho, mu)}
    -> the same after the exchange.  A rank keeps its inside markers in order (:60-76) and appends, for
    neighbour index i = 1..8, the markers that the rank opposite direction i (dstToSrcIdx, :198-202) sent
    in direction i, shifted by (lx - dx, ly - dy) times the step (:77-79), in the sender's order."""
    hx, hy = dx / 2, dy / 2
    dimx, dimy = dims
    kept, sent = {}, {}
    for (cx, cy), (x, y, r, m) in markers.items():
        d = _pos_to_neighbour_idx(x, y, lx, ly, hx, hy, cx, cy, dimx, dimy)
        k = d == 0
        kept[(cx, cy)] = (x[k], y[k], r[k], m[k])
        for i, (sx, sy) in _SHIFT.items():
            s = d == i
            sent[((cx, cy), i)] = (x[s] - (lx - dx) * sx, y[s] - (ly - dy) * sy, r[s], m[s])
    out = {}
    for (cx, cy) in markers:
        parts = [kept[(cx, cy)]]
        for i in range(1, 9):
            src_dir = i + 4 if i < 5 else (i + 4) % 9 + 1
            sx, sy = _SHIFT[src_dir]
            src = (cx + sx, cy + sy)
            if src in markers:
                parts.append(sent[(src, i)])
        out[(cx, cy)] = tuple(np.concatenate([p[q] for p in parts]) for q in range(4))
    return out


# --------------------------------------------------------------------------
# the StokesFlow2D timestep on a grid of ranks, composed from the pieces above
# --------------------------------------------------------------------------
# entries of each array beyond the rank's Nx x Ny grid (StokesFlow2D_multixpu.jl:89-109)
_RANK_ARRAY_EXTRA = {"rho_vy": (1, 0), "mu_b": (0, 0), "mu_p": (-1, -1), "Vx": (2, 1), "Vy": (1, 2)}


def rank_slices(name, coord, Nx, Ny):
    """The global index range of a rank's array: ImplicitGlobalGrid with overlap 2 puts local point i of the
    rank at coordinate c at global point c (N - 2) + i, in every array."""
    sx, sy = _RANK_ARRAY_EXTRA[name]
    x0, y0 = coord[0] * (Nx - 2), coord[1] * (Ny - 2)
    return slice(x0, x0 + Nx + sx), slice(y0, y0 + Ny + sy)


def rank_markers(dims, Nx, Ny, Lx, Ly, model: PlumeModel, marker_density, jitter=0.0, seed=0):
    """initializeMarkersCPU + setInitialMarkerProperties! on every rank (StokesFlow2D_multixpu.jl:135-136):
    {(cx, cy): (x, y, rho, mu)} in local coordinates; jitter with an odd density is followed by the exchange
    (common.jl:93-97) before the properties are set; the jitter seed of a rank is seed + its MPI rank."""
    nx_g, ny_g = dims[0] * (Nx - 2) + 2, dims[1] * (Ny - 2) + 2
    dx, dy = Lx / (nx_g - 1), Ly / (ny_g - 1)
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    out = {}
    for cx in range(dims[0]):
        for cy in range(dims[1]):
            x, y = initialize_markers_rank(marker_density, lx, ly, dx, dy, Nx, Ny, (cx, cy), dims, jitter,
                                           seed + cx * dims[1] + cy)
            out[(cx, cy)] = (x, y, np.zeros_like(x), np.zeros_like(x))
    if jitter != 0.0 and marker_density % 2 == 1:
        out = exchange_markers(out, dims, lx, ly, dx, dy)
    for (cx, cy), (x, y, _, _) in out.items():
        rho, mu = set_marker_properties(model, x, y, cx * (Nx - 2) * dx, cy * (Ny - 2) * dy)
        out[(cx, cy)] = (x, y, rho, mu)
    return out


def stokes_flow_2d_ranks(Nt, dims, Nx, Ny, Lx, Ly, markers: dict, stokes_eps=1e-5, iter_max=100000, g_y=9.81,
                         maxdisp=0.5, nthreads=1):
    """StokesFlow2D_multixpu.jl:157-191 on dims[0] x dims[1] ranks of Nx x Ny local points, from oracle pieces:
    per-rank deposits onto the (Nx+1, Ny) interpolation arrays, sumOverlappingValues!, safeDivision; the solve
    on the global grid (the decomposed PT iterate is the global one; the stopping test uses the one-rank err,
    which only moves the stopping iteration); per-rank RK4 on the local slices of V; exchangeMarkers.
    markers: {(cx, cy): (x, y, rho, mu)} in local coordinates (rank_markers).  Returns (Vx_glob, Vy_glob,
    t_tot, markers, dts) with V as gather_V_grid hands it back."""
    nx_g, ny_g = dims[0] * (Nx - 2) + 2, dims[1] * (Ny - 2) + 2
    dx, dy = Lx / (nx_g - 1), Ly / (ny_g - 1)
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    o = node_origins(dx, dy)
    a = stokes_arrays(nx_g, ny_g)
    grids = {c: {n: zeros(Nx + s[0], Ny + s[1]) for n, s in _RANK_ARRAY_EXTRA.items() if n not in ("Vx", "Vy")}
             for c in markers}
    markers = {c: tuple(v.copy() for v in m) for c, m in markers.items()}
    dt, t_tot, dts = 0.0, 0.0, []
    for _ in range(Nt):
        for name, (xo, yo), q in (("rho_vy", ("x_rho", "y_rho"), 2), ("mu_b", ("x", "y"), 3),
                                  ("mu_p", ("x_p", "y_p"), 3)):                    # :164-166
            vws = {c: zeros(Nx + 1, Ny) for c in markers}
            ws = {c: zeros(Nx + 1, Ny) for c in markers}
            for c, m in markers.items():
                bilinear_marker_to_grid(o[xo], o[yo], grids[c][name], m[0], m[1], m[q], dx, dy, vws[c], ws[c])
            sum_overlapping_values(ws, dims, Nx, Ny)
            sum_overlapping_values(vws, dims, Nx, Ny)
            for c in markers:                                                     # safeDivision
                g = grids[c][name]
                nxv, nyv = g.shape
                nz = ws[c][:nxv, :nyv] != 0
                g[nz] = vws[c][:nxv, :nyv][nz] / ws[c][:nxv, :nyv][nz]
                xs, ys = rank_slices(name, c, Nx, Ny)
                a[name][xs, ys] = g
        r = solve_stokes(a, g_y, dx, dy, nx_g, ny_g, dt, maxdisp, True, stokes_eps, iter_max, nthreads)
        dt = r.dt
        dts.append(dt)
        for c, m in markers.items():                                              # :181, local domain
            xs, ys = rank_slices("Vx", c, Nx, Ny)
            vx = np.asfortranarray(a["Vx"][xs, ys])
            xs, ys = rank_slices("Vy", c, Nx, Ny)
            vy = np.asfortranarray(a["Vy"][xs, ys])
            move_markers_rk4(m[0], m[1], vx, vy, o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, lx, ly, dx, dy,
                             nthreads)
        markers = exchange_markers(markers, dims, lx, ly, dx, dy)                # :186-191
        t_tot += dt
    return a["Vx"], a["Vy"], t_tot, markers, dts
