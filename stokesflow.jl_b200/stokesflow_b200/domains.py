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
