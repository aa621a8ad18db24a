"""The rest of a decomposed timestep: sumOverlappingValues!, the decomposed deposit (MarkerToGrid.jl:18-38
with :183-269) and exchangeMarkers (MarkerExchange.jl:8-163).  The numpy restatements in the oracle are pinned
by known answers on the CPU; the device versions must match them bit for bit on the GPU."""
import numpy as np
import pytest
import torch

import oracle
from stokesflow_b200 import domains


def ones_ranks(dims, nx, ny):
    return {(cx, cy): np.ones((nx, ny), order="F") for cx in range(dims[0]) for cy in range(dims[1])}


def test_oracle_overlap_sum_known_answer():
    Nx, Ny, dims = 8, 6, (2, 2)
    a = ones_ranks(dims, Nx + 1, Ny)           # the (Nx+1, Ny) interpolation arrays: ox = 3, oy = 2
    oracle.sum_overlapping_values(a, dims, Nx, Ny)
    r00 = a[(0, 0)]
    assert np.all(r00[:Nx + 1 - 3, :Ny - 2] == 1)        # own interior
    assert np.all(r00[Nx + 1 - 3:, :Ny - 2] == 2)        # shared with the right neighbour
    assert np.all(r00[:Nx + 1 - 3, Ny - 2:] == 2)        # shared with the neighbour below
    assert np.all(r00[Nx + 1 - 3:, Ny - 2:] == 4)        # the corner: all four
    r11 = a[(1, 1)]
    assert np.all(r11[:3, :2] == 4) and np.all(r11[3:, 2:] == 1)


def test_oracle_exchange_known_answer():
    lx, ly, dx, dy, dims = 1.0, 0.5, 0.125, 0.0625, (2, 1)
    f = lambda *v: np.array(v, dtype=np.float64)  # noqa: E731
    markers = {(0, 0): (f(0.5, 0.99, 0.95, 0.01), f(0.2, 0.2, 0.3, 0.2), f(1, 2, 3, 4), f(5, 6, 7, 8)),
               (1, 0): (f(0.5, 0.02, 0.99), f(0.1, 0.3, 0.1), f(9, 10, 11), f(12, 13, 14))}
    out = oracle.exchange_markers(markers, dims, lx, ly, dx, dy)
    x0, y0, r0, m0 = out[(0, 0)]
    x1, y1, r1, m1 = out[(1, 0)]
    # rank 0 keeps 0.5, 0.01 (x < dx/2 but it is the physical boundary); 0.99 and 0.95 (> lx - dx/2) go right
    assert r0.tolist() == [1, 4, 10] and x0[-1] == 0.02 + (lx - dx)
    # rank 1 keeps 0.5 and 0.99 (the physical boundary), then receives rank 0's two, shifted left by lx - dx
    assert r1.tolist() == [9, 11, 2, 3] and x1[2] == 0.99 - (lx - dx) and x1[3] == 0.95 - (lx - dx)
    assert y1.tolist()[2:] == [0.2, 0.3]


def random_rank_markers(dims, lx, ly, n, seed):
    rng = np.random.default_rng(seed)
    out = {}
    for cx in range(dims[0]):
        for cy in range(dims[1]):
            # many near the edges, some far inside, a few at the corners
            x = np.concatenate([rng.uniform(0, lx, n), rng.uniform(0, 0.1, n // 4) * lx, lx - rng.uniform(0, 0.1, n // 4) * lx])
            y = np.concatenate([rng.uniform(0, ly, n), ly - rng.uniform(0, 0.1, n // 4) * ly, rng.uniform(0, 0.1, n // 4) * ly])
            k = len(x)
            out[(cx, cy)] = (x, y, rng.uniform(0.5, 1.5, k), rng.uniform(0.01, 1, k))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(2, 1), (3, 2)])
def test_exchange_matches_oracle(sf, dims):
    lx, ly, dx, dy = 1.0, 0.75, 1 / 32, 1 / 24
    mk = random_rank_markers(dims, lx, ly, 20000, 3)
    ctxs = {c: sf.Context() for c in mk}
    dev = {c: tuple(torch.from_numpy(a).cuda() for a in v) for c, v in mk.items()}
    got = domains.exchange_markers(dev, dims, lx, ly, dx, dy, ctxs)
    ref = oracle.exchange_markers(mk, dims, lx, ly, dx, dy)
    moved = 0
    for c in mk:
        for q in range(4):
            assert np.array_equal(got[c][q].cpu().numpy(), ref[c][q]), (c, q)
        moved += abs(len(ref[c][0]) - len(mk[c][0]))
    assert moved > 0
    assert sum(len(v[0]) for v in ref.values()) == sum(len(v[0]) for v in mk.values())   # none lost


@pytest.mark.gpu
def test_overlap_sum_and_decomposed_deposit_match_oracle(sf):
    dims, Nx, Ny = (3, 2), 20, 14
    dx, dy = 1 / ((Nx - 2) * dims[0] + 1), 1 / ((Ny - 2) * dims[1] + 1)
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    rng = np.random.default_rng(5)
    arrs = {(cx, cy): np.asfortranarray(rng.standard_normal((Nx + 1, Ny))) for cx in range(3) for cy in range(2)}
    ctxs = {c: sf.Context() for c in arrs}
    dev = {c: torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t() for c, a in arrs.items()}
    domains.sum_overlapping_values(dev, dims, Nx, Ny, ctxs)
    oracle.sum_overlapping_values(arrs, dims, Nx, Ny)
    for c in arrs:
        assert np.array_equal(dev[c].cpu().numpy(), arrs[c]), c
    # the decomposed deposit of rho onto rho_vy (origin (-dx/2, 0)), from markers in each rank's local domain
    mk = random_rank_markers(dims, lx, ly, 3000, 8)
    o = oracle.node_origins(dx, dy)
    prev = {c: np.asfortranarray(rng.uniform(2, 3, (Nx + 1, Ny))) for c in mk}   # what an empty node keeps
    grids = {c: torch.from_numpy(np.ascontiguousarray(p.T)).cuda().t() for c, p in prev.items()}
    dmk = {c: (torch.from_numpy(v[0]).cuda(), torch.from_numpy(v[1]).cuda(), torch.from_numpy(v[2]).cuda()) for c, v in mk.items()}
    domains.deposit_decomposed(o["x_rho"], o["y_rho"], grids, dmk, dx, dy, dims, Nx, Ny, ctxs)
    torch.cuda.synchronize()
    # oracle: each rank's sums (its own deposit), overlap sums, safeDivision keeping the previous value
    vws, ws = {}, {}
    for c, (x, y, r, m) in mk.items():
        g = prev[c].copy(order="F")
        vws[c], ws[c] = oracle.zeros(Nx + 1, Ny), oracle.zeros(Nx + 1, Ny)
        oracle.bilinear_marker_to_grid(o["x_rho"], o["y_rho"], g, x, y, r, dx, dy, vws[c], ws[c])
    oracle.sum_overlapping_values(ws, dims, Nx, Ny)
    oracle.sum_overlapping_values(vws, dims, Nx, Ny)
    for c in mk:
        expect = prev[c].copy(order="F")
        nz = ws[c] != 0
        expect[nz] = vws[c][nz] / ws[c][nz]
        assert np.array_equal(grids[c].cpu().numpy(), expect), c


def _initial_markers(dims, Nx, Ny, dx, dy, per_rank, seed):
    """Seeded markers of every rank inside its own part of the domain (half a cell clear of the edges shared
    with a neighbour, as the reference's layout keeps them), with smooth rho / mu of the global position."""
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    rng = np.random.default_rng(seed)
    out = {}
    for cx in range(dims[0]):
        for cy in range(dims[1]):
            x0 = 0.0 if cx == 0 else dx / 2 + 1e-9
            x1 = lx if cx == dims[0] - 1 else lx - dx / 2 - 1e-9
            y0 = 0.0 if cy == 0 else dy / 2 + 1e-9
            y1 = ly if cy == dims[1] - 1 else ly - dy / 2 - 1e-9
            x, y = rng.uniform(x0, x1, per_rank), rng.uniform(y0, y1, per_rank)
            gx, gy = x + cx * (lx - dx), y + cy * (ly - dy)
            rho = 1.0 + 0.1 * np.sin(3 * gx) * np.cos(2 * gy)
            mu = np.exp(np.sin(2 * gx + gy))
            out[(cx, cy)] = (x, y, rho, mu)
    return out


def _oracle_decomposed_steps(mk, dims, Nx, Ny, Lx, Ly, steps, iters):
    """The decomposed timestep from oracle pieces (oracle.stokes_flow_2d_ranks), a fixed iteration count."""
    vx, vy, _, markers, dts = oracle.stokes_flow_2d_ranks(steps, dims, Nx, Ny, Lx, Ly, mk, stokes_eps=1e-300,
                                                          iter_max=iters, nthreads=4)
    return markers, {"Vx": vx, "Vy": vy}, dts


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(2, 1), (2, 2)])
def test_decomposed_timesteps_match_oracle(sf, dims):
    Nx, Ny, Lx, Ly, steps, iters = 18, 14, 1.0, 0.8, 2, 600
    nx_g, ny_g = domains.global_size(dims[0], Nx), domains.global_size(dims[1], Ny)
    dx, dy = Lx / (nx_g - 1), Ly / (ny_g - 1)
    mk = _initial_markers(dims, Nx, Ny, dx, dy, 2500, 11)
    st = domains.DecomposedStokesFlow2D(dims, Nx, Ny, Lx, Ly, {c: tuple(torch.from_numpy(v) for v in m) for c, m in mk.items()},
                                        eps=1e-300, iter_max=iters)
    dts = [st.step()["dt"] for _ in range(steps)]
    ref_markers, ref_a, ref_dts = _oracle_decomposed_steps(mk, dims, Nx, Ny, Lx, Ly, steps, iters)
    assert dts == ref_dts
    vx, vy = st.velocities()
    assert np.array_equal(vx.cpu().numpy(), ref_a["Vx"]) and np.array_equal(vy.cpu().numpy(), ref_a["Vy"])
    for c in mk:
        for q in range(4):
            assert np.array_equal(st.markers[c][q].cpu().numpy(), ref_markers[c][q]), (c, q)
    moved = sum(abs(len(ref_markers[c][0]) - len(mk[c][0])) for c in mk)
    assert moved > 0          # markers did cross between ranks


def test_reference_marker_to_grid_multi_process():
    """test/test_MarkerToGrid.jl:43-148 (TEST 2) as the reference runs it: 2 x 2 ranks of 10 x 8 points, 25
    random markers per cell in each rank's own part of the domain, deposited per rank onto three grids (origins
    (dx/2, dy/2), (0, 0), (-dx/2, 0)) with sumOverlappingValues! on the (Nx+1, Ny) sums and safeDivision,
    gathered as create_grid_view does; a one-process deposit of the gathered markers onto the global grids
    agrees elementwise at isapprox's default tolerance."""
    dims, Nx, Ny, dx, dy = (2, 2), 10, 8, 0.3, 0.4
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    origins = {"mu_p": (0.5 * dx, 0.5 * dy), "mu_b": (0.0, 0.0), "rho_vy": (-0.5 * dx, 0.0)}   # grid1..3, :62-67
    rng = np.random.default_rng(2)
    nm = 25 * (Nx - 1) * (Ny - 1)
    markers = {}
    for cx in range(2):
        for cy in range(2):
            rank = cx * 2 + cy
            x = rng.random(nm) * (lx - 0.5 * dx) + (0.5 * dx if cx > 0 else 0.0)      # :75-77
            y = rng.random(nm) * (ly - 0.5 * dy) + (0.5 * dy if cy > 0 else 0.0)
            markers[(cx, cy)] = (x, y, rng.random(nm) + 2 * (rank + 1))
    local = {}
    for name, (gx, gy) in origins.items():
        sx, sy = domains.ARRAYS[name]
        grids = {c: oracle.zeros(Nx + sx, Ny + sy) for c in markers}
        vws = {c: oracle.zeros(Nx + 1, Ny) for c in markers}
        ws = {c: oracle.zeros(Nx + 1, Ny) for c in markers}
        for c, (x, y, v) in markers.items():
            oracle.bilinear_marker_to_grid(gx, gy, grids[c], x, y, v, dx, dy, vws[c], ws[c])
        oracle.sum_overlapping_values(ws, dims, Nx, Ny)
        oracle.sum_overlapping_values(vws, dims, Nx, Ny)
        for c in markers:
            g = grids[c]
            nz = ws[c][:g.shape[0], :g.shape[1]] != 0
            g[nz] = vws[c][:g.shape[0], :g.shape[1]][nz] / ws[c][:g.shape[0], :g.shape[1]][nz]
        local[name] = {c: {name: torch.from_numpy(np.ascontiguousarray(g))} for c, g in grids.items()}
    # gather_markers! (:88) and the one-process deposit (:119-138)
    xg, yg, vg, _ = (t.numpy() for t in domains.gather_markers(
        {c: tuple(torch.from_numpy(a) for a in (x, y, v, v)) for c, (x, y, v) in markers.items()}, dims, lx, ly, dx,
        dy))
    nxg, nyg = domains.global_size(2, Nx), domains.global_size(2, Ny)
    assert (nxg, nyg) == (18, 14)
    tol = np.sqrt(np.finfo(np.float64).eps)
    for name, (gx, gy) in origins.items():
        sx, sy = domains.ARRAYS[name]
        single = oracle.zeros(nxg + sx, nyg + sy)
        vws, ws = oracle.zeros(nxg + 1, nyg), oracle.zeros(nxg + 1, nyg)
        oracle.bilinear_marker_to_grid(gx, gy, single, xg, yg, vg, dx, dy, vws, ws)
        multi = domains.gather(local[name], name, dims, Nx, Ny).numpy()
        assert multi.shape == single.shape
        assert np.all(np.abs(multi - single) <= tol * np.maximum(np.abs(multi), np.abs(single))), name   # :141-143


@pytest.mark.parametrize("dims, n_dev", [((3, 2), 4), ((2, 2), 2), ((1, 3), 8), ((4, 4), 8), ((5, 3), 4)])
def test_rank_devices_are_contiguous_balanced_runs(dims, n_dev):
    """The rank -> GPU assignment of the decomposition: contiguous runs in MPI rank order (x slowest), run
    lengths differing by at most one, every GPU used when there are at least as many ranks, one rank per GPU
    otherwise, and the same answer every time."""
    from stokesflow_b200.domains import rank_devices
    a = rank_devices(dims, n_dev)
    assert a == rank_devices(dims, n_dev)
    order = [a[(cx, cy)] for cx in range(dims[0]) for cy in range(dims[1])]   # MPI rank order
    n = dims[0] * dims[1]
    assert order == sorted(order) and all(0 <= d < n_dev for d in order)
    sizes = [order.count(d) for d in sorted(set(order))]
    assert max(sizes) - min(sizes) <= 1
    assert len(set(order)) == min(n, n_dev)
