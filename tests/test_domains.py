"""Domain decomposition of the PT solve (sf_solve_stokes_decomposed): the ImplicitGlobalGrid index
arithmetic on the CPU, and on the GPU the decomposed iterate against the single-domain one, bit for bit,
with every rank's local arrays (halos and overlaps included) equal to the slices of the global result."""
import numpy as np
import pytest
import torch

from fields import random_fields
from stokesflow_b200 import domains


def test_sizes_and_slices_tile_the_global_grid():
    for dims, n_local in ((1, 10), (2, 34), (3, 18), (4, 6)):
        n_g = domains.global_size(dims, n_local)
        assert domains.local_size(dims, n_g) == n_local
    with pytest.raises(ValueError):
        domains.local_size(3, 66)            # 64 does not split in 3
    Nx, Ny, dims = 6, 5, (3, 2)
    nx_g, ny_g = domains.global_size(dims[0], Nx), domains.global_size(dims[1], Ny)
    for name, (sx, sy) in domains.ARRAYS.items():
        cover = np.zeros((nx_g + sx, ny_g + sy), dtype=int)
        for cy in range(dims[1]):
            for cx in range(dims[0]):
                xs, ys = domains.local_slices(name, (cx, cy), Nx, Ny)
                assert xs.stop - xs.start == Nx + sx and ys.stop - ys.start == Ny + sy
                cover[xs, ys] += 1
        assert cover.min() >= 1, name               # every global entry is held by some rank
        assert cover[-1, -1] == 1 and cover[0, 0] == 1


def test_split_keeps_the_overlap_consistent():
    Nx, Ny, dims = 8, 6, (2, 2)
    nx_g, ny_g = domains.global_size(2, Nx), domains.global_size(2, Ny)
    g = torch.arange(float(nx_g * (ny_g + 1)), dtype=torch.float64).reshape(ny_g + 1, nx_g).t()   # Vx_s layout
    loc = domains.split({"Vx_s": g}, dims, Nx, Ny)
    a, b = loc[(0, 0)]["Vx_s"], loc[(1, 0)]["Vx_s"]
    assert a.stride() == (1, a.shape[0])
    whole = domains.split({"Vx_s": g}, (1, 1), nx_g, ny_g)[(0, 0)]["Vx_s"]
    assert torch.equal(whole, g) and whole.data_ptr() != g.data_ptr()   # a copy, never a view
    assert torch.equal(a[-2:, :], b[:2, :])         # the two overlapping x planes
    c = loc[(0, 1)]["Vx_s"]
    assert torch.equal(a[:, -3:], c[:, :3])         # Vx_s is one entry longer in y: three planes overlap


def test_gather_inverts_split():
    """With consistent overlaps (as after update_halo!) the gathered array is the global one, for every
    staggering; the kept ranges tile each dimension without gaps."""
    Nx, Ny, dims = 7, 6, (3, 2)
    nx_g, ny_g = domains.global_size(dims[0], Nx), domains.global_size(dims[1], Ny)
    g = {}
    for name, (sx, sy) in domains.ARRAYS.items():
        g[name] = torch.randn(ny_g + sy, nx_g + sx, dtype=torch.float64).t()
    loc = domains.split(g, dims, Nx, Ny)
    for name in domains.ARRAYS:
        assert torch.equal(domains.gather(loc, name, dims, Nx, Ny), g[name]), name


def test_gather_markers_order_and_shift():
    dims, lx, ly, dx, dy = (2, 2), 1.0, 0.5, 0.25, 0.125
    mk = {}
    for cx in range(2):
        for cy in range(2):
            base = 10 * cx + cy
            mk[(cx, cy)] = (torch.tensor([0.1, 0.2], dtype=torch.float64), torch.tensor([0.3, 0.4], dtype=torch.float64),
                            torch.tensor([base, base], dtype=torch.float64), torch.tensor([1.0, 2.0], dtype=torch.float64))
    x, y, r, m = domains.gather_markers(mk, dims, lx, ly, dx, dy)
    assert r.tolist() == [0, 0, 1, 1, 10, 10, 11, 11]          # rank order: x coordinate slowest
    assert x.tolist()[4:6] == [0.1 + 1 * (lx - dx), 0.2 + 1 * (lx - dx)]
    assert y.tolist()[2:4] == [0.3 + 1 * (ly - dy), 0.4 + 1 * (ly - dy)]


def _global_problem(sf, nx_g, ny_g, seed=4):
    rho, mub, mup = random_fields(nx_g, ny_g, seed=seed, contrast=10.0)
    rng = np.random.default_rng(seed + 1)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda().t()  # noqa: E731
    z = sf.zeros
    g = {"rho_vy": dev(rho), "mu_b": dev(mub), "mu_p": dev(mup), "P": dev(1e-3 * rng.standard_normal((nx_g - 1, ny_g - 1))),
         "Vx_s": dev(1e-3 * rng.standard_normal((nx_g, ny_g + 1))), "Vy_s": dev(1e-3 * rng.standard_normal((nx_g + 1, ny_g))),
         "dVxdt": z(nx_g - 2, ny_g - 1), "dVydt": z(nx_g - 1, ny_g - 2), "Vx_pad": z(nx_g + 2, ny_g + 1),
         "Vy_pad": z(nx_g + 1, ny_g + 2)}
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(1, 1), (2, 1), (2, 2), (3, 2)])
def test_decomposed_solve_is_the_global_solve(sf, dims):
    nx_g, ny_g = 74, 50
    Nx, Ny = domains.local_size(dims[0], nx_g), domains.local_size(dims[1], ny_g)
    g = _global_problem(sf, nx_g, ny_g)
    ranks = domains.split(g, dims, Nx, Ny)          # copies of the initial state
    dx, dy = 1.0 / (nx_g - 1), 1.0 / (ny_g - 1)
    iters = 600                                      # checks at 250 and 500, a dt update at 500
    info = sf.solve_stokes_info(g["P"], g["Vx_pad"], g["Vy_pad"], g["rho_vy"], g["mu_b"], g["mu_p"], None, None, None,
                                None, None, None, None, g["dVxdt"], g["dVydt"], None, None, g["Vx_s"], g["Vy_s"], 9.81,
                                dx, dy, nx_g, ny_g, 1e-4, 0.5, eps=1e-300, iter_max=iters)
    dinfo = domains.solve_stokes_decomposed(ranks, dims, Nx, Ny, 9.81, dx, dy, 1e-4, 0.5, eps=1e-300, iter_max=iters)
    torch.cuda.synchronize()
    assert dinfo["iters"] == info["iters"] == iters and dinfo["n_checks"] == info["n_checks"] == 2
    assert dinfo["dt"] == info["dt"]
    if dims == (1, 1):
        assert dinfo["err"] == info["err"]
    else:   # the reference's multi-rank err averages per-rank means: close, not equal
        assert abs(dinfo["err"] - info["err"]) <= 0.5 * info["err"]
    for coord, loc in ranks.items():
        for name in domains.ARRAYS:
            xs, ys = domains.local_slices(name, coord, Nx, Ny)
            assert torch.equal(loc[name], g[name][xs, ys]), f"rank {coord} {name}"
    for name in ("Vx_pad", "Vy_pad", "P"):   # what gather_V_grid hands back
        assert torch.equal(domains.gather(ranks, name, dims, Nx, Ny), g[name]), name


# test/test_StokesSolver.jl:17-41: the 26 x 32-point global grid on 1 to 4 ranks
SOLVER_GRIDS = [((1, 2), 26, 17), ((2, 1), 14, 32), ((1, 3), 26, 12), ((3, 1), 10, 32), ((4, 1), 8, 32),
                ((2, 2), 14, 17)]


@pytest.mark.gpu
@pytest.mark.parametrize("dims,Nx,Ny", SOLVER_GRIDS)
def test_decomposed_solve_meets_the_solver_golden_values(sf, dims, Nx, Ny):
    """test/test_StokesSolver.jl:48-140 on the reference's rank grids, through the decomposed solve (halo updates,
    the multi-rank err and dt): the gathered velocities match the reference's golden values as its `≈` does
    (norm-relative sqrt(eps)), and the free-slip / mirror identities of the padded arrays hold exactly."""
    from fields import golden, solver_test_fields
    g = golden()["stokes_solver"]
    nx_g, ny_g, dx, dy = g["Nx"], g["Ny"], g["dx"], g["dy"]
    assert (domains.global_size(dims[0], Nx), domains.global_size(dims[1], Ny)) == (nx_g, ny_g)
    rho, mub, mup = solver_test_fields(nx_g, ny_g, dx, dy)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda().t()  # noqa: E731
    z = sf.zeros
    glob = {"rho_vy": dev(rho), "mu_b": dev(mub), "mu_p": dev(mup), "P": z(nx_g - 1, ny_g - 1),
            "Vx_s": z(nx_g, ny_g + 1), "Vy_s": z(nx_g + 1, ny_g), "dVxdt": z(nx_g - 2, ny_g - 1),
            "dVydt": z(nx_g - 1, ny_g - 2), "Vx_pad": z(nx_g + 2, ny_g + 1), "Vy_pad": z(nx_g + 1, ny_g + 2)}
    ranks = domains.split(glob, dims, Nx, Ny)
    info = domains.solve_stokes_decomposed(ranks, dims, Nx, Ny, g["g_y"], dx, dy, 0.0, g["maxdisp"], eps=g["eps"],
                                           iter_max=100000)
    assert info["converged"] == 1
    vx = domains.gather(ranks, "Vx_pad", dims, Nx, Ny).cpu().numpy()
    vy = domains.gather(ranks, "Vy_pad", dims, Nx, Ny).cpu().numpy()
    inds = np.array(g["inds"]) - 1
    tol = np.sqrt(np.finfo(np.float64).eps)
    for got, ref in ((vx.ravel(order="F")[inds], np.array(g["vx_ref"])), (vy.ravel(order="F")[inds], np.array(g["vy_ref"]))):
        assert np.linalg.norm(got - ref) <= tol * max(np.linalg.norm(got), np.linalg.norm(ref))
    assert np.array_equal(vx[0], -vx[2]) and np.all(vx[1] == 0) and np.array_equal(vx[-1], -vx[-3]) and np.all(vx[-2] == 0)
    assert np.array_equal(vx[:, 0], vx[:, 1]) and np.array_equal(vx[:, -1], vx[:, -2])
    assert np.array_equal(vy[:, 0], -vy[:, 2]) and np.all(vy[:, 1] == 0) and np.array_equal(vy[:, -1], -vy[:, -3])
    assert np.all(vy[:, -2] == 0) and np.array_equal(vy[0], vy[1]) and np.array_equal(vy[-1], vy[-2])
