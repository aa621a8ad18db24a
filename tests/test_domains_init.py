"""initializeMarkersCPU on a grid of ranks (common.jl:40-97) and setInitialMarkerProperties! at the ranks'
global offsets (common.jl:104-110, StokesFlow2D_multixpu.jl:80-81, 135-136).

CPU: the oracle's rank layouts tile the one-domain layout of the global grid (counts and positions), and the
library's host-side counts agree with the oracle.  GPU: each rank's markers and properties are bit-identical
to the oracle's, including the exchange that follows jitter with an odd density."""
import numpy as np
import pytest
import torch

import oracle
from stokesflow_b200 import domains
from stokesflow_b200._lib import StokesFlowError

DIMS = [(1, 1), (2, 1), (1, 2), (2, 2), (3, 2)]


def geometry(dims, Nx, Ny, Lx=1.0, Ly=1.3):
    dx = Lx / (domains.global_size(dims[0], Nx) - 1)
    dy = Ly / (domains.global_size(dims[1], Ny) - 1)
    return dx, dy, (Nx - 1) * dx, (Ny - 1) * dy


def coords_of(dims):
    return [(cx, cy) for cx in range(dims[0]) for cy in range(dims[1])]


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("md", [1, 2, 3, 4, 5])
def test_rank_counts_tile_the_global_count(dims, md):
    Nx, Ny = 11, 9
    gx, gy = oracle.marker_counts(md, domains.global_size(dims[0], Nx), domains.global_size(dims[1], Ny))
    assert sum(oracle.marker_counts_rank(md, Nx, Ny, (cx, 0), dims)[0] for cx in range(dims[0])) == gx
    assert sum(oracle.marker_counts_rank(md, Nx, Ny, (0, cy), dims)[1] for cy in range(dims[1])) == gy
    for c in coords_of(dims):                                   # the library's host-side count agrees
        assert domains.marker_count_rank(md, Nx, Ny, c, dims) == oracle.marker_counts_rank(md, Nx, Ny, c, dims)


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("md", [2, 3, 4, 5])
def test_rank_layouts_tile_the_global_layout(dims, md):
    """Without jitter, the ranks' markers moved by the offsets x0 = cx (Nx - 2) dx are the global lattice."""
    Nx, Ny = 10, 8
    dx, dy, lx, ly = geometry(dims, Nx, Ny)
    xs, ys = [], []
    for cx, cy in coords_of(dims):
        x, y = oracle.initialize_markers_rank(md, lx, ly, dx, dy, Nx, Ny, (cx, cy), dims)
        xs.append(x + cx * (Nx - 2) * dx)
        ys.append(y + cy * (Ny - 2) * dy)
    x, y = np.concatenate(xs), np.concatenate(ys)
    nxg, nyg = domains.global_size(dims[0], Nx), domains.global_size(dims[1], Ny)
    xg, yg = oracle.initialize_markers(md, (nxg - 1) * dx, (nyg - 1) * dy, dx, dy, nxg, nyg)
    assert x.size == xg.size
    order = np.lexsort((np.round(y / dy * md * 4), np.round(x / dx * md * 4)))
    order_g = np.lexsort((np.round(yg / dy * md * 4), np.round(xg / dx * md * 4)))
    assert np.allclose(x[order], xg[order_g], rtol=0, atol=1e-12)
    assert np.allclose(y[order], yg[order_g], rtol=0, atol=1e-12)


def test_one_rank_is_the_one_domain_layout():
    dx, dy, lx, ly = geometry((1, 1), 17, 13)
    a = oracle.initialize_markers_rank(3, lx, ly, dx, dy, 17, 13, (0, 0), (1, 1), 0.5, 11)
    b = oracle.initialize_markers(3, lx, ly, dx, dy, 17, 13, 0.5, 11)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_rank_count_rejects_bad_coords():
    with pytest.raises(StokesFlowError):
        domains.marker_count_rank(4, 10, 10, (2, 0), (2, 1))
    with pytest.raises(StokesFlowError):
        domains.marker_count_rank(4, 10, 10, (0, 0), (0, 1))


def oracle_rank_markers(dims, Nx, Ny, Lx, Ly, md, jitter, seed, model):
    dx, dy, lx, ly = geometry(dims, Nx, Ny, Lx, Ly)
    out = {}
    for c in coords_of(dims):
        x, y = oracle.initialize_markers_rank(md, lx, ly, dx, dy, Nx, Ny, c, dims, jitter,
                                              domains.rank_seed(seed, c, dims))
        out[c] = (x, y, np.zeros_like(x), np.zeros_like(x))
    if jitter != 0.0 and md % 2 == 1:
        out = oracle.exchange_markers(out, dims, lx, ly, dx, dy)
    om = oracle.PlumeModel(**{f: getattr(model, f) for f in model.FIELDS})
    for c, (x, y, _, _) in out.items():
        rho, mu = oracle.set_marker_properties(om, x, y, c[0] * (Nx - 2) * dx, c[1] * (Ny - 2) * dy)
        out[c] = (x, y, rho, mu)
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(1, 1), (2, 1), (2, 2), (3, 2)])
@pytest.mark.parametrize("md,jitter", [(4, 0.0), (4, 1.0), (3, 0.0), (3, 1.0), (5, 0.8)])
def test_initialize_markers_decomposed_matches_oracle(sf, dims, md, jitter):
    Nx, Ny, Lx, Ly = 24, 20, 1.0, 1.0
    model = sf.plume_model_unit_square()
    ctx = {c: sf.Context(0) for c in coords_of(dims)}
    got = domains.initialize_markers_decomposed(dims, Nx, Ny, Lx, Ly, model, md, ctx, jitter=jitter, seed=5)
    want = oracle_rank_markers(dims, Nx, Ny, Lx, Ly, md, jitter, 5, model)
    for c in coords_of(dims):
        for g, w, name in zip(got[c], want[c], ("x", "y", "rho", "mu")):
            assert np.array_equal(g.cpu().numpy(), w), (c, name)
    if jitter != 0.0 and md % 2 == 1 and dims != (1, 1):   # the exchange moved some markers between ranks
        dx, dy, lx, ly = geometry(dims, Nx, Ny, Lx, Ly)
        laid = sum(np.prod(oracle.marker_counts_rank(md, Nx, Ny, c, dims)) for c in coords_of(dims))
        assert sum(got[c][0].numel() for c in coords_of(dims)) == laid
        assert any(got[c][0].numel() != np.prod(oracle.marker_counts_rank(md, Nx, Ny, c, dims))
                   for c in coords_of(dims))


@pytest.mark.gpu
def test_decomposed_flow_from_model_steps(sf):
    """The multi-rank timestep loop set up from a material model: markers laid out by the ranks, one step."""
    model = sf.plume_model_unit_square()
    model.mu_air = 1e-2
    flow = domains.DecomposedStokesFlow2D((2, 2), 18, 18, 1.0, 1.0, model=model, marker_density=4, jitter=0.5,
                                          seed=1, eps=1e-4)
    rec = flow.step()
    assert rec["dt"] > 0 and rec["info"]["converged"]
    assert all(torch.isfinite(v).all() for v in flow.velocities())


@pytest.mark.gpu
@pytest.mark.parametrize("dims,nx,ny", [((2, 2), 11, 14), ((3, 2), 8, 14), ((1, 3), 20, 10)])
def test_decomposed_flow_meets_the_reference_golden_values(sf, dims, nx, ny):
    """test/test_StokesFlow2D.jl:91-110 on the GPU's decomposed timestep: the 20 x 26-point plume case split
    over the reference's rank grids, 5 timesteps, markers laid out by the ranks, the reference's golden values
    at its tolerance (atol 1e-6)."""
    from fields import golden
    g = golden()["stokes_flow_2d"]
    model = sf.PlumeModel(**g["model"])
    flow = domains.DecomposedStokesFlow2D(dims, nx, ny, g["Lx"], g["Ly"], model=model,
                                          marker_density=g["marker_density"], eps=g["stokes_eps"])
    for _ in range(g["Nt"]):
        flow.step()
    vx, vy = (v.cpu().numpy() for v in flow.velocities())
    assert vx.shape == (g["Nx"] + 2, g["Ny"] + 1) and vy.shape == (g["Nx"] + 1, g["Ny"] + 2)
    inds = np.array(g["inds"]) - 1
    assert np.allclose(vx.ravel(order="F")[inds], g["vx_ref"], rtol=0, atol=g["atol"])
    assert np.allclose(vy.ravel(order="F")[inds], g["vy_ref"], rtol=0, atol=g["atol"])


# test/test_InitialMarkerCoords.jl:17-56: the 20 x 26-point global grid on 1 to 9 ranks
INIT_GRIDS = [((1, 1), 20, 26), ((1, 2), 20, 14), ((2, 1), 11, 26), ((1, 3), 20, 10), ((3, 1), 8, 26),
              ((1, 4), 20, 8), ((2, 3), 11, 10), ((3, 2), 8, 14), ((2, 4), 11, 8), ((3, 3), 8, 10)]


@pytest.mark.parametrize("dims,nx,ny", INIT_GRIDS)
def test_reference_initial_marker_coords_on_ranks(dims, nx, ny):
    """test/test_InitialMarkerCoords.jl:67-134 as the reference runs it: 3 markers per cell, the ranks' layouts
    gathered with gather_markers! and sorted by x * Lx * 2 + y equal the global lattice (same count; `≈` on the
    whole vectors)."""
    md, Lx, Ly = 3, 10.0, 10.0
    nxg, nyg = domains.global_size(dims[0], nx), domains.global_size(dims[1], ny)
    assert (nxg, nyg) == (20, 26)
    dx, dy = Lx / (nxg - 1), Ly / (nyg - 1)
    lx, ly = (nx - 1) * dx, (ny - 1) * dy
    ranks = {}
    for c in coords_of(dims):
        x, y = oracle.initialize_markers_rank(md, lx, ly, dx, dy, nx, ny, c, dims)
        z = torch.zeros(x.size, dtype=torch.float64)
        ranks[c] = (torch.from_numpy(x), torch.from_numpy(y), z, z)
    xg, yg, _, _ = (t.numpy() for t in domains.gather_markers(ranks, dims, lx, ly, dx, dy))
    order = np.argsort(xg * Lx * 2 + yg, kind="stable")
    xg, yg = xg[order], yg[order]
    # the reference lattice (:101-124), LinRange elements as (1 - t) a + t b
    nmx, nmy = md * (nxg - 1), md * (nyg - 1)
    dxm, dym = dx / md, dy / md

    def linrange(a, b, n):
        t = np.arange(n) / (n - 1)
        return (1 - t) * a + t * b

    xr = np.repeat(linrange(0.5 * dxm, Lx - 0.5 * dxm, nmx), nmy)
    yr = np.tile(linrange(0.5 * dym, Ly - 0.5 * dym, nmy), nmx)
    order = np.argsort(xr * Lx * 2 + yr, kind="stable")
    xr, yr = xr[order], yr[order]
    assert xg.size == xr.size == nmx * nmy                                            # :126-127
    tol = np.sqrt(np.finfo(np.float64).eps)                                           # isapprox's default rtol
    assert np.linalg.norm(xg - xr) <= tol * max(np.linalg.norm(xg), np.linalg.norm(xr))   # :129
    assert np.linalg.norm(yg - yr) <= tol * max(np.linalg.norm(yg), np.linalg.norm(yr))   # :130
