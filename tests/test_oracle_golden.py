"""Pins the CPU oracle against the reference's own known-answer tests.

Each test restates one of the reference's tests (cited) against the C oracle.
The values come from tests/golden/reference_golden.json (extracted verbatim
from the reference's test files by tests/golden/make_golden.py) or, for the
closed-form checks, from the formulas the reference's tests use.
"""
import math

import numpy as np
import pytest

from fields import F, golden, solver_test_fields


def julia_isapprox(a, b, rtol=math.sqrt(np.finfo(np.float64).eps)):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.linalg.norm(a - b) <= rtol * max(np.linalg.norm(a), np.linalg.norm(b))


def test_stokes_solver_golden(oracle_lib):
    """test/test_StokesSolver.jl:48-140 on one rank."""
    O = oracle_lib
    g = golden()["stokes_solver"]
    Nx, Ny, dx, dy = g["Nx"], g["Ny"], g["dx"], g["dy"]
    a = O.stokes_arrays(Nx, Ny)
    a["rho_vy"][:], a["mu_b"][:], a["mu_p"][:] = solver_test_fields(Nx, Ny, dx, dy)
    r = O.solve_stokes(a, g["g_y"], dx, dy, Nx, Ny, 0.0, g["maxdisp"], True, g["eps"], 100000)
    Vx, Vy = a["Vx"], a["Vy"]
    inds = np.array(g["inds"]) - 1
    assert julia_isapprox(Vx.ravel(order="F")[inds], g["vx_ref"])          # :125
    assert julia_isapprox(Vy.ravel(order="F")[inds], g["vy_ref"])          # :126
    # :116 returned dt
    dt_ref = g["maxdisp"] * min(dx / np.abs(Vx[1:-1, :]).max(), dy / np.abs(Vy[:, 1:-1]).max())
    assert math.isclose(r.dt, dt_ref, rel_tol=1.5e-8)
    assert r.err <= g["eps"]
    # :128-140 boundary identities, exact
    assert np.all(Vx[0, :] == -Vx[2, :]) and np.all(Vx[1, :] == 0.0)
    assert np.all(Vx[-1, :] == -Vx[-3, :]) and np.all(Vx[-2, :] == 0.0)
    assert np.all(Vx[:, 0] == Vx[:, 1]) and np.all(Vx[:, -1] == Vx[:, -2])
    assert np.all(Vy[:, 0] == -Vy[:, 2]) and np.all(Vy[:, 1] == 0.0)
    assert np.all(Vy[:, -1] == -Vy[:, -3]) and np.all(Vy[:, -2] == 0.0)
    assert np.all(Vy[0, :] == Vy[1, :]) and np.all(Vy[-1, :] == Vy[-2, :])


def test_marker_to_grid_kat(oracle_lib):
    """test/test_MarkerToGrid.jl:24-37: hand-computed 3x2 deposit (work arrays start at ones)."""
    O = oracle_lib
    g = golden()["marker_to_grid_kat"]
    val = F(*g["shape"])
    vws = np.ones(g["shape"], order="F")
    ws = np.ones(g["shape"], order="F")
    nb, ne = O.bilinear_marker_to_grid(g["x_grid_min"], g["y_grid_min"], val, np.array(g["x_m"]),
                                       np.array(g["y_m"]), np.array(g["val_m"]), g["dx"], g["dy"], vws, ws)
    ref = np.array(g["reference_columns"]).T
    assert nb == 0 and ne == 0
    assert np.allclose(val, ref, rtol=1.5e-8, atol=0)


def test_marker_to_grid_matches_direct_sum(oracle_lib):
    """The serial deposit equals an independent weighted-average restatement (README 'Details of Marker Methods')."""
    O = oracle_lib
    rng = np.random.default_rng(3)
    nx, ny, dx, dy = 9, 7, 0.3, 0.4
    xmin, ymin = -0.5 * dx, 0.0
    nm = 400
    x = rng.random(nm) * (nx - 1) * dx
    y = rng.random(nm) * (ny - 1) * dy
    v = rng.random(nm) + 1.0
    val = F(nx, ny)
    vws, ws = F(nx + 1, ny), F(nx + 1, ny)
    O.bilinear_marker_to_grid(xmin, ymin, val, x, y, v, dx, dy, vws, ws)
    num = np.zeros((nx, ny))
    den = np.zeros((nx, ny))
    for k in range(nm):
        fx, fy = (x[k] - xmin) / dx, (y[k] - ymin) / dy
        ix, iy = int(math.floor(fx)), int(math.floor(fy))   # 0-based cell; its nodes are ix+1, ix+2 (1-based)
        ax, ay = (x[k] - (xmin + ix * dx)) / dx, (y[k] - (ymin + iy * dy)) / dy
        for cx, wx in ((ix + 1, 1 - ax), (ix + 2, ax)):
            for cy, wy in ((iy + 1, 1 - ay), (iy + 2, ay)):
                if 1 <= cx <= nx and 1 <= cy <= ny:
                    num[cx - 1, cy - 1] += wx * wy * v[k]
                    den[cx - 1, cy - 1] += wx * wy
    mask = den > 0
    assert np.allclose(val[mask], num[mask] / den[mask], rtol=1e-13)
    assert np.allclose(ws[:nx, :], den, rtol=1e-13, atol=1e-15)


def test_marker_to_grid_bad_and_empty(oracle_lib):
    """MarkerToGrid.jl:66-67 (erroneous markers skipped) and :164-172 (empty nodes keep their value)."""
    O = oracle_lib
    nx, ny = 6, 5
    val = np.full((nx, ny), 7.0, order="F")
    vws, ws = F(nx, ny), F(nx, ny)
    x = np.array([0.05, 100.0, -5.0])
    y = np.array([0.05, 0.1, 0.1])
    nb, ne = O.bilinear_marker_to_grid(0.0, 0.0, val, x, y, np.array([2.0, 3.0, 4.0]), 0.1, 0.1, vws, ws)
    assert nb == 2
    assert ne == nx * ny - 4
    assert np.all(val[:2, :2] == 2.0)
    assert val[3, 3] == 7.0


def test_move_markers_constant_field(oracle_lib):
    """test/test_MoveMarkers.jl:16-47: a constant velocity field translates every marker exactly."""
    O = oracle_lib
    Nx, Ny, dx, dy = 10, 13, 0.4, 0.7
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    rng = np.random.default_rng(0)
    nm = 25 * (Nx - 1) * (Ny - 1)
    x = rng.random(nm) * (lx - dx) + 0.5 * dx
    y = rng.random(nm) * (ly - dy) + 0.5 * dy
    x0, y0 = x.copy(), y.copy()
    Vx = np.ones((Nx + 2, Ny + 1), order="F")
    Vy = np.ones((Nx + 1, Ny + 2), order="F") * -2
    dt = 0.5 * min(dx / 1.0, dy / 2.0)
    nf = O.move_markers_rk4(x, y, Vx, Vy, -dx, -0.5 * dy, -0.5 * dx, -dy, dt, lx, ly, dx, dy)
    assert nf == 0
    assert np.allclose(x, x0 + 1.0 * dt, rtol=1.5e-8)
    assert np.allclose(y, y0 - 2.0 * dt, rtol=1.5e-8)


@pytest.mark.parametrize("quadrant", [0, 1, 2, 3])
def test_interpolate_v_quadrants(oracle_lib, quadrant):
    """test/test_MoveMarkers.jl:50-152: interpolateV against the closed-form bilinear +
    continuity-correction expressions in each quarter of a cell."""
    O = oracle_lib
    dx, dy = 0.4, 0.7
    rng = np.random.default_rng(10 + quadrant)
    Vx = np.asfortranarray(rng.random((4, 3)))
    Vy = np.asfortranarray(rng.random((3, 4)))
    sx, sy = [(0, 0), (0, 1), (1, 0), (1, 1)][quadrant]
    x = (0.99 * rng.random() + 0.005 + sx) * 0.5 * dx
    y = (0.99 * rng.random() + 0.005 + sy) * 0.5 * dy
    vx, vy, nf = O.interpolate_v(x, y, Vx, Vy, -dx, -0.5 * dy, -0.5 * dx, -dy, dx, dy)
    assert nf == 0
    V = lambda a, i, j: a[i - 1, j - 1]  # noqa: E731  (Julia 1-based)
    ix, iy, a, b = O.topleft_index_rel_dist(-dx, -0.5 * dy, x, y, dx, dy)
    assert ix == 2 and iy == (1 if sy == 0 else 2)
    bil = (1 - a) * (1 - b) * V(Vx, ix, iy) + a * (1 - b) * V(Vx, ix + 1, iy) + a * b * V(Vx, ix + 1, iy + 1) \
        + (1 - a) * b * V(Vx, ix, iy + 1)
    if a >= 0.5:
        c = 0.5 * (a - 0.5) ** 2 * ((1 - b) * (V(Vx, ix, iy) - 2 * V(Vx, ix + 1, iy) + V(Vx, ix + 2, iy))
                                    + b * (V(Vx, ix, iy + 1) - 2 * V(Vx, ix + 1, iy + 1) + V(Vx, ix + 2, iy + 1)))
    else:
        c = 0.5 * (a - 0.5) ** 2 * ((1 - b) * (V(Vx, ix - 1, iy) - 2 * V(Vx, ix, iy) + V(Vx, ix + 1, iy))
                                    + b * (V(Vx, ix - 1, iy + 1) - 2 * V(Vx, ix, iy + 1) + V(Vx, ix + 1, iy + 1)))
    assert math.isclose(vx, bil + c, rel_tol=1.5e-8)
    ix, iy, a, b = O.topleft_index_rel_dist(-0.5 * dx, -dy, x, y, dx, dy)
    assert iy == 2 and ix == (1 if sx == 0 else 2)
    bil = (1 - a) * (1 - b) * V(Vy, ix, iy) + a * (1 - b) * V(Vy, ix + 1, iy) + a * b * V(Vy, ix + 1, iy + 1) \
        + (1 - a) * b * V(Vy, ix, iy + 1)
    if b >= 0.5:
        c = 0.5 * (b - 0.5) ** 2 * ((1 - a) * (V(Vy, ix, iy) - 2 * V(Vy, ix, iy + 1) + V(Vy, ix, iy + 2))
                                    + a * (V(Vy, ix + 1, iy) - 2 * V(Vy, ix + 1, iy + 1) + V(Vy, ix + 1, iy + 2)))
    else:
        c = 0.5 * (b - 0.5) ** 2 * ((1 - a) * (V(Vy, ix, iy - 1) - 2 * V(Vy, ix, iy) + V(Vy, ix, iy + 1))
                                    + a * (V(Vy, ix + 1, iy - 1) - 2 * V(Vy, ix + 1, iy) + V(Vy, ix + 1, iy + 1)))
    assert math.isclose(vy, bil + c, rel_tol=1.5e-8)


def test_interpolate_v_failsafe(oracle_lib):
    """MoveMarkers.jl:80-99: positions outside the padded grid hit the index failsafes."""
    O = oracle_lib
    Vx = np.ones((6, 5), order="F")
    Vy = np.ones((5, 6), order="F")
    vx, vy, nf = O.interpolate_v(-10.0, 50.0, Vx, Vy, -1.0, -0.5, -0.5, -1.0, 1.0, 1.0)
    assert nf == 4 and vx == 1.0 and vy == 1.0


def test_initial_marker_coords(oracle_lib):
    """test/test_InitialMarkerCoords.jl:58-132 on one rank: the unjittered layout is
    LinRange(dxm/2, L - dxm/2, Nm) in x (outer) and y (inner)."""
    O = oracle_lib
    Nx, Ny, L, md = 20, 26, 10.0, 3
    dx, dy = L / (Nx - 1), L / (Ny - 1)
    x, y = O.initialize_markers(md, (Nx - 1) * dx, (Ny - 1) * dy, dx, dy, Nx, Ny)
    nmx, nmy = md * (Nx - 1), md * (Ny - 1)
    assert x.size == nmx * nmy
    xr = np.linspace(0.5 * dx / md, L - 0.5 * dx / md, nmx)
    yr = np.linspace(0.5 * dy / md, L - 0.5 * dy / md, nmy)
    assert np.allclose(x, np.repeat(xr, nmy), rtol=1.5e-8)
    assert np.allclose(y, np.tile(yr, nmx), rtol=1.5e-8)


def test_initial_marker_jitter_bounds(oracle_lib):
    """Jitter of width j sub-spacings keeps every marker within +-j/2 sub-spacings of its site."""
    O = oracle_lib
    Nx = Ny = 9
    dx = dy = 1.0 / 8
    x0, y0 = O.initialize_markers(4, 1.0, 1.0, dx, dy, Nx, Ny)
    x, y = O.initialize_markers(4, 1.0, 1.0, dx, dy, Nx, Ny, jitter=0.5, seed=0)
    dxm = dx / 4
    assert np.all(np.abs(x - x0) <= 0.25 * dxm + 1e-15) and np.all(np.abs(y - y0) <= 0.25 * dxm + 1e-15)
    assert np.std((x - x0) / dxm) > 0.1


def test_stokes_flow_2d_golden(oracle_lib):
    """test/test_StokesFlow2D.jl:53-110: 5 timesteps of the 20 x 26-point plume case with unjittered markers,
    against the reference's golden values at the reference's own tolerance (atol 1e-6).

    The marker lattice of that case puts markers exactly on the plume circle in exact arithmetic, so their
    material depends on the last bit of Julia's LinRange; the oracle uses the element formula the golden values
    fit, (1 - t) a + t b (test_linrange_form_decides_a_boundary_marker)."""
    O = oracle_lib
    g = golden()["stokes_flow_2d"]
    model = O.PlumeModel(**g["model"])
    Vx, Vy, t_tot = O.stokes_flow_2d(g["Nt"], g["Nx"], g["Ny"], g["Lx"], g["Ly"], model,
                                     marker_density=g["marker_density"], stokes_eps=g["stokes_eps"])
    assert Vx.shape == (g["Nx"] + 2, g["Ny"] + 1) and Vy.shape == (g["Nx"] + 1, g["Ny"] + 2)   # :103-104
    inds = np.array(g["inds"]) - 1
    assert np.allclose(Vx.ravel(order="F")[inds], g["vx_ref"], rtol=0, atol=g["atol"])      # :107
    assert np.allclose(Vy.ravel(order="F")[inds], g["vy_ref"], rtol=0, atol=g["atol"])      # :108


def test_linrange_form_decides_a_boundary_marker(oracle_lib):
    """In the golden case (dy = 0.4, 5 markers per cell) the 38th marker row is y = 3 in exact arithmetic, on
    the plume circle around (5, 5) of radius 2 for the marker column x = 5.  The form (1 - t) a + t b gives
    exactly 3.0, so that marker is matrix; the fma form gives 3.0000000000000004, which is plume."""
    O = oracle_lib
    g = golden()["stokes_flow_2d"]
    dx, dy = g["Lx"] / (g["Nx"] - 1), g["Ly"] / (g["Ny"] - 1)
    x, y = O.initialize_markers(g["marker_density"], (g["Nx"] - 1) * dx, (g["Ny"] - 1) * dy, dx, dy, g["Nx"],
                                g["Ny"])
    nmy = g["marker_density"] * (g["Ny"] - 1)
    k = 47 * nmy + 37                       # column 48 (x = 5), row 38 (y = 3)
    assert x[k] == 5.0 and y[k] == 3.0
    rho, _ = O.set_marker_properties(O.PlumeModel(**g["model"]), x[k:k + 1], y[k:k + 1])
    assert rho[0] == g["model"]["rho_matrix"]


# test/test_StokesFlow2D.jl:16-51: the same 20 x 26-point global grid split over 1 to 9 ranks
RANK_GRIDS = [((1, 1), 20, 26), ((1, 2), 20, 14), ((2, 1), 11, 26), ((1, 3), 20, 10), ((3, 1), 8, 26),
              ((2, 2), 11, 14), ((2, 3), 11, 10), ((3, 2), 8, 14), ((3, 3), 8, 10)]


@pytest.mark.parametrize("dims,nx,ny", RANK_GRIDS)
def test_stokes_flow_2d_golden_on_ranks(oracle_lib, dims, nx, ny):
    """test/test_StokesFlow2D.jl:91-110 on every rank grid the reference runs it on: the rank layouts of
    initializeMarkersCPU, the overlap sums of the deposits, the marker exchange and gather_V_grid, composed from
    the oracle's pieces, give the reference's golden values at its tolerance (atol 1e-6) in every split."""
    O = oracle_lib
    g = golden()["stokes_flow_2d"]
    model = O.PlumeModel(**g["model"])
    mk = O.rank_markers(dims, nx, ny, g["Lx"], g["Ly"], model, g["marker_density"])
    assert sum(v[0].size for v in mk.values()) == (g["marker_density"] * (g["Nx"] - 1)) * \
        (g["marker_density"] * (g["Ny"] - 1))                                    # the ranks tile the lattice
    Vx, Vy, t_tot, _, _ = O.stokes_flow_2d_ranks(g["Nt"], dims, nx, ny, g["Lx"], g["Ly"], mk,
                                                 stokes_eps=g["stokes_eps"])
    assert Vx.shape == (g["Nx"] + 2, g["Ny"] + 1) and Vy.shape == (g["Nx"] + 1, g["Ny"] + 2)   # :103-104
    inds = np.array(g["inds"]) - 1
    assert np.allclose(Vx.ravel(order="F")[inds], g["vx_ref"], rtol=0, atol=g["atol"])      # :107
    assert np.allclose(Vy.ravel(order="F")[inds], g["vy_ref"], rtol=0, atol=g["atol"])      # :108


def test_oracle_threads_do_not_change_bits(oracle_lib):
    """The timed CPU baseline and the full-size GPU parity test run the oracle's stencil and advection on
    several OpenMP threads: every array, dt, err and the iteration count are the same bits as on one thread
    (each point is written by one thread, and the residual means are summed serially)."""
    O = oracle_lib
    g = golden()["stokes_solver"]
    Nx, Ny, dx, dy = g["Nx"], g["Ny"], g["dx"], g["dy"]
    runs = {}
    for nt in (1, 4):
        a = O.stokes_arrays(Nx, Ny)
        a["rho_vy"][:], a["mu_b"][:], a["mu_p"][:] = solver_test_fields(Nx, Ny, dx, dy)
        r = O.solve_stokes(a, g["g_y"], dx, dy, Nx, Ny, 0.0, g["maxdisp"], True, g["eps"], 100000, nthreads=nt)
        o = O.node_origins(dx, dy)
        x, y = O.initialize_markers(4, dx * (Nx - 1), dy * (Ny - 1), dx, dy, Nx, Ny, 0.5, 3)
        nf = O.move_markers_rk4(x, y, a["Vx"], a["Vy"], o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], r.dt,
                                dx * (Nx - 1), dy * (Ny - 1), dx, dy, nthreads=nt)
        runs[nt] = (a, r, x, y, nf)
    (a1, r1, x1, y1, f1), (a4, r4, x4, y4, f4) = runs[1], runs[4]
    assert (r1.dt, r1.err, r1.iters, r1.n_checks) == (r4.dt, r4.err, r4.iters, r4.n_checks)
    for k in a1:
        assert np.array_equal(a1[k], a4[k]), k
    assert np.array_equal(x1, x4) and np.array_equal(y1, y4) and f1 == f4
