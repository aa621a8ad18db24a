"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Deposit, PT iterates and marker positions are expected BIT-IDENTICAL to the
oracle (same expression order, no FMA contraction, reference summation order
in the deposit).  The only floating-point difference allowed anywhere is the
summation order inside the residual norm `err`, which can only move the
stopping iteration when err lands within ~1e-15 of eps; the full-timestep
tests therefore also check the required bar (1e-10 relative L2) explicitly.
"""
import math

import numpy as np
import pytest
import torch

from fields import F, golden, random_fields, rel_l2, solver_test_fields

pytestmark = pytest.mark.gpu

TOL_REL_L2 = 1e-10   # plain FP64 path vs oracle, V / P / marker positions


def dev(a: np.ndarray) -> torch.Tensor:
    """numpy (Julia layout, Fortran order) -> column-major CUDA tensor of the same shape."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        return torch.from_numpy(a.copy()).cuda()
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def host(t: torch.Tensor) -> np.ndarray:
    if t.dim() == 1:
        return t.cpu().numpy()
    return np.asfortranarray(t.t().contiguous().cpu().numpy().T)


# ---------------------------------------------------------------------------
# deposit
# ---------------------------------------------------------------------------
def test_deposit_kat(sf):
    g = golden()["marker_to_grid_kat"]
    val = sf.zeros(*g["shape"])
    vws = dev(np.ones(g["shape"], order="F"))
    ws = dev(np.ones(g["shape"], order="F"))
    sf.bilinear_marker_to_grid(g["x_grid_min"], g["y_grid_min"], val, dev(np.array(g["x_m"])),
                               dev(np.array(g["y_m"])), dev(np.array(g["val_m"])), g["dx"], g["dy"], vws, ws)
    assert np.allclose(host(val), np.array(g["reference_columns"]).T, rtol=1.5e-8, atol=0)


@pytest.mark.parametrize("which", ["rho", "mu_b", "mu_p"])
def test_deposit_bitexact_random(sf, oracle_lib, which):
    """Random markers (with 3 erroneous ones) onto each of the three staggered grids."""
    O = oracle_lib
    Nx, Ny = 37, 29
    dx, dy = 1.0 / (Nx - 1), 0.8 / (Ny - 1)
    o = O.node_origins(dx, dy)
    x0, y0, shape = {"rho": (o["x_rho"], o["y_rho"], (Nx + 1, Ny)), "mu_b": (o["x"], o["y"], (Nx, Ny)),
                     "mu_p": (o["x_p"], o["y_p"], (Nx - 1, Ny - 1))}[which]
    rng = np.random.default_rng(5)
    nm = 30 * (Nx - 1) * (Ny - 1)
    x = rng.random(nm) * (Nx - 1) * dx
    y = rng.random(nm) * (Ny - 1) * dy
    x[:3] = [-1.0, 5.0, np.nan]
    v = np.exp(rng.normal(size=nm))
    ref = np.asfortranarray(rng.random(shape))
    vws_o, ws_o = F(Nx + 1, Ny), F(Nx + 1, Ny)
    ref_before = ref.copy(order="F")
    nb, ne = O.bilinear_marker_to_grid(x0, y0, ref, x, y, v, dx, dy, vws_o, ws_o)
    got = dev(ref_before)
    vws, ws = sf.zeros(Nx + 1, Ny), sf.zeros(Nx + 1, Ny)
    sf.get_warnings(reset=True)
    sf.bilinear_marker_to_grid(x0, y0, got, dev(x), dev(y), dev(v), dx, dy, vws, ws)
    w = sf.get_warnings(reset=True)
    assert np.array_equal(host(got), ref)
    assert np.array_equal(host(ws), ws_o) and np.array_equal(host(vws), vws_o)
    assert w["bad_markers"] == nb == 3
    assert w["empty_nodes"] == ne


def test_deposit_no_markers_keeps_values(sf):
    val = dev(np.full((5, 4), 3.0, order="F"))
    empty = torch.empty(0, dtype=torch.float64, device="cuda")
    sf.get_warnings(reset=True)
    sf.bilinear_marker_to_grid(0.0, 0.0, val, empty, empty, empty, 0.1, 0.1)
    assert np.all(host(val) == 3.0)
    assert sf.get_warnings(reset=True)["empty_nodes"] == 20


def test_deposit_clustered_markers(sf, oracle_lib):
    """Many markers in few cells (long segments) and markers exactly on nodes."""
    O = oracle_lib
    nx, ny, dx, dy = 8, 6, 0.5, 0.25
    rng = np.random.default_rng(9)
    x = np.concatenate([rng.random(3000) * 0.3 + 1.0, np.arange(nx) * dx])
    y = np.concatenate([rng.random(3000) * 0.2 + 0.5, np.full(nx, 2 * dy)])
    v = rng.random(x.size)
    ref = F(nx, ny)
    O.bilinear_marker_to_grid(0.0, 0.0, ref, x, y, v, dx, dy, F(nx, ny), F(nx, ny))
    got = sf.zeros(nx, ny)
    sf.bilinear_marker_to_grid(0.0, 0.0, got, dev(x), dev(y), dev(v), dx, dy)
    assert np.array_equal(host(got), ref)


@pytest.mark.parametrize("order", ["x_fastest", "y_fastest", "reversed", "cell_blocks", "alternating_rows"])
def test_deposit_marker_orders(sf, oracle_lib, order):
    """A jittered lattice of 5x5 markers per cell in orders that give the gather's merge long runs from one
    cell (cell blocks), runs that alternate between neighbouring cells (lattice rows), and runs in reverse
    order; all three staggered grids, bit for bit against the oracle's serial loop."""
    O = oracle_lib
    Nx, Ny = 26, 19
    dx, dy = 1.0 / (Nx - 1), 0.7 / (Ny - 1)
    k = 5
    mx, my = (Nx - 1) * k, (Ny - 1) * k
    rng = np.random.default_rng(21)
    ii, jj = np.meshgrid(np.arange(mx), np.arange(my), indexing="ij")    # ii: x index, jj: y index
    x = (ii + 0.5 + 0.4 * (rng.random(ii.shape) - 0.5)) * dx / k
    y = (jj + 0.5 + 0.4 * (rng.random(jj.shape) - 0.5)) * dy / k
    if order == "x_fastest":
        idx = np.ravel_multi_index((ii.T.ravel(), jj.T.ravel()), ii.shape)
    elif order == "y_fastest":
        idx = np.arange(ii.size)
    elif order == "reversed":
        idx = np.ravel_multi_index((ii.T.ravel(), jj.T.ravel()), ii.shape)[::-1]
    elif order == "cell_blocks":
        cell = (ii // k) + (jj // k) * (Nx - 1)
        idx = np.argsort(cell.ravel(), kind="stable")
    else:   # lattice rows in x order, every second row reversed
        rows = [np.ravel_multi_index((np.arange(mx)[::(1 if j % 2 == 0 else -1)], np.full(mx, j)), ii.shape)
                for j in range(my)]
        idx = np.concatenate(rows)
    x, y = x.ravel()[idx], y.ravel()[idx]
    v = np.exp(rng.normal(size=x.size))
    o = O.node_origins(dx, dy)
    xt, yt, vt = dev(x), dev(y), dev(v)
    for x0, y0, shape in ((o["x_rho"], o["y_rho"], (Nx + 1, Ny)), (o["x"], o["y"], (Nx, Ny)),
                          (o["x_p"], o["y_p"], (Nx - 1, Ny - 1))):
        ref = F(*shape)
        O.bilinear_marker_to_grid(x0, y0, ref, x, y, v, dx, dy, F(Nx + 1, Ny), F(Nx + 1, Ny))
        got = sf.zeros(*shape)
        sf.bilinear_marker_to_grid(x0, y0, got, xt, yt, vt, dx, dy)
        assert np.array_equal(host(got), ref), (order, shape)


@pytest.mark.parametrize("ngrids", [1, 3, 4])
def test_deposit_grids_equals_one_call_per_grid(sf, oracle_lib, ngrids):
    """The fused deposit of a timestep's grids equals one bilinear_marker_to_grid call per grid in order, bit
    for bit: every grid, the sum arrays (the last grid's sums), and the warning counters; and the oracle."""
    O = oracle_lib
    Nx, Ny = 33, 27
    dx, dy = 1.0 / (Nx - 1), 0.9 / (Ny - 1)
    o = O.node_origins(dx, dy)
    rng = np.random.default_rng(31)
    nm = 20 * (Nx - 1) * (Ny - 1)
    x = rng.random(nm) * (Nx - 1) * dx
    y = rng.random(nm) * (Ny - 1) * dy
    x[:4] = [-1.0, 5.0, np.nan, 2.0]
    y[100:102] = [-3.0, np.inf]
    vals = [np.exp(rng.normal(size=nm)) for _ in range(4)]
    specs = [(o["x_rho"], o["y_rho"], (Nx + 1, Ny), 0), (o["x"], o["y"], (Nx, Ny), 1),
             (o["x_p"], o["y_p"], (Nx - 1, Ny - 1), 1), (o["x_vx"], o["y_vx"], (Nx + 1, Ny - 1), 2)][:ngrids]
    xt, yt = dev(x), dev(y)
    vt = [dev(v) for v in vals]
    starts = [np.asfortranarray(rng.random(shape)) for _, _, shape, _ in specs]
    # one call per grid
    one = [dev(a) for a in starts]
    vws1, ws1 = sf.zeros(Nx + 1, Ny), sf.zeros(Nx + 1, Ny)
    sf.get_warnings(reset=True)
    for (x0, y0, _, vi), g in zip(specs, one):
        sf.bilinear_marker_to_grid(x0, y0, g, xt, yt, vt[vi], dx, dy, vws1, ws1)
    w1 = sf.get_warnings(reset=True)
    # fused
    fused = [dev(a) for a in starts]
    vws2 = dev(np.full((Nx + 1, Ny), 7.0, order="F"))
    ws2 = dev(np.full((Nx + 1, Ny), 7.0, order="F"))
    sf.bilinear_marker_to_grids([(x0, y0, g, vt[vi]) for (x0, y0, _, vi), g in zip(specs, fused)], xt, yt, dx, dy,
                                vws2, ws2)
    w2 = sf.get_warnings(reset=True)
    for a, b in zip(one, fused):
        assert torch.equal(a, b)
    assert torch.equal(vws1, vws2) and torch.equal(ws1, ws2)
    assert w1["bad_markers"] == w2["bad_markers"] > 0 and w1["empty_nodes"] == w2["empty_nodes"]
    for (x0, y0, shape, vi), a, g in zip(specs, starts, fused):
        ref = a.copy(order="F")
        O.bilinear_marker_to_grid(x0, y0, ref, x, y, vals[vi], dx, dy, F(Nx + 1, Ny), F(Nx + 1, Ny))
        assert np.array_equal(host(g), ref)


def test_deposit_grids_with_markers_piled_in_cells(sf, oracle_lib):
    """The fused deposit with cells holding 3*10^4 and 2000 markers (each grid's long-cell radix sort works in
    that grid's own slice of the key buffer), against the oracle on all three staggered grids."""
    O = oracle_lib
    Nx, Ny = 30, 24
    dx, dy = 0.04, 0.05
    rng = np.random.default_rng(41)
    n0, n1, n2 = 20_000, 30_000, 2_000
    x = np.concatenate([rng.random(n0) * (Nx - 1) * dx, (5 + rng.random(n1)) * dx, (20 + rng.random(n2)) * dx])
    y = np.concatenate([rng.random(n0) * (Ny - 1) * dy, (7 + rng.random(n1)) * dy, (15 + rng.random(n2)) * dy])
    order = rng.permutation(x.size)
    x, y = x[order], y[order]
    rho, mu = np.exp(rng.normal(size=x.size)), np.exp(rng.normal(size=x.size))
    o = O.node_origins(dx, dy)
    specs = [(o["x_rho"], o["y_rho"], (Nx + 1, Ny), rho), (o["x"], o["y"], (Nx, Ny), mu),
             (o["x_p"], o["y_p"], (Nx - 1, Ny - 1), mu)]
    grids = [sf.zeros(*shape) for _, _, shape, _ in specs]
    sf.bilinear_marker_to_grids([(x0, y0, g, dev(v)) for (x0, y0, _, v), g in zip(specs, grids)], dev(x), dev(y),
                                dx, dy)
    for (x0, y0, shape, v), g in zip(specs, grids):
        ref = F(*shape)
        O.bilinear_marker_to_grid(x0, y0, ref, x, y, v, dx, dy, F(Nx + 1, Ny), F(Nx + 1, Ny))
        assert np.array_equal(host(g), ref), shape


def test_deposit_grids_arguments(sf):
    g = sf.zeros(6, 5)
    x = torch.zeros(10, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        sf.bilinear_marker_to_grids([], x, x, 0.1, 0.1)
    with pytest.raises(ValueError):
        sf.bilinear_marker_to_grids([(0.0, 0.0, g, x)] * 5, x, x, 0.1, 0.1)
    with pytest.raises(ValueError):
        sf.bilinear_marker_to_grids([(0.0, 0.0, g, x[:5])], x, x, 0.1, 0.1)
    empty = torch.empty(0, dtype=torch.float64, device="cuda")
    val = dev(np.full((5, 4), 3.0, order="F"))
    sf.get_warnings(reset=True)
    sf.bilinear_marker_to_grids([(0.0, 0.0, val, empty), (0.05, 0.05, val, empty)], empty, empty, 0.1, 0.1)
    assert np.all(host(val) == 3.0)
    assert sf.get_warnings(reset=True)["empty_nodes"] == 40


def test_deposit_and_rebin_with_markers_piled_in_one_cell(sf, oracle_lib):
    """Markers piled into single cells, as markers clamped into a corner pile up: one cell holds 10^5 markers
    (more than a shared-memory window of the segment sort), another 2000, the rest of the grid ~25 per cell,
    all indices shuffled.  The deposit (regular and allocation-free) equals the oracle's serial loop bit for
    bit, and the rebin's permutation is sorted inside every cell."""
    O = oracle_lib
    nx, ny, dx, dy = 40, 30, 0.025, 0.03
    rng = np.random.default_rng(12)
    n0, n1, n2 = 30_000, 100_000, 2_000
    x = np.concatenate([rng.random(n0) * (nx - 1) * dx, (5 + rng.random(n1)) * dx, (30 + rng.random(n2)) * dx])
    y = np.concatenate([rng.random(n0) * (ny - 1) * dy, (7 + rng.random(n1)) * dy, (20 + rng.random(n2)) * dy])
    order = rng.permutation(x.size)
    x, y = x[order], y[order]
    v = np.exp(rng.normal(size=x.size))
    ref = F(nx, ny)
    O.bilinear_marker_to_grid(0.0, 0.0, ref, x, y, v, dx, dy, F(nx, ny), F(nx, ny))
    got = sf.zeros(nx, ny)
    xt, yt, vt = dev(x), dev(y), dev(v)
    sf.bilinear_marker_to_grid(0.0, 0.0, got, xt, yt, vt, dx, dy)
    assert np.array_equal(host(got), ref)
    na = sf.zeros(nx, ny)
    sf.bilinear_marker_to_grid_noalloc(0.0, 0.0, na, xt, yt, vt, dx, dy)
    assert np.array_equal(host(na), ref)
    counts_o, _ = O.cell_counts(x, y, 0.0, 0.0, dx, dy, nx, ny)
    counts, offsets, perm = sf.rebin_markers(xt, yt, 0.0, 0.0, dx, dy, nx, ny)
    assert np.array_equal(counts.cpu().numpy(), counts_o) and counts_o.max() >= n1
    off = offsets.cpu().numpy()
    p = perm.cpu().numpy()[: off[-1]]
    assert np.array_equal(np.sort(p), np.arange(x.size))
    for c in range(counts_o.size):
        assert np.all(np.diff(p[off[c]:off[c + 1]]) > 0), f"cell {c} not in marker order"


# ---------------------------------------------------------------------------
# solver
# ---------------------------------------------------------------------------
NAMES = ["P", "Vx", "Vy", "rho_vy", "mu_b", "mu_p", "txx", "tyy", "txy", "divV", "dtPt", "Rx", "Ry", "dVxdt",
         "dVydt", "dtVx", "dtVy", "Vx_s", "Vy_s"]


def gpu_solve(sf, a_np, g_y, dx, dy, Nx, Ny, dt, maxdisp, stab, eps, iter_max):
    t = {k: dev(v) for k, v in a_np.items()}
    info = sf.solve_stokes_info(*[t[k] for k in NAMES], g_y, dx, dy, Nx, Ny, dt, maxdisp,
                                use_free_surface_stabilization=stab, eps=eps, iter_max=iter_max)
    return {k: host(v) for k, v in t.items()}, info


def test_solver_golden(sf, oracle_lib):
    """test/test_StokesSolver.jl:48-140 on the GPU; bit-identical to the oracle."""
    O = oracle_lib
    g = golden()["stokes_solver"]
    Nx, Ny, dx, dy = g["Nx"], g["Ny"], g["dx"], g["dy"]
    a = O.stokes_arrays(Nx, Ny)
    a["rho_vy"][:], a["mu_b"][:], a["mu_p"][:] = solver_test_fields(Nx, Ny, dx, dy)
    b, info = gpu_solve(sf, {k: v.copy(order="F") for k, v in a.items()}, g["g_y"], dx, dy, Nx, Ny, 0.0,
                        g["maxdisp"], True, g["eps"], 100000)
    r = O.solve_stokes(a, g["g_y"], dx, dy, Nx, Ny, 0.0, g["maxdisp"], True, g["eps"], 100000)
    inds = np.array(g["inds"]) - 1
    vx = b["Vx"].ravel(order="F")[inds]
    assert np.linalg.norm(vx - g["vx_ref"]) <= 1.5e-8 * np.linalg.norm(g["vx_ref"])
    vy = b["Vy"].ravel(order="F")[inds]
    assert np.linalg.norm(vy - g["vy_ref"]) <= 1.5e-8 * np.linalg.norm(g["vy_ref"])
    assert info["iters"] == r.iters and info["n_checks"] == r.n_checks and info["converged"] == 1
    assert info["dt"] == r.dt
    assert math.isclose(info["err"], r.err, rel_tol=1e-12)
    for k in NAMES:
        assert np.array_equal(b[k], a[k]), f"{k} differs from the oracle"


@pytest.mark.parametrize("Nx,Ny,iters,stab,dt0", [(67, 45, 700, True, 0.0), (40, 70, 1234, True, 3e-3),
                                                  (33, 33, 500, False, 0.0), (130, 97, 2100, True, 1e-3)])
def test_solver_fixed_iterations_bitexact(sf, oracle_lib, Nx, Ny, iters, stab, dt0):
    """Warm-started solves from a non-trivial state with a node-to-node random 10x viscosity contrast
    (larger per-node contrasts make the reference scheme itself diverge), a fixed iteration count
    (dt updates, checks and a final partial chunk inside), Nx != Ny: every array bit-identical."""
    O = oracle_lib
    dx, dy = 1.0 / (Nx - 1), 1.2 / (Ny - 1)
    a = O.stokes_arrays(Nx, Ny)
    a["rho_vy"][:], a["mu_b"][:], a["mu_p"][:] = random_fields(Nx, Ny, seed=Nx, contrast=10.0)
    rng = np.random.default_rng(Ny)
    for k in ("P", "Vx_s", "Vy_s", "dVxdt", "dVydt"):
        a[k][:] = 1e-3 * rng.normal(size=a[k].shape)
    b, info = gpu_solve(sf, {k: v.copy(order="F") for k, v in a.items()}, 9.81, dx, dy, Nx, Ny, dt0, 0.5, stab,
                        1e-300, iters)
    r = O.solve_stokes(a, 9.81, dx, dy, Nx, Ny, dt0, 0.5, stab, 1e-300, iters)
    assert info["iters"] == r.iters == iters
    assert info["dt"] == r.dt
    for k in NAMES:
        assert np.array_equal(b[k], a[k]), f"{k} differs from the oracle"


def test_solver_nonfinite_status(sf):
    Nx = Ny = 16
    a = {k: np.zeros(s, order="F") for k, s in _shapes(Nx, Ny).items()}
    a["rho_vy"][:] = 1.0
    a["mu_b"][:] = 1.0
    a["mu_p"][:] = 1.0
    a["P"][3, 3] = np.nan
    with pytest.raises(sf.StokesFlowError) as e:
        gpu_solve(sf, a, 9.81, 0.1, 0.1, Nx, Ny, 0.0, 0.5, True, 1e-8, 10000)
    assert e.value.status == 5


def _shapes(Nx, Ny):
    return dict(P=(Nx - 1, Ny - 1), Vx=(Nx + 2, Ny + 1), Vy=(Nx + 1, Ny + 2), rho_vy=(Nx + 1, Ny), mu_b=(Nx, Ny),
                mu_p=(Nx - 1, Ny - 1), txx=(Nx - 1, Ny - 1), tyy=(Nx - 1, Ny - 1), txy=(Nx, Ny),
                divV=(Nx - 1, Ny - 1), dtPt=(Nx - 1, Ny - 1), Rx=(Nx - 2, Ny - 1), Ry=(Nx - 1, Ny - 2),
                dVxdt=(Nx - 2, Ny - 1), dVydt=(Nx - 1, Ny - 2), dtVx=(Nx - 2, Ny - 1), dtVy=(Nx - 1, Ny - 2),
                Vx_s=(Nx, Ny + 1), Vy_s=(Nx + 1, Ny))


# ---------------------------------------------------------------------------
# advection + rebin
# ---------------------------------------------------------------------------
def _grid_line_markers(rng, xmins, ymins, dx, dy, kx, ky, n_rand):
    """Markers on the grid lines of every given origin (x = xmin + k dx exactly, as the reference computes the
    node coordinate) and one and two ulps to either side, plus random ones: the positions where
    floor((x - xmin)/dx) and (x - x_ix)/dx sit on their boundaries."""
    xs, ys = [], []
    for x0, y0 in zip(xmins, ymins):
        for k in range(kx):
            base = x0 + k * dx
            for v in (base, np.nextafter(base, -np.inf), np.nextafter(base, np.inf),
                      np.nextafter(np.nextafter(base, -np.inf), -np.inf), np.nextafter(np.nextafter(base, np.inf), np.inf)):
                xs.append(v)
                ys.append(y0 + rng.integers(0, ky) * dy + rng.random() * dy)
        for k in range(ky):
            base = y0 + k * dy
            for v in (base, np.nextafter(base, -np.inf), np.nextafter(base, np.inf)):
                ys.append(v)
                xs.append(x0 + rng.integers(0, kx) * dx + rng.random() * dx)
    x = np.concatenate([np.array(xs), rng.random(n_rand) * (kx - 1) * dx])
    y = np.concatenate([np.array(ys), rng.random(n_rand) * (ky - 1) * dy])
    return x, y


def test_divisions_on_grid_lines_bitexact(sf, oracle_lib):
    """topleftIndexRelDist's divisions run as a reciprocal multiply with a proved correctly rounded result
    (the IEEE division where the proof fails): on markers sitting on the grid lines of all three deposit grids
    and of the velocity grids, and 1-2 ulps off them, the deposits and the RK4 advection stay bit-identical to
    the oracle's IEEE divisions."""
    O = oracle_lib
    Nx, Ny = 33, 27
    dx, dy = 1.0 / (Nx - 1), 0.9 / (Ny - 1)
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    o = O.node_origins(dx, dy)
    rng = np.random.default_rng(21)
    x, y = _grid_line_markers(rng, [o["x"], o["x_p"], o["x_rho"], o["x_vx"], o["x_vy"]],
                              [o["y"], o["y_p"], o["y_rho"], o["y_vx"], o["y_vy"]], dx, dy, Nx, Ny, 20000)
    x = np.clip(x, 0.0, lx)
    y = np.clip(y, 0.0, ly)
    v = np.exp(rng.normal(size=x.size))
    for x0, y0, shape in ((o["x_rho"], o["y_rho"], (Nx + 1, Ny)), (o["x"], o["y"], (Nx, Ny)),
                          (o["x_p"], o["y_p"], (Nx - 1, Ny - 1))):
        ref = F(*shape)
        O.bilinear_marker_to_grid(x0, y0, ref, x, y, v, dx, dy, F(Nx + 1, Ny), F(Nx + 1, Ny))
        got = sf.zeros(*shape)
        sf.bilinear_marker_to_grid(x0, y0, got, dev(x), dev(y), dev(v), dx, dy)
        assert np.array_equal(host(got), ref), f"deposit origin ({x0}, {y0})"
    Vx = np.asfortranarray(rng.normal(size=(Nx + 2, Ny + 1)))
    Vy = np.asfortranarray(rng.normal(size=(Nx + 1, Ny + 2)))
    dt = 0.3 * min(dx, dy)
    xo, yo = x.copy(), y.copy()
    O.move_markers_rk4(xo, yo, Vx, Vy, o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, lx, ly, dx, dy)
    xg, yg = dev(x), dev(y)
    sf.move_markers_rk4(xg, yg, dev(Vx), dev(Vy), o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, lx, ly, dx, dy)
    assert np.array_equal(host(xg), xo) and np.array_equal(host(yg), yo)


def test_advection_bitexact(sf, oracle_lib):
    O = oracle_lib
    Nx, Ny = 41, 35
    dx, dy = 1.0 / (Nx - 1), 1.0 / (Ny - 1)
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    rng = np.random.default_rng(2)
    Vx = np.asfortranarray(rng.normal(size=(Nx + 2, Ny + 1)))
    Vy = np.asfortranarray(rng.normal(size=(Nx + 1, Ny + 2)))
    nm = 50000
    x = rng.random(nm) * lx
    y = rng.random(nm) * ly
    x[:4] = [0.0, lx, -0.3, 2.0]   # on / beyond the walls: exercises the clamps and failsafes
    y[:4] = [ly, 0.0, 0.5, -1.0]
    dt = 0.5 * min(dx / np.abs(Vx).max(), dy / np.abs(Vy).max())
    xg, yg = dev(x), dev(y)
    sf.get_warnings(reset=True)
    o = O.node_origins(dx, dy)
    sf.move_markers_rk4(xg, yg, dev(Vx), dev(Vy), o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, lx, ly, dx, dy)
    nf = O.move_markers_rk4(x, y, Vx, Vy, o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, lx, ly, dx, dy)
    assert np.array_equal(host(xg), x) and np.array_equal(host(yg), y)
    assert sf.get_warnings(reset=True)["interp_failsafe"] == nf > 0


def test_advection_constant_field(sf):
    """test/test_MoveMarkers.jl:16-47 on the GPU."""
    Nx, Ny, dx, dy = 10, 13, 0.4, 0.7
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    rng = np.random.default_rng(0)
    nm = 25 * (Nx - 1) * (Ny - 1)
    x = rng.random(nm) * (lx - dx) + 0.5 * dx
    y = rng.random(nm) * (ly - dy) + 0.5 * dy
    xg, yg = dev(x), dev(y)
    dt = 0.5 * min(dx / 1.0, dy / 2.0)
    sf.move_markers_rk4(xg, yg, dev(np.ones((Nx + 2, Ny + 1), order="F")),
                        dev(-2 * np.ones((Nx + 1, Ny + 2), order="F")), -dx, -0.5 * dy, -0.5 * dx, -dy, dt, lx, ly,
                        dx, dy)
    assert np.allclose(host(xg), x + dt, rtol=1.5e-8) and np.allclose(host(yg), y - 2 * dt, rtol=1.5e-8)


def test_rebin_counts_and_order(sf, oracle_lib):
    O = oracle_lib
    nx, ny, dx, dy = 50, 40, 0.02, 0.025
    rng = np.random.default_rng(4)
    nm = 100000
    x = rng.random(nm) * (nx - 1) * dx
    y = rng.random(nm) * (ny - 1) * dy
    x[:2] = [-5.0, 100.0]
    counts_o, nout = O.cell_counts(x, y, 0.0, 0.0, dx, dy, nx, ny)
    sf.get_warnings(reset=True)
    counts, offsets, perm = sf.rebin_markers(dev(x), dev(y), 0.0, 0.0, dx, dy, nx, ny)
    assert np.array_equal(counts.cpu().numpy(), counts_o)
    assert sf.get_warnings(reset=True)["markers_outside"] == nout == 2
    off = offsets.cpu().numpy()
    p = perm.cpu().numpy()[: off[-1]]
    assert off[-1] == nm - 2
    assert np.array_equal(np.sort(p), np.arange(2, nm))
    for c in range(counts_o.size):
        seg = p[off[c]:off[c + 1]]
        assert np.all(np.diff(seg) > 0)


# ---------------------------------------------------------------------------
# full timesteps
# ---------------------------------------------------------------------------
def test_flow_golden_matches_oracle(sf, oracle_lib):
    """test/test_StokesFlow2D.jl:53-110 (5 timesteps) on the GPU: against the oracle, and against the reference's
    golden values at the reference's tolerance (atol 1e-6, :107-108)."""
    O = oracle_lib
    g = golden()["stokes_flow_2d"]
    model = sf.PlumeModel(**g["model"])
    Vx, Vy, t_tot = sf.stokes_flow_2d(g["Nt"], g["Nx"], g["Ny"], g["Lx"], g["Ly"], model,
                                      marker_density=g["marker_density"], stokes_eps=g["stokes_eps"])
    Vxo, Vyo, t_o = O.stokes_flow_2d(g["Nt"], g["Nx"], g["Ny"], g["Lx"], g["Ly"], O.PlumeModel(**g["model"]),
                                     marker_density=g["marker_density"], stokes_eps=g["stokes_eps"])
    assert rel_l2(Vx, Vxo) <= TOL_REL_L2 and rel_l2(Vy, Vyo) <= TOL_REL_L2
    assert math.isclose(t_tot, t_o, rel_tol=1e-12)
    inds = np.array(g["inds"]) - 1
    assert np.allclose(Vx.ravel(order="F")[inds], g["vx_ref"], rtol=0, atol=g["atol"])
    assert np.allclose(Vy.ravel(order="F")[inds], g["vy_ref"], rtol=0, atol=g["atol"])


def test_plume_64_five_timesteps(sf, oracle_lib):
    """The CPU-runnable plume case (63x63 cells, 4x4 markers per cell jittered +-0.25 from seed 0,
    relative residual 1e-6, 5 timesteps, air viscosity 1e-2) against the oracle:
    V, P, marker positions within 1e-10 relative L2 and identical markers-per-cell counts."""
    O = oracle_lib
    m = sf.plume_model_unit_square()
    m.mu_air = 1e-2
    st = sf.StokesFlow2D(64, 64, 1.0, 1.0, m, marker_density=4, stokes_rtol=1e-6, jitter=0.5, seed=0, rebin=True)
    om = O.PlumeModel(**{f: getattr(m, f) for f in m.FIELDS})
    dx = dy = 1.0 / 63
    a = O.stokes_arrays(64, 64)
    vws, ws = F(65, 64), F(65, 64)
    o = O.node_origins(dx, dy)
    x, y = O.initialize_markers(4, 1.0, 1.0, dx, dy, 64, 64, 0.5, 0)
    rho, mu = O.set_marker_properties(om, x, y)
    dt = 0.0
    for _ in range(5):
        rec = st.step()
        O.bilinear_marker_to_grid(o["x_rho"], o["y_rho"], a["rho_vy"], x, y, rho, dx, dy, vws, ws)
        O.bilinear_marker_to_grid(o["x"], o["y"], a["mu_b"], x, y, mu, dx, dy, vws, ws)
        O.bilinear_marker_to_grid(o["x_p"], o["y_p"], a["mu_p"], x, y, mu, dx, dy, vws, ws)
        eps = 1e-6 * np.mean(np.abs(9.81 * a["rho_vy"][1:-1, 1:-1]))
        r = O.solve_stokes(a, 9.81, dx, dy, 64, 64, dt, 0.5, True, eps, 100000)
        dt = r.dt
        O.move_markers_rk4(x, y, a["Vx"], a["Vy"], o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, 1.0, 1.0, dx, dy)
        assert rec["info"]["converged"] == 1 and rec["info"]["iters"] == r.iters
        for k, t in (("Vx", st.Vx), ("Vy", st.Vy), ("P", st.P)):
            assert rel_l2(host(t), a[k]) <= TOL_REL_L2, k
        assert rel_l2(host(st.x_m), x) <= TOL_REL_L2 and rel_l2(host(st.y_m), y) <= TOL_REL_L2
        counts_o, _ = O.cell_counts(x, y, 0.0, 0.0, dx, dy, 64, 64)
        assert np.array_equal(st.counts.cpu().numpy(), counts_o)
    # with every piece bit-identical, so is the whole run
    assert np.array_equal(host(st.Vx), a["Vx"]) and np.array_equal(host(st.x_m), x)
