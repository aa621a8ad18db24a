"""The benchmark's own size on the GPU: the plume at 2047 x 2047 cells with 16 markers per cell (67 M markers,
jittered from seed 0, air viscosity 1e-2), checked against the oracle.

* deposit: all three grids (rho on the Vy nodes, mu on the nodes and on the cell centres) and the weight and
  value sums bit-identical to the oracle's serial loop over all 67 M markers;
* PT solve: 60 iterations from the deposited fields, every array bit-identical to the oracle (OpenMP);
* advection: a seeded sample of 1 M markers moved on the GPU and by the oracle, bit-identical; all 67 M moved
  markers finite and inside the domain;
* rebin: markers-per-cell counts of all 67 M markers identical to the oracle's; the permutation is a
  permutation, ordered by cell and stable inside each cell.
"""
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

N = 2048          # grid points per side
MD = 4            # 4 x 4 markers per cell
THREADS = max(1, min(32, os.cpu_count() or 1))


def host(t):
    if t.dim() == 1:
        return t.cpu().numpy()
    return np.asfortranarray(t.t().contiguous().cpu().numpy().T)


@pytest.fixture(scope="module")
def flow(sf):
    m = sf.plume_model_unit_square()
    m.mu_air = 1e-2
    st = sf.StokesFlow2D(N, N, 1.0, 1.0, m, marker_density=MD, jitter=0.5, seed=0)
    st.deposit()
    torch.cuda.synchronize()
    return st


@pytest.fixture(scope="module")
def markers_host(flow):
    return tuple(t.cpu().numpy() for t in (flow.x_m, flow.y_m, flow.rho_m, flow.mu_m))


def test_fullsize_deposit_bitexact(flow, markers_host, oracle_lib):
    O = oracle_lib
    x, y, rho, mu = markers_host
    assert x.size == (MD * (N - 1)) ** 2
    o = flow.o
    for name, xo, yo, val in (("rho_vy", "x_rho", "y_rho", rho), ("mu_b", "x", "y", mu), ("mu_p", "x_p", "y_p", mu)):
        g = getattr(flow, name)
        want = O.zeros(*g.shape)
        vws, ws = O.zeros(N + 1, N), O.zeros(N + 1, N)
        O.bilinear_marker_to_grid(o[xo], o[yo], want, x, y, val, flow.dx, flow.dy, vws, ws)
        assert np.array_equal(host(g), want), f"{name} differs from the oracle"
    # the interpolation sums the GPU kept from its last deposit (mu on the cell centres), bit for bit
    assert np.array_equal(host(flow.wt_sum), ws) and np.array_equal(host(flow.val_wt_sum), vws)


NAMES = ["P", "Vx", "Vy", "rho_vy", "mu_b", "mu_p", "txx", "tyy", "txy", "divV", "dtPt", "Rx", "Ry", "dVxdt",
         "dVydt", "dtVx", "dtVy", "Vx_s", "Vy_s"]
ITERS = 60


@pytest.fixture(scope="module")
def solved(sf, flow, oracle_lib):
    """ITERS PT iterations on the GPU from the deposited fields (from rest, dt 0): the arrays and the info."""
    a = oracle_lib.stokes_arrays(N, N)
    for k in ("rho_vy", "mu_b", "mu_p"):
        a[k][:] = host(getattr(flow, k))
    dev = {k: torch.from_numpy(np.ascontiguousarray(v.T)).cuda().t() for k, v in a.items()}
    info = sf.solve_stokes_info(*[dev[k] for k in NAMES], 9.81, flow.dx, flow.dy, N, N, 0.0, 0.5,
                                use_free_surface_stabilization=True, eps=1e-300, iter_max=ITERS)
    return a, dev, info


def test_fullsize_pt_iterations_bitexact(flow, solved, oracle_lib):
    a, dev, info = solved
    r = oracle_lib.solve_stokes(a, 9.81, flow.dx, flow.dy, N, N, 0.0, 0.5, True, 1e-300, ITERS, nthreads=THREADS)
    assert info["iters"] == r.iters == ITERS and info["dt"] == r.dt
    for k in ("P", "Vx", "Vy", "dVxdt", "dVydt", "Vx_s", "Vy_s"):
        assert np.array_equal(host(dev[k]), a[k]), f"{k} differs from the oracle"
    assert np.abs(a["Vy"]).max() > 0


def test_fullsize_advection(sf, flow, solved, oracle_lib):
    O = oracle_lib
    o = flow.o
    _, dev, info = solved
    Vx, Vy, dt = dev["Vx"], dev["Vy"], info["dt"]
    assert np.isfinite(dt) and dt > 0
    g = torch.Generator(device="cuda").manual_seed(5)
    idx = torch.randperm(flow.n_markers, generator=g, device="cuda")[:1_000_000]
    xs, ys = flow.x_m[idx].contiguous(), flow.y_m[idx].contiguous()
    xh, yh = xs.cpu().numpy(), ys.cpu().numpy()
    sf.move_markers_rk4(xs, ys, Vx, Vy, o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, flow.lx, flow.ly, flow.dx,
                        flow.dy)
    O.move_markers_rk4(xh, yh, host(Vx), host(Vy), o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, flow.lx, flow.ly,
                       flow.dx, flow.dy, nthreads=THREADS)
    assert np.array_equal(xs.cpu().numpy(), xh) and np.array_equal(ys.cpu().numpy(), yh)
    assert not np.array_equal(xh, flow.x_m[idx].cpu().numpy()), "the sample did not move"
    x, y = flow.x_m.clone(), flow.y_m.clone()             # all 67 M
    sf.move_markers_rk4(x, y, Vx, Vy, o["x_vx"], o["y_vx"], o["x_vy"], o["y_vy"], dt, flow.lx, flow.ly, flow.dx,
                        flow.dy)
    assert bool(torch.isfinite(x).all()) and bool(torch.isfinite(y).all())
    assert float(x.min()) >= 0.0 and float(x.max()) <= flow.lx
    assert float(y.min()) >= 0.0 and float(y.max()) <= flow.ly
    assert torch.equal(x[idx], xs) and torch.equal(y[idx], ys)   # the sample moves the same inside the full set


def test_fullsize_rebin(sf, flow, oracle_lib):
    O = oracle_lib
    o = flow.o
    counts, offsets, perm = sf.rebin_markers(flow.x_m, flow.y_m, o["x"], o["y"], flow.dx, flow.dy, N, N)
    want, nout = O.cell_counts(flow.x_m.cpu().numpy(), flow.y_m.cpu().numpy(), o["x"], o["y"], flow.dx, flow.dy,
                               N, N)
    assert np.array_equal(counts.cpu().numpy(), want)
    assert nout == 0
    nm = flow.n_markers
    assert int(offsets[-1]) == nm
    p = perm[:nm].long()
    assert torch.equal(torch.sort(p).values, torch.arange(nm, device=p.device))
    cell = torch.repeat_interleave(torch.arange(counts.numel(), device=p.device), counts.long())
    same = cell[1:] == cell[:-1]
    assert bool((p[1:][same] > p[:-1][same]).all()), "not stable inside a cell"
