"""Where the reference's pseudo-transient scheme converges, on the CPU oracle.

The reference's iteration (StokesSolver_multixpu.jl:14-96: Vdmp = 4, Vsc = 0.45,
Ptsc = 1/2, the pseudo-time step Vsc min(dx,dy)^2 / av(mu_p) / 4.1 of
compute_timesteps!, :128-133) converges only for a band of viscosity contrasts.
These tests run the oracle's restatement of that iteration, unchanged, on a
63 x 63 cell unit square with the sticky-air layer (mu 1e-2, rho 1e-3, y < 0.1)
and one circular body of viscosity mu_body in a matrix of mu = 1, and assert
on which side of the band each case falls:

* stiff bodies (radius 0.15 at (0.5, 0.6), rho 1.1): 20x converges to relative
  residual 1e-6, 50x diverges (the residual grows without bound);
* soft bodies (the benchmark's plume, radius 0.1 at (0.5, 0.75), rho 0.9):
  1e-2 converges, 1e-3 diverges (non-finite within a few hundred iterations).

Measured on the oracle across grids of 31 to 127 cells: stiff bodies converge
up to 20x and diverge from 30x (30x converges only on the 31-cell grid); soft
bodies converge down to 1e-2 (3e-3 on the 127-cell grid) and diverge from
3e-3 (1e-3 on the 127-cell grid).  The batching and serving workloads draw
body viscosities inside this band (workloads.batch_specs: 10**[-2, 1]); the
checks below keep that default inside it.
"""
import numpy as np
import pytest

N = 64            # grid points per side (63 cells)
RTOL = 1e-6
STIFF = (0.5, 0.6, 0.15, 1.1)
SOFT = (0.5, 0.75, 0.1, 0.9)


def solve(O, mu_body, body, iter_max):
    dx = dy = 1.0 / (N - 1)
    bx, by, br, brho = body
    m = O.PlumeModel(air_height=0.1, plume_x=bx, plume_y=by, plume_r=br, rho_air=1e-3, rho_matrix=1.0,
                     rho_plume=brho, mu_air=1e-2, mu_matrix=1.0, mu_plume=mu_body)
    x, y = O.initialize_markers(4, 1.0, 1.0, dx, dy, N, N, 0.5, 0)
    rho, mu = O.set_marker_properties(m, x, y)
    arr = O.stokes_arrays(N, N)
    o = O.node_origins(dx, dy)
    vws, ws = O.zeros(N + 1, N), O.zeros(N + 1, N)
    O.bilinear_marker_to_grid(o["x_rho"], o["y_rho"], arr["rho_vy"], x, y, rho, dx, dy, vws, ws)
    O.bilinear_marker_to_grid(o["x"], o["y"], arr["mu_b"], x, y, mu, dx, dy, vws, ws)
    O.bilinear_marker_to_grid(o["x_p"], o["y_p"], arr["mu_p"], x, y, mu, dx, dy, vws, ws)
    # relative residual: eps = rtol * mean|g_y rho_vy| over the Ry interior (the residual of V = P = 0)
    scale = float(np.mean(np.abs(9.81 * arr["rho_vy"][1:N, 1:N - 1])))
    r = O.solve_stokes(arr, 9.81, dx, dy, N, N, 0.0, 0.5, True, RTOL * scale, iter_max, 4)
    return r.err / scale, r.iters


@pytest.mark.parametrize("mu_body, body", [(20.0, STIFF), (1e-2, SOFT)], ids=["stiff_20x", "soft_1e-2"])
def test_inside_the_band_converges(oracle_lib, mu_body, body):
    err, iters = solve(oracle_lib, mu_body, body, 100_000)
    assert err <= RTOL, (err, iters)


@pytest.mark.parametrize("mu_body, body", [(50.0, STIFF), (1e-3, SOFT)], ids=["stiff_50x", "soft_1e-3"])
def test_outside_the_band_diverges(oracle_lib, mu_body, body):
    err, iters = solve(oracle_lib, mu_body, body, 60_000)
    assert not (err <= 1.0), f"relative residual {err:.3g} after {iters} iterations: expected divergence"


def test_workload_viscosities_lie_inside_the_band():
    import inspect
    from stokesflow_b200 import workloads
    lo, hi = inspect.signature(workloads.batch_specs).parameters["mu_log10"].default
    assert 10.0 ** lo >= 1e-2 and 10.0 ** hi <= 20.0
