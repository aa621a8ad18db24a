"""Mixed-precision / batched solver (sf_solve_stokes_batch_mixed) on the GPU.

* accuracy at the tolerance the forms are timed at: the FP64 oracle of a mixed solve is the plain FP64
  solver (bit-identical to the reference's solveStokes!) on the same inputs and the same relative
  residual 1e-6.  The mixed solve keeps the reference loop's schedule (dt updates every ndtupdate,
  residual checks every ncheck, the reference's check quantities), so it stops at the same iteration,
  and its V and P lie within REL_L2_BAR (the required 1e-5) of the oracle's, relative L2;
* batch invariance: an instance solved inside a batch of differently sized instances gives
  bit-identical results to the same instance solved alone (its arithmetic and its stopping decisions
  depend only on itself).
"""
import numpy as np
import pytest
import torch

from fields import rel_l2, solver_test_fields

pytestmark = pytest.mark.gpu

REL_L2_BAR = 1e-5     # relative L2 error against the FP64 oracle, at relative residual 1e-6
RTOL = 1e-6


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)).cuda().t()


def host(t):
    return np.asfortranarray(t.t().contiguous().cpu().numpy().T)


def make_problem(sf, Nx, Ny, dx, dy, fields, dt=0.0):
    rho, mub, mup = fields
    z = sf.zeros
    a = dict(P=z(Nx - 1, Ny - 1), Vx_pad=z(Nx + 2, Ny + 1), Vy_pad=z(Nx + 1, Ny + 2), rho_vy=dev(rho), mu_b=dev(mub),
             mu_p=dev(mup), Vx_s=z(Nx, Ny + 1), Vy_s=z(Nx + 1, Ny))
    return a


def plume_fields(sf, N, mu_air=1e-2):
    """rho_vy, mu_b, mu_p of the unit-square plume model deposited from markers (one timestep's input)."""
    m = sf.plume_model_unit_square()
    m.mu_air = mu_air
    st = sf.StokesFlow2D(N, N, 1.0, 1.0, m, marker_density=4, jitter=0.5, seed=0, keep_work_arrays=False)
    st.deposit()
    return host(st.rho_vy), host(st.mu_b), host(st.mu_p), st.dx, st.dy


def fp64_solve(sf, Nx, Ny, dx, dy, fields, rtol):
    a = make_problem(sf, Nx, Ny, dx, dy, fields)
    z = sf.zeros
    scale = sf.residual_scale(a["rho_vy"], Nx, Ny, 9.81)
    info = sf.solve_stokes_info(a["P"], a["Vx_pad"], a["Vy_pad"], a["rho_vy"], a["mu_b"], a["mu_p"], None, None, None,
                                None, None, None, None, z(Nx - 2, Ny - 1), z(Nx - 1, Ny - 2), None, None, a["Vx_s"],
                                a["Vy_s"], 9.81, dx, dy, Nx, Ny, 0.0, 0.5, eps=rtol * scale, iter_max=2_000_000)
    return {k: host(v) for k, v in a.items()}, info


def mixed_solve(sf, problems_spec, rtol, **opts):
    probs, arrs = [], []
    for (Nx, Ny, dx, dy, fields) in problems_spec:
        a = make_problem(sf, Nx, Ny, dx, dy, fields)
        arrs.append(a)
        probs.append(sf.MixedProblem(a["P"], a["Vx_pad"], a["Vy_pad"], a["rho_vy"], a["mu_b"], a["mu_p"], a["Vx_s"],
                                     a["Vy_s"], 9.81, dx, dy, Nx, Ny, 0.0, 0.5, rel_tol=rtol))
    res = sf.solve_stokes_batch_mixed(probs, options=sf.mixed_options(**opts) if opts else None)
    return [{k: host(v) for k, v in a.items()} for a in arrs], res


def assert_matches_oracle(got, res, ref, info, what):
    """The mixed result against the FP64 oracle's at the same tolerance: same stopping iteration, V and P
    within the bar."""
    assert res["status"] == 0 and res["converged"] == 1 and info["converged"] == 1, (what, res, info)
    assert res["inner_iters"] == info["iters"], f"{what}: stopped at {res['inner_iters']}, FP64 at {info['iters']}"
    for k in ("Vx_pad", "Vy_pad", "P"):
        e = rel_l2(got[k], ref[k])
        assert e <= REL_L2_BAR, f"{what} {k}: relative L2 {e:.2e} against the FP64 oracle"


def test_mixed_meets_the_bar_at_rtol_1e6_plume(sf):
    """The benchmark's plume model at 127 x 127 cells, cold start, relative residual 1e-6: the mixed solve
    stops at the FP64 solver's iteration and is within 1e-5 of its V and P."""
    rho, mub, mup, dx, dy = plume_fields(sf, 128)
    f = (rho, mub, mup)
    ref, info = fp64_solve(sf, 128, 128, dx, dy, f, RTOL)
    (got,), (r,) = mixed_solve(sf, [(128, 128, dx, dy, f)], RTOL)
    assert_matches_oracle(got, r, ref, info, "plume 127^2")
    assert abs(r["dt_out"] - info["dt"]) <= 1e-5 * abs(info["dt"])
    # the same boundary identities as the reference's solver test (test_StokesSolver.jl:128-140)
    Vx, Vy = got["Vx_pad"], got["Vy_pad"]
    assert np.all(Vx[0, :] == -Vx[2, :]) and np.all(Vx[1, :] == 0.0) and np.all(Vx[:, 0] == Vx[:, 1])
    assert np.all(Vy[:, 0] == -Vy[:, 2]) and np.all(Vy[:, 1] == 0.0) and np.all(Vy[0, :] == Vy[1, :])


def test_mixed_meets_the_bar_on_random_inclusions(sf):
    """A batch of random-inclusion instances of uneven grids (the batching workload's sampler, smaller
    grids) at relative residual 1e-6: every instance stops at its FP64 solve's iteration and is within 1e-5
    of it."""
    from stokesflow_b200.workloads import batch_specs
    specs = batch_specs(8, seed=3, cells=(31, 160))
    spec_f = []
    for s in specs:
        st = sf.StokesFlow2D(s.Nx, s.Ny, 1.0, 1.0, s.model, marker_density=s.md, jitter=0.5, seed=s.seed,
                             keep_work_arrays=False)
        st.deposit()
        spec_f.append((s.Nx, s.Ny, st.dx, st.dy, (host(st.rho_vy), host(st.mu_b), host(st.mu_p))))
    got, res = mixed_solve(sf, spec_f, RTOL)
    for q, (Nx, Ny, dx, dy, f) in enumerate(spec_f):
        ref, info = fp64_solve(sf, Nx, Ny, dx, dy, f, RTOL)
        assert_matches_oracle(got[q], res[q], ref, info, f"instance {q} ({Nx}x{Ny})")


def test_mixed_timesteps_match_fp64(sf):
    """Three timesteps of the plume model (63 x 63 cells, 16 markers per cell) with the mixed solver against
    the plain FP64 path, each carrying its own state (V, P, damped rates, dt, markers) forward: every solve
    stops at the FP64 iteration, and V, P and the marker positions stay within 1e-5."""
    m = sf.plume_model_unit_square()
    m.mu_air = 1e-2
    runs = {}
    for solver in ("fp64", "mixed"):
        st = sf.StokesFlow2D(64, 64, 1.0, 1.0, m, marker_density=4, jitter=0.5, seed=0, stokes_rtol=RTOL,
                             keep_work_arrays=False, solver=solver, iter_max=2_000_000)
        iters = [int(st.step()["info"]["iters"]) for _ in range(3)]
        runs[solver] = (st, iters)
    (a, ia), (b, ib) = runs["fp64"], runs["mixed"]
    assert ia == ib, (ia, ib)
    for k in ("Vx", "Vy", "P", "x_m", "y_m"):
        ta, tb = getattr(a, k), getattr(b, k)
        e = rel_l2(tb.detach().cpu().numpy(), ta.detach().cpu().numpy())
        assert e <= REL_L2_BAR, f"{k}: {e:.2e}"
    assert abs(a.t_tot - b.t_tot) <= 1e-5 * a.t_tot


def test_mixed_tight_tolerance_reaches_the_converged_solution(sf):
    """FP32 sweeps with FP64 correction are not limited by FP32 rounding: the mixed solve reaches an FP64
    residual of 1e-10 relative (far below FP32's 6e-8 unit roundoff), where it is within 2e-6 in V and
    1e-7 in P of the FP64 solution converged to 1e-11.  The remaining distance is convergence, which the
    stopping tolerance sets for both solvers: against the FP64 solver stopped at the same 1e-10 it is within
    1e-7."""
    rho, mub, mup, dx, dy = plume_fields(sf, 64)
    f = (rho, mub, mup)
    ref, info = fp64_solve(sf, 64, 64, dx, dy, f, 1e-11)
    same, info10 = fp64_solve(sf, 64, 64, dx, dy, f, 1e-10)
    assert info["converged"] == 1 and info10["converged"] == 1
    (mix, ), (r, ) = mixed_solve(sf, [(64, 64, dx, dy, f)], 1e-10)
    assert r["converged"] == 1 and r["status"] == 0 and r["err"] <= r["eps_used"]
    assert r["inner_iters"] == info10["iters"]
    for k in ("Vx_pad", "Vy_pad", "P"):
        assert rel_l2(mix[k], ref[k]) <= (1e-7 if k == "P" else 2e-6), f"{k}: against the converged solution"
        assert rel_l2(mix[k], same[k]) <= 1e-7, f"{k}: against FP64 at 1e-10"


def test_mixed_golden_solver_case(sf):
    """test/test_StokesSolver.jl's case through the mixed path, against the FP64 path."""
    Nx, Ny, dx, dy = 26, 32, 0.5, 0.4
    f = solver_test_fields(Nx, Ny, dx, dy)
    ref, _ = fp64_solve(sf, Nx, Ny, dx, dy, f, 1e-12)
    (got,), (r,) = mixed_solve(sf, [(Nx, Ny, dx, dy, f)], 1e-10)
    assert r["converged"] == 1
    assert rel_l2(got["Vx_pad"], ref["Vx_pad"]) <= 1e-7 and rel_l2(got["Vy_pad"], ref["Vy_pad"]) <= 1e-7


def test_batch_is_bit_identical_to_solo(sf):
    rng = np.random.default_rng(7)
    specs = []
    for Nx, Ny in [(40, 37), (64, 64), (100, 70), (33, 90), (129, 65)]:
        dx, dy = 1.0 / (Nx - 1), 1.0 / (Ny - 1)
        specs.append((Nx, Ny, dx, dy, solver_test_fields(Nx, Ny, dx * 12.5 / 1.0, dy * 12.4 / 1.0)))
    rng.shuffle(specs)
    batch, res_b = mixed_solve(sf, specs, 1e-8, fold_every=100)
    for q, spec in enumerate(specs):
        (solo,), (r,) = mixed_solve(sf, [spec], 1e-8, fold_every=100)
        assert r["converged"] == 1 and res_b[q]["converged"] == 1
        assert r["inner_iters"] == res_b[q]["inner_iters"]
        for k in ("Vx_pad", "Vy_pad", "P"):
            assert np.array_equal(batch[q][k], solo[k]), f"instance {q} {k} differs in the batch"


def inclusion_fields(sf, N, mu_inc, mu_air=1e-2, rho_inc=1.1):
    m = sf.PlumeModel(air_height=0.1, plume_x=0.5, plume_y=0.6, plume_r=0.15, rho_air=1e-3, rho_matrix=1.0,
                      rho_plume=rho_inc, mu_air=mu_air, mu_matrix=1.0, mu_plume=mu_inc)
    st = sf.StokesFlow2D(N, N, 1.0, 1.0, m, marker_density=4, jitter=0.5, seed=0, keep_work_arrays=False)
    st.deposit()
    return host(st.rho_vy), host(st.mu_b), host(st.mu_p), st.dx, st.dy


def test_local_max_dtau_same_solution(sf):
    """The pseudo-time step only preconditions the iteration: with the reference's averaged dtau and with
    the stencil-maximum dtau the mixed solver reaches the same discrete solution (a 10x stiff inclusion,
    where the reference's scheme converges)."""
    rho, mub, mup, dx, dy = inclusion_fields(sf, 64, 10.0)
    f = (rho, mub, mup)
    (a,), (ra,) = mixed_solve(sf, [(64, 64, dx, dy, f)], 1e-10, dtau_local_max=False)
    (b,), (rb,) = mixed_solve(sf, [(64, 64, dx, dy, f)], 1e-10, dtau_local_max=True)
    assert ra["converged"] == 1 and rb["converged"] == 1
    for k in ("Vx_pad", "Vy_pad", "P"):
        assert rel_l2(a[k], b[k]) <= REL_L2_BAR, k


@pytest.mark.parametrize("local_max", [False, True])
def test_soft_inclusion_converges(sf, local_max):
    """A 100x soft inclusion converges to relative residual 1e-8 with either pseudo-time step."""
    rho, mub, mup, dx, dy = inclusion_fields(sf, 64, 1e-2)
    (a,), (r,) = mixed_solve(sf, [(64, 64, dx, dy, (rho, mub, mup))], 1e-8, dtau_local_max=local_max)
    assert r["status"] == 0 and r["converged"] == 1, r
    assert np.all(np.isfinite(a["Vx_pad"])) and np.all(np.isfinite(a["P"]))


def test_diverging_instance_reports_nonfinite_and_leaves_others(sf):
    """A 1000x stiff inclusion diverges under the reference's scheme (NaN on the CPU oracle as well): the
    instance ends with SF_ERR_NONFINITE while a well-posed instance in the same batch converges to the
    same bits as alone."""
    rho, mub, mup, dx, dy = inclusion_fields(sf, 48, 1e3)
    good = plume_fields(sf, 40)
    specs = [(48, 48, dx, dy, (rho, mub, mup)), (40, 40, good[3], good[4], good[:3])]
    batch, res = mixed_solve(sf, specs, 1e-8, max_sweeps=200_000)
    (solo,), (rs,) = mixed_solve(sf, specs[1:], 1e-8, max_sweeps=200_000)
    assert res[0]["status"] == 5 and res[0]["converged"] == 0, res[0]
    assert res[1]["status"] == 0 and res[1]["converged"] == 1 and rs["converged"] == 1
    for k in ("Vx_pad", "Vy_pad", "P"):
        assert np.array_equal(batch[1][k], solo[k]), k


def test_mixed_without_graphs_matches_graphs(sf):
    rho, mub, mup, dx, dy = plume_fields(sf, 48)
    (a,), _ = mixed_solve(sf, [(48, 48, dx, dy, (rho, mub, mup))], 1e-8, use_graphs=False)
    (b,), _ = mixed_solve(sf, [(48, 48, dx, dy, (rho, mub, mup))], 1e-8, use_graphs=True)
    assert np.array_equal(a["Vx_pad"], b["Vx_pad"]) and np.array_equal(a["P"], b["P"])
