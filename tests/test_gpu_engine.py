"""Resident solve engine (sf_engine_*) and the serving loop on the GPU.

* an instance's result does not depend on what else is in the engine or when it joined: staggered
  admission gives the same bits as the blocking batch call and as solving it alone;
* admission control: SF_ERR_BUSY (None in Python) when the arena is full, SF_ERR_TOO_LARGE when the
  instance can never fit;
* serving: a request's final state is the same alone and in a mix of requests.
"""
import numpy as np
import pytest
import torch

from fields import solver_test_fields
from test_gpu_mixed import make_problem, host, plume_fields

pytestmark = pytest.mark.gpu


def specs_for(sizes):
    out = []
    for Nx, Ny in sizes:
        dx, dy = 1.0 / (Nx - 1), 1.0 / (Ny - 1)
        out.append((Nx, Ny, dx, dy, solver_test_fields(Nx, Ny, dx * 12.5, dy * 12.4)))
    return out


def problems(sf, specs, rtol=1e-8):
    arrs, probs = [], []
    for (Nx, Ny, dx, dy, f) in specs:
        a = make_problem(sf, Nx, Ny, dx, dy, f)
        arrs.append(a)
        probs.append(sf.MixedProblem(a["P"], a["Vx_pad"], a["Vy_pad"], a["rho_vy"], a["mu_b"], a["mu_p"], a["Vx_s"],
                                     a["Vy_s"], 9.81, dx, dy, Nx, Ny, 0.0, 0.5, rel_tol=rtol))
    return arrs, probs


def arena_for(sf, specs):
    return sum(sf.Engine.instance_bytes(s[0], s[1]) for s in specs)


def test_staggered_admission_matches_blocking_batch(sf):
    specs = specs_for([(40, 37), (64, 64), (100, 70), (33, 90), (129, 65)])
    opts = sf.mixed_options(fold_every=100)
    a_ref, p_ref = problems(sf, specs)
    sf.solve_stokes_batch_mixed(p_ref, options=opts)
    a_eng, p_eng = problems(sf, specs)
    with sf.Engine(arena_for(sf, specs), 8, options=opts) as eng:
        done = []
        # two join at once, the others one per round while the first ones iterate
        for p in p_eng[:2]:
            assert eng.submit(p) is not None
        for p in p_eng[2:]:
            done += eng.step()
            assert eng.submit(p) is not None
        while eng.active:
            done += eng.step()
        st = eng.stats()
    assert len(done) == len(specs) and st["finished"] == len(specs) and st["active"] == 0
    torch.cuda.synchronize()
    for q in range(len(specs)):
        assert p_eng[q].result["converged"] == 1
        assert p_eng[q].result["inner_iters"] == p_ref[q].result["inner_iters"]
        assert p_eng[q].result["dt_out"] == p_ref[q].result["dt_out"]
        for k in ("Vx_pad", "Vy_pad", "P", "Vx_s", "Vy_s"):
            assert torch.equal(a_eng[q][k], a_ref[q][k]), f"instance {q} {k}"


def test_admission_busy_then_admitted_and_too_large(sf):
    specs = specs_for([(64, 64), (60, 58)])
    one = max(sf.Engine.instance_bytes(s[0], s[1]) for s in specs)
    a_eng, p_eng = problems(sf, specs)
    a_solo, p_solo = problems(sf, specs[1:])
    sf.solve_stokes_batch_mixed(p_solo)
    with sf.Engine(one, 4) as eng:
        assert eng.submit(p_eng[0]) is not None
        assert eng.submit(p_eng[1]) is None          # arena full: not admitted, nothing changed
        rounds = 0
        while eng.active:
            eng.step()
            rounds += 1
        assert eng.submit(p_eng[1]) is not None      # room again
        while eng.active:
            eng.step()
        big = problems(sf, specs_for([(200, 200)]))[1][0]
        with pytest.raises(sf.StokesFlowError) as ei:
            eng.submit(big)
        assert ei.value.status == 6
        st = eng.stats()
        assert st["arena_used"] == 0 and st["arena_peak"] <= st["arena_bytes"]
    assert rounds >= 2
    torch.cuda.synchronize()
    for k in ("Vx_pad", "Vy_pad", "P"):
        assert torch.equal(a_eng[1][k], a_solo[0][k]), k


def test_engine_reports_diverging_instance(sf):
    """A 1000x stiff inclusion diverges under the reference's scheme: it leaves with SF_ERR_NONFINITE, the
    other instance is unaffected."""
    from test_gpu_mixed import inclusion_fields
    rho, mub, mup, dx, dy = inclusion_fields(sf, 48, 1e3)
    good = plume_fields(sf, 40)
    specs = [(48, 48, dx, dy, (rho, mub, mup)), (40, 40, good[3], good[4], good[:3])]
    a, p = problems(sf, specs)
    opts = sf.mixed_options(max_sweeps=200_000)
    with sf.Engine(arena_for(sf, specs), 4, options=opts) as eng:
        for x in p:
            assert eng.submit(x) is not None
        while eng.active:
            eng.step()
    assert p[0].result["status"] == 5 and p[1].result["status"] == 0 and p[1].result["converged"] == 1


def test_retry_rescues_a_diverging_layout(sf):
    """A 0.015-viscosity inclusion overlapping a 4.3 one (57^2 points): the reference's pseudo-time step
    diverges (non-finite after the first fold); with the default retry the instance restarts from its
    untouched inputs with the stencil-maximum step and converges -- to the same bits as a solve that used
    that step from the start, since the restart depends on nothing but the inputs."""
    from stokesflow_b200 import workloads
    N = 57
    m = workloads.InclusionModel(inclusions=[(0.41097438276340365, 0.5557518051240106, 0.1352829024064631,
                                               0.9281545598641852, 0.01517583353528039),
                                              (0.43634253798256306, 0.5888521117278834, 0.1352829024064631,
                                               1.1863722075708387, 4.262449612501063)])
    st = sf.StokesFlow2D(N, N, 1.0, 1.0, m, marker_density=4, jitter=0.5, seed=0, keep_work_arrays=False)
    st.deposit()
    f = (host(st.rho_vy), host(st.mu_b), host(st.mu_p))
    spec = [(N, N, st.dx, st.dy, f)]
    runs = {}
    for name, opts in (("plain", dict(retry_local_max=False)), ("retry", {}), ("local_max", dict(dtau_local_max=True))):
        arrs, probs = problems(sf, spec)
        res = sf.solve_stokes_batch_mixed(probs, options=sf.mixed_options(max_sweeps=400_000, **opts))
        runs[name] = (arrs[0], res[0])
    assert runs["plain"][1]["status"] == 5 and runs["plain"][1]["retried"] == 0
    r, l = runs["retry"][1], runs["local_max"][1]
    assert r["status"] == 0 and r["converged"] == 1 and r["retried"] == 1
    assert l["converged"] == 1 and l["retried"] == 0
    assert r["inner_iters"] > l["inner_iters"]            # the diverged attempt's sweeps count too
    for k in ("Vx_pad", "Vy_pad", "P"):
        assert torch.equal(runs["retry"][0][k], runs["local_max"][0][k]), k


def test_serving_same_alone_and_in_mix(sf):
    from stokesflow_b200 import serving
    reqs = serving.poisson_requests(4, rate=0.0, seed=3, cells=(31, 90), timesteps=(2, 3))
    with_mix = serving.StokesServer(1 << 30, keep_final=True, options=sf.mixed_options(fold_every=100))
    summary = with_mix.run(reqs)
    with_mix.close()
    assert summary["completed"] == 4 and summary["solves"] == sum(r.timesteps for r in reqs)
    assert summary["converged_solves"] == summary["solves"]
    for r in reqs:
        alone = serving.poisson_requests(4, rate=0.0, seed=3, cells=(31, 90), timesteps=(2, 3))[r.rid]
        srv = serving.StokesServer(1 << 30, keep_final=True, options=sf.mixed_options(fold_every=100))
        srv.run([alone])
        srv.close()
        for k in ("P", "Vx", "Vy", "x_m", "y_m"):
            assert np.array_equal(alone.final[k], r.final[k]), f"request {r.rid} {k}"
        assert alone.final["t_tot"] == r.final["t_tot"]


def test_serving_admission_by_budget(sf):
    """A budget that holds about one request's state at a time: the rest wait in arrival order, the peak
    stays within the budget, and every request ends with the same results as with room for all."""
    from stokesflow_b200 import serving
    kw = dict(rate=0.0, seed=9, cells=(40, 60), timesteps=(1, 2))
    reqs = serving.poisson_requests(3, **kw)
    biggest = max(serving.state_bytes(r.spec) for r in reqs)
    opts = sf.mixed_options(fold_every=100)
    tight = serving.StokesServer(2 * biggest + biggest // 2, engine_share=0.5, keep_final=True, options=opts)
    s = tight.run(reqs)
    assert s["completed"] == 3 and s["failed"] == 0
    assert tight.peak_state <= tight.state_budget
    assert tight.peak_state < sum(serving.state_bytes(r.spec) for r in reqs)   # they did not all fit at once
    order = sorted(reqs, key=lambda r: r.t_admit)
    assert [r.rid for r in order] == [0, 1, 2]
    tight.close()
    roomy_reqs = serving.poisson_requests(3, **kw)
    roomy = serving.StokesServer(1 << 30, keep_final=True, options=opts)
    roomy.run(roomy_reqs)
    roomy.close()
    for a, b in zip(reqs, roomy_reqs):
        for k in ("P", "Vx", "Vy", "x_m", "y_m"):
            assert np.array_equal(a.final[k], b.final[k]), f"request {a.rid} {k}"


def test_serving_state_bytes_and_fp64_server(sf):
    from stokesflow_b200 import serving
    reqs = serving.poisson_requests(2, rate=0.0, seed=5, cells=(31, 50), timesteps=(1, 2))
    st = serving.StokesServer(1 << 30, solver="fp64")._new_state(reqs[0])
    assert serving.state_bytes(reqs[0].spec) == st.device_bytes()
    srv = serving.StokesServer(1 << 30, solver="fp64")
    s = srv.run(reqs)
    assert s["completed"] == 2 and s["converged_solves"] == s["solves"]
    assert s["p99_latency_s"] >= s["p50_latency_s"] > 0
