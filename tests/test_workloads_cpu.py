"""Host-side logic of the batched and served forms (no GPU): seeded workloads, material assignment,
admission sizes and the latency summary."""
import math

import numpy as np
import torch

from stokesflow_b200 import serving, workloads


def test_batch_specs_are_seeded_and_in_range():
    a = workloads.batch_specs(64, seed=11)
    b = workloads.batch_specs(64, seed=11)
    c = workloads.batch_specs(64, seed=12)
    key = lambda s: [(x.Nx, x.Ny, x.md, x.model.inclusions) for x in s]  # noqa: E731
    assert key(a) == key(b) and key(a) != key(c)
    for s in a:
        assert 128 <= s.Nx <= 1024 and 128 <= s.Ny <= 1024 and 3 <= s.md <= 5
        assert 1 <= len(s.model.inclusions) <= 3
        inc = s.model.inclusions
        for (cx, cy, r, rho, mu) in inc:
            assert 0.05 <= r <= 0.2 and 0.8 <= rho <= 1.2 and 1e-2 <= mu <= 1e1
            assert cy - r >= 0.1 + 0.05 - 1e-12  # clear of the air layer
        for i in range(len(inc)):                 # and of each other, by a gap of matrix
            for j in range(i):
                d = math.hypot(inc[i][0] - inc[j][0], inc[i][1] - inc[j][1])
                assert d >= inc[i][2] + inc[j][2] + workloads.INCLUSION_GAP - 1e-12


def test_log_uniform_sizes_cover_the_range():
    rng = np.random.default_rng(0)
    xs = np.array([workloads.log_uniform_int(rng, 127, 1023) for _ in range(4000)])
    assert xs.min() >= 127 and xs.max() <= 1023
    # log-uniform: the median sits near the geometric mean
    assert abs(math.log(np.median(xs)) - 0.5 * (math.log(127) + math.log(1023))) < 0.1


def test_inclusion_model_properties():
    m = workloads.InclusionModel(air_height=0.1, rho_air=1e-3, mu_air=1e-2,
                                 inclusions=[(0.5, 0.5, 0.2, 1.2, 10.0), (0.6, 0.5, 0.1, 0.8, 0.05)])
    x = torch.tensor([0.4, 0.6, 0.9, 0.5, 0.05], dtype=torch.float64)
    y = torch.tensor([0.5, 0.5, 0.9, 0.05, 0.95], dtype=torch.float64)
    rho, mu = m.marker_properties(x, y)
    assert rho.tolist() == [1.2, 0.8, 1.0, 1e-3, 1.0]      # later inclusion wins, air wins over all
    assert mu.tolist() == [10.0, 0.05, 1.0, 1e-2, 1.0]


def test_poisson_trace():
    r = serving.poisson_requests(400, rate=5.0, seed=2, cells=(63, 2047), timesteps=(1, 20))
    t = np.array([q.arrival for q in r])
    assert np.all(np.diff(t) > 0)
    assert abs(np.mean(np.diff(t)) - 0.2) < 0.03            # mean inter-arrival 1/rate
    assert all(64 <= q.spec.Nx <= 2048 and q.spec.Nx == q.spec.Ny and 1 <= q.timesteps <= 20 for q in r)
    r0 = serving.poisson_requests(3, rate=0.0, seed=2)
    assert all(q.arrival == 0.0 for q in r0)


def test_state_bytes_formula():
    spec = workloads.InstanceSpec(10, 7, 3, workloads.InclusionModel(), 0)
    Nx, Ny = 10, 7
    grids = [(Nx - 1, Ny - 1), (Nx + 2, Ny + 1), (Nx + 1, Ny + 2), (Nx + 1, Ny), (Nx, Ny), (Nx - 1, Ny - 1),
             (Nx - 2, Ny - 1), (Nx - 1, Ny - 2), (Nx, Ny + 1), (Nx + 1, Ny)]
    assert serving.state_bytes(spec) == 8 * (4 * 9 * (Nx - 1) * (Ny - 1) + sum(a * b for a, b in grids))


def test_summary_percentiles():
    reqs = []
    for k, lat in enumerate([1.0, 2.0, 3.0, 10.0]):
        q = serving.Request(k, None, 2, arrival=float(k))
        q.t_done = q.arrival + lat
        q.solves = 2
        reqs.append(q)
    s = serving.summarize(reqs)
    assert s["completed"] == 4 and s["solves"] == 8
    assert s["p50_latency_s"] == 2.5 and abs(s["p99_latency_s"] - 9.79) < 1e-9
    assert s["makespan_s"] == 13.0 - 0.0 and abs(s["solves_per_s"] - 8 / 13.0) < 1e-12
