"""The serving loop's host logic on the CPU: HBM-budget admission, continuous batching, the waiting line
for a full engine arena, and a failed solve ending only its own request.

The engine and the per-request timestep state are replaced by fakes that count rounds; the loop itself
(`StokesServer._run_mixed`) is the product code.  The numerics of the served solves are covered by the
GPU tests (each result the same alone and in the mix)."""
import time

import pytest

from stokesflow_b200 import serving
from stokesflow_b200.workloads import InstanceSpec


class FakeProblem:
    def __init__(self, rid, rounds, fail):
        self.rid, self.rounds, self.fail = rid, rounds, fail
        self.done_rounds = 0
        self.result = None


class FakeEngine:
    """An arena of `slots` solves; every step is one round of every solve in it."""
    slots = 2
    log = []

    def __init__(self, arena, max_instances, options=None, ctx=None):
        self.in_arena = []
        FakeEngine.log = []

    @property
    def active(self):
        return len(self.in_arena)

    def submit(self, problem, stream=None):
        if len(self.in_arena) >= FakeEngine.slots:
            return None
        self.in_arena.append(problem)
        return len(self.in_arena)

    def step(self, stream=None):
        time.sleep(0.002)
        FakeEngine.log.append(sorted({p.rid for p in self.in_arena}))
        done = []
        for p in list(self.in_arena):
            p.done_rounds += 1
            if p.done_rounds >= p.rounds:
                p.result = {"converged": int(not p.fail), "inner_iters": 8 * p.rounds, "status": 5 if p.fail else 0}
                self.in_arena.remove(p)
                done.append(p)
        return done

    def close(self):
        pass


class FakeState:
    """A request's timestep state: seed encodes (request id, rounds per solve, failing solve or -1)."""

    def __init__(self, Nx, Ny, lx, ly, model, *, seed, **kw):
        self.rid, self.rounds, self.fail_at = seed
        self.steps = 0

    def begin_timestep(self):
        return FakeProblem(self.rid, self.rounds, self.steps == self.fail_at)

    def end_timestep(self, result):
        assert result["status"] == 0
        self.steps += 1


class FakeStream:
    def synchronize(self):
        pass


@pytest.fixture
def server(monkeypatch):
    monkeypatch.setattr(serving.api, "Engine", FakeEngine)
    monkeypatch.setattr(serving.api, "default_context", lambda: object())
    monkeypatch.setattr(serving, "StokesFlow2D", FakeState)
    monkeypatch.setattr(serving.torch.cuda, "current_stream", lambda: FakeStream())
    seen = []
    orig = serving.StokesServer._new_state

    def new_state(self, r):   # called once the request's bytes are counted in state_used
        seen.append((r.rid, self.state_used, self.state_budget))
        return orig(self, r)

    monkeypatch.setattr(serving.StokesServer, "_new_state", new_state)
    return seen


def request(rid, n, timesteps, arrival, rounds=3, fail_at=-1, md=3):
    return serving.Request(rid, InstanceSpec(n, n, md, None, (rid, rounds, fail_at)), timesteps, arrival)


def test_budget_bounds_the_admitted_state(server):
    reqs = [request(k, 33, 2, 0.0) for k in range(6)]
    one = serving.state_bytes(reqs[0].spec)
    srv = serving.StokesServer(4 * one + 1, solver="mixed", engine_share=0.5)   # room for 2 requests' state
    FakeEngine.slots = 8
    out = srv.run(reqs)
    assert out["completed"] == 6 and out["failed"] == 0 and out["solves"] == 12
    assert srv.peak_state == 2 * one <= srv.state_budget
    assert all(used <= budget for _, used, budget in server)
    assert max(len(ids) for ids in FakeEngine.log) == 2
    assert srv.state_used == 0
    # arrival order is kept: admission times never decrease with the request id
    assert [r.rid for r in sorted(reqs, key=lambda r: (r.t_admit, r.rid))] == list(range(6))


def test_an_oversized_request_runs_alone(server):
    small = serving.state_bytes(request(0, 33, 1, 0.0).spec)
    reqs = [request(0, 33, 1, 0.0), request(1, 129, 1, 0.0), request(2, 33, 1, 0.0)]
    srv = serving.StokesServer(2 * (2 * small), solver="mixed", engine_share=0.5)  # 2 small ones fit, the big not
    FakeEngine.slots = 8
    out = srv.run(reqs)
    assert out["completed"] == 3
    big = [s for s in server if s[0] == 1][0]
    assert big[1] == serving.state_bytes(reqs[1].spec) > big[2]   # admitted only once nothing else held state
    assert [1] in FakeEngine.log and not any(1 in ids and len(ids) > 1 for ids in FakeEngine.log)


def test_a_late_request_joins_while_others_run(server):
    reqs = [request(0, 33, 1, 0.0, rounds=150), request(1, 33, 2, 0.05, rounds=5)]
    srv = serving.StokesServer(1 << 40, solver="mixed")
    FakeEngine.slots = 8
    srv.run(reqs)
    assert reqs[1].t_admit < reqs[0].t_done
    assert reqs[1].t_done < reqs[0].t_done   # the short request does not wait for the long one
    assert any(ids == [0, 1] for ids in FakeEngine.log)


def test_full_arena_holds_solves_in_line(server):
    reqs = [request(k, 33, 3, 0.0, rounds=2 + k) for k in range(5)]
    srv = serving.StokesServer(1 << 40, solver="mixed")
    FakeEngine.slots = 2
    out = srv.run(reqs)
    assert out["completed"] == 5 and out["solves"] == 15
    assert max(len(ids) for ids in FakeEngine.log) == 2
    assert all(r.solves == 3 and r.converged == 3 for r in reqs)


def test_a_failed_solve_ends_only_its_request(server):
    reqs = [request(0, 33, 4, 0.0), request(1, 33, 4, 0.0, fail_at=1), request(2, 33, 4, 0.0)]
    srv = serving.StokesServer(1 << 40, solver="mixed")
    FakeEngine.slots = 8
    out = srv.run(reqs)
    assert out["completed"] == 3 and out["failed"] == 1
    assert reqs[1].failed and reqs[1].solves == 2 and reqs[1].converged == 1
    assert not reqs[0].failed and reqs[0].solves == 4 and not reqs[2].failed and reqs[2].solves == 4
    assert srv.state_used == 0


def test_summary_of_the_served_trace(server):
    reqs = [request(k, 33, 1 + k % 3, 0.01 * k) for k in range(8)]
    srv = serving.StokesServer(1 << 40, solver="mixed")
    FakeEngine.slots = 4
    out = srv.run(reqs)
    assert out["completed"] == 8 and out["solves"] == sum(1 + k % 3 for k in range(8))
    assert 0 < out["p50_latency_s"] <= out["p99_latency_s"]
    assert all(r.t_admit >= r.arrival and r.t_done >= r.t_admit for r in reqs)


def _concurrent_fakes(monkeypatch):
    """Fakes for the plain FP64 server's workers: no device, a request 'solve' is a sleep."""
    import contextlib
    import threading

    class Ctx:
        def __init__(self, device=None):
            pass

        def close(self):
            pass

    monkeypatch.setattr(serving.api, "default_context", lambda: object())
    monkeypatch.setattr(serving.api, "Context", Ctx)
    monkeypatch.setattr(serving.torch.cuda, "current_device", lambda: 0)
    monkeypatch.setattr(serving.torch.cuda, "set_device", lambda d: None)
    monkeypatch.setattr(serving.torch.cuda, "Stream", lambda: None)
    monkeypatch.setattr(serving.torch.cuda, "stream", lambda s: contextlib.nullcontext())
    monkeypatch.setattr(serving.torch.cuda, "synchronize", lambda d=None: None)
    lock = threading.Lock()
    seen = {"running": 0, "peak": 0, "starts": []}

    def serve(self, r, ctx=None):
        with lock:
            seen["running"] += 1
            seen["peak"] = max(seen["peak"], seen["running"])
            seen["starts"].append(r.rid)
        time.sleep(0.02 * r.timesteps)
        r.solves = r.converged = r.timesteps
        with lock:
            seen["running"] -= 1

    monkeypatch.setattr(serving.StokesServer, "_serve_fp64", serve)
    return seen


def test_concurrent_fp64_server_keeps_order_workers_and_budget(monkeypatch):
    """The plain FP64 server with K workers: requests start in arrival order, at most K run at once, the HBM
    budget bounds the state held, and every request completes once."""
    seen = _concurrent_fakes(monkeypatch)
    reqs = [request(k, 33, 1 + k % 3, 0.005 * k) for k in range(9)]
    srv = serving.StokesServer(1 << 40, solver="fp64", concurrency=3)
    out = srv.run(reqs)
    assert out["completed"] == 9 and out["solves"] == sum(1 + k % 3 for k in range(9))
    assert seen["starts"] == list(range(9)) and seen["peak"] == 3
    assert srv.state_used == 0 and all(r.t_done >= r.t_admit >= r.arrival for r in reqs)

    seen = _concurrent_fakes(monkeypatch)
    reqs = [request(k, 33, 2, 0.0) for k in range(6)]
    one = serving.state_bytes(reqs[0].spec)
    srv = serving.StokesServer(2 * one, solver="fp64", concurrency=4)     # room for two requests' state
    out = srv.run(reqs)
    assert out["completed"] == 6 and seen["peak"] == 2 and srv.peak_state == 2 * one


def test_concurrency_only_for_the_fp64_server():
    with pytest.raises(ValueError):
        serving.StokesServer(1 << 30, solver="mixed", concurrency=2)
    with pytest.raises(ValueError):
        serving.StokesServer(1 << 30, solver="fp64", concurrency=0)
