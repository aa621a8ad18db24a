"""Serving form: a stream of StokesFlow2D runs (requests) on one GPU.

A request is one StokesFlow2D run (scripts/StokesFlow2D_multixpu.jl:55-235)
of its own grid, markers and material for a given number of timesteps.  Its
state (markers, grid arrays) stays on the device from admission to
completion.  Admission is by HBM budget: a request is admitted when the
device bytes of its state fit what the budget has left and its solve fits
the engine's arena; otherwise it waits in arrival order.

Two servers over the same request trace:

* ``solver="mixed"`` (continuous batching): every admitted request's current
  Stokes solve lives in one resident :class:`api.Engine`.  Each loop turn is
  one engine round; a request whose solve converged in it advects, deposits
  its next timestep and re-enters the engine at once, while newly admitted
  requests join between rounds -- no request waits for a batch to drain.
* ``solver="fp64"``: the plain path, each timestep a blocking ``solveStokes!``
  (bit-identical to the reference).  With ``concurrency=1`` one request at a
  time in arrival order; with ``concurrency=K`` K worker threads, each with its
  own context and CUDA stream, take requests in arrival order, so up to K
  plain solves share the GPU (HBM admission as for the mixed server).

Latency of a request = completion time - arrival time.
"""
from __future__ import annotations

import math
import threading
import time
from collections import deque
from dataclasses import dataclass

import numpy as np
import torch

from . import api
from ._lib import StokesFlowError
from .driver import StokesFlow2D
from .workloads import InstanceSpec, log_uniform_int, random_inclusion_model


@dataclass
class Request:
    rid: int
    spec: InstanceSpec
    timesteps: int
    arrival: float                 # seconds after the server starts
    t_admit: float | None = None
    t_done: float | None = None
    solves: int = 0
    converged: int = 0
    sweeps: int = 0
    failed: bool = False           # a solve ended non-finite: the request stops there
    state: StokesFlow2D | None = None
    problem: api.MixedProblem | None = None
    state_bytes: int = 0
    final: dict | None = None      # host copies of the final state (keep_final)

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def poisson_requests(n: int, rate: float, seed: int = 0, *, cells=(63, 2047), timesteps=(1, 20), md=(3, 5),
                     mu_log10=(-2.0, 1.0), mu_air=1e-2) -> list[Request]:
    """n requests with exponential inter-arrival times of mean 1/rate seconds; cells per side log-uniform
    in `cells` (square grids), timesteps uniform in `timesteps`, materials as workloads.batch_specs."""
    # arrivals and request contents from two streams of the seed, so that one does not shift the other
    rng_t = np.random.default_rng([seed, 0])
    rng = np.random.default_rng([seed, 1])
    t = 0.0
    out = []
    for k in range(n):
        t += float(rng_t.exponential(1.0 / rate)) if rate > 0 else 0.0
        c = log_uniform_int(rng, *cells)
        m = int(rng.integers(md[0], md[1] + 1))
        model = random_inclusion_model(rng, mu_log10=mu_log10, mu_air=mu_air)
        steps = int(rng.integers(timesteps[0], timesteps[1] + 1))
        out.append(Request(k, InstanceSpec(c + 1, c + 1, m, model, seed * 100003 + k), steps, t))
    return out


def state_bytes(spec: InstanceSpec) -> int:
    """Device bytes of a request's state: 4 marker arrays and the grid arrays of StokesFlow2D without the
    reference's work arrays (P, Vx, Vy, rho_vy, mu_b, mu_p, dVxdt, dVydt, Vx_s, Vy_s), FP64."""
    Nx, Ny = spec.Nx, spec.Ny
    markers = spec.md * spec.md * (Nx - 1) * (Ny - 1)
    grid = ((Nx - 1) * (Ny - 1) + (Nx + 2) * (Ny + 1) + (Nx + 1) * (Ny + 2) + (Nx + 1) * Ny + Nx * Ny +
            (Nx - 1) * (Ny - 1) + (Nx - 2) * (Ny - 1) + (Nx - 1) * (Ny - 2) + Nx * (Ny + 1) + (Nx + 1) * Ny)
    return 8 * (4 * markers + grid)


def percentile(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if xs else float("nan")


class StokesServer:
    """See the module docstring.  hbm_budget: device bytes for request state plus (mixed) the engine arena,
    which takes `engine_share` of it."""

    def __init__(self, hbm_budget: int, *, solver: str = "mixed", rtol: float = 1e-6, options=None,
                 max_instances: int = 1024, engine_share: float = 0.5, iter_max: int = 4_000_000,
                 keep_final: bool = False, concurrency: int = 1, ctx: api.Context | None = None):
        if solver not in ("mixed", "fp64"):
            raise ValueError("solver must be 'mixed' or 'fp64'")
        if concurrency < 1 or (concurrency > 1 and solver != "fp64"):
            raise ValueError("concurrency: a positive worker count, for the fp64 server")
        self.solver = solver
        self.concurrency = int(concurrency)
        self.rtol = rtol
        self.iter_max = iter_max
        self.keep_final = keep_final
        self.ctx = ctx or api.default_context()
        self.engine = None
        if solver == "mixed":
            arena = int(hbm_budget * engine_share)
            self.engine = api.Engine(arena, max_instances, options=options, ctx=self.ctx)
            self.state_budget = hbm_budget - arena
        else:
            self.state_budget = hbm_budget
        self.state_used = 0
        self.peak_state = 0

    def close(self):
        if self.engine is not None:
            self.engine.close()
            self.engine = None

    # ------------------------------------------------------------------
    def _new_state(self, r: Request, ctx: api.Context | None = None) -> StokesFlow2D:
        s = r.spec
        return StokesFlow2D(s.Nx, s.Ny, 1.0, 1.0, s.model, marker_density=s.md, stokes_rtol=self.rtol, jitter=0.5,
                            seed=s.seed, keep_work_arrays=False, solver=self.solver, iter_max=self.iter_max,
                            ctx=ctx or self.ctx)

    def _finish(self, r: Request, now: float):
        r.t_done = now
        if self.keep_final:
            st = r.state
            r.final = {k: v.detach().cpu().numpy().copy() for k, v in
                       (("P", st.P), ("Vx", st.Vx), ("Vy", st.Vy), ("x_m", st.x_m), ("y_m", st.y_m))}
            r.final["t_tot"] = st.t_tot
        r.state = None
        r.problem = None
        self.state_used -= r.state_bytes

    def run(self, requests: list[Request]) -> dict:
        """Serve `requests` (arrival times relative to the call); returns the summary."""
        pending = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        t0 = time.perf_counter()
        if self.solver == "mixed":
            self._run_mixed(pending, t0)
        elif self.concurrency > 1:
            self._run_fp64_concurrent(pending, t0)
        else:
            self._run_fp64(pending, t0)
        return summarize(requests)

    def _run_mixed(self, pending: deque, t0: float):
        eng = self.engine
        queue: deque = deque()
        waiting: deque = deque()    # admitted, its current solve not yet in the engine (arena full)
        owner = {}
        stream = torch.cuda.current_stream()

        def enter(r: Request) -> bool:
            t = eng.submit(r.problem, stream=stream)
            if t is None:
                return False
            owner[id(r.problem)] = r
            return True

        while pending or queue or waiting or eng.active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.popleft())
            while waiting and enter(waiting[0]):
                waiting.popleft()
            while queue and not waiting:
                r = queue[0]
                b = state_bytes(r.spec)
                if self.state_used + b > self.state_budget and self.state_used > 0:
                    break
                queue.popleft()
                r.state_bytes = b
                self.state_used += b
                self.peak_state = max(self.peak_state, self.state_used)
                r.t_admit = now
                r.state = self._new_state(r)
                r.problem = r.state.begin_timestep()
                if not enter(r):
                    waiting.append(r)
            if eng.active:
                done = eng.step(stream=stream)
                finished = []
                for p in done:
                    r = owner.pop(id(p))
                    r.solves += 1
                    r.converged += int(p.result["converged"])
                    r.sweeps += int(p.result["inner_iters"])
                    if p.result["status"] != 0:
                        r.failed = True
                        finished.append(r)
                        continue
                    r.state.end_timestep(p.result)
                    if r.solves < r.timesteps:
                        r.problem = r.state.begin_timestep()
                        if not enter(r):
                            waiting.append(r)
                    else:
                        finished.append(r)
                if finished:
                    stream.synchronize()
                    now = time.perf_counter() - t0
                    for r in finished:
                        self._finish(r, now)
            elif pending and not queue and not waiting:
                time.sleep(max(0.0, pending[0].arrival - (time.perf_counter() - t0)))

    def _serve_fp64(self, r: Request, ctx: api.Context | None = None):
        """All timesteps of request r with the plain path, on the calling thread's current stream."""
        r.state = self._new_state(r, ctx)
        for _ in range(r.timesteps):
            r.solves += 1
            try:
                rec = r.state.step()
            except StokesFlowError as e:
                if e.status != 5:   # SF_ERR_NONFINITE ends the request; anything else is an error
                    raise
                r.failed = True
                break
            info = rec["info"]
            r.converged += int(info["converged"])
            r.sweeps += int(info["iters"])
        torch.cuda.current_stream().synchronize()

    def _run_fp64(self, pending: deque, t0: float):
        while pending:
            r = pending.popleft()
            now = time.perf_counter() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
                now = time.perf_counter() - t0
            r.t_admit = now
            r.state_bytes = state_bytes(r.spec)
            self.state_used = r.state_bytes
            self.peak_state = max(self.peak_state, self.state_used)
            self._serve_fp64(r)
            self._finish(r, time.perf_counter() - t0)

    def _run_fp64_concurrent(self, pending: deque, t0: float):
        """K workers, each with its own context and stream; a worker takes the next request in arrival order
        once it has arrived and its state fits what the HBM budget has left."""
        lock = threading.Condition()
        errors = []
        device = torch.cuda.current_device()

        def next_request():
            with lock:
                while True:
                    if errors or not pending:
                        return None
                    r = pending[0]
                    b = state_bytes(r.spec)
                    now = time.perf_counter() - t0
                    fits = self.state_used + b <= self.state_budget or self.state_used == 0
                    if r.arrival <= now and fits:
                        break
                    lock.wait(timeout=max(1e-3, r.arrival - now) if fits else None)
                pending.popleft()
                r.t_admit = now
                r.state_bytes = b
                self.state_used += b
                self.peak_state = max(self.peak_state, self.state_used)
                return r

        def worker():
            ctx = None
            try:
                torch.cuda.set_device(device)
                ctx = api.Context(device)
                with torch.cuda.stream(torch.cuda.Stream()):
                    while (r := next_request()) is not None:
                        self._serve_fp64(r, ctx)
                        with lock:
                            self._finish(r, time.perf_counter() - t0)
                            lock.notify_all()
            except BaseException as e:   # surfaced after the join
                with lock:
                    errors.append(e)
                    lock.notify_all()
            finally:
                if ctx is not None:
                    torch.cuda.synchronize(device)
                    ctx.close()

        threads = [threading.Thread(target=worker, daemon=True) for _ in range(self.concurrency)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if errors:
            raise errors[0]


def summarize(requests: list[Request]) -> dict:
    done = [r for r in requests if r.t_done is not None]
    lat = [r.latency for r in done]
    solves = sum(r.solves for r in done)
    t_first = min((r.arrival for r in requests), default=0.0)
    t_last = max((r.t_done for r in done), default=0.0)
    span = max(t_last - t_first, 1e-9)
    return {"requests": len(requests), "completed": len(done), "failed": sum(1 for r in done if r.failed),
            "solves": solves,
            "converged_solves": sum(r.converged for r in done), "sweeps": sum(r.sweeps for r in done),
            "makespan_s": span, "solves_per_s": solves / span, "p50_latency_s": percentile(lat, 50),
            "p99_latency_s": percentile(lat, 99), "mean_latency_s": float(np.mean(lat)) if lat else math.nan}
