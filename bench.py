"""Benchmark: the StokesFlow.jl per-timestep hot path on B200.

Workload (one "step" = one timestep: deposit rho/mu onto the three staggered
grids -> PT Stokes solve to relative residual 1e-6 -> RK4 advection ->
marker rebin): the plume model on the unit square, 2047 x 2047 cells
(Nx = Ny = 2048 grid points), 16 markers per cell (4 x 4 sub-grid, jittered
+-0.25 sub-spacing from seed 0; 67,043,344 markers), FP64, warm-started
timesteps as in StokesFlow2D.

Metric: PT T_eff = essential HBM bytes of the PT iterations (read + write
Vx, Vy, P, dVx, dVy; read rho_vy, mu_b, mu_p = ~104 Nx Ny bytes per
iteration) x iterations / timed-region time, in GB/s.  `value` is over the
whole timed steps (deposit and advection included in the time); the solve-only
figure, solves/s and the per-phase split are reported beside it.

--impl reference times the reference algorithm on the host cores: the C
restatement in oracle/ (the Julia reference has no toolchain here), OpenMP over
all cores, on a bounded sample of the same workload.

Multi-GPU: the path does not shard (single domain); --gpus N runs N
independent replicas (one per rank) and `value` sums their bytes over the
max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "stokesflow.jl_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

METRIC = "PT T_eff (essential HBM bytes of the PT iterations / time), FP64, relative residual 1e-6"
UNIT = "GB/s"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
TRAFFIC_PER_LAUNCH_2048 = 402.079e6   # dram__bytes_read.sum + dram__bytes_write.sum, k_pt_iter, 2047^2 points


# ---------------------------------------------------------------------------
def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", "--grid-points", dest="n", type=int, default=2048,
                    help="grid points per side (cells = n - 1); under torchrun spell it --grid-points, since "
                         "torchrun's own parser takes --n for a prefix of its options")
    ap.add_argument("--markers-per-cell", type=int, default=16)
    ap.add_argument("--rtol", type=float, default=1e-6)
    ap.add_argument("--iter-max", type=int, default=400000,
                    help="PT iteration cap per solve (reference default 100000; a cold 2048^2 start needs ~250k)")
    ap.add_argument("--mu-air", type=float, default=1e-2,
                    help="air viscosity; with 1e-3 (a 1000x jump) the reference PT scheme diverges")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=12, help="PT iterations in the CPU baseline sample")
    ap.add_argument("--pt-probe", type=int, default=0, metavar="ITERS",
                    help="kernel probe: run ITERS fused PT iterations of an n x n solve (smooth random fields, no "
                         "markers) and print the kernel time; used for ncu captures")
    ap.add_argument("--pt32-probe", type=int, default=0, metavar="SWEEPS",
                    help="kernel probe: one n x n instance through the mixed engine for exactly SWEEPS FP32 sweeps "
                         "(one fold); prints the sweep time; used for ncu captures of k_pt32")
    ap.add_argument("--form", default="timestep",
                    choices=["timestep", "precision", "batch", "serve", "tune", "decomposed"],
                    help="timestep: the plain FP64 timestep (default line); precision: the same timesteps with FP32 "
                         "sweeps + FP64 correction beside the plain path; batch: many independent solves in one "
                         "engine vs a loop of plain FP64 solves; serve: a Poisson request stream, continuous "
                         "batching vs plain FP64 serving; tune: the sweep tuner's table of tile shapes and schedules; "
                         "decomposed: the PT solve over a grid of ranks vs the single-domain solve of the same grid")
    ap.add_argument("--dims", default="2,2", help="decomposed form: ranks in x and y")
    ap.add_argument("--decomposed-iters", type=int, default=2000, help="decomposed form: PT iterations timed")
    ap.add_argument("--precision-cases", type=int, default=2, help="precision form: plume contrasts drawn from seed")
    ap.add_argument("--precision-contrast", default="0,2",
                    help="precision form: log10 range of matrix/plume viscosity, log-uniform (soft plume)")
    ap.add_argument("--precision-steps", type=int, default=3, help="precision form: timesteps per case")
    ap.add_argument("--batch-instances", type=int, default=256)
    ap.add_argument("--batch-cells", default="127,1023", help="cells per side, log-uniform range")
    ap.add_argument("--mu-log10", default="-2,1", help="inclusion viscosity range (log10), log-uniform")
    ap.add_argument("--fp64-concurrency", type=int, default=8,
                    help="batch and serve forms: also time plain FP64 with this many solves at a time (host "
                         "threads, own contexts and streams); 1: only one at a time")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--serve-requests", type=int, default=32)
    ap.add_argument("--serve-rate", type=float, default=6.0, help="requests per second (Poisson)")
    ap.add_argument("--serve-cells", default="63,1023", help="cells per side of a request, log-uniform range")
    ap.add_argument("--serve-steps", default="1,20", help="timesteps per request, uniform range")
    ap.add_argument("--hbm-budget-gb", type=float, default=64.0)
    ap.add_argument("--no-forms", action="store_true",
                    help="default line without the bounded precision / batch / serve forms object")
    ap.add_argument("--forms-batch", type=int, default=64, help="forms object: batch instances")
    ap.add_argument("--forms-requests", type=int, default=16, help="forms object: serve requests")
    ap.add_argument("--forms-rate", type=float, default=16.0,
                    help="forms object: serve requests per second (above both servers' capacity, so that solves/s "
                         "measures throughput, not the arrival rate)")
    ap.add_argument("--forms-cells", default="63,511", help="forms object: serve cells per side")
    ap.add_argument("--forms-precision-n", type=int, default=1024, help="forms object: precision grid points")
    ap.add_argument("--forms-precision-steps", type=int, default=3, help="forms object: precision timesteps")
    ap.add_argument("--fold-every", type=int, default=400)
    ap.add_argument("--tile-rows", type=int, default=0,
                    help="rows of the FP32 sweep tiles (8, 16, 32); 0: the autotuner chooses rows and schedule")
    ap.add_argument("--tile-schedule", default=None, choices=["strided", "chunked"],
                    help="schedule of the sweep tiles, with --tile-rows")
    return ap.parse_args()


def _pair(s, typ=float):
    a, b = s.split(",")
    return typ(a), typ(b)


def pt_probe(a):
    """Fused PT iteration alone: ITERS iterations (no residual check falls inside when ITERS < 2000)."""
    import stokesflow_b200 as sf
    n, iters = a.n, a.pt_probe
    z = sf.zeros
    P, Vx, Vy = z(n - 1, n - 1), z(n + 2, n + 1), z(n + 1, n + 2)
    rho, mub, mup = z(n + 1, n), z(n, n), z(n - 1, n - 1)
    g = torch.Generator(device="cuda").manual_seed(0)
    for arr in (rho, mub, mup):
        arr.copy_(1.0 + 0.5 * torch.rand(arr.shape[1], arr.shape[0], device="cuda", dtype=torch.float64,
                                         generator=g).t())
    dVx, dVy, Vxs, Vys = z(n - 2, n - 1), z(n - 1, n - 2), z(n, n + 1), z(n + 1, n)
    info = sf.solve_stokes_info(P, Vx, Vy, rho, mub, mup, None, None, None, None, None, None, None, dVx, dVy, None,
                                None, Vxs, Vys, 9.81, 1 / (n - 1), 1 / (n - 1), n, n, 0.0, 0.5, eps=1e-300,
                                iter_max=iters)
    peak, src = peak_hbm()
    us = info["loop_ms"] * 1e3 / iters
    gbs = info["bytes_per_iter"] / (us * 1e-6) / 1e9
    print(json.dumps({"probe": "k_pt_iter", "n": n, "iters": iters, "us_per_iter": round(us, 3),
                      "t_eff_gbs": round(gbs, 1), "frac_of_peak": round(gbs / peak, 4), "peak_source": src,
                      "bytes_per_iter": info["bytes_per_iter"]}), flush=True)


def pt32_probe(a):
    """FP32 sweeps of the mixed engine alone: one n x n instance (smooth random fields), SWEEPS sweeps in one
    fold, timed by the engine's device clock; the fold's FP64 residual evaluations are a small extra."""
    import stokesflow_b200 as sf
    n, sweeps = a.n, a.pt32_probe
    z = sf.zeros
    P, Vx, Vy, Vxs, Vys = z(n - 1, n - 1), z(n + 2, n + 1), z(n + 1, n + 2), z(n, n + 1), z(n + 1, n)
    rho, mub, mup = z(n + 1, n), z(n, n), z(n - 1, n - 1)
    g = torch.Generator(device="cuda").manual_seed(0)
    for arr in (rho, mub, mup):
        arr.copy_(1.0 + 0.5 * torch.rand(arr.shape[1], arr.shape[0], device="cuda", dtype=torch.float64,
                                         generator=g).t())
    # a fixed sweep shape (16 rows strided unless given), so that every launch is the same kernel
    opts = sf.mixed_options(max_sweeps=sweeps, fold_every=sweeps, tile_rows=a.tile_rows or 16,
                            tile_schedule=a.tile_schedule if a.tile_rows else "strided")
    h = 1.0 / (n - 1)
    for rep in range(2):   # the first run captures the graph
        p = sf.MixedProblem(P, Vx, Vy, rho, mub, mup, Vxs, Vys, 9.81, h, h, n, n, 0.0, 0.5, eps=1e-300)
        r = sf.solve_stokes_batch_mixed([p], options=opts)[0]
    peak, src = peak_hbm()
    us = r["batch_ms"] * 1e3 / max(1, r["inner_iters"])
    pts = (n - 1) * (n - 1)
    gbs = sf.driver.MIXED_BYTES_PER_POINT * pts / (us * 1e-6) / 1e9
    print(json.dumps({"probe": "k_pt32", "n": n, "sweeps": r["inner_iters"], "us_per_sweep": round(us, 3),
                      "gpts_per_s": round(pts / us / 1e3, 2), "t_eff_gbs": round(gbs, 1),
                      "frac_of_peak": round(gbs / peak, 4), "peak_source": src}), flush=True)


def run_decomposed_form(a):
    """The decomposed PT solve (sf_solve_stokes_decomposed: a grid of ranks with halo updates and the global
    reductions) on the ranks' devices -- here all on this GPU -- against the single-domain solve of the same
    global grid: the same plume fields, split as the ranks hold them, iterated a fixed number of times from rest
    (no residual small enough to stop them).  Reports microseconds per PT iteration of each; the decomposed solve
    issues its launches and halo copies from the host, rank by rank, every iteration."""
    import stokesflow_b200 as sf
    from stokesflow_b200 import domains
    torch.cuda.set_device(0)
    dims = _pair(a.dims, int)
    n = a.n
    nloc = domains.local_size(dims[0], n), domains.local_size(dims[1], n)
    iters = a.decomposed_iters
    model = sf.plume_model_unit_square()
    model.mu_air = a.mu_air
    md = sf.driver.marker_density_for(a.markers_per_cell)
    st = sf.StokesFlow2D(n, n, 1.0, 1.0, model, marker_density=md, stokes_rtol=a.rtol, jitter=0.5, seed=0,
                         iter_max=iters, keep_work_arrays=False)
    st.deposit()
    names = ("P", "Vx_pad", "Vy_pad", "rho_vy", "mu_b", "mu_p", "dVxdt", "dVydt", "Vx_s", "Vy_s")
    glob = {"P": st.P, "Vx_pad": st.Vx, "Vy_pad": st.Vy, "rho_vy": st.rho_vy, "mu_b": st.mu_b, "mu_p": st.mu_p,
            "dVxdt": st.dVxdt, "dVydt": st.dVydt, "Vx_s": st.Vx_s, "Vy_s": st.Vy_s}
    ranks = domains.split({k: glob[k] for k in names}, dims, nloc[0], nloc[1])
    ctxs = {c: sf.Context(0) for c in ranks}
    out = {}
    for rep in range(2):   # the first of each is a warm-up
        t = {}
        info = sf.solve_stokes_info(st.P, st.Vx, st.Vy, st.rho_vy, st.mu_b, st.mu_p, None, None, None, None, None,
                                    None, None, st.dVxdt, st.dVydt, None, None, st.Vx_s, st.Vy_s, st.g_y, st.dx,
                                    st.dy, n, n, 0.0, st.maxdisp, eps=1e-300, iter_max=iters, ctx=st.ctx)
        t["single"] = (info["loop_ms"], info["iters"])
        loc = {c: {k: v.clone() for k, v in r.items()} for c, r in ranks.items()}
        d = domains.solve_stokes_decomposed(loc, dims, nloc[0], nloc[1], st.g_y, st.dx, st.dy, 0.0, st.maxdisp,
                                            eps=1e-300, iter_max=iters, contexts=ctxs)
        t["decomposed"] = (d["loop_ms"], d["iters"])
        out = t
    us = {k: v[0] * 1e3 / max(1, v[1]) for k, v in out.items()}
    for c in ctxs.values():
        c.close()
    return {"form": "decomposed", "metric": "microseconds per PT iteration, FP64", "unit": "us",
            "us_per_iter_single_domain": round(us["single"], 2), "us_per_iter_decomposed": round(us["decomposed"], 2),
            "decomposed_over_single": round(us["decomposed"] / us["single"], 3),
            "iterations": {k: v[1] for k, v in out.items()},
            "config": {"workload": f"plume, {n}x{n} grid points, fields deposited from {md * md} markers per cell; "
                                   f"{dims[0]}x{dims[1]} ranks of {nloc[0]}x{nloc[1]} points, all on one GPU",
                       "note": "single-domain time from the library's CUDA events over the PT loop; decomposed time "
                               "from its host clock over the loop (launches and halo copies issued rank by rank)"}}


def run_tune_form(a):
    """The sweep autotuner's candidate table: G point-sweeps/s of each tile shape (8, 16, 32 rows) and schedule
    (strided, chunked) as the engine times them in its first round, on (1) the instance sizes of the batch
    form's workload and (2) one n x n instance.  Smooth random fields; 2 folds of fold_every sweeps each."""
    import stokesflow_b200 as sf
    from stokesflow_b200 import workloads
    torch.cuda.set_device(0)
    g = torch.Generator(device="cuda").manual_seed(a.seed)

    def problem(nx, ny):
        z = sf.zeros
        arr = dict(P=z(nx - 1, ny - 1), Vx=z(nx + 2, ny + 1), Vy=z(nx + 1, ny + 2), Vxs=z(nx, ny + 1),
                   Vys=z(nx + 1, ny), rho=z(nx + 1, ny), mub=z(nx, ny), mup=z(nx - 1, ny - 1))
        for k in ("rho", "mub", "mup"):
            t = arr[k]
            t.copy_(1.0 + 0.5 * torch.rand(t.shape[1], t.shape[0], device="cuda", dtype=torch.float64,
                                           generator=g).t())
        p = sf.MixedProblem(arr["P"], arr["Vx"], arr["Vy"], arr["rho"], arr["mub"], arr["mup"], arr["Vxs"],
                            arr["Vys"], 9.81, 1.0 / (nx - 1), 1.0 / (ny - 1), nx, ny, 0.0, 0.5, eps=1e-300)
        return p, arr

    specs = workloads.batch_specs(a.batch_instances, a.seed, cells=_pair(a.batch_cells, int))
    cases = {f"batch {len(specs)} instances, cells {a.batch_cells}": [(sp.Nx, sp.Ny) for sp in specs],
             f"one instance {a.n}x{a.n}": [(a.n, a.n)]}
    opts = sf.mixed_options(max_sweeps=2 * a.fold_every, fold_every=a.fold_every)
    out = {}
    for name, sizes in cases.items():
        ctx = sf.Context(0)                  # a fresh context: no choice recorded yet
        made = [problem(nx, ny) for nx, ny in sizes]
        sf.solve_stokes_batch_mixed([p for p, _ in made], options=opts, ctx=ctx)
        st = sf.batch_stats(ctx)
        launch = "overlapped" if st["overlap_launches"] else "serial"
        out[name] = {"chosen": f"{st['tile_rows']}/{st['tile_schedule']}/{launch}", "tuner": st["tune_state"],
                     "grid_points": int(sum((nx - 1) * (ny - 1) for nx, ny in sizes)),
                     "gpts_per_s": {k: round(1.0 / v, 2) for k, v in st["tune_ns"].items() if v > 0}}
        del made
        torch.cuda.empty_cache()
    return {"form": "tune", "metric": "FP32 sweep throughput per tile shape, schedule and launch mode, as the "
                                      "engine's tuner times it", "unit": "G point-sweeps/s", "cases": out,
            "data": "synthetic (smooth random fields, seeded)", "fold_every": a.fold_every, "seed": a.seed}


def bench_config(a):
    return {"workload": f"plume, {a.n - 1}x{a.n - 1} cells, {a.markers_per_cell} markers/cell, FP64, "
                        f"PT to relative residual {a.rtol:g}, warm-started timesteps",
            "grid_points": [a.n, a.n], "markers_per_cell": a.markers_per_cell,
            "n_markers": (int(round(a.markers_per_cell ** 0.5)) * (a.n - 1)) ** 2, "rtol": a.rtol,
            "iter_max": a.iter_max, "mu_air": a.mu_air, "rho_air": 1e-3, "jitter": "+-0.25 sub-spacing, seed 0",
            "l2": "inputs larger than L2: 13 arrays x 34 MB per PT iteration",
            "parallelism": "replicas only (single-domain path)"}


def peak_hbm():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples during the timed region (sm clock, max clock, throttle reasons)."""
    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for nm, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def aggregate(bytes_local: float, ms_local: float, extra_sum=()):
    """Whole-job aggregate over ranks: bytes (and extra_sum) summed, time = max over ranks."""
    if dist.is_available() and dist.is_initialized():
        dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
        s = torch.tensor([bytes_local, *extra_sum], dtype=torch.float64, device=dev)
        m = torch.tensor([ms_local], dtype=torch.float64, device=dev)
        dist.all_reduce(s, op=dist.ReduceOp.SUM)
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        s, m = s.cpu().tolist(), m.item()
        return s[0], m, s[1:]
    return bytes_local, ms_local, list(extra_sum)


def barrier():
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


# ---------------------------------------------------------------------------
def make_state(a, host_markers=False):
    import stokesflow_b200 as sf
    model = sf.plume_model_unit_square()
    model.mu_air = a.mu_air
    md = sf.driver.marker_density_for(a.markers_per_cell)
    return sf.StokesFlow2D(a.n, a.n, 1.0, 1.0, model, marker_density=md, stokes_rtol=a.rtol, jitter=0.5, seed=0,
                           iter_max=a.iter_max, rebin=True, keep_work_arrays=False, host_markers=host_markers)


def run_ours(a, rank, world, local_rank):
    import stokesflow_b200 as sf
    torch.cuda.set_device(local_rank)
    peak, peak_src = peak_hbm()
    st = make_state(a)
    ctx = st.ctx
    for _ in range(a.warmup):
        st.step()
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = ctx.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record()
    recs = [st.step() for _ in range(a.steps)]
    ev1.record()
    torch.cuda.synchronize()
    launches = ctx.launch_count() - launches0
    clk = clocks.stop()
    ms_local = ev0.elapsed_time(ev1)
    bytes_local = sum(r["info"]["bytes_per_iter"] * r["info"]["iters"] for r in recs)
    solve_ms = sum(r["times"].solve_ms for r in recs)
    loop_ms = sum(r["info"]["loop_ms"] for r in recs)
    iters = sum(r["info"]["iters"] for r in recs)
    tot_bytes, tot_ms, (tot_steps,) = aggregate(bytes_local, ms_local, (float(len(recs)),))
    value = tot_bytes / (tot_ms * 1e-3) / 1e9
    out = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": round(tot_ms / a.steps, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded plume model)",
           "config": bench_config(a)}
    bpi = recs[0]["info"]["bytes_per_iter"]
    out["solve"] = {
        "iters_per_step": [r["info"]["iters"] for r in recs],
        "converged": [int(r["info"]["converged"]) for r in recs],
        "t_eff_solve_gbs": round(bytes_local / (solve_ms * 1e-3) / 1e9, 2),
        "t_eff_reference_def_gbs": round(sum(r["info"]["T_eff"] for r in recs) / len(recs), 2),
        "solves_per_s": round(tot_steps / (tot_ms * 1e-3), 4),
        "bytes_per_iter": bpi, "us_per_iter": round(loop_ms * 1e3 / max(iters, 1), 3)}
    out["ms_per_timestep"] = {k: round(sum(getattr(r["times"], k) for r in recs) / len(recs), 3)
                              for k in ("deposit_ms", "solve_ms", "advect_ms", "rebin_ms")}
    achieved = bytes_local / (loop_ms * 1e-3) / 1e9
    # DRAM bytes (read + write) of one k_pt_iter launch, measured by ncu at 2047^2 points, scaled by the
    # point count (the kernel streams each field once, so its traffic grows with the points)
    traffic = TRAFFIC_PER_LAUNCH_2048 * ((a.n - 1) / 2047.0) ** 2
    out["roofline"] = {"bound": "hbm", "kernel": "k_pt_iter (fused PT iteration)", "achieved": round(achieved, 1),
                       "peak": peak, "peak_source": peak_src, "unit": "GB/s", "frac": round(achieved / peak, 4),
                       "traffic": round(traffic), "algorithmic_bytes_per_launch": bpi,
                       "note": "achieved = bytes_per_iter x iterations / PT-loop device time (CUDA events; checks and "
                               "dt updates included, pack/unpack excluded); traffic from ncu per launch"}
    out["clocks"] = clk
    out["gpu_launches"] = launches
    # ---- end to end through the public API with host buffers ----
    if not a.no_e2e:
        st.x_host = st.x_m.cpu().pin_memory()
        st.y_host = st.y_m.cpu().pin_memory()
        st.rho_host = st.rho_m.cpu().pin_memory()
        st.mu_host = st.mu_m.cpu().pin_memory()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        erecs = [st.step(host_io=True) for _ in range(a.steps)]
        e1.record()
        torch.cuda.synchronize()
        ebytes = sum(r["info"]["bytes_per_iter"] * r["info"]["iters"] for r in erecs)
        eb, ems, _ = aggregate(ebytes, e0.elapsed_time(e1))
        out["e2e"] = {"value": round(eb / (ems * 1e-3) / 1e9, 2), "unit": UNIT,
                      "h2d_bytes_per_step": st.h2d_bytes_per_step(), "d2h_bytes_per_step": st.d2h_bytes_per_step(),
                      "ms_per_step": round(ems / a.steps, 3),
                      "note": "same timesteps continued, markers H2D from pinned host memory before and "
                              "markers + padded velocities D2H after every step"}
    if rank == 0 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(a)
    return out


# ---------------------------------------------------------------------------
def cpu_sample(a, iters, nthreads):
    """The oracle (reference algorithm restated in C) on the host: deposit of the three grids, then `iters`
    PT iterations of the same 2048^2 plume solve; returns (T_eff GB/s, details)."""
    import numpy as np

    import oracle as O
    n = a.n
    dx = dy = 1.0 / (n - 1)
    md = int(round(a.markers_per_cell ** 0.5))
    m = O.PlumeModel(air_height=0.1, plume_x=0.5, plume_y=0.75, plume_r=0.1, rho_air=1e-3, rho_matrix=1.0,
                     rho_plume=0.9, mu_air=a.mu_air, mu_matrix=1.0, mu_plume=0.1)
    x, y = O.initialize_markers(md, 1.0, 1.0, dx, dy, n, n, 0.5, 0)
    rho, mu = O.set_marker_properties(m, x, y)
    arr = O.stokes_arrays(n, n)
    o = O.node_origins(dx, dy)
    vws, ws = O.zeros(n + 1, n), O.zeros(n + 1, n)
    t0 = time.perf_counter()
    O.bilinear_marker_to_grid(o["x_rho"], o["y_rho"], arr["rho_vy"], x, y, rho, dx, dy, vws, ws)
    t_dep = time.perf_counter() - t0
    O.bilinear_marker_to_grid(o["x"], o["y"], arr["mu_b"], x, y, mu, dx, dy, vws, ws)
    O.bilinear_marker_to_grid(o["x_p"], o["y_p"], arr["mu_p"], x, y, mu, dx, dy, vws, ws)
    t0 = time.perf_counter()
    r = O.solve_stokes(arr, 9.81, dx, dy, n, n, 0.0, 0.5, True, 1e-300, iters, nthreads)
    t_solve = time.perf_counter() - t0
    bpi = 8.0 * (2.0 * (n * (n + 1) + (n + 1) * n + (n - 1) ** 2 + (n - 2) * (n - 1) + (n - 1) * (n - 2))
                 + (n + 1) * n + n * n + (n - 1) ** 2)
    teff = bpi * r.iters / t_solve / 1e9
    del np
    return teff, {"iters": r.iters, "solve_s": round(t_solve, 3), "deposit_one_grid_s": round(t_dep, 3),
                  "us_per_iter": round(t_solve / r.iters * 1e6, 1)}


def cpu_baseline(a):
    n = os.cpu_count() or 1
    teff, det = cpu_sample(a, a.cpu_iters, n)
    return {"value": round(teff, 3), "unit": UNIT, "cores": n, "kind": "port",
            "sample": f"{a.cpu_iters} PT iterations of the same {a.n}^2 solve (cold start) after the rho deposit, "
                      f"OpenMP over {n} threads; deposit timed on one grid, serial as in the reference",
            "detail": det, "cpu": _cpu_model()}


def _cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


# ---------------------------------------------------------------------------
# batched and served forms (single GPU; printed as their own JSON lines)
# ---------------------------------------------------------------------------
SOLVE_CAP = 4_000_000   # PT iterations / FP32 sweeps a solve may take in the batch and serve forms


def _deposit_instances(sf, specs):
    """rho_vy, mu_b, mu_p of every instance deposited from its markers (markers freed afterwards)."""
    out = []
    for sp in specs:
        st = sf.StokesFlow2D(sp.Nx, sp.Ny, 1.0, 1.0, sp.model, marker_density=sp.md, jitter=0.5, seed=sp.seed,
                             keep_work_arrays=False)
        st.deposit()
        out.append(dict(spec=sp, rho_vy=st.rho_vy, mu_b=st.mu_b, mu_p=st.mu_p, dx=st.dx, dy=st.dy,
                        markers=st.n_markers))
        del st
    torch.cuda.synchronize()
    return out


def _state_arrays(sf, Nx, Ny):
    z = sf.zeros
    return dict(P=z(Nx - 1, Ny - 1), Vx_pad=z(Nx + 2, Ny + 1), Vy_pad=z(Nx + 1, Ny + 2), Vx_s=z(Nx, Ny + 1),
                Vy_s=z(Nx + 1, Ny), dVx=z(Nx - 2, Ny - 1), dVy=z(Nx - 1, Ny - 2))


def _rel_l2(a, b):
    d = torch.linalg.vector_norm((a - b).flatten()).item()
    n = torch.linalg.vector_norm(b.flatten()).item()
    return d / n if n > 0 else d


def _fields_l2(got, ref, names):
    return {f: _rel_l2(got[f], ref[f]) for f in names}


def _worst(rows, names):
    return {f: max((r[f] for r in rows), default=None) for f in names}


def run_precision_form(a, *, n=None, cases=None, steps=None, contrast=None):
    """Precision form: the plume timesteps of the default workload (n x n grid points, markers per cell as
    given) with the plume viscosity drawn from seed (matrix/plume contrast log-uniform over
    10**contrast), each timestep solved by the plain FP64 path (the oracle) and by FP32 sweeps + FP64 defect
    correction, both to relative residual rtol, each carrying its own state (V, P, damped rates, dt,
    markers) forward.  Reported per timestep: solve time and iterations of each, and the relative L2
    distance of V, P and the marker positions between them."""
    import numpy as np
    import stokesflow_b200 as sf
    torch.cuda.set_device(0)
    n = n or a.n
    cases = cases or a.precision_cases
    steps = steps or a.precision_steps
    contrast = contrast or a.precision_contrast
    rng = np.random.default_rng(a.seed)
    lo, hi = _pair(contrast)
    md = sf.driver.marker_density_for(a.markers_per_cell)
    opts = sf.mixed_options(max_sweeps=SOLVE_CAP, fold_every=a.fold_every, tile_rows=a.tile_rows,
                            tile_schedule=a.tile_schedule)
    names = ("rel_l2_Vx", "rel_l2_Vy", "rel_l2_P", "rel_l2_markers_x", "rel_l2_markers_y")
    clocks = ClockSampler(0)
    clocks.start()
    out_cases = []
    for c in range(cases):
        C = float(10.0 ** rng.uniform(lo, hi))
        model = sf.plume_model_unit_square()
        model.mu_air = a.mu_air
        model.mu_plume = model.mu_matrix / C
        # the mixed path on a context of its own: its sweep tuner measures this workload instead of reusing a
        # choice recorded for another form's instances in the same workload class
        mctx = sf.Context(0)
        states = {s: sf.StokesFlow2D(n, n, 1.0, 1.0, model, marker_density=md, stokes_rtol=a.rtol, jitter=0.5,
                                     seed=0, iter_max=SOLVE_CAP, keep_work_arrays=False, solver=s, mixed_opts=opts,
                                     ctx=mctx if s == "mixed" else None)
                  for s in ("fp64", "mixed")}
        rows = []
        for k in range(steps):
            rec = {s: st.step() for s, st in states.items()}
            f, m = states["fp64"], states["mixed"]
            rows.append({"fp64_solve_ms": round(rec["fp64"]["times"].solve_ms, 2),
                         "mixed_solve_ms": round(rec["mixed"]["times"].solve_ms, 2),
                         "fp64_iters": int(rec["fp64"]["info"]["iters"]),
                         "mixed_sweeps": int(rec["mixed"]["info"]["inner_iters"]),
                         "rel_l2_Vx": _rel_l2(m.Vx, f.Vx), "rel_l2_Vy": _rel_l2(m.Vy, f.Vy),
                         "rel_l2_P": _rel_l2(m.P, f.P), "rel_l2_markers_x": _rel_l2(m.x_m, f.x_m),
                         "rel_l2_markers_y": _rel_l2(m.y_m, f.y_m)})
        fs = sum(r["fp64_solve_ms"] for r in rows)
        ms = sum(r["mixed_solve_ms"] for r in rows)
        eng = sf.batch_stats(mctx)
        out_cases.append({"contrast": C, "mu_plume": model.mu_plume, "fp64_solve_ms_total": round(fs, 1),
                          "mixed_solve_ms_total": round(ms, 1), "solve_speedup": round(fs / ms, 3),
                          "same_iterations": all(r["fp64_iters"] == r["mixed_sweeps"] for r in rows),
                          "sweeps": {k: eng.get(k) for k in ("tile_rows", "tile_schedule", "overlap_launches",
                                                             "tune_state")},
                          "steps": rows})
        del states
        mctx.close()
        torch.cuda.empty_cache()
    clk = clocks.stop()
    fs = sum(cs["fp64_solve_ms_total"] for cs in out_cases)
    ms = sum(cs["mixed_solve_ms_total"] for cs in out_cases)
    nsolves = cases * steps
    return {"form": "precision", "metric": f"solve time and rel L2 vs plain FP64, relative residual {a.rtol:g}",
            "unit": "ms / rel L2", "solves_per_s": round(nsolves / (ms * 1e-3), 4),
            "fp64_solves_per_s": round(nsolves / (fs * 1e-3), 4), "solve_speedup": round(fs / ms, 3),
            "max_rel_l2": _worst([r for cs in out_cases for r in cs["steps"]], names),
            "same_iterations": all(cs["same_iterations"] for cs in out_cases), "cases": out_cases,
            "dtype": "f32 sweeps + f64 correction / f64", "data": "synthetic (seeded markers and contrasts)",
            "clocks": clk,
            "config": {"workload": f"plume, {n - 1}x{n - 1} cells, {a.markers_per_cell} markers/cell, matrix/"
                                   f"plume viscosity contrast log-uniform 10**[{contrast}], {steps} timesteps per "
                                   f"case from a cold start, air mu {a.mu_air:g}",
                       "oracle": "plain FP64 path (bit-identical to the reference) at the same tolerance",
                       "fold_every": a.fold_every, "seed": a.seed}}


def run_batch_form(a, *, instances=None, cells=None, concurrency=None):
    """Batching form: N independent problems (seeded random grids and inclusion layouts) solved to relative
    residual rtol in one resident engine (FP32 sweeps + FP64 defect correction, one launch per sweep for all
    instances, graph replay, the tuner's sweep shapes) against the plain FP64 path on the same problems:
    a loop of solves one after the other (the plain form as it is called), and, with concurrency K > 1, K
    host threads each with its own context and stream, so that K plain solves share the GPU.  Every
    instance's result is compared with its plain FP64 result (the oracle at the same tolerance).  Latency of
    an instance: from the start of the run to its completion."""
    import statistics as stats

    import stokesflow_b200 as sf
    from stokesflow_b200 import workloads
    torch.cuda.set_device(0)
    instances = instances or a.batch_instances
    cells = cells or a.batch_cells
    concurrency = a.fp64_concurrency if concurrency is None else concurrency
    specs = workloads.batch_specs(instances, a.seed, cells=_pair(cells, int), mu_log10=_pair(a.mu_log10),
                                  mu_air=a.mu_air)
    inst = _deposit_instances(sf, specs)
    opts = sf.mixed_options(max_sweeps=SOLVE_CAP, fold_every=a.fold_every, tile_rows=a.tile_rows,
                            tile_schedule=a.tile_schedule)

    def mixed_problems(subset):
        probs, arrs = [], []
        for d in subset:
            sp = d["spec"]
            s = _state_arrays(sf, sp.Nx, sp.Ny)
            arrs.append(s)
            probs.append(sf.MixedProblem(s["P"], s["Vx_pad"], s["Vy_pad"], d["rho_vy"], d["mu_b"], d["mu_p"],
                                         s["Vx_s"], s["Vy_s"], 9.81, d["dx"], d["dy"], sp.Nx, sp.Ny, 0.0, 0.5,
                                         rel_tol=a.rtol, dVxdt=s["dVx"], dVydt=s["dVy"]))
        return probs, arrs

    def fp64_solve(d, s, ctx=None):
        sp = d["spec"]
        scale = sf.residual_scale(d["rho_vy"], sp.Nx, sp.Ny, 9.81, ctx=ctx)
        try:
            return sf.solve_stokes_info(s["P"], s["Vx_pad"], s["Vy_pad"], d["rho_vy"], d["mu_b"], d["mu_p"], None,
                                        None, None, None, None, None, None, s["dVx"], s["dVy"], None, None, s["Vx_s"],
                                        s["Vy_s"], 9.81, d["dx"], d["dy"], sp.Nx, sp.Ny, 0.0, 0.5,
                                        eps=a.rtol * scale, iter_max=SOLVE_CAP, ctx=ctx)
        except sf.StokesFlowError as e:
            if e.status != 5:   # SF_ERR_NONFINITE: the instance diverged; anything else is an error
                raise
            return {"converged": 0, "iters": 0, "nonfinite": 1}

    # warm-up of both paths on the two smallest instances (graph capture, occupancy queries, scratch growth)
    small = sorted(inst, key=lambda d: d["spec"].points)[:2]
    sf.solve_stokes_batch_mixed(mixed_problems(small)[0], options=opts)
    for d in small:
        fp64_solve(d, _state_arrays(sf, d["spec"].Nx, d["spec"].Ny))
    probs, arrs = mixed_problems(inst)
    arena = sum(sf.Engine.instance_bytes(d["spec"].Nx, d["spec"].Ny) for d in inst)
    clocks = ClockSampler(0)
    clocks.start()
    # ---- the engine: every instance admitted at once, rounds until all have left ----
    lat_m = [None] * len(inst)
    with sf.Engine(arena, len(inst), options=opts) as eng:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pid = {id(p): q for q, p in enumerate(probs)}
        for p in probs:
            assert eng.submit(p) is not None
        while eng.active:
            for p in eng.step():
                lat_m[pid[id(p)]] = time.perf_counter() - t0
        torch.cuda.synchronize()
        mixed_s = time.perf_counter() - t0
        tiles = eng.stats()
    res = [p.result for p in probs]
    # ---- plain FP64, one solve after the other ----
    fp64_arrs = [_state_arrays(sf, d["spec"].Nx, d["spec"].Ny) for d in inst]
    lat_f, infos = [], []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for d, s in zip(inst, fp64_arrs):
        infos.append(fp64_solve(d, s))
        lat_f.append(time.perf_counter() - t0)
    fp64_s = time.perf_counter() - t0
    # ---- plain FP64, K solves at a time ----
    conc = None
    if concurrency > 1:
        conc_arrs = [_state_arrays(sf, d["spec"].Nx, d["spec"].Ny) for d in inst]
        nxt = iter(range(len(inst)))
        lock = threading.Lock()
        lat_c = [None] * len(inst)
        errs = []

        def worker():
            ctx = sf.Context(0)
            try:
                with torch.cuda.stream(torch.cuda.Stream()):
                    while True:
                        with lock:
                            q = next(nxt, None)
                        if q is None or errs:
                            break
                        fp64_solve(inst[q], conc_arrs[q], ctx)
                        lat_c[q] = time.perf_counter() - t1
            except BaseException as e:
                errs.append(e)
            finally:
                torch.cuda.synchronize()
                ctx.close()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ths = [threading.Thread(target=worker) for _ in range(concurrency)]
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        if errs:
            raise errs[0]
        conc_s = time.perf_counter() - t1
        conc = {"workers": concurrency, "solves_per_s": round(len(inst) / conc_s, 4), "s": round(conc_s, 3),
                "p50_latency_s": round(stats.median(lat_c), 3),
                "p99_latency_s": round(float(_percentile(lat_c, 99)), 3)}
        del conc_arrs
    clk = clocks.stop()
    names = ("Vx_pad", "Vy_pad", "P")
    ok = [q for q in range(len(inst)) if res[q]["status"] == 0 and infos[q]["converged"] and res[q]["converged"]]
    l2 = [_fields_l2(arrs[q], fp64_arrs[q], names) for q in ok]
    pts = [d["spec"].points for d in inst]
    mixed_rate = len(inst) / mixed_s
    fp64_rate = len(inst) / fp64_s
    out = {"form": "batch", "metric": f"Stokes solves/s to relative residual {a.rtol:g}, independent instances",
           "unit": "solves/s", "solves_per_s": round(mixed_rate, 4), "fp64_loop_solves_per_s": round(fp64_rate, 4),
           "speedup_solves_per_s": round(mixed_rate / fp64_rate, 3),
           "p50_latency_s": round(stats.median(lat_m), 3), "p99_latency_s": round(float(_percentile(lat_m, 99)), 3),
           "fp64_loop_p50_latency_s": round(stats.median(lat_f), 3),
           "fp64_loop_p99_latency_s": round(float(_percentile(lat_f, 99)), 3),
           "max_rel_l2": {f: max((x[f] for x in l2), default=None) for f in names},
           "median_rel_l2": {f: (sorted(x[f] for x in l2)[len(l2) // 2] if l2 else None) for f in names},
           "same_iterations": sum(1 for q in ok if res[q]["inner_iters"] == infos[q]["iters"]),
           "compared": len(ok), "instances": len(inst),
           "converged": sum(r["converged"] for r in res), "fp64_converged": sum(int(i["converged"]) for i in infos),
           "nonfinite": sum(1 for r in res if r["status"] == 5),
           "fp64_nonfinite": sum(int(i.get("nonfinite", 0)) for i in infos),
           "retried": sum(int(r.get("retried", 0)) for r in res),
           "mixed_s": round(mixed_s, 3), "fp64_loop_s": round(fp64_s, 3),
           "mixed_sweeps_total": int(sum(r["inner_iters"] for r in res)),
           "fp64_iters_total": int(sum(i["iters"] for i in infos)),
           "fp32_sweep_gpts": round(sum(r["inner_iters"] * pts[q] for q, r in enumerate(res)) / mixed_s / 1e9, 3),
           "sweep_tiles": {"rows": tiles["tile_rows"], "schedule": tiles["tile_schedule"],
                           "overlapped_launches": tiles["overlap_launches"], "tuner": tiles["tune_state"],
                           "classes_measured": tiles["tune_rounds"], "classes_recalled": tiles["tune_hits"]},
           "dtype": "f32 sweeps + f64 correction", "data": "synthetic (seeded random inclusion layouts)",
           "clocks": clk,
           "config": {"workload": f"{len(inst)} instances, cells per side log-uniform {cells}, 9-25 "
                                  f"markers/cell, 1-3 inclusions mu log10-uniform {a.mu_log10}, air mu "
                                  f"{a.mu_air:g}", "grid_points_total": int(sum(pts)),
                      "markers_total": int(sum(d['markers'] for d in inst)), "fold_every": a.fold_every,
                      "oracle": "plain FP64 path (bit-identical to the reference) at the same tolerance",
                      "seed": a.seed, "solve_cap": SOLVE_CAP}}
    if conc is not None:
        out["fp64_concurrent"] = conc
        out["speedup_vs_fp64_concurrent"] = round(mixed_rate / conc["solves_per_s"], 3)
    return out


def _percentile(xs, q):
    import numpy as np
    return np.percentile(np.asarray(xs, dtype=np.float64), q)


def run_serve_form(a, *, requests=None, rate=None, cells=None, concurrency=None):
    """Serving form: a Poisson stream of StokesFlow2D requests (1-20 timesteps each, random grids and
    inclusion layouts), continuous batching through the resident engine against plain FP64 serving on the
    same request trace: one request at a time in arrival order (the plain form as it is called), and, with
    concurrency K > 1, K workers with their own contexts and streams.  Each mixed request's final state
    (V, P, markers) is compared with the plain FP64 server's for the same request."""
    import stokesflow_b200 as sf
    from stokesflow_b200 import serving
    torch.cuda.set_device(0)
    requests = requests or a.serve_requests
    rate = rate or a.serve_rate
    cells = cells or a.serve_cells
    concurrency = a.fp64_concurrency if concurrency is None else concurrency
    kw = dict(cells=_pair(cells, int), timesteps=_pair(a.serve_steps, int), mu_log10=_pair(a.mu_log10),
              mu_air=a.mu_air)
    budget = int(a.hbm_budget_gb * 2 ** 30)
    opts = sf.mixed_options(max_sweeps=SOLVE_CAP, fold_every=a.fold_every, tile_rows=a.tile_rows,
                            tile_schedule=a.tile_schedule)
    # warm-up: one small request through each server
    for solver in ("mixed", "fp64"):
        w = serving.poisson_requests(1, 0.0, a.seed + 1, cells=(31, 31), timesteps=(1, 1))
        srv = serving.StokesServer(budget // 8, solver=solver, rtol=a.rtol, options=opts, iter_max=SOLVE_CAP)
        srv.run(w)
        srv.close()
    clocks = ClockSampler(0)
    clocks.start()
    out, finals = {}, {}
    runs = [("mixed", 1), ("fp64", 1)] + ([("fp64", concurrency)] if concurrency > 1 else [])
    for solver, k in runs:
        key = solver if k == 1 else f"fp64_x{k}"
        reqs = serving.poisson_requests(requests, rate, a.seed, **kw)
        srv = serving.StokesServer(budget, solver=solver, rtol=a.rtol, options=opts, iter_max=SOLVE_CAP,
                                   keep_final=(k == 1), concurrency=k)
        out[key] = srv.run(reqs)
        out[key]["peak_state_bytes"] = srv.peak_state
        if srv.engine is not None:
            out[key]["engine"] = srv.engine.stats()
        srv.close()
        if k == 1:
            finals[key] = {r.rid: r for r in reqs}
    clk = clocks.stop()
    names = ("Vx", "Vy", "P", "x_m", "y_m")
    l2 = []
    for rid, rm in finals["mixed"].items():
        rf = finals["fp64"][rid]
        if rm.failed or rf.failed or rm.final is None or rf.final is None:
            continue
        l2.append({f: _rel_l2(torch.from_numpy(rm.final[f]), torch.from_numpy(rf.final[f])) for f in names})
    m, f = out["mixed"], out["fp64"]
    res = {"form": "serve", "metric": f"p50/p99 request latency and solves/s at relative residual {a.rtol:g}",
           "unit": "s / solves/s", "solves_per_s": round(m["solves_per_s"], 3),
           "p50_latency_s": round(m["p50_latency_s"], 4), "p99_latency_s": round(m["p99_latency_s"], 4),
           "fp64_solves_per_s": round(f["solves_per_s"], 3), "fp64_p50_latency_s": round(f["p50_latency_s"], 4),
           "fp64_p99_latency_s": round(f["p99_latency_s"], 4),
           "speedup_solves_per_s": round(m["solves_per_s"] / f["solves_per_s"], 3),
           "max_rel_l2": {k: max((x[k] for x in l2), default=None) for k in names},
           "median_rel_l2": {k: (sorted(x[k] for x in l2)[len(l2) // 2] if l2 else None) for k in names},
           "compared_requests": len(l2), "mixed": m, "fp64": f, "clocks": clk,
           "data": "synthetic (seeded Poisson trace, random inclusion layouts)",
           "config": {"workload": f"{requests} requests at {rate:g}/s, square grids with cells per side "
                                  f"log-uniform {cells}, {a.serve_steps} timesteps, 9-25 markers/cell, inclusion "
                                  f"mu log10-uniform {a.mu_log10}, air mu {a.mu_air:g}",
                      "hbm_budget_bytes": budget, "fold_every": a.fold_every, "seed": a.seed,
                      "oracle": "the plain FP64 server's final V, P and markers of the same request"}}
    if concurrency > 1:
        c = out[f"fp64_x{concurrency}"]
        res["fp64_concurrent"] = {"workers": concurrency, "solves_per_s": round(c["solves_per_s"], 3),
                                  "p50_latency_s": round(c["p50_latency_s"], 4),
                                  "p99_latency_s": round(c["p99_latency_s"], 4)}
        res["speedup_vs_fp64_concurrent"] = round(m["solves_per_s"] / c["solves_per_s"], 3)
    return res


def _brief(d, keys):
    return {k: d[k] for k in keys if k in d}


def run_forms(a):
    """The three further forms, bounded so that they add a few minutes to the default run: a batch of
    forms_batch instances of the batching workload with the full plain FP64 loop over the same instances, a
    serve trace of forms_requests requests (against the plain FP64 server one request at a time and with
    fp64_concurrency workers), and one precision case of forms_precision_n^2 grid points."""
    forms = {}
    t0 = time.perf_counter()
    b = run_batch_form(a, instances=a.forms_batch, cells=a.batch_cells, concurrency=1)
    forms["batch"] = _brief(b, ("solves_per_s", "fp64_loop_solves_per_s", "speedup_solves_per_s", "p50_latency_s",
                                "p99_latency_s", "fp64_loop_p50_latency_s", "fp64_loop_p99_latency_s", "max_rel_l2",
                                "median_rel_l2", "same_iterations", "compared", "instances", "converged",
                                "fp64_converged", "clocks", "config"))
    # the plain FP64 server both one request at a time (the plain form as it is called) and with
    # fp64_concurrency workers, so that the batching gain and the precision gain can be told apart
    s = run_serve_form(a, requests=a.forms_requests, rate=a.forms_rate, cells=a.forms_cells,
                       concurrency=a.fp64_concurrency)
    forms["serve"] = _brief(s, ("solves_per_s", "p50_latency_s", "p99_latency_s", "fp64_solves_per_s",
                                "fp64_p50_latency_s", "fp64_p99_latency_s", "speedup_solves_per_s",
                                "fp64_concurrent", "speedup_vs_fp64_concurrent", "max_rel_l2", "median_rel_l2",
                                "compared_requests", "clocks", "config"))
    forms["serve"]["requests"] = s["mixed"]["requests"]
    forms["serve"]["solves"] = s["mixed"]["solves"]
    p = run_precision_form(a, n=a.forms_precision_n, cases=1, steps=a.forms_precision_steps,
                           contrast=a.precision_contrast)
    forms["precision"] = _brief(p, ("solves_per_s", "fp64_solves_per_s", "solve_speedup", "max_rel_l2",
                                    "same_iterations", "clocks", "config"))
    forms["precision"]["iterations"] = [[r["fp64_iters"], r["mixed_sweeps"]] for r in p["cases"][0]["steps"]]
    forms["precision"]["sweeps"] = p["cases"][0]["sweeps"]
    forms["wall_s"] = round(time.perf_counter() - t0, 1)
    forms["bar"] = {"rel_l2": 1e-5, "speedup_solves_per_s": 1.8,
                    "note": "rel L2 of the FP32-with-correction result against the plain FP64 path (the oracle) at "
                            "the same relative residual; speed-ups against the plain FP64 path on the same GPU"}
    return forms


def run_reference(a, rank):
    if rank != 0:
        return None
    n = os.cpu_count() or 1
    cpu_sample(a, 2, n)  # warm the oracle (first touch of the arrays)
    vals, dets = [], []
    for _ in range(max(a.warmup, 0)):
        cpu_sample(a, a.cpu_iters, n)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        v, d = cpu_sample(a, a.cpu_iters, n)
        vals.append(v)
        dets.append(d)
    wall = time.perf_counter() - t0
    value = statistics.median(vals)
    return {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(wall * 1e3 / a.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded plume model)", "config": bench_config(a),
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": n, "kind": "port",
                             "sample": f"each step: deposit of rho_vy + {a.cpu_iters} PT iterations of the "
                                       f"{a.n}^2 solve, OpenMP over {n} threads",
                             "cpu": _cpu_model(), "detail": dets},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0,
            "note": "a step here is one bounded sample (one grid's serial deposit, then the PT iterations above), "
                    "timed on the host cores; value is the sample's PT T_eff (the deposit is outside it), so "
                    "ms_per_step is not a timestep"}


# ---------------------------------------------------------------------------
def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if a.pt_probe:
        torch.cuda.set_device(local_rank)
        pt_probe(a)
        return
    if a.pt32_probe:
        torch.cuda.set_device(local_rank)
        pt32_probe(a)
        return
    if a.form != "timestep" and a.impl == "ours":
        if rank == 0:
            run = {"precision": run_precision_form, "batch": run_batch_form, "serve": run_serve_form,
                   "tune": run_tune_form, "decomposed": run_decomposed_form}[a.form]
            print(json.dumps(run(a)), flush=True)
        return
    if a.impl == "reference":
        out = run_reference(a, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if world > 1:
        import datetime
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        out = run_ours(a, rank, world, local_rank)
        if world == 1 and not a.no_forms:
            out["forms"] = run_forms(a)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
