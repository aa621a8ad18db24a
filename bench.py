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
TRAFFIC_PER_LAUNCH_2048 = 469.078e6   # dram__bytes_read.sum + dram__bytes_write.sum, k_pt_iter, 2047^2 points


# ---------------------------------------------------------------------------
def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=2048, help="grid points per side (cells = n - 1)")
    ap.add_argument("--markers-per-cell", type=int, default=16)
    ap.add_argument("--rtol", type=float, default=1e-6)
    ap.add_argument("--iter-max", type=int, default=400000,
                    help="PT iteration cap per solve (reference default 100000; a cold 2048^2 start needs ~250k)")
    ap.add_argument("--mu-air", type=float, default=1e-2,
                    help="air viscosity; 1e-3 makes the reference PT scheme diverge (see DESIGN.md)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-iters", type=int, default=12, help="PT iterations in the CPU baseline sample")
    ap.add_argument("--pt-probe", type=int, default=0, metavar="ITERS",
                    help="kernel probe: run ITERS fused PT iterations of an n x n solve (smooth random fields, no "
                         "markers) and print the kernel time; used for ncu captures")
    return ap.parse_args()


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
    # DRAM bytes (read + write) of one k_pt_iter launch from the ncu capture in
    # profiles/k_pt_iter_plume2048.md (2047^2 points), scaled by the point count
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
            "gpu_launches": 0}


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
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
