"""The sweep autotuner of the batched / served forms (sf_mixed_options.tile_rows / tile_schedule,
sf_ctx_batch_stats).

Every sweep tile shape (32 x 8, 32 x 16, 32 x 32) and schedule (strided, chunked) computes the same
arithmetic per point, so a batch solved with any fixed choice, or by the tuner (which switches between rounds
while it times them), gives bit-identical results; the tuner keeps the candidate it timed fastest, and the
context keeps that for the next solve of the same workload class."""
import numpy as np
import pytest

from fields import solver_test_fields
from stokesflow_b200._lib import StokesFlowError

pytestmark = pytest.mark.gpu


def specs():
    out = []
    for Nx, Ny in [(40, 37), (64, 64), (100, 70), (33, 90), (129, 65), (200, 131)]:
        dx, dy = 1.0 / (Nx - 1), 1.0 / (Ny - 1)
        out.append((Nx, Ny, dx, dy, solver_test_fields(Nx, Ny, dx * 12.5, dy * 12.4)))
    return out


def solve(sf, ctx, tile_rows, fold_every=50, schedule=None, overlap=False):
    import torch
    probs, arrs = [], []
    for (Nx, Ny, dx, dy, (rho, mub, mup)) in specs():
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()  # noqa: E731
        z = sf.zeros
        a = dict(P=z(Nx - 1, Ny - 1), Vx_pad=z(Nx + 2, Ny + 1), Vy_pad=z(Nx + 1, Ny + 2), rho_vy=dev(rho),
                 mu_b=dev(mub), mu_p=dev(mup), Vx_s=z(Nx, Ny + 1), Vy_s=z(Nx + 1, Ny))
        arrs.append(a)
        probs.append(sf.MixedProblem(a["P"], a["Vx_pad"], a["Vy_pad"], a["rho_vy"], a["mu_b"], a["mu_p"],
                                     a["Vx_s"], a["Vy_s"], 9.81, dx, dy, Nx, Ny, 0.0, 0.5, rel_tol=1e-8))
    opts = sf.mixed_options(fold_every=fold_every, tile_rows=tile_rows, tile_schedule=schedule,
                            overlap_launches=overlap)
    res = sf.solve_stokes_batch_mixed(probs, options=opts, ctx=ctx)
    out = [{k: a[k].cpu().numpy() for k in ("P", "Vx_pad", "Vy_pad")} for a in arrs]
    return out, res, sf.batch_stats(ctx)


def same(a, b):
    return all(np.array_equal(x[k], y[k]) for x, y in zip(a, b) for k in x)


def chosen(st):
    return f'{st["tile_rows"]}/{st["tile_schedule"]}/{"overlapped" if st["overlap_launches"] else "serial"}'


def test_every_shape_and_the_tuner_give_the_same_bits(sf):
    ctx = sf.Context(0)
    ref, res_ref, st = solve(sf, ctx, 16)
    assert st["tile_rows"] == 16 and st["tile_schedule"] == "strided" and st["tune_state"] == "fixed"
    assert all(r["converged"] == 1 for r in res_ref)
    for rows in (8, 16, 32):
        for sched in ("strided", "chunked"):
            for overlap in (False, True):
                if (rows, sched, overlap) == (16, "strided", False):
                    continue
                got, res, st = solve(sf, ctx, rows, schedule=sched, overlap=overlap)
                assert (st["tile_rows"], st["tile_schedule"], st["overlap_launches"]) == (rows, sched, int(overlap))
                assert [r["inner_iters"] for r in res] == [r["inner_iters"] for r in res_ref]
                assert same(got, ref), f"{rows}-row {sched} tiles (overlapped {overlap}) differ from the reference run"
    got, res, st = solve(sf, ctx, 0)               # the tuner times every candidate while it solves
    assert st["tune_rounds"] >= 1 and st["tune_classes"] >= 1, st
    assert all(v > 0 for v in st["tune_ns"].values())
    if st["tune_state"] == "measured":
        assert chosen(st) == min(st["tune_ns"], key=st["tune_ns"].get)
    assert same(got, ref), "the tuned solve differs"
    classes = st["tune_classes"]
    got, res, st = solve(sf, ctx, 0)               # the same classes again: the context remembers them
    assert st["tune_hits"] >= 1 and st["tune_classes"] >= classes, st
    assert same(got, ref)


def test_bad_tile_options_rejected(sf):
    with pytest.raises(StokesFlowError):
        solve(sf, sf.Context(0), 12)
    for field in ("tile_schedule", "overlap_launches"):   # without a fixed shape
        bad = sf.mixed_options()
        setattr(bad, field, 1)
        with pytest.raises(StokesFlowError):
            sf.Engine(arena_bytes=64 << 20, options=bad)


def test_engine_reports_its_shape(sf):
    with sf.Engine(arena_bytes=64 << 20, options=sf.mixed_options(tile_rows=32, tile_schedule="chunked")) as eng:
        st = eng.stats()
        assert st["tile_rows"] == 32 and st["tile_schedule"] == "chunked" and st["tune_state"] == "fixed"
    with sf.Engine(arena_bytes=64 << 20) as eng:
        assert eng.stats()["tune_state"] == "measuring"
