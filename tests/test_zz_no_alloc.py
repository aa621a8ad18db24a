"""The allocation-free deposit, sf_bilinear_marker_to_grid_noalloc.

It exists for callers that cannot let a library allocate device memory: a
host runtime that owns the GPU memory through its own pool, a stream loop that
cudaMalloc / cudaFree would stall with their device-wide synchronisation, or a
process held to a fixed memory budget.  Its scratch is a fixed array inside
the library that every call shares, so these tests call it twice in a row
(and once more with the first inputs) and check each result against the
regular entry point, sf_bilinear_marker_to_grid, bit for bit -- the tolerance
every deposit test here uses.  Both entry points are called through the C ABI.
One case is also checked directly against the CPU oracle's serial deposit, and
one test checks the property the entry point exists for: a call, after the
first on the device, leaves the device's free memory and the context's scratch
exactly as they were.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _col(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda().t()


def _case(seed, nx, ny, nm, dx, dy, x0, y0):
    rng = np.random.default_rng(seed)
    x = rng.random(nm) * (nx - 1) * dx + x0
    y = rng.random(nm) * (ny - 1) * dy + y0
    x[:2] = [x0 - 10.0, np.nan]            # two erroneous markers (skipped by both)
    v = np.exp(rng.normal(size=nm))
    start = np.asfortranarray(rng.random((nx, ny)))   # nodes without markers keep this
    return x, y, v, start


def _call_noalloc(sf, x0, y0, grid, xt, yt, vt, dx, dy):
    L = sf.lib()
    rc = L.sf_bilinear_marker_to_grid_noalloc(x0, y0, grid.data_ptr(), grid.shape[0], grid.shape[1], xt.data_ptr(),
                                              yt.data_ptr(), vt.data_ptr(), xt.numel(), dx, dy,
                                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    sf._lib.check(rc, "sf_bilinear_marker_to_grid_noalloc")


def _call_regular(sf, x0, y0, grid, xt, yt, vt, dx, dy):
    ctx = sf.default_context()
    L = sf.lib()
    rc = L.sf_bilinear_marker_to_grid(ctx.handle, x0, y0, grid.data_ptr(), grid.shape[0], grid.shape[1],
                                      xt.data_ptr(), yt.data_ptr(), vt.data_ptr(), xt.numel(), dx, dy, None, None, 0,
                                      0, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    sf._lib.check(rc, "sf_bilinear_marker_to_grid")


CASES = [
    # seed, nx, ny, markers, dx, dy, origin x, origin y  (2nd case: other grid, more markers, sparse corner)
    (1, 61, 47, 200_000, 0.02, 0.03, -0.01, 0.0),
    (2, 300, 200, 1_000_000, 0.005, 0.004, 0.0025, 0.002),
]


def test_noalloc_matches_regular_deposit_on_consecutive_calls(sf):
    results = []
    for seed, nx, ny, nm, dx, dy, x0, y0 in CASES + CASES[:1]:
        x, y, v, start = _case(seed, nx, ny, nm, dx, dy, x0, y0)
        xt, yt, vt = (torch.from_numpy(a).cuda() for a in (x, y, v))
        g_na, g_ref = _col(start), _col(start)
        _call_noalloc(sf, x0, y0, g_na, xt, yt, vt, dx, dy)
        _call_regular(sf, x0, y0, g_ref, xt, yt, vt, dx, dy)
        a, b = g_na.cpu().numpy(), g_ref.cpu().numpy()
        assert np.array_equal(a, b), f"noalloc deposit differs from the regular one (case seed {seed})"
        assert not np.array_equal(a, start.T.T)  # something was deposited
        results.append(a)
    # the third call repeats the first inputs after a larger call: nothing stale leaks through
    assert np.array_equal(results[0], results[2])


def test_noalloc_rejects_sizes_beyond_its_scratch(sf):
    L = sf.lib()
    t = torch.zeros(4, dtype=torch.float64, device="cuda")
    g = torch.zeros((2, 2), dtype=torch.float64, device="cuda")
    rc = L.sf_bilinear_marker_to_grid_noalloc(0.0, 0.0, g.data_ptr(), 2, 2, t.data_ptr(), t.data_ptr(), t.data_ptr(),
                                              sf._lib.SF_NOALLOC_MAX_MARKERS + 1, 1.0, 1.0, None)
    assert rc == sf._lib.SF_ERR_TOO_LARGE
    assert b"exceed" in L.sf_last_error()
    rc = L.sf_bilinear_marker_to_grid_noalloc(0.0, 0.0, g.data_ptr(), 600, 600, t.data_ptr(), t.data_ptr(),
                                              t.data_ptr(), 4, 1.0, 1.0, None)
    assert rc == sf._lib.SF_ERR_TOO_LARGE


def test_noalloc_matches_the_oracle(sf, oracle_lib):
    """The first case against the oracle's serial deposit (MarkerToGrid.jl:110-172 restated in C): the
    same bits, erroneous markers skipped and empty nodes keeping their value in both."""
    seed, nx, ny, nm, dx, dy, x0, y0 = CASES[0]
    x, y, v, start = _case(seed, nx, ny, nm, dx, dy, x0, y0)
    xt, yt, vt = (torch.from_numpy(a).cuda() for a in (x, y, v))
    g = _col(start)
    _call_noalloc(sf, x0, y0, g, xt, yt, vt, dx, dy)
    ref = np.asfortranarray(start.copy())
    vws, ws = oracle_lib.zeros(nx, ny), oracle_lib.zeros(nx, ny)
    oracle_lib.bilinear_marker_to_grid(x0, y0, ref, x, y, v, dx, dy, vws, ws)
    assert np.array_equal(g.cpu().numpy(), ref)


def test_noalloc_allocates_nothing(sf):
    """After a first call (which looks up the scratch address and loads the kernels), further calls on new
    grid sizes and marker counts change neither the device's free memory nor the default context's
    scratch."""
    seed, nx, ny, nm, dx, dy, x0, y0 = CASES[1]
    x, y, v, start = _case(seed, nx, ny, nm, dx, dy, x0, y0)
    xt, yt, vt = (torch.from_numpy(a).cuda() for a in (x, y, v))
    g = _col(start)
    _call_noalloc(sf, x0, y0, g, xt, yt, vt, dx, dy)
    small = _col(np.zeros((40, 30)))
    torch.cuda.synchronize()
    scratch0 = sf.default_context().scratch_bytes()
    free0, _ = torch.cuda.mem_get_info()
    for grid, k in ((small, nm // 3), (g, nm)):
        _call_noalloc(sf, x0, y0, grid, xt[:k], yt[:k], vt[:k], 0.025 if grid is small else dx,
                      0.035 if grid is small else dy)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert sf.default_context().scratch_bytes() == scratch0
