"""The bounded waits of the persistent kernels, made to run out on the GPU without a fault: a barrier that
nothing completes (no trap, no bad address, no endless loop).  The wait gives up after its budget, the host
reads the status, and the context keeps working."""
import time

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_completed_barrier_does_not_time_out(sf):
    assert sf.selftest_bounded_wait(True, 200_000_000) is False


def test_wait_gives_up_after_its_budget_and_the_context_stays_usable(sf, oracle_lib):
    t0 = time.perf_counter()
    assert sf.selftest_bounded_wait(False, 50_000_000) is True
    elapsed = time.perf_counter() - t0
    assert 0.045 <= elapsed < 2.0
    # the same context runs a deposit afterwards, bit for bit as the oracle
    O = oracle_lib
    nx, ny, dx, dy = 9, 7, 0.25, 0.2
    rng = np.random.default_rng(3)
    x, y = rng.random(500) * (nx - 1) * dx, rng.random(500) * (ny - 1) * dy
    v = rng.random(500)
    ref = np.zeros((nx, ny), order="F")
    O.bilinear_marker_to_grid(0.0, 0.0, ref, x, y, v, dx, dy, np.zeros((nx, ny), order="F"),
                              np.zeros((nx, ny), order="F"))
    got = sf.zeros(nx, ny)
    d = lambda a: torch.from_numpy(a.copy()).cuda()  # noqa: E731
    sf.bilinear_marker_to_grid(0.0, 0.0, got, d(x), d(y), d(v), dx, dy)
    assert np.array_equal(np.asfortranarray(got.t().contiguous().cpu().numpy().T), ref)
    assert sf.selftest_bounded_wait(True, 200_000_000) is False


def test_budget_is_checked(sf):
    with pytest.raises(Exception):
        sf.selftest_bounded_wait(False, 0)
    with pytest.raises(Exception):
        sf.selftest_bounded_wait(False, 3_000_000_000)
