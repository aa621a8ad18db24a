"""The end-to-end timestep the benchmark's e2e figure measures: markers set up on the host and copied in from
pinned host memory before every step, markers and padded velocities copied out after it.  It computes the same
timesteps, bit for bit, as the device-resident state, and the host copies hold each step's results."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def _state(sf, **kw):
    model = sf.plume_model_unit_square()
    return sf.StokesFlow2D(41, 33, 1.0, 1.0, model, marker_density=4, stokes_rtol=1e-6, jitter=0.5, seed=3,
                           iter_max=40000, rebin=True, **kw)


def test_host_io_timesteps_equal_device_timesteps(sf):
    a = _state(sf)
    b = _state(sf, host_markers=True)
    for t in ("x_m", "y_m", "rho_m", "mu_m"):     # the host and device marker set-ups agree bit for bit
        assert torch.equal(getattr(a, t), getattr(b, t)), t
    for _ in range(3):
        ra, rb = a.step(), b.step(host_io=True)
        assert ra["info"]["iters"] == rb["info"]["iters"] and ra["dt"] == rb["dt"]
        for t in ("Vx", "Vy", "P", "x_m", "y_m", "rho_vy", "mu_b", "mu_p"):
            assert torch.equal(getattr(a, t), getattr(b, t)), t
        # what was copied out after the step is the step's result
        assert torch.equal(b.x_host, b.x_m.cpu()) and torch.equal(b.y_host, b.y_m.cpu())
        assert torch.equal(b._vx_host, b.Vx.t().cpu()) and torch.equal(b._vy_host, b.Vy.t().cpu())
        assert rb["times"].h2d_ms > 0.0 and rb["times"].d2h_ms > 0.0
    assert torch.equal(a.counts, b.counts) and torch.equal(a.cell_perm, b.cell_perm)
    nm = b.n_markers
    assert b.h2d_bytes_per_step() == 4 * 8 * nm
    assert b.d2h_bytes_per_step() == 2 * 8 * nm + 8 * (b.Vx.numel() + b.Vy.numel())
