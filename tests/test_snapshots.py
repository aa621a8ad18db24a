"""Snapshot files in the reference's .mat layout (StokesFlow2D_multixpu.jl:242-299): names, variables,
Float32 values in the Julia shapes, coordinate vectors of :117-124."""
import os
from types import SimpleNamespace

import numpy as np
import pytest
import scipy.io
import torch

from stokesflow_b200.snapshots import SnapshotWriter, grid_coordinates


def julia_array(nx, ny, base):
    """A column-major (nx, ny) CPU tensor, like the library's grids: entry (i, j) = base + i + 1000 j."""
    t = torch.empty(ny, nx, dtype=torch.float64).t()
    i = torch.arange(nx, dtype=torch.float64)[:, None]
    j = torch.arange(ny, dtype=torch.float64)[None, :]
    t.copy_(base + i + 1000.0 * j + 0.123456789)
    return t


def fake_state(Nx=7, Ny=5, nm=11):
    return SimpleNamespace(Nx=Nx, Ny=Ny, dx=1.0 / (Nx - 1), dy=1.0 / (Ny - 1),
                           x_m=torch.linspace(0, 1, nm, dtype=torch.float64),
                           y_m=torch.linspace(1, 0, nm, dtype=torch.float64),
                           rho_m=torch.arange(nm, dtype=torch.float64) / 3.0,
                           mu_b=julia_array(Nx, Ny, 1.0), P=julia_array(Nx - 1, Ny - 1, 2.0),
                           Vx=julia_array(Nx + 2, Ny + 1, 3.0), Vy=julia_array(Nx + 1, Ny + 2, 4.0))


def test_coordinates_follow_the_reference():
    c = grid_coordinates(4, 3, 0.5, 0.25)
    assert np.allclose(c["x"], [0, 0.5, 1.0, 1.5]) and np.allclose(c["y"], [0, 0.25, 0.5])
    assert np.allclose(c["x_p"], [0.25, 0.75, 1.25]) and np.allclose(c["y_p"], [0.125, 0.375])
    assert np.allclose(c["x_vx"], [-0.5, 0, 0.5, 1.0, 1.5, 2.0]) and np.allclose(c["y_vx"], [-0.125, 0.125, 0.375, 0.625])
    assert np.allclose(c["x_vy"], [-0.25, 0.25, 0.75, 1.25, 1.75]) and np.allclose(c["y_vy"], [-0.25, 0, 0.25, 0.5, 0.75])


def test_snapshot_files_cpu(tmp_path):
    st = fake_state()
    w = SnapshotWriter(str(tmp_path), st)
    w.snapshot(0)
    st.Vx.add_(1.0)          # the second snapshot sees the state as it is when taken
    w.snapshot(1)
    w.close()
    names = sorted(os.listdir(tmp_path))
    assert names == ["grid_0000_0000.mat", "grid_0001_0000.mat", "markers_0000_0000.mat", "markers_0001_0000.mat",
                     "stats.mat"]
    stats = scipy.io.loadmat(tmp_path / "stats.mat")
    assert int(stats["nt"].ravel()[0]) == 1 and stats["dims"].ravel().tolist() == [1, 1, 1]
    m = scipy.io.loadmat(tmp_path / "markers_0001_0000.mat")
    for k in ("x_m", "y_m", "rho_m"):
        assert m[k].dtype == np.float32 and m[k].shape == (11, 1)
        assert np.array_equal(m[k].ravel(), getattr(st, k).numpy().astype(np.float32))
    g0 = scipy.io.loadmat(tmp_path / "grid_0000_0000.mat")
    g1 = scipy.io.loadmat(tmp_path / "grid_0001_0000.mat")
    c = grid_coordinates(st.Nx, st.Ny, st.dx, st.dy)
    for k, v in c.items():
        assert g1[k].dtype == np.float32 and g1[k].shape == (v.size, 1)
        assert np.array_equal(g1[k].ravel(), v.astype(np.float32))
    for k in ("mu_b", "P", "Vx", "Vy"):
        ref = getattr(st, k).numpy().astype(np.float32)          # (nx, ny), Julia orientation
        assert g1[k].dtype == np.float32 and g1[k].shape == ref.shape
        assert np.array_equal(g1[k], ref), k
    assert np.array_equal(g0["Vx"] + 1.0, g1["Vx"])


@pytest.mark.gpu
def test_snapshots_of_a_run(sf, tmp_path):
    model = sf.plume_model_unit_square()
    model.mu_air = 1e-2
    Vx, Vy, t_tot, st = sf.stokes_flow_2d(2, 24, 20, 1.0, 1.0, model, marker_density=3, stokes_rtol=1e-6,
                                         save_to_file=True, out_dir=str(tmp_path), return_state=True)
    names = sorted(os.listdir(tmp_path))
    assert names == ["grid_0000_0000.mat", "grid_0001_0000.mat", "grid_0002_0000.mat", "markers_0000_0000.mat",
                     "markers_0001_0000.mat", "markers_0002_0000.mat", "stats.mat"]
    g = scipy.io.loadmat(tmp_path / "grid_0002_0000.mat")
    assert np.array_equal(g["Vx"], Vx.astype(np.float32)) and np.array_equal(g["Vy"], Vy.astype(np.float32))
    m = scipy.io.loadmat(tmp_path / "markers_0002_0000.mat")
    assert np.array_equal(m["x_m"].ravel(), st.x_m.cpu().numpy().astype(np.float32))
    g0 = scipy.io.loadmat(tmp_path / "grid_0000_0000.mat")
    assert not g0["Vx"].any() and not g0["mu_b"].any()      # saved before the first deposit, as the reference
