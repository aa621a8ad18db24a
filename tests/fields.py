"""Test inputs shared by the CPU and GPU tests (numpy, Julia layout)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_golden.json")


def golden():
    with open(GOLDEN) as f:
        return json.load(f)


def F(*shape):
    return np.zeros(shape, dtype=np.float64, order="F")


def solver_test_fields(Nx=26, Ny=32, dx=0.5, dy=0.4):
    """rho_vy, mu_b, mu_p of test/test_StokesSolver.jl:62-82 (Gaussian blobs)."""
    lxg, lyg = dx * (Nx - 1), dy * (Ny - 1)
    xmid, ymid = 0.5 * lxg, 0.5 * lyg
    x = np.array([(ix - 1) * dx for ix in range(1, Nx + 1)])
    y = np.array([(iy - 1) * dy for iy in range(1, Ny + 1)])
    xp = np.array([(ix - 1) * dx + 0.5 * dx for ix in range(1, Nx)])
    yp = np.array([(iy - 1) * dy + 0.5 * dy for iy in range(1, Ny)])
    xr = np.array([(ix - 1) * dx - 0.5 * dx for ix in range(1, Nx + 2)])
    yr = np.array([(iy - 1) * dy for iy in range(1, Ny + 1)])
    rho = np.asfortranarray(3.3 * np.exp(-0.01 * ((xr[:, None] - 1.1 * xmid) ** 2 + (yr[None, :] - 1.3 * ymid) ** 2)))
    mub = np.asfortranarray(np.exp(-0.025 * ((x[:, None] - 1.1 * xmid) ** 2 + (y[None, :] - 1.3 * ymid) ** 2)))
    mup = np.asfortranarray(np.exp(-0.025 * ((xp[:, None] - 1.1 * xmid) ** 2 + (yp[None, :] - 1.3 * ymid) ** 2)))
    return rho, mub, mup


def random_fields(Nx, Ny, seed=1, contrast=1e3):
    """Smooth-ish random parameter fields with a large viscosity contrast."""
    rng = np.random.default_rng(seed)
    rho = np.asfortranarray(0.8 + 0.4 * rng.random((Nx + 1, Ny)))
    mub = np.asfortranarray(np.exp(np.log(contrast) * rng.random((Nx, Ny))) / contrast ** 0.5)
    mup = np.asfortranarray(np.exp(np.log(contrast) * rng.random((Nx - 1, Ny - 1))) / contrast ** 0.5)
    return rho, mub, mup


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)
