"""Seeded synthetic workloads for the batched and served solve forms.

The reference has one material model (a plume in a matrix under sticky air:
the density / viscosity functions of scripts/StokesFlow2D_multixpu.jl:382-404,
applied per marker by ``setInitialMarkerProperties!``, scripts/common.jl:104-110).
The batched and
served forms run many independent problems of the same physics; each gets a
matrix with one to three circular inclusions of their own density and
viscosity under the same sticky-air layer.  Grid sizes are drawn
log-uniformly.  Everything is drawn from ``numpy.random.default_rng(seed)``,
so a workload is reproducible from its seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch


@dataclass
class InclusionModel:
    """Matrix + circular inclusions + sticky air for y < air_height (y grows downward, gravity +y).
    Inclusions are (x, y, r, rho, mu); a later inclusion overrides an earlier one where they overlap, and
    the air layer overrides both, as the air test comes first in the reference's plume model
    (StokesFlow2D_multixpu.jl:387-404)."""
    air_height: float = 0.1
    rho_air: float = 1e-3
    mu_air: float = 1e-2
    rho_matrix: float = 1.0
    mu_matrix: float = 1.0
    inclusions: list = field(default_factory=list)

    def marker_properties(self, x: torch.Tensor, y: torch.Tensor):
        """(rho_m, mu_m) of markers at (x, y) (device tensors)."""
        rho = torch.full_like(x, self.rho_matrix)
        mu = torch.full_like(x, self.mu_matrix)
        for (cx, cy, r, rh, m) in self.inclusions:
            inside = (x - cx) ** 2 + (y - cy) ** 2 < r * r
            rho = torch.where(inside, torch.full_like(x, rh), rho)
            mu = torch.where(inside, torch.full_like(x, m), mu)
        air = y < self.air_height
        rho = torch.where(air, torch.full_like(x, self.rho_air), rho)
        mu = torch.where(air, torch.full_like(x, self.mu_air), mu)
        return rho.contiguous(), mu.contiguous()


@dataclass
class InstanceSpec:
    """One problem of a batch: grid points (Nx, Ny) on the unit square, md x md markers per cell, material."""
    Nx: int
    Ny: int
    md: int
    model: InclusionModel
    seed: int

    @property
    def points(self) -> int:
        return self.Nx * self.Ny


def log_uniform_int(rng, lo, hi) -> int:
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


# gap of matrix kept between two inclusions, and draws of a position before an inclusion is left out
INCLUSION_GAP = 0.03
PLACEMENT_TRIES = 100


def random_inclusion_model(rng, *, n_inclusions=(1, 3), radius=(0.05, 0.2), rho=(0.8, 1.2), mu_log10=(-2.0, 1.0),
                           air_height=0.1, rho_air=1e-3, mu_air=1e-2) -> InclusionModel:
    """1-3 circular inclusions in a matrix of mu = 1, each touching only the matrix: it stays clear of the
    air layer and of the other inclusions by a gap of matrix.  The reference's PT scheme converges for a
    body of 1e-2 to 20 times the matrix viscosity against the matrix alone; a stiff body against the air
    (1e3) or against a soft body (1e-2 next to 10 is a 1e3 jump) makes it diverge (tests/
    test_oracle_contrast.py)."""
    k = int(rng.integers(n_inclusions[0], n_inclusions[1] + 1))
    inc = []
    for _ in range(k):
        r = float(rng.uniform(*radius))
        rh = float(rng.uniform(*rho))
        mu = float(10.0 ** rng.uniform(*mu_log10))
        top = air_height + r + 0.05
        for _ in range(PLACEMENT_TRIES):
            cx = float(rng.uniform(0.2, 0.8))
            cy = float(rng.uniform(top, max(top, 0.95 - r)))
            if all((cx - x) ** 2 + (cy - y) ** 2 >= (r + q + INCLUSION_GAP) ** 2 for (x, y, q, _, _) in inc):
                inc.append((cx, cy, r, rh, mu))
                break
    return InclusionModel(air_height=air_height, rho_air=rho_air, mu_air=mu_air, inclusions=inc)


def batch_specs(n: int, seed: int = 0, *, cells=(127, 1023), md=(3, 5), mu_log10=(-2.0, 1.0),
                mu_air=1e-2) -> list[InstanceSpec]:
    """n instances: cells per side log-uniform in `cells` (each side drawn on its own), md x md markers per
    cell with md uniform in `md` (3..5: 9-25 markers per cell), 1-3 inclusions with viscosity
    log-uniform over 10**mu_log10."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = log_uniform_int(rng, *cells)
        ny = log_uniform_int(rng, *cells)
        m = int(rng.integers(md[0], md[1] + 1))
        model = random_inclusion_model(rng, mu_log10=mu_log10, mu_air=mu_air)
        out.append(InstanceSpec(nx + 1, ny + 1, m, model, seed * 100003 + k))
    return out
