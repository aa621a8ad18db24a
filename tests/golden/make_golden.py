"""Extract the reference's golden vectors into tests/golden/reference_golden.json.

Reads the Julia test files of dastrm/StokesFlow.jl as text (nothing is run)
and records the known-answer values they assert, with the file:line they come
from, so the tests can pin the oracle without the reference present:

* test/test_StokesSolver.jl:49-51   solver, padded Vx / Vy at 20 linear indices
* test/test_StokesFlow2D.jl:86-88   5 timesteps of the full loop, Vx / Vy at 10 indices
* test/test_MarkerToGrid.jl:24-37   hand-computed 3x2 deposit

Usage:  python tests/golden/make_golden.py <StokesFlow.jl checkout>   (or set STOKESFLOW_REFERENCE)
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _array(src: str, name: str):
    m = re.search(r"^\s*" + re.escape(name) + r"\s*=\s*\[([^\]]*)\]", src, re.M)
    if not m:
        raise KeyError(name)
    line = src[: m.start()].count("\n") + 1
    vals = [float(v) if ("." in v or "e" in v.lower()) else int(v) for v in m.group(1).replace(",", " ").split()]
    return vals, line


def main(ref: str) -> None:
    out = {"source": "dastrm/StokesFlow.jl test files (values copied verbatim)"}
    src = open(os.path.join(ref, "test", "test_StokesSolver.jl")).read()
    inds, l1 = _array(src, "test_inds")
    vx, l2 = _array(src, "vx_ref")
    vy, l3 = _array(src, "vy_ref")
    out["stokes_solver"] = dict(
        cite=f"test/test_StokesSolver.jl:{l1}-{l3}", Nx=26, Ny=32, dx=0.5, dy=0.4, eps=1e-8, g_y=9.81, maxdisp=0.5,
        inds=inds, vx_ref=vx, vy_ref=vy,
        note="Julia `isapprox` on the vectors: norm(a-b) <= sqrt(eps(Float64)) * max(norm(a), norm(b))")
    src = open(os.path.join(ref, "test", "test_StokesFlow2D.jl")).read()
    inds, l1 = _array(src, "inds")
    vx, l2 = _array(src, "vxref")
    vy, l3 = _array(src, "vyref")
    out["stokes_flow_2d"] = dict(
        cite=f"test/test_StokesFlow2D.jl:{l1}-{l3}", Nt=5, Nx=20, Ny=26, Lx=10.0, Ly=10.0, marker_density=5,
        stokes_eps=1e-8, inds=inds, vx_ref=vx, vy_ref=vy, atol=1e-6,
        model=dict(air_height=2.0, plume_x=5.0, plume_y=5.0, plume_r=2.0, rho_air=1e-2, rho_matrix=3.3,
                   rho_plume=3.2, mu_air=1e-1, mu_matrix=1.0, mu_plume=5e-1))
    src = open(os.path.join(ref, "test", "test_MarkerToGrid.jl")).read()
    m = re.search(r"^reference = \[\[([^\]]*)\]\s*\[([^\]]*)\]\]", src, re.M)
    line = src[: m.start()].count("\n") + 1
    col1 = [float(v) for v in m.group(1).split(",")]
    col2 = [float(v) for v in m.group(2).split(",")]
    out["marker_to_grid_kat"] = dict(
        cite=f"test/test_MarkerToGrid.jl:25-{line}", x_grid_min=3.0, dx=1.4, y_grid_min=4.5, dy=2.0,
        x_m=[4.3, 5.6], y_m=[6.0, 4.8], val_m=[13.5, 10.0], shape=[3, 2], reference_columns=[col1, col2])
    with open(os.path.join(HERE, "reference_golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "reference_golden.json"))


if __name__ == "__main__":
    # the reference checkout: first argument, else $STOKESFLOW_REFERENCE
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("STOKESFLOW_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <StokesFlow.jl checkout>  (or set STOKESFLOW_REFERENCE)")
    main(ref)
