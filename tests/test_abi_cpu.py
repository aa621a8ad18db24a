"""CPU-side checks of the product library: it builds for sm_100a, loads without a
GPU, exports every function include/*.h declares, and its host-only entry
points (marker layout, material properties, seeded generator) agree bit for
bit with the oracle.  No device compute is called here."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest
import torch

import stokesflow_b200 as sf
from stokesflow_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(sf_[A-Za-z0-9_]+)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def L():
    sf.build()
    return sf.lib()


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("sf_bilinear_marker_to_grid", "sf_solve_stokes", "sf_move_markers_rk4", "sf_rebin_markers",
                 "sf_ctx_create", "sf_ctx_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol(L):
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_ctypes_prototypes_cover_header():
    assert set(_lib.PROTOTYPES) == set(declared_functions())


def test_library_is_sm100a_build():
    so = open(_lib.LIB_PATH, "rb").read()
    assert b"sm_100a" in so or b"compute_100a" in so


def test_struct_layouts_match_the_header(tmp_path):
    """Every struct of the C ABI has the size and field offsets of its ctypes mirror (a C program compiled
    against include/stokesflow_b200.h prints them)."""
    mirrors = {}
    for cls in vars(_lib).values():
        if isinstance(cls, type) and issubclass(cls, C.Structure) and cls.__doc__:
            m = re.match(r"(sf_[a-z_]+)\.", cls.__doc__.strip())
            if m:
                mirrors[m.group(1)] = cls
    assert len(mirrors) >= 9
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "stokesflow_b200.h"', "int main(void) {"]
    for name, cls in mirrors.items():
        lines.append(f'printf("{name} %zu\\n", sizeof({name}));')
        for f, _ in cls._fields_:
            lines.append(f'printf("{name}.{f} %zu\\n", offsetof({name}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    import subprocess
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                        text=True).stdout.splitlines())
    for name, cls in mirrors.items():
        assert int(got[name]) == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert int(got[f"{name}.{f}"]) == getattr(cls, f).offset, f"{name}.{f}"


def test_status_strings(L):
    assert L.sf_status_string(0) == b"ok"
    assert L.sf_status_string(_lib.SF_ERR_NONFINITE) == b"non-finite residual"
    assert L.sf_version() >> 8 == 1


def test_ctx_create_without_gpu_fails_cleanly(L):
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = L.sf_ctx_create(0, C.byref(h))
    assert rc == _lib.SF_ERR_NO_DEVICE and not h.value


def test_uniform_matches_oracle(L, oracle_lib):
    for seed in (0, 1, 12345):
        for k in (0, 1, 2, 1000, 2**40 + 7):
            assert L.sf_uniform(seed, k) == oracle_lib.uniform(seed, k)


@pytest.mark.parametrize("md,jitter", [(3, 0.0), (4, 0.5), (5, 1.0)])
def test_host_marker_init_matches_oracle(oracle_lib, md, jitter):
    Nx, Ny = 17, 12
    dx, dy = 1.0 / (Nx - 1), 1.3 / (Ny - 1)
    lx, ly = (Nx - 1) * dx, (Ny - 1) * dy
    x, y = sf.api.initialize_markers_host(md, lx, ly, dx, dy, Nx, Ny, jitter, 7)
    xo, yo = oracle_lib.initialize_markers(md, lx, ly, dx, dy, Nx, Ny, jitter, 7)
    assert np.array_equal(x.numpy(), xo) and np.array_equal(y.numpy(), yo)


def test_host_marker_properties_match_oracle(oracle_lib):
    m = sf.plume_model_unit_square()
    om = oracle_lib.PlumeModel(**{f: getattr(m, f) for f in m.FIELDS})
    x, y = sf.api.initialize_markers_host(4, 1.0, 1.0, 1 / 32, 1 / 32, 33, 33, 0.5, 0)
    rho, mu = sf.set_initial_marker_properties(x, y, m)
    ro, mo = oracle_lib.set_marker_properties(om, x.numpy(), y.numpy())
    assert np.array_equal(rho.numpy(), ro) and np.array_equal(mu.numpy(), mo)
    assert set(np.unique(ro)) == {1e-3, 0.9, 1.0}


def test_marker_count():
    assert sf.marker_count(4, 2048, 2048) == (8188, 8188)
    with pytest.raises(sf.StokesFlowError):
        sf.marker_count(0, 10, 10)


def test_api_rejects_host_tensors():
    with pytest.raises(TypeError):
        sf.api._grid(torch.zeros(3, 4, dtype=torch.float64), "A")


def test_node_origins_match_reference_formulas(oracle_lib):
    dx, dy = 10 / 19, 10 / 25
    assert sf.node_origins(dx, dy) == oracle_lib.node_origins(dx, dy)


def test_engine_instance_bytes_is_the_arena_layout(L):
    """An instance's arena block: 14 FP32 fields then 6 FP64 fields, each field LD x (Ny + 3) entries with
    LD = roundup(Nx + 4, 32), each part rounded up to 256 B.  Serving admits requests by this figure."""
    b = C.c_int64()
    for nx, ny in ((4, 4), (64, 64), (127, 1023), (2048, 2048), (1000, 33)):
        assert L.sf_engine_instance_bytes(nx, ny, C.byref(b)) == 0
        ld = -(-(nx + 4) // 32) * 32
        f = ld * (ny + 3)
        r256 = lambda v: -(-v // 256) * 256  # noqa: E731
        assert b.value == r256(14 * f * 4) + r256(6 * f * 8), (nx, ny)
    assert L.sf_engine_instance_bytes(3, 10, C.byref(b)) == _lib.SF_ERR_INVALID_ARG
    assert sf.Engine.instance_bytes(64, 64) == r256(14 * 96 * 67 * 4) + r256(6 * 96 * 67 * 8)
