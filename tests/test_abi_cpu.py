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


def _ctypes_for_c(decl):
    """The ctypes types a C parameter (or return type) declaration may be bound with, by kind and width."""
    t = re.sub(r"\s+", "", re.sub(r"\b[A-Za-z_]\w*$", "", decl.strip()) if re.search(r"[\s*]\w+$", decl.strip())
               else decl)
    t = t.replace("const", "")
    structs = {c.__doc__.strip().rstrip("."): c for c in vars(_lib).values()
               if isinstance(c, type) and issubclass(c, C.Structure) and c.__doc__}
    scalars = {"double": (C.c_double,), "int64_t": (C.c_int64,), "int": (C.c_int, C.c_int32),
               "int32_t": (C.c_int32, C.c_int), "uint64_t": (C.c_uint64,), "char*": (C.c_char_p,)}
    if t in scalars:
        return scalars[t]
    if t in ("void*", "sf_ctx*", "sf_engine*"):
        return (C.c_void_p,)
    if t in ("sf_ctx**", "sf_engine**"):
        return (C.POINTER(C.c_void_p),)
    if t == "double*":                   # a device array passed as an address, or a host result
        return (C.c_void_p, C.POINTER(C.c_double))
    if t in ("int64_t*", "int32_t*"):   # a host result, or a device array passed as an address
        return (C.POINTER(scalars[t[:-1]][0]), C.c_void_p)
    if t.endswith("*") and t[:-1] in structs:
        return (C.POINTER(structs[t[:-1]]),)
    raise AssertionError(f"no ctypes rule for {decl!r}")


def _header_prototypes():
    text = re.sub(r"/\*.*?\*/", " ", "".join(open(h).read() for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))), flags=re.S)
    out = {}
    for m in re.finditer(r"\n\s*((?:const\s+)?[A-Za-z_]\w*\s*\**)\s*(sf_\w+)\s*\(([^;]*?)\)\s*;", text):
        params = m.group(3).strip()
        out[m.group(2)] = (m.group(1), [] if params in ("", "void") else [p.strip() for p in params.split(",")])
    return out


@pytest.mark.parametrize("name", sorted(_lib.PROTOTYPES))
def test_ctypes_prototype_matches_header(name):
    """Each ctypes prototype passes one argument per C parameter, of the same kind and width, so that no
    call truncates an int64_t or shifts the arguments after it."""
    protos = _header_prototypes()
    assert name in protos
    cret, cparams = protos[name]
    res, args = _lib.PROTOTYPES[name]
    assert res in _ctypes_for_c(cret), f"{name}: returns {cret}, bound as {res}"
    assert len(args) == len(cparams), f"{name}: {len(args)} ctypes arguments for {len(cparams)} C parameters"
    for k, (a, p) in enumerate(zip(args, cparams)):
        assert a in _ctypes_for_c(p), f"{name}: parameter {k} ({p}) bound as {a}"
