"""The C ABI from a plain C program: tests/c_abi_timestep.c is compiled against include/stokesflow_b200.h, linked
with the library and the CUDA runtime, and run -- one timestep (marker set-up, the fused deposit checked
against one call per grid, the PT solve, advection, rebin) with no Python between the caller and the kernels."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def test_c_program_runs_a_timestep_through_the_abi(sf, tmp_path):
    sf.build()
    libdir = os.path.dirname(sf.LIB_PATH)
    exe = tmp_path / "c_abi_timestep"
    subprocess.run(["gcc", "-std=c11", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "c_abi_timestep.c"),
                    "-L", libdir, "-lstokesflow_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart", "-lm",
                    "-o", str(exe)], check=True)
    env = dict(os.environ, LD_LIBRARY_PATH=os.pathsep.join([libdir, os.path.join(CUDA, "lib64"),
                                                            os.environ.get("LD_LIBRARY_PATH", "")]))
    r = subprocess.run([str(exe)], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("c abi ok")
