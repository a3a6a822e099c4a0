"""The C header checked by a C compiler: tests/c/tbfp_abi_check.c includes
include/tbfp.h, is built with gcc -std=c99 -Wall -Wextra -Werror -pedantic and
linked against the in-tree libtbfp.so.  On the CPU it runs the calls that need
no device; on a GPU it makes one host-pointer solveFPS, compared with the same
solve through the Python binding (1e-12 relative)."""
import os
import subprocess

import numpy as np
import pytest

from tbfsolver_b200 import _native as N
from tbfsolver_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c", "tbfp_abi_check.c")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    build()
    out = str(tmp_path_factory.mktemp("cabi") / "tbfp_abi_check")
    libdir = os.path.dirname(N.LIB_PATH)
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-O1", "-I", os.path.join(ROOT, "include"),
           SRC, "-o", out, "-L", libdir, "-ltbfp", f"-Wl,-rpath,{libdir}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return out


def test_c_caller_compiles_and_runs_the_host_checks(exe):
    r = subprocess.run([exe, "cpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cpu checks ok" in r.stdout


@pytest.mark.gpu
def test_c_caller_solve_matches_the_python_binding(exe, tmp_path):
    import torch

    from tbfsolver_b200.fields import Field
    from tbfsolver_b200.grid import Grid
    from tbfsolver_b200.solver import FastPoissonSolver

    out = str(tmp_path / "psi.bin")
    r = subprocess.run([exe, "gpu", out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    nx, ny, nz = 32, 24, 16
    got = np.fromfile(out, dtype=np.float64).reshape(nz + 2, ny + 2, nx + 2)
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, True, 1.5)
    s = Field("cl", 1, nx, ny, nz)
    i = np.arange(1, nx + 1)[None, None, :]
    j = np.arange(1, ny + 1)[None, :, None]
    k = np.arange(1, nz + 1)[:, None, None]
    v = np.cos(2.0 * i * g.dx_fft) * np.sin(1.0 * j) + 0.25 * np.cos(3.0 * k * g.dz_fft)
    V = g.dxf.r(1, nx)[None, None, :] * g.dyf.r(1, ny)[None, :, None] * g.dzf.r(1, nz)[:, None, None]
    s.interior()[...] = v - np.sum(v * V) / np.sum(V)
    with FastPoissonSolver(g) as fps:
        p = Field("cl", 1, nx, ny, nz, torch.zeros(s.a.shape, dtype=torch.float64, device="cuda"))
        fps.solve_fps(p, Field.like(s, torch.from_numpy(s.a.copy()).cuda()))
        want = p.a.cpu().numpy()
    assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < 1e-12
