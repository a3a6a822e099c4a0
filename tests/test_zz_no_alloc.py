"""The allocation-free solve (tbfp_solve_fps_noalloc) against the handle-based
solve (tbfp_solve_fps_dev), through the C ABI.

The no-allocation entry point serves callers that cannot call cudaMalloc: a
driver that only hands over arrays it allocated itself, or code whose device
memory belongs to another runtime's pool.  It keeps its scratch in one static
device array shared by every call, so this test makes calls in a row -- two
sources on one grid, then a third call on a grid of other sizes (other
transform lengths and table sizes in the same array) -- and checks each against
the regular entry point, within the parity tolerance of the other GPU tests
(1e-12 relative).  This file is collected last so that a failure here does not
hide the others.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from tbfsolver_b200 import _native as N
from tbfsolver_b200.fields import Field
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import FastPoissonSolver

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _desc(g: Grid, keep: dict) -> N.TbfpDesc:
    nx, ny, nz = g.nx, g.ny, g.nz
    keep.update(dxf=np.ascontiguousarray(g.dxf.r(1, nx)), dxc=np.ascontiguousarray(g.dxc.r(1, nx + 1)),
                dyf=np.ascontiguousarray(g.dyf.r(1, ny)), dyc=np.ascontiguousarray(g.dyc.r(1, ny + 1)),
                dzf=np.ascontiguousarray(g.dzf.r(1, nz)), dzc=np.ascontiguousarray(g.dzc.r(1, nz + 1)))
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    return N.TbfpDesc(nx=nx, ny=ny, nz=nz, hd_psi=1, hd_u=2, hd_rho=1, hd_st=1, dx_fft=g.dx_fft, dz_fft=g.dz_fft,
                      dxf=p(keep["dxf"]), dxc=p(keep["dxc"]), dyf=p(keep["dyf"]), dyc=p(keep["dyc"]),
                      dzf=p(keep["dzf"]), dzc=p(keep["dzc"]), s_Vg=g.s_Vg, precision=0, tol=1e-10, max_iter=1,
                      device=-1, stream=None, flags=0)


def _source(g: Grid, seed: int) -> Field:
    """A seeded source with zero volume integral (compatible with the Neumann walls)."""
    rng = np.random.default_rng(seed)
    s = Field("cl", 1, g.nx, g.ny, g.nz)
    s.interior()[...] = rng.standard_normal((g.nz, g.ny, g.nx))
    V = (g.dxf.r(1, g.nx)[None, None, :] * g.dyf.r(1, g.ny)[None, :, None]) * g.dzf.r(1, g.nz)[:, None, None]
    s.interior()[...] -= np.sum(s.interior() * V) / g.s_Vg
    return Field.like(s, torch.from_numpy(s.a).cuda())


def _check_against_handle(lib, g: Grid, seed: int):
    keep = {}
    d = _desc(g, keep)
    with FastPoissonSolver(g) as fps:
        s = _source(g, seed)
        want = Field("cl", 1, g.nx, g.ny, g.nz, torch.zeros_like(s.a))
        fps.solve_fps(want, s)
        got = Field("cl", 1, g.nx, g.ny, g.nz, torch.full_like(s.a, 3.0))
        rc = lib.tbfp_solve_fps_noalloc(C.byref(d), s.a.data_ptr(), got.a.data_ptr())
        assert rc == 0, lib.tbfp_last_error(None)
        torch.cuda.synchronize()
        a, b = got.a.cpu().numpy(), want.a.cpu().numpy()
        assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < TOL, (g.nx, g.ny, g.nz, seed)


def test_noalloc_matches_the_handle_path_on_consecutive_calls():
    torch.cuda.set_device(0)
    lib = N.load()
    g = Grid(96, 64, 48, 2 * np.pi, 2.0, np.pi, y_stretched=True, gamma=1.5)
    for seed in (1, 2):  # two calls in a row share the static scratch
        _check_against_handle(lib, g, seed)
    # a third call on other sizes: stale tables or offsets of the previous grid would show here
    _check_against_handle(lib, Grid(64, 48, 32, 2 * np.pi, 2.0, np.pi, y_stretched=False, gamma=1.5), 3)
    assert torch.cuda.current_device() == 0


def test_noalloc_rejects_bad_metrics():
    lib = N.load()
    g = Grid(32, 24, 16, 2 * np.pi, 2.0, np.pi, y_stretched=True, gamma=1.5)
    keep = {}
    d = _desc(g, keep)
    keep["dyf"][3] = 0.0
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.tbfp_solve_fps_noalloc(C.byref(d), dummy.data_ptr(), dummy.data_ptr())
    assert rc == N.TBFP_EINVAL
    assert b"dyf" in lib.tbfp_last_error(None)


def test_noalloc_rejects_grids_beyond_its_static_scratch():
    lib = N.load()
    g = Grid(512, 384, 256, 2 * np.pi, 2.0, np.pi, y_stretched=True, gamma=1.5)
    keep = {}
    d = _desc(g, keep)
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = lib.tbfp_solve_fps_noalloc(C.byref(d), dummy.data_ptr(), dummy.data_ptr())
    assert rc == N.TBFP_EUNSUPPORTED
    assert b"static scratch" in lib.tbfp_last_error(None)
