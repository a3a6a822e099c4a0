"""CPU tests of the C ABI boundary: the in-tree library builds/loads, exports
exactly what include/tbfp.h declares, and validates descriptors before touching
a GPU.  No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from tbfsolver_b200 import _native as N
from tbfsolver_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(tbfp_[a-z0-9_]+)\s*\(", txt))
    return names


@pytest.fixture(scope="module")
def lib():
    build()
    return N.load()


def test_library_exports_every_declared_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\bT (tbfp_\w+)", out.stdout))
    declared = declared_symbols()
    assert declared, "no declarations parsed"
    assert declared <= exported, f"declared but not exported: {sorted(declared - exported)}"
    assert set(N.PROTOTYPES) == declared, "ctypes prototypes and header disagree"


def test_version_and_strerror(lib):
    assert lib.tbfp_abi_version() == 1
    for code in (0, 1, -1, -2, -3, -4, -5, -6, -7, -8):
        assert lib.tbfp_strerror(code) != b"unknown status"
    assert lib.tbfp_strerror(12345) == b"unknown status"


def _desc(nx=16, ny=12, nz=8, **kw):
    arrs = {k: np.ones(n) for k, n in (("dxf", nx), ("dxc", nx + 1), ("dyf", ny), ("dyc", ny + 1), ("dzf", nz),
                                       ("dzc", nz + 1))}
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    d = N.TbfpDesc(nx=nx, ny=ny, nz=nz, hd_psi=1, hd_u=2, hd_rho=1, hd_st=1, dx_fft=1.0, dz_fft=1.0,
                   dxf=p(arrs["dxf"]), dxc=p(arrs["dxc"]), dyf=p(arrs["dyf"]), dyc=p(arrs["dyc"]),
                   dzf=p(arrs["dzf"]), dzc=p(arrs["dzc"]), s_Vg=0.0, precision=0, tol=1e-10, max_iter=4,
                   device=-1, stream=None, flags=0)
    for k, v in kw.items():
        setattr(d, k, v)
    return d, arrs


@pytest.mark.parametrize("bad,code", [
    (dict(nx=15), N.TBFP_EINVAL),        # odd nx: no r2c along x
    (dict(ny=2), N.TBFP_EINVAL),
    (dict(hd_psi=0), N.TBFP_EINVAL),     # the stencils read one ghost layer
    (dict(dx_fft=0.0), N.TBFP_EINVAL),
    (dict(precision=7), N.TBFP_EINVAL),
    (dict(nx=14), N.TBFP_EUNSUPPORTED),  # nx/2 = 7 has no 2/3 factorisation
])
def test_create_rejects_bad_descriptors(lib, bad, code):
    d, keep = _desc(**bad)
    h = C.c_void_p()
    rc = lib.tbfp_create(C.byref(d), C.byref(h))
    assert rc == code
    assert not h.value
    assert lib.tbfp_last_error(None)


def test_create_null_arguments(lib):
    h = C.c_void_p()
    assert lib.tbfp_create(None, C.byref(h)) == N.TBFP_ENULL
    d, keep = _desc()
    d.dyf = None
    assert lib.tbfp_create(C.byref(d), C.byref(h)) == N.TBFP_ENULL


def test_entry_points_reject_null_handle(lib):
    assert lib.tbfp_solve_fps(None, None, None) == N.TBFP_ENULL
    assert lib.tbfp_projection_dev(None, *([None] * 9), None, None, 1.0, 1.0, 1.0, None, None) == N.TBFP_ENULL
    assert lib.tbfp_destroy(None) == 0


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(N.TbfpError):
        N.load(str(tmp_path / "nope.so"))
