"""ctypes wrapper of the C/OpenMP oracle (oracle/tbfp_oracle.c).

TEST INFRASTRUCTURE ONLY: used by the tests as a second checker and by
bench.py as the timed CPU baseline.  Build with ``make -C oracle``.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libtbfp_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        P = C.c_void_p
        D = C.c_double
        I = C.c_int
        lib.tbfo_projection.restype = I
        lib.tbfo_projection.argtypes = [I, I, I, I, I, I, P, P, P, P, P, P, D, D, D, P, P, P, P, P, P, D, D, D, P,
                                        C.POINTER(D), I, I]
        lib.tbfo_max_threads.restype = I
        _lib = lib
    return _lib


def _p(a):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def projection(mesh, ux, uy, uz, rho, psi_n, psi_nm1, dt, alpha, rho0, psi, nthreads=0, pin00=False):
    """One projection on numpy arrays in the Fortran layout (u corrected in place,
    psi written); mesh is an oracle Mesh or a package Grid.  pin00 selects the
    exact gauge of the (0,0) system instead of the reference's epsilon pivot.
    Returns max|div u|."""
    lib = load()
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    m = [np.ascontiguousarray(x) for x in (mesh.dxf.r(1, nx), mesh.dxc.r(1, nx + 1), mesh.dyf.r(1, ny),
                                           mesh.dyc.r(1, ny + 1), mesh.dzf.r(1, nz), mesh.dzc.r(1, nz + 1))]
    hd_u = (ux.shape[2] - (nx + 1)) // 2
    hd_rho = (rho.shape[2] - nx) // 2
    hd_psi = (psi.shape[2] - nx) // 2
    md = C.c_double()
    rc = lib.tbfo_projection(nx, ny, nz, hd_psi, hd_u, hd_rho, *[_p(x) for x in m],
                             mesh.xc[2] - mesh.xc[1], mesh.zc[2] - mesh.zc[1], mesh.s_Vg,
                             _p(ux), _p(uy), _p(uz), _p(rho), _p(psi_n), _p(psi_nm1), dt, alpha, rho0, _p(psi),
                             C.byref(md), int(nthreads), int(bool(pin00)))
    if rc != 0:
        raise RuntimeError(f"tbfo_projection failed: {rc}")
    return md.value


def max_threads():
    return int(load().tbfo_max_threads())
