"""Channel grid of the reference solver (gridCTOR, src/grid/grid.f90:156-215).

Host-side set-up only: coordinates and metrics for one rank (local == global
mesh), with the halo gHD=3 the reference uses (grid.f90:173).  x and z are
uniform and periodic (checkGridSpacing, grid.f90:219-230); y is uniform or
tanh-stretched (coord_hyper_c/f, grid.f90:288-330) with the stretching factor
as a parameter (the reference hard-codes 1.4 at grid.f90:27).

Arrays are stored with their Fortran lower bound: ``g.dyc.v[j - g.dyc.lb]`` is
dyc(j); ``g.dyc.r(a, b)`` is the inclusive range dyc(a:b).
"""
from __future__ import annotations

import math

import numpy as np


class Arr1:
    """1-D array with a Fortran lower bound."""

    def __init__(self, lb: int, values):
        self.lb = int(lb)
        self.v = np.ascontiguousarray(values, dtype=np.float64)

    def __getitem__(self, i: int) -> float:
        return float(self.v[i - self.lb])

    def r(self, a: int, b: int) -> np.ndarray:
        return self.v[a - self.lb : b - self.lb + 1]


def _unif_c(lb, ub, L, n):  # grid.f90:235-257
    delta = L / n
    i = np.arange(lb, ub + 1, dtype=np.float64)
    return 0.5 * delta + (i - 1.0) * delta


def _unif_f(lb, ub, L, n):  # grid.f90:261-283
    delta = L / n
    return np.arange(lb, ub + 1, dtype=np.float64) * delta


def _hyper_c(lb, ub, L, n, gamma):  # grid.f90:288-307
    i = np.arange(lb, ub + 1, dtype=np.float64)
    return 0.5 * L * (1.0 + np.tanh(-gamma + 2.0 * gamma * (i - 0.5) / n) / math.tanh(gamma))


def _hyper_f(lb, ub, L, n, gamma):  # grid.f90:311-330
    i = np.arange(lb, ub + 1, dtype=np.float64)
    return 0.5 * L * (1.0 + np.tanh(-gamma + 2.0 * gamma * i / n) / math.tanh(gamma))


class Grid:
    """Mesh coordinates and metrics (grid.f90:633-807, :933-951)."""

    def __init__(self, nx: int, ny: int, nz: int, Lx: float, Ly: float, Lz: float,
                 y_stretched: bool = False, gamma: float = 1.4, hd: int = 3):
        if nx % 2:
            raise ValueError("nx must be even")
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.y_stretched, self.gamma, self.hd = bool(y_stretched), float(gamma), int(hd)
        g = self.hd
        self.xc = Arr1(1 - g, _unif_c(1 - g, nx + g, Lx, nx))
        self.zc = Arr1(1 - g, _unif_c(1 - g, nz + g, Lz, nz))
        self.xf = Arr1(-g, _unif_f(-g, nx + g, Lx, nx))
        self.zf = Arr1(-g, _unif_f(-g, nz + g, Lz, nz))
        if y_stretched:
            self.yc = Arr1(1 - g, _hyper_c(1 - g, ny + g, Ly, ny, gamma))
            self.yf = Arr1(-g, _hyper_f(-g, ny + g, Ly, ny, gamma))
        else:
            self.yc = Arr1(1 - g, _unif_c(1 - g, ny + g, Ly, ny))
            self.yf = Arr1(-g, _unif_f(-g, ny + g, Ly, ny))
        # metrics_centroids / metrics_faces (grid.f90:334-399)
        self.dxc = Arr1(self.xc.lb + 1, np.diff(self.xc.v))
        self.dyc = Arr1(self.yc.lb + 1, np.diff(self.yc.v))
        self.dzc = Arr1(self.zc.lb + 1, np.diff(self.zc.v))
        self.dxf = Arr1(self.xf.lb + 1, np.diff(self.xf.v))
        self.dyf = Arr1(self.yf.lb + 1, np.diff(self.yf.v))
        self.dzf = Arr1(self.zf.lb + 1, np.diff(self.zf.v))
        self.s_Vg = self._total_volume()

    def _total_volume(self) -> float:
        """totalVolume (grid.f90:933-951): sequential sum in loop order k, j, i."""
        dxf = self.dxf.r(1, self.nx)
        dyf = self.dyf.r(1, self.ny)
        dzf = self.dzf.r(1, self.nz)
        s = 0.0
        for k in range(self.nz):
            # V(i,j,k) = dxf(i)*dyf(j)*dzf(k) (grid.f90:801); cumsum is a strictly
            # left-to-right accumulation, so seeding it with the carry reproduces
            # the scalar loop bit for bit
            blk = ((dxf[None, :] * dyf[:, None]) * dzf[k]).ravel()
            s = float(np.cumsum(np.concatenate(([s], blk)))[-1])
        return s

    @property
    def dx_fft(self) -> float:
        """xc(2) - xc(1): the spacing of the x eigenvalues (fastPoissonSolver.f90:222)."""
        return self.xc[2] - self.xc[1]

    @property
    def dz_fft(self) -> float:
        return self.zc[2] - self.zc[1]

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz
