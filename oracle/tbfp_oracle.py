"""CPU oracle for the TBFsolver pressure-projection step (numpy/scipy restatement).

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library imports or calls this
module; only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it, and only as the checker.

Every function restates the reference Fortran (cifanip/TBFsolver) line by line
and cites the file:line it follows.  The reference itself cannot be built in
this environment (no Fortran compiler, MPI, FFTW, LAPACK or MUMPS), and the
reference ships no tests, golden vectors or fixtures for this path
(its example case ``channel_18`` has its input fields missing).  PARITY IS
UNPINNED against reference outputs; the restatement is pinned instead by
analytic known-answer tests (manufactured discrete solutions, single Fourier
modes, post-projection divergence) and by the fact that the tridiagonal step
calls the very LAPACK routines (``zgttrf``/``zgttrs``) the reference calls.

Array convention
----------------
A Fortran array ``f_(ilo:ihi, jlo:jhi, klo:khi)`` is held as a C-ordered numpy
array of shape ``(khi-klo+1, jhi-jlo+1, ihi-ilo+1)`` -- byte-for-byte the same
memory image as the Fortran column-major array.  ``FField`` carries the lower
bounds so code can index with the reference's (i, j, k) ranges.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field as dc_field

import numpy as np
from scipy.linalg import lapack

EPS64 = float(np.finfo(np.float64).eps)  # Fortran epsilon(0.d0)
TINY64 = float(np.finfo(np.float64).tiny)  # Fortran tiny(0.d0)

# field.f90:28-30 boundary types
FIXED_VALUE, NORMAL_GRADIENT, PERIODIC = 1, 2, 3


# ---------------------------------------------------------------------------
# 1-D arrays with Fortran lower bounds
# ---------------------------------------------------------------------------
class FArr1:
    """1-D array with a Fortran lower bound: ``a[i]`` and ``a.r(i0, i1)`` (inclusive)."""

    def __init__(self, lb: int, values: np.ndarray):
        self.lb = int(lb)
        self.v = np.asarray(values, dtype=np.float64)

    @property
    def ub(self) -> int:
        return self.lb + self.v.size - 1

    def __getitem__(self, i: int) -> float:
        return float(self.v[i - self.lb])

    def r(self, i0: int, i1: int) -> np.ndarray:
        return self.v[i0 - self.lb : i1 - self.lb + 1]


# ---------------------------------------------------------------------------
# grid.f90 restatement (single rank: local mesh == global mesh)
# ---------------------------------------------------------------------------
def _coord_unif_c(lb, ub, L, n):
    # grid.f90:235-257  q(i) = 0.5*delta + (n-1)*delta, n starting at i0-gHD == lb
    delta = L / n
    idx = np.arange(lb, ub + 1, dtype=np.float64)
    return 0.5 * delta + (idx - 1.0) * delta


def _coord_unif_f(lb, ub, L, n):
    # grid.f90:261-283  q(i) = n*delta, n starting at i0-1-gHD == lb
    delta = L / n
    idx = np.arange(lb, ub + 1, dtype=np.float64)
    return idx * delta


def _coord_hyper_c(lb, ub, L, n, gamma):
    # grid.f90:288-307 (the reference hard-codes s_gamma=1.4 at grid.f90:27;
    # the restatement takes gamma as a parameter)
    idx = np.arange(lb, ub + 1, dtype=np.float64)
    return 0.5 * L * (1.0 + np.tanh(-gamma + 2.0 * gamma * (idx - 0.5) / n) / math.tanh(gamma))


def _coord_hyper_f(lb, ub, L, n, gamma):
    # grid.f90:311-330
    idx = np.arange(lb, ub + 1, dtype=np.float64)
    return 0.5 * L * (1.0 + np.tanh(-gamma + 2.0 * gamma * idx / n) / math.tanh(gamma))


@dataclass
class Mesh:
    """Restatement of ``gridCTOR`` (grid.f90:156-215) for one rank, halo gHD=3."""

    nx: int
    ny: int
    nz: int
    Lx: float
    Ly: float
    Lz: float
    y_uniform: bool = True
    gamma: float = 1.4
    hd: int = 3
    xc: FArr1 = dc_field(init=False)
    yc: FArr1 = dc_field(init=False)
    zc: FArr1 = dc_field(init=False)
    xf: FArr1 = dc_field(init=False)
    yf: FArr1 = dc_field(init=False)
    zf: FArr1 = dc_field(init=False)
    dxc: FArr1 = dc_field(init=False)
    dyc: FArr1 = dc_field(init=False)
    dzc: FArr1 = dc_field(init=False)
    dxf: FArr1 = dc_field(init=False)
    dyf: FArr1 = dc_field(init=False)
    dzf: FArr1 = dc_field(init=False)
    s_Vg: float = dc_field(init=False)

    def __post_init__(self):
        g = self.hd
        nx, ny, nz = self.nx, self.ny, self.nz
        # computeCoordinates grid.f90:633-688 (x, z uniform: checkGridSpacing :219-230)
        self.xc = FArr1(1 - g, _coord_unif_c(1 - g, nx + g, self.Lx, nx))
        self.zc = FArr1(1 - g, _coord_unif_c(1 - g, nz + g, self.Lz, nz))
        self.xf = FArr1(0 - g, _coord_unif_f(0 - g, nx + g, self.Lx, nx))
        self.zf = FArr1(0 - g, _coord_unif_f(0 - g, nz + g, self.Lz, nz))
        if self.y_uniform:
            self.yc = FArr1(1 - g, _coord_unif_c(1 - g, ny + g, self.Ly, ny))
            self.yf = FArr1(0 - g, _coord_unif_f(0 - g, ny + g, self.Ly, ny))
        else:
            self.yc = FArr1(1 - g, _coord_hyper_c(1 - g, ny + g, self.Ly, ny, self.gamma))
            self.yf = FArr1(0 - g, _coord_hyper_f(0 - g, ny + g, self.Ly, ny, self.gamma))
        # metrics_centroids grid.f90:334-364: dxc(i) = xc(i)-xc(i-1), i = lb+1..ub
        self.dxc = FArr1(self.xc.lb + 1, np.diff(self.xc.v))
        self.dyc = FArr1(self.yc.lb + 1, np.diff(self.yc.v))
        self.dzc = FArr1(self.zc.lb + 1, np.diff(self.zc.v))
        # metrics_faces grid.f90:368-399
        self.dxf = FArr1(self.xf.lb + 1, np.diff(self.xf.v))
        self.dyf = FArr1(self.yf.lb + 1, np.diff(self.yf.v))
        self.dzf = FArr1(self.zf.lb + 1, np.diff(self.zf.v))
        # computeVolume grid.f90:784-807 and totalVolume :933-951 (loop order k, j, i)
        s = 0.0
        dxf = self.dxf.r(1, nx)
        dyf = self.dyf.r(1, ny)
        dzf = self.dzf.r(1, nz)
        for k in range(nz):
            # sequential accumulation in the Fortran loop order (cumsum is strictly
            # left to right; the carry is prepended)
            blk = ((dxf[None, :] * dyf[:, None]) * dzf[k]).ravel()
            s = float(np.cumsum(np.concatenate(([s], blk)))[-1])
        self.s_Vg = s

    def volume(self) -> np.ndarray:
        """V(i,j,k) = dxf(i)*dyf(j)*dzf(k) on the interior, shape (nz, ny, nx) (grid.f90:801)."""
        dxf = self.dxf.r(1, self.nx)
        dyf = self.dyf.r(1, self.ny)
        dzf = self.dzf.r(1, self.nz)
        return (dxf[None, None, :] * dyf[None, :, None]) * dzf[:, None, None]


# ---------------------------------------------------------------------------
# field.f90 restatement: storage with halos
# ---------------------------------------------------------------------------
_KIND_LO = {"cl": (1, 1, 1), "sx": (0, 1, 1), "sy": (1, 0, 1), "sz": (1, 1, 0)}


class FField:
    """Field ``f_(is-hd:ie+hd, js-hd:je+hd, ks-hd:ke+hd)`` (field.f90:271-273, :1746-1789)."""

    def __init__(self, kind: str, hd: int, nx: int, ny: int, nz: int, data: np.ndarray | None = None):
        lo = _KIND_LO[kind]
        self.kind, self.hd = kind, hd
        self.nx, self.ny, self.nz = nx, ny, nz
        self.lb = (lo[0] - hd, lo[1] - hd, lo[2] - hd)
        self.ub = (nx + hd, ny + hd, nz + hd)
        shape = (self.ub[2] - self.lb[2] + 1, self.ub[1] - self.lb[1] + 1, self.ub[0] - self.lb[0] + 1)
        if data is None:
            self.a = np.zeros(shape, dtype=np.float64)
        else:
            assert data.shape == shape, (data.shape, shape)
            self.a = data

    def v(self, i0, i1, j0, j1, k0, k1) -> np.ndarray:
        """View of the inclusive Fortran range (i0:i1, j0:j1, k0:k1)."""
        lb = self.lb
        return self.a[k0 - lb[2] : k1 - lb[2] + 1, j0 - lb[1] : j1 - lb[1] + 1, i0 - lb[0] : i1 - lb[0] + 1]

    def copy(self) -> "FField":
        return FField(self.kind, self.hd, self.nx, self.ny, self.nz, self.a.copy())

    def interior(self) -> np.ndarray:
        lo = _KIND_LO[self.kind]
        return self.v(lo[0], self.nx, lo[1], self.ny, lo[2], self.nz)


def update_boundaries_cl_channel(f: FField) -> None:
    """updateBoundaries (field.f90:950-974) for a cell field of the channel:
    normalGradient (bf=0) at the y walls (boundaryField_S.f90:694-727, one ghost
    layer on the interior i,k range), then the periodic halo exchange in x and
    then z over the full extended ranges (field.f90:708-788 with a single rank,
    whose Cartesian neighbours are itself)."""
    nx, ny, nz, hd = f.nx, f.ny, f.nz, f.hd
    f.v(1, nx, 0, 0, 1, nz)[...] = f.v(1, nx, 1, 1, 1, nz)
    f.v(1, nx, ny + 1, ny + 1, 1, nz)[...] = f.v(1, nx, ny, ny, 1, nz)
    jl, jh, kl, kh = 1 - hd, ny + hd, 1 - hd, nz + hd
    il, ih = 1 - hd, nx + hd
    # x: recv from right into ie+1.. <- is..is+hd-1 ; recv from left into is-hd.. <- ie-hd+1..ie
    f.v(nx + 1, nx + hd, jl, jh, kl, kh)[...] = f.v(1, hd, jl, jh, kl, kh)
    f.v(1 - hd, 0, jl, jh, kl, kh)[...] = f.v(nx - hd + 1, nx, jl, jh, kl, kh)
    # z (front-back) over all i, j
    f.v(il, ih, jl, jh, nz + 1, nz + hd)[...] = f.v(il, ih, jl, jh, 1, hd)
    f.v(il, ih, jl, jh, 1 - hd, 0)[...] = f.v(il, ih, jl, jh, nz - hd + 1, nz)


def equate_periodic_bc(ux: FField, uz: FField) -> None:
    """equatePeriodicBC (vfield.f90:124-189) on one rank: ux(0,:,:) = ux(nx,:,:),
    uz(:,:,0) = uz(:,:,nz) (y is wall-bounded, so uy is left alone)."""
    ux.v(0, 0, ux.lb[1], ux.ub[1], ux.lb[2], ux.ub[2])[...] = ux.v(ux.nx, ux.nx, ux.lb[1], ux.ub[1], ux.lb[2], ux.ub[2])
    uz.v(uz.lb[0], uz.ub[0], uz.lb[1], uz.ub[1], 0, 0)[...] = uz.v(uz.lb[0], uz.ub[0], uz.lb[1], uz.ub[1], uz.nz, uz.nz)


def wall_metrics(mesh: Mesh, kind: str):
    """setMetrics (boundaryField_S.f90:138-214) at the y walls:
    ((dhb, dhi) of the bottom, (dhb, dhi) of the top) for a field of type kind."""
    ny = mesh.ny
    if kind == "sy":
        return ((mesh.dyf[0], mesh.dyf[0] + mesh.dyf[1]), (mesh.dyf[ny + 1], mesh.dyf[ny] + mesh.dyf[ny + 1]))
    return ((mesh.yf[0] - mesh.yc[0], mesh.dyc[1]), (mesh.yc[ny + 1] - mesh.yf[ny], mesh.dyc[ny + 1]))


def update_boundaries_v_channel(mesh: Mesh, ux: FField, uy: FField, uz: FField, ubot=(0.0, 0.0, 0.0),
                                utop=(0.0, 0.0, 0.0)) -> None:
    """updateBoundariesV (vfield.f90:111-119) for the channel on one rank.  Per
    component, updateBoundaries (field.f90:950-974): the fixedValue walls in y
    (updateFixedValueBoundary, boundaryField_S.f90:593-690: one ghost layer over
    the interior i, k range, from the first interior layer -- the second for a
    'sy' field, whose walls are the faces j = 0 and ny -- with setMetrics'
    spacings), then the periodic halo exchanges in x and then z over the full
    extended ranges (updateHalo, field.f90:708-946; the rank is its own x and z
    neighbour, y has none); then equatePeriodicBC (vfield.f90:124-189).  ubot,
    utop: the wall values of ux, uy, uz (bvx3/bvx4 ... of the case's u file)."""
    for f, bb, bt in zip((ux, uy, uz), ubot, utop):
        nx, ny, nz, hd = f.nx, f.ny, f.nz, f.hd
        is_, js, ks = _KIND_LO[f.kind]
        ie, je, ke = nx, ny, nz
        (hb, hi), (tb, ti) = wall_metrics(mesh, f.kind)
        jb = js + 1 if f.kind == "sy" else js
        jt = je - 1 if f.kind == "sy" else je
        f.v(is_, ie, js - 1, js - 1, ks, ke)[...] = (f.v(is_, ie, jb, jb, ks, ke) * hb - bb * hi) / (hb - hi)
        f.v(is_, ie, je + 1, je + 1, ks, ke)[...] = (f.v(is_, ie, jt, jt, ks, ke) * tb - bt * ti) / (tb - ti)
        il, ih, jl, jh, kl, kh = is_ - hd, ie + hd, js - hd, je + hd, ks - hd, ke + hd
        # x: receive from the right into ie+1.. what it sends to the left, and
        # from the left into is-hd.. what it sends to the right
        if f.kind == "sx":
            f.v(ie + 1, ie + hd, jl, jh, kl, kh)[...] = f.v(is_ + 1, is_ + hd, jl, jh, kl, kh)
            f.v(is_ - hd, is_ - 1, jl, jh, kl, kh)[...] = f.v(ie - hd, ie - 1, jl, jh, kl, kh)
        else:
            f.v(ie + 1, ie + hd, jl, jh, kl, kh)[...] = f.v(is_, is_ + hd - 1, jl, jh, kl, kh)
            f.v(is_ - hd, is_ - 1, jl, jh, kl, kh)[...] = f.v(ie - hd + 1, ie, jl, jh, kl, kh)
        # z over all i, j
        if f.kind == "sz":
            f.v(il, ih, jl, jh, ke + 1, ke + hd)[...] = f.v(il, ih, jl, jh, ks + 1, ks + hd)
            f.v(il, ih, jl, jh, ks - hd, ks - 1)[...] = f.v(il, ih, jl, jh, ke - hd, ke - 1)
        else:
            f.v(il, ih, jl, jh, ke + 1, ke + hd)[...] = f.v(il, ih, jl, jh, ks, ks + hd - 1)
            f.v(il, ih, jl, jh, ks - hd, ks - 1)[...] = f.v(il, ih, jl, jh, ke - hd + 1, ke)
    equate_periodic_bc(ux, uz)


def _seq_sum(v: np.ndarray) -> float:
    """A sum in element order (loop order), one rounding per addition."""
    return float(np.cumsum(np.concatenate(([0.0], np.ravel(v))))[-1])


def staggered_x_volume(mesh: Mesh) -> np.ndarray:
    """Vsx(i,j,k) = dxc(i+1)*dyf(j)*dzf(k), i = 0..nx (grid.f90:812-838), as (nz, ny, nx+1)."""
    dx = mesh.dxc.r(1, mesh.nx + 1)[None, None, :]
    return (dx * mesh.dyf.r(1, mesh.ny)[None, :, None]) * mesh.dzf.r(1, mesh.nz)[:, None, None]


def set_press_grad(mesh: Mesh, rho: FField, flow_ctrl: int, ret: float, rhol: float, mul: float, g: float) -> float:
    """setPressGrad (auxiliaryRoutines.f90:336-393): fs from the mean density at
    the ux faces i = 0..nx-1 (the reference's OpenMP reduction has no fixed
    order; the restatement sums in loop order)."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    x = 0.5 * (rho.v(1, nx, 1, ny, 1, nz) + rho.v(0, nx - 1, 1, ny, 1, nz))
    rho_av = _seq_sum(x * staggered_x_volume(mesh)[:, :, :nx]) / mesh.s_Vg
    if flow_ctrl == 1:
        nul = mul / rhol
        re = 1.0 / nul
        tauw = (ret / re) * (ret / re)
        return tauw - rho_av * g
    if flow_ctrl in (2, 3):
        return -rho_av * g
    return 0.0


def compute_flow_rate(mesh: Mesh, ux: FField) -> float:
    """computeFlowRate (auxiliaryRoutines.f90:517-546): sum of ux*Vsx over i = 0..nx-1."""
    nx = mesh.nx
    return _seq_sum(ux.v(0, nx - 1, 1, mesh.ny, 1, mesh.nz) * staggered_x_volume(mesh)[:, :, :nx])


def set_flow_rate(mesh: Mesh, ux: FField, uy: FField, uz: FField, q0: float, flow_ctrl: int, ubot=(0.0, 0.0, 0.0),
                  utop=(0.0, 0.0, 0.0)) -> None:
    """setFlowRate (auxiliaryRoutines.f90:467-513): for flow_ctrl 2, ux += (Q0 - Q)/s_Vg
    over ux(0:nx,1:ny,1:nz), then updateBoundariesV."""
    if flow_ctrl != 2:
        return
    uf = (q0 - compute_flow_rate(mesh, ux)) / mesh.s_Vg
    t = ux.v(0, mesh.nx, 1, mesh.ny, 1, mesh.nz)
    t[...] = t + uf
    update_boundaries_v_channel(mesh, ux, uy, uz, ubot, utop)


# ---------------------------------------------------------------------------
# poissonEqn.f90 (FAST_MODE): split right-hand side
# ---------------------------------------------------------------------------
def compute_source_fast(mesh: Mesh, psi_n: FField, psi_nm1: FField, rho: FField,
                        ux: FField, uy: FField, uz: FField, dt: float, alpha: float, rho0: float,
                        st_n=None, st_nm1=None) -> np.ndarray:
    """computeSource (poissonEqn.f90:193-256) + computeOldPressDiv (:258-305), nl=2.

    ``st_n``/``st_nm1`` are (stx, sty, stz) FField triples or None (zero surface
    tension).  Returns the interior source s, shape (nz, ny, nx)."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    r = 1.0 / (alpha * dt)
    dxf1, dzf1 = mesh.dxf[1], mesh.dzf[1]
    dxc1, dzc1 = mesh.dxc[1], mesh.dzc[1]
    dyf = mesh.dyf.r(1, ny)[None, :, None]
    dycp = mesh.dyc.r(2, ny + 1)[None, :, None]  # dyc(j+1)
    dycm = mesh.dyc.r(1, ny)[None, :, None]  # dyc(j)

    def P(f, di=0, dj=0, dk=0):
        return f.v(1 + di, nx + di, 1 + dj, ny + dj, 1 + dk, nz + dk)

    ddx = (P(ux) - P(ux, di=-1)) / dxf1
    ddy = (P(uy) - P(uy, dj=-1)) / dyf
    ddz = (P(uz) - P(uz, dk=-1)) / dzf1
    s = ((ddx + ddy) + ddz) * r * rho0

    irc = 1.0 / P(rho)
    apx = 1.0 - rho0 * 0.5 * (1.0 / P(rho, di=1) + irc)
    amx = 1.0 - rho0 * 0.5 * (1.0 / P(rho, di=-1) + irc)
    apy = 1.0 - rho0 * 0.5 * (1.0 / P(rho, dj=1) + irc)
    amy = 1.0 - rho0 * 0.5 * (1.0 / P(rho, dj=-1) + irc)
    apz = 1.0 - rho0 * 0.5 * (1.0 / P(rho, dk=1) + irc)
    amz = 1.0 - rho0 * 0.5 * (1.0 / P(rho, dk=-1) + irc)

    def grad(dc, sh_p, sh_m):
        # 2*(pn(+)-pn(-)) - (pnm1(+)-pnm1(-)), divided by the centroid spacing
        g = 2.0 * (P(psi_n, **sh_p) - P(psi_n, **sh_m))
        g = g - (P(psi_nm1, **sh_p) - P(psi_nm1, **sh_m))
        return g / dc

    dpxp = grad(dxc1, dict(di=1), {})
    dpxm = grad(dxc1, {}, dict(di=-1))
    dpyp = grad(dycp, dict(dj=1), {})
    dpym = grad(dycm, {}, dict(dj=-1))
    dpzp = grad(dzc1, dict(dk=1), {})
    dpzm = grad(dzc1, {}, dict(dk=-1))
    if st_n is not None:
        sxn, syn, szn = st_n
        sxo, syo, szo = st_nm1
        dpxp = dpxp - 2.0 * P(sxn) + P(sxo)
        dpxm = dpxm - 2.0 * P(sxn, di=-1) + P(sxo, di=-1)
        dpyp = dpyp - 2.0 * P(syn) + P(syo)
        dpym = dpym - 2.0 * P(syn, dj=-1) + P(syo, dj=-1)
        dpzp = dpzp - 2.0 * P(szn) + P(szo)
        dpzm = dpzm - 2.0 * P(szn, dk=-1) + P(szo, dk=-1)

    ddx = (apx * dpxp - amx * dpxm) / dxf1
    ddy = (apy * dpyp - amy * dpym) / dyf
    ddz = (apz * dpzp - amz * dpzm) / dzf1
    return ((s + ddx) + ddy) + ddz


# ---------------------------------------------------------------------------
# fastPoissonSolver.f90: FFT(x,z) + tridiagonal(y) direct solve
# ---------------------------------------------------------------------------
def fps_eigenvalues(mesh: Mesh):
    """computeEigenvalues (fastPoissonSolver.f90:215-251): lx(i), i=1..nx, and lz(k)."""
    dx = mesh.xc[2] - mesh.xc[1]
    dz = mesh.zc[2] - mesh.zc[1]
    vx = np.arange(mesh.nx, dtype=np.float64) * 2.0 * math.pi
    vz = np.arange(mesh.nz, dtype=np.float64) * 2.0 * math.pi
    lx = 2.0 * (np.cos(vx / mesh.nx) - 1.0) / (dx * dx)
    lz = 2.0 * (np.cos(vz / mesh.nz) - 1.0) / (dz * dz)
    return lx, lz


def fps_offdiag(mesh: Mesh):
    """initOffDiagMatrix (fastPoissonSolver.f90:255-276): am(j), ap(j), j=1..ny."""
    ny = mesh.ny
    am = 1.0 / (mesh.dyc.r(1, ny) * mesh.dyf.r(1, ny))
    am[0] = 0.0
    ap = 1.0 / (mesh.dyc.r(2, ny + 1) * mesh.dyf.r(1, ny))
    ap[-1] = 0.0
    return am, ap


def solve_tridiag_lapack(spec: np.ndarray, lx: np.ndarray, lz: np.ndarray, am: np.ndarray, ap: np.ndarray,
                         pin00: bool = False) -> None:
    """solveTriDiag (fastPoissonSolver.f90:280-333) with the LAPACK routines the
    reference calls.  ``spec`` has shape (nz, ny, nkx) (complex, modified in place);
    system (kx, kz) runs along axis 1.  Row scaling by r=1/(lx+lz-am-ap) so the
    diagonal is 1; ``zgttrf``; if info != 0 the last U pivot becomes epsilon
    (:318-322); ``zgttrs``.

    pin00=True gauges the singular (0,0) system exactly instead: its last
    equation is replaced by x_ny = 0.  In exact arithmetic the epsilon pivot
    solves the same consistent system (the compatibility defect lands in the
    last row) shifted by a constant of order defect/epsilon, which the zero-mean
    step removes; in floating point that constant costs up to ~1e-11 relative
    accuracy, so parity checks at 1e-12 use the exact gauge."""
    nz, ny, nkx = spec.shape
    for kz in range(nz):
        for kx in range(nkx):
            r = 1.0 / (lx[kx] + lz[kz] - am - ap)
            am_s = (am * r).astype(np.complex128)
            ap_s = (ap * r).astype(np.complex128)
            ac = np.ones(ny, dtype=np.complex128)
            fy = spec[kz, :, kx] * r
            if pin00 and kx == 0 and kz == 0:
                am_s[ny - 1] = 0.0
                fy[ny - 1] = 0.0
            dl, d, du, du2, ipiv, info = lapack.zgttrf(am_s[1:].copy(), ac, ap_s[:-1].copy())
            if info != 0:
                d[ny - 1] = EPS64
            x, info2 = lapack.zgttrs(dl, d, du, du2, ipiv, fy)
            spec[kz, :, kx] = x


def solve_tridiag_thomas(spec: np.ndarray, lx: np.ndarray, lz: np.ndarray, am: np.ndarray, ap: np.ndarray,
                         pin00: bool = True) -> None:
    """Vectorised no-pivoting LU of the same scaled systems (a faster stand-in for
    the LAPACK call on large grids).  The singular (kx,kz)=(0,0) system is gauged
    exactly (last unknown pinned, see solve_tridiag_lapack) unless pin00=False,
    in which case it gets the epsilon-pivot rule of :318-322."""
    nz, ny, nkx = spec.shape
    lam = lz[:, None] + lx[None, :nkx]  # (nz, nkx)
    pin = np.zeros(lam.shape, dtype=bool)
    if pin00:
        pin[0, 0] = True
    cp = np.empty((ny, nz, nkx))
    dp = np.empty((ny, nz, nkx), dtype=np.complex128)
    r0 = 1.0 / (lam - am[0] - ap[0])
    c_prev = ap[0] * r0  # U(1,1) = 1
    d_prev = spec[:, 0, :] * r0
    cp[0] = c_prev
    dp[0] = d_prev
    piv = np.ones_like(lam)
    for j in range(1, ny):
        r = 1.0 / (lam - am[j] - ap[j])
        a = am[j] * r
        rhs = spec[:, j, :] * r
        if j == ny - 1:
            a = np.where(pin, 0.0, a)
            rhs = np.where(pin, 0.0, rhs)
        den = 1.0 - a * c_prev
        if j == ny - 1:
            den = np.where(den == 0.0, EPS64, den)
        c_prev = (ap[j] * r) / den
        d_prev = (rhs - a * d_prev) / den
        cp[j] = c_prev
        dp[j] = d_prev
    x = dp[ny - 1]
    spec[:, ny - 1, :] = x
    for j in range(ny - 2, -1, -1):
        x = dp[j] - cp[j] * x
        spec[:, j, :] = x
    del piv


def solve_fps(mesh: Mesh, s: np.ndarray, psi: FField, tridiag: str = "lapack-pinned") -> None:
    """solveFPS (fastPoissonSolver.f90:337-384): r2c along x (:353), c2c along z
    (:357), tridiagonal along y (:363), inverse z (:367) and c2r x (:371), scale by
    1/(nx*nz) (:374), zero volume-weighted mean (:380, :388-423), then
    updateBoundaries (:381).  All transforms unnormalised as FFTW's.
    tridiag: "lapack" (the reference's epsilon pivot), "lapack-pinned" (same
    routines, exact gauge of the (0,0) system; the default) or "thomas"."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    spec = np.fft.rfft(s, axis=2)  # (nz, ny, nx/2+1), unnormalised forward
    spec = np.fft.fft(spec, axis=0)
    lx, lz = fps_eigenvalues(mesh)
    am, ap = fps_offdiag(mesh)
    if tridiag == "lapack":
        solve_tridiag_lapack(spec, lx, lz, am, ap)
    elif tridiag == "lapack-pinned":
        solve_tridiag_lapack(spec, lx, lz, am, ap, pin00=True)
    elif tridiag == "thomas":
        solve_tridiag_thomas(spec, lx, lz, am, ap)
    else:
        raise ValueError(tridiag)
    spec = np.fft.ifft(spec, axis=0, norm="forward")  # unnormalised backward
    p = np.fft.irfft(spec, n=nx, axis=2, norm="forward")
    p = p / (nx * nz)
    psi.v(1, nx, 1, ny, 1, nz)[...] = p
    zero_average_pressure(mesh, psi)
    update_boundaries_cl_channel(psi)


def zero_average_pressure(mesh: Mesh, p: FField) -> None:
    """zeroAveragePressure (fastPoissonSolver.f90:388-423): p -= sum(p*V)/s_Vg,
    applied to the whole array including the halo (:421)."""
    av = float(np.sum(p.interior() * mesh.volume()))
    avg = av / mesh.s_Vg
    p.a -= avg


# ---------------------------------------------------------------------------
# momentumEqn.f90 (FAST_MODE) velocity correction
# ---------------------------------------------------------------------------
def make_velocity_div_free(mesh: Mesh, ux: FField, uy: FField, uz: FField, psi: FField,
                           psi_n: FField, psi_nm1: FField, rho: FField,
                           dt: float, alpha: float, rho0: float, st_n=None, st_nm1=None) -> None:
    """makeVelocityDivFree FAST (momentumEqn.f90:999-1090) + computeOldPressGrad
    (:1092-1127), in place.  Loop ranges follow setEqnBounds (:1134-1190) for the
    channel: ux i=0..nx (periodic), uy j=1..ny-1 (fixedValue walls excluded), uz
    k=0..nz.  Ends with the periodic equate of updateBoundariesV (vfield.f90:118,
    :124-189); the remaining ghost/halo refresh of u is the caller's."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    r = dt * alpha
    invrho0 = 1.0 / rho0

    def upd(u, i0, i1, j0, j1, k0, k1, di, dj, dk, dc, stc):
        def S(f, o=0):
            return f.v(i0 + di * o, i1 + di * o, j0 + dj * o, j1 + dj * o, k0 + dk * o, k1 + dk * o)

        invrho = 0.5 * (1.0 / S(rho, 1) + 1.0 / S(rho))
        dpr = (S(psi, 1) - S(psi)) / dc
        dpr0 = (2.0 * (S(psi_n, 1) - S(psi_n)) - (S(psi_nm1, 1) - S(psi_nm1))) / dc
        if st_n is not None:
            dpr0 = dpr0 - 2.0 * S(st_n[stc]) + S(st_nm1[stc])
        tgt = u.v(i0, i1, j0, j1, k0, k1)
        tgt -= r * (invrho0 * dpr + (invrho - invrho0) * dpr0)

    upd(ux, 0, nx, 1, ny, 1, nz, 1, 0, 0, mesh.dxc[1], 0)
    upd(uy, 1, nx, 1, ny - 1, 1, nz, 0, 1, 0, mesh.dyc.r(2, ny)[None, :, None], 1)
    upd(uz, 1, nx, 1, ny, 0, nz, 0, 0, 1, mesh.dzc[1], 2)
    equate_periodic_bc(ux, uz)


def compute_continuity_error(mesh: Mesh, ux: FField, uy: FField, uz: FField) -> float:
    """max|div u| over the interior (auxiliaryRoutines.f90:42-91), WITHOUT the
    final multiplication by dt (:82) so both forms can be reported."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    dxf = mesh.dxf.r(1, nx)[None, None, :]
    dyf = mesh.dyf.r(1, ny)[None, :, None]
    dzf = mesh.dzf.r(1, nz)[:, None, None]
    d = (ux.v(1, nx, 1, ny, 1, nz) - ux.v(0, nx - 1, 1, ny, 1, nz)) / dxf
    d = d + (uy.v(1, nx, 1, ny, 1, nz) - uy.v(1, nx, 0, ny - 1, 1, nz)) / dyf
    d = d + (uz.v(1, nx, 1, ny, 1, nz) - uz.v(1, nx, 1, ny, 0, nz - 1)) / dzf
    return float(np.max(np.abs(d))) if d.size else -1.0


def divergence(mesh: Mesh, ux: FField, uy: FField, uz: FField) -> np.ndarray:
    """The cell divergence field used by compute_continuity_error (auxiliaryRoutines.f90:71-75)."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    dxf = mesh.dxf.r(1, nx)[None, None, :]
    dyf = mesh.dyf.r(1, ny)[None, :, None]
    dzf = mesh.dzf.r(1, nz)[:, None, None]
    d = (ux.v(1, nx, 1, ny, 1, nz) - ux.v(0, nx - 1, 1, ny, 1, nz)) / dxf
    d = d + (uy.v(1, nx, 1, ny, 1, nz) - uy.v(1, nx, 0, ny - 1, 1, nz)) / dyf
    return d + (uz.v(1, nx, 1, ny, 1, nz) - uz.v(1, nx, 1, ny, 0, nz - 1)) / dzf


# ---------------------------------------------------------------------------
# The 7-point operator the split solve inverts (beta == 1 form of pcg.f90:163-176
# with the am/ap of fastPoissonSolver.f90:265-273 and periodic x, z).
# ---------------------------------------------------------------------------
def laplacian_fps(mesh: Mesh, psi: FField) -> np.ndarray:
    """L_h psi on the interior for a psi whose ghosts are up to date (Neumann walls
    via the ghost rows, periodic x/z via halos).  x and z use the uniform spacing
    dx=xc(2)-xc(1) exactly as the eigenvalues do; y uses am/ap."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    dx = mesh.xc[2] - mesh.xc[1]
    dz = mesh.zc[2] - mesh.zc[1]
    am, ap = fps_offdiag(mesh)
    c = psi.v(1, nx, 1, ny, 1, nz)
    lx = (psi.v(2, nx + 1, 1, ny, 1, nz) - 2.0 * c + psi.v(0, nx - 1, 1, ny, 1, nz)) / (dx * dx)
    lz = (psi.v(1, nx, 1, ny, 2, nz + 1) - 2.0 * c + psi.v(1, nx, 1, ny, 0, nz - 1)) / (dz * dz)
    ly = ap[None, :, None] * (psi.v(1, nx, 2, ny + 1, 1, nz) - c) - am[None, :, None] * (c - psi.v(1, nx, 0, ny - 1, 1, nz))
    return lx + ly + lz


# ---------------------------------------------------------------------------
# one projection, as called from main.f90:197-215 (FAST_MODE)
# ---------------------------------------------------------------------------
@dataclass
class ProjectionResult:
    psi: FField
    ux: FField
    uy: FField
    uz: FField
    s: np.ndarray
    max_div: float  # max|div u| (raw)
    cont_err: float  # dt * max|div u| (auxiliaryRoutines.f90:82)


def projection(mesh: Mesh, ux: FField, uy: FField, uz: FField, rho: FField, psi_n: FField,
               psi_nm1: FField, dt: float, alpha: float, rho0: float, st_n=None, st_nm1=None,
               tridiag: str = "lapack-pinned") -> ProjectionResult:
    """solvePoissonEqn (poissonEqn.f90:347-370) -> makeVelocityDivFree
    (momentumEqn.f90:999) -> computeContinuityError (auxiliaryRoutines.f90:42)
    on copies of the inputs.  psi_n / psi_nm1 are psi%ptrf_ and psi%ptrf_%ptrf_."""
    s = compute_source_fast(mesh, psi_n, psi_nm1, rho, ux, uy, uz, dt, alpha, rho0, st_n, st_nm1)
    psi = FField("cl", psi_n.hd, mesh.nx, mesh.ny, mesh.nz)
    solve_fps(mesh, s, psi, tridiag=tridiag)
    uxo, uyo, uzo = ux.copy(), uy.copy(), uz.copy()
    make_velocity_div_free(mesh, uxo, uyo, uzo, psi, psi_n, psi_nm1, rho, dt, alpha, rho0, st_n, st_nm1)
    md = compute_continuity_error(mesh, uxo, uyo, uzo)
    return ProjectionResult(psi, uxo, uyo, uzo, s, md, md * dt)


def alpha_rks(scheme: int, substep: int = 1) -> float:
    """alphaRKS (time.f90:99-105) with the tables of initRK3coef (time.f90:365-405)."""
    if scheme == 0:
        gamma, xi = (1.5, 0.0, 0.0), (-0.5, 0.0, 0.0)
    elif scheme == 1:
        gamma, xi = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0), (0.0, -17.0 / 60.0, -5.0 / 12.0)
    else:
        raise ValueError("invalid time integration scheme")
    return gamma[substep - 1] + xi[substep - 1]


# ===========================================================================
# MG_MODE: variable-coefficient oracle (PCG preconditioned by a red-black
# Gauss-Seidel multigrid V-cycle with a direct coarsest-level solve)
# ===========================================================================
class Level:
    """One multigrid level: grid metrics (coarsenGrid, grid.f90:490-544, halo 2
    on coarse levels), red/black masks (rbgsCTOR, rbgs.f90:115-153) and the
    1/(dc*df) metric tables (storeMetrics, rbgs.f90:489-521)."""

    def __init__(self, mesh: Mesh):
        self.m = mesh
        nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
        i = np.arange(1, nx + 1)[None, None, :]
        j = np.arange(1, ny + 1)[None, :, None]
        k = np.arange(1, nz + 1)[:, None, None]
        self.red = ((i + j + k) % 2 == 0)
        self.black = ~self.red
        self.invx1 = 1.0 / (mesh.dxc.r(2, nx + 1) * mesh.dxf.r(1, nx))  # invx(1,i)
        self.invx2 = 1.0 / (mesh.dxc.r(1, nx) * mesh.dxf.r(1, nx))      # invx(2,i)
        self.invy1 = 1.0 / (mesh.dyc.r(2, ny + 1) * mesh.dyf.r(1, ny))
        self.invy2 = 1.0 / (mesh.dyc.r(1, ny) * mesh.dyf.r(1, ny))
        self.invz1 = 1.0 / (mesh.dzc.r(2, nz + 1) * mesh.dzf.r(1, nz))
        self.invz2 = 1.0 / (mesh.dzc.r(1, nz) * mesh.dzf.r(1, nz))

    def coeffs(self, beta: FField):
        """Face coefficients aR..aBa of rbgs.f90:215-220 (and pcg.f90:163-168)."""
        nx, ny, nz = self.m.nx, self.m.ny, self.m.nz
        B = lambda di=0, dj=0, dk=0: beta.v(1 + di, nx + di, 1 + dj, ny + dj, 1 + dk, nz + dk)  # noqa: E731
        bc = B()
        aR = 0.5 * (B(di=1) + bc) * self.invx1[None, None, :]
        aL = 0.5 * (bc + B(di=-1)) * self.invx2[None, None, :]
        aT = 0.5 * (B(dj=1) + bc) * self.invy1[None, :, None]
        aBo = 0.5 * (bc + B(dj=-1)) * self.invy2[None, :, None]
        aF = 0.5 * (B(dk=1) + bc) * self.invz1[:, None, None]
        aBa = 0.5 * (bc + B(dk=-1)) * self.invz2[:, None, None]
        return aR, aL, aT, aBo, aF, aBa


def coarse_mesh(m: Mesh) -> Mesh:
    """coarsenGrid (grid.f90:490-544): half the cells, same box and stretching,
    coordinates recomputed with the reference formulas, halo 2."""
    return Mesh(m.nx // 2, m.ny // 2, m.nz // 2, m.Lx, m.Ly, m.Lz, y_uniform=m.y_uniform, gamma=m.gamma, hd=2)


def apply_L(lev: Level, p: FField, beta: FField, coeffs=None) -> np.ndarray:
    """L_beta p on the interior: the operator of computeQv (pcg.f90:171-176) and
    computeResiduals (rbgs.f90:308-317)."""
    m = lev.m
    nx, ny, nz = m.nx, m.ny, m.nz
    aR, aL, aT, aBo, aF, aBa = coeffs or lev.coeffs(beta)
    P = lambda di=0, dj=0, dk=0: p.v(1 + di, nx + di, 1 + dj, ny + dj, 1 + dk, nz + dk)  # noqa: E731
    c = P()
    return (aR * (P(di=1) - c) - aL * (c - P(di=-1)) + aT * (P(dj=1) - c) - aBo * (c - P(dj=-1))
            + aF * (P(dk=1) - c) - aBa * (c - P(dk=-1)))


def correct_full_neumann(m: Mesh, p: FField) -> None:
    """correctFullNeumann (rbgs.f90:403-446): remove the unweighted interior mean
    from the whole array (halo included)."""
    avg = float(np.sum(p.interior())) / (m.nx * m.ny * m.nz)
    p.a -= avg


def rbgs_iterate(lev: Level, p: FField, beta: FField, q: np.ndarray, n_iter: int, reset: bool, coeffs=None) -> None:
    """iterateGS (rbgs.f90:186-272): red sweep, boundary update, black sweep,
    boundary update, full-Neumann mean removal; every colour is updated from the
    values (and ghosts) left by the previous boundary update."""
    m = lev.m
    nx, ny, nz = m.nx, m.ny, m.nz
    if reset:
        p.a[...] = 0.0
    aR, aL, aT, aBo, aF, aBa = coeffs or lev.coeffs(beta)
    den = aR + aL + aT + aBo + aF + aBa
    P = lambda di=0, dj=0, dk=0: p.v(1 + di, nx + di, 1 + dj, ny + dj, 1 + dk, nz + dk)  # noqa: E731
    for _ in range(n_iter):
        for mask in (lev.red, lev.black):
            new = (-q + (aR * P(di=1) + aL * P(di=-1)) + (aT * P(dj=1) + aBo * P(dj=-1))
                   + (aF * P(dk=1) + aBa * P(dk=-1))) / den
            c = P()
            c[mask] = new[mask]
            update_boundaries_cl_channel(p)
        correct_full_neumann(m, p)


def compute_residuals(lev: Level, p: FField, beta: FField, q_full: FField, coeffs=None):
    """computeResiduals (rbgs.f90:276-333): resV = q - L_beta p and
    res = ||resV||_2 / (||q||_2 + tiny), the q norm over q's whole array."""
    resV = q_full.interior() - apply_L(lev, p, beta, coeffs)
    res = math.sqrt(float(np.sum(resV * resV))) / (math.sqrt(float(np.sum(q_full.a * q_full.a))) + TINY64)
    return resV, res


def restriction(mf: Mesh, mc: Mesh, qf: np.ndarray) -> np.ndarray:
    """restrictionOp3D (interpolation.f90:80-124): trilinear restriction from the
    fine centroids to the coarse centroids (interior arrays)."""
    xf, yf, zf = mf.xc.r(1, mf.nx), mf.yc.r(1, mf.ny), mf.zc.r(1, mf.nz)
    xc, yc, zc = mc.xc.r(1, mc.nx), mc.yc.r(1, mc.ny), mc.zc.r(1, mc.nz)
    xo, xe = xf[0::2], xf[1::2]  # xf(2i-1), xf(2i)
    yo, ye = yf[0::2], yf[1::2]
    zo, ze = zf[0::2], zf[1::2]
    X1, X2 = (xe - xc)[None, None, :], (xc - xo)[None, None, :]
    Y1, Y2 = (ye - yc)[None, :, None], (yc - yo)[None, :, None]
    Z1, Z2 = (ze - zc)[:, None, None], (zc - zo)[:, None, None]
    V = ((xe - xo)[None, None, :] * (ye - yo)[None, :, None]) * (ze - zo)[:, None, None]
    q = lambda a, b, c: qf[c::2, b::2, a::2]  # qf(2i-1+a, 2j-1+b, 2k-1+c)  # noqa: E731
    s = (X1 * Y1) * Z1 * q(0, 0, 0)
    s = s + (X2 * Y1) * Z1 * q(1, 0, 0)
    s = s + (X1 * Y2) * Z1 * q(0, 1, 0)
    s = s + (X2 * Y2) * Z1 * q(1, 1, 0)
    s = s + (X1 * Y1) * Z2 * q(0, 0, 1)
    s = s + (X2 * Y1) * Z2 * q(1, 0, 1)
    s = s + (X1 * Y2) * Z2 * q(0, 1, 1)
    s = s + (X2 * Y2) * Z2 * q(1, 1, 1)
    return s / V


def prolongation(mf: Mesh, mc: Mesh, pc: FField) -> np.ndarray:
    """prolongationOp3D (interpolation.f90:129-181): trilinear interpolation of
    the coarse field (ghosts included) to the fine centroids; fine cell i lies
    between coarse centroids ih = i/2 (integer division) and ih+1."""
    nxf, nyf, nzf = mf.nx, mf.ny, mf.nz
    xf, yf, zf = mf.xc.r(1, nxf), mf.yc.r(1, nyf), mf.zc.r(1, nzf)
    ih = np.arange(1, nxf + 1) // 2
    jh = np.arange(1, nyf + 1) // 2
    kh = np.arange(1, nzf + 1) // 2
    xc0, xc1 = mc.xc.v[ih - mc.xc.lb], mc.xc.v[ih + 1 - mc.xc.lb]
    yc0, yc1 = mc.yc.v[jh - mc.yc.lb], mc.yc.v[jh + 1 - mc.yc.lb]
    zc0, zc1 = mc.zc.v[kh - mc.zc.lb], mc.zc.v[kh + 1 - mc.zc.lb]
    X1, X2 = (xc1 - xf)[None, None, :], (xf - xc0)[None, None, :]
    Y1, Y2 = (yc1 - yf)[None, :, None], (yf - yc0)[None, :, None]
    Z1, Z2 = (zc1 - zf)[:, None, None], (zf - zc0)[:, None, None]
    V = ((xc1 - xc0)[None, None, :] * (yc1 - yc0)[None, :, None]) * (zc1 - zc0)[:, None, None]
    lb = pc.lb
    Q = lambda a, b, c: pc.a[(kh + c - lb[2])[:, None, None], (jh + b - lb[1])[None, :, None],  # noqa: E731
                             (ih + a - lb[0])[None, None, :]]
    s = (X1 * Y1) * Z1 * Q(0, 0, 0)
    s = s + (X2 * Y1) * Z1 * Q(1, 0, 0)
    s = s + (X1 * Y2) * Z1 * Q(0, 1, 0)
    s = s + (X2 * Y2) * Z1 * Q(1, 1, 0)
    s = s + (X1 * Y1) * Z2 * Q(0, 0, 1)
    s = s + (X2 * Y1) * Z2 * Q(1, 0, 1)
    s = s + (X1 * Y2) * Z2 * Q(0, 1, 1)
    s = s + (X2 * Y2) * Z2 * Q(1, 1, 1)
    return s / V


def coarse_direct_solve(lev: Level, p: FField, beta: FField, s: np.ndarray) -> None:
    """solveMat (poissMat.f90:289-312): the coarsest-level system assembled as
    V*(-L_beta) with true Neumann walls (computeInternalMatrixValues :714-772 and
    the boundary values :802-971), right-hand side -V*s (computeRHS :1081-1118;
    the homogeneous error boundary conditions add nothing), bordered by the
    Lagrange-multiplier row sum(p) = 0 (:467-503, :776-798) and solved directly
    (the reference factorises with MUMPS on every call)."""
    m = lev.m
    nx, ny, nz = m.nx, m.ny, m.nz
    n = nx * ny * nz
    idx = lambda i, j, k: ((k % nz) * ny + j) * nx + (i % nx)  # noqa: E731
    aR, aL, aT, aBo, aF, aBa = lev.coeffs(beta)
    V = m.volume()
    A = np.zeros((n + 1, n + 1))
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                r = idx(i, j, k)
                v = V[k, j, i]
                terms = [(aR[k, j, i], idx(i + 1, j, k)), (aL[k, j, i], idx(i - 1, j, k)),
                         (aF[k, j, i], idx(i, j, k + 1)), (aBa[k, j, i], idx(i, j, k - 1))]
                if j < ny - 1:
                    terms.append((aT[k, j, i], idx(i, j + 1, k)))
                if j > 0:
                    terms.append((aBo[k, j, i], idx(i, j - 1, k)))
                for a, c in terms:
                    A[r, c] -= v * a
                    A[r, r] += v * a
                A[r, n] = 1.0
                A[n, r] = 1.0
    b = np.zeros(n + 1)
    b[:n] = (-V * s).reshape(-1)
    x = np.linalg.solve(A, b)
    p.v(1, nx, 1, ny, 1, nz)[...] = x[:n].reshape(nz, ny, nx)
    update_boundaries_cl_channel(p)


class MGOracle:
    """multiGrid + rbgs + poissMat + pcg restated (multiGrid.f90, rbgs.f90,
    poissMat.f90, pcg.f90) for one rank, all in FP64."""

    def __init__(self, mesh: Mesh, n_levels: int = 6, n_pre: int = 2, n_post: int = 2, tol_mg: float = 0.4,
                 max_iter_mg: int = 100, tol_pcg: float = 1e-10, max_iter_pcg: int = 100):
        for l in range(1, n_levels):  # checkLevelsNumber (multiGrid.f90:116-145)
            for n in (mesh.nx, mesh.ny, mesh.nz):
                if n % (2 ** l):
                    raise ValueError("grid not divisible for the requested multigrid levels")
        self.n_levels, self.n_pre, self.n_post = n_levels, n_pre, n_post
        self.tol_mg, self.max_iter_mg = tol_mg, max_iter_mg
        self.tol_pcg, self.max_iter_pcg = tol_pcg, max_iter_pcg
        meshes = [mesh]
        for _ in range(n_levels - 1):
            meshes.append(coarse_mesh(meshes[-1]))
        self.levels = [Level(m) for m in meshes]  # index 0 = finest (level nLevels)
        self.mg_iters = []

    def _field(self, li):
        m = self.levels[li].m
        return FField("cl", 1, m.nx, m.ny, m.nz)

    def restrict_beta(self, beta: FField):
        """restrictField(beta) on every level (field.f90:1442-1470) with boundary updates."""
        betas = [beta]
        for li in range(1, self.n_levels):
            mf, mc = self.levels[li - 1].m, self.levels[li].m
            bc = self._field(li)
            bc.v(1, mc.nx, 1, mc.ny, 1, mc.nz)[...] = restriction(mf, mc, betas[-1].interior())
            update_boundaries_cl_channel(bc)
            betas.append(bc)
        return betas

    def vcycle(self, li: int, p: FField, betas, s_full: FField, coeffs) -> None:
        """mgVcycle (multiGrid.f90:186-232); li = 0 is the finest level."""
        lev = self.levels[li]
        if li == self.n_levels - 1:
            coarse_direct_solve(lev, p, betas[li], s_full.interior())
            return
        rbgs_iterate(lev, p, betas[li], s_full.interior(), self.n_pre, reset=(li != 0), coeffs=coeffs[li])
        resV, _ = compute_residuals(lev, p, betas[li], s_full, coeffs[li])
        mc = self.levels[li + 1].m
        sc = self._field(li + 1)
        sc.v(1, mc.nx, 1, mc.ny, 1, mc.nz)[...] = restriction(lev.m, mc, resV)
        update_boundaries_cl_channel(sc)
        pc = self._field(li + 1)
        self.vcycle(li + 1, pc, betas, sc, coeffs)
        m = lev.m
        p.v(1, m.nx, 1, m.ny, 1, m.nz)[...] += prolongation(m, mc, pc)
        update_boundaries_cl_channel(p)
        rbgs_iterate(lev, p, betas[li], s_full.interior(), self.n_post, reset=False, coeffs=coeffs[li])

    def solve_mg(self, p: FField, betas, s_full: FField, coeffs) -> int:
        """solveMG (multiGrid.f90:165-182) with continueIterating (:237-279)."""
        lev = self.levels[0]
        _, res = compute_residuals(lev, p, betas[0], s_full, coeffs[0])
        it = 0
        while True:
            if it == self.max_iter_mg:
                break
            if not res > self.tol_mg:
                break
            it += 1
            self.vcycle(0, p, betas, s_full, coeffs)
            _, res = compute_residuals(lev, p, betas[0], s_full, coeffs[0])
        return it

    def solve_pcg(self, psi: FField, beta: FField, q: np.ndarray):
        """solvePCG (pcg.f90:103-140): psi is the initial guess and the result
        (ghosts updated); returns (iterations, ||r||/||q||)."""
        lev = self.levels[0]
        m = lev.m
        nx, ny, nz = m.nx, m.ny, m.nz
        betas = self.restrict_beta(beta)
        coeffs = [lv.coeffs(b) for lv, b in zip(self.levels, betas)]
        qf = FField("cl", 1, nx, ny, nz)
        qf.v(1, nx, 1, ny, 1, nz)[...] = q
        resV, _ = compute_residuals(lev, psi, beta, qf, coeffs[0])
        r = FField("cl", 1, nx, ny, nz)
        r.v(1, nx, 1, ny, 1, nz)[...] = resV
        d = FField("cl", 1, nx, ny, nz)
        self.mg_iters.append(self.solve_mg(d, betas, r, coeffs))
        deltaN = float(np.sum(r.interior() * d.interior()))
        qn = math.sqrt(float(np.sum(q * q)) + TINY64)
        it = 0
        res = math.sqrt(float(np.sum(r.interior() ** 2))) / qn
        while True:
            if it == self.max_iter_pcg:
                break
            res = math.sqrt(float(np.sum(r.interior() ** 2))) / qn
            if not res > self.tol_pcg:
                break
            it += 1
            qv = apply_L(lev, d, beta, coeffs[0])
            alpha = deltaN / float(np.sum(d.interior() * qv))
            psi.a += alpha * d.a
            r.v(1, nx, 1, ny, 1, nz)[...] -= alpha * qv
            d0 = d.interior().copy()
            d.a[...] = 0.0
            self.mg_iters.append(self.solve_mg(d, betas, r, coeffs))
            delta0 = deltaN
            deltaN = float(np.sum(r.interior() * d.interior()))
            gamma = deltaN / delta0
            d0 = d.interior() + gamma * d0
            d.v(1, nx, 1, ny, 1, nz)[...] = d0
            update_boundaries_cl_channel(d)
        update_boundaries_cl_channel(psi)
        return it, res


def compute_source_mg(mesh: Mesh, ux: FField, uy: FField, uz: FField) -> np.ndarray:
    """computeSource MG (poissonEqn.f90:155-190): s = div u* with per-index metrics."""
    return divergence(mesh, ux, uy, uz)


def compute_beta(mesh: Mesh, rho: FField, dt: float, alpha: float) -> FField:
    """computeBeta (poissonEqn.f90:311-342): beta = dt*alpha/rho, then its boundary update."""
    b = FField("cl", 1, mesh.nx, mesh.ny, mesh.nz)
    b.v(1, mesh.nx, 1, mesh.ny, 1, mesh.nz)[...] = (dt * alpha) / rho.interior()
    update_boundaries_cl_channel(b)
    return b


def add_pressure_grad(mesh: Mesh, ux: FField, uy: FField, uz: FField, p: FField, rho: FField,
                      dt: float, alpha: float) -> None:
    """makeVelocityDivFree MG = addPressureGrad (momentumEqn.f90:795-869, :980-993),
    loop ranges of setEqnBounds, then the periodic equate."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz

    def upd(u, i0, i1, j0, j1, k0, k1, di, dj, dk, dc):
        S = lambda f, o=0: f.v(i0 + di * o, i1 + di * o, j0 + dj * o, j1 + dj * o, k0 + dk * o, k1 + dk * o)  # noqa: E731
        invrho = 0.5 * (1.0 / S(rho, 1) + 1.0 / S(rho))
        tgt = u.v(i0, i1, j0, j1, k0, k1)
        tgt -= dt * alpha * invrho * (S(p, 1) - S(p)) / dc

    upd(ux, 0, nx, 1, ny, 1, nz, 1, 0, 0, mesh.dxc.r(1, nx + 1)[None, None, :])
    upd(uy, 1, nx, 1, ny - 1, 1, nz, 0, 1, 0, mesh.dyc.r(2, ny)[None, :, None])
    upd(uz, 1, nx, 1, ny, 0, nz, 0, 0, 1, mesh.dzc.r(1, nz + 1)[:, None, None])
    equate_periodic_bc(ux, uz)


# ---------------------------------------------------------------------------
# Material properties: updateMaterialProps (VOF.f90:197-233) with smoothVF
# (VOF.f90:235-262), cellToVertex / vertexToCell (interpolation.f90:188-276)
# ---------------------------------------------------------------------------
def cell_to_vertex(mesh: Mesh, q: FField) -> np.ndarray:
    """cellToVertex (interpolation.f90:188-229) onto the vertex array s_cv(0:nx, 0:ny, 0:nz)
    (VOF.f90:156): the trilinear value at vertex (i, j, k) from cells i..i+1,
    j..j+1, k..k+1, weights w1..w8 and volume V as written there, summed in
    the same order.  Returns shape (nz+1, ny+1, nx+1)."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    x, y, z = mesh.xc.r(0, nx + 1), mesh.yc.r(0, ny + 1), mesh.zc.r(0, nz + 1)
    xv, yv, zv = mesh.xf.r(0, nx), mesh.yf.r(0, ny), mesh.zf.r(0, nz)
    X1, X2 = (x[1:] - xv)[None, None, :], (xv - x[:-1])[None, None, :]   # x(i+1)-xv(i), xv(i)-x(i)
    Y1, Y2 = (yv - y[:-1])[None, :, None], (y[1:] - yv)[None, :, None]   # yv(j)-y(j), y(j+1)-yv(j)
    Z1, Z2 = (z[1:] - zv)[:, None, None], (zv - z[:-1])[:, None, None]   # z(k+1)-zv(k), zv(k)-z(k)
    V = ((x[1:] - x[:-1])[None, None, :] * (y[1:] - y[:-1])[None, :, None]) * (z[1:] - z[:-1])[:, None, None]
    Q = lambda di, dj, dk: q.v(di, nx + di, dj, ny + dj, dk, nz + dk)  # noqa: E731  q(i+di, j+dj, k+dk)
    s = (X1 * Y1) * Z1 * Q(0, 1, 0)
    s = s + (X2 * Y1) * Z1 * Q(1, 1, 0)
    s = s + (X1 * Y1) * Z2 * Q(0, 1, 1)
    s = s + (X2 * Y1) * Z2 * Q(1, 1, 1)
    s = s + (X1 * Y2) * Z1 * Q(0, 0, 0)
    s = s + (X2 * Y2) * Z1 * Q(1, 0, 0)
    s = s + (X1 * Y2) * Z2 * Q(0, 0, 1)
    s = s + (X2 * Y2) * Z2 * Q(1, 0, 1)
    return s / V


def vertex_to_cell(mesh: Mesh, qv: np.ndarray, q: FField) -> None:
    """vertexToCell (interpolation.f90:234-276): the interior cells of q from
    their 8 vertices (qv as returned by cell_to_vertex)."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    x, y, z = mesh.xc.r(1, nx), mesh.yc.r(1, ny), mesh.zc.r(1, nz)
    xv, yv, zv = mesh.xf.r(0, nx), mesh.yf.r(0, ny), mesh.zf.r(0, nz)
    X1, X2 = (xv[1:] - x)[None, None, :], (x - xv[:-1])[None, None, :]   # xv(i)-x(i), x(i)-xv(i-1)
    Y1, Y2 = (y - yv[:-1])[None, :, None], (yv[1:] - y)[None, :, None]   # y(j)-yv(j-1), yv(j)-y(j)
    Z1, Z2 = (zv[1:] - z)[:, None, None], (z - zv[:-1])[:, None, None]   # zv(k)-z(k), z(k)-zv(k-1)
    V = ((xv[1:] - xv[:-1])[None, None, :] * (yv[1:] - yv[:-1])[None, :, None]) * (zv[1:] - zv[:-1])[:, None, None]
    P = lambda di, dj, dk: qv[dk:dk + nz, dj:dj + ny, di:di + nx]  # noqa: E731  qv(i-1+di, j-1+dj, k-1+dk)
    s = (X1 * Y1) * Z1 * P(0, 1, 0)
    s = s + (X2 * Y1) * Z1 * P(1, 1, 0)
    s = s + (X1 * Y1) * Z2 * P(0, 1, 1)
    s = s + (X2 * Y1) * Z2 * P(1, 1, 1)
    s = s + (X1 * Y2) * Z1 * P(0, 0, 0)
    s = s + (X2 * Y2) * Z1 * P(1, 0, 0)
    s = s + (X1 * Y2) * Z2 * P(0, 0, 1)
    s = s + (X2 * Y2) * Z2 * P(1, 0, 1)
    q.interior()[...] = s / V


def smooth_vf(mesh: Mesh, c: FField) -> FField:
    """smoothVF (VOF.f90:235-262), smooth_level = 1: cell -> vertex -> cell from c,
    boundary update, once more from cs, boundary update.  c's ghosts must be
    current; cs has c's halo."""
    cs = FField("cl", c.hd, c.nx, c.ny, c.nz)
    vertex_to_cell(mesh, cell_to_vertex(mesh, c), cs)
    update_boundaries_cl_channel(cs)
    vertex_to_cell(mesh, cell_to_vertex(mesh, cs), cs)
    update_boundaries_cl_channel(cs)
    return cs


def update_material_props(mesh: Mesh, c: FField, rhol: float, rhog: float, mul: float, mug: float):
    """updateMaterialProps (VOF.f90:197-233): cs = smoothVF(c), then over the
    whole arrays (halos included) mu = mug*cs + (1-cs)*mul, rho = rhog*cs + (1-cs)*rhol.
    Returns (cs, rho, mu)."""
    cs = smooth_vf(mesh, c)
    rho = FField("cl", c.hd, c.nx, c.ny, c.nz, rhog * cs.a + (1.0 - cs.a) * rhol)
    mu = FField("cl", c.hd, c.nx, c.ny, c.nz, mug * cs.a + (1.0 - cs.a) * mul)
    return cs, rho, mu


# ---------------------------------------------------------------------------
# Momentum predictor: solveMomentumEqn FAST (momentumEqn.f90:161-194) without
# its closing updateBoundariesV: copyOldFluxes / resetFluxes, updateConveDiff
# (:198-607), addConvDiff (:738-791), addSource (:874-973)
# ---------------------------------------------------------------------------
def approx_zero(d: np.ndarray) -> np.ndarray:
    """approx_zero (auxiliaryRoutines.f90:553-565)."""
    return np.where(d == 0.0, 1e-50, d)


def compute_limiters(vc, vm, vp, vpp, vmm, cxp, cxm, cyp, cym, czp, czm, scheme: int):
    """compute_limiters (momentumEqn.f90:611-663) with the limiters of :667-734:
    0 central, 1 upwind, 2 QUICK, 3 van Leer, 4 superbee, 5 superbee where the
    volume fraction varies (dc > epsilon in any direction), central elsewhere."""
    if scheme == 0:
        one = np.ones_like(vc)
        return one, one, one, one
    if scheme == 1:
        z = np.zeros_like(vc)
        return z, z, z, z
    rs = [(vc - vm) / approx_zero(vp - vc), (vpp - vp) / approx_zero(vp - vc),
          (vm - vmm) / approx_zero(vc - vm), (vp - vc) / approx_zero(vc - vm)]

    def quick(r):
        return (r + 3.0) / 4.0

    def vanleer(r):
        r = np.maximum(0.0, r)
        return (r + np.abs(r)) / (1.0 + np.abs(r))

    def superbee(r):
        r = np.maximum(0.0, r)
        return np.maximum(np.maximum(0.0, np.minimum(2.0 * r, 1.0)), np.minimum(r, 2.0))

    if scheme == 2:
        return tuple(quick(r) for r in rs)
    if scheme == 3:
        return tuple(vanleer(r) for r in rs)
    if scheme == 4:
        return tuple(superbee(r) for r in rs)
    if scheme == 5:
        small = EPS64
        sharp = ((cxp - cxm) > small) | ((cyp - cym) > small) | ((czp - czm) > small)
        return tuple(np.where(sharp, superbee(r), 1.0) for r in rs)
    raise ValueError(f"unknown convection scheme {scheme}")


def _flux(q, a, b, psi_up, psi_um):
    """F = max(q,0)*A + min(q,0)*B with A = a + psi_up/2 (b - a), B = b + psi_um/2 (a - b)."""
    A = a + 0.5 * psi_up * (b - a)
    B = b + 0.5 * psi_um * (a - b)
    return np.maximum(q, 0.0) * A + np.minimum(q, 0.0) * B


def momentum_fluxes(mesh: Mesh, ux: FField, uy: FField, uz: FField, c: FField, mu: FField, rho: FField,
                    scheme: int):
    """updateConveDiff (momentumEqn.f90:198-607): the convection + diffusion
    fluxes phiX, phiY, phiZ on the equation bounds of setEqnBounds (:1134-1190)
    for the channel: ux i=0..nx, uy j=1..ny-1 (fixed walls), uz k=0..nz.
    Returns dense (k, j, i) arrays."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    out = []
    for comp, (i0, i1, j0, j1, k0, k1) in enumerate([(0, nx, 1, ny, 1, nz), (1, nx, 1, ny - 1, 1, nz),
                                                     (1, nx, 1, ny, 0, nz)]):
        S = lambda f, di=0, dj=0, dk=0: f.v(i0 + di, i1 + di, j0 + dj, j1 + dj, k0 + dk, k1 + dk)  # noqa: E731
        X = lambda a, d=0: a.r(i0 + d, i1 + d)[None, None, :]  # noqa: E731
        Y = lambda a, d=0: a.r(j0 + d, j1 + d)[None, :, None]  # noqa: E731
        Z = lambda a, d=0: a.r(k0 + d, k1 + d)[:, None, None]  # noqa: E731
        if comp == 0:
            u = ux
            cl = (S(c, 1), S(c), S(c, 0, 1), S(c, 0, -1), S(c, 0, 0, 1), S(c, 0, 0, -1))
        elif comp == 1:
            u = uy
            cl = (S(c, 1), S(c, -1), S(c, 0, 1), S(c), S(c, 0, 0, 1), S(c, 0, 0, -1))
        else:
            u = uz
            cl = (S(c, 1), S(c, -1), S(c, 0, 1), S(c, 0, -1), S(c, 0, 0, 1), S(c))
        U = lambda di=0, dj=0, dk=0: S(u, di, dj, dk)  # noqa: E731

        def lim(d):
            e = [(1 if d == n else 0) for n in range(3)]
            p = lambda s: U(*[s * x for x in e])  # noqa: E731
            return compute_limiters(U(), p(-1), p(1), p(2), p(-2), *cl, scheme)

        phi = np.zeros_like(U())
        # --- convection
        if comp == 0:
            l = lim(0)
            qp, qm = 0.5 * (U() + U(1)), 0.5 * (U() + U(-1))
            phi = phi - (_flux(qp, U(), U(1), l[0], l[1]) - _flux(qm, U(-1), U(), l[2], l[3])) / X(mesh.dxc, 1)
            l = lim(1)
            qp, qm = 0.5 * (S(uy, 1) + S(uy)), 0.5 * (S(uy, 1, -1) + S(uy, 0, -1))
            phi = phi - (_flux(qp, U(), U(0, 1), l[0], l[1]) - _flux(qm, U(0, -1), U(), l[2], l[3])) / Y(mesh.dyf)
            l = lim(2)
            qp, qm = 0.5 * (S(uz) + S(uz, 1)), 0.5 * (S(uz, 0, 0, -1) + S(uz, 1, 0, -1))
            phi = phi - (_flux(qp, U(), U(0, 0, 1), l[0], l[1]) - _flux(qm, U(0, 0, -1), U(), l[2], l[3])) / Z(mesh.dzf)
        elif comp == 1:
            l = lim(0)
            qp = 0.5 * (S(ux, 0, 1) * Y(mesh.dyf, 1) + S(ux) * Y(mesh.dyf)) / Y(mesh.dyc, 1)
            qm = 0.5 * (S(ux, -1, 1) * Y(mesh.dyf, 1) + S(ux, -1) * Y(mesh.dyf)) / Y(mesh.dyc, 1)
            phi = phi - (_flux(qp, U(), U(1), l[0], l[1]) - _flux(qm, U(-1), U(), l[2], l[3])) / X(mesh.dxf)
            l = lim(1)
            qp, qm = 0.5 * (U() + U(0, 1)), 0.5 * (U() + U(0, -1))
            phi = phi - (_flux(qp, U(), U(0, 1), l[0], l[1]) - _flux(qm, U(0, -1), U(), l[2], l[3])) / Y(mesh.dyc, 1)
            l = lim(2)
            qp = 0.5 * (S(uz, 0, 1) * Y(mesh.dyf, 1) + S(uz) * Y(mesh.dyf)) / Y(mesh.dyc, 1)
            qm = 0.5 * (S(uz, 0, 1, -1) * Y(mesh.dyf, 1) + S(uz, 0, 0, -1) * Y(mesh.dyf)) / Y(mesh.dyc, 1)
            phi = phi - (_flux(qp, U(), U(0, 0, 1), l[0], l[1]) - _flux(qm, U(0, 0, -1), U(), l[2], l[3])) / Z(mesh.dzf)
        else:
            l = lim(0)
            qp, qm = 0.5 * (S(ux) + S(ux, 0, 0, 1)), 0.5 * (S(ux, -1) + S(ux, -1, 0, 1))
            phi = phi - (_flux(qp, U(), U(1), l[0], l[1]) - _flux(qm, U(-1), U(), l[2], l[3])) / X(mesh.dxf)
            l = lim(1)
            qp, qm = 0.5 * (S(uy) + S(uy, 0, 0, 1)), 0.5 * (S(uy, 0, -1) + S(uy, 0, -1, 1))
            phi = phi - (_flux(qp, U(), U(0, 1), l[0], l[1]) - _flux(qm, U(0, -1), U(), l[2], l[3])) / Y(mesh.dyf)
            l = lim(2)
            qp, qm = 0.5 * (U() + U(0, 0, 1)), 0.5 * (U() + U(0, 0, -1))
            phi = phi - (_flux(qp, U(), U(0, 0, 1), l[0], l[1]) - _flux(qm, U(0, 0, -1), U(), l[2], l[3])) / Z(mesh.dzc, 1)
        # --- diffusion
        M = lambda di=0, dj=0, dk=0: S(mu, di, dj, dk)  # noqa: E731
        if comp == 0:
            mur, mul = M(1), M()
            dxx = (mur * (U(1) - U()) / X(mesh.dxf, 1) - mul * (U() - U(-1)) / X(mesh.dxf)) / X(mesh.dxc, 1)
            dxxt = dxx
            mur = 0.25 * (M(1) + M() + M(1, 1) + M(0, 1))
            mul = 0.25 * (M(1) + M() + M(1, -1) + M(0, -1))
            dyy = (mur * (U(0, 1) - U()) / Y(mesh.dyc, 1) - mul * (U() - U(0, -1)) / Y(mesh.dyc)) / Y(mesh.dyf)
            dyyt = (mur * (S(uy, 1) - S(uy)) / X(mesh.dxc, 1) - mul * (S(uy, 1, -1) - S(uy, 0, -1)) / X(mesh.dxc, 1)) / Y(mesh.dyf)
            mur = 0.25 * (M(1) + M() + M(1, 0, 1) + M(0, 0, 1))
            mul = 0.25 * (M(1) + M() + M(1, 0, -1) + M(0, 0, -1))
            dzz = (mur * (U(0, 0, 1) - U()) / Z(mesh.dzc, 1) - mul * (U() - U(0, 0, -1)) / Z(mesh.dzc)) / Z(mesh.dzf)
            dzzt = (mur * (S(uz, 1) - S(uz)) / X(mesh.dxc, 1) - mul * (S(uz, 1, 0, -1) - S(uz, 0, 0, -1)) / X(mesh.dxc, 1)) / Z(mesh.dzf)
            invrho = 0.5 * (1.0 / S(rho, 1) + 1.0 / S(rho))
        elif comp == 1:
            mur = 0.25 * (M() + M(1) + M(0, 1) + M(1, 1))
            mul = 0.25 * (M() + M(-1) + M(0, 1) + M(-1, 1))
            dxx = (mur * (U(1) - U()) / X(mesh.dxc, 1) - mul * (U() - U(-1)) / X(mesh.dxc)) / X(mesh.dxf)
            dxxt = (mur * (S(ux, 0, 1) - S(ux)) / Y(mesh.dyc, 1) - mul * (S(ux, -1, 1) - S(ux, -1)) / Y(mesh.dyc, 1)) / X(mesh.dxf)
            mur, mul = M(0, 1), M()
            dyy = (mur * (U(0, 1) - U()) / Y(mesh.dyf, 1) - mul * (U() - U(0, -1)) / Y(mesh.dyf)) / Y(mesh.dyc, 1)
            dyyt = dyy
            mur = 0.25 * (M() + M(0, 0, 1) + M(0, 1) + M(0, 1, 1))
            mul = 0.25 * (M() + M(0, 0, -1) + M(0, 1) + M(0, 1, -1))
            dzz = (mur * (U(0, 0, 1) - U()) / Z(mesh.dzc, 1) - mul * (U() - U(0, 0, -1)) / Z(mesh.dzc)) / Z(mesh.dzf)
            dzzt = (mur * (S(uz, 0, 1) - S(uz)) / Y(mesh.dyc, 1) - mul * (S(uz, 0, 1, -1) - S(uz, 0, 0, -1)) / Y(mesh.dyc, 1)) / Z(mesh.dzf)
            invrho = 0.5 * (1.0 / S(rho, 0, 1) + 1.0 / S(rho))
        else:
            mur = 0.25 * (M() + M(0, 0, 1) + M(1) + M(1, 0, 1))
            mul = 0.25 * (M() + M(0, 0, 1) + M(-1) + M(-1, 0, 1))
            dxx = (mur * (U(1) - U()) / X(mesh.dxc, 1) - mul * (U() - U(-1)) / X(mesh.dxc)) / X(mesh.dxf)
            dxxt = (mur * (S(ux, 0, 0, 1) - S(ux)) / Z(mesh.dzc, 1) - mul * (S(ux, -1, 0, 1) - S(ux, -1)) / Z(mesh.dzc, 1)) / X(mesh.dxf)
            mur = 0.25 * (M() + M(0, 0, 1) + M(0, 1) + M(0, 1, 1))
            mul = 0.25 * (M() + M(0, 0, 1) + M(0, -1) + M(0, -1, 1))
            dyy = (mur * (U(0, 1) - U()) / Y(mesh.dyc, 1) - mul * (U() - U(0, -1)) / Y(mesh.dyc)) / Y(mesh.dyf)
            dyyt = (mur * (S(uy, 0, 0, 1) - S(uy)) / Z(mesh.dzc, 1) - mul * (S(uy, 0, -1, 1) - S(uy, 0, -1)) / Z(mesh.dzc, 1)) / Y(mesh.dyf)
            mur, mul = M(0, 0, 1), M()
            dzz = (mur * (U(0, 0, 1) - U()) / Z(mesh.dzf, 1) - mul * (U() - U(0, 0, -1)) / Z(mesh.dzf)) / Z(mesh.dzc, 1)
            dzzt = dzz
            invrho = 0.5 * (1.0 / S(rho, 0, 0, 1) + 1.0 / S(rho))
        phi = phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho
        out.append(phi)
    return tuple(out)


def momentum_predictor(mesh: Mesh, ux: FField, uy: FField, uz: FField, c: FField, mu: FField, rho: FField,
                       phi_prev, dt: float, alpha: float, gamma: float, xi: float, rho0: float,
                       gch: float = 0.0, g: float = 0.0, fs: float = 0.0, st=None, scheme: int = 2):
    """solveMomentumEqn FAST (momentumEqn.f90:161-194) without the closing
    updateBoundariesV: the new fluxes from u, then u += dt*(gamma*phi + xi*phi_prev)
    (addConvDiff :738-791) and the sources of addSource (:874-973):
    ux += r/rho0 st_x + invrho_x r fs + r gCH, uy += r/rho0 st_y + r g,
    uz += r/rho0 st_z, r = dt*alpha.  Updates u in place; returns the new fluxes
    (the next call's phi_prev)."""
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    phi = momentum_fluxes(mesh, ux, uy, uz, c, mu, rho, scheme)
    boxes = [(0, nx, 1, ny, 1, nz), (1, nx, 1, ny - 1, 1, nz), (1, nx, 1, ny, 0, nz)]
    r = dt * alpha
    invrho0 = 1.0 / rho0
    for d, (u, (i0, i1, j0, j1, k0, k1)) in enumerate(zip((ux, uy, uz), boxes)):
        t = u.v(i0, i1, j0, j1, k0, k1)
        t[...] = t + dt * (gamma * phi[d] + xi * phi_prev[d])
    for d, (u, (i0, i1, j0, j1, k0, k1)) in enumerate(zip((ux, uy, uz), boxes)):
        t = u.v(i0, i1, j0, j1, k0, k1)
        s = st[d].v(i0, i1, j0, j1, k0, k1) if st is not None else 0.0
        if d == 0:
            invrho = 0.5 * (1.0 / rho.v(i0 + 1, i1 + 1, j0, j1, k0, k1) + 1.0 / rho.v(i0, i1, j0, j1, k0, k1))
            t[...] = t + invrho0 * r * s + invrho * r * fs + r * gch
        elif d == 1:
            t[...] = t + invrho0 * r * s + r * g
        else:
            t[...] = t + invrho0 * r * s
    return phi


# ---------------------------------------------------------------------------
# Surface tension: height-function curvature and the face force
# (computeSurfaceTension / computeBlockST, VOF.f90:1872-2002; curvature
# computeBlockCurvature / hfColumn, VOF.f90:2070-2290, Popinet 2009).
#
# A grid-wide restatement.  The reference works on per-bubble blocks whose
# bounds stop the height columns and falls back to a parabolic fit through
# interface centroids when no direction gives nine valid columns; here the
# columns walk at most L cells each way over the whole grid, and a cell with no
# valid direction gets curvature 0.  The interface cells, the face force and the
# averaging of the curvature onto the faces follow the reference:
#   mixed: eps <= c <= 1-eps; full: c >= 1-eps (VOF.f90:1094-1108);
#   a full cell with an empty 6-neighbour becomes mixed with c = 1-2 eps
#   (search_full_interface_cells, :672-726);
#   st_d = sigma * k_f * (c(Q) - c(P)) / dc on the face between P and Q, k_f the
#   mean of the two cells' curvatures if both are mixed, else the mixed one's,
#   else 0 (computeBlockST, :1904-1996).
# Arrays are dense interior arrays [k, j, i] (0-based); dyf[0..ny-1] = dyf(1..ny),
# dyc[0..ny] = dyc(1..ny+1) as in the library descriptor.
# ---------------------------------------------------------------------------
ST_EPS = 1e-12
ST_COLUMN = 6  # cells a height column may walk from its start cell, each way


def st_classify(c: np.ndarray, eps: float = ST_EPS):
    """(c', mixed, full) after the promotion of full interface cells."""
    mixed0 = (c >= 0.0 + eps) & (c <= 1.0 - eps)
    full0 = c >= 1.0 - eps
    empty0 = ~full0 & ~mixed0
    nb_empty = np.zeros_like(full0)
    for ax in (0, 2):  # z and x periodic
        nb_empty |= np.roll(empty0, 1, axis=ax) | np.roll(empty0, -1, axis=ax)
    # y: the ghost rows copy the wall cells, so a wall cell's outer neighbour is itself
    up = np.concatenate([empty0[:, 1:, :], empty0[:, -1:, :]], axis=1)
    dn = np.concatenate([empty0[:, :1, :], empty0[:, :-1, :]], axis=1)
    nb_empty |= up | dn
    promote = full0 & nb_empty
    cp = np.where(promote, 1.0 - 2.0 * eps, c)
    return cp, mixed0 | promote, full0 & ~promote


def st_curvature(cp, mixed, full, dx, dz, dyf, dyc, L: int = ST_COLUMN):
    """Height-function curvature at the mixed cells (0 elsewhere).  Positive for a
    bubble (c = 1 inside): 2/R on a sphere of radius R."""
    nz, ny, nx = cp.shape
    n_ = (nx, ny, nz)
    empty = ~mixed & ~full
    yf0 = np.zeros(ny + 1)  # face positions, sequential sums of dyf
    acc = 0.0
    for m in range(ny):
        acc = acc + dyf[m]
        yf0[m + 1] = acc
    w = (1.0, 2.0, 1.0)

    def cell(ijk):  # wrap x, z; None outside the walls in y
        i, j, k = ijk
        if j < 0 or j >= ny:
            return None
        return (k % nz, j, i % nx)

    def cyc(j):  # clamped y index
        return min(max(j, 0), ny - 1)

    def ydist(jm, jp):
        s = 0.0
        for J in range(jm + 1, jp + 1):
            s = s + dyc[J]
        return s

    def face_pos(d, q):  # position of face q (0-based: lower face of cell q) along d
        if d == 0:
            return q * dx
        if d == 2:
            return q * dz
        return yf0[q]

    def width(d, q):
        return dx if d == 0 else (dz if d == 2 else dyf[q])

    kap = np.zeros_like(cp)
    ks, js, is_ = np.nonzero(mixed)
    for k, j, i in zip(ks, js, is_):
        # normal: central differences smoothed over the transverse 3x3 (weights 1,2,1)
        nx_ = 0.0
        ny_ = 0.0
        nz_ = 0.0
        for b in range(3):
            for e in range(3):
                jj = cyc(j + b - 1)
                nx_ = nx_ + w[b] * w[e] * (cp[(k + e - 1) % nz, jj, (i + 1) % nx] - cp[(k + e - 1) % nz, jj, (i - 1) % nx])
        jm, jp = cyc(j - 1), cyc(j + 1)
        for a in range(3):
            for e in range(3):
                ny_ = ny_ + w[a] * w[e] * (cp[(k + e - 1) % nz, jp, (i + a - 1) % nx] - cp[(k + e - 1) % nz, jm, (i + a - 1) % nx])
        for a in range(3):
            for b in range(3):
                jj = cyc(j + b - 1)
                nz_ = nz_ + w[a] * w[b] * (cp[(k + 1) % nz, jj, (i + a - 1) % nx] - cp[(k - 1) % nz, jj, (i + a - 1) % nx])
        nvec = [nx_ / (2.0 * dx), (ny_ / ydist(jm, jp)) if jp > jm else 0.0, nz_ / (2.0 * dz)]
        order = []
        mag = [abs(v) for v in nvec]
        for _ in range(3):  # maxloc: the first largest remaining
            best = -1
            for d in range(3):
                if d in order:
                    continue
                if best < 0 or mag[d] > mag[best]:
                    best = d
            order.append(best)
        P = (i, j, k)
        for d in order:
            s = 1 if nvec[d] >= 0.0 else -1
            t1, t2 = [x for x in (0, 1, 2) if x != d]
            F = np.zeros((3, 3))
            ok = True
            for a in (-1, 0, 1):
                for b in (-1, 0, 1):
                    st0 = list(P)
                    st0[t1] += a
                    st0[t2] += b
                    if cell(tuple(st0)) is None:
                        ok = False
                        break
                    q0 = st0[d]

                    def at(t):
                        x = list(st0)
                        x[d] = q0 + s * t
                        return cell(tuple(x))

                    tf = te = -1
                    for t in range(L + 1):
                        cc = at(t)
                        if cc is None:
                            break
                        if full[cc]:
                            tf = t
                            break
                    for t in range(L + 1):
                        cc = at(-t)
                        if cc is None:
                            break
                        if empty[cc]:
                            te = t
                            break
                    if tf < 0 or te < 0:
                        ok = False
                        break
                    hsum = 0.0
                    for t in range(-te, tf + 1):
                        cc = at(t)
                        qq = q0 + s * t
                        hsum = hsum + cp[cc] * width(d, qq % n_[d] if d != 1 else qq)
                    qf = q0 + s * tf
                    xf_ = face_pos(d, qf + 1) if s > 0 else face_pos(d, qf)
                    F[a + 1, b + 1] = xf_ - s * hsum
                if not ok:
                    break
            if not ok:
                continue

            def spacing(tdir, p):
                if tdir == 0:
                    return dx, dx
                if tdir == 2:
                    return dz, dz
                return dyc[p], dyc[p + 1]

            h1m, h1p = spacing(t1, P[t1])
            h2m, h2p = spacing(t2, P[t2])
            den1 = h1p * h1m * (h1p + h1m)
            den2 = h2p * h2m * (h2p + h2m)
            d1 = (h1m * h1m * F[2, 1] - h1p * h1p * F[0, 1] + (h1p * h1p - h1m * h1m) * F[1, 1]) / den1
            d11 = 2.0 * (h1m * F[2, 1] - (h1p + h1m) * F[1, 1] + h1p * F[0, 1]) / den1
            d2 = (h2m * h2m * F[1, 2] - h2p * h2p * F[1, 0] + (h2p * h2p - h2m * h2m) * F[1, 1]) / den2
            d22 = 2.0 * (h2m * F[1, 2] - (h2p + h2m) * F[1, 1] + h2p * F[1, 0]) / den2
            d12 = (F[2, 2] - F[2, 0] - F[0, 2] + F[0, 0]) / ((h1p + h1m) * (h2p + h2m))
            num = d11 * (1.0 + d2 * d2) + d22 * (1.0 + d1 * d1) - 2.0 * d1 * d2 * d12
            g = 1.0 + d1 * d1 + d2 * d2
            kap[k, j, i] = s * num / (g * np.sqrt(g))
            break
    return kap


def st_faces(cp, mixed, kap, sigma, dx, dz, dyc):
    """Face force of computeBlockST on every face: stx[k, j, f] for x faces
    f = 0..nx (face f between cells f-1 and f, periodic), sty[k, f, i] for
    f = 0..ny (zero on the walls), stz[f, j, i] for f = 0..nz."""
    nz, ny, nx = cp.shape

    def kf(kp, mp, kq, mq):
        return np.where(mp & mq, 0.5 * (kq + kp), np.where(mq, kq, np.where(mp, kp, 0.0)))

    def along(ax, n, dc):
        lo = [slice(None)] * 3
        idx_p = np.arange(-1, n) % n  # cell below face f
        idx_q = np.arange(0, n + 1) % n
        cp_p, cp_q = np.take(cp, idx_p, axis=ax), np.take(cp, idx_q, axis=ax)
        mp, mq = np.take(mixed, idx_p, axis=ax), np.take(mixed, idx_q, axis=ax)
        kp, kq = np.take(kap, idx_p, axis=ax), np.take(kap, idx_q, axis=ax)
        del lo
        return sigma * kf(kp, mp, kq, mq) * ((cp_q - cp_p) / dc)

    stx = along(2, nx, dx)
    stz = along(0, nz, dz)
    sty = np.zeros((nz, ny + 1, nx))
    for f in range(1, ny):
        mp, mq = mixed[:, f - 1, :], mixed[:, f, :]
        sty[:, f, :] = sigma * kf(kap[:, f - 1, :], mp, kap[:, f, :], mq) * ((cp[:, f, :] - cp[:, f - 1, :]) / dyc[f])
    return stx, sty, stz


def surface_tension(c, sigma, dx, dz, dyf, dyc, eps: float = ST_EPS, L: int = ST_COLUMN):
    """computeSurfaceTension restated grid-wide: (curvature, stx, sty, stz) from
    the interior volume fraction c[k, j, i]."""
    cp, mixed, full = st_classify(c, eps)
    kap = st_curvature(cp, mixed, full, dx, dz, np.asarray(dyf), np.asarray(dyc), L)
    return (kap,) + st_faces(cp, mixed, kap, sigma, dx, dz, np.asarray(dyc))
