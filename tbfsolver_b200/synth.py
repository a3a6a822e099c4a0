"""Seeded synthetic inputs for the projection step, built with the reference's
own initial-condition recipe (no dataset or checkpoint is available).

* Bubble volume fraction: ``init_Bubble_vf`` (src/initialConditions/initialConditions.f90:192-398):
  cells whose centre is inside get 1; cells with 1..7 of their 8 vertices
  inside are re-integrated on an nref^3 sub-grid.  Bubbles are spheres of
  radius R at seeded, non-overlapping positions (periodic in x and z).
* Smoothing: ``smoothVF`` (src/VOF/VOF.f90:235-262), two cell->vertex->cell
  trilinear passes (interpolation.f90:188-276) with the field's boundary update
  in between.
* Density: ``updateMaterialProps`` (VOF.f90:197-231): rho = rhog*cs + (1-cs)*rhol
  on the whole array including the halo.
* Velocity u*: laminar Poiseuille icA*y*(Ly-y) with unit bulk velocity (the form
  of initChFlowVelocity, initialConditions.f90:77) plus uniform noise in
  [-0.05, 0.05] on every interior face; uy = 0 on the wall faces; periodic
  duplicate faces equated (vfield.f90:124-189).

Noise comes from a counter-based generator (splitmix64 of seed, field id and
linear index), so the same inputs are produced on the CPU and on any GPU.
All arrays are torch tensors in the Fortran layout of ``fields.Field``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from .fields import Field, VField, field_shape
from .grid import Grid

TWO_PI = 2.0 * math.pi


@dataclass
class ChannelSpec:
    """One channel of the benchmark suite (box, grid, bubbles, densities)."""

    name: str
    nx: int
    ny: int
    nz: int
    Lx: float = TWO_PI
    Ly: float = 2.0
    Lz: float = math.pi
    y_stretched: bool = False
    gamma: float = 1.5
    nbubbles: int = 0
    radius: float = 0.1
    rhol: float = 1.0
    rhog: float = 0.1
    dt: float = 1e-4
    nref: int = 16

    @property
    def ncells(self) -> int:
        return self.nx * self.ny * self.nz

    def grid(self) -> Grid:
        return Grid(self.nx, self.ny, self.nz, self.Lx, self.Ly, self.Lz, self.y_stretched, self.gamma)


# The workloads named by the benchmark configurations.
CONFIGS = {
    "c1": ChannelSpec("c1-128x128x64-uniform", 128, 128, 64, nbubbles=18, radius=0.25, rhol=1.0, rhog=0.1),
    "c2": ChannelSpec("c2-512x384x256-tanh1.5", 512, 384, 256, y_stretched=True, gamma=1.5, nbubbles=200,
                      radius=0.1, rhol=1.0, rhog=0.02),
    "c3": ChannelSpec("c3-1024x512x512-tanh1.5", 1024, 512, 512, y_stretched=True, gamma=1.5, nbubbles=800,
                      radius=0.06, rhol=1.0, rhog=0.02),
    "c5": ChannelSpec("c5-256x256x128-tanh1.5", 256, 256, 128, y_stretched=True, gamma=1.5, nbubbles=60,
                      radius=0.15, rhol=1.0, rhog=0.01),
    # half of c2's planes: the same x and y transforms and y-solve instance
    # (384 rows) with a spectrum (202 MB) still larger than L2, for profiling
    # captures that must stay small
    "c6": ChannelSpec("c6-512x384x128-tanh1.5", 512, 384, 128, y_stretched=True, gamma=1.5, nbubbles=100,
                      radius=0.1, rhol=1.0, rhog=0.02),
    # c3's y-solve instance (512 rows) on a small grid whose spectrum (135 MB)
    # is still larger than L2, for profiling captures
    "c7": ChannelSpec("c7-256x512x128-tanh1.5", 256, 512, 128, y_stretched=True, gamma=1.5, nbubbles=60,
                      radius=0.15, rhol=1.0, rhog=0.02),
}



def ensemble_specs(n: int = 64, seed: int = 4) -> list:
    """The ensemble workload: n channels of the reference's minimal channel box
    (pi x 2 x pi/2, channel_18/specs/mesh:20-22), each with a seeded grid
    nx in {64, 96, 128}, ny in {96, 128, 192}, nz in {32, 48, 64} (tanh
    gamma 1.5), 4-24 bubbles of radius R in [0.2, 0.3], rho_l/rho_g = 1/0.05."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n):
        nx = int(rng.choice([64, 96, 128]))
        ny = int(rng.choice([96, 128, 192]))
        nz = int(rng.choice([32, 48, 64]))
        nb = int(rng.integers(4, 25))
        r = float(rng.uniform(0.2, 0.3))
        out.append(ChannelSpec(f"c4-{c:02d}-{nx}x{ny}x{nz}", nx, ny, nz, Lx=math.pi, Ly=2.0, Lz=0.5 * math.pi,
                               y_stretched=True, gamma=1.5, nbubbles=nb, radius=r, rhol=1.0, rhog=0.05))
    return out


# ---------------------------------------------------------------------------
# counter-based noise
# ---------------------------------------------------------------------------
_M64 = (1 << 64) - 1


def _s64(v: int) -> int:
    """Interpret an unsigned 64-bit constant as a signed int64."""
    v &= _M64
    return v - (1 << 64) if v >= (1 << 63) else v


def _lsr(z: torch.Tensor, s: int) -> torch.Tensor:
    """Logical right shift of int64 bit patterns."""
    return (z >> s) & ((1 << (64 - s)) - 1)


def splitmix64(x: torch.Tensor) -> torch.Tensor:
    """splitmix64 finaliser on int64 tensors (two's-complement wrap-around)."""
    z = x + _s64(0x9E3779B97F4A7C15)
    z = (z ^ _lsr(z, 30)) * _s64(0xBF58476D1CE4E5B9)
    z = (z ^ _lsr(z, 27)) * _s64(0x94D049BB133111EB)
    return z ^ _lsr(z, 31)


def uniform01(seed: int, field_id: int, n: int, device) -> torch.Tensor:
    """n uniform doubles in [0,1) from the top 53 bits of splitmix64(key)."""
    idx = torch.arange(n, dtype=torch.int64, device=device)
    key = idx ^ ((int(seed) & 0xFFFFF) << 44) ^ ((int(field_id) & 0xF) << 40)
    z = splitmix64(key)
    return _lsr(z, 11).to(torch.float64) * (1.0 / 9007199254740992.0)


def splitmix64_numpy(x: np.ndarray) -> np.ndarray:
    """Same generator on numpy uint64 (reference for the torch version)."""
    with np.errstate(over="ignore"):
        z = x.astype(np.uint64) + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


# ---------------------------------------------------------------------------
# boundary update of a cell field (periodic x/z, zero-gradient y walls)
# ---------------------------------------------------------------------------
def update_boundaries_cl(a: torch.Tensor, hd: int, nx: int, ny: int, nz: int) -> None:
    """updateBoundaries (field.f90:950-974) on one rank for the channel: the
    first y ghost copies the wall cell on the interior i,k range, then periodic
    halos in x and then in z over the full extent."""
    o = hd  # offset of index 1
    a[o : o + nz, o - 1, o : o + nx] = a[o : o + nz, o, o : o + nx]
    a[o : o + nz, o + ny, o : o + nx] = a[o : o + nz, o + ny - 1, o : o + nx]
    a[:, :, o + nx : o + nx + hd] = a[:, :, o : o + hd]
    a[:, :, o - hd : o] = a[:, :, o + nx - hd : o + nx]
    a[o + nz : o + nz + hd, :, :] = a[o : o + hd, :, :]
    a[o - hd : o, :, :] = a[o + nz - hd : o + nz, :, :]


# ---------------------------------------------------------------------------
# bubbles
# ---------------------------------------------------------------------------
def bubble_centres(spec: ChannelSpec, seed: int):
    """Seeded rejection sampling of non-overlapping centres (periodic distance
    >= 2R + 3h in x and z, h the largest cell size; 3h clearance from the walls)."""
    g = spec.grid()
    h = max(g.dxf[1], g.dzf[1], float(np.max(g.dyf.r(1, g.ny))))
    R = spec.radius
    rng = np.random.default_rng(seed)
    cen = []
    ylo, yhi = R + 3.0 * h, spec.Ly - R - 3.0 * h
    if yhi < ylo:  # coarse test grids: centre the bubbles between the walls
        ylo = yhi = 0.5 * spec.Ly
    dmin = 2.0 * R + 3.0 * h
    tries = 0
    while len(cen) < spec.nbubbles and tries < 200000:
        tries += 1
        c = np.array([rng.uniform(0, spec.Lx), rng.uniform(ylo, yhi), rng.uniform(0, spec.Lz)])
        ok = True
        for d in cen:
            dx = abs(c[0] - d[0])
            dx = min(dx, spec.Lx - dx)
            dz = abs(c[2] - d[2])
            dz = min(dz, spec.Lz - dz)
            if dx * dx + (c[1] - d[1]) ** 2 + dz * dz < dmin * dmin:
                ok = False
                break
        if ok:
            cen.append(c)
    return np.array(cen).reshape(-1, 3)


def vof_field(spec: ChannelSpec, centres, device="cpu", hd: int = 1) -> torch.Tensor:
    """Sharp volume fraction c ('cl', halo hd) with its boundary update."""
    g = spec.grid()
    nx, ny, nz = g.nx, g.ny, g.nz
    dx, dz = spec.Lx / nx, spec.Lz / nz
    R = spec.radius
    nref = spec.nref
    c = torch.zeros(field_shape("cl", hd, nx, ny, nz), dtype=torch.float64, device=device)
    yc = torch.tensor(g.yc.r(1, ny), dtype=torch.float64, device=device)
    yf = torch.tensor(g.yf.r(0, ny), dtype=torch.float64, device=device)
    sub = (torch.arange(nref, dtype=torch.float64, device=device) + 0.5) / nref
    for (x0, y0, z0) in centres:
        ia = int(math.floor((x0 - R) / dx)) - 1
        ib = int(math.floor((x0 + R) / dx)) + 2
        ka = int(math.floor((z0 - R) / dz)) - 1
        kb = int(math.floor((z0 + R) / dz)) + 2
        ii = torch.arange(ia, ib + 1, device=device)  # 1-based, unwrapped
        kk = torch.arange(ka, kb + 1, device=device)
        jsel = torch.nonzero((yf[1:] >= y0 - R - 1e-12) & (yf[:-1] <= y0 + R + 1e-12)).flatten()
        jj = jsel + 1
        xcb = 0.5 * dx + (ii.to(torch.float64) - 1.0) * dx
        zcb = 0.5 * dz + (kk.to(torch.float64) - 1.0) * dz
        ycb = yc[jj - 1]
        xfm, xfp = (ii.to(torch.float64) - 1.0) * dx, ii.to(torch.float64) * dx
        zfm, zfp = (kk.to(torch.float64) - 1.0) * dz, kk.to(torch.float64) * dz
        yfm, yfp = yf[jj - 1], yf[jj]
        X = (xcb - x0)[None, None, :]
        Y = (ycb - y0)[None, :, None]
        Z = (zcb - z0)[:, None, None]
        blk = ((X * X + Y * Y + Z * Z) <= R * R).to(torch.float64)
        cnt = torch.zeros_like(blk)
        for vx in (xfm, xfp):
            for vy in (yfm, yfp):
                for vz in (zfm, zfp):
                    r2 = ((vx - x0) ** 2)[None, None, :] + ((vy - y0) ** 2)[None, :, None] + ((vz - z0) ** 2)[:, None, None]
                    cnt += (r2 <= R * R).to(torch.float64)
        iface = (cnt > 0) & (cnt < 8)
        idx = torch.nonzero(iface)
        if idx.numel():
            # nref^3 sub-cell integration of interface cells (initialConditions.f90:349-377)
            for chunk in torch.split(idx, 4096):
                kq, jq, iq = chunk[:, 0], chunk[:, 1], chunk[:, 2]
                px = xfm[iq][:, None] + sub[None, :] * dx
                py = yfm[jq][:, None] + sub[None, :] * (yfp[jq] - yfm[jq])[:, None]
                pz = zfm[kq][:, None] + sub[None, :] * dz
                r2 = ((px - x0) ** 2)[:, None, None, :] + ((py - y0) ** 2)[:, None, :, None] + \
                    ((pz - z0) ** 2)[:, :, None, None]
                frac = (r2 <= R * R).sum(dim=(1, 2, 3)).to(torch.float64) / float(nref ** 3)
                blk[kq, jq, iq] = frac
        # scatter into the periodic domain (x, z wrap)
        iw = ((ii - 1) % nx) + hd
        kw = ((kk - 1) % nz) + hd
        jw = jj - 1 + hd
        c[kw[:, None, None], jw[None, :, None], iw[None, None, :]] += blk
    c.clamp_(0.0, 1.0)
    update_boundaries_cl(c, hd, nx, ny, nz)
    return c


def _cell_to_vertex(q, g: Grid, hd: int):
    """cellToVertex (interpolation.f90:188-229) onto vertices 0..n in each direction."""
    nx, ny, nz = g.nx, g.ny, g.nz
    dev = q.device
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)  # noqa: E731
    x, y, z = t(g.xc.r(0, nx + 1)), t(g.yc.r(0, ny + 1)), t(g.zc.r(0, nz + 1))
    xv, yv, zv = t(g.xf.r(0, nx)), t(g.yf.r(0, ny)), t(g.zf.r(0, nz))
    ax1, ax2 = x[1:] - xv, xv - x[:-1]
    ay1, ay2 = yv - y[:-1], y[1:] - yv
    az1, az2 = z[1:] - zv, zv - z[:-1]
    V = ((x[1:] - x[:-1])[None, None, :] * (y[1:] - y[:-1])[None, :, None]) * (z[1:] - z[:-1])[:, None, None]
    o = hd
    Q = lambda di, dj, dk: q[o - 1 + dk : o + nz + dk, o - 1 + dj : o + ny + dj, o - 1 + di : o + nx + di]  # noqa: E731
    X1, X2 = ax1[None, None, :], ax2[None, None, :]
    Y1, Y2 = ay1[None, :, None], ay2[None, :, None]
    Z1, Z2 = az1[:, None, None], az2[:, None, None]
    s = (X1 * Y1) * Z1 * Q(0, 1, 0)
    s = s + (X2 * Y1) * Z1 * Q(1, 1, 0)
    s = s + (X1 * Y1) * Z2 * Q(0, 1, 1)
    s = s + (X2 * Y1) * Z2 * Q(1, 1, 1)
    s = s + (X1 * Y2) * Z1 * Q(0, 0, 0)
    s = s + (X2 * Y2) * Z1 * Q(1, 0, 0)
    s = s + (X1 * Y2) * Z2 * Q(0, 0, 1)
    s = s + (X2 * Y2) * Z2 * Q(1, 0, 1)
    return s / V


def _vertex_to_cell(qv, out, g: Grid, hd: int):
    """vertexToCell (interpolation.f90:234-276) onto the interior cells of out."""
    nx, ny, nz = g.nx, g.ny, g.nz
    dev = qv.device
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)  # noqa: E731
    x, y, z = t(g.xc.r(1, nx)), t(g.yc.r(1, ny)), t(g.zc.r(1, nz))
    xv, yv, zv = t(g.xf.r(0, nx)), t(g.yf.r(0, ny)), t(g.zf.r(0, nz))
    bx1, bx2 = xv[1:] - x, x - xv[:-1]
    by1, by2 = y - yv[:-1], yv[1:] - y
    bz1, bz2 = zv[1:] - z, z - zv[:-1]
    V = ((xv[1:] - xv[:-1])[None, None, :] * (yv[1:] - yv[:-1])[None, :, None]) * (zv[1:] - zv[:-1])[:, None, None]
    P = lambda di, dj, dk: qv[dk : dk + nz, dj : dj + ny, di : di + nx]  # qv(i-1+di, j-1+dj, k-1+dk)  # noqa: E731
    X1, X2 = bx1[None, None, :], bx2[None, None, :]
    Y1, Y2 = by1[None, :, None], by2[None, :, None]
    Z1, Z2 = bz1[:, None, None], bz2[:, None, None]
    s = (X1 * Y1) * Z1 * P(0, 1, 0)
    s = s + (X2 * Y1) * Z1 * P(1, 1, 0)
    s = s + (X1 * Y1) * Z2 * P(0, 1, 1)
    s = s + (X2 * Y1) * Z2 * P(1, 1, 1)
    s = s + (X1 * Y2) * Z1 * P(0, 0, 0)
    s = s + (X2 * Y2) * Z1 * P(1, 0, 0)
    s = s + (X1 * Y2) * Z2 * P(0, 0, 1)
    s = s + (X2 * Y2) * Z2 * P(1, 0, 1)
    o = hd
    out[o : o + nz, o : o + ny, o : o + nx] = s / V


def smooth_vf(c: torch.Tensor, g: Grid, hd: int = 1) -> torch.Tensor:
    """smoothVF (VOF.f90:235-262): two cell->vertex->cell passes with boundary updates."""
    cs = torch.zeros_like(c)
    _vertex_to_cell(_cell_to_vertex(c, g, hd), cs, g, hd)
    update_boundaries_cl(cs, hd, g.nx, g.ny, g.nz)
    _vertex_to_cell(_cell_to_vertex(cs, g, hd), cs, g, hd)
    update_boundaries_cl(cs, hd, g.nx, g.ny, g.nz)
    return cs


def velocity(spec: ChannelSpec, seed: int, device="cpu", hd: int = 2) -> VField:
    """u* = Poiseuille + U[-0.05, 0.05] noise on interior faces, uy = 0 on the
    walls, periodic duplicates equated."""
    g = spec.grid()
    nx, ny, nz = g.nx, g.ny, g.nz
    icA = 1.5 * 4.0 / (spec.Ly * spec.Ly)  # unit bulk velocity
    comps = []
    for fid, kind in enumerate(("sx", "sy", "sz")):
        f = Field(kind, hd, nx, ny, nz, torch.zeros(field_shape(kind, hd, nx, ny, nz), dtype=torch.float64,
                                                    device=device))
        inner = f.interior()
        noise = uniform01(seed, fid, inner.numel(), device).reshape(inner.shape)
        inner.copy_(-0.05 + 0.1 * noise)
        comps.append(f)
    ux, uy, uz = comps
    yc = torch.tensor(g.yc.r(1, ny), dtype=torch.float64, device=device)
    prof = icA * yc * (spec.Ly - yc)
    ux.interior().add_(prof[None, :, None])
    uy.v(1, nx, 0, 0, 1, nz).zero_()
    uy.v(1, nx, ny, ny, 1, nz).zero_()
    ux.v(0, 0, 1, ny, 1, nz).copy_(ux.v(nx, nx, 1, ny, 1, nz))
    uz.v(1, nx, 1, ny, 0, 0).copy_(uz.v(1, nx, 1, ny, nz, nz))
    return VField(ux, uy, uz)


@dataclass
class ProjectionInputs:
    spec: ChannelSpec
    grid: Grid
    u: VField
    rho: Field
    cs: Field
    psi_n: Field
    psi_nm1: Field
    dt: float
    alpha: float
    rho0: float
    c: Field | None = None  # the sharp volume fraction before smoothVF (surface tension reads it)


def make_inputs(spec: ChannelSpec, seed: int = 1234, device="cpu", hd_u: int = 2, hd_psi: int = 1,
                hd_rho: int = 1) -> ProjectionInputs:
    """Inputs of the first call of a projection chain (psi^n = psi^{n-1} = 0)."""
    g = spec.grid()
    nx, ny, nz = g.nx, g.ny, g.nz
    cen = bubble_centres(spec, seed)
    c = vof_field(spec, cen, device=device, hd=hd_rho)
    cs = smooth_vf(c, g, hd_rho)
    rho = spec.rhog * cs + (1.0 - cs) * spec.rhol  # VOF.f90:223, whole array
    u = velocity(spec, seed, device=device, hd=hd_u)
    z = lambda: Field("cl", hd_psi, nx, ny, nz, torch.zeros(field_shape("cl", hd_psi, nx, ny, nz),  # noqa: E731
                                                            dtype=torch.float64, device=device))
    return ProjectionInputs(spec, g, u, Field("cl", hd_rho, nx, ny, nz, rho), Field("cl", hd_rho, nx, ny, nz, cs),
                            z(), z(), spec.dt, 1.0, min(spec.rhol, spec.rhog), Field("cl", hd_rho, nx, ny, nz, c))


def small_spec(nx=32, ny=24, nz=16, stretched=True, nbubbles=3, radius=0.3, rhog=0.05, **kw) -> ChannelSpec:
    """A quick test channel with the same box and recipe."""
    return ChannelSpec(f"small-{nx}x{ny}x{nz}", nx, ny, nz, y_stretched=stretched, gamma=1.5, nbubbles=nbubbles,
                       radius=radius, rhol=1.0, rhog=rhog, **kw)
