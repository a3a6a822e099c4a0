"""Multi-GPU layer of the projection: one process per GPU over torch.distributed.

The path spreads over GPUs in two ways.

* Replicas -- the ensemble workload: every rank projects its own channels and
  nothing on the data path is exchanged; only the timing is reduced (the
  maximum over ranks).
* Slabs -- one channel over P ranks: physical space is split into z slabs (the
  x transform is local; the RHS and correction stencils need one ghost plane
  from each z neighbour, periodic in z), spectral space into kx slabs (the z
  transform and the y solve are local).  Two all-to-alls per solve move the
  spectrum between the two layouts; this is the job of the reference's pencil
  transposes (pencilDec.f90:359-562) with a single pencil direction (py = 1).

This module holds the host side of both: the partitions, the packing of the
spectrum for the all-to-alls, and the z ghost-plane exchange.  It works on
tensors of any device (NCCL between GPUs; gloo on the CPU in the tests).

Spectrum layouts (the single-GPU library's S[kx][row], row = k*ny + j, kept
per rank):
  z-slab form:  S_z[kx][k_local][j]   for all kx = 0..nx/2, local k;
  kx-slab form: S_x[kx_local][k][j]   for local kx, all k.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist


def split(n: int, parts: int, r: int) -> tuple[int, int]:
    """Balanced block partition of range(n) into `parts`: (start, count) of part r."""
    base, extra = divmod(n, parts)
    count = base + (1 if r < extra else 0)
    start = r * base + min(r, extra)
    return start, count


@dataclass
class Slabs:
    """Ownership of one channel nx x ny x nz over `world` ranks."""

    nx: int
    ny: int
    nz: int
    world: int
    rank: int

    def __post_init__(self):
        self.nkx = self.nx // 2 + 1
        if self.nz < self.world or self.nkx < self.world:
            raise ValueError("every rank needs at least one z plane and one kx")
        self.k0, self.nz_loc = split(self.nz, self.world, self.rank)
        self.kx0, self.nkx_loc = split(self.nkx, self.world, self.rank)

    def zslab(self, r: int) -> tuple[int, int]:
        return split(self.nz, self.world, r)

    def kxslab(self, r: int) -> tuple[int, int]:
        return split(self.nkx, self.world, r)


def _real(t: torch.Tensor) -> torch.Tensor:
    return torch.view_as_real(t) if t.is_complex() else t


def kx_send_chunks(sz: torch.Tensor, s: Slabs) -> list:
    """S_z[nkx, nz_loc, ny] cut into the flat chunks for every destination rank
    (destination q gets its kx range, all local k)."""
    assert sz.shape[0] == s.nkx and sz.shape[1] == s.nz_loc
    xr = _real(sz.contiguous())
    return [xr[s.kxslab(q)[0]:s.kxslab(q)[0] + s.kxslab(q)[1]].reshape(-1) for q in range(s.world)]


def kx_assemble(chunks: list, s: Slabs, ny: int, cplx: bool) -> torch.Tensor:
    """S_x[nkx_loc, nz, ny] from the chunks received from every source rank."""
    tail = (2,) if cplx else ()
    out = torch.empty((s.nkx_loc, s.nz, ny) + tail, dtype=chunks[0].dtype, device=chunks[0].device)
    for p, c in enumerate(chunks):
        k0, nzp = s.zslab(p)
        out[:, k0:k0 + nzp] = c.reshape((s.nkx_loc, nzp, ny) + tail)
    return torch.view_as_complex(out) if cplx else out


def z_send_chunks(sx: torch.Tensor, s: Slabs) -> list:
    """S_x[nkx_loc, nz, ny] cut for every destination (its k range, local kx)."""
    assert sx.shape[0] == s.nkx_loc and sx.shape[1] == s.nz
    xr = _real(sx)
    return [xr[:, s.zslab(q)[0]:s.zslab(q)[0] + s.zslab(q)[1]].reshape(-1) for q in range(s.world)]


def z_assemble(chunks: list, s: Slabs, ny: int, cplx: bool) -> torch.Tensor:
    """S_z[nkx, nz_loc, ny] from the chunks of every source (kx ranges in order)."""
    out = torch.cat(chunks).reshape((s.nkx, s.nz_loc, ny) + ((2,) if cplx else ()))
    return torch.view_as_complex(out) if cplx else out


def _all_to_all(chunks: list, sizes_in: list, group) -> list:
    send = torch.cat(chunks)
    recv = torch.empty(sum(sizes_in), dtype=send.dtype, device=send.device)
    dist.all_to_all_single(recv, send, sizes_in, [c.numel() for c in chunks], group=group)
    return list(torch.split(recv, sizes_in))


def z_starts(s: Slabs) -> list:
    """First z plane of every rank's slab, and the channel's nz last."""
    return [s.zslab(r)[0] for r in range(s.world)] + [s.nz]


def to_kx_slabs(sz: torch.Tensor, s: Slabs, group=None, chan=None) -> torch.Tensor:
    """S_z[nkx, nz_loc, ny] -> S_x[nkx_loc, nz, ny] (the first all-to-all of a solve).
    With chan (the rank's SlabChannel) and device tensors, S_z is the send
    buffer as it is and one library kernel unpacks the received chunks."""
    ny = sz.shape[2]
    if chan is not None and sz.is_cuda:
        recv = sz.contiguous()
        if s.world > 1:
            recv = torch.empty(s.nkx_loc * s.nz * ny, dtype=sz.dtype, device=sz.device)
            ins = [s.nkx_loc * s.zslab(p)[1] * ny * 2 for p in range(s.world)]
            outs = [s.kxslab(q)[1] * s.nz_loc * ny * 2 for q in range(s.world)]
            dist.all_to_all_single(torch.view_as_real(recv).reshape(-1),
                                   torch.view_as_real(sz.contiguous()).reshape(-1), ins, outs, group=group)
        sx = torch.empty((s.nkx_loc, s.nz, ny), dtype=sz.dtype, device=sz.device)
        chan.unpack_kx(recv, sx)
        return sx
    chunks = kx_send_chunks(sz, s)
    if s.world > 1:
        per = 2 if sz.is_complex() else 1
        chunks = _all_to_all(chunks, [s.nkx_loc * s.zslab(p)[1] * ny * per for p in range(s.world)], group)
    return kx_assemble(chunks, s, ny, sz.is_complex())


def to_z_slabs(sx: torch.Tensor, s: Slabs, group=None, chan=None) -> torch.Tensor:
    """S_x[nkx_loc, nz, ny] -> S_z[nkx, nz_loc, ny] (the second all-to-all).  With
    chan and device tensors one library kernel packs the chunks and what the
    rank receives is S_z as it is."""
    ny = sx.shape[2]
    if chan is not None and sx.is_cuda:
        send = torch.empty(s.nkx_loc * s.nz * ny, dtype=sx.dtype, device=sx.device)
        chan.pack_z(sx, send)
        if s.world == 1:
            return send.reshape(s.nkx, s.nz_loc, ny)
        sz = torch.empty((s.nkx, s.nz_loc, ny), dtype=sx.dtype, device=sx.device)
        ins = [s.kxslab(p)[1] * s.nz_loc * ny * 2 for p in range(s.world)]
        outs = [s.nkx_loc * s.zslab(q)[1] * ny * 2 for q in range(s.world)]
        dist.all_to_all_single(torch.view_as_real(sz).reshape(-1), torch.view_as_real(send).reshape(-1), ins, outs,
                               group=group)
        return sz
    chunks = z_send_chunks(sx, s)
    if s.world > 1:
        per = 2 if sx.is_complex() else 1
        chunks = _all_to_all(chunks, [s.kxslab(p)[1] * s.nz_loc * ny * per for p in range(s.world)], group)
    return z_assemble(chunks, s, ny, sx.is_complex())


def exchange_z_ghosts(f: torch.Tensor, s: Slabs, hd: int, group=None) -> None:
    """Fill the hd ghost planes on each side of a z-slab field f[nz_loc + 2hd, ...]
    with the neighbours' interior planes (periodic in z, as updateBoundaries
    does for the reference's z ghosts)."""
    if s.nz_loc < hd:
        raise ValueError("a slab must hold at least hd planes")
    lo_int = f[hd:2 * hd]                      # first interior planes -> rank below's upper ghosts
    hi_int = f[s.nz_loc:s.nz_loc + hd]         # last interior planes -> rank above's lower ghosts
    if s.world == 1:
        f[0:hd] = hi_int
        f[s.nz_loc + hd:s.nz_loc + 2 * hd] = lo_int
        return
    below, above = (s.rank - 1) % s.world, (s.rank + 1) % s.world
    recv_lo = torch.empty_like(lo_int)
    recv_hi = torch.empty_like(hi_int)
    # tag 1: planes travelling up (k+), tag 2: down (k-); with two ranks the
    # neighbour below is also the one above, and the tags keep the pairs apart
    ops = [dist.P2POp(dist.isend, hi_int.contiguous(), above, group, 1),
           dist.P2POp(dist.irecv, recv_lo, below, group, 1),
           dist.P2POp(dist.isend, lo_int.contiguous(), below, group, 2),
           dist.P2POp(dist.irecv, recv_hi, above, group, 2)]
    for w in dist.batch_isend_irecv(ops):
        w.wait()
    f[0:hd] = recv_lo
    f[s.nz_loc + hd:s.nz_loc + 2 * hd] = recv_hi


def exchange_z_ghosts_sz(f: torch.Tensor, s: Slabs, hd: int, group=None) -> None:
    """The z exchange of a z-staggered field (uz, planes -hd..nz_loc+hd) on a
    slab: the hd ghost planes on each side and the periodic duplicate
    uz(:,:,0) = the rank below's uz(:,:,nz_loc) (updateHalo's 'sz' case,
    field.f90:910-930, and equatePeriodicBC, vfield.f90:124-189): the planes
    nz_loc-hd..nz_loc of the rank below land in -hd..0, the planes 1..hd of
    the rank above in nz_loc+1..nz_loc+hd."""
    n = s.nz_loc
    if n < hd + 1:
        raise ValueError("a slab must hold more than hd planes")
    up = f[n:n + hd + 1]              # k = nz_loc-hd..nz_loc -> rank above's -hd..0
    down = f[hd + 1:2 * hd + 1]       # k = 1..hd -> rank below's nz_loc+1..nz_loc+hd
    if s.world == 1:
        f[0:hd + 1] = up.clone()
        f[n + hd + 1:n + 2 * hd + 1] = down.clone()
        return
    below, above = (s.rank - 1) % s.world, (s.rank + 1) % s.world
    recv_lo = torch.empty_like(up)
    recv_hi = torch.empty_like(down)
    ops = [dist.P2POp(dist.isend, up.contiguous(), above, group, 3),
           dist.P2POp(dist.irecv, recv_lo, below, group, 3),
           dist.P2POp(dist.isend, down.contiguous(), below, group, 4),
           dist.P2POp(dist.irecv, recv_hi, above, group, 4)]
    for w in dist.batch_isend_irecv(ops):
        w.wait()
    f[0:hd + 1] = recv_lo
    f[n + hd + 1:n + 2 * hd + 1] = recv_hi


def exchange_v_ghosts(u, s: Slabs, hd: int, group=None) -> None:
    """The z part of updateBoundariesV on a slab (after tbfp_update_boundaries_v
    did the walls and x halos): ux and uy as cell-like fields, uz with its
    periodic duplicate."""
    exchange_z_ghosts(u.ux.a, s, hd, group)
    exchange_z_ghosts(u.uy.a, s, hd, group)
    exchange_z_ghosts_sz(u.uz.a, s, hd, group)


def slab_material_props(vof, c, cs, rho, mu, tmp, s: Slabs, group=None, exchange=None) -> None:
    """updateMaterialProps on a slab: the two smoothing passes, each followed by
    the z ghost exchange of what it wrote (the reference's updateBoundaries of
    cs between the passes; rho and mu are computed over the whole arrays
    there, so their ghost planes are the neighbours' values too).  exchange
    (fields) replaces the collective exchange, e.g. by copies between slabs
    held in one process; by default exchange_z_ghosts on each field."""
    ex = exchange or (lambda fs: [exchange_z_ghosts(f.a, s, 1, group) for f in fs])
    vof.smooth_pass(c, tmp)
    ex([tmp])
    vof.smooth_pass(tmp, cs, rho, mu)
    ex([cs, rho, mu])


def sum_over_ranks(x: float, device="cpu", group=None) -> float:
    """A volume sum over the ranks of a split channel (the reference's Mpi_Allreduce)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(x)
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return float(t.item())


def max_over_ranks(x: float, device="cpu", group=None) -> float:
    """The maximum of a per-rank value (device times are reported this way)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(x)
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's own channel (replicas): independent inputs per GPU."""
    return seed + rank


def exchange_z_ghosts_local(fields: list, slabs: list, hd: int) -> None:
    """The ghost exchange of exchange_z_ghosts for several ranks held by one
    process (fields[r] is rank r's slab): the same planes move, by copies."""
    P = len(fields)
    lows = [f[hd:2 * hd].clone() for f in fields]
    highs = [f[s.nz_loc:s.nz_loc + hd].clone() for f, s in zip(fields, slabs)]
    for r, (f, s) in enumerate(zip(fields, slabs)):
        f[0:hd] = highs[(r - 1) % P]
        f[s.nz_loc + hd:s.nz_loc + 2 * hd] = lows[(r + 1) % P]


def exchange_z_ghosts_sz_local(fields: list, slabs: list, hd: int) -> None:
    """exchange_z_ghosts_sz for several ranks held by one process, by copies."""
    P = len(fields)
    ups = [f[s.nz_loc:s.nz_loc + hd + 1].clone() for f, s in zip(fields, slabs)]
    downs = [f[hd + 1:2 * hd + 1].clone() for f in fields]
    for r, (f, s) in enumerate(zip(fields, slabs)):
        f[0:hd + 1] = ups[(r - 1) % P]
        f[s.nz_loc + hd + 1:s.nz_loc + 2 * hd + 1] = downs[(r + 1) % P]


def all_to_all_local(sends: list) -> list:
    """sends[p][q] -> recv[q][p] for several ranks held by one process."""
    P = len(sends)
    return [[sends[p][q] for p in range(P)] for q in range(P)]


class SlabChannel:
    """One rank's share of a channel split over ranks (tbfp_slab_*): solveFPS on
    z slabs / kx slabs with the two all-to-alls and the ghost exchange of this
    module.  The local arrays use the single-channel layout of the slab
    (nz_loc planes plus halos)."""

    def __init__(self, mesh, world: int, rank: int, hd_psi: int = 1, hd_u: int = 2, hd_rho: int = 1,
                 device: int = -1):
        import ctypes as C

        import numpy as np

        from ._native import TbfpDesc, check, load
        from .solver import _dptr

        self.lib = load()
        self.mesh, self.world, self.rank = mesh, world, rank
        self.s = s = Slabs(mesh.nx, mesh.ny, mesh.nz, world, rank)
        self.hd_psi, self.hd_u, self.hd_rho = hd_psi, hd_u, hd_rho
        nx, ny = mesh.nx, mesh.ny
        k0, nzl = s.k0, s.nz_loc
        self._m = {
            "dxf": np.ascontiguousarray(mesh.dxf.r(1, nx)), "dxc": np.ascontiguousarray(mesh.dxc.r(1, nx + 1)),
            "dyf": np.ascontiguousarray(mesh.dyf.r(1, ny)), "dyc": np.ascontiguousarray(mesh.dyc.r(1, ny + 1)),
            "dzf": np.ascontiguousarray(mesh.dzf.r(k0 + 1, k0 + nzl)),
            "dzc": np.ascontiguousarray(mesh.dzc.r(k0 + 1, k0 + nzl + 1)),
        }
        m = self._m
        d = TbfpDesc(nx=nx, ny=ny, nz=nzl, hd_psi=hd_psi, hd_u=hd_u, hd_rho=hd_rho, hd_st=1, dx_fft=mesh.dx_fft,
                     dz_fft=mesh.dz_fft, dxf=_dptr(m["dxf"]), dxc=_dptr(m["dxc"]), dyf=_dptr(m["dyf"]),
                     dyc=_dptr(m["dyc"]), dzf=_dptr(m["dzf"]), dzc=_dptr(m["dzc"]), s_Vg=mesh.s_Vg, precision=0,
                     tol=1e-10, max_iter=1, device=device, stream=None, flags=0)
        h = C.c_void_p()
        check(self.lib.tbfp_slab_create(C.byref(d), mesh.nz, k0, s.kx0, s.nkx_loc, C.byref(h)), None)
        self.h = h
        dev = torch.device("cuda", torch.cuda.current_device() if device < 0 else device)
        self.spec_z = torch.empty((s.nkx, nzl, ny), dtype=torch.complex128, device=dev)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.tbfp_destroy(self.h)
            self.h = None

    def forward_x(self, s_field) -> torch.Tensor:
        from ._native import check
        check(self.lib.tbfp_slab_forward_x(self.h, s_field.address(), self.spec_z.data_ptr()), self.h)
        return self.spec_z

    def spectral(self, spec_x: torch.Tensor) -> None:
        from ._native import check
        check(self.lib.tbfp_slab_spectral(self.h, spec_x.data_ptr()), self.h)

    def inverse_x(self, spec_z: torch.Tensor, psi) -> None:
        from ._native import check
        check(self.lib.tbfp_slab_inverse_x(self.h, spec_z.contiguous().data_ptr(), psi.address()), self.h)

    def _zs(self):
        import ctypes as C

        if not hasattr(self, "_zs_arr"):
            zs = z_starts(self.s)
            self._zs_arr = (C.c_int * len(zs))(*zs)
        return self._zs_arr

    def unpack_kx(self, recv: torch.Tensor, spec_x: torch.Tensor) -> None:
        """The chunks received in the first all-to-all (rank order) -> S_x (tbfp_slab_unpack_kx)."""
        from ._native import check
        check(self.lib.tbfp_slab_unpack_kx(self.h, self.world, self._zs(), recv.data_ptr(), spec_x.data_ptr()),
              self.h)

    def pack_z(self, spec_x: torch.Tensor, send: torch.Tensor) -> None:
        """S_x -> the chunks for every destination of the second all-to-all (tbfp_slab_pack_z)."""
        from ._native import check
        check(self.lib.tbfp_slab_pack_z(self.h, self.world, self._zs(), spec_x.data_ptr(), send.data_ptr()), self.h)

    def solve_fps(self, psi, s_field, group=None) -> None:
        """solveFPS on this rank's slab (a collective: every rank calls it)."""
        sz = self.forward_x(s_field)
        sx = to_kx_slabs(sz, self.s, group, chan=self)
        self.spectral(sx)
        self.inverse_x(to_z_slabs(sx, self.s, group, chan=self), psi)
        exchange_z_ghosts(psi.a, self.s, self.hd_psi, group)
