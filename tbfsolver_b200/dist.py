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


def to_kx_slabs(sz: torch.Tensor, s: Slabs, group=None) -> torch.Tensor:
    """S_z[nkx, nz_loc, ny] -> S_x[nkx_loc, nz, ny] (the first all-to-all of a solve)."""
    assert sz.shape[0] == s.nkx and sz.shape[1] == s.nz_loc
    ny = sz.shape[2]
    send = _real(sz.contiguous()).reshape(-1)
    per_entry = send.numel() // (s.nkx * s.nz_loc * ny)  # 2 for complex
    in_splits = [s.kxslab(q)[1] * s.nz_loc * ny * per_entry for q in range(s.world)]
    out_splits = [s.nkx_loc * s.zslab(p)[1] * ny * per_entry for p in range(s.world)]
    recv = torch.empty(sum(out_splits), dtype=send.dtype, device=send.device)
    if s.world == 1:
        recv.copy_(send)
    else:
        dist.all_to_all_single(recv, send, out_splits, in_splits, group=group)
    out = torch.empty((s.nkx_loc, s.nz, ny) + ((2,) if sz.is_complex() else ()), dtype=send.dtype,
                      device=send.device)
    off = 0
    for p in range(s.world):
        k0, nzp = s.zslab(p)
        blk = recv[off:off + out_splits[p]].reshape((s.nkx_loc, nzp, ny) + out.shape[3:])
        out[:, k0:k0 + nzp] = blk
        off += out_splits[p]
    return torch.view_as_complex(out) if sz.is_complex() else out


def to_z_slabs(sx: torch.Tensor, s: Slabs, group=None) -> torch.Tensor:
    """S_x[nkx_loc, nz, ny] -> S_z[nkx, nz_loc, ny] (the second all-to-all)."""
    assert sx.shape[0] == s.nkx_loc and sx.shape[1] == s.nz
    ny = sx.shape[2]
    xr = _real(sx)
    per_entry = 2 if sx.is_complex() else 1
    # pack for each destination q its k range, kx-major
    send = torch.cat([xr[:, s.zslab(q)[0]:s.zslab(q)[0] + s.zslab(q)[1]].reshape(-1) for q in range(s.world)])
    in_splits = [s.nkx_loc * s.zslab(q)[1] * ny * per_entry for q in range(s.world)]
    out_splits = [s.kxslab(p)[1] * s.nz_loc * ny * per_entry for p in range(s.world)]
    recv = torch.empty(sum(out_splits), dtype=send.dtype, device=send.device)
    if s.world == 1:
        recv.copy_(send)
    else:
        dist.all_to_all_single(recv, send, out_splits, in_splits, group=group)
    out = recv.reshape((s.nkx, s.nz_loc, ny) + ((2,) if sx.is_complex() else ()))
    return torch.view_as_complex(out) if sx.is_complex() else out


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
