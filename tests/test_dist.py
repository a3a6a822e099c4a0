"""Host side of the multi-GPU layer (tbfsolver_b200.dist) with world_size 2 on
the CPU (gloo): the spectrum all-to-alls between z slabs and kx slabs, the z
ghost-plane exchange of the slab stencils, and the max-over-ranks timing of
replicas.  Each rank checks its piece against the same seeded global array."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from tbfsolver_b200.dist import (Slabs, exchange_z_ghosts, exchange_z_ghosts_sz, exchange_z_ghosts_sz_local,
                                 max_over_ranks, split, sum_over_ranks, to_kx_slabs, to_z_slabs)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nx, ny, nz, errq):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=__import__("datetime").timedelta(seconds=60))
        s = Slabs(nx, ny, nz, world, rank)
        rng = np.random.default_rng(7)
        g = rng.standard_normal((s.nkx, nz, ny)) + 1j * rng.standard_normal((s.nkx, nz, ny))
        full = torch.from_numpy(g)
        sz = full[:, s.k0:s.k0 + s.nz_loc].clone()
        sx = to_kx_slabs(sz, s)
        assert torch.equal(sx, full[s.kx0:s.kx0 + s.nkx_loc])
        back = to_z_slabs(sx, s)
        assert torch.equal(back, sz)
        # z ghost planes, hd = 1 and 2, periodic
        for hd in (1, 2):
            f = torch.from_numpy(rng.standard_normal((nz, 3, 5)))
            loc = torch.zeros((s.nz_loc + 2 * hd, 3, 5), dtype=torch.float64)
            loc[hd:hd + s.nz_loc] = f[s.k0:s.k0 + s.nz_loc]
            exchange_z_ghosts(loc, s, hd)
            idx = [(s.k0 - hd + m) % nz for m in range(s.nz_loc + 2 * hd)]
            assert torch.equal(loc, f[idx])
        # uz-like arrays (planes -hd..nz_loc+hd): ghosts and the periodic duplicate
        # plane 0 = the rank below's nz_loc; global faces 0..nz with face 0 == face nz
        for hd in (1, 2):
            faces = torch.from_numpy(rng.standard_normal((nz, 3, 5)))  # faces 1..nz at index 0..nz-1
            loc = torch.full((s.nz_loc + 1 + 2 * hd, 3, 5), float("nan"), dtype=torch.float64)
            loc[hd + 1:hd + 1 + s.nz_loc] = faces[s.k0:s.k0 + s.nz_loc]
            exchange_z_ghosts_sz(loc, s, hd)
            idx = [(s.k0 - hd + m - 1) % nz for m in range(s.nz_loc + 1 + 2 * hd)]
            assert torch.equal(loc, faces[idx])
        assert sum_over_ranks(float(rank + 1)) == float(world * (world + 1) // 2)
        assert max_over_ranks(float(rank + 1)) == float(world)
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report to the parent
        errq.put(f"rank {rank}: {e!r}")
        raise


@pytest.mark.parametrize("dims", [(16, 6, 8), (12, 5, 7)])  # even and uneven partitions
def test_slab_exchanges_world2(dims):
    ctx = mp.get_context("spawn")
    errq = ctx.Queue()
    mp.spawn(_worker, args=(2, _free_port(), *dims, errq), nprocs=2, join=True)
    assert errq.empty()


def test_partition():
    assert [split(10, 3, r) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]
    s = Slabs(16, 4, 8, 1, 0)
    sz = torch.randn(s.nkx, 8, 4, dtype=torch.complex128)
    assert torch.equal(to_z_slabs(to_kx_slabs(sz, s), s), sz)
    f = torch.arange(12.0).reshape(12, 1) * torch.ones(1, 2)
    loc = torch.zeros(14, 2)
    loc[1:13] = f[:12]
    s1 = Slabs(16, 4, 12, 1, 0)
    exchange_z_ghosts(loc, s1, 1)
    assert torch.equal(loc[0], f[11]) and torch.equal(loc[13], f[0])


def test_sz_exchange_one_process_matches_the_periodic_faces():
    """exchange_z_ghosts_sz_local over three slabs held by one process: every
    slab's planes -hd..nz_loc+hd hold the periodic faces k0-hd..k0+nz_loc+hd."""
    nz, hd = 10, 2
    slabs = [Slabs(8, 4, nz, 3, r) for r in range(3)]
    faces = torch.arange(float(nz)).reshape(nz, 1)  # faces 1..nz at index 0..nz-1
    locs = []
    for s in slabs:
        loc = torch.full((s.nz_loc + 1 + 2 * hd, 1), float("nan"))
        loc[hd + 1:hd + 1 + s.nz_loc] = faces[s.k0:s.k0 + s.nz_loc]
        locs.append(loc)
    exchange_z_ghosts_sz_local(locs, slabs, hd)
    for s, loc in zip(slabs, locs):
        idx = [(s.k0 - hd + m - 1) % nz for m in range(s.nz_loc + 1 + 2 * hd)]
        assert torch.equal(loc, faces[idx])
