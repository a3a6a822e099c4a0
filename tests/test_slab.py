"""The slab form of the projection (tbfp_slab_*, tbfsolver_b200.dist) on one
GPU: P ranks of one channel are held by this process and their exchanges are
done by copies (the same planes the collectives move between GPUs).  Every
stage runs the single-channel kernels on the rank's rows, kx values or planes,
so the assembled result must equal the whole-channel result bit for bit:
solveFPS alone, and a full projection (split RHS, solve, correction) with the
z ghost planes of the inputs taken from the neighbouring slabs."""
import numpy as np
import pytest
import torch

from tbfsolver_b200 import synth
from tbfsolver_b200.dist import (SlabChannel, all_to_all_local, exchange_z_ghosts_local, kx_assemble,
                                 kx_send_chunks, z_assemble, z_send_chunks)
from tbfsolver_b200.fields import Field, VField
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import FastPoissonSolver, PoissonEqn, make_velocity_div_free
from tests._helpers import mesh_of

pytestmark = pytest.mark.gpu


def _zslice(f: Field, k0: int, nzl: int) -> Field:
    """Rank slab of a whole-channel field (interior planes k0+1..k0+nzl plus the
    halo planes around them), as a field of the slab's own layout."""
    extra = 1 if f.kind == "sz" else 0
    a = f.a[k0:k0 + nzl + extra + 2 * f.hd].clone()
    return Field(f.kind, f.hd, f.nx, f.ny, nzl, a)


def _slab_solve(chans, s_loc, psi_loc):
    """solveFPS over the ranks of chans, exchanges by copies."""
    spec_z = [c.forward_x(s).clone() for c, s in zip(chans, s_loc)]
    recv = all_to_all_local([kx_send_chunks(z, c.s) for z, c in zip(spec_z, chans)])
    spec_x = [kx_assemble(r, c.s, c.mesh.ny, True).contiguous() for r, c in zip(recv, chans)]
    for c, x in zip(chans, spec_x):
        c.spectral(x)
    recv = all_to_all_local([z_send_chunks(x, c.s) for x, c in zip(spec_x, chans)])
    for r, c, p in zip(recv, chans, psi_loc):
        c.inverse_x(z_assemble(r, c.s, c.mesh.ny, True), p)
    exchange_z_ghosts_local([p.a for p in psi_loc], [c.s for c in chans], chans[0].hd_psi)


@pytest.mark.parametrize("P,dims", [(2, (64, 48, 32)), (3, (48, 40, 24)), (4, (32, 24, 16)), (2, (128, 300, 32))])
def test_slab_solve_fps_is_the_whole_channel_solve(P, dims):
    nx, ny, nz = dims
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, True, 1.5)
    m = mesh_of(g)
    rng = np.random.default_rng(P)
    s = Field("cl", 1, nx, ny, nz)
    s.interior()[...] = rng.standard_normal((nz, ny, nx))
    s.interior()[...] -= np.sum(s.interior() * m.volume()) / m.s_Vg
    s = Field.like(s, torch.from_numpy(s.a).cuda())
    with FastPoissonSolver(g) as fps:
        whole = Field.like(s, torch.zeros_like(s.a))
        fps.solve_fps(whole, s)
    chans = [SlabChannel(g, P, r) for r in range(P)]
    try:
        s_loc = [_zslice(s, c.s.k0, c.s.nz_loc) for c in chans]
        psi_loc = [Field("cl", 1, nx, ny, c.s.nz_loc, torch.zeros_like(x.a)) for c, x in zip(chans, s_loc)]
        _slab_solve(chans, s_loc, psi_loc)
        for c, p in zip(chans, psi_loc):
            assert torch.equal(p.a, _zslice(whole, c.s.k0, c.s.nz_loc).a), c.rank
    finally:
        for c in chans:
            c.close()


class _Eqn:
    """The slab handle seen through PoissonEqn's interface (for the RHS and
    correction wrappers)."""

    def __init__(self, chan, rho0):
        self.solver = chan
        self.rho0 = rho0


def test_slab_projection_is_the_whole_channel_projection():
    spec = synth.small_spec(64, 48, 32, nbubbles=3, radius=0.3, rhog=0.05)
    inp = synth.make_inputs(spec, seed=13, device="cuda")
    g, dt, alpha = inp.grid, inp.dt, inp.alpha
    eqn = PoissonEqn(g, spec.rhol, spec.rhog)
    # history from a first projection, then the compared one, both in place
    u = VField(*[Field.like(f, f.a.clone()) for f in inp.u.components()])
    pn = Field.like(inp.psi_n, torch.zeros_like(inp.psi_n.a))
    eqn.projection(pn, inp.psi_n, inp.psi_nm1, inp.rho, u, dt, alpha)
    pnm1 = inp.psi_n
    u0 = [f.a.clone() for f in u.components()]
    psi = Field.like(pn, torch.zeros_like(pn.a))
    s = Field.like(pn, torch.zeros_like(pn.a))
    eqn.compute_source(s, pn, pnm1, inp.rho, u, dt, alpha)
    eqn.solver.solve_fps(psi, s)
    make_velocity_div_free(eqn, u, psi, pn, pnm1, inp.rho, dt, alpha)
    eqn.close()

    P = 2
    chans = [SlabChannel(g, P, r) for r in range(P)]
    try:
        uin = VField(*[Field.like(f, a) for f, a in zip(inp.u.components(), u0)])
        loc = []
        for c in chans:
            k0, nzl = c.s.k0, c.s.nz_loc
            loc.append(dict(u=VField(*[_zslice(f, k0, nzl) for f in uin.components()]),
                            rho=_zslice(inp.rho, k0, nzl), pn=_zslice(pn, k0, nzl), pnm1=_zslice(pnm1, k0, nzl)))
        s_loc, psi_loc = [], []
        for c, L in zip(chans, loc):
            e = _Eqn(c, eqn.rho0)
            sl = Field("cl", 1, g.nx, g.ny, c.s.nz_loc, torch.zeros_like(L["pn"].a))
            PoissonEqn.compute_source(e, sl, L["pn"], L["pnm1"], L["rho"], L["u"], dt, alpha)
            assert torch.equal(sl.interior(), _zslice(s, c.s.k0, c.s.nz_loc).interior()), c.rank
            s_loc.append(sl)
            psi_loc.append(Field("cl", 1, g.nx, g.ny, c.s.nz_loc, torch.zeros_like(L["pn"].a)))
        _slab_solve(chans, s_loc, psi_loc)
        for c, L, p in zip(chans, loc, psi_loc):
            make_velocity_div_free(_Eqn(c, eqn.rho0), L["u"], p, L["pn"], L["pnm1"], L["rho"], dt, alpha)
            k0, nzl = c.s.k0, c.s.nz_loc
            assert torch.equal(p.a, _zslice(psi, k0, nzl).a)
            for got, want in zip(L["u"].components(), u.components()):
                w = _zslice(want, k0, nzl)
                hd = got.hd
                lo = 1 + hd if got.kind == "sz" else hd  # the slab writes its own faces k0+1..k0+nzl
                assert torch.equal(got.a[lo:hd + nzl + (1 if got.kind == "sz" else 0)],
                                   w.a[lo:hd + nzl + (1 if got.kind == "sz" else 0)]), got.kind
    finally:
        for c in chans:
            c.close()


@pytest.mark.parametrize("P,dims", [(1, (32, 24, 16)), (3, (48, 40, 16)), (4, (64, 24, 24))])
def test_library_packing_matches_the_torch_packing(P, dims):
    """tbfp_slab_unpack_kx / tbfp_slab_pack_z against the torch chunk functions,
    uneven partitions included: bit for bit, and the whole split solve through
    the library packing equals the whole-channel solve."""
    nx, ny, nz = dims
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, True, 1.5)
    chans = [SlabChannel(g, P, r) for r in range(P)]
    try:
        gen = torch.Generator(device="cuda").manual_seed(P)
        sz = [torch.randn((c.s.nkx, c.s.nz_loc, ny), dtype=torch.complex128, device="cuda", generator=gen)
              for c in chans]
        sends = [kx_send_chunks(z, c.s) for z, c in zip(sz, chans)]
        recv = all_to_all_local(sends)
        for r, c in zip(recv, chans):
            want = kx_assemble(r, c.s, ny, True)
            flat = torch.view_as_complex(torch.cat(r).reshape(-1, 2))
            got = torch.empty_like(want)
            c.unpack_kx(flat, got)
            assert torch.equal(got, want)
            send = torch.empty(c.s.nkx_loc * nz * ny, dtype=torch.complex128, device="cuda")
            c.pack_z(want.contiguous(), send)
            chunks = z_send_chunks(want.contiguous(), c.s)
            assert torch.equal(torch.view_as_real(send).reshape(-1), torch.cat(chunks))
        # a whole solve with the library packing and local exchanges
        m = mesh_of(g)
        rng = np.random.default_rng(7)
        s = Field("cl", 1, nx, ny, nz)
        s.interior()[...] = rng.standard_normal((nz, ny, nx))
        s.interior()[...] -= np.sum(s.interior() * m.volume()) / m.s_Vg
        s = Field.like(s, torch.from_numpy(s.a).cuda())
        with FastPoissonSolver(g) as fps:
            whole = Field.like(s, torch.zeros_like(s.a))
            fps.solve_fps(whole, s)
        s_loc = [_zslice(s, c.s.k0, c.s.nz_loc) for c in chans]
        psi_loc = [Field("cl", 1, nx, ny, c.s.nz_loc, torch.zeros_like(x.a)) for c, x in zip(chans, s_loc)]
        spec_z = [c.forward_x(x).clone() for c, x in zip(chans, s_loc)]
        recv = all_to_all_local([[z[c2.s.kx0:c2.s.kx0 + c2.s.nkx_loc].reshape(-1) for c2 in chans] for z in spec_z])
        spec_x = []
        for r, c in zip(recv, chans):
            sx = torch.empty((c.s.nkx_loc, nz, ny), dtype=torch.complex128, device="cuda")
            c.unpack_kx(torch.cat(r), sx)
            c.spectral(sx)
            spec_x.append(sx)
        sends = []
        for x, c in zip(spec_x, chans):
            send = torch.empty(c.s.nkx_loc * nz * ny, dtype=torch.complex128, device="cuda")
            c.pack_z(x, send)
            offs = [c.s.nkx_loc * ny * c2.s.k0 for c2 in chans] + [c.s.nkx_loc * ny * nz]
            sends.append([send[offs[q]:offs[q + 1]] for q in range(P)])
        recv = all_to_all_local(sends)
        for r, c, p in zip(recv, chans, psi_loc):
            c.inverse_x(torch.cat(r).reshape(c.s.nkx, c.s.nz_loc, ny), p)
        exchange_z_ghosts_local([p.a for p in psi_loc], [c.s for c in chans], chans[0].hd_psi)
        for c, p in zip(chans, psi_loc):
            assert torch.equal(p.a, _zslice(whole, c.s.k0, c.s.nz_loc).a), c.rank
    finally:
        for c in chans:
            c.close()
