"""The momentum step (predictor + updateBoundariesV) and the material
properties on the slabs of a z-split channel, the ranks held by one process on
one GPU and their exchanges done by copies (the planes dist.exchange_v_ghosts
and dist.slab_material_props move between GPUs): every rank runs the
whole-channel kernels on its planes with its ghost planes from the
neighbours, so the assembled fields and fluxes equal the whole channel's bit
for bit."""
import numpy as np
import pytest
import torch

from oracle import tbfp_oracle as O
from tbfsolver_b200 import synth
from tbfsolver_b200.dist import SlabChannel, exchange_z_ghosts_local, exchange_z_ghosts_sz_local
from tbfsolver_b200.fields import Field, VField, field_shape
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import FastPoissonSolver, MomentumEqn
from tests._helpers import mesh_of

pytestmark = pytest.mark.gpu


def _zslice(f: Field, k0: int, nzl: int) -> Field:
    extra = 1 if f.kind == "sz" else 0
    return Field(f.kind, f.hd, f.nx, f.ny, nzl, f.a[k0:k0 + nzl + extra + 2 * f.hd].clone())


@pytest.mark.parametrize("P,dims,scheme", [(2, (32, 24, 16), 2), (3, (48, 40, 24), 4), (4, (32, 24, 16), 5)])
def test_slab_momentum_step_is_the_whole_channel_step(P, dims, scheme):
    nx, ny, nz = dims
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, True, 1.5)
    m = mesh_of(g)
    rng = np.random.default_rng(P)
    u = [O.FField(k, 2, nx, ny, nz, rng.uniform(-0.05, 0.05, field_shape(k, 2, nx, ny, nz))) for k in ("sx", "sy", "sz")]
    u[0].a += (1.5 * g.yc.r(-1, ny + 2) * (2.0 - g.yc.r(-1, ny + 2)))[None, :, None]
    O.update_boundaries_v_channel(m, *u)
    spec = synth.small_spec(nx, ny, nz, stretched=True, nbubbles=3, radius=0.35)
    c = O.FField("cl", 1, nx, ny, nz, synth.vof_field(spec, synth.bubble_centres(spec, P), hd=1).numpy().copy())
    _, rho, mu = O.update_material_props(m, c, 1.0, 0.05, 1e-3, 5e-5)
    dev = lambda f: Field(f.kind, f.hd, nx, ny, nz, torch.from_numpy(f.a.copy()).cuda())  # noqa: E731
    kw = dict(dt=2e-3, alpha=1.0, rho0=0.05, fs=0.2)
    steps = ((1.0, 0.0), (1.5, -0.5))
    # the whole channel
    with FastPoissonSolver(g) as fps:
        mom = MomentumEqn(fps, scheme=scheme, gch=0.3)
        wu = VField(*[dev(f) for f in u])
        wc, wmu, wrho = dev(c), dev(mu), dev(rho)
        for gamma, xi in steps:
            mom.solve(wu, wc, wmu, wrho, gamma=gamma, xi=xi, **kw)
        whole_phi = mom.fluxes()
    # the slabs
    chans = [SlabChannel(g, P, r) for r in range(P)]
    try:
        moms = [MomentumEqn(ch, scheme=scheme, gch=0.3) for ch in chans]
        su = [VField(*[_zslice(dev(f), ch.s.k0, ch.s.nz_loc) for f in u]) for ch in chans]
        sc = [[_zslice(f, ch.s.k0, ch.s.nz_loc) for f in (dev(c), dev(mu), dev(rho))] for ch in chans]
        slabs = [ch.s for ch in chans]
        for gamma, xi in steps:
            for mo, uu, (cc, mm, rr) in zip(moms, su, sc):
                mo.predictor(uu, cc, mm, rr, gamma=gamma, xi=xi, **kw)
                mo.update_boundaries_v(uu)
            exchange_z_ghosts_local([uu.ux.a for uu in su], slabs, 2)
            exchange_z_ghosts_local([uu.uy.a for uu in su], slabs, 2)
            exchange_z_ghosts_sz_local([uu.uz.a for uu in su], slabs, 2)
        for ch, uu, mo in zip(chans, su, moms):
            k0, nzl = ch.s.k0, ch.s.nz_loc
            for got, want in zip(uu.components(), wu.components()):
                assert torch.equal(got.a, _zslice(want, k0, nzl).a), ch.rank
            for got, want, kz in zip(mo.fluxes(), whole_phi, (0, 0, 1)):
                assert np.array_equal(got, want[k0:k0 + nzl + kz]), ch.rank
    finally:
        for ch in chans:
            ch.close()


@pytest.mark.parametrize("P,dims", [(2, (32, 24, 16)), (3, (48, 40, 24))])
def test_slab_material_props_are_the_whole_channel_props(P, dims):
    """updateMaterialProps on slabs: pass, z ghost exchange, pass, exchange
    (dist.slab_material_props, here with the exchanges done by copies between
    slabs held in one process) gives the whole channel's cs, rho, mu bit for
    bit, ghost planes included."""
    from tbfsolver_b200.solver import VOF

    nx, ny, nz = dims
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, True, 1.5)
    props = dict(rhol=1.0, rhog=0.05, mul=1e-3, mug=5e-5)
    spec = synth.small_spec(nx, ny, nz, stretched=True, nbubbles=3, radius=0.35)
    c = Field("cl", 1, nx, ny, nz, synth.vof_field(spec, synth.bubble_centres(spec, P), hd=1).cuda())
    zeros = lambda f: Field.like(f, torch.zeros_like(f.a))  # noqa: E731
    with FastPoissonSolver(g) as fps:
        vof = VOF(fps, **props)
        w = [zeros(c) for _ in range(3)]
        vof.update_material_props(c, *w)
    chans = [SlabChannel(g, P, r) for r in range(P)]
    try:
        vofs = [VOF(ch, **props) for ch in chans]
        sc = [_zslice(c, ch.s.k0, ch.s.nz_loc) for ch in chans]
        tmp = [zeros(x) for x in sc]
        outs = [[zeros(x) for _ in range(3)] for x in sc]
        slabs = [ch.s for ch in chans]
        for v, x, t in zip(vofs, sc, tmp):
            v.smooth_pass(x, t)
        exchange_z_ghosts_local([t.a for t in tmp], slabs, 1)
        for v, t, (cs, rho, mu) in zip(vofs, tmp, outs):
            v.smooth_pass(t, cs, rho, mu)
        for q in range(3):
            exchange_z_ghosts_local([o[q].a for o in outs], slabs, 1)
        for ch, o in zip(chans, outs):
            for got, want in zip(o, w):
                assert torch.equal(got.a, _zslice(want, ch.s.k0, ch.s.nz_loc).a), ch.rank
    finally:
        for ch in chans:
            ch.close()
