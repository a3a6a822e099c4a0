"""Flow control of the channel (setPressGrad, computeFlowRate, setFlowRate,
auxiliaryRoutines.f90:336-546): oracle known answers on the CPU and the CUDA
volume sums and shift against the oracle on the GPU."""
import numpy as np
import pytest
import torch

from oracle import tbfp_oracle as O
from tbfsolver_b200 import synth
from tbfsolver_b200.fields import Field, VField, field_shape
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import FastPoissonSolver, FlowControl, MomentumEqn
from tests._helpers import mesh_of, rel_linf


def _grid(nx, ny, nz, stretched):
    return Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, stretched, 1.5)


def _velocity(g, seed):
    rng = np.random.default_rng(seed)
    u = [O.FField(k, 2, g.nx, g.ny, g.nz, rng.uniform(-0.05, 0.05, field_shape(k, 2, g.nx, g.ny, g.nz)))
         for k in ("sx", "sy", "sz")]
    yc = g.yc.r(-1, g.ny + 2)
    u[0].a += (1.5 * yc * (2.0 - yc))[None, :, None]
    return u


def _rho(g, seed):
    spec = synth.small_spec(g.nx, g.ny, g.nz, stretched=g.y_stretched, nbubbles=3, radius=0.35)
    c = synth.vof_field(spec, synth.bubble_centres(spec, seed), device="cpu", hd=1).numpy().copy()
    _, rho, _ = O.update_material_props(mesh_of(g), O.FField("cl", 1, g.nx, g.ny, g.nz, c), 1.0, 0.02, 1e-3, 2e-5)
    return rho


# --- oracle known answers (CPU) ---------------------------------------------
@pytest.mark.parametrize("stretched", [False, True])
def test_uniform_fields_give_their_value_times_the_volume(stretched):
    """The staggered volumes of the faces i = 0..nx-1 tile the channel once:
    a uniform density is its own mean, a uniform ux carries U*Lx*Ly*Lz."""
    g = _grid(16, 12, 8, stretched)
    m = mesh_of(g)
    rho = O.FField("cl", 1, 16, 12, 8, np.full(field_shape("cl", 1, 16, 12, 8), 0.7))
    assert O.set_press_grad(m, rho, 2, 0.0, 1.0, 1e-3, 0.3) == pytest.approx(-0.7 * 0.3, rel=1e-13)
    nul = 1e-3 / 1.0
    assert O.set_press_grad(m, rho, 1, 180.0, 1.0, 1e-3, 0.3) == pytest.approx((180.0 * nul) ** 2 - 0.21, rel=1e-13)
    assert O.set_press_grad(m, rho, 0, 180.0, 1.0, 1e-3, 0.3) == 0.0
    ux = O.FField("sx", 2, 16, 12, 8, np.full(field_shape("sx", 2, 16, 12, 8), 1.25))
    assert O.compute_flow_rate(m, ux) == pytest.approx(1.25 * 2 * np.pi * 2.0 * np.pi, rel=1e-13)


def test_set_flow_rate_reaches_the_target():
    g = _grid(16, 12, 8, True)
    m = mesh_of(g)
    u = _velocity(g, 2)
    O.update_boundaries_v_channel(m, *u)
    q0 = 1.1 * O.compute_flow_rate(m, u[0])
    O.set_flow_rate(m, *u, q0, 2)
    assert O.compute_flow_rate(m, u[0]) == pytest.approx(q0, rel=1e-13)
    assert np.array_equal(u[0].v(0, 0, -1, 14, -1, 10), u[0].v(16, 16, -1, 14, -1, 10))


# --- CUDA path vs oracle (GPU) ---------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("where", ["host", "device"])
def test_sums_and_shift_match_the_oracle(where):
    nx, ny, nz = 32, 24, 16
    g = _grid(nx, ny, nz, True)
    m = mesh_of(g)
    u = _velocity(g, 3)
    O.update_boundaries_v_channel(m, *u)
    rho = _rho(g, 4)
    mk = (lambda f: Field(f.kind, f.hd, nx, ny, nz, torch.from_numpy(f.a.copy()).cuda())) if where == "device" else \
        (lambda f: Field(f.kind, f.hd, nx, ny, nz, f.a.copy()))  # noqa: E731
    with FastPoissonSolver(g) as fps:
        mom = MomentumEqn(fps, scheme=2)
        du = VField(*[mk(f) for f in u])
        drho = mk(rho)
        for ctrl in (1, 2, 3, 0):
            fc = FlowControl(fps, ctrl, ret=127.3)
            want = O.set_press_grad(m, rho, ctrl, 127.3, 1.0, 3.3e-4, 0.1)
            assert fc.set_press_grad(drho, 1.0, 3.3e-4, 0.1) == pytest.approx(want, rel=1e-13, abs=0)
        q = O.compute_flow_rate(m, u[0])
        assert FlowControl(fps, 2).flow_rate(du) == pytest.approx(q, rel=1e-13)
        fc = FlowControl(fps, 2, q0=1.05 * q)
        fc.set_flow_rate(mom, du)
        got = [f.a.cpu().numpy() if where == "device" else f.a for f in du.components()]
    O.set_flow_rate(m, *u, 1.05 * q, 2)
    for a, b in zip(got, u):
        assert rel_linf(a, b.a) < 1e-14


@pytest.mark.gpu
def test_two_fast_substeps_on_the_gpu_match_the_oracle_chain():
    """fast_substep twice (AB2 on the second, pressure levels rotated between):
    material properties, setPressGrad (flowCtrl 1), solveMomentumEqn,
    projection, updateBoundariesV, against the oracle's routines in the same
    order."""
    from tbfsolver_b200.solver import VOF, PoissonEqn, fast_substep

    nx, ny, nz = 32, 24, 16
    g = _grid(nx, ny, nz, True)
    m = mesh_of(g)
    props = dict(rhol=1.0, rhog=0.1, mul=3.3e-4, mug=3.3e-4)
    spec = synth.small_spec(nx, ny, nz, stretched=True, nbubbles=3, radius=0.35)
    c = O.FField("cl", 1, nx, ny, nz, synth.vof_field(spec, synth.bubble_centres(spec, 8), hd=1).numpy().copy())
    u = _velocity(g, 9)
    O.update_boundaries_v_channel(m, *u)
    dt, alpha, gch, ret = 2e-3, 1.0, 0.1, 127.3
    rho0 = min(props["rhol"], props["rhog"])
    dev = lambda f: Field(f.kind, f.hd, nx, ny, nz, torch.from_numpy(f.a.copy()).cuda())  # noqa: E731
    zero = lambda: O.FField("cl", 1, nx, ny, nz)  # noqa: E731
    eqn = PoissonEqn(g, props["rhol"], props["rhog"])
    try:
        vof = VOF(eqn.solver, **props)
        mom = MomentumEqn(eqn.solver, scheme=2, gch=gch)
        flow = FlowControl(eqn.solver, 1, ret=ret)
        du = VField(*[dev(f) for f in u])
        dc, dcs, drho, dmu = dev(c), dev(zero()), dev(zero()), dev(zero())
        dpsi, dpn, dpm = dev(zero()), dev(zero()), dev(zero())
        # oracle state
        pn, pm, prev = zero(), zero(), [np.zeros(s) for s in mom._shapes()]
        for gamma, xi in ((1.0, 0.0), (1.5, -0.5)):
            fast_substep(eqn, vof, mom, flow, dc, dcs, drho, dmu, du, dpsi, dpn, dpm, dt, alpha, gamma, xi)
            dpn, dpm, dpsi = PoissonEqn.update_pressure(dpsi, dpn, dpm)
            cs_o, rho_o, mu_o = O.update_material_props(m, c, **props)
            fs = O.set_press_grad(m, rho_o, 1, ret, props["rhol"], props["mul"], gch)
            prev = O.momentum_predictor(m, *u, c, mu_o, rho_o, prev, dt, alpha, gamma, xi, rho0, gch=gch, fs=fs)
            O.update_boundaries_v_channel(m, *u)
            res = O.projection(m, *u, rho_o, pn, pm, dt, alpha, rho0)
            u = [res.ux, res.uy, res.uz]
            O.update_boundaries_v_channel(m, *u)
            pn, pm = res.psi, pn
        got = [f.a.cpu().numpy() for f in du.components()]
        for a, b in zip(got, u):
            assert rel_linf(a, b.a) < 1e-11
        assert rel_linf(dpn.a.cpu().numpy()[1:-1, 1:-1, 1:-1], pn.a[1:-1, 1:-1, 1:-1]) < 1e-10
    finally:
        eqn.close()


@pytest.mark.gpu
def test_double_buffered_substep_matches_the_in_place_one():
    """fast_substep with a u_star scratch (out-of-place predictor, projection
    from u_star back into u) gives the in-place chain's velocity and pressure."""
    from tbfsolver_b200.solver import VOF, PoissonEqn, fast_substep

    nx, ny, nz = 32, 24, 16
    g = _grid(nx, ny, nz, True)
    m = mesh_of(g)
    props = dict(rhol=1.0, rhog=0.1, mul=3.3e-4, mug=3.3e-4)
    spec = synth.small_spec(nx, ny, nz, stretched=True, nbubbles=3, radius=0.35)
    c0 = synth.vof_field(spec, synth.bubble_centres(spec, 8), hd=1).numpy().copy()
    u0 = _velocity(g, 9)
    O.update_boundaries_v_channel(m, *u0)
    dev = lambda a, kind="cl", hd=1: Field(kind, hd, nx, ny, nz, torch.from_numpy(a.copy()).cuda())  # noqa: E731
    out = []
    for star in (False, True):
        eqn = PoissonEqn(g, props["rhol"], props["rhog"])
        try:
            vof = VOF(eqn.solver, **props)
            mom = MomentumEqn(eqn.solver, scheme=2, gch=0.1)
            flow = FlowControl(eqn.solver, 1, ret=127.3)
            du = VField(*[dev(f.a, f.kind, f.hd) for f in u0])
            us = VField(*[dev(np.zeros_like(f.a), f.kind, f.hd) for f in u0]) if star else None
            z = np.zeros(field_shape("cl", 1, nx, ny, nz))
            dc, dcs, drho, dmu, dpsi, dpn, dpm = (dev(a) for a in (c0, z, z, z, z, z, z))
            for gamma, xi in ((1.0, 0.0), (1.5, -0.5)):
                fast_substep(eqn, vof, mom, flow, dc, dcs, drho, dmu, du, dpsi, dpn, dpm, 2e-3, 1.0, gamma, xi,
                             u_star=us)
                dpn, dpm, dpsi = PoissonEqn.update_pressure(dpsi, dpn, dpm)
            out.append(([f.a.cpu().numpy() for f in du.components()], dpn.a.cpu().numpy()))
        finally:
            eqn.close()
    (ua, pa), (ub, pb) = out
    for a, b in zip(ua, ub):
        assert rel_linf(b, a) < 1e-13
    assert rel_linf(pb, pa) < 1e-12


@pytest.mark.gpu
def test_new_entry_points_refuse_bad_calls():
    """The momentum, boundary, flow and property entry points fail loudly
    (TbfpError with the library's message) instead of computing garbage."""
    from tbfsolver_b200._native import TBFP_EINVAL, TBFP_ENULL, TbfpError, load
    from tbfsolver_b200.dist import SlabChannel
    from tbfsolver_b200.solver import VOF

    g = _grid(16, 12, 8, True)
    lib = load()
    with FastPoissonSolver(g) as fps:
        mom = MomentumEqn.__new__(MomentumEqn)  # a wrapper without setup
        mom.solver = fps
        u = VField(*[Field(k, 2, 16, 12, 8, torch.zeros(field_shape(k, 2, 16, 12, 8), dtype=torch.float64,
                                                      device="cuda")) for k in ("sx", "sy", "sz")])
        with pytest.raises(TbfpError) as e:
            mom.update_boundaries_v(u)
        assert e.value.code == TBFP_EINVAL and "tbfp_momentum_setup" in str(e.value)
        assert lib.tbfp_update_boundaries_v_dev(fps.h, None, None, None) == TBFP_ENULL
        mom = MomentumEqn(fps, scheme=2)
        cl = lambda: Field("cl", 1, 16, 12, 8, torch.ones(field_shape("cl", 1, 16, 12, 8), dtype=torch.float64,  # noqa: E731
                                                            device="cuda"))
        with pytest.raises(TbfpError) as e:  # u_out aliasing u
            mom.predictor(u, cl(), cl(), cl(), dt=1e-3, alpha=1.0, gamma=1.0, xi=0.0, rho0=1.0, u_out=u)
        assert e.value.code == TBFP_EINVAL
        with pytest.raises(TbfpError):  # dt must be positive
            mom.predictor(u, cl(), cl(), cl(), dt=0.0, alpha=1.0, gamma=1.0, xi=0.0, rho0=1.0)
        with pytest.raises(TbfpError):  # a second setup on the handle
            MomentumEqn(fps, scheme=2)
    chan = SlabChannel(g, 2, 0)
    try:
        vof = VOF(chan, rhol=1.0, rhog=0.1, mul=1e-3, mug=1e-4)
        c = Field("cl", 1, 16, 12, chan.s.nz_loc,
                  torch.zeros(field_shape("cl", 1, 16, 12, chan.s.nz_loc), dtype=torch.float64, device="cuda"))
        outs = [Field.like(c, torch.zeros_like(c.a)) for _ in range(3)]
        with pytest.raises(TbfpError) as e:  # a slab needs the two passes with exchanges
            vof.update_material_props(c, *outs)
        assert "tbfp_material_props_pass_dev" in str(e.value)
    finally:
        chan.close()
