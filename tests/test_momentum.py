"""Momentum predictor (solveMomentumEqn FAST, momentumEqn.f90:161-194, without
its closing updateBoundariesV): oracle known answers on the CPU, and the CUDA
path (tbfp_momentum_predictor) against the oracle on the GPU, every
convection scheme, host and device fields, two calls so that the second one
uses the flux history (AB2)."""
import numpy as np
import pytest
import torch

from oracle import tbfp_oracle as O
from tbfsolver_b200 import synth
from tbfsolver_b200.fields import Field, VField, field_shape
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import FastPoissonSolver, MomentumEqn
from tests._helpers import mesh_of, rel_linf

PROPS = dict(rhol=1.0, rhog=0.02, mul=1e-3, mug=2e-5)
HD_U, HD_RHO, HD_ST = 2, 1, 1


def _grid(nx, ny, nz, stretched):
    return Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, stretched, 1.5)


def _velocity(g, seed):
    """Poiseuille + noise over the WHOLE arrays, ghosts and halos included, so
    every ghost value the stencils read is a distinct number."""
    rng = np.random.default_rng(seed)
    out = []
    for kind in ("sx", "sy", "sz"):
        a = rng.uniform(-0.05, 0.05, field_shape(kind, HD_U, g.nx, g.ny, g.nz))
        out.append(O.FField(kind, HD_U, g.nx, g.ny, g.nz, a))
    yc = g.yc.r(1 - HD_U, g.ny + HD_U)
    out[0].a += (1.5 * yc * (2.0 - yc))[None, :, None]
    return out


def _props(g, seed):
    """c from seeded bubbles; cs, rho, mu from it (updateMaterialProps)."""
    spec = synth.small_spec(g.nx, g.ny, g.nz, stretched=g.y_stretched, nbubbles=3, radius=0.35)
    c = synth.vof_field(spec, synth.bubble_centres(spec, seed), device="cpu", hd=HD_RHO).numpy().copy()
    fc = O.FField("cl", HD_RHO, g.nx, g.ny, g.nz, c)
    _, rho, mu = O.update_material_props(mesh_of(g), fc, **PROPS)
    return fc, mu, rho


def _st(g, seed):
    rng = np.random.default_rng(seed)
    return [O.FField(k, HD_ST, g.nx, g.ny, g.nz, rng.uniform(-1, 1, field_shape(k, HD_ST, g.nx, g.ny, g.nz)))
            for k in ("sx", "sy", "sz")]


# --- oracle known answers (CPU) ---------------------------------------------
@pytest.mark.parametrize("scheme", range(6))
def test_uniform_flow_has_no_fluxes(scheme):
    """Constant u: every face flux is U^2 on both sides and every difference
    quotient is zero, whatever the limiter."""
    g = _grid(12, 10, 8, True)
    m = mesh_of(g)
    u = [O.FField(k, HD_U, 12, 10, 8, np.full(field_shape(k, HD_U, 12, 10, 8), v))
         for k, v in (("sx", 0.7), ("sy", -0.2), ("sz", 0.3))]
    c, mu, rho = _props(g, 5)
    phi = O.momentum_fluxes(m, *u, c, mu, rho, scheme)
    for p in phi:
        assert np.max(np.abs(p)) == 0.0


def test_parabolic_profile_gives_the_viscous_term():
    """ux = a*y^2 + b*y on a uniform grid, uy = uz = 0, mu and rho constant: the
    second difference is exact, so phi_x = 2*a*mu/rho everywhere (the walls'
    ghosts hold the same parabola) and phi_y = phi_z = 0."""
    nx, ny, nz = 8, 12, 6
    g = _grid(nx, ny, nz, False)
    m = mesh_of(g)
    a, b, mu0, rho0 = -1.3, 0.4, 2e-3, 0.8
    ux = O.FField("sx", HD_U, nx, ny, nz)
    yc = m.yc.r(1 - HD_U, ny + HD_U)
    ux.a[...] = (a * yc * yc + b * yc)[None, :, None]
    uy = O.FField("sy", HD_U, nx, ny, nz)
    uz = O.FField("sz", HD_U, nx, ny, nz)
    cl = lambda v: O.FField("cl", HD_RHO, nx, ny, nz, np.full(field_shape("cl", HD_RHO, nx, ny, nz), v))  # noqa: E731
    for scheme in (0, 2, 4):
        px, py, pz = O.momentum_fluxes(m, ux, uy, uz, cl(0.0), cl(mu0), cl(rho0), scheme)
        assert np.allclose(px, 2 * a * mu0 / rho0, rtol=1e-9, atol=0)
        assert np.max(np.abs(py)) == 0.0 and np.max(np.abs(pz)) == 0.0


def test_localvf_is_central_where_the_fraction_is_flat():
    """Scheme 5 uses superbee only where c varies; with c constant it is the
    central scheme, and on a sharp interface it differs from it."""
    g = _grid(16, 12, 8, True)
    m = mesh_of(g)
    u = _velocity(g, 3)
    c, mu, rho = _props(g, 3)
    flat = O.FField("cl", HD_RHO, 16, 12, 8, np.full_like(c.a, 0.4))
    for p5, p0 in zip(O.momentum_fluxes(m, *u, flat, mu, rho, 5), O.momentum_fluxes(m, *u, flat, mu, rho, 0)):
        assert np.array_equal(p5, p0)
    diff = [np.max(np.abs(a - b)) for a, b in zip(O.momentum_fluxes(m, *u, c, mu, rho, 5),
                                                   O.momentum_fluxes(m, *u, c, mu, rho, 0))]
    assert max(diff) > 0.0


def test_predictor_adds_the_sources():
    """With no fluxes (uniform u) the update is the source term of addSource
    alone: ux += r*(st_x/rho0 + fs*invrho_x + gCH), uy += r*(st_y/rho0 + g),
    uz += r*st_z/rho0 with r = dt*alpha."""
    nx, ny, nz = 10, 8, 6
    g = _grid(nx, ny, nz, True)
    m = mesh_of(g)
    u = [O.FField(k, HD_U, nx, ny, nz, np.full(field_shape(k, HD_U, nx, ny, nz), 0.5)) for k in ("sx", "sy", "sz")]
    u0 = [f.copy() for f in u]
    c, mu, rho = _props(g, 9)
    st = _st(g, 2)
    dt, alpha, rho0, fs, gch, gy = 1e-3, 0.5, 0.02, 0.3, 1.1, -9.8
    prev = [np.zeros(s) for s in ((nz, ny, nx + 1), (nz, ny - 1, nx), (nz + 1, ny, nx))]
    O.momentum_predictor(m, *u, c, mu, rho, prev, dt, alpha, 1.5, -0.5, rho0, gch=gch, g=gy, fs=fs, st=st)
    r = dt * alpha
    invrho = 0.5 * (1.0 / rho.v(1, nx + 1, 1, ny, 1, nz) + 1.0 / rho.v(0, nx, 1, ny, 1, nz))
    want_x = 0.5 + r / rho0 * st[0].v(0, nx, 1, ny, 1, nz) + invrho * r * fs + r * gch
    want_y = 0.5 + r / rho0 * st[1].v(1, nx, 1, ny - 1, 1, nz) + r * gy
    want_z = 0.5 + r / rho0 * st[2].v(1, nx, 1, ny, 0, nz)
    assert np.allclose(u[0].v(0, nx, 1, ny, 1, nz), want_x, rtol=1e-14, atol=0)
    assert np.allclose(u[1].v(1, nx, 1, ny - 1, 1, nz), want_y, rtol=1e-14, atol=0)
    assert np.allclose(u[2].v(1, nx, 1, ny, 0, nz), want_z, rtol=1e-14, atol=0)
    # wall faces of uy and the ghosts are not touched
    assert np.array_equal(u[1].v(1, nx, 0, 0, 1, nz), u0[1].v(1, nx, 0, 0, 1, nz))
    assert np.array_equal(u[0].a[:, :, :HD_U], u0[0].a[:, :, :HD_U])


# --- CUDA path vs oracle (GPU) ---------------------------------------------
def _to_dev(f, where):
    a = torch.from_numpy(f.a.copy()).cuda() if where == "device" else f.a.copy()
    return Field(f.kind, f.hd, f.nx, f.ny, f.nz, a)


def _host(f):
    return f.a.cpu().numpy() if hasattr(f.a, "cpu") else f.a


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", range(6))
@pytest.mark.parametrize("dims,stretched,where", [((32, 24, 16), True, "device"), ((24, 20, 12), False, "host"),
                                                  ((48, 36, 24), True, "host")])
def test_momentum_predictor_matches_the_oracle(scheme, dims, stretched, where):
    nx, ny, nz = dims
    g = _grid(nx, ny, nz, stretched)
    m = mesh_of(g)
    u = _velocity(g, nx + scheme)
    c, mu, rho = _props(g, ny + scheme)
    st = _st(g, nz)
    kw = dict(dt=2e-3, alpha=1.0, rho0=0.02, fs=0.25)
    gch, gy = 0.7, -0.3
    with FastPoissonSolver(g, hd_u=HD_U, hd_rho=HD_RHO, hd_st=HD_ST) as fps:
        mom = MomentumEqn(fps, scheme=scheme, gch=gch, g=gy)
        du = VField(*[_to_dev(f, where) for f in u])
        dc, dmu, drho = (_to_dev(f, where) for f in (c, mu, rho))
        dst = [_to_dev(f, where) for f in st]
        prev = [np.zeros(s) for s in mom._shapes()]
        # first step: Euler-like (gamma=1, xi=0) from a zero history, as in the first step of the reference
        # second step: AB2 (gamma=1.5, xi=-0.5) with the first step's fluxes as history
        for gamma, xi in ((1.0, 0.0), (1.5, -0.5)):
            mom.predictor(du, dc, dmu, drho, gamma=gamma, xi=xi, st=dst, **kw)
            prev = O.momentum_predictor(m, *u, c, mu, rho, prev, kw["dt"], kw["alpha"], gamma, xi, kw["rho0"],
                                        gch=gch, g=gy, fs=kw["fs"], st=st, scheme=scheme)
            for got, want in zip(du.components(), u):
                assert rel_linf(_host(got), want.a) < 1e-13
        for got, want in zip(mom.fluxes(), prev):
            assert rel_linf(got, want) < 1e-12


@pytest.mark.gpu
def test_flux_history_is_loaded_and_read_back():
    """tbfp_momentum_fluxes(set=1) loads phi_prev (initOldTimeFlux); a step with
    gamma=0, xi=1 then adds dt*phi_prev to u (plus the sources, here none); the
    device may fuse the multiply-add, hence one rounding of slack."""
    nx, ny, nz = 24, 16, 12
    g = _grid(nx, ny, nz, True)
    u = _velocity(g, 1)
    c, mu, rho = _props(g, 1)
    rng = np.random.default_rng(4)
    with FastPoissonSolver(g, hd_u=HD_U, hd_rho=HD_RHO) as fps:
        mom = MomentumEqn(fps, scheme=2)
        hist = [rng.standard_normal(s) for s in mom._shapes()]
        mom.set_fluxes(hist)
        for a, b in zip(mom.fluxes(), hist):
            assert np.array_equal(a, b)
        du = VField(*[_to_dev(f, "device") for f in u])
        dc, dmu, drho = (_to_dev(f, "device") for f in (c, mu, rho))
        dt = 1e-3
        mom.predictor(du, dc, dmu, drho, dt=dt, alpha=1.0, gamma=0.0, xi=1.0, rho0=0.02)
        boxes = [(0, nx, 1, ny, 1, nz), (1, nx, 1, ny - 1, 1, nz), (1, nx, 1, ny, 0, nz)]
        for f, f0, h, b in zip(du.components(), u, hist, boxes):
            got = Field(f.kind, f.hd, nx, ny, nz, _host(f)).v(*b)
            assert np.max(np.abs(got - (f0.v(*b) + dt * h))) <= 2.3e-16 * np.max(np.abs(got))


@pytest.mark.gpu
def test_flux_history_round_trips_through_phi0_files(tmp_path):
    """printOldTimeFlux writes phi0x/y/z of the output folder in the field
    format; initOldTimeFlux reads them back (an absent component as zero)."""
    from tbfsolver_b200 import io

    nx, ny, nz = 16, 12, 8
    g = _grid(nx, ny, nz, True)
    rng = np.random.default_rng(11)
    with FastPoissonSolver(g) as fps:
        mom = MomentumEqn(fps, scheme=2)
        hist = [rng.standard_normal(s) for s in mom._shapes()]
        mom.set_fluxes(hist)
        mom.write_old_time_flux(str(tmp_path), 7)
    fy = Field("sy", 1, nx, ny, nz)
    io.read_field(str(tmp_path), 7, "phi0y", fy)
    assert np.array_equal(fy.v(1, nx, 1, ny - 1, 1, nz), hist[1])
    assert not fy.v(1, nx, 0, 0, 1, nz).any() and not fy.v(1, nx, ny, ny, 1, nz).any()
    (tmp_path / "7" / "phi0z").unlink()
    with FastPoissonSolver(g) as fps:
        mom = MomentumEqn(fps, scheme=2)
        mom.read_old_time_flux(str(tmp_path), 7)
        got = mom.fluxes()
    assert np.array_equal(got[0], hist[0]) and np.array_equal(got[1], hist[1])
    assert not got[2].any()


# --- updateBoundariesV --------------------------------------------------------
def test_wall_ghosts_mirror_the_first_layer_on_a_uniform_grid():
    """No-slip walls on a uniform grid: the wall sits halfway between the ghost
    and the first cell centre (ux, uz), or the ghost face mirrors face 1 about
    the wall face (uy), so the ghost is minus the first value (to the rounding
    of the coordinate differences in setMetrics); the x and z halos and the
    periodic duplicates are copies."""
    nx, ny, nz = 8, 6, 4
    g = _grid(nx, ny, nz, False)
    m = mesh_of(g)
    u = _velocity(g, 21)
    O.update_boundaries_v_channel(m, *u)
    ux, uy, uz = u
    assert np.allclose(ux.v(0, nx, 0, 0, 1, nz), -ux.v(0, nx, 1, 1, 1, nz), rtol=1e-13, atol=0)
    assert np.allclose(ux.v(0, nx, ny + 1, ny + 1, 1, nz), -ux.v(0, nx, ny, ny, 1, nz), rtol=1e-13, atol=0)
    assert np.allclose(uy.v(1, nx, -1, -1, 1, nz), -uy.v(1, nx, 1, 1, 1, nz), rtol=1e-13, atol=0)
    assert np.allclose(uz.v(1, nx, 0, 0, 0, nz), -uz.v(1, nx, 1, 1, 0, nz), rtol=1e-13, atol=0)
    full = (-HD_U + 1, ny + HD_U, -HD_U + 1, nz + HD_U)
    assert np.array_equal(ux.v(-2, -1, *full), ux.v(nx - 2, nx - 1, *full))
    assert np.array_equal(ux.v(0, 0, *full), ux.v(nx, nx, *full))
    assert np.array_equal(uz.v(-1, nx + 2, -1, ny + 2, 0, 0), uz.v(-1, nx + 2, -1, ny + 2, nz, nz))
    assert np.array_equal(uy.v(-1, nx + 2, -2, ny + 2, nz + 1, nz + 2), uy.v(-1, nx + 2, -2, ny + 2, 1, 2))


@pytest.mark.gpu
@pytest.mark.parametrize("hd,where", [(2, "device"), (2, "host"), (3, "device")])
def test_boundaries_match_the_oracle_bit_for_bit(hd, where):
    """tbfp_update_boundaries_v against the oracle's literal sequence (walls,
    x exchange, z exchange, equate) on random arrays, moving walls included."""
    from tbfsolver_b200.fields import field_shape as fsh

    nx, ny, nz = 24, 20, 12
    g = _grid(nx, ny, nz, True)
    rng = np.random.default_rng(hd)
    u = [O.FField(k, hd, nx, ny, nz, rng.standard_normal(fsh(k, hd, nx, ny, nz))) for k in ("sx", "sy", "sz")]
    ub, ut = (0.25, 0.0, -0.5), (1.0, 0.0, 0.125)
    with FastPoissonSolver(g, hd_u=hd) as fps:
        mom = MomentumEqn(fps, scheme=2, ubot=ub, utop=ut)
        du = VField(*[_to_dev(f, where) for f in u])
        mom.update_boundaries_v(du)
        got = [_host(f) for f in du.components()]
    O.update_boundaries_v_channel(mesh_of(g), *u, ub, ut)
    for a, b in zip(got, u):
        assert np.array_equal(a, b.a)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [2, 4])
def test_two_momentum_steps_with_boundaries_match_the_oracle(scheme):
    """solveMomentumEqn twice (predictor + updateBoundariesV, AB2 on the second
    step): the second step's stencils read the halos the first one refreshed."""
    nx, ny, nz = 32, 24, 16
    g = _grid(nx, ny, nz, True)
    m = mesh_of(g)
    u = _velocity(g, 5)
    c, mu, rho = _props(g, 6)
    O.update_boundaries_v_channel(m, *u)
    kw = dict(dt=2e-3, alpha=1.0, rho0=0.02)
    with FastPoissonSolver(g, hd_u=HD_U, hd_rho=HD_RHO) as fps:
        mom = MomentumEqn(fps, scheme=scheme, gch=0.4)
        du = VField(*[_to_dev(f, "device") for f in u])
        dc, dmu, drho = (_to_dev(f, "device") for f in (c, mu, rho))
        prev = [np.zeros(s) for s in mom._shapes()]
        for gamma, xi in ((1.0, 0.0), (1.5, -0.5)):
            mom.solve(du, dc, dmu, drho, gamma=gamma, xi=xi, **kw)
            prev = O.momentum_predictor(m, *u, c, mu, rho, prev, kw["dt"], kw["alpha"], gamma, xi, kw["rho0"],
                                        gch=0.4, scheme=scheme)
            O.update_boundaries_v_channel(m, *u)
            for got, want in zip(du.components(), u):
                assert rel_linf(_host(got), want.a) < 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", [2, 4, 5])
def test_out_of_place_predictor_equals_the_in_place_one(scheme):
    """tbfp_momentum_predictor_out_dev: the update fused into the flux kernel
    gives the in-place step's values on the boxes (to the rounding of a fused
    multiply-add), u's values elsewhere, the same flux history, and leaves u
    untouched."""
    nx, ny, nz = 48, 24, 16
    g = _grid(nx, ny, nz, True)
    u = _velocity(g, 30 + scheme)
    c, mu, rho = _props(g, 31)
    st = _st(g, 32)
    kw = dict(dt=2e-3, alpha=0.5, gamma=1.5, xi=-0.5, rho0=0.02, fs=0.3)
    res = []
    for out in (False, True):
        with FastPoissonSolver(g, hd_u=HD_U, hd_rho=HD_RHO, hd_st=HD_ST) as fps:
            mom = MomentumEqn(fps, scheme=scheme, gch=0.2, g=-0.1)
            hist = [np.random.default_rng(7).standard_normal(s) for s in mom._shapes()]
            mom.set_fluxes(hist)
            du = VField(*[_to_dev(f, "device") for f in u])
            dc, dmu, drho = (_to_dev(f, "device") for f in (c, mu, rho))
            dst = [_to_dev(f, "device") for f in st]
            if out:
                uo = VField(*[Field(f.kind, f.hd, nx, ny, nz, torch.full_like(f.a, np.nan)) for f in du.components()])
                mom.predictor(du, dc, dmu, drho, st=dst, u_out=uo, **kw)
                for a, b in zip(du.components(), u):
                    assert np.array_equal(_host(a), b.a)
                du = uo
            else:
                mom.predictor(du, dc, dmu, drho, st=dst, **kw)
            res.append(([_host(f) for f in du.components()], mom.fluxes()))
    (ua, pa), (ub, pb) = res
    for a, b in zip(ua, ub):
        assert not np.isnan(b).any()
        assert rel_linf(b, a) < 1e-15
    for a, b in zip(pa, pb):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("hd_u,hd_rho", [(3, 1), (2, 2), (3, 2)])
def test_predictor_with_wider_halos_matches_the_oracle(hd_u, hd_rho):
    """The kernels address every array through its layout: wider velocity or
    cell halos than the reference's 2 and 1 give the same step."""
    nx, ny, nz = 24, 20, 12
    g = _grid(nx, ny, nz, True)
    m = mesh_of(g)
    rng = np.random.default_rng(hd_u * 10 + hd_rho)
    u = [O.FField(k, hd_u, nx, ny, nz, rng.uniform(-0.5, 0.5, field_shape(k, hd_u, nx, ny, nz))) for k in ("sx", "sy", "sz")]
    cl = lambda lo, hi: O.FField("cl", hd_rho, nx, ny, nz, rng.uniform(lo, hi, field_shape("cl", hd_rho, nx, ny, nz)))  # noqa: E731
    c, mu, rho = cl(0.0, 1.0), cl(1e-4, 1e-3), cl(0.1, 1.0)
    kw = dict(dt=2e-3, alpha=1.0, gamma=1.0, xi=0.0, rho0=0.1, fs=0.2)
    with FastPoissonSolver(g, hd_u=hd_u, hd_rho=hd_rho) as fps:
        mom = MomentumEqn(fps, scheme=5, gch=0.3)
        du = VField(*[_to_dev(f, "device") for f in u])
        dc, dmu, drho = (_to_dev(f, "device") for f in (c, mu, rho))
        mom.predictor(du, dc, dmu, drho, **kw)
        got = [_host(f) for f in du.components()]
    prev = [np.zeros(s) for s in ((nz, ny, nx + 1), (nz, ny - 1, nx), (nz + 1, ny, nx))]
    O.momentum_predictor(m, *u, c, mu, rho, prev, kw["dt"], kw["alpha"], kw["gamma"], kw["xi"], kw["rho0"],
                         gch=0.3, fs=kw["fs"], scheme=5)
    for a, b in zip(got, u):
        assert rel_linf(a, b.a) < 1e-13
