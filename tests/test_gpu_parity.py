"""GPU parity tests: the CUDA path, called through the C ABI, against the CPU
oracle and the golden fixtures.

Tolerances (the floating-point bar of the task): pressure and velocity within
1e-12 relative (L-infinity, relative to the field's max magnitude), max|div u|
within 1e-12 absolute.
"""
import glob
import os

import numpy as np
import pytest
import torch

from oracle import tbfp_oracle as O
from tbfsolver_b200 import synth
from tbfsolver_b200._native import TbfpError
from tbfsolver_b200.fields import Field, VField
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import FastPoissonSolver, PoissonEqn, compute_continuity_error, make_velocity_div_free
from tests._helpers import mesh_of, rel_linf, to_oracle

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL_P = 1e-12
TOL_DIV = 1e-12


def _grid_from(z):
    return Grid(int(z["nx"]), int(z["ny"]), int(z["nz"]), float(z["Lx"]), float(z["Ly"]), float(z["Lz"]),
                bool(z["stretched"]), float(z["gamma"]))


def _cuda(f: Field) -> Field:
    a = f.a if isinstance(f.a, torch.Tensor) else torch.from_numpy(np.asarray(f.a))
    return Field.like(f, a.to("cuda").contiguous())


def _np(f: Field) -> Field:
    a = f.a.detach().cpu().numpy() if isinstance(f.a, torch.Tensor) else np.asarray(f.a)
    return Field.like(f, np.ascontiguousarray(a, dtype=np.float64).copy())


# ---------------------------------------------------------------------------
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "kat_*.npz"))))
@pytest.mark.parametrize("where", ["host", "device"])
def test_golden_kat_solve_fps(path, where):
    """Manufactured solution: solve_fps(s = L_h psi*) == psi* - mean, ghosts included."""
    z = np.load(path)
    g = _grid_from(z)
    with FastPoissonSolver(g) as fps:
        s = Field("cl", 1, g.nx, g.ny, g.nz, z["s"].copy())
        p = Field("cl", 1, g.nx, g.ny, g.nz)
        if where == "device":
            s, p = _cuda(s), _cuda(p)
        fps.solve_fps(p, s)
        got = _np(p).a
    assert rel_linf(got, z["psi_expected"]) < TOL_P


def _golden_fields(z, device):
    nx, ny, nz = int(z["nx"]), int(z["ny"]), int(z["nz"])
    hu = int(z["hd_u"])
    mk = lambda kind, key, hd: Field(kind, hd, nx, ny, nz, z[key].copy())  # noqa: E731
    u = VField(mk("sx", "ux", hu), mk("sy", "uy", hu), mk("sz", "uz", hu))
    rest = [mk("cl", k, 1) for k in ("rho", "psi_n", "psi_nm1")]
    st_n = st_nm1 = None
    if "stn_x" in z:
        st_n = [mk(k, "stn_" + c, 1) for k, c in zip(("sx", "sy", "sz"), "xyz")]
        st_nm1 = [mk(k, "sto_" + c, 1) for k, c in zip(("sx", "sy", "sz"), "xyz")]
    if device:
        u = VField(*[_cuda(f) for f in u.components()])
        rest = [_cuda(f) for f in rest]
        if st_n:
            st_n = [_cuda(f) for f in st_n]
            st_nm1 = [_cuda(f) for f in st_nm1]
    return u, rest, st_n, st_nm1


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "proj_*.npz"))))
@pytest.mark.parametrize("mode", ["host", "device_inplace", "device_outofplace"])
def test_golden_projection(path, mode):
    """One projection (computeSource, solveFPS, makeVelocityDivFree, continuity check)."""
    z = np.load(path)
    g = _grid_from(z)
    dev = mode != "host"
    u, (rho, pn, pnm1), st_n, st_nm1 = _golden_fields(z, dev)
    eqn = PoissonEqn(g, 1.0, float(z["rho0"]), hd_u=int(z["hd_u"]))
    try:
        psi = Field("cl", 1, g.nx, g.ny, g.nz)
        if dev:
            psi = _cuda(psi)
        uo = None
        if mode == "device_outofplace":
            uo = VField(*[Field.like(f, torch.full_like(f.a, 7.0)) for f in u.components()])
        st = eqn.projection(psi, pn, pnm1, rho, u, float(z["dt"]), float(z["alpha"]), st_n, st_nm1, u_out=uo)
        res = uo or u
        assert rel_linf(_np(psi).a, z["psi"]) < TOL_P
        for c, f in zip("xyz", res.components()):
            a = _np(f).a
            want = z[f"u{c}_out"]
            if mode == "device_outofplace":  # halos are not written out of place: compare interiors
                a = Field.like(f, a).interior()
                want = Field.like(f, want).interior()
            assert rel_linf(a, want) < TOL_P, c
        assert abs(st.max_div - float(z["max_div"])) < TOL_DIV
        assert st.cont_err == pytest.approx(st.max_div * float(z["dt"]), rel=1e-15)
    finally:
        eqn.close()


def _widen(f: Field, hd: int) -> Field:
    """f re-embedded with halo hd >= f.hd; the extra outer layers hold NaN,
    so any read of them shows up in the results."""
    w = Field(f.kind, hd, f.nx, f.ny, f.nz, torch.full(
        tuple(s + 2 * (hd - f.hd) for s in f.a.shape), float("nan"), dtype=f.a.dtype, device=f.a.device))
    d = hd - f.hd
    w.a[d:d + f.a.shape[0], d:d + f.a.shape[1], d:d + f.a.shape[2]] = f.a
    return w


@pytest.mark.gpu
def test_projection_with_wider_halos_matches_default_halos():
    """The out-of-place projection with psi and rho halos of 2 and velocity
    halos of 3 against the same projection with the default halos (1 and 2).
    Odd and even halos shift the tensor-map boxes of the staged correction by
    one column (the 16-byte start rule), so both offsets of every box run here;
    x tiles of 128 with a partial last tile, ny not a multiple of the tile
    height.  The arithmetic is the same, so the interiors agree to the bit."""
    spec = synth.small_spec(192, 20, 12, stretched=True, nbubbles=2, radius=0.3, rhog=0.05)
    inp = synth.make_inputs(spec, seed=13, device="cuda")
    g = inp.grid
    out = []
    for hps, hu in ((1, 2), (2, 3)):
        rho, pn, pnm1 = (_widen(f, hps) for f in (inp.rho, inp.psi_n, inp.psi_nm1))
        u = VField(*[_widen(f, hu) for f in inp.u.components()])
        psi = Field("cl", hps, g.nx, g.ny, g.nz, torch.zeros(
            tuple(s + 2 * (hps - 1) for s in inp.psi_n.a.shape), dtype=torch.float64, device="cuda"))
        uo = VField(*[Field.like(f, torch.zeros_like(f.a)) for f in u.components()])
        eqn = PoissonEqn(g, spec.rhol, spec.rhog, hd_psi=hps, hd_rho=hps, hd_u=hu)
        try:
            st = eqn.projection(psi, pn, pnm1, rho, u, inp.dt, inp.alpha, u_out=uo)
        finally:
            eqn.close()
        out.append(([_np(psi).interior().copy()] + [_np(f).interior().copy() for f in uo.components()], st.max_div))
    (a, mda), (b, mdb) = out
    for x, y in zip(a, b):
        assert np.isfinite(y).all()
        assert np.array_equal(x, y)
    assert mda == mdb and np.isfinite(mdb)


# ---------------------------------------------------------------------------
def _case(nx, ny, nz, stretched, nb=2, radius=0.3, seed=5, rhog=0.05):
    spec = synth.small_spec(nx, ny, nz, stretched=stretched, nbubbles=nb, radius=radius, rhog=rhog)
    return synth.make_inputs(spec, seed=seed)


@pytest.mark.parametrize("dims,stretched", [((32, 24, 16), True), ((64, 64, 32), False), ((96, 48, 48), True),
                                            ((128, 96, 64), True), ((48, 100, 24), False), ((256, 40, 12), True)])
def test_solve_fps_random_rhs(dims, stretched):
    """solveFPS on a seeded random right-hand side vs the oracle (LAPACK path);
    covers radix-2/4/8 and radix-3 lengths and ny not a multiple of 32.  The
    right-hand side is made compatible with the Neumann walls (zero volume
    integral), as every projection source is."""
    nx, ny, nz = dims
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, stretched, 1.5)
    m = mesh_of(g)
    rng = np.random.default_rng(nx + ny + nz)
    s = Field("cl", 1, nx, ny, nz)
    s.interior()[...] = rng.standard_normal((nz, ny, nx))
    s.interior()[...] -= np.sum(s.interior() * m.volume()) / m.s_Vg
    want = O.FField("cl", 1, nx, ny, nz)
    O.solve_fps(m, s.interior().copy(), want, tridiag="lapack-pinned" if nx * nz <= 8192 else "thomas")
    with FastPoissonSolver(g) as fps:
        p = _cuda(Field("cl", 1, nx, ny, nz))
        fps.solve_fps(p, _cuda(s))
        got = _np(p).a
    assert rel_linf(got, want.a) < TOL_P


@pytest.mark.parametrize("ny", [260, 300, 333, 384, 420, 500])
def test_persistent_y_solve_against_the_oracle_and_across_calls(ny):
    """ny in 257..384 takes the persistent one-warp-per-pair y solve (9..12
    rows per lane), ny in 385..512 the two-warp team form (7 or 8 rows per
    thread; the two warps' reduced systems meet through the spike column).
    Both prefetch their next pair and take pairs by ticket.  256 x ny x 64 has
    4257 pairs, several per warp or team.  Three solves on one handle give the
    same bits (the ticket counters return to zero after each launch), and the
    answer matches the oracle."""
    nx, nz = 256, 64
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, True, 1.5)
    m = mesh_of(g)
    rng = np.random.default_rng(ny)
    s = Field("cl", 1, nx, ny, nz)
    s.interior()[...] = rng.standard_normal((nz, ny, nx))
    s.interior()[...] -= np.sum(s.interior() * m.volume()) / m.s_Vg
    want = O.FField("cl", 1, nx, ny, nz)
    O.solve_fps(m, s.interior().copy(), want, tridiag="thomas")
    sd = _cuda(s)
    with FastPoissonSolver(g) as fps:
        outs = []
        for _ in range(3):
            p = _cuda(Field("cl", 1, nx, ny, nz))
            fps.solve_fps(p, sd)
            outs.append(p.a.clone())
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[0], outs[2])
    got = outs[0].cpu().numpy()
    assert rel_linf(got, want.a) < TOL_P


def test_solve_fps_two_layer_halo():
    """hd_psi = 2: the same interior as hd_psi = 1, with both x and z ghost
    layers periodic images and the first y ghost layer a copy of the wall cell
    (updateBoundaries on one rank)."""
    nx, ny, nz = 32, 24, 16
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, True, 1.5)
    m = mesh_of(g)
    rng = np.random.default_rng(11)
    src = rng.standard_normal((nz, ny, nx))
    src -= np.sum(src * m.volume()) / m.s_Vg
    out = {}
    for hd in (1, 2):
        s = Field("cl", hd, nx, ny, nz)
        s.interior()[...] = src
        with FastPoissonSolver(g, hd_psi=hd) as fps:
            p = _cuda(Field("cl", hd, nx, ny, nz))
            fps.solve_fps(p, _cuda(s))
            out[hd] = _np(p).a
    a1, a2 = out[1], out[2]
    assert np.array_equal(a2[2:-2, 2:-2, 2:-2], a1[1:-1, 1:-1, 1:-1])
    # Fortran index f -> array index f + hd - 1 (hd = 2: f + 1)
    ix = lambda f: f + 1  # noqa: E731
    J, K = slice(ix(1), ix(ny) + 1), slice(ix(1), ix(nz) + 1)
    for gh, src_i in ((-1, nx - 1), (0, nx), (nx + 1, 1), (nx + 2, 2)):
        assert np.array_equal(a2[K, J, ix(gh)], a2[K, J, ix(src_i)]), gh
    I = slice(ix(1), ix(nx) + 1)
    for gh, src_k in ((-1, nz - 1), (0, nz), (nz + 1, 1), (nz + 2, 2)):
        assert np.array_equal(a2[ix(gh), J, I], a2[ix(src_k), J, I]), gh
    assert np.array_equal(a2[K, ix(0), I], a2[K, ix(1), I])
    assert np.array_equal(a2[K, ix(ny + 1), I], a2[K, ix(ny), I])


@pytest.mark.parametrize("stretched", [True, False])
def test_incompatible_rhs_is_solved_with_the_defect_on_the_top_wall(stretched):
    """A source with a non-zero volume integral has no Neumann solution.  The
    reference's epsilon pivot (fastPoissonSolver.f90:318-322) then returns the
    solution of the system whose defect is moved to the last y row (the top
    wall), shifted by a constant of order defect/epsilon that the zero-mean
    step cancels (losing most of its digits).  The library solves the same
    consistent system with an exact gauge: the residual L psi - s vanishes
    except on the top-wall plane, where it is uniform and equals
    -sum(s V) / (dyf(ny) Lx Lz)."""
    nx, ny, nz = 32, 24, 16
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, stretched, 1.5)
    m = mesh_of(g)
    rng = np.random.default_rng(5)
    s = Field("cl", 1, nx, ny, nz)
    s.interior()[...] = 1.0 + rng.standard_normal((nz, ny, nx))
    with FastPoissonSolver(g) as fps:
        p = _cuda(Field("cl", 1, nx, ny, nz))
        fps.solve_fps(p, _cuda(s))
        psi = O.FField("cl", 1, nx, ny, nz, _np(p).a)
    res = O.laplacian_fps(m, psi) - s.interior()
    scale = np.max(np.abs(s.interior()))
    assert np.max(np.abs(res[:, :-1, :])) < 1e-12 * scale
    defect = -np.sum(s.interior() * m.volume()) / (m.dyf[ny] * (nx * m.dx_fft if hasattr(m, "dx_fft") else g.Lx)
                                                   * g.Lz)
    assert np.max(np.abs(res[:, -1, :] - defect)) < 1e-11 * scale
    assert abs(np.sum(psi.interior() * m.volume())) / m.s_Vg < 1e-12 * np.max(np.abs(psi.interior()))


@pytest.mark.parametrize("stretched", [True, False])
def test_rhs_correct_and_continuity_separately(stretched):
    """tbfp_rhs_split, tbfp_correct and tbfp_continuity_error against
    computeSource, makeVelocityDivFree and computeContinuityError."""
    inp = _case(48, 32, 24, stretched, seed=11)
    g = inp.grid
    m = mesh_of(g)
    rng = np.random.default_rng(2)
    pn, pnm1 = _np(inp.psi_n), _np(inp.psi_nm1)
    pn.a[...] = rng.standard_normal(pn.a.shape)
    pnm1.a[...] = rng.standard_normal(pn.a.shape)
    o = {k: to_oracle(f, g) for k, f in (("ux", inp.u.ux), ("uy", inp.u.uy), ("uz", inp.u.uz), ("rho", inp.rho))}
    opn, opnm1 = to_oracle(pn, g), to_oracle(pnm1, g)
    s_ref = O.compute_source_fast(m, opn, opnm1, o["rho"], o["ux"], o["uy"], o["uz"], inp.dt, inp.alpha, inp.rho0)
    eqn = PoissonEqn(g, 1.0, inp.rho0)
    try:
        u = VField(*[_cuda(f) for f in inp.u.components()])
        s = _cuda(Field("cl", 1, g.nx, g.ny, g.nz))
        eqn.compute_source(s, _cuda(pn), _cuda(pnm1), _cuda(inp.rho), u, inp.dt, inp.alpha)
        assert rel_linf(_np(s).interior(), s_ref) < TOL_P
        # correction with a given psi
        psi = _np(Field("cl", 1, g.nx, g.ny, g.nz))
        psi.a[...] = rng.standard_normal(psi.a.shape)
        opsi = to_oracle(psi, g)
        O.update_boundaries_cl_channel(opsi)
        psi.a[...] = opsi.a
        ux, uy, uz = o["ux"].copy(), o["uy"].copy(), o["uz"].copy()
        O.make_velocity_div_free(m, ux, uy, uz, opsi, opn, opnm1, o["rho"], inp.dt, inp.alpha, inp.rho0)
        make_velocity_div_free(eqn, u, _cuda(psi), _cuda(pn), _cuda(pnm1), _cuda(inp.rho), inp.dt, inp.alpha)
        for f, want in zip(u.components(), (ux, uy, uz)):
            a = Field.like(f, _np(f).a)
            assert rel_linf(a.interior(), Field.like(f, want.a).interior()) < TOL_P
        md, ce = compute_continuity_error(eqn.solver, u, inp.dt)
        md_ref = O.compute_continuity_error(m, ux, uy, uz)
        assert abs(md - md_ref) <= 1e-12 * max(1.0, md_ref)
        assert ce == pytest.approx(md * inp.dt, rel=1e-15)
    finally:
        eqn.close()


@pytest.mark.parametrize("name", ["c1"])
def test_projection_chain_full_config(name):
    """Config 1 at full size (128x128x64, 18 bubbles): a 3-call projection chain on
    the GPU vs the oracle chain, compared at every call."""
    spec = synth.CONFIGS[name]
    inp = synth.make_inputs(spec, seed=2024)
    g = inp.grid
    m = mesh_of(g)
    ou = [to_oracle(f, g) for f in inp.u.components()]
    orho, opn, opnm1 = to_oracle(inp.rho, g), to_oracle(inp.psi_n, g), to_oracle(inp.psi_nm1, g)
    eqn = PoissonEqn(g, spec.rhol, spec.rhog)
    try:
        u0 = VField(*[_cuda(f) for f in inp.u.components()])
        rho, pn, pnm1 = _cuda(inp.rho), _cuda(inp.psi_n), _cuda(inp.psi_nm1)
        for call in range(3):
            r = O.projection(m, *ou, orho, opn, opnm1, inp.dt, inp.alpha, inp.rho0)
            psi = _cuda(Field("cl", 1, g.nx, g.ny, g.nz))
            uo = VField(*[Field.like(f, torch.empty_like(f.a)) for f in u0.components()])
            st = eqn.projection(psi, pn, pnm1, rho, u0, inp.dt, inp.alpha, u_out=uo)
            assert rel_linf(_np(psi).a, r.psi.a) < TOL_P, call
            for f, want in zip(uo.components(), (r.ux, r.uy, r.uz)):
                assert rel_linf(Field.like(f, _np(f).a).interior(), Field.like(f, want.a).interior()) < TOL_P
            assert abs(st.max_div - r.max_div) < TOL_DIV
            opnm1, opn = opn, r.psi
            pnm1, pn = pn, psi
    finally:
        eqn.close()


def test_host_and_device_paths_identical():
    inp = _case(32, 24, 16, True, seed=3)
    g = inp.grid
    eqn = PoissonEqn(g, 1.0, inp.rho0)
    try:
        uh = VField(*[_np(f) for f in inp.u.components()])
        ph = Field("cl", 1, g.nx, g.ny, g.nz)
        sh = eqn.projection(ph, _np(inp.psi_n), _np(inp.psi_nm1), _np(inp.rho), uh, inp.dt, inp.alpha)
        ud = VField(*[_cuda(f) for f in inp.u.components()])
        pd = _cuda(Field("cl", 1, g.nx, g.ny, g.nz))
        sd = eqn.projection(pd, _cuda(inp.psi_n), _cuda(inp.psi_nm1), _cuda(inp.rho), ud, inp.dt, inp.alpha)
        assert np.array_equal(ph.a, _np(pd).a)
        for a, b in zip(uh.components(), ud.components()):
            assert np.array_equal(a.a, _np(b).a)
        assert sh.max_div == sd.max_div
    finally:
        eqn.close()


def test_errors_are_raised_not_hidden():
    g = Grid(16, 12, 8, 1.0, 2.0, 1.0)
    with FastPoissonSolver(g) as fps:
        with pytest.raises(TbfpError):
            fps.solve_fps(_cuda(Field("cl", 1, 16, 12, 8)), Field("cl", 1, 16, 12, 8))  # mixed placement
        eqn = PoissonEqn(g, 1.0, 0.1)
        u = VField.zeros(2, 16, 12, 8)
        f = Field("cl", 1, 16, 12, 8)
        with pytest.raises(TbfpError):
            eqn.projection(f, f, f, f, u, dt=-1.0, alpha=1.0)
        eqn.close()
