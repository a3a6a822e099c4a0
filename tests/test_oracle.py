"""CPU tests of the oracle (oracle/tbfp_oracle.py): analytic known answers, the
golden fixtures, and internal cross-checks.  No GPU needed."""
import glob
import os

import numpy as np
import pytest

from oracle import tbfp_oracle as O
from tests._helpers import rel_linf

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _mesh(nx, ny, nz, stretched, gamma=1.5, L=(2 * np.pi, 2.0, np.pi)):
    return O.Mesh(nx, ny, nz, *L, y_uniform=not stretched, gamma=gamma)


def _manufactured(m, seed):
    rng = np.random.default_rng(seed)
    ps = O.FField("cl", 1, m.nx, m.ny, m.nz)
    ps.v(1, m.nx, 1, m.ny, 1, m.nz)[...] = rng.standard_normal((m.nz, m.ny, m.nx))
    O.update_boundaries_cl_channel(ps)
    s = O.laplacian_fps(m, ps)
    ex = ps.interior() - np.sum(ps.interior() * m.volume()) / m.s_Vg
    return s, ex


@pytest.mark.parametrize("mode", ["lapack", "lapack-pinned", "thomas"])
@pytest.mark.parametrize("dims,stretched", [((16, 12, 8), False), ((16, 12, 8), True), ((32, 24, 16), True),
                                            ((24, 12, 12), False), ((48, 20, 6), True)])
def test_manufactured_solution(dims, stretched, mode):
    """KAT 1: s = L_h psi*, the solve must return psi* - mean (fastPoissonSolver.f90:337-423)."""
    m = _mesh(*dims, stretched)
    s, ex = _manufactured(m, 3)
    psi = O.FField("cl", 1, *dims)
    O.solve_fps(m, s, psi, tridiag=mode)
    assert rel_linf(psi.interior(), ex) < 1e-12
    # zero volume-weighted mean and updated ghosts
    assert abs(np.sum(psi.interior() * m.volume())) / m.s_Vg < 1e-13 * np.max(np.abs(ex))
    g = psi.copy()
    O.update_boundaries_cl_channel(g)
    assert np.array_equal(g.a, psi.a)


@pytest.mark.parametrize("dims,stretched", [((64, 64, 32), False), ((32, 24, 16), True), ((128, 96, 64), True)])
def test_epsilon_pivot_noise_of_the_reference(dims, stretched):
    """The reference's epsilon pivot for the singular (0,0) system
    (fastPoissonSolver.f90:318-322) and the exact gauge solve the same
    consistent system; in floating point the epsilon variant carries an extra
    error of up to a few 1e-11 (relative), which bounds how reproducible the
    reference's own pressure is.  Both leave a residual at rounding level."""
    m = _mesh(*dims, stretched)
    rng = np.random.default_rng(sum(dims))
    s = rng.standard_normal((m.nz, m.ny, m.nx))
    s -= np.sum(s * m.volume()) / m.s_Vg
    out = {}
    for mode in ("lapack", "lapack-pinned", "thomas"):
        p = O.FField("cl", 1, *dims)
        O.solve_fps(m, s, p, tridiag=mode)
        assert rel_linf(O.laplacian_fps(m, p), s) < 1e-12
        out[mode] = p.interior().copy()
    assert rel_linf(out["lapack-pinned"], out["thomas"]) < 1e-13
    assert rel_linf(out["lapack"], out["lapack-pinned"]) < 1e-10


def test_single_mode_eigenvalues():
    """KAT 2: psi = cos(2 pi m x/Lx) cos(2 pi n z/Lz) f(y) is an eigenfunction of the
    x/z second differences with lambda = 2(cos(2 pi m/nx)-1)/dx^2 (fastPoissonSolver.f90:235-248)."""
    nx, ny, nz = 32, 16, 24
    m = _mesh(nx, ny, nz, True)
    lx, lz = O.fps_eigenvalues(m)
    mx, mz = 3, 5
    x = m.xc.r(1, nx)
    z = m.zc.r(1, nz)
    y = m.yc.r(1, ny)
    f = np.cos(np.pi * y / 2.0)
    ps = O.FField("cl", 1, nx, ny, nz)
    ps.v(1, nx, 1, ny, 1, nz)[...] = (np.cos(2 * np.pi * mz * z / m.Lz)[:, None, None] * f[None, :, None]
                                       * np.cos(2 * np.pi * mx * x / m.Lx)[None, None, :])
    O.update_boundaries_cl_channel(ps)
    L = O.laplacian_fps(m, ps)
    am, ap = O.fps_offdiag(m)
    c = ps.v(1, nx, 1, ny, 1, nz)
    ly = ap[None, :, None] * (ps.v(1, nx, 2, ny + 1, 1, nz) - c) - am[None, :, None] * (c - ps.v(1, nx, 0, ny - 1, 1, nz))
    expect = (lx[mx] + lz[mz]) * c + ly
    assert rel_linf(L, expect) < 1e-12
    psi = O.FField("cl", 1, nx, ny, nz)
    O.solve_fps(m, L, psi)
    ex = c - np.sum(c * m.volume()) / m.s_Vg
    assert rel_linf(psi.interior(), ex) < 1e-12


def test_lapack_and_thomas_agree_on_projection():
    """Cross-check: the LAPACK zgttrf/zgttrs path and a vectorised Thomas give the same projection."""
    from tbfsolver_b200 import synth
    from tests._helpers import mesh_of, to_oracle

    spec = synth.small_spec(32, 24, 16, nbubbles=2, radius=0.3)
    inp = synth.make_inputs(spec, seed=5)
    g = inp.grid
    m = mesh_of(g)
    args = [to_oracle(f, g) for f in (inp.u.ux, inp.u.uy, inp.u.uz, inp.rho, inp.psi_n, inp.psi_nm1)]
    a = O.projection(m, *args, inp.dt, inp.alpha, inp.rho0, tridiag="lapack")
    b = O.projection(m, *args, inp.dt, inp.alpha, inp.rho0, tridiag="thomas")
    assert rel_linf(a.psi.a, b.psi.a) < 1e-12
    assert rel_linf(a.ux.a, b.ux.a) < 1e-13


def test_projection_is_divergence_free():
    """KAT 3: after the correction dt*max|div u| is at rounding level
    (auxiliaryRoutines.f90:42-91), for a chain of three calls with the split term active."""
    from tbfsolver_b200 import synth
    from tests._helpers import mesh_of, to_oracle

    spec = synth.small_spec(32, 24, 16, nbubbles=2, radius=0.3, rhog=0.02)
    inp = synth.make_inputs(spec, seed=9)
    g = inp.grid
    m = mesh_of(g)
    ux, uy, uz, rho, pn, pnm1 = [to_oracle(f, g) for f in
                                 (inp.u.ux, inp.u.uy, inp.u.uz, inp.rho, inp.psi_n, inp.psi_nm1)]
    div0 = O.compute_continuity_error(m, ux, uy, uz)
    for _ in range(3):
        r = O.projection(m, ux, uy, uz, rho, pn, pnm1, inp.dt, inp.alpha, inp.rho0)
        pnm1, pn = pn, r.psi
        assert r.max_div < 1e-12 * max(1.0, div0)
        assert r.cont_err == r.max_div * inp.dt


def test_constant_density_reduces_to_plain_projection():
    """KAT 5 (FFT side): with rho == const the split term vanishes and psi solves
    L psi = rho0/(alpha dt) div u*."""
    from tbfsolver_b200 import synth
    from tests._helpers import mesh_of, to_oracle

    spec = synth.small_spec(16, 12, 8, nbubbles=0)
    inp = synth.make_inputs(spec, seed=4)
    g = inp.grid
    m = mesh_of(g)
    ux, uy, uz, rho, pn, pnm1 = [to_oracle(f, g) for f in
                                 (inp.u.ux, inp.u.uy, inp.u.uz, inp.rho, inp.psi_n, inp.psi_nm1)]
    rng = np.random.default_rng(0)
    pn.a[...] = rng.standard_normal(pn.a.shape)
    pnm1.a[...] = rng.standard_normal(pn.a.shape)
    rho.a[...] = 1.0
    s = O.compute_source_fast(m, pn, pnm1, rho, ux, uy, uz, inp.dt, 1.0, 1.0)
    div = O.divergence(m, ux, uy, uz)
    assert rel_linf(s, div / inp.dt) < 1e-13


def test_alpha_tables():
    assert O.alpha_rks(0) == 1.0
    assert O.alpha_rks(1, 1) == pytest.approx(8.0 / 15.0)
    assert O.alpha_rks(1, 2) == pytest.approx(5.0 / 12.0 - 17.0 / 60.0)
    assert O.alpha_rks(1, 3) == pytest.approx(3.0 / 4.0 - 5.0 / 12.0)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "kat_*.npz"))))
def test_golden_kat(path):
    z = np.load(path)
    m = _mesh(int(z["nx"]), int(z["ny"]), int(z["nz"]), bool(z["stretched"]), float(z["gamma"]),
              (float(z["Lx"]), float(z["Ly"]), float(z["Lz"])))
    s = O.FField("cl", 1, m.nx, m.ny, m.nz, z["s"].copy())
    psi = O.FField("cl", 1, m.nx, m.ny, m.nz)
    O.solve_fps(m, s.interior(), psi)
    assert rel_linf(psi.a, z["psi_expected"]) < 1e-12


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "proj_*.npz"))))
def test_golden_projection(path):
    z = np.load(path)
    nx, ny, nz = int(z["nx"]), int(z["ny"]), int(z["nz"])
    m = _mesh(nx, ny, nz, bool(z["stretched"]), float(z["gamma"]), (float(z["Lx"]), float(z["Ly"]), float(z["Lz"])))
    hu = int(z["hd_u"])
    F = lambda kind, key, hd: O.FField(kind, hd, nx, ny, nz, z[key].copy())  # noqa: E731
    st_n = st_nm1 = None
    if "stn_x" in z:
        st_n = tuple(F(k, "stn_" + c, 1) for k, c in zip(("sx", "sy", "sz"), "xyz"))
        st_nm1 = tuple(F(k, "sto_" + c, 1) for k, c in zip(("sx", "sy", "sz"), "xyz"))
    r = O.projection(m, F("sx", "ux", hu), F("sy", "uy", hu), F("sz", "uz", hu), F("cl", "rho", 1),
                     F("cl", "psi_n", 1), F("cl", "psi_nm1", 1), float(z["dt"]), float(z["alpha"]),
                     float(z["rho0"]), st_n, st_nm1)
    assert rel_linf(r.psi.a, z["psi"]) < 1e-13
    for c in "xyz":
        assert rel_linf(getattr(r, "u" + c).a, z[f"u{c}_out"]) < 1e-14
    assert abs(r.max_div - float(z["max_div"])) < 1e-12


@pytest.mark.parametrize("path", sorted(p for p in glob.glob(os.path.join(GOLDEN, "proj_*.npz")) if "_st_" not in p))
def test_c_oracle_matches_golden(path):
    """The C/OpenMP restatement (timed CPU baseline) agrees with the numpy oracle's fixtures."""
    from oracle import cref

    cref.build()
    z = np.load(path)
    nx, ny, nz = int(z["nx"]), int(z["ny"]), int(z["nz"])
    m = _mesh(nx, ny, nz, bool(z["stretched"]), float(z["gamma"]), (float(z["Lx"]), float(z["Ly"]), float(z["Lz"])))
    ux, uy, uz = z["ux"].copy(), z["uy"].copy(), z["uz"].copy()
    psi = np.zeros_like(z["psi"])
    md = cref.projection(m, ux, uy, uz, z["rho"].copy(), z["psi_n"].copy(), z["psi_nm1"].copy(), float(z["dt"]),
                         float(z["alpha"]), float(z["rho0"]), psi, nthreads=2)
    assert rel_linf(psi, z["psi"]) < 1e-12
    hu = int(z["hd_u"])
    for c, a in zip("xyz", (ux, uy, uz)):
        f = O.FField("s" + c, hu, nx, ny, nz, a)
        g = O.FField("s" + c, hu, nx, ny, nz, z[f"u{c}_out"].copy())
        assert rel_linf(f.interior(), g.interior()) < 1e-12
    assert abs(md - float(z["max_div"])) < 1e-12
