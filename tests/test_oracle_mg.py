"""CPU tests of the MG_MODE oracle (PCG + red-black Gauss-Seidel multigrid +
direct coarsest-level solve): grid-transfer identities, the bordered coarse
solve, convergence, and agreement with the FFT path at constant density."""
import numpy as np
import pytest

from oracle import tbfp_oracle as O
from tests._helpers import mesh_of, rel_linf, to_oracle


def _mesh(nx, ny, nz, stretched=True):
    return O.Mesh(nx, ny, nz, 2 * np.pi, 2.0, np.pi, y_uniform=not stretched, gamma=1.5)


@pytest.mark.parametrize("stretched", [False, True])
def test_transfer_operators_preserve_constants(stretched):
    mf = _mesh(16, 16, 8, stretched)
    mc = O.coarse_mesh(mf)
    q = np.full((8, 16, 16), 3.25)
    assert np.allclose(O.restriction(mf, mc, q), 3.25, rtol=0, atol=1e-14)
    pc = O.FField("cl", 1, 8, 8, 4)
    pc.a[...] = -1.5
    assert np.allclose(O.prolongation(mf, mc, pc), -1.5, rtol=0, atol=1e-14)


def test_restriction_is_the_child_average_on_a_uniform_grid():
    mf = _mesh(8, 8, 4, stretched=False)
    mc = O.coarse_mesh(mf)
    rng = np.random.default_rng(0)
    q = rng.standard_normal((4, 8, 8))
    avg = q.reshape(2, 2, 4, 2, 4, 2).mean(axis=(1, 3, 5))
    assert rel_linf(O.restriction(mf, mc, q), avg) < 1e-14


def test_coarse_direct_solve_satisfies_the_bordered_system():
    m = _mesh(8, 8, 4)
    lev = O.Level(m)
    rng = np.random.default_rng(1)
    beta = O.FField("cl", 1, 8, 8, 4)
    beta.v(1, 8, 1, 8, 1, 4)[...] = 0.5 + rng.random((4, 8, 8))
    O.update_boundaries_cl_channel(beta)
    s = rng.standard_normal((4, 8, 8))
    p = O.FField("cl", 1, 8, 8, 4)
    O.coarse_direct_solve(lev, p, beta, s)
    assert abs(np.sum(p.interior())) < 1e-12 * np.max(np.abs(p.interior()))
    V = m.volume()
    lam = -np.sum(V * s) / s.size  # the Lagrange multiplier of the sum(p)=0 row
    # V*(-L p) + lam = -V*s  <=>  L p = s + lam / V
    assert rel_linf(O.apply_L(lev, p, beta), s + lam / V) < 1e-11


def _mg_case(nx, ny, nz, rhog, seed, const_rho=False):
    from tbfsolver_b200 import synth

    spec = synth.small_spec(nx, ny, nz, nbubbles=2, radius=0.3, rhog=rhog)
    inp = synth.make_inputs(spec, seed=seed)
    g = inp.grid
    m = mesh_of(g)
    ux, uy, uz, rho = [to_oracle(f, g) for f in (inp.u.ux, inp.u.uy, inp.u.uz, inp.rho)]
    if const_rho:
        rho.a[...] = 1.0
    return inp, m, ux, uy, uz, rho


@pytest.mark.parametrize("levels", [2, 3])
def test_pcg_converges_and_projects(levels):
    """solvePCG reaches tolPCG; addPressureGrad then leaves max|div u| at the
    tolerance level (pcg.f90:103-140, momentumEqn.f90:795-869)."""
    inp, m, ux, uy, uz, rho = _mg_case(32, 32, 16, 0.01, 4)
    q = O.compute_source_mg(m, ux, uy, uz)
    beta = O.compute_beta(m, rho, inp.dt, inp.alpha)
    mg = O.MGOracle(m, n_levels=levels, n_pre=2, n_post=2, tol_mg=0.4, tol_pcg=1e-10)
    p = O.FField("cl", 1, m.nx, m.ny, m.nz)
    it, res = mg.solve_pcg(p, beta, q)
    assert res <= 1e-10 and 0 < it < 100
    assert rel_linf(O.apply_L(mg.levels[0], p, beta), q) < 1e-9
    div0 = O.compute_continuity_error(m, ux, uy, uz)
    O.add_pressure_grad(m, ux, uy, uz, p, rho, inp.dt, inp.alpha)
    assert O.compute_continuity_error(m, ux, uy, uz) < 1e-8 * div0


def test_constant_density_mg_agrees_with_fft_path():
    """KAT 5: with rho == const the PCG (MG_MODE) and split-FFT (FAST_MODE)
    projections solve the same equation; pressures agree to the PCG tolerance
    once both gauges are removed, and so do the projected velocities."""
    inp, m, ux, uy, uz, rho = _mg_case(32, 16, 16, 0.01, 6, const_rho=True)
    q = O.compute_source_mg(m, ux, uy, uz)
    beta = O.compute_beta(m, rho, inp.dt, inp.alpha)
    mg = O.MGOracle(m, n_levels=3, tol_pcg=1e-12)
    p = O.FField("cl", 1, m.nx, m.ny, m.nz)
    mg.solve_pcg(p, beta, q)
    zero = O.FField("cl", 1, m.nx, m.ny, m.nz)
    r = O.projection(m, ux, uy, uz, rho, zero, zero, inp.dt, inp.alpha, 1.0)
    a = p.interior() - np.mean(p.interior())
    b = r.psi.interior() - np.mean(r.psi.interior())
    assert rel_linf(a, b) < 1e-8
    u2 = [f.copy() for f in (ux, uy, uz)]
    O.add_pressure_grad(m, *u2, p, rho, inp.dt, inp.alpha)
    for c in range(3):
        assert rel_linf(u2[c].interior(), (r.ux, r.uy, r.uz)[c].interior()) < 1e-8
