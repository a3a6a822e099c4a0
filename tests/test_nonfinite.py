"""Failure detection without a GPU fault: a NaN or Inf planted in an input on
the host must come back as the hard status TBFP_ENONFINITE from every solver
entry point.  A NaN compares false against every tolerance, so an unguarded
loop would read it as converged.  The reference aborts in that case
(errorHandler.f90:30-48).  After the error the handle stays usable: the same
call on clean inputs succeeds."""
import numpy as np
import pytest
import torch

from tbfsolver_b200 import synth
from tbfsolver_b200._native import TBFP_ENONFINITE, TbfpError
from tbfsolver_b200.fields import Field, VField
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import PCG, FastPoissonSolver, PoissonEqn

pytestmark = pytest.mark.gpu


def _inputs():
    spec = synth.small_spec(64, 48, 32, nbubbles=2, radius=0.3, rhog=0.05)
    return spec, synth.make_inputs(spec, seed=9, device="cuda")


def _clone_u(u):
    return VField(*[Field.like(f, f.a.clone()) for f in u.components()])


def _poison(t: torch.Tensor, value: float, where: float = 0.37):
    flat = t.view(-1)
    flat[int(where * flat.numel())] = value


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
# (rho = Inf is not in the list: 1/rho = 0 is a finite inverse density and every
# coefficient stays finite, so there is nothing to report; rho = 0 makes 1/rho
# infinite and must be reported)
@pytest.mark.parametrize("field,value", [("ux", float("nan")), ("uz", float("inf")), ("rho", float("nan")),
                                         ("rho", 0.0), ("psi_n", float("nan"))])
def test_projection_reports_nonfinite_inputs(precision, field, value):
    spec, inp = _inputs()
    g = inp.grid
    eqn = PoissonEqn(g, spec.rhol, spec.rhog, precision=precision, tol=1e-10, max_iter=6)
    try:
        u = _clone_u(inp.u)
        rho = Field.like(inp.rho, inp.rho.a.clone())
        pn = Field.like(inp.psi_n, inp.psi_n.a.clone())
        target = {"ux": u.ux.a, "uz": u.uz.a, "rho": rho.a, "psi_n": pn.a}[field]
        _poison(target, value)
        psi = Field.like(inp.psi_n, torch.zeros_like(inp.psi_n.a))
        uo = _clone_u(inp.u)
        with pytest.raises(TbfpError) as ei:
            eqn.projection(psi, pn, inp.psi_nm1, rho, u, inp.dt, inp.alpha, u_out=uo)
        assert ei.value.code == TBFP_ENONFINITE
        # the handle and the context stay usable
        st = eqn.projection(psi, inp.psi_n, inp.psi_nm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=uo)
        assert np.isfinite(st.max_div) and st.max_div < 1e-9
    finally:
        eqn.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solve_fps_reports_a_nan_source(precision):
    g = Grid(64, 48, 32, 2 * np.pi, 2.0, np.pi, True, 1.5)
    rng = np.random.default_rng(3)
    s = Field("cl", 1, g.nx, g.ny, g.nz)
    s.interior()[...] = rng.standard_normal((g.nz, g.ny, g.nx))
    s.interior()[...] -= s.interior().mean()
    sd = Field.like(s, torch.from_numpy(s.a.copy()).cuda())
    bad = Field.like(s, sd.a.clone())
    bad.a[5, 7, 9] = float("nan")
    with FastPoissonSolver(g, precision=precision, tol=1e-10, max_iter=6) as fps:
        p = Field.like(s, torch.zeros_like(sd.a))
        with pytest.raises(TbfpError) as ei:
            fps.solve_fps(p, bad)
        assert ei.value.code == TBFP_ENONFINITE
        assert fps.solve_fps(p, sd) == 0


def test_pcg_reports_a_nan_source():
    from oracle import tbfp_oracle as O
    from tests._helpers import mesh_of, to_oracle

    spec, inp = _inputs()
    g = inp.grid
    m = mesh_of(g)
    ux, uy, uz, rho = [to_oracle(f, g) for f in (inp.u.ux, inp.u.uy, inp.u.uz, inp.rho)]
    q = O.compute_source_mg(m, ux, uy, uz)  # div u*: compatible with the Neumann walls
    beta = O.compute_beta(m, rho, inp.dt, inp.alpha)
    qf = Field("cl", 1, g.nx, g.ny, g.nz)
    qf.interior()[...] = q
    cu = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    qd = Field.like(qf, cu(qf.a))
    bd = Field.like(qf, cu(beta.a))
    bad = Field.like(qf, qd.a.clone())
    bad.a[4, 6, 8] = float("nan")
    with PCG(g, n_levels=4, tol_pcg=1e-10) as pcg:
        psi = Field.like(qf, torch.zeros_like(qd.a))
        with pytest.raises(TbfpError) as ei:
            pcg.solve_pcg(psi, bd, bad)
        assert ei.value.code == TBFP_ENONFINITE
        psi.a.zero_()
        st = pcg.solve_pcg(psi, bd, qd)
        assert st.rel_residual <= 1e-10


def test_correction_copy_wait_limit_reports_a_timeout():
    """The staged correction bounds each wait for the bulk copies of its input
    planes.  With the bound at zero cycles a copy that has not landed at the
    first look counts as late: the kernel lets its copies in flight land, ends,
    and the call returns TBFP_ETIMEOUT (not a divergence error).  With the
    default bound restored the same handle gives the same answer as before."""
    from tbfsolver_b200._native import TBFP_ETIMEOUT

    spec, inp = _inputs()
    g = inp.grid
    eqn = PoissonEqn(g, spec.rhol, spec.rhog)

    def run():
        psi = Field.like(inp.psi_n, torch.zeros_like(inp.psi_n.a))
        uo = VField(*[Field.like(f, torch.zeros_like(f.a)) for f in inp.u.components()])
        st = eqn.projection(psi, inp.psi_n, inp.psi_nm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=uo)
        return [psi.a.clone()] + [f.a.clone() for f in uo.components()], st.max_div

    try:
        want, md = run()
        eqn.solver.set_wait_limit(0)
        with pytest.raises(TbfpError) as ei:
            run()
        assert ei.value.code == TBFP_ETIMEOUT
        eqn.solver.set_wait_limit(4_000_000_000)
        got, md2 = run()
        assert md2 == md
        for a, b in zip(want, got):
            assert torch.equal(a, b)
        with pytest.raises(TbfpError):
            eqn.solver.set_wait_limit(-1)
    finally:
        eqn.close()
