"""Mixed precision (TBFP_MIXED): FP32 spectrum transforms with FP64 defect
correction, through the C ABI, against the FP64 path (itself held to the
oracle by test_gpu_parity.py).

Bar: the refined solve stops at ||s - L psi||_2/||s||_2 <= tol (1e-10 here,
the target of the mixed path) within a few sweeps, and its pressure agrees with
the FP64 direct solve to the accuracy that residual implies (1e-8 relative,
L-infinity); the projected velocity keeps max|div u| at the FP64 level of the
residual (1e-8 of the source's scale).
"""
import numpy as np
import pytest
import torch

from tbfsolver_b200 import synth
from tbfsolver_b200._native import TBFP_ENOTCONVERGED
from tbfsolver_b200.fields import Field, VField
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import FastPoissonSolver, PoissonEqn
from tests._helpers import mesh_of, rel_linf

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _cuda(f: Field) -> Field:
    return Field.like(f, torch.from_numpy(np.ascontiguousarray(f.a)).to("cuda"))


def _rhs(g: Grid, seed: int, compatible: bool = True) -> Field:
    m = mesh_of(g)
    rng = np.random.default_rng(seed)
    s = Field("cl", 1, g.nx, g.ny, g.nz)
    s.interior()[...] = rng.standard_normal((g.nz, g.ny, g.nx))
    if compatible:
        s.interior()[...] -= np.sum(s.interior() * m.volume()) / m.s_Vg
    else:
        s.interior()[...] += 1.0
    return s


def _solve(g, s, **kw):
    with FastPoissonSolver(g, **kw) as fps:
        p = _cuda(Field("cl", 1, g.nx, g.ny, g.nz))
        rc = fps.solve_fps(p, _cuda(s))
        st = fps.last_stats()
        return rc, st, p.a.cpu().numpy()


@pytest.mark.parametrize("dims,stretched", [((64, 48, 32), True), ((96, 64, 48), False), ((128, 96, 64), True),
                                            ((48, 100, 24), True)])
def test_mixed_solve_reaches_tolerance(dims, stretched):
    g = Grid(*dims, 2 * np.pi, 2.0, np.pi, stretched, 1.5)
    s = _rhs(g, sum(dims))
    rc, st, p_mixed = _solve(g, s, precision="mixed", tol=TOL, max_iter=8)
    assert rc == 0 and st.rel_residual <= TOL and 2 <= st.iterations <= 4, (rc, st.rel_residual, st.iterations)
    rc64, st64, p64 = _solve(g, s, residual=True)
    assert rc64 == 0 and st64.iterations == 1 and 0 <= st64.rel_residual < 1e-13
    assert rel_linf(p_mixed, p64) < 1e-8


def test_mixed_incompatible_rhs_matches_the_fp64_system():
    """The residual of the mixed path is that of the system the FP64 path
    solves, so a source with a non-zero volume integral still converges to the
    FP64 answer (the defect on the top wall)."""
    g = Grid(32, 24, 16, 2 * np.pi, 2.0, np.pi, True, 1.5)
    s = _rhs(g, 5, compatible=False)
    rc, st, p_mixed = _solve(g, s, precision="mixed", tol=TOL, max_iter=8)
    assert rc == 0 and st.rel_residual <= TOL
    _, st64, p64 = _solve(g, s, residual=True)
    assert st64.rel_residual < 1e-12
    assert rel_linf(p_mixed, p64) < 1e-8


def test_mixed_iteration_cap_is_a_soft_status():
    g = Grid(64, 48, 32, 2 * np.pi, 2.0, np.pi, True, 1.5)
    s = _rhs(g, 9)
    rc, st, _ = _solve(g, s, precision="mixed", tol=1e-30, max_iter=2)
    assert rc == TBFP_ENOTCONVERGED and st.iterations == 2 and st.rel_residual > 0.0


def test_mixed_long_run_keeps_its_residual():
    """An unreachable tolerance with a long cap: every sweep's residual is
    summed afresh, so after many sweeps the reported residual stays at the
    FP64 floor (it must not grow with the sweep count)."""
    g = Grid(64, 48, 32, 2 * np.pi, 2.0, np.pi, True, 1.5)
    s = _rhs(g, 12)
    rc5, st5, p5 = _solve(g, s, precision="mixed", tol=1e-30, max_iter=5)
    rc, st, p = _solve(g, s, precision="mixed", tol=1e-30, max_iter=70)
    assert rc5 == rc == TBFP_ENOTCONVERGED and st.iterations == 70
    assert 0.0 < st.rel_residual < 1e-13 and st.rel_residual < 10 * st5.rel_residual
    assert rel_linf(p, p5) < 1e-12


def test_mixed_projection_matches_fp64():
    spec = synth.small_spec(64, 48, 32, nbubbles=3, radius=0.3, rhog=0.02)
    inp = synth.make_inputs(spec, seed=3, device="cuda")
    g = inp.grid
    out = {}
    for prec in ("fp64", "mixed"):
        eqn = PoissonEqn(g, spec.rhol, spec.rhog, precision=prec, tol=TOL, max_iter=8)
        psi = Field.like(inp.psi_n, torch.zeros_like(inp.psi_n.a))
        u_out = VField(*[Field.like(f, f.a.clone()) for f in inp.u.components()])  # same halos in both runs
        st = eqn.projection(psi, inp.psi_n, inp.psi_nm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=u_out)
        out[prec] = (st, psi.a.cpu().numpy(), [f.a.cpu().numpy() for f in u_out.components()])
        eqn.close()
    st64, p64, u64 = out["fp64"]
    stm, pm, um = out["mixed"]
    assert stm.rel_residual <= TOL and stm.iterations >= 2
    assert rel_linf(pm, p64) < 1e-8
    for a, b in zip(um, u64):
        assert rel_linf(a, b) < 1e-9
    # the loop also stops on the divergence: max|div u| <= tol, as the FP64 path
    assert stm.max_div <= TOL, stm.max_div


def test_mixed_projection_asynchronous_and_stats_later():
    """Without stats an asynchronous handle does not read the loop's outcome
    back; the result is the same as a synchronous call's to 1e-11 (not bit for
    bit: the residual sums are atomics in no fixed order)."""
    spec = synth.small_spec(64, 48, 32, nbubbles=3, radius=0.3, rhog=0.02)
    inp = synth.make_inputs(spec, seed=4, device="cuda")
    g = inp.grid
    res = []
    for asyn in (False, True):
        eqn = PoissonEqn(g, spec.rhol, spec.rhog, precision="mixed", tol=TOL, max_iter=8, asynchronous=asyn)
        psi = Field.like(inp.psi_n, torch.zeros_like(inp.psi_n.a))
        u_out = VField(*[Field.like(f, f.a.clone()) for f in inp.u.components()])
        for _ in range(2):  # the second call replays the cached refinement graph
            eqn.projection(psi, inp.psi_n, inp.psi_nm1, inp.rho, inp.u, inp.dt, inp.alpha, u_out=u_out,
                           want_stats=False)
        torch.cuda.synchronize()
        res.append(psi.a.cpu().numpy())
        eqn.close()
    assert rel_linf(res[1], res[0]) < 1e-11
