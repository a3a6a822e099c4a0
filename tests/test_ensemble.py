"""The ensemble entry point (tbfp_ensemble_*): several channels of different
sizes projected in one call, through the C ABI, against one projection per
channel with the single-channel entry point.  The kernels are the same, so
the FP64 results must agree bit for bit, on the first call (graph capture),
on a replay, and after the arrays change (re-capture).  A mixed-precision
ensemble runs inside the same captured graph, each member's refinement loop a
conditional node on the device; it must reach its residual and divergence
targets on the first call and on replays, and agree with single-channel mixed
calls to 1e-11, well inside the mixed path's own 1e-8 bar against FP64.  They
do not agree bit for bit: the residual passes sum with atomics in no fixed
order, and the sum of s dyf sets the top-wall term of the residual.)"""
import numpy as np
import pytest
import torch

from tbfsolver_b200 import synth
from tbfsolver_b200.fields import Field, VField
from tbfsolver_b200.solver import Ensemble, PoissonEqn

pytestmark = pytest.mark.gpu


def _members(specs, seed):
    out = []
    for c, spec in enumerate(specs):
        inp = synth.make_inputs(spec, seed=seed + c, device="cuda")
        # psi^n from one projection of the chain, so the split term is active
        eqn = PoissonEqn(inp.grid, spec.rhol, spec.rhog)
        psi1, pn, pnm1, rho, u, uo = _io(inp)
        eqn.projection(psi1, pn, pnm1, rho, u, inp.dt, inp.alpha, u_out=uo)
        eqn.close()
        inp.psi_n = psi1
        out.append(inp)
    return out


def _io(inp):
    psi = Field.like(inp.psi_n, torch.zeros_like(inp.psi_n.a))
    uo = VField(*[Field.like(f, f.a.clone()) for f in inp.u.components()])
    return (psi, inp.psi_n, inp.psi_nm1, inp.rho, inp.u, uo)


def _reference(inp, rho0):
    eqn = PoissonEqn(inp.grid, inp.spec.rhol, inp.spec.rhog)
    psi, pn, pnm1, rho, u, uo = _io(inp)
    st = eqn.projection(psi, pn, pnm1, rho, u, inp.dt, inp.alpha, u_out=uo)
    eqn.close()
    return st, psi, uo


def test_ensemble_matches_single_channel_projections():
    specs = [synth.small_spec(64, 48, 32, nbubbles=2, rhog=0.05), synth.small_spec(48, 40, 24, nbubbles=1, rhog=0.05),
             synth.small_spec(96, 64, 48, nbubbles=3, rhog=0.05)]
    inps = _members(specs, 11)
    rho0 = 0.05
    with Ensemble([i.grid for i in inps], nstreams=2, mode="graph") as ens:
        for rep in range(3):
            if rep == 2:  # new arrays: the graph is captured again
                inps = _members(specs, 21)
            members = [_io(i) for i in inps]
            stats = ens.projection(members, inps[0].dt, inps[0].alpha, rho0)
            for inp, m, st in zip(inps, members, stats):
                want_st, want_psi, want_u = _reference(inp, rho0)
                assert torch.equal(m[0].a, want_psi.a)
                for a, b in zip(m[5].components(), want_u.components()):
                    assert torch.equal(a.a, b.a)
                assert st.max_div == want_st.max_div and st.max_div < 1e-9


def _reference_mixed(inp, rho0):
    eqn = PoissonEqn(inp.grid, inp.spec.rhol, inp.spec.rhog, precision="mixed", tol=1e-10, max_iter=8)
    psi, pn, pnm1, rho, u, uo = _io(inp)
    st = eqn.projection(psi, pn, pnm1, rho, u, inp.dt, inp.alpha, u_out=uo)
    eqn.close()
    return st, psi, uo


def test_mixed_ensemble_reaches_tolerance():
    specs = [synth.small_spec(64, 48, 32, nbubbles=2, rhog=0.05), synth.small_spec(48, 40, 24, nbubbles=1, rhog=0.05),
             synth.small_spec(96, 64, 48, nbubbles=3, rhog=0.05)]
    inps = _members(specs, 5)
    with Ensemble([i.grid for i in inps], nstreams=2, precision="mixed", tol=1e-10) as ens:
        members = [_io(i) for i in inps]
        for rep in range(3):  # capture, then replays of the graph with its conditional loops
            for m in members:
                m[0].a.zero_()
            stats = ens.projection(members, inps[0].dt, inps[0].alpha, 0.05)
            for inp, m, st in zip(inps, members, stats):
                assert st.rel_residual <= 1e-10 and st.iterations >= 2 and st.max_div <= 1e-10, (rep, st.iterations)
                want_st, want_psi, want_u = _reference_mixed(inp, 0.05)
                assert st.iterations == want_st.iterations
                a, b = m[0].a.cpu().numpy(), want_psi.a.cpu().numpy()
                assert np.max(np.abs(a - b)) / np.max(np.abs(b)) < 1e-11
                _, p64, _ = _reference(inp, 0.05)
                c = p64.a.cpu().numpy()
                assert np.max(np.abs(a - c)) / np.max(np.abs(c)) < 1e-8


def _specs_small():
    return [synth.small_spec(64, 48, 32, nbubbles=2, rhog=0.05), synth.small_spec(48, 40, 24, nbubbles=1, rhog=0.05),
            synth.small_spec(96, 64, 48, nbubbles=3, rhog=0.05), synth.small_spec(128, 96, 64, nbubbles=2, rhog=0.05)]


def _close(a, b, tol=1e-12):
    a, b = a.detach().cpu().numpy(), b.detach().cpu().numpy()
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) < tol


def test_persistent_form_matches_single_channel_projections():
    """One persistent launch (a device work queue over (member, stage, tile))
    runs the same tile bodies as the standalone kernels, inlined into another
    kernel: the compiler may contract and order the arithmetic differently, so
    the results agree with the single-channel ones to rounding (the 1e-12
    parity bar), on the first call, on a replay and after the arrays change."""
    specs = _specs_small()
    inps = _members(specs, 31)
    with Ensemble([i.grid for i in inps], nstreams=2, mode="persistent") as ens:
        for rep in range(3):
            if rep == 2:
                inps = _members(specs, 41)
            members = [_io(i) for i in inps]
            stats = ens.projection(members, inps[0].dt, inps[0].alpha, 0.05)
            assert ens.mode()[0] == "persistent"
            for inp, m, st in zip(inps, members, stats):
                want_st, want_psi, want_u = _reference(inp, 0.05)
                assert _close(m[0].a, want_psi.a)
                for a, b in zip(m[5].components(), want_u.components()):
                    assert _close(Field.like(a, a.a).interior(), Field.like(b, b.a).interior())
                assert abs(st.max_div - want_st.max_div) < 1e-12 and st.max_div < 1e-9


def test_auto_form_is_measured_once_and_cached(tmp_path, monkeypatch):
    cache = tmp_path / "tune.txt"
    monkeypatch.setenv("TBFP_TUNE_CACHE", str(cache))
    specs = _specs_small()
    inps = _members(specs, 51)
    members = [_io(i) for i in inps]
    with Ensemble([i.grid for i in inps], nstreams=2) as ens:
        ens.projection(members, inps[0].dt, inps[0].alpha, 0.05)
        form, param, ms = ens.mode()
    assert form in ("graph", "persistent") and ms[0] > 0 and ms[1] > 0
    lines = cache.read_text().split()
    assert len(lines) == 4 and int(lines[1]) == {"graph": 1, "persistent": 2}[form]
    with Ensemble([i.grid for i in inps], nstreams=2) as ens2:  # same sizes: the choice is read back
        stats = ens2.projection(members, inps[0].dt, inps[0].alpha, 0.05)
        f2, p2, ms2 = ens2.mode()
    assert (f2, p2) == (form, param) and ms2 == [-1.0, -1.0, -1.0]
    for inp, m, st in zip(inps, members, stats):
        _, want_psi, _ = _reference(inp, 0.05)
        assert _close(m[0].a, want_psi.a)


def test_persistent_wait_limit_reports_a_timeout():
    """Failure detection without a fault: with a zero poll budget the first
    dependency wait of the persistent kernel runs out, the launch stops and the
    call returns TBFP_ETIMEOUT; with the budget restored the same ensemble
    projects correctly."""
    from tbfsolver_b200._native import TBFP_ETIMEOUT, TbfpError

    specs = _specs_small()
    inps = _members(specs, 61)
    members = [_io(i) for i in inps]
    with Ensemble([i.grid for i in inps], nstreams=2, mode="persistent") as ens:
        ens.set_wait_limit(0)
        with pytest.raises(TbfpError) as ei:
            ens.projection(members, inps[0].dt, inps[0].alpha, 0.05)
        assert ei.value.code == TBFP_ETIMEOUT
        ens.set_wait_limit(10_000_000)
        stats = ens.projection(members, inps[0].dt, inps[0].alpha, 0.05)
        for inp, m, st in zip(inps, members, stats):
            _, want_psi, _ = _reference(inp, 0.05)
            assert _close(m[0].a, want_psi.a)


def test_persistent_form_needs_out_of_place_members():
    from tbfsolver_b200._native import TBFP_EUNSUPPORTED, TbfpError

    specs = _specs_small()[:2]
    inps = _members(specs, 71)
    members = [(psi, pn, pnm1, rho, u, u) for (psi, pn, pnm1, rho, u, _) in (_io(i) for i in inps)]
    with Ensemble([i.grid for i in inps], nstreams=2, mode="persistent") as ens:
        with pytest.raises(TbfpError) as ei:
            ens.projection(members, inps[0].dt, inps[0].alpha, 0.05)
        assert ei.value.code == TBFP_EUNSUPPORTED
