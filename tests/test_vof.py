"""Material properties from the volume fraction (updateMaterialProps with
smoothVF, VOF.f90:197-262): the oracle pinned by known answers on the CPU,
and the CUDA path (tbfp_material_props) against the oracle on the GPU."""
import numpy as np
import pytest
import torch

from oracle import tbfp_oracle as O
from tbfsolver_b200 import synth
from tbfsolver_b200.fields import Field
from tbfsolver_b200.grid import Grid
from tbfsolver_b200.solver import VOF, FastPoissonSolver
from tests._helpers import mesh_of, rel_linf

PROPS = dict(rhol=1.0, rhog=0.02, mul=1e-3, mug=2e-5)


def _vf(nx, ny, nz, stretched, seed, nbub=3):
    spec = synth.small_spec(nx, ny, nz, stretched=stretched, nbubbles=nbub, radius=0.3)
    c = synth.vof_field(spec, synth.bubble_centres(spec, seed), device="cpu", hd=1)
    return spec.grid(), c.numpy().copy()


# --- oracle known answers (CPU) ---------------------------------------------
def test_constant_fraction_is_kept_and_sets_the_phase_properties():
    g = Grid(16, 12, 8, 2 * np.pi, 2.0, np.pi, True, 1.5)
    m = mesh_of(g)
    for v in (0.0, 1.0, 0.3):
        c = O.FField("cl", 1, 16, 12, 8, np.full((10, 14, 18), v))
        cs, rho, mu = O.update_material_props(m, c, **PROPS)
        assert np.allclose(cs.a, v, rtol=0, atol=1e-15)
        assert np.allclose(rho.a, PROPS["rhog"] * v + (1 - v) * PROPS["rhol"], rtol=1e-13, atol=0)
        assert np.allclose(mu.a, PROPS["mug"] * v + (1 - v) * PROPS["mul"], rtol=1e-13, atol=1e-18)


@pytest.mark.parametrize("stretched", [True, False])
def test_smoothing_reproduces_a_field_linear_in_y_away_from_the_walls(stretched):
    """Trilinear interpolation is exact for linear functions: two passes keep
    c = a + b*yc on cells whose stencils stay off the wall ghosts (j = 3..ny-2)."""
    nx, ny, nz = 12, 20, 8
    g = Grid(nx, ny, nz, 2 * np.pi, 2.0, np.pi, stretched, 1.5)
    m = mesh_of(g)
    c = O.FField("cl", 1, nx, ny, nz)
    yc = m.yc.r(0, ny + 1)
    c.a[...] = 0.25 + 0.3 * yc[None, :, None]
    O.update_boundaries_cl_channel(c)
    cs = O.smooth_vf(m, c)
    got = cs.v(1, nx, 3, ny - 2, 1, nz)
    want = c.v(1, nx, 3, ny - 2, 1, nz)
    assert np.max(np.abs(got - want)) < 1e-14


def test_oracle_matches_the_input_generator():
    """The seeded inputs smooth their volume fraction with a torch restatement
    of the same routines; the two agree bit for bit."""
    g, c = _vf(32, 24, 16, True, 3)
    cs_t = synth.smooth_vf(torch.from_numpy(c), g, 1).numpy()
    cs_o = O.smooth_vf(mesh_of(g), O.FField("cl", 1, 32, 24, 16, c.copy()))
    assert np.array_equal(cs_o.a, cs_t)


# --- CUDA path vs oracle (GPU) ---------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("dims,stretched", [((32, 24, 16), True), ((64, 48, 32), False), ((48, 40, 24), True)])
@pytest.mark.parametrize("where", ["host", "device"])
def test_material_props_match_the_oracle(dims, stretched, where):
    nx, ny, nz = dims
    g, c = _vf(nx, ny, nz, stretched, nx + ny)
    cs_o, rho_o, mu_o = O.update_material_props(mesh_of(g), O.FField("cl", 1, nx, ny, nz, c.copy()), **PROPS)
    with FastPoissonSolver(g) as fps:
        vof = VOF(fps, **PROPS)
        mk = (lambda a: torch.from_numpy(a).cuda()) if where == "device" else (lambda a: a)  # noqa: E731
        fc = Field("cl", 1, nx, ny, nz, mk(c.copy()))
        outs = [Field("cl", 1, nx, ny, nz, mk(np.zeros_like(c))) for _ in range(3)]
        vof.update_material_props(fc, *outs)
        got = [o.a.cpu().numpy() if where == "device" else o.a for o in outs]
    for a, b in zip(got, (cs_o.a, rho_o.a, mu_o.a)):
        assert rel_linf(a, b) < 1e-14


@pytest.mark.gpu
def test_material_props_feed_the_projection_inputs():
    """rho from tbfp_material_props is the rho the seeded projection inputs use."""
    spec = synth.small_spec(64, 48, 32, nbubbles=4, radius=0.3, rhog=0.05)
    inp = synth.make_inputs(spec, seed=11, device="cuda")
    g = inp.grid
    c = synth.vof_field(spec, synth.bubble_centres(spec, 11), device="cuda", hd=1)
    with FastPoissonSolver(g) as fps:
        vof = VOF(fps, rhol=spec.rhol, rhog=spec.rhog, mul=1e-3, mug=1e-5)
        cs, rho, mu = (Field("cl", 1, g.nx, g.ny, g.nz, torch.zeros_like(c)) for _ in range(3))
        vof.update_material_props(Field("cl", 1, g.nx, g.ny, g.nz, c), cs, rho, mu)
    assert rel_linf(cs.a.cpu().numpy(), inp.cs.a.cpu().numpy()) < 1e-14
    assert rel_linf(rho.a.cpu().numpy(), inp.rho.a.cpu().numpy()) < 1e-14


@pytest.mark.gpu
def test_material_props_errors():
    g = Grid(16, 12, 8, 2 * np.pi, 2.0, np.pi, True, 1.5)
    with FastPoissonSolver(g) as fps:
        f = Field("cl", 1, 16, 12, 8, torch.zeros((10, 14, 18), dtype=torch.float64, device="cuda"))
        rc = fps.lib.tbfp_material_props_dev(fps.h, f.address(), f.address(), f.address(), f.address())
        assert rc < 0  # no tbfp_vof_setup yet
        VOF(fps, **PROPS)
        rc = fps.lib.tbfp_material_props_dev(fps.h, f.address(), f.address(), f.address(), f.address())
        assert rc < 0  # aliased outputs
