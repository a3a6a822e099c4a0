"""CPU tests of the host-side logic: grid set-up, field layout, synthetic
inputs.  No GPU needed."""
import numpy as np
import pytest
import torch

from oracle import tbfp_oracle as O
from tbfsolver_b200 import synth
from tbfsolver_b200.fields import Field, field_shape
from tbfsolver_b200.grid import Grid


@pytest.mark.parametrize("stretched", [False, True])
def test_grid_matches_oracle_bitwise(stretched):
    g = Grid(48, 40, 24, 2 * np.pi, 2.0, np.pi, y_stretched=stretched, gamma=1.5)
    m = O.Mesh(48, 40, 24, 2 * np.pi, 2.0, np.pi, y_uniform=not stretched, gamma=1.5)
    for name in ("xc", "yc", "zc", "xf", "yf", "zf", "dxc", "dyc", "dzc", "dxf", "dyf", "dzf"):
        a, b = getattr(g, name), getattr(m, name)
        assert a.lb == b.lb and np.array_equal(a.v, b.v), name
    assert g.s_Vg == m.s_Vg
    assert g.dx_fft == m.xc[2] - m.xc[1]


def test_total_volume_is_sequential_sum():
    g = Grid(8, 6, 4, 1.0, 2.0, 3.0, y_stretched=True, gamma=1.5)
    s = 0.0
    for k in range(1, 5):
        for j in range(1, 7):
            for i in range(1, 9):
                s += g.dxf[i] * g.dyf[j] * g.dzf[k]
    assert g.s_Vg == s
    assert abs(s - 6.0) < 1e-13


def test_tanh_grid_is_symmetric_and_stretched():
    g = Grid(8, 64, 4, 1.0, 2.0, 1.0, y_stretched=True, gamma=1.5)
    yf = g.yf.r(0, 64)
    assert abs(yf[0]) < 1e-15 and abs(yf[-1] - 2.0) < 1e-14
    dy = np.diff(yf)
    assert np.allclose(dy, dy[::-1], rtol=1e-12, atol=1e-15)
    assert dy[0] < dy[32] / 3.0


@pytest.mark.parametrize("kind,lo", [("cl", (1, 1, 1)), ("sx", (0, 1, 1)), ("sy", (1, 0, 1)), ("sz", (1, 1, 0))])
def test_field_layout_is_fortran_column_major(kind, lo):
    nx, ny, nz, hd = 5, 4, 3, 2
    f = Field(kind, hd, nx, ny, nz)
    assert f.a.shape == field_shape(kind, hd, nx, ny, nz)
    # element (i,j,k) at offset (i-ilo) + (j-jlo)*ni + (k-klo)*ni*nj
    ni, nj = f.a.shape[2], f.a.shape[1]
    i, j, k = 2, 3, 1
    f.v(i, i, j, j, k, k)[...] = 7.0
    off = (i - (lo[0] - hd)) + (j - (lo[1] - hd)) * ni + (k - (lo[2] - hd)) * ni * nj
    assert f.a.reshape(-1)[off] == 7.0


def test_splitmix_torch_matches_numpy():
    idx = np.arange(100000, dtype=np.uint64) ^ (np.uint64(77) << np.uint64(44))
    ref = synth.splitmix64_numpy(idx)
    t = synth.splitmix64(torch.from_numpy(idx.astype(np.int64)))
    assert np.array_equal(t.numpy().view(np.uint64), ref)
    u = synth.uniform01(77, 0, 1000, "cpu")
    assert float(u.min()) >= 0.0 and float(u.max()) < 1.0


def test_synthetic_inputs_follow_the_recipe():
    spec = synth.small_spec(32, 24, 16, nbubbles=2, radius=0.3, rhog=0.05)
    inp = synth.make_inputs(spec, seed=3)
    g = inp.grid
    cs = inp.cs.interior()
    assert float(cs.min()) >= 0.0 and float(cs.max()) <= 1.0 and float(cs.max()) > 0.2
    rho = inp.rho.a
    assert float(rho.min()) >= spec.rhog - 1e-15 and float(rho.max()) <= spec.rhol + 1e-15
    ux, uy, uz = inp.u.ux, inp.u.uy, inp.u.uz
    # walls, periodic duplicates
    assert float(uy.v(1, g.nx, 0, 0, 1, g.nz).abs().max()) == 0.0
    assert float(uy.v(1, g.nx, g.ny, g.ny, 1, g.nz).abs().max()) == 0.0
    assert torch.equal(ux.v(0, 0, 1, g.ny, 1, g.nz), ux.v(g.nx, g.nx, 1, g.ny, 1, g.nz))
    assert torch.equal(uz.v(1, g.nx, 1, g.ny, 0, 0), uz.v(1, g.nx, 1, g.ny, g.nz, g.nz))
    # bulk (dy-weighted) velocity of the Poiseuille profile ~ 1
    w = torch.from_numpy(g.dyf.r(1, g.ny))[None, :, None]
    ub = float((ux.v(1, g.nx, 1, g.ny, 1, g.nz) * w).sum() / (w.sum() * g.nx * g.nz))
    assert abs(ub - 1.0) < 0.02
    # deterministic
    inp2 = synth.make_inputs(spec, seed=3)
    assert torch.equal(inp2.rho.a, inp.rho.a) and torch.equal(inp2.u.uz.a, uz.a)


def test_update_boundaries_matches_oracle():
    nx, ny, nz = 6, 5, 4
    rng = np.random.default_rng(1)
    a = rng.standard_normal(field_shape("cl", 1, nx, ny, nz))
    f = O.FField("cl", 1, nx, ny, nz, a.copy())
    O.update_boundaries_cl_channel(f)
    t = torch.from_numpy(a.copy())
    synth.update_boundaries_cl(t, 1, nx, ny, nz)
    assert np.array_equal(t.numpy(), f.a)


def test_bubble_volume_close_to_sphere():
    spec = synth.small_spec(64, 64, 32, stretched=False, nbubbles=1, radius=0.4)
    cen = synth.bubble_centres(spec, 1)
    c = synth.vof_field(spec, cen, hd=1)
    g = spec.grid()
    V = float((torch.from_numpy(g.dxf.r(1, 64))[None, None, :] * torch.from_numpy(g.dyf.r(1, 64))[None, :, None]
               * torch.from_numpy(g.dzf.r(1, 32))[:, None, None] * c[1:-1, 1:-1, 1:-1]).sum())
    assert abs(V - 4.0 / 3.0 * np.pi * 0.4 ** 3) / (4.0 / 3.0 * np.pi * 0.4 ** 3) < 2e-3
