"""Generate the golden fixtures under tests/golden/ (run from the repo root):

    python tests/golden/make_golden.py

The reference (Fortran + MPI + FFTW + LAPACK + MUMPS) cannot be built in this
environment and ships no golden vectors, so the fixtures come from two sources:

* ``kat_*``  -- analytic known answers: a seeded pressure psi* is pushed through
  the discrete 7-point operator that the FFT/tridiagonal solve inverts
  (fastPoissonSolver.f90:235-273), s = L_h psi*; the expected solution is psi*
  minus its volume-weighted mean (zeroAveragePressure, :388-423).  These pin the
  solver independently of any implementation.
* ``proj_*`` -- outputs of the CPU oracle (oracle/tbfp_oracle.py, LAPACK
  zgttrf/zgttrs mode) for the third call of a seeded projection chain on small
  grids, kept as regression fixtures for both the oracle and the CUDA path.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import tbfp_oracle as O  # noqa: E402
from tbfsolver_b200 import synth  # noqa: E402


def grid_meta(spec):
    return dict(nx=spec.nx, ny=spec.ny, nz=spec.nz, Lx=spec.Lx, Ly=spec.Ly, Lz=spec.Lz,
                stretched=int(spec.y_stretched), gamma=spec.gamma)


def make_kat(name, nx, ny, nz, stretched, seed):
    m = O.Mesh(nx, ny, nz, 2 * np.pi, 2.0, np.pi, y_uniform=not stretched, gamma=1.5)
    rng = np.random.default_rng(seed)
    ps = O.FField("cl", 1, nx, ny, nz)
    ps.v(1, nx, 1, ny, 1, nz)[...] = rng.standard_normal((nz, ny, nx))
    O.update_boundaries_cl_channel(ps)
    s = O.FField("cl", 1, nx, ny, nz)
    s.v(1, nx, 1, ny, 1, nz)[...] = O.laplacian_fps(m, ps)
    ex = ps.copy()
    ex.a -= np.sum(ps.interior() * m.volume()) / m.s_Vg
    np.savez_compressed(os.path.join(HERE, name + ".npz"), s=s.a, psi_expected=ex.a,
                        nx=nx, ny=ny, nz=nz, Lx=2 * np.pi, Ly=2.0, Lz=np.pi, stretched=int(stretched), gamma=1.5)


def make_proj(name, spec, seed, with_st=False):
    inp = synth.make_inputs(spec, seed=seed, hd_u=1)
    g = inp.grid
    m = O.Mesh(g.nx, g.ny, g.nz, g.Lx, g.Ly, g.Lz, y_uniform=not g.y_stretched, gamma=g.gamma)

    def F(f):
        return O.FField(f.kind, f.hd, g.nx, g.ny, g.nz, f.a.numpy().copy())

    ux, uy, uz, rho = F(inp.u.ux), F(inp.u.uy), F(inp.u.uz), F(inp.rho)
    pn, pnm1 = F(inp.psi_n), F(inp.psi_nm1)
    st_n = st_nm1 = None
    if with_st:
        rng = np.random.default_rng(seed + 1)
        st_n = tuple(O.FField(k, 1, g.nx, g.ny, g.nz) for k in ("sx", "sy", "sz"))
        st_nm1 = tuple(O.FField(k, 1, g.nx, g.ny, g.nz) for k in ("sx", "sy", "sz"))
        for f in st_n + st_nm1:
            f.a[...] = 0.3 * rng.standard_normal(f.a.shape)
        # clean_st_prev_bc (poissonEqn.f90:419-459): the old surface-tension levels
        # are zero on the Neumann walls of psi (uy at j = lbj..lbj+hd and
        # ubj-hd..ubj), which keeps the split source compatible
        for f in (st_n[1], st_nm1[1]):
            f.v(f.lb[0], f.ub[0], -1, 0, f.lb[2], f.ub[2])[...] = 0.0
            f.v(f.lb[0], f.ub[0], g.ny, g.ny + 1, f.lb[2], f.ub[2])[...] = 0.0
        # the periodic duplicate faces are equal (equatePeriodicBC, vfield.f90:124-189)
        for lev in (st_n, st_nm1):
            O.equate_periodic_bc(lev[0], lev[2])
    for _ in range(2):  # calls 1 and 2 of the chain, then rotate the history
        r = O.projection(m, ux, uy, uz, rho, pn, pnm1, inp.dt, inp.alpha, inp.rho0, st_n, st_nm1)
        pnm1, pn = pn, r.psi
    r = O.projection(m, ux, uy, uz, rho, pn, pnm1, inp.dt, inp.alpha, inp.rho0, st_n, st_nm1)
    out = dict(ux=ux.a, uy=uy.a, uz=uz.a, rho=rho.a, psi_n=pn.a, psi_nm1=pnm1.a,
               psi=r.psi.a, ux_out=r.ux.a, uy_out=r.uy.a, uz_out=r.uz.a, s=r.s, max_div=r.max_div,
               dt=inp.dt, alpha=inp.alpha, rho0=inp.rho0, hd_u=1, **grid_meta(spec))
    if with_st:
        for c, f in zip("xyz", st_n):
            out["stn_" + c] = f.a
        for c, f in zip("xyz", st_nm1):
            out["sto_" + c] = f.a
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


if __name__ == "__main__":
    make_kat("kat_16x12x8_tanh", 16, 12, 8, True, 11)
    make_kat("kat_24x16x12_uniform", 24, 16, 12, False, 12)
    make_proj("proj_12x8x8_tanh", synth.small_spec(12, 8, 8, nbubbles=1, radius=0.45), 21)
    make_proj("proj_16x12x8_tanh", synth.small_spec(16, 12, 8, nbubbles=1, radius=0.4), 22)
    make_proj("proj_24x16x12_uniform", synth.small_spec(24, 16, 12, stretched=False, nbubbles=1, radius=0.35), 23)
    make_proj("proj_st_16x12x8_tanh", synth.small_spec(16, 12, 8, nbubbles=1, radius=0.4), 24, with_st=True)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
