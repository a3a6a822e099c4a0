"""Python mirror of the reference's projection-step interface over the C ABI.

Names and argument meaning follow the Fortran modules they replace:

* ``FastPoissonSolver``  -- fastPoissonSolverMod (src/fastPoissonSolver/fastPoissonSolver.f90):
  ``FastPoissonSolver(mesh)`` is fastPoissonSolverCTOR (:123), ``solve_fps(p, s)`` is solveFPS (:337).
* ``PoissonEqn``         -- poissonEqnMod in FAST_MODE (src/poissonEqn/poissonEqn.f90):
  ``compute_source`` (:193), ``solve_poisson_eqn`` (:347), ``update_pressure`` (:374).
* ``make_velocity_div_free`` -- momentumEqn.f90:999 (FAST_MODE).
* ``compute_continuity_error`` -- auxiliaryRoutines.f90:42 (returns the value
  instead of printing it).
* ``Ensemble``           -- many independent channels per GPU in one call (no
  counterpart in the reference, which runs one channel per job).
* ``PCG``                -- pcgMod (src/pcg/pcg.f90) with its multigrid preconditioner
  (multiGridMod, rbgsMod, poissMatMod): ``PCG(mesh, ...)`` is pcgCTOR (:62),
  ``solve_pcg(psi, beta, q)`` is solvePCG (:103).
* ``VOF``                -- the VOF type's material properties (src/VOF/VOF.f90:197-262).
* ``MomentumEqn``        -- momentumEqnMod in FAST_MODE (src/momentumEqn/momentumEqn.f90):
  ``solve`` is solveMomentumEqn (:161) with updateBoundariesV (vfield.f90:111),
  ``write_old_time_flux`` / ``read_old_time_flux`` are printOldTimeFlux /
  initOldTimeFlux (:1254-1290).
* ``FlowControl``        -- setPressGrad, computeFlowRate, setFlowRate
  (src/auxiliaryRoutines/auxiliaryRoutines.f90:336-546).
* ``fast_substep``       -- one Runge-Kutta substep of tph_flow_solver (src/main.f90:177-209)
  after the VOF advection.

The reference's old time levels ``psi%ptrf_`` and ``psi%ptrf_%ptrf_`` are
passed explicitly as ``psi_n`` and ``psi_nm1``; the surface-tension old levels
as ``st_n``/``st_nm1`` triples (or None for zero surface tension).  Errors the
reference turns into mpiABORT raise ``TbfpError``; soft conditions are returned.

Fields holding numpy arrays go through the host entry points (copies in and
out); fields holding CUDA tensors go through the ``*_dev`` entry points.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import (TBFP_EINVAL, TBFP_FLAG_ASYNC, TBFP_FLAG_RESIDUAL, TBFP_FLAG_TIMING, TBFP_FP64, TBFP_MIXED,
                      TbfpDesc, TbfpError, TbfpMemberIO, TbfpMgParams, TbfpStats,
                      TbfpMomentumDesc, TbfpVofDesc, check, load)
from .fields import Field, VField
from .grid import Grid


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _placement(fields) -> bool:
    """True if every field is on a CUDA device, False if every one is on the host."""
    flags = {f.on_cuda for f in fields if f is not None}
    if len(flags) != 1:
        raise TbfpError(TBFP_EINVAL, "fields must all live on the host or all on the device")
    return flags.pop()


class _PtrTriple:
    """A ``const double *const[3]`` argument kept alive for one call."""

    def __init__(self, st):
        if st is None:
            self.arr = None
            self.addr = None
        else:
            if len(st) != 3:
                raise ValueError("surface tension must be a (x, y, z) triple of fields")
            self.arr = (C.c_void_p * 3)(*[f.address() for f in st])
            self.addr = C.cast(self.arr, C.c_void_p).value


def _metrics(mesh: Grid) -> dict:
    nx, ny, nz = mesh.nx, mesh.ny, mesh.nz
    return {
        "dxf": np.ascontiguousarray(mesh.dxf.r(1, nx)), "dxc": np.ascontiguousarray(mesh.dxc.r(1, nx + 1)),
        "dyf": np.ascontiguousarray(mesh.dyf.r(1, ny)), "dyc": np.ascontiguousarray(mesh.dyc.r(1, ny + 1)),
        "dzf": np.ascontiguousarray(mesh.dzf.r(1, nz)), "dzc": np.ascontiguousarray(mesh.dzc.r(1, nz + 1)),
    }


def _desc(mesh: Grid, m: dict, hd_psi, hd_u, hd_rho, hd_st, precision, tol, max_iter, device, stream, flags):
    prec = {"fp64": TBFP_FP64, "mixed": TBFP_MIXED}[precision]
    return TbfpDesc(nx=mesh.nx, ny=mesh.ny, nz=mesh.nz, hd_psi=hd_psi, hd_u=hd_u, hd_rho=hd_rho, hd_st=hd_st,
                    dx_fft=mesh.dx_fft, dz_fft=mesh.dz_fft, dxf=_dptr(m["dxf"]), dxc=_dptr(m["dxc"]),
                    dyf=_dptr(m["dyf"]), dyc=_dptr(m["dyc"]), dzf=_dptr(m["dzf"]), dzc=_dptr(m["dzc"]),
                    s_Vg=mesh.s_Vg, precision=prec, tol=tol, max_iter=max_iter, device=device, stream=stream,
                    flags=flags)


class FastPoissonSolver:
    """The split-constant-coefficient direct Poisson solver on one GPU."""

    def __init__(self, mesh: Grid, hd_psi: int = 1, hd_u: int = 2, hd_rho: int = 1, hd_st: int = 1,
                 precision: str = "fp64", tol: float = 1e-10, max_iter: int = 8, device: int = -1,
                 stream: int | None = None, asynchronous: bool = False, timing: bool = False,
                 residual: bool = False):
        self.lib = load()
        self.mesh = mesh
        self.hd_psi, self.hd_u, self.hd_rho, self.hd_st = hd_psi, hd_u, hd_rho, hd_st
        # keep the metric arrays alive while the descriptor is read
        self._m = _metrics(mesh)
        d = _desc(mesh, self._m, hd_psi, hd_u, hd_rho, hd_st, precision, tol, max_iter, device, stream,
                  (TBFP_FLAG_ASYNC if asynchronous else 0) | (TBFP_FLAG_TIMING if timing else 0)
                  | (TBFP_FLAG_RESIDUAL if residual else 0))
        h = C.c_void_p()
        check(self.lib.tbfp_create(C.byref(d), C.byref(h)), None)
        self.h = h

    # --- lifecycle -------------------------------------------------------
    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.tbfp_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass

    @property
    def device_bytes(self) -> int:
        return int(self.lib.tbfp_device_bytes(self.h))

    # --- fields ----------------------------------------------------------
    def new_field(self, kind: str, hd: int | None = None) -> Field:
        m = self.mesh
        if hd is None:
            hd = {"cl": self.hd_psi, "sx": self.hd_u, "sy": self.hd_u, "sz": self.hd_u}[kind]
        return Field(kind, hd, m.nx, m.ny, m.nz)

    def _check_psi(self, *fs):
        for f in fs:
            if f.kind != "cl" or f.hd != self.hd_psi:
                raise TbfpError(TBFP_EINVAL, f"expected a 'cl' field with halo {self.hd_psi}")

    def last_stats(self) -> TbfpStats:
        """Statistics of the last solve or projection (tbfp_get_stats)."""
        st = TbfpStats()
        check(self.lib.tbfp_get_stats(self.h, C.byref(st)), self.h)
        return st

    def set_wait_limit(self, cycles: int) -> None:
        """Bound, in SM clock cycles, on each wait of the velocity correction for the copies
        that stage its inputs (tbfp_set_wait_limit; default 4e9, about 2 s).  A wait that runs
        out makes the projection raise TbfpError with TBFP_ETIMEOUT; the handle stays usable."""
        check(self.lib.tbfp_set_wait_limit(self.h, int(cycles)), self.h)

    # --- solveFPS ----------------------------------------------------------
    def solve_fps(self, p: Field, s: Field) -> int:
        """solveFPS (fastPoissonSolver.f90:337-384): p <- L^{-1} s with zero volume-weighted
        mean, ghosts updated.  Returns the status (0, or TBFP_ENOTCONVERGED when the
        mixed path hit max_iter); iterations and residual are in last_stats()."""
        self._check_psi(p, s)
        dev = _placement([p, s])
        fn = self.lib.tbfp_solve_fps_dev if dev else self.lib.tbfp_solve_fps
        return check(fn(self.h, s.address(), p.address()), self.h)


class PoissonEqn:
    """The FAST_MODE pressure equation (poissonEqnCTOR, poissonEqn.f90:89-150)."""

    def __init__(self, mesh: Grid, rhol: float, rhog: float, **solver_kw):
        self.mesh = mesh
        self.rho0 = min(rhol, rhog)  # poissonEqn.f90:127
        self.nl = 2  # number of pressure levels (:145)
        self.solver = FastPoissonSolver(mesh, **solver_kw)

    def close(self):
        self.solver.close()

    def compute_source(self, s: Field, psi_n: Field, psi_nm1: Field, rho: Field, u: VField, dt: float,
                       alpha: float, st_n=None, st_nm1=None) -> None:
        """computeSource FAST (poissonEqn.f90:193-305) into s."""
        sv = self.solver
        fields = [s, psi_n, psi_nm1, rho, *u.components()] + list(st_n or []) + list(st_nm1 or [])
        dev = _placement(fields)
        a, b = _PtrTriple(st_n), _PtrTriple(st_nm1)
        fn = sv.lib.tbfp_rhs_split_dev if dev else sv.lib.tbfp_rhs_split
        check(fn(sv.h, u.ux.address(), u.uy.address(), u.uz.address(), rho.address(), psi_n.address(),
                 psi_nm1.address(), a.addr, b.addr, dt, alpha, self.rho0, s.address()), sv.h)

    def solve_poisson_eqn(self, psi: Field, psi_n: Field, psi_nm1: Field, rho: Field, u: VField, dt: float,
                          alpha: float, st_n=None, st_nm1=None) -> None:
        """solvePoissonEqn FAST (poissonEqn.f90:347-370): computeSource then solveFPS."""
        s = Field.like(psi, _zeros_like(psi.a))
        self.compute_source(s, psi_n, psi_nm1, rho, u, dt, alpha, st_n, st_nm1)
        self.solver.solve_fps(psi, s)

    def projection(self, psi: Field, psi_n: Field, psi_nm1: Field, rho: Field, u: VField, dt: float,
                   alpha: float, st_n=None, st_nm1=None, u_out: VField | None = None,
                   want_stats: bool = True) -> TbfpStats | None:
        """One projection as main.f90:197-212 calls it: solvePoissonEqn, makeVelocityDivFree
        and computeContinuityError in one library call.  u is overwritten with the
        projected velocity unless u_out is given (device fields only).  With
        want_stats=False no statistics are read back, so an asynchronous solver
        does not synchronise."""
        sv = self.solver
        fields = [psi, psi_n, psi_nm1, rho, *u.components()] + list(st_n or []) + list(st_nm1 or [])
        dev = _placement(fields)
        a, b = _PtrTriple(st_n), _PtrTriple(st_nm1)
        st = TbfpStats() if want_stats else None
        stp = C.byref(st) if want_stats else None
        if dev:
            uo = u_out or u
            check(sv.lib.tbfp_projection_dev(sv.h, u.ux.address(), u.uy.address(), u.uz.address(),
                                             uo.ux.address(), uo.uy.address(), uo.uz.address(), rho.address(),
                                             psi_n.address(), psi_nm1.address(), a.addr, b.addr, dt, alpha,
                                             self.rho0, psi.address(), stp), sv.h)
        else:
            if u_out is not None:
                raise TbfpError(TBFP_EINVAL, "u_out is only supported for device fields")
            check(sv.lib.tbfp_projection(sv.h, u.ux.address(), u.uy.address(), u.uz.address(), rho.address(),
                                         psi_n.address(), psi_nm1.address(), a.addr, b.addr, dt, alpha,
                                         self.rho0, psi.address(), stp), sv.h)
        return st

    @staticmethod
    def update_pressure(psi: Field, psi_n: Field, psi_nm1: Field):
        """updatePressure's history shift (poissonEqn.f90:400-401, storeOldField
        field.f90:1590-1603) as a rotation of buffers: returns the new
        (psi_n, psi_nm1, spare) -- psi becomes psi^n, psi^n becomes psi^{n-1}."""
        return psi, psi_n, psi_nm1


def make_velocity_div_free(eqn: PoissonEqn, u: VField, psi: Field, psi_n: Field, psi_nm1: Field, rho: Field,
                           dt: float, alpha: float, st_n=None, st_nm1=None) -> None:
    """makeVelocityDivFree FAST (momentumEqn.f90:999-1127), in place on u."""
    sv = eqn.solver
    fields = [psi, psi_n, psi_nm1, rho, *u.components()] + list(st_n or []) + list(st_nm1 or [])
    dev = _placement(fields)
    a, b = _PtrTriple(st_n), _PtrTriple(st_nm1)
    fn = sv.lib.tbfp_correct_dev if dev else sv.lib.tbfp_correct
    check(fn(sv.h, u.ux.address(), u.uy.address(), u.uz.address(), psi.address(), psi_n.address(),
             psi_nm1.address(), rho.address(), a.addr, b.addr, dt, alpha, eqn.rho0), sv.h)


def compute_continuity_error(solver: FastPoissonSolver, u: VField, dt: float):
    """computeContinuityError (auxiliaryRoutines.f90:42-91): returns
    (max|div u|, dt*max|div u|)."""
    dev = _placement(list(u.components()))
    md, ce = C.c_double(), C.c_double()
    fn = solver.lib.tbfp_continuity_error_dev if dev else solver.lib.tbfp_continuity_error
    check(fn(solver.h, u.ux.address(), u.uy.address(), u.uz.address(), dt, C.byref(md), C.byref(ce)), solver.h)
    return md.value, ce.value


def _zeros_like(a):
    if isinstance(a, np.ndarray):
        return np.zeros_like(a)
    import torch  # noqa: PLC0415

    return torch.zeros_like(a)


class VOF:
    """Material properties of the two-phase mixture (the VOF type's
    updateMaterialProps, VOF.f90:197-233, with smoothVF, :235-262) on a solver's
    handle: cs = smoothed volume fraction, rho and mu from cs.  The fields c, cs,
    rho, mu are cell fields with the solver's rho halo."""

    def __init__(self, solver: FastPoissonSolver, rhol: float, rhog: float, mul: float, mug: float):
        m = solver.mesh
        nx, ny = m.nx, m.ny
        # a rank of a z-split channel (dist.SlabChannel) holds planes k0+1..k0+nz
        slab = getattr(solver, "s", None)
        k0, nz = (slab.k0, slab.nz_loc) if slab is not None else (0, m.nz)
        self.solver = solver
        self.rhol, self.rhog, self.mul, self.mug = rhol, rhog, mul, mug
        self._c = {
            "xc": np.ascontiguousarray(m.xc.r(0, nx + 1)), "yc": np.ascontiguousarray(m.yc.r(0, ny + 1)),
            "zc": np.ascontiguousarray(m.zc.r(k0, k0 + nz + 1)), "xf": np.ascontiguousarray(m.xf.r(0, nx)),
            "yf": np.ascontiguousarray(m.yf.r(0, ny)), "zf": np.ascontiguousarray(m.zf.r(k0, k0 + nz)),
        }
        v = TbfpVofDesc(rhol=rhol, rhog=rhog, mul=mul, mug=mug,
                        **{k: a.ctypes.data_as(C.c_void_p) for k, a in self._c.items()})
        check(solver.lib.tbfp_vof_setup(solver.h, C.byref(v)), solver.h)

    def update_material_props(self, c: Field, cs: Field, rho: Field, mu: Field) -> None:
        """updateMaterialProps (VOF.f90:197-233): cs, rho and mu from c (c's ghosts current)."""
        sv = self.solver
        dev = _placement([c, cs, rho, mu])
        fn = sv.lib.tbfp_material_props_dev if dev else sv.lib.tbfp_material_props
        check(fn(sv.h, c.address(), cs.address(), rho.address(), mu.address()), sv.h)

    def smooth_pass(self, inp: Field, out: Field, rho: Field | None = None, mu: Field | None = None) -> None:
        """One smoothing pass (device fields, halo 1); with rho and mu the second
        pass with the properties.  On a slab the caller exchanges the z ghost
        planes of out (rho, mu) after it (dist.slab_material_props)."""
        sv = self.solver
        _placement([inp, out, rho, mu])
        check(sv.lib.tbfp_material_props_pass_dev(sv.h, inp.address(), out.address(),
                                                  rho.address() if rho is not None else None,
                                                  mu.address() if mu is not None else None), sv.h)


def compute_surface_tension(solver: FastPoissonSolver, c: Field, sigma: float, st: VField,
                            kappa: Field | None = None) -> None:
    """computeSurfaceTension (VOF.f90:1872-2002) on the grid: the face force
    sigma * k_f * grad c into st (the three staggered components with halo
    hd_st), from the volume fraction c (rho's layout) and the height-function
    curvature (also into kappa when given).  See include/tbfp.h for the method."""
    fields = [c, *st.components()] + ([kappa] if kappa is not None else [])
    dev = _placement(fields)
    fn = solver.lib.tbfp_surface_tension_dev if dev else solver.lib.tbfp_surface_tension
    check(fn(solver.h, c.address(), float(sigma), kappa.address() if kappa is not None else None, st.ux.address(),
             st.uy.address(), st.uz.address()), solver.h)


class MomentumEqn:
    """The momentum predictor of FAST_MODE (momentumEqnCTOR, momentumEqn.f90:98-157;
    solveMomentumEqn :161-194 without its closing updateBoundariesV) on a
    solver's handle.  The flux history (phi of the last step, for AB2) lives in
    the library; fluxes() / set_fluxes() read and load it (printOldTimeFlux /
    initOldTimeFlux)."""

    def __init__(self, solver: FastPoissonSolver, scheme: int = 2, gch: float = 0.0, g: float = 0.0,
                 ubot=(0.0, 0.0, 0.0), utop=(0.0, 0.0, 0.0)):
        self.solver = solver
        self.scheme, self.gch, self.g = int(scheme), float(gch), float(g)
        g_ = solver.mesh
        # a rank of a z-split channel (dist.SlabChannel) holds planes k0+1..k0+nz
        slab = getattr(solver, "s", None)
        self._k0, self._nz = (slab.k0, slab.nz_loc) if slab is not None else (0, g_.nz)
        k0, nzl = self._k0, self._nz
        self._t = {n: np.ascontiguousarray(getattr(g_, n).r(0, nn + 1))
                   for n, nn in (("dxf", g_.nx), ("dxc", g_.nx), ("dyf", g_.ny), ("dyc", g_.ny), ("yc", g_.ny))}
        for n in ("dzf", "dzc"):
            self._t[n] = np.ascontiguousarray(getattr(g_, n).r(k0, k0 + nzl + 1))
        self._t["yf"] = np.ascontiguousarray(g_.yf.r(0, g_.ny))
        m = TbfpMomentumDesc(scheme=scheme, gch=gch, g=g, ubot=(C.c_double * 3)(*ubot),
                             utop=(C.c_double * 3)(*utop),
                             **{n: a.ctypes.data_as(C.c_void_p).value for n, a in self._t.items()})
        check(solver.lib.tbfp_momentum_setup(solver.h, C.byref(m)), solver.h)

    @classmethod
    def from_specs(cls, solver: FastPoissonSolver, specs_dir: str) -> "MomentumEqn":
        """Settings read as momentumEqnCTOR reads them: convection_scheme from
        specs/schemes, g and gCH from specs/parameters; the wall values from
        specs/fstart_bc/u when present."""
        from .io import ParFile  # noqa: PLC0415

        from .io import velocity_walls  # noqa: PLC0415

        par = ParFile("parameters", specs_dir)
        ubot, utop = velocity_walls(specs_dir)
        return cls(solver, scheme=ParFile("schemes", specs_dir).read_int("convection_scheme"),
                   gch=par.read_real("gCH"), g=par.read_real("g"), ubot=ubot, utop=utop)

    def _shapes(self):
        m, nz = self.solver.mesh, self._nz
        return [(nz, m.ny, m.nx + 1), (nz, m.ny - 1, m.nx), (nz + 1, m.ny, m.nx)]

    def fluxes(self):
        """The fluxes of the last step (phi_x, phi_y, phi_z) over the equation boxes."""
        out = [np.zeros(s) for s in self._shapes()]
        sv = self.solver
        check(sv.lib.tbfp_momentum_fluxes(sv.h, *[a.ctypes.data_as(C.c_void_p) for a in out], 0), sv.h)
        return tuple(out)

    def set_fluxes(self, phi) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in phi]
        for a, s in zip(arrs, self._shapes()):
            if a.shape != s:
                raise TbfpError(TBFP_EINVAL, f"flux array of shape {a.shape}, expected {s}")
        sv = self.solver
        check(sv.lib.tbfp_momentum_fluxes(sv.h, *[a.ctypes.data_as(C.c_void_p) for a in arrs], 1), sv.h)

    def _boxes(self):
        if self._nz != self.solver.mesh.nz:
            raise TbfpError(TBFP_EINVAL, "the phi0 files hold the whole channel: gather the slabs' fluxes first")
        m = self.solver.mesh
        return [(0, m.nx, 1, m.ny, 1, m.nz), (1, m.nx, 1, m.ny - 1, 1, m.nz), (1, m.nx, 1, m.ny, 0, m.nz)]

    def write_old_time_flux(self, case_dir: str, n: int) -> None:
        """printOldTimeFlux (momentumEqn.f90:1279-1290): the flux history as the
        vector field phi0 of time folder n (files phi0x, phi0y, phi0z in the
        field format), the equation boxes filled and the uy wall faces zero (phi0
        is created zeroed, initOpt=-1)."""
        from . import io  # noqa: PLC0415

        m = self.solver.mesh
        for comp, kind, phi, b in zip("xyz", ("sx", "sy", "sz"), self.fluxes(), self._boxes()):
            f = Field(kind, 1, m.nx, m.ny, m.nz)
            f.v(*b)[...] = phi
            io.write_field(case_dir, n, "phi0" + comp, f)

    def read_old_time_flux(self, case_dir: str, n: int) -> None:
        """initOldTimeFlux (momentumEqn.f90:1254-1275): phi0 of time folder n
        into the flux history; a component file that is absent reads as zero
        (readField_if_present, field.f90:308-326)."""
        import os  # noqa: PLC0415

        from . import io  # noqa: PLC0415

        m = self.solver.mesh
        hist = []
        for comp, kind, b in zip("xyz", ("sx", "sy", "sz"), self._boxes()):
            f = Field(kind, 1, m.nx, m.ny, m.nz)
            if os.path.exists(io.field_path(case_dir, n, "phi0" + comp)):
                io.read_field(case_dir, n, "phi0" + comp, f)
            hist.append(np.ascontiguousarray(f.v(*b)))
        self.set_fluxes(hist)

    def update_boundaries_v(self, u: VField) -> None:
        """updateBoundariesV (vfield.f90:111-189): wall ghosts, periodic halos and
        duplicates of u, in place."""
        sv = self.solver
        dev = _placement(list(u.components()))
        fn = sv.lib.tbfp_update_boundaries_v_dev if dev else sv.lib.tbfp_update_boundaries_v
        check(fn(sv.h, u.ux.address(), u.uy.address(), u.uz.address()), sv.h)

    def solve(self, u: VField, c: Field, mu: Field, rho: Field, dt: float, alpha: float, gamma: float, xi: float,
              rho0: float, fs: float = 0.0, st=None, u_out: VField | None = None) -> None:
        """solveMomentumEqn (momentumEqn.f90:161-194): the predictor, then
        updateBoundariesV, so the result comes out ready for the next stencils;
        in u, or in u_out (device fields) with u left as it was."""
        self.predictor(u, c, mu, rho, dt, alpha, gamma, xi, rho0, fs, st, u_out=u_out)
        self.update_boundaries_v(u_out if u_out is not None else u)

    def predictor(self, u: VField, c: Field, mu: Field, rho: Field, dt: float, alpha: float, gamma: float,
                  xi: float, rho0: float, fs: float = 0.0, st=None, u_out: VField | None = None) -> None:
        """solveMomentumEqn FAST without its boundary update: u <- u + dt*(gamma*phi +
        xi*phi_prev) + sources, in place, or into u_out (device fields; the update
        then runs inside the flux kernel and u is only read)."""
        sv = self.solver
        fields = [*u.components(), c, mu, rho] + list(st or [])
        dev = _placement(fields + (list(u_out.components()) if u_out is not None else []))
        s = _PtrTriple(st)
        if u_out is not None:
            if not dev:
                raise TbfpError(TBFP_EINVAL, "u_out is only supported for device fields")
            check(sv.lib.tbfp_momentum_predictor_out_dev(
                sv.h, u.ux.address(), u.uy.address(), u.uz.address(), u_out.ux.address(), u_out.uy.address(),
                u_out.uz.address(), c.address(), mu.address(), rho.address(), s.addr, dt, alpha, gamma, xi, rho0,
                fs), sv.h)
            return
        fn = sv.lib.tbfp_momentum_predictor_dev if dev else sv.lib.tbfp_momentum_predictor
        check(fn(sv.h, u.ux.address(), u.uy.address(), u.uz.address(), c.address(), mu.address(), rho.address(),
                 s.addr, dt, alpha, gamma, xi, rho0, fs), sv.h)


class FlowControl:
    """The channel's flow control (momentumEqnCTOR, momentumEqn.f90:109-146, and
    auxiliaryRoutines.f90:336-546): flow_ctrl 1 drives ux with the pressure
    gradient of the friction Reynolds number ret, 2 holds the flow rate at q0,
    3 only balances gravity, anything else does nothing.  The volume sums run
    on the GPU (tbfp_rho_face_sum, tbfp_flow_rate); the scalar formulas are
    the reference's."""

    def __init__(self, solver: FastPoissonSolver, flow_ctrl: int, ret: float = 0.0, q0: float = 0.0, group=None):
        self.solver = solver
        self.flow_ctrl, self.ret, self.q0 = int(flow_ctrl), float(ret), float(q0)
        # on a rank of a z-split channel the volume sums add over the ranks (Mpi_Allreduce)
        self._slab = getattr(solver, "s", None) is not None
        self.group = group

    def _global(self, x: float) -> float:
        if not self._slab:
            return x
        from .dist import sum_over_ranks  # noqa: PLC0415

        return sum_over_ranks(x, group=self.group)

    @classmethod
    def from_specs(cls, solver: FastPoissonSolver, specs_dir: str, u: VField | None = None) -> "FlowControl":
        """As momentumEqnCTOR reads specs/flowControl: flowCtrl; Ret for 1; for 2
        flow_rate (times Lx*Lz) when read_flow_rate is true, else the flow rate
        of the initial u."""
        from .io import ParFile  # noqa: PLC0415

        pf = ParFile("flowControl", specs_dir)
        ctrl = pf.read_int("flowCtrl")
        fc = cls(solver, ctrl)
        if ctrl == 1:
            fc.ret = pf.read_real("Ret")
        if ctrl == 2:
            if pf.read_bool("read_flow_rate"):
                m = solver.mesh
                fc.q0 = pf.read_real("flow_rate") * m.Lx * m.Lz
            else:
                if u is None:
                    raise TbfpError(TBFP_EINVAL, "flowCtrl 2 without read_flow_rate needs the initial velocity")
                fc.q0 = fc.flow_rate(u)
        return fc

    def rho_face_sum(self, rho: Field) -> float:
        sv = self.solver
        out = C.c_double(0.0)
        fn = sv.lib.tbfp_rho_face_sum_dev if _placement([rho]) else sv.lib.tbfp_rho_face_sum
        check(fn(sv.h, rho.address(), C.byref(out)), sv.h)
        return self._global(out.value)

    def flow_rate(self, u: VField) -> float:
        """computeFlowRate: the sum of ux*Vsx over the faces i = 0..nx-1."""
        sv = self.solver
        out = C.c_double(0.0)
        fn = sv.lib.tbfp_flow_rate_dev if _placement([u.ux]) else sv.lib.tbfp_flow_rate
        check(fn(sv.h, u.ux.address(), C.byref(out)), sv.h)
        return self._global(out.value)

    def set_press_grad(self, rho: Field, rhol: float, mul: float, g: float) -> float:
        """setPressGrad (auxiliaryRoutines.f90:336-393): the forcing fs of the
        momentum predictor; g is the momentum equation's gCH."""
        rho_av = self.rho_face_sum(rho) / self.solver.mesh.s_Vg
        if self.flow_ctrl == 1:
            nul = mul / rhol
            re = 1.0 / nul
            tauw = (self.ret / re) * (self.ret / re)
            return tauw - rho_av * g
        if self.flow_ctrl in (2, 3):
            return -rho_av * g
        return 0.0

    def set_flow_rate(self, mom: "MomentumEqn", u: VField) -> None:
        """setFlowRate (auxiliaryRoutines.f90:467-513): for flowCtrl 2, ux += (Q0 - Q)/s_Vg
        over ux(0:nx,1:ny,1:nz), then updateBoundariesV."""
        if self.flow_ctrl != 2:
            return
        uf = (self.q0 - self.flow_rate(u)) / self.solver.mesh.s_Vg
        sv = self.solver
        fn = sv.lib.tbfp_add_ux_dev if _placement([u.ux]) else sv.lib.tbfp_add_ux
        check(fn(sv.h, u.ux.address(), uf), sv.h)
        mom.update_boundaries_v(u)


def fast_substep(eqn: PoissonEqn, vof: VOF, mom: MomentumEqn, flow: FlowControl, c: Field, cs: Field, rho: Field,
                 mu: Field, u: VField, psi: Field, psi_n: Field, psi_nm1: Field, dt: float, alpha: float,
                 gamma: float, xi: float, st_n=None, st_nm1=None, want_stats: bool = True,
                 u_star: VField | None = None):
    """One Runge-Kutta substep of tph_flow_solver (main.f90:177-209) from
    updateMaterialProps on, all on the GPU when the fields are device fields:
    updateMaterialProps, setPressGrad, solveMomentumEqn (predictor +
    updateBoundariesV), solvePoissonEqn + makeVelocityDivFree (with its closing
    updateBoundariesV) + computeContinuityError, setFlowRate.  The VOF
    advection and the surface tension before it, and updatePressure's level
    rotation after it (PoissonEqn.update_pressure), stay with the caller.  vof,
    mom and flow must live on eqn's handle.  With a scratch u_star (device
    fields) the predictor writes u* there and the projection writes the result
    back into u, so the predictor's update needs no pass of its own.  Returns
    the projection's stats."""
    vof.update_material_props(c, cs, rho, mu)
    fs = flow.set_press_grad(rho, vof.rhol, vof.mul, mom.gch)
    if u_star is not None:
        mom.solve(u, c, mu, rho, dt, alpha, gamma, xi, eqn.rho0, fs=fs, st=st_n, u_out=u_star)
        stats = eqn.projection(psi, psi_n, psi_nm1, rho, u_star, dt, alpha, st_n, st_nm1, u_out=u,
                               want_stats=want_stats)
    else:
        mom.solve(u, c, mu, rho, dt, alpha, gamma, xi, eqn.rho0, fs=fs, st=st_n)
        stats = eqn.projection(psi, psi_n, psi_nm1, rho, u, dt, alpha, st_n, st_nm1, want_stats=want_stats)
    mom.update_boundaries_v(u)
    flow.set_flow_rate(mom, u)
    return stats


class PCG:
    """MG_MODE pressure solver (pcgCTOR, pcg.f90:62-99): FP64 conjugate gradients
    preconditioned by FP32 red-black Gauss-Seidel multigrid V-cycles.  Defaults
    are those of the 256x256x128 MG workload (6 levels, 2 + 2 sweeps); a case's
    own settings come from its specs/pcg_solver file through from_specs."""

    @classmethod
    def from_specs(cls, mesh: Grid, specs_dir: str, **kw) -> "PCG":
        """pcgCTOR / multiGridCTOR reading specs/pcg_solver (pcg.f90:82-85,
        multiGrid.f90:81-86): nLevels, nPreSweep, nPostSweep, tolMG, maxIterMG,
        tolPCG, maxIterPCG."""
        from .io import ParFile  # noqa: PLC0415

        p = ParFile("pcg_solver", specs_dir)
        return cls(mesh, n_levels=p.read_int("nLevels"), n_pre=p.read_int("nPreSweep"),
                   n_post=p.read_int("nPostSweep"), tol_mg=p.read_real("tolMG"), max_iter_mg=p.read_int("maxIterMG"),
                   tol_pcg=p.read_real("tolPCG"), max_iter_pcg=p.read_int("maxIterPCG"), **kw)

    def __init__(self, mesh: Grid, n_levels: int = 6, n_pre: int = 2, n_post: int = 2, tol_mg: float = 0.4,
                 max_iter_mg: int = 100, tol_pcg: float = 1e-10, max_iter_pcg: int = 100, hd_psi: int = 1,
                 hd_rho: int = 1, device: int = -1, stream: int | None = None):
        self.solver = FastPoissonSolver(mesh, hd_psi=hd_psi, hd_rho=hd_rho, device=device, stream=stream)
        self.lib, self.h, self.mesh = self.solver.lib, self.solver.h, mesh
        self.params = TbfpMgParams(n_levels=n_levels, n_pre=n_pre, n_post=n_post, tol_mg=tol_mg,
                                   max_iter_mg=max_iter_mg, tol_pcg=tol_pcg, max_iter_pcg=max_iter_pcg)
        check(self.lib.tbfp_pcg_setup(self.h, C.byref(self.params)), self.h)

    def close(self):
        self.solver.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve_pcg(self, psi: Field, beta: Field, q: Field) -> TbfpStats:
        """solvePCG (pcg.f90:103-140): psi (initial guess, result with ghosts)
        solves L_beta psi = q.  Returns the statistics (iterations, ||r||/||q||);
        an iteration cap is a soft condition (the stats say so)."""
        dev = _placement([psi, beta, q])
        st = TbfpStats()
        fn = self.lib.tbfp_pcg_solve_dev if dev else self.lib.tbfp_pcg_solve
        check(fn(self.h, psi.address(), beta.address(), q.address(), C.byref(st)), self.h)
        return st

    def projection(self, psi: Field, rho: Field, u: VField, dt: float, alpha: float,
                   u_out: VField | None = None) -> TbfpStats:
        """One MG_MODE projection (computeSource MG, computeBeta, solvePCG,
        addPressureGrad, computeContinuityError): psi is the initial guess and
        the pressure; u is corrected in place unless u_out is given (device
        fields only)."""
        dev = _placement([psi, rho, *u.components()])
        st = TbfpStats()
        if dev:
            uo = u_out or u
            check(self.lib.tbfp_projection_mg_dev(self.h, u.ux.address(), u.uy.address(), u.uz.address(),
                                                  uo.ux.address(), uo.uy.address(), uo.uz.address(), rho.address(),
                                                  dt, alpha, psi.address(), C.byref(st)), self.h)
        else:
            if u_out is not None:
                raise TbfpError(TBFP_EINVAL, "u_out is only supported for device fields")
            check(self.lib.tbfp_projection_mg(self.h, u.ux.address(), u.uy.address(), u.uz.address(),
                                              rho.address(), dt, alpha, psi.address(), C.byref(st)), self.h)
        return st


class Ensemble:
    """Many independent channels on one GPU (tbfp_ensemble_*): each member has
    its own grid; one call projects every member, either as a replayed CUDA
    graph of every member's kernels on a pool of streams (mode "graph"), or as
    one persistent launch that runs every stage of every member from a device
    work queue (mode "persistent": FP64, out-of-place members up to
    nx = 256, nz = 128, ny = 256).  Mode "auto" measures both on the first
    call and keeps the faster, recorded in the tuning cache file."""

    MODES = {"auto": 0, "graph": 1, "persistent": 2}

    def __init__(self, meshes, nstreams: int = 8, precision: str = "fp64", tol: float = 1e-10, max_iter: int = 8,
                 device: int = -1, mode: str = "auto", blocks_per_sm: int = 0):
        self.lib = load()
        self.meshes = list(meshes)
        self._m = [_metrics(g) for g in self.meshes]
        descs = (TbfpDesc * len(self.meshes))(*[_desc(g, m, 1, 2, 1, 1, precision, tol, max_iter, device, None, 0)
                                                for g, m in zip(self.meshes, self._m)])
        h = C.c_void_p()
        check(self.lib.tbfp_ensemble_create(len(self.meshes), descs, nstreams, C.byref(h)), None)
        self.h = h
        if mode != "auto" or blocks_per_sm:
            self.set_mode(mode, blocks_per_sm)

    def set_mode(self, mode: str, blocks_per_sm: int = 0) -> None:
        check(self.lib.tbfp_ensemble_set_mode(self.h, self.MODES[mode], blocks_per_sm), None)

    def mode(self):
        """(form in use, its parameter, measured ms of [graph, persistent x1, persistent x2])."""
        m, p = C.c_int(), C.c_int()
        ms = (C.c_float * 3)()
        check(self.lib.tbfp_ensemble_get_mode(self.h, C.byref(m), C.byref(p), ms), None)
        names = {0: None, 1: "graph", 2: "persistent"}
        return names[m.value], p.value, [float(x) for x in ms]

    def set_wait_limit(self, polls: int) -> None:
        check(self.lib.tbfp_ensemble_set_wait_limit(self.h, int(polls)), None)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.tbfp_ensemble_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass

    def projection(self, members, dt: float, alpha: float, rho0: float, want_stats: bool = True):
        """members: one (psi, psi_n, psi_nm1, rho, u, u_out) tuple of device fields per
        channel (u_out may be u).  Returns the per-member statistics or None."""
        n = len(self.meshes)
        if len(members) != n:
            raise TbfpError(TBFP_EINVAL, f"expected {n} members")
        io = (TbfpMemberIO * n)()
        for k, (psi, pn, pnm1, rho, u, uo) in enumerate(members):
            if not _placement([psi, pn, pnm1, rho, *u.components(), *uo.components()]):
                raise TbfpError(TBFP_EINVAL, "ensemble members must be device fields")
            io[k] = TbfpMemberIO(u.ux.address(), u.uy.address(), u.uz.address(), uo.ux.address(), uo.uy.address(),
                                 uo.uz.address(), rho.address(), pn.address(), pnm1.address(), psi.address())
        st = (TbfpStats * n)() if want_stats else None
        check(self.lib.tbfp_ensemble_projection_dev(self.h, io, dt, alpha, rho0, st), None)
        return list(st) if want_stats else None
