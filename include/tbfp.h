/*
 * tbfp.h -- C ABI of the B200-native pressure-projection library for
 * TBFsolver-style bubbly channel flow.
 *
 * The library replaces, behind plain C calls, the Fortran subroutines of the
 * reference's FAST_MODE projection step:
 *
 *   fastPoissonSolverCTOR   src/fastPoissonSolver/fastPoissonSolver.f90:123  -> tbfp_create
 *   solveFPS                src/fastPoissonSolver/fastPoissonSolver.f90:337  -> tbfp_solve_fps[_dev]
 *   computeSource (FAST)    src/poissonEqn/poissonEqn.f90:193                -> tbfp_rhs_split[_dev]
 *   makeVelocityDivFree     src/momentumEqn/momentumEqn.f90:999              -> tbfp_correct[_dev]
 *   computeContinuityError  src/auxiliaryRoutines/auxiliaryRoutines.f90:42   -> tbfp_continuity_error[_dev]
 *   solvePoissonEqn + makeVelocityDivFree + computeContinuityError
 *                           src/main.f90:197-212                             -> tbfp_projection[_dev]
 *
 * Array convention.  Every field argument is the base address of a Fortran
 * allocatable WITH its halo, exactly as the reference allocates it
 * (field.f90:271-273): a cell field ('cl') is f(1-hd:nx+hd, 1-hd:ny+hd,
 * 1-hd:nz+hd); the staggered velocity components are ux(-hd:nx+hd, ...) ('sx'),
 * uy(.., -hd:ny+hd, ..) ('sy'), uz(.., .., -hd:nz+hd) ('sz'), column-major
 * (i fastest).  The halo widths are given once in tbfp_desc.  Host-pointer
 * entry points copy to and from device buffers owned by the handle; the
 * *_dev entry points take device pointers with the same layout.
 *
 * Return convention (mirrors the reference's error handling, errorHandler.f90):
 *   0   TBFP_OK
 *   >0  soft condition; results are valid (e.g. an iteration cap was reached,
 *       the reference's warning at pcg.f90:366-373)
 *   <0  hard error; a Fortran caller maps it to mpiABORT(tbfp_strerror(rc)).
 * A singular tridiagonal pivot is NOT an error (fastPoissonSolver.f90:318-322).
 *
 * Threading: one handle per host thread; calls on one handle are not
 * re-entrant.  All calls are synchronous (they return after the device work
 * has completed) unless TBFP_FLAG_ASYNC is set at create time.
 */
#ifndef TBFP_H
#define TBFP_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TBFP_ABI_VERSION 1

/* status codes */
#define TBFP_OK 0
#define TBFP_ENOTCONVERGED 1 /* soft: iteration cap reached */
#define TBFP_EINVAL (-1)     /* invalid descriptor or argument */
#define TBFP_ENULL (-2)      /* a required pointer is NULL */
#define TBFP_ECUDA (-3)      /* CUDA runtime error */
#define TBFP_ENOMEM (-4)     /* device allocation failed */
#define TBFP_EUNSUPPORTED (-5) /* size or feature not supported */
#define TBFP_ENODEVICE (-6)  /* no usable CUDA device */
#define TBFP_ENONFINITE (-7) /* a NaN or Inf reached a residual, the pressure or max|div u|: a
                                non-finite input, or a breakdown (the reference aborts) */
#define TBFP_ESINGULAR (-8)  /* MG_MODE: the coarsest-level system is singular (beta not positive) */
#define TBFP_ETIMEOUT (-9)   /* a bounded device-side wait ran out (persistent ensemble kernel, staged correction) */

/* precision modes */
#define TBFP_FP64 0  /* plain FP64: the drop-in for solveFPS */
#define TBFP_MIXED 1 /* FP32 transforms + FP64 defect correction: psi = solve32(s), then
                        psi += solve32(s - L psi) until ||s - L psi||_2/||s||_2 <= tol and,
                        in a projection, also max|div u| <= tol (div u of the corrected
                        velocity is alpha*dt/rho0 * (s - L psi) cell by cell).  The
                        residual is that of the system the FP64 path solves (the
                        incompatible part of s, sum s V != 0, sits on the top wall).  The
                        loop runs on the device (a CUDA graph with a conditional WHILE
                        node, also inside a caller's stream capture): no host round trip
                        per sweep.  A synchronous call reads the outcome back; with
                        TBFP_FLAG_ASYNC and no stats the sweep count is reported as -1. */

/* create-time flags */
#define TBFP_FLAG_ASYNC 1u  /* do not synchronise the stream before returning */
#define TBFP_FLAG_TIMING 2u /* record per-stage device times into tbfp_stats.ms_stage */
#define TBFP_FLAG_RESIDUAL 4u /* TBFP_FP64: also compute tbfp_stats.rel_residual (one more pass) */

/* stages of one projection, indices into tbfp_stats.ms_stage */
#define TBFP_STAGE_RECIP 0      /* 1/rho */
#define TBFP_STAGE_RHS_FFTX 1   /* split RHS + forward x transform */
#define TBFP_STAGE_FFTZ_FWD 2   /* forward z transform */
#define TBFP_STAGE_TRIDIAG 3    /* y tridiagonal systems + gauge */
#define TBFP_STAGE_FFTZ_INV 4   /* backward z transform */
#define TBFP_STAGE_FFTX_INV 5   /* backward x transform, psi + ghosts */
#define TBFP_STAGE_CORRECT 6    /* velocity correction (+ continuity check) */
#define TBFP_STAGE_DIV 7        /* separate continuity check (in-place path) */
#define TBFP_NSTAGES 8

typedef struct tbfp_handle tbfp_handle;

/*
 * Create-time descriptor.  Grid metrics are the reference mesh arrays
 * (grid.f90:334-399) for the interior index ranges given below; they are
 * copied at create time.  x and z must be uniform and periodic, y
 * wall-bounded (grid.f90:219-230, mpiControl.f90:206-228).
 */
typedef struct {
  int nx, ny, nz;      /* global cell counts */
  int hd_psi;          /* halo of psi, its old levels and s (reference: 1) */
  int hd_u;            /* halo of ux, uy, uz (reference: 2) */
  int hd_rho;          /* halo of rho (reference: 1) */
  int hd_st;           /* halo of the surface-tension components (reference: 1) */
  double dx_fft;       /* xc(2)-xc(1), spacing of the x eigenvalues (fastPoissonSolver.f90:222) */
  double dz_fft;       /* zc(2)-zc(1) (fastPoissonSolver.f90:223) */
  const double *dxf;   /* dxf(1..nx)   */
  const double *dxc;   /* dxc(1..nx+1) */
  const double *dyf;   /* dyf(1..ny)   */
  const double *dyc;   /* dyc(1..ny+1) */
  const double *dzf;   /* dzf(1..nz)   */
  const double *dzc;   /* dzc(1..nz+1) */
  double s_Vg;         /* total volume (grid.f90:933-951); <= 0: computed from dxf,dyf,dzf */
  int precision;       /* TBFP_FP64 or TBFP_MIXED */
  double tol;          /* TBFP_MIXED: target ||s - L psi||_2 / ||s||_2 */
  int max_iter;        /* TBFP_MIXED: cap on defect-correction sweeps */
  int device;          /* CUDA device ordinal; < 0 selects the current device */
  void *stream;        /* cudaStream_t to run on; NULL: the library creates one */
  unsigned flags;      /* TBFP_FLAG_* */
} tbfp_desc;

/* Per-call statistics (the reference prints these to stdout). */
typedef struct {
  int iterations;       /* defect-correction sweeps (1 for TBFP_FP64) */
  double rel_residual;  /* ||s - L psi||_2/||s||_2 when computed, else -1 */
  double max_div;       /* max|div u| after the correction (auxiliaryRoutines.f90:75) */
  double cont_err;      /* dt * max_div, the reference's "continuity error" (:82) */
  double ms_device;     /* device time of the call, ms (CUDA events) */
  double ms_stage[8];   /* per-stage device time (TBFP_FLAG_TIMING), else 0 */
} tbfp_stats;

/* MG_MODE settings (the reference's specs/pcg_solver file, read by pcgCTOR,
 * pcg.f90:62-99, and multiGridCTOR, multiGrid.f90:60-112). */
typedef struct {
  int n_levels;       /* multigrid levels; nx, ny, nz divisible by 2^(n_levels-1) */
  int n_pre, n_post;  /* red-black Gauss-Seidel sweeps before / after the coarse correction */
  double tol_mg;      /* V-cycles repeat while ||q - L p||/||q|| > tol_mg (0.4 in channel_18) */
  int max_iter_mg;    /* cap on V-cycles per preconditioner application */
  double tol_pcg;     /* PCG stops at ||r||_2/||q||_2 <= tol_pcg */
  int max_iter_pcg;   /* cap on PCG iterations (soft TBFP_ENOTCONVERGED) */
} tbfp_mg_params;

/* --- lifecycle --------------------------------------------------------- */
int tbfp_abi_version(void);
const char *tbfp_strerror(int status);
/* Last error message of a handle (or of the last failed tbfp_create if h is NULL). */
const char *tbfp_last_error(const tbfp_handle *h);
/* fastPoissonSolverCTOR (fastPoissonSolver.f90:123-156): eigenvalues, off-diagonals,
   transform plans and device work buffers. */
int tbfp_create(const tbfp_desc *d, tbfp_handle **h);
int tbfp_destroy(tbfp_handle *h);
/* Bytes of device memory the handle holds. */
size_t tbfp_device_bytes(const tbfp_handle *h);
/* Statistics of the handle's last solve or projection (iterations and
 * rel_residual of TBFP_MIXED / TBFP_FLAG_RESIDUAL, device time).  No
 * counterpart in the reference, which prints them (pcg.f90:366-373). */
int tbfp_get_stats(const tbfp_handle *h, tbfp_stats *out);

/* --- solveFPS (fastPoissonSolver.f90:337-384) -------------------------- */
/* s: cell field (hd_psi), read on the interior.  psi: cell field (hd_psi),
   written on the interior and on the ghost cells (the updateBoundaries of
   fastPoissonSolver.f90:381: Neumann at the y walls, periodic in x and z). */
int tbfp_solve_fps(tbfp_handle *h, const double *s, double *psi);
int tbfp_solve_fps_dev(tbfp_handle *h, const double *s, double *psi);

/* --- computeSource, FAST_MODE (poissonEqn.f90:193-305) ----------------- */
/* psi_n = psi%ptrf_, psi_nm1 = psi%ptrf_%ptrf_.  st_n / st_nm1: arrays of the
   three staggered surface-tension components at the old levels, or NULL for
   zero surface tension.  s: cell field (hd_psi), interior written. */
int tbfp_rhs_split(tbfp_handle *h, const double *ux, const double *uy, const double *uz,
                   const double *rho, const double *psi_n, const double *psi_nm1,
                   const double *const *st_n, const double *const *st_nm1,
                   double dt, double alpha, double rho0, double *s);
int tbfp_rhs_split_dev(tbfp_handle *h, const double *ux, const double *uy, const double *uz,
                       const double *rho, const double *psi_n, const double *psi_nm1,
                       const double *const *st_n, const double *const *st_nm1,
                       double dt, double alpha, double rho0, double *s);

/* --- makeVelocityDivFree, FAST_MODE (momentumEqn.f90:999-1127) --------- */
/* In place on ux, uy, uz: faces of setEqnBounds (momentumEqn.f90:1134-1190)
   are corrected and the periodic duplicate faces are equated
   (vfield.f90:124-189).  The rest of the routine's closing updateBoundariesV
   (momentumEqn.f90:1088: wall ghosts and halos) is tbfp_update_boundaries_v. */
int tbfp_correct(tbfp_handle *h, double *ux, double *uy, double *uz, const double *psi,
                 const double *psi_n, const double *psi_nm1, const double *rho,
                 const double *const *st_n, const double *const *st_nm1,
                 double dt, double alpha, double rho0);
int tbfp_correct_dev(tbfp_handle *h, double *ux, double *uy, double *uz, const double *psi,
                     const double *psi_n, const double *psi_nm1, const double *rho,
                     const double *const *st_n, const double *const *st_nm1,
                     double dt, double alpha, double rho0);

/* --- computeContinuityError (auxiliaryRoutines.f90:42-91) -------------- */
/* max_div = max|div u| over the interior; cont_err = dt * max_div.  Either
   output pointer may be NULL. */
int tbfp_continuity_error(tbfp_handle *h, const double *ux, const double *uy, const double *uz,
                          double dt, double *max_div, double *cont_err);
int tbfp_continuity_error_dev(tbfp_handle *h, const double *ux, const double *uy,
                              const double *uz, double dt, double *max_div, double *cont_err);

/* --- one projection (main.f90:197-212) ---------------------------------- */
/* computeSource -> solveFPS -> makeVelocityDivFree -> computeContinuityError.
   ux, uy, uz are read as u* and overwritten with the projected velocity; psi
   receives the new pressure (interior + ghosts).  stats may be NULL. */
int tbfp_projection(tbfp_handle *h, double *ux, double *uy, double *uz, const double *rho,
                    const double *psi_n, const double *psi_nm1,
                    const double *const *st_n, const double *const *st_nm1,
                    double dt, double alpha, double rho0, double *psi, tbfp_stats *stats);
/* Device-pointer form.  u*_in are read, u*_out written: they may be the same
   arrays (in place).  Every interior face of u*_out is written; halos are not. */
int tbfp_projection_dev(tbfp_handle *h, const double *ux_in, const double *uy_in,
                        const double *uz_in, double *ux_out, double *uy_out, double *uz_out,
                        const double *rho, const double *psi_n, const double *psi_nm1,
                        const double *const *st_n, const double *const *st_nm1,
                        double dt, double alpha, double rho0, double *psi, tbfp_stats *stats);

/* --- MG_MODE: PCG with a multigrid preconditioner ----------------------- */
/* pcgCTOR (pcg.f90:62-99) + multiGridCTOR (multiGrid.f90:60-112): builds the
   level hierarchy on the handle's grid (metrics from its tbfp_desc). */
int tbfp_pcg_setup(tbfp_handle *h, const tbfp_mg_params *p);
/* solvePCG (pcg.f90:103-140): L_beta psi = q with face coefficient
   (beta_P + beta_nb)/2/(dc df), periodic x/z, Neumann walls; FP64 CG
   preconditioned by FP32 red-black Gauss-Seidel V-cycles (solveMG,
   multiGrid.f90:165-232) with a direct coarsest solve (poissMat.f90:289-312).
   psi (layout of psi, hd_psi) is the initial guess and the result, ghosts
   updated; beta has rho's layout (hd_rho), q psi's.  stats: iterations = PCG
   iterations, rel_residual = ||r||_2/||q||_2.  Returns TBFP_ENOTCONVERGED
   (soft) at max_iter_pcg. */
int tbfp_pcg_solve(tbfp_handle *h, double *psi, const double *beta, const double *q, tbfp_stats *stats);
int tbfp_pcg_solve_dev(tbfp_handle *h, double *psi, const double *beta, const double *q, tbfp_stats *stats);

/* One MG_MODE projection (main.f90:197-212 with the MG branches):
   q = div u* (computeSource, poissonEqn.f90:155-190), beta = dt*alpha/rho
   (computeBeta, :311-342), tbfp_pcg_solve, addPressureGrad
   (momentumEqn.f90:795-869) with the periodic equate, and max|div u| into
   stats (computeContinuityError).  psi: initial guess in, pressure out.  The
   _dev form reads u*_in and writes u*_out (may alias); the host form
   corrects u in place. */
int tbfp_projection_mg(tbfp_handle *h, double *ux, double *uy, double *uz, const double *rho, double dt,
                       double alpha, double *psi, tbfp_stats *stats);
int tbfp_projection_mg_dev(tbfp_handle *h, const double *ux_in, const double *uy_in, const double *uz_in,
                           double *ux_out, double *uy_out, double *uz_out, const double *rho, double dt,
                           double alpha, double *psi, tbfp_stats *stats);

/* --- material properties from the volume fraction ---------------------- */
/* updateMaterialProps (VOF.f90:197-233) with smoothVF (VOF.f90:235-262), the
   step that produces rho for the projection: cs = two cell -> vertex -> cell
   passes of c (cellToVertex / vertexToCell, interpolation.f90:188-276), each
   followed by the boundary update of a cell field; then, over the whole
   arrays (halos included), rho = rhog*cs + (1-cs)*rhol and
   mu = mug*cs + (1-cs)*mul.  c, cs, rho, mu are cell fields with rho's layout
   (halo hd_rho); c's ghosts must be current (the reference updates them).
   tbfp_vof_setup takes the grid coordinates (grid.f90:633-688: centroids
   xc(0:nx+1), yc(0:ny+1), zc(0:nz+1) and faces xf(0:nx), yf(0:ny), zf(0:nz))
   and the phase properties (VOFCTOR), once per handle (on a slab handle:
   the local planes' z coordinates zc(k0:k0+nz+1), zf(k0:k0+nz), hd_rho = 1). */
typedef struct {
  const double *xc, *yc, *zc; /* centroids, Fortran indices 0..n+1 */
  const double *xf, *yf, *zf; /* faces, Fortran indices 0..n */
  double rhol, rhog, mul, mug;
} tbfp_vof_desc;
int tbfp_vof_setup(tbfp_handle *h, const tbfp_vof_desc *v);
int tbfp_material_props(tbfp_handle *h, const double *c, double *cs, double *rho, double *mu);
int tbfp_material_props_dev(tbfp_handle *h, const double *c, double *cs, double *rho, double *mu);
/* One of the two smoothing passes (hd_rho = 1, device pointers): out = the
   cell -> vertex -> cell pass of in with its ghost images; with rho and mu
   (the second pass) also the properties.  On a slab handle (a z-split
   channel) the pass writes no z ghost images: the caller exchanges the z ghost
   planes of out (and rho, mu) with the neighbours after each pass, as the
   reference's updateBoundaries does.  tbfp_material_props is
   pass(c -> scratch), pass(scratch -> cs, rho, mu) on a whole channel. */
int tbfp_material_props_pass_dev(tbfp_handle *h, const double *in, double *out, double *rho, double *mu);

/* --- momentum predictor ------------------------------------------------ */
/* solveMomentumEqn FAST (momentumEqn.f90:161-194) without its closing
   updateBoundariesV, which stays with the caller as for the projection: the
   convection (flux-limited) and diffusion (variable viscosity) fluxes of
   updateConveDiff from the current u, u += dt*(gamma*phi + xi*phi_prev)
   (addConvDiff), then the sources of addSource: ux += dt*alpha*(st_x/rho0 +
   fs/rho_x + gCH), uy += dt*alpha*(st_y/rho0 + g), uz += dt*alpha*st_z/rho0,
   on the equation boxes (ux faces 0..nx, uy faces 1..ny-1, uz faces 0..nz,
   setEqnBounds :1134-1190).  u is updated in place; c, mu and rho are cell
   fields with rho's layout; st is NULL or the three surface-tension
   components (hd_st).  u needs its two-layer halo current (the limiters read
   u at +-2).  The library keeps the flux history (phi of the last call);
   tbfp_momentum_setup starts it at zero (initFluxes), tbfp_momentum_fluxes
   loads or reads it (initOldTimeFlux / printOldTimeFlux) as host arrays over
   the equation boxes in Fortran order: phi_x (0:nx,1:ny,1:nz),
   phi_y (1:nx,1:ny-1,1:nz), phi_z (1:nx,1:ny,0:nz).  The spacings are the
   mesh's own metrics (grid.f90:334-399) including the ghost entries the
   stencils reach: dxf(0:nx+1), dxc(0:nx+1), dyf(0:ny+1), dyc(0:ny+1),
   dzf(0:nz+1), dzc(0:nz+1), n+2 values each.  yc(0:ny+1), yf(0:ny) and the
   wall values serve tbfp_update_boundaries_v. */
typedef struct {
  int scheme; /* specs/schemes convection_scheme: 0 central, 1 upwind, 2 QUICK, 3 van Leer,
                 4 superbee, 5 superbee where the volume fraction varies, central elsewhere */
  double gch; /* specs/parameters gCH: streamwise driving added to ux */
  double g;   /* specs/parameters g: body force added to uy */
  const double *dxf, *dxc, *dyf, *dyc, *dzf, *dzc;
  const double *yc, *yf;       /* y centroids (0:ny+1) and faces (0:ny) */
  double ubot[3], utop[3];     /* fixedValue of ux, uy, uz at the bottom and top walls (bvx3, bvx4, ...) */
} tbfp_momentum_desc;
int tbfp_momentum_setup(tbfp_handle *h, const tbfp_momentum_desc *m);
int tbfp_momentum_fluxes(tbfp_handle *h, double *phi_x, double *phi_y, double *phi_z, int set);
int tbfp_momentum_predictor(tbfp_handle *h, double *ux, double *uy, double *uz, const double *c, const double *mu,
                            const double *rho, const double *const *st, double dt, double alpha, double gamma,
                            double xi, double rho0, double fs);
int tbfp_momentum_predictor_dev(tbfp_handle *h, double *ux, double *uy, double *uz, const double *c,
                                const double *mu, const double *rho, const double *const *st, double dt,
                                double alpha, double gamma, double xi, double rho0, double fs);
/* The same step out of place, device pointers only: u is read, u_out (no
   alias of u) receives the updated boxes and u's values everywhere else; the
   update runs inside the flux kernel (no separate pass over u), which suits a
   pipeline that keeps u and u* in two buffers (the projection's _dev form
   reads u* and writes u). */
int tbfp_momentum_predictor_out_dev(tbfp_handle *h, const double *ux, const double *uy, const double *uz,
                                    double *ux_out, double *uy_out, double *uz_out, const double *c, const double *mu,
                                    const double *rho, const double *const *st, double dt, double alpha, double gamma,
                                    double xi, double rho0, double fs);
/* updateBoundariesV (vfield.f90:111-189) for the channel, in place on u: the
   fixedValue walls in y (one ghost layer, boundaryField_S.f90:593-690, with
   the spacings of setMetrics :138-214), the periodic halos in x and z
   (updateHalo, field.f90:708-946, the rank being its own neighbour) and the
   periodic duplicates ux(0,:,:) = ux(nx,:,:), uz(:,:,0) = uz(:,:,nz).  Other
   y-ghost layers are only copied periodically, as in the reference.
   solveMomentumEqn is tbfp_momentum_predictor followed by this call.  Needs
   tbfp_momentum_setup. */
int tbfp_update_boundaries_v(tbfp_handle *h, double *ux, double *uy, double *uz);
int tbfp_update_boundaries_v_dev(tbfp_handle *h, double *ux, double *uy, double *uz);

/* --- flow control (auxiliaryRoutines.f90:336-540) ----------------------- */
/* Volume sums over the ux faces i = 0..nx-1, j = 1..ny, k = 1..nz with the
   staggered volume Vsx = dxc(i+1)*dyf(j)*dzf(k) (grid.f90:812-838):
   tbfp_rho_face_sum: sum of 0.5*(rho(i+1)+rho(i))*Vsx, setPressGrad's rho_sum
   (its mean density is the sum over s_Vg; fs follows on the host);
   tbfp_flow_rate: sum of ux*Vsx, computeFlowRate's Q.  On a slab handle the
   sums cover the local planes and the caller adds them over the ranks (the
   reference's Mpi_Allreduce).  tbfp_add_ux: ux(0:nx,1:ny,1:nz) += uf,
   setFlowRate's shift (updateBoundariesV follows). */
int tbfp_rho_face_sum(tbfp_handle *h, const double *rho, double *sum);
int tbfp_rho_face_sum_dev(tbfp_handle *h, const double *rho, double *sum);
int tbfp_flow_rate(tbfp_handle *h, const double *ux, double *q);
int tbfp_flow_rate_dev(tbfp_handle *h, const double *ux, double *q);
int tbfp_add_ux(tbfp_handle *h, double *ux, double uf);
int tbfp_add_ux_dev(tbfp_handle *h, double *ux, double uf);

/* --- surface tension ---------------------------------------------------- */
/* computeSurfaceTension (VOF.f90:1872-2002): the face force st = sigma * k_f *
   (c(Q) - c(P)) / dc on every face, from the volume fraction c (a cell field
   with rho's layout, hd_rho; ghosts not read: x and z wrap, the walls copy).
   Interface cells as the reference's: mixed eps <= c <= 1-eps, full
   c >= 1-eps (eps = 1e-12), a full cell with an empty 6-neighbour counts as
   mixed with c = 1-2 eps; k_f is the mean curvature of the face's two cells if
   both are mixed, else the mixed one's, else 0.  The curvature of a mixed cell
   is the generalised height-function estimate (computeBlockCurvature,
   :2070-2290) computed over the whole grid rather than per bubble block: nine
   height columns across the cell in the largest normal direction (then the
   second, the third), each walking at most 6 cells toward the full and the
   empty phase and stopping at the walls; a cell with no valid direction gets
   0 where the reference fits a parabola.  Positive for a bubble (c = 1 inside):
   2/R on a sphere.  kappa: NULL, or the curvature as a cell field (rho's layout;
   y ghost rows 0).  st_x, st_y, st_z: the staggered components with halo hd_st,
   every element written (x and z halos periodic; wall faces and y ghost rows
   0), ready for the st_n / st_nm1 arguments of the projection. */
int tbfp_surface_tension(tbfp_handle *h, const double *c, double sigma, double *kappa, double *st_x, double *st_y,
                         double *st_z);
int tbfp_surface_tension_dev(tbfp_handle *h, const double *c, double sigma, double *kappa, double *st_x,
                             double *st_y, double *st_z);

/* --- slab form: one channel split over several GPUs --------------------- */
/* One rank's share of a channel split over P ranks (the reference's pencil
   decomposition with py = 1, pencilDec.f90:359-562): in physical space the z
   planes k0 .. k0+d->nz-1 of nz_total (d describes the local slab: d->nz and
   dzf/dzc are local, d->s_Vg is the whole channel's and must be given), in
   spectral space the wavenumbers kx0 .. kx0+nkx_loc-1.  solveFPS becomes
     tbfp_slab_forward_x(s -> S_z[nx/2+1][nz_loc][ny]),  all-to-all to
     S_x[nkx_loc][nz_total][ny],  tbfp_slab_spectral(S_x),  all-to-all back,
     tbfp_slab_inverse_x(S_z -> psi),  z ghost planes of psi exchanged,
   with the exchanges done by the caller (tbfsolver_b200.dist).  tbfp_rhs_split
   and tbfp_correct on a slab handle read the z neighbours of the end planes
   from the ghost planes (exchanged by the caller) instead of wrapping.
   Spectra are complex FP64, interleaved. */
int tbfp_slab_create(const tbfp_desc *d, int nz_total, int k0, int kx0, int nkx_loc, tbfp_handle **out);
int tbfp_slab_forward_x(tbfp_handle *h, const double *s, double *spec_z);
int tbfp_slab_spectral(tbfp_handle *h, double *spec_x);
int tbfp_slab_inverse_x(tbfp_handle *h, const double *spec_z, double *psi);
/* The packing of the two all-to-alls (no counterpart in the reference, whose
   pencil transposes pack with loops, pencilDec.f90:359-562).  z_start[0..world]:
   the first z plane of every rank's slab in rank order (z_start[world] = the
   channel's nz).  In the first exchange rank p sends S_z[kx range of q][nz_p][ny]
   to rank q -- contiguous slices of its S_z, so S_z is the send buffer as it
   is -- and tbfp_slab_unpack_kx turns the received chunks (in rank order, each
   [nkx_loc][nz_p][ny]) into S_x[nkx_loc][nz][ny].  In the second exchange
   tbfp_slab_pack_z writes S_x as the chunks for every destination q
   ([nkx_loc][nz_q][ny], in rank order); what rank q receives, in rank order, is
   its S_z as it is.  One strided copy on the device each way. */
int tbfp_slab_unpack_kx(tbfp_handle *h, int world, const int *z_start, const double *recv, double *spec_x);
int tbfp_slab_pack_z(tbfp_handle *h, int world, const int *z_start, const double *spec_x, double *send);

/* --- ensemble: many independent channels per GPU ----------------------- */
/* No counterpart in the reference, which runs one channel per job.  Each
   member is a channel with its own descriptor (sizes may differ); its arrays
   are device arrays laid out as for tbfp_projection_dev.  Members run on a
   pool of nstreams streams; the whole step (TBFP_MIXED members with their
   device-side refinement loops included) is captured once as a CUDA graph and
   replayed while the arrays and scalars stay the same.  Calls are synchronous.  Surface tension is not supported in
   an ensemble. */
typedef struct tbfp_ensemble tbfp_ensemble;
typedef struct {
  const double *ux_in, *uy_in, *uz_in; /* u*: read */
  double *ux_out, *uy_out, *uz_out;    /* projected u: written (may alias u*_in) */
  const double *rho, *psi_n, *psi_nm1;
  double *psi;                         /* pressure: written with ghosts */
} tbfp_member_io;
/* Execution forms of an ensemble. */
#define TBFP_ENS_AUTO 0       /* choose by measurement on the first call, cached per device and sizes */
#define TBFP_ENS_GRAPH 1      /* each member's kernels on a pool of streams, one replayed CUDA graph */
#define TBFP_ENS_PERSISTENT 2 /* one persistent launch of every stage of every member (a device work
                                 queue of (member, stage, tile) items with per-member stage counters),
                                 replayed as a CUDA graph; FP64 members with out-of-place velocity,
                                 nx/2 <= 128, nz <= 128, ny <= 256 */
int tbfp_ensemble_create(int n, const tbfp_desc *descs, int nstreams, tbfp_ensemble **out);
int tbfp_ensemble_destroy(tbfp_ensemble *e);
int tbfp_ensemble_size(const tbfp_ensemble *e);
/* Request a form (TBFP_ENS_*); param: blocks per SM of the persistent form (0: as many as fit).
   TBFP_ENS_AUTO, the default, times the graph and the persistent kernel at one and two blocks per
   SM on the first call for a set of arrays (when every member is out of place), keeps the fastest,
   and appends the choice to the tuning cache file: $TBFP_TUNE_CACHE, else
   $XDG_CACHE_HOME/tbfp_tune.txt, else $HOME/.cache/tbfp_tune.txt (one line per decision:
   key, form, param, ms).  An ensemble of the same sizes on the same device reads it back. */
int tbfp_ensemble_set_mode(tbfp_ensemble *e, int mode, int param);
/* The form in use (0 before the first call) and its param; tuned_ms (NULL or 3 entries): the
   measured ms of the graph and of the persistent form at 1 and 2 blocks per SM (-1: not measured). */
int tbfp_ensemble_get_mode(const tbfp_ensemble *e, int *mode, int *param, float *tuned_ms);
/* Bound on each wait of the velocity correction for the bulk copies that stage its inputs in
   shared memory (the FP64 out-of-place correction of tbfp_projection[_dev] and of each ensemble
   member), in SM clock cycles; default 4e9 (about 2 s), 0: a copy not complete at the first look
   counts as late.  A wait that runs out ends the kernel after its copies in flight have landed:
   the call returns TBFP_ETIMEOUT and the handle stays usable.  No counterpart in the reference
   (its loops run on the host and cannot wait on a copy engine). */
int tbfp_set_wait_limit(tbfp_handle *h, long long cycles);
/* Bound on each dependency wait of the persistent kernel, in polls of about 0.1 us (default 1e7,
   about a second).  A wait that runs out stops the launch: the call returns TBFP_ETIMEOUT. */
int tbfp_ensemble_set_wait_limit(tbfp_ensemble *e, long long polls);
/* One projection of every member; stats: NULL or n entries (max_div per member). */
int tbfp_ensemble_projection_dev(tbfp_ensemble *e, const tbfp_member_io *io, double dt, double alpha,
                                 double rho0, tbfp_stats *stats);

/* --- solveFPS without device allocation ------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
   memory (code under a memory pool another runtime owns, or a driver that
   only hands over arrays it allocated itself): the same
   solve as tbfp_solve_fps_dev, on the caller's device arrays s and psi, with no
   handle.  Work spectrum and set-up tables live in one static device array that
   every GPU loading the library holds until exit, which limits the grid to
   (nx/2+1)*ny*nz <= TBFP_NOALLOC_MAX_SPECTRUM complex entries (64 MiB),
   nx <= 4096, ny <= 2048, nz <= 2048 (else TBFP_EUNSUPPORTED).  The first call
   on a device looks up the array's address; make it before any stream capture.
   All calls share the array: calls that overlap on the GPU race.  Runs on
   d->stream (NULL: the legacy default stream), synchronous; the caller's
   current device is restored before returning; error text via
   tbfp_last_error(NULL).  Only the fields nx, ny, nz, hd_psi, dx_fft, dz_fft,
   dxf, dyf, dyc, dzf, s_Vg, device and stream of d are read. */
#define TBFP_NOALLOC_MAX_SPECTRUM 4194304
int tbfp_solve_fps_noalloc(const tbfp_desc *d, const double *s, double *psi);

#ifdef __cplusplus
}
#endif

#endif /* TBFP_H */
