/*
 * tbfp_oracle.c -- C/OpenMP restatement of the reference projection step.
 *
 * TEST INFRASTRUCTURE ONLY: the CPU checker and the timed CPU baseline.  The
 * shipped library never links or calls it.  PARITY UNPINNED: the Fortran
 * reference (cifanip/TBFsolver, FAST_MODE) cannot be built here (no Fortran
 * compiler, MPI, FFTW or LAPACK) and ships no golden vectors; this file is
 * cross-checked against the numpy/scipy oracle (oracle/tbfp_oracle.py, which
 * calls LAPACK's zgttrf/zgttrs) and the analytic fixtures in tests/golden/.
 *
 * One call of tbfo_projection does what main.f90:197-212 does for one rank:
 *   computeSource FAST      poissonEqn.f90:193-305
 *   solveFPS                fastPoissonSolver.f90:337-384
 *     x r2c / z c2c         (FFTW guru plans :160-211; here a Stockham FFT, unnormalised)
 *     solveTriDiag          :280-333 (row scaling, zgttrf, epsilon pivot, zgttrs)
 *     scale 1/(nx*nz)       :374
 *     zeroAveragePressure   :388-423
 *     updateBoundaries      field.f90:950-974 (Neumann y walls, periodic x/z)
 *   makeVelocityDivFree     momentumEqn.f90:999-1127 + equatePeriodicBC vfield.f90:124-189
 *   computeContinuityError  auxiliaryRoutines.f90:42-91 (max|div u|, without dt)
 * The tridiagonal factorisation restates the published LAPACK algorithms
 * ZGTTRF (LU with partial pivoting of a tridiagonal matrix) and ZGTTS2 (the
 * solve behind ZGTTRS) for real coefficients and a complex right-hand side.
 *
 * Array layout: Fortran column-major with halos, as in include/tbfp.h.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double re, im;
} cpx;

typedef struct {
  int ilo, jlo, klo;
  long sj, sk;
} lay_t;

static inline long AT(const lay_t *L, int i, int j, int k) {
  return (long)(i - L->ilo) + (long)(j - L->jlo) * L->sj + (long)(k - L->klo) * L->sk;
}

static lay_t mklay(int ilo, int jlo, int klo, int ni, int nj, int hd) {
  lay_t L;
  L.ilo = ilo - hd;
  L.jlo = jlo - hd;
  L.klo = klo - hd;
  L.sj = ni + 2 * hd;
  L.sk = (long)(ni + 2 * hd) * (nj + 2 * hd);
  return L;
}

/* ------------------------------------------------------------------------- */
/* Stockham FFT (radix 2, 3, 4) with an accurate twiddle table.              */
/* ------------------------------------------------------------------------- */
typedef struct {
  int n, nrad, rad[40];
  cpx *tw; /* exp(-2 pi i m / n) */
} plan_t;

static int make_plan(plan_t *p, int n) {
  p->n = n;
  p->nrad = 0;
  int m = n;
  while (m % 4 == 0) { p->rad[p->nrad++] = 4; m /= 4; }
  while (m % 2 == 0) { p->rad[p->nrad++] = 2; m /= 2; }
  while (m % 3 == 0) { p->rad[p->nrad++] = 3; m /= 3; }
  if (m != 1) return -1;
  p->tw = (cpx *)malloc(sizeof(cpx) * (size_t)n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < n; ++k) {
    long double a = 2.0L * pi * (long double)k / (long double)n;
    p->tw[k].re = (double)cosl(a);
    p->tw[k].im = (double)(-sinl(a));
  }
  return 0;
}

static void free_plan(plan_t *p) { free(p->tw); }

/* x (length n) transformed in place; work must hold n values; sgn = -1 forward, +1 backward. */
static void fft_run(const plan_t *p, cpx *x, cpx *work, int sgn) {
  const int n = p->n;
  cpx *a = x, *b = work;
  int Ns = 1;
  for (int q = 0; q < p->nrad; ++q) {
    const int R = p->rad[q];
    const int per = n / R;
    const int st = n / (Ns * R);
    for (int j = 0; j < per; ++j) {
      const int k0 = j % Ns;
      cpx v[4];
      for (int r = 0; r < R; ++r) {
        cpx t = a[j + r * per];
        if (r > 0) {
          cpx w = p->tw[k0 * r * st];
          if (sgn > 0) w.im = -w.im;
          cpx u = {t.re * w.re - t.im * w.im, t.re * w.im + t.im * w.re};
          t = u;
        }
        v[r] = t;
      }
      cpx y[4];
      if (R == 2) {
        y[0].re = v[0].re + v[1].re; y[0].im = v[0].im + v[1].im;
        y[1].re = v[0].re - v[1].re; y[1].im = v[0].im - v[1].im;
      } else if (R == 4) {
        cpx t0 = {v[0].re + v[2].re, v[0].im + v[2].im}, t1 = {v[0].re - v[2].re, v[0].im - v[2].im};
        cpx t2 = {v[1].re + v[3].re, v[1].im + v[3].im}, d = {v[1].re - v[3].re, v[1].im - v[3].im};
        cpx t3 = (sgn < 0) ? (cpx){d.im, -d.re} : (cpx){-d.im, d.re};
        y[0].re = t0.re + t2.re; y[0].im = t0.im + t2.im;
        y[2].re = t0.re - t2.re; y[2].im = t0.im - t2.im;
        y[1].re = t1.re + t3.re; y[1].im = t1.im + t3.im;
        y[3].re = t1.re - t3.re; y[3].im = t1.im - t3.im;
      } else { /* R == 3 */
        const double c = -0.5, s = (sgn < 0) ? -0.86602540378443864676 : 0.86602540378443864676;
        cpx t = {v[1].re + v[2].re, v[1].im + v[2].im}, d = {v[1].re - v[2].re, v[1].im - v[2].im};
        cpx m = {v[0].re + c * t.re, v[0].im + c * t.im};
        cpx id = {-s * d.im, s * d.re};
        y[0].re = v[0].re + t.re; y[0].im = v[0].im + t.im;
        y[1].re = m.re + id.re; y[1].im = m.im + id.im;
        y[2].re = m.re - id.re; y[2].im = m.im - id.im;
      }
      const int dd = (j / Ns) * Ns * R + k0;
      for (int r = 0; r < R; ++r) b[dd + r * Ns] = y[r];
    }
    cpx *t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  if (a != x) memcpy(x, a, sizeof(cpx) * (size_t)n);
}

/* ------------------------------------------------------------------------- */
/* ZGTTRF / ZGTTS2 restated for real coefficients and a complex RHS.         */
/* dl[0..n-2], d[0..n-1], du[0..n-2], du2[0..n-3], ipiv[0..n-1] (0-based).    */
/* Returns info (0 or the 1-based index of the first exactly-zero pivot).    */
/* ------------------------------------------------------------------------- */
static int gttrf(int n, double *dl, double *d, double *du, double *du2, int *ipiv) {
  for (int i = 0; i < n; ++i) ipiv[i] = i;
  for (int i = 0; i < n - 2; ++i) du2[i] = 0.0;
  for (int i = 0; i < n - 2; ++i) {
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] != 0.0) {
        const double f = dl[i] / d[i];
        dl[i] = f;
        d[i + 1] = d[i + 1] - f * du[i];
      }
    } else {
      const double f = d[i] / dl[i];
      d[i] = dl[i];
      dl[i] = f;
      const double t = du[i];
      du[i] = d[i + 1];
      d[i + 1] = t - f * d[i + 1];
      du2[i] = du[i + 1];
      du[i + 1] = -f * du[i + 1];
      ipiv[i] = i + 1;
    }
  }
  if (n > 1) {
    const int i = n - 2;
    if (fabs(d[i]) >= fabs(dl[i])) {
      if (d[i] != 0.0) {
        const double f = dl[i] / d[i];
        dl[i] = f;
        d[i + 1] = d[i + 1] - f * du[i];
      }
    } else {
      const double f = d[i] / dl[i];
      d[i] = dl[i];
      dl[i] = f;
      const double t = du[i];
      du[i] = d[i + 1];
      d[i + 1] = t - f * d[i + 1];
      ipiv[i] = i + 1;
    }
  }
  for (int i = 0; i < n; ++i)
    if (d[i] == 0.0) return i + 1;
  return 0;
}

static void gtts2(int n, const double *dl, const double *d, const double *du, const double *du2, const int *ipiv,
                  cpx *b) {
  for (int i = 0; i < n - 1; ++i) {
    if (ipiv[i] == i) {
      b[i + 1].re -= dl[i] * b[i].re;
      b[i + 1].im -= dl[i] * b[i].im;
    } else {
      const cpx t = b[i];
      b[i] = b[i + 1];
      b[i + 1].re = t.re - dl[i] * b[i].re;
      b[i + 1].im = t.im - dl[i] * b[i].im;
    }
  }
  b[n - 1].re /= d[n - 1];
  b[n - 1].im /= d[n - 1];
  if (n > 1) {
    b[n - 2].re = (b[n - 2].re - du[n - 2] * b[n - 1].re) / d[n - 2];
    b[n - 2].im = (b[n - 2].im - du[n - 2] * b[n - 1].im) / d[n - 2];
  }
  for (int i = n - 3; i >= 0; --i) {
    b[i].re = (b[i].re - du[i] * b[i + 1].re - du2[i] * b[i + 2].re) / d[i];
    b[i].im = (b[i].im - du[i] * b[i + 1].im - du2[i] * b[i + 2].im) / d[i];
  }
}

/* ------------------------------------------------------------------------- */
typedef struct {
  int nx, ny, nz, hd_psi, hd_u, hd_rho;
  const double *dxf, *dxc, *dyf, *dyc, *dzf, *dzc; /* dxf[i-1] = dxf(i), dxc[i-1] = dxc(i), ... */
  double dx_fft, dz_fft, s_Vg;
} tbfo_grid;

/* computeSource FAST (poissonEqn.f90:224-253, computeOldPressDiv :270-301), no surface tension. */
static void compute_source(const tbfo_grid *g, const double *ux, const double *uy, const double *uz,
                           const double *rho, const double *pn, const double *po, double dt, double alpha,
                           double rho0, double *s /* interior nx*ny*nz, i fastest */) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const lay_t Lu = mklay(0, 1, 1, nx + 1, ny, g->hd_u), Lv = mklay(1, 0, 1, nx, ny + 1, g->hd_u),
              Lw = mklay(1, 1, 0, nx, ny, g->hd_u), Lr = mklay(1, 1, 1, nx, ny, g->hd_rho),
              Lp = mklay(1, 1, 1, nx, ny, g->hd_psi);
  const double r = 1.0 / (alpha * dt);
  const double dxf1 = g->dxf[0], dzf1 = g->dzf[0], dxc1 = g->dxc[0], dzc1 = g->dzc[0];
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) {
      const double dyfj = g->dyf[j - 1], dycp = g->dyc[j], dycm = g->dyc[j - 1];
      for (int i = 1; i <= nx; ++i) {
        double ddx = (ux[AT(&Lu, i, j, k)] - ux[AT(&Lu, i - 1, j, k)]) / dxf1;
        double ddy = (uy[AT(&Lv, i, j, k)] - uy[AT(&Lv, i, j - 1, k)]) / dyfj;
        double ddz = (uz[AT(&Lw, i, j, k)] - uz[AT(&Lw, i, j, k - 1)]) / dzf1;
        double sv = (ddx + ddy + ddz) * r * rho0;
        const long c = AT(&Lr, i, j, k);
        const double irc = 1.0 / rho[c];
        const double apx = 1.0 - rho0 * 0.5 * (1.0 / rho[c + 1] + irc);
        const double amx = 1.0 - rho0 * 0.5 * (1.0 / rho[c - 1] + irc);
        const double apy = 1.0 - rho0 * 0.5 * (1.0 / rho[c + Lr.sj] + irc);
        const double amy = 1.0 - rho0 * 0.5 * (1.0 / rho[c - Lr.sj] + irc);
        const double apz = 1.0 - rho0 * 0.5 * (1.0 / rho[c + Lr.sk] + irc);
        const double amz = 1.0 - rho0 * 0.5 * (1.0 / rho[c - Lr.sk] + irc);
        const long p = AT(&Lp, i, j, k);
        const long sj = Lp.sj, sk = Lp.sk;
        const double pc = pn[p], oc = po[p];
        const double dpxp = (2.0 * (pn[p + 1] - pc) - (po[p + 1] - oc)) / dxc1;
        const double dpxm = (2.0 * (pc - pn[p - 1]) - (oc - po[p - 1])) / dxc1;
        const double dpyp = (2.0 * (pn[p + sj] - pc) - (po[p + sj] - oc)) / dycp;
        const double dpym = (2.0 * (pc - pn[p - sj]) - (oc - po[p - sj])) / dycm;
        const double dpzp = (2.0 * (pn[p + sk] - pc) - (po[p + sk] - oc)) / dzc1;
        const double dpzm = (2.0 * (pc - pn[p - sk]) - (oc - po[p - sk])) / dzc1;
        sv = sv + (apx * dpxp - amx * dpxm) / dxf1 + (apy * dpyp - amy * dpym) / dyfj + (apz * dpzp - amz * dpzm) / dzf1;
        s[((long)(k - 1) * ny + (j - 1)) * nx + (i - 1)] = sv;
      }
    }
}

/* solveFPS (fastPoissonSolver.f90:337-384): s interior -> psi with ghosts. */
static int solve_fps(const tbfo_grid *g, const double *s, double *psi, int nthreads, int pin00) {
  const int nx = g->nx, ny = g->ny, nz = g->nz, nkx = nx / 2 + 1;
  const long R = (long)ny * nz;
  plan_t px, pz;
  if (make_plan(&px, nx) || make_plan(&pz, nz)) return -1;
  cpx *S = (cpx *)malloc(sizeof(cpx) * (size_t)nkx * R); /* S[(kx*nz + k)*ny + j] */
  if (!S) return -2;
  const double pi = 3.14159265358979323846;
  double *lx = (double *)malloc(sizeof(double) * nkx), *lz = (double *)malloc(sizeof(double) * nz);
  double *am = (double *)malloc(sizeof(double) * ny), *ap = (double *)malloc(sizeof(double) * ny);
  for (int i = 0; i < nkx; ++i) lx[i] = 2.0 * (cos((i * 2.0 * pi) / nx) - 1.0) / (g->dx_fft * g->dx_fft);
  for (int k = 0; k < nz; ++k) lz[k] = 2.0 * (cos((k * 2.0 * pi) / nz) - 1.0) / (g->dz_fft * g->dz_fft);
  for (int j = 0; j < ny; ++j) {
    am[j] = 1.0 / (g->dyc[j] * g->dyf[j]);
    ap[j] = 1.0 / (g->dyc[j + 1] * g->dyf[j]);
  }
  am[0] = 0.0;
  ap[ny - 1] = 0.0;
  /* forward x (r2c via a full complex transform of the real row) */
#pragma omp parallel num_threads(nthreads)
  {
    cpx *row = (cpx *)malloc(sizeof(cpx) * nx), *work = (cpx *)malloc(sizeof(cpx) * nx);
#pragma omp for schedule(static)
    for (long rr = 0; rr < R; ++rr) {
      const double *src = s + rr * nx;
      for (int i = 0; i < nx; ++i) { row[i].re = src[i]; row[i].im = 0.0; }
      fft_run(&px, row, work, -1);
      const int k = (int)(rr / ny), j = (int)(rr % ny);
      for (int kx = 0; kx < nkx; ++kx) S[((long)kx * nz + k) * ny + j] = row[kx];
    }
    free(row);
    free(work);
  }
  /* forward z, tridiagonal y, backward z: per kx plane */
#pragma omp parallel num_threads(nthreads)
  {
    cpx *col = (cpx *)malloc(sizeof(cpx) * nz), *work = (cpx *)malloc(sizeof(cpx) * (nz > ny ? nz : ny));
    double *dl = (double *)malloc(sizeof(double) * ny), *d = (double *)malloc(sizeof(double) * ny);
    double *du = (double *)malloc(sizeof(double) * ny), *du2 = (double *)malloc(sizeof(double) * ny);
    int *ipiv = (int *)malloc(sizeof(int) * ny);
    cpx *fy = (cpx *)malloc(sizeof(cpx) * ny);
#pragma omp for schedule(static)
    for (long q = 0; q < (long)nkx * ny; ++q) {
      const int kx = (int)(q / ny), j = (int)(q % ny);
      cpx *base = S + (long)kx * R + j;
      for (int k = 0; k < nz; ++k) col[k] = base[(long)k * ny];
      fft_run(&pz, col, work, -1);
      for (int k = 0; k < nz; ++k) base[(long)k * ny] = col[k];
    }
#pragma omp for schedule(static)
    for (long q = 0; q < (long)nkx * nz; ++q) {
      const int kx = (int)(q / nz), kz = (int)(q % nz);
      cpx *sys = S + (long)kx * R + (long)kz * ny;
      for (int j = 0; j < ny; ++j) {
        const double r = 1.0 / (lx[kx] + lz[kz] - am[j] - ap[j]);
        if (j > 0) dl[j - 1] = am[j] * r;
        if (j < ny - 1) du[j] = ap[j] * r;
        d[j] = 1.0;
        fy[j].re = sys[j].re * r;
        fy[j].im = sys[j].im * r;
      }
      if (pin00 && kx == 0 && kz == 0) { /* exact gauge: last equation x_ny = 0 */
        dl[ny - 2] = 0.0;
        fy[ny - 1].re = 0.0;
        fy[ny - 1].im = 0.0;
      }
      const int info = gttrf(ny, dl, d, du, du2, ipiv);
      if (info != 0) d[ny - 1] = 2.220446049250313e-16; /* epsilon(0.d0), :318-322 */
      gtts2(ny, dl, d, du, du2, ipiv, fy);
      memcpy(sys, fy, sizeof(cpx) * ny);
    }
#pragma omp for schedule(static)
    for (long q = 0; q < (long)nkx * ny; ++q) {
      const int kx = (int)(q / ny), j = (int)(q % ny);
      cpx *base = S + (long)kx * R + j;
      for (int k = 0; k < nz; ++k) col[k] = base[(long)k * ny];
      fft_run(&pz, col, work, +1);
      for (int k = 0; k < nz; ++k) base[(long)k * ny] = col[k];
    }
    free(col); free(work); free(dl); free(d); free(du); free(du2); free(ipiv); free(fy);
  }
  /* backward x (c2r: Hermitian extension, imaginary parts of DC/Nyquist dropped), scale */
  const lay_t Lp = mklay(1, 1, 1, nx, ny, g->hd_psi);
  const double scale = (double)nx * (double)nz;
#pragma omp parallel num_threads(nthreads)
  {
    cpx *row = (cpx *)malloc(sizeof(cpx) * nx), *work = (cpx *)malloc(sizeof(cpx) * nx);
#pragma omp for schedule(static)
    for (long rr = 0; rr < R; ++rr) {
      const int k = (int)(rr / ny), j = (int)(rr % ny);
      for (int kx = 0; kx < nkx; ++kx) row[kx] = S[((long)kx * nz + k) * ny + j];
      row[0].im = 0.0;
      row[nx / 2].im = 0.0;
      for (int kx = nkx; kx < nx; ++kx) { row[kx].re = row[nx - kx].re; row[kx].im = -row[nx - kx].im; }
      fft_run(&px, row, work, +1);
      for (int i = 0; i < nx; ++i) psi[AT(&Lp, i + 1, j + 1, k + 1)] = row[i].re / scale;
    }
    free(row);
    free(work);
  }
  /* zeroAveragePressure */
  double av = 0.0;
#pragma omp parallel for reduction(+ : av) collapse(2) num_threads(nthreads)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) av += psi[AT(&Lp, i, j, k)] * (g->dxf[i - 1] * g->dyf[j - 1] * g->dzf[k - 1]);
  const double avg = av / g->s_Vg;
  const long ntot = (long)(nx + 2 * g->hd_psi) * (ny + 2 * g->hd_psi) * (nz + 2 * g->hd_psi);
#pragma omp parallel for num_threads(nthreads)
  for (long t = 0; t < ntot; ++t) psi[t] -= avg;
  /* updateBoundaries: y walls, then periodic x, then periodic z */
  const int hd = g->hd_psi;
  for (int k = 1; k <= nz; ++k)
    for (int i = 1; i <= nx; ++i) {
      psi[AT(&Lp, i, 0, k)] = psi[AT(&Lp, i, 1, k)];
      psi[AT(&Lp, i, ny + 1, k)] = psi[AT(&Lp, i, ny, k)];
    }
  for (int k = 1 - hd; k <= nz + hd; ++k)
    for (int j = 1 - hd; j <= ny + hd; ++j)
      for (int h = 0; h < hd; ++h) {
        psi[AT(&Lp, nx + 1 + h, j, k)] = psi[AT(&Lp, 1 + h, j, k)];
        psi[AT(&Lp, 1 - hd + h, j, k)] = psi[AT(&Lp, nx - hd + 1 + h, j, k)];
      }
  for (int h = 0; h < hd; ++h)
    for (int j = 1 - hd; j <= ny + hd; ++j)
      for (int i = 1 - hd; i <= nx + hd; ++i) {
        psi[AT(&Lp, i, j, nz + 1 + h)] = psi[AT(&Lp, i, j, 1 + h)];
        psi[AT(&Lp, i, j, 1 - hd + h)] = psi[AT(&Lp, i, j, nz - hd + 1 + h)];
      }
  free(S); free(lx); free(lz); free(am); free(ap);
  free_plan(&px);
  free_plan(&pz);
  return 0;
}

/* makeVelocityDivFree FAST (momentumEqn.f90:1017-1084) in place, then the periodic equate. */
static void correct(const tbfo_grid *g, double *ux, double *uy, double *uz, const double *psi, const double *pn,
                    const double *po, const double *rho, double dt, double alpha, double rho0, int nthreads) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const lay_t Lu = mklay(0, 1, 1, nx + 1, ny, g->hd_u), Lv = mklay(1, 0, 1, nx, ny + 1, g->hd_u),
              Lw = mklay(1, 1, 0, nx, ny, g->hd_u), Lr = mklay(1, 1, 1, nx, ny, g->hd_rho),
              Lp = mklay(1, 1, 1, nx, ny, g->hd_psi);
  const double r = dt * alpha, ir0 = 1.0 / rho0, dxc1 = g->dxc[0], dzc1 = g->dzc[0];
#pragma omp parallel for collapse(2) num_threads(nthreads)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        const long c = AT(&Lr, i, j, k), p = AT(&Lp, i, j, k);
        const double ir = 0.5 * (1.0 / rho[c + 1] + 1.0 / rho[c]);
        const double dpr = (psi[p + 1] - psi[p]) / dxc1;
        const double dpr0 = (2.0 * (pn[p + 1] - pn[p]) - (po[p + 1] - po[p])) / dxc1;
        ux[AT(&Lu, i, j, k)] -= r * (ir0 * dpr + (ir - ir0) * dpr0);
      }
#pragma omp parallel for collapse(2) num_threads(nthreads)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny - 1; ++j)
      for (int i = 1; i <= nx; ++i) {
        const long c = AT(&Lr, i, j, k), p = AT(&Lp, i, j, k);
        const double ir = 0.5 * (1.0 / rho[c + Lr.sj] + 1.0 / rho[c]);
        const double dy = g->dyc[j];
        const double dpr = (psi[p + Lp.sj] - psi[p]) / dy;
        const double dpr0 = (2.0 * (pn[p + Lp.sj] - pn[p]) - (po[p + Lp.sj] - po[p])) / dy;
        uy[AT(&Lv, i, j, k)] -= r * (ir0 * dpr + (ir - ir0) * dpr0);
      }
#pragma omp parallel for collapse(2) num_threads(nthreads)
  for (int k = 0; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const long c = AT(&Lr, i, j, k), p = AT(&Lp, i, j, k);
        const double ir = 0.5 * (1.0 / rho[c + Lr.sk] + 1.0 / rho[c]);
        const double dpr = (psi[p + Lp.sk] - psi[p]) / dzc1;
        const double dpr0 = (2.0 * (pn[p + Lp.sk] - pn[p]) - (po[p + Lp.sk] - po[p])) / dzc1;
        uz[AT(&Lw, i, j, k)] -= r * (ir0 * dpr + (ir - ir0) * dpr0);
      }
  /* equatePeriodicBC on the interior rows */
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j) ux[AT(&Lu, 0, j, k)] = ux[AT(&Lu, nx, j, k)];
  for (int j = 1; j <= ny; ++j)
    for (int i = 1; i <= nx; ++i) uz[AT(&Lw, i, j, 0)] = uz[AT(&Lw, i, j, nz)];
}

static double max_div(const tbfo_grid *g, const double *ux, const double *uy, const double *uz, int nthreads) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const lay_t Lu = mklay(0, 1, 1, nx + 1, ny, g->hd_u), Lv = mklay(1, 0, 1, nx, ny + 1, g->hd_u),
              Lw = mklay(1, 1, 0, nx, ny, g->hd_u);
  double m = -1.0;
#pragma omp parallel for reduction(max : m) collapse(2) num_threads(nthreads)
  for (int k = 1; k <= nz; ++k)
    for (int j = 1; j <= ny; ++j)
      for (int i = 1; i <= nx; ++i) {
        const double d = (ux[AT(&Lu, i, j, k)] - ux[AT(&Lu, i - 1, j, k)]) / g->dxf[i - 1] +
                         (uy[AT(&Lv, i, j, k)] - uy[AT(&Lv, i, j - 1, k)]) / g->dyf[j - 1] +
                         (uz[AT(&Lw, i, j, k)] - uz[AT(&Lw, i, j, k - 1)]) / g->dzf[k - 1];
        if (fabs(d) > m) m = fabs(d);
      }
  return m;
}

/* One projection.  u* is read from ux..uz and the projected velocity written
   back in place; psi receives the pressure with ghosts.  pin00 = 0 keeps the
   reference's epsilon pivot for the singular (0,0) system; pin00 = 1 gauges it
   exactly (last unknown pinned).  Returns 0 on success. */
int tbfo_projection(int nx, int ny, int nz, int hd_psi, int hd_u, int hd_rho, const double *dxf, const double *dxc,
                    const double *dyf, const double *dyc, const double *dzf, const double *dzc, double dx_fft,
                    double dz_fft, double s_Vg, double *ux, double *uy, double *uz, const double *rho,
                    const double *psi_n, const double *psi_nm1, double dt, double alpha, double rho0, double *psi,
                    double *out_max_div, int nthreads, int pin00) {
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  omp_set_num_threads(nthreads);
  tbfo_grid g = {nx, ny, nz, hd_psi, hd_u, hd_rho, dxf, dxc, dyf, dyc, dzf, dzc, dx_fft, dz_fft, s_Vg};
  double *s = (double *)malloc(sizeof(double) * (size_t)nx * ny * nz);
  if (!s) return -2;
  compute_source(&g, ux, uy, uz, rho, psi_n, psi_nm1, dt, alpha, rho0, s);
  int rc = solve_fps(&g, s, psi, nthreads, pin00);
  free(s);
  if (rc) return rc;
  correct(&g, ux, uy, uz, psi, psi_n, psi_nm1, rho, dt, alpha, rho0, nthreads);
  if (out_max_div) *out_max_div = max_div(&g, ux, uy, uz, nthreads);
  return 0;
}

int tbfo_max_threads(void) { return omp_get_max_threads(); }
