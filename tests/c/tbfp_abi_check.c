/* A C caller of the library, compiled against include/tbfp.h by the tests so
 * that the header is checked by a C compiler (gcc -std=c99 -Wall -Wextra
 * -Werror -pedantic), not only by ctypes.
 *
 *   tbfp_abi_check cpu        calls that need no GPU: version, status texts,
 *                             descriptor validation before any device work
 *   tbfp_abi_check gpu OUT    one solveFPS on a 32x24x16 tanh grid through the
 *                             host-pointer entry point; writes psi to OUT
 *
 * Exit status 0 on success.  The grid metrics follow the reference's tanh
 * channel (grid.f90:288-330, gamma 1.5): faces yf(j) = 1 + tanh(g (2j/ny - 1))
 * / tanh(g), centres yc(j) = the same map at j - 1/2, j = 0..ny+1. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "tbfp.h"

#define NX 32
#define NY 24
#define NZ 16

static int fail(const char *what, int rc) {
  fprintf(stderr, "%s: %d (%s) %s\n", what, rc, tbfp_strerror(rc), tbfp_last_error(NULL));
  return 1;
}

static void metrics(double *dxf, double *dxc, double *dyf, double *dyc, double *dzf, double *dzc, double *dx,
                    double *dz) {
  const double pi = 3.14159265358979323846, g = 1.5;
  double yf[NY + 1], yc[NY + 2];
  int i;
  *dx = 2.0 * pi / NX;
  *dz = pi / NZ;
  for (i = 0; i < NX; ++i) dxf[i] = *dx;
  for (i = 0; i <= NX; ++i) dxc[i] = *dx;
  for (i = 0; i < NZ; ++i) dzf[i] = *dz;
  for (i = 0; i <= NZ; ++i) dzc[i] = *dz;
  for (i = 0; i <= NY; ++i) yf[i] = 1.0 + tanh(g * (2.0 * i / NY - 1.0)) / tanh(g);
  /* centres: the same map at half-integer indices, ghost centres included */
  for (i = 0; i <= NY + 1; ++i) yc[i] = 1.0 + tanh(g * ((2.0 * i - 1.0) / NY - 1.0)) / tanh(g);
  for (i = 0; i < NY; ++i) dyf[i] = yf[i + 1] - yf[i];
  for (i = 0; i <= NY; ++i) dyc[i] = yc[i + 1] - yc[i];
}

static tbfp_desc make_desc(double *m[6], double dx, double dz) {
  tbfp_desc d;
  memset(&d, 0, sizeof(d));
  d.nx = NX;
  d.ny = NY;
  d.nz = NZ;
  d.hd_psi = 1;
  d.hd_u = 2;
  d.hd_rho = 1;
  d.hd_st = 1;
  d.dx_fft = dx;
  d.dz_fft = dz;
  d.dxf = m[0];
  d.dxc = m[1];
  d.dyf = m[2];
  d.dyc = m[3];
  d.dzf = m[4];
  d.dzc = m[5];
  d.s_Vg = 0.0;
  d.precision = TBFP_FP64;
  d.tol = 1e-10;
  d.max_iter = 4;
  d.device = -1;
  d.stream = NULL;
  d.flags = 0u;
  return d;
}

int main(int argc, char **argv) {
  double dxf[NX], dxc[NX + 1], dyf[NY], dyc[NY + 1], dzf[NZ], dzc[NZ + 1], dx, dz;
  double *m[6];
  tbfp_desc d;
  tbfp_handle *h = NULL;
  int rc, code;
  m[0] = dxf;
  m[1] = dxc;
  m[2] = dyf;
  m[3] = dyc;
  m[4] = dzf;
  m[5] = dzc;
  metrics(dxf, dxc, dyf, dyc, dzf, dzc, &dx, &dz);
  if (argc < 2) return 2;

  if (strcmp(argv[1], "cpu") == 0) {
    if (tbfp_abi_version() != TBFP_ABI_VERSION) return fail("abi version", tbfp_abi_version());
    for (code = TBFP_ESINGULAR; code <= TBFP_ENOTCONVERGED; ++code)
      if (!tbfp_strerror(code) || strcmp(tbfp_strerror(code), "unknown status") == 0) return fail("strerror", code);
    d = make_desc(m, dx, dz);
    d.nx = NX - 1; /* odd: no real-to-complex transform along x */
    rc = tbfp_create(&d, &h);
    if (rc != TBFP_EINVAL || h != NULL) return fail("odd nx accepted", rc);
    d = make_desc(m, dx, dz);
    d.dyf = NULL;
    rc = tbfp_create(&d, &h);
    if (rc != TBFP_ENULL) return fail("NULL metric accepted", rc);
    if (tbfp_solve_fps(NULL, NULL, NULL) != TBFP_ENULL) return fail("NULL handle accepted", 0);
    if (tbfp_destroy(NULL) != TBFP_OK) return fail("destroy(NULL)", 0);
    printf("cpu checks ok\n");
    return 0;
  }

  if (strcmp(argv[1], "gpu") == 0 && argc >= 3) {
    const size_t n = (size_t)(NX + 2) * (NY + 2) * (NZ + 2);
    double *s = (double *)calloc(n, sizeof(double)), *psi = (double *)calloc(n, sizeof(double));
    double vol = 0.0, mean = 0.0;
    int i, j, k;
    FILE *f;
    if (!s || !psi) return 3;
    /* a smooth source with zero volume integral on the interior (compatible with the walls) */
    for (k = 1; k <= NZ; ++k)
      for (j = 1; j <= NY; ++j)
        for (i = 1; i <= NX; ++i) {
          const double v = cos(2.0 * i * dx) * sin((double)j) + 0.25 * cos(3.0 * k * dz);
          const double w = dxf[i - 1] * dyf[j - 1] * dzf[k - 1];
          s[(size_t)i + (NX + 2) * ((size_t)j + (NY + 2) * (size_t)k)] = v;
          mean += v * w;
          vol += w;
        }
    for (k = 1; k <= NZ; ++k)
      for (j = 1; j <= NY; ++j)
        for (i = 1; i <= NX; ++i) s[(size_t)i + (NX + 2) * ((size_t)j + (NY + 2) * (size_t)k)] -= mean / vol;
    d = make_desc(m, dx, dz);
    rc = tbfp_create(&d, &h);
    if (rc != TBFP_OK) return fail("tbfp_create", rc);
    rc = tbfp_solve_fps(h, s, psi);
    if (rc != TBFP_OK) return fail("tbfp_solve_fps", rc);
    tbfp_destroy(h);
    f = fopen(argv[2], "wb");
    if (!f || fwrite(psi, sizeof(double), n, f) != n) return 4;
    fclose(f);
    free(s);
    free(psi);
    printf("gpu solve ok\n");
    return 0;
  }
  return 2;
}
