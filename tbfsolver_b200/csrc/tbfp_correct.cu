// FP64 velocity correction and continuity check of the split-pressure
// projection (FAST_MODE of the reference).
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"

namespace tbfp {

// ---------------------------------------------------------------------------
// Velocity correction (makeVelocityDivFree FAST, momentumEqn.f90:999-1127):
//   u_d -= dt*alpha*[ (1/rho0) d psi + (1/rho_f - 1/rho0)(2 d psi^n - d psi^{n-1} - (2 st^n - st^{n-1})) ]
// One face value per helper; faces are indexed like the staggered arrays.
// ---------------------------------------------------------------------------
template <bool ST>
__device__ __forceinline__ double corr_x(const CorrArgs &a, const GridK &g, int i, int j, int k) {
  const long pc = at(a.Lpsi, i, j, k), rc = at(a.Lrho, i, j, k);
  const double invrho = 0.5 * (a.irho[rc + 1] + a.irho[rc]);
  const double dpr = (a.psi[pc + 1] - a.psi[pc]) * g.idxc1;
  double dpr0 = (2.0 * (a.pn[pc + 1] - a.pn[pc]) - (a.pnm1[pc + 1] - a.pnm1[pc])) * g.idxc1;
  if constexpr (ST) {
    const long q = at(a.Lst[0], i, j, k);
    dpr0 = dpr0 - 2.0 * a.stn[0][q] + a.sto[0][q];
  }
  return a.uxi[at(a.Lux, i, j, k)] - a.r * (a.invrho0 * dpr + (invrho - a.invrho0) * dpr0);
}
template <bool ST>
__device__ __forceinline__ double corr_y(const CorrArgs &a, const GridK &g, int i, int j, int k) {
  const long pc = at(a.Lpsi, i, j, k), rc = at(a.Lrho, i, j, k);
  const long sj = a.Lpsi.sj;
  const double invrho = 0.5 * (a.irho[rc + a.Lrho.sj] + a.irho[rc]);
  const double idy = g.idyc[j];  // 1/dyc(j+1)
  const double dpr = (a.psi[pc + sj] - a.psi[pc]) * idy;
  double dpr0 = (2.0 * (a.pn[pc + sj] - a.pn[pc]) - (a.pnm1[pc + sj] - a.pnm1[pc])) * idy;
  if constexpr (ST) {
    const long q = at(a.Lst[1], i, j, k);
    dpr0 = dpr0 - 2.0 * a.stn[1][q] + a.sto[1][q];
  }
  return a.uyi[at(a.Luy, i, j, k)] - a.r * (a.invrho0 * dpr + (invrho - a.invrho0) * dpr0);
}
template <bool ST>
__device__ __forceinline__ double corr_z(const CorrArgs &a, const GridK &g, int i, int j, int k) {
  const long pc = at(a.Lpsi, i, j, k), rc = at(a.Lrho, i, j, k);
  const long sk = a.Lpsi.sk;
  const double invrho = 0.5 * (a.irho[rc + a.Lrho.sk] + a.irho[rc]);
  const double dpr = (a.psi[pc + sk] - a.psi[pc]) * g.idzc1;
  double dpr0 = (2.0 * (a.pn[pc + sk] - a.pn[pc]) - (a.pnm1[pc + sk] - a.pnm1[pc])) * g.idzc1;
  if constexpr (ST) {
    const long q = at(a.Lst[2], i, j, k);
    dpr0 = dpr0 - 2.0 * a.stn[2][q] + a.sto[2][q];
  }
  return a.uzi[at(a.Luz, i, j, k)] - a.r * (a.invrho0 * dpr + (invrho - a.invrho0) * dpr0);
}

__device__ __forceinline__ void block_max_atomic(double v, unsigned long long *out) {
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) v = nanmax_nonneg(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = nanmax_nonneg(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (l == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
  }
}

// Out-of-place correction fused with the continuity check.  Grid (x tiles of
// 128, y chunks of kJC rows, nz); a thread owns column (i, k) of a y chunk and
// walks it in j with one pointer per array and neighbour, so the lower y face
// of a cell is the upper face computed one step before.  Every thread computes
// both of its x faces (the lower one is the upper face of cell i-1, or of cell
// nx at i = 1: the periodic image), which keeps the warp free of divergent
// recomputation.  The periodic duplicates ux(0)=ux(nx), uz(.,.,0)=uz(.,.,nz) are
// the equated values of vfield.f90:124-189 and the uy wall faces are copied
// through.  |div u| (auxiliaryRoutines.f90:71-75) is reduced per block and
// folded into *maxdiv with one atomic.
constexpr int kJC = 32;

// Face update of makeVelocityDivFree FAST for one face: u - r*(invrho0*dpr + (invrho-invrho0)*dpr0),
// dpr = (psi+ - psi)*idc, dpr0 = (2(pn+ - pn) - (po+ - po))*idc [- 2 st^n + st^{n-1}].
__device__ __forceinline__ double face_update(double u, double r, double ir0, double irp, double irc, double idc,
                                              double ps_p, double ps_c, double pn_p, double pn_c, double po_p,
                                              double po_c, double st) {
  const double invrho = 0.5 * (irp + irc);
  const double dpr = (ps_p - ps_c) * idc;
  const double dpr0 = (2.0 * (pn_p - pn_c) - (po_p - po_c)) * idc - st;
  return u - r * (ir0 * dpr + (invrho - ir0) * dpr0);
}

template <bool ST>
__global__ void __launch_bounds__(128, 8) k_correct_div(CorrArgs a, GridK g, unsigned long long *__restrict__ maxdiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.z + 1;
  const int j0 = blockIdx.y * kJC + 1, j1 = min(j0 + kJC - 1, g.ny);
  const bool valid = i <= g.nx;
  const int ic = valid ? i : g.nx;  // clamped index keeps every load in bounds
  const int km = (k == 1 && !g.slab) ? g.nz : k - 1;
  // 32-bit element offsets (tbfp_create checks every array has < 2^31 elements)
  const int pjs = (int)a.Lpsi.sj, rjs = (int)a.Lrho.sj;
  const int xjs = (int)a.Lux.sj, yjs = (int)a.Luy.sj, zjs = (int)a.Luz.sj;
  // offset of the lower x neighbour's centre: cell i-1, or cell nx at i = 1
  const int xo = (ic == 1) ? g.nx - 1 : -1;
  int op = (int)at(a.Lpsi, ic, j0, k), oq = (int)at(a.Lrho, ic, j0, k);
  const int pz = (int)a.Lpsi.sk, pm = (km - k) * (int)a.Lpsi.sk;
  const int qz = (int)a.Lrho.sk, qm = (km - k) * (int)a.Lrho.sk;
  int ox = (int)at(a.Lux, ic, j0, k), oy = (int)at(a.Luy, ic, j0, k), oz = (int)at(a.Luz, ic, j0, k);
  const int zm = (km - k) * (int)a.Luz.sk;
  const double *__restrict__ ps = a.psi;
  const double *__restrict__ pn = a.pn;
  const double *__restrict__ po = a.pnm1;
  const double *__restrict__ ir = a.irho;
  const double *__restrict__ uxi = a.uxi;
  const double *__restrict__ uyi = a.uyi;
  const double *__restrict__ uzi = a.uzi;
  double *__restrict__ uxo = a.uxo;
  double *__restrict__ uyo = a.uyo;
  double *__restrict__ uzo = a.uzo;
  const double r = a.r, ir0 = a.invrho0;
  const double idxc = g.idxc1, idzc = g.idzc1;
  const double idx = g.idxf[ic - 1], idz = g.idzf[k - 1];
  // surface-tension terms of one face (zero without surface tension)
  auto stf = [&](int c, int ii, int jj, int kk) -> double {
    if constexpr (ST) {
      const long q = at(a.Lst[c], ii, jj, kk);
      return 2.0 * a.stn[c][q] - a.sto[c][q];
    } else return 0.0;
  };

  // centre values of the current cell, carried along j
  double psc = ps[op], pnc = pn[op], poc = po[op], irc = ir[oq];
  double uym;
  if (j0 > 1) {
    uym = face_update(uyi[oy - yjs], r, ir0, irc, ir[oq - rjs], g.idyc[j0 - 1], psc, ps[op - pjs], pnc,
                      pn[op - pjs], poc, po[op - pjs], stf(1, ic, j0 - 1, k));
  } else {
    uym = uyi[oy - yjs];
    if (valid) uyo[oy - yjs] = uym;
  }
  double vmax = 0.0;
  for (int j = j0; j <= j1; ++j) {
    // every load of this step, issued together
    const int ow = op + xo, qw = oq + xo;
    const double psx = ps[op + 1], pnx = pn[op + 1], pox = po[op + 1], irx = ir[oq + 1];
    // the lower x face is the upper face of lane - 1; lane 0 computes it
    const bool lead = (threadIdx.x & 31) == 0;
    double psw = 0.0, pnw = 0.0, pow_ = 0.0, irw = 0.0, psw1 = 0.0, pnw1 = 0.0, pow1 = 0.0, irw1 = 0.0, ux_w = 0.0;
    if (lead) {
      psw = ps[ow];
      pnw = pn[ow];
      pow_ = po[ow];
      irw = ir[qw];
      psw1 = ps[ow + 1];
      pnw1 = pn[ow + 1];
      pow1 = po[ow + 1];
      irw1 = ir[qw + 1];
      ux_w = uxi[ox + xo];
    }
    const double psy = ps[op + pjs], pny = pn[op + pjs], poy = po[op + pjs], iry = ir[oq + rjs];
    const double psz = ps[op + pz], pnz = pn[op + pz], poz = po[op + pz], irz = ir[oq + qz];
    const double psm = ps[op + pm], pnm = pn[op + pm], pom = po[op + pm], irm = ir[oq + qm];
    const double ux_c = uxi[ox], uy_c = uyi[oy], uz_c = uzi[oz], uz_m = uzi[oz + zm];

    const double uxp = face_update(ux_c, r, ir0, irx, irc, idxc, psx, psc, pnx, pnc, pox, poc, stf(0, ic, j, k));
    const double uxl = lead ? face_update(ux_w, r, ir0, irw1, irw, idxc, psw1, psw, pnw1, pnw, pow1, pow_,
                                          stf(0, ic + xo, j, k))
                            : 0.0;
    const double uxs = __shfl_up_sync(0xffffffffu, uxp, 1);
    const double uxm = lead ? uxl : uxs;
    const double uyp = (j < g.ny) ? face_update(uy_c, r, ir0, iry, irc, g.idyc[j], psy, psc, pny, pnc, poy, poc,
                                                stf(1, ic, j, k))
                                  : uy_c;
    const double uzp = face_update(uz_c, r, ir0, irz, irc, idzc, psz, psc, pnz, pnc, poz, poc, stf(2, ic, j, k));
    const double uzq = face_update(uz_m, r, ir0, irc, irm, idzc, psc, psm, pnc, pnm, poc, pom, stf(2, ic, j, km));
    if (valid) {
      uxo[ox] = uxp;
      if (i == g.nx) uxo[ox - ic] = uxp;  // ux(0, j, k)
      uyo[oy] = uyp;
      uzo[oz] = uzp;
      if (k == g.nz && !g.slab) uzo[oz - k * (int)a.Luz.sk] = uzp;  // uz(i, j, 0)
      double dv = (uxp - uxm) * idx;
      dv = dv + (uyp - uym) * g.idyf[j - 1];
      dv = dv + (uzp - uzq) * idz;
      vmax = nanmax_nonneg(vmax, dv);
    }
    uym = uyp;
    psc = psy;
    pnc = pny;
    poc = poy;
    irc = iry;
    op += pjs;
    oq += rjs;
    ox += xjs;
    oy += yjs;
    oz += zjs;
  }
  block_max_atomic(vmax, maxdiv);
}

void launch_correct_div(const CorrArgs &ca, bool has_st, const GridK &g, unsigned long long *maxdiv,
                        cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, (g.ny + kJC - 1) / kJC, g.nz);
  if (has_st) k_correct_div<true><<<grid, 128, 0, st>>>(ca, g, maxdiv);
  else k_correct_div<false><<<grid, 128, 0, st>>>(ca, g, maxdiv);
}

// In-place correction: each thread reads and writes only the faces it owns.
template <bool ST>
__global__ void __launch_bounds__(128) k_correct_inplace(CorrArgs a, GridK g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  if (i > g.nx) return;
  const double uxp = corr_x<ST>(a, g, i, j, k);
  const double uzp = corr_z<ST>(a, g, i, j, k);
  if (j < g.ny) a.uyo[at(a.Luy, i, j, k)] = corr_y<ST>(a, g, i, j, k);
  a.uxo[at(a.Lux, i, j, k)] = uxp;
  if (i == g.nx) a.uxo[at(a.Lux, 0, j, k)] = uxp;
  a.uzo[at(a.Luz, i, j, k)] = uzp;
  if (k == g.nz && !g.slab) a.uzo[at(a.Luz, i, j, 0)] = uzp;
}

void launch_correct_inplace(const CorrArgs &ca, bool has_st, const GridK &g, cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, g.ny, g.nz);
  if (has_st) k_correct_inplace<true><<<grid, 128, 0, st>>>(ca, g);
  else k_correct_inplace<false><<<grid, 128, 0, st>>>(ca, g);
}

// computeContinuityError (auxiliaryRoutines.f90:67-80), max|div u| only.
__global__ void __launch_bounds__(128) k_div(const double *__restrict__ ux, const double *__restrict__ uy,
                                             const double *__restrict__ uz, Lay Lux, Lay Luy, Lay Luz, GridK g,
                                             unsigned long long *__restrict__ maxdiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.z + 1;
  const int j0 = blockIdx.y * kJC + 1, j1 = min(j0 + kJC - 1, g.ny);
  double vmax = 0.0;
  if (i <= g.nx) {
    const double idx = g.idxf[i - 1], idz = g.idzf[k - 1];
    for (int j = j0; j <= j1; ++j) {
      double dv = (ux[at(Lux, i, j, k)] - ux[at(Lux, i - 1, j, k)]) * idx;
      dv = dv + (uy[at(Luy, i, j, k)] - uy[at(Luy, i, j - 1, k)]) * g.idyf[j - 1];
      dv = dv + (uz[at(Luz, i, j, k)] - uz[at(Luz, i, j, k - 1)]) * idz;
      vmax = nanmax_nonneg(vmax, dv);
    }
  }
  block_max_atomic(vmax, maxdiv);
}

void launch_div(const double *ux, const double *uy, const double *uz, Lay Lux, Lay Luy, Lay Luz, const GridK &g,
                unsigned long long *maxdiv, cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, (g.ny + kJC - 1) / kJC, g.nz);
  k_div<<<grid, 128, 0, st>>>(ux, uy, uz, Lux, Luy, Luz, g, maxdiv);
}

// Raise the dynamic shared-memory limits of every transform kernel; once per device.
cudaError_t prepare_kernels() {
  cudaError_t e = prepare_xfft_kernels();
  const cudaError_t e2 = prepare_yz_kernels();
  return e != cudaSuccess ? e : e2;
}

}  // namespace tbfp

namespace tbfp {

// ---------------------------------------------------------------------------
// MG_MODE source and coefficient: q = div u* (computeSource MG,
// poissonEqn.f90:155-190, metrics per index) and beta = dt*alpha/rho
// (computeBeta, :311-342) on the interior; beta is written with rho's layout.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_mg_source_beta(const double *__restrict__ ux, const double *__restrict__ uy,
                                                       const double *__restrict__ uz, Lay Lux, Lay Luy, Lay Luz,
                                                       const double *__restrict__ rho, Lay Lrho, GridK g, double dta,
                                                       double *__restrict__ q, Lay Lq, double *__restrict__ beta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  if (i > g.nx) return;
  double d = (ux[at(Lux, i, j, k)] - ux[at(Lux, i - 1, j, k)]) * g.idxf[i - 1];
  d = d + (uy[at(Luy, i, j, k)] - uy[at(Luy, i, j - 1, k)]) * g.idyf[j - 1];
  d = d + (uz[at(Luz, i, j, k)] - uz[at(Luz, i, j, k - 1)]) * g.idzf[k - 1];
  q[at(Lq, i, j, k)] = d;
  const long r = at(Lrho, i, j, k);
  beta[r] = dta / rho[r];
}

void launch_mg_source_beta(const double *ux, const double *uy, const double *uz, Lay Lux, Lay Luy, Lay Luz,
                           const double *rho, Lay Lrho, const GridK &g, double dta, double *q, Lay Lq, double *beta,
                           cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, g.ny, g.nz);
  k_mg_source_beta<<<grid, 128, 0, st>>>(ux, uy, uz, Lux, Luy, Luz, rho, Lrho, g, dta, q, Lq, beta);
}

// ---------------------------------------------------------------------------
// makeVelocityDivFree MG = addPressureGrad (momentumEqn.f90:795-869, :980-993):
//   u_d -= dt*alpha * (1/rho)_face * (p(+) - p) / dc_d
// with (1/rho)_face = (1/rho(+) + 1/rho)/2, on the setEqnBounds ranges (wall
// faces of uy copied through), then the periodic equate ux(0)=ux(nx),
// uz(.,.,0)=uz(.,.,nz) (vfield.f90:124-189).  p and rho are read with their
// ghosts (periodic images, wall copies).  Out of place or in place: a thread
// reads and writes only its own cell's faces.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_add_pressure_grad(const double *__restrict__ uxi, const double *__restrict__ uyi,
                                                          const double *__restrict__ uzi, double *__restrict__ uxo,
                                                          double *__restrict__ uyo, double *__restrict__ uzo,
                                                          Lay Lux, Lay Luy, Lay Luz, const double *__restrict__ p,
                                                          Lay Lp, const double *__restrict__ rho, Lay Lrho, GridK g,
                                                          const double *__restrict__ idxc, const double *__restrict__ idzc,
                                                          double dta) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  if (i > g.nx) return;
  const long pc = at(Lp, i, j, k), rc = at(Lrho, i, j, k);
  const double irc = 1.0 / rho[rc];
  {  // x face i+1/2: dxc(i+1)
    const double ir = 0.5 * (1.0 / rho[rc + 1] + irc);
    const long o = at(Lux, i, j, k);
    const double v = uxi[o] - dta * ir * (p[pc + 1] - p[pc]) * idxc[i];
    uxo[o] = v;
    if (i == g.nx) uxo[at(Lux, 0, j, k)] = v;
  }
  {  // y face j+1/2: dyc(j+1); the wall faces j = 0 and j = ny keep their values
    const long o = at(Luy, i, j, k);
    if (j < g.ny) {
      const double ir = 0.5 * (1.0 / rho[rc + Lrho.sj] + irc);
      uyo[o] = uyi[o] - dta * ir * (p[pc + Lp.sj] - p[pc]) * g.idyc[j];
    } else {
      uyo[o] = uyi[o];
    }
    if (j == 1) uyo[at(Luy, i, 0, k)] = uyi[at(Luy, i, 0, k)];
  }
  {  // z face k+1/2: dzc(k+1)
    const double ir = 0.5 * (1.0 / rho[rc + Lrho.sk] + irc);
    const long o = at(Luz, i, j, k);
    const double v = uzi[o] - dta * ir * (p[pc + Lp.sk] - p[pc]) * idzc[k];
    uzo[o] = v;
    if (k == g.nz) uzo[at(Luz, i, j, 0)] = v;
  }
}

void launch_add_pressure_grad(const double *uxi, const double *uyi, const double *uzi, double *uxo, double *uyo,
                              double *uzo, Lay Lux, Lay Luy, Lay Luz, const double *p, Lay Lp, const double *rho,
                              Lay Lrho, const GridK &g, const double *idxc, const double *idzc, double dta,
                              cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, g.ny, g.nz);
  k_add_pressure_grad<<<grid, 128, 0, st>>>(uxi, uyi, uzi, uxo, uyo, uzo, Lux, Luy, Luz, p, Lp, rho, Lrho, g, idxc,
                                            idzc, dta);
}

}  // namespace tbfp
