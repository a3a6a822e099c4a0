// FP64 velocity correction and continuity check of the split-pressure
// projection (FAST_MODE of the reference).
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"
#include "tbfp_stages.cuh"

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

template <bool ST>
__global__ void __launch_bounds__(128, 8) k_correct_div(CorrArgs a, GridK g, unsigned long long *__restrict__ maxdiv) {
  correct_div_body<ST>(a, g, maxdiv, blockIdx.x, blockIdx.y, blockIdx.z, threadIdx.x);
}

void launch_correct_div(const CorrArgs &ca, bool has_st, const GridK &g, unsigned long long *maxdiv,
                        cudaStream_t st) {
  if (!has_st) {  // the TMA-staged z march (tbfp_correct_tma.cu) wherever tensor maps describe the arrays
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        launch_correct_div_tma(ca, g, maxdiv, sms, st))
      return;
  }
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
  const cudaError_t e3 = prepare_correct_tma_kernel();
  if (e == cudaSuccess) e = e3;
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
