// Device-side types shared by the projection kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "fft_smem.cuh"

namespace tbfp {

// Layout of a Fortran array f(ilo:.., jlo:.., klo:..), column-major.
struct Lay {
  int ilo, jlo, klo;
  long sj, sk;
};
__host__ __device__ __forceinline__ long at(const Lay &L, int i, int j, int k) {
  return (long)(i - L.ilo) + (long)(j - L.jlo) * L.sj + (long)(k - L.klo) * L.sk;
}

// Grid constants and metric tables (device pointers, 0-based: table[j-1] holds the
// reference's value at Fortran index j).
struct GridK {
  int nx, ny, nz, nkx, M;  // M = nx/2 (length of the half-length complex x transform)
  long R;                  // ny*nz: number of x rows
  double idxf1, idzf1;     // 1/dxf(1), 1/dzf(1)
  double idxc1, idzc1;     // 1/dxc(1), 1/dzc(1)
  const double *idyf;      // 1/dyf(j), j=1..ny
  const double *idyc;      // 1/dyc(j), j=1..ny+1
  const double *idxf;      // 1/dxf(i), i=1..nx
  const double *idzf;      // 1/dzf(k), k=1..nz
};

// Inputs of the split right-hand side (poissonEqn.f90:193-305).
struct RhsArgs {
  const double *ux, *uy, *uz;
  const double *irho;  // 1/rho, laid out like rho
  const double *pn, *pnm1;
  const double *stn[3], *sto[3];
  Lay Lux, Luy, Luz, Lrho, Lpsi, Lst[3];
  double r;     // 1/(alpha*dt)
  double rho0;
};

// Inputs of the velocity correction (momentumEqn.f90:999-1127).
struct CorrArgs {
  const double *uxi, *uyi, *uzi;
  double *uxo, *uyo, *uzo;
  const double *psi, *pn, *pnm1, *irho;
  const double *stn[3], *sto[3];
  Lay Lux, Luy, Luz, Lpsi, Lrho, Lst[3];
  double r;  // dt*alpha
  double invrho0;
};

// Error text returned by tbfp_last_error(NULL) (defined in tbfp_api.cu).
void set_global_error(const std::string &msg);

// Kernel launchers (defined in tbfp_kernels.cu).
void launch_recip(const double *rho, double *irho, long n, cudaStream_t st);
cudaError_t prepare_kernels();
int fft_max_length();
int fftx_rows_per_cta(int M);
int fftz_cols_per_cta(int nz);
size_t fftx_smem_bytes(int M);
size_t fftz_smem_bytes(int nz);
size_t tridiag_smem_bytes(int ny);

void launch_fftx_fwd_from_s(const double *s, Lay Ls, const GridK &g, const FftPlan &pl, const double2 *twx,
                            double2 *spec, cudaStream_t st);
void launch_fftx_fwd_rhs(const RhsArgs &ra, bool has_st, const GridK &g, const FftPlan &pl, const double2 *twx,
                         double2 *spec, cudaStream_t st);
void launch_rhs(const RhsArgs &ra, bool has_st, const GridK &g, double *s, Lay Ls, cudaStream_t st);
void launch_fftz(double2 *spec, const GridK &g, const FftPlan &pl, const double2 *twz, bool inverse,
                 cudaStream_t st);
void launch_tridiag(double2 *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                    const double *ap, const double *dyf, double mean_c, double nxnz, cudaStream_t st);
void launch_fftx_inv(const double2 *spec, double *psi, Lay Lp, int hd, const GridK &g, const FftPlan &pl,
                     const double2 *twx, double scale, cudaStream_t st);
void launch_correct_div(const CorrArgs &ca, bool has_st, const GridK &g, unsigned long long *maxdiv,
                        cudaStream_t st);
void launch_correct_inplace(const CorrArgs &ca, bool has_st, const GridK &g, cudaStream_t st);
void launch_div(const double *ux, const double *uy, const double *uz, Lay Lux, Lay Luy, Lay Luz, const GridK &g,
                unsigned long long *maxdiv, cudaStream_t st);

}  // namespace tbfp
