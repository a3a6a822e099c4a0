// Flow control of the channel (auxiliaryRoutines.f90:336-540): the volume
// sums behind setPressGrad (the mean density at the ux faces) and
// computeFlowRate (the ux flux), and setFlowRate's uniform shift of ux.
// A sum runs over the ux faces i = 0..nx-1, j = 1..ny, k = 1..nz with the
// staggered volume Vsx(i,j,k) = dxc(i+1)*dyf(j)*dzf(k) (grid.f90:812-838):
// one block per (j, k) row into a partial, then one block adds the partials
// in a fixed order, so a sum is the same on every call (its order differs
// from the reference's sequential loop: agreement to rounding).
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"

namespace tbfp {

namespace {

constexpr int kRT = 128;

template <int MODE>  // 0: 0.5*(rho(i+1)+rho(i)), 1: ux(i)
__global__ void __launch_bounds__(kRT) k_face_sum_rows(const double *__restrict__ f, Lay L,
                                                       const double *__restrict__ dxc, const double *__restrict__ dyf,
                                                       const double *__restrict__ dzf, int nx, int ny,
                                                       double *__restrict__ part) {
  const int j = blockIdx.x + 1, k = blockIdx.y + 1;
  const double dy = dyf[j - 1], dz = dzf[k - 1];
  double s = 0.0;
  for (int i = threadIdx.x; i < nx; i += kRT) {
    const long o = at(L, i, j, k);
    const double x = MODE == 0 ? 0.5 * (f[o + 1] + f[o]) : f[o];
    const double dV = dxc[i] * dy * dz;  // dxc(i+1)*dyf(j)*dzf(k)
    s += x * dV;
  }
  __shared__ double red[kRT];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = kRT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[(long)(k - 1) * ny + (j - 1)] = red[0];
}

__global__ void __launch_bounds__(1024) k_sum_partials(const double *__restrict__ part, long n,
                                                       double *__restrict__ out) {
  double s = 0.0;
  for (long e = threadIdx.x; e < n; e += 1024) s += part[e];
  __shared__ double red[1024];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// setFlowRate: ux(0:nx, 1:ny, 1:nz) += uf
__global__ void __launch_bounds__(kRT) k_add_ux(double *__restrict__ ux, Lay L, int nx, double uf) {
  const int i = blockIdx.x * kRT + threadIdx.x, j = blockIdx.y + 1, k = blockIdx.z + 1;
  if (i > nx) return;
  const long o = at(L, i, j, k);
  ux[o] = ux[o] + uf;
}

}  // namespace

void launch_face_sum(int mode, const double *f, Lay L, const double *dxc, const double *dyf, const double *dzf, int nx,
                     int ny, int nz, double *part, double *out, cudaStream_t st) {
  const dim3 grid(ny, nz);
  if (mode == 0) k_face_sum_rows<0><<<grid, kRT, 0, st>>>(f, L, dxc, dyf, dzf, nx, ny, part);
  else k_face_sum_rows<1><<<grid, kRT, 0, st>>>(f, L, dxc, dyf, dzf, nx, ny, part);
  k_sum_partials<<<1, 1024, 0, st>>>(part, (long)ny * nz, out);
}

void launch_add_ux(double *ux, Lay L, int nx, int ny, int nz, double uf, cudaStream_t st) {
  k_add_ux<<<dim3((nx + 1 + kRT - 1) / kRT, ny, nz), kRT, 0, st>>>(ux, L, nx, uf);
}

}  // namespace tbfp
