// FP64 x-direction kernels of the split-pressure projection (FAST_MODE of the
// reference): 1/rho, the split right-hand side, the forward real-to-complex x
// transform, and the inverse complex-to-real x transform that writes psi with
// its ghost images.
//
// Spectrum layout in HBM: S[kx][row], row = (k-1)*ny + (j-1), kx = 0..nx/2.
// For a fixed kx the x rows are contiguous, so the x transforms (one CTA per
// tile of consecutive rows) write/read contiguous runs of the tile's rows for
// every kx.  This replaces the pencil transposes of pencilDec.f90:359-562.
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"
#include "tbfp_stages.cuh"

namespace tbfp {

// ---------------------------------------------------------------------------
// 1/rho over the whole (halo-inclusive) density array.
// ---------------------------------------------------------------------------
__global__ void k_recip(const double *__restrict__ rho, double *__restrict__ irho, long n) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    irho[t] = 1.0 / rho[t];
}

void launch_recip(const double *rho, double *irho, long n, cudaStream_t st) {
  int blocks = (int)((n + 255) / 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_recip<<<blocks, 256, 0, st>>>(rho, irho, n);
}

// ---------------------------------------------------------------------------
// Forward x transform of a tile of rows: real rows (s, or the refinement
// residual, see XSrc) -> half-length complex FFT -> r2c post-processing ->
// S[kx][row].  A warp owns 2^LOGRPW rows; the CTA's 8 warps own TJ consecutive
// rows.  V = double2 (FP64) or float2 (the FP32 spectrum of the mixed path).
// ---------------------------------------------------------------------------
template <typename V, int M, int MODE>
__global__ void __launch_bounds__(kNT, (M >= 384 ? 2 : 3)) k_fftx_fwd(XSrc src, GridK g, const V *__restrict__ twx,
                                                  const V *__restrict__ tpx, V *__restrict__ spec) {
  extern __shared__ __align__(16) unsigned char smx[];
  fftx_fwd_body<V, M, MODE>(src, g, twx, tpx, spec, blockIdx.x, smx);
}

template <typename V, int M, int MODE>
static void launch_x_fwd_n(const XSrc &src, const GridK &g, const V *twx, const V *tpx, V *spec, cudaStream_t st) {
  constexpr int TJ = fftx_rows_per_cta(M);
  const long nblk = (g.R + TJ - 1) / TJ;
  k_fftx_fwd<V, M, MODE><<<(unsigned)nblk, kNT, fftx_smem_bytes(M, sizeof(V)), st>>>(src, g, twx, tpx, spec);
}

template <typename V, int MODE>
static void launch_x_fwd_t(const XSrc &src, const GridK &g, const V *twx, const V *tpx, V *spec, cudaStream_t st) {
  switch (g.M) {
#define TBFP_CASE(L) \
  case L: launch_x_fwd_n<V, L, MODE>(src, g, twx, tpx, spec, st); break;
    TBFP_FFT_LENGTHS(TBFP_CASE)
#undef TBFP_CASE
    default: break;  // lengths are validated by tbfp_create
  }
}

void launch_fftx_fwd_from_s(const double *s, Lay Ls, const GridK &g, const double2 *twx, const double2 *tpx,
                            double2 *spec, cudaStream_t st) {
  XSrc src{};
  src.s = s;
  src.Ls = Ls;
  launch_x_fwd_t<double2, 0>(src, g, twx, tpx, spec, st);
}
void launch_fftx_fwd(const XSrc &src, bool residual, const GridK &g, const double2 *twx, const double2 *tpx,
                     double2 *spec, cudaStream_t st) {
  if (residual) launch_x_fwd_t<double2, 1>(src, g, twx, tpx, spec, st);
  else launch_x_fwd_t<double2, 0>(src, g, twx, tpx, spec, st);
}
void launch_fftx_fwd(const XSrc &src, bool residual, const GridK &g, const float2 *twx, const float2 *tpx,
                     float2 *spec, cudaStream_t st) {
  if (residual) launch_x_fwd_t<float2, 1>(src, g, twx, tpx, spec, st);
  else launch_x_fwd_t<float2, 0>(src, g, twx, tpx, spec, st);
}

// ---------------------------------------------------------------------------
// Device-side control of the mixed-precision refinement (MixedCtl).
// ---------------------------------------------------------------------------
__global__ void k_mixed_params(MixedCtl *ctl, double *acc, double tol, double dtol, double dscale, int max_iter) {
  acc[0] = 0.0;
  acc[1] = 0.0;
  acc[2] = 0.0;
  acc[3] = 0.0;
  ctl->tol = tol;
  ctl->dtol = dtol;
  ctl->dscale = dscale;
  ctl->max_iter = max_iter;
  ctl->iters = 1;
  ctl->rel = -1.0;
  ctl->div = -1.0;
  ctl->status = 0;
  ctl->done = 0;
}

__global__ void k_mixed_decide(MixedCtl *ctl, const double *acc, double *acc_r, cudaGraphConditionalHandle cond,
                               int use_cond) {
  const double ss = acc[1], rr = acc_r[0];
  const double rel = ss > 0.0 ? sqrt(rr / ss) : sqrt(rr);
  const double div = ctl->dscale > 0.0 ? ctl->dscale * acc_r[1] : 0.0;
  acc_r[0] = 0.0;  // the next residual pass accumulates afresh
  acc_r[1] = 0.0;
  ctl->rel = rel;
  ctl->div = ctl->dscale > 0.0 ? div : -1.0;
  int done = 1;
  if (!isfinite(rel) || !isfinite(div)) ctl->status = -7;  // TBFP_ENONFINITE
  else if (rel <= ctl->tol && div <= ctl->dtol) ctl->status = 0;
  else if (ctl->iters >= ctl->max_iter) ctl->status = 1;  // TBFP_ENOTCONVERGED
  else {
    done = 0;
    ctl->iters += 1;  // the sweep that follows
  }
  ctl->done = done;
  if (use_cond) cudaGraphSetConditional(cond, done ? 0u : 1u);
}

void launch_mixed_params(MixedCtl *ctl, double *acc, double tol, double dtol, double dscale, int max_iter,
                         cudaStream_t st) {
  k_mixed_params<<<1, 1, 0, st>>>(ctl, acc, tol, dtol, dscale, max_iter);
}
void launch_mixed_decide(MixedCtl *ctl, const double *acc, double *acc_r, cudaGraphConditionalHandle cond,
                         bool use_cond, cudaStream_t st) {
  k_mixed_decide<<<1, 1, 0, st>>>(ctl, acc, acc_r, cond, use_cond ? 1 : 0);
}

// Split RHS into s on the interior (tbfp_rhs_split and the projection).  Grid
// (x tiles of 128, y chunks of kRJ rows, nz); a thread owns column (i, k) of a y
// chunk and walks it in j with 32-bit element offsets, carrying the centre
// values of 1/rho, psi^n and psi^(n-1) to the next row as its lower y
// neighbours.  computeSource (poissonEqn.f90:224-253) with computeOldPressDiv
// (:270-301), nl = 2; divisions by metrics are products with host-computed
// reciprocals, 1/rho comes from the precomputed array.

template <bool ST>
__global__ void __launch_bounds__(128, 6) k_rhs(RhsArgs a, GridK g, double *__restrict__ s, Lay Ls) {
  rhs_body<ST>(a, g, s, Ls, blockIdx.x, blockIdx.y, blockIdx.z, threadIdx.x);
}

void launch_rhs(const RhsArgs &ra, bool has_st, const GridK &g, double *s, Lay Ls, cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, (g.ny + kRJ - 1) / kRJ, g.nz);
  if (has_st) k_rhs<true><<<grid, 128, 0, st>>>(ra, g, s, Ls);
  else k_rhs<false><<<grid, 128, 0, st>>>(ra, g, s, Ls);
}

// ---------------------------------------------------------------------------
// Inverse x transform of a tile of rows: S[kx][row] -> c2r -> psi rows scaled
// by 1/(nx*nz) (fastPoissonSolver.f90:371-378), written with every ghost image
// of updateBoundaries (field.f90:950-974 on one rank): the first y ghost layer
// copies the wall cell (normalGradient, bf=0), x and z ghosts are periodic.
// The imaginary parts of X[0] and X[nx/2] are ignored, as FFTW's c2r does.
// ---------------------------------------------------------------------------

template <typename V, int M, bool ACC>
__global__ void __launch_bounds__(kNT, (M >= 384 ? 2 : 3)) k_fftx_inv(const V *__restrict__ spec, double *__restrict__ psi, Lay Lp,
                                                  int hd, GridK g, const V *__restrict__ twx,
                                                  const V *__restrict__ tpx, double scale) {
  extern __shared__ __align__(16) unsigned char smx[];
  fftx_inv_body<V, M, ACC>(spec, psi, Lp, hd, g, twx, tpx, scale, blockIdx.x, smx);
}

template <typename V, int M, bool ACC>
static void launch_fftx_inv_n(const V *spec, double *psi, Lay Lp, int hd, const GridK &g, const V *twx, const V *tpx,
                              double scale, cudaStream_t st) {
  constexpr int TJ = fftx_rows_per_cta(M);
  const long nblk = (g.R + TJ - 1) / TJ;
  k_fftx_inv<V, M, ACC><<<(unsigned)nblk, kNT, fftx_smem_bytes(M, sizeof(V)), st>>>(spec, psi, Lp, hd, g, twx, tpx,
                                                                                     scale);
}

template <typename V, bool ACC>
static void launch_fftx_inv_t(const V *spec, double *psi, Lay Lp, int hd, const GridK &g, const V *twx,
                              const V *tpx, double scale, cudaStream_t st) {
  switch (g.M) {
#define TBFP_CASE(L) \
  case L: launch_fftx_inv_n<V, L, ACC>(spec, psi, Lp, hd, g, twx, tpx, scale, st); break;
    TBFP_FFT_LENGTHS(TBFP_CASE)
#undef TBFP_CASE
    default: break;
  }
}

void launch_fftx_inv(const double2 *spec, double *psi, Lay Lp, int hd, const GridK &g, const double2 *twx,
                     const double2 *tpx, double scale, cudaStream_t st) {
  launch_fftx_inv_t<double2, false>(spec, psi, Lp, hd, g, twx, tpx, scale, st);
}
void launch_fftx_inv(const float2 *spec, double *psi, Lay Lp, int hd, const GridK &g, const float2 *twx,
                     const float2 *tpx, double scale, bool accumulate, cudaStream_t st) {
  if (accumulate) launch_fftx_inv_t<float2, true>(spec, psi, Lp, hd, g, twx, tpx, scale, st);
  else launch_fftx_inv_t<float2, false>(spec, psi, Lp, hd, g, twx, tpx, scale, st);
}

cudaError_t prepare_xfft_kernels() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void *fn, size_t bytes) {
    const cudaError_t ee = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (ee != cudaSuccess) e = ee;
  };
#define TBFP_CASE(L)                                                         \
  set((const void *)k_fftx_fwd<double2, L, 0>, fftx_smem_bytes(L, 16));      \
  set((const void *)k_fftx_fwd<double2, L, 1>, fftx_smem_bytes(L, 16));      \
  set((const void *)k_fftx_fwd<float2, L, 0>, fftx_smem_bytes(L, 8));        \
  set((const void *)k_fftx_fwd<float2, L, 1>, fftx_smem_bytes(L, 8));        \
  set((const void *)k_fftx_inv<double2, L, false>, fftx_smem_bytes(L, 16));  \
  set((const void *)k_fftx_inv<float2, L, false>, fftx_smem_bytes(L, 8));    \
  set((const void *)k_fftx_inv<float2, L, true>, fftx_smem_bytes(L, 8));
  TBFP_FFT_LENGTHS(TBFP_CASE)
#undef TBFP_CASE
  return e;
}

}  // namespace tbfp
