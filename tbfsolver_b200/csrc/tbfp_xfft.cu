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

// The same with 16-byte accesses, two in flight per thread (both arrays
// 16-byte aligned; the odd last element, if any, by the scalar kernel's rule).
__global__ void k_recip2(const double2 *__restrict__ rho, double2 *__restrict__ irho, long n2) {
  const long stride = (long)gridDim.x * blockDim.x;
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  for (; t + stride < n2; t += 2 * stride) {
    const double2 a = __ldcs(rho + t), b = __ldcs(rho + t + stride);
    __stcs(irho + t, make_double2(1.0 / a.x, 1.0 / a.y));
    __stcs(irho + t + stride, make_double2(1.0 / b.x, 1.0 / b.y));
  }
  if (t < n2) {
    const double2 a = __ldcs(rho + t);
    __stcs(irho + t, make_double2(1.0 / a.x, 1.0 / a.y));
  }
}

void launch_recip(const double *rho, double *irho, long n, cudaStream_t st) {
  if (((reinterpret_cast<uintptr_t>(rho) | reinterpret_cast<uintptr_t>(irho)) & 15) == 0 && n >= 2) {
    const long n2 = n / 2;
    long blocks = (n2 + 511) / 512;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_recip2<<<(unsigned)blocks, 256, 0, st>>>(reinterpret_cast<const double2 *>(rho),
                                              reinterpret_cast<double2 *>(irho), n2);
    if (n & 1) k_recip<<<1, 32, 0, st>>>(rho + (n - 1), irho + (n - 1), 1);
    return;
  }
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
  using T = decltype(V::x);
  constexpr int LOGRPW = ct_lognb(M), RPW = 1 << LOGRPW, LOGTJ = LOGRPW + 3, TJ = 1 << LOGTJ;
  constexpr int LD = x_row_stride(M), NX = 2 * M, NXC = (NX + 31) / 32;
  extern __shared__ __align__(16) unsigned char smx[];
  V *sm = reinterpret_cast<V *>(smx);
  V *tw = sm + TJ * LD;
  __shared__ double red[kNW][3];
  for (int t = threadIdx.x; t < ct_twiddle_len(M); t += kNT) tw[t] = tpx[t];
  const int r0 = blockIdx.x << LOGTJ;
  const int nrows = min(TJ, (int)g.R - r0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *wsm = sm + warp * RPW * LD;  // this warp's rows
  T *wsr = reinterpret_cast<T *>(wsm);
  const bool sums = (MODE == 0) ? src.acc != nullptr : true;
  const double ctop = (MODE == 1) ? src.acc[0] * src.ctop_scale : 0.0;
  double sum0 = 0.0, sum1 = 0.0, vmax = 0.0;

#pragma unroll
  for (int rl = 0; rl < RPW; ++rl) {
    const int row = warp * RPW + rl;
    T *dst = wsr + rl * 2 * LD;
    if (row < nrows) {
      const unsigned rr = (unsigned)(r0 + row);
      const int k = (int)(rr / (unsigned)g.ny) + 1, j = (int)(rr - (unsigned)(k - 1) * g.ny) + 1;
      const double *srow = src.s + at(src.Ls, 0, j, k);
      if constexpr (MODE == 0) {
        const double wy = sums ? src.dyf[j - 1] : 0.0;
#pragma unroll
        for (int c = 0; c < NXC; ++c) {
          const int ii = lane + 32 * c;
          if (NX % 32 == 0 || ii < NX) {
            const double v = srow[ii + 1];
            sum0 += v * wy;
            sum1 += v * v;
            dst[2 * pad8(ii >> 1) + (ii & 1)] = (T)v;
          }
        }
      } else {
        // r = s - c [j == ny] - L psi (the operator whose eigenvectors the solve uses)
        const double *p = src.psi + at(src.Lp, 0, j, k);
        const long sj = src.Lp.sj, sk = src.Lp.sk;
        const double amj = src.am[j - 1], apj = src.ap[j - 1];
        const double cj = (j == g.ny) ? ctop : 0.0;
#pragma unroll
        for (int c = 0; c < NXC; ++c) {
          const int ii = lane + 32 * c;
          if (NX % 32 == 0 || ii < NX) {
            const int i = ii + 1;
            const double p0 = p[i];
            const double lap = (p[i + 1] + p[i - 1] - 2.0 * p0) * src.idx2 + amj * (p[i - sj] - p0) +
                               apj * (p[i + sj] - p0) + (p[i + sk] + p[i - sk] - 2.0 * p0) * src.idz2;
            const double v = (srow[i] - cj) - lap;
            sum1 += v * v;
            vmax = nanmax_nonneg(vmax, v + cj);
            dst[2 * pad8(ii >> 1) + (ii & 1)] = (T)v;
          }
        }
      }
    } else {
#pragma unroll
      for (int c = 0; c < NXC; ++c) {
        const int ii = lane + 32 * c;
        if (NX % 32 == 0 || ii < NX) dst[2 * pad8(ii >> 1) + (ii & 1)] = T(0);
      }
    }
  }
  if (sums) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sum0 += __shfl_xor_sync(0xffffffffu, sum0, o);
      sum1 += __shfl_xor_sync(0xffffffffu, sum1, o);
      if constexpr (MODE == 1) vmax = nanmax_nonneg(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    }
    if (lane == 0) {
      red[warp][0] = sum0;
      red[warp][1] = sum1;
      red[warp][2] = vmax;
    }
  }
  __syncthreads();  // twiddle table, rows and partial sums in place
  if (sums && threadIdx.x == 0) {
    double a0 = 0.0, a1 = 0.0, m = 0.0;
    for (int w = 0; w < kNW; ++w) {
      a0 += red[w][0];
      a1 += red[w][1];
      m = nanmax_nonneg(m, red[w][2]);
    }
    if constexpr (MODE == 0) {
      atomicAdd(src.acc, a0);
      atomicAdd(src.acc + 1, a1);
    } else {
      atomicAdd(src.acc_r, a1);
      atomicMax(reinterpret_cast<unsigned long long *>(src.acc_r + 1), (unsigned long long)__double_as_longlong(m));
    }
  }
  fft_warp<V, M, LOGRPW, 1, LD, false, 0, ct_nrad(M) - 1>(wsm, lane, tw);  // all passes but the last
  __syncthreads();
  // the last pass with the r2c pair step and the store of S[kx][r0 + row]
  fwd_last_pass_r2c_store<V, M, LOGTJ>(sm, tw, twx, spec, g.R, r0, nrows);
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
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.z + 1;
  const int j0 = blockIdx.y * kRJ + 1, j1 = min(j0 + kRJ - 1, g.ny);
  if (i > g.nx) return;  // no block-level barrier in this kernel
  const int pjs = (int)a.Lpsi.sj, pks = (int)a.Lpsi.sk, rjs = (int)a.Lrho.sj, rks = (int)a.Lrho.sk;
  const int xjs = (int)a.Lux.sj, yjs = (int)a.Luy.sj, zjs = (int)a.Luz.sj, zks = (int)a.Luz.sk;
  const int sjs = (int)Ls.sj;
  int op = (int)at(a.Lpsi, i, j0, k), oq = (int)at(a.Lrho, i, j0, k);
  int ox = (int)at(a.Lux, i, j0, k), oy = (int)at(a.Luy, i, j0, k), oz = (int)at(a.Luz, i, j0, k);
  int os = (int)at(Ls, i, j0, k);
  const double *__restrict__ ux = a.ux;
  const double *__restrict__ uy = a.uy;
  const double *__restrict__ uz = a.uz;
  const double *__restrict__ ir = a.irho;
  const double *__restrict__ pn = a.pn;
  const double *__restrict__ po = a.pnm1;
  const double h = a.rho0 * 0.5;
  const double idxf = g.idxf1, idzf = g.idzf1, idxc = g.idxc1, idzc = g.idzc1;
  // carried along j: centre values and the lower y face
  double irc = ir[oq], pc = pn[op], oc = po[op];
  double irm = ir[oq - rjs], pm = pn[op - pjs], om = po[op - pjs];
  double uym = uy[oy - yjs];
  for (int j = j0; j <= j1; ++j) {
    const double uxc = ux[ox], uxm = ux[ox - 1], uyc = uy[oy], uzc = uz[oz], uzm = uz[oz - zks];
    const double irxp = ir[oq + 1], irxm = ir[oq - 1], iryp = ir[oq + rjs], irzp = ir[oq + rks], irzm = ir[oq - rks];
    const double pxp = pn[op + 1], pxm = pn[op - 1], pyp = pn[op + pjs], pzp = pn[op + pks], pzm = pn[op - pks];
    const double oxp = po[op + 1], oxm = po[op - 1], oyp = po[op + pjs], ozp = po[op + pks], ozm = po[op - pks];
    const double idyf = g.idyf[j - 1], idycp = g.idyc[j], idycm = g.idyc[j - 1];

    const double ddx = (uxc - uxm) * idxf;
    const double ddy = (uyc - uym) * idyf;
    const double ddz = (uzc - uzm) * idzf;
    double r = ((ddx + ddy) + ddz) * a.r * a.rho0;
    const double apx = 1.0 - h * (irxp + irc);
    const double amx = 1.0 - h * (irxm + irc);
    const double apy = 1.0 - h * (iryp + irc);
    const double amy = 1.0 - h * (irm + irc);
    const double apz = 1.0 - h * (irzp + irc);
    const double amz = 1.0 - h * (irzm + irc);
    double dpxp = (2.0 * (pxp - pc) - (oxp - oc)) * idxc;
    double dpxm = (2.0 * (pc - pxm) - (oc - oxm)) * idxc;
    double dpyp = (2.0 * (pyp - pc) - (oyp - oc)) * idycp;
    double dpym = (2.0 * (pc - pm) - (oc - om)) * idycm;
    double dpzp = (2.0 * (pzp - pc) - (ozp - oc)) * idzc;
    double dpzm = (2.0 * (pc - pzm) - (oc - ozm)) * idzc;
    if constexpr (ST) {
      const long x0 = at(a.Lst[0], i, j, k), y0 = at(a.Lst[1], i, j, k), z0 = at(a.Lst[2], i, j, k);
      dpxp = dpxp - 2.0 * a.stn[0][x0] + a.sto[0][x0];
      dpxm = dpxm - 2.0 * a.stn[0][x0 - 1] + a.sto[0][x0 - 1];
      dpyp = dpyp - 2.0 * a.stn[1][y0] + a.sto[1][y0];
      dpym = dpym - 2.0 * a.stn[1][y0 - a.Lst[1].sj] + a.sto[1][y0 - a.Lst[1].sj];
      dpzp = dpzp - 2.0 * a.stn[2][z0] + a.sto[2][z0];
      dpzm = dpzm - 2.0 * a.stn[2][z0 - a.Lst[2].sk] + a.sto[2][z0 - a.Lst[2].sk];
    }
    r = r + (apx * dpxp - amx * dpxm) * idxf;
    r = r + (apy * dpyp - amy * dpym) * idyf;
    r = r + (apz * dpzp - amz * dpzm) * idzf;
    s[os] = r;
    irm = irc;
    pm = pc;
    om = oc;
    irc = iryp;
    pc = pyp;
    oc = oyp;
    uym = uyc;
    op += pjs;
    oq += rjs;
    ox += xjs;
    oy += yjs;
    oz += zjs;
    os += sjs;
  }
}

void launch_rhs(const RhsArgs &ra, bool has_st, const GridK &g, double *s, Lay Ls, cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, (g.ny + kRJ - 1) / kRJ, g.nz);
  if (has_st) k_rhs<true><<<grid, 128, 0, st>>>(ra, g, s, Ls);
  else k_rhs<false><<<grid, 128, 0, st>>>(ra, g, s, Ls);
}

// ---------------------------------------------------------------------------
// The split right-hand side and the forward x transform in one kernel (the
// FP64 direct solve).  The CTA computes the right-hand side of its TJ rows
// straight into its x tile in shared memory, so s never goes through HBM
// (403 MB written and read back at 512x384x256).  Threads own columns and
// march along the tile's rows with the centre values and lower y neighbours
// carried from row to row, the arithmetic of k_rhs term for term; a row at
// j = 1 (the start of a z plane) reloads them.  The transform, the r2c
// post-processing and the transposed store are those of k_fftx_fwd.
// ---------------------------------------------------------------------------
template <int M, bool ST>
__global__ void __launch_bounds__(kNT, (M >= 384 ? 2 : 3))
    k_rhs_fftx(RhsArgs a, GridK g, const double2 *__restrict__ twx, const double2 *__restrict__ tpx,
               double2 *__restrict__ spec) {
  using V = double2;
  constexpr int LOGRPW = ct_lognb(M), RPW = 1 << LOGRPW, LOGTJ = LOGRPW + 3, TJ = 1 << LOGTJ;
  constexpr int LD = x_row_stride(M), NX = 2 * M;
  // column ownership: NG groups of NX threads (NX <= kNT), each marching RG
  // rows, or one group with NCOL columns per thread
  constexpr int NG = NX <= kNT ? kNT / NX : 1;
  constexpr int NCOL = NX <= kNT ? 1 : (NX + kNT - 1) / kNT;
  constexpr int RG = (TJ + NG - 1) / NG;
  extern __shared__ __align__(16) unsigned char smx[];
  V *sm = reinterpret_cast<V *>(smx);
  double *smr = reinterpret_cast<double *>(smx);
  V *tw = sm + TJ * LD;
  for (int t = threadIdx.x; t < ct_twiddle_len(M); t += kNT) tw[t] = __ldg(tpx + t);
  const int r0 = blockIdx.x << LOGTJ;
  const int nrows = min(TJ, (int)g.R - r0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  const int grp = NX <= kNT ? (int)threadIdx.x / NX : 0;
  if (grp < NG) {
    const int col0 = (int)threadIdx.x - grp * (NX <= kNT ? NX : 0);
    const int rl0 = grp * RG, rl1 = min(rl0 + RG, TJ);
    const int pjs = (int)a.Lpsi.sj, pks = (int)a.Lpsi.sk, rjs = (int)a.Lrho.sj, rks = (int)a.Lrho.sk;
    const int xjs = (int)a.Lux.sj, yjs = (int)a.Luy.sj, zjs = (int)a.Luz.sj, zks = (int)a.Luz.sk;
    const double *__restrict__ ux = a.ux;
    const double *__restrict__ uy = a.uy;
    const double *__restrict__ uz = a.uz;
    const double *__restrict__ ir = a.irho;
    const double *__restrict__ pn = a.pn;
    const double *__restrict__ po = a.pnm1;
    const double h = a.rho0 * 0.5;
    const double idxf = g.idxf1, idzf = g.idzf1, idxc = g.idxc1, idzc = g.idzc1;
#pragma unroll 1
    for (int c = 0; c < NCOL; ++c) {
      const int ii = col0 + c * kNT;
      if (NCOL > 1 && ii >= NX) break;
      const int i = ii + 1;
      double *dst = smr + 2 * pad8(ii >> 1) + (ii & 1);
      double irc = 0.0, pc = 0.0, oc = 0.0, irm = 0.0, pm = 0.0, om = 0.0, uym = 0.0;
      // (j, k) and the element offsets of the march's first row; later rows step
      // one row stride, a new z plane starts afresh
      const unsigned rr0 = (unsigned)(r0 + rl0);
      int k = (int)(rr0 / (unsigned)g.ny) + 1, j = (int)(rr0 - (unsigned)(k - 1) * g.ny) + 1;
      int op = (int)at(a.Lpsi, i, j, k), oq = (int)at(a.Lrho, i, j, k);
      int ox = (int)at(a.Lux, i, j, k), oy = (int)at(a.Luy, i, j, k), oz = (int)at(a.Luz, i, j, k);
      bool fresh = true;
#pragma unroll
      for (int rl = rl0; rl < rl1; ++rl) {
        double r = 0.0;
        if (rl < nrows) {
          if (fresh) {  // first row of the march or of a z plane
            irc = __ldg(ir + oq);
            pc = __ldg(pn + op);
            oc = __ldg(po + op);
            irm = __ldg(ir + (oq - rjs));
            pm = __ldg(pn + (op - pjs));
            om = __ldg(po + (op - pjs));
            uym = __ldg(uy + (oy - yjs));
            fresh = false;
          }
          const double uxc = __ldg(ux + ox), uyc = __ldg(uy + oy), uzc = __ldg(uz + oz), uzm = __ldg(uz + (oz - zks));
          const double iryp = __ldg(ir + (oq + rjs)), irzp = __ldg(ir + (oq + rks)), irzm = __ldg(ir + (oq - rks));
          const double pyp = __ldg(pn + (op + pjs)), pzp = __ldg(pn + (op + pks)), pzm = __ldg(pn + (op - pks));
          const double oyp = __ldg(po + (op + pjs)), ozp = __ldg(po + (op + pks)), ozm = __ldg(po + (op - pks));
          const double uxm = __ldg(ux + (ox - 1));
          const double irxm = __ldg(ir + (oq - 1)), irxp = __ldg(ir + (oq + 1));
          const double pxm = __ldg(pn + (op - 1)), pxp = __ldg(pn + (op + 1));
          const double oxm = __ldg(po + (op - 1)), oxp = __ldg(po + (op + 1));
          const double idyf = g.idyf[j - 1], idycp = g.idyc[j], idycm = g.idyc[j - 1];

          const double ddx = (uxc - uxm) * idxf;
          const double ddy = (uyc - uym) * idyf;
          const double ddz = (uzc - uzm) * idzf;
          r = ((ddx + ddy) + ddz) * a.r * a.rho0;
          const double apx = 1.0 - h * (irxp + irc);
          const double amx = 1.0 - h * (irxm + irc);
          const double apy = 1.0 - h * (iryp + irc);
          const double amy = 1.0 - h * (irm + irc);
          const double apz = 1.0 - h * (irzp + irc);
          const double amz = 1.0 - h * (irzm + irc);
          double dpxp = (2.0 * (pxp - pc) - (oxp - oc)) * idxc;
          double dpxm = (2.0 * (pc - pxm) - (oc - oxm)) * idxc;
          double dpyp = (2.0 * (pyp - pc) - (oyp - oc)) * idycp;
          double dpym = (2.0 * (pc - pm) - (oc - om)) * idycm;
          double dpzp = (2.0 * (pzp - pc) - (ozp - oc)) * idzc;
          double dpzm = (2.0 * (pc - pzm) - (oc - ozm)) * idzc;
          if constexpr (ST) {
            const long x0 = at(a.Lst[0], i, j, k), y0 = at(a.Lst[1], i, j, k), z0 = at(a.Lst[2], i, j, k);
            dpxp = dpxp - 2.0 * a.stn[0][x0] + a.sto[0][x0];
            dpxm = dpxm - 2.0 * a.stn[0][x0 - 1] + a.sto[0][x0 - 1];
            dpyp = dpyp - 2.0 * a.stn[1][y0] + a.sto[1][y0];
            dpym = dpym - 2.0 * a.stn[1][y0 - a.Lst[1].sj] + a.sto[1][y0 - a.Lst[1].sj];
            dpzp = dpzp - 2.0 * a.stn[2][z0] + a.sto[2][z0];
            dpzm = dpzm - 2.0 * a.stn[2][z0 - a.Lst[2].sk] + a.sto[2][z0 - a.Lst[2].sk];
          }
          r = r + (apx * dpxp - amx * dpxm) * idxf;
          r = r + (apy * dpyp - amy * dpym) * idyf;
          r = r + (apz * dpzp - amz * dpzm) * idzf;
          irm = irc;
          pm = pc;
          om = oc;
          irc = iryp;
          pc = pyp;
          oc = oyp;
          uym = uyc;
        }
        dst[rl * 2 * LD] = r;
        if (++j > g.ny) {
          j = 1;
          ++k;
          op = (int)at(a.Lpsi, i, j, k);
          oq = (int)at(a.Lrho, i, j, k);
          ox = (int)at(a.Lux, i, j, k);
          oy = (int)at(a.Luy, i, j, k);
          oz = (int)at(a.Luz, i, j, k);
          fresh = true;
        } else {
          op += pjs;
          oq += rjs;
          ox += xjs;
          oy += yjs;
          oz += zjs;
        }
      }
    }
  }
  __syncthreads();  // twiddle table and rows in place
  V *wsm = sm + warp * RPW * LD;  // this warp's rows
  fft_warp<V, M, LOGRPW, 1, LD, false, 0, ct_nrad(M) - 1>(wsm, lane, tw);  // all passes but the last
  __syncthreads();
  // the last pass with the r2c pair step and the store of S[kx][r0 + row]
  fwd_last_pass_r2c_store<V, M, LOGTJ>(sm, tw, twx, spec, g.R, r0, nrows);
}

template <int M>
static void launch_rhs_fftx_n(const RhsArgs &ra, bool has_st, const GridK &g, const double2 *twx,
                              const double2 *tpx, double2 *spec, cudaStream_t st) {
  constexpr int TJ = fftx_rows_per_cta(M);
  const unsigned nblk = (unsigned)((g.R + TJ - 1) / TJ);
  const size_t smem = fftx_smem_bytes(M, 16);
  if (has_st) k_rhs_fftx<M, true><<<nblk, kNT, smem, st>>>(ra, g, twx, tpx, spec);
  else k_rhs_fftx<M, false><<<nblk, kNT, smem, st>>>(ra, g, twx, tpx, spec);
}

void launch_rhs_fftx(const RhsArgs &ra, bool has_st, const GridK &g, const double2 *twx, const double2 *tpx,
                     double2 *spec, cudaStream_t st) {
  switch (g.M) {
#define TBFP_CASE(L) \
  case L: launch_rhs_fftx_n<L>(ra, has_st, g, twx, tpx, spec, st); break;
    TBFP_FFT_LENGTHS(TBFP_CASE)
#undef TBFP_CASE
    default: break;  // lengths are validated by tbfp_create
  }
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
  using T = decltype(V::x);
  constexpr int LOGRPW = ct_lognb(M), RPW = 1 << LOGRPW, LOGTJ = LOGRPW + 3, TJ = 1 << LOGTJ;
  constexpr int LD = x_row_stride(M);
  extern __shared__ __align__(16) unsigned char smx[];
  V *sm = reinterpret_cast<V *>(smx);
  V *tw = sm + TJ * LD;
  for (int t = threadIdx.x; t < ct_twiddle_len(M); t += kNT) tw[t] = tpx[t];
  const int r0 = blockIdx.x << LOGTJ;
  const int nrows = min(TJ, (int)g.R - r0);
  // Z[n] = (X_n + conj X_{M-n}) + i conj(W^n) (X_n - conj X_{M-n}),  n = 0..M-1,
  // made as the spectrum comes in and fed straight into the first radix-R0
  // pass: thread (b, row) loads X_n and X_{M-n} for its butterfly's inputs
  // n = b + r M/R0 (eight rows of one n are 128 contiguous bytes), transforms
  // them in registers and writes the pass's outputs
  constexpr int R0 = ct_rad(M, 0), PER = M / R0, NB0 = PER << LOGTJ;
#pragma unroll
  for (int t = threadIdx.x; t < NB0; t += kNT) {
    const int jb = t >> LOGTJ, row = t & (TJ - 1);
    V v[R0];
#pragma unroll
    for (int r = 0; r < R0; ++r) {
      const int n = jb + r * PER, m = M - n;
      V xa = mk<V>(T(0), T(0)), xb = xa;
      if (row < nrows) {
        xa = spec[(long)n * g.R + r0 + row];
        xb = spec[(long)m * g.R + r0 + row];
      }
      if (n == 0) {
        v[r] = mk<V>(xa.x + xb.x, xa.x - xb.x);  // the imaginary parts of X_0 and X_M are ignored
      } else {
        const V wa = cconj(twx[n]);
        V ep = mk<V>(xa.x + xb.x, xa.y - xb.y);
        V em = mk<V>(xa.x - xb.x, xa.y + xb.y);
        V t1 = cmul(wa, em);
        v[r] = mk<V>(ep.x - t1.y, ep.y + t1.x);  // ep + i t1
      }
    }
    bfly<V, R0, true>(v);
    V *X = sm + row * LD;
#pragma unroll
    for (int r = 0; r < R0; ++r) X[pad8(jb * R0 + r)] = v[r];
  }
  __shared__ RowPtrs rp[TJ];  // the tile's psi rows and their ghost images
  for (int r = threadIdx.x; r < nrows; r += kNT) rp[r] = psi_row_ptrs(psi, Lp, hd, g, r0, r);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *wsm = sm + warp * RPW * LD;
  fft_warp<V, M, LOGRPW, 1, LD, true, 1, ct_nrad(M) - 1>(wsm, lane, tw);  // the middle passes
  __syncthreads();
  // the last pass with the store of psi and its ghost images
  inv_last_pass_store<V, M, LOGTJ, ACC>(sm, tw, psi, Lp, hd, g, scale, r0, nrows, rp);
}

// The same transform (FP64, M = 128 or 256) as a persistent grid of 3 CTAs
// per SM that stages each tile's spectrum in shared memory by cp.async, one
// tile ahead: the copies of tile t+1 (the (M+1) x TJ entries, TJ*16 contiguous
// bytes per kx) are issued as soon as the first pass of tile t has read its
// stage, so they land while tile t's middle passes, last pass and psi stores
// run.  k_fftx_inv issues a tile's loads only when its CTA starts and then
// waits for them.  Tiles go round-robin over the CTAs (every tile costs the
// same); the launcher takes this form only when every CTA gets two tiles or
// more.
template <int M>
__host__ __device__ constexpr size_t fftx_inv_pf_smem_bytes() {
  return fftx_smem_bytes(M, 16) + (size_t)(M + 1) * fftx_rows_per_cta(M) * 16;
}

template <int M>
__global__ void __launch_bounds__(kNT, 3) k_fftx_inv_pf(const double2 *__restrict__ spec, double *__restrict__ psi,
                                                       Lay Lp, int hd, GridK g, const double2 *__restrict__ twx,
                                                       const double2 *__restrict__ tpx, double scale) {
  using V = double2;
  constexpr int LOGRPW = ct_lognb(M), RPW = 1 << LOGRPW, LOGTJ = LOGRPW + 3, TJ = 1 << LOGTJ;
  constexpr int LD = x_row_stride(M);
  extern __shared__ __align__(16) unsigned char smx[];
  V *sm = reinterpret_cast<V *>(smx);
  V *tw = sm + TJ * LD;
  V *stg = tw + M;  // stage: entry (kx, row) at kx*TJ + row
  __shared__ RowPtrs rp[TJ];  // the tile's psi rows and their ghost images
  for (int t = threadIdx.x; t < ct_twiddle_len(M); t += kNT) tw[t] = tpx[t];
  const int ntile = (int)((g.R + TJ - 1) / TJ);
  auto stage = [&](int tile) {
    const int r0 = tile << LOGTJ, nrows = min(TJ, (int)g.R - r0);
    for (int t = threadIdx.x; t < (M + 1) * TJ; t += kNT) {
      const int kx = t >> LOGTJ, row = t & (TJ - 1);
      if (row < nrows) cp_async16(stg + t, spec + (long)kx * g.R + r0 + row);
    }
    cp_async_commit();
  };
  int tile = blockIdx.x;
  if (tile < ntile) stage(tile);
  constexpr int R0 = ct_rad(M, 0), PER = M / R0, NB0 = PER << LOGTJ;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (; tile < ntile; tile += gridDim.x) {
    const int r0 = tile << LOGTJ, nrows = min(TJ, (int)g.R - r0);
    cp_async_wait_all();
    __syncthreads();  // the stage holds this tile; the previous tile's stores have read sm
    // first pass: Z[n] = (X_n + conj X_{M-n}) + i conj(W^n) (X_n - conj X_{M-n}), as in k_fftx_inv
#pragma unroll
    for (int t = threadIdx.x; t < NB0; t += kNT) {
      const int jb = t >> LOGTJ, row = t & (TJ - 1);
      V v[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) {
        const int n = jb + r * PER, m = M - n;
        V xa = mk<V>(0.0, 0.0), xb = xa;
        if (row < nrows) {
          xa = stg[(n << LOGTJ) + row];
          xb = stg[(m << LOGTJ) + row];
        }
        if (n == 0) {
          v[r] = mk<V>(xa.x + xb.x, xa.x - xb.x);  // the imaginary parts of X_0 and X_M are ignored
        } else {
          const V wa = cconj(twx[n]);
          V ep = mk<V>(xa.x + xb.x, xa.y - xb.y);
          V em = mk<V>(xa.x - xb.x, xa.y + xb.y);
          V t1 = cmul(wa, em);
          v[r] = mk<V>(ep.x - t1.y, ep.y + t1.x);  // ep + i t1
        }
      }
      bfly<V, R0, true>(v);
      V *X = sm + row * LD;
#pragma unroll
      for (int r = 0; r < R0; ++r) X[pad8(jb * R0 + r)] = v[r];
    }
    for (int r = threadIdx.x; r < nrows; r += kNT) rp[r] = psi_row_ptrs(psi, Lp, hd, g, r0, r);
    __syncthreads();  // the stage is free, the first pass is in sm, the row pointers are in rp
    if (tile + (int)gridDim.x < ntile) stage(tile + gridDim.x);
    V *wsm = sm + warp * RPW * LD;
    fft_warp<V, M, LOGRPW, 1, LD, true, 1, ct_nrad(M) - 1>(wsm, lane, tw);  // the middle passes
    __syncthreads();
    inv_last_pass_store<V, M, LOGTJ, false>(sm, tw, psi, Lp, hd, g, scale, r0, nrows, rp);
  }
  cp_async_wait_all();
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

template <int M>
static void launch_fftx_inv_pf(const double2 *spec, double *psi, Lay Lp, int hd, const GridK &g, const double2 *twx,
                               const double2 *tpx, double scale, int sms, cudaStream_t st) {
  constexpr int TJ = fftx_rows_per_cta(M);
  long nblk = (g.R + TJ - 1) / TJ;
  if (nblk > 3L * sms) nblk = 3L * sms;
  k_fftx_inv_pf<M><<<(unsigned)nblk, kNT, fftx_inv_pf_smem_bytes<M>(), st>>>(spec, psi, Lp, hd, g, twx, tpx, scale);
}

void launch_fftx_inv(const double2 *spec, double *psi, Lay Lp, int hd, const GridK &g, const double2 *twx,
                     const double2 *tpx, double scale, cudaStream_t st) {
  int dev = 0, sms = 0;
  if ((g.M == 128 || g.M == 256) && cudaGetDevice(&dev) == cudaSuccess &&
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0) {
    const long ntile = (g.R + fftx_rows_per_cta(g.M) - 1) / fftx_rows_per_cta(g.M);
    if (ntile >= 6L * sms) {  // two tiles or more per CTA
      if (g.M == 128) launch_fftx_inv_pf<128>(spec, psi, Lp, hd, g, twx, tpx, scale, sms, st);
      else launch_fftx_inv_pf<256>(spec, psi, Lp, hd, g, twx, tpx, scale, sms, st);
      return;
    }
  }
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
  set((const void *)k_fftx_inv<float2, L, true>, fftx_smem_bytes(L, 8));     \
  set((const void *)k_rhs_fftx<L, false>, fftx_smem_bytes(L, 16));           \
  set((const void *)k_rhs_fftx<L, true>, fftx_smem_bytes(L, 16));
  TBFP_FFT_LENGTHS(TBFP_CASE)
#undef TBFP_CASE
  set((const void *)k_fftx_inv_pf<128>, fftx_inv_pf_smem_bytes<128>());
  set((const void *)k_fftx_inv_pf<256>, fftx_inv_pf_smem_bytes<256>());
  return e;
}

}  // namespace tbfp
