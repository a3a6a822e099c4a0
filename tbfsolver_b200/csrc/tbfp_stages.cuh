// Tile bodies of the FP64/FP32 projection kernels as device functions.
//
// The z transform, y solve and correction kernels (tbfp_yz.cu, tbfp_correct.cu)
// are thin __global__ wrappers that call these bodies with their block
// coordinates; the persistent ensemble kernel (tbfp_ensemble.cu) calls the
// same bodies for the tiles it takes from its work queue.  The RHS and the two
// x transforms (tbfp_xfft.cu) keep kernel-form copies of the same code: called
// as device functions they ran 15-25 % slower at 512x384x256 (same box, CUDA
// events; explicit read-only loads did not recover it), so the x-direction
// bodies below serve the persistent kernel only and must be kept equal to the
// kernels there.  COH = true reads
// the buffers that are written during the same launch (1/rho, s, the spectrum,
// psi) through L2 (ld.global.cg): a persistent kernel consumes data that other
// blocks of the same launch produced, which the read-only and L1 paths of a
// plain load do not guarantee to see.  The standalone kernels use COH = false.
#pragma once
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"

namespace tbfp {

// Loads of data that the standalone kernel only reads: the read-only path
// (__ldg; a kernel parameter declared const __restrict__ got it implicitly, a
// device function's parameter does not).  COH: through L2 (the persistent
// kernel, where another block of the launch may have written the data).
template <bool COH, typename X>
__device__ __forceinline__ X ldc(const X *p) {
  if constexpr (COH) return __ldcg(p);
  else return __ldg(p);
}
// Loads of data the kernel itself writes elsewhere (the in-place z transform).
template <bool COH, typename X>
__device__ __forceinline__ X ldw(const X *p) {
  if constexpr (COH) return __ldcg(p);
  else return *p;
}

constexpr int kRJ = 32;                // y rows walked by one thread of the RHS kernel
constexpr int kNoGhost = -(1 << 30);  // no ghost image of this index

// 1/rho over elements [t0, t1) of the (halo-inclusive) density array.
__device__ __forceinline__ void recip_body(const double *__restrict__ rho, double *__restrict__ irho, long t0,
                                           long t1, int tid, int nthreads) {
  for (long t = t0 + tid; t < t1; t += nthreads) irho[t] = 1.0 / rho[t];
}

__device__ __forceinline__ double shup(double v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ double shdn(double v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

// ---------------------------------------------------------------------------
// Forward x transform (see k_fftx_fwd in tbfp_xfft.cu)
// ---------------------------------------------------------------------------
// The last Stockham pass of the forward half-length transforms of a tile of
// TJ = 2^LOGTJ rows (the earlier passes done, rows at sm + row*LD in the pad8
// layout), fused with the r2c pair step
//   X[k] = 1/2[(Z_k + conj Z_{M-k}) - i W^k (Z_k - conj Z_{M-k})], W = exp(-2 pi i/nx)
// and the store of S[kx][r0 + row].  Output k = b + r*NS of last-pass butterfly
// b pairs with output M-k of butterfly NS-b, so thread (b, row) runs both
// butterflies in registers and stores both halves of every pair: the last
// pass's shared-memory writes and the pair step's reads are gone.
template <typename V, int M, int LOGTJ>
__device__ __forceinline__ void fwd_last_pass_r2c_store(const V *sm, const V *tw, const V *__restrict__ twx,
                                                        V *__restrict__ spec, long R, int r0, int nrows) {
  using T = decltype(V::x);
  constexpr int TJ = 1 << LOGTJ, LD = x_row_stride(M);
  constexpr int PL = ct_nrad(M) - 1, RL = ct_rad(M, PL), NS = ct_ns(M, PL), TWO = NS - ct_rad(M, 0);
  constexpr int NITEM = NS == 1 ? 1 : NS / 2 + 1;  // butterflies b = 0 .. NS/2
  const T half = T(0.5);
  auto pair = [&](V zk, V zm, int k, int row) {  // X_k and X_{M-k} from Z_k, Z_{M-k}
    V *o = spec + r0 + row;
    const int m = M - k;
    const V wa = twx[k], wb = twx[m];
    V ep = mk<V>(zk.x + zm.x, zk.y - zm.y);  // Z_k + conj Z_{M-k}
    V em = mk<V>(zk.x - zm.x, zk.y + zm.y);  // Z_k - conj Z_{M-k}
    V t1 = cmul(wa, em);                      // W^k * em
    o[(long)k * R] = mk<V>(half * (ep.x + t1.y), half * (ep.y - t1.x));  // (ep - i t1)/2
    if (m != k) {
      V fp = mk<V>(zm.x + zk.x, zm.y - zk.y);
      V fm = mk<V>(zm.x - zk.x, zm.y + zk.y);
      V t2 = cmul(wb, fm);
      o[(long)m * R] = mk<V>(half * (fp.x + t2.y), half * (fp.y - t2.x));
    }
  };
  auto butterfly = [&](const V *X, int b, V *v) {  // last-pass butterfly b of one row
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      V x = X[pad8(b + r * NS)];
      if constexpr (NS > 1) {
        if (r > 0) x = cmul(x, tw[TWO + b * (RL - 1) + (r - 1)]);
      }
      v[r] = x;
    }
    bfly<V, RL, false>(v);
  };
#pragma unroll
  for (int t = threadIdx.x; t < (NITEM << LOGTJ); t += kNT) {
    const int b = t >> LOGTJ, row = t & (TJ - 1);
    if (row >= nrows) continue;
    const V *X = sm + row * LD;
    V u[RL];
    butterfly(X, b, u);
    if (b == 0) {  // outputs r*NS: Z_0 with Z_M (the Nyquist term), r with RL - r
      V *o = spec + r0 + row;
      o[0] = mk<V>(u[0].x + u[0].y, T(0));
      o[(long)M * R] = mk<V>(u[0].x - u[0].y, T(0));
#pragma unroll
      for (int r = 1; r <= RL / 2; ++r) pair(u[r], u[RL - r], r * NS, row);
    } else if (2 * b == NS) {  // outputs NS/2 + r*NS: r with RL - 1 - r
#pragma unroll
      for (int r = 0; 2 * r <= RL - 1; ++r) pair(u[r], u[RL - 1 - r], b + r * NS, row);
    } else {  // with butterfly NS - b: r with RL - 1 - r
      V w[RL];
      butterfly(X, NS - b, w);
#pragma unroll
      for (int r = 0; r < RL; ++r) pair(u[r], w[RL - 1 - r], b + r * NS, row);
    }
  }
}

template <typename V, int M, int MODE, bool COH = false>
__device__ __forceinline__ void fftx_fwd_body(XSrc src, GridK g, const V *__restrict__ twx,
                                              const V *__restrict__ tpx, V *__restrict__ spec, int bx,
                                              unsigned char * /*dynamic shared memory: named below*/) {
  extern __shared__ __align__(16) unsigned char smx[];  // the launch's dynamic shared memory
  using T = decltype(V::x);
  constexpr int LOGRPW = ct_lognb(M), RPW = 1 << LOGRPW, LOGTJ = LOGRPW + 3, TJ = 1 << LOGTJ;
  constexpr int LD = x_row_stride(M), NX = 2 * M, NXC = (NX + 31) / 32;
  V *sm = reinterpret_cast<V *>(smx);
  V *tw = sm + TJ * LD;
  __shared__ double red[kNW][3];
  for (int t = threadIdx.x; t < ct_twiddle_len(M); t += kNT) tw[t] = __ldg(tpx + t);
  const int r0 = bx << LOGTJ;
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
            const double v = ldc<COH>(srow + ii + 1);
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
  fwd_last_pass_r2c_store<V, M, LOGTJ>(sm, tw, twx, spec, g.R, r0, nrows);
}

// ---------------------------------------------------------------------------
// Split right-hand side (see k_rhs in tbfp_xfft.cu)
// ---------------------------------------------------------------------------
template <bool ST, bool COH = false>
__device__ __forceinline__ void rhs_body(RhsArgs a, GridK g, double *__restrict__ s, Lay Ls, int bx, int by, int bz,
                                         int tx) {
  const int i = bx * 128 + tx + 1;
  const int k = bz + 1;
  const int j0 = by * kRJ + 1, j1 = min(j0 + kRJ - 1, g.ny);
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
  double irc = ldc<COH>(ir + (oq)), pc = __ldg(pn + (op)), oc = __ldg(po + (op));
  double irm = ldc<COH>(ir + (oq - rjs)), pm = __ldg(pn + (op - pjs)), om = __ldg(po + (op - pjs));
  double uym = __ldg(uy + (oy - yjs));
  for (int j = j0; j <= j1; ++j) {
    const double uxc = __ldg(ux + (ox)), uxm = __ldg(ux + (ox - 1)), uyc = __ldg(uy + (oy)), uzc = __ldg(uz + (oz)), uzm = __ldg(uz + (oz - zks));
    const double irxp = ldc<COH>(ir + (oq + 1)), irxm = ldc<COH>(ir + (oq - 1)), iryp = ldc<COH>(ir + (oq + rjs)), irzp = ldc<COH>(ir + (oq + rks)), irzm = ldc<COH>(ir + (oq - rks));
    const double pxp = __ldg(pn + (op + 1)), pxm = __ldg(pn + (op - 1)), pyp = __ldg(pn + (op + pjs)), pzp = __ldg(pn + (op + pks)), pzm = __ldg(pn + (op - pks));
    const double oxp = __ldg(po + (op + 1)), oxm = __ldg(po + (op - 1)), oyp = __ldg(po + (op + pjs)), ozp = __ldg(po + (op + pks)), ozm = __ldg(po + (op - pks));
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

// ---------------------------------------------------------------------------
// Inverse x transform (see k_fftx_inv in tbfp_xfft.cu)
// ---------------------------------------------------------------------------
// The last Stockham pass of the inverse half-length transforms of a tile of
// TJ = 2^LOGTJ rows (the earlier passes done, rows at sm + row*LD in the pad8
// layout), fused with the store of the psi rows: complex output n of a row
// holds psi at i = 2n+1 and 2n+2, scaled by 1/(nx*nz) (plus the old psi when
// ACC), written with every ghost image of updateBoundaries (field.f90:950-974
// on one rank): periodic x, the first y ghost layer copying the wall cell, and
// periodic z unless the rows belong to a z slab.  Thread (b, row) runs
// last-pass butterfly b of one row; 32 consecutive b write 512 contiguous
// bytes.  For a one-pass length the tile is already transformed and is
// stored as it stands.
// The psi row (x index 0) of spectrum row r0 + row and its ghost images
// (y wall copy, periodic z), null where a row has none.
struct RowPtrs {
  double *p00, *p10, *p01, *p11;
};
__device__ __forceinline__ RowPtrs psi_row_ptrs(double *psi, Lay Lp, int hd, const GridK &g, int r0, int row) {
  const unsigned rr = (unsigned)(r0 + row);
  const int k = (int)(rr / (unsigned)g.ny) + 1, j = (int)(rr - (unsigned)(k - 1) * g.ny) + 1;
  const int jg = (j == 1) ? 0 : (j == g.ny ? g.ny + 1 : -1);
  const int kg = g.slab ? kNoGhost : ((k <= hd) ? k + g.nz : (k > g.nz - hd ? k - g.nz : kNoGhost));
  RowPtrs q;
  q.p00 = psi + at(Lp, 0, j, k);
  q.p10 = (jg >= 0) ? psi + at(Lp, 0, jg, k) : nullptr;
  q.p01 = (kg != kNoGhost) ? psi + at(Lp, 0, j, kg) : nullptr;
  q.p11 = (q.p10 && q.p01) ? psi + at(Lp, 0, jg, kg) : nullptr;
  return q;
}

// rp: the tile's row pointers made beforehand (one per row, in shared
// memory), or null to make them per butterfly
template <typename V, int M, int LOGTJ, bool ACC>
__device__ __forceinline__ void inv_last_pass_store(const V *sm, const V *tw, double *__restrict__ psi, Lay Lp,
                                                    int hd, const GridK &g, double scale, int r0, int nrows,
                                                    const RowPtrs *rp = nullptr) {
  using T = decltype(V::x);
  constexpr int LD = x_row_stride(M), NX = 2 * M;
  constexpr int NP = ct_nrad(M), RL = ct_rad(M, NP - 1), NSL = ct_ns(M, NP - 1), TWL = NSL - ct_rad(M, 0);
  auto row_ptrs = [&](int row) { return rp ? rp[row] : psi_row_ptrs(psi, Lp, hd, g, r0, row); };
  auto put = [&](const RowPtrs &q, int i, double v) {
    if constexpr (ACC) v += q.p00[i];  // refinement: psi += correction
    const int ig = (i <= hd) ? i + NX : (i > NX - hd ? i - NX : kNoGhost);
    q.p00[i] = v;
    if (ig != kNoGhost) q.p00[ig] = v;
    if (q.p10) {
      q.p10[i] = v;
      if (ig != kNoGhost) q.p10[ig] = v;
    }
    if (q.p01) {
      q.p01[i] = v;
      if (ig != kNoGhost) q.p01[ig] = v;
    }
    if (q.p11) {
      q.p11[i] = v;
      if (ig != kNoGhost) q.p11[ig] = v;
    }
  };
  if constexpr (NP == 1) {
    constexpr int LNX = ct_log2(NX);  // NX = 8 or 16
#pragma unroll 1
    for (int t = threadIdx.x; t < (NX << LOGTJ); t += kNT) {
      const int ii = t & (NX - 1), row = t >> LNX;
      if (row >= nrows) continue;
      const T *src = reinterpret_cast<const T *>(sm + row * LD);
      put(row_ptrs(row), ii + 1, (double)src[2 * pad8(ii >> 1) + (ii & 1)] * scale);
    }
  } else {
    constexpr int LNSL = ct_log2(NSL);
#pragma unroll 1
    for (int t = threadIdx.x; t < (NSL << LOGTJ); t += kNT) {
      const int b = t & (NSL - 1), row = t >> LNSL;
      if (row >= nrows) continue;
      const V *X = sm + row * LD;
      V v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        V x = X[pad8(b + r * NSL)];
        if (r > 0) {
          V w = tw[TWL + b * (RL - 1) + (r - 1)];
          w.y = -w.y;
          x = cmul(x, w);
        }
        v[r] = x;
      }
      bfly<V, RL, true>(v);
      const RowPtrs q = row_ptrs(row);
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const int n = b + r * NSL;
        put(q, 2 * n + 1, (double)v[r].x * scale);
        put(q, 2 * n + 2, (double)v[r].y * scale);
      }
    }
  }
}

template <typename V, int M, bool ACC, bool COH = false>
__device__ __forceinline__ void fftx_inv_body(const V *__restrict__ spec, double *__restrict__ psi, Lay Lp, int hd,
                                              GridK g, const V *__restrict__ twx, const V *__restrict__ tpx,
                                              double scale, int bx, unsigned char * /*dynamic shared memory: named below*/) {
  extern __shared__ __align__(16) unsigned char smx[];  // the launch's dynamic shared memory
  using T = decltype(V::x);
  constexpr int LOGRPW = ct_lognb(M), RPW = 1 << LOGRPW, LOGTJ = LOGRPW + 3, TJ = 1 << LOGTJ;
  constexpr int LD = x_row_stride(M);
  V *sm = reinterpret_cast<V *>(smx);
  V *tw = sm + TJ * LD;
  for (int t = threadIdx.x; t < ct_twiddle_len(M); t += kNT) tw[t] = __ldg(tpx + t);
  const int r0 = bx << LOGTJ;
  const int nrows = min(TJ, (int)g.R - r0);
  // Z[n] = (X_n + conj X_{M-n}) + i conj(W^n) (X_n - conj X_{M-n}), made as the
  // spectrum comes in and fed straight into the first radix-R0 pass (as k_fftx_inv)
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
        xa = ldc<COH>(spec + ((long)n * g.R + r0 + row));
        xb = ldc<COH>(spec + ((long)m * g.R + r0 + row));
      }
      if (n == 0) {
        v[r] = mk<V>(xa.x + xb.x, xa.x - xb.x);  // the imaginary parts of X_0 and X_M are ignored
      } else {
        const V wa = cconj(__ldg(twx + n));
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
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  V *wsm = sm + warp * RPW * LD;
  fft_warp<V, M, LOGRPW, 1, LD, true, 1, ct_nrad(M) - 1>(wsm, lane, tw);  // the middle passes
  __syncthreads();
  inv_last_pass_store<V, M, LOGTJ, ACC>(sm, tw, psi, Lp, hd, g, scale, r0, nrows);
}

// ---------------------------------------------------------------------------
// z transform and y systems (see k_fftz and k_tridiag_t in tbfp_yz.cu)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rcp_nr(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

template <int T>
__host__ __device__ constexpr int tri_min_blocks() {
  return T <= 6 ? 6 : (T <= 8 ? 4 : 3);
}


template <typename V, bool INV, int NZ, bool COH = false>
__device__ __forceinline__ void fftz_body(V *__restrict__ spec, GridK g, const V *__restrict__ tpz, int bx, int by,
                                          unsigned char * /*dynamic shared memory: named below*/) {
  extern __shared__ __align__(16) unsigned char smz[];  // the launch's dynamic shared memory
  constexpr int LOGCPW = ct_lognb(NZ), LOGT = LOGCPW + 3, TJZ = 1 << LOGT;
  constexpr int ES = z_row_stride(NZ), ROWS = pad8(NZ - 1) + 1;
  V *sm = reinterpret_cast<V *>(smz);
  V *tw = sm + ES * ROWS;
  const int kx = by;
  const int j0 = bx << LOGT;
  const int nj = min(TJZ, g.ny - j0);
  const int ny = g.ny;
  V *base = spec + (long)kx * g.R + j0;
  using T = decltype(V::x);
  // The first pass reads its inputs from HBM and the last pass writes its
  // outputs to HBM, so the tile goes through shared memory only between
  // passes.  Thread (b, column): butterfly b of one column; eight columns of
  // one k are 128 contiguous bytes.
  constexpr int NP = ct_nrad(NZ), R0 = ct_rad(NZ, 0), PER0 = NZ / R0;
  constexpr int RL = ct_rad(NZ, NP - 1), NSL = ct_ns(NZ, NP - 1), TWL = NSL - R0;
  auto load_col = [&](int k, int jj) -> V {
    return (jj < nj) ? ldw<COH>(base + ((long)k * ny + jj)) : mk<V>(T(0), T(0));
  };
  if constexpr (NP == 1) {  // one pass: HBM -> registers -> HBM
#pragma unroll
    for (int t = threadIdx.x; t < TJZ; t += kNT) {
      V v[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) v[r] = load_col(r, t);
      bfly<V, R0, INV>(v);
      if (t < nj) {
#pragma unroll
        for (int r = 0; r < R0; ++r) base[(long)r * ny + t] = v[r];
      }
    }
    return;
  } else {
    for (int t = threadIdx.x; t < ct_twiddle_len(NZ); t += kNT) tw[t] = tpz[t];
#pragma unroll
    for (int t = threadIdx.x; t < (PER0 << LOGT); t += kNT) {
      const int b = t >> LOGT, jj = t & (TJZ - 1);
      V v[R0];
#pragma unroll
      for (int r = 0; r < R0; ++r) v[r] = load_col(b + r * PER0, jj);
      bfly<V, R0, INV>(v);
#pragma unroll
      for (int r = 0; r < R0; ++r) sm[pad8(b * R0 + r) * ES + jj] = v[r];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    fft_warp<V, NZ, LOGCPW, ES, 1, INV, 1, NP - 1>(sm + (warp << LOGCPW), lane, tw);  // the middle passes
    __syncthreads();
#pragma unroll
    for (int t = threadIdx.x; t < (NSL << LOGT); t += kNT) {
      const int b = t >> LOGT, jj = t & (TJZ - 1);
      V v[RL];
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        V x = sm[pad8(b + r * NSL) * ES + jj];
        if (r > 0) {
          V w = tw[TWL + b * (RL - 1) + (r - 1)];
          if constexpr (INV) w.y = -w.y;
          x = cmul(x, w);
        }
        v[r] = x;
      }
      bfly<V, RL, INV>(v);
      if (jj < nj) {
#pragma unroll
        for (int r = 0; r < RL; ++r) base[(long)(b + r * NSL) * ny + jj] = v[r];
      }
    }
  }
}

// Serial Thomas sweep of the pinned (0,0) y system on one thread: row e's
// right-hand side at d0[slot(e)], its off-diagonals from am_at(e), ap_at(e);
// the elimination factors go to cpin[slot(e)] and the solution back to d0.
// The last unknown is pinned to zero (Neumann walls make the system
// singular).  The next row's operands are loaded one step ahead, so the loads
// stay off the dependent chain of the elimination, and the reciprocal is the
// Newton-refined rcp_nr of the parallel elimination.
template <typename SlotF, typename AmF, typename ApF>
__device__ __forceinline__ void pinned_sweep(double2 *d0, double *cpin, double lam, int ny, SlotF slot, AmF am_at,
                                             ApF ap_at) {
  double ct_p = 0.0;
  double2 dt_p = mk<double2>(0.0, 0.0);
  double a_n = am_at(0), c_n = ap_at(0);
  double2 f_n = d0[slot(0)];
  for (int e = 0; e < ny - 1; ++e) {
    const double a = a_n, c = c_n;
    const double2 f = f_n;
    const int sl = slot(e);
    if (e + 1 < ny - 1) {
      a_n = am_at(e + 1);
      c_n = ap_at(e + 1);
      f_n = d0[slot(e + 1)];
    }
    const double gi = rcp_nr((lam - a - c) - a * ct_p);
    ct_p = c * gi;
    dt_p = mk<double2>((f.x - a * dt_p.x) * gi, (f.y - a * dt_p.y) * gi);
    cpin[sl] = ct_p;
    d0[sl] = dt_p;
  }
  {
    const int sl = slot(ny - 1);
    cpin[sl] = 0.0;
    d0[sl] = mk<double2>(0.0, 0.0);
  }
  double2 xn = mk<double2>(0.0, 0.0);
  double c_b = cpin[slot(ny - 2)];
  double2 d_b = d0[slot(ny - 2)];
  for (int e = ny - 2; e >= 0; --e) {
    const double c = c_b;
    const double2 dv = d_b;
    const int sl = slot(e);
    if (e > 0) {
      c_b = cpin[slot(e - 1)];
      d_b = d0[slot(e - 1)];
    }
    xn = mk<double2>(dv.x - c * xn.x, dv.y - c * xn.y);
    d0[sl] = xn;
  }
}

// The same sweep with the elimination factors of the pinned system taken from
// a table (fs[2e] = 1/pivot, fs[2e+1] = ct_e for e < ny-1, made once per
// handle by k_pin_factors with the arithmetic above): the system's matrix does
// not change between calls, so only the right-hand side's recurrence is left
// on the dependent chain.
template <typename SlotF, typename AmF>
__device__ __forceinline__ void pinned_sweep_f(double2 *d0, const double *fs, int ny, SlotF slot, AmF am_at) {
  double2 dt_p = mk<double2>(0.0, 0.0);
  double a_n = am_at(0), g_n = fs[0];
  double2 f_n = d0[slot(0)];
  for (int e = 0; e < ny - 1; ++e) {
    const double a = a_n, gi = g_n;
    const double2 f = f_n;
    const int sl = slot(e);
    if (e + 1 < ny - 1) {
      a_n = am_at(e + 1);
      g_n = fs[2 * (e + 1)];
      f_n = d0[slot(e + 1)];
    }
    dt_p = mk<double2>((f.x - a * dt_p.x) * gi, (f.y - a * dt_p.y) * gi);
    d0[sl] = dt_p;
  }
  d0[slot(ny - 1)] = mk<double2>(0.0, 0.0);
  double2 xn = mk<double2>(0.0, 0.0);
  double c_b = fs[2 * (ny - 2) + 1];
  double2 d_b = d0[slot(ny - 2)];
  for (int e = ny - 2; e >= 0; --e) {
    const double c = c_b;
    const double2 dv = d_b;
    const int sl = slot(e);
    if (e > 0) {
      c_b = fs[2 * (e - 1) + 1];
      d_b = d0[slot(e - 1)];
    }
    xn = mk<double2>(dv.x - c * xn.x, dv.y - c * xn.y);
    d0[sl] = xn;
  }
}

// Right-hand sides of the y systems (kx, kz) and (kx, nz - kz) into d0 / d1:
// row e lives in lane e / T at slot (e mod T)*33 + lane, padding rows are zero.
// FP64 rows go by cp.async (the caller waits for them); FP32 rows are widened
// through registers.
template <typename V, int T>
__device__ __forceinline__ void tri_pair_fill(const V *S0, const V *S1, bool two, int ny, int lane, double2 *d0,
                                              double2 *d1) {
#pragma unroll
  for (int c = 0; c < T; ++c) {
    const int e = lane + 32 * c;
    const int l = e / T, sl = (e - l * T) * 33 + l;
    if (e < ny) {
      if constexpr (sizeof(V) == sizeof(double2)) {
        cp_async16(d0 + sl, S0 + e);
        if (two) cp_async16(d1 + sl, S1 + e);
      } else {
        const V v0 = S0[e];
        d0[sl] = mk<double2>((double)v0.x, (double)v0.y);
        if (two) {
          const V v1 = S1[e];
          d1[sl] = mk<double2>((double)v1.x, (double)v1.y);
        }
      }
    } else {
      d0[sl] = mk<double2>(0.0, 0.0);
      d1[sl] = mk<double2>(0.0, 0.0);
    }
  }
}

template <typename V, int T, bool SMC = false>
__device__ __forceinline__ void tri_pair_solve(V *S0, V *S1, bool two, double lam, bool pin,
                                               const double *__restrict__ am, const double *__restrict__ ap,
                                               const double *__restrict__ dyf, double mean_c, double nxnz, int ny,
                                               int lane, double2 *d0, double2 *d1, const double *cam = nullptr,
                                               const double *cap = nullptr, const double *pinf = nullptr);

template <typename V, int T>
__device__ __forceinline__ void tridiag_t_body(V *__restrict__ spec, GridK g, const double *__restrict__ lamx,
                                               const double *__restrict__ lamz, const double *__restrict__ am,
                                               const double *__restrict__ ap, const double *__restrict__ dyf,
                                               double mean_c, double nxnz, unsigned q, int warp,
                                               unsigned char * /*dynamic shared memory: named below*/,
                                               const double *pinf = nullptr) {
  extern __shared__ __align__(16) unsigned char smraw[];  // the launch's dynamic shared memory
  constexpr int W = 33 * T;
  const int ny = g.ny, nz = g.nz;
  const int lane = threadIdx.x & 31;
  double2 *d0 = reinterpret_cast<double2 *>(smraw) + warp * 2 * W;
  double2 *d1 = d0 + W;
  const int nzh = nz / 2 + 1;
  if (q >= (unsigned)(g.nkx * nzh)) return;  // whole warp leaves; no block-level barrier follows
  const int kx = (int)(q / (unsigned)nzh), kz = (int)(q - (unsigned)kx * nzh);
  const int kz2 = (kz == 0) ? 0 : nz - kz;
  const bool two = kz2 != kz;
  V *S0 = spec + (long)kx * g.R + (long)kz * ny;
  V *S1 = spec + (long)kx * g.R + (long)kz2 * ny;
  tri_pair_fill<V, T>(S0, S1, two, ny, lane, d0, d1);
  const double lam = lamx[kx + g.kx0] + lamz[kz];
  const bool pin = (kx + g.kx0 == 0 && kz == 0);
  if constexpr (sizeof(V) == sizeof(double2)) cp_async_wait_all();
  __syncwarp();
  tri_pair_solve<V, T>(S0, S1, two, lam, pin, am, ap, dyf, mean_c, nxnz, ny, lane, d0, d1, nullptr, nullptr, pinf);
}

// Solve of the pair whose right-hand sides tri_pair_fill put in d0 / d1 (every
// lane's copies landed and a __syncwarp passed); the solutions go to S0 / S1.
// The (0,0) system (pin) has no partner, so d1 serves it as scratch.  SMC: the
// elimination reads the off-diagonals of the lane's rows from shared copies
// cam / cap (row t of lane l at [t*33 + l], zero on padding rows) instead of
// the global tables, whose lane-strided reads touch a cache line per lane.
template <typename V, int T, bool SMC>
__device__ __forceinline__ void tri_pair_solve(V *S0, V *S1, bool two, double lam, bool pin,
                                               const double *__restrict__ am, const double *__restrict__ ap,
                                               const double *__restrict__ dyf, double mean_c, double nxnz, int ny,
                                               int lane, double2 *d0, double2 *d1, const double *cam,
                                               const double *cap, const double *pinf) {
  using VT = decltype(V::x);
  auto st = [](double2 v) { return mk<V>((VT)v.x, (VT)v.y); };
  const int s0 = lane * T;

  if (pin) {  // single system: pinned serial Thomas, factors in d1
    double *cpin = reinterpret_cast<double *>(d1);
    auto slot = [&](int e) { return (e % T) * 33 + e / T; };
    if constexpr (SMC) {
      if (pinf) {  // the factor table, copied by the warp into d1
        for (int i = lane; i < 2 * (ny - 1); i += 32) cpin[i] = pinf[i];
        __syncwarp();
        if (lane == 0) pinned_sweep_f(d0, cpin, ny, slot, [&](int e) { return cam[slot(e)]; });
      } else if (lane == 0) {  // the shared copies use the right-hand sides' slots
        pinned_sweep(d0, cpin, lam, ny, slot, [&](int e) { return cam[slot(e)]; },
                     [&](int e) { return cap[slot(e)]; });
      }
    } else if (pinf) {  // the factor table, copied by the warp into d1
      for (int i = lane; i < 2 * (ny - 1); i += 32) cpin[i] = pinf[i];
      __syncwarp();
      if (lane == 0) pinned_sweep_f(d0, cpin, ny, slot, [&](int e) { return am[e]; });
    } else if (lane == 0) {
      pinned_sweep(d0, cpin, lam, ny, slot, [&](int e) { return am[e]; }, [&](int e) { return ap[e]; });
    }
    __syncwarp();
    double sx = 0.0, sy = 0.0;
    for (int e = lane; e < ny; e += 32) {
      const double2 v = d0[slot(e)];
      sx += v.x * dyf[e];
      sy += v.y * dyf[e];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sx += __shfl_xor_sync(0xffffffffu, sx, o);
      sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    const double subx = sx * mean_c * nxnz, suby = sy * mean_c * nxnz;
    for (int e = lane; e < ny; e += 32) {
      const int sl = slot(e);
      S0[e] = st(mk<double2>(d0[sl].x - subx, d0[sl].y - suby));
    }
    return;
  }

  // forward elimination within the lane's block (padding rows: diagonal one)
  double at_r[T], ct_r[T];
  double at_p = -1.0, ct_p = 0.0;
  double2 p0 = mk<double2>(0.0, 0.0), p1 = mk<double2>(0.0, 0.0);
#pragma unroll
  for (int t = 0; t < T; ++t) {
    const bool real = s0 + t < ny;  // off-diagonals zero, diagonal one on padding rows
    double a, c;
    if constexpr (SMC) {
      a = cam[t * 33 + lane];
      c = cap[t * 33 + lane];
    } else {
      a = real ? am[s0 + t] : 0.0;
      c = real ? ap[s0 + t] : 0.0;
    }
    const double dg = real ? lam : 1.0;
    const int sl = t * 33 + lane;
    const double gi = rcp_nr((dg - a - c) - a * ct_p);
    const double2 f0 = d0[sl], f1 = d1[sl];
    p0 = mk<double2>((f0.x - a * p0.x) * gi, (f0.y - a * p0.y) * gi);
    p1 = mk<double2>((f1.x - a * p1.x) * gi, (f1.y - a * p1.y) * gi);
    d0[sl] = p0;
    d1[sl] = p1;
    at_p = -a * at_p * gi;
    ct_p = c * gi;
    at_r[t] = at_p;
    ct_r[t] = ct_p;
  }
  // running backward pass: x_s = hd - ha x_{s-1} - hc x_e
  double ha = 0.0, hc = -1.0;
  double2 h0 = mk<double2>(0.0, 0.0), h1 = mk<double2>(0.0, 0.0);
  if constexpr (T >= 2) {
    h0 = d0[(T - 2) * 33 + lane];
    h1 = d1[(T - 2) * 33 + lane];
    ha = at_r[T - 2];
    hc = ct_r[T - 2];
#pragma unroll
    for (int t = T - 3; t >= 0; --t) {
      const double2 v0 = d0[t * 33 + lane], v1 = d1[t * 33 + lane];
      const double ct = ct_r[t];
      h0 = mk<double2>(v0.x - ct * h0.x, v0.y - ct * h0.y);
      h1 = mk<double2>(v1.x - ct * h1.x, v1.y - ct * h1.y);
      ha = at_r[t] - ct * ha;
      hc = -ct * hc;
    }
  }
  // reduced equation of this lane: A y_{l-1} + B y_l + C y_{l+1} = D
  const double ha_n = shdn(ha, 1), hc_n = shdn(hc, 1);
  const double h0x = shdn(h0.x, 1), h0y = shdn(h0.y, 1), h1x = shdn(h1.x, 1), h1y = shdn(h1.y, 1);
  const double at_e = at_r[T - 1], ct_e = ct_r[T - 1];
  double A = at_e, B = 1.0, C = 0.0;
  double D[4] = {p0.x, p0.y, p1.x, p1.y};
  if (lane < 31) {
    B = 1.0 - ct_e * ha_n;
    C = -ct_e * hc_n;
    D[0] -= ct_e * h0x;
    D[1] -= ct_e * h0y;
    D[2] -= ct_e * h1x;
    D[3] -= ct_e * h1y;
  }
  // parallel cyclic reduction over the 32 reduced equations
#pragma unroll
  for (int h = 1; h < 32; h <<= 1) {
    const double iB = rcp_nr(B);
    double Am = shup(A, h), iBm = shup(iB, h), Cm = shup(C, h);
    double Ap = shdn(A, h), iBp = shdn(iB, h), Cp = shdn(C, h);
    double Dm[4], Dp[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      Dm[c] = shup(D[c], h);
      Dp[c] = shdn(D[c], h);
    }
    const bool lo = lane < h, hi = lane + h >= 32;
    const double k1 = lo ? 0.0 : A * iBm, k2 = hi ? 0.0 : C * iBp;
    if (lo) Am = Cm = 0.0;
    if (hi) Ap = Cp = 0.0;
    B = B - k1 * Cm - k2 * Ap;
    A = -k1 * Am;
    C = -k2 * Cp;
#pragma unroll
    for (int c = 0; c < 4; ++c) D[c] = D[c] - k1 * Dm[c] - k2 * Dp[c];
  }
  const double iBf = rcp_nr(B);
  double y[4], ys[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) y[c] = D[c] * iBf;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double v = shup(y[c], 1);  // every lane takes part in the shuffle
    ys[c] = (lane == 0) ? 0.0 : v;
  }
  double2 x0 = mk<double2>(y[0], y[1]), x1 = mk<double2>(y[2], y[3]);
  d0[(T - 1) * 33 + lane] = x0;
  d1[(T - 1) * 33 + lane] = x1;
#pragma unroll
  for (int t = T - 2; t >= 0; --t) {
    const int sl = t * 33 + lane;
    const double a = at_r[t], c = ct_r[t];
    const double2 v0 = d0[sl], v1 = d1[sl];
    x0 = mk<double2>(v0.x - a * ys[0] - c * x0.x, v0.y - a * ys[1] - c * x0.y);
    x1 = mk<double2>(v1.x - a * ys[2] - c * x1.x, v1.y - a * ys[3] - c * x1.y);
    d0[sl] = x0;
    d1[sl] = x1;
  }
  __syncwarp();
#pragma unroll
  for (int c = 0; c < T; ++c) {
    const int e = lane + 32 * c;
    if (e < ny) {
      const int l = e / T, sl = (e - l * T) * 33 + l;
      S0[e] = st(d0[sl]);
      if (two) S1[e] = st(d1[sl]);
    }
  }
}

// ---------------------------------------------------------------------------
// Velocity correction with the continuity check (see k_correct_div in tbfp_correct.cu)
// ---------------------------------------------------------------------------
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


template <bool ST, bool COH = false>
__device__ __forceinline__ void correct_div_body(CorrArgs a, GridK g, unsigned long long *__restrict__ maxdiv, int bx,
                                                 int by, int bz, int tx) {
  const int i = bx * 128 + tx + 1;
  const int k = bz + 1;
  const int j0 = by * kJC + 1, j1 = min(j0 + kJC - 1, g.ny);
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
  double psc = ldc<COH>(ps + (op)), pnc = __ldg(pn + (op)), poc = __ldg(po + (op)), irc = ldc<COH>(ir + (oq));
  double uym;
  if (j0 > 1) {
    uym = face_update(__ldg(uyi + (oy - yjs)), r, ir0, irc, ldc<COH>(ir + (oq - rjs)), g.idyc[j0 - 1], psc, ldc<COH>(ps + (op - pjs)), pnc,
                      __ldg(pn + (op - pjs)), poc, __ldg(po + (op - pjs)), stf(1, ic, j0 - 1, k));
  } else {
    uym = __ldg(uyi + (oy - yjs));
    if (valid) uyo[oy - yjs] = uym;
  }
  double vmax = 0.0;
  for (int j = j0; j <= j1; ++j) {
    // every load of this step, issued together
    const int ow = op + xo, qw = oq + xo;
    const double psx = ldc<COH>(ps + (op + 1)), pnx = __ldg(pn + (op + 1)), pox = __ldg(po + (op + 1)), irx = ldc<COH>(ir + (oq + 1));
    // the lower x face is the upper face of lane - 1; lane 0 computes it
    const bool lead = (threadIdx.x & 31) == 0;
    double psw = 0.0, pnw = 0.0, pow_ = 0.0, irw = 0.0, psw1 = 0.0, pnw1 = 0.0, pow1 = 0.0, irw1 = 0.0, ux_w = 0.0;
    if (lead) {
      psw = ldc<COH>(ps + (ow));
      pnw = __ldg(pn + (ow));
      pow_ = __ldg(po + (ow));
      irw = ldc<COH>(ir + (qw));
      psw1 = ldc<COH>(ps + (ow + 1));
      pnw1 = __ldg(pn + (ow + 1));
      pow1 = __ldg(po + (ow + 1));
      irw1 = ldc<COH>(ir + (qw + 1));
      ux_w = __ldg(uxi + (ox + xo));
    }
    const double psy = ldc<COH>(ps + (op + pjs)), pny = __ldg(pn + (op + pjs)), poy = __ldg(po + (op + pjs)), iry = ldc<COH>(ir + (oq + rjs));
    const double psz = ldc<COH>(ps + (op + pz)), pnz = __ldg(pn + (op + pz)), poz = __ldg(po + (op + pz)), irz = ldc<COH>(ir + (oq + qz));
    const double psm = ldc<COH>(ps + (op + pm)), pnm = __ldg(pn + (op + pm)), pom = __ldg(po + (op + pm)), irm = ldc<COH>(ir + (oq + qm));
    const double ux_c = __ldg(uxi + (ox)), uy_c = __ldg(uyi + (oy)), uz_c = __ldg(uzi + (oz)), uz_m = __ldg(uzi + (oz + zm));

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

}  // namespace tbfp
