// FP64 kernels of the split-pressure projection (FAST_MODE of the reference).
//
// Spectrum layout in HBM: S[kx][row], row = (k-1)*ny + (j-1), kx = 0..nx/2.
// For a fixed kx the x rows are contiguous, so
//   * the x transforms (one CTA per tile of consecutive rows) write/read
//     contiguous runs of the tile's rows for every kx,
//   * the z transform of a fixed (kx, j) column strides by ny (a CTA stages a
//     tile of consecutive j columns for all k in shared memory),
//   * the y system of a fixed (kx, kz) is the contiguous run S[kx][kz*ny ...].
// This replaces the six pencil transposes of pencilDec.f90:359-562.
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"

namespace tbfp {

constexpr int kNT = 256;   // threads per CTA of the transform kernels (8 warps)
constexpr int kNW = kNT / 32;
constexpr int kWPB = 4;    // warps per CTA of the tridiagonal kernel

static int pow2_floor(int v) {
  int p = 1;
  while (2 * p <= v) p *= 2;
  return p;
}
static int ilog2i(int v) {
  int l = 0;
  while ((2 << l) <= v) ++l;
  return l;
}
// Each warp transforms its own sequences (rows of x, columns of z) with
// __syncwarp only; a warp holds 8 complex values per lane (16 for lengths 512).
// Sequences per warp: the largest power of two keeping n*spw <= 256, or 1.
static int seq_per_warp(int n) { return n >= 256 ? 1 : pow2_floor(256 / n); }
static int elems_per_lane(int n) { return n * seq_per_warp(n) / 32; }
int fft_max_length() { return 512; }
int fftx_rows_per_cta(int M) { return kNW * seq_per_warp(M); }
int fftz_cols_per_cta(int nz) { return kNW * seq_per_warp(nz); }
// Row stride of an x tile (complex slots): holds pad8(M)+1 slots; with nb rows
// per warp interleaved in a phase of 8 lanes, rows must land on distinct
// 16-byte bank groups: stride = (8/nb)*odd (mod 8) for nb < 8, odd for nb >= 8.
static int x_row_stride(int M) {
  const int nb = seq_per_warp(M);
  int ld = pad8(M) + 1;
  if (nb == 1) return ld;
  const int want = nb >= 8 ? 1 : 8 / nb;  // required residue pattern
  while (!((ld % 8) % want == 0 && ((ld % 8) / want) % 2 == 1)) ++ld;
  return ld;
}
// Row stride of a z tile: the tile's 8*nb columns plus a skew for small nb.
static int z_row_stride(int nz) {
  const int nb = seq_per_warp(nz);
  return 8 * nb + (nb <= 4 ? nb : 0);
}
size_t fftx_smem_bytes(int M) { return (size_t)fftx_rows_per_cta(M) * x_row_stride(M) * sizeof(double2); }
size_t fftz_smem_bytes(int nz) { return (size_t)z_row_stride(nz) * (pad8(nz - 1) + 1) * sizeof(double2); }
// per warp: (rows per lane + 1) x 33 slots of (complex rhs, two real coefficients)
static int tri_rows_per_lane(int ny) {
  const int NL = ny / 2 < 32 ? ny / 2 : 32;
  return (ny + NL - 1) / NL;
}
size_t tridiag_smem_bytes(int ny) {
  return (size_t)kWPB * 33 * tri_rows_per_lane(ny) * (sizeof(double2) + 2 * sizeof(double));
}

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
// Split right-hand side at one cell: computeSource (poissonEqn.f90:224-253) with
// computeOldPressDiv (:270-301), nl = 2.  Divisions by metrics are products with
// host-computed reciprocals; 1/rho comes from the precomputed array.
// ---------------------------------------------------------------------------
template <bool ST>
__device__ __forceinline__ double rhs_cell(const RhsArgs &a, const GridK &g, int i, int j, int k) {
  const double ddx = (a.ux[at(a.Lux, i, j, k)] - a.ux[at(a.Lux, i - 1, j, k)]) * g.idxf1;
  const double ddy = (a.uy[at(a.Luy, i, j, k)] - a.uy[at(a.Luy, i, j - 1, k)]) * g.idyf[j - 1];
  const double ddz = (a.uz[at(a.Luz, i, j, k)] - a.uz[at(a.Luz, i, j, k - 1)]) * g.idzf1;
  double s = ((ddx + ddy) + ddz) * a.r * a.rho0;

  const long c = at(a.Lrho, i, j, k);
  const double irc = a.irho[c];
  const double h = a.rho0 * 0.5;
  const double apx = 1.0 - h * (a.irho[c + 1] + irc);
  const double amx = 1.0 - h * (a.irho[c - 1] + irc);
  const double apy = 1.0 - h * (a.irho[c + a.Lrho.sj] + irc);
  const double amy = 1.0 - h * (a.irho[c - a.Lrho.sj] + irc);
  const double apz = 1.0 - h * (a.irho[c + a.Lrho.sk] + irc);
  const double amz = 1.0 - h * (a.irho[c - a.Lrho.sk] + irc);

  const long p = at(a.Lpsi, i, j, k);
  const long sj = a.Lpsi.sj, sk = a.Lpsi.sk;
  const double pc = a.pn[p], oc = a.pnm1[p];
  double dpxp = (2.0 * (a.pn[p + 1] - pc) - (a.pnm1[p + 1] - oc)) * g.idxc1;
  double dpxm = (2.0 * (pc - a.pn[p - 1]) - (oc - a.pnm1[p - 1])) * g.idxc1;
  double dpyp = (2.0 * (a.pn[p + sj] - pc) - (a.pnm1[p + sj] - oc)) * g.idyc[j];
  double dpym = (2.0 * (pc - a.pn[p - sj]) - (oc - a.pnm1[p - sj])) * g.idyc[j - 1];
  double dpzp = (2.0 * (a.pn[p + sk] - pc) - (a.pnm1[p + sk] - oc)) * g.idzc1;
  double dpzm = (2.0 * (pc - a.pn[p - sk]) - (oc - a.pnm1[p - sk])) * g.idzc1;
  if constexpr (ST) {
    const long x0 = at(a.Lst[0], i, j, k), y0 = at(a.Lst[1], i, j, k), z0 = at(a.Lst[2], i, j, k);
    dpxp = dpxp - 2.0 * a.stn[0][x0] + a.sto[0][x0];
    dpxm = dpxm - 2.0 * a.stn[0][x0 - 1] + a.sto[0][x0 - 1];
    dpyp = dpyp - 2.0 * a.stn[1][y0] + a.sto[1][y0];
    dpym = dpym - 2.0 * a.stn[1][y0 - a.Lst[1].sj] + a.sto[1][y0 - a.Lst[1].sj];
    dpzp = dpzp - 2.0 * a.stn[2][z0] + a.sto[2][z0];
    dpzm = dpzm - 2.0 * a.stn[2][z0 - a.Lst[2].sk] + a.sto[2][z0 - a.Lst[2].sk];
  }
  s = s + (apx * dpxp - amx * dpxm) * g.idxf1;
  s = s + (apy * dpyp - amy * dpym) * g.idyf[j - 1];
  s = s + (apz * dpzp - amz * dpzm) * g.idzf1;
  return s;
}

// ---------------------------------------------------------------------------
// Forward x transform of a tile of rows: real rows (from s, or computed by the
// split RHS) -> half-length complex FFT -> r2c post-processing -> S[kx][row].
// ---------------------------------------------------------------------------
template <int MODE, bool ST, int EMAX>
__global__ void __launch_bounds__(kNT, 2) k_fftx_fwd(const double *__restrict__ s_in, Lay Ls, RhsArgs ra, GridK g,
                                                  FftPlan pl, const double2 *__restrict__ twx,
                                                  double2 *__restrict__ spec, int logrpw, int ld) {
  extern __shared__ double2 sm[];
  const int RPW = 1 << logrpw;         // rows per warp
  const int logTJ = logrpw + 3;        // kNW = 8 warps
  const int TJ = 1 << logTJ;
  const int M = g.M, nx = g.nx;
  const int r0 = blockIdx.x << logTJ;
  const int nrows = min(TJ, (int)g.R - r0);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *wsm = sm + (long)warp * RPW * ld;  // this warp's rows
  double *wsr = reinterpret_cast<double *>(wsm);

  for (int rl = 0; rl < RPW; ++rl) {
    const int row = warp * RPW + rl;
    double *dst = wsr + (long)rl * 2 * ld;
    if (row < nrows) {
      const unsigned rr = (unsigned)(r0 + row);
      const int k = (int)(rr / (unsigned)g.ny) + 1, j = (int)(rr - (unsigned)(k - 1) * g.ny) + 1;
#pragma unroll 4
      for (int ii = lane; ii < nx; ii += 32) {
        const int slot = 2 * pad8(ii >> 1) + (ii & 1);
        if constexpr (MODE == 0) dst[slot] = s_in[at(Ls, ii + 1, j, k)];
        else dst[slot] = rhs_cell<ST>(ra, g, ii + 1, j, k);
      }
    } else {
      for (int ii = lane; ii < nx; ii += 32) dst[2 * pad8(ii >> 1) + (ii & 1)] = 0.0;
    }
  }
  __syncwarp();
  fft_group<double2, EMAX, false, 32>(wsm, lane, pl, logrpw, 1, ld, twx, 2);

  // X[k] = 1/2[(Z_k + conj Z_{M-k}) - i W^k (Z_k - conj Z_{M-k})], W = exp(-2 pi i/nx)
  const int npair = M / 2 + 1;
  for (int rl = 0; rl < RPW; ++rl) {
    double2 *Z = wsm + (long)rl * ld;
    for (int kk = lane; kk < npair; kk += 32) {
      if (kk == 0) {
        const double2 z0 = Z[0];
        Z[0] = mk<double2>(z0.x + z0.y, 0.0);
        Z[pad8(M)] = mk<double2>(z0.x - z0.y, 0.0);
      } else {
        const int km = M - kk;
        const double2 a = Z[pad8(kk)], b = Z[pad8(km)];
        const double2 wa = twx[kk], wb = twx[km];
        double2 ep = mk<double2>(a.x + b.x, a.y - b.y);  // Z_k + conj Z_{M-k}
        double2 em = mk<double2>(a.x - b.x, a.y + b.y);  // Z_k - conj Z_{M-k}
        double2 t1 = cmul(wa, em);                        // W^k * em
        Z[pad8(kk)] = mk<double2>(0.5 * (ep.x + t1.y), 0.5 * (ep.y - t1.x));  // (ep - i t1)/2
        if (km != kk) {
          double2 fp = mk<double2>(b.x + a.x, b.y - a.y);
          double2 fm = mk<double2>(b.x - a.x, b.y + a.y);
          double2 t2 = cmul(wb, fm);
          Z[pad8(km)] = mk<double2>(0.5 * (fp.x + t2.y), 0.5 * (fp.y - t2.x));
        }
      }
    }
  }
  __syncthreads();
  // S[kx][r0 + row]: consecutive threads take consecutive rows of one kx
  for (int t = threadIdx.x; t < ((M + 1) << logTJ); t += kNT) {
    const int kx = t >> logTJ, row = t & (TJ - 1);
    if (row < nrows) spec[(long)kx * g.R + r0 + row] = sm[(long)row * ld + pad8(kx)];
  }
}

template <int MODE, bool ST>
static void launch_x_fwd(const double *s, Lay Ls, const RhsArgs &ra, const GridK &g, const FftPlan &pl,
                         const double2 *twx, double2 *spec, cudaStream_t st) {
  const int TJ = fftx_rows_per_cta(g.M);
  const long nblk = (g.R + TJ - 1) / TJ;
  const int lr = ilog2i(seq_per_warp(g.M)), ld = x_row_stride(g.M);
  if (elems_per_lane(g.M) <= 8)
    k_fftx_fwd<MODE, ST, 8><<<(unsigned)nblk, kNT, fftx_smem_bytes(g.M), st>>>(s, Ls, ra, g, pl, twx, spec, lr, ld);
  else
    k_fftx_fwd<MODE, ST, 16><<<(unsigned)nblk, kNT, fftx_smem_bytes(g.M), st>>>(s, Ls, ra, g, pl, twx, spec, lr, ld);
}

void launch_fftx_fwd_from_s(const double *s, Lay Ls, const GridK &g, const FftPlan &pl, const double2 *twx,
                            double2 *spec, cudaStream_t st) {
  RhsArgs ra{};
  launch_x_fwd<0, false>(s, Ls, ra, g, pl, twx, spec, st);
}

void launch_fftx_fwd_rhs(const RhsArgs &ra, bool has_st, const GridK &g, const FftPlan &pl, const double2 *twx,
                         double2 *spec, cudaStream_t st) {
  Lay Ls{};
  if (has_st) launch_x_fwd<1, true>(nullptr, Ls, ra, g, pl, twx, spec, st);
  else launch_x_fwd<1, false>(nullptr, Ls, ra, g, pl, twx, spec, st);
}

// Standalone split RHS (tbfp_rhs_split): s on the interior; grid (x tiles, ny, nz).
template <bool ST>
__global__ void __launch_bounds__(128) k_rhs(RhsArgs ra, GridK g, double *__restrict__ s, Lay Ls) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  if (i <= g.nx) s[at(Ls, i, j, k)] = rhs_cell<ST>(ra, g, i, j, k);
}

void launch_rhs(const RhsArgs &ra, bool has_st, const GridK &g, double *s, Lay Ls, cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, g.ny, g.nz);
  if (has_st) k_rhs<true><<<grid, 128, 0, st>>>(ra, g, s, Ls);
  else k_rhs<false><<<grid, 128, 0, st>>>(ra, g, s, Ls);
}

// ---------------------------------------------------------------------------
// z transform (forward or backward) of a tile of TJz consecutive j columns of
// one kx plane: S[kx][(k-1)*ny + j-1], k = 1..nz, staged in shared memory.
// ---------------------------------------------------------------------------
template <bool INV, int EMAX>
__global__ void __launch_bounds__(kNT, 2) k_fftz(double2 *__restrict__ spec, GridK g, FftPlan pl,
                                              const double2 *__restrict__ twz, int logcpw, int ES) {
  extern __shared__ double2 sm[];
  const int logT = logcpw + 3;  // columns per CTA (8 warps)
  const int TJz = 1 << logT;
  const int kx = blockIdx.y;
  const int j0 = blockIdx.x << logT;
  const int nj = min(TJz, g.ny - j0);
  double2 *base = spec + (long)kx * g.R + j0;
  const int nz = g.nz, ny = g.ny;
  for (int t = threadIdx.x; t < (nz << logT); t += kNT) {
    const int k = t >> logT, jj = t & (TJz - 1);
    sm[pad8(k) * ES + jj] = (jj < nj) ? base[(long)k * ny + jj] : mk<double2>(0.0, 0.0);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  fft_group<double2, EMAX, INV, 32>(sm + (warp << logcpw), lane, pl, logcpw, ES, 1, twz, 1);
  __syncthreads();
  for (int t = threadIdx.x; t < (nz << logT); t += kNT) {
    const int k = t >> logT, jj = t & (TJz - 1);
    if (jj < nj) base[(long)k * ny + jj] = sm[pad8(k) * ES + jj];
  }
}

void launch_fftz(double2 *spec, const GridK &g, const FftPlan &pl, const double2 *twz, bool inverse,
                 cudaStream_t st) {
  const int TJz = fftz_cols_per_cta(g.nz);
  const int lc = ilog2i(seq_per_warp(g.nz));
  dim3 grid((g.ny + TJz - 1) / TJz, g.nkx);
  const size_t sb = fftz_smem_bytes(g.nz);
  const int es = z_row_stride(g.nz);
  const bool e8 = elems_per_lane(g.nz) <= 8;
  if (inverse) {
    if (e8) k_fftz<true, 8><<<grid, kNT, sb, st>>>(spec, g, pl, twz, lc, es);
    else k_fftz<true, 16><<<grid, kNT, sb, st>>>(spec, g, pl, twz, lc, es);
  } else {
    if (e8) k_fftz<false, 8><<<grid, kNT, sb, st>>>(spec, g, pl, twz, lc, es);
    else k_fftz<false, 16><<<grid, kNT, sb, st>>>(spec, g, pl, twz, lc, es);
  }
}

// ---------------------------------------------------------------------------
// y systems (solveTriDiag, fastPoissonSolver.f90:280-333): one warp per (kx,kz).
// Row j (0-based) scaled as in the reference, r = 1/(lam - am - ap):
//     a_j x_{j-1} + x_j + c_j x_{j+1} = d_j,  a = am*r, c = ap*r, d = f*r.
// Each lane owns a contiguous block [s,e] of rows (partition method):
//   forward within the block:  at_i x_{s-1} + x_i + ct_i x_{i+1} = dt_i
//   running backward pass:     x_s = hd - ha x_{s-1} - hc x_e
// which gives one reduced equation per lane in y_l = x_{e_l}:
//   at_e y_{l-1} + (1 - ct_e ha') y_l - ct_e hc' y_{l+1} = dt_e - ct_e hd'
// (primes: the next lane's hat values), solved by parallel cyclic reduction
// over the warp; then x_i = dt_i - at_i y_{l-1} - ct_i x_{i+1}.
// The singular (0,0) system (Neumann walls) is gauged by pinning its last
// unknown to zero, then its volume-weighted mean is removed in spectral space:
// sum_{i,k} p(i,j,k) = X(0,j,0), so zeroAveragePressure (:388-423) is
// X(0,j,0) -= nx*nz * dx*dz*sum_j dyf(j) X(0,j,0) / s_Vg.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double shup(double v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
__device__ __forceinline__ double shdn(double v, int d) { return __shfl_down_sync(0xffffffffu, v, d); }

__global__ void __launch_bounds__(kWPB * 32) k_tridiag(double2 *__restrict__ spec, GridK g,
                                                       const double *__restrict__ lamx,
                                                       const double *__restrict__ lamz,
                                                       const double *__restrict__ am, const double *__restrict__ ap,
                                                       const double *__restrict__ dyf, double mean_c, double nxnz,
                                                       int T) {
  extern __shared__ unsigned char smraw[];
  const int ny = g.ny;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // per warp, interleaved by lane: row t of lane l at [t*33 + l]
  const int W = 33 * T;
  double2 *d = reinterpret_cast<double2 *>(smraw) + (long)warp * W;
  double *ca = reinterpret_cast<double *>(reinterpret_cast<double2 *>(smraw) + (long)kWPB * W) + (long)warp * 2 * W;
  double *cc = ca + W;
  const long q = (long)blockIdx.x * kWPB + warp;
  if (q >= (long)g.nkx * g.nz) return;  // whole warp leaves; no block-level barrier follows
  const int kx = (int)(q / g.nz), kz = (int)(q % g.nz);
  double2 *S = spec + (long)kx * g.R + (long)kz * ny;

  const int NL = min(32, ny / 2);
  const int nb = ny / NL, rem = ny - nb * NL;
  const int split = rem * (nb + 1);  // rows owned by the lanes with nb+1 rows
  // slot of global row e
  auto slot = [&](int e) -> int {
    int l, t;
    if (e < split) {
      l = e / (nb + 1);
      t = e - l * (nb + 1);
    } else {
      const int f = e - split;
      l = rem + f / nb;
      t = f - (l - rem) * nb;
    }
    return t * 33 + l;
  };
  for (int e = lane; e < ny; e += 32) d[slot(e)] = S[e];
  __syncwarp();

  const double lam = lamx[kx] + lamz[kz];
  const bool pin = (kx == 0 && kz == 0);
  const bool active = lane < NL;
  const int s0 = lane * nb + min(lane, rem);  // first global row of this lane
  const int len = active ? nb + (lane < rem ? 1 : 0) : 0;

  double at_e = 0.0, ct_e = 0.0;
  double2 dt_e = mk<double2>(0.0, 0.0);
  if (active) {
    double at_p = 0.0, ct_p = 0.0;
    double2 dt_p = mk<double2>(0.0, 0.0);
    for (int t = 0; t < len; ++t) {
      const int i = s0 + t;
      const double r = 1.0 / (lam - am[i] - ap[i]);
      double a = am[i] * r, c = ap[i] * r;
      const int sl = t * 33 + lane;
      double2 dd = cscale(d[sl], r);
      if (pin && i == ny - 1) {
        a = 0.0;
        c = 0.0;
        dd = mk<double2>(0.0, 0.0);
      }
      double at, ct;
      double2 dt;
      if (t == 0) {
        at = a;
        ct = c;
        dt = dd;
      } else {
        const double inv = 1.0 / (1.0 - a * ct_p);
        at = -a * at_p * inv;
        ct = c * inv;
        dt = mk<double2>((dd.x - a * dt_p.x) * inv, (dd.y - a * dt_p.y) * inv);
      }
      ca[sl] = at;
      cc[sl] = ct;
      d[sl] = dt;
      at_p = at;
      ct_p = ct;
      dt_p = dt;
    }
    at_e = at_p;
    ct_e = ct_p;
    dt_e = dt_p;
  }
  // running backward pass for x_s in terms of x_{s-1} and x_e
  double ha = 0.0, hc = -1.0;
  double2 hd = mk<double2>(0.0, 0.0);
  if (active && len >= 2) {
    int sl = (len - 2) * 33 + lane;
    hd = d[sl];
    ha = ca[sl];
    hc = cc[sl];
    for (int t = len - 3; t >= 0; --t) {
      sl = t * 33 + lane;
      const double ct = cc[sl];
      const double2 dv = d[sl];
      hd = mk<double2>(dv.x - ct * hd.x, dv.y - ct * hd.y);
      ha = ca[sl] - ct * ha;
      hc = -ct * hc;
    }
  }
  const double ha_n = shdn(ha, 1), hc_n = shdn(hc, 1);
  const double hdx_n = shdn(hd.x, 1), hdy_n = shdn(hd.y, 1);
  double A = 0.0, B = 1.0, C = 0.0, Dx = 0.0, Dy = 0.0;
  if (active) {
    A = at_e;
    if (lane + 1 < NL) {
      B = 1.0 - ct_e * ha_n;
      C = -ct_e * hc_n;
      Dx = dt_e.x - ct_e * hdx_n;
      Dy = dt_e.y - ct_e * hdy_n;
    } else {
      Dx = dt_e.x;
      Dy = dt_e.y;
    }
  }
  // parallel cyclic reduction over the 32 reduced equations
#pragma unroll
  for (int h = 1; h < 32; h <<= 1) {
    double Am = shup(A, h), Bm = shup(B, h), Cm = shup(C, h), Dxm = shup(Dx, h), Dym = shup(Dy, h);
    double Ap = shdn(A, h), Bp = shdn(B, h), Cp = shdn(C, h), Dxp = shdn(Dx, h), Dyp = shdn(Dy, h);
    if (lane < h) {
      Am = 0.0; Bm = 1.0; Cm = 0.0; Dxm = 0.0; Dym = 0.0;
    }
    if (lane + h >= 32) {
      Ap = 0.0; Bp = 1.0; Cp = 0.0; Dxp = 0.0; Dyp = 0.0;
    }
    const double k1 = A / Bm, k2 = C / Bp;
    const double nA = -k1 * Am, nC = -k2 * Cp;
    const double nB = B - k1 * Cm - k2 * Ap;
    const double nDx = Dx - k1 * Dxm - k2 * Dxp, nDy = Dy - k1 * Dym - k2 * Dyp;
    A = nA; B = nB; C = nC; Dx = nDx; Dy = nDy;
  }
  const double iB = 1.0 / B;
  const double yx = Dx * iB, yy = Dy * iB;
  double xsx = shup(yx, 1), xsy = shup(yy, 1);
  if (lane == 0) { xsx = 0.0; xsy = 0.0; }
  if (active) {
    double2 xn = mk<double2>(yx, yy);
    d[(len - 1) * 33 + lane] = xn;
    for (int t = len - 2; t >= 0; --t) {
      const int sl = t * 33 + lane;
      const double a = ca[sl], c = cc[sl];
      const double2 dv = d[sl];
      xn = mk<double2>(dv.x - a * xsx - c * xn.x, dv.y - a * xsy - c * xn.y);
      d[sl] = xn;
    }
  }
  __syncwarp();
  if (pin) {
    double sx = 0.0, sy = 0.0;
    for (int e = lane; e < ny; e += 32) {
      const double2 v = d[slot(e)];
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
      d[sl] = mk<double2>(d[sl].x - subx, d[sl].y - suby);
    }
    __syncwarp();
  }
  for (int e = lane; e < ny; e += 32) S[e] = d[slot(e)];
}

void launch_tridiag(double2 *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                    const double *ap, const double *dyf, double mean_c, double nxnz, cudaStream_t st) {
  const long nsys = (long)g.nkx * g.nz;
  const long nblk = (nsys + kWPB - 1) / kWPB;
  k_tridiag<<<(unsigned)nblk, kWPB * 32, tridiag_smem_bytes(g.ny), st>>>(spec, g, lamx, lamz, am, ap, dyf, mean_c,
                                                                         nxnz, tri_rows_per_lane(g.ny));
}

// ---------------------------------------------------------------------------
// Inverse x transform of a tile of rows: S[kx][row] -> c2r -> psi rows scaled
// by 1/(nx*nz) (fastPoissonSolver.f90:371-378), written with every ghost image
// of updateBoundaries (field.f90:950-974 on one rank): the first y ghost layer
// copies the wall cell (normalGradient, bf=0), x and z ghosts are periodic.
// The imaginary parts of X[0] and X[nx/2] are ignored, as FFTW's c2r does.
// ---------------------------------------------------------------------------
template <int EMAX>
__global__ void __launch_bounds__(kNT, 2) k_fftx_inv(const double2 *__restrict__ spec, double *__restrict__ psi,
                                                  Lay Lp, int hd, GridK g, FftPlan pl,
                                                  const double2 *__restrict__ twx, double scale, int logrpw,
                                                  int ld) {
  extern __shared__ double2 sm[];
  const int RPW = 1 << logrpw;
  const int logTJ = logrpw + 3;
  const int TJ = 1 << logTJ;
  const int M = g.M, nx = g.nx;
  const int r0 = blockIdx.x << logTJ;
  const int nrows = min(TJ, (int)g.R - r0);
  for (int t = threadIdx.x; t < ((M + 1) << logTJ); t += kNT) {
    const int kx = t >> logTJ, row = t & (TJ - 1);
    sm[(long)row * ld + pad8(kx)] = (row < nrows) ? spec[(long)kx * g.R + r0 + row] : mk<double2>(0.0, 0.0);
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *wsm = sm + (long)warp * RPW * ld;
  // Z[k] = (X_k + conj X_{M-k}) + i conj(W^k) (X_k - conj X_{M-k}),  k = 0..M-1
  const int npair = M / 2 + 1;
  for (int rl = 0; rl < RPW; ++rl) {
    double2 *X = wsm + (long)rl * ld;
    for (int kk = lane; kk < npair; kk += 32) {
      if (kk == 0) {
        const double a = X[0].x, b = X[pad8(M)].x;
        X[0] = mk<double2>(a + b, a - b);
      } else {
        const int km = M - kk;
        const double2 a = X[pad8(kk)], b = X[pad8(km)];
        const double2 wa = cconj(twx[kk]), wb = cconj(twx[km]);
        double2 ep = mk<double2>(a.x + b.x, a.y - b.y);
        double2 em = mk<double2>(a.x - b.x, a.y + b.y);
        double2 t1 = cmul(wa, em);
        X[pad8(kk)] = mk<double2>(ep.x - t1.y, ep.y + t1.x);  // ep + i t1
        if (km != kk) {
          double2 fp = mk<double2>(b.x + a.x, b.y - a.y);
          double2 fm = mk<double2>(b.x - a.x, b.y + a.y);
          double2 t2 = cmul(wb, fm);
          X[pad8(km)] = mk<double2>(fp.x - t2.y, fp.y + t2.x);
        }
      }
    }
  }
  __syncwarp();
  fft_group<double2, EMAX, true, 32>(wsm, lane, pl, logrpw, 1, ld, twx, 2);
  const double *wsr = reinterpret_cast<const double *>(wsm);
  for (int rl = 0; rl < RPW; ++rl) {
    const int row = warp * RPW + rl;
    if (row >= nrows) break;
    const unsigned rr = (unsigned)(r0 + row);
    const int k = (int)(rr / (unsigned)g.ny) + 1, j = (int)(rr - (unsigned)(k - 1) * g.ny) + 1;
    // ghost images of the row: first y ghost layer (wall copy), periodic z
    int js[2], ks[2];
    int nj = 1, nk = 1;
    js[0] = j;
    ks[0] = k;
    if (j == 1) js[nj++] = 0;
    else if (j == g.ny) js[nj++] = g.ny + 1;
    if (k <= hd) ks[nk++] = k + g.nz;
    else if (k > g.nz - hd) ks[nk++] = k - g.nz;
    const double *src = wsr + (long)rl * 2 * ld;
    for (int ii = lane; ii < nx; ii += 32) {
      const double v = src[2 * pad8(ii >> 1) + (ii & 1)] * scale;
      const int i = ii + 1;
      int is[2];
      int ni = 1;
      is[0] = i;
      if (i <= hd) is[ni++] = i + nx;
      else if (i > nx - hd) is[ni++] = i - nx;
      for (int c = 0; c < nk; ++c)
        for (int b = 0; b < nj; ++b) {
          double *prow = psi + at(Lp, 0, js[b], ks[c]);
          for (int a = 0; a < ni; ++a) prow[is[a] - Lp.ilo] = v;
        }
    }
  }
}

void launch_fftx_inv(const double2 *spec, double *psi, Lay Lp, int hd, const GridK &g, const FftPlan &pl,
                     const double2 *twx, double scale, cudaStream_t st) {
  const int TJ = fftx_rows_per_cta(g.M);
  const long nblk = (g.R + TJ - 1) / TJ;
  const int lr = ilog2i(seq_per_warp(g.M)), ld = x_row_stride(g.M);
  if (elems_per_lane(g.M) <= 8)
    k_fftx_inv<8><<<(unsigned)nblk, kNT, fftx_smem_bytes(g.M), st>>>(spec, psi, Lp, hd, g, pl, twx, scale, lr, ld);
  else
    k_fftx_inv<16><<<(unsigned)nblk, kNT, fftx_smem_bytes(g.M), st>>>(spec, psi, Lp, hd, g, pl, twx, scale, lr, ld);
}

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
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (l == 0) atomicMax(out, (unsigned long long)__double_as_longlong(v));
  }
}

// Out-of-place correction fused with the continuity check.  Grid (x tiles of
// 128, y chunks of kJC rows, nz); a thread owns column (i, k) of a y chunk and
// walks it in j, so the lower y face of a cell is the upper face computed one
// step before; the lower x face comes from the neighbouring lane (recomputed
// by lane 0 and at i = 1).  The periodic duplicates ux(0)=ux(nx),
// uz(.,.,0)=uz(.,.,nz) are the equated values of vfield.f90:124-189 and the uy
// wall faces are copied through.  |div u| (auxiliaryRoutines.f90:71-75) is
// reduced per block and folded into *maxdiv with one atomic.
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
__global__ void __launch_bounds__(128, 7) k_correct_div(CorrArgs a, GridK g, unsigned long long *__restrict__ maxdiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int k = blockIdx.z + 1;
  const int j0 = blockIdx.y * kJC + 1, j1 = min(j0 + kJC - 1, g.ny);
  const bool valid = i <= g.nx;
  const int lane = threadIdx.x & 31;
  const int ic = valid ? i : g.nx;  // clamped index keeps every load in bounds
  const int km = (k == 1) ? g.nz : k - 1;
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
  const long pjs = a.Lpsi.sj, pks = a.Lpsi.sk, rjs = a.Lrho.sj, rks = a.Lrho.sk;
  const double r = a.r, ir0 = a.invrho0;
  const double idxc = g.idxc1, idzc = g.idzc1;
  const double idx = g.idxf[ic - 1], idz = g.idzf[k - 1];
  // surface-tension terms of one face (zero without surface tension)
  auto stx = [&](int ii, int jj, int kk) -> double {
    if constexpr (ST) {
      const long q = at(a.Lst[0], ii, jj, kk);
      return 2.0 * a.stn[0][q] - a.sto[0][q];
    } else return 0.0;
  };
  auto sty = [&](int ii, int jj, int kk) -> double {
    if constexpr (ST) {
      const long q = at(a.Lst[1], ii, jj, kk);
      return 2.0 * a.stn[1][q] - a.sto[1][q];
    } else return 0.0;
  };
  auto stz = [&](int ii, int jj, int kk) -> double {
    if constexpr (ST) {
      const long q = at(a.Lst[2], ii, jj, kk);
      return 2.0 * a.stn[2][q] - a.sto[2][q];
    } else return 0.0;
  };

  // centre values of the current cell, carried along j
  long p = at(a.Lpsi, ic, j0, k), q = at(a.Lrho, ic, j0, k);
  double psc = ps[p], pnc = pn[p], poc = po[p], irc = ir[q];
  double uym;
  if (j0 > 1) {
    const double psm = ps[p - pjs], pnm = pn[p - pjs], pom = po[p - pjs], irm = ir[q - rjs];
    uym = face_update(uyi[at(a.Luy, ic, j0 - 1, k)], r, ir0, irc, irm, g.idyc[j0 - 1], psc, psm, pnc, pnm, poc, pom,
                      sty(ic, j0 - 1, k));
  } else {
    uym = uyi[at(a.Luy, ic, 0, k)];
  }
  if (valid && j0 == 1) uyo[at(a.Luy, i, 0, k)] = uym;
  const long pxw = (i == 1) ? (long)(g.nx - 1) : -1;  // offset to the lower x neighbour's centre
  double vmax = 0.0;
  for (int j = j0; j <= j1; ++j) {
    // every load of this step, issued together
    const double psx = ps[p + 1], pnx = pn[p + 1], pox = po[p + 1], irx = ir[q + 1];
    const double psy = ps[p + pjs], pny = pn[p + pjs], poy = po[p + pjs], iry = ir[q + rjs];
    const double psz = ps[p + pks], pnz = pn[p + pks], poz = po[p + pks], irz = ir[q + rks];
    const long pm = (k == 1) ? p + (long)(g.nz - 1) * pks : p - pks;
    const long qm = (k == 1) ? q + (long)(g.nz - 1) * rks : q - rks;
    const double psm = ps[pm], pnm = pn[pm], pom = po[pm], irm = ir[qm];
    const double ux_c = uxi[at(a.Lux, ic, j, k)];
    const double uy_c = uyi[at(a.Luy, ic, j, k)];
    const double uz_c = uzi[at(a.Luz, ic, j, k)];
    const double uz_m = uzi[at(a.Luz, ic, j, km)];

    const double uxp = face_update(ux_c, r, ir0, irx, irc, idxc, psx, psc, pnx, pnc, pox, poc, stx(ic, j, k));
    const double up = __shfl_up_sync(0xffffffffu, uxp, 1);
    double uxm = up;
    if (lane == 0 || i == 1) {  // lower x face: recompute (periodic wrap at i = 1)
      const long pw = (i == 1) ? p + pxw : p - 1;
      const long qw = (i == 1) ? q + pxw : q - 1;
      const int iw = (i == 1) ? g.nx : ic - 1;
      uxm = face_update(uxi[at(a.Lux, iw, j, k)], r, ir0, ir[qw + 1], ir[qw], idxc, ps[pw + 1], ps[pw], pn[pw + 1],
                        pn[pw], po[pw + 1], po[pw], stx(iw, j, k));
    }
    const double uyp = (j < g.ny) ? face_update(uy_c, r, ir0, iry, irc, g.idyc[j], psy, psc, pny, pnc, poy, poc,
                                                sty(ic, j, k))
                                  : uy_c;
    const double uzp = face_update(uz_c, r, ir0, irz, irc, idzc, psz, psc, pnz, pnc, poz, poc, stz(ic, j, k));
    const double uzm = face_update(uz_m, r, ir0, irc, irm, idzc, psc, psm, pnc, pnm, poc, pom, stz(ic, j, km));
    if (valid) {
      uxo[at(a.Lux, i, j, k)] = uxp;
      if (i == g.nx) uxo[at(a.Lux, 0, j, k)] = uxp;
      uyo[at(a.Luy, i, j, k)] = uyp;
      uzo[at(a.Luz, i, j, k)] = uzp;
      if (k == g.nz) uzo[at(a.Luz, i, j, 0)] = uzp;
      double dv = (uxp - uxm) * idx;
      dv = dv + (uyp - uym) * g.idyf[j - 1];
      dv = dv + (uzp - uzm) * idz;
      vmax = fmax(vmax, fabs(dv));
    }
    uym = uyp;
    psc = psy;
    pnc = pny;
    poc = poy;
    irc = iry;
    p += pjs;
    q += rjs;
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
  if (k == g.nz) a.uzo[at(a.Luz, i, j, 0)] = uzp;
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
      vmax = fmax(vmax, fabs(dv));
    }
  }
  block_max_atomic(vmax, maxdiv);
}

void launch_div(const double *ux, const double *uy, const double *uz, Lay Lux, Lay Luy, Lay Luz, const GridK &g,
                unsigned long long *maxdiv, cudaStream_t st) {
  dim3 grid((g.nx + 127) / 128, (g.ny + kJC - 1) / kJC, g.nz);
  k_div<<<grid, 128, 0, st>>>(ux, uy, uz, Lux, Luy, Luz, g, maxdiv);
}

// Raise the dynamic shared-memory limits once per process.
cudaError_t prepare_kernels() {
  const int big = 227 * 1024;
  cudaError_t e = cudaSuccess;
#define TBFP_ATTR(fn)                                                                 \
  do {                                                                                \
    cudaError_t ee = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, big); \
    if (ee != cudaSuccess) e = ee;                                                    \
  } while (0)
  TBFP_ATTR((k_fftx_fwd<0, false, 8>));
  TBFP_ATTR((k_fftx_fwd<1, false, 8>));
  TBFP_ATTR((k_fftx_fwd<1, true, 8>));
  TBFP_ATTR((k_fftx_fwd<0, false, 16>));
  TBFP_ATTR((k_fftx_fwd<1, false, 16>));
  TBFP_ATTR((k_fftx_fwd<1, true, 16>));
  TBFP_ATTR((k_fftz<false, 8>));
  TBFP_ATTR((k_fftz<true, 8>));
  TBFP_ATTR((k_fftz<false, 16>));
  TBFP_ATTR((k_fftz<true, 16>));
  TBFP_ATTR(k_tridiag);
  TBFP_ATTR(k_fftx_inv<8>);
  TBFP_ATTR(k_fftx_inv<16>);
#undef TBFP_ATTR
  return e;
}

}  // namespace tbfp
