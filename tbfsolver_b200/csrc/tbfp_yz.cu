// FP64 z transforms and y (tridiagonal) solves of the split-pressure
// projection (FAST_MODE of the reference), on the spectrum S[kx][row],
// row = (k-1)*ny + (j-1):
//   * the z transform of a fixed (kx, j) column strides by ny (a CTA stages a
//     tile of consecutive j columns for all k in shared memory),
//   * the y system of a fixed (kx, kz) is the contiguous run S[kx][kz*ny ...].
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"
#include "tbfp_stages.cuh"

namespace tbfp {

// ---------------------------------------------------------------------------
// z transform (forward or backward) of a tile of TJZ consecutive j columns of
// one kx plane, staged in shared memory (row k of the tile at pad8(k)*ES).
// ---------------------------------------------------------------------------
template <typename V, bool INV, int NZ>
__global__ void __launch_bounds__(kNT, (NZ >= 384 ? 2 : 3)) k_fftz(V *__restrict__ spec, GridK g,
                                                               const V *__restrict__ tpz) {
  extern __shared__ __align__(16) unsigned char smz[];
  fftz_body<V, INV, NZ>(spec, g, tpz, blockIdx.x, blockIdx.y, smz);
}

template <typename V, int NZ>
static void launch_fftz_n(V *spec, const GridK &g, const V *tpz, bool inverse, cudaStream_t st) {
  constexpr int TJZ = fftz_cols_per_cta(NZ);
  constexpr size_t smem = fftz_smem_bytes(NZ, sizeof(V));
  dim3 grid((g.ny + TJZ - 1) / TJZ, g.nkx);
  if (inverse) k_fftz<V, true, NZ><<<grid, kNT, smem, st>>>(spec, g, tpz);
  else k_fftz<V, false, NZ><<<grid, kNT, smem, st>>>(spec, g, tpz);
}

template <typename V>
static void launch_fftz_t(V *spec, const GridK &g, const V *tpz, bool inverse, cudaStream_t st) {
  switch (g.nz) {
#define TBFP_CASE(L) \
  case L: launch_fftz_n<V, L>(spec, g, tpz, inverse, st); break;
    TBFP_FFT_LENGTHS(TBFP_CASE)
#undef TBFP_CASE
    default: break;  // lengths are validated by tbfp_create
  }
}
void launch_fftz(double2 *spec, const GridK &g, const double2 *tpz, bool inverse, cudaStream_t st) {
  launch_fftz_t(spec, g, tpz, inverse, st);
}
void launch_fftz(float2 *spec, const GridK &g, const float2 *tpz, bool inverse, cudaStream_t st) {
  launch_fftz_t(spec, g, tpz, inverse, st);
}

// ---------------------------------------------------------------------------
// y systems (solveTriDiag, fastPoissonSolver.f90:280-333).  Row j (0-based) of
// the reference, before its row scaling by r = 1/(lam - am - ap), is
//     am_j x_{j-1} + (lam - am_j - ap_j) x_j + ap_j x_{j+1} = f_j,
// lam = lamx(kx) + lamz(kz).  lamz is even in kz (the host table is built
// symmetric), so the systems kz and nz-kz have the same matrix: one warp solves
// both, computing the elimination coefficients once for two right-hand sides.
// Lane l owns the T = ceil(ny/32) consecutive rows [l*T, l*T+len) (partition
// method).  Forward within the block, with g_i = 1/(lam - am_i - ap_i - am_i ct_{i-1})
// (ct, dt = 0 and at = -1 before the block):
//   at_i x_{s-1} + x_i + ct_i x_{i+1} = dt_i,
//   at_i = -am_i at_{i-1} g_i,  ct_i = ap_i g_i,  dt_i = (f_i - am_i dt_{i-1}) g_i,
// which is the reference's scaled elimination (a = am r, c = ap r, d = f r)
// with r cancelled.  A running backward pass gives
//   x_s = hd - ha x_{s-1} - hc x_e,
// so each lane contributes one reduced equation in y_l = x_{e_l}:
//   at_e y_{l-1} + (1 - ct_e ha') y_l - ct_e hc' y_{l+1} = dt_e - ct_e hd'
// (primes: the next lane's values), solved by parallel cyclic reduction over
// the warp; then x_i = dt_i - at_i y_{l-1} - ct_i x_{i+1}.
// The singular (0,0) system (Neumann walls) is gauged by pinning its last
// unknown to zero and solved by one lane (Thomas: the cyclic reduction loses
// digits on this only weakly diagonally dominant system); then its
// volume-weighted mean is removed in spectral space:
// sum_{i,k} p(i,j,k) = X(0,j,0), so zeroAveragePressure (:388-423) is
// X(0,j,0) -= nx*nz * dx*dz*sum_j dyf(j) X(0,j,0) / s_Vg.
// Shared memory per warp: row t of lane l at [t*33 + l] (conflict-free) for the
// two right-hand sides and the two coefficient arrays.  The arithmetic is FP64
// for both spectrum types (float2 spectra are widened on load).
// ---------------------------------------------------------------------------

// TM > 0: every lane holds at most TM rows and keeps their elimination
// coefficients at_i, ct_i in registers (shared memory holds only the two
// right-hand sides, so more warps fit per SM); TM = 0: any T, coefficients in
// shared memory.
template <typename V, int TM>
__global__ void __launch_bounds__(kWPB * 32) k_tridiag(V *__restrict__ spec, GridK g,
                                                       const double *__restrict__ lamx,
                                                       const double *__restrict__ lamz,
                                                       const double *__restrict__ am, const double *__restrict__ ap,
                                                       const double *__restrict__ dyf, double mean_c, double nxnz,
                                                       int T, unsigned magicT) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int ny = g.ny, nz = g.nz;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int W = 33 * T;
  double2 *d0 = reinterpret_cast<double2 *>(smraw) + warp * 2 * W;
  double2 *d1 = d0 + W;
  double *ca = nullptr, *cc = nullptr;
  if constexpr (TM == 0) {
    ca = reinterpret_cast<double *>(reinterpret_cast<double2 *>(smraw) + kWPB * 2 * W) + warp * 2 * W;
    cc = ca + W;
  }
  const int nzh = nz / 2 + 1;  // kz = 0..nz/2 (nz is even)
  const unsigned q = blockIdx.x * kWPB + warp;
  if (q >= (unsigned)(g.nkx * nzh)) return;  // whole warp leaves; no block-level barrier follows
  const int kx = (int)(q / (unsigned)nzh), kz = (int)(q - (unsigned)kx * nzh);
  const int kz2 = (kz == 0) ? 0 : nz - kz;  // partner system (itself at kz = 0 and nz/2)
  const bool two = kz2 != kz;
  V *S0 = spec + (long)kx * g.R + (long)kz * ny;
  V *S1 = spec + (long)kx * g.R + (long)kz2 * ny;
  using VT = decltype(V::x);
  auto ld = [](const V v) { return mk<double2>((double)v.x, (double)v.y); };
  auto st = [](double2 v) { return mk<V>((VT)v.x, (VT)v.y); };

  // slot of global row e: lane e/T (by the multiplier, exact for e < 2^16), row e mod T
  auto slot = [&](int e) -> int {
    const int l = (T == 1) ? e : (int)__umulhi((unsigned)e, magicT);
    return (e - l * T) * 33 + l;
  };
  if constexpr (sizeof(V) == sizeof(double2)) {
    // all of the lane's rows in flight at once
    for (int e = lane; e < ny; e += 32) {
      const int sl = slot(e);
      cp_async16(d0 + sl, S0 + e);
      if (two) cp_async16(d1 + sl, S1 + e);
    }
    cp_async_wait_all();
  } else {
#pragma unroll 4
    for (int e = lane; e < ny; e += 32) {
      const int sl = slot(e);
      d0[sl] = ld(S0[e]);
      if (two) d1[sl] = ld(S1[e]);
    }
  }
  __syncwarp();

  const double lam = lamx[kx + g.kx0] + lamz[kz];
  const bool pin = (kx + g.kx0 == 0 && kz == 0);
  if (pin) {
    // single system: its factors c_j go where the partner's right-hand side would be
    double *cpin = (TM == 0) ? cc : reinterpret_cast<double *>(d1);
    if (lane == 0) {
      double ct_p = 0.0;
      double2 dt_p = mk<double2>(0.0, 0.0);
      for (int e = 0; e < ny; ++e) {
        const int sl = slot(e);
        double ct = 0.0;
        double2 dt = mk<double2>(0.0, 0.0);
        if (e < ny - 1) {
          const double a = am[e], c = ap[e];
          const double2 f = d0[sl];
          const double gi = 1.0 / ((lam - a - c) - a * ct_p);
          ct = c * gi;
          dt = mk<double2>((f.x - a * dt_p.x) * gi, (f.y - a * dt_p.y) * gi);
        }
        cpin[sl] = ct;
        d0[sl] = dt;
        ct_p = ct;
        dt_p = dt;
      }
      double2 xn = d0[slot(ny - 1)];
      for (int e = ny - 2; e >= 0; --e) {
        const int sl = slot(e);
        const double c = cpin[sl];
        xn = mk<double2>(d0[sl].x - c * xn.x, d0[sl].y - c * xn.y);
        d0[sl] = xn;
      }
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

  const int NL = (ny + T - 1) / T;  // active lanes
  const bool active = lane < NL;
  const int s0 = lane * T;
  const int len = active ? min(T, ny - s0) : 0;
  constexpr int TR = TM > 0 ? TM : 1;
  double at_r[TR], ct_r[TR];
  // forward elimination within the lane's block
  double at_e = 0.0, ct_e = 0.0;
  double2 e0 = mk<double2>(0.0, 0.0), e1 = mk<double2>(0.0, 0.0);
  if (active) {
    double at_p = -1.0, ct_p = 0.0;
    double2 p0 = mk<double2>(0.0, 0.0), p1 = mk<double2>(0.0, 0.0);
    auto row = [&](int t) {
      const int i = s0 + t;
      const double a = am[i], c = ap[i];
      const int sl = t * 33 + lane;
      const double gi = 1.0 / ((lam - a - c) - a * ct_p);
      const double at = -a * at_p * gi, ct = c * gi;
      const double2 f0 = d0[sl], f1 = d1[sl];
      p0 = mk<double2>((f0.x - a * p0.x) * gi, (f0.y - a * p0.y) * gi);
      p1 = mk<double2>((f1.x - a * p1.x) * gi, (f1.y - a * p1.y) * gi);
      d0[sl] = p0;
      d1[sl] = p1;
      at_p = at;
      ct_p = ct;
    };
    if constexpr (TM > 0) {
#pragma unroll
      for (int t = 0; t < TM; ++t)
        if (t < len) {
          row(t);
          at_r[t] = at_p;
          ct_r[t] = ct_p;
        }
    } else {
      for (int t = 0; t < len; ++t) {
        row(t);
        ca[t * 33 + lane] = at_p;
        cc[t * 33 + lane] = ct_p;
      }
    }
    at_e = at_p;
    ct_e = ct_p;
    e0 = p0;
    e1 = p1;
  }
  // running backward pass for x_s in terms of x_{s-1} and x_e
  double ha = 0.0, hc = -1.0;
  double2 h0 = mk<double2>(0.0, 0.0), h1 = mk<double2>(0.0, 0.0);
  auto back_run = [&](int t, double at, double ct) {
    const int sl = t * 33 + lane;
    const double2 v0 = d0[sl], v1 = d1[sl];
    if (t == len - 2) {
      h0 = v0;
      h1 = v1;
      ha = at;
      hc = ct;
    } else {
      h0 = mk<double2>(v0.x - ct * h0.x, v0.y - ct * h0.y);
      h1 = mk<double2>(v1.x - ct * h1.x, v1.y - ct * h1.y);
      ha = at - ct * ha;
      hc = -ct * hc;
    }
  };
  if constexpr (TM > 0) {
#pragma unroll
    for (int t = TM - 2; t >= 0; --t)
      if (t <= len - 2) back_run(t, at_r[t], ct_r[t]);
  } else {
    for (int t = len - 2; t >= 0; --t) back_run(t, ca[t * 33 + lane], cc[t * 33 + lane]);
  }
  // reduced equation of this lane: A y_{l-1} + B y_l + C y_{l+1} = D
  const double ha_n = shdn(ha, 1), hc_n = shdn(hc, 1);
  const double h0x = shdn(h0.x, 1), h0y = shdn(h0.y, 1), h1x = shdn(h1.x, 1), h1y = shdn(h1.y, 1);
  double A = 0.0, B = 1.0, C = 0.0;
  double D[4] = {0.0, 0.0, 0.0, 0.0};
  if (active) {
    A = at_e;
    D[0] = e0.x;
    D[1] = e0.y;
    D[2] = e1.x;
    D[3] = e1.y;
    if (lane + 1 < NL) {
      B = 1.0 - ct_e * ha_n;
      C = -ct_e * hc_n;
      D[0] -= ct_e * h0x;
      D[1] -= ct_e * h0y;
      D[2] -= ct_e * h1x;
      D[3] -= ct_e * h1y;
    }
  }
  // parallel cyclic reduction over the 32 reduced equations
#pragma unroll
  for (int h = 1; h < 32; h <<= 1) {
    double Am = shup(A, h), Bm = shup(B, h), Cm = shup(C, h);
    double Ap = shdn(A, h), Bp = shdn(B, h), Cp = shdn(C, h);
    double Dm[4], Dp[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      Dm[c] = shup(D[c], h);
      Dp[c] = shdn(D[c], h);
    }
    const bool lo = lane < h, hi = lane + h >= 32;
    if (lo) { Am = 0.0; Bm = 1.0; Cm = 0.0; }
    if (hi) { Ap = 0.0; Bp = 1.0; Cp = 0.0; }
    const double k1 = A / Bm, k2 = C / Bp;
    const double nB = B - k1 * Cm - k2 * Ap;
    A = -k1 * Am;
    C = -k2 * Cp;
    B = nB;
#pragma unroll
    for (int c = 0; c < 4; ++c) D[c] = D[c] - (lo ? 0.0 : k1 * Dm[c]) - (hi ? 0.0 : k2 * Dp[c]);
  }
  const double iB = 1.0 / B;
  double y[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) y[c] = D[c] * iB;
  double ys[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const double v = shup(y[c], 1);  // every lane takes part in the shuffle
    ys[c] = (lane == 0) ? 0.0 : v;
  }
  if (active) {
    double2 x0 = mk<double2>(y[0], y[1]), x1 = mk<double2>(y[2], y[3]);
    d0[(len - 1) * 33 + lane] = x0;
    d1[(len - 1) * 33 + lane] = x1;
    auto back_sub = [&](int t, double a, double c) {
      const int sl = t * 33 + lane;
      const double2 v0 = d0[sl], v1 = d1[sl];
      x0 = mk<double2>(v0.x - a * ys[0] - c * x0.x, v0.y - a * ys[1] - c * x0.y);
      x1 = mk<double2>(v1.x - a * ys[2] - c * x1.x, v1.y - a * ys[3] - c * x1.y);
      d0[sl] = x0;
      d1[sl] = x1;
    };
    if constexpr (TM > 0) {
#pragma unroll
      for (int t = TM - 2; t >= 0; --t)
        if (t <= len - 2) back_sub(t, at_r[t], ct_r[t]);
    } else {
      for (int t = len - 2; t >= 0; --t) back_sub(t, ca[t * 33 + lane], cc[t * 33 + lane]);
    }
  }
  __syncwarp();
  for (int e = lane; e < ny; e += 32) {
    const int sl = slot(e);
    S0[e] = st(d0[sl]);
    if (two) S1[e] = st(d1[sl]);
  }
}

// ---------------------------------------------------------------------------
// The same solve with the rows per lane T a compile-time constant (T <= 16).
// The system is padded to 32*T rows: a row i >= ny is the decoupled equation
// x_i = 0 (its off-diagonals are zero and its diagonal is one), so every lane
// eliminates exactly T rows and the loops unroll with no per-lane guard; the
// off-diagonals of the lane's rows are loaded before the elimination starts.
// The reciprocals on the elimination's dependent chain are Newton-Raphson
// iterations (y <- y + y(1 - x y), twice) from the PTX rcp.approx.ftz.f64
// seed: fewer dependent instructions than a division, within an ulp of 1/x
// (the arguments are bounded away from zero: |lam - am - ap| >= am + ap and the
// reduced diagonals stay near one).  The off-diagonals are read inside the
// unrolled elimination (L1-resident tables), so only the elimination
// coefficients of the lane's rows stay in registers.  The cyclic reduction takes one reciprocal
// per lane and level (1/B, exchanged with the neighbours) in place of two
// divisions.  The singular (0,0) system keeps the serial pinned path.
// ---------------------------------------------------------------------------
template <typename V, int T>
__global__ void __launch_bounds__(kWPB * 32, tri_min_blocks<T>()) k_tridiag_t(
    V *__restrict__ spec, GridK g, const double *__restrict__ lamx, const double *__restrict__ lamz,
    const double *__restrict__ am, const double *__restrict__ ap, const double *__restrict__ dyf, double mean_c,
    double nxnz, const double *__restrict__ pinf) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int warp = threadIdx.x >> 5;
  tridiag_t_body<V, T>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, blockIdx.x * kWPB + warp, warp, smraw, pinf);
}

// ---------------------------------------------------------------------------
// The same solve (FP64 spectrum, 9 <= T <= 12) as a persistent grid whose
// warps overlap the copies of their next pair with the solve of the current
// one.  k_tridiag_t waits for each pair's 12 KB (T = 12) before its
// latency-bound elimination starts, and its 168 registers hold it at 12 warps
// per SM; here each warp owns two buffers of a pair and, while it solves the
// pair in one, the cp.async copies of its next pair land in the other.  The
// off-diagonals of every lane's rows are copied once per CTA into shared
// memory (row t of lane l at [t*33 + l]): the elimination's reads of the
// global tables are lane-strided (a cache line per lane) and sat on its
// dependent chain.  Pairs are handed out by tickets: the first pair of warp w
// is w, the next ones come from atomicAdd on ctl[0] (one ticket ahead, so its
// latency hides behind the solve).  The warp that takes the (0,0) system and
// its serial pinned sweep takes fewer of the others.  The last warp to retire
// (ctl[1] counts them) returns both words to zero for the next launch on the
// stream.  No warp waits on another: the grid needs no co-residency.
// At T <= 8 the spectrum of the cases this library meets is small (it fits in
// L2 at 256x256x128) and k_tridiag_t, at 16 warps per SM, is faster.
// ---------------------------------------------------------------------------
template <int T>
__host__ __device__ constexpr int tri_pf_min_blocks() {
  static_assert(T >= 9 && T <= 12, "the persistent y solve is built for 9..12 rows per lane");
  return 2;
}
template <int T>
__host__ __device__ constexpr size_t tri_pf_smem_bytes() {
  return (size_t)kWPB * 4 * 33 * T * sizeof(double2) + 2 * 33 * T * sizeof(double);
}

template <int T>
__global__ void __launch_bounds__(kWPB * 32, tri_pf_min_blocks<T>()) k_tridiag_pf(
    double2 *__restrict__ spec, GridK g, const double *__restrict__ lamx, const double *__restrict__ lamz,
    const double *__restrict__ am, const double *__restrict__ ap, const double *__restrict__ dyf, double mean_c,
    double nxnz, unsigned *__restrict__ ctl, const double *__restrict__ pinf) {
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int W = 33 * T;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double2 *buf = reinterpret_cast<double2 *>(smraw) + warp * 4 * W;  // two buffers of (d0, d1)
  double *cam = reinterpret_cast<double *>(reinterpret_cast<double2 *>(smraw) + kWPB * 4 * W);
  double *cap = cam + W;
  const int ny = g.ny, nz = g.nz, nzh = nz / 2 + 1;
  // the off-diagonals of every lane's rows, once per CTA (zero on padding rows)
  for (int i = threadIdx.x; i < W; i += kWPB * 32) {
    const int t = i / 33, l = i - t * 33, r = l * T + t;
    const bool real = l < 32 && r < ny;
    cam[i] = real ? am[r] : 0.0;
    cap[i] = real ? ap[r] : 0.0;
  }
  __syncthreads();
  const unsigned ntask = (unsigned)(g.nkx * nzh);
  const unsigned nw = gridDim.x * kWPB;
  auto pair = [&](unsigned q, int &kx, int &kz, bool &two, double2 *&S0, double2 *&S1) {
    kx = (int)(q / (unsigned)nzh);
    kz = (int)(q - (unsigned)kx * nzh);
    const int kz2 = (kz == 0) ? 0 : nz - kz;
    two = kz2 != kz;
    S0 = spec + (long)kx * g.R + (long)kz * ny;
    S1 = spec + (long)kx * g.R + (long)kz2 * ny;
  };
  auto fill = [&](unsigned q, double2 *d) {
    int kx, kz;
    bool two;
    double2 *S0, *S1;
    pair(q, kx, kz, two, S0, S1);
    tri_pair_fill<double2, T>(S0, S1, two, ny, lane, d, d + W);
  };
  unsigned q = blockIdx.x * kWPB + warp;
  unsigned qn = ntask;
  if (q < ntask) {
    fill(q, buf);
    cp_async_commit();
    unsigned t = 0;
    if (lane == 0) t = atomicAdd(ctl, 1u);
    qn = __shfl_sync(0xffffffffu, t, 0) + nw;
  }
  for (int it = 0; q < ntask; ++it) {
    double2 *cur = buf + (it & 1) * 2 * W, *nxt = buf + ((it + 1) & 1) * 2 * W;
    const bool more = qn < ntask;
    if (more) fill(qn, nxt);
    cp_async_commit();  // one group per iteration (empty on the last)
    unsigned t = 0;
    if (more && lane == 0) t = atomicAdd(ctl, 1u);  // the pair after next; read after the solve
    int kx, kz;
    bool two;
    double2 *S0, *S1;
    pair(q, kx, kz, two, S0, S1);
    const double lam = lamx[kx + g.kx0] + lamz[kz];
    const bool pin = (kx + g.kx0 == 0 && kz == 0);
    cp_async_wait_group<1>();  // this pair's copies have landed; the next pair's may be in flight
    __syncwarp();
    tri_pair_solve<double2, T, true>(S0, S1, two, lam, pin, am, ap, dyf, mean_c, nxnz, ny, lane, cur, cur + W, cam,
                                     cap, pinf);
    __syncwarp();  // every lane is done with cur before it is refilled
    const unsigned b = __shfl_sync(0xffffffffu, t, 0);
    q = qn;
    qn = more ? b + nw : ntask;
  }
  cp_async_wait_all();
  if (lane == 0) {
    __threadfence();
    if (atomicAdd(ctl + 1, 1u) == nw - 1) {  // every other warp has taken its last ticket
      atomicExch(ctl, 0u);
      atomicExch(ctl + 1, 0u);
    }
  }
}

// ---------------------------------------------------------------------------
// The same solve split over a team of two warps per pair (FP64, persistent,
// prefetching, off-diagonals in shared memory): team thread l = 0..63 owns the
// U = ceil(ny/64) consecutive rows [l*U, l*U+U), so each thread's elimination
// chain is half as long as with one warp per pair.  The 64 reduced equations
// are two closed systems of 32, one per warp, once the couplings across the
// warp boundary (C of equation 31 to y_32, A of equation 32 to y_31) move to a
// fifth right-hand-side column (spike): warp 0 solves y = u + v y_32 and warp 1
// y = u' + v' y_31 by the same cyclic reduction over shuffles, and the two
// interface unknowns come from
//   y_31 = (u_31 + v_31 u'_0) / (1 - v_31 v'_0),  y_32 = u'_0 + v'_0 y_31,
// which is block Gaussian elimination of the reduced system.  The two warps
// meet at named barriers (one per team): after the copies land, for the
// neighbour terms of equation 31, for the interface values, and before a
// buffer is refilled.  The (0,0) system keeps the serial pinned sweep (warp 0).
// Tickets, retirement and the control block work as in k_tridiag_pf.
// Used for 385 <= ny <= 512 (7 or 8 rows per thread), where one warp per pair
// would hold 13..16 rows per lane and spill: at 1024 x 512 x 512 the y stage
// went from 1.483 to 1.034 ms.  At 257 <= ny <= 384 k_tridiag_pf, whose warps
// hold 8 pairs per SM in flight against 6 teams here, stays faster (0.190
// against 0.209 ms at 512 x 384 x 256).
// ---------------------------------------------------------------------------
template <int U>
__host__ __device__ constexpr size_t tri_team_smem_bytes(int teams) {
  return (size_t)teams * 4 * 65 * U * sizeof(double2) + 2 * 65 * U * sizeof(double) +
         (size_t)teams * 16 * sizeof(double) + (size_t)teams * 8;
}

__device__ __forceinline__ void team_bar(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }

template <int U, int TPC>
__global__ void __launch_bounds__(TPC * 64, 3) k_tridiag_team(
    double2 *__restrict__ spec, GridK g, const double *__restrict__ lamx, const double *__restrict__ lamz,
    const double *__restrict__ am, const double *__restrict__ ap, const double *__restrict__ dyf, double mean_c,
    double nxnz, unsigned *__restrict__ ctl, const double *__restrict__ pinf) {
  extern __shared__ __align__(16) unsigned char smraw[];
  constexpr int W = 65 * U;
  const int team = threadIdx.x >> 6, l = threadIdx.x & 63, w = l >> 5, lane = threadIdx.x & 31;
  const int bar = 1 + team;
  double2 *buf = reinterpret_cast<double2 *>(smraw) + team * 4 * W;  // two buffers of (d0, d1)
  double *cam = reinterpret_cast<double *>(reinterpret_cast<double2 *>(smraw) + TPC * 4 * W);
  double *cap = cam + W;
  double *xch = cap + W + team * 16;  // [0, 6): neighbour terms of equation 31; [6, 16): interface values
  unsigned *tks = reinterpret_cast<unsigned *>(cap + W + TPC * 16) + 2 * team;
  const int ny = g.ny, nz = g.nz, nzh = nz / 2 + 1;
  const unsigned ntask = (unsigned)(g.nkx * nzh);
  const unsigned nw = gridDim.x * TPC;
  for (int i = threadIdx.x; i < W; i += TPC * 64) {
    const int t = i / 65, o = i - t * 65, r = o * U + t;
    const bool real = o < 64 && r < ny;
    cam[i] = real ? am[r] : 0.0;
    cap[i] = real ? ap[r] : 0.0;
  }
  __syncthreads();
  auto pair = [&](unsigned q, int &kx, int &kz, bool &two, double2 *&S0, double2 *&S1) {
    kx = (int)(q / (unsigned)nzh);
    kz = (int)(q - (unsigned)kx * nzh);
    const int kz2 = (kz == 0) ? 0 : nz - kz;
    two = kz2 != kz;
    S0 = spec + (long)kx * g.R + (long)kz * ny;
    S1 = spec + (long)kx * g.R + (long)kz2 * ny;
  };
  // row e of the pair at team thread e / U, slot (e mod U)*65 + e / U
  auto fill = [&](unsigned q, double2 *d0) {
    int kx, kz;
    bool two;
    double2 *S0, *S1;
    pair(q, kx, kz, two, S0, S1);
    double2 *d1 = d0 + W;
#pragma unroll
    for (int c = 0; c < U; ++c) {
      const int e = l + 64 * c;
      const int o = e / U, sl = (e - o * U) * 65 + o;
      if (e < ny) {
        cp_async16(d0 + sl, S0 + e);
        if (two) cp_async16(d1 + sl, S1 + e);
      } else {
        d0[sl] = mk<double2>(0.0, 0.0);
        d1[sl] = mk<double2>(0.0, 0.0);
      }
    }
  };
  unsigned q = blockIdx.x * TPC + team;
  unsigned qn = ntask;
  if (q < ntask) {
    fill(q, buf);
    cp_async_commit();
    if (l == 0) tks[0] = atomicAdd(ctl, 1u);
    team_bar(bar);
    qn = tks[0] + nw;
  }
  for (int it = 0; q < ntask; ++it) {
    double2 *d0 = buf + (it & 1) * 2 * W, *d1 = d0 + W, *nxt = buf + ((it + 1) & 1) * 2 * W;
    const bool more = qn < ntask;
    if (more) fill(qn, nxt);
    cp_async_commit();
    unsigned tk = 0;
    if (more && l == 0) tk = atomicAdd(ctl, 1u);
    int kx, kz;
    bool two;
    double2 *S0, *S1;
    pair(q, kx, kz, two, S0, S1);
    const double lam = lamx[kx + g.kx0] + lamz[kz];
    const bool pin = (kx + g.kx0 == 0 && kz == 0);
    cp_async_wait_group<1>();
    team_bar(bar);  // both warps' copies of this pair are visible
    if (pin) {
      if (w == 0) {  // serial pinned Thomas (as tri_pair_solve), factors in d1
        double *cpin = reinterpret_cast<double *>(d1);
        auto slot = [&](int e) { return (e % U) * 65 + e / U; };
        if (pinf) {  // the factor table, copied by the warp into d1
          for (int i = lane; i < 2 * (ny - 1); i += 32) cpin[i] = pinf[i];
          __syncwarp();
          if (lane == 0) pinned_sweep_f(d0, cpin, ny, slot, [&](int e) { return cam[slot(e)]; });
        } else if (lane == 0) {  // the shared off-diagonals use the right-hand sides' slots
          pinned_sweep(d0, cpin, lam, ny, slot, [&](int e) { return cam[slot(e)]; },
                       [&](int e) { return cap[slot(e)]; });
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
          S0[e] = mk<double2>(d0[sl].x - subx, d0[sl].y - suby);
        }
      }
    } else {
      const int s0 = l * U;
      // forward elimination within the thread's block (padding rows: diagonal one)
      double at_r[U], ct_r[U];
      double at_p = -1.0, ct_p = 0.0;
      double2 p0 = mk<double2>(0.0, 0.0), p1 = mk<double2>(0.0, 0.0);
#pragma unroll
      for (int t = 0; t < U; ++t) {
        const bool real = s0 + t < ny;
        const double a = cam[t * 65 + l], c = cap[t * 65 + l];
        const double dg = real ? lam : 1.0;
        const int sl = t * 65 + l;
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
      if constexpr (U >= 2) {
        h0 = d0[(U - 2) * 65 + l];
        h1 = d1[(U - 2) * 65 + l];
        ha = at_r[U - 2];
        hc = ct_r[U - 2];
#pragma unroll
        for (int t = U - 3; t >= 0; --t) {
          const double2 v0 = d0[t * 65 + l], v1 = d1[t * 65 + l];
          const double ct = ct_r[t];
          h0 = mk<double2>(v0.x - ct * h0.x, v0.y - ct * h0.y);
          h1 = mk<double2>(v1.x - ct * h1.x, v1.y - ct * h1.y);
          ha = at_r[t] - ct * ha;
          hc = -ct * hc;
        }
      }
      // the next thread's terms: by shuffle inside a warp, through xch across
      if (w == 1 && lane == 0) {
        xch[0] = ha;
        xch[1] = hc;
        xch[2] = h0.x;
        xch[3] = h0.y;
        xch[4] = h1.x;
        xch[5] = h1.y;
      }
      double ha_n = shdn(ha, 1), hc_n = shdn(hc, 1);
      double h0x = shdn(h0.x, 1), h0y = shdn(h0.y, 1), h1x = shdn(h1.x, 1), h1y = shdn(h1.y, 1);
      team_bar(bar);
      if (w == 0 && lane == 31) {
        ha_n = xch[0];
        hc_n = xch[1];
        h0x = xch[2];
        h0y = xch[3];
        h1x = xch[4];
        h1y = xch[5];
      }
      const double at_e = at_r[U - 1], ct_e = ct_r[U - 1];
      double A = at_e, B = 1.0, C = 0.0;
      double D[5] = {p0.x, p0.y, p1.x, p1.y, 0.0};
      if (l < 63) {
        B = 1.0 - ct_e * ha_n;
        C = -ct_e * hc_n;
        D[0] -= ct_e * h0x;
        D[1] -= ct_e * h0y;
        D[2] -= ct_e * h1x;
        D[3] -= ct_e * h1y;
      }
      // the coupling across the warp boundary becomes the spike column
      if (w == 0 && lane == 31) {
        D[4] = -C;
        C = 0.0;
      }
      if (w == 1 && lane == 0) {
        D[4] = -A;
        A = 0.0;
      }
#pragma unroll
      for (int h = 1; h < 32; h <<= 1) {
        const double iB = rcp_nr(B);
        double Am = shup(A, h), iBm = shup(iB, h), Cm = shup(C, h);
        double Ap = shdn(A, h), iBp = shdn(iB, h), Cp = shdn(C, h);
        double Dm[5], Dp[5];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
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
        for (int c = 0; c < 5; ++c) D[c] = D[c] - k1 * Dm[c] - k2 * Dp[c];
      }
      const double iBf = rcp_nr(B);
      double y[5];
#pragma unroll
      for (int c = 0; c < 5; ++c) y[c] = D[c] * iBf;
      // interface unknowns y_31 and y_32
      if (w == 0 && lane == 31) {
#pragma unroll
        for (int c = 0; c < 5; ++c) xch[6 + c] = y[c];
      }
      if (w == 1 && lane == 0) {
#pragma unroll
        for (int c = 0; c < 5; ++c) xch[11 + c] = y[c];
      }
      team_bar(bar);
      const double v31 = xch[10], v32 = xch[15];
      const double den = 1.0 - v31 * v32;
      double y31[4], y32[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        y31[c] = (xch[6 + c] + v31 * xch[11 + c]) / den;
        y32[c] = xch[11 + c] + v32 * y31[c];
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) y[c] = y[c] + y[4] * (w == 0 ? y32[c] : y31[c]);
      double ys[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const double v = shup(y[c], 1);  // every lane takes part in the shuffle
        ys[c] = (lane == 0) ? (w == 0 ? 0.0 : y31[c]) : v;
      }
      double2 x0 = mk<double2>(y[0], y[1]), x1 = mk<double2>(y[2], y[3]);
      d0[(U - 1) * 65 + l] = x0;
      d1[(U - 1) * 65 + l] = x1;
#pragma unroll
      for (int t = U - 2; t >= 0; --t) {
        const int sl = t * 65 + l;
        const double a = at_r[t], c = ct_r[t];
        const double2 v0 = d0[sl], v1 = d1[sl];
        x0 = mk<double2>(v0.x - a * ys[0] - c * x0.x, v0.y - a * ys[1] - c * x0.y);
        x1 = mk<double2>(v1.x - a * ys[2] - c * x1.x, v1.y - a * ys[3] - c * x1.y);
        d0[sl] = x0;
        d1[sl] = x1;
      }
      team_bar(bar);  // every row of the pair is solved
#pragma unroll
      for (int c = 0; c < U; ++c) {
        const int e = l + 64 * c;
        if (e < ny) {
          const int o = e / U, sl = (e - o * U) * 65 + o;
          S0[e] = d0[sl];
          if (two) S1[e] = d1[sl];
        }
      }
    }
    if (l == 0) tks[0] = tk;
    team_bar(bar);  // the buffer is free for the refill; the ticket is visible
    const unsigned b = tks[0];
    q = qn;
    qn = more ? b + nw : ntask;
  }
  cp_async_wait_all();
  if (l == 0) {
    __threadfence();
    if (atomicAdd(ctl + 1, 1u) == nw - 1) {  // every other team has taken its last ticket
      atomicExch(ctl, 0u);
      atomicExch(ctl + 1, 0u);
    }
  }
}

// shared memory of a k_tridiag<V, TM> block: the two right-hand sides per warp,
// plus the coefficient arrays when TM == 0
static size_t tridiag_block_smem(int T, int TM) {
  return (size_t)kWPB * 33 * T * (2 * sizeof(double2) + (TM == 0 ? 2 * sizeof(double) : 0));
}

template <typename V>
static void launch_tridiag_t(V *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                             const double *ap, const double *dyf, double mean_c, double nxnz, cudaStream_t st,
                             const double *pinf = nullptr) {
  const long nwarps = (long)g.nkx * (g.nz / 2 + 1);
  const unsigned nblk = (unsigned)((nwarps + kWPB - 1) / kWPB);
  const int T = tri_rows_per_lane(g.ny);
  // e/T == umulhi(e, floor(2^32/T) + 1) for every e < 2^16 (and T <= 2^16)
  const unsigned magic = T > 1 ? (unsigned)((1ull << 32) / (unsigned long long)T + 1ull) : 0u;
  const dim3 blk(kWPB * 32);
  const size_t sm2 = (size_t)kWPB * 2 * 33 * T * sizeof(double2);
  switch (T) {
#define TBFP_TRI_T(TT) \
  case TT: k_tridiag_t<V, TT><<<nblk, blk, sm2, st>>>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, pinf); return;
    TBFP_TRI_T(1) TBFP_TRI_T(2) TBFP_TRI_T(3) TBFP_TRI_T(4) TBFP_TRI_T(5) TBFP_TRI_T(6) TBFP_TRI_T(7)
    TBFP_TRI_T(8) TBFP_TRI_T(9) TBFP_TRI_T(10) TBFP_TRI_T(11) TBFP_TRI_T(12) TBFP_TRI_T(13) TBFP_TRI_T(14)
    TBFP_TRI_T(15) TBFP_TRI_T(16)
#undef TBFP_TRI_T
    default: break;
  }
  if (T <= 4) k_tridiag<V, 4><<<nblk, blk, tridiag_block_smem(T, 4), st>>>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, T, magic);
  else if (T <= 8) k_tridiag<V, 8><<<nblk, blk, tridiag_block_smem(T, 8), st>>>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, T, magic);
  else if (T <= 12) k_tridiag<V, 12><<<nblk, blk, tridiag_block_smem(T, 12), st>>>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, T, magic);
  else if (T <= 16) k_tridiag<V, 16><<<nblk, blk, tridiag_block_smem(T, 16), st>>>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, T, magic);
  else k_tridiag<V, 0><<<nblk, blk, tridiag_block_smem(T, 0), st>>>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, T, magic);
}
void launch_tridiag(double2 *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                    const double *ap, const double *dyf, double mean_c, double nxnz, cudaStream_t st) {
  launch_tridiag_t(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, st);
}

template <int T>
static void launch_tridiag_pf_n(double2 *spec, const GridK &g, const double *lamx, const double *lamz,
                                const double *am, const double *ap, const double *dyf, double mean_c, double nxnz,
                                unsigned *ctl, int sms, const double *pinf, cudaStream_t st) {
  const long npair = (long)g.nkx * (g.nz / 2 + 1);
  long nblk = (npair + kWPB - 1) / kWPB;
  const long resident = (long)sms * tri_pf_min_blocks<T>();
  if (nblk > resident) nblk = resident;
  k_tridiag_pf<T><<<(unsigned)nblk, kWPB * 32, tri_pf_smem_bytes<T>(), st>>>(spec, g, lamx, lamz, am, ap, dyf,
                                                                           mean_c, nxnz, ctl, pinf);
}

template <int U, int TPC>
static void launch_tridiag_team_n(double2 *spec, const GridK &g, const double *lamx, const double *lamz,
                                  const double *am, const double *ap, const double *dyf, double mean_c, double nxnz,
                                  unsigned *ctl, int sms, const double *pinf, cudaStream_t st) {
  const long npair = (long)g.nkx * (g.nz / 2 + 1);
  long nblk = (npair + TPC - 1) / TPC;
  const size_t smem = tri_team_smem_bytes<U>(TPC);
  long per_sm = (long)(233472 / (smem + 1024));  // shared memory per SM, 1 KB reserved per CTA
  if (per_sm > 3) per_sm = 3;
  if (per_sm < 1) per_sm = 1;
  if (nblk > per_sm * sms) nblk = per_sm * sms;
  k_tridiag_team<U, TPC><<<(unsigned)nblk, TPC * 64, smem, st>>>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, ctl,
                                                                  pinf);
}

void launch_tridiag(double2 *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                    const double *ap, const double *dyf, double mean_c, double nxnz, unsigned *ctl, int sms,
                    const double *pinf, cudaStream_t st) {
  const int T = tri_rows_per_lane(g.ny);
  if (ctl && sms > 0) {
    switch ((g.ny + 63) / 64) {  // 385 <= ny <= 512: two-warp teams
      case 7: launch_tridiag_team_n<7, 2>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, ctl, sms, pinf, st); return;
      case 8: launch_tridiag_team_n<8, 2>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, ctl, sms, pinf, st); return;
      default: break;
    }
    switch (T) {
#define TBFP_TRI_PF(TT) \
  case TT: launch_tridiag_pf_n<TT>(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, ctl, sms, pinf, st); return;
      TBFP_TRI_PF(9) TBFP_TRI_PF(10) TBFP_TRI_PF(11) TBFP_TRI_PF(12)
#undef TBFP_TRI_PF
      default: break;
    }
  }
  launch_tridiag_t(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, st, pinf);
}
void launch_tridiag(float2 *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                    const double *ap, const double *dyf, double mean_c, double nxnz, cudaStream_t st) {
  launch_tridiag_t(spec, g, lamx, lamz, am, ap, dyf, mean_c, nxnz, st);
}

// ---------------------------------------------------------------------------
// The kx-slab spectrum S_x[kx][k][j] of a split channel and the chunks that
// the all-to-alls move: the chunk of rank p (source in the first exchange,
// destination in the second) is [kx][k - zs[p]][j] for its planes k.  One
// thread per complex entry, j fastest in both layouts (coalesced).
// ---------------------------------------------------------------------------
__global__ void k_slab_chunks(GridK g, SlabParts parts, int to_x, const double2 *__restrict__ src,
                              double2 *__restrict__ dst) {
  const int ny = g.ny, nz = g.nz;
  const long n = (long)g.nkx * nz * ny;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int j = (int)(t % ny);
    const long r = t / ny;
    const int k = (int)(r % nz), kx = (int)(r / nz);
    int p = 0;
    while (k >= parts.zs[p + 1]) ++p;  // the rank that owns plane k (parts.n is small)
    const int z0 = parts.zs[p], nzp = parts.zs[p + 1] - z0;
    const long c = (long)g.nkx * ny * z0 + ((long)kx * nzp + (k - z0)) * ny + j;
    if (to_x) dst[t] = src[c];
    else dst[c] = src[t];
  }
}

void launch_slab_chunks(const GridK &g, const SlabParts &parts, bool to_x, const double2 *src, double2 *dst,
                        cudaStream_t st) {
  const long n = (long)g.nkx * g.nz * g.ny;
  long nb = (n + 255) / 256;
  if (nb > 148L * 32) nb = 148L * 32;
  k_slab_chunks<<<(unsigned)(nb < 1 ? 1 : nb), 256, 0, st>>>(g, parts, to_x ? 1 : 0, src, dst);
}

// Elimination factors of the pinned (0,0) y system, once per handle (its
// matrix does not change between calls): f[2e] = 1/pivot_e, f[2e+1] = ct_e for
// e < ny-1, with the arithmetic of pinned_sweep.  One thread: ny steps.
__global__ void k_pin_factors(const double *__restrict__ am, const double *__restrict__ ap,
                              const double *__restrict__ lamx, const double *__restrict__ lamz, int ny,
                              double *__restrict__ f) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double lam = lamx[0] + lamz[0];
  double ct_p = 0.0;
  for (int e = 0; e < ny - 1; ++e) {
    const double a = am[e], c = ap[e];
    const double gi = rcp_nr((lam - a - c) - a * ct_p);
    ct_p = c * gi;
    f[2 * e] = gi;
    f[2 * e + 1] = ct_p;
  }
}

void launch_pin_factors(const double *am, const double *ap, const double *lamx, const double *lamz, int ny, double *f,
                        cudaStream_t st) {
  k_pin_factors<<<1, 32, 0, st>>>(am, ap, lamx, lamz, ny, f);
}

cudaError_t prepare_yz_kernels() {
  cudaError_t e = cudaSuccess;
  auto set = [&](const void *fn, size_t bytes) {
    const cudaError_t ee = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (ee != cudaSuccess) e = ee;
  };
#define TBFP_CASE(L)                                                             \
  set((const void *)k_fftz<double2, false, L>, fftz_smem_bytes(L, 16));          \
  set((const void *)k_fftz<double2, true, L>, fftz_smem_bytes(L, 16));           \
  set((const void *)k_fftz<float2, false, L>, fftz_smem_bytes(L, 8));            \
  set((const void *)k_fftz<float2, true, L>, fftz_smem_bytes(L, 8));
  TBFP_FFT_LENGTHS(TBFP_CASE)
#undef TBFP_CASE
#define TBFP_TRI(TM)                                          \
  set((const void *)k_tridiag<double2, TM>, 227 * 1024);      \
  set((const void *)k_tridiag<float2, TM>, 227 * 1024);
  TBFP_TRI(0) TBFP_TRI(4) TBFP_TRI(8) TBFP_TRI(12) TBFP_TRI(16)
#undef TBFP_TRI
#define TBFP_TRI_T(TT)                                        \
  set((const void *)k_tridiag_t<double2, TT>, 227 * 1024);    \
  set((const void *)k_tridiag_t<float2, TT>, 227 * 1024);
  TBFP_TRI_T(1) TBFP_TRI_T(2) TBFP_TRI_T(3) TBFP_TRI_T(4) TBFP_TRI_T(5) TBFP_TRI_T(6) TBFP_TRI_T(7)
  TBFP_TRI_T(8) TBFP_TRI_T(9) TBFP_TRI_T(10) TBFP_TRI_T(11) TBFP_TRI_T(12) TBFP_TRI_T(13) TBFP_TRI_T(14)
  TBFP_TRI_T(15) TBFP_TRI_T(16)
#undef TBFP_TRI_T
  set((const void *)k_tridiag_team<7, 2>, tri_team_smem_bytes<7>(2));
  set((const void *)k_tridiag_team<8, 2>, tri_team_smem_bytes<8>(2));
#define TBFP_TRI_PF(TT) set((const void *)k_tridiag_pf<TT>, tri_pf_smem_bytes<TT>());
  TBFP_TRI_PF(9) TBFP_TRI_PF(10) TBFP_TRI_PF(11) TBFP_TRI_PF(12)
#undef TBFP_TRI_PF
  return e;
}

}  // namespace tbfp
