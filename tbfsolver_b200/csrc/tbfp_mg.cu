// MG_MODE pressure solve: FP64 preconditioned conjugate gradients (solvePCG,
// pcg.f90:103-140) on L_beta psi = q, preconditioned by FP32 red-black
// Gauss-Seidel multigrid V-cycles (solveMG/mgVcycle, multiGrid.f90:165-232;
// iterateGS/computeResiduals, rbgs.f90:186-333; restrictionOp3D /
// prolongationOp3D, interpolation.f90:80-181) with a direct solve of the
// Lagrange-bordered system on the coarsest level (poissMat.f90:289-312).
//
// Operator (computeQv, pcg.f90:163-176): face coefficients
//   aR = (beta(i+1)+beta(i))/2 / (dxc(i+1) dxf(i)),  aL = (beta(i)+beta(i-1))/2 / (dxc(i) dxf(i)),
// likewise in y and z; L p = aR (p(i+1)-p) - aL (p-p(i-1)) + ... .  x and z are
// periodic, y has Neumann walls: the ghost values the reference's boundary
// update writes (periodic images, wall copies) are read here through wrapped
// (x, z) and clamped (y) indices, which is the same arithmetic.
//
// Level arrays (FP32 p, q, beta, residual) are dense nz x ny x nx, no halo.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "tbfp_mg.cuh"

namespace tbfp {

namespace {

constexpr int kMgThreads = 256;

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }
__device__ __forceinline__ int clampi(int j, int n) { return j < 0 ? 0 : (j >= n ? n - 1 : j); }

// Launch shape of the stencil kernels: grid (x tiles of kWalkX, y chunks of J
// rows, z planes) with J = ceil(ny / gridDim.y); a thread owns column (i, k) of
// a y chunk and walks it, so there is no integer division per cell.  Kernels
// without a reduction are launched with J = 1 (one cell per thread, most
// parallelism); reductions with J = kMgJ (one block sum per kMgJ rows).  Dense
// level arrays: t = (k*ny + j)*nx + i (32-bit: every level holds fewer than
// 2^31 cells, checked at set-up).
constexpr int kMgJ = 16;
constexpr int kWalkX = 128;  // threads per block of the column-walk kernels
struct Walk {
  int i, j0, j1, k;
};
__device__ __forceinline__ Walk walk(int ny) {
  Walk w;
  const int J = (ny + (int)gridDim.y - 1) / (int)gridDim.y;
  w.i = blockIdx.x * blockDim.x + threadIdx.x;
  w.k = blockIdx.z;
  w.j0 = blockIdx.y * J;
  w.j1 = min(w.j0 + J, ny);
  return w;
}

// Face coefficients of cell (i, j, k) (0-based) from a dense beta.
template <typename T>
struct Coef {
  T aR, aL, aT, aB, aF, aK;
};
template <typename T, typename B>
__device__ __forceinline__ Coef<T> coef(const MgLev &L, const B *beta, int i, int j, int k) {
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  auto at3 = [&](int ii, int jj, int kk) { return ((long)kk * ny + jj) * nx + ii; };
  const T bc = (T)beta[at3(i, j, k)];
  const T h = T(0.5);
  Coef<T> c;
  c.aR = h * ((T)beta[at3(wrap(i + 1, nx), j, k)] + bc) * (T)L.invx1[i];
  c.aL = h * (bc + (T)beta[at3(wrap(i - 1, nx), j, k)]) * (T)L.invx2[i];
  c.aT = h * ((T)beta[at3(i, clampi(j + 1, ny), k)] + bc) * (T)L.invy1[j];
  c.aB = h * (bc + (T)beta[at3(i, clampi(j - 1, ny), k)]) * (T)L.invy2[j];
  c.aF = h * ((T)beta[at3(i, j, wrap(k + 1, nz))] + bc) * (T)L.invz1[k];
  c.aK = h * (bc + (T)beta[at3(i, j, wrap(k - 1, nz))]) * (T)L.invz2[k];
  return c;
}

__device__ __forceinline__ void block_sum2(double a, double b, double *out_a, double *out_b) {
  __shared__ double red[2][32];
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    red[0][w] = a;
    red[1][w] = b;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (int)(blockDim.x >> 5);
    a = l < nw ? red[0][l] : 0.0;
    b = l < nw ? red[1][l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_xor_sync(0xffffffffu, a, o);
      b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if (l == 0) {
      if (out_a) atomicAdd(out_a, a);
      if (out_b) atomicAdd(out_b, b);
    }
  }
}

// ---------------------------------------------------------------------------
// One colour of iterateGS (rbgs.f90:215-250): cells with (i+j+k) mod 2 == colour
// (1-based indices, red = 0) take p = (-q + sum a_nb p_nb) / sum a_nb.
// ---------------------------------------------------------------------------
// sum: when not NULL, the sum of the updated cells is added to *sum (the last
// red and black sweeps of a smoothing call give sum(p) for correctFullNeumann
// without another pass).  A wall cell's clamped y neighbour is the cell
// itself, so a sweep also reads cells of its own colour there.
__global__ void __launch_bounds__(kWalkX) k_rbgs_colour(MgLev L, float *__restrict__ p,
                                                       const float *__restrict__ q,
                                                       const float *__restrict__ beta, int colour,
                                                       double *__restrict__ sum) {
  const Walk w = walk(L.ny);
  const int nx = L.nx, ny = L.ny, nz = L.nz, k = w.k;
  double acc = 0.0;
  if (w.i < (nx + 1) / 2) {
    for (int j = w.j0; j < w.j1; ++j) {
      // colour of 1-based (i+1, j+1, k+1) is (i + j + k + 3) mod 2, so the row's
      // first 0-based index of this colour is (colour + j + k + 1) mod 2
      const int ii = 2 * w.i + ((colour + j + k + 1) & 1);
      if (ii >= nx) continue;
      auto at3 = [&](int a, int b, int c) { return (c * ny + b) * nx + a; };
      const Coef<float> c = coef<float>(L, beta, ii, j, k);
      const float den = c.aR + c.aL + c.aT + c.aB + c.aF + c.aK;
      const float pR = p[at3(wrap(ii + 1, nx), j, k)], pL = p[at3(wrap(ii - 1, nx), j, k)];
      const float pT = p[at3(ii, clampi(j + 1, ny), k)], pB = p[at3(ii, clampi(j - 1, ny), k)];
      const float pF = p[at3(ii, j, wrap(k + 1, nz))], pK = p[at3(ii, j, wrap(k - 1, nz))];
      const float v =
          (-q[at3(ii, j, k)] + (c.aR * pR + c.aL * pL) + (c.aT * pT + c.aB * pB) + (c.aF * pF + c.aK * pK)) / den;
      p[at3(ii, j, k)] = v;
      acc += v;
    }
  }
  if (sum) block_sum2(acc, 0.0, sum, nullptr);  // sum is uniform over the grid
}

// p -= sum/n (correctFullNeumann, rbgs.f90:403-446)
__global__ void __launch_bounds__(kMgThreads) k_sub_mean(float *__restrict__ p, long n,
                                                        const double *__restrict__ sum) {
  const float avg = (float)(*sum / (double)n);
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) p[t] -= avg;
}

// res = q - L p (computeResiduals, rbgs.f90:308-317); optional sum res^2, sum q^2
__global__ void __launch_bounds__(kMgThreads) k_mg_residual(MgLev L, const float *__restrict__ p,
                                                           const float *__restrict__ q,
                                                           const float *__restrict__ beta, float *__restrict__ res,
                                                           double *__restrict__ nrm) {
  const Walk w = walk(L.ny);
  const int nx = L.nx, ny = L.ny, nz = L.nz, i = w.i, k = w.k;
  double rr = 0.0, qq = 0.0;
  if (i < nx) {
    auto at3 = [&](int a, int b, int c) { return (c * ny + b) * nx + a; };
#pragma unroll 4
    for (int j = w.j0; j < w.j1; ++j) {
      const int t = at3(i, j, k);
      const Coef<float> c = coef<float>(L, beta, i, j, k);
      const float pc = p[t];
      const float Lp = c.aR * (p[at3(wrap(i + 1, nx), j, k)] - pc) - c.aL * (pc - p[at3(wrap(i - 1, nx), j, k)]) +
                       c.aT * (p[at3(i, clampi(j + 1, ny), k)] - pc) - c.aB * (pc - p[at3(i, clampi(j - 1, ny), k)]) +
                       c.aF * (p[at3(i, j, wrap(k + 1, nz))] - pc) - c.aK * (pc - p[at3(i, j, wrap(k - 1, nz))]);
      const float v = q[t] - Lp;
      res[t] = v;
      rr += (double)v * v;
      qq += (double)q[t] * q[t];
    }
  }
  if (nrm) block_sum2(rr, qq, nrm, nrm + 1);
}

// restrictionOp3D (interpolation.f90:80-124): coarse = sum of the 8 children with
// separable trilinear weights w[I][a] (a = 0: child 2I-1, a = 1: child 2I, 1-based).
__global__ void __launch_bounds__(kMgThreads) k_restrict(MgLev F, MgLev C, const float *__restrict__ fine,
                                                        float *__restrict__ coarse) {
  const Walk w = walk(C.ny);
  const int I = w.i, K = w.k;
  if (I >= C.nx) return;  // no block-level barrier in this kernel
  const float x0 = C.rx[2 * I], x1 = C.rx[2 * I + 1];
  const float z0 = C.rz[2 * K], z1 = C.rz[2 * K + 1];
  for (int J = w.j0; J < w.j1; ++J) {
    auto f = [&](int a, int b, int c) { return fine[((2 * K + c) * F.ny + (2 * J + b)) * F.nx + (2 * I + a)]; };
    const float y0 = C.ry[2 * J], y1 = C.ry[2 * J + 1];
    float s = (x0 * y0) * z0 * f(0, 0, 0);
    s += (x1 * y0) * z0 * f(1, 0, 0);
    s += (x0 * y1) * z0 * f(0, 1, 0);
    s += (x1 * y1) * z0 * f(1, 1, 0);
    s += (x0 * y0) * z1 * f(0, 0, 1);
    s += (x1 * y0) * z1 * f(1, 0, 1);
    s += (x0 * y1) * z1 * f(0, 1, 1);
    s += (x1 * y1) * z1 * f(1, 1, 1);
    coarse[(K * C.ny + J) * C.nx + I] = s;
  }
}

// prolongationOp3D (interpolation.f90:129-181): fine += trilinear interpolation
// between coarse centroids ih = i/2 and ih+1 (1-based, the coarse ghosts read
// through wrapped / clamped indices).
// The means left by the smoothing calls (correctFullNeumann) are removed here:
// fsum/finv the fine level's pre-smoothing sum and 1/cells, csum/cinv the
// coarse level's post-smoothing sum (NULL: nothing pending); the weights sum
// to 1, so interpolating p - mean subtracts the mean.
__global__ void __launch_bounds__(kMgThreads) k_prolong_add(MgLev F, MgLev C, const float *__restrict__ coarse,
                                                           float *__restrict__ fine, const double *__restrict__ fsum,
                                                           double finv, const double *__restrict__ csum,
                                                           double cinv) {
  const Walk w = walk(F.ny);
  const int i = w.i, k = w.k;
  if (i >= F.nx) return;  // no block-level barrier in this kernel
  const float mf = fsum ? (float)(*fsum * finv) : 0.0f, mc = csum ? (float)(*csum * cinv) : 0.0f;
  // 1-based fine index i+1 -> ih = (i+1)/2, coarse 0-based ih-1 and ih
  const int ih = (i + 1) / 2 - 1, kh = (k + 1) / 2 - 1;
  const int xa = wrap(ih, C.nx), xb = wrap(ih + 1, C.nx);
  const int za = wrap(kh, C.nz), zb = wrap(kh + 1, C.nz);
  const float x0 = F.px[2 * i], x1 = F.px[2 * i + 1];
  const float z0 = F.pz[2 * k], z1 = F.pz[2 * k + 1];
  auto c = [&](int a, int b, int cc) { return coarse[(cc * C.ny + b) * C.nx + a]; };
  for (int j = w.j0; j < w.j1; ++j) {
    const int jh = (j + 1) / 2 - 1;
    const int ya = clampi(jh, C.ny), yb = clampi(jh + 1, C.ny);
    const float y0 = F.py[2 * j], y1 = F.py[2 * j + 1];
    float s = (x0 * y0) * z0 * c(xa, ya, za);
    s += (x1 * y0) * z0 * c(xb, ya, za);
    s += (x0 * y1) * z0 * c(xa, yb, za);
    s += (x1 * y1) * z0 * c(xb, yb, za);
    s += (x0 * y0) * z1 * c(xa, ya, zb);
    s += (x1 * y0) * z1 * c(xb, ya, zb);
    s += (x0 * y1) * z1 * c(xa, yb, zb);
    s += (x1 * y1) * z1 * c(xb, yb, zb);
    const int t = (k * F.ny + j) * F.nx + i;
    fine[t] = (fine[t] - mf) + (s - mc);
  }
}

__global__ void k_fill(float *__restrict__ p, long n, float v) {
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) p[t] = v;
}

// ---------------------------------------------------------------------------
// Coarsest level (solveMat, poissMat.f90:289-312): the system V*(-L) p = -V*s
// with Neumann walls, bordered by the Lagrange row sum(p) = 0, in FP64.  The
// bordered matrix depends only on beta, so it is inverted once per PCG solve
// and every V-cycle applies the inverse (the reference refactorises with MUMPS
// on every call; the result is the same linear solve).
//
// Inversion: blocked Gauss-Jordan on [K | I] without pivoting, in the order
// cells 0..n-2, border, cell n-1 (unknowns n-1 and n swapped).  K's cell block
// A = V*(-L) is an irreducible singular M-matrix, so its proper leading
// submatrices are nonsingular M-matrices, the bordered leading block
// [A_11 1; 1^T 0] is nonsingular (1^T A_11^-1 1 > 0) and so is K: every
// leading minor of the reordered matrix is nonzero and elimination needs no
// row exchanges.  Panels of kGB columns: one CTA inverts the panel's diagonal
// block and scales the panel rows by it; the other rows take the rank-kGB
// update from many CTAs.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int coarse_perm(int x, int n) { return x == n - 1 ? n : (x == n ? n - 1 : x); }

__global__ void k_coarse_assemble(MgLev L, const float *__restrict__ beta, double *__restrict__ M, int n1) {
  const int n = n1 - 1;
  const int ld = 2 * n1;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < (long)n1 * ld; e += (long)gridDim.x * blockDim.x)
    M[e] = 0.0;
  __syncthreads();  // one CTA
  for (int r0 = threadIdx.x; r0 < n; r0 += blockDim.x) {
    const int r = coarse_perm(r0, n);
    const int i = r0 % L.nx, j = (r0 / L.nx) % L.ny, k = r0 / (L.nx * L.ny);
    const Coef<double> c = coef<double>(L, beta, i, j, k);
    const double V = (double)L.vx[i] * (double)L.vy[j] * (double)L.vz[k];
    auto idx = [&](int a, int b, int cc) { return coarse_perm((cc * L.ny + b) * L.nx + a, n); };
    double diag = 0.0;
    auto term = [&](double a, int col) {
      M[(long)r * ld + col] -= V * a;
      diag += V * a;
    };
    term(c.aR, idx(wrap(i + 1, L.nx), j, k));
    term(c.aL, idx(wrap(i - 1, L.nx), j, k));
    term(c.aF, idx(i, j, wrap(k + 1, L.nz)));
    term(c.aK, idx(i, j, wrap(k - 1, L.nz)));
    if (j < L.ny - 1) term(c.aT, idx(i, j + 1, k));
    if (j > 0) term(c.aB, idx(i, j - 1, k));
    M[(long)r * ld + r] += diag;
    const int bdr = coarse_perm(n, n);
    M[(long)r * ld + bdr] = 1.0;
    M[(long)bdr * ld + r] = 1.0;
  }
  __syncthreads();
  for (int r = threadIdx.x; r < n1; r += blockDim.x) M[(long)r * ld + n1 + r] = 1.0;  // [K | I]
}

constexpr int kGB = 32;     // panel width
constexpr int kGPT = 256;   // threads of the panel kernel
// Rows p0 .. p0+pb-1 of [K | I]: D = K[p0.., p0..] is inverted in shared memory
// (Gauss-Jordan, no exchanges), the panel rows become D^-1 times themselves
// (columns p0.. on; the columns before p0 are already unit vectors), and the
// panel's column block of every row is saved in Cb (the update's multipliers).
__global__ void __launch_bounds__(kGPT) k_gj_panel(double *__restrict__ M, int n1, int p0, double *__restrict__ Cb,
                                                  int *__restrict__ fail) {
  const int ld = 2 * n1, pb = min(kGB, n1 - p0), tid = threadIdx.x;
  __shared__ double A[kGB][2 * kGB + 1];
  for (int e = tid; e < kGB * 2 * kGB; e += kGPT) {
    const int r = e / (2 * kGB), c = e % (2 * kGB);
    double v = 0.0;
    if (r < pb && c < pb) v = M[(long)(p0 + r) * ld + p0 + c];
    else if (c >= kGB) v = (c - kGB == r) ? 1.0 : 0.0;
    else if (r >= pb && c == r) v = 1.0;  // unused rows of a short last panel
    A[r][c] = v;
  }
  for (long e = tid; e < (long)n1 * pb; e += kGPT) {
    const int r = (int)(e / pb), t = (int)(e % pb);
    Cb[(long)r * kGB + t] = M[(long)r * ld + p0 + t];
  }
  __shared__ double fcol[kGB];
  __syncthreads();
  for (int k = 0; k < kGB; ++k) {
    const double piv = A[k][k];
    __syncthreads();  // every thread has read the pivot before row k is scaled
    if (tid == 0 && !(fabs(piv) > 0.0 && fabs(piv) < 1e300)) *fail = 1;
    const double ip = 1.0 / piv;
    for (int c = tid; c < 2 * kGB; c += kGPT) A[k][c] *= ip;
    for (int r = tid; r < kGB; r += kGPT) fcol[r] = A[r][k];  // row k's own entry is not used
    __syncthreads();
    for (int e = tid; e < kGB * 2 * kGB; e += kGPT) {
      const int r = e / (2 * kGB), c = e % (2 * kGB);
      if (r != k) A[r][c] -= fcol[r] * A[k][c];
    }
    __syncthreads();
  }
  // panel rows, column by column (each thread owns columns): R = D^-1 * rows
  for (int c = p0 + tid; c < ld; c += kGPT) {
    double x[kGB];
#pragma unroll
    for (int s = 0; s < kGB; ++s) x[s] = s < pb ? M[(long)(p0 + s) * ld + c] : 0.0;
    for (int t = 0; t < pb; ++t) {
      double y = 0.0;
#pragma unroll
      for (int s = 0; s < kGB; ++s) y += A[t][kGB + s] * x[s];
      M[(long)(p0 + t) * ld + c] = y;
    }
  }
}

// Rows outside the panel: M[r][c] -= sum_t Cb[r][t] * M[p0+t][c], c >= p0.
// CTA tile: 32 rows x 128 columns; thread = one column, 16 rows.
__global__ void __launch_bounds__(256) k_gj_update(double *__restrict__ M, int n1, int p0,
                                                   const double *__restrict__ Cb) {
  const int ld = 2 * n1, pb = min(kGB, n1 - p0);
  const int r0 = blockIdx.y * 32, c0 = p0 + blockIdx.x * 128;
  __shared__ double Ct[32][kGB + 1];
  __shared__ double Rt[kGB][128];
  const int tid = threadIdx.x;
  for (int e = tid; e < 32 * kGB; e += 256) {
    const int r = e / kGB, t = e % kGB;
    Ct[r][t] = (r0 + r < n1 && t < pb) ? Cb[(long)(r0 + r) * kGB + t] : 0.0;
  }
  for (int e = tid; e < kGB * 128; e += 256) {
    const int t = e / 128, c = e % 128;
    Rt[t][c] = (t < pb && c0 + c < ld) ? M[(long)(p0 + t) * ld + c0 + c] : 0.0;
  }
  __syncthreads();
  const int c = tid & 127, rh = (tid >> 7) * 16;
  if (c0 + c >= ld) return;  // no barrier follows
#pragma unroll 1
  for (int rr = 0; rr < 16; ++rr) {
    const int r = r0 + rh + rr;
    if (r >= n1 || (r >= p0 && r < p0 + pb)) continue;
    double acc = 0.0;
#pragma unroll
    for (int t = 0; t < kGB; ++t) acc += Ct[rh + rr][t] * Rt[t][c];
    M[(long)r * ld + c0 + c] -= acc;
  }
}

// p = K^-1 (-V s) on the coarsest level (the Lagrange row's right-hand side is
// 0); the inverse is stored in the reordered basis.
__global__ void k_coarse_apply(MgLev L, const double *__restrict__ M, int n1, const float *__restrict__ s,
                               float *__restrict__ p) {
  const int n = n1 - 1, ld = 2 * n1;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n) return;
  const long row = (long)coarse_perm(warp, n) * ld + n1;
  double acc = 0.0;
  for (int c = lane; c < n; c += 32) {
    const int i = c % L.nx, j = (c / L.nx) % L.ny, k = c / (L.nx * L.ny);
    const double V = (double)L.vx[i] * (double)L.vy[j] * (double)L.vz[k];
    acc += M[row + coarse_perm(c, n)] * (-V * (double)s[c]);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) p[warp] = (float)acc;
}

// ---------------------------------------------------------------------------
// FP64 PCG kernels on the finest level.  psi uses the caller's layout (halo
// hd_psi), q and beta theirs; r, d, qv are dense.
// ---------------------------------------------------------------------------
struct Fine {
  int nx, ny, nz;
  const double *ix1, *ix2, *iy1, *iy2, *iz1, *iz2;  // FP64 1/(dc*df) tables
  const double *beta;
  Lay Lb;
};

__device__ __forceinline__ Coef<double> coef64(const Fine &F, int i, int j, int k) {
  auto b = [&](int a, int bb, int c) { return F.beta[at(F.Lb, a + 1, bb + 1, c + 1)]; };
  const double bc = b(i, j, k);
  Coef<double> c;
  c.aR = 0.5 * (b(wrap(i + 1, F.nx), j, k) + bc) * F.ix1[i];
  c.aL = 0.5 * (bc + b(wrap(i - 1, F.nx), j, k)) * F.ix2[i];
  c.aT = 0.5 * (b(i, clampi(j + 1, F.ny), k) + bc) * F.iy1[j];
  c.aB = 0.5 * (bc + b(i, clampi(j - 1, F.ny), k)) * F.iy2[j];
  c.aF = 0.5 * (b(i, j, wrap(k + 1, F.nz)) + bc) * F.iz1[k];
  c.aK = 0.5 * (bc + b(i, j, wrap(k - 1, F.nz))) * F.iz2[k];
  return c;
}

template <typename G>
__device__ __forceinline__ double apply_L64(const Fine &F, const Coef<double> &c, G get, int i, int j, int k) {
  const double pc = get(i, j, k);
  return c.aR * (get(wrap(i + 1, F.nx), j, k) - pc) - c.aL * (pc - get(wrap(i - 1, F.nx), j, k)) +
         c.aT * (get(i, clampi(j + 1, F.ny), k) - pc) - c.aB * (pc - get(i, clampi(j - 1, F.ny), k)) +
         c.aF * (get(i, j, wrap(k + 1, F.nz)) - pc) - c.aK * (pc - get(i, j, wrap(k - 1, F.nz)));
}

// r = q - L psi; sum q^2 -> acc[0], sum r^2 -> acc[1]; r32 = (float) r
__global__ void __launch_bounds__(kMgThreads) k_pcg_init(Fine F, const double *__restrict__ psi, Lay Lp,
                                                        const double *__restrict__ q, Lay Lq, double *__restrict__ r,
                                                        float *__restrict__ r32, double *__restrict__ acc) {
  const Walk w = walk(F.ny);
  const int i = w.i, k = w.k;
  double qq = 0.0, rr = 0.0;
  if (i < F.nx) {
    auto get = [&](int a, int b, int cc) { return psi[at(Lp, a + 1, b + 1, cc + 1)]; };
#pragma unroll 4
    for (int j = w.j0; j < w.j1; ++j) {
      const int t = (k * F.ny + j) * F.nx + i;
      const Coef<double> c = coef64(F, i, j, k);
      const double qv = q[at(Lq, i + 1, j + 1, k + 1)];
      const double v = qv - apply_L64(F, c, get, i, j, k);
      r[t] = v;
      r32[t] = (float)v;
      qq += qv * qv;
      rr += v * v;
    }
  }
  block_sum2(qq, rr, acc, acc + 1);
}

// qv = L d, sum d*qv -> *dq
__global__ void __launch_bounds__(kMgThreads) k_pcg_qv(Fine F, const double *__restrict__ d, double *__restrict__ qv,
                                                      double *__restrict__ dq) {
  const Walk w = walk(F.ny);
  const int i = w.i, k = w.k;
  double s = 0.0;
  if (i < F.nx) {
    auto get = [&](int a, int b, int cc) { return d[(cc * F.ny + b) * F.nx + a]; };
#pragma unroll 4
    for (int j = w.j0; j < w.j1; ++j) {
      const int t = (k * F.ny + j) * F.nx + i;
      const Coef<double> c = coef64(F, i, j, k);
      const double v = apply_L64(F, c, get, i, j, k);
      qv[t] = v;
      s += d[t] * v;
    }
  }
  block_sum2(s, 0.0, dq, nullptr);
}

// alpha = deltaN / dq; psi += alpha d; r -= alpha qv; sum r^2 -> *rr; r32 = (float) r
__global__ void __launch_bounds__(kMgThreads) k_pcg_update(Fine F, double *__restrict__ psi, Lay Lp,
                                                          const double *__restrict__ d, const double *__restrict__ qv,
                                                          double *__restrict__ r, float *__restrict__ r32,
                                                          const double *__restrict__ sc, double *__restrict__ rr) {
  const Walk w = walk(F.ny);
  const int i = w.i, k = w.k;
  const double alpha = sc[0] / sc[1];  // deltaN / (d . qv)
  double s = 0.0;
  if (i < F.nx) {
#pragma unroll 4
    for (int j = w.j0; j < w.j1; ++j) {
      const int t = (k * F.ny + j) * F.nx + i;
      psi[at(Lp, i + 1, j + 1, k + 1)] += alpha * d[t];
      const double v = r[t] - alpha * qv[t];
      r[t] = v;
      r32[t] = (float)v;
      s += v * v;
    }
  }
  block_sum2(s, 0.0, rr, nullptr);
}

// deltaN_new = r . z (z the preconditioned residual, FP32)
__global__ void __launch_bounds__(kMgThreads) k_pcg_dot(const double *__restrict__ r, const float *__restrict__ z,
                                                       long n, double *__restrict__ out) {
  double s = 0.0;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    s += r[t] * (double)z[t];
  block_sum2(s, 0.0, out, nullptr);
}

// d = z + gamma d, gamma = deltaN_new / deltaN (gamma = 0 for the first direction)
__global__ void __launch_bounds__(kMgThreads) k_pcg_dir(const float *__restrict__ z, double *__restrict__ d, long n,
                                                       const double *__restrict__ sc, int first) {
  const double gamma = first ? 0.0 : sc[2] / sc[3];
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x)
    d[t] = (double)z[t] + gamma * d[t];
}

// beta (caller layout, FP64) -> dense FP32 level-0 copy
__global__ void k_beta32(Fine F, float *__restrict__ b32) {
  const Walk w = walk(F.ny);
  const int i = w.i, k = w.k;
  if (i >= F.nx) return;
  for (int j = w.j0; j < w.j1; ++j) b32[(k * F.ny + j) * F.nx + i] = (float)F.beta[at(F.Lb, i + 1, j + 1, k + 1)];
}

// ghost images of psi (updateBoundaries on one rank): x, z periodic, first y
// ghost layer a copy of the wall cell
__global__ void k_psi_ghosts(double *__restrict__ psi, Lay Lp, int hd, int nx, int ny, int nz) {
  const int ex = nx + 2 * hd, ey = ny + 2 * hd, ez = nz + 2 * hd;
  const long n = (long)ex * ey * ez;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int a = (int)(t % ex) + 1 - hd;
    const long rw = t / ex;
    const int b = (int)(rw % ey) + 1 - hd, c = (int)(rw / ey) + 1 - hd;
    const bool gi = a < 1 || a > nx, gk = c < 1 || c > nz;
    const bool gj = b < 1 || b > ny;
    if (!gi && !gj && !gk) continue;
    if (gj && b != 0 && b != ny + 1) continue;  // deeper y layers are not written
    const int ia = a < 1 ? a + nx : (a > nx ? a - nx : a);
    const int ic = c < 1 ? c + nz : (c > nz ? c - nz : c);
    const int jb = b < 1 ? 1 : (b > ny ? ny : b);
    psi[at(Lp, a, b, c)] = psi[at(Lp, ia, jb, ic)];
  }
}

dim3 wgrid(int nxe, int ny, int nz, int J) {
  return dim3((unsigned)((nxe + kWalkX - 1) / kWalkX), (unsigned)((ny + J - 1) / J), (unsigned)nz);
}
// Rows per block of the level kernels without a reduction: a walk of up to
// jmax rows where the grid stays above rows/div blocks.  One row per block on
// every level made the finest level's kernels launch-rate bound (65,536
// blocks of one row for a residual on 256x256x128): walking up to 4 rows
// (sweeps up to 16) was 7 % faster over a PCG solve.
int rows_j(int nxe, int ny, int nz, long div, int jmax) {
  const long rows = (long)((nxe + kWalkX - 1) / kWalkX) * ny * nz;
  return (int)std::max<long>(1, std::min<long>(jmax, rows / div));
}
// Rows per block of a summing sweep: up to kMgJ (fewer atomics on the sum),
// but never so many that the grid drops below ~8 blocks per SM -- a walk of J
// rows is a serial chain, and on the coarse levels (a few thousand rows) J =
// kMgJ left a few dozen blocks walking 16 rows each (15 us per sweep where
// one row per block takes 3-5 us).
int sum_rows(int nxe, int ny, int nz) {
  const long rows = (long)((nxe + kWalkX - 1) / kWalkX) * ny * nz;
  return (int)std::max<long>(1, std::min<long>(kMgJ, rows / (148L * 8)));
}
unsigned nblk_grid(long n) {
  long b = (n + kMgThreads - 1) / kMgThreads;
  return (unsigned)std::min<long>(b, 148L * 8);
}

}  // namespace

// ===========================================================================
// host side
// ===========================================================================
namespace {
// one direction of one level: faces f(0..n), centroids c(0..n+1) (ghosts included)
struct Axis {
  int n = 0;
  bool periodic = false;
  std::vector<double> f, c;
  double df(int i) const { return f[i] - f[i - 1]; }  // i = 1..n
  double dc(int i) const { return c[i] - c[i - 1]; }  // i = 1..n+1
};

Axis axis_from_metrics(int n, const double *df, const double *dc, bool periodic) {
  Axis a;
  a.n = n;
  a.periodic = periodic;
  a.f.assign(n + 1, 0.0);
  for (int i = 1; i <= n; ++i) a.f[i] = a.f[i - 1] + df[i - 1];
  // centroids from the centroid spacings dc(2..n), anchored so that the grid is
  // symmetric (c(1) + c(n) = f(0) + f(n)): exact for the reference's uniform and
  // tanh grids; ghosts from dc(1) and dc(n+1)
  double span = 0.0;
  for (int i = 2; i <= n; ++i) span += dc[i - 1];
  a.c.assign(n + 2, 0.0);
  a.c[1] = 0.5 * (a.f[0] + a.f[n] - span);
  for (int i = 2; i <= n; ++i) a.c[i] = a.c[i - 1] + dc[i - 1];
  a.c[0] = a.c[1] - dc[0];
  a.c[n + 1] = a.c[n] + dc[n];
  return a;
}

// coarsenGrid (grid.f90:490-544): every other face; the coarse centroid I is the
// fine face 2I-1 (the reference recomputes both from the grid formula, and for
// its uniform and tanh grids they coincide); ghost centroids are periodic
// images in x, z and mirror images through the wall in y (their values are
// copies of the wall cell, so they only enter the smoother's wall weights).
Axis coarsen(const Axis &a) {
  Axis b;
  b.n = a.n / 2;
  b.periodic = a.periodic;
  b.f.resize(b.n + 1);
  for (int I = 0; I <= b.n; ++I) b.f[I] = a.f[2 * I];
  b.c.resize(b.n + 2);
  for (int I = 1; I <= b.n; ++I) b.c[I] = a.f[2 * I - 1];
  const double L = b.f[b.n] - b.f[0];
  if (b.periodic) {
    b.c[0] = b.c[b.n] - L;
    b.c[b.n + 1] = b.c[1] + L;
  } else {
    b.c[0] = 2.0 * b.f[0] - b.c[1];
    b.c[b.n + 1] = 2.0 * b.f[b.n] - b.c[b.n];
  }
  return b;
}
}  // namespace

struct MgSolver::Impl {
  struct Level {
    int nx, ny, nz;
    long n;
    float *p = nullptr, *q = nullptr, *beta = nullptr, *res = nullptr;
    float *tab = nullptr;  // invx1, invx2, invy1, invy2, invz1, invz2, vx, vy, vz, rx, ry, rz, px, py, pz
    MgLev L{};
  };
  std::vector<Level> lv;
  tbfp_mg_params prm{};
  int nx = 0, ny = 0, nz = 0;
  long n = 0;
  // FP64 fine tables and PCG vectors
  double *ix1 = nullptr, *ix2 = nullptr, *iy1 = nullptr, *iy2 = nullptr, *iz1 = nullptr, *iz2 = nullptr;
  double *r = nullptr, *d = nullptr, *qv = nullptr, *sc = nullptr;  // sc: scalars and norms
  float *r32 = nullptr;
  double *Minv = nullptr;
  double *Cb = nullptr;  // multipliers of one Gauss-Jordan panel (n1 x kGB)
  double *msum = nullptr;  // per level: pending sums of p after pre- and post-smoothing
  int n1 = 0;
  int *fail = nullptr;
  std::vector<void *> allocs;
  size_t bytes = 0;
  cudaGraphExec_t vgraph = nullptr;  // one V-cycle from the finest level
  bool graph_failed = false;

  template <typename T>
  cudaError_t alloc(T **p, size_t count) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(count * sizeof(T), 16));
    if (e != cudaSuccess) return e;
    allocs.push_back(q);
    bytes += count * sizeof(T);
    *p = static_cast<T *>(q);
    return cudaSuccess;
  }
  ~Impl() {
    if (vgraph) cudaGraphExecDestroy(vgraph);
    for (void *p : allocs) cudaFree(p);
  }
};

MgSolver::MgSolver() : d_(new Impl) {}
MgSolver::~MgSolver() { delete d_; }
size_t MgSolver::device_bytes() const { return d_->bytes; }

int MgSolver::init(const tbfp_mg_params &prm, int nx, int ny, int nz, const double *dxf, const double *dxc,
                   const double *dyf, const double *dyc, const double *dzf, const double *dzc, std::string *err) {
  Impl &m = *d_;
  if (prm.n_levels < 1 || prm.n_pre < 0 || prm.n_post < 0 || prm.max_iter_mg < 0 || prm.max_iter_pcg < 0 ||
      !(prm.tol_mg > 0.0) || !(prm.tol_pcg > 0.0))
    return *err = "tbfp_pcg_setup: invalid multigrid parameters", TBFP_EINVAL;
  const int f = 1 << (prm.n_levels - 1);
  if (nx % f || ny % f || nz % f)  // checkLevelsNumber (multiGrid.f90:116-145)
    return *err = "tbfp_pcg_setup: nx, ny, nz must be divisible by 2^(n_levels-1)", TBFP_EINVAL;
  m.prm = prm;
  m.nx = nx;
  m.ny = ny;
  m.nz = nz;
  m.n = (long)nx * ny * nz;
  std::vector<Axis> ax{axis_from_metrics(nx, dxf, dxc, true)}, ay{axis_from_metrics(ny, dyf, dyc, false)},
      az{axis_from_metrics(nz, dzf, dzc, true)};
  for (int l = 1; l < prm.n_levels; ++l) {
    ax.push_back(coarsen(ax.back()));
    ay.push_back(coarsen(ay.back()));
    az.push_back(coarsen(az.back()));
  }
  const long ncoarse = (long)ax.back().n * ay.back().n * az.back().n;
  if (ncoarse > 2048)
    return *err = "tbfp_pcg_setup: coarsest level has more than 2048 cells; use more levels", TBFP_EUNSUPPORTED;
  m.n1 = (int)ncoarse + 1;
  if ((long)nx * ny * nz >= (1L << 31) || nz > 65535)
    return *err = "tbfp_pcg_setup: grid too large (2^31 cells or nz > 65535)", TBFP_EUNSUPPORTED;
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t x) {
    if (x != cudaSuccess && e == cudaSuccess) e = x;
  };
  m.lv.resize(prm.n_levels);
  for (int l = 0; l < prm.n_levels; ++l) {
    auto &L = m.lv[l];
    const Axis &X = ax[l], &Y = ay[l], &Z = az[l];
    L.nx = X.n;
    L.ny = Y.n;
    L.nz = Z.n;
    L.n = (long)L.nx * L.ny * L.nz;
    ck(m.alloc(&L.p, L.n));
    ck(m.alloc(&L.q, L.n));
    ck(m.alloc(&L.beta, L.n));
    ck(m.alloc(&L.res, L.n));
    // tables
    std::vector<float> t;
    auto put = [&](const std::vector<double> &v) {
      const size_t off = t.size();
      for (double x : v) t.push_back((float)x);
      return off;
    };
    auto inv = [&](const Axis &A, int which) {  // which 1: 1/(dc(i+1) df(i)), 2: 1/(dc(i) df(i))
      std::vector<double> v(A.n);
      for (int i = 1; i <= A.n; ++i) v[i - 1] = 1.0 / ((which == 1 ? A.dc(i + 1) : A.dc(i)) * A.df(i));
      return v;
    };
    auto vol = [&](const Axis &A) {
      std::vector<double> v(A.n);
      for (int i = 1; i <= A.n; ++i) v[i - 1] = A.df(i);
      return v;
    };
    // restriction weights of this level's cells from the finer level l-1
    auto rweights = [&](const Axis &Fa, const Axis &Ca) {
      std::vector<double> w(2 * Ca.n);
      for (int I = 1; I <= Ca.n; ++I) {
        const double xo = Fa.c[2 * I - 1], xe = Fa.c[2 * I], xc = Ca.c[I];
        w[2 * (I - 1)] = (xe - xc) / (xe - xo);
        w[2 * (I - 1) + 1] = (xc - xo) / (xe - xo);
      }
      return w;
    };
    // prolongation weights of this level's cells from the coarser level l+1
    auto pweights = [&](const Axis &Fa, const Axis &Ca) {
      std::vector<double> w(2 * Fa.n);
      for (int i = 1; i <= Fa.n; ++i) {
        const int ih = i / 2;
        const double c0 = Ca.c[ih], c1 = Ca.c[ih + 1], xf = Fa.c[i];
        w[2 * (i - 1)] = (c1 - xf) / (c1 - c0);
        w[2 * (i - 1) + 1] = (xf - c0) / (c1 - c0);
      }
      return w;
    };
    size_t o[15];
    o[0] = put(inv(X, 1));
    o[1] = put(inv(X, 2));
    o[2] = put(inv(Y, 1));
    o[3] = put(inv(Y, 2));
    o[4] = put(inv(Z, 1));
    o[5] = put(inv(Z, 2));
    o[6] = put(vol(X));
    o[7] = put(vol(Y));
    o[8] = put(vol(Z));
    if (l > 0) {
      o[9] = put(rweights(ax[l - 1], X));
      o[10] = put(rweights(ay[l - 1], Y));
      o[11] = put(rweights(az[l - 1], Z));
    } else {
      o[9] = o[10] = o[11] = 0;
    }
    if (l + 1 < prm.n_levels) {
      o[12] = put(pweights(X, ax[l + 1]));
      o[13] = put(pweights(Y, ay[l + 1]));
      o[14] = put(pweights(Z, az[l + 1]));
    } else {
      o[12] = o[13] = o[14] = 0;
    }
    ck(m.alloc(&L.tab, t.size()));
    if (e == cudaSuccess) ck(cudaMemcpy(L.tab, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
    MgLev &G = L.L;
    G.nx = L.nx;
    G.ny = L.ny;
    G.nz = L.nz;
    G.invx1 = L.tab + o[0];
    G.invx2 = L.tab + o[1];
    G.invy1 = L.tab + o[2];
    G.invy2 = L.tab + o[3];
    G.invz1 = L.tab + o[4];
    G.invz2 = L.tab + o[5];
    G.vx = L.tab + o[6];
    G.vy = L.tab + o[7];
    G.vz = L.tab + o[8];
    G.rx = L.tab + o[9];
    G.ry = L.tab + o[10];
    G.rz = L.tab + o[11];
    G.px = L.tab + o[12];
    G.py = L.tab + o[13];
    G.pz = L.tab + o[14];
  }
  // FP64 fine tables from the caller's metrics (the reference's own values)
  std::vector<double> x1(nx), x2(nx), y1(ny), y2(ny), z1(nz), z2(nz);
  for (int i = 0; i < nx; ++i) {
    x1[i] = 1.0 / (dxc[i + 1] * dxf[i]);
    x2[i] = 1.0 / (dxc[i] * dxf[i]);
  }
  for (int j = 0; j < ny; ++j) {
    y1[j] = 1.0 / (dyc[j + 1] * dyf[j]);
    y2[j] = 1.0 / (dyc[j] * dyf[j]);
  }
  for (int k = 0; k < nz; ++k) {
    z1[k] = 1.0 / (dzc[k + 1] * dzf[k]);
    z2[k] = 1.0 / (dzc[k] * dzf[k]);
  }
  auto up = [&](double **dst, const std::vector<double> &v) {
    ck(m.alloc(dst, v.size()));
    if (e == cudaSuccess) ck(cudaMemcpy(*dst, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
  };
  up(&m.ix1, x1);
  up(&m.ix2, x2);
  up(&m.iy1, y1);
  up(&m.iy2, y2);
  up(&m.iz1, z1);
  up(&m.iz2, z2);
  ck(m.alloc(&m.r, m.n));
  ck(m.alloc(&m.d, m.n));
  ck(m.alloc(&m.qv, m.n));
  ck(m.alloc(&m.r32, m.n));
  ck(m.alloc(&m.sc, 16));
  ck(m.alloc(&m.Minv, (size_t)m.n1 * 2 * m.n1));
  ck(m.alloc(&m.Cb, (size_t)m.n1 * kGB));
  ck(m.alloc(&m.msum, 2 * m.lv.size()));
  ck(m.alloc(&m.fail, 1));
  if (e != cudaSuccess) {
    *err = std::string("tbfp_pcg_setup: ") + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? TBFP_ENOMEM : TBFP_ECUDA;
  }
  return TBFP_OK;
}

// sc layout: [0] deltaN, [1] d.qv, [2] deltaN_new, [3] deltaN_old, [4] sum q^2, [5] sum r^2,
//            [6] MG residual sum res^2, [7] MG sum q^2
namespace {
struct Run {
  MgSolver::Impl &m;
  cudaStream_t st;

  // iterateGS (rbgs.f90:186-272).  The reference removes the mean
  // (correctFullNeumann) after every red+black iteration.  A sweep commutes
  // with adding a constant to p (the update is an average of neighbours, q
  // fixed), so removing the mean once after the last iteration gives the same
  // p.
  // The mean of p is not removed in a separate pass: the last red and black
  // sweeps of a smoothing call add sum(p) into `slot`, and the kernel that
  // next combines p with another level (k_prolong_add) subtracts it; the
  // residual in between does not need it (L p ignores constants).  Returns
  // whether a sum is pending in `slot`.  With reset, p starts from 0.
  bool rbgs(int l, int n_iter, bool reset, double *slot) {
    auto &L = m.lv[l];
    if (reset) k_fill<<<nblk_grid(L.n), kMgThreads, 0, st>>>(L.p, L.n, 0.0f);
    if (n_iter == 0) return false;
    for (int it = 0; it < n_iter; ++it) {
      const bool last = it == n_iter - 1;
      const int J = last ? sum_rows((L.nx + 1) / 2, L.ny, L.nz) : rows_j((L.nx + 1) / 2, L.ny, L.nz, 4096, kMgJ);
      double *sum = last ? slot : nullptr;
      k_rbgs_colour<<<wgrid((L.nx + 1) / 2, L.ny, L.nz, J), kWalkX, 0, st>>>(L.L, L.p, L.q, L.beta, 0, sum);
      k_rbgs_colour<<<wgrid((L.nx + 1) / 2, L.ny, L.nz, J), kWalkX, 0, st>>>(L.L, L.p, L.q, L.beta, 1, sum);
    }
    return true;
  }

  void vcycle(int l) {
    const int last = (int)m.lv.size() - 1;
    auto &L = m.lv[l];
    if (l == 0) cudaMemsetAsync(m.msum, 0, 2 * m.lv.size() * sizeof(double), st);
    if (l == last) {
      k_coarse_apply<<<(unsigned)((L.n * 32 + 255) / 256), 256, 0, st>>>(L.L, m.Minv, m.n1, L.q, L.p);
      return;  // the bordered solve gives sum(p) = 0: nothing pending
    }
    double *pre = m.msum + 2 * l, *post = m.msum + 2 * l + 1;
    const bool hpre = rbgs(l, m.prm.n_pre, l != 0, pre);
    k_mg_residual<<<wgrid(L.nx, L.ny, L.nz, rows_j(L.nx, L.ny, L.nz, 4096, 4)), kWalkX, 0, st>>>(L.L, L.p, L.q, L.beta, L.res, nullptr);
    auto &C = m.lv[l + 1];
    k_restrict<<<wgrid(C.nx, C.ny, C.nz, rows_j(C.nx, C.ny, C.nz, 4096, 4)), kWalkX, 0, st>>>(L.L, C.L, L.res, C.q);
    vcycle(l + 1);
    const bool hcpost = l + 1 < last && m.prm.n_post > 0;
    k_prolong_add<<<wgrid(L.nx, L.ny, L.nz, rows_j(L.nx, L.ny, L.nz, 4096, 4)), kWalkX, 0, st>>>(
        L.L, C.L, C.p, L.p, hpre ? pre : nullptr, 1.0 / (double)L.n, hcpost ? m.msum + 2 * (l + 1) + 1 : nullptr,
        1.0 / (double)C.n);
    const bool hpost = rbgs(l, m.prm.n_post, false, post);
    if (l == 0 && hpost) k_sub_mean<<<nblk_grid(L.n), kMgThreads, 0, st>>>(L.p, L.n, post);
  }

  // ||q - L p|| / ||q|| at the finest level (computeResiduals' res) into *res;
  // a CUDA error returns TBFP_ECUDA with its text in *err.
  int fine_residual(double *res, std::string *err) {
    auto &L = m.lv[0];
    cudaMemsetAsync(m.sc + 6, 0, 2 * sizeof(double), st);
    k_mg_residual<<<wgrid(L.nx, L.ny, L.nz, kMgJ), kWalkX, 0, st>>>(L.L, L.p, L.q, L.beta, L.res, m.sc + 6);
    double v[2] = {0.0, 0.0};
    cudaMemcpyAsync(v, m.sc + 6, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    const cudaError_t e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      *err = std::string("tbfp_pcg_solve (multigrid residual): ") + cudaGetErrorString(e);
      return TBFP_ECUDA;
    }
    *res = std::sqrt(v[0]) / (std::sqrt(v[1]) + 1e-300);
    return TBFP_OK;
  }

  // solveMG (multiGrid.f90:165-182): p starts at 0, V-cycles while res > tol_mg.
  // Each V-cycle is one launch of a CUDA graph captured once per hierarchy
  // (its buffers never move); without a graph the kernels are launched one by one.
  // Adds the V-cycles to *cycles.  A non-finite residual (the FP32 hierarchy
  // overflowed, or a NaN reached it) is a hard error.
  int solve_mg(int *cycles, std::string *err) {
    auto &L = m.lv[0];
    k_fill<<<nblk_grid(L.n), kMgThreads, 0, st>>>(L.p, L.n, 0.0f);
    double res = 0.0;
    int rc = fine_residual(&res, err);
    int it = 0;
    while (rc == TBFP_OK && std::isfinite(res) && it < m.prm.max_iter_mg && res > m.prm.tol_mg) {
      ++it;
      if (m.vgraph) cudaGraphLaunch(m.vgraph, st);
      else vcycle(0);
      rc = fine_residual(&res, err);
    }
    *cycles += it;
    if (rc) return rc;
    if (!std::isfinite(res)) {
      *err = "tbfp_pcg_solve: non-finite multigrid residual (NaN or Inf in q, beta or the iterate)";
      return TBFP_ENONFINITE;
    }
    return TBFP_OK;
  }

  void capture() {
    if (m.vgraph || m.graph_failed) return;
    cudaStream_t cs = nullptr;
    cudaGraph_t gr = nullptr;
    bool ok = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) == cudaSuccess;
    if (ok) ok = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      Run r{m, cs};
      r.vcycle(0);
      ok = cudaStreamEndCapture(cs, &gr) == cudaSuccess && gr != nullptr;
    }
    if (ok) ok = cudaGraphInstantiate(&m.vgraph, gr, 0) == cudaSuccess;
    if (gr) cudaGraphDestroy(gr);
    if (cs) cudaStreamDestroy(cs);
    if (!ok) {
      m.vgraph = nullptr;
      m.graph_failed = true;
      cudaGetLastError();  // clear a capture error; the eager path is used instead
    }
  }
};
}  // namespace

int MgSolver::solve(double *psi, Lay Lp, int hd_psi, const double *beta, Lay Lb, const double *q, Lay Lq,
                    cudaStream_t st, int *iters, double *rel, int *mg_cycles, std::string *err) {
  Impl &m = *d_;
  Fine F{};
  F.nx = m.nx;
  F.ny = m.ny;
  F.nz = m.nz;
  F.ix1 = m.ix1;
  F.ix2 = m.ix2;
  F.iy1 = m.iy1;
  F.iy2 = m.iy2;
  F.iz1 = m.iz1;
  F.iz2 = m.iz2;
  F.beta = beta;
  F.Lb = Lb;
  Run run{m, st};
  run.capture();
  *mg_cycles = 0;
  // beta on every level (restrictField, field.f90:1442-1470)
  k_beta32<<<wgrid(m.nx, m.ny, m.nz, 1), kWalkX, 0, st>>>(F, m.lv[0].beta);
  for (size_t l = 1; l < m.lv.size(); ++l)
    k_restrict<<<wgrid(m.lv[l].nx, m.lv[l].ny, m.lv[l].nz, 1), kWalkX, 0, st>>>(m.lv[l - 1].L, m.lv[l].L,
                                                                                 m.lv[l - 1].beta, m.lv[l].beta);
  // coarsest bordered system, inverted once for this beta
  auto &C = m.lv.back();
  cudaMemsetAsync(m.fail, 0, sizeof(int), st);
  k_coarse_assemble<<<1, 1024, 0, st>>>(C.L, C.beta, m.Minv, m.n1);
  for (int p0 = 0; p0 < m.n1; p0 += kGB) {
    k_gj_panel<<<1, kGPT, 0, st>>>(m.Minv, m.n1, p0, m.Cb, m.fail);
    const dim3 ug((unsigned)((2 * m.n1 - p0 + 127) / 128), (unsigned)((m.n1 + 31) / 32));
    k_gj_update<<<ug, 256, 0, st>>>(m.Minv, m.n1, p0, m.Cb);
  }
  // r = q - L psi (psi: the initial guess), z = MG(r), d = z
  cudaMemsetAsync(m.sc, 0, 16 * sizeof(double), st);
  k_pcg_init<<<wgrid(m.nx, m.ny, m.nz, kMgJ), kWalkX, 0, st>>>(F, psi, Lp, q, Lq, m.r, m.lv[0].q, m.sc + 4);
  int rc = run.solve_mg(mg_cycles, err);
  if (rc) return rc;
  k_pcg_dot<<<nblk_grid(m.n), kMgThreads, 0, st>>>(m.r, m.lv[0].p, m.n, m.sc + 0);
  k_pcg_dir<<<nblk_grid(m.n), kMgThreads, 0, st>>>(m.lv[0].p, m.d, m.n, m.sc, 1);
  double nrm[2];
  int fail = 0;
  cudaMemcpyAsync(nrm, m.sc + 4, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&fail, m.fail, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    *err = std::string("tbfp_pcg_solve: ") + cudaGetErrorString(e);
    return TBFP_ECUDA;
  }
  if (fail) {
    *err = "tbfp_pcg_solve: singular coarsest-level system";
    return TBFP_ESINGULAR;
  }
  const double qn = std::sqrt(nrm[0] + 1e-300);
  double rr = nrm[1];
  int it = 0;
  double res = std::sqrt(rr) / qn;
  while (true) {
    res = std::sqrt(rr) / qn;
    if (!std::isfinite(res)) {  // a NaN would otherwise fail every comparison and read as converged
      *err = "tbfp_pcg_solve: non-finite PCG residual (NaN or Inf in q, beta or the initial guess)";
      return TBFP_ENONFINITE;
    }
    if (it == m.prm.max_iter_pcg || !(res > m.prm.tol_pcg)) break;
    ++it;
    cudaMemsetAsync(m.sc + 1, 0, sizeof(double), st);
    k_pcg_qv<<<wgrid(m.nx, m.ny, m.nz, kMgJ), kWalkX, 0, st>>>(F, m.d, m.qv, m.sc + 1);
    cudaMemsetAsync(m.sc + 5, 0, sizeof(double), st);
    k_pcg_update<<<wgrid(m.nx, m.ny, m.nz, kMgJ), kWalkX, 0, st>>>(F, psi, Lp, m.d, m.qv, m.r, m.lv[0].q, m.sc, m.sc + 5);
    rc = run.solve_mg(mg_cycles, err);
    if (rc) return rc;
    cudaMemcpyAsync(m.sc + 3, m.sc + 0, sizeof(double), cudaMemcpyDeviceToDevice, st);  // deltaN_old
    cudaMemsetAsync(m.sc + 2, 0, sizeof(double), st);
    k_pcg_dot<<<nblk_grid(m.n), kMgThreads, 0, st>>>(m.r, m.lv[0].p, m.n, m.sc + 2);
    k_pcg_dir<<<nblk_grid(m.n), kMgThreads, 0, st>>>(m.lv[0].p, m.d, m.n, m.sc, 0);
    cudaMemcpyAsync(m.sc + 0, m.sc + 2, sizeof(double), cudaMemcpyDeviceToDevice, st);  // deltaN = new
    cudaMemcpyAsync(&rr, m.sc + 5, sizeof(double), cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      *err = std::string("tbfp_pcg_solve: ") + cudaGetErrorString(e);
      return TBFP_ECUDA;
    }
  }
  k_psi_ghosts<<<nblk_grid((long)(m.nx + 2 * hd_psi) * (m.ny + 2 * hd_psi) * (m.nz + 2 * hd_psi)), kMgThreads, 0,
                 st>>>(psi, Lp, hd_psi, m.nx, m.ny, m.nz);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    *err = std::string("tbfp_pcg_solve: ") + cudaGetErrorString(e);
    return TBFP_ECUDA;
  }
  *iters = it;
  *rel = res;
  return (res > m.prm.tol_pcg) ? TBFP_ENOTCONVERGED : TBFP_OK;
}

}  // namespace tbfp
