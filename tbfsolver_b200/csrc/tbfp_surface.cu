// Surface tension on the grid: the interface cells, the height-function
// curvature and the face force that the projection reads as st (the reference's
// computeSurfaceTension, VOF.f90:1872-2002, with computeBlockCurvature and
// hfColumn, :2070-2290, after Popinet 2009).
//
// The reference works on per-bubble blocks; this is a grid-wide restatement:
//   * interface cells: mixed eps <= c <= 1-eps, full c >= 1-eps (VOF.f90:1094-1108);
//     a full cell with an empty 6-neighbour becomes mixed with c = 1-2 eps
//     (search_full_interface_cells, :672-726);
//   * curvature at a mixed cell: the height-function direction is the largest
//     component of a smoothed central-difference normal (then the second, then
//     the third); in that direction nine columns (the cell's 3x3 neighbourhood
//     across it) each walk at most kStColumn cells toward the full phase and
//     toward the empty phase; the column height is the sum of c times the cell
//     width between the two ends, the interface position is the full end's outer
//     face minus that height; with all nine columns valid the curvature is
//     s * div(grad f / sqrt(1 + |grad f|^2)) of the positions f by second-order
//     (non-uniform in y) differences, s the orientation of the column.  Columns
//     stop at the walls; a cell without a valid direction gets curvature 0 (the
//     reference fits a parabola through interface centroids there);
//   * face force: sigma * k_f * (c(Q) - c(P)) / dc, k_f the mean curvature of the
//     two cells if both are mixed, else the mixed one's, else 0 (computeBlockST,
//     :1904-1996); zero on the wall faces.
// The decisions (the normal's ranking, the column sums) use adds and multiplies
// that the compiler does not contract, so they are those of the oracle's
// restatement in oracle/tbfp_oracle.py (surface_tension).
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"

namespace tbfp {

namespace {

constexpr int kStColumn = 6;

__device__ __forceinline__ long dix(const StGrid &g, int i, int j, int k) {  // dense index, wrap x and z
  i = (i % g.nx + g.nx) % g.nx;
  k = (k % g.nz + g.nz) % g.nz;
  return (long)i + (long)g.nx * ((long)j + (long)g.ny * k);
}
__device__ __forceinline__ int clampj(const StGrid &g, int j) { return j < 0 ? 0 : (j >= g.ny ? g.ny - 1 : j); }

// classes of the original field: 1 mixed, 2 full (both bits when c == 1-eps)
__device__ __forceinline__ int cls0(double c, double eps) {
  return ((c >= 0.0 + eps && c <= 1.0 - eps) ? 1 : 0) | (c >= 1.0 - eps ? 2 : 0);
}

__global__ void k_st_classify(const double *__restrict__ c, Lay Lc, StGrid g, double eps, double *__restrict__ cp,
                              unsigned char *__restrict__ fl) {
  const long n = (long)g.nx * g.ny * g.nz;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) {
    const int i = (int)(t % g.nx), j = (int)((t / g.nx) % g.ny), k = (int)(t / ((long)g.nx * g.ny));
    auto cv = [&](int ii, int jj, int kk) {
      ii = (ii % g.nx + g.nx) % g.nx;
      kk = (kk % g.nz + g.nz) % g.nz;
      return c[at(Lc, ii + 1, clampj(g, jj) + 1, kk + 1)];
    };
    const double c0 = cv(i, j, k);
    int f = cls0(c0, eps);
    double cout = c0;
    if (f & 2) {  // a full cell next to an empty one is an interface cell
      const int nb[6] = {cls0(cv(i + 1, j, k), eps), cls0(cv(i - 1, j, k), eps), cls0(cv(i, j + 1, k), eps),
                         cls0(cv(i, j - 1, k), eps), cls0(cv(i, j, k + 1), eps), cls0(cv(i, j, k - 1), eps)};
      bool empty_nb = false;
      for (int q = 0; q < 6; ++q) empty_nb = empty_nb || nb[q] == 0;
      if (empty_nb) {
        f = 1;
        cout = 1.0 - 2.0 * eps;
      }
    }
    cp[t] = cout;
    fl[t] = (unsigned char)f;
  }
}

__device__ __forceinline__ double face_pos(const StGrid &g, int d, int q) {
  return d == 0 ? q * g.dx : (d == 2 ? q * g.dz : g.yf[q]);
}

__global__ void __launch_bounds__(128) k_st_curvature(const double *__restrict__ cp, const unsigned char *__restrict__ fl,
                                                      StGrid g, double *__restrict__ kap) {
  const long n = (long)g.nx * g.ny * g.nz;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  kap[t] = 0.0;
  if (!(fl[t] & 1)) return;
  const int i = (int)(t % g.nx), j = (int)((t / g.nx) % g.ny), k = (int)(t / ((long)g.nx * g.ny));
  const double w[3] = {1.0, 2.0, 1.0};
  double nxs = 0.0, nys = 0.0, nzs = 0.0;
  for (int b = 0; b < 3; ++b)
    for (int e = 0; e < 3; ++e) {
      const int jj = clampj(g, j + b - 1);
      const double dd = __dsub_rn(cp[dix(g, i + 1, jj, k + e - 1)], cp[dix(g, i - 1, jj, k + e - 1)]);
      nxs = __dadd_rn(nxs, __dmul_rn(__dmul_rn(w[b], w[e]), dd));
    }
  const int jm = clampj(g, j - 1), jp = clampj(g, j + 1);
  for (int a = 0; a < 3; ++a)
    for (int e = 0; e < 3; ++e) {
      const double dd = __dsub_rn(cp[dix(g, i + a - 1, jp, k + e - 1)], cp[dix(g, i + a - 1, jm, k + e - 1)]);
      nys = __dadd_rn(nys, __dmul_rn(__dmul_rn(w[a], w[e]), dd));
    }
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      const int jj = clampj(g, j + b - 1);
      const double dd = __dsub_rn(cp[dix(g, i + a - 1, jj, k + 1)], cp[dix(g, i + a - 1, jj, k - 1)]);
      nzs = __dadd_rn(nzs, __dmul_rn(__dmul_rn(w[a], w[b]), dd));
    }
  double ydist = 0.0;
  for (int J = jm + 1; J <= jp; ++J) ydist = __dadd_rn(ydist, g.dyc[J]);
  const double nv[3] = {nxs / (2.0 * g.dx), jp > jm ? nys / ydist : 0.0, nzs / (2.0 * g.dz)};
  int order[3];
  bool used[3] = {false, false, false};
  for (int r = 0; r < 3; ++r) {  // maxloc: the first largest remaining component
    int best = -1;
    for (int d = 0; d < 3; ++d)
      if (!used[d] && (best < 0 || fabs(nv[d]) > fabs(nv[best]))) best = d;
    order[r] = best;
    used[best] = true;
  }
  const int P[3] = {i, j, k};
  const int nn[3] = {g.nx, g.ny, g.nz};
  for (int r = 0; r < 3; ++r) {
    const int d = order[r];
    const int s = nv[d] >= 0.0 ? 1 : -1;
    const int t1 = d == 0 ? 1 : 0, t2 = d == 2 ? 1 : 2;
    double F[3][3];
    bool ok = true;
    for (int a = -1; a <= 1 && ok; ++a)
      for (int b = -1; b <= 1 && ok; ++b) {
        int st0[3] = {P[0], P[1], P[2]};
        st0[t1] += a;
        st0[t2] += b;
        if (st0[1] < 0 || st0[1] >= g.ny) {
          ok = false;
          break;
        }
        const int q0 = st0[d];
        auto cell = [&](int tt, long *out) -> bool {  // false: outside the walls
          int x[3] = {st0[0], st0[1], st0[2]};
          x[d] = q0 + s * tt;
          if (x[1] < 0 || x[1] >= g.ny) return false;
          *out = dix(g, x[0], x[1], x[2]);
          return true;
        };
        int tf = -1, te = -1;
        for (int tt = 0; tt <= kStColumn; ++tt) {
          long cc;
          if (!cell(tt, &cc)) break;
          if (fl[cc] & 2) {
            tf = tt;
            break;
          }
        }
        for (int tt = 0; tt <= kStColumn; ++tt) {
          long cc;
          if (!cell(-tt, &cc)) break;
          if (fl[cc] == 0) {
            te = tt;
            break;
          }
        }
        if (tf < 0 || te < 0) {
          ok = false;
          break;
        }
        double hs = 0.0;
        for (int tt = -te; tt <= tf; ++tt) {
          long cc;
          cell(tt, &cc);
          const int qq = q0 + s * tt;
          const double wd = d == 0 ? g.dx : (d == 2 ? g.dz : g.dyf[qq]);
          hs = __dadd_rn(hs, __dmul_rn(cp[cc], wd));
        }
        const int qf = q0 + s * tf;
        const double xf = s > 0 ? face_pos(g, d, qf + 1) : face_pos(g, d, qf);
        (void)nn;
        F[a + 1][b + 1] = s > 0 ? __dsub_rn(xf, hs) : __dadd_rn(xf, hs);
      }
    if (!ok) continue;
    auto spacing = [&](int tdir, int p, double *hm, double *hp) {
      if (tdir == 0) *hm = *hp = g.dx;
      else if (tdir == 2) *hm = *hp = g.dz;
      else {
        *hm = g.dyc[p];
        *hp = g.dyc[p + 1];
      }
    };
    double h1m, h1p, h2m, h2p;
    spacing(t1, P[t1], &h1m, &h1p);
    spacing(t2, P[t2], &h2m, &h2p);
    const double den1 = h1p * h1m * (h1p + h1m), den2 = h2p * h2m * (h2p + h2m);
    const double d1 = (h1m * h1m * F[2][1] - h1p * h1p * F[0][1] + (h1p * h1p - h1m * h1m) * F[1][1]) / den1;
    const double d11 = 2.0 * (h1m * F[2][1] - (h1p + h1m) * F[1][1] + h1p * F[0][1]) / den1;
    const double d2 = (h2m * h2m * F[1][2] - h2p * h2p * F[1][0] + (h2p * h2p - h2m * h2m) * F[1][1]) / den2;
    const double d22 = 2.0 * (h2m * F[1][2] - (h2p + h2m) * F[1][1] + h2p * F[1][0]) / den2;
    const double d12 = (F[2][2] - F[2][0] - F[0][2] + F[0][0]) / ((h1p + h1m) * (h2p + h2m));
    const double num = d11 * (1.0 + d2 * d2) + d22 * (1.0 + d1 * d1) - 2.0 * d1 * d2 * d12;
    const double gg = 1.0 + d1 * d1 + d2 * d2;
    kap[t] = s * num / (gg * sqrt(gg));
    return;
  }
}

__device__ __forceinline__ double face_k(double kp, bool mp, double kq, bool mq) {
  return (mp && mq) ? 0.5 * (kq + kp) : (mq ? kq : (mp ? kp : 0.0));
}

// st on every element of the three staggered arrays (their halos included):
// component d, face index along d (Fortran, 0..n), the other two indices wrap
// periodically; y faces 0 and ny and the y ghost rows are zero.
__global__ void k_st_faces(const double *__restrict__ cp, const unsigned char *__restrict__ fl,
                           const double *__restrict__ kap, StGrid g, double sigma, double *__restrict__ sx,
                           Lay Lx, long nsx, double *__restrict__ sy, Lay Ly, long nsy, double *__restrict__ sz,
                           Lay Lz, long nsz) {
  const long tot = nsx + nsy + nsz;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
    int d;
    long e;
    const Lay *L;
    double *out;
    if (t < nsx) {
      d = 0, e = t, L = &Lx, out = sx;
    } else if (t < nsx + nsy) {
      d = 1, e = t - nsx, L = &Ly, out = sy;
    } else {
      d = 2, e = t - nsx - nsy, L = &Lz, out = sz;
    }
    // Fortran indices of element e
    const long i = e % L->sj + L->ilo, j = (e / L->sj) % (L->sk / L->sj) + L->jlo, k = e / L->sk + L->klo;
    double v = 0.0;
    if (d == 1) {
      if (j >= 1 && j <= g.ny - 1) {  // face j between cells j and j+1 (Fortran)
        const long p = dix(g, (int)i - 1, (int)j - 1, (int)k - 1), q = dix(g, (int)i - 1, (int)j, (int)k - 1);
        v = sigma * face_k(kap[p], fl[p] & 1, kap[q], fl[q] & 1) * ((cp[q] - cp[p]) / g.dyc[j]);
      }
    } else if (j >= 1 && j <= g.ny) {
      long p, q;
      if (d == 0) {  // face i between cells i and i+1 (Fortran), periodic
        p = dix(g, (int)i - 1, (int)j - 1, (int)k - 1);
        q = dix(g, (int)i, (int)j - 1, (int)k - 1);
      } else {
        p = dix(g, (int)i - 1, (int)j - 1, (int)k - 1);
        q = dix(g, (int)i - 1, (int)j - 1, (int)k);
      }
      const double dc = d == 0 ? g.dx : g.dz;
      v = sigma * face_k(kap[p], fl[p] & 1, kap[q], fl[q] & 1) * ((cp[q] - cp[p]) / dc);
    }
    out[e] = v;
  }
}

// curvature as a cell field with the layout of c: interior, x/z ghosts periodic, y ghosts 0
__global__ void k_st_kappa_out(const double *__restrict__ kap, StGrid g, double *__restrict__ out, Lay L, long n) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const long i = e % L.sj + L.ilo, j = (e / L.sj) % (L.sk / L.sj) + L.jlo, k = e / L.sk + L.klo;
    out[e] = (j >= 1 && j <= g.ny) ? kap[dix(g, (int)i - 1, (int)j - 1, (int)k - 1)] : 0.0;
  }
}

int grid_blocks(long n, int threads) {
  long b = (n + threads - 1) / threads;
  return (int)(b < 148 * 32 ? (b < 1 ? 1 : b) : 148 * 32);
}

}  // namespace

void launch_surface_tension(const double *c, Lay Lc, const StGrid &g, double eps, double sigma, double *cp,
                            unsigned char *fl, double *kap, double *kap_out, Lay Lk, long nk, double *sx, Lay Lx,
                            long nsx, double *sy, Lay Ly, long nsy, double *sz, Lay Lz, long nsz, cudaStream_t st) {
  const long n = (long)g.nx * g.ny * g.nz;
  k_st_classify<<<grid_blocks(n, 256), 256, 0, st>>>(c, Lc, g, eps, cp, fl);
  k_st_curvature<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(cp, fl, g, kap);
  k_st_faces<<<grid_blocks(nsx + nsy + nsz, 256), 256, 0, st>>>(cp, fl, kap, g, sigma, sx, Lx, nsx, sy, Ly, nsy, sz,
                                                               Lz, nsz);
  if (kap_out) k_st_kappa_out<<<grid_blocks(nk, 256), 256, 0, st>>>(kap, g, kap_out, Lk, nk);
}

}  // namespace tbfp
