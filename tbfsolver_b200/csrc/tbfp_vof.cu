// Material properties from the volume fraction: updateMaterialProps
// (VOF.f90:197-233) with smoothVF (VOF.f90:235-262).  cs is c after two
// cell -> vertex -> cell passes (cellToVertex / vertexToCell,
// interpolation.f90:188-276), each followed by the boundary update of a cell
// field (zero normal gradient at the y walls, periodic halos in x then z);
// then rho = rhog*cs + (1-cs)*rhol and mu = mug*cs + (1-cs)*mul over the whole
// arrays, halos included.  FP64; the weights of both interpolations are
// products of per-direction distances, tabulated on the host.
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"

namespace tbfp {

namespace {

constexpr int kVT = 128;

// vertex (i, j, k), 0 <= i <= nx: from cells i..i+1 (and j, k likewise)
__global__ void __launch_bounds__(kVT) k_cell_to_vertex(VofTab t, const double *__restrict__ q, Lay L,
                                                        double *__restrict__ qv, int nx, int ny, int nz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i > nx) return;
  const int o = (int)at(L, i, j, k), sj = (int)L.sj, sk = (int)L.sk;
  const double X1 = t.cx1[i], X2 = t.cx2[i], Y1 = t.cy1[j], Y2 = t.cy2[j], Z1 = t.cz1[k], Z2 = t.cz2[k];
  // weights and sum in the order of interpolation.f90:206-224
  const double w1 = (X1 * Y1) * Z1, w2 = (X2 * Y1) * Z1, w3 = (X1 * Y1) * Z2, w4 = (X2 * Y1) * Z2;
  const double w5 = (X1 * Y2) * Z1, w6 = (X2 * Y2) * Z1, w7 = (X1 * Y2) * Z2, w8 = (X2 * Y2) * Z2;
  const double V = (t.hx[i] * t.hy[j]) * t.hz[k];
  double s = w1 * q[o + sj];
  s = s + w2 * q[o + 1 + sj];
  s = s + w3 * q[o + sj + sk];
  s = s + w4 * q[o + 1 + sj + sk];
  s = s + w5 * q[o];
  s = s + w6 * q[o + 1];
  s = s + w7 * q[o + sk];
  s = s + w8 * q[o + 1 + sk];
  qv[((long)k * (ny + 1) + j) * (nx + 1) + i] = s / V;
}

// interior cell (i, j, k), 1 <= i <= nx: from vertices i-1..i
__global__ void __launch_bounds__(kVT) k_vertex_to_cell(VofTab t, const double *__restrict__ qv,
                                                        double *__restrict__ q, Lay L, int nx, int ny) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1, k = blockIdx.z + 1;
  if (i > nx) return;
  const long vj = nx + 1, vk = (long)(ny + 1) * (nx + 1);
  const long v = (long)(k - 1) * vk + (long)(j - 1) * vj + (i - 1);  // qv(i-1, j-1, k-1)
  const double X1 = t.vx1[i - 1], X2 = t.vx2[i - 1], Y1 = t.vy1[j - 1], Y2 = t.vy2[j - 1];
  const double Z1 = t.vz1[k - 1], Z2 = t.vz2[k - 1];
  // weights and sum in the order of interpolation.f90:252-271
  const double w1 = (X1 * Y1) * Z1, w2 = (X2 * Y1) * Z1, w3 = (X1 * Y1) * Z2, w4 = (X2 * Y1) * Z2;
  const double w5 = (X1 * Y2) * Z1, w6 = (X2 * Y2) * Z1, w7 = (X1 * Y2) * Z2, w8 = (X2 * Y2) * Z2;
  const double V = (t.Vx[i - 1] * t.Vy[j - 1]) * t.Vz[k - 1];
  double s = w1 * qv[v + vj];
  s = s + w2 * qv[v + 1 + vj];
  s = s + w3 * qv[v + vj + vk];
  s = s + w4 * qv[v + 1 + vj + vk];
  s = s + w5 * qv[v];
  s = s + w6 * qv[v + 1];
  s = s + w7 * qv[v + vk];
  s = s + w8 * qv[v + 1 + vk];
  q[at(L, i, j, k)] = s / V;
}

// updateBoundaries of a cell field of the channel (field.f90:950-974):
// phase 0, zero normal gradient at the y walls on the interior i, k range
// (one ghost layer, boundaryField_S.f90:694-727); phase 1, periodic x halos
// over all j, k; phase 2, periodic z halos over all i, j.
__global__ void k_bc_cell(double *__restrict__ f, Lay L, int nx, int ny, int nz, int hd, int phase) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x, b = blockIdx.y;
  if (phase == 0) {
    const int i = a + 1, k = b + 1;
    if (i > nx) return;
    f[at(L, i, 0, k)] = f[at(L, i, 1, k)];
    f[at(L, i, ny + 1, k)] = f[at(L, i, ny, k)];
  } else if (phase == 1) {
    const int j = a + 1 - hd, k = b + 1 - hd;  // j, k over the extended ranges
    if (j > ny + hd) return;
    for (int g = 0; g < hd; ++g) {
      f[at(L, nx + 1 + g, j, k)] = f[at(L, 1 + g, j, k)];
      f[at(L, 1 - hd + g, j, k)] = f[at(L, nx - hd + 1 + g, j, k)];
    }
  } else {
    const int i = a + 1 - hd, j = b + 1 - hd;  // i, j over the extended ranges
    if (i > nx + hd) return;
    for (int g = 0; g < hd; ++g) {
      f[at(L, i, j, nz + 1 + g)] = f[at(L, i, j, 1 + g)];
      f[at(L, i, j, 1 - hd + g)] = f[at(L, i, j, nz - hd + 1 + g)];
    }
  }
}

// rho and mu over the whole arrays (VOF.f90:220-221)
__global__ void k_props(const double *__restrict__ cs, double *__restrict__ rho, double *__restrict__ mu, long n,
                        double rhol, double rhog, double mul, double mug) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const double c = cs[e];
    mu[e] = mug * c + (1.0 - c) * mul;
    rho[e] = rhog * c + (1.0 - c) * rhol;
  }
}

void bc_cell(double *f, Lay L, int nx, int ny, int nz, int hd, cudaStream_t st) {
  k_bc_cell<<<dim3((nx + kVT - 1) / kVT, nz), kVT, 0, st>>>(f, L, nx, ny, nz, hd, 0);
  k_bc_cell<<<dim3((ny + 2 * hd + kVT - 1) / kVT, nz + 2 * hd), kVT, 0, st>>>(f, L, nx, ny, nz, hd, 1);
  k_bc_cell<<<dim3((nx + 2 * hd + kVT - 1) / kVT, ny + 2 * hd), kVT, 0, st>>>(f, L, nx, ny, nz, hd, 2);
}

// One smoothing pass (cellToVertex then vertexToCell) for halo 1, in
// separable form.  Both interpolations are products of 1-D linear weights
// (w = X*Y*Z / (hx*hy*hz)), so a pass is, per direction, the 3-point stencil
//   out(i) = m(i) in(i-1) + z(i) in(i) + p(i) in(i+1)
// with m, z, p from the distance tables (VofSep, built on the host), applied
// in z, then y, then x: 9 FMAs per cell instead of the 16 products and 2
// divisions per vertex and cell of the direct form (same operator; rounding
// differs in the last bits).  A CTA owns a kMX x kMY tile of (i, j) columns
// and marches up a chunk of kMKC planes: the input planes k-1, k, k+1 (with
// their in-plane halo) sit in a ring of eight shared-memory slots, planes
// k+2..k+4 in flight by cp.async (one commit group per plane, three planes
// of prefetch cover the DRAM latency of the short per-plane steps) while plane
// k is combined in z, then y, then x.  Each input plane is read once per chunk
// (the halo rows and columns add a third).
// The boundary update that follows a pass in the reference (y walls, then x,
// then z halos over the extended ranges) leaves each ghost cell equal to the
// interior cell reached by mapping every coordinate independently (x: 0 -> nx,
// nx+1 -> 1; y: 0 -> 1, ny+1 -> ny; z: 0 -> nz, nz+1 -> 1), so each cell also
// writes the ghost cells that copy it.  PROPS: the final pass, which also
// writes rho and mu (VOF.f90:220-221) at the cell and its ghost images.
// zimg = 0 (a slab of a z-split channel): no z ghost images, the neighbours'
// planes arrive by the caller's exchange between the passes.
constexpr int kMX = 32, kMY = 8, kMKC = 32, kMT2 = kMX * kMY;

template <bool PROPS>
__global__ void __launch_bounds__(kMT2, 4) k_smooth_march(VofSep w, const double *__restrict__ in,
                                                       double *__restrict__ out, double *__restrict__ rho,
                                                       double *__restrict__ mu, Lay L, int nx, int ny, int nz,
                                                       double rhol, double rhog, double mul, double mug, int zimg) {
  constexpr int CX = kMX + 2, CY = kMY + 2, NP = CX * CY, NY = kMY * CX;
  static_assert(NP <= 2 * kMT2 && NY <= 2 * kMT2, "two elements per thread");
  __shared__ double ring[8][NP];     // input planes, slot = plane & 7
  __shared__ double c1[NP];          // after z
  __shared__ double c2[kMY][CX];     // after y
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kMX + tx;
  const int i0 = blockIdx.x * kMX + 1, j0 = blockIdx.y * kMY + 1;
  const int kb = blockIdx.z * kMKC + 1, ke = min(kb + kMKC - 1, nz);
  // everything that does not change up the march, once: the thread's (up to)
  // two tile elements with their plane-0 offsets, its y-pass elements with
  // their weights, its x weights and output offset
  long src[2];
  bool ld[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = tid + q * kMT2, cx = e % CX, cy = e / CX;
    const int gi = i0 - 1 + cx, gj = j0 - 1 + cy;
    ld[q] = e < NP && gi <= nx + 1 && gj <= ny + 1;
    src[q] = ld[q] ? at(L, gi, gj, 0) : 0;
  }
  int ye[2];
  double ywm[2], yw0[2], ywp[2];
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int e = tid + q * kMT2, cx = e % CX, oy = e / CX;
    ye[q] = e < NY ? oy * CX + cx : -1;
    const int jj = min(j0 + min(oy, kMY - 1), ny) - 1;
    ywm[q] = w.ym[jj];
    yw0[q] = w.y0[jj];
    ywp[q] = w.yp[jj];
  }
  const int i = i0 + tx, j = j0 + ty;
  const bool in_tile = i <= nx && j <= ny;
  const int ic = min(i, nx) - 1;
  const double xwm = w.xm[ic], xw0 = w.x0[ic], xwp = w.xp[ic];
  const long oij = at(L, min(i, nx), min(j, ny), 0);
  const int xs1 = i == nx ? 0 : (i == 1 ? nx + 1 : -1), ys1 = j == 1 ? 0 : (j == ny ? ny + 1 : -1);
  auto load = [&](int kp) {  // plane kp of 0..nz+1
    double *dst = ring[kp & 7];
    const long ko = (long)kp * L.sk;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int e = tid + q * kMT2;
      if (ld[q]) cp_async8(dst + e, in + src[q] + ko);
      else if (e < NP) dst[e] = 0.0;
    }
  };
  // groups: {kb-1, kb, kb+1}, {kb+2}, {kb+3}; then one per step (possibly empty)
  load(kb - 1);
  load(kb);
  load(kb + 1);
  cp_async_commit();
  if (kb + 2 <= ke + 1) load(kb + 2);
  cp_async_commit();
  if (kb + 3 <= ke + 1) load(kb + 3);
  cp_async_commit();
  cp_async_wait_group<2>();
  __syncthreads();
  for (int k = kb; k <= ke; ++k) {
    // plane k+4 into the slot of plane k-4, read four steps ago
    if (k + 4 <= ke + 1) load(k + 4);
    cp_async_commit();
    {
      const double zm = w.zm[k - 1], z0 = w.z0[k - 1], zp = w.zp[k - 1];
      const double *pm = ring[(k - 1) & 7], *p0 = ring[k & 7], *pp = ring[(k + 1) & 7];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int e = tid + q * kMT2;
        if (e < NP) c1[e] = zm * pm[e] + z0 * p0[e] + zp * pp[e];
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int e = ye[q];
      if (e >= 0) (&c2[0][0])[e] = ywm[q] * c1[e] + yw0[q] * c1[e + CX] + ywp[q] * c1[e + 2 * CX];
    }
    __syncthreads();
    if (in_tile) {
      const double c = xwm * c2[ty][tx] + xw0 * c2[ty][tx + 1] + xwp * c2[ty][tx + 2];
      const double m = mug * c + (1.0 - c) * mul, r = rhog * c + (1.0 - c) * rhol;
      const int zs1 = !zimg ? -1 : (k == nz ? 0 : (k == 1 ? nz + 1 : -1));
      if (xs1 < 0 && ys1 < 0 && zs1 < 0) {
        const long o = oij + (long)k * L.sk;
        out[o] = c;
        if constexpr (PROPS) {
          mu[o] = m;
          rho[o] = r;
        }
      } else {
        // the cell and the ghost cells equal to it
        const int xs[2] = {i, xs1}, ys[2] = {j, ys1}, zs[2] = {k, zs1};
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int d = 0; d < 2; ++d) {
              if (xs[a] < 0 || ys[b] < 0 || zs[d] < 0) continue;
              const long o = at(L, xs[a], ys[b], zs[d]);
              out[o] = c;
              if constexpr (PROPS) {
                mu[o] = m;
                rho[o] = r;
              }
            }
      }
    }
    cp_async_wait_group<2>();  // plane k+2 has landed (k+3, k+4 may be in flight)
    __syncthreads();
  }
  cp_async_wait_all();
}

}  // namespace

// Halo-1 fields (the reference's c, cs, rho, mu): two fused passes, the first
// into the scratch tmp (laid out like the fields), the second into cs with
// rho and mu.
void launch_material_props_fused(const VofSep &w, const double *c, double *cs, double *rho, double *mu, double *tmp,
                                 Lay L, int nx, int ny, int nz, double rhol, double rhog, double mul, double mug,
                                 cudaStream_t st) {
  const dim3 grid((nx + kMX - 1) / kMX, (ny + kMY - 1) / kMY, (nz + kMKC - 1) / kMKC), blk(kMX, kMY);
  k_smooth_march<false><<<grid, blk, 0, st>>>(w, c, tmp, nullptr, nullptr, L, nx, ny, nz, 0.0, 0.0, 0.0, 0.0, 1);
  k_smooth_march<true><<<grid, blk, 0, st>>>(w, tmp, cs, rho, mu, L, nx, ny, nz, rhol, rhog, mul, mug, 1);
}

void launch_smooth_pass(const VofSep &w, const double *in, double *out, double *rho, double *mu, Lay L, int nx, int ny,
                        int nz, double rhol, double rhog, double mul, double mug, bool zimg, cudaStream_t st) {
  const dim3 grid((nx + kMX - 1) / kMX, (ny + kMY - 1) / kMY, (nz + kMKC - 1) / kMKC), blk(kMX, kMY);
  if (rho)
    k_smooth_march<true><<<grid, blk, 0, st>>>(w, in, out, rho, mu, L, nx, ny, nz, rhol, rhog, mul, mug, zimg);
  else
    k_smooth_march<false><<<grid, blk, 0, st>>>(w, in, out, nullptr, nullptr, L, nx, ny, nz, 0.0, 0.0, 0.0, 0.0, zimg);
}

void launch_material_props(const VofTab &t, const double *c, double *cs, double *rho, double *mu, double *qv, Lay L,
                           long n, int nx, int ny, int nz, int hd, double rhol, double rhog, double mul, double mug,
                           cudaStream_t st) {
  const dim3 gv((nx + 1 + kVT - 1) / kVT, ny + 1, nz + 1), gc((nx + kVT - 1) / kVT, ny, nz);
  k_cell_to_vertex<<<gv, kVT, 0, st>>>(t, c, L, qv, nx, ny, nz);
  k_vertex_to_cell<<<gc, kVT, 0, st>>>(t, qv, cs, L, nx, ny);
  bc_cell(cs, L, nx, ny, nz, hd, st);
  k_cell_to_vertex<<<gv, kVT, 0, st>>>(t, cs, L, qv, nx, ny, nz);
  k_vertex_to_cell<<<gc, kVT, 0, st>>>(t, qv, cs, L, nx, ny);
  bc_cell(cs, L, nx, ny, nz, hd, st);
  long blocks = (n + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_props<<<(unsigned)blocks, 256, 0, st>>>(cs, rho, mu, n, rhol, rhog, mul, mug);
}

}  // namespace tbfp
