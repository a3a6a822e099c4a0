// Momentum predictor: solveMomentumEqn FAST (momentumEqn.f90:161-194) without
// its closing updateBoundariesV (the caller's halo refresh, as for the
// projection).  Kernel 1, updateConveDiff (:198-607): the convection (flux
// limited, compute_limiters :611-734) and diffusion (variable viscosity, with
// the transposed stress terms) of each velocity component on its equation
// box (setEqnBounds :1134-1190: ux i = 0..nx, uy j = 1..ny-1, uz k = 0..nz),
// into the flux arrays.  Kernel 2, addConvDiff (:738-791) and addSource
// (:874-973): u += dt*(gamma*phi + xi*phi_prev), then the surface-tension,
// forcing and body-force sources.  Every expression follows the reference's
// operand order; metrics are the reference's spacings (x and z extended
// periodically over one ghost).
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"

namespace tbfp {

namespace {

constexpr int kMT = 128;

__device__ __forceinline__ double approx_zero(double d) { return d == 0.0 ? 1e-50 : d; }

__device__ __forceinline__ double superbee(double r) {
  r = fmax(0.0, r);
  return fmax(fmax(0.0, fmin(2.0 * r, 1.0)), fmin(r, 2.0));
}

// compute_limiters (momentumEqn.f90:611-663); psi = {hpup, hpum, hmup, hmum}
__device__ __forceinline__ void limiters(double vc, double vm, double vp, double vpp, double vmm, double cxp,
                                         double cxm, double cyp, double cym, double czp, double czm, int scheme,
                                         double psi[4]) {
  if (scheme == 0 || scheme == 1) {
    const double v = scheme == 0 ? 1.0 : 0.0;
    psi[0] = psi[1] = psi[2] = psi[3] = v;
    return;
  }
  double r[4];
  r[0] = (vc - vm) / approx_zero(vp - vc);
  r[1] = (vpp - vp) / approx_zero(vp - vc);
  r[2] = (vm - vmm) / approx_zero(vc - vm);
  r[3] = (vp - vc) / approx_zero(vc - vm);
  bool sharp = true;
  if (scheme == 5) {
    const double small = 2.220446049250313e-16;  // epsilon(0.d0)
    sharp = (cxp - cxm) > small || (cyp - cym) > small || (czp - czm) > small;
  }
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const double x = r[e];
    if (scheme == 2) psi[e] = (x + 3.0) / 4.0;
    else if (scheme == 3) {
      const double y = fmax(0.0, x);
      psi[e] = (y + fabs(y)) / (1.0 + fabs(y));
    } else if (scheme == 4) psi[e] = superbee(x);
    else psi[e] = sharp ? superbee(x) : 1.0;
  }
}

// F = max(q,0)*A + min(q,0)*B (momentumEqn.f90:247-256 and the like)
__device__ __forceinline__ double flux(double q, double a, double b, double pu, double pm) {
  const double A = a + 0.5 * pu * (b - a);
  const double B = b + 0.5 * pm * (a - b);
  return fmax(q, 0.0) * A + fmin(q, 0.0) * B;
}

struct MomArgs {
  const double *ux, *uy, *uz, *c, *mu, *rho;
  Lay Lux, Luy, Luz, Lc;  // c, mu, rho share Lc
  // spacings, Fortran index -> table[index] (x, z: 0..n+1; y: dyf 1..ny at [j], dyc 1..ny+1 at [j])
  const double *dxf, *dxc, *dyf, *dyc, *dzf, *dzc;
  double *phx, *phy, *phz;  // fluxes, dense over the equation boxes
  int nx, ny, nz, scheme;
};

__device__ __forceinline__ long box_x(const MomArgs &a, int i, int j, int k) {
  return ((long)(k - 1) * a.ny + (j - 1)) * (a.nx + 1) + i;
}
__device__ __forceinline__ long box_y(const MomArgs &a, int i, int j, int k) {
  return ((long)(k - 1) * (a.ny - 1) + (j - 1)) * a.nx + (i - 1);
}
__device__ __forceinline__ long box_z(const MomArgs &a, int i, int j, int k) {
  return ((long)k * a.ny + (j - 1)) * a.nx + (i - 1);
}

// updateConveDiff, x component at face (i, j, k) (momentumEqn.f90:228-341)
__device__ double phi_x(const MomArgs &a, int i, int j, int k) {
  const double *U = a.ux, *V = a.uy, *W = a.uz, *C = a.c, *M = a.mu, *R = a.rho;
  auto u = [&](int di, int dj, int dk) { return U[at(a.Lux, i + di, j + dj, k + dk)]; };
  auto v = [&](int di, int dj, int dk) { return V[at(a.Luy, i + di, j + dj, k + dk)]; };
  auto w = [&](int di, int dj, int dk) { return W[at(a.Luz, i + di, j + dj, k + dk)]; };
  auto c = [&](int di, int dj, int dk) { return C[at(a.Lc, i + di, j + dj, k + dk)]; };
  auto m = [&](int di, int dj, int dk) { return M[at(a.Lc, i + di, j + dj, k + dk)]; };
  const double cxp = c(1, 0, 0), cxm = c(0, 0, 0), cyp = c(0, 1, 0), cym = c(0, -1, 0), czp = c(0, 0, 1),
               czm = c(0, 0, -1);
  const double uc = u(0, 0, 0);
  double phi = 0.0, ps[4], qp, qm;
  // d(uu)/dx
  limiters(uc, u(-1, 0, 0), u(1, 0, 0), u(2, 0, 0), u(-2, 0, 0), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (uc + u(1, 0, 0));
  qm = 0.5 * (uc + u(-1, 0, 0));
  phi = phi - (flux(qp, uc, u(1, 0, 0), ps[0], ps[1]) - flux(qm, u(-1, 0, 0), uc, ps[2], ps[3])) / a.dxc[i + 1];
  // d(vu)/dy
  limiters(uc, u(0, -1, 0), u(0, 1, 0), u(0, 2, 0), u(0, -2, 0), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (v(1, 0, 0) + v(0, 0, 0));
  qm = 0.5 * (v(1, -1, 0) + v(0, -1, 0));
  phi = phi - (flux(qp, uc, u(0, 1, 0), ps[0], ps[1]) - flux(qm, u(0, -1, 0), uc, ps[2], ps[3])) / a.dyf[j];
  // d(wu)/dz
  limiters(uc, u(0, 0, -1), u(0, 0, 1), u(0, 0, 2), u(0, 0, -2), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (w(0, 0, 0) + w(1, 0, 0));
  qm = 0.5 * (w(0, 0, -1) + w(1, 0, -1));
  phi = phi - (flux(qp, uc, u(0, 0, 1), ps[0], ps[1]) - flux(qm, u(0, 0, -1), uc, ps[2], ps[3])) / a.dzf[k];
  // diffusion
  double mur = m(1, 0, 0), mul = m(0, 0, 0);
  const double dxx =
      (mur * (u(1, 0, 0) - uc) / a.dxf[i + 1] - mul * (uc - u(-1, 0, 0)) / a.dxf[i]) / a.dxc[i + 1];
  const double dxxt = dxx;
  mur = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 1, 0) + m(0, 1, 0));
  mul = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, -1, 0) + m(0, -1, 0));
  const double dyy = (mur * (u(0, 1, 0) - uc) / a.dyc[j + 1] - mul * (uc - u(0, -1, 0)) / a.dyc[j]) / a.dyf[j];
  const double dyyt =
      (mur * (v(1, 0, 0) - v(0, 0, 0)) / a.dxc[i + 1] - mul * (v(1, -1, 0) - v(0, -1, 0)) / a.dxc[i + 1]) / a.dyf[j];
  mur = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 0, 1) + m(0, 0, 1));
  mul = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 0, -1) + m(0, 0, -1));
  const double dzz = (mur * (u(0, 0, 1) - uc) / a.dzc[k + 1] - mul * (uc - u(0, 0, -1)) / a.dzc[k]) / a.dzf[k];
  const double dzzt =
      (mur * (w(1, 0, 0) - w(0, 0, 0)) / a.dxc[i + 1] - mul * (w(1, 0, -1) - w(0, 0, -1)) / a.dxc[i + 1]) / a.dzf[k];
  const double invrho = 0.5 * (1.0 / R[at(a.Lc, i + 1, j, k)] + 1.0 / R[at(a.Lc, i, j, k)]);
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}

// y component at face (i, j, k) (momentumEqn.f90:344-467)
__device__ double phi_y(const MomArgs &a, int i, int j, int k) {
  const double *U = a.ux, *V = a.uy, *W = a.uz, *C = a.c, *M = a.mu, *R = a.rho;
  auto u = [&](int di, int dj, int dk) { return U[at(a.Lux, i + di, j + dj, k + dk)]; };
  auto v = [&](int di, int dj, int dk) { return V[at(a.Luy, i + di, j + dj, k + dk)]; };
  auto w = [&](int di, int dj, int dk) { return W[at(a.Luz, i + di, j + dj, k + dk)]; };
  auto c = [&](int di, int dj, int dk) { return C[at(a.Lc, i + di, j + dj, k + dk)]; };
  auto m = [&](int di, int dj, int dk) { return M[at(a.Lc, i + di, j + dj, k + dk)]; };
  const double cxp = c(1, 0, 0), cxm = c(-1, 0, 0), cyp = c(0, 1, 0), cym = c(0, 0, 0), czp = c(0, 0, 1),
               czm = c(0, 0, -1);
  const double vc = v(0, 0, 0);
  const double dyfj = a.dyf[j], dyfp = a.dyf[j + 1], dycp = a.dyc[j + 1];
  double phi = 0.0, ps[4], qp, qm;
  // d(uv)/dx
  limiters(vc, v(-1, 0, 0), v(1, 0, 0), v(2, 0, 0), v(-2, 0, 0), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (u(0, 1, 0) * dyfp + u(0, 0, 0) * dyfj) / dycp;
  qm = 0.5 * (u(-1, 1, 0) * dyfp + u(-1, 0, 0) * dyfj) / dycp;
  phi = phi - (flux(qp, vc, v(1, 0, 0), ps[0], ps[1]) - flux(qm, v(-1, 0, 0), vc, ps[2], ps[3])) / a.dxf[i];
  // d(vv)/dy
  limiters(vc, v(0, -1, 0), v(0, 1, 0), v(0, 2, 0), v(0, -2, 0), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (vc + v(0, 1, 0));
  qm = 0.5 * (vc + v(0, -1, 0));
  phi = phi - (flux(qp, vc, v(0, 1, 0), ps[0], ps[1]) - flux(qm, v(0, -1, 0), vc, ps[2], ps[3])) / dycp;
  // d(wv)/dz
  limiters(vc, v(0, 0, -1), v(0, 0, 1), v(0, 0, 2), v(0, 0, -2), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (w(0, 1, 0) * dyfp + w(0, 0, 0) * dyfj) / dycp;
  qm = 0.5 * (w(0, 1, -1) * dyfp + w(0, 0, -1) * dyfj) / dycp;
  phi = phi - (flux(qp, vc, v(0, 0, 1), ps[0], ps[1]) - flux(qm, v(0, 0, -1), vc, ps[2], ps[3])) / a.dzf[k];
  // diffusion
  double mur = 0.25 * (m(0, 0, 0) + m(1, 0, 0) + m(0, 1, 0) + m(1, 1, 0));
  double mul = 0.25 * (m(0, 0, 0) + m(-1, 0, 0) + m(0, 1, 0) + m(-1, 1, 0));
  const double dxx = (mur * (v(1, 0, 0) - vc) / a.dxc[i + 1] - mul * (vc - v(-1, 0, 0)) / a.dxc[i]) / a.dxf[i];
  const double dxxt =
      (mur * (u(0, 1, 0) - u(0, 0, 0)) / dycp - mul * (u(-1, 1, 0) - u(-1, 0, 0)) / dycp) / a.dxf[i];
  mur = m(0, 1, 0);
  mul = m(0, 0, 0);
  const double dyy = (mur * (v(0, 1, 0) - vc) / dyfp - mul * (vc - v(0, -1, 0)) / dyfj) / dycp;
  const double dyyt = dyy;
  mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, 1, 0) + m(0, 1, 1));
  mul = 0.25 * (m(0, 0, 0) + m(0, 0, -1) + m(0, 1, 0) + m(0, 1, -1));
  const double dzz = (mur * (v(0, 0, 1) - vc) / a.dzc[k + 1] - mul * (vc - v(0, 0, -1)) / a.dzc[k]) / a.dzf[k];
  const double dzzt =
      (mur * (w(0, 1, 0) - w(0, 0, 0)) / dycp - mul * (w(0, 1, -1) - w(0, 0, -1)) / dycp) / a.dzf[k];
  const double invrho = 0.5 * (1.0 / R[at(a.Lc, i, j + 1, k)] + 1.0 / R[at(a.Lc, i, j, k)]);
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}

// z component at face (i, j, k) (momentumEqn.f90:470-603)
__device__ double phi_z(const MomArgs &a, int i, int j, int k) {
  const double *U = a.ux, *V = a.uy, *W = a.uz, *C = a.c, *M = a.mu, *R = a.rho;
  auto u = [&](int di, int dj, int dk) { return U[at(a.Lux, i + di, j + dj, k + dk)]; };
  auto v = [&](int di, int dj, int dk) { return V[at(a.Luy, i + di, j + dj, k + dk)]; };
  auto w = [&](int di, int dj, int dk) { return W[at(a.Luz, i + di, j + dj, k + dk)]; };
  auto c = [&](int di, int dj, int dk) { return C[at(a.Lc, i + di, j + dj, k + dk)]; };
  auto m = [&](int di, int dj, int dk) { return M[at(a.Lc, i + di, j + dj, k + dk)]; };
  const double cxp = c(1, 0, 0), cxm = c(-1, 0, 0), cyp = c(0, 1, 0), cym = c(0, -1, 0), czp = c(0, 0, 1),
               czm = c(0, 0, 0);
  const double wc = w(0, 0, 0);
  double phi = 0.0, ps[4], qp, qm;
  // d(uw)/dx
  limiters(wc, w(-1, 0, 0), w(1, 0, 0), w(2, 0, 0), w(-2, 0, 0), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (u(0, 0, 0) + u(0, 0, 1));
  qm = 0.5 * (u(-1, 0, 0) + u(-1, 0, 1));
  phi = phi - (flux(qp, wc, w(1, 0, 0), ps[0], ps[1]) - flux(qm, w(-1, 0, 0), wc, ps[2], ps[3])) / a.dxf[i];
  // d(vw)/dy
  limiters(wc, w(0, -1, 0), w(0, 1, 0), w(0, 2, 0), w(0, -2, 0), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (v(0, 0, 0) + v(0, 0, 1));
  qm = 0.5 * (v(0, -1, 0) + v(0, -1, 1));
  phi = phi - (flux(qp, wc, w(0, 1, 0), ps[0], ps[1]) - flux(qm, w(0, -1, 0), wc, ps[2], ps[3])) / a.dyf[j];
  // d(ww)/dz
  limiters(wc, w(0, 0, -1), w(0, 0, 1), w(0, 0, 2), w(0, 0, -2), cxp, cxm, cyp, cym, czp, czm, a.scheme, ps);
  qp = 0.5 * (wc + w(0, 0, 1));
  qm = 0.5 * (wc + w(0, 0, -1));
  phi = phi - (flux(qp, wc, w(0, 0, 1), ps[0], ps[1]) - flux(qm, w(0, 0, -1), wc, ps[2], ps[3])) / a.dzc[k + 1];
  // diffusion
  double mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(1, 0, 0) + m(1, 0, 1));
  double mul = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(-1, 0, 0) + m(-1, 0, 1));
  const double dxx = (mur * (w(1, 0, 0) - wc) / a.dxc[i + 1] - mul * (wc - w(-1, 0, 0)) / a.dxc[i]) / a.dxf[i];
  const double dxxt =
      (mur * (u(0, 0, 1) - u(0, 0, 0)) / a.dzc[k + 1] - mul * (u(-1, 0, 1) - u(-1, 0, 0)) / a.dzc[k + 1]) / a.dxf[i];
  mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, 1, 0) + m(0, 1, 1));
  mul = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, -1, 0) + m(0, -1, 1));
  const double dyy = (mur * (w(0, 1, 0) - wc) / a.dyc[j + 1] - mul * (wc - w(0, -1, 0)) / a.dyc[j]) / a.dyf[j];
  const double dyyt =
      (mur * (v(0, 0, 1) - v(0, 0, 0)) / a.dzc[k + 1] - mul * (v(0, -1, 1) - v(0, -1, 0)) / a.dzc[k + 1]) / a.dyf[j];
  mur = m(0, 0, 1);
  mul = m(0, 0, 0);
  const double dzz = (mur * (w(0, 0, 1) - wc) / a.dzf[k + 1] - mul * (wc - w(0, 0, -1)) / a.dzf[k]) / a.dzc[k + 1];
  const double dzzt = dzz;
  const double invrho = 0.5 * (1.0 / R[at(a.Lc, i, j, k + 1)] + 1.0 / R[at(a.Lc, i, j, k)]);
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}

// grid over i = 0..nx, j = 1..ny, k = 0..nz; each thread the components whose box holds it
__global__ void __launch_bounds__(kMT) k_momentum_fluxes(MomArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y + 1, k = blockIdx.z;
  if (i > a.nx) return;
  if (k >= 1) a.phx[box_x(a, i, j, k)] = phi_x(a, i, j, k);
  if (i >= 1 && k >= 1 && j <= a.ny - 1) a.phy[box_y(a, i, j, k)] = phi_y(a, i, j, k);
  if (i >= 1) a.phz[box_z(a, i, j, k)] = phi_z(a, i, j, k);
}

struct MomUpd {
  double *ux, *uy, *uz;
  const double *rho, *stx, *sty, *stz;
  Lay Lux, Luy, Luz, Lc, Lsx, Lsy, Lsz;
  const double *phx, *phy, *phz, *ppx, *ppy, *ppz;
  double dt, gamma, xi, r, invrho0, fs, gch, g;
  int nx, ny, nz;
};

// addConvDiff then addSource (FAST), element by element in the reference's order
__global__ void __launch_bounds__(kMT) k_momentum_update(MomUpd a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y + 1, k = blockIdx.z;
  if (i > a.nx) return;
  MomArgs b;
  b.nx = a.nx;
  b.ny = a.ny;
  if (k >= 1) {
    const long o = at(a.Lux, i, j, k), q = box_x(b, i, j, k);
    double u = a.ux[o] + a.dt * (a.gamma * a.phx[q] + a.xi * a.ppx[q]);
    const double invrho = 0.5 * (1.0 / a.rho[at(a.Lc, i + 1, j, k)] + 1.0 / a.rho[at(a.Lc, i, j, k)]);
    const double st = a.stx ? a.stx[at(a.Lsx, i, j, k)] : 0.0;
    a.ux[o] = u + a.invrho0 * a.r * st + invrho * a.r * a.fs + a.r * a.gch;
  }
  if (i >= 1 && k >= 1 && j <= a.ny - 1) {
    const long o = at(a.Luy, i, j, k), q = box_y(b, i, j, k);
    double u = a.uy[o] + a.dt * (a.gamma * a.phy[q] + a.xi * a.ppy[q]);
    const double st = a.sty ? a.sty[at(a.Lsy, i, j, k)] : 0.0;
    a.uy[o] = u + a.invrho0 * a.r * st + a.r * a.g;
  }
  if (i >= 1) {
    const long o = at(a.Luz, i, j, k), q = box_z(b, i, j, k);
    double u = a.uz[o] + a.dt * (a.gamma * a.phz[q] + a.xi * a.ppz[q]);
    const double st = a.stz ? a.stz[at(a.Lsz, i, j, k)] : 0.0;
    a.uz[o] = u + a.invrho0 * a.r * st;
  }
}

}  // namespace

void launch_momentum(const MomentumTabs &t, double *ux, double *uy, double *uz, const double *c, const double *mu,
                     const double *rho, const double *const *st, Lay Lux, Lay Luy, Lay Luz, Lay Lc, const Lay *Lst,
                     double *const phi[3], const double *const prev[3], int nx, int ny, int nz, int scheme, double dt,
                     double alpha, double gamma, double xi, double rho0, double fs, double gch, double g,
                     cudaStream_t st_) {
  MomArgs a{};
  a.ux = ux;
  a.uy = uy;
  a.uz = uz;
  a.c = c;
  a.mu = mu;
  a.rho = rho;
  a.Lux = Lux;
  a.Luy = Luy;
  a.Luz = Luz;
  a.Lc = Lc;
  a.dxf = t.dxf;
  a.dxc = t.dxc;
  a.dyf = t.dyf;
  a.dyc = t.dyc;
  a.dzf = t.dzf;
  a.dzc = t.dzc;
  a.phx = phi[0];
  a.phy = phi[1];
  a.phz = phi[2];
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.scheme = scheme;
  const dim3 grid((nx + 1 + kMT - 1) / kMT, ny, nz + 1);
  k_momentum_fluxes<<<grid, kMT, 0, st_>>>(a);
  MomUpd b{};
  b.ux = ux;
  b.uy = uy;
  b.uz = uz;
  b.rho = rho;
  b.stx = st ? st[0] : nullptr;
  b.sty = st ? st[1] : nullptr;
  b.stz = st ? st[2] : nullptr;
  b.Lux = Lux;
  b.Luy = Luy;
  b.Luz = Luz;
  b.Lc = Lc;
  if (st) {
    b.Lsx = Lst[0];
    b.Lsy = Lst[1];
    b.Lsz = Lst[2];
  }
  b.phx = phi[0];
  b.phy = phi[1];
  b.phz = phi[2];
  b.ppx = prev[0];
  b.ppy = prev[1];
  b.ppz = prev[2];
  b.dt = dt;
  b.gamma = gamma;
  b.xi = xi;
  b.r = dt * alpha;
  b.invrho0 = 1.0 / rho0;
  b.fs = fs;
  b.gch = gch;
  b.g = g;
  b.nx = nx;
  b.ny = ny;
  b.nz = nz;
  k_momentum_update<<<grid, kMT, 0, st_>>>(b);
}

}  // namespace tbfp
