// Momentum predictor: solveMomentumEqn FAST (momentumEqn.f90:161-194) without
// its closing updateBoundariesV (the caller's halo refresh, as for the
// projection).  Kernel 1, updateConveDiff (:198-607): the convection (flux
// limited, compute_limiters :611-734) and diffusion (variable viscosity, with
// the transposed stress terms) of each velocity component on its equation
// box (setEqnBounds :1134-1190: ux i = 0..nx, uy j = 1..ny-1, uz k = 0..nz),
// into the flux arrays.  Kernel 2, addConvDiff (:738-791) and addSource
// (:874-973): u += dt*(gamma*phi + xi*phi_prev), then the surface-tension,
// forcing and body-force sources.  Every expression follows the reference's
// operand order, with one substitution: a quotient by a grid spacing is a
// product with the spacing's reciprocal (tables built once on the host, each
// the correctly rounded 1/d), and the four limiter ratios of one direction
// share the reciprocals of their two denominators.  Each such term then
// differs from the reference's quotient by at most an ulp or two, and FP64
// divisions -- 96 per cell in the literal form, the kernel's whole cost --
// drop to 24 reciprocals.  The kernel is specialised per convection scheme.
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

// compute_limiters (momentumEqn.f90:611-663); psi = {hpup, hpum, hmup, hmum}.
// sharp: the localVF test of the cell (dc > epsilon(0.d0) in any direction)
template <int S>
__device__ __forceinline__ void limiters(double vc, double vm, double vp, double vpp, double vmm, bool sharp,
                                         double psi[4]) {
  if constexpr (S == 0 || S == 1) {
    psi[0] = psi[1] = psi[2] = psi[3] = S == 0 ? 1.0 : 0.0;
    return;
  }
  if (S == 5 && !sharp) {
    psi[0] = psi[1] = psi[2] = psi[3] = 1.0;
    return;
  }
  const double ip = 1.0 / approx_zero(vp - vc), im = 1.0 / approx_zero(vc - vm);
  const double r[4] = {(vc - vm) * ip, (vpp - vp) * ip, (vm - vmm) * im, (vp - vc) * im};
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const double x = r[e];
    if constexpr (S == 2) psi[e] = (x + 3.0) * 0.25;  // (r+3)/4, exact as a product
    else if constexpr (S == 3) {
      const double y = fmax(0.0, x);
      psi[e] = (y + fabs(y)) / (1.0 + fabs(y));
    } else psi[e] = superbee(x);
  }
}

template <int S>
__device__ __forceinline__ bool sharp_cell(double cxp, double cxm, double cyp, double cym, double czp, double czm) {
  if constexpr (S != 5) return true;
  const double small = 2.220446049250313e-16;  // epsilon(0.d0)
  return (cxp - cxm) > small || (cyp - cym) > small || (czp - czm) > small;
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
  // spacings and their reciprocals, Fortran index 0..n+1 -> table[index]
  const double *dyf, *rdxf, *rdxc, *rdyf, *rdyc, *rdzf, *rdzc;
  double *phx, *phy, *phz;  // fluxes, dense over the equation boxes
  int nx, ny, nz;
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

// Each field is read through a pointer to the thread's own element and 32-bit
// strides: a neighbour costs one address computation per distinct (dj, dk)
// and a load with an immediate i offset.  c, mu and rho share one layout.
#define TBFP_MOM_ACCESSORS                                                                    \
  const double *__restrict__ pU = a.ux + at(a.Lux, i, j, k);                                  \
  const double *__restrict__ pV = a.uy + at(a.Luy, i, j, k);                                  \
  const double *__restrict__ pW = a.uz + at(a.Luz, i, j, k);                                  \
  const long oc = at(a.Lc, i, j, k);                                                          \
  const double *__restrict__ pC = a.c + oc;                                                   \
  const double *__restrict__ pM = a.mu + oc;                                                  \
  const double *__restrict__ pR = a.rho + oc;                                                 \
  const int uj = (int)a.Lux.sj, uk = (int)a.Lux.sk, vj = (int)a.Luy.sj, vk = (int)a.Luy.sk;   \
  const int wj = (int)a.Luz.sj, wk = (int)a.Luz.sk, cj = (int)a.Lc.sj, ck = (int)a.Lc.sk;     \
  auto u = [&](int di, int dj, int dk) { return __ldg(pU + (di + dj * uj + dk * uk)); };       \
  auto v = [&](int di, int dj, int dk) { return __ldg(pV + (di + dj * vj + dk * vk)); };       \
  auto w = [&](int di, int dj, int dk) { return __ldg(pW + (di + dj * wj + dk * wk)); };       \
  auto c = [&](int di, int dj, int dk) { return __ldg(pC + (di + dj * cj + dk * ck)); };       \
  auto m = [&](int di, int dj, int dk) { return __ldg(pM + (di + dj * cj + dk * ck)); };       \
  auto rho = [&](int di, int dj, int dk) { return __ldg(pR + (di + dj * cj + dk * ck)); };     \
  (void)c

// updateConveDiff, x component at face (i, j, k) (momentumEqn.f90:228-341)
template <int S>
__device__ double phi_x(const MomArgs &a, int i, int j, int k) {
  TBFP_MOM_ACCESSORS;
  const bool sh = sharp_cell<S>(c(1, 0, 0), c(0, 0, 0), c(0, 1, 0), c(0, -1, 0), c(0, 0, 1), c(0, 0, -1));
  const double uc = u(0, 0, 0);
  const double rxc = a.rdxc[i + 1], ryf = a.rdyf[j], rzf = a.rdzf[k];
  double phi = 0.0, ps[4], qp, qm;
  // d(uu)/dx
  limiters<S>(uc, u(-1, 0, 0), u(1, 0, 0), u(2, 0, 0), u(-2, 0, 0), sh, ps);
  qp = 0.5 * (uc + u(1, 0, 0));
  qm = 0.5 * (uc + u(-1, 0, 0));
  phi = phi - (flux(qp, uc, u(1, 0, 0), ps[0], ps[1]) - flux(qm, u(-1, 0, 0), uc, ps[2], ps[3])) * rxc;
  // d(vu)/dy
  limiters<S>(uc, u(0, -1, 0), u(0, 1, 0), u(0, 2, 0), u(0, -2, 0), sh, ps);
  qp = 0.5 * (v(1, 0, 0) + v(0, 0, 0));
  qm = 0.5 * (v(1, -1, 0) + v(0, -1, 0));
  phi = phi - (flux(qp, uc, u(0, 1, 0), ps[0], ps[1]) - flux(qm, u(0, -1, 0), uc, ps[2], ps[3])) * ryf;
  // d(wu)/dz
  limiters<S>(uc, u(0, 0, -1), u(0, 0, 1), u(0, 0, 2), u(0, 0, -2), sh, ps);
  qp = 0.5 * (w(0, 0, 0) + w(1, 0, 0));
  qm = 0.5 * (w(0, 0, -1) + w(1, 0, -1));
  phi = phi - (flux(qp, uc, u(0, 0, 1), ps[0], ps[1]) - flux(qm, u(0, 0, -1), uc, ps[2], ps[3])) * rzf;
  // diffusion
  double mur = m(1, 0, 0), mul = m(0, 0, 0);
  const double dxx = (mur * (u(1, 0, 0) - uc) * a.rdxf[i + 1] - mul * (uc - u(-1, 0, 0)) * a.rdxf[i]) * rxc;
  const double dxxt = dxx;
  mur = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 1, 0) + m(0, 1, 0));
  mul = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, -1, 0) + m(0, -1, 0));
  const double dyy = (mur * (u(0, 1, 0) - uc) * a.rdyc[j + 1] - mul * (uc - u(0, -1, 0)) * a.rdyc[j]) * ryf;
  const double dyyt = (mur * (v(1, 0, 0) - v(0, 0, 0)) * rxc - mul * (v(1, -1, 0) - v(0, -1, 0)) * rxc) * ryf;
  mur = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 0, 1) + m(0, 0, 1));
  mul = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 0, -1) + m(0, 0, -1));
  const double dzz = (mur * (u(0, 0, 1) - uc) * a.rdzc[k + 1] - mul * (uc - u(0, 0, -1)) * a.rdzc[k]) * rzf;
  const double dzzt = (mur * (w(1, 0, 0) - w(0, 0, 0)) * rxc - mul * (w(1, 0, -1) - w(0, 0, -1)) * rxc) * rzf;
  const double invrho = 0.5 * (1.0 / rho(1, 0, 0) + 1.0 / rho(0, 0, 0));
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}

// y component at face (i, j, k) (momentumEqn.f90:344-467)
template <int S>
__device__ double phi_y(const MomArgs &a, int i, int j, int k) {
  TBFP_MOM_ACCESSORS;
  const bool sh = sharp_cell<S>(c(1, 0, 0), c(-1, 0, 0), c(0, 1, 0), c(0, 0, 0), c(0, 0, 1), c(0, 0, -1));
  const double vc = v(0, 0, 0);
  const double dyfj = a.dyf[j], dyfp = a.dyf[j + 1], rycp = a.rdyc[j + 1];
  const double rxf = a.rdxf[i], rzf = a.rdzf[k];
  double phi = 0.0, ps[4], qp, qm;
  // d(uv)/dx
  limiters<S>(vc, v(-1, 0, 0), v(1, 0, 0), v(2, 0, 0), v(-2, 0, 0), sh, ps);
  qp = 0.5 * (u(0, 1, 0) * dyfp + u(0, 0, 0) * dyfj) * rycp;
  qm = 0.5 * (u(-1, 1, 0) * dyfp + u(-1, 0, 0) * dyfj) * rycp;
  phi = phi - (flux(qp, vc, v(1, 0, 0), ps[0], ps[1]) - flux(qm, v(-1, 0, 0), vc, ps[2], ps[3])) * rxf;
  // d(vv)/dy
  limiters<S>(vc, v(0, -1, 0), v(0, 1, 0), v(0, 2, 0), v(0, -2, 0), sh, ps);
  qp = 0.5 * (vc + v(0, 1, 0));
  qm = 0.5 * (vc + v(0, -1, 0));
  phi = phi - (flux(qp, vc, v(0, 1, 0), ps[0], ps[1]) - flux(qm, v(0, -1, 0), vc, ps[2], ps[3])) * rycp;
  // d(wv)/dz
  limiters<S>(vc, v(0, 0, -1), v(0, 0, 1), v(0, 0, 2), v(0, 0, -2), sh, ps);
  qp = 0.5 * (w(0, 1, 0) * dyfp + w(0, 0, 0) * dyfj) * rycp;
  qm = 0.5 * (w(0, 1, -1) * dyfp + w(0, 0, -1) * dyfj) * rycp;
  phi = phi - (flux(qp, vc, v(0, 0, 1), ps[0], ps[1]) - flux(qm, v(0, 0, -1), vc, ps[2], ps[3])) * rzf;
  // diffusion
  double mur = 0.25 * (m(0, 0, 0) + m(1, 0, 0) + m(0, 1, 0) + m(1, 1, 0));
  double mul = 0.25 * (m(0, 0, 0) + m(-1, 0, 0) + m(0, 1, 0) + m(-1, 1, 0));
  const double dxx = (mur * (v(1, 0, 0) - vc) * a.rdxc[i + 1] - mul * (vc - v(-1, 0, 0)) * a.rdxc[i]) * rxf;
  const double dxxt = (mur * (u(0, 1, 0) - u(0, 0, 0)) * rycp - mul * (u(-1, 1, 0) - u(-1, 0, 0)) * rycp) * rxf;
  mur = m(0, 1, 0);
  mul = m(0, 0, 0);
  const double dyy = (mur * (v(0, 1, 0) - vc) * a.rdyf[j + 1] - mul * (vc - v(0, -1, 0)) * a.rdyf[j]) * rycp;
  const double dyyt = dyy;
  mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, 1, 0) + m(0, 1, 1));
  mul = 0.25 * (m(0, 0, 0) + m(0, 0, -1) + m(0, 1, 0) + m(0, 1, -1));
  const double dzz = (mur * (v(0, 0, 1) - vc) * a.rdzc[k + 1] - mul * (vc - v(0, 0, -1)) * a.rdzc[k]) * rzf;
  const double dzzt = (mur * (w(0, 1, 0) - w(0, 0, 0)) * rycp - mul * (w(0, 1, -1) - w(0, 0, -1)) * rycp) * rzf;
  const double invrho = 0.5 * (1.0 / rho(0, 1, 0) + 1.0 / rho(0, 0, 0));
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}

// z component at face (i, j, k) (momentumEqn.f90:470-603)
template <int S>
__device__ double phi_z(const MomArgs &a, int i, int j, int k) {
  TBFP_MOM_ACCESSORS;
  const bool sh = sharp_cell<S>(c(1, 0, 0), c(-1, 0, 0), c(0, 1, 0), c(0, -1, 0), c(0, 0, 1), c(0, 0, 0));
  const double wc = w(0, 0, 0);
  const double rxf = a.rdxf[i], ryf = a.rdyf[j], rzcp = a.rdzc[k + 1];
  double phi = 0.0, ps[4], qp, qm;
  // d(uw)/dx
  limiters<S>(wc, w(-1, 0, 0), w(1, 0, 0), w(2, 0, 0), w(-2, 0, 0), sh, ps);
  qp = 0.5 * (u(0, 0, 0) + u(0, 0, 1));
  qm = 0.5 * (u(-1, 0, 0) + u(-1, 0, 1));
  phi = phi - (flux(qp, wc, w(1, 0, 0), ps[0], ps[1]) - flux(qm, w(-1, 0, 0), wc, ps[2], ps[3])) * rxf;
  // d(vw)/dy
  limiters<S>(wc, w(0, -1, 0), w(0, 1, 0), w(0, 2, 0), w(0, -2, 0), sh, ps);
  qp = 0.5 * (v(0, 0, 0) + v(0, 0, 1));
  qm = 0.5 * (v(0, -1, 0) + v(0, -1, 1));
  phi = phi - (flux(qp, wc, w(0, 1, 0), ps[0], ps[1]) - flux(qm, w(0, -1, 0), wc, ps[2], ps[3])) * ryf;
  // d(ww)/dz
  limiters<S>(wc, w(0, 0, -1), w(0, 0, 1), w(0, 0, 2), w(0, 0, -2), sh, ps);
  qp = 0.5 * (wc + w(0, 0, 1));
  qm = 0.5 * (wc + w(0, 0, -1));
  phi = phi - (flux(qp, wc, w(0, 0, 1), ps[0], ps[1]) - flux(qm, w(0, 0, -1), wc, ps[2], ps[3])) * rzcp;
  // diffusion
  double mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(1, 0, 0) + m(1, 0, 1));
  double mul = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(-1, 0, 0) + m(-1, 0, 1));
  const double dxx = (mur * (w(1, 0, 0) - wc) * a.rdxc[i + 1] - mul * (wc - w(-1, 0, 0)) * a.rdxc[i]) * rxf;
  const double dxxt = (mur * (u(0, 0, 1) - u(0, 0, 0)) * rzcp - mul * (u(-1, 0, 1) - u(-1, 0, 0)) * rzcp) * rxf;
  mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, 1, 0) + m(0, 1, 1));
  mul = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, -1, 0) + m(0, -1, 1));
  const double dyy = (mur * (w(0, 1, 0) - wc) * a.rdyc[j + 1] - mul * (wc - w(0, -1, 0)) * a.rdyc[j]) * ryf;
  const double dyyt = (mur * (v(0, 0, 1) - v(0, 0, 0)) * rzcp - mul * (v(0, -1, 1) - v(0, -1, 0)) * rzcp) * ryf;
  mur = m(0, 0, 1);
  mul = m(0, 0, 0);
  const double dzz = (mur * (w(0, 0, 1) - wc) * a.rdzf[k + 1] - mul * (wc - w(0, 0, -1)) * a.rdzf[k]) * rzcp;
  const double dzzt = dzz;
  const double invrho = 0.5 * (1.0 / rho(0, 0, 1) + 1.0 / rho(0, 0, 0));
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}
#undef TBFP_MOM_ACCESSORS

// grid over i = 1..nx, j = 1..ny, k = 0..nz; each thread the components whose
// box holds it, and the thread at i = nx also the x component's face i = 0
template <int S>
__global__ void __launch_bounds__(kMT) k_momentum_fluxes(MomArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1, k = blockIdx.z;
  if (i > a.nx) return;
  if (k >= 1) {
    a.phx[box_x(a, i, j, k)] = phi_x<S>(a, i, j, k);
    if (i == a.nx) a.phx[box_x(a, 0, j, k)] = phi_x<S>(a, 0, j, k);
    if (j <= a.ny - 1) a.phy[box_y(a, i, j, k)] = phi_y<S>(a, i, j, k);
  }
  a.phz[box_z(a, i, j, k)] = phi_z<S>(a, i, j, k);
}

struct MomUpd {
  double *ux, *uy, *uz;
  const double *rho, *stx, *sty, *stz;
  Lay Lux, Luy, Luz, Lc, Lsx, Lsy, Lsz;
  const double *phx, *phy, *phz, *ppx, *ppy, *ppz;
  double dt, gamma, xi, r, invrho0, fs, gch, g;
  int nx, ny, nz;
};

__device__ __forceinline__ void update_x(const MomUpd &a, const MomArgs &b, int i, int j, int k) {
  const long o = at(a.Lux, i, j, k), q = box_x(b, i, j, k);
  double u = a.ux[o] + a.dt * (a.gamma * a.phx[q] + a.xi * a.ppx[q]);
  const double invrho = 0.5 * (1.0 / a.rho[at(a.Lc, i + 1, j, k)] + 1.0 / a.rho[at(a.Lc, i, j, k)]);
  const double st = a.stx ? a.stx[at(a.Lsx, i, j, k)] : 0.0;
  a.ux[o] = u + a.invrho0 * a.r * st + invrho * a.r * a.fs + a.r * a.gch;
}

// addConvDiff then addSource (FAST), element by element in the reference's
// order; the flux kernel's grid (i = 1..nx, the thread at nx also ux at i = 0)
__global__ void __launch_bounds__(kMT) k_momentum_update(MomUpd a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1, j = blockIdx.y + 1, k = blockIdx.z;
  if (i > a.nx) return;
  MomArgs b;
  b.nx = a.nx;
  b.ny = a.ny;
  if (k >= 1) {
    update_x(a, b, i, j, k);
    if (i == a.nx) update_x(a, b, 0, j, k);
    if (j <= a.ny - 1) {
      const long o = at(a.Luy, i, j, k), q = box_y(b, i, j, k);
      double u = a.uy[o] + a.dt * (a.gamma * a.phy[q] + a.xi * a.ppy[q]);
      const double st = a.sty ? a.sty[at(a.Lsy, i, j, k)] : 0.0;
      a.uy[o] = u + a.invrho0 * a.r * st + a.r * a.g;
    }
  }
  const long o = at(a.Luz, i, j, k), q = box_z(b, i, j, k);
  double u = a.uz[o] + a.dt * (a.gamma * a.phz[q] + a.xi * a.ppz[q]);
  const double st = a.stz ? a.stz[at(a.Lsz, i, j, k)] : 0.0;
  a.uz[o] = u + a.invrho0 * a.r * st;
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
  a.dyf = t.dyf;
  a.rdxf = t.rdxf;
  a.rdxc = t.rdxc;
  a.rdyf = t.rdyf;
  a.rdyc = t.rdyc;
  a.rdzf = t.rdzf;
  a.rdzc = t.rdzc;
  a.phx = phi[0];
  a.phy = phi[1];
  a.phz = phi[2];
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  const dim3 grid((nx + kMT - 1) / kMT, ny, nz + 1);
  switch (scheme) {
    case 0: k_momentum_fluxes<0><<<grid, kMT, 0, st_>>>(a); break;
    case 1: k_momentum_fluxes<1><<<grid, kMT, 0, st_>>>(a); break;
    case 2: k_momentum_fluxes<2><<<grid, kMT, 0, st_>>>(a); break;
    case 3: k_momentum_fluxes<3><<<grid, kMT, 0, st_>>>(a); break;
    case 4: k_momentum_fluxes<4><<<grid, kMT, 0, st_>>>(a); break;
    default: k_momentum_fluxes<5><<<grid, kMT, 0, st_>>>(a); break;
  }
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
