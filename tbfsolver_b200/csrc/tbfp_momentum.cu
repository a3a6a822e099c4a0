// Momentum predictor: solveMomentumEqn FAST (momentumEqn.f90:161-194), and
// its closing updateBoundariesV (vfield.f90:111-189) as a launch of its own.
// The flux kernel, updateConveDiff (:198-607): the convection (flux limited,
// compute_limiters :611-734) and diffusion (variable viscosity, with the
// transposed stress terms) of each velocity component on its equation box
// (setEqnBounds :1134-1190: ux i = 0..nx, uy j = 1..ny-1, uz k = 0..nz), into
// the flux arrays; a tiled kernel that marches up z with the stencil planes in
// shared memory, plus a small launch for the ux faces i = 0.  The update,
// addConvDiff (:738-791) and addSource (:874-973): u += dt*(gamma*phi +
// xi*phi_prev), then the surface-tension, forcing and body-force sources --
// a separate pass over u in place, or inside the flux kernel when u* goes to
// a second buffer.  Every expression follows the reference's operand order,
// with these substitutions: a quotient by a grid spacing is a product with the
// spacing's reciprocal (tables built once on the host, each the correctly
// rounded 1/d); the four limiter ratios of one direction share the
// reciprocals of their two denominators; QUICK's ratio cancels against the
// face difference it multiplies (exact zero differences kept).  Each such term
// differs from the reference's by an ulp or two, and the 96 FP64 divisions per
// cell of the literal form drop to at most 22 reciprocals (4 for QUICK).  The
// kernels are specialised per convection scheme.
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

// Fp - Fm of one direction: the limited flux through the upper face (between
// vc and vp) minus the one through the lower face (between vm and vc)
// (momentumEqn.f90:240-256 and the like).  QUICK's limiter is psi = (r+3)/4
// with r a ratio whose denominator is the face's own difference d, so the
// flux's psi*d/2 is ((numerator) + 3d)/8 without the division; d == 0 keeps
// the reference's value (approx_zero makes psi*d exactly 0 there).
template <int S>
__device__ __forceinline__ double conv_diff(double qp, double qm, double vmm, double vm, double vc, double vp,
                                            double vpp, bool sh) {
  if constexpr (S == 2) {
    const double d = vp - vc, e = vc - vm;
    const double Ap = d == 0.0 ? vc : vc + 0.125 * (e + 3.0 * d);
    const double Bp = d == 0.0 ? vp : vp - 0.125 * ((vpp - vp) + 3.0 * d);
    const double Am = e == 0.0 ? vm : vm + 0.125 * ((vm - vmm) + 3.0 * e);
    const double Bm = e == 0.0 ? vc : vc - 0.125 * (d + 3.0 * e);
    return (fmax(qp, 0.0) * Ap + fmin(qp, 0.0) * Bp) - (fmax(qm, 0.0) * Am + fmin(qm, 0.0) * Bm);
  } else {
    double ps[4];
    limiters<S>(vc, vm, vp, vpp, vmm, sh, ps);
    return flux(qp, vc, vp, ps[0], ps[1]) - flux(qm, vm, vc, ps[2], ps[3]);
  }
}

// the limiter of one ratio (momentumEqn.f90:667-734) for schemes 3 and 4
template <int S>
__device__ __forceinline__ double lim(double x) {
  if constexpr (S == 3) {
    const double y = fmax(0.0, x);
    return (y + fabs(y)) / (1.0 + fabs(y));
  } else {
    return superbee(x);
  }
}

// The limited flux through the face between vc and vp (vm and vpp the next
// values outward), for schemes 0-4, whose limiters depend on the face alone:
// the upper face of one cell is then the lower face of the next bit for bit
// (the lower face's ratios have the same numerators and denominator), so a
// face is computed once.
template <int S>
__device__ __forceinline__ double face_flux(double q, double vm, double vc, double vp, double vpp) {
  if constexpr (S == 2) {
    const double d = vp - vc;
    const double A = d == 0.0 ? vc : vc + 0.125 * ((vc - vm) + 3.0 * d);
    const double B = d == 0.0 ? vp : vp - 0.125 * ((vpp - vp) + 3.0 * d);
    return fmax(q, 0.0) * A + fmin(q, 0.0) * B;
  } else if constexpr (S == 0 || S == 1) {
    const double p = S == 0 ? 1.0 : 0.0;
    return flux(q, vc, vp, p, p);
  } else {
    const double ip = 1.0 / approx_zero(vp - vc);
    return flux(q, vc, vp, lim<S>((vc - vm) * ip), lim<S>((vpp - vp) * ip));
  }
}

struct MomArgs {
  const double *ux, *uy, *uz, *c, *mu, *rho;
  Lay Lux, Luy, Luz, Lc;  // c, mu, rho share Lc
  // spacings and their reciprocals, Fortran index 0..n+1 -> table[index]
  const double *dyf, *rdxf, *rdxc, *rdyf, *rdyc, *rdzf, *rdzc;
  double *phx, *phy, *phz;  // fluxes, dense over the equation boxes
  int nx, ny, nz;
  int hdu, hdc;  // halos of the velocity and cell arrays
  // the out-of-place form's update (addConvDiff + addSource) into uxo, uyo, uzo
  double *uxo, *uyo, *uzo;
  const double *ppx, *ppy, *ppz, *stx, *sty, *stz;
  Lay Lsx, Lsy, Lsz;
  double dt, gamma, xi, r, invrho0, fs, gch, g;
};

// one component's flux into its buffer and, in the out-of-place form, its
// addConvDiff + addSource update from the thread's own u (the expressions of
// k_momentum_update, so both forms give the same values)
template <bool OUT>
__device__ __forceinline__ void emit_x(const MomArgs &a, int i, int j, int k, double phi, double uc, double invrho);
template <bool OUT>
__device__ __forceinline__ void emit_y(const MomArgs &a, int i, int j, int k, double phi, double uc);
template <bool OUT>
__device__ __forceinline__ void emit_z(const MomArgs &a, int i, int j, int k, double phi, double uc);

__device__ __forceinline__ long box_x(const MomArgs &a, int i, int j, int k) {
  return ((long)(k - 1) * a.ny + (j - 1)) * (a.nx + 1) + i;
}
__device__ __forceinline__ long box_y(const MomArgs &a, int i, int j, int k) {
  return ((long)(k - 1) * (a.ny - 1) + (j - 1)) * a.nx + (i - 1);
}
__device__ __forceinline__ long box_z(const MomArgs &a, int i, int j, int k) {
  return ((long)k * a.ny + (j - 1)) * a.nx + (i - 1);
}

template <bool OUT>
__device__ __forceinline__ void emit_x(const MomArgs &a, int i, int j, int k, double phi, double uc, double invrho) {
  const long q = box_x(a, i, j, k);
  a.phx[q] = phi;
  if constexpr (OUT) {
    const double u = uc + a.dt * (a.gamma * phi + a.xi * __ldg(a.ppx + q));
    const double st = a.stx ? __ldg(a.stx + at(a.Lsx, i, j, k)) : 0.0;
    a.uxo[at(a.Lux, i, j, k)] = u + a.invrho0 * a.r * st + invrho * a.r * a.fs + a.r * a.gch;
  }
}
template <bool OUT>
__device__ __forceinline__ void emit_y(const MomArgs &a, int i, int j, int k, double phi, double uc) {
  const long q = box_y(a, i, j, k);
  a.phy[q] = phi;
  if constexpr (OUT) {
    const double u = uc + a.dt * (a.gamma * phi + a.xi * __ldg(a.ppy + q));
    const double st = a.sty ? __ldg(a.sty + at(a.Lsy, i, j, k)) : 0.0;
    a.uyo[at(a.Luy, i, j, k)] = u + a.invrho0 * a.r * st + a.r * a.g;
  }
}
template <bool OUT>
__device__ __forceinline__ void emit_z(const MomArgs &a, int i, int j, int k, double phi, double uc) {
  const long q = box_z(a, i, j, k);
  a.phz[q] = phi;
  if constexpr (OUT) {
    const double u = uc + a.dt * (a.gamma * phi + a.xi * __ldg(a.ppz + q));
    const double st = a.stz ? __ldg(a.stz + at(a.Lsz, i, j, k)) : 0.0;
    a.uzo[at(a.Luz, i, j, k)] = u + a.invrho0 * a.r * st;
  }
}

// Two ways to reach a field's neighbours.  GAcc reads global memory through
// a pointer to the thread's own element and 32-bit strides (one address per
// distinct (dj, dk), an immediate i offset).  SAcc reads the shared-memory
// plane rings of the tiled kernel: the thread's own element of ring slot 0
// plus the offset of the slot holding plane k + dk.  c, mu and rho share one
// layout.
struct GAcc {
  const double *__restrict__ pU;
  const double *__restrict__ pV;
  const double *__restrict__ pW;
  const double *__restrict__ pC;
  const double *__restrict__ pM;
  const double *__restrict__ pR;
  int uj, uk, vj, vk, wj, wk, cj, ck;
  __device__ GAcc(const MomArgs &a, int i, int j, int k)
      : pU(a.ux + at(a.Lux, i, j, k)), pV(a.uy + at(a.Luy, i, j, k)), pW(a.uz + at(a.Luz, i, j, k)),
        pC(a.c + at(a.Lc, i, j, k)), pM(a.mu + at(a.Lc, i, j, k)), pR(a.rho + at(a.Lc, i, j, k)),
        uj((int)a.Lux.sj), uk((int)a.Lux.sk), vj((int)a.Luy.sj), vk((int)a.Luy.sk), wj((int)a.Luz.sj),
        wk((int)a.Luz.sk), cj((int)a.Lc.sj), ck((int)a.Lc.sk) {}
  __device__ double u(int di, int dj, int dk) const { return __ldg(pU + (di + dj * uj + dk * uk)); }
  __device__ double v(int di, int dj, int dk) const { return __ldg(pV + (di + dj * vj + dk * vk)); }
  __device__ double w(int di, int dj, int dk) const { return __ldg(pW + (di + dj * wj + dk * wk)); }
  __device__ double c(int di, int dj, int dk) const { return __ldg(pC + (di + dj * cj + dk * ck)); }
  __device__ double m(int di, int dj, int dk) const { return __ldg(pM + (di + dj * cj + dk * ck)); }
  __device__ double r(int di, int dj, int dk) const { return __ldg(pR + (di + dj * cj + dk * ck)); }
};

// tiled kernel geometry: a 32 x 8 tile of (i, j) columns marches up in k; the
// velocity planes k-2..k+2 (in-plane halo 2) and the cell planes k-1..k+1
// (halo 1) sit in rings of shared memory, the next plane loading meanwhile
constexpr int kTX = 32, kTY = 8, kKC = 64;
constexpr int kHV = 2, kHC = 1;
constexpr int kPV = kTX + 2 * kHV, kPC = kTX + 2 * kHC;  // row pitches
constexpr int kNV = kPV * (kTY + 2 * kHV), kNC = kPC * (kTY + 2 * kHC);  // doubles per plane
constexpr int kRV = 6, kRC = 4;  // ring depths: 5 + 1 and 3 + 1 planes

struct SAcc {
  const double *sU, *sV, *sW, *sC, *sM, *sR;
  int ov[5], oc[3];  // slot offsets of planes k-2..k+2 (velocity), k-1..k+1 (cell)
  __device__ double u(int di, int dj, int dk) const { return sU[ov[dk + 2] + dj * kPV + di]; }
  __device__ double v(int di, int dj, int dk) const { return sV[ov[dk + 2] + dj * kPV + di]; }
  __device__ double w(int di, int dj, int dk) const { return sW[ov[dk + 2] + dj * kPV + di]; }
  __device__ double c(int di, int dj, int dk) const { return sC[oc[dk + 1] + dj * kPC + di]; }
  __device__ double m(int di, int dj, int dk) const { return sM[oc[dk + 1] + dj * kPC + di]; }
  __device__ double r(int di, int dj, int dk) const { return sR[oc[dk + 1] + dj * kPC + di]; }
  // the accessor of the cell (di, dj) columns away in the same plane
  __device__ SAcc shifted(int di, int dj) const {
    SAcc b = *this;
    b.sU += di + dj * kPV;
    b.sV += di + dj * kPV;
    b.sW += di + dj * kPV;
    b.sC += di + dj * kPC;
    b.sM += di + dj * kPC;
    b.sR += di + dj * kPC;
    return b;
  }
  // the accessor of the cell one plane down (reaches planes k-2..k+1 only)
  __device__ SAcc down() const {
    SAcc b = *this;
#pragma unroll
    for (int d = 4; d > 0; --d) b.ov[d] = ov[d - 1];
#pragma unroll
    for (int d = 2; d > 0; --d) b.oc[d] = oc[d - 1];
    return b;
  }
};

// the spacings one cell's stencils use (reciprocals, and dyf at j, j+1),
// loaded once per cell through the read-only path
struct Met {
  double rxf0, rxf1, rxc0, rxc1, ryf0, ryf1, ryc0, ryc1, dyf0, dyf1, rzf0, rzf1, rzc0, rzc1;
  __device__ Met(const MomArgs &a, int i, int j, int k)
      : rxf0(__ldg(a.rdxf + i)), rxf1(__ldg(a.rdxf + i + 1)), rxc0(__ldg(a.rdxc + i)), rxc1(__ldg(a.rdxc + i + 1)),
        ryf0(__ldg(a.rdyf + j)), ryf1(__ldg(a.rdyf + j + 1)), ryc0(__ldg(a.rdyc + j)), ryc1(__ldg(a.rdyc + j + 1)),
        dyf0(__ldg(a.dyf + j)), dyf1(__ldg(a.dyf + j + 1)), rzf0(__ldg(a.rdzf + k)), rzf1(__ldg(a.rdzf + k + 1)),
        rzc0(__ldg(a.rdzc + k)), rzc1(__ldg(a.rdzc + k + 1)) {}
};

#define TBFP_MOM_ACCESSORS                                                       \
  auto u = [&](int di, int dj, int dk) { return A.u(di, dj, dk); };              \
  auto v = [&](int di, int dj, int dk) { return A.v(di, dj, dk); };              \
  auto w = [&](int di, int dj, int dk) { return A.w(di, dj, dk); };              \
  auto c = [&](int di, int dj, int dk) { return A.c(di, dj, dk); };              \
  auto m = [&](int di, int dj, int dk) { return A.m(di, dj, dk); };              \
  auto rho = [&](int di, int dj, int dk) { return A.r(di, dj, dk); };            \
  (void)c

// The upper-face fluxes of the nine (component, direction) pairs at the
// accessor's cell (updateConveDiff, momentumEqn.f90:228-603): ux faces
template <int S, class Acc>
__device__ __forceinline__ double F_xx(const Acc &A) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (u(0, 0, 0) + u(1, 0, 0)), u(-1, 0, 0), u(0, 0, 0), u(1, 0, 0), u(2, 0, 0));
}
template <int S, class Acc>
__device__ __forceinline__ double F_xy(const Acc &A) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (v(1, 0, 0) + v(0, 0, 0)), u(0, -1, 0), u(0, 0, 0), u(0, 1, 0), u(0, 2, 0));
}
template <int S, class Acc>
__device__ __forceinline__ double F_xz(const Acc &A) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (w(0, 0, 0) + w(1, 0, 0)), u(0, 0, -1), u(0, 0, 0), u(0, 0, 1), u(0, 0, 2));
}
// uy faces
template <int S, class Acc>
__device__ __forceinline__ double F_yx(const Acc &A, const Met &g) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (u(0, 1, 0) * g.dyf1 + u(0, 0, 0) * g.dyf0) * g.ryc1, v(-1, 0, 0), v(0, 0, 0), v(1, 0, 0),
                      v(2, 0, 0));
}
template <int S, class Acc>
__device__ __forceinline__ double F_yy(const Acc &A) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (v(0, 0, 0) + v(0, 1, 0)), v(0, -1, 0), v(0, 0, 0), v(0, 1, 0), v(0, 2, 0));
}
template <int S, class Acc>
__device__ __forceinline__ double F_yz(const Acc &A, const Met &g) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (w(0, 1, 0) * g.dyf1 + w(0, 0, 0) * g.dyf0) * g.ryc1, v(0, 0, -1), v(0, 0, 0), v(0, 0, 1),
                      v(0, 0, 2));
}
// uz faces
template <int S, class Acc>
__device__ __forceinline__ double F_zx(const Acc &A) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (u(0, 0, 0) + u(0, 0, 1)), w(-1, 0, 0), w(0, 0, 0), w(1, 0, 0), w(2, 0, 0));
}
template <int S, class Acc>
__device__ __forceinline__ double F_zy(const Acc &A) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (v(0, 0, 0) + v(0, 0, 1)), w(0, -1, 0), w(0, 0, 0), w(0, 1, 0), w(0, 2, 0));
}
template <int S, class Acc>
__device__ __forceinline__ double F_zz(const Acc &A) {
  TBFP_MOM_ACCESSORS;
  return face_flux<S>(0.5 * (w(0, 0, 0) + w(0, 0, 1)), w(0, 0, -1), w(0, 0, 0), w(0, 0, 1), w(0, 0, 2));
}

// x component at face (i, j, k) (momentumEqn.f90:228-341) from the convective
// flux differences (upper minus lower face) of its three directions, plus the
// diffusion with its transposed terms
template <class Acc>
__device__ __forceinline__ double tail_x(const Acc &A, const Met &g, double invrho, double cx, double cy, double cz) {
  TBFP_MOM_ACCESSORS;
  const double uc = u(0, 0, 0);
  const double rxc = g.rxc1, ryf = g.ryf0, rzf = g.rzf0;
  double phi = 0.0;
  phi = phi - cx * rxc;  // d(uu)/dx
  phi = phi - cy * ryf;  // d(vu)/dy
  phi = phi - cz * rzf;  // d(wu)/dz
  double mur = m(1, 0, 0), mul = m(0, 0, 0);
  const double dxx = (mur * (u(1, 0, 0) - uc) * g.rxf1 - mul * (uc - u(-1, 0, 0)) * g.rxf0) * rxc;
  const double dxxt = dxx;
  mur = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 1, 0) + m(0, 1, 0));
  mul = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, -1, 0) + m(0, -1, 0));
  const double dyy = (mur * (u(0, 1, 0) - uc) * g.ryc1 - mul * (uc - u(0, -1, 0)) * g.ryc0) * ryf;
  const double dyyt = (mur * (v(1, 0, 0) - v(0, 0, 0)) * rxc - mul * (v(1, -1, 0) - v(0, -1, 0)) * rxc) * ryf;
  mur = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 0, 1) + m(0, 0, 1));
  mul = 0.25 * (m(1, 0, 0) + m(0, 0, 0) + m(1, 0, -1) + m(0, 0, -1));
  const double dzz = (mur * (u(0, 0, 1) - uc) * g.rzc1 - mul * (uc - u(0, 0, -1)) * g.rzc0) * rzf;
  const double dzzt = (mur * (w(1, 0, 0) - w(0, 0, 0)) * rxc - mul * (w(1, 0, -1) - w(0, 0, -1)) * rxc) * rzf;
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}

// y component at face (i, j, k) (momentumEqn.f90:344-467)
template <class Acc>
__device__ __forceinline__ double tail_y(const Acc &A, const Met &g, double invrho, double cx, double cy, double cz) {
  TBFP_MOM_ACCESSORS;
  const double vc = v(0, 0, 0);
  const double rycp = g.ryc1, rxf = g.rxf0, rzf = g.rzf0;
  double phi = 0.0;
  phi = phi - cx * rxf;   // d(uv)/dx
  phi = phi - cy * rycp;  // d(vv)/dy
  phi = phi - cz * rzf;   // d(wv)/dz
  double mur = 0.25 * (m(0, 0, 0) + m(1, 0, 0) + m(0, 1, 0) + m(1, 1, 0));
  double mul = 0.25 * (m(0, 0, 0) + m(-1, 0, 0) + m(0, 1, 0) + m(-1, 1, 0));
  const double dxx = (mur * (v(1, 0, 0) - vc) * g.rxc1 - mul * (vc - v(-1, 0, 0)) * g.rxc0) * rxf;
  const double dxxt = (mur * (u(0, 1, 0) - u(0, 0, 0)) * rycp - mul * (u(-1, 1, 0) - u(-1, 0, 0)) * rycp) * rxf;
  mur = m(0, 1, 0);
  mul = m(0, 0, 0);
  const double dyy = (mur * (v(0, 1, 0) - vc) * g.ryf1 - mul * (vc - v(0, -1, 0)) * g.ryf0) * rycp;
  const double dyyt = dyy;
  mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, 1, 0) + m(0, 1, 1));
  mul = 0.25 * (m(0, 0, 0) + m(0, 0, -1) + m(0, 1, 0) + m(0, 1, -1));
  const double dzz = (mur * (v(0, 0, 1) - vc) * g.rzc1 - mul * (vc - v(0, 0, -1)) * g.rzc0) * rzf;
  const double dzzt = (mur * (w(0, 1, 0) - w(0, 0, 0)) * rycp - mul * (w(0, 1, -1) - w(0, 0, -1)) * rycp) * rzf;
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}

// z component at face (i, j, k) (momentumEqn.f90:470-603)
template <class Acc>
__device__ __forceinline__ double tail_z(const Acc &A, const Met &g, double invrho, double cx, double cy, double cz) {
  TBFP_MOM_ACCESSORS;
  const double wc = w(0, 0, 0);
  const double rxf = g.rxf0, ryf = g.ryf0, rzcp = g.rzc1;
  double phi = 0.0;
  phi = phi - cx * rxf;   // d(uw)/dx
  phi = phi - cy * ryf;   // d(vw)/dy
  phi = phi - cz * rzcp;  // d(ww)/dz
  double mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(1, 0, 0) + m(1, 0, 1));
  double mul = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(-1, 0, 0) + m(-1, 0, 1));
  const double dxx = (mur * (w(1, 0, 0) - wc) * g.rxc1 - mul * (wc - w(-1, 0, 0)) * g.rxc0) * rxf;
  const double dxxt = (mur * (u(0, 0, 1) - u(0, 0, 0)) * rzcp - mul * (u(-1, 0, 1) - u(-1, 0, 0)) * rzcp) * rxf;
  mur = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, 1, 0) + m(0, 1, 1));
  mul = 0.25 * (m(0, 0, 0) + m(0, 0, 1) + m(0, -1, 0) + m(0, -1, 1));
  const double dyy = (mur * (w(0, 1, 0) - wc) * g.ryc1 - mul * (wc - w(0, -1, 0)) * g.ryc0) * ryf;
  const double dyyt = (mur * (v(0, 0, 1) - v(0, 0, 0)) * rzcp - mul * (v(0, -1, 1) - v(0, -1, 0)) * rzcp) * ryf;
  mur = m(0, 0, 1);
  mul = m(0, 0, 0);
  const double dzz = (mur * (w(0, 0, 1) - wc) * g.rzf1 - mul * (wc - w(0, 0, -1)) * g.rzf0) * rzcp;
  const double dzzt = dzz;
  return phi + (dxx + dyy + dzz + dxxt + dyyt + dzzt) * invrho;
}

// The per-cell forms (every scheme; scheme 5's limiters depend on the cell):
// both faces of each direction at the cell itself
template <int S, class Acc>
__device__ __forceinline__ double phi_x(const Acc &A, const Met &g, double invrho) {
  TBFP_MOM_ACCESSORS;
  const bool sh = sharp_cell<S>(c(1, 0, 0), c(0, 0, 0), c(0, 1, 0), c(0, -1, 0), c(0, 0, 1), c(0, 0, -1));
  const double uc = u(0, 0, 0);
  const double cx = conv_diff<S>(0.5 * (uc + u(1, 0, 0)), 0.5 * (uc + u(-1, 0, 0)), u(-2, 0, 0), u(-1, 0, 0), uc,
                                 u(1, 0, 0), u(2, 0, 0), sh);
  const double cy = conv_diff<S>(0.5 * (v(1, 0, 0) + v(0, 0, 0)), 0.5 * (v(1, -1, 0) + v(0, -1, 0)), u(0, -2, 0),
                                 u(0, -1, 0), uc, u(0, 1, 0), u(0, 2, 0), sh);
  const double cz = conv_diff<S>(0.5 * (w(0, 0, 0) + w(1, 0, 0)), 0.5 * (w(0, 0, -1) + w(1, 0, -1)), u(0, 0, -2),
                                 u(0, 0, -1), uc, u(0, 0, 1), u(0, 0, 2), sh);
  return tail_x(A, g, invrho, cx, cy, cz);
}

template <int S, class Acc>
__device__ __forceinline__ double phi_y(const Acc &A, const Met &g, double invrho) {
  TBFP_MOM_ACCESSORS;
  const bool sh = sharp_cell<S>(c(1, 0, 0), c(-1, 0, 0), c(0, 1, 0), c(0, 0, 0), c(0, 0, 1), c(0, 0, -1));
  const double vc = v(0, 0, 0);
  const double dyfj = g.dyf0, dyfp = g.dyf1, rycp = g.ryc1;
  const double cx = conv_diff<S>(0.5 * (u(0, 1, 0) * dyfp + u(0, 0, 0) * dyfj) * rycp,
                                 0.5 * (u(-1, 1, 0) * dyfp + u(-1, 0, 0) * dyfj) * rycp, v(-2, 0, 0), v(-1, 0, 0), vc,
                                 v(1, 0, 0), v(2, 0, 0), sh);
  const double cy = conv_diff<S>(0.5 * (vc + v(0, 1, 0)), 0.5 * (vc + v(0, -1, 0)), v(0, -2, 0), v(0, -1, 0), vc,
                                 v(0, 1, 0), v(0, 2, 0), sh);
  const double cz = conv_diff<S>(0.5 * (w(0, 1, 0) * dyfp + w(0, 0, 0) * dyfj) * rycp,
                                 0.5 * (w(0, 1, -1) * dyfp + w(0, 0, -1) * dyfj) * rycp, v(0, 0, -2), v(0, 0, -1), vc,
                                 v(0, 0, 1), v(0, 0, 2), sh);
  return tail_y(A, g, invrho, cx, cy, cz);
}

template <int S, class Acc>
__device__ __forceinline__ double phi_z(const Acc &A, const Met &g, double invrho) {
  TBFP_MOM_ACCESSORS;
  const bool sh = sharp_cell<S>(c(1, 0, 0), c(-1, 0, 0), c(0, 1, 0), c(0, -1, 0), c(0, 0, 1), c(0, 0, 0));
  const double wc = w(0, 0, 0);
  const double cx = conv_diff<S>(0.5 * (u(0, 0, 0) + u(0, 0, 1)), 0.5 * (u(-1, 0, 0) + u(-1, 0, 1)), w(-2, 0, 0),
                                 w(-1, 0, 0), wc, w(1, 0, 0), w(2, 0, 0), sh);
  const double cy = conv_diff<S>(0.5 * (v(0, 0, 0) + v(0, 0, 1)), 0.5 * (v(0, -1, 0) + v(0, -1, 1)), w(0, -2, 0),
                                 w(0, -1, 0), wc, w(0, 1, 0), w(0, 2, 0), sh);
  const double cz = conv_diff<S>(0.5 * (wc + w(0, 0, 1)), 0.5 * (wc + w(0, 0, -1)), w(0, 0, -2), w(0, 0, -1), wc,
                                 w(0, 0, 1), w(0, 0, 2), sh);
  return tail_z(A, g, invrho, cx, cy, cz);
}
#undef TBFP_MOM_ACCESSORS

// Computing each face once (schemes 0-4) costs a barrier, shared-memory
// traffic and the edge faces; it pays where the limiter is expensive (van
// Leer's and superbee's divisions and branches: 27 % and 22 % faster on
// 512x384x256) and loses where it is cheap (central, upwind, QUICK: 8-10 %
// slower), so those keep both faces per cell, as scheme 5 must.
__host__ __device__ constexpr bool share_faces(int S) { return S == 3 || S == 4; }

// Tiled form: block (32, 8) over a tile of (i, j) columns, i = 1..nx,
// j = 1..ny, marching k over a chunk of kKC planes of 0..nz; each thread the
// components whose box holds its (i, j, k).  A plane outside a field's array
// is not loaded: no stencil of a computed component reaches it.
template <int S, bool OUT>
__global__ void __launch_bounds__(kTX * kTY, 2) k_momentum_fluxes(MomArgs a) {
  extern __shared__ double sm[];
  double *rU = sm, *rV = rU + kRV * kNV, *rW = rV + kRV * kNV;
  double *rM = rW + kRV * kNV, *rR = rM + kRC * kNC, *rC = rR + kRC * kNC;
  // face fluxes of one plane (schemes 0-4): x faces [3][kTY][kTX+1], y faces [3][kTY+1][kTX]
  double *fx = rC, *fy = fx + 3 * kTY * (kTX + 1);
  double fzl0 = 0.0, fzl1 = 0.0, fzl2 = 0.0;  // lower z faces of the current plane
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * kTX + tx;
  const int i0 = blockIdx.x * kTX + 1, j0 = blockIdx.y * kTY + 1;
  const int kb = blockIdx.z * kKC, ke = min(kb + kKC - 1, a.nz);
  const int i = i0 + tx, j = j0 + ty;
  const bool in = i <= a.nx && j <= a.ny;
  const int vhi = a.hdu, chi = a.hdc;  // upper bound of every array: n + halo

  auto load_v = [&](double *ring, const double *f, const Lay &L, int kp) {
    if (kp < L.klo || kp > a.nz + vhi) return;
    double *dst = ring + ((kp + 3 * kRV) % kRV) * kNV;
    for (int e = tid; e < kNV; e += kTX * kTY) {
      const int rr = e / kPV, cc = e - rr * kPV;
      const int gi = i0 - kHV + cc, gj = j0 - kHV + rr;
      if (gi >= L.ilo && gi <= a.nx + vhi && gj >= L.jlo && gj <= a.ny + vhi) cp_async8(dst + e, f + at(L, gi, gj, kp));
    }
  };
  auto load_c = [&](double *ring, const double *f, int kp) {
    const Lay &L = a.Lc;
    if (kp < L.klo || kp > a.nz + chi) return;
    double *dst = ring + ((kp + 3 * kRC) % kRC) * kNC;
    for (int e = tid; e < kNC; e += kTX * kTY) {
      const int rr = e / kPC, cc = e - rr * kPC;
      const int gi = i0 - kHC + cc, gj = j0 - kHC + rr;
      if (gi >= L.ilo && gi <= a.nx + chi && gj >= L.jlo && gj <= a.ny + chi) cp_async8(dst + e, f + at(L, gi, gj, kp));
    }
  };
  auto load_planes = [&](int kv, int kcl) {
    load_v(rU, a.ux, a.Lux, kv);
    load_v(rV, a.uy, a.Luy, kv);
    load_v(rW, a.uz, a.Luz, kv);
    load_c(rM, a.mu, kcl);
    load_c(rR, a.rho, kcl);
    if (S == 5) load_c(rC, a.c, kcl);
  };
  for (int d = -2; d <= 2; ++d) {
    load_v(rU, a.ux, a.Lux, kb + d);
    load_v(rV, a.uy, a.Luy, kb + d);
    load_v(rW, a.uz, a.Luz, kb + d);
  }
  for (int d = -1; d <= 1; ++d) {
    load_c(rM, a.mu, kb + d);
    load_c(rR, a.rho, kb + d);
    if (S == 5) load_c(rC, a.c, kb + d);
  }
  cp_async_wait_all();
  __syncthreads();
  SAcc A;
  A.sU = rU + (ty + kHV) * kPV + tx + kHV;
  A.sV = rV + (ty + kHV) * kPV + tx + kHV;
  A.sW = rW + (ty + kHV) * kPV + tx + kHV;
  A.sM = rM + (ty + kHC) * kPC + tx + kHC;
  A.sR = rR + (ty + kHC) * kPC + tx + kHC;
  A.sC = rC + (ty + kHC) * kPC + tx + kHC;
  for (int k = kb; k <= ke; ++k) {
    // planes k+3 (velocity) and k+2 (cell) into the slots of k-3 and k-2, read by the previous step only
    if (k < ke) load_planes(k + 3, k + 2);
#pragma unroll
    for (int d = 0; d < 5; ++d) A.ov[d] = ((k + d - 2 + 3 * kRV) % kRV) * kNV;
#pragma unroll
    for (int d = 0; d < 3; ++d) A.oc[d] = ((k + d - 1 + 3 * kRC) % kRC) * kNC;
    if constexpr (!share_faces(S)) {
      if (in) {
        const double irc = 1.0 / A.r(0, 0, 0);  // 1/rho of the own cell, shared by the three components
        const Met g(a, i, j, k);
        if (k >= 1) {
          const double ivx = 0.5 * (1.0 / A.r(1, 0, 0) + irc);
          emit_x<OUT>(a, i, j, k, phi_x<S>(A, g, ivx), A.u(0, 0, 0), ivx);
          if (j <= a.ny - 1) emit_y<OUT>(a, i, j, k, phi_y<S>(A, g, 0.5 * (1.0 / A.r(0, 1, 0) + irc)), A.v(0, 0, 0));
        }
        emit_z<OUT>(a, i, j, k, phi_z<S>(A, g, 0.5 * (1.0 / A.r(0, 0, 1) + irc)), A.w(0, 0, 0));
      }
    } else {
      // each face once: the cell's upper x, y faces into shared memory, its
      // upper z faces in registers (the next plane's lower ones); the tile's
      // lower edge faces by warp 0 (x, 8 rows) and warp 1 (y, 32 columns)
      double fzn0 = 0.0, fzn1 = 0.0, fzn2 = 0.0;
      if (in) {
        const Met g(a, i, j, k);
        fx[(0 * kTY + ty) * (kTX + 1) + tx + 1] = F_xx<S>(A);
        fx[(1 * kTY + ty) * (kTX + 1) + tx + 1] = F_yx<S>(A, g);
        fx[(2 * kTY + ty) * (kTX + 1) + tx + 1] = F_zx<S>(A);
        fy[(0 * (kTY + 1) + ty + 1) * kTX + tx] = F_xy<S>(A);
        fy[(1 * (kTY + 1) + ty + 1) * kTX + tx] = F_yy<S>(A);
        fy[(2 * (kTY + 1) + ty + 1) * kTX + tx] = F_zy<S>(A);
        fzn0 = F_xz<S>(A);
        fzn1 = F_yz<S>(A, g);
        fzn2 = F_zz<S>(A);
        if (k == kb) {  // the chunk's first lower z faces (ux, uy need none at k = 0)
          const SAcc B = A.down();
          if (kb > 0) {
            fzl0 = F_xz<S>(B);
            fzl1 = F_yz<S>(B, g);
          }
          fzl2 = F_zz<S>(B);
        }
      }
      if (ty == 0 && tx < kTY && j0 + tx <= a.ny) {
        const SAcc E = A.shifted(-1 - tx, tx);
        const Met ge(a, i0 - 1, j0 + tx, k);
        fx[(0 * kTY + tx) * (kTX + 1)] = F_xx<S>(E);
        fx[(1 * kTY + tx) * (kTX + 1)] = F_yx<S>(E, ge);
        fx[(2 * kTY + tx) * (kTX + 1)] = F_zx<S>(E);
      } else if (ty == 1 && i0 + tx <= a.nx) {
        const SAcc E = A.shifted(0, -2);
        fy[(0 * (kTY + 1)) * kTX + tx] = F_xy<S>(E);
        fy[(1 * (kTY + 1)) * kTX + tx] = F_yy<S>(E);
        fy[(2 * (kTY + 1)) * kTX + tx] = F_zy<S>(E);
      }
      __syncthreads();
      if (in) {
        const Met g(a, i, j, k);
        const double irc = 1.0 / A.r(0, 0, 0);
        auto cxd = [&](int c) { return fx[(c * kTY + ty) * (kTX + 1) + tx + 1] - fx[(c * kTY + ty) * (kTX + 1) + tx]; };
        auto cyd = [&](int c) { return fy[(c * (kTY + 1) + ty + 1) * kTX + tx] - fy[(c * (kTY + 1) + ty) * kTX + tx]; };
        if (k >= 1) {
          const double ivx = 0.5 * (1.0 / A.r(1, 0, 0) + irc);
          emit_x<OUT>(a, i, j, k, tail_x(A, g, ivx, cxd(0), cyd(0), fzn0 - fzl0), A.u(0, 0, 0), ivx);
          if (j <= a.ny - 1)
            emit_y<OUT>(a, i, j, k, tail_y(A, g, 0.5 * (1.0 / A.r(0, 1, 0) + irc), cxd(1), cyd(1), fzn1 - fzl1),
                        A.v(0, 0, 0));
        }
        emit_z<OUT>(a, i, j, k, tail_z(A, g, 0.5 * (1.0 / A.r(0, 0, 1) + irc), cxd(2), cyd(2), fzn2 - fzl2),
                    A.w(0, 0, 0));
      }
      fzl0 = fzn0;
      fzl1 = fzn1;
      fzl2 = fzn2;
    }
    cp_async_wait_all();
    __syncthreads();
  }
}

__host__ __device__ constexpr size_t tiled_smem_bytes(int S) {
  return sizeof(double) * (3 * kRV * kNV + 2 * kRC * kNC + (S == 5 ? kRC * kNC : 0) +
                           (share_faces(S) ? 3 * kTY * (kTX + 1) + 3 * (kTY + 1) * kTX : 0));
}

// the x component's face i = 0 (the periodic duplicate of i = nx, computed
// from its own stencil), one thread per (j, k)
template <int S, bool OUT>
__global__ void __launch_bounds__(kMT) k_momentum_fluxes_i0(MomArgs a) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x + 1, k = blockIdx.y + 1;
  if (j > a.ny) return;
  const GAcc A(a, 0, j, k);
  const double ivx = 0.5 * (1.0 / A.r(1, 0, 0) + 1.0 / A.r(0, 0, 0));
  emit_x<OUT>(a, 0, j, k, phi_x<S>(A, Met(a, 0, j, k), ivx), A.u(0, 0, 0), ivx);
}

// The out-of-place form leaves the elements outside the equation boxes to
// this copy from u_in: uy's wall faces, every ghost and halo layer (the
// boundary update that follows rewrites the ones the reference rewrites).
// It visits, per component, the planes outside the box's k range, the rows
// outside its j range and the columns outside its i range.
struct Cmp {
  const double *in;
  double *out;
  Lay L;
  int ilo, ihi, jlo, jhi, klo, khi;  // array
  int bi0, bi1, bj0, bj1, bk0, bk1;  // equation box
  long n_planes, n_total;
};
struct CmpArgs {
  Cmp c[3];
};

__global__ void __launch_bounds__(256) k_copy_outside_box(CmpArgs a) {
  const Cmp &c = a.c[blockIdx.y];
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= c.n_total) return;
  const int NI = c.ihi - c.ilo + 1, NJ = c.jhi - c.jlo + 1;
  const int nkl = c.bk0 - c.klo, njl = c.bj0 - c.jlo, njh = c.jhi - c.bj1, nil = c.bi0 - c.ilo, nih = c.ihi - c.bi1;
  int i, j, k;
  if (t < c.n_planes) {
    const long pl = (long)NI * NJ;
    const int p = (int)(t / pl), r = (int)(t - p * pl);
    k = p < nkl ? c.klo + p : c.bk1 + 1 + (p - nkl);
    j = c.jlo + r / NI;
    i = c.ilo + r % NI;
  } else {
    const long u = t - c.n_planes;
    const long per_k = (long)(njl + njh) * NI + (long)(c.bj1 - c.bj0 + 1) * (nil + nih);
    k = c.bk0 + (int)(u / per_k);
    const int r = (int)(u - (k - c.bk0) * per_k);
    if (r < (njl + njh) * NI) {
      const int rr = r / NI;
      j = rr < njl ? c.jlo + rr : c.bj1 + 1 + (rr - njl);
      i = c.ilo + r % NI;
    } else {
      const int q = r - (njl + njh) * NI, jj = q / (nil + nih), ii = q - jj * (nil + nih);
      j = c.bj0 + jj;
      i = ii < nil ? c.ilo + ii : c.bi1 + 1 + (ii - nil);
    }
  }
  const long o = at(c.L, i, j, k);
  c.out[o] = c.in[o];
}

template <int S, bool OUT>
void launch_fluxes(const MomArgs &a, cudaStream_t st) {
  static bool attr[64] = {};  // per device: the attribute belongs to the device's context
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !attr[dev]) {
    cudaFuncSetAttribute(k_momentum_fluxes<S, OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)tiled_smem_bytes(S));
    if (dev < 64) attr[dev] = true;
  }
  const dim3 blk(kTX, kTY), grid((a.nx + kTX - 1) / kTX, (a.ny + kTY - 1) / kTY, (a.nz + 1 + kKC - 1) / kKC);
  k_momentum_fluxes<S, OUT><<<grid, blk, tiled_smem_bytes(S), st>>>(a);
  k_momentum_fluxes_i0<S, OUT><<<dim3((a.ny + kMT - 1) / kMT, a.nz), kMT, 0, st>>>(a);
}

template <bool OUT>
void launch_fluxes_scheme(int scheme, const MomArgs &a, cudaStream_t st) {
  switch (scheme) {
    case 0: launch_fluxes<0, OUT>(a, st); break;
    case 1: launch_fluxes<1, OUT>(a, st); break;
    case 2: launch_fluxes<2, OUT>(a, st); break;
    case 3: launch_fluxes<3, OUT>(a, st); break;
    case 4: launch_fluxes<4, OUT>(a, st); break;
    default: launch_fluxes<5, OUT>(a, st); break;
  }
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

// updateBoundariesV for the channel (vfield.f90:111-189): fixedValue walls in
// y, periodic halos in x and z, the periodic duplicates ux(0) = ux(nx),
// uz(0) = uz(nz).  The reference's sequence (wall ghost layer on the interior
// i, k range; x exchange over all j, k; z exchange over whole planes; equate)
// leaves every written element equal to a function of elements it never
// writes: with mx(i) = i + nx for i < 1, i - nx for i > nx (the equate is
// mx(0) = nx), likewise mz, the element (i, j, k) becomes
//   j = js-1 or je+1 (the wall ghosts): the wall formula of (mx(i), jb/jt, mz(k)),
//   any other j:                        the element (mx(i), j, mz(k)),
// so one gather pass in place is race-free.  It visits the halo planes
// k < 1 and k > nz (all i, j) and, for k = 1..nz, the wall ghost rows (all i)
// and the x halo columns (and ux's i = 0) of the other rows.  On a slab of a
// z-split channel the z ghost planes and uz's plane 0 belong to the
// neighbours' exchange: the pass covers the planes ks..nz without z wrap.
struct BcComp {
  double *f;
  Lay L;
  int ilo, ihi, jlo, jhi, klo, khi;  // allocated extents
  int js, je, jb, jt;                // interior j range, the wall formulas' source rows
  double hb, hi, tb, ti, bb, bt;     // dhb, dhi and wall value: bottom, top
  int kin0;                          // first plane of the row/column part (1; ks on a slab)
  long n_planes, n_total;            // elements visited in the halo planes; in all
};
struct BcArgs {
  BcComp c[3];
  int nx, nz;
  int slab;  // 1: no z wrap (planes ks..nz only, mz = identity)
};

__device__ __forceinline__ double wall(double v, double dhb, double dhi, double bf) {
  // (f*dhb - bf*dhi)/(dhb - dhi), rounded as written
  return __ddiv_rn(__dsub_rn(__dmul_rn(v, dhb), __dmul_rn(bf, dhi)), __dsub_rn(dhb, dhi));
}

__global__ void __launch_bounds__(256) k_boundaries_v(BcArgs a) {
  const BcComp &c = a.c[blockIdx.y];
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= c.n_total) return;
  const int NI = c.ihi - c.ilo + 1, NJ = c.jhi - c.jlo + 1;
  int i, j, k;
  if (t < c.n_planes) {
    const long pl = NI * (long)NJ;
    const int p = (int)(t / pl), r = (int)(t - p * pl);
    const int nlow = 1 - c.klo;  // planes klo..0
    k = p < nlow ? c.klo + p : a.nz + 1 + (p - nlow);
    j = c.jlo + r / NI;
    i = c.ilo + r % NI;
  } else {
    const long u = t - c.n_planes;
    const int nxh = (1 - c.ilo) + (c.ihi - a.nx);  // x halo columns (ux: with i = 0)
    const long per_k = 2L * NI + (long)(NJ - 2) * nxh;
    k = c.kin0 + (int)(u / per_k);
    const int r = (int)(u - (k - c.kin0) * per_k);
    if (r < 2 * NI) {
      j = r < NI ? c.js - 1 : c.je + 1;
      i = c.ilo + r % NI;
    } else {
      const int q = r - 2 * NI, jj = q / nxh, ii = q - jj * nxh;
      j = c.jlo + jj;
      if (j >= c.js - 1) ++j;
      if (j >= c.je + 1) ++j;
      i = ii < 1 - c.ilo ? c.ilo + ii : a.nx + 1 + (ii - (1 - c.ilo));
    }
  }
  const int mi = i < 1 ? i + a.nx : (i > a.nx ? i - a.nx : i);
  const int mk = a.slab ? k : (k < 1 ? k + a.nz : (k > a.nz ? k - a.nz : k));
  double v;
  if (j == c.js - 1) v = wall(c.f[at(c.L, mi, c.jb, mk)], c.hb, c.hi, c.bb);
  else if (j == c.je + 1) v = wall(c.f[at(c.L, mi, c.jt, mk)], c.tb, c.ti, c.bt);
  else v = c.f[at(c.L, mi, j, mk)];
  c.f[at(c.L, i, j, k)] = v;
}

}  // namespace

void launch_momentum(const MomentumTabs &t, double *ux, double *uy, double *uz, const double *c, const double *mu,
                     const double *rho, const double *const *st, Lay Lux, Lay Luy, Lay Luz, Lay Lc, const Lay *Lst,
                     double *const phi[3], const double *const prev[3], int nx, int ny, int nz, int scheme, double dt,
                     double alpha, double gamma, double xi, double rho0, double fs, double gch, double g, int hdu,
                     int hdc, double *const *u_out, cudaStream_t st_) {
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
  a.hdu = hdu;
  a.hdc = hdc;
  if (u_out) {
    // fused: the flux kernel also writes u_out on the boxes; the rest of u_out is copied from u
    a.uxo = u_out[0];
    a.uyo = u_out[1];
    a.uzo = u_out[2];
    a.ppx = prev[0];
    a.ppy = prev[1];
    a.ppz = prev[2];
    a.stx = st ? st[0] : nullptr;
    a.sty = st ? st[1] : nullptr;
    a.stz = st ? st[2] : nullptr;
    if (st) {
      a.Lsx = Lst[0];
      a.Lsy = Lst[1];
      a.Lsz = Lst[2];
    }
    a.dt = dt;
    a.gamma = gamma;
    a.xi = xi;
    a.r = dt * alpha;
    a.invrho0 = 1.0 / rho0;
    a.fs = fs;
    a.gch = gch;
    a.g = g;
    launch_fluxes_scheme<true>(scheme, a, st_);
    CmpArgs ca{};
    const double *in[3] = {ux, uy, uz};
    const Lay L[3] = {Lux, Luy, Luz};
    long most = 0;
    for (int e = 0; e < 3; ++e) {
      Cmp &c = ca.c[e];
      const int is = e == 0 ? 0 : 1, js = e == 1 ? 0 : 1, ks = e == 2 ? 0 : 1;
      c.in = in[e];
      c.out = u_out[e];
      c.L = L[e];
      c.ilo = is - hdu;
      c.ihi = nx + hdu;
      c.jlo = js - hdu;
      c.jhi = ny + hdu;
      c.klo = ks - hdu;
      c.khi = nz + hdu;
      // equation boxes: ux (0:nx,1:ny,1:nz), uy (1:nx,1:ny-1,1:nz), uz (1:nx,1:ny,0:nz)
      c.bi0 = e == 0 ? 0 : 1;
      c.bi1 = nx;
      c.bj0 = 1;
      c.bj1 = e == 1 ? ny - 1 : ny;
      c.bk0 = e == 2 ? 0 : 1;
      c.bk1 = nz;
      const long NI = c.ihi - c.ilo + 1, NJ = c.jhi - c.jlo + 1;
      const long nk_out = (c.bk0 - c.klo) + (c.khi - c.bk1), nj_out = (c.bj0 - c.jlo) + (c.jhi - c.bj1);
      const long ni_out = (c.bi0 - c.ilo) + (c.ihi - c.bi1);
      c.n_planes = nk_out * NI * NJ;
      c.n_total = c.n_planes + (long)(c.bk1 - c.bk0 + 1) * (nj_out * NI + (long)(c.bj1 - c.bj0 + 1) * ni_out);
      most = c.n_total > most ? c.n_total : most;
    }
    k_copy_outside_box<<<dim3((unsigned)((most + 255) / 256), 3), 256, 0, st_>>>(ca);
    return;
  }
  launch_fluxes_scheme<false>(scheme, a, st_);
  const dim3 grid((nx + kMT - 1) / kMT, ny, nz + 1);
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

void launch_boundaries_v(const WallTabs &w, double *ux, double *uy, double *uz, Lay Lux, Lay Luy, Lay Luz, int nx,
                         int ny, int nz, int hd, bool slab, cudaStream_t st) {
  BcArgs a{};
  a.nx = nx;
  a.nz = nz;
  a.slab = slab ? 1 : 0;
  double *f[3] = {ux, uy, uz};
  const Lay L[3] = {Lux, Luy, Luz};
  long most = 0;
  for (int e = 0; e < 3; ++e) {
    BcComp &c = a.c[e];
    const int is = e == 0 ? 0 : 1, js = e == 1 ? 0 : 1, ks = e == 2 ? 0 : 1;
    c.f = f[e];
    c.L = L[e];
    c.ilo = is - hd;
    c.ihi = nx + hd;
    c.jlo = js - hd;
    c.jhi = ny + hd;
    c.klo = ks - hd;
    c.khi = nz + hd;
    c.js = js;
    c.je = ny;
    c.jb = e == 1 ? js + 1 : js;
    c.jt = e == 1 ? ny - 1 : ny;
    c.hb = w.hb[e];
    c.hi = w.hi[e];
    c.tb = w.tb[e];
    c.ti = w.ti[e];
    c.bb = w.bb[e];
    c.bt = w.bt[e];
    const long NI = c.ihi - c.ilo + 1, NJ = c.jhi - c.jlo + 1;
    const long nplanes = (1 - c.klo) + hd, nxh = (1 - c.ilo) + hd;
    // a slab leaves its z ghost planes (and uz's plane 0) to the exchange and
    // does the walls and x halos of its planes ks..nz
    c.kin0 = slab ? ks : 1;
    c.n_planes = slab ? 0 : nplanes * NI * NJ;
    c.n_total = c.n_planes + (long)(nz - c.kin0 + 1) * (2 * NI + (NJ - 2) * nxh);
    most = c.n_total > most ? c.n_total : most;
  }
  k_boundaries_v<<<dim3((unsigned)((most + 255) / 256), 3), 256, 0, st>>>(a);
}

}  // namespace tbfp
