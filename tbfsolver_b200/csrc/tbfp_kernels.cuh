// Device-side types, tile geometry and kernel launchers of the projection.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <string>

#include "fft_smem.cuh"

namespace tbfp {

// Layout of a Fortran array f(ilo:.., jlo:.., klo:..), column-major.
struct Lay {
  int ilo, jlo, klo;
  long sj, sk;
};
__host__ __device__ __forceinline__ long at(const Lay &L, int i, int j, int k) {
  return (long)(i - L.ilo) + (long)(j - L.jlo) * L.sj + (long)(k - L.klo) * L.sk;
}

// Grid constants and metric tables (device pointers, 0-based: table[j-1] holds the
// reference's value at Fortran index j).
struct GridK {
  int nx, ny, nz, nkx, M;  // M = nx/2 (length of the half-length complex x transform)
  long R;                  // ny*nz: number of x rows
  double idxf1, idzf1;     // 1/dxf(1), 1/dz_fft
  double idxc1, idzc1;     // 1/dxc(1), 1/dz_fft
  const double *idyf;      // 1/dyf(j), j=1..ny
  const double *idyc;      // 1/dyc(j), j=1..ny+1
  const double *idxf;      // 1/dxf(i), i=1..nx
  const double *idzf;      // 1/dzf(k), k=1..nz
  // slab form (one rank of a channel split over ranks): 0 for a whole channel.
  // With slab = 1 the z neighbours of the first and last plane are the ghost
  // planes the caller exchanged (no periodic wrap, no z ghost images written),
  // and kx0 is the global index of the first local kx (spectral stage).
  int slab, kx0;
};

// Inputs of the split right-hand side (poissonEqn.f90:193-305).
struct RhsArgs {
  const double *ux, *uy, *uz;
  const double *irho;  // 1/rho, laid out like rho
  const double *pn, *pnm1;
  const double *stn[3], *sto[3];
  Lay Lux, Luy, Luz, Lrho, Lpsi, Lst[3];
  double r;     // 1/(alpha*dt)
  double rho0;
};

// Inputs of the velocity correction (momentumEqn.f90:999-1127).
struct CorrArgs {
  const double *uxi, *uyi, *uzi;
  double *uxo, *uyo, *uzo;
  const double *psi, *pn, *pnm1, *irho;
  const double *stn[3], *sto[3];
  Lay Lux, Luy, Luz, Lpsi, Lrho, Lst[3];
  double r;  // dt*alpha
  double invrho0;
  long long wait_cycles;  // bound on each wait of the TMA-staged correction for its copies (SM cycles)
};
// The max|div u| word of a correction whose copy wait ran out: a NaN with its
// own payload, above the canonical NaN, so the host tells it from NaN data.
constexpr unsigned long long kWaitTimeoutBits = 0x7ff8dead00000001ull;
constexpr long long kDefaultWaitCycles = 4000000000LL;  // about 2 s of SM clock

// Source rows of the forward x transform.
//   residual = false: s; with acc != nullptr also acc[0] += sum s*dyf(j) and
//     acc[1] += sum s^2;
//   residual = true: the refinement residual r = s - c [j == ny] - L psi of
//     solveFPS's operator, with c = acc[0] * ctop_scale (the incompatible part
//     of s, which the pinned (0,0) solve leaves on the top wall, so that the
//     residual of the FP64 solution is zero), and acc_r[0] += sum r^2.
//   With acc_r, the residual pass also folds max|s - L psi| (= max|r + c [j == ny]|,
//   the quantity that bounds the divergence the correction leaves) into acc_r[1]
//   as the bits of a non-negative double (a NaN wins).
struct XSrc {
  const double *s;
  Lay Ls;
  const double *psi;
  Lay Lp;
  const double *am, *ap, *dyf;  // y operator coefficients and dyf(j), 0-based
  double idx2, idz2;            // 1/dx^2, 1/dz^2 of the uniform x and z spacing
  double ctop_scale;            // 1/(dyf(ny) nx nz)
  double *acc, *acc_r;
};

// Device-side control of the mixed-precision refinement loop.  Per call the
// host sets tol, dtol, dscale and max_iter (launch_mixed_params, which also
// clears the sums); after every residual pass launch_mixed_decide evaluates
//   rel = ||r||_2/||s||_2 from acc[1] and acc_r[0],  div = dscale * max|s - L psi|
// and stops the loop (done = 1) when rel <= tol and, with dscale > 0, div <= dtol
// (status TBFP_OK); when the sweeps reach max_iter (status TBFP_ENOTCONVERGED);
// or when rel or div is not finite (status TBFP_ENONFINITE).  For the
// projection dscale = alpha*dt/rho0, because the corrected velocity has
// div u = alpha*dt/rho0 * (s - L psi) cell by cell, so div is max|div u|.
struct MixedCtl {
  double tol, dtol, dscale;  // set per call
  double rel, div;           // of the last residual pass
  int max_iter;              // set per call
  int iters;                 // FP32 solves so far
  int status;                // TBFP_OK, TBFP_ENOTCONVERGED or TBFP_ENONFINITE once done
  int done;
};

// One member of an ensemble as the persistent kernel sees it (tbfp_ensemble.cu):
// its grid, the arguments of each stage and its tile counts.  Built on the host
// from the member's handle and arrays, copied to the device once per set of
// arrays.  Stages: 0 1/rho, 1 split RHS, 2 forward x, 3 forward z, 4 y systems,
// 5 backward z, 6 backward x, 7 correction with the continuity check.
constexpr int kEnsStages = 8;
struct EnsMember {
  GridK g;
  RhsArgs ra;
  CorrArgs ca;
  XSrc xs;                        // s -> forward x (acc = nullptr)
  const double *rho;
  double *irho, *s;
  long n_rho;
  double2 *spec;
  double *psi;
  Lay Lpsi;
  int hd_psi;
  const double2 *twx, *tpx, *tpz;
  const double *lamx, *lamz, *am, *ap, *dyf;
  double mean_c, nxnz, scale;
  unsigned long long *maxdiv;
  int T;                          // rows per lane of the y systems
  int items[kEnsStages];          // work items of each stage (256-thread tiles)
};
// Work-queue state of one persistent launch (zeroed before the launch):
// next item, items finished per (member, stage), and the abort word (1 = a
// dependency wait ran out of its spin budget).
struct EnsCtl {
  int next;
  int abort;
  int pad[2];
  int done[1];  // [members * kEnsStages], allocated with the block
};
// Lengths the persistent kernel is compiled for: nx/2 and nz up to 128, rows
// per lane (ceil(ny/32)) up to 8.  Larger members use the graph form.
constexpr int kEnsMaxLen = 128, kEnsMaxT = 8;
inline bool ens_supported(int M, int nz, int T) {
  return M <= kEnsMaxLen && nz <= kEnsMaxLen && T <= kEnsMaxT;
}
// Work items of each stage of a member, and the dynamic shared memory the
// persistent kernel needs for it.
void ens_items(const GridK &g, long n_rho, int T, int *items);
size_t ens_smem_bytes(int M, int nz, int T);
// One persistent launch over every member: grid = blocks_per_sm x SMs;
// spin_limit bounds each dependency wait (iterations of ~0.1 us).  qstart
// holds the prefix sums of the items, stage-major: qstart[s*n + m].
cudaError_t launch_ensemble_persistent(const EnsMember *mem, int n, const int *qstart, EnsCtl *ctl,
                                       long long spin_limit, int blocks, size_t smem, cudaStream_t st);
cudaError_t prepare_ensemble_kernel(size_t smem);
int ensemble_blocks_per_sm(size_t smem);

// Transform lengths with a compiled kernel (nx/2 and nz): 2^a and 3*2^a, 4..512.
#define TBFP_FFT_LENGTHS(X) \
  X(4) X(6) X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512)
inline bool fft_length_supported(int n) {
  switch (n) {
#define TBFP_CASE(L) case L:
    TBFP_FFT_LENGTHS(TBFP_CASE)
#undef TBFP_CASE
    return true;
    default:
      return false;
  }
}

// --- tile geometry (shared by the host launchers and the kernels) -----------
// Asynchronous 16-byte copy global -> shared (cp.async, no register staging):
// a thread issues all its copies back to back and waits once.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// all but the N most recently committed groups complete
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Maximum of two non-negative values that lets a NaN win (fmax would drop it,
// and a NaN must reach the host): the bit patterns of non-negative doubles
// order like their values, and a NaN with its sign cleared lies above +Inf.
// The sign is cleared on the bits, not by fabs: a NaN that the device makes
// (Inf - Inf, 0 * Inf) can keep its sign bit through fabs, and a negative
// pattern would lose to every finite value.
__device__ __forceinline__ double abs_bits(double v) {
  return __longlong_as_double(__double_as_longlong(v) & 0x7fffffffffffffffLL);
}
__device__ __forceinline__ double nanmax_nonneg(double a, double b) {
  return __longlong_as_double(max(__double_as_longlong(abs_bits(a)), __double_as_longlong(abs_bits(b))));
}

constexpr int kNT = 256;  // threads per CTA of the transform kernels (8 warps)
constexpr int kNW = kNT / 32;
constexpr int kWPB = 4;   // warps per CTA of the tridiagonal kernel

// Each warp transforms its own sequences (rows of x, columns of z) with
// __syncwarp only, 8 complex values per lane (16 for length 512).
// Sequences per warp: the largest power of two keeping n*spw <= 256, or 1.
__host__ __device__ constexpr int ct_lognb(int n) { return n >= 256 ? 0 : ct_log2(256 / n); }
// Row stride of an x tile (complex slots): holds pad8(M)+1 slots; with nb rows
// per warp interleaved in a phase of 8 lanes, rows must land on distinct
// 16-byte bank groups: stride = (8/nb)*odd (mod 8) for nb < 8, odd for nb >= 8.
__host__ __device__ constexpr int x_row_stride(int M) {
  const int nb = 1 << ct_lognb(M);
  int ld = pad8(M) + 1;
  if (nb == 1) return ld;
  const int want = nb >= 8 ? 1 : 8 / nb;  // required residue pattern
  while (!((ld % 8) % want == 0 && ((ld % 8) / want) % 2 == 1)) ++ld;
  return ld;
}
// Row stride of a z tile: the tile's 8*nb columns plus a skew for small nb.
__host__ __device__ constexpr int z_row_stride(int nz) {
  const int nb = 1 << ct_lognb(nz);
  return 8 * nb + (nb <= 4 ? nb : 0);
}
__host__ __device__ constexpr int fftx_rows_per_cta(int M) { return kNW << ct_lognb(M); }
__host__ __device__ constexpr int fftz_cols_per_cta(int nz) { return kNW << ct_lognb(nz); }
// dynamic shared memory: tile + twiddle table, elements of esz bytes (16 for
// double2, 8 for float2)
__host__ __device__ constexpr size_t fftx_smem_bytes(int M, size_t esz = 16) {
  return ((size_t)fftx_rows_per_cta(M) * x_row_stride(M) + M) * esz;
}
__host__ __device__ constexpr size_t fftz_smem_bytes(int nz, size_t esz = 16) {
  return ((size_t)z_row_stride(nz) * (pad8(nz - 1) + 1) + nz) * esz;
}
// y systems: one lane owns T = ceil(ny/32) consecutive rows; a warp holds two
// complex right-hand sides and two real coefficients per row
inline int tri_rows_per_lane(int ny) { return (ny + 31) / 32; }
inline size_t tridiag_smem_bytes(int ny) {
  return (size_t)kWPB * 33 * tri_rows_per_lane(ny) * (2 * sizeof(double2) + 2 * sizeof(double));
}

// Pass-ordered twiddle table of a length-n transform (fft_smem.cuh), n
// entries (the last R_0 unused), evaluated in extended precision.
inline void fft_pass_twiddles(int n, double2 *out) {
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int e = 0; e < n; ++e) out[e] = make_double2(0.0, 0.0);
  const int r0 = ct_rad(n, 0);
  for (int p = 1; p < ct_nrad(n); ++p) {
    const int R = ct_rad(n, p), NS = ct_ns(n, p);
    for (int k0 = 0; k0 < NS; ++k0)
      for (int r = 1; r < R; ++r) {
        const long double a = 2.0L * pi * (long double)(k0 * r) / (long double)(NS * R);
        out[NS - r0 + k0 * (R - 1) + (r - 1)] = make_double2((double)cosl(a), (double)(-sinl(a)));
      }
  }
}
// exp(-2*pi*i*m/n), m = 0..n-1 (the r2c/c2r post-processing factors for n = nx).
inline void fft_unit_twiddles(int n, double2 *out) {
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int m = 0; m < n; ++m) {
    const long double a = 2.0L * pi * (long double)m / (long double)n;
    out[m] = make_double2((double)cosl(a), (double)(-sinl(a)));
  }
}

// Error text returned by tbfp_last_error(NULL) (defined in tbfp_api.cu).
void set_global_error(const std::string &msg);

// Kernel launchers.  The x launchers take twx (fft_unit_twiddles(nx)) and tpx
// (fft_pass_twiddles(nx/2)); the z launcher takes tpz (fft_pass_twiddles(nz)).
cudaError_t prepare_kernels();  // raises the shared-memory limits; once per device
void launch_recip(const double *rho, double *irho, long n, cudaStream_t st);
void launch_fftx_fwd_from_s(const double *s, Lay Ls, const GridK &g, const double2 *twx, const double2 *tpx,
                            double2 *spec, cudaStream_t st);
void launch_rhs(const RhsArgs &ra, bool has_st, const GridK &g, double *s, Lay Ls, cudaStream_t st);
// the correction with its inputs staged by TMA; false when the arrays do not
// suit a tensor map (then nothing is launched)
bool launch_correct_div_tma(const CorrArgs &ca, const GridK &g, unsigned long long *maxdiv, int sms,
                            cudaStream_t st);
cudaError_t prepare_correct_tma_kernel();
// the right-hand side computed into the forward x transform's tiles (s is not stored)
void launch_rhs_fftx(const RhsArgs &ra, bool has_st, const GridK &g, const double2 *twx, const double2 *tpx,
                     double2 *spec, cudaStream_t st);
void launch_fftz(double2 *spec, const GridK &g, const double2 *tpz, bool inverse, cudaStream_t st);
void launch_fftz(float2 *spec, const GridK &g, const float2 *tpz, bool inverse, cudaStream_t st);
void launch_tridiag(double2 *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                    const double *ap, const double *dyf, double mean_c, double nxnz, cudaStream_t st);
// FP64 spectrum with a two-word control block (zero before the first launch;
// every launch leaves it zero) and the device's SM count: the persistent
// prefetching forms for 257 <= ny <= 512 (one warp per pair up to 384 rows,
// a two-warp team per pair above), k_tridiag_t otherwise
void launch_tridiag(double2 *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                    const double *ap, const double *dyf, double mean_c, double nxnz, unsigned *ctl, int sms,
                    const double *pinf, cudaStream_t st);
// the pinned (0,0) system's elimination factors (2*(ny-1) doubles) for the
// persistent forms; pinf == nullptr makes them compute the factors inline
void launch_pin_factors(const double *am, const double *ap, const double *lamx, const double *lamz, int ny, double *f,
                        cudaStream_t st);
void launch_tridiag(float2 *spec, const GridK &g, const double *lamx, const double *lamz, const double *am,
                    const double *ap, const double *dyf, double mean_c, double nxnz, cudaStream_t st);
void launch_fftx_inv(const double2 *spec, double *psi, Lay Lp, int hd, const GridK &g, const double2 *twx,
                     const double2 *tpx, double scale, cudaStream_t st);
// mixed path: FP32 spectrum, psi = (accumulate ? psi : 0) + scale * c2r(spec)
void launch_fftx_inv(const float2 *spec, double *psi, Lay Lp, int hd, const GridK &g, const float2 *twx,
                     const float2 *tpx, double scale, bool accumulate, cudaStream_t st);
void launch_fftx_fwd(const XSrc &src, bool residual, const GridK &g, const double2 *twx, const double2 *tpx,
                     double2 *spec, cudaStream_t st);
void launch_fftx_fwd(const XSrc &src, bool residual, const GridK &g, const float2 *twx, const float2 *tpx,
                     float2 *spec, cudaStream_t st);
// Mixed-precision loop control (MixedCtl): params clears acc[0..3] and starts
// the count at one solve; decide reads acc[1] (sum s^2) and acc_r[0..1], writes
// ctl and clears acc_r for the next pass; with cond it also sets the WHILE
// condition of the graph it runs in (1: run another sweep).
void launch_mixed_params(MixedCtl *ctl, double *acc, double tol, double dtol, double dscale, int max_iter,
                         cudaStream_t st);
void launch_mixed_decide(MixedCtl *ctl, const double *acc, double *acc_r, cudaGraphConditionalHandle cond,
                         bool use_cond, cudaStream_t st);
void launch_correct_div(const CorrArgs &ca, bool has_st, const GridK &g, unsigned long long *maxdiv,
                        cudaStream_t st);
void launch_correct_inplace(const CorrArgs &ca, bool has_st, const GridK &g, cudaStream_t st);
void launch_div(const double *ux, const double *uy, const double *uz, Lay Lux, Lay Luy, Lay Luz, const GridK &g,
                unsigned long long *maxdiv, cudaStream_t st);

// Material properties (updateMaterialProps + smoothVF, tbfp_vof.cu).  Distance
// tables of the two interpolations (interpolation.f90:188-276), per direction:
// cellToVertex at vertex i = 0..n: c*1 = x(i+1)-xv(i) (x) / yv(j)-y(j) (y) /
// z(k+1)-zv(k) (z), c*2 = xv(i)-x(i) / y(j+1)-yv(j) / zv(k)-z(k), h* = x(i+1)-x(i);
// vertexToCell at cell i = 1..n (table index i-1): v*1 = xv(i)-x(i) / y(j)-yv(j-1) /
// zv(k)-z(k), v*2 = x(i)-xv(i-1) / yv(j)-y(j) / z(k)-zv(k-1), V* = xv(i)-xv(i-1).
struct VofTab {
  const double *cx1, *cx2, *hx, *cy1, *cy2, *hy, *cz1, *cz2, *hz;
  const double *vx1, *vx2, *Vx, *vy1, *vy2, *Vy, *vz1, *vz2, *Vz;
};
// qv: (nx+1)(ny+1)(nz+1) scratch; c, cs, rho, mu laid out by L (n elements, halo hd)
void launch_material_props(const VofTab &t, const double *c, double *cs, double *rho, double *mu, double *qv, Lay L,
                           long n, int nx, int ny, int nz, int hd, double rhol, double rhog, double mul, double mug,
                           cudaStream_t st);
// Separable form of one cell -> vertex -> cell pass, per direction and cell
// i = 1..n (table index i-1): out(i) = m(i) in(i-1) + z(i) in(i) + p(i) in(i+1).
struct VofSep {
  const double *xm, *x0, *xp, *ym, *y0, *yp, *zm, *z0, *zp;
};
// the same for halo 1 in two fused launches; tmp: a scratch field laid out by L
void launch_material_props_fused(const VofSep &w, const double *c, double *cs, double *rho, double *mu, double *tmp,
                                 Lay L, int nx, int ny, int nz, double rhol, double rhog, double mul, double mug,
                                 cudaStream_t st);
// One fused smoothing pass (halo 1); rho, mu non-NULL: the final pass with the
// properties.  zimg = false on a slab: no periodic z ghost images.
void launch_smooth_pass(const VofSep &w, const double *in, double *out, double *rho, double *mu, Lay L, int nx, int ny,
                        int nz, double rhol, double rhog, double mul, double mug, bool zimg, cudaStream_t st);

// Momentum predictor (tbfp_momentum.cu).  Spacings indexed by the Fortran
// index: dxf, dxc, dzf, dzc over 0..n+1 (x and z periodic), dyf over 1..ny and
// dyc over 1..ny+1 (tables of ny+2 entries).
// dyf and the reciprocals of every spacing, Fortran index 0..n+1 -> [index]
struct MomentumTabs {
  const double *dyf, *rdxf, *rdxc, *rdyf, *rdyc, *rdzf, *rdzc;
};
// phi: the new fluxes (written), prev: the previous call's; dense over the
// equation boxes ux (0:nx,1:ny,1:nz), uy (1:nx,1:ny-1,1:nz), uz (1:nx,1:ny,0:nz).
// u_out NULL: u is updated in place; else u is read only and u_out (no alias
// of u) receives the update on the boxes and u's values elsewhere.
void launch_momentum(const MomentumTabs &t, double *ux, double *uy, double *uz, const double *c, const double *mu,
                     const double *rho, const double *const *st, Lay Lux, Lay Luy, Lay Luz, Lay Lc, const Lay *Lst,
                     double *const phi[3], const double *const prev[3], int nx, int ny, int nz, int scheme, double dt,
                     double alpha, double gamma, double xi, double rho0, double fs, double gch, double g, int hdu,
                     int hdc, double *const *u_out, cudaStream_t st_);

// updateBoundariesV for the channel: the y-wall spacings of setMetrics (dhb,
// dhi at the bottom and top) and the wall values, per component ux, uy, uz
struct WallTabs {
  double hb[3], hi[3], tb[3], ti[3], bb[3], bt[3];
};
// slab: a rank of a z-split channel; its z ghost planes and uz's plane k = 0
// come from the neighbours (the caller's exchange), so only the wall ghosts
// and the x halos of the planes ks..nz are written here.
void launch_boundaries_v(const WallTabs &w, double *ux, double *uy, double *uz, Lay Lux, Lay Luy, Lay Luz, int nx,
                         int ny, int nz, int hd, bool slab, cudaStream_t st);

// Flow control: mode 0 sums 0.5*(rho(i+1)+rho(i))*Vsx, mode 1 sums ux*Vsx over
// i = 0..nx-1, j = 1..ny, k = 1..nz into *out (device); part holds ny*nz
// partials.  dxc, dyf, dzf: device tables of dxc(1..nx), dyf(1..ny), dzf(1..nz).
void launch_face_sum(int mode, const double *f, Lay L, const double *dxc, const double *dyf, const double *dzf, int nx,
                     int ny, int nz, double *part, double *out, cudaStream_t st);
void launch_add_ux(double *ux, Lay L, int nx, int ny, int nz, double uf, cudaStream_t st);

// MG_MODE source/beta (computeSource MG, computeBeta) and addPressureGrad.
// idxc, idzc: 1/dxc(i), 1/dzc(k) for Fortran i = 1..nx+1 (0-based tables).
void launch_mg_source_beta(const double *ux, const double *uy, const double *uz, Lay Lux, Lay Luy, Lay Luz,
                           const double *rho, Lay Lrho, const GridK &g, double dta, double *q, Lay Lq, double *beta,
                           cudaStream_t st);
void launch_add_pressure_grad(const double *uxi, const double *uyi, const double *uzi, double *uxo, double *uyo,
                              double *uzo, Lay Lux, Lay Luy, Lay Luz, const double *p, Lay Lp, const double *rho,
                              Lay Lrho, const GridK &g, const double *idxc, const double *idzc, double dta,
                              cudaStream_t st);

// Surface tension (tbfp_surface.cu): grid constants; dyf[0..ny-1] = dyf(1..ny),
// dyc[0..ny] = dyc(1..ny+1), yf[0..ny] the y face positions as sequential sums
// of dyf from yf[0] = 0 (device tables).
struct StGrid {
  int nx, ny, nz;
  double dx, dz;
  const double *dyf, *dyc, *yf;
};
// c: volume fraction (layout Lc); cp, fl, kap: dense scratch (c after the
// promotion of full interface cells, class bits 1 mixed / 2 full, curvature);
// kap_out (NULL or layout Lk, nk elements); sx, sy, sz: the three staggered
// st arrays (nsx, nsy, nsz elements).
void launch_surface_tension(const double *c, Lay Lc, const StGrid &g, double eps, double sigma, double *cp,
                            unsigned char *fl, double *kap, double *kap_out, Lay Lk, long nk, double *sx, Lay Lx,
                            long nsx, double *sy, Lay Ly, long nsy, double *sz, Lay Lz, long nsz, cudaStream_t st);

// The all-to-all chunks of a channel split over ranks (z slabs <-> kx slabs).
// zs[0..n]: the z-slab starts of the n ranks (zs[n] = nz of the channel).
constexpr int kSlabMaxRanks = 64;
struct SlabParts {
  int n;
  int zs[kSlabMaxRanks + 1];
};
// to_x: chunks[p] = [nkx_loc][nz_p][ny] in rank order -> S_x[nkx_loc][nz][ny];
// else the inverse (S_x -> the chunks for every destination).  g: the slab
// handle's spectral grid (nkx = nkx_loc, nz = the channel's nz).
void launch_slab_chunks(const GridK &g, const SlabParts &parts, bool to_x, const double2 *src, double2 *dst,
                        cudaStream_t st);

// per-file parts of prepare_kernels()
cudaError_t prepare_xfft_kernels();
cudaError_t prepare_yz_kernels();

}  // namespace tbfp
