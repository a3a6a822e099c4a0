// tbfp_solve_fps_noalloc: the solveFPS path for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc: a code whose device memory belongs to
// a pool that another runtime owns, or a framework that forbids allocation on
// its solver path (a Fortran driver that hands over device arrays it allocated
// itself is the typical case).  This entry point takes the grid descriptor and
// the caller's device arrays and allocates nothing: its work spectrum and its
// set-up tables live in one file-scope __device__ array of fixed size that
// every GPU loading the library holds until the process exits.
//
// * Limits: (nx/2+1)*ny*nz <= TBFP_NOALLOC_MAX_SPECTRUM complex entries
//   (64 MiB), nx <= 4096, ny <= 2048, nz <= 2048; larger sizes are rejected
//   with TBFP_EUNSUPPORTED and a message.
// * Set-up: the first call on a device looks up the array's device address
//   with cudaGetSymbolAddress (with that device current) and caches it; make
//   that first call before any stream capture.
// * Sharing: every call on a device uses the same array, which keeps the last
//   call's contents.  Nothing needs to start at zero (the forward transform
//   overwrites every spectrum entry before it is read; the tables are rewritten
//   by every call), but calls that overlap on the GPU -- from two host threads,
//   or on two streams -- race on the array and must be serialised by the caller.
//   (Within one process the host side of this function holds a lock and
//   synchronises its stream before returning, which serialises its own calls.)
// * The caller's current device is the same after the call as before it.
// * Errors: the status code, with the message in tbfp_last_error(NULL).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "tbfp.h"
#include "tbfp_kernels.cuh"

using namespace tbfp;

namespace {

constexpr int kNxMax = 4096, kNyMax = 2048, kNzMax = 2048;
constexpr long kSpecMax = TBFP_NOALLOC_MAX_SPECTRUM;
// region sizes rounded up to 32 doubles (256 bytes), so every region is aligned
constexpr long rup(long n) { return (n + 31) / 32 * 32; }
// table layout (in doubles) inside the scratch array, after the spectrum
constexpr long kOffLamx = 2 * kSpecMax;                   // nx/2+1
constexpr long kOffLamz = kOffLamx + rup(kNxMax / 2 + 1); // nz
constexpr long kOffAm = kOffLamz + rup(kNzMax);           // ny
constexpr long kOffAp = kOffAm + rup(kNyMax);             // ny
constexpr long kOffDyf = kOffAp + rup(kNyMax);            // ny
constexpr long kOffIdyf = kOffDyf + rup(kNyMax);          // ny
constexpr long kOffIdyc = kOffIdyf + rup(kNyMax);         // ny+1
constexpr long kOffIdxf = kOffIdyc + rup(kNyMax + 1);     // nx
constexpr long kOffIdzf = kOffIdxf + rup(kNxMax);         // nz
constexpr long kOffTwx = kOffIdzf + rup(kNzMax);          // nx complex: r2c/c2r factors
constexpr long kOffTpx = kOffTwx + rup(2 * kNxMax);       // nx/2 complex: pass twiddles of nx/2
constexpr long kOffTpz = kOffTpx + rup(kNxMax);           // nz complex: pass twiddles of nz
constexpr long kTableEnd = kOffTpz + rup(2 * kNzMax);
constexpr long kTableDoubles = kTableEnd - kOffLamx;

// The scratch array: spectrum, then the set-up tables.  256-byte aligned so
// every carved region (all at even double offsets) is 16-byte aligned.
static __device__ __align__(256) double g_noalloc_scratch[kTableEnd];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double *g_scratch_ptr[kMaxDevices] = {};
// host staging of the tables (no allocation per call)
double g_host_tables[kTableDoubles];

int fail(int code, const std::string &msg) {
  set_global_error(msg);  // read back with tbfp_last_error(NULL)
  return code;
}

int solve_fps_noalloc(const tbfp_desc *d, const double *s, double *psi);

}  // namespace

// The caller's current device is restored on every return path.
extern "C" int tbfp_solve_fps_noalloc(const tbfp_desc *d, const double *s, double *psi) {
  int prev = -1;
  const bool have_prev = cudaGetDevice(&prev) == cudaSuccess;
  const int rc = solve_fps_noalloc(d, s, psi);
  if (have_prev) {
    int now = -1;
    if (cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
  }
  return rc;
}

namespace {

int solve_fps_noalloc(const tbfp_desc *d, const double *s, double *psi) {
  set_global_error("");
  if (!d || !s || !psi) return fail(TBFP_ENULL, "tbfp_solve_fps_noalloc: NULL argument");
  if (d->nx < 4 || d->ny < 4 || d->nz < 2 || (d->nx % 2) != 0 || d->hd_psi < 1)
    return fail(TBFP_EINVAL, "tbfp_solve_fps_noalloc: need nx even >= 4, ny >= 4, nz >= 2, hd_psi >= 1");
  if (!d->dxf || !d->dyf || !d->dyc || !d->dzf)
    return fail(TBFP_ENULL, "tbfp_solve_fps_noalloc: a grid metric array is NULL");
  if (!(d->dx_fft > 0.0) || !(d->dz_fft > 0.0))
    return fail(TBFP_EINVAL, "tbfp_solve_fps_noalloc: dx_fft and dz_fft must be positive");
  const int nx = d->nx, ny = d->ny, nz = d->nz, nkx = nx / 2 + 1;
  if (nx <= kNxMax && ny <= kNyMax && nz <= kNzMax) {  // the same metric checks as tbfp_create
    for (int i = 0; i < nx; ++i)
      if (!(d->dxf[i] > 0.0)) return fail(TBFP_EINVAL, "tbfp_solve_fps_noalloc: dxf must be positive");
    for (int j = 0; j < ny; ++j)
      if (!(d->dyf[j] > 0.0)) return fail(TBFP_EINVAL, "tbfp_solve_fps_noalloc: dyf must be positive");
    for (int j = 0; j <= ny; ++j)
      if (!(d->dyc[j] > 0.0)) return fail(TBFP_EINVAL, "tbfp_solve_fps_noalloc: dyc must be positive");
    for (int k = 0; k < nz; ++k)
      if (!(d->dzf[k] > 0.0)) return fail(TBFP_EINVAL, "tbfp_solve_fps_noalloc: dzf must be positive");
  }
  const long R = (long)ny * nz;
  if (nx > kNxMax || ny > kNyMax || nz > kNzMax || (long)nkx * R > kSpecMax)
    return fail(TBFP_EUNSUPPORTED,
                "tbfp_solve_fps_noalloc: grid exceeds the static scratch ((nx/2+1)*ny*nz <= 4194304, "
                "nx <= 4096, ny <= 2048, nz <= 2048); use tbfp_create/tbfp_solve_fps_dev");
  if (!fft_length_supported(nx / 2) || !fft_length_supported(nz))
    return fail(TBFP_EUNSUPPORTED, "tbfp_solve_fps_noalloc: nx/2 and nz must be 2^a or 3*2^a between 4 and 512");
  if (tridiag_smem_bytes(ny) > 227 * 1024)
    return fail(TBFP_EUNSUPPORTED, "tbfp_solve_fps_noalloc: ny too large for the shared-memory tiles");

  int dev = 0;
  if (d->device >= 0) {
    if (cudaSetDevice(d->device) != cudaSuccess) return fail(TBFP_ENODEVICE, "tbfp_solve_fps_noalloc: bad device");
    dev = d->device;
  } else if (cudaGetDevice(&dev) != cudaSuccess) {
    return fail(TBFP_ENODEVICE, "tbfp_solve_fps_noalloc: no CUDA device");
  }
  if (dev < 0 || dev >= kMaxDevices) return fail(TBFP_ENODEVICE, "tbfp_solve_fps_noalloc: device ordinal too large");

  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {  // once per device, with that device current
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(TBFP_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    e = prepare_kernels();
    if (e != cudaSuccess) return fail(TBFP_ECUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<double *>(p);
  }
  double *base = g_scratch_ptr[dev];

  // set-up tables (fastPoissonSolver.f90:215-276), staged on the host
  double *t = g_host_tables;
  auto T = [&](long off) { return t + (off - kOffLamx); };
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < nkx; ++i) T(kOffLamx)[i] = 2.0 * (std::cos(((double)i * 2.0 * pi) / nx) - 1.0) / (d->dx_fft * d->dx_fft);
  for (int k = 0; k < nz; ++k) {  // even in k, as in tbfp_create
    const int kk = k < nz - k ? k : nz - k;
    T(kOffLamz)[k] = 2.0 * (std::cos(((double)kk * 2.0 * pi) / nz) - 1.0) / (d->dz_fft * d->dz_fft);
  }
  for (int j = 0; j < ny; ++j) {
    T(kOffAm)[j] = 1.0 / (d->dyc[j] * d->dyf[j]);
    T(kOffAp)[j] = 1.0 / (d->dyc[j + 1] * d->dyf[j]);
    T(kOffDyf)[j] = d->dyf[j];
    T(kOffIdyf)[j] = 1.0 / d->dyf[j];
  }
  T(kOffAm)[0] = 0.0;
  T(kOffAp)[ny - 1] = 0.0;
  for (int j = 0; j <= ny; ++j) T(kOffIdyc)[j] = 1.0 / d->dyc[j];
  for (int i = 0; i < nx; ++i) T(kOffIdxf)[i] = 1.0 / d->dxf[i];
  for (int k = 0; k < nz; ++k) T(kOffIdzf)[k] = 1.0 / d->dzf[k];
  fft_unit_twiddles(nx, reinterpret_cast<double2 *>(T(kOffTwx)));
  fft_pass_twiddles(nx / 2, reinterpret_cast<double2 *>(T(kOffTpx)));
  fft_pass_twiddles(nz, reinterpret_cast<double2 *>(T(kOffTpz)));
  double sVg = d->s_Vg;
  if (!(sVg > 0.0)) {
    sVg = 0.0;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) sVg += d->dxf[i] * d->dyf[j] * d->dzf[k];
  }
  cudaStream_t st = static_cast<cudaStream_t>(d->stream);
  cudaError_t e = cudaMemcpyAsync(base + kOffLamx, g_host_tables, sizeof(double) * kTableDoubles,
                                  cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return fail(TBFP_ECUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));

  GridK g{};
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.nkx = nkx;
  g.M = nx / 2;
  g.R = R;
  g.idxf1 = 1.0 / d->dxf[0];
  g.idzf1 = 1.0 / d->dzf[0];
  g.idxc1 = d->dxc ? 1.0 / d->dxc[0] : 0.0;
  g.idzc1 = d->dzc ? 1.0 / d->dzc[0] : 0.0;
  g.idyf = base + kOffIdyf;
  g.idyc = base + kOffIdyc;
  g.idxf = base + kOffIdxf;
  g.idzf = base + kOffIdzf;
  Lay Lp;
  Lp.ilo = 1 - d->hd_psi;
  Lp.jlo = 1 - d->hd_psi;
  Lp.klo = 1 - d->hd_psi;
  Lp.sj = nx + 2 * d->hd_psi;
  Lp.sk = Lp.sj * (ny + 2 * d->hd_psi);
  double2 *spec = reinterpret_cast<double2 *>(base);
  const double2 *twx = reinterpret_cast<const double2 *>(base + kOffTwx);
  const double2 *tpx = reinterpret_cast<const double2 *>(base + kOffTpx);
  const double2 *tpz = reinterpret_cast<const double2 *>(base + kOffTpz);

  launch_fftx_fwd_from_s(s, Lp, g, twx, tpx, spec, st);
  launch_fftz(spec, g, tpz, false, st);
  launch_tridiag(spec, g, base + kOffLamx, base + kOffLamz, base + kOffAm, base + kOffAp, base + kOffDyf,
                 d->dx_fft * d->dz_fft / sVg, (double)nx * (double)nz, st);
  launch_fftz(spec, g, tpz, true, st);
  launch_fftx_inv(spec, psi, Lp, d->hd_psi, g, twx, tpx, 1.0 / ((double)nx * (double)nz), st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(TBFP_ECUDA, std::string("tbfp_solve_fps_noalloc launch: ") + cudaGetErrorString(e));
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail(TBFP_ECUDA, std::string("tbfp_solve_fps_noalloc: ") + cudaGetErrorString(e));
  return TBFP_OK;
}

}  // namespace
