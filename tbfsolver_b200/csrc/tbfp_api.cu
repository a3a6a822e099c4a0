// C ABI of the projection library: handle lifecycle, set-up tables and the
// orchestration of the kernels in tbfp_kernels.cu.  See include/tbfp.h.
#include <cuda_runtime.h>
#include <sys/stat.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "tbfp.h"
#include "tbfp_kernels.cuh"
#include "tbfp_mg.cuh"

using namespace tbfp;

namespace {

thread_local std::string g_create_error;

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
};

}  // namespace

namespace tbfp {
void set_global_error(const std::string &msg) { g_create_error = msg; }
}  // namespace tbfp

// An executable graph of the mixed refinement for one (s, psi) pair of arrays.
struct MixedGraph {
  const double *s = nullptr;
  double *psi = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long used = 0;
};

struct tbfp_handle {
  int nx = 0, ny = 0, nz = 0, nkx = 0;
  long R = 0;
  int hd_psi = 1, hd_u = 2, hd_rho = 1, hd_st = 1;
  long long wait_cycles = kDefaultWaitCycles;  // bound on each copy wait of the staged correction
  Lay Lpsi{}, Lux{}, Luy{}, Luz{}, Lrho{}, Lst[3]{};
  size_t n_psi = 0, n_ux = 0, n_uy = 0, n_uz = 0, n_rho = 0, n_st[3]{};
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  unsigned flags = 0;
  int precision = TBFP_FP64;
  double tol = 1e-10;
  int max_iter = 8;

  GridK g{};
  double s_Vg = 0.0, dx_fft = 0.0, dz_fft = 0.0, mean_c = 0.0, nxnz = 0.0, scale = 0.0;

  // device tables
  double *d_lamx = nullptr, *d_lamz = nullptr, *d_am = nullptr, *d_ap = nullptr, *d_dyf = nullptr;
  double *d_idyf = nullptr, *d_idyc = nullptr, *d_idxf = nullptr, *d_idzf = nullptr;
  double *d_idxc = nullptr, *d_idzc = nullptr;  // 1/dxc(1..nx+1), 1/dzc(1..nz+1) (MG_MODE correction)
  double2 *d_twx = nullptr;                     // exp(-2 pi i m/nx), the r2c/c2r factors
  double2 *d_tpx = nullptr, *d_tpz = nullptr;  // pass-ordered twiddles of lengths nx/2 and nz
  float2 *d_twx32 = nullptr, *d_tpx32 = nullptr, *d_tpz32 = nullptr;  // FP32 copies (TBFP_MIXED)
  double *d_acc = nullptr;  // reductions of the residual passes: [0] sum s dyf, [1] sum s^2, [2] sum r^2,
                            // [3] max|s - L psi| (bits)
  MixedCtl *d_ctl = nullptr;  // device-side control of the mixed refinement loop
  cudaStream_t cap = nullptr, cap_body = nullptr;  // capture streams of the mixed-refinement graphs
  MixedGraph mgr[4];          // executable refinement graphs, least recently used evicted
  unsigned long long mgr_tick = 0;
  bool mgr_off = false;       // the runtime refused the conditional graph: host-driven loop
  double idx2 = 0.0, idz2 = 0.0, ctop_scale = 0.0;
  tbfp_stats last{};        // statistics of the last solve or projection
  bool slab = false;        // one rank's slab of a channel (tbfp_slab_create)
  GridK gs{};               // slab form: the spectral stage's grid (local kx, all kz)
  int nz_total = 0;
  // material properties (tbfp_vof_setup)
  bool vof = false;
  VofTab vt{};
  VofSep vsep{};
  double *d_qv = nullptr;                     // vertex scratch, (nx+1)(ny+1)(nz+1)
  double rhol = 0.0, rhog = 0.0, mul = 0.0, mug = 0.0;
  double *h_vof[4] = {nullptr, nullptr, nullptr, nullptr};  // c, cs, rho, mu for tbfp_material_props
  // momentum predictor (tbfp_momentum_setup)
  bool mom = false;
  int mom_scheme = 2;
  double mom_gch = 0.0, mom_g = 0.0;
  MomentumTabs mt{};
  double *d_phi[2][3] = {};  // flux history: [cur][component], swapped per call
  int phi_cur = 0;
  size_t n_phi[3] = {0, 0, 0};
  double *h_mom[2] = {nullptr, nullptr};  // c, mu copies for tbfp_momentum_predictor
  WallTabs wt{};                           // updateBoundariesV wall spacings and values
  // flow control: dxc(1..nx), dyf(1..ny), dzf(1..nz) on the device, ny*nz row partials + the sum
  double *d_fdxc = nullptr, *d_fdyf = nullptr, *d_fdzf = nullptr, *d_fpart = nullptr;
  // surface tension (tbfp_surface_tension): tables and dense scratch, made on first use
  double *d_st_dyc = nullptr, *d_st_yf = nullptr, *d_st_cp = nullptr, *d_st_kap = nullptr, *h_kap = nullptr;
  unsigned char *d_st_fl = nullptr;
  MgSolver *mg = nullptr;   // MG_MODE hierarchy (tbfp_pcg_setup)
  std::vector<double> mdxf, mdxc, mdyf, mdyc, mdzf, mdzc;  // caller's metrics, kept for tbfp_pcg_setup
  double *h_beta = nullptr, *h_q = nullptr;                // device copies for tbfp_pcg_solve
  // work
  double2 *d_spec = nullptr;
  double *d_s = nullptr;  // split right-hand side, laid out like psi
  double *d_irho = nullptr;
  unsigned long long *d_maxdiv = nullptr;
  unsigned *d_tri_ctl = nullptr;  // ticket and retire counts of the persistent y solve (zero between launches)
  double *d_pinf = nullptr;       // elimination factors of the pinned (0,0) y system
  int sms = 0;                    // SMs of the handle's device
  // device copies used by the host-pointer entry points
  double *h_ux = nullptr, *h_uy = nullptr, *h_uz = nullptr;
  double *h_rho = nullptr, *h_pn = nullptr, *h_pnm1 = nullptr, *h_psi = nullptr, *h_s = nullptr;
  double *h_st[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evs[TBFP_NSTAGES + 1] = {};
  size_t dev_bytes = 0;
  std::vector<void *> allocs;
  std::string err;
};

namespace {

int set_err(tbfp_handle *h, int code, const std::string &msg) {
  if (h) h->err = msg;
  else g_create_error = msg;
  return code;
}

int cuda_err(tbfp_handle *h, cudaError_t e, const char *where) {
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorMemoryAllocation) return set_err(h, TBFP_ENOMEM, m);
  return set_err(h, TBFP_ECUDA, m);
}

#define TBFP_CK(h, call)                                  \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return cuda_err((h), _e, #call); \
  } while (0)

template <typename T>
int dev_alloc(tbfp_handle *h, T **p, size_t count) {
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16);
  if (e != cudaSuccess) return cuda_err(h, e, "cudaMalloc");
  h->allocs.push_back(q);
  h->dev_bytes += count * sizeof(T);
  *p = static_cast<T *>(q);
  return TBFP_OK;
}

template <typename T>
int upload(tbfp_handle *h, T **p, const std::vector<T> &v) {
  int rc = dev_alloc(h, p, v.size());
  if (rc) return rc;
  TBFP_CK(h, cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return TBFP_OK;
}

// Fortran array layout: interior lower bounds lo, halo hd.
Lay make_lay(int ilo, int jlo, int klo, int ni, int nj, int hd, size_t *count, int nk) {
  Lay L;
  L.ilo = ilo - hd;
  L.jlo = jlo - hd;
  L.klo = klo - hd;
  const long ei = ni + 2 * hd, ej = nj + 2 * hd, ek = nk + 2 * hd;
  L.sj = ei;
  L.sk = ei * ej;
  *count = (size_t)(ei * ej * ek);
  return L;
}

std::vector<double2> unit_twiddles(int n) {
  std::vector<double2> t(n);
  fft_unit_twiddles(n, t.data());
  return t;
}
std::vector<double2> pass_twiddles(int n) {
  std::vector<double2> t(n);
  fft_pass_twiddles(n, t.data());
  return t;
}
std::vector<double> inv_of(const double *a, int n) {
  std::vector<double> t(n);
  for (int i = 0; i < n; ++i) t[i] = 1.0 / a[i];
  return t;
}
std::vector<float2> to_f32(const std::vector<double2> &v) {
  std::vector<float2> t(v.size());
  for (size_t i = 0; i < v.size(); ++i) t[i] = make_float2((float)v[i].x, (float)v[i].y);
  return t;
}

int ensure_host_bufs(tbfp_handle *h, bool st) {
  if (!h->h_ux) {
    int rc;
    if ((rc = dev_alloc(h, &h->h_ux, h->n_ux))) return rc;
    if ((rc = dev_alloc(h, &h->h_uy, h->n_uy))) return rc;
    if ((rc = dev_alloc(h, &h->h_uz, h->n_uz))) return rc;
    if ((rc = dev_alloc(h, &h->h_rho, h->n_rho))) return rc;
    if ((rc = dev_alloc(h, &h->h_pn, h->n_psi))) return rc;
    if ((rc = dev_alloc(h, &h->h_pnm1, h->n_psi))) return rc;
    if ((rc = dev_alloc(h, &h->h_psi, h->n_psi))) return rc;
    if ((rc = dev_alloc(h, &h->h_s, h->n_psi))) return rc;
  }
  if (st && !h->h_st[0]) {
    for (int c = 0; c < 6; ++c) {
      int rc = dev_alloc(h, &h->h_st[c], h->n_st[c % 3]);
      if (rc) return rc;
    }
  }
  return TBFP_OK;
}

int h2d(tbfp_handle *h, double *dst, const double *src, size_t n) {
  TBFP_CK(h, cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  return TBFP_OK;
}
int d2h(tbfp_handle *h, double *dst, const double *src, size_t n) {
  TBFP_CK(h, cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return TBFP_OK;
}

int finish(tbfp_handle *h, const char *where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(h, e, where);
  if (!(h->flags & TBFP_FLAG_ASYNC)) {
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, where);
  }
  return TBFP_OK;
}

bool st_present(const double *const *st_n, const double *const *st_nm1) {
  return st_n != nullptr && st_nm1 != nullptr;
}

RhsArgs rhs_args(tbfp_handle *h, const double *ux, const double *uy, const double *uz, const double *psi_n,
                 const double *psi_nm1, const double *const *st_n, const double *const *st_nm1, double dt,
                 double alpha, double rho0) {
  RhsArgs a{};
  a.ux = ux;
  a.uy = uy;
  a.uz = uz;
  a.irho = h->d_irho;
  a.pn = psi_n;
  a.pnm1 = psi_nm1;
  for (int c = 0; c < 3; ++c) {
    a.stn[c] = st_n ? st_n[c] : nullptr;
    a.sto[c] = st_nm1 ? st_nm1[c] : nullptr;
    a.Lst[c] = h->Lst[c];
  }
  a.Lux = h->Lux;
  a.Luy = h->Luy;
  a.Luz = h->Luz;
  a.Lrho = h->Lrho;
  a.Lpsi = h->Lpsi;
  a.r = 1.0 / (alpha * dt);  // poissonEqn.f90:215
  a.rho0 = rho0;
  return a;
}

CorrArgs corr_args(tbfp_handle *h, const double *uxi, const double *uyi, const double *uzi, double *uxo,
                   double *uyo, double *uzo, const double *psi, const double *psi_n, const double *psi_nm1,
                   const double *const *st_n, const double *const *st_nm1, double dt, double alpha,
                   double rho0) {
  CorrArgs a{};
  a.uxi = uxi;
  a.uyi = uyi;
  a.uzi = uzi;
  a.uxo = uxo;
  a.uyo = uyo;
  a.uzo = uzo;
  a.psi = psi;
  a.pn = psi_n;
  a.pnm1 = psi_nm1;
  a.irho = h->d_irho;
  for (int c = 0; c < 3; ++c) {
    a.stn[c] = st_n ? st_n[c] : nullptr;
    a.sto[c] = st_nm1 ? st_nm1[c] : nullptr;
    a.Lst[c] = h->Lst[c];
  }
  a.Lux = h->Lux;
  a.Luy = h->Luy;
  a.Luz = h->Luz;
  a.Lpsi = h->Lpsi;
  a.Lrho = h->Lrho;
  a.r = dt * alpha;  // momentumEqn.f90:1012
  a.invrho0 = 1.0 / rho0;
  a.wait_cycles = h->wait_cycles;
  return a;
}

// solveFPS body on device data: spectrum already holds the forward x transform.
void fps_spectral_solve(tbfp_handle *h) {
  launch_fftz(h->d_spec, h->g, h->d_tpz, false, h->stream);
  launch_tridiag(h->d_spec, h->g, h->d_lamx, h->d_lamz, h->d_am, h->d_ap, h->d_dyf, h->mean_c, h->nxnz, h->d_tri_ctl,
                 h->sms, h->d_pinf, h->stream);
  launch_fftz(h->d_spec, h->g, h->d_tpz, true, h->stream);
}

XSrc xsrc(tbfp_handle *h, const double *s, const double *psi) {
  XSrc x{};
  x.s = s;
  x.Ls = h->Lpsi;
  x.psi = psi;
  x.Lp = h->Lpsi;
  x.am = h->d_am;
  x.ap = h->d_ap;
  x.dyf = h->d_dyf;
  x.idx2 = h->idx2;
  x.idz2 = h->idz2;
  x.ctop_scale = h->ctop_scale;
  x.acc = h->d_acc;
  return x;
}

// Read back acc[1] (sum s^2) and acc[slot] (sum r^2): the relative residual
// ||r||_2/||s||_2 (pcg.f90:408-429 uses the same ratio of 2-norms).
int read_rel_residual(tbfp_handle *h, int slot, double *rel) {
  double v[2];
  TBFP_CK(h, cudaMemcpyAsync(&v[0], h->d_acc + 1, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  TBFP_CK(h, cudaMemcpyAsync(&v[1], h->d_acc + slot, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  *rel = v[0] > 0.0 ? std::sqrt(v[1] / v[0]) : std::sqrt(v[1]);
  if (!std::isfinite(*rel)) return set_err(h, TBFP_ENONFINITE, "tbfp_solve_fps: non-finite residual (NaN or Inf in s)");
  return TBFP_OK;
}

// --- mixed precision: FP32 spectral solves, FP64 residuals, device-side loop ---
// Sums: acc[0] = sum s dyf, acc[1] = sum s^2 (first pass); acc[2] = sum r^2 and
// acc[3] = max|s - L psi| of the latest residual pass (cleared by each decision).
XSrc mixed_x(tbfp_handle *h, const double *s, const double *psi) {
  XSrc x = xsrc(h, s, psi);
  x.acc = h->d_acc;
  x.acc_r = h->d_acc + 2;
  return x;
}

void mixed_spectral32(tbfp_handle *h, float2 *sp, cudaStream_t st) {
  launch_fftz(sp, h->g, h->d_tpz32, false, st);
  launch_tridiag(sp, h->g, h->d_lamx, h->d_lamz, h->d_am, h->d_ap, h->d_dyf, h->mean_c, h->nxnz, st);
  launch_fftz(sp, h->g, h->d_tpz32, true, st);
}

// psi = solve32(s), then the first residual pass (r transformed into the
// spectrum for the next sweep) and its decision.
void mixed_head(tbfp_handle *h, const double *s, double *psi, cudaStream_t st, cudaGraphConditionalHandle cond,
                bool use_cond) {
  float2 *sp = reinterpret_cast<float2 *>(h->d_spec);
  const XSrc x = mixed_x(h, s, psi);
  launch_fftx_fwd(x, false, h->g, h->d_twx32, h->d_tpx32, sp, st);
  mixed_spectral32(h, sp, st);
  launch_fftx_inv(sp, psi, h->Lpsi, h->hd_psi, h->g, h->d_twx32, h->d_tpx32, h->scale, false, st);
  launch_fftx_fwd(x, true, h->g, h->d_twx32, h->d_tpx32, sp, st);
  launch_mixed_decide(h->d_ctl, h->d_acc, h->d_acc + 2, cond, use_cond, st);
}

// One refinement sweep psi += solve32(r), then the residual pass and decision.
void mixed_body(tbfp_handle *h, const double *s, double *psi, cudaStream_t st, cudaGraphConditionalHandle cond,
                bool use_cond) {
  float2 *sp = reinterpret_cast<float2 *>(h->d_spec);
  const XSrc x = mixed_x(h, s, psi);
  mixed_spectral32(h, sp, st);
  launch_fftx_inv(sp, psi, h->Lpsi, h->hd_psi, h->g, h->d_twx32, h->d_tpx32, h->scale, true, st);
  launch_fftx_fwd(x, true, h->g, h->d_twx32, h->d_tpx32, sp, st);
  launch_mixed_decide(h->d_ctl, h->d_acc, h->d_acc + 2, cond, use_cond, st);
}

// Emit the whole refinement into the capture that st belongs to: the head,
// then a WHILE conditional node whose body (captured on the handle's second
// capture stream) is one sweep; the decision kernels set the condition, so the
// loop runs on the device with no host round trip.  Returns false if the
// runtime refused a step (the capture is then invalid).
bool emit_mixed_loop(tbfp_handle *h, const double *s, double *psi, cudaStream_t st) {
  cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  if (cudaStreamGetCaptureInfo(st, &cst, nullptr, &g, nullptr, nullptr) != cudaSuccess ||
      cst != cudaStreamCaptureStatusActive || !g)
    return false;
  if (!h->cap_body && cudaStreamCreateWithFlags(&h->cap_body, cudaStreamNonBlocking) != cudaSuccess) return false;
  cudaGraphConditionalHandle hc{};
  if (cudaGraphConditionalHandleCreate(&hc, g, 0, cudaGraphCondAssignDefault) != cudaSuccess) return false;
  mixed_head(h, s, psi, st, hc, true);
  const cudaGraphNode_t *deps = nullptr;
  size_t nd = 0;
  if (cudaStreamGetCaptureInfo(st, &cst, nullptr, &g, &deps, &nd) != cudaSuccess) return false;
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = hc;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cn = nullptr;
  if (cudaGraphAddNode(&cn, g, deps, nd, &cp) != cudaSuccess) return false;
  if (cudaStreamUpdateCaptureDependencies(st, &cn, 1, cudaStreamSetCaptureDependencies) != cudaSuccess) return false;
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  if (cudaStreamBeginCaptureToGraph(h->cap_body, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) !=
      cudaSuccess)
    return false;
  mixed_body(h, s, psi, h->cap_body, hc, true);
  cudaGraph_t bout = nullptr;
  return cudaStreamEndCapture(h->cap_body, &bout) == cudaSuccess;
}

// An executable graph of the whole refinement for the arrays (s, psi).
cudaGraphExec_t build_mixed_graph(tbfp_handle *h, const double *s, double *psi) {
  if (!h->cap && cudaStreamCreateWithFlags(&h->cap, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ex = nullptr;
  bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
  if (ok) ok = cudaStreamBeginCaptureToGraph(h->cap, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
               cudaSuccess;
  if (ok) {
    ok = emit_mixed_loop(h, s, psi, h->cap);
    cudaGraph_t gout = nullptr;
    ok = (cudaStreamEndCapture(h->cap, &gout) == cudaSuccess) && ok;
  }
  if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
  if (g) cudaGraphDestroy(g);
  if (!ok) {
    if (ex) cudaGraphExecDestroy(ex);
    ex = nullptr;
    cudaGetLastError();  // clear the refusal; the host-driven loop is used instead
  }
  return ex;
}

// The refinement of s into psi on stream st: device-side loop (a cached graph
// per (s, psi), or emitted into the caller's capture), else a host-driven loop
// that reads the decision after every pass.  dscale > 0 adds the divergence
// bar of the projection (MixedCtl).  The outcome is in h->d_ctl.
int mixed_solve(tbfp_handle *h, const double *s, double *psi, double dscale, cudaStream_t st) {
  launch_mixed_params(h->d_ctl, h->d_acc, h->tol, h->tol, dscale, h->max_iter, st);
  cudaStreamCaptureStatus cst = cudaStreamCaptureStatusNone;
  TBFP_CK(h, cudaStreamIsCapturing(st, &cst));
  if (cst == cudaStreamCaptureStatusActive) {  // e.g. an ensemble being captured
    if (!emit_mixed_loop(h, s, psi, st))
      return set_err(h, TBFP_ECUDA, "mixed refinement: cannot add the device-side loop to the capture");
    return TBFP_OK;
  }
  cudaGraphExec_t ex = nullptr;
  if (!h->mgr_off) {
    MixedGraph *hit = nullptr, *lru = &h->mgr[0];
    for (MixedGraph &m : h->mgr) {
      if (m.exec && m.s == s && m.psi == psi) hit = &m;
      if (m.used < lru->used) lru = &m;
    }
    if (!hit) {
      cudaGraphExec_t fresh = build_mixed_graph(h, s, psi);
      if (!fresh) {
        h->mgr_off = true;
      } else {
        if (lru->exec) {  // evicted: let a launch still in flight finish first
          TBFP_CK(h, cudaStreamSynchronize(st));
          cudaGraphExecDestroy(lru->exec);
        }
        *lru = MixedGraph{s, psi, fresh, 0};
        hit = lru;
      }
    }
    if (hit) {
      hit->used = ++h->mgr_tick;
      ex = hit->exec;
    }
  }
  if (ex) {
    TBFP_CK(h, cudaGraphLaunch(ex, st));
    return TBFP_OK;
  }
  const cudaGraphConditionalHandle none{};
  mixed_head(h, s, psi, st, none, false);
  for (;;) {
    MixedCtl c{};
    TBFP_CK(h, cudaMemcpyAsync(&c, h->d_ctl, sizeof(c), cudaMemcpyDeviceToHost, st));
    TBFP_CK(h, cudaStreamSynchronize(st));
    if (c.done) break;
    mixed_body(h, s, psi, st, none, false);
  }
  return TBFP_OK;
}

// The refinement's outcome (one read of the control block): status TBFP_OK,
// TBFP_ENOTCONVERGED or TBFP_ENONFINITE (with its message).
int read_mixed(tbfp_handle *h, int *iters, double *rel, double *div) {
  MixedCtl c{};
  TBFP_CK(h, cudaMemcpyAsync(&c, h->d_ctl, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  *iters = c.iters;
  *rel = c.rel;
  if (div) *div = c.div;
  if (c.status == TBFP_ENONFINITE)
    return set_err(h, TBFP_ENONFINITE, "mixed refinement: non-finite residual (NaN or Inf in the inputs)");
  return c.status;
}

// solveFPS (fastPoissonSolver.f90:337-384) on device arrays, including the
// zero-mean gauge and the ghost update of psi.
//   TBFP_FP64: one FP64 direct solve; with TBFP_FLAG_RESIDUAL one more pass
//     computes ||s - L psi||/||s|| (and reads it back).
//   TBFP_MIXED: direct solves with an FP32 spectrum (FP64 tridiagonal
//     arithmetic) and FP64 defect correction, psi = solve32(s), then
//     psi += solve32(r) with r = s - L psi recomputed in FP64 by the forward x
//     pass, until the device-side decision stops the loop (MixedCtl; dscale as
//     there).  With read the outcome is read back: iterations, residual, status.
int device_solve(tbfp_handle *h, const double *s, double *psi, double dscale, bool read, int *iters, double *rel) {
  cudaStream_t st = h->stream;
  *iters = 1;
  *rel = -1.0;
  if (h->precision == TBFP_FP64) {
    const bool want_res = (h->flags & TBFP_FLAG_RESIDUAL) != 0;
    if (want_res) TBFP_CK(h, cudaMemsetAsync(h->d_acc, 0, 4 * sizeof(double), st));
    XSrc x = xsrc(h, s, psi);
    if (!want_res) x.acc = nullptr;
    launch_fftx_fwd(x, false, h->g, h->d_twx, h->d_tpx, h->d_spec, st);
    fps_spectral_solve(h);
    launch_fftx_inv(h->d_spec, psi, h->Lpsi, h->hd_psi, h->g, h->d_twx, h->d_tpx, h->scale, st);
    if (want_res) {
      x.acc_r = h->d_acc + 2;
      launch_fftx_fwd(x, true, h->g, h->d_twx, h->d_tpx, h->d_spec, st);  // residual (spectrum is scratch)
      return read_rel_residual(h, 2, rel);
    }
    return TBFP_OK;
  }
  int rc = mixed_solve(h, s, psi, dscale, st);
  if (rc) return rc;
  if (!read) {
    *iters = -1;  // not read back (asynchronous call)
    return TBFP_OK;
  }
  return read_mixed(h, iters, rel, nullptr);
}

bool aliased(const void *a, const void *b) { return a == b; }

int check_ptrs(tbfp_handle *h, std::initializer_list<const void *> ps) {
  if (!h) return TBFP_ENULL;
  for (const void *p : ps)
    if (!p) return set_err(h, TBFP_ENULL, "a required array pointer is NULL");
  return TBFP_OK;
}

int check_st(tbfp_handle *h, const double *const *st_n, const double *const *st_nm1) {
  if ((st_n == nullptr) != (st_nm1 == nullptr))
    return set_err(h, TBFP_EINVAL, "st_n and st_nm1 must both be given or both be NULL");
  if (st_n)
    for (int c = 0; c < 3; ++c)
      if (!st_n[c] || !st_nm1[c]) return set_err(h, TBFP_ENULL, "a surface-tension component pointer is NULL");
  return TBFP_OK;
}

int device_projection(tbfp_handle *h, const double *uxi, const double *uyi, const double *uzi, double *uxo,
                      double *uyo, double *uzo, const double *rho, const double *psi_n, const double *psi_nm1,
                      const double *const *st_n, const double *const *st_nm1, double dt, double alpha,
                      double rho0, double *psi, tbfp_stats *stats) {
  const bool st = st_present(st_n, st_nm1);
  const bool timing = (h->flags & TBFP_FLAG_TIMING) != 0;
  cudaStream_t s = h->stream;
  auto mark = [&](int i) {
    if (timing) cudaEventRecord(h->evs[i], s);
  };
  TBFP_CK(h, cudaEventRecord(h->ev0, s));
  TBFP_CK(h, cudaMemsetAsync(h->d_maxdiv, 0, sizeof(unsigned long long), s));
  mark(0);
  launch_recip(rho, h->d_irho, (long)h->n_rho, s);
  mark(1);
  RhsArgs ra = rhs_args(h, uxi, uyi, uzi, psi_n, psi_nm1, st_n, st_nm1, dt, alpha, rho0);
  int iters = 1, solve_rc = TBFP_OK;
  double rel = -1.0;
  const bool read = stats != nullptr || !(h->flags & TBFP_FLAG_ASYNC);
  if (h->precision == TBFP_FP64 && !(h->flags & TBFP_FLAG_RESIDUAL)) {
    launch_rhs_fftx(ra, st, h->g, h->d_twx, h->d_tpx, h->d_spec, s);  // s stays on chip
    mark(2);
    launch_fftz(h->d_spec, h->g, h->d_tpz, false, s);
    mark(3);
    launch_tridiag(h->d_spec, h->g, h->d_lamx, h->d_lamz, h->d_am, h->d_ap, h->d_dyf, h->mean_c, h->nxnz,
                   h->d_tri_ctl, h->sms, h->d_pinf, s);
    mark(4);
    launch_fftz(h->d_spec, h->g, h->d_tpz, true, s);
    mark(5);
    launch_fftx_inv(h->d_spec, psi, h->Lpsi, h->hd_psi, h->g, h->d_twx, h->d_tpx, h->scale, s);
    mark(6);
  } else {  // iterative or checked solve: its passes are timed as one stage (TRIDIAG)
    launch_rhs(ra, st, h->g, h->d_s, h->Lpsi, s);
    mark(2);
    mark(3);
    // the mixed loop also stops on max|div u| = alpha*dt/rho0 * max|s - L psi| <= tol
    solve_rc = device_solve(h, h->d_s, psi, alpha * dt / rho0, false, &iters, &rel);
    if (solve_rc < 0) return solve_rc;
    mark(4);
    mark(5);
    mark(6);
  }
  CorrArgs ca = corr_args(h, uxi, uyi, uzi, uxo, uyo, uzo, psi, psi_n, psi_nm1, st_n, st_nm1, dt, alpha, rho0);
  const bool inplace = aliased(uxi, uxo) || aliased(uyi, uyo) || aliased(uzi, uzo);
  if (!inplace) {
    launch_correct_div(ca, st, h->g, h->d_maxdiv, s);
    mark(7);
    mark(8);
  } else {
    launch_correct_inplace(ca, st, h->g, s);
    mark(7);
    launch_div(uxo, uyo, uzo, h->Lux, h->Luy, h->Luz, h->g, h->d_maxdiv, s);
    mark(8);
  }
  TBFP_CK(h, cudaEventRecord(h->ev1, s));
  tbfp_stats out{};
  out.iterations = iters;
  out.rel_residual = rel;
  out.max_div = -1.0;
  out.cont_err = -1.0;
  if (read) {  // one read-back: max|div u| (NaN-propagating) and the mixed loop's outcome
    unsigned long long bits = 0;
    MixedCtl c{};
    TBFP_CK(h, cudaMemcpyAsync(&bits, h->d_maxdiv, sizeof(bits), cudaMemcpyDeviceToHost, s));
    if (h->precision == TBFP_MIXED) TBFP_CK(h, cudaMemcpyAsync(&c, h->d_ctl, sizeof(c), cudaMemcpyDeviceToHost, s));
    TBFP_CK(h, cudaStreamSynchronize(s));
    double md;
    std::memcpy(&md, &bits, sizeof(md));
    out.max_div = md;
    out.cont_err = md * dt;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    out.ms_device = ms;
    for (int i = 0; i < TBFP_NSTAGES; ++i) {
      float m = 0.f;
      if (timing) cudaEventElapsedTime(&m, h->evs[i], h->evs[i + 1]);
      out.ms_stage[i] = m;
    }
    if (h->precision == TBFP_MIXED) {
      out.iterations = c.iters;
      out.rel_residual = c.rel;
      solve_rc = c.status;
    }
    if (bits == kWaitTimeoutBits) {
      h->last = out;
      if (stats) *stats = out;
      return set_err(h, TBFP_ETIMEOUT,
                     "tbfp_projection: a staged copy of the velocity correction did not complete within the wait "
                     "limit (tbfp_set_wait_limit)");
    }
    if (!std::isfinite(md) || solve_rc == TBFP_ENONFINITE) {
      h->last = out;
      if (stats) *stats = out;
      return set_err(h, TBFP_ENONFINITE,
                     "tbfp_projection: non-finite max|div u| or residual (NaN or Inf in u*, rho, psi^n or psi^n-1)");
    }
  } else if (h->precision == TBFP_MIXED) {
    out.iterations = -1;  // the loop's outcome is on the device; not read back
  }
  h->last = out;
  if (stats) *stats = out;
  const int frc = finish(h, "tbfp_projection");
  return frc ? frc : solve_rc;
}

// solveFPS body of tbfp_solve_fps[_dev]; with read the call waits for the
// device and reads back the outcome: the mixed loop's status, or for the FP64
// path one pressure value, which a NaN or Inf anywhere in s reaches (every
// transform output depends on every input, and every unknown of a tridiagonal
// system on every right-hand side entry).
int solve_fps_core(tbfp_handle *h, const double *s, double *psi, bool read) {
  int rc = check_ptrs(h, {s, psi});
  if (rc) return rc;
  if (h->slab) return set_err(h, TBFP_EINVAL, "tbfp_solve_fps: a slab handle solves with tbfp_slab_*");
  cudaSetDevice(h->device);
  TBFP_CK(h, cudaEventRecord(h->ev0, h->stream));
  int iters = 1;
  double rel = -1.0;
  const int src = device_solve(h, s, psi, 0.0, read, &iters, &rel);
  if (src < 0) return src;
  TBFP_CK(h, cudaEventRecord(h->ev1, h->stream));
  h->last = tbfp_stats{};
  h->last.iterations = iters;
  h->last.rel_residual = rel;
  h->last.max_div = -1.0;
  h->last.cont_err = -1.0;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(h, e, "tbfp_solve_fps");
  if (read) {
    double p111 = 0.0;
    TBFP_CK(h, cudaMemcpyAsync(&p111, psi + at(h->Lpsi, 1, 1, 1), sizeof(double), cudaMemcpyDeviceToHost,
                               h->stream));
    TBFP_CK(h, cudaStreamSynchronize(h->stream));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) h->last.ms_device = ms;
    if (!std::isfinite(p111)) return set_err(h, TBFP_ENONFINITE, "tbfp_solve_fps: non-finite pressure (NaN or Inf in s)");
  }
  return src;
}

}  // namespace

extern "C" {

int tbfp_abi_version(void) { return TBFP_ABI_VERSION; }

const char *tbfp_strerror(int status) {
  switch (status) {
    case TBFP_OK: return "success";
    case TBFP_ENOTCONVERGED: return "iteration cap reached before the tolerance (results valid)";
    case TBFP_EINVAL: return "invalid descriptor or argument";
    case TBFP_ENULL: return "a required pointer is NULL";
    case TBFP_ECUDA: return "CUDA runtime error";
    case TBFP_ENOMEM: return "device memory allocation failed";
    case TBFP_EUNSUPPORTED: return "size or feature not supported";
    case TBFP_ENODEVICE: return "no usable CUDA device";
    case TBFP_ENONFINITE: return "non-finite value (NaN or Inf) in a residual or a result";
    case TBFP_ESINGULAR: return "singular coarsest-level system";
    case TBFP_ETIMEOUT: return "a bounded device-side wait ran out";
    default: return "unknown status";
  }
}

const char *tbfp_last_error(const tbfp_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

size_t tbfp_device_bytes(const tbfp_handle *h) { return h ? h->dev_bytes : 0; }

int tbfp_get_stats(const tbfp_handle *h, tbfp_stats *out) {
  if (!h || !out) return TBFP_ENULL;
  *out = h->last;
  return TBFP_OK;
}

int tbfp_destroy(tbfp_handle *h) {
  if (!h) return TBFP_OK;
  int dev_prev = 0;
  cudaGetDevice(&dev_prev);
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  delete h->mg;
  h->mg = nullptr;
  for (MixedGraph &m : h->mgr)
    if (m.exec) cudaGraphExecDestroy(m.exec);
  if (h->cap) cudaStreamDestroy(h->cap);
  if (h->cap_body) cudaStreamDestroy(h->cap_body);
  for (void *p : h->allocs) cudaFree(p);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  for (cudaEvent_t e : h->evs)
    if (e) cudaEventDestroy(e);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  cudaSetDevice(dev_prev);
  delete h;
  return TBFP_OK;
}

}  // extern "C"

namespace {
// Geometry of a slab handle: this rank holds the planes k0 .. k0+nz-1 of a
// channel of nz_total planes (physical space) and the kx0 .. kx0+nkx_loc-1
// wavenumbers (spectral space).
struct SlabSpec {
  int nz_total, k0, kx0, nkx_loc;
};

int create_impl(const tbfp_desc *d, const SlabSpec *sl, tbfp_handle **out) {
  g_create_error.clear();
  if (!d || !out) return set_err(nullptr, TBFP_ENULL, "tbfp_create: NULL descriptor or output");
  *out = nullptr;
  if (d->nx < 4 || d->ny < 4 || d->nz < (sl ? 1 : 2) || (d->nx % 2) != 0)
    return set_err(nullptr, TBFP_EINVAL, "tbfp_create: need nx even >= 4, ny >= 4, nz >= 2");
  if (sl) {
    if (sl->nz_total < d->nz || sl->k0 < 0 || sl->k0 + d->nz > sl->nz_total || sl->kx0 < 0 || sl->nkx_loc < 1 ||
        sl->kx0 + sl->nkx_loc > d->nx / 2 + 1 || d->nz < d->hd_psi)
      return set_err(nullptr, TBFP_EINVAL, "tbfp_slab_create: inconsistent slab geometry");
    if (!(d->s_Vg > 0.0) || d->precision != TBFP_FP64)
      return set_err(nullptr, TBFP_EINVAL, "tbfp_slab_create: needs the channel's s_Vg and TBFP_FP64");
  }
  if (d->hd_psi < 1 || d->hd_rho < 1 || d->hd_u < 0 || d->hd_st < 0)
    return set_err(nullptr, TBFP_EINVAL, "tbfp_create: halo widths must be hd_psi>=1, hd_rho>=1, hd_u>=0, hd_st>=0");
  if (!d->dxf || !d->dxc || !d->dyf || !d->dyc || !d->dzf || !d->dzc)
    return set_err(nullptr, TBFP_ENULL, "tbfp_create: a grid metric array is NULL");
  if (!(d->dx_fft > 0.0) || !(d->dz_fft > 0.0))
    return set_err(nullptr, TBFP_EINVAL, "tbfp_create: dx_fft and dz_fft must be positive");
  if (d->precision != TBFP_FP64 && d->precision != TBFP_MIXED)
    return set_err(nullptr, TBFP_EINVAL, "tbfp_create: unknown precision mode");
  if (d->precision == TBFP_MIXED && (!(d->tol > 0.0) || d->max_iter < 1))
    return set_err(nullptr, TBFP_EINVAL, "tbfp_create: TBFP_MIXED needs tol > 0 and max_iter >= 1");
  for (int i = 0; i < d->nx; ++i)
    if (!(d->dxf[i] > 0.0)) return set_err(nullptr, TBFP_EINVAL, "tbfp_create: dxf must be positive");
  for (int j = 0; j < d->ny; ++j)
    if (!(d->dyf[j] > 0.0)) return set_err(nullptr, TBFP_EINVAL, "tbfp_create: dyf must be positive");
  for (int j = 0; j <= d->ny; ++j)
    if (!(d->dyc[j] > 0.0)) return set_err(nullptr, TBFP_EINVAL, "tbfp_create: dyc must be positive");
  for (int k = 0; k < d->nz; ++k)
    if (!(d->dzf[k] > 0.0)) return set_err(nullptr, TBFP_EINVAL, "tbfp_create: dzf must be positive");
  if (!(d->dxc[0] > 0.0) || !(d->dzc[0] > 0.0))
    return set_err(nullptr, TBFP_EINVAL, "tbfp_create: dxc(1), dzc(1) must be positive");

  if (!fft_length_supported(d->nx / 2) || !fft_length_supported(sl ? sl->nz_total : d->nz))
    return set_err(nullptr, TBFP_EUNSUPPORTED,
                   "tbfp_create: nx/2 and nz must be 2^a or 3*2^a between 4 and 512");
  if (tridiag_smem_bytes(d->ny) > 227 * 1024)
    return set_err(nullptr, TBFP_EUNSUPPORTED, "tbfp_create: ny too large for the shared-memory tiles");

  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(nullptr, TBFP_ENODEVICE, "tbfp_create: no CUDA device");

  tbfp_handle *h = new tbfp_handle();
  h->nx = d->nx;
  h->ny = d->ny;
  h->nz = d->nz;
  h->nkx = d->nx / 2 + 1;
  h->R = (long)d->ny * d->nz;
  h->hd_psi = d->hd_psi;
  h->hd_u = d->hd_u;
  h->hd_rho = d->hd_rho;
  h->hd_st = d->hd_st;
  h->flags = d->flags;
  h->precision = d->precision;
  h->tol = d->tol;
  h->max_iter = d->max_iter;
  if (d->device >= 0) h->device = d->device;
  else cudaGetDevice(&h->device);
  int dev_prev = 0;
  cudaGetDevice(&dev_prev);
  if (cudaSetDevice(h->device) != cudaSuccess) {
    delete h;
    return set_err(nullptr, TBFP_ENODEVICE, "tbfp_create: cannot select the CUDA device");
  }
  const int nx = h->nx, ny = h->ny, nz = h->nz;
  const int nzt = sl ? sl->nz_total : nz;  // planes of the whole channel (z transform length)
  h->slab = sl != nullptr;
  h->nz_total = nzt;
  h->Lpsi = make_lay(1, 1, 1, nx, ny, h->hd_psi, &h->n_psi, nz);
  h->Lrho = make_lay(1, 1, 1, nx, ny, h->hd_rho, &h->n_rho, nz);
  h->Lux = make_lay(0, 1, 1, nx + 1, ny, h->hd_u, &h->n_ux, nz);
  h->Luy = make_lay(1, 0, 1, nx, ny + 1, h->hd_u, &h->n_uy, nz);
  h->Luz = make_lay(1, 1, 0, nx, ny, h->hd_u, &h->n_uz, nz + 1);
  h->Lst[0] = make_lay(0, 1, 1, nx + 1, ny, h->hd_st, &h->n_st[0], nz);
  h->Lst[1] = make_lay(1, 0, 1, nx, ny + 1, h->hd_st, &h->n_st[1], nz);
  h->Lst[2] = make_lay(1, 1, 0, nx, ny, h->hd_st, &h->n_st[2], nz + 1);
  // the stencil kernels index fields with 32-bit element offsets
  const size_t nmax = std::max({h->n_psi, h->n_rho, h->n_ux, h->n_uy, h->n_uz, h->n_st[0], h->n_st[1], h->n_st[2]});
  if (nmax >= (size_t)INT32_MAX) {
    delete h;
    cudaSetDevice(dev_prev);
    return set_err(nullptr, TBFP_EUNSUPPORTED, "tbfp_create: a field has 2^31 or more elements");
  }

  int rc = TBFP_OK;
  auto fail = [&](int code) {
    std::string m = h->err;
    tbfp_destroy(h);
    cudaSetDevice(dev_prev);
    return set_err(nullptr, code, m);
  };
  cudaError_t ce = prepare_kernels();
  if (ce != cudaSuccess) {
    cuda_err(h, ce, "cudaFuncSetAttribute");
    return fail(TBFP_ECUDA);
  }
  if (d->stream) {
    h->stream = static_cast<cudaStream_t>(d->stream);
  } else {
    if ((ce = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) {
      cuda_err(h, ce, "cudaStreamCreate");
      return fail(TBFP_ECUDA);
    }
    h->own_stream = true;
  }
  if ((ce = cudaEventCreate(&h->ev0)) != cudaSuccess || (ce = cudaEventCreate(&h->ev1)) != cudaSuccess) {
    cuda_err(h, ce, "cudaEventCreate");
    return fail(TBFP_ECUDA);
  }
  if (h->flags & TBFP_FLAG_TIMING) {
    for (cudaEvent_t &e : h->evs) {
      if ((ce = cudaEventCreate(&e)) != cudaSuccess) {
        cuda_err(h, ce, "cudaEventCreate");
        return fail(TBFP_ECUDA);
      }
    }
  }

  // --- tables: computeEigenvalues (fastPoissonSolver.f90:215-251) and
  //     initOffDiagMatrix (:255-276); reciprocal metrics for the stencils.
  const double pi = 3.14159265358979323846;
  h->dx_fft = d->dx_fft;
  h->mdxf.assign(d->dxf, d->dxf + nx);
  h->mdxc.assign(d->dxc, d->dxc + nx + 1);
  h->mdyf.assign(d->dyf, d->dyf + ny);
  h->mdyc.assign(d->dyc, d->dyc + ny + 1);
  h->mdzf.assign(d->dzf, d->dzf + nz);
  h->mdzc.assign(d->dzc, d->dzc + nz + 1);
  h->dz_fft = d->dz_fft;
  std::vector<double> lamx(h->nkx), lamz(nzt), am(ny), ap(ny), dyf(ny), idyf(ny), idyc(ny + 1), idxf(nx), idzf(nz);
  for (int i = 0; i < h->nkx; ++i)
    lamx[i] = 2.0 * (std::cos(((double)i * 2.0 * pi) / nx) - 1.0) / (d->dx_fft * d->dx_fft);
  // lamz(k) of fastPoissonSolver.f90:215-251, evaluated at min(k, nz-k) so the
  // table is exactly even in k (the y solve pairs kz with nz-kz)
  for (int k = 0; k < nzt; ++k) {
    const int kk = std::min(k, nzt - k);
    lamz[k] = 2.0 * (std::cos(((double)kk * 2.0 * pi) / nzt) - 1.0) / (d->dz_fft * d->dz_fft);
  }
  for (int j = 0; j < ny; ++j) {
    am[j] = 1.0 / (d->dyc[j] * d->dyf[j]);
    ap[j] = 1.0 / (d->dyc[j + 1] * d->dyf[j]);
    dyf[j] = d->dyf[j];
    idyf[j] = 1.0 / d->dyf[j];
  }
  am[0] = 0.0;
  ap[ny - 1] = 0.0;
  for (int j = 0; j <= ny; ++j) idyc[j] = 1.0 / d->dyc[j];
  for (int i = 0; i < nx; ++i) idxf[i] = 1.0 / d->dxf[i];
  for (int k = 0; k < nz; ++k) idzf[k] = 1.0 / d->dzf[k];
  double sVg = d->s_Vg;
  if (!(sVg > 0.0)) {  // totalVolume (grid.f90:933-951), loop order k, j, i
    sVg = 0.0;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) sVg += d->dxf[i] * d->dyf[j] * d->dzf[k];
  }
  h->s_Vg = sVg;
  h->mean_c = d->dx_fft * d->dz_fft / sVg;
  h->nxnz = (double)nx * (double)nzt;
  h->scale = 1.0 / ((double)nx * (double)nzt);
  h->idx2 = 1.0 / (d->dx_fft * d->dx_fft);
  h->idz2 = 1.0 / (d->dz_fft * d->dz_fft);
  h->ctop_scale = 1.0 / (d->dyf[ny - 1] * (double)nx * (double)nzt);

  if ((rc = upload(h, &h->d_lamx, lamx)) || (rc = upload(h, &h->d_lamz, lamz)) || (rc = upload(h, &h->d_am, am)) ||
      (rc = upload(h, &h->d_ap, ap)) || (rc = upload(h, &h->d_dyf, dyf)) || (rc = upload(h, &h->d_idyf, idyf)) ||
      (rc = upload(h, &h->d_idyc, idyc)) || (rc = upload(h, &h->d_idxf, idxf)) || (rc = upload(h, &h->d_idzf, idzf)) ||
      (rc = upload(h, &h->d_twx, unit_twiddles(nx))) || (rc = upload(h, &h->d_tpx, pass_twiddles(nx / 2))) ||
      (rc = upload(h, &h->d_tpz, pass_twiddles(nzt))) || (rc = upload(h, &h->d_twx32, to_f32(unit_twiddles(nx)))) ||
      (rc = upload(h, &h->d_tpx32, to_f32(pass_twiddles(nx / 2)))) ||
      (rc = upload(h, &h->d_tpz32, to_f32(pass_twiddles(nzt)))) ||
      (rc = upload(h, &h->d_acc, std::vector<double>(64, 0.0))) || (rc = upload(h, &h->d_idxc, inv_of(d->dxc, nx + 1))) ||
      (rc = upload(h, &h->d_idzc, inv_of(d->dzc, nz + 1))))
    return fail(rc);
  if ((rc = dev_alloc(h, &h->d_spec, (size_t)h->nkx * h->R)) || (rc = dev_alloc(h, &h->d_irho, h->n_rho)) ||
      (rc = dev_alloc(h, &h->d_s, h->n_psi)) ||
      (rc = dev_alloc(h, &h->d_maxdiv, 1)) || (rc = dev_alloc(h, &h->d_ctl, 1)) ||
      (rc = dev_alloc(h, &h->d_tri_ctl, 2)) || (rc = dev_alloc(h, &h->d_pinf, (size_t)2 * ny)))
    return fail(rc);
  {
    cudaError_t e = cudaMemset(h->d_tri_ctl, 0, 2 * sizeof(unsigned));
    if (e != cudaSuccess) return fail(cuda_err(h, e, "cudaMemset"));
    launch_pin_factors(h->d_am, h->d_ap, h->d_lamx, h->d_lamz, ny, h->d_pinf, h->stream);
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return fail(cuda_err(h, e, "k_pin_factors"));
    if (cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess) h->sms = 0;
  }

  GridK &g = h->g;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.nkx = h->nkx;
  g.M = nx / 2;
  g.R = h->R;
  g.idxf1 = 1.0 / d->dxf[0];
  g.idxc1 = 1.0 / d->dxc[0];
  // z is uniform (the FFT direction): its metric is the channel's dz_fft, the
  // same number on every rank of a split channel, so a slab's stencils round
  // exactly as the whole channel's (dzf(k), dzc(k) differ from it by rounding)
  g.idzf1 = 1.0 / d->dz_fft;
  g.idzc1 = 1.0 / d->dz_fft;
  g.idyf = h->d_idyf;
  g.idyc = h->d_idyc;
  g.idxf = h->d_idxf;
  g.idzf = h->d_idzf;
  if (sl) {
    g.slab = 1;
    h->gs = g;
    h->gs.nz = nzt;
    h->gs.nkx = sl->nkx_loc;
    h->gs.R = (long)ny * nzt;
    h->gs.kx0 = sl->kx0;
  }
  cudaSetDevice(dev_prev);
  *out = h;
  return TBFP_OK;
}
}  // namespace

extern "C" {

int tbfp_create(const tbfp_desc *d, tbfp_handle **out) { return create_impl(d, nullptr, out); }

int tbfp_slab_create(const tbfp_desc *d, int nz_total, int k0, int kx0, int nkx_loc, tbfp_handle **out) {
  const SlabSpec sl{nz_total, k0, kx0, nkx_loc};
  return create_impl(d, &sl, out);
}

int tbfp_slab_forward_x(tbfp_handle *h, const double *s, double *spec_z) {
  int rc = check_ptrs(h, {s, spec_z});
  if (rc) return rc;
  if (!h->slab) return set_err(h, TBFP_EINVAL, "tbfp_slab_forward_x: not a slab handle");
  cudaSetDevice(h->device);
  launch_fftx_fwd_from_s(s, h->Lpsi, h->g, h->d_twx, h->d_tpx, reinterpret_cast<double2 *>(spec_z), h->stream);
  return finish(h, "tbfp_slab_forward_x");
}

int tbfp_slab_spectral(tbfp_handle *h, double *spec_x) {
  int rc = check_ptrs(h, {spec_x});
  if (rc) return rc;
  if (!h->slab) return set_err(h, TBFP_EINVAL, "tbfp_slab_spectral: not a slab handle");
  cudaSetDevice(h->device);
  double2 *sp = reinterpret_cast<double2 *>(spec_x);
  launch_fftz(sp, h->gs, h->d_tpz, false, h->stream);
  launch_tridiag(sp, h->gs, h->d_lamx, h->d_lamz, h->d_am, h->d_ap, h->d_dyf, h->mean_c, h->nxnz, h->d_tri_ctl, h->sms,
                 h->d_pinf, h->stream);
  launch_fftz(sp, h->gs, h->d_tpz, true, h->stream);
  return finish(h, "tbfp_slab_spectral");
}

int tbfp_slab_inverse_x(tbfp_handle *h, const double *spec_z, double *psi) {
  int rc = check_ptrs(h, {spec_z, psi});
  if (rc) return rc;
  if (!h->slab) return set_err(h, TBFP_EINVAL, "tbfp_slab_inverse_x: not a slab handle");
  cudaSetDevice(h->device);
  launch_fftx_inv(reinterpret_cast<const double2 *>(spec_z), psi, h->Lpsi, h->hd_psi, h->g, h->d_twx, h->d_tpx,
                  h->scale, h->stream);
  return finish(h, "tbfp_slab_inverse_x");
}

}  // extern "C"

namespace {

int slab_chunks(tbfp_handle *h, int world, const int *z_start, bool to_x, const double *src, double *dst,
                const char *where) {
  int rc = check_ptrs(h, {z_start, src, dst});
  if (rc) return rc;
  if (!h->slab) return set_err(h, TBFP_EINVAL, std::string(where) + ": not a slab handle");
  if (world < 1 || world > kSlabMaxRanks)
    return set_err(h, TBFP_EINVAL, std::string(where) + ": world must be 1..64");
  SlabParts parts{};
  parts.n = world;
  if (z_start[0] != 0 || z_start[world] != h->nz_total)
    return set_err(h, TBFP_EINVAL, std::string(where) + ": z_start must run from 0 to the channel's nz");
  for (int r = 0; r <= world; ++r) {
    if (r > 0 && z_start[r] <= z_start[r - 1])
      return set_err(h, TBFP_EINVAL, std::string(where) + ": every rank needs at least one z plane");
    parts.zs[r] = z_start[r];
  }
  cudaSetDevice(h->device);
  launch_slab_chunks(h->gs, parts, to_x, reinterpret_cast<const double2 *>(src), reinterpret_cast<double2 *>(dst),
                     h->stream);
  return finish(h, where);
}

}  // namespace

extern "C" {

int tbfp_slab_unpack_kx(tbfp_handle *h, int world, const int *z_start, const double *recv, double *spec_x) {
  return slab_chunks(h, world, z_start, true, recv, spec_x, "tbfp_slab_unpack_kx");
}

int tbfp_slab_pack_z(tbfp_handle *h, int world, const int *z_start, const double *spec_x, double *send) {
  return slab_chunks(h, world, z_start, false, spec_x, send, "tbfp_slab_pack_z");
}

// ---------------------------------------------------------------------------
int tbfp_solve_fps_dev(tbfp_handle *h, const double *s, double *psi) {
  return solve_fps_core(h, s, psi, !(h && (h->flags & TBFP_FLAG_ASYNC)));
}

int tbfp_solve_fps(tbfp_handle *h, const double *s, double *psi) {
  int rc = check_ptrs(h, {s, psi});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, false))) return rc;
  if ((rc = h2d(h, h->h_s, s, h->n_psi))) return rc;
  // keep the caller's untouched entries (deep y ghost layers) as they are
  if (h->hd_psi > 1 && (rc = h2d(h, h->h_psi, psi, h->n_psi))) return rc;
  const int src = solve_fps_core(h, h->h_s, h->h_psi, true);
  if (src < 0) return src;
  if ((rc = d2h(h, psi, h->h_psi, h->n_psi))) return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return src;
}

int tbfp_rhs_split_dev(tbfp_handle *h, const double *ux, const double *uy, const double *uz, const double *rho,
                       const double *psi_n, const double *psi_nm1, const double *const *st_n,
                       const double *const *st_nm1, double dt, double alpha, double rho0, double *s) {
  int rc = check_ptrs(h, {ux, uy, uz, rho, psi_n, psi_nm1, s});
  if (rc) return rc;
  if ((rc = check_st(h, st_n, st_nm1))) return rc;
  if (!(dt > 0.0) || !(alpha > 0.0) || !(rho0 > 0.0))
    return set_err(h, TBFP_EINVAL, "tbfp_rhs_split: dt, alpha and rho0 must be positive");
  cudaSetDevice(h->device);
  launch_recip(rho, h->d_irho, (long)h->n_rho, h->stream);
  RhsArgs ra = rhs_args(h, ux, uy, uz, psi_n, psi_nm1, st_n, st_nm1, dt, alpha, rho0);
  launch_rhs(ra, st_present(st_n, st_nm1), h->g, s, h->Lpsi, h->stream);
  return finish(h, "tbfp_rhs_split");
}

int tbfp_rhs_split(tbfp_handle *h, const double *ux, const double *uy, const double *uz, const double *rho,
                   const double *psi_n, const double *psi_nm1, const double *const *st_n,
                   const double *const *st_nm1, double dt, double alpha, double rho0, double *s) {
  int rc = check_ptrs(h, {ux, uy, uz, rho, psi_n, psi_nm1, s});
  if (rc) return rc;
  if ((rc = check_st(h, st_n, st_nm1))) return rc;
  cudaSetDevice(h->device);
  const bool st = st_present(st_n, st_nm1);
  if ((rc = ensure_host_bufs(h, st))) return rc;
  if ((rc = h2d(h, h->h_ux, ux, h->n_ux)) || (rc = h2d(h, h->h_uy, uy, h->n_uy)) ||
      (rc = h2d(h, h->h_uz, uz, h->n_uz)) || (rc = h2d(h, h->h_rho, rho, h->n_rho)) ||
      (rc = h2d(h, h->h_pn, psi_n, h->n_psi)) || (rc = h2d(h, h->h_pnm1, psi_nm1, h->n_psi)) ||
      (rc = h2d(h, h->h_s, s, h->n_psi)))
    return rc;
  const double *dn[3] = {nullptr, nullptr, nullptr}, *do_[3] = {nullptr, nullptr, nullptr};
  if (st) {
    for (int c = 0; c < 3; ++c) {
      if ((rc = h2d(h, h->h_st[c], st_n[c], h->n_st[c])) || (rc = h2d(h, h->h_st[3 + c], st_nm1[c], h->n_st[c])))
        return rc;
      dn[c] = h->h_st[c];
      do_[c] = h->h_st[3 + c];
    }
  }
  const unsigned fl = h->flags;
  h->flags |= TBFP_FLAG_ASYNC;
  rc = tbfp_rhs_split_dev(h, h->h_ux, h->h_uy, h->h_uz, h->h_rho, h->h_pn, h->h_pnm1, st ? dn : nullptr,
                          st ? do_ : nullptr, dt, alpha, rho0, h->h_s);
  h->flags = fl;
  if (rc) return rc;
  if ((rc = d2h(h, s, h->h_s, h->n_psi))) return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return TBFP_OK;
}

int tbfp_correct_dev(tbfp_handle *h, double *ux, double *uy, double *uz, const double *psi, const double *psi_n,
                     const double *psi_nm1, const double *rho, const double *const *st_n,
                     const double *const *st_nm1, double dt, double alpha, double rho0) {
  int rc = check_ptrs(h, {ux, uy, uz, psi, psi_n, psi_nm1, rho});
  if (rc) return rc;
  if ((rc = check_st(h, st_n, st_nm1))) return rc;
  if (!(dt > 0.0) || !(alpha > 0.0) || !(rho0 > 0.0))
    return set_err(h, TBFP_EINVAL, "tbfp_correct: dt, alpha and rho0 must be positive");
  cudaSetDevice(h->device);
  launch_recip(rho, h->d_irho, (long)h->n_rho, h->stream);
  CorrArgs ca = corr_args(h, ux, uy, uz, ux, uy, uz, psi, psi_n, psi_nm1, st_n, st_nm1, dt, alpha, rho0);
  launch_correct_inplace(ca, st_present(st_n, st_nm1), h->g, h->stream);
  return finish(h, "tbfp_correct");
}

int tbfp_correct(tbfp_handle *h, double *ux, double *uy, double *uz, const double *psi, const double *psi_n,
                 const double *psi_nm1, const double *rho, const double *const *st_n, const double *const *st_nm1,
                 double dt, double alpha, double rho0) {
  int rc = check_ptrs(h, {ux, uy, uz, psi, psi_n, psi_nm1, rho});
  if (rc) return rc;
  if ((rc = check_st(h, st_n, st_nm1))) return rc;
  cudaSetDevice(h->device);
  const bool st = st_present(st_n, st_nm1);
  if ((rc = ensure_host_bufs(h, st))) return rc;
  if ((rc = h2d(h, h->h_ux, ux, h->n_ux)) || (rc = h2d(h, h->h_uy, uy, h->n_uy)) ||
      (rc = h2d(h, h->h_uz, uz, h->n_uz)) || (rc = h2d(h, h->h_rho, rho, h->n_rho)) ||
      (rc = h2d(h, h->h_psi, psi, h->n_psi)) || (rc = h2d(h, h->h_pn, psi_n, h->n_psi)) ||
      (rc = h2d(h, h->h_pnm1, psi_nm1, h->n_psi)))
    return rc;
  const double *dn[3] = {nullptr, nullptr, nullptr}, *do_[3] = {nullptr, nullptr, nullptr};
  if (st) {
    for (int c = 0; c < 3; ++c) {
      if ((rc = h2d(h, h->h_st[c], st_n[c], h->n_st[c])) || (rc = h2d(h, h->h_st[3 + c], st_nm1[c], h->n_st[c])))
        return rc;
      dn[c] = h->h_st[c];
      do_[c] = h->h_st[3 + c];
    }
  }
  const unsigned fl = h->flags;
  h->flags |= TBFP_FLAG_ASYNC;
  rc = tbfp_correct_dev(h, h->h_ux, h->h_uy, h->h_uz, h->h_psi, h->h_pn, h->h_pnm1, h->h_rho, st ? dn : nullptr,
                        st ? do_ : nullptr, dt, alpha, rho0);
  h->flags = fl;
  if (rc) return rc;
  if ((rc = d2h(h, ux, h->h_ux, h->n_ux)) || (rc = d2h(h, uy, h->h_uy, h->n_uy)) || (rc = d2h(h, uz, h->h_uz, h->n_uz)))
    return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return TBFP_OK;
}

int tbfp_continuity_error_dev(tbfp_handle *h, const double *ux, const double *uy, const double *uz, double dt,
                              double *max_div, double *cont_err) {
  int rc = check_ptrs(h, {ux, uy, uz});
  if (rc) return rc;
  cudaSetDevice(h->device);
  TBFP_CK(h, cudaMemsetAsync(h->d_maxdiv, 0, sizeof(unsigned long long), h->stream));
  launch_div(ux, uy, uz, h->Lux, h->Luy, h->Luz, h->g, h->d_maxdiv, h->stream);
  unsigned long long bits = 0;
  TBFP_CK(h, cudaMemcpyAsync(&bits, h->d_maxdiv, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(h, e, "tbfp_continuity_error");
  double md;
  std::memcpy(&md, &bits, sizeof(md));
  if (max_div) *max_div = md;
  if (cont_err) *cont_err = md * dt;  // auxiliaryRoutines.f90:82
  return TBFP_OK;
}

int tbfp_continuity_error(tbfp_handle *h, const double *ux, const double *uy, const double *uz, double dt,
                          double *max_div, double *cont_err) {
  int rc = check_ptrs(h, {ux, uy, uz});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, false))) return rc;
  if ((rc = h2d(h, h->h_ux, ux, h->n_ux)) || (rc = h2d(h, h->h_uy, uy, h->n_uy)) || (rc = h2d(h, h->h_uz, uz, h->n_uz)))
    return rc;
  return tbfp_continuity_error_dev(h, h->h_ux, h->h_uy, h->h_uz, dt, max_div, cont_err);
}

int tbfp_projection_dev(tbfp_handle *h, const double *ux_in, const double *uy_in, const double *uz_in,
                        double *ux_out, double *uy_out, double *uz_out, const double *rho, const double *psi_n,
                        const double *psi_nm1, const double *const *st_n, const double *const *st_nm1, double dt,
                        double alpha, double rho0, double *psi, tbfp_stats *stats) {
  int rc = check_ptrs(h, {ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, rho, psi_n, psi_nm1, psi});
  if (rc) return rc;
  if ((rc = check_st(h, st_n, st_nm1))) return rc;
  if (h->slab) return set_err(h, TBFP_EINVAL, "tbfp_projection: a slab handle solves with tbfp_slab_*");
  if (!(dt > 0.0) || !(alpha > 0.0) || !(rho0 > 0.0))
    return set_err(h, TBFP_EINVAL, "tbfp_projection: dt, alpha and rho0 must be positive");
  cudaSetDevice(h->device);
  return device_projection(h, ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, rho, psi_n, psi_nm1, st_n, st_nm1, dt,
                           alpha, rho0, psi, stats);
}

int tbfp_projection(tbfp_handle *h, double *ux, double *uy, double *uz, const double *rho, const double *psi_n,
                    const double *psi_nm1, const double *const *st_n, const double *const *st_nm1, double dt,
                    double alpha, double rho0, double *psi, tbfp_stats *stats) {
  int rc = check_ptrs(h, {ux, uy, uz, rho, psi_n, psi_nm1, psi});
  if (rc) return rc;
  if ((rc = check_st(h, st_n, st_nm1))) return rc;
  if (!(dt > 0.0) || !(alpha > 0.0) || !(rho0 > 0.0))
    return set_err(h, TBFP_EINVAL, "tbfp_projection: dt, alpha and rho0 must be positive");
  cudaSetDevice(h->device);
  const bool st = st_present(st_n, st_nm1);
  if ((rc = ensure_host_bufs(h, st))) return rc;
  // u is corrected in place in the device copy, so the caller's halos come back
  // unchanged.  With hd_psi == 1 every entry of psi (interior and ghosts) is
  // written; deeper halos are preserved by uploading psi first.
  if ((rc = h2d(h, h->h_ux, ux, h->n_ux)) || (rc = h2d(h, h->h_uy, uy, h->n_uy)) ||
      (rc = h2d(h, h->h_uz, uz, h->n_uz)) || (rc = h2d(h, h->h_rho, rho, h->n_rho)) ||
      (rc = h2d(h, h->h_pn, psi_n, h->n_psi)) || (rc = h2d(h, h->h_pnm1, psi_nm1, h->n_psi)))
    return rc;
  if (h->hd_psi > 1 && (rc = h2d(h, h->h_psi, psi, h->n_psi))) return rc;
  const double *dn[3] = {nullptr, nullptr, nullptr}, *do_[3] = {nullptr, nullptr, nullptr};
  if (st) {
    for (int c = 0; c < 3; ++c) {
      if ((rc = h2d(h, h->h_st[c], st_n[c], h->n_st[c])) || (rc = h2d(h, h->h_st[3 + c], st_nm1[c], h->n_st[c])))
        return rc;
      dn[c] = h->h_st[c];
      do_[c] = h->h_st[3 + c];
    }
  }
  const unsigned fl = h->flags;
  h->flags |= TBFP_FLAG_ASYNC;
  const int prc = device_projection(h, h->h_ux, h->h_uy, h->h_uz, h->h_ux, h->h_uy, h->h_uz, h->h_rho, h->h_pn,
                                    h->h_pnm1, st ? dn : nullptr, st ? do_ : nullptr, dt, alpha, rho0, h->h_psi, stats);
  h->flags = fl;
  if (prc < 0) return prc;
  if ((rc = d2h(h, ux, h->h_ux, h->n_ux)) || (rc = d2h(h, uy, h->h_uy, h->n_uy)) ||
      (rc = d2h(h, uz, h->h_uz, h->n_uz)) || (rc = d2h(h, psi, h->h_psi, h->n_psi)))
    return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return prc;
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// updateMaterialProps (VOF.f90:197-233) with smoothVF (:235-262)
// ---------------------------------------------------------------------------
void run_material_props(tbfp_handle *h, const double *c, double *cs, double *rho, double *mu) {
  if (h->hd_rho == 1)
    launch_material_props_fused(h->vsep, c, cs, rho, mu, h->d_qv, h->Lrho, h->nx, h->ny, h->nz, h->rhol, h->rhog, h->mul,
                                h->mug, h->stream);
  else
    launch_material_props(h->vt, c, cs, rho, mu, h->d_qv, h->Lrho, (long)h->n_rho, h->nx, h->ny, h->nz, h->hd_rho,
                          h->rhol, h->rhog, h->mul, h->mug, h->stream);
}

int tbfp_vof_setup(tbfp_handle *h, const tbfp_vof_desc *v) {
  if (!h || !v) return TBFP_ENULL;
  if (!v->xc || !v->yc || !v->zc || !v->xf || !v->yf || !v->zf)
    return set_err(h, TBFP_ENULL, "tbfp_vof_setup: a coordinate array is NULL");
  if (h->slab && h->hd_rho != 1)
    return set_err(h, TBFP_EUNSUPPORTED, "tbfp_vof_setup: a slab handle needs hd_rho = 1 (the fused passes)");
  if (h->vof) return set_err(h, TBFP_EINVAL, "tbfp_vof_setup: already set up for this handle");
  const int nx = h->nx, ny = h->ny, nz = h->nz;
  // distance tables of cellToVertex / vertexToCell (interpolation.f90:188-276)
  auto c2v = [](const double *c, const double *f, int n, int dir, std::vector<double> &a1, std::vector<double> &a2,
                std::vector<double> &hh) {
    a1.resize(n + 1);
    a2.resize(n + 1);
    hh.resize(n + 1);
    for (int i = 0; i <= n; ++i) {
      if (dir == 1) {  // y: yv(j)-y(j), y(j+1)-yv(j)
        a1[i] = f[i] - c[i];
        a2[i] = c[i + 1] - f[i];
      } else {  // x, z: x(i+1)-xv(i), xv(i)-x(i)
        a1[i] = c[i + 1] - f[i];
        a2[i] = f[i] - c[i];
      }
      hh[i] = c[i + 1] - c[i];
    }
  };
  auto v2c = [](const double *c, const double *f, int n, int dir, std::vector<double> &a1, std::vector<double> &a2,
                std::vector<double> &vv) {
    a1.resize(n);
    a2.resize(n);
    vv.resize(n);
    for (int i = 1; i <= n; ++i) {
      if (dir == 1) {  // y: y(j)-yv(j-1), yv(j)-y(j)
        a1[i - 1] = c[i] - f[i - 1];
        a2[i - 1] = f[i] - c[i];
      } else {  // x, z: xv(i)-x(i), x(i)-xv(i-1)
        a1[i - 1] = f[i] - c[i];
        a2[i - 1] = c[i] - f[i - 1];
      }
      vv[i - 1] = f[i] - f[i - 1];
    }
  };
  std::vector<double> t[18];
  c2v(v->xc, v->xf, nx, 0, t[0], t[1], t[2]);
  c2v(v->yc, v->yf, ny, 1, t[3], t[4], t[5]);
  c2v(v->zc, v->zf, nz, 2, t[6], t[7], t[8]);
  v2c(v->xc, v->xf, nx, 0, t[9], t[10], t[11]);
  v2c(v->yc, v->yf, ny, 1, t[12], t[13], t[14]);
  v2c(v->zc, v->zf, nz, 2, t[15], t[16], t[17]);
  for (int i = 0; i <= nx; ++i)
    if (!(t[2][i] > 0.0)) return set_err(h, TBFP_EINVAL, "tbfp_vof_setup: xc must increase");
  for (int j = 0; j <= ny; ++j)
    if (!(t[5][j] > 0.0)) return set_err(h, TBFP_EINVAL, "tbfp_vof_setup: yc must increase");
  for (int k = 0; k <= nz; ++k)
    if (!(t[8][k] > 0.0)) return set_err(h, TBFP_EINVAL, "tbfp_vof_setup: zc must increase");
  cudaSetDevice(h->device);
  double *d[18];
  int rc;
  for (int e = 0; e < 18; ++e)
    if ((rc = upload(h, &d[e], t[e]))) return rc;
  // halo 1 (the reference's): two fused passes through a field-shaped scratch;
  // otherwise the vertex array of the reference's s_cv
  const size_t nscr = h->hd_rho == 1 ? h->n_rho : (size_t)(nx + 1) * (ny + 1) * (nz + 1);
  if ((rc = dev_alloc(h, &h->d_qv, nscr))) return rc;
  h->vt = VofTab{d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8],
                 d[9], d[10], d[11], d[12], d[13], d[14], d[15], d[16], d[17]};
  // separable pass per direction: cell i takes vertices i-1 (weight a) and i
  // (weight b) of vertexToCell, vertex v takes cells v (weight e) and v+1
  // (weight f) of cellToVertex; in y the tables hold the weights in the other
  // order (interpolation.f90:206-224, 252-271).
  auto sep = [](const std::vector<double> &c1, const std::vector<double> &c2, const std::vector<double> &hh,
                const std::vector<double> &v1, const std::vector<double> &v2, const std::vector<double> &VV, int n,
                bool ydir, std::vector<double> &m, std::vector<double> &z, std::vector<double> &p) {
    m.resize(n);
    z.resize(n);
    p.resize(n);
    for (int i = 1; i <= n; ++i) {
      const double a = (ydir ? v2[i - 1] : v1[i - 1]) / VV[i - 1], b = (ydir ? v1[i - 1] : v2[i - 1]) / VV[i - 1];
      const double e0 = (ydir ? c2[i - 1] : c1[i - 1]) / hh[i - 1], f0 = (ydir ? c1[i - 1] : c2[i - 1]) / hh[i - 1];
      const double e1 = (ydir ? c2[i] : c1[i]) / hh[i], f1 = (ydir ? c1[i] : c2[i]) / hh[i];
      m[i - 1] = a * e0;
      z[i - 1] = a * f0 + b * e1;
      p[i - 1] = b * f1;
    }
  };
  std::vector<double> sw[9];
  sep(t[0], t[1], t[2], t[9], t[10], t[11], nx, false, sw[0], sw[1], sw[2]);
  sep(t[3], t[4], t[5], t[12], t[13], t[14], ny, true, sw[3], sw[4], sw[5]);
  sep(t[6], t[7], t[8], t[15], t[16], t[17], nz, false, sw[6], sw[7], sw[8]);
  double *ds[9];
  for (int e = 0; e < 9; ++e)
    if ((rc = upload(h, &ds[e], sw[e]))) return rc;
  h->vsep = VofSep{ds[0], ds[1], ds[2], ds[3], ds[4], ds[5], ds[6], ds[7], ds[8]};
  h->rhol = v->rhol;
  h->rhog = v->rhog;
  h->mul = v->mul;
  h->mug = v->mug;
  h->vof = true;
  return TBFP_OK;
}

int tbfp_material_props_pass_dev(tbfp_handle *h, const double *in, double *out, double *rho, double *mu) {
  int rc = check_ptrs(h, {in, out});
  if (rc) return rc;
  if (!h->vof) return set_err(h, TBFP_EINVAL, "tbfp_material_props_pass: call tbfp_vof_setup first");
  if (h->hd_rho != 1) return set_err(h, TBFP_EUNSUPPORTED, "tbfp_material_props_pass: needs hd_rho = 1");
  if ((rho == nullptr) != (mu == nullptr))
    return set_err(h, TBFP_EINVAL, "tbfp_material_props_pass: rho and mu are both given or both NULL");
  if (aliased(in, out) || (rho && (aliased(in, rho) || aliased(in, mu) || aliased(out, rho) || aliased(out, mu) ||
                                   aliased(rho, mu))))
    return set_err(h, TBFP_EINVAL, "tbfp_material_props_pass: the arrays must be distinct");
  cudaSetDevice(h->device);
  launch_smooth_pass(h->vsep, in, out, rho, mu, h->Lrho, h->nx, h->ny, h->nz, h->rhol, h->rhog, h->mul, h->mug,
                     !h->slab, h->stream);
  return finish(h, "tbfp_material_props_pass");
}

int tbfp_material_props_dev(tbfp_handle *h, const double *c, double *cs, double *rho, double *mu) {
  int rc = check_ptrs(h, {c, cs, rho, mu});
  if (rc) return rc;
  if (!h->vof) return set_err(h, TBFP_EINVAL, "tbfp_material_props: call tbfp_vof_setup first");
  if (h->slab)
    return set_err(h, TBFP_EINVAL, "tbfp_material_props: on a slab handle run the two passes "
                                   "(tbfp_material_props_pass_dev) with the z ghost exchange between them");
  if (aliased(c, cs) || aliased(c, rho) || aliased(c, mu) || aliased(cs, rho) || aliased(cs, mu) || aliased(rho, mu))
    return set_err(h, TBFP_EINVAL, "tbfp_material_props: c, cs, rho and mu must be distinct arrays");
  cudaSetDevice(h->device);
  run_material_props(h, c, cs, rho, mu);
  return finish(h, "tbfp_material_props");
}

int tbfp_material_props(tbfp_handle *h, const double *c, double *cs, double *rho, double *mu) {
  int rc = check_ptrs(h, {c, cs, rho, mu});
  if (rc) return rc;
  if (!h->vof) return set_err(h, TBFP_EINVAL, "tbfp_material_props: call tbfp_vof_setup first");
  if (h->slab)
    return set_err(h, TBFP_EINVAL, "tbfp_material_props: on a slab handle run the two passes "
                                   "(tbfp_material_props_pass_dev) with the z ghost exchange between them");
  cudaSetDevice(h->device);
  for (double *&b : h->h_vof)
    if (!b && (rc = dev_alloc(h, &b, h->n_rho))) return rc;
  const size_t n = h->n_rho;
  if ((rc = h2d(h, h->h_vof[0], c, n))) return rc;
  run_material_props(h, h->h_vof[0], h->h_vof[1], h->h_vof[2], h->h_vof[3]);
  if ((rc = d2h(h, cs, h->h_vof[1], n)) || (rc = d2h(h, rho, h->h_vof[2], n)) || (rc = d2h(h, mu, h->h_vof[3], n)))
    return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return finish(h, "tbfp_material_props");
}

// ---------------------------------------------------------------------------
// solveMomentumEqn FAST (momentumEqn.f90:161-194)
// ---------------------------------------------------------------------------
int tbfp_momentum_setup(tbfp_handle *h, const tbfp_momentum_desc *m) {
  if (!h || !m) return TBFP_ENULL;
  if (h->mom) return set_err(h, TBFP_EINVAL, "tbfp_momentum_setup: already set up for this handle");
  if (m->scheme < 0 || m->scheme > 5) return set_err(h, TBFP_EINVAL, "tbfp_momentum_setup: scheme must be 0..5");
  if (h->hd_u < 2 || h->hd_rho < 1)
    return set_err(h, TBFP_EINVAL, "tbfp_momentum_setup: needs hd_u >= 2 and hd_rho >= 1");
  if (!m->dxf || !m->dxc || !m->dyf || !m->dyc || !m->dzf || !m->dzc || !m->yc || !m->yf)
    return set_err(h, TBFP_ENULL, "tbfp_momentum_setup: a spacing or coordinate table is NULL");
  const int nx = h->nx, ny = h->ny, nz = h->nz;
  // spacings by Fortran index 0..n+1, as the mesh holds them
  std::vector<double> dxf(m->dxf, m->dxf + nx + 2), dxc(m->dxc, m->dxc + nx + 2);
  std::vector<double> dyf(m->dyf, m->dyf + ny + 2), dyc(m->dyc, m->dyc + ny + 2);
  std::vector<double> dzf(m->dzf, m->dzf + nz + 2), dzc(m->dzc, m->dzc + nz + 2);
  cudaSetDevice(h->device);
  // the kernel multiplies by reciprocals, each the correctly rounded 1/d
  auto recip = [](const std::vector<double> &v) {
    std::vector<double> r(v.size());
    for (size_t e = 0; e < v.size(); ++e) r[e] = 1.0 / v[e];
    return r;
  };
  const std::vector<double> tabs[7] = {dyf, recip(dxf), recip(dxc), recip(dyf), recip(dyc), recip(dzf), recip(dzc)};
  double *d[7];
  int rc;
  for (int e = 0; e < 7; ++e)
    if ((rc = upload(h, &d[e], tabs[e]))) return rc;
  h->mt = MomentumTabs{d[0], d[1], d[2], d[3], d[4], d[5], d[6]};
  h->n_phi[0] = (size_t)(nx + 1) * ny * nz;
  h->n_phi[1] = (size_t)nx * (ny - 1) * nz;
  h->n_phi[2] = (size_t)nx * ny * (nz + 1);
  for (int b = 0; b < 2; ++b)
    for (int c = 0; c < 3; ++c) {
      if ((rc = dev_alloc(h, &h->d_phi[b][c], h->n_phi[c]))) return rc;
      TBFP_CK(h, cudaMemset(h->d_phi[b][c], 0, h->n_phi[c] * sizeof(double)));  // initFluxes
    }
  // setMetrics at the y walls: 'cl'-type spacings for ux and uz, face spacings for uy
  for (int e = 0; e < 3; ++e) {
    if (e == 1) {
      h->wt.hb[e] = m->dyf[0];
      h->wt.hi[e] = m->dyf[0] + m->dyf[1];
      h->wt.tb[e] = m->dyf[ny + 1];
      h->wt.ti[e] = m->dyf[ny] + m->dyf[ny + 1];
    } else {
      h->wt.hb[e] = m->yf[0] - m->yc[0];
      h->wt.hi[e] = m->dyc[1];
      h->wt.tb[e] = m->yc[ny + 1] - m->yf[ny];
      h->wt.ti[e] = m->dyc[ny + 1];
    }
    h->wt.bb[e] = m->ubot[e];
    h->wt.bt[e] = m->utop[e];
  }
  h->mom_scheme = m->scheme;
  h->mom_gch = m->gch;
  h->mom_g = m->g;
  h->phi_cur = 0;
  h->mom = true;
  return TBFP_OK;
}

int tbfp_momentum_fluxes(tbfp_handle *h, double *phi_x, double *phi_y, double *phi_z, int set) {
  int rc = check_ptrs(h, {phi_x, phi_y, phi_z});
  if (rc) return rc;
  if (!h->mom) return set_err(h, TBFP_EINVAL, "tbfp_momentum_fluxes: call tbfp_momentum_setup first");
  cudaSetDevice(h->device);
  double *host[3] = {phi_x, phi_y, phi_z};
  for (int c = 0; c < 3; ++c) {
    if (set) rc = h2d(h, h->d_phi[h->phi_cur][c], host[c], h->n_phi[c]);
    else rc = d2h(h, host[c], h->d_phi[h->phi_cur][c], h->n_phi[c]);
    if (rc) return rc;
  }
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return TBFP_OK;
}

int tbfp_momentum_predictor_dev(tbfp_handle *h, double *ux, double *uy, double *uz, const double *c,
                                const double *mu, const double *rho, const double *const *st, double dt,
                                double alpha, double gamma, double xi, double rho0, double fs) {
  int rc = check_ptrs(h, {ux, uy, uz, c, mu, rho});
  if (rc) return rc;
  if (!h->mom) return set_err(h, TBFP_EINVAL, "tbfp_momentum_predictor: call tbfp_momentum_setup first");
  if (st && (!st[0] || !st[1] || !st[2]))
    return set_err(h, TBFP_ENULL, "tbfp_momentum_predictor: a surface-tension component pointer is NULL");
  if (!(dt > 0.0) || !(rho0 > 0.0))
    return set_err(h, TBFP_EINVAL, "tbfp_momentum_predictor: dt and rho0 must be positive");
  cudaSetDevice(h->device);
  // copyOldFluxes + resetFluxes: the previous fluxes stay where they are and
  // the new ones go to the other buffer
  const int prev = h->phi_cur, cur = 1 - h->phi_cur;
  double *const phi[3] = {h->d_phi[cur][0], h->d_phi[cur][1], h->d_phi[cur][2]};
  const double *const pp[3] = {h->d_phi[prev][0], h->d_phi[prev][1], h->d_phi[prev][2]};
  launch_momentum(h->mt, ux, uy, uz, c, mu, rho, st, h->Lux, h->Luy, h->Luz, h->Lrho, h->Lst, phi, pp, h->nx, h->ny,
                  h->nz, h->mom_scheme, dt, alpha, gamma, xi, rho0, fs, h->mom_gch, h->mom_g, h->hd_u, h->hd_rho,
                  nullptr, h->stream);
  h->phi_cur = cur;
  return finish(h, "tbfp_momentum_predictor");
}

int tbfp_momentum_predictor_out_dev(tbfp_handle *h, const double *ux, const double *uy, const double *uz,
                                    double *ux_out, double *uy_out, double *uz_out, const double *c, const double *mu,
                                    const double *rho, const double *const *st, double dt, double alpha, double gamma,
                                    double xi, double rho0, double fs) {
  int rc = check_ptrs(h, {ux, uy, uz, ux_out, uy_out, uz_out, c, mu, rho});
  if (rc) return rc;
  if (!h->mom) return set_err(h, TBFP_EINVAL, "tbfp_momentum_predictor_out: call tbfp_momentum_setup first");
  if (st && (!st[0] || !st[1] || !st[2]))
    return set_err(h, TBFP_ENULL, "tbfp_momentum_predictor_out: a surface-tension component pointer is NULL");
  if (!(dt > 0.0) || !(rho0 > 0.0))
    return set_err(h, TBFP_EINVAL, "tbfp_momentum_predictor_out: dt and rho0 must be positive");
  const double *ins[3] = {ux, uy, uz};
  const double *outs[3] = {ux_out, uy_out, uz_out};
  for (const double *o : outs)
    for (const double *i : ins)
      if (o == i) return set_err(h, TBFP_EINVAL, "tbfp_momentum_predictor_out: u_out must not alias u");
  cudaSetDevice(h->device);
  const int prev = h->phi_cur, cur = 1 - h->phi_cur;
  double *const phi[3] = {h->d_phi[cur][0], h->d_phi[cur][1], h->d_phi[cur][2]};
  const double *const pp[3] = {h->d_phi[prev][0], h->d_phi[prev][1], h->d_phi[prev][2]};
  double *const uo[3] = {ux_out, uy_out, uz_out};
  launch_momentum(h->mt, const_cast<double *>(ux), const_cast<double *>(uy), const_cast<double *>(uz), c, mu, rho, st,
                  h->Lux, h->Luy, h->Luz, h->Lrho, h->Lst, phi, pp, h->nx, h->ny, h->nz, h->mom_scheme, dt, alpha,
                  gamma, xi, rho0, fs, h->mom_gch, h->mom_g, h->hd_u, h->hd_rho, uo, h->stream);
  h->phi_cur = cur;
  return finish(h, "tbfp_momentum_predictor_out");
}

int tbfp_update_boundaries_v_dev(tbfp_handle *h, double *ux, double *uy, double *uz) {
  int rc = check_ptrs(h, {ux, uy, uz});
  if (rc) return rc;
  if (!h->mom) return set_err(h, TBFP_EINVAL, "tbfp_update_boundaries_v: call tbfp_momentum_setup first");
  cudaSetDevice(h->device);
  launch_boundaries_v(h->wt, ux, uy, uz, h->Lux, h->Luy, h->Luz, h->nx, h->ny, h->nz, h->hd_u, h->slab != 0,
                      h->stream);
  return finish(h, "tbfp_update_boundaries_v");
}

int tbfp_update_boundaries_v(tbfp_handle *h, double *ux, double *uy, double *uz) {
  int rc = check_ptrs(h, {ux, uy, uz});
  if (rc) return rc;
  if (!h->mom) return set_err(h, TBFP_EINVAL, "tbfp_update_boundaries_v: call tbfp_momentum_setup first");
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, false))) return rc;
  if ((rc = h2d(h, h->h_ux, ux, h->n_ux)) || (rc = h2d(h, h->h_uy, uy, h->n_uy)) || (rc = h2d(h, h->h_uz, uz, h->n_uz)))
    return rc;
  launch_boundaries_v(h->wt, h->h_ux, h->h_uy, h->h_uz, h->Lux, h->Luy, h->Luz, h->nx, h->ny, h->nz, h->hd_u,
                      h->slab != 0, h->stream);
  if ((rc = d2h(h, ux, h->h_ux, h->n_ux)) || (rc = d2h(h, uy, h->h_uy, h->n_uy)) || (rc = d2h(h, uz, h->h_uz, h->n_uz)))
    return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return finish(h, "tbfp_update_boundaries_v");
}

int tbfp_momentum_predictor(tbfp_handle *h, double *ux, double *uy, double *uz, const double *c, const double *mu,
                            const double *rho, const double *const *st, double dt, double alpha, double gamma,
                            double xi, double rho0, double fs) {
  int rc = check_ptrs(h, {ux, uy, uz, c, mu, rho});
  if (rc) return rc;
  if (!h->mom) return set_err(h, TBFP_EINVAL, "tbfp_momentum_predictor: call tbfp_momentum_setup first");
  if (st && (!st[0] || !st[1] || !st[2]))
    return set_err(h, TBFP_ENULL, "tbfp_momentum_predictor: a surface-tension component pointer is NULL");
  cudaSetDevice(h->device);
  const bool has_st = st != nullptr;
  if ((rc = ensure_host_bufs(h, has_st))) return rc;
  for (double *&b : h->h_mom)
    if (!b && (rc = dev_alloc(h, &b, h->n_rho))) return rc;
  if ((rc = h2d(h, h->h_ux, ux, h->n_ux)) || (rc = h2d(h, h->h_uy, uy, h->n_uy)) ||
      (rc = h2d(h, h->h_uz, uz, h->n_uz)) || (rc = h2d(h, h->h_rho, rho, h->n_rho)) ||
      (rc = h2d(h, h->h_mom[0], c, h->n_rho)) || (rc = h2d(h, h->h_mom[1], mu, h->n_rho)))
    return rc;
  const double *dst[3] = {nullptr, nullptr, nullptr};
  if (has_st) {
    for (int e = 0; e < 3; ++e) {
      if ((rc = h2d(h, h->h_st[e], st[e], h->n_st[e]))) return rc;
      dst[e] = h->h_st[e];
    }
  }
  const int flags = h->flags;
  h->flags |= TBFP_FLAG_ASYNC;
  rc = tbfp_momentum_predictor_dev(h, h->h_ux, h->h_uy, h->h_uz, h->h_mom[0], h->h_mom[1], h->h_rho,
                                   has_st ? dst : nullptr, dt, alpha, gamma, xi, rho0, fs);
  h->flags = flags;
  if (rc) return rc;
  if ((rc = d2h(h, ux, h->h_ux, h->n_ux)) || (rc = d2h(h, uy, h->h_uy, h->n_uy)) || (rc = d2h(h, uz, h->h_uz, h->n_uz)))
    return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return finish(h, "tbfp_momentum_predictor");
}

// ---------------------------------------------------------------------------
// flow control (auxiliaryRoutines.f90:336-540)
// ---------------------------------------------------------------------------
namespace {
int face_sum(tbfp_handle *h, int mode, const double *f, Lay L, double *out) {
  int rc;
  if (!h->d_fpart) {
    const std::vector<double> dxc(h->mdxc.begin(), h->mdxc.begin() + h->nx);
    if ((rc = upload(h, &h->d_fdxc, dxc)) || (rc = upload(h, &h->d_fdyf, h->mdyf)) ||
        (rc = upload(h, &h->d_fdzf, h->mdzf)) || (rc = dev_alloc(h, &h->d_fpart, (size_t)h->ny * h->nz + 1)))
      return rc;
  }
  double *sum = h->d_fpart + (size_t)h->ny * h->nz;
  launch_face_sum(mode, f, L, h->d_fdxc, h->d_fdyf, h->d_fdzf, h->nx, h->ny, h->nz, h->d_fpart, sum, h->stream);
  TBFP_CK(h, cudaMemcpyAsync(out, sum, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return TBFP_OK;
}
}  // namespace

int tbfp_rho_face_sum_dev(tbfp_handle *h, const double *rho, double *sum) {
  int rc = check_ptrs(h, {rho, sum});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = face_sum(h, 0, rho, h->Lrho, sum))) return rc;
  return finish(h, "tbfp_rho_face_sum");
}

int tbfp_rho_face_sum(tbfp_handle *h, const double *rho, double *sum) {
  int rc = check_ptrs(h, {rho, sum});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, false)) || (rc = h2d(h, h->h_rho, rho, h->n_rho))) return rc;
  if ((rc = face_sum(h, 0, h->h_rho, h->Lrho, sum))) return rc;
  return finish(h, "tbfp_rho_face_sum");
}

int tbfp_flow_rate_dev(tbfp_handle *h, const double *ux, double *q) {
  int rc = check_ptrs(h, {ux, q});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = face_sum(h, 1, ux, h->Lux, q))) return rc;
  return finish(h, "tbfp_flow_rate");
}

int tbfp_flow_rate(tbfp_handle *h, const double *ux, double *q) {
  int rc = check_ptrs(h, {ux, q});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, false)) || (rc = h2d(h, h->h_ux, ux, h->n_ux))) return rc;
  if ((rc = face_sum(h, 1, h->h_ux, h->Lux, q))) return rc;
  return finish(h, "tbfp_flow_rate");
}

int tbfp_add_ux_dev(tbfp_handle *h, double *ux, double uf) {
  int rc = check_ptrs(h, {ux});
  if (rc) return rc;
  cudaSetDevice(h->device);
  launch_add_ux(ux, h->Lux, h->nx, h->ny, h->nz, uf, h->stream);
  return finish(h, "tbfp_add_ux");
}

int tbfp_add_ux(tbfp_handle *h, double *ux, double uf) {
  int rc = check_ptrs(h, {ux});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, false)) || (rc = h2d(h, h->h_ux, ux, h->n_ux))) return rc;
  launch_add_ux(h->h_ux, h->Lux, h->nx, h->ny, h->nz, uf, h->stream);
  if ((rc = d2h(h, ux, h->h_ux, h->n_ux))) return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return finish(h, "tbfp_add_ux");
}

// ---------------------------------------------------------------------------
// surface tension (computeSurfaceTension, VOF.f90:1872-2002), grid-wide
// ---------------------------------------------------------------------------
int tbfp_surface_tension_dev(tbfp_handle *h, const double *c, double sigma, double *kappa, double *st_x,
                             double *st_y, double *st_z) {
  int rc = check_ptrs(h, {c, st_x, st_y, st_z});
  if (rc) return rc;
  if (h->slab) return set_err(h, TBFP_EINVAL, "tbfp_surface_tension: not available on a slab handle");
  if (!std::isfinite(sigma)) return set_err(h, TBFP_EINVAL, "tbfp_surface_tension: sigma must be finite");
  cudaSetDevice(h->device);
  const long n = (long)h->nx * h->ny * h->nz;
  if (!h->d_st_cp) {
    std::vector<double> dyc(h->mdyc.begin(), h->mdyc.end()), yf(h->ny + 1, 0.0);
    double acc = 0.0;
    for (int m = 0; m < h->ny; ++m) {  // face positions: sequential sums of dyf
      acc = acc + h->mdyf[m];
      yf[m + 1] = acc;
    }
    if ((rc = upload(h, &h->d_st_dyc, dyc)) || (rc = upload(h, &h->d_st_yf, yf)) ||
        (rc = dev_alloc(h, &h->d_st_cp, (size_t)n)) || (rc = dev_alloc(h, &h->d_st_kap, (size_t)n)) ||
        (rc = dev_alloc(h, &h->d_st_fl, (size_t)n)))
      return rc;
  }
  StGrid g{};
  g.nx = h->nx;
  g.ny = h->ny;
  g.nz = h->nz;
  g.dx = h->dx_fft;
  g.dz = h->dz_fft;
  g.dyf = h->d_dyf;
  g.dyc = h->d_st_dyc;
  g.yf = h->d_st_yf;
  launch_surface_tension(c, h->Lrho, g, 1e-12, sigma, h->d_st_cp, h->d_st_fl, h->d_st_kap, kappa, h->Lrho,
                         (long)h->n_rho, st_x, h->Lst[0], (long)h->n_st[0], st_y, h->Lst[1], (long)h->n_st[1], st_z,
                         h->Lst[2], (long)h->n_st[2], h->stream);
  return finish(h, "tbfp_surface_tension");
}

int tbfp_surface_tension(tbfp_handle *h, const double *c, double sigma, double *kappa, double *st_x, double *st_y,
                         double *st_z) {
  int rc = check_ptrs(h, {c, st_x, st_y, st_z});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, true))) return rc;
  if (kappa && !h->h_kap && (rc = dev_alloc(h, &h->h_kap, h->n_rho))) return rc;
  if ((rc = h2d(h, h->h_rho, c, h->n_rho))) return rc;
  const unsigned fl = h->flags;
  h->flags |= TBFP_FLAG_ASYNC;
  rc = tbfp_surface_tension_dev(h, h->h_rho, sigma, kappa ? h->h_kap : nullptr, h->h_st[0], h->h_st[1], h->h_st[2]);
  h->flags = fl;
  if (rc) return rc;
  if ((rc = d2h(h, st_x, h->h_st[0], h->n_st[0])) || (rc = d2h(h, st_y, h->h_st[1], h->n_st[1])) ||
      (rc = d2h(h, st_z, h->h_st[2], h->n_st[2])))
    return rc;
  if (kappa && (rc = d2h(h, kappa, h->h_kap, h->n_rho))) return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return TBFP_OK;
}

int tbfp_pcg_setup(tbfp_handle *h, const tbfp_mg_params *p) {
  if (!h || !p) return TBFP_ENULL;
  cudaSetDevice(h->device);
  MgSolver *mg = new MgSolver();
  std::string e;
  const int rc = mg->init(*p, h->nx, h->ny, h->nz, h->mdxf.data(), h->mdxc.data(), h->mdyf.data(), h->mdyc.data(),
                          h->mdzf.data(), h->mdzc.data(), &e);
  if (rc != TBFP_OK) {
    delete mg;
    return set_err(h, rc, e);
  }
  delete h->mg;
  h->mg = mg;
  return TBFP_OK;
}

int tbfp_pcg_solve_dev(tbfp_handle *h, double *psi, const double *beta, const double *q, tbfp_stats *stats) {
  int rc = check_ptrs(h, {psi, beta, q});
  if (rc) return rc;
  if (!h->mg) return set_err(h, TBFP_EINVAL, "tbfp_pcg_solve: call tbfp_pcg_setup first");
  cudaSetDevice(h->device);
  TBFP_CK(h, cudaEventRecord(h->ev0, h->stream));
  int iters = 0, cycles = 0;
  double rel = -1.0;
  std::string err;
  const int src = h->mg->solve(psi, h->Lpsi, h->hd_psi, beta, h->Lrho, q, h->Lpsi, h->stream, &iters, &rel, &cycles,
                               &err);
  if (src < 0) return set_err(h, src, err);
  TBFP_CK(h, cudaEventRecord(h->ev1, h->stream));
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last = tbfp_stats{};
  h->last.iterations = iters;
  h->last.rel_residual = rel;
  h->last.max_div = -1.0;
  h->last.cont_err = -1.0;
  h->last.ms_device = ms;
  h->last.ms_stage[0] = cycles;  // V-cycles in total (informational)
  if (stats) *stats = h->last;
  return src;
}

int tbfp_projection_mg_dev(tbfp_handle *h, const double *ux_in, const double *uy_in, const double *uz_in,
                           double *ux_out, double *uy_out, double *uz_out, const double *rho, double dt, double alpha,
                           double *psi, tbfp_stats *stats) {
  int rc = check_ptrs(h, {ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, rho, psi});
  if (rc) return rc;
  if (!h->mg) return set_err(h, TBFP_EINVAL, "tbfp_projection_mg: call tbfp_pcg_setup first");
  if (!(dt > 0.0) || !(alpha > 0.0)) return set_err(h, TBFP_EINVAL, "tbfp_projection_mg: dt and alpha must be positive");
  cudaSetDevice(h->device);
  cudaStream_t s = h->stream;
  const double dta = dt * alpha;
  TBFP_CK(h, cudaEventRecord(h->ev0, s));
  // q = div u* into the s scratch, beta = dt alpha / rho into the 1/rho scratch
  launch_mg_source_beta(ux_in, uy_in, uz_in, h->Lux, h->Luy, h->Luz, rho, h->Lrho, h->g, dta, h->d_s, h->Lpsi,
                        h->d_irho, s);
  int iters = 0, cycles = 0;
  double rel = -1.0;
  std::string err;
  const int src = h->mg->solve(psi, h->Lpsi, h->hd_psi, h->d_irho, h->Lrho, h->d_s, h->Lpsi, s, &iters, &rel, &cycles,
                               &err);
  if (src < 0) return set_err(h, src, err);
  launch_add_pressure_grad(ux_in, uy_in, uz_in, ux_out, uy_out, uz_out, h->Lux, h->Luy, h->Luz, psi, h->Lpsi, rho,
                           h->Lrho, h->g, h->d_idxc, h->d_idzc, dta, s);
  TBFP_CK(h, cudaMemsetAsync(h->d_maxdiv, 0, sizeof(unsigned long long), s));
  launch_div(ux_out, uy_out, uz_out, h->Lux, h->Luy, h->Luz, h->g, h->d_maxdiv, s);
  TBFP_CK(h, cudaEventRecord(h->ev1, s));
  unsigned long long bits = 0;
  TBFP_CK(h, cudaMemcpyAsync(&bits, h->d_maxdiv, sizeof(bits), cudaMemcpyDeviceToHost, s));
  TBFP_CK(h, cudaStreamSynchronize(s));
  double md;
  std::memcpy(&md, &bits, sizeof(md));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->last = tbfp_stats{};
  h->last.iterations = iters;
  h->last.rel_residual = rel;
  h->last.max_div = md;
  h->last.cont_err = md * dt;
  h->last.ms_device = ms;
  h->last.ms_stage[0] = cycles;
  if (stats) *stats = h->last;
  const int frc = finish(h, "tbfp_projection_mg");
  return frc ? frc : src;
}

int tbfp_projection_mg(tbfp_handle *h, double *ux, double *uy, double *uz, const double *rho, double dt, double alpha,
                       double *psi, tbfp_stats *stats) {
  int rc = check_ptrs(h, {ux, uy, uz, rho, psi});
  if (rc) return rc;
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, false))) return rc;
  if ((rc = h2d(h, h->h_ux, ux, h->n_ux)) || (rc = h2d(h, h->h_uy, uy, h->n_uy)) ||
      (rc = h2d(h, h->h_uz, uz, h->n_uz)) || (rc = h2d(h, h->h_rho, rho, h->n_rho)) ||
      (rc = h2d(h, h->h_psi, psi, h->n_psi)))
    return rc;
  const int prc = tbfp_projection_mg_dev(h, h->h_ux, h->h_uy, h->h_uz, h->h_ux, h->h_uy, h->h_uz, h->h_rho, dt, alpha,
                                         h->h_psi, stats);
  if (prc < 0) return prc;
  if ((rc = d2h(h, ux, h->h_ux, h->n_ux)) || (rc = d2h(h, uy, h->h_uy, h->n_uy)) ||
      (rc = d2h(h, uz, h->h_uz, h->n_uz)) || (rc = d2h(h, psi, h->h_psi, h->n_psi)))
    return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return prc;
}

int tbfp_pcg_solve(tbfp_handle *h, double *psi, const double *beta, const double *q, tbfp_stats *stats) {
  int rc = check_ptrs(h, {psi, beta, q});
  if (rc) return rc;
  if (!h->mg) return set_err(h, TBFP_EINVAL, "tbfp_pcg_solve: call tbfp_pcg_setup first");
  cudaSetDevice(h->device);
  if ((rc = ensure_host_bufs(h, false))) return rc;
  if (!h->h_beta && ((rc = dev_alloc(h, &h->h_beta, h->n_rho)) || (rc = dev_alloc(h, &h->h_q, h->n_psi)))) return rc;
  if ((rc = h2d(h, h->h_psi, psi, h->n_psi)) || (rc = h2d(h, h->h_beta, beta, h->n_rho)) ||
      (rc = h2d(h, h->h_q, q, h->n_psi)))
    return rc;
  const int src = tbfp_pcg_solve_dev(h, h->h_psi, h->h_beta, h->h_q, stats);
  if (src < 0) return src;
  if ((rc = d2h(h, psi, h->h_psi, h->n_psi))) return rc;
  TBFP_CK(h, cudaStreamSynchronize(h->stream));
  return src;
}

// ---------------------------------------------------------------------------
// Ensemble: many independent channels per GPU in one call, in one of two forms:
//   graph:      each member's kernels on a pool of streams, captured once as a
//               CUDA graph and replayed while the arrays and scalars stay the
//               same (TBFP_MIXED members keep their device-side refinement
//               loops inside the graph);
//   persistent: every stage of every member in ONE launch of resident blocks
//               that take (member, stage, tile) items from a device work queue
//               (tbfp_ensemble.cu), that launch captured in a graph with the
//               reset of the queue.  FP64 out-of-place members whose lengths
//               the persistent kernel is compiled for (nx/2, nz <= 128,
//               ceil(ny/32) <= 8).
// TBFP_ENS_AUTO times the candidates (the graph, the persistent kernel at one
// and two blocks per SM) on the first call for a set of arrays, keeps the
// fastest and records it in the tuning cache file, keyed by the device and
// the members' sizes; later ensembles of the same sizes read the choice back.
// ---------------------------------------------------------------------------
}  // extern "C"

struct tbfp_ensemble {
  std::vector<tbfp_handle *> h;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> ev;  // [0] fork, [1..] joins
  int device = 0;
  bool graphable = true;        // the multi-stream form may be captured
  bool persistent_ok = true;    // every member fits the persistent kernel
  int mode = TBFP_ENS_AUTO;     // requested form
  int param = 0;                // requested blocks per SM of the persistent form (0: occupancy)
  int use_mode = 0, use_param = 0;  // form in use once chosen
  long long spin_limit = 10000000;  // polls of a dependency wait (~0.1 us each)
  std::string sizes_key;
  // graph form
  cudaGraphExec_t graph = nullptr;
  std::vector<tbfp_member_io> key;
  double kdt = 0.0, kalpha = 0.0, krho0 = 0.0;
  // persistent form
  size_t smem = 0;
  EnsMember *d_mem = nullptr;
  int *d_qstart = nullptr;
  EnsCtl *d_ctl = nullptr;
  size_t ctl_bytes = 0;
  int total_items = 0;
  cudaGraphExec_t pgraph = nullptr;
  int pgraph_blocks = 0;
  std::vector<tbfp_member_io> pkey;
  double pdt = 0.0, palpha = 0.0, prho0 = 0.0;
  float tuned_ms[3] = {-1.f, -1.f, -1.f};  // graph, persistent x1, persistent x2
};

namespace {
bool same_io(const tbfp_member_io &a, const tbfp_member_io &b) { return std::memcmp(&a, &b, sizeof(a)) == 0; }

int ensemble_launch_all(tbfp_ensemble *e, const tbfp_member_io *io, double dt, double alpha, double rho0) {
  const int ns = (int)e->streams.size();
  for (int s = 1; s < ns; ++s) cudaStreamWaitEvent(e->streams[s], e->ev[0], 0);
  for (size_t i = 0; i < e->h.size(); ++i) {
    const tbfp_member_io &m = io[i];
    const int rc = device_projection(e->h[i], m.ux_in, m.uy_in, m.uz_in, m.ux_out, m.uy_out, m.uz_out, m.rho,
                                     m.psi_n, m.psi_nm1, nullptr, nullptr, dt, alpha, rho0, m.psi, nullptr);
    if (rc < 0) {
      set_global_error(e->h[i]->err);
      return rc;
    }
  }
  for (int s = 1; s < ns; ++s) {
    cudaEventRecord(e->ev[s], e->streams[s]);
    cudaStreamWaitEvent(e->streams[0], e->ev[s], 0);
  }
  return TBFP_OK;
}

// The graph form: capture (when the arrays or scalars changed) and launch.
int ensemble_run_graph(tbfp_ensemble *e, const tbfp_member_io *io, double dt, double alpha, double rho0) {
  const int n = (int)e->h.size();
  cudaStream_t s0 = e->streams[0];
  if (!e->graphable) {
    cudaEventRecord(e->ev[0], s0);
    return ensemble_launch_all(e, io, dt, alpha, rho0);
  }
  bool reuse = e->graph && e->kdt == dt && e->kalpha == alpha && e->krho0 == rho0 && (int)e->key.size() == n;
  for (int i = 0; reuse && i < n; ++i) reuse = same_io(e->key[i], io[i]);
  if (!reuse) {
    if (e->graph) cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
    cudaGraph_t g = nullptr;
    int rc = TBFP_OK;
    cudaError_t ce = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      cudaEventRecord(e->ev[0], s0);
      rc = ensemble_launch_all(e, io, dt, alpha, rho0);
      ce = cudaStreamEndCapture(s0, &g);
    }
    if (rc < 0) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (ce != cudaSuccess)
      return set_err(nullptr, TBFP_ECUDA, std::string("tbfp_ensemble_projection: graph: ") + cudaGetErrorString(ce));
    e->key.assign(io, io + n);
    e->kdt = dt;
    e->kalpha = alpha;
    e->krho0 = rho0;
  }
  const cudaError_t ce = cudaGraphLaunch(e->graph, s0);
  if (ce != cudaSuccess)
    return set_err(nullptr, TBFP_ECUDA, std::string("tbfp_ensemble_projection: ") + cudaGetErrorString(ce));
  return TBFP_OK;
}

// A member as the persistent kernel sees it.
EnsMember ens_member(tbfp_handle *h, const tbfp_member_io &m, double dt, double alpha, double rho0) {
  EnsMember em{};
  em.g = h->g;
  em.ra = rhs_args(h, m.ux_in, m.uy_in, m.uz_in, m.psi_n, m.psi_nm1, nullptr, nullptr, dt, alpha, rho0);
  em.ca = corr_args(h, m.ux_in, m.uy_in, m.uz_in, m.ux_out, m.uy_out, m.uz_out, m.psi, m.psi_n, m.psi_nm1, nullptr,
                    nullptr, dt, alpha, rho0);
  em.xs = XSrc{};
  em.xs.s = h->d_s;
  em.xs.Ls = h->Lpsi;
  em.rho = m.rho;
  em.irho = h->d_irho;
  em.s = h->d_s;
  em.n_rho = (long)h->n_rho;
  em.spec = h->d_spec;
  em.psi = m.psi;
  em.Lpsi = h->Lpsi;
  em.hd_psi = h->hd_psi;
  em.twx = h->d_twx;
  em.tpx = h->d_tpx;
  em.tpz = h->d_tpz;
  em.lamx = h->d_lamx;
  em.lamz = h->d_lamz;
  em.am = h->d_am;
  em.ap = h->d_ap;
  em.dyf = h->d_dyf;
  em.mean_c = h->mean_c;
  em.nxnz = h->nxnz;
  em.scale = h->scale;
  em.maxdiv = h->d_maxdiv;
  em.T = tri_rows_per_lane(h->ny);
  ens_items(h->g, (long)h->n_rho, em.T, em.items);
  return em;
}

bool all_out_of_place(const tbfp_member_io *io, int n) {
  for (int i = 0; i < n; ++i)
    if (aliased(io[i].ux_in, io[i].ux_out) || aliased(io[i].uy_in, io[i].uy_out) ||
        aliased(io[i].uz_in, io[i].uz_out))
      return false;
  return true;
}

// The persistent form: upload the member table (when the arrays or scalars
// changed), capture [reset of the queue, one launch] as a graph, launch it.
int ensemble_run_persistent(tbfp_ensemble *e, const tbfp_member_io *io, double dt, double alpha, double rho0,
                            int blocks_per_sm) {
  const int n = (int)e->h.size();
  cudaStream_t s0 = e->streams[0];
  int dev_sms = 0;
  cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, e->device);
  const int occ = ensemble_blocks_per_sm(e->smem);
  if (occ < 1) return set_err(nullptr, TBFP_EUNSUPPORTED, "tbfp_ensemble_projection: persistent kernel does not fit");
  const int bps = (blocks_per_sm > 0 && blocks_per_sm < occ) ? blocks_per_sm : occ;
  const int blocks = bps * dev_sms;
  bool same = e->pgraph && e->pgraph_blocks == blocks && e->pdt == dt && e->palpha == alpha && e->prho0 == rho0 &&
              (int)e->pkey.size() == n;
  for (int i = 0; same && i < n; ++i) same = same_io(e->pkey[i], io[i]);
  if (!same) {
    bool table_same = (int)e->pkey.size() == n && e->pdt == dt && e->palpha == alpha && e->prho0 == rho0;
    for (int i = 0; table_same && i < n; ++i) table_same = same_io(e->pkey[i], io[i]);
    if (!table_same) {
      std::vector<EnsMember> mem(n);
      std::vector<int> qs(kEnsStages * n + 1, 0);
      for (int i = 0; i < n; ++i) mem[i] = ens_member(e->h[i], io[i], dt, alpha, rho0);
      int run = 0;
      for (int st = 0; st < kEnsStages; ++st)
        for (int i = 0; i < n; ++i) {
          qs[st * n + i] = run;
          run += mem[i].items[st];
        }
      qs[kEnsStages * n] = run;
      e->total_items = run;
      cudaStreamSynchronize(s0);  // the previous launch may still read the table
      if (cudaMemcpy(e->d_mem, mem.data(), sizeof(EnsMember) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(e->d_qstart, qs.data(), sizeof(int) * qs.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        return set_err(nullptr, TBFP_ECUDA, "tbfp_ensemble_projection: uploading the member table");
    }
    if (e->pgraph) cudaGraphExecDestroy(e->pgraph);
    e->pgraph = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal);
    if (ce == cudaSuccess) {
      cudaMemsetAsync(e->d_ctl, 0, e->ctl_bytes, s0);
      launch_ensemble_persistent(e->d_mem, n, e->d_qstart, e->d_ctl, e->spin_limit, blocks, e->smem, s0);
      ce = cudaStreamEndCapture(s0, &g);
    }
    if (ce == cudaSuccess) ce = cudaGraphInstantiate(&e->pgraph, g, 0);
    if (g) cudaGraphDestroy(g);
    if (ce != cudaSuccess)
      return set_err(nullptr, TBFP_ECUDA, std::string("tbfp_ensemble_projection: persistent graph: ") +
                                              cudaGetErrorString(ce));
    e->pgraph_blocks = blocks;
    e->pkey.assign(io, io + n);
    e->pdt = dt;
    e->palpha = alpha;
    e->prho0 = rho0;
  }
  const cudaError_t ce = cudaGraphLaunch(e->pgraph, s0);
  if (ce != cudaSuccess)
    return set_err(nullptr, TBFP_ECUDA, std::string("tbfp_ensemble_projection: ") + cudaGetErrorString(ce));
  return TBFP_OK;
}

// --- the tuning cache: one line per decision, "<key> <mode> <param> <ms>" ---
std::string tune_cache_path() {
  if (const char *p = std::getenv("TBFP_TUNE_CACHE")) return p;
  if (const char *x = std::getenv("XDG_CACHE_HOME")) return std::string(x) + "/tbfp_tune.txt";
  if (const char *hm = std::getenv("HOME")) return std::string(hm) + "/.cache/tbfp_tune.txt";
  return "";
}

bool tune_lookup(const std::string &key, int *mode, int *param) {
  const std::string path = tune_cache_path();
  if (path.empty()) return false;
  FILE *f = std::fopen(path.c_str(), "r");
  if (!f) return false;
  char k[512];
  int m = 0, p = 0;
  float ms = 0.f;
  bool found = false;
  while (std::fscanf(f, "%511s %d %d %f", k, &m, &p, &ms) == 4)
    if (key == k) {  // the last line for a key wins
      *mode = m;
      *param = p;
      found = true;
    }
  std::fclose(f);
  return found;
}

void tune_record(const std::string &key, int mode, int param, float ms) {
  const std::string path = tune_cache_path();
  if (path.empty()) return;
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos && slash > 0) mkdir(path.substr(0, slash).c_str(), 0755);  // one level, if missing
  FILE *f = std::fopen(path.c_str(), "a");
  if (!f) return;  // an unwritable cache only costs a new tuning next time
  std::fprintf(f, "%s %d %d %.4f\n", key.c_str(), mode, param, ms);
  std::fclose(f);
}

// Device time of one call of a form (after one untimed call).
int time_form(tbfp_ensemble *e, const tbfp_member_io *io, double dt, double alpha, double rho0, int mode, int param,
              float *ms) {
  cudaStream_t s0 = e->streams[0];
  cudaEvent_t a = nullptr, b = nullptr;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int rc = TBFP_OK;
  for (int rep = 0; rep < 4 && rc == TBFP_OK; ++rep) {
    if (rep == 1) cudaEventRecord(a, s0);
    rc = (mode == TBFP_ENS_GRAPH) ? ensemble_run_graph(e, io, dt, alpha, rho0)
                                  : ensemble_run_persistent(e, io, dt, alpha, rho0, param);
  }
  cudaEventRecord(b, s0);
  cudaError_t ce = cudaEventSynchronize(b);
  float t = 0.f;
  if (rc == TBFP_OK && ce == cudaSuccess) cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  if (ce != cudaSuccess) return set_err(nullptr, TBFP_ECUDA, std::string("ensemble tuning: ") + cudaGetErrorString(ce));
  *ms = t / 3.f;
  return TBFP_OK;
}

// Choose the form: the requested one, the cached choice, or a measurement.
int ensemble_choose(tbfp_ensemble *e, const tbfp_member_io *io, double dt, double alpha, double rho0) {
  const int n = (int)e->h.size();
  const bool pers = e->persistent_ok && all_out_of_place(io, n);
  if (e->mode == TBFP_ENS_GRAPH || (e->mode == TBFP_ENS_PERSISTENT && !pers)) {
    if (e->mode == TBFP_ENS_PERSISTENT)
      return set_err(nullptr, TBFP_EUNSUPPORTED,
                     "tbfp_ensemble_projection: the persistent form needs FP64 out-of-place members with "
                     "nx/2, nz <= 128 and ny <= 256");
    e->use_mode = TBFP_ENS_GRAPH;
    e->use_param = (int)e->streams.size();
    return TBFP_OK;
  }
  if (e->mode == TBFP_ENS_PERSISTENT) {
    e->use_mode = TBFP_ENS_PERSISTENT;
    e->use_param = e->param;
    return TBFP_OK;
  }
  if (!pers) {  // nothing to choose between
    e->use_mode = TBFP_ENS_GRAPH;
    e->use_param = (int)e->streams.size();
    return TBFP_OK;
  }
  int m = 0, p = 0;
  if (tune_lookup(e->sizes_key, &m, &p) && (m == TBFP_ENS_GRAPH || m == TBFP_ENS_PERSISTENT)) {
    e->use_mode = m;
    e->use_param = p;
    return TBFP_OK;
  }
  // measure: the graph, then the persistent kernel at 1 and 2 blocks per SM
  float best = 0.f;
  int bm = TBFP_ENS_GRAPH, bp = (int)e->streams.size();
  const int occ = ensemble_blocks_per_sm(e->smem);
  for (int c = 0; c < 3; ++c) {
    const int mode = c == 0 ? TBFP_ENS_GRAPH : TBFP_ENS_PERSISTENT;
    const int param = c == 0 ? (int)e->streams.size() : c;
    if (c > 0 && c > occ) continue;
    float ms = 0.f;
    const int rc = time_form(e, io, dt, alpha, rho0, mode, param, &ms);
    if (rc) return rc;
    e->tuned_ms[c] = ms;
    if (c == 0 || ms < best) {
      best = ms;
      bm = mode;
      bp = param;
    }
  }
  e->use_mode = bm;
  e->use_param = bp;
  tune_record(e->sizes_key, bm, bp, best);
  return TBFP_OK;
}
}  // namespace

extern "C" {

int tbfp_ensemble_create(int n, const tbfp_desc *descs, int nstreams, tbfp_ensemble **out) {
  set_global_error("");
  if (!descs || !out) return TBFP_ENULL;
  *out = nullptr;
  if (n < 1 || nstreams < 1) return set_err(nullptr, TBFP_EINVAL, "tbfp_ensemble_create: need n >= 1 and nstreams >= 1");
  tbfp_ensemble *e = new tbfp_ensemble();
  e->device = descs[0].device;
  if (e->device < 0) cudaGetDevice(&e->device);
  cudaSetDevice(e->device);
  const int ns = std::min(nstreams, n);
  e->streams.resize(ns, nullptr);
  e->ev.resize(ns, nullptr);
  auto fail = [&](int rc) {
    tbfp_ensemble_destroy(e);
    return rc;
  };
  for (int s = 0; s < ns; ++s) {
    if (cudaStreamCreateWithFlags(&e->streams[s], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->ev[s], cudaEventDisableTiming) != cudaSuccess)
      return fail(set_err(nullptr, TBFP_ECUDA, "tbfp_ensemble_create: stream or event creation failed"));
  }
  cudaDeviceProp prop{};
  cudaGetDeviceProperties(&prop, e->device);
  std::string sig;
  for (int i = 0; i < n; ++i) {
    tbfp_desc d = descs[i];
    if (d.device >= 0 && d.device != e->device)
      return fail(set_err(nullptr, TBFP_EINVAL, "tbfp_ensemble_create: members must share one device"));
    d.device = e->device;
    d.stream = e->streams[i % ns];
    d.flags = (d.flags | TBFP_FLAG_ASYNC) & ~TBFP_FLAG_TIMING;
    if (d.flags & TBFP_FLAG_RESIDUAL) e->graphable = false;  // reads its residual back on the host
    tbfp_handle *h = nullptr;
    const int rc = tbfp_create(&d, &h);
    if (rc < 0) {
      const std::string m = "tbfp_ensemble_create: member " + std::to_string(i) + ": " + g_create_error;
      tbfp_ensemble_destroy(e);
      return set_err(nullptr, rc, m);
    }
    e->h.push_back(h);
    const int T = tri_rows_per_lane(d.ny);
    if (d.precision != TBFP_FP64 || (d.flags & TBFP_FLAG_RESIDUAL) || !ens_supported(d.nx / 2, d.nz, T))
      e->persistent_ok = false;
    else e->smem = std::max(e->smem, ens_smem_bytes(d.nx / 2, d.nz, T));
    sig += std::to_string(d.nx) + "x" + std::to_string(d.ny) + "x" + std::to_string(d.nz) + ";";
  }
  // tuning-cache key: the device and the members' sizes (FNV-1a of the list)
  unsigned long long hsh = 1469598103934665603ull;
  for (char c : sig) hsh = (hsh ^ (unsigned char)c) * 1099511628211ull;
  std::string dev = prop.name;
  for (char &c : dev)
    if (c == ' ') c = '_';
  char kb[64];
  std::snprintf(kb, sizeof(kb), "%d-%016llx", n, hsh);
  e->sizes_key = "ensemble|" + dev + "|" + kb;
  if (e->persistent_ok) {
    e->ctl_bytes = sizeof(EnsCtl) + sizeof(int) * (size_t)n * kEnsStages;
    if (prepare_ensemble_kernel(e->smem) != cudaSuccess || cudaMalloc(&e->d_mem, sizeof(EnsMember) * n) != cudaSuccess ||
        cudaMalloc(&e->d_qstart, sizeof(int) * ((size_t)kEnsStages * n + 1)) != cudaSuccess ||
        cudaMalloc(&e->d_ctl, e->ctl_bytes) != cudaSuccess)
      return fail(set_err(nullptr, TBFP_ENOMEM, "tbfp_ensemble_create: persistent-form buffers"));
  }
  *out = e;
  return TBFP_OK;
}

int tbfp_ensemble_destroy(tbfp_ensemble *e) {
  if (!e) return TBFP_OK;
  cudaSetDevice(e->device);
  for (cudaStream_t s : e->streams)
    if (s) cudaStreamSynchronize(s);
  if (e->graph) cudaGraphExecDestroy(e->graph);
  if (e->pgraph) cudaGraphExecDestroy(e->pgraph);
  for (tbfp_handle *h : e->h) tbfp_destroy(h);
  for (cudaEvent_t v : e->ev)
    if (v) cudaEventDestroy(v);
  for (cudaStream_t s : e->streams)
    if (s) cudaStreamDestroy(s);
  if (e->d_mem) cudaFree(e->d_mem);
  if (e->d_qstart) cudaFree(e->d_qstart);
  if (e->d_ctl) cudaFree(e->d_ctl);
  delete e;
  return TBFP_OK;
}

int tbfp_ensemble_size(const tbfp_ensemble *e) { return e ? (int)e->h.size() : 0; }

int tbfp_ensemble_set_mode(tbfp_ensemble *e, int mode, int param) {
  set_global_error("");
  if (!e) return TBFP_ENULL;
  if (mode != TBFP_ENS_AUTO && mode != TBFP_ENS_GRAPH && mode != TBFP_ENS_PERSISTENT)
    return set_err(nullptr, TBFP_EINVAL, "tbfp_ensemble_set_mode: unknown mode");
  if (mode == TBFP_ENS_PERSISTENT && !e->persistent_ok)
    return set_err(nullptr, TBFP_EUNSUPPORTED,
                   "tbfp_ensemble_set_mode: the persistent form needs FP64 members with nx/2, nz <= 128 and "
                   "ny <= 256");
  e->mode = mode;
  e->param = param;
  e->use_mode = 0;  // choose again on the next call
  return TBFP_OK;
}

int tbfp_ensemble_get_mode(const tbfp_ensemble *e, int *mode, int *param, float *tuned_ms) {
  if (!e) return TBFP_ENULL;
  if (mode) *mode = e->use_mode;
  if (param) *param = e->use_param;
  if (tuned_ms)
    for (int c = 0; c < 3; ++c) tuned_ms[c] = e->tuned_ms[c];
  return TBFP_OK;
}

int tbfp_set_wait_limit(tbfp_handle *h, long long cycles) {
  if (!h) return TBFP_ENULL;
  if (cycles < 0) return set_err(h, TBFP_EINVAL, "tbfp_set_wait_limit: negative limit");
  h->wait_cycles = cycles;
  return TBFP_OK;
}

int tbfp_ensemble_set_wait_limit(tbfp_ensemble *e, long long polls) {
  if (!e) return TBFP_ENULL;
  if (polls < 0) return set_err(nullptr, TBFP_EINVAL, "tbfp_ensemble_set_wait_limit: negative limit");
  e->spin_limit = polls;
  if (e->pgraph) cudaGraphExecDestroy(e->pgraph);  // the limit is a launch argument: capture again
  e->pgraph = nullptr;
  return TBFP_OK;
}

int tbfp_ensemble_projection_dev(tbfp_ensemble *e, const tbfp_member_io *io, double dt, double alpha, double rho0,
                                 tbfp_stats *stats) {
  set_global_error("");
  if (!e || !io) return TBFP_ENULL;
  const int n = (int)e->h.size();
  for (int i = 0; i < n; ++i) {
    const tbfp_member_io &m = io[i];
    if (!m.ux_in || !m.uy_in || !m.uz_in || !m.ux_out || !m.uy_out || !m.uz_out || !m.rho || !m.psi_n ||
        !m.psi_nm1 || !m.psi)
      return set_err(nullptr, TBFP_ENULL, "tbfp_ensemble_projection: member " + std::to_string(i) + ": NULL array");
  }
  if (!(dt > 0.0) || !(alpha > 0.0) || !(rho0 > 0.0))
    return set_err(nullptr, TBFP_EINVAL, "tbfp_ensemble_projection: dt, alpha and rho0 must be positive");
  cudaSetDevice(e->device);
  cudaStream_t s0 = e->streams[0];
  int rc = TBFP_OK;
  if (e->use_mode == 0 || (e->use_mode == TBFP_ENS_PERSISTENT && !all_out_of_place(io, n))) {
    if (e->use_mode == TBFP_ENS_PERSISTENT) e->use_mode = 0;
    if ((rc = ensemble_choose(e, io, dt, alpha, rho0))) return rc;
  }
  rc = (e->use_mode == TBFP_ENS_PERSISTENT) ? ensemble_run_persistent(e, io, dt, alpha, rho0, e->use_param)
                                            : ensemble_run_graph(e, io, dt, alpha, rho0);
  if (rc < 0) return rc;
  const cudaError_t ce = cudaStreamSynchronize(s0);
  if (ce != cudaSuccess)
    return set_err(nullptr, TBFP_ECUDA, std::string("tbfp_ensemble_projection: ") + cudaGetErrorString(ce));
  if (e->use_mode == TBFP_ENS_PERSISTENT) {  // a dependency wait that ran out of polls stops the launch
    int abort_word = 0;
    if (cudaMemcpy(&abort_word, &e->d_ctl->abort, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return set_err(nullptr, TBFP_ECUDA, "tbfp_ensemble_projection: reading the work-queue state");
    if (abort_word)
      return set_err(nullptr, TBFP_ETIMEOUT,
                     "tbfp_ensemble_projection: a dependency wait of the persistent kernel ran out of polls");
  }
  rc = TBFP_OK;
  if (stats) {
    for (int i = 0; i < n; ++i) {
      unsigned long long bits = 0;
      if (cudaMemcpy(&bits, e->h[i]->d_maxdiv, sizeof(bits), cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_err(nullptr, TBFP_ECUDA, "tbfp_ensemble_projection: reading the continuity error");
      double md;
      std::memcpy(&md, &bits, sizeof(md));
      stats[i] = tbfp_stats{};
      stats[i].iterations = 1;
      stats[i].rel_residual = -1.0;
      stats[i].max_div = md;
      stats[i].cont_err = md * dt;
      if (e->h[i]->precision == TBFP_MIXED) {
        const int mrc = read_mixed(e->h[i], &stats[i].iterations, &stats[i].rel_residual, nullptr);
        if (mrc < 0) return set_err(nullptr, mrc, "tbfp_ensemble_projection: member " + std::to_string(i) + ": " +
                                                       e->h[i]->err);
        if (mrc > rc) rc = mrc;
      }
      if (!std::isfinite(md))
        return set_err(nullptr, TBFP_ENONFINITE,
                       "tbfp_ensemble_projection: member " + std::to_string(i) + ": non-finite max|div u|");
    }
  }
  return rc;
}

}  // extern "C"
