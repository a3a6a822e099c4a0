// Velocity correction with the continuity check (makeVelocityDivFree FAST,
// momentumEqn.f90:999-1127, and computeContinuityError,
// auxiliaryRoutines.f90:42-91), with its inputs staged by the tensor memory
// accelerator (TMA).
//
// A CTA owns an x-y tile of kCTX x TY cells and marches a chunk of z planes.
// For every plane, one thread issues the tiled bulk copies
// (cp.async.bulk.tensor, no multicast): psi, psi^n, psi^(n-1) and 1/rho with a
// one-cell halo in x and y, and the tile's ux, uy (with the face below the
// tile) and uz.  The copies of a plane complete on one mbarrier.  NS slots
// form a ring: while the threads correct plane k from the slots of planes k
// and k+1, the copies of planes k+2 .. k+NS-2 are in flight, so the load
// parallelism comes from the copy engine instead of from resident warps.  The
// lower z face of a plane is the upper face of the plane before (carried in
// registers); the chunk's first plane computes it from one extra plane.  The x
// face below cell i = 1 is the upper face of cell nx (the periodic image),
// whose nine inputs per row come in by 8-byte cp.async copies in the same ring.
//
// Every face is computed with the arguments and in the operation order of
// correct_div_body (the kernel form, which serves surface tension and arrays
// that a tensor map cannot describe).  A wait on a copy is bounded
// (CorrArgs::wait_cycles): past the limit the CTA waits (with the default
// bound) for its copies in flight, folds kWaitTimeoutBits into *maxdiv, which
// the host reports as TBFP_ETIMEOUT, and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"
#include "tbfp_stages.cuh"

namespace tbfp {

namespace {

constexpr int kCTX = 128;  // tile width; a CTA's threads are 128 columns x NT/128 row groups
constexpr int kPer = 9;                               // periodic inputs per row
constexpr int kCorrTmaMaxSmem = 220 * 1024;  // under the opt-in limit with the static reduction buffer

__host__ __device__ constexpr int align128(int b) { return (b + 127) & ~127; }

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_test_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// A first look that does not block, then waits (try_wait suspends the thread
// for a while inside the instruction) until the bound in SM cycles runs out.
__device__ bool mbar_wait_bounded(unsigned bar, unsigned parity, long long limit) {
  if (mbar_test_wait(bar, parity)) return true;
  if (limit <= 0) return false;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}
__device__ __forceinline__ void tma_load2(unsigned dst, const CUtensorMap *map, int x, int y, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void tma_load3(unsigned dst, const CUtensorMap *map, int x, int y, int z, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// Box geometry of one array: the first box column/row (array indices, for the
// tile at the origin), the offset of the first needed column inside the box
// (the box starts on an even index: 16-byte rule), the box width, and the
// array index of plane 0.
struct BoxGeom {
  int xo, dx, w, yo, zo;
};
// ux rows are nx + 1 + 2 halo long (odd), so its row stride is no multiple of
// 16 bytes: its tensor map is 2-D (the flattened x-y plane, z) and each tile
// row is its own box of kUxW values starting on an even element.
constexpr int kUxW = kCTX + 2;
constexpr int kUxLd = 144;  // shared-memory row slot of ux: kUxW values, 1152 bytes (a copy lands on 128 bytes)
struct UxGeom {
  int fx, yo, zo, sj;  // x index of face i0-1 at the origin tile, row index of row j0 = 1, plane 0, row stride
};
struct CorrTmaGeom {
  BoxGeom ps, ir, uy, uz;  // psi, psi^n, psi^(n-1) share the psi layout
  UxGeom ux;
  int nzc;  // planes per chunk
};

// shared-memory carve-up of one ring slot (bytes), from the box widths
struct CorrTmaSmem {
  int sps, sir;             // one psi-layout plane, one 1/rho plane
  int sux, suy, suz, sper;  // velocity boxes, the periodic column
  int slot, total;
};
__host__ __device__ inline CorrTmaSmem corr_tma_smem(const CorrTmaGeom &q, int ty, int ns) {
  CorrTmaSmem m;
  m.sps = align128(q.ps.w * (ty + 2) * 8);
  m.sir = align128(q.ir.w * (ty + 2) * 8);
  m.sux = kUxLd * ty * 8;
  m.suy = align128(q.uy.w * (ty + 1) * 8);
  m.suz = align128(q.uz.w * ty * 8);
  m.sper = align128(kPer * ty * 8);
  m.slot = 3 * m.sps + m.sir + m.sux + m.suy + m.suz + m.sper;
  m.total = ns * m.slot + ns * 8;
  return m;
}

template <int TY, int NS, int NT>
__global__ void __launch_bounds__(NT, 1)
    k_correct_tma(const __grid_constant__ CUtensorMap m_ps, const __grid_constant__ CUtensorMap m_pn,
                  const __grid_constant__ CUtensorMap m_po, const __grid_constant__ CUtensorMap m_ir,
                  const __grid_constant__ CUtensorMap m_ux, const __grid_constant__ CUtensorMap m_uy,
                  const __grid_constant__ CUtensorMap m_uz, CorrArgs a, GridK g, CorrTmaGeom q,
                  unsigned long long *__restrict__ maxdiv) {
  constexpr int NG = NT / kCTX, RPT = TY / NG;  // row groups, consecutive rows per thread
  static_assert(NT % kCTX == 0 && TY % NG == 0 && NS >= 3, "whole row groups; at least one plane in flight");
  extern __shared__ __align__(128) unsigned char smc[];
  const int tid = threadIdx.x, tx = tid & (kCTX - 1), tg = tid / kCTX;
  const int bx = blockIdx.x, by = blockIdx.y;
  const int i0 = 1 + kCTX * bx, j0 = 1 + TY * by;
  const int k0 = 1 + q.nzc * (int)blockIdx.z;
  if (k0 > g.nz) return;  // whole CTA
  const int k1 = min(k0 + q.nzc - 1, g.nz);
  const int km0 = (k0 == 1 && !g.slab) ? g.nz : k0 - 1;
  const CorrTmaSmem L = corr_tma_smem(q, TY, NS);
  // NS slots [psi | psi^n | psi^(n-1) | 1/rho | ux | uy | uz | periodic], copy
  // destinations on 128-byte boundaries (the launch adds 128 bytes of slack)
  unsigned char *base = smc + ((128u - (smem_u32(smc) & 127u)) & 127u);
  unsigned long long *bars = reinterpret_cast<unsigned long long *>(base + NS * L.slot);
  const int o_pn = L.sps, o_po = 2 * L.sps, o_ir = 3 * L.sps, o_ux = o_ir + L.sir, o_uy = o_ux + L.sux,
            o_uz = o_uy + L.suy, o_per = o_uz + L.suz;
  const unsigned bps = (unsigned)(q.ps.w * (TY + 2) * 8), bir = (unsigned)(q.ir.w * (TY + 2) * 8);
  const unsigned bux = (unsigned)(kUxW * TY * 8), buy = (unsigned)(q.uy.w * (TY + 1) * 8),
                 buz = (unsigned)(q.uz.w * TY * 8);

  if (tid == 0) {
    for (int m = 0; m < NS; ++m) mbar_init(smem_u32(bars + m), 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  __syncthreads();

  // stage t: plane p_t (p_{-1} = km0, p_t = k0 + t) into slot (t+1)%NS on
  // mbarrier (t+1)%NS: the four scalar boxes and uz, and for t >= 0 also ux,
  // uy and the periodic column
  auto issue = [&](int t) {
    const int pl = (t < 0) ? km0 : k0 + t;
    const int S = (t + 1) % NS;
    unsigned char *s = base + S * L.slot;
    if (tid == 0) {
      const unsigned bar = smem_u32(bars + S);
      mbar_expect_tx(bar, 3 * bps + bir + buz + (t >= 0 ? bux + buy : 0u));
      const int xs = q.ps.xo + kCTX * bx, ys = q.ps.yo + TY * by, zs = q.ps.zo + pl;
      tma_load3(smem_u32(s), &m_ps, xs, ys, zs, bar);
      tma_load3(smem_u32(s + o_pn), &m_pn, xs, ys, zs, bar);
      tma_load3(smem_u32(s + o_po), &m_po, xs, ys, zs, bar);
      tma_load3(smem_u32(s + o_ir), &m_ir, q.ir.xo + kCTX * bx, q.ir.yo + TY * by, q.ir.zo + pl, bar);
      if (t >= 0) {
        for (int r = 0; r < TY; ++r) {
          const int e = (q.ux.yo + TY * by + r) * q.ux.sj + q.ux.fx + kCTX * bx;
          tma_load2(smem_u32(s + o_ux + r * kUxLd * 8), &m_ux, e & ~1, q.ux.zo + pl, bar);
        }
        tma_load3(smem_u32(s + o_uy), &m_uy, q.uy.xo + kCTX * bx, q.uy.yo + TY * by, q.uy.zo + pl, bar);
      }
      tma_load3(smem_u32(s + o_uz), &m_uz, q.uz.xo + kCTX * bx, q.uz.yo + TY * by, q.uz.zo + pl, bar);
    }
    if (bx == 0 && t >= 0 && tid < kPer * TY) {
      // inputs of the upper x face of cell nx, row j (clamped into the array)
      const int r = tid / kPer, v = tid - r * kPer, j = min(j0 + r, g.ny);
      const int ic = g.nx + (v < 8 ? (v & 1) : 0);
      const double *src;
      if (v < 2) src = a.psi + at(a.Lpsi, ic, j, pl);
      else if (v < 4) src = a.pn + at(a.Lpsi, ic, j, pl);
      else if (v < 6) src = a.pnm1 + at(a.Lpsi, ic, j, pl);
      else if (v < 8) src = a.irho + at(a.Lrho, ic, j, pl);
      else src = a.uxi + at(a.Lux, g.nx, j, pl);
      cp_async8(reinterpret_cast<double *>(s + o_per) + v * TY + r, src);
    }
    cp_async_commit();
  };

  const int nlast = k1 - k0, tmax = nlast + 1;
  int waited = -1;  // the next stage to wait for
  int issued = -1;  // the last stage issued
  for (int t = -1; t <= NS - 2; ++t) {  // one cp.async group per stage, issued or not
    if (t <= tmax) {
      issue(t);
      issued = t;
    } else {
      cp_async_commit();
    }
  }
  auto drain_and_fail = [&]() {
    // the copies in flight land before the CTA leaves (waits of the default bound)
    if (tid == 0)
      for (int t = waited; t <= issued; ++t)
        mbar_wait_bounded(smem_u32(bars + (t + 1) % NS), (unsigned)(((t + 1) / NS) & 1), kDefaultWaitCycles);
    cp_async_wait_all();
    __syncthreads();
    if (tid == 0) atomicMax(maxdiv, kWaitTimeoutBits);  // a copy did not complete within the bound
  };
  const long long lim = a.wait_cycles;

  const double R = a.r, ir0 = a.invrho0, idxc = g.idxc1, idzc = g.idzc1;
  const int i = i0 + tx;
  const bool col = i <= g.nx;
  const double idx = col ? g.idxf[i - 1] : 0.0;
  auto dslot = [&](int S, int off) { return reinterpret_cast<const double *>(base + S * L.slot + off); };

  // the lower z face of the chunk's first plane, from planes km0 (slot 0) and
  // k0 (slot 1); plane k0+1 (slot 2) is waited for as well
  double uzq[RPT];
  {
    bool bad = !mbar_wait_bounded(smem_u32(bars + 0), 0u, lim);
    bad = !mbar_wait_bounded(smem_u32(bars + 1), 0u, lim) || bad;
    bad = !mbar_wait_bounded(smem_u32(bars + 2 % NS), (unsigned)((2 / NS) & 1), lim) || bad;
    cp_async_wait_group<NS - 2>();  // the periodic columns of stages -1 and 0
    if (__syncthreads_or(bad)) {
      drain_and_fail();
      return;
    }
    waited = 2;
    const double *P0 = dslot(0, 0), *P1 = dslot(1, 0), *Uzm = dslot(0, o_uz);
    const int so = L.sps / 8, io = o_ir / 8;
#pragma unroll
    for (int qq = 0; qq < RPT; ++qq) {
      const int r = RPT * tg + qq;
      const int rs = (r + 1) * q.ps.w + q.ps.dx + 1 + tx, ri = (r + 1) * q.ir.w + q.ir.dx + 1 + tx;
      uzq[qq] = face_update(Uzm[r * q.uz.w + q.uz.dx + tx], R, ir0, P1[io + ri], P0[io + ri], idzc, P1[rs], P0[rs],
                            P1[so + rs], P0[so + rs], P1[2 * so + rs], P0[2 * so + rs], 0.0);
    }
  }
  __syncthreads();  // slot 0 (plane km0) is free
  if (NS - 1 <= tmax) {
    issue(NS - 1);
    issued = NS - 1;
  } else {
    cp_async_commit();  // keeps one group per stage
  }

  // One barrier per plane: after plane k, wait for the copies of plane k+2
  // and the periodic column of plane k+1, then one barrier both publishes
  // them to every thread and frees the slot of plane k for plane k+NS.
  // y metrics of the thread's rows, read once (a store to u may alias the
  // tables as far as the compiler knows, so they would be reloaded per plane)
  double m_idycp[RPT], m_idyf[RPT], m_idycm = 0.0;
#pragma unroll
  for (int qq = 0; qq < RPT; ++qq) {
    const int j = j0 + RPT * tg + qq;
    m_idycp[qq] = (j < g.ny) ? g.idyc[j] : 0.0;
    m_idyf[qq] = (j <= g.ny) ? g.idyf[j - 1] : 0.0;
  }
  {
    const int j = j0 + RPT * tg;
    if (j > 1 && j <= g.ny) m_idycm = g.idyc[j - 1];
  }

  double vmax = 0.0;
  for (int n = 0; n <= nlast; ++n) {
    const int k = k0 + n;
    const int K = (n + 1) % NS, K1 = (n + 2) % NS;
    const double *Sps = dslot(K, 0), *Spn = dslot(K, o_pn), *Spo = dslot(K, o_po), *Sir = dslot(K, o_ir);
    const double *Tps = dslot(K1, 0), *Tpn = dslot(K1, o_pn), *Tpo = dslot(K1, o_po), *Tir = dslot(K1, o_ir);
    const double *Ux = dslot(K, o_ux), *Uy = dslot(K, o_uy), *Uz = dslot(K, o_uz), *Pe = dslot(K, o_per);
    const double idz = g.idzf[k - 1];
    double uym = 0.0;
#pragma unroll
    for (int qq = 0; qq < RPT; ++qq) {
      const int r = RPT * tg + qq, j = j0 + r;
      const int rs = (r + 1) * q.ps.w + q.ps.dx + 1 + tx, ri = (r + 1) * q.ir.w + q.ir.dx + 1 + tx;
      const double psc = Sps[rs], pnc = Spn[rs], poc = Spo[rs], irc = Sir[ri];
      // upper and lower x faces (ux(i) at column rx + 1 of the row's box)
      const int rx = r * kUxLd + (((q.ux.yo + TY * by + r) * q.ux.sj + q.ux.fx) & 1) + tx;
      const double uxp = face_update(Ux[rx + 1], R, ir0, Sir[ri + 1], irc, idxc, Sps[rs + 1], psc, Spn[rs + 1], pnc,
                                     Spo[rs + 1], poc, 0.0);
      double uxm;
      if (i == 1) {
        uxm = face_update(Pe[8 * TY + r], R, ir0, Pe[7 * TY + r], Pe[6 * TY + r], idxc, Pe[1 * TY + r],
                          Pe[0 * TY + r], Pe[3 * TY + r], Pe[2 * TY + r], Pe[5 * TY + r], Pe[4 * TY + r], 0.0);
      } else {
        uxm = face_update(Ux[rx], R, ir0, irc, Sir[ri - 1], idxc, psc, Sps[rs - 1], pnc, Spn[rs - 1], poc,
                          Spo[rs - 1], 0.0);
      }
      // upper y face (the top wall face is copied), lower y face
      const double uyc = Uy[(r + 1) * q.uy.w + q.uy.dx + tx];
      const double uyp = (j < g.ny) ? face_update(uyc, R, ir0, Sir[ri + q.ir.w], irc, m_idycp[qq], Sps[rs + q.ps.w],
                                                  psc, Spn[rs + q.ps.w], pnc, Spo[rs + q.ps.w], poc, 0.0)
                                    : uyc;
      if (qq == 0) {
        const double uyb = Uy[r * q.uy.w + q.uy.dx + tx];
        if (j == 1) {
          uym = uyb;
          if (col) a.uyo[at(a.Luy, i, 0, k)] = uyb;  // the wall face below row 1
        } else if (j <= g.ny) {
          uym = face_update(uyb, R, ir0, irc, Sir[ri - q.ir.w], m_idycm, psc, Sps[rs - q.ps.w], pnc,
                            Spn[rs - q.ps.w], poc, Spo[rs - q.ps.w], 0.0);
        } else {
          uym = 0.0;  // a row past ny: nothing is stored
        }
      }
      // upper z face; the lower one is the previous plane's upper face
      const double uzp = face_update(Uz[r * q.uz.w + q.uz.dx + tx], R, ir0, Tir[ri], irc, idzc, Tps[rs], psc,
                                     Tpn[rs], pnc, Tpo[rs], poc, 0.0);
      const double uzl = uzq[qq];
      uzq[qq] = uzp;
      if (col && j <= g.ny) {
        const long ox = at(a.Lux, i, j, k);
        a.uxo[ox] = uxp;
        if (i == g.nx) a.uxo[ox - i] = uxp;  // ux(0, j, k)
        a.uyo[at(a.Luy, i, j, k)] = uyp;
        const long oz = at(a.Luz, i, j, k);
        a.uzo[oz] = uzp;
        if (k == g.nz && !g.slab) a.uzo[oz - (long)k * a.Luz.sk] = uzp;  // uz(i, j, 0)
        double dv = (uxp - uxm) * idx;
        dv = dv + (uyp - uym) * m_idyf[qq];
        dv = dv + (uzp - uzl) * idz;
        vmax = nanmax_nonneg(vmax, dv);
      }
      uym = uyp;
    }
    if (n == nlast) break;
    {
      const int t = n + 2;  // plane k+2 (t <= tmax since n < nlast)
      const bool bad = !mbar_wait_bounded(smem_u32(bars + (t + 1) % NS), (unsigned)(((t + 1) / NS) & 1), lim);
      cp_async_wait_group<NS - 2>();  // the periodic column of plane k+1
      if (__syncthreads_or(bad)) {
        drain_and_fail();
        return;
      }
      waited = t + 1;
    }
    if (n + NS <= tmax) {  // into the slot of plane k
      issue(n + NS);
      issued = n + NS;
    } else {
      cp_async_commit();
    }
  }
  cp_async_wait_all();  // the periodic copies of stages past the chunk (not read)
  block_max_atomic(vmax, maxdiv);
}

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = []() -> EncodeTiledFn {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &qr) != cudaSuccess ||
        qr != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

// Box geometry of an array with layout Ly: needed columns start at x index
// fx (first cell or face minus ilo) and span nx_need, rows at fy and span
// ny_need; nk_nom planes around the nominal first plane klo_nom.
bool box_geom(const Lay &Ly, int first_i, int nx_need, int first_j, int ny_need, int klo_nom, BoxGeom *b) {
  const int fx = first_i - Ly.ilo;
  if (fx < 0 || first_j - Ly.jlo < 0 || klo_nom - Ly.klo < 1) return false;  // needs a halo on every side
  b->xo = fx & ~1;
  b->dx = fx & 1;
  b->w = (b->dx + nx_need + 1) & ~1;
  b->yo = first_j - Ly.jlo;
  b->zo = -Ly.klo;
  return b->w <= 256 && ny_need <= 256;
}

bool encode_box(CUtensorMap *m, const double *base, const Lay &Ly, long nk, const BoxGeom &b, int box_h) {
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (Ly.sj & 1) != 0 || (Ly.sk & 1) != 0) return false;
  const EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)Ly.sj, (cuuint64_t)(Ly.sk / Ly.sj), (cuuint64_t)nk};
  cuuint64_t strides[2] = {(cuuint64_t)Ly.sj * 8, (cuuint64_t)Ly.sk * 8};
  cuuint32_t box[3] = {(cuuint32_t)b.w, (cuuint32_t)box_h, 1};
  cuuint32_t es[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double *>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the 2-D map of ux: dims (plane of sk values, planes), boxes of one row of kUxW
bool encode_rows(CUtensorMap *m, const double *base, const Lay &Ly, long nk) {
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0 || (Ly.sk & 1) != 0) return false;
  const EncodeTiledFn fn = encode_tiled();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)Ly.sk, (cuuint64_t)nk};
  cuuint64_t strides[1] = {(cuuint64_t)Ly.sk * 8};
  cuuint32_t box[2] = {(cuuint32_t)kUxW, 1};
  cuuint32_t es[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims, strides, box, es,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// planes per chunk: the chunk count that best fills whole waves of one CTA
// per SM, counting the extra plane each chunk loads, with at least 8 planes a
// chunk (small channels run several at once in an ensemble and need not fill
// the GPU alone)
int pick_chunk(int tiles, int nz, int sms) {
  int best = nz;
  double best_eff = -1.0;
  for (int c = 1; c <= 32 && c <= nz; ++c) {
    const int len = (nz + c - 1) / c, chunks = (nz + len - 1) / len;
    if (len < 8 && len < nz) break;  // a chunk loads one plane more than it corrects
    const long ctas = (long)tiles * chunks, waves = (ctas + sms - 1) / sms;
    const double eff = (double)ctas / (double)(waves * sms) * (double)len / (double)(len + 1);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = len;
    }
  }
  return best;
}

}  // namespace

// tile height and ring depth of the launch
constexpr int kTY = 8, kNS = 3, kCNT = 512;

cudaError_t prepare_correct_tma_kernel() {
  return cudaFuncSetAttribute((const void *)k_correct_tma<kTY, kNS, kCNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              kCorrTmaMaxSmem);
}

bool launch_correct_div_tma(const CorrArgs &ca, const GridK &g, unsigned long long *maxdiv, int sms,
                            cudaStream_t st) {
  CorrTmaGeom q{};
  if (!box_geom(ca.Lpsi, 0, kCTX + 2, 0, kTY + 2, 1, &q.ps) || !box_geom(ca.Lrho, 0, kCTX + 2, 0, kTY + 2, 1, &q.ir) ||
      !box_geom(ca.Luy, 1, kCTX, 0, kTY + 1, 1, &q.uy) || !box_geom(ca.Luz, 1, kCTX, 1, kTY, 0, &q.uz))
    return false;
  q.ux.fx = 0 - ca.Lux.ilo;  // face i0 - 1 of the origin tile
  q.ux.yo = 1 - ca.Lux.jlo;
  q.ux.zo = -ca.Lux.klo;
  q.ux.sj = (int)ca.Lux.sj;
  if (q.ux.fx < 1 || q.ux.yo < 1 || q.ux.zo < 0 || (ca.Lux.sk & 1) != 0) return false;  // a halo on every side
  const CorrTmaSmem L = corr_tma_smem(q, kTY, kNS);
  if (L.total + 128 > kCorrTmaMaxSmem) return false;
  // planes in each array: the nominal range plus the halo on both sides
  const long nk_s = g.nz + 2L * (1 - ca.Lpsi.klo), nk_r = g.nz + 2L * (1 - ca.Lrho.klo);
  const long nk_u = g.nz + 2L * (1 - ca.Lux.klo), nk_v = g.nz + 2L * (1 - ca.Luy.klo);
  const long nk_w = g.nz + 1 + 2L * (0 - ca.Luz.klo);
  CUtensorMap m[7];
  if (!encode_box(&m[0], ca.psi, ca.Lpsi, nk_s, q.ps, kTY + 2) || !encode_box(&m[1], ca.pn, ca.Lpsi, nk_s, q.ps, kTY + 2) ||
      !encode_box(&m[2], ca.pnm1, ca.Lpsi, nk_s, q.ps, kTY + 2) ||
      !encode_box(&m[3], ca.irho, ca.Lrho, nk_r, q.ir, kTY + 2) || !encode_rows(&m[4], ca.uxi, ca.Lux, nk_u) ||
      !encode_box(&m[5], ca.uyi, ca.Luy, nk_v, q.uy, kTY + 1) || !encode_box(&m[6], ca.uzi, ca.Luz, nk_w, q.uz, kTY))
    return false;
  const int nbx = (g.nx + kCTX - 1) / kCTX, nby = (g.ny + kTY - 1) / kTY;
  q.nzc = pick_chunk(nbx * nby, g.nz, sms > 0 ? sms : 148);
  const dim3 grid((unsigned)nbx, (unsigned)nby, (unsigned)((g.nz + q.nzc - 1) / q.nzc));
  k_correct_tma<kTY, kNS, kCNT><<<grid, kCNT, (size_t)L.total + 128, st>>>(m[0], m[1], m[2], m[3], m[4], m[5], m[6], ca, g, q, maxdiv);
  return true;
}

}  // namespace tbfp
