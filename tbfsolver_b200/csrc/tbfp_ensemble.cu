// The ensemble as one persistent launch: every stage of every member's FP64
// projection, run by resident 256-thread blocks that take work items from a
// device queue.
//
// Items are numbered stage-major: all members' 1/rho tiles, then all their
// RHS tiles, and so on up to the correction (qstart holds the prefix sums).
// A block takes the next item with one atomic and, for a stage s > 0, waits
// until its member's stage s-1 has finished every item (a per-(member, stage)
// counter that each finished item raises after a release fence).  Items are
// handed out in order and an item only waits on items handed out before it,
// all held by running blocks, so the queue cannot deadlock.  The wait is
// bounded: after spin_limit polls the block sets the abort word, every block
// stops taking items, and the host reports the timeout.
//
// Each item is one tile of the standalone kernel's grid (the same device
// bodies, tbfp_stages.cuh), or two tiles of a 128-thread kernel, or eight y
// systems (one per warp).  Data produced inside the launch (1/rho, s, the
// spectrum, psi) is read through L2 (COH = true).
#include <cuda_runtime.h>

#include "tbfp_kernels.cuh"
#include "tbfp_stages.cuh"

namespace tbfp {

namespace {

constexpr int kEnsThreads = 256;
constexpr int kRecipChunk = kEnsThreads * 32;  // elements of 1/rho per item
constexpr int kEnsWarps = kEnsThreads / 32;    // y systems (pairs) per item

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// (bx, by, bz) of tile t of a 128-thread stencil grid (x tiles of 128, y chunks of rows, z planes)
__device__ __forceinline__ void stencil_tile(const GridK &g, int rows, int t, int *bx, int *by, int *bz) {
  const int nbx = (g.nx + 127) / 128, nby = (g.ny + rows - 1) / rows;
  *bx = t % nbx;
  *by = (t / nbx) % nby;
  *bz = t / (nbx * nby);
}

// Each stage is its own (not inlined) function, so that each gets its own
// register allocation: one function holding every length spilled.
template <int M>
__device__ __noinline__ void x_stage(const EnsMember *__restrict__ mp, bool inverse, int item, unsigned char *sm) {
  const EnsMember &m = *mp;
  if (inverse)
    fftx_inv_body<double2, M, false, true>(m.spec, m.psi, m.Lpsi, m.hd_psi, m.g, m.twx, m.tpx, m.scale, item, sm);
  else
    fftx_fwd_body<double2, M, 0, true>(m.xs, m.g, m.twx, m.tpx, m.spec, item, sm);
}

template <int NZ>
__device__ __noinline__ void z_stage(const EnsMember *__restrict__ mp, bool inverse, int item, unsigned char *sm) {
  const EnsMember &m = *mp;
  constexpr int TJZ = fftz_cols_per_cta(NZ);
  const int nbx = (m.g.ny + TJZ - 1) / TJZ;
  if (inverse) fftz_body<double2, true, NZ, true>(m.spec, m.g, m.tpz, item % nbx, item / nbx, sm);
  else fftz_body<double2, false, NZ, true>(m.spec, m.g, m.tpz, item % nbx, item / nbx, sm);
}

template <int T>
__device__ __noinline__ void y_stage(const EnsMember *__restrict__ mp, int item, unsigned char *sm) {
  const EnsMember &m = *mp;
  const int warp = threadIdx.x >> 5;
  tridiag_t_body<double2, T>(m.spec, m.g, m.lamx, m.lamz, m.am, m.ap, m.dyf, m.mean_c, m.nxnz,
                             (unsigned)(item * kEnsWarps + warp), warp, sm);
}

__device__ __noinline__ void recip_stage(const EnsMember *__restrict__ mp, int item) {
  const EnsMember &m = *mp;
  if (item == 0 && threadIdx.x == 0) *m.maxdiv = 0ull;  // the correction (stage 7) of this member comes later
  const long t0 = (long)item * kRecipChunk, t1 = min(t0 + kRecipChunk, m.n_rho);
  recip_body(m.rho, m.irho, t0, t1, threadIdx.x, kEnsThreads);
}

__device__ __noinline__ void rhs_stage(const EnsMember *__restrict__ mp, int item) {
  const EnsMember &m = *mp;  // two 128-thread tiles (nz is even)
  int bx, by, bz;
  stencil_tile(m.g, kRJ, item * 2 + (threadIdx.x >> 7), &bx, &by, &bz);
  rhs_body<false, true>(m.ra, m.g, m.s, m.Lpsi, bx, by, bz, threadIdx.x & 127);
}

__device__ __noinline__ void correct_stage(const EnsMember *__restrict__ mp, int item) {
  const EnsMember &m = *mp;
  int bx, by, bz;
  stencil_tile(m.g, kJC, item * 2 + (threadIdx.x >> 7), &bx, &by, &bz);
  correct_div_body<false, true>(m.ca, m.g, m.maxdiv, bx, by, bz, threadIdx.x & 127);
}

__device__ __forceinline__ void run_item(const EnsMember *__restrict__ mp, int stage, int item, unsigned char *sm) {
  switch (stage) {
    case 0:
      recip_stage(mp, item);
      break;
    case 1:
      rhs_stage(mp, item);
      break;
    case 2:
    case 6: {
      const bool inv = stage == 6;
      switch (mp->g.M) {
#define TBFP_X(L) \
  case L: x_stage<L>(mp, inv, item, sm); break;
        TBFP_X(4) TBFP_X(6) TBFP_X(8) TBFP_X(12) TBFP_X(16) TBFP_X(24) TBFP_X(32) TBFP_X(48) TBFP_X(64) TBFP_X(96)
        TBFP_X(128)
#undef TBFP_X
        default: break;
      }
      break;
    }
    case 3:
    case 5: {
      const bool inv = stage == 5;
      switch (mp->g.nz) {
#define TBFP_Z(L) \
  case L: z_stage<L>(mp, inv, item, sm); break;
        TBFP_Z(4) TBFP_Z(6) TBFP_Z(8) TBFP_Z(12) TBFP_Z(16) TBFP_Z(24) TBFP_Z(32) TBFP_Z(48) TBFP_Z(64) TBFP_Z(96)
        TBFP_Z(128)
#undef TBFP_Z
        default: break;
      }
      break;
    }
    case 4: {
      switch (mp->T) {
#define TBFP_T(TT) \
  case TT: y_stage<TT>(mp, item, sm); break;
        TBFP_T(1) TBFP_T(2) TBFP_T(3) TBFP_T(4) TBFP_T(5) TBFP_T(6) TBFP_T(7) TBFP_T(8)
#undef TBFP_T
        default: break;
      }
      break;
    }
    case 7:
      correct_stage(mp, item);
      break;
    default:
      break;
  }
}

__global__ void __launch_bounds__(kEnsThreads, 2) k_ensemble(const EnsMember *__restrict__ mem, int n,
                                                            const int *__restrict__ qstart, EnsCtl *ctl,
                                                            long long spin_limit) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ int s_stage, s_mem, s_item, s_quit;
  const int total = qstart[kEnsStages * n];
  for (;;) {
    if (threadIdx.x == 0) {
      int quit = ld_acquire(&ctl->abort) != 0;
      const int it = quit ? total : atomicAdd(&ctl->next, 1);
      if (it >= total) quit = 1;
      int stage = 0, m = 0, local = 0;
      if (!quit) {
        int lo = 0, hi = kEnsStages * n - 1;  // largest idx with qstart[idx] <= it
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (qstart[mid] <= it) lo = mid;
          else hi = mid - 1;
        }
        stage = lo / n;
        m = lo - stage * n;
        local = it - qstart[lo];
        if (stage > 0) {
          const int prev = (stage - 1) * n + m;
          const int need = qstart[prev + 1] - qstart[prev];
          const int *cnt = &ctl->done[m * kEnsStages + stage - 1];
          long long polls = 0;
          while (ld_acquire(cnt) < need) {
            if (++polls > spin_limit) {
              atomicExch(&ctl->abort, 1);
              quit = 1;
              break;
            }
            if (ld_acquire(&ctl->abort)) {
              quit = 1;
              break;
            }
            __nanosleep(100);
          }
        }
      }
      s_quit = quit;
      s_stage = stage;
      s_mem = m;
      s_item = local;
    }
    __syncthreads();
    if (s_quit) break;
    const int stage = s_stage, m = s_mem, item = s_item;
    run_item(mem + m, stage, item, sm);
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();  // the item's writes before its count
      atomicAdd(&ctl->done[m * kEnsStages + stage], 1);
    }
  }
}

}  // namespace

void ens_items(const GridK &g, long n_rho, int T, int *items) {
  const long nbx = (g.nx + 127) / 128;
  items[0] = (int)((n_rho + kRecipChunk - 1) / kRecipChunk);
  items[1] = (int)(nbx * ((g.ny + kRJ - 1) / kRJ) * g.nz / 2);
  const int TJ = fftx_rows_per_cta(g.M);
  items[2] = items[6] = (int)((g.R + TJ - 1) / TJ);
  const int TJZ = fftz_cols_per_cta(g.nz);
  items[3] = items[5] = (int)(((g.ny + TJZ - 1) / TJZ) * g.nkx);
  const long pairs = (long)g.nkx * (g.nz / 2 + 1);
  items[4] = (int)((pairs + kEnsWarps - 1) / kEnsWarps);
  items[7] = (int)(nbx * ((g.ny + kJC - 1) / kJC) * g.nz / 2);
  (void)T;
}

size_t ens_smem_bytes(int M, int nz, int T) {
  size_t b = fftx_smem_bytes(M, 16);
  const size_t z = fftz_smem_bytes(nz, 16), y = (size_t)kEnsWarps * 2 * 33 * T * sizeof(double2);
  if (z > b) b = z;
  if (y > b) b = y;
  return b;
}

cudaError_t prepare_ensemble_kernel(size_t smem) {
  return cudaFuncSetAttribute((const void *)k_ensemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

int ensemble_blocks_per_sm(size_t smem) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_ensemble, kEnsThreads, smem) != cudaSuccess) return 0;
  return nb;
}

cudaError_t launch_ensemble_persistent(const EnsMember *mem, int n, const int *qstart, EnsCtl *ctl,
                                       long long spin_limit, int blocks, size_t smem, cudaStream_t st) {
  k_ensemble<<<blocks, kEnsThreads, smem, st>>>(mem, n, qstart, ctl, spin_limit);
  return cudaGetLastError();
}

}  // namespace tbfp
