// Batched complex FFTs held in shared memory (Stockham autosort, radix 2/3/4/8),
// specialised at compile time for each supported length.
//
// Replaces the FFTW guru plans of the reference (fastPoissonSolver.f90:160-211):
// all transforms are unnormalised, forward = exp(-2*pi*i*k*n/N), exactly FFTW's
// convention.  One warp transforms NB = 2^LOGNB sequences of length N that sit in
// shared memory with element stride ES and sequence stride BS (in complex
// elements).  Each radix pass reads a lane's butterfly inputs into registers,
// synchronises the warp, and writes the outputs back in place, so no second
// buffer is needed.  N, NB, ES, BS and the radix sequence are template
// constants, so every index is a shift, a mask or a constant offset.
//
// Twiddles come from a pass-ordered table (built on the host in extended
// precision, staged in shared memory by the kernel): pass p with Ns_p > 1 reads
// tw[Ns_p - R_0 + k0*(R_p-1) + r-1] = exp(-2*pi*i*k0*r/(Ns_p*R_p)); the table has
// N - R_0 entries in total (sum over p of Ns_{p+1} - Ns_p).
#pragma once
#include <cuda_runtime.h>

namespace tbfp {

template <typename V> __device__ __forceinline__ V mk(decltype(V::x) a, decltype(V::x) b) {
  V r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename V> __device__ __forceinline__ V cadd(V a, V b) { return mk<V>(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V csub(V a, V b) { return mk<V>(a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V cmul(V a, V b) {
  return mk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename V> __device__ __forceinline__ V cconj(V a) { return mk<V>(a.x, -a.y); }
template <typename V> __device__ __forceinline__ V cscale(V a, decltype(V::x) s) { return mk<V>(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <typename V, bool INV> __device__ __forceinline__ V rot90(V a) {
  return INV ? mk<V>(-a.y, a.x) : mk<V>(a.y, -a.x);
}

// --- compile-time radix plan: radix 8 while possible, then 4, then 2, and at
// most one radix 3 as the last pass (n = 2^a or 3*2^a) -----------------------
__host__ __device__ constexpr int ct_nrad(int n) {
  int k = 0, m = n;
  while (m % 8 == 0 && m > 1) { ++k; m /= 8; }
  while (m % 4 == 0) { ++k; m /= 4; }
  while (m % 2 == 0) { ++k; m /= 2; }
  if (m % 3 == 0) { ++k; m /= 3; }
  return m == 1 ? k : -1;
}
__host__ __device__ constexpr int ct_rad(int n, int p) {
  int k = 0, m = n;
  while (m % 8 == 0 && m > 1) { if (k == p) return 8; ++k; m /= 8; }
  while (m % 4 == 0) { if (k == p) return 4; ++k; m /= 4; }
  while (m % 2 == 0) { if (k == p) return 2; ++k; m /= 2; }
  if (m % 3 == 0 && k == p) return 3;
  return 1;
}
__host__ __device__ constexpr int ct_ns(int n, int p) {
  int s = 1;
  for (int q = 0; q < p; ++q) s *= ct_rad(n, q);
  return s;
}
__host__ __device__ constexpr int ct_log2(int v) {
  int l = 0;
  while ((1 << (l + 1)) <= v) ++l;
  return l;
}
// Entries of the pass-ordered twiddle table of a length-n transform.
__host__ __device__ constexpr int ct_twiddle_len(int n) { return n - ct_rad(n, 0); }

// --- radix butterflies (in registers) --------------------------------------
template <typename V, bool INV> __device__ __forceinline__ void bfly2(V *v) {
  V a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <typename V, bool INV> __device__ __forceinline__ void bfly4(V &x0, V &x1, V &x2, V &x3) {
  V t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = rot90<V, INV>(csub(x1, x3));
  x0 = cadd(t0, t2);
  x2 = csub(t0, t2);
  x1 = cadd(t1, t3);
  x3 = csub(t1, t3);
}

template <typename V, bool INV> __device__ __forceinline__ void bfly3(V *v) {
  using T = decltype(V::x);
  const T c = T(-0.5);
  // sin(2*pi/3) = sqrt(3)/2
  const T s = INV ? T(0.86602540378443864676) : T(-0.86602540378443864676);
  V t = cadd(v[1], v[2]);
  V d = csub(v[1], v[2]);
  V m = mk<V>(v[0].x + c * t.x, v[0].y + c * t.y);
  V id = mk<V>(-s * d.y, s * d.x);  // i*s*d
  v[0] = cadd(v[0], t);
  v[1] = cadd(m, id);
  v[2] = csub(m, id);
}

template <typename V, bool INV> __device__ __forceinline__ void bfly8(V *v) {
  using T = decltype(V::x);
  const T h = T(0.70710678118654752440);  // sqrt(2)/2
  // radix-4 on evens and odds
  V a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
  V b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
  bfly4<V, INV>(a0, a1, a2, a3);
  bfly4<V, INV>(b0, b1, b2, b3);
  // twiddles W8^k (forward W8 = exp(-i*pi/4))
  // W8^1 = h(1 -+ i), W8^2 = -+i, W8^3 = h(-1 -+ i)
  V w1b = INV ? mk<V>(h * (b1.x - b1.y), h * (b1.x + b1.y)) : mk<V>(h * (b1.x + b1.y), h * (b1.y - b1.x));
  V w2b = rot90<V, INV>(b2);
  V w3b = INV ? mk<V>(-h * (b3.x + b3.y), h * (b3.x - b3.y)) : mk<V>(h * (b3.y - b3.x), -h * (b3.x + b3.y));
  v[0] = cadd(a0, b0);
  v[4] = csub(a0, b0);
  v[1] = cadd(a1, w1b);
  v[5] = csub(a1, w1b);
  v[2] = cadd(a2, w2b);
  v[6] = csub(a2, w2b);
  v[3] = cadd(a3, w3b);
  v[7] = csub(a3, w3b);
}

template <typename V, int R, bool INV> __device__ __forceinline__ void bfly(V *v) {
  if constexpr (R == 2) bfly2<V, INV>(v);
  else if constexpr (R == 3) bfly3<V, INV>(v);
  else if constexpr (R == 4) bfly4<V, INV>(v[0], v[1], v[2], v[3]);
  else bfly8<V, INV>(v);
}

// Shared-memory slot of element e of a sequence: one empty slot after every 8
// elements, which makes the stride-R writes of the early Stockham passes (and
// the reads of the late ones) free of bank conflicts for 16-byte elements.
__host__ __device__ __forceinline__ constexpr int pad8(int e) { return e + (e >> 3); }

// Passes P .. PEND-1 of a length-N transform of NB = 2^LOGNB sequences by one warp.
// Butterfly b reads x[b + r*N/R], applies twiddle exp(-+2*pi*i*(b mod Ns)*r/(Ns*R)),
// transforms, and writes y[(b/Ns)*Ns*R + b mod Ns + r*Ns].  Butterflies are
// numbered sequence-fastest (b = jj*NB + sequence).
template <typename V, int N, int LOGNB, int ES, int BS, bool INV, int P = 0, int PEND = ct_nrad(N)>
__device__ __forceinline__ void fft_warp(V *buf, int lane, const V *__restrict__ tw) {
  if constexpr (P < PEND) {
    constexpr int R = ct_rad(N, P), NS = ct_ns(N, P), LNS = ct_log2(NS), PER = N / R;
    constexpr int NB = 1 << LOGNB, TOT = PER * NB, Q = (TOT + 31) / 32;
    constexpr int TWO = NS - ct_rad(N, 0);  // this pass's offset in the twiddle table
    V v[Q][R];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int b = lane + 32 * q;
      if (TOT % 32 == 0 || b < TOT) {
        const int bt = b & (NB - 1), jj = b >> LOGNB;
        const V *base = buf + bt * BS;
        const int k0 = jj & (NS - 1);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          V x = base[pad8(jj + r * PER) * ES];
          if constexpr (NS > 1) {
            if (r > 0) {
              V w = tw[TWO + k0 * (R - 1) + (r - 1)];
              if constexpr (INV) w.y = -w.y;
              x = cmul(x, w);
            }
          }
          v[q][r] = x;
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int b = lane + 32 * q;
      if (TOT % 32 == 0 || b < TOT) {
        const int bt = b & (NB - 1), jj = b >> LOGNB;
        bfly<V, R, INV>(v[q]);
        V *base = buf + bt * BS;
        const int d = (((jj >> LNS) * R) << LNS) + (jj & (NS - 1));
#pragma unroll
        for (int r = 0; r < R; ++r) base[pad8(d + r * NS) * ES] = v[q][r];
      }
    }
    __syncwarp();
    fft_warp<V, N, LOGNB, ES, BS, INV, P + 1, PEND>(buf, lane, tw);
  }
}

}  // namespace tbfp
