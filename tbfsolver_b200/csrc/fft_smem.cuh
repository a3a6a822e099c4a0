// Batched complex FFTs held in shared memory (Stockham autosort, radix 2/3/4/8).
//
// Replaces the FFTW guru plans of the reference (fastPoissonSolver.f90:160-211):
// all transforms are unnormalised, forward = exp(-2*pi*i*k*n/N), exactly FFTW's
// convention.  A CTA transforms `nb` sequences of length n that already sit in
// shared memory with element stride `es` and batch stride `bs` (in complex
// elements).  Each radix pass reads all of a thread's butterfly inputs into
// registers, synchronises, and writes the outputs back in place, so no second
// buffer is needed.  Twiddles come from a table tw[m] = exp(-2*pi*i*m/Ntab)
// computed on the host in double precision; a length-n transform reads it with
// stride twmul = Ntab/n.
#pragma once
#include <cuda_runtime.h>

namespace tbfp {

template <typename T> struct cplx_t;
template <> struct cplx_t<double> { using type = double2; };
template <> struct cplx_t<float> { using type = float2; };

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

// A transform plan: length and radix sequence (product == n).  n = 2^a or
// 3*2^a; powers of two first (radix 8, then 4, then 2), the radix 3 last.
struct FftPlan {
  int n;
  int nrad;
  int rad[16];
};

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
__host__ __device__ __forceinline__ int pad8(int e) { return e + (e >> 3); }

// One Stockham pass of radix R over a group of G threads (a warp, G = 32, or a
// whole block).  Butterfly b of a length-n transform reads x[b + r*n/R],
// applies twiddle exp(-+2*pi*i*(b mod Ns)*r/(Ns*R)), transforms, and writes
// y[(b/Ns)*Ns*R + b mod Ns + r*Ns].  Butterflies are numbered batch-fastest
// (b = jj*nb + batch), nb and Ns are powers of two (the plan puts its single
// radix-3 pass last), so all index arithmetic is shifts and masks.  QMAX
// bounds the butterflies a thread owns (ceil(elements per thread / R)).
template <int G>
__device__ __forceinline__ void group_sync() {
  if constexpr (G == 32) __syncwarp();
  else __syncthreads();
}

template <typename V, int R, int QMAX, bool INV, int G>
__device__ __forceinline__ void stockham_pass(V *buf, int tid, int n, int lognb, int es, int bs, int logNs,
                                              const V *__restrict__ tw, int twmul) {
  const int per = n / R;
  const int total = per << lognb;
  const int nbm = (1 << lognb) - 1, Nsm = (1 << logNs) - 1;
  const int stride_tw = (n / R) >> logNs;  // n/(Ns*R)
  V v[QMAX][R];
#pragma unroll
  for (int q = 0; q < QMAX; ++q) {
    const int b = tid + q * G;
    if (b < total) {
      const int bt = b & nbm, jj = b >> lognb;
      const V *base = buf + bt * bs;
      const int k0 = jj & Nsm;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        V x = base[pad8(jj + r * per) * es];
        if (r > 0) {
          V w = tw[(k0 * r * stride_tw) * twmul];
          if (INV) w.y = -w.y;
          x = cmul(x, w);
        }
        v[q][r] = x;
      }
    }
  }
  group_sync<G>();
#pragma unroll
  for (int q = 0; q < QMAX; ++q) {
    const int b = tid + q * G;
    if (b < total) {
      const int bt = b & nbm, jj = b >> lognb;
      bfly<V, R, INV>(v[q]);
      V *base = buf + bt * bs;
      const int d = (((jj >> logNs) * R) << logNs) + (jj & Nsm);
#pragma unroll
      for (int r = 0; r < R; ++r) base[pad8(d + (r << logNs)) * es] = v[q][r];
    }
  }
  group_sync<G>();
}

// Full transform of nb = 2^lognb sequences by a group of G threads (tid is the
// thread's index in the group).  EMAX = upper bound of n*nb/G.
template <typename V, int EMAX, bool INV, int G>
__device__ void fft_group(V *buf, int tid, const FftPlan &pl, int lognb, int es, int bs, const V *__restrict__ tw,
                          int twmul) {
  int logNs = 0;
  for (int p = 0; p < pl.nrad; ++p) {
    const int R = pl.rad[p];
    switch (R) {
      case 2:
        stockham_pass<V, 2, (EMAX + 1) / 2, INV, G>(buf, tid, pl.n, lognb, es, bs, logNs, tw, twmul);
        logNs += 1;
        break;
      case 3:  // always the last pass
        stockham_pass<V, 3, (EMAX + 2) / 3, INV, G>(buf, tid, pl.n, lognb, es, bs, logNs, tw, twmul);
        break;
      case 4:
        stockham_pass<V, 4, (EMAX + 3) / 4, INV, G>(buf, tid, pl.n, lognb, es, bs, logNs, tw, twmul);
        logNs += 2;
        break;
      default:
        stockham_pass<V, 8, (EMAX + 7) / 8, INV, G>(buf, tid, pl.n, lognb, es, bs, logNs, tw, twmul);
        logNs += 3;
        break;
    }
  }
}

}  // namespace tbfp
