// pf_fft.cuh -- shared-memory Stockham FFT building blocks for sm_100a.
//
// Replaces the FFTW plans of the reference (r2cfieldbackend.hh:210-274,
// r2cmatrixbackend.hh:254-321, dctmatrixbackend.hh:240-309, dftfieldbackend.hh:186-247).
// A multi-dimensional transform is a sequence of "pencil passes": each CTA loads a
// tile of B pencils of one axis from HBM into shared memory with coalesced accesses,
// runs every radix stage of the 1D transform in shared memory (Stockham autosort,
// Govindaraju et al., SC 2008), and writes the tile back, so every pass reads and
// writes the array exactly once.  Load and store functors fuse the work around the
// transform (covariance evaluation, noise scaling, zero padding, pruning of unused
// outputs, eigenvalue multiplication, value transforms).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace pf {

template <typename T>
struct cplx_of;
template <>
struct cplx_of<float> {
  using type = float2;
};
template <>
struct cplx_of<double> {
  using type = double2;
};
template <typename T>
using cx = typename cplx_of<T>::type;

template <typename T>
__device__ __forceinline__ cx<T> mk(T a, T b) {
  cx<T> r;
  r.x = a;
  r.y = b;
  return r;
}
template <typename T>
__device__ __forceinline__ cx<T> cadd(cx<T> a, cx<T> b) {
  return mk<T>(a.x + b.x, a.y + b.y);
}
template <typename T>
__device__ __forceinline__ cx<T> csub(cx<T> a, cx<T> b) {
  return mk<T>(a.x - b.x, a.y - b.y);
}
template <typename T>
__device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
__device__ __forceinline__ cx<T> cscale(cx<T> a, T s) {
  return mk<T>(a.x * s, a.y * s);
}
// a * (sign * i)
template <typename T>
__device__ __forceinline__ cx<T> mul_si(cx<T> a, int sign) {
  return sign < 0 ? mk<T>(a.y, -a.x) : mk<T>(-a.y, a.x);
}
template <typename T>
__device__ __forceinline__ cx<T> conjg(cx<T> a) {
  return mk<T>(a.x, -a.y);
}

// twiddle exp(sign * 2 pi i m / L) from a table holding exp(-2 pi i m / L)
template <typename T>
__device__ __forceinline__ cx<T> twiddle(const cx<T>* __restrict__ tw, int m, int sign) {
  cx<T> w = __ldg(tw + m);
  if (sign > 0) w.y = -w.y;
  return w;
}

// ---------------------------------------------------------------------------
// in-register DFTs: out[q] = sum_r v[r] exp(sign 2 pi i r q / R)
// ---------------------------------------------------------------------------
template <typename T, int R>
struct Dft;

template <typename T>
struct Dft<T, 2> {
  static __device__ __forceinline__ void run(cx<T>* v, int, const cx<T>*, int) {
    cx<T> a = v[0], b = v[1];
    v[0] = cadd<T>(a, b);
    v[1] = csub<T>(a, b);
  }
};

template <typename T>
struct Dft<T, 4> {
  static __device__ __forceinline__ void run(cx<T>* v, int sign, const cx<T>*, int) {
    cx<T> a = cadd<T>(v[0], v[2]), b = csub<T>(v[0], v[2]);
    cx<T> c = cadd<T>(v[1], v[3]), d = mul_si<T>(csub<T>(v[1], v[3]), sign);
    v[0] = cadd<T>(a, c);
    v[2] = csub<T>(a, c);
    v[1] = cadd<T>(b, d);
    v[3] = csub<T>(b, d);
  }
};

template <typename T>
struct Dft<T, 8> {
  static __device__ __forceinline__ void run(cx<T>* v, int sign, const cx<T>*, int) {
    const T h = (T)0.70710678118654752440084436210484903928;
    cx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cx<T> o[4] = {v[1], v[3], v[5], v[7]};
    Dft<T, 4>::run(e, sign, nullptr, 0);
    Dft<T, 4>::run(o, sign, nullptr, 0);
    // o[q] *= W8^q, W8 = exp(sign 2 pi i / 8)
    cx<T> o1 = o[1], o3 = o[3];
    o[1] = mk<T>(h * (o1.x - sign * o1.y), h * (o1.y + sign * o1.x));
    o[2] = mul_si<T>(o[2], sign);
    o[3] = mk<T>(h * (-o3.x - sign * o3.y), h * (-o3.y + sign * o3.x));
#pragma unroll
    for (int q = 0; q < 4; q++) {
      v[q] = cadd<T>(e[q], o[q]);
      v[q + 4] = csub<T>(e[q], o[q]);
    }
  }
};

template <typename T>
struct Dft<T, 3> {
  static __device__ __forceinline__ void run(cx<T>* v, int sign, const cx<T>*, int) {
    const T s3 = (T)0.86602540378443864676372317075293618347;
    cx<T> a = v[0], s = cadd<T>(v[1], v[2]), d = csub<T>(v[1], v[2]);
    cx<T> m = mk<T>(a.x - (T)0.5 * s.x, a.y - (T)0.5 * s.y);
    cx<T> t = mul_si<T>(cscale<T>(d, s3), sign);
    v[0] = cadd<T>(a, s);
    v[1] = cadd<T>(m, t);
    v[2] = csub<T>(m, t);
  }
};

template <typename T>
struct Dft<T, 5> {
  static __device__ __forceinline__ void run(cx<T>* v, int sign, const cx<T>*, int) {
    const T c1 = (T)0.30901699437494742410229341718281905886;   // cos(2pi/5)
    const T c2 = (T)-0.80901699437494742410229341718281905886;  // cos(4pi/5)
    const T s1 = (T)0.95105651629515357211643933337938214340;   // sin(2pi/5)
    const T s2 = (T)0.58778525229247312916870595463907276860;   // sin(4pi/5)
    cx<T> a0 = v[0];
    cx<T> p1 = cadd<T>(v[1], v[4]), m1 = csub<T>(v[1], v[4]);
    cx<T> p2 = cadd<T>(v[2], v[3]), m2 = csub<T>(v[2], v[3]);
    cx<T> r1 = mk<T>(a0.x + c1 * p1.x + c2 * p2.x, a0.y + c1 * p1.y + c2 * p2.y);
    cx<T> r2 = mk<T>(a0.x + c2 * p1.x + c1 * p2.x, a0.y + c2 * p1.y + c1 * p2.y);
    cx<T> i1 = mul_si<T>(mk<T>(s1 * m1.x + s2 * m2.x, s1 * m1.y + s2 * m2.y), sign);
    cx<T> i2 = mul_si<T>(mk<T>(s2 * m1.x - s1 * m2.x, s2 * m1.y - s1 * m2.y), sign);
    v[0] = cadd<T>(a0, cadd<T>(p1, p2));
    v[1] = cadd<T>(r1, i1);
    v[4] = csub<T>(r1, i1);
    v[2] = cadd<T>(r2, i2);
    v[3] = csub<T>(r2, i2);
  }
};

// generic small odd prime R: O(R^2) with the pencil's twiddle table (L divisible by R)
template <typename T, int R>
struct Dft {
  static __device__ __forceinline__ void run(cx<T>* v, int sign, const cx<T>* tw, int L) {
    cx<T> out[R];
    const int step = L / R;
#pragma unroll
    for (int q = 0; q < R; q++) {
      cx<T> s = v[0];
#pragma unroll
      for (int r = 1; r < R; r++) s = cadd<T>(s, cmul<T>(v[r], twiddle<T>(tw, ((r * q) % R) * step, sign)));
      out[q] = s;
    }
#pragma unroll
    for (int q = 0; q < R; q++) v[q] = out[q];
  }
};

// ---------------------------------------------------------------------------
// one Stockham stage over a tile of B pencils in shared memory.
// element (b, j) of the tile lives at b*sb + j*sj.
// ---------------------------------------------------------------------------
struct TileShape {
  int L;       // transform length
  int B;       // pencils in the tile
  int sb, sj;  // shared-memory strides
  int bfast;   // thread order: b fastest (strided passes) or butterfly fastest
};

template <typename T, int R>
__device__ __forceinline__ void stage_r(const cx<T>* __restrict__ src, cx<T>* __restrict__ dst,
                                        const TileShape& ts, int Ns, const cx<T>* __restrict__ tw,
                                        int sign) {
  const int nbf = ts.L / R;
  const int total = nbf * ts.B;
  const int twstride = ts.L / (Ns * R);
  for (int u = threadIdx.x; u < total; u += blockDim.x) {
    int b, t;
    if (ts.bfast) {
      b = u % ts.B;
      t = u / ts.B;
    } else {
      t = u % nbf;
      b = u / nbf;
    }
    const int k = t % Ns;
    cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      cx<T> a = src[b * ts.sb + (t + r * nbf) * ts.sj];
      if (r > 0 && k > 0) a = cmul<T>(a, twiddle<T>(tw, r * k * twstride, sign));
      v[r] = a;
    }
    Dft<T, R>::run(v, sign, tw, ts.L);
    const int base = (t / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) dst[b * ts.sb + (base + r * Ns) * ts.sj] = v[r];
  }
}

// radix schedule of one transform length (host-computed)
struct Radices {
  int n;
  int r[20];
};

// Runs all stages; input in buf[0], returns the buffer holding the result.
template <typename T>
__device__ cx<T>* fft_tile(cx<T>* b0, cx<T>* b1, const TileShape& ts, const Radices& rad,
                           const cx<T>* __restrict__ tw, int sign) {
  cx<T>* src = b0;
  cx<T>* dst = b1;
  int Ns = 1;
  for (int s = 0; s < rad.n; s++) {
    const int R = rad.r[s];
    switch (R) {
      case 2: stage_r<T, 2>(src, dst, ts, Ns, tw, sign); break;
      case 3: stage_r<T, 3>(src, dst, ts, Ns, tw, sign); break;
      case 4: stage_r<T, 4>(src, dst, ts, Ns, tw, sign); break;
      case 5: stage_r<T, 5>(src, dst, ts, Ns, tw, sign); break;
      case 7: stage_r<T, 7>(src, dst, ts, Ns, tw, sign); break;
      case 8: stage_r<T, 8>(src, dst, ts, Ns, tw, sign); break;
      case 11: stage_r<T, 11>(src, dst, ts, Ns, tw, sign); break;
      case 13: stage_r<T, 13>(src, dst, ts, Ns, tw, sign); break;
      default: break;
    }
    __syncthreads();
    cx<T>* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  return src;
}

// ---------------------------------------------------------------------------
// Bluestein (chirp-z) transform for lengths with a prime factor above 13
// (L. Bluestein, "A linear filtering approach to the computation of the discrete Fourier
// transform", 1970): with w_j = exp(s pi i (j^2 mod 2L) / L),
//   X_k = w_k sum_j (x_j w_j) conj(w_{k-j}),
// a circular convolution of length M >= 2L-1 (power of two) done in shared memory as an
// in-place decimation-in-frequency FFT (natural -> bit-reversed order), a pointwise
// product with the precomputed FFT of conj(w) (bit-reversed order, 1/M folded in), and an
// in-place decimation-in-time inverse FFT (bit-reversed -> natural order).
// Tables (sign -1; sign +1 uses their conjugates since conj(w) is symmetric):
//   chirp[j] = exp(-pi i (j^2 mod 2L)/L), j < L;   bhat[m] = FFT_M(conj chirp)[rev(m)] / M;
//   twM[m] = exp(-2 pi i m / M), m < M/2.
// ---------------------------------------------------------------------------
struct Blue {
  int M;              // 0: the length is 13-smooth (Stockham stages instead)
  const void* chirp;  // cx<T>[L]
  const void* bhat;   // cx<T>[M]
  const void* twM;    // cx<T>[M/2]
};

template <typename T>
__device__ __forceinline__ cx<T> cj_if(cx<T> v, bool c) {
  if (c) v.y = -v.y;
  return v;
}

// in place on the B = 2^lgB pencils of x, element j of pencil b at x[j*B + b] (j < L);
// work holds M*B elements of shared memory in the same interleaved layout.  M, the
// butterfly spans and the pencil count are powers of two, so every index is a shift/mask.
template <typename T>
__device__ void bluestein(cx<T>* x, cx<T>* work, int L, const Blue& bl, int sign, int lgB = 0) {
  const int M = bl.M;
  const int B = 1 << lgB, bm = B - 1;
  const int lgM = __ffs(M) - 1;
  const cx<T>* chirp = (const cx<T>*)bl.chirp;
  const cx<T>* bhat = (const cx<T>*)bl.bhat;
  const cx<T>* twM = (const cx<T>*)bl.twM;
  const bool c = sign > 0;
  for (int u = threadIdx.x; u < (M << lgB); u += blockDim.x) {
    const int j = u >> lgB;
    work[u] = j < L ? cmul<T>(x[u], cj_if<T>(__ldg(chirp + j), c)) : mk<T>(0, 0);
  }
  __syncthreads();
  // forward DIF, natural -> bit-reversed; two radix-2 stages (half H, H/2) per pass over
  // shared memory, a last single stage when log2 M is odd
  int half = M >> 1, lgh = lgM - 1;
  for (; half >= 2; half >>= 2, lgh -= 2) {
    const int q = half >> 1, lgq = lgh - 1;
    const int lts = lgM - 1 - lgh;  // log2(M / (2 half))
    for (int u = threadIdx.x; u < ((M >> 2) << lgB); u += blockDim.x) {
      const int b = u & bm, v = u >> lgB;
      const int g = v >> lgq, pos = v & (q - 1);
      const int i0 = g * 2 * half + pos;
      cx<T>* w0 = work + ((size_t)i0 << lgB) + b;
      const size_t sq = (size_t)q << lgB, sh = (size_t)half << lgB;
      cx<T> a0 = w0[0], a1 = w0[sq], a2 = w0[sh], a3 = w0[sh + sq];
      const cx<T> wA0 = __ldg(twM + (pos << lts)), wA1 = __ldg(twM + ((pos + q) << lts)),
                  wB = __ldg(twM + (pos << (lts + 1)));
      cx<T> s0 = cadd<T>(a0, a2), d0 = cmul<T>(csub<T>(a0, a2), wA0);
      cx<T> s1 = cadd<T>(a1, a3), d1 = cmul<T>(csub<T>(a1, a3), wA1);
      w0[0] = cadd<T>(s0, s1);
      w0[sq] = cmul<T>(csub<T>(s0, s1), wB);
      w0[sh] = cadd<T>(d0, d1);
      w0[sh + sq] = cmul<T>(csub<T>(d0, d1), wB);
    }
    __syncthreads();
  }
  if (half == 1) {
    for (int u = threadIdx.x; u < ((M >> 1) << lgB); u += blockDim.x) {
      const int b = u & bm, v = u >> lgB;
      cx<T>* w0 = work + ((size_t)(2 * v) << lgB) + b;
      const cx<T> a = w0[0], bb = w0[B];
      w0[0] = cadd<T>(a, bb);
      w0[B] = csub<T>(a, bb);
    }
    __syncthreads();
  }
  for (int u = threadIdx.x; u < (M << lgB); u += blockDim.x)
    work[u] = cmul<T>(work[u], cj_if<T>(__ldg(bhat + (u >> lgB)), c));
  __syncthreads();
  // inverse DIT, bit-reversed -> natural; radix-2 stage first when log2 M is odd, then
  // pairs of stages (half h, 2h)
  int h = 1, lgh2 = 0;
  if (lgM & 1) {
    for (int u = threadIdx.x; u < ((M >> 1) << lgB); u += blockDim.x) {
      const int b = u & bm, v = u >> lgB;
      cx<T>* w0 = work + ((size_t)(2 * v) << lgB) + b;
      const cx<T> a = w0[0], bb = w0[B];
      w0[0] = cadd<T>(a, bb);
      w0[B] = csub<T>(a, bb);
    }
    __syncthreads();
    h = 2;
    lgh2 = 1;
  }
  for (; h < M; h <<= 2, lgh2 += 2) {
    const int ltA = lgM - 1 - lgh2, ltB = lgM - 2 - lgh2;  // log2(M / 2h), log2(M / 4h)
    for (int u = threadIdx.x; u < ((M >> 2) << lgB); u += blockDim.x) {
      const int b = u & bm, v = u >> lgB;
      const int g = v >> lgh2, pos = v & (h - 1);
      const int i0 = g * 4 * h + pos;
      cx<T>* w0 = work + ((size_t)i0 << lgB) + b;
      const size_t s1h = (size_t)h << lgB;
      const cx<T> wA = conjg<T>(__ldg(twM + (pos << ltA)));
      const cx<T> wB0 = conjg<T>(__ldg(twM + (pos << ltB))), wB1 = conjg<T>(__ldg(twM + ((pos + h) << ltB)));
      const cx<T> a0 = w0[0], a1 = cmul<T>(w0[s1h], wA);
      const cx<T> a2 = w0[2 * s1h], a3 = cmul<T>(w0[3 * s1h], wA);
      const cx<T> s0 = cadd<T>(a0, a1), d0 = csub<T>(a0, a1);
      const cx<T> s1 = cadd<T>(a2, a3), d1 = csub<T>(a2, a3);
      const cx<T> t0 = cmul<T>(s1, wB0), t1 = cmul<T>(d1, wB1);
      w0[0] = cadd<T>(s0, t0);
      w0[2 * s1h] = csub<T>(s0, t0);
      w0[s1h] = cadd<T>(d0, t1);
      w0[3 * s1h] = csub<T>(d0, t1);
    }
    __syncthreads();
  }
  for (int u = threadIdx.x; u < (L << lgB); u += blockDim.x)
    x[u] = cmul<T>(work[u], cj_if<T>(__ldg(chirp + (u >> lgB)), c));
  __syncthreads();
}

}  // namespace pf
