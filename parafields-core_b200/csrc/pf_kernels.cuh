// pf_kernels.cuh -- pass kernels and the functors fused into their load/store stages.
#pragma once

#include <math.h>

#include "pf_fft.cuh"

namespace pf {

#ifndef PF_THREADS
#define PF_THREADS 256
#endif
constexpr int kThreads = PF_THREADS;

// Set by any functor whose computed index falls outside its buffer; the access is
// skipped instead of performed, and the host turns the flag into an error.
__device__ unsigned int g_bounds_error;

__device__ __forceinline__ bool in_bounds(long long i, long long n) {
  if (i >= 0 && i < n) return true;
  atomicOr(&g_bounds_error, 1u);
  return false;
}
// 32-bit element indices (every buffer of a plan holds fewer than 2^32 elements)
__device__ __forceinline__ bool in_bounds32(unsigned i, unsigned n) {
  if (i < n) return true;
  atomicOr(&g_bounds_error, 1u);
  return false;
}

// ---------------------------------------------------------------------------
// pass descriptor
// ---------------------------------------------------------------------------
struct PassArgs {
  int L;               // complex transform length
  int Lout;            // outputs stored per pencil (pruning)
  int B;               // pencils per tile
  int pitch;           // shared-memory pitch of one pencil (contiguous passes)
  long long npencil;   // contiguous: rows; strided: inner extent
  long long nouter;    // strided: outer extent
  int sign, sign2;     // first / second (fused) transform direction
  Radices rad;         // radix schedule of L
  Blue blue;           // Bluestein tables when L has a prime factor above 13 (then B = 1)
};

// the 1D transforms of a tile: Stockham stages, or Bluestein (one pencil per tile, unit
// stride, scratch of blue.M elements after the tile buffers); returns the result buffer
template <typename T>
__device__ __forceinline__ cx<T>* fft_any(cx<T>* b0, cx<T>* b1, cx<T>* work, const TileShape& ts, const PassArgs& a,
                                          const cx<T>* __restrict__ tw, int sign) {
  if (a.blue.M) {  // strided tiles hold B = 2^k interleaved pencils, row tiles one
    bluestein<T>(b0, work, a.L, a.blue, sign, ts.bfast ? __ffs(ts.B) - 1 : 0);
    return b0;
  }
  return fft_tile<T>(b0, b1, ts, a.rad, tw, sign);
}

struct NoMid {
  static constexpr bool active = false;
  template <typename T>
  __device__ cx<T> operator()(long long, int, long long, cx<T> v) const {
    return v;
  }
};

// loaders that produce elements j and j + L/2 of a pencil from one generator call
struct R2CNoise;
template <class Ld>
struct has_pair_load : std::false_type {};
template <>
struct has_pair_load<R2CNoise> : std::true_type {};

// Generic complex pencil pass.  CONTIG: pencils are rows (element j of row p at
// stride 1); otherwise pencil p of outer block o has element j at p + j*jstride +
// o*ostride, and one tile holds B consecutive p so every row segment is coalesced.
// Registers are capped for two resident CTAs per SM (the Bluestein tiles allow two).
template <typename T, bool CONTIG, class Ld, class Mid, class St>
__global__ void __launch_bounds__(kThreads, 2) k_pass(const PassArgs a, const cx<T>* __restrict__ tw,
                                                      Ld ld, Mid mid, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  TileShape ts;
  ts.L = a.L;
  ts.B = a.B;
  if (CONTIG) {
    ts.sb = a.pitch;
    ts.sj = 1;
    ts.bfast = 0;
  } else {
    ts.sb = 1;
    ts.sj = a.B;
    ts.bfast = 1;
  }
  cx<T>* b1 = b0 + (CONTIG ? a.B * a.pitch : a.B * a.L);
  long long p0, io;
  if (CONTIG) {
    p0 = (long long)blockIdx.x * a.B;
    io = 0;
  } else {
    const long long tpo = (a.npencil + a.B - 1) / a.B;
    io = blockIdx.x / tpo;
    p0 = (blockIdx.x - io * tpo) * a.B;
  }
  const int tot = a.B * a.L;
  bool loaded = false;
  if constexpr (has_pair_load<Ld>::value) {
    if (a.L % 2 == 0) {  // one generator call for elements j and j + L/2
      const int h = a.L / 2;
      for (int u = threadIdx.x; u < a.B * h; u += blockDim.x) {
        int b, j;
        if (CONTIG) {
          b = u / h;
          j = u - b * h;
        } else {
          b = u % a.B;
          j = u / a.B;
        }
        const long long p = p0 + b;
        cx<T> v0 = mk<T>(0, 0), v1 = mk<T>(0, 0);
        if (p < a.npencil) ld.template load2<T>((int)p, j, (int)io, v0, v1);
        b0[b * ts.sb + j * ts.sj] = v0;
        b0[b * ts.sb + (j + h) * ts.sj] = v1;
      }
      loaded = true;
    }
  }
  if (!loaded)
    for (int u = threadIdx.x; u < tot; u += blockDim.x) {
      int b, j;
      if (CONTIG) {
        b = u / a.L;
        j = u - b * a.L;
      } else {
        b = u % a.B;
        j = u / a.B;
      }
      const long long p = p0 + b;
      b0[b * ts.sb + j * ts.sj] = (p < a.npencil) ? ld.template load<T>(p, j, io) : mk<T>(0, 0);
    }
  __syncthreads();
  cx<T>* wk = b1;  // Bluestein scratch (b1 is not used as a Stockham buffer then)
  cx<T>* r = fft_any<T>(b0, b1, wk, ts, a, tw, a.sign);
  if (Mid::active) {
    for (int u = threadIdx.x; u < tot; u += blockDim.x) {
      int b, j;
      if (CONTIG) {
        b = u / a.L;
        j = u - b * a.L;
      } else {
        b = u % a.B;
        j = u / a.B;
      }
      const long long p = p0 + b;
      if (p < a.npencil) r[b * ts.sb + j * ts.sj] = mid.template operator()<T>(p, j, io, r[b * ts.sb + j * ts.sj]);
    }
    __syncthreads();
    r = fft_any<T>(r, r == b0 ? b1 : b0, wk, ts, a, tw, a.sign2);
  }
  const int tout = a.B * a.Lout;
  for (int u = threadIdx.x; u < tout; u += blockDim.x) {
    int b, j;
    if (CONTIG) {
      b = u / a.Lout;
      j = u - b * a.Lout;
    } else {
      b = u % a.B;
      j = u / a.B;
    }
    const long long p = p0 + b;
    if (p < a.npencil) st.template store<T>(p, j, io, r[b * ts.sb + j * ts.sj]);
  }
}

// Real-to-complex pass along dimension 0 (rows of 2L reals -> L+1 complex), via the
// half-length complex FFT of z_m = x_{2m} + i x_{2m+1} and the standard split
// X_k = (Z_k + conj Z_{L-k})/2 - i/2 e^{-2 pi i k/2L} (Z_k - conj Z_{L-k}).
// twT holds exp(-2 pi i m / 2L).
template <typename T, class Ld, class St>
__global__ void __launch_bounds__(kThreads, 2) k_r2c(const PassArgs a, const cx<T>* __restrict__ tw,
                                                     const cx<T>* __restrict__ twT, Ld ld, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* b1 = b0 + a.B * a.pitch;
  TileShape ts{a.L, a.B, a.pitch, 1, 0};
  const long long p0 = (long long)blockIdx.x * a.B;
  const int tot = a.B * a.L;
  for (int u = threadIdx.x; u < tot; u += blockDim.x) {
    const int b = u / a.L, m = u - b * a.L;
    const long long p = p0 + b;
    cx<T> z = mk<T>(0, 0);
    if (p < a.npencil) z = mk<T>(ld.template real<T>(p, 2 * m), ld.template real<T>(p, 2 * m + 1));
    b0[b * a.pitch + m] = z;
  }
  __syncthreads();
  cx<T>* Z = fft_any<T>(b0, b1, b1 + a.B * a.pitch, ts, a, tw, -1);
  cx<T>* X = (Z == b0) ? b1 : b0;
  const int L = a.L;
  for (int u = threadIdx.x; u < a.B * (L + 1); u += blockDim.x) {
    const int b = u / (L + 1), k = u - b * (L + 1);
    const cx<T> zk = Z[b * a.pitch + (k == L ? 0 : k)];
    const cx<T> zm = conjg<T>(Z[b * a.pitch + (k == 0 ? 0 : L - k)]);
    const cx<T> e = cscale<T>(cadd<T>(zk, zm), (T)0.5);
    const cx<T> o = cscale<T>(csub<T>(zk, zm), (T)0.5);  // (Zk - conj Z_{L-k})/2
    // o / i = -i o ; times w = exp(-2 pi i k / 2L)
    const cx<T> oi = mk<T>(o.y, -o.x);
    const cx<T> w = (k == L) ? mk<T>(-1, 0) : __ldg(twT + k);
    X[b * a.pitch + k] = cadd<T>(e, cmul<T>(oi, w));
  }
  __syncthreads();
  for (int u = threadIdx.x; u < a.B * a.Lout; u += blockDim.x) {
    const int b = u / a.Lout, k = u - b * a.Lout;
    const long long p = p0 + b;
    if (p < a.npencil) st.template store<T>(p, k, 0, X[b * a.pitch + k]);
  }
}

// Complex-to-real pass along dimension 0 with FFTW c2r semantics (imaginary parts of
// the DC and Nyquist entries ignored): Z_k = (X_k + conj X_{L-k}) + i e^{+2 pi i k/2L}
// (X_k - conj X_{L-k}), z = IDFT_L(Z), out_{2m} = Re z_m, out_{2m+1} = Im z_m.
template <typename T, class Ld, class St>
__global__ void __launch_bounds__(kThreads, 2) k_c2r(const PassArgs a, const cx<T>* __restrict__ tw,
                                                     const cx<T>* __restrict__ twT, Ld ld, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* b1 = b0 + a.B * a.pitch;
  TileShape ts{a.L, a.B, a.pitch, 1, 0};
  const long long p0 = (long long)blockIdx.x * a.B;
  const int L = a.L;
  for (int u = threadIdx.x; u < a.B * (L + 1); u += blockDim.x) {
    const int b = u / (L + 1), k = u - b * (L + 1);
    const long long p = p0 + b;
    cx<T> v = (p < a.npencil) ? ld.template load<T>(p, k, 0) : mk<T>(0, 0);
    if (k == 0 || k == L) v.y = 0;
    b1[b * a.pitch + k] = v;
  }
  __syncthreads();
  for (int u = threadIdx.x; u < a.B * L; u += blockDim.x) {
    const int b = u / L, k = u - b * L;
    const cx<T> xk = b1[b * a.pitch + k];
    const cx<T> xm = conjg<T>(b1[b * a.pitch + L - k]);
    const cx<T> s = cadd<T>(xk, xm);
    const cx<T> d = csub<T>(xk, xm);
    const cx<T> w = conjg<T>(__ldg(twT + k));  // exp(+2 pi i k / 2L)
    const cx<T> t = cmul<T>(d, w);
    b0[b * a.pitch + k] = mk<T>(s.x - t.y, s.y + t.x);  // s + i t
  }
  __syncthreads();
  cx<T>* z = fft_any<T>(b0, b1, b1 + a.B * a.pitch, ts, a, tw, +1);
  for (int u = threadIdx.x; u < a.B * a.Lout; u += blockDim.x) {
    const int b = u / a.Lout, j = u - b * a.Lout;
    const long long p = p0 + b;
    if (p < a.npencil) {
      const cx<T> v = z[b * a.pitch + (j >> 1)];
      st.template real<T>(p, j, (j & 1) ? v.y : v.x);
    }
  }
}

// ---------------------------------------------------------------------------
// array load/store functors (element p + j*jstride + o*ostride, complex)
// ---------------------------------------------------------------------------
template <typename S>
struct ArrLoad {
  const S* ptr;  // S = float2 or double2
  unsigned jstride, ostride, rowstride;
  unsigned n;  // elements in the buffer
  int Lin;     // j >= Lin reads zero (input pruning / zero padding)
  template <typename T>
  __device__ __forceinline__ cx<T> load(long long p, int j, long long o) const {
    if (j >= Lin) return mk<T>(0, 0);
    const unsigned i = (unsigned)p * rowstride + (unsigned)j * jstride + (unsigned)o * ostride;
    if (!in_bounds32(i, n)) return mk<T>(0, 0);
    const S v = ptr[i];
    return mk<T>((T)v.x, (T)v.y);
  }
};

// ArrLoad over an array that holds only the indices j <= T/2 of an even sequence of
// period T along the pencil axis: element j reads index min(j, T - j)
template <typename S>
struct MirrorLoad {
  const S* ptr;
  unsigned jstride, ostride, rowstride;
  unsigned n;
  int T;
  template <typename T_>
  __device__ __forceinline__ cx<T_> load(long long p, int j, long long o) const {
    const int m = j <= T - j ? j : T - j;
    const unsigned i = (unsigned)p * rowstride + (unsigned)m * jstride + (unsigned)o * ostride;
    if (!in_bounds32(i, n)) return mk<T_>(0, 0);
    const S v = ptr[i];
    return mk<T_>((T_)v.x, (T_)v.y);
  }
};

template <typename S>
struct ArrStore {
  S* ptr;
  unsigned jstride, ostride, rowstride;
  unsigned n;
  template <typename T>
  __device__ __forceinline__ void store(long long p, int j, long long o, cx<T> v) const {
    const unsigned i = (unsigned)p * rowstride + (unsigned)j * jstride + (unsigned)o * ostride;
    if (!in_bounds32(i, n)) return;
    S w;
    w.x = v.x;
    w.y = v.y;
    ptr[i] = w;
  }
};

// ---------------------------------------------------------------------------
// value transforms (mutators.hh:35-118)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T apply_mutator(int kind, T lam, T v) {
  switch (kind) {
    case 1: return exp(v);
    case 2: return fabs(v);
    case 3: return v < (T)0 ? (T)-1 : (T)1;
    case 4: return pow(v * lam + (T)1, -lam);
    default: return v;
  }
}

// real row load of a field embedded in the torus (fieldToExtendedField,
// r2cfieldbackend.hh:352-368): row p holds x[p*n0 + j] for j < n0, zero beyond
template <typename S>
struct FieldRowLoad {
  const S* x;
  int n0;
  unsigned n;
  template <typename T>
  __device__ __forceinline__ T real(long long p, int j) const {
    if (j >= n0) return (T)0;
    const unsigned i = (unsigned)p * (unsigned)n0 + (unsigned)j;
    return in_bounds32(i, n) ? (T)x[i] : (T)0;
  }
};

// real row store of the original-domain corner (extendedFieldToField,
// r2cfieldbackend.hh:433-441) with an optional value transform
template <typename S>
struct FieldRowStore {
  S* out;
  int n0;
  int transform;
  double boxcox;
  unsigned n;
  template <typename T>
  __device__ __forceinline__ void real(long long p, int j, T v) const {
    if (transform) v = apply_mutator<T>(transform, (T)boxcox, v);
    const unsigned i = (unsigned)p * (unsigned)n0 + (unsigned)j;
    if (in_bounds32(i, n)) out[i] = (S)v;
  }
};

// complex row store splitting Re / Im into two fields (DFT backend, component 0/1,
// dftfieldbackend.hh:380-393)
template <typename S>
struct SplitStore {
  S* re;
  S* im;  // may be null
  long long rowlen;
  int transform;
  double boxcox;
  unsigned n;
  template <typename T>
  __device__ __forceinline__ void store(long long p, int j, long long, cx<T> v) const {
    T a = v.x, b = v.y;
    if (transform) {
      a = apply_mutator<T>(transform, (T)boxcox, a);
      b = apply_mutator<T>(transform, (T)boxcox, b);
    }
    const unsigned i = (unsigned)p * (unsigned)rowlen + (unsigned)j;
    if (!in_bounds32(i, n)) return;
    re[i] = (S)a;
    if (im) im[i] = (S)b;
  }
};

// Re of a complex row into a real field, replacing (first symmetry type) or adding to the
// field (later types): DCTDSTFieldBackend::extendedFieldToField with `additive`
// (dctdstfieldbackend.hh:631-771)
template <typename S>
struct AccStore {
  S* out;
  int n0;
  int accumulate;
  unsigned n;
  template <typename T>
  __device__ __forceinline__ void store(long long p, int j, long long, cx<T> v) const {
    const unsigned i = (unsigned)p * (unsigned)n0 + (unsigned)j;
    if (!in_bounds32(i, n)) return;
    out[i] = accumulate ? (S)(out[i] + (S)v.x) : (S)v.x;
  }
};

// complex row load of a real field (DFT backend embedding, dftfieldbackend.hh:307-325)
template <typename S>
struct FieldComplexLoad {
  const S* x;
  int n0;
  unsigned n;
  template <typename T>
  __device__ __forceinline__ cx<T> load(long long p, int j, long long) const {
    if (j >= n0) return mk<T>(0, 0);
    const unsigned i = (unsigned)p * (unsigned)n0 + (unsigned)j;
    return mk<T>(in_bounds32(i, n) ? (T)x[i] : (T)0, (T)0);
  }
};

// ---------------------------------------------------------------------------
// covariance evaluation on the torus (matrix.hh:615-638, covariance.hh)
// ---------------------------------------------------------------------------
struct CovParams {
  int dim;
  int cov;
  int aniso;
  int T[3];
  int rowcells[3];  // cells of the row decomposition (dim 0 is the pencil)
  double h[3];
  double half[3];   // 0.5 * ext * factor
  double wrap[3];   // ext * factor
  double geo[9];    // transformation applied to coordinates
  double variance;
  double p0, p1;    // gamma / alpha / beta; matern: sqrt(2 nu), 2^(1-nu)
  double p2, p3;    // matern: Gamma(nu), nu
  // merge periodization (matrix.hh:652-775)
  int per;          // 0 classical mirroring, 1 merge
  int sig;          // 0 smoothstep, 1 smooth
  int radial;       // radial or radialPlus combination of the sigmoids
  int plus;         // radialPlus: remainder filled with the covariance at half the torus
  int rec;          // sigmoid recursions
  double sstart, send, factor;
  double ext[3];
  // fold periodization (matrix.hh:791-890): zero edge of the sigmoid and Gauss-Legendre rule
  double fold_beta;
  double gl_x[16], gl_w[16];
  // cofold periodization (matrix.hh:905-1013): {active, alpha, beta, offset} on the device,
  // written by k_cofold_finish before the spectrum passes read it
  const double* cof;
};
constexpr int kFoldNodes = 16;

// Modified Bessel function of the second kind K_nu(x), nu >= 0, x > 0.
// Temme's series (N. M. Temme, J. Comput. Phys. 19, 324-337, 1975) for x <= 2 and
// Steed's continued fraction CF2 (I. J. Thompson and A. R. Barnett, J. Comput. Phys.
// 64, 490-509, 1986) for x > 2 give K_mu and K_mu+1 with |mu| <= 1/2; the upward
// recurrence K_{m+1} = K_{m-1} + (2m/x) K_m reaches nu.  1/Gamma(1+z) enters through
// its Taylor series (Abramowitz & Stegun 6.1.34; coefficients from the definition).
__device__ __constant__ double RGAMMA_SERIES[24] = {1.0, 0.5772156649015328606065, -0.655878071520253881077, -0.042002635034095235529,
    0.1665386113822914895017, -0.04219773455554433674821, -0.009621971527876973562115,
    0.007218943246663099542395, -0.001165167591859065112114, -0.0002152416741149509728157,
    0.0001280502823881161861532, -0.00002013485478078823865569, -0.000001250493482142670657345,
    0.000001133027231981695882374, -2.05633841697760710345e-7, 6.116095104481415817862e-9,
    5.002007644469222930056e-9, -1.181274570487020144588e-9, 1.043426711691100510492e-10,
    7.78226343990507125405e-12, -3.696805618642205708188e-12, 5.100370287454475979015e-13,
    -2.058326053566506783222e-14, -5.34812253942301798237e-15};

__device__ inline double bessel_k(double nu, double x) {
  const int nl = (int)(nu + 0.5);
  const double mu = nu - nl, mu2 = mu * mu;
  double kmu, kmu1;
  if (x <= 2.0) {
    const double x2 = 0.5 * x;
    const double pimu = 3.14159265358979323846264338327950288 * mu;
    const double fact = fabs(pimu) < 1e-15 ? 1.0 : pimu / sin(pimu);
    const double d = -log(x2);
    double e = mu * d;
    const double fact2 = fabs(e) < 1e-15 ? 1.0 : sinh(e) / e;
    double gam1 = 0.0, gam2 = 0.0, pw = 1.0;
    for (int k = 0; k < 12; k++) {
      gam2 += RGAMMA_SERIES[2 * k] * pw;
      gam1 -= RGAMMA_SERIES[2 * k + 1] * pw;
      pw *= mu2;
    }
    const double gampl = gam2 - mu * gam1; /* 1/Gamma(1+mu) */
    const double gammi = gam2 + mu * gam1; /* 1/Gamma(1-mu) */
    double ff = fact * (gam1 * cosh(e) + gam2 * fact2 * d);
    double sum = ff;
    e = exp(e);
    double p = 0.5 * e / gampl;
    double q = 0.5 / (e * gammi);
    double c = 1.0;
    const double dd = x2 * x2;
    double sum1 = p;
    for (int i = 1; i < 500; i++) {
      ff = (i * ff + p + q) / (i * (double)i - mu2);
      c *= dd / i;
      p /= (i - mu);
      q /= (i + mu);
      const double del = c * ff;
      sum += del;
      sum1 += c * (p - i * ff);
      if (fabs(del) < fabs(sum) * 1e-17) break;
    }
    kmu = sum;
    kmu1 = sum1 * (2.0 / x);
  } else {
    double b = 2.0 * (1.0 + x);
    double d = 1.0 / b;
    double h = d, delh = d;
    double q1 = 0.0, q2 = 1.0;
    const double a1 = 0.25 - mu2;
    double q = a1, c = a1, a = -a1;
    double s = 1.0 + q * delh;
    for (int i = 2; i < 100000; i++) {
      a -= 2 * (i - 1);
      c = -a * c / i;
      const double qnew = (q1 - b * q2) / a;
      q1 = q2;
      q2 = qnew;
      q += c * qnew;
      b += 2.0;
      d = 1.0 / (b + a * d);
      delh = (b * d - 1.0) * delh;
      h += delh;
      const double dels = q * delh;
      s += dels;
      if (fabs(dels / s) < 1e-17) break;
    }
    h = a1 * h;
    kmu = sqrt(3.14159265358979323846264338327950288 / (2.0 * x)) * exp(-x) / s;
    kmu1 = kmu * (mu + x + 0.5 - h) / x;
  }
  double km = kmu, kp = kmu1;
  for (int i = 1; i <= nl; i++) {
    const double kn = km + (2.0 * (mu + i) / x) * kp;
    km = kp;
    kp = kn;
  }
  return km;
}

__device__ __forceinline__ double cov_eval(const CovParams& c, const double* xt) {
  const double var = c.variance;
  const int dim = c.dim;
  double sum = 0.;
  for (int i = 0; i < dim; i++) sum += xt[i] * xt[i];
  switch (c.cov) {
    case 2: {  // spherical, covariance.hh:310-340
      const double h = sqrt(sum);
      if (h > 1.) return 0.;
      if (dim == 3) return var * (1. - 1.5 * h + 0.5 * pow(h, 3.));
      if (dim == 2)
        return var * (1. - 2. / 3.14159265358979323846 * (h * sqrt(1. - pow(h, 2.)) + asin(h)));
      return var * (1. - h);
    }
    case 0: return var * exp(-sqrt(sum));                   // exponential
    case 8: return var * exp(-pow(sqrt(sum), c.p0));        // gammaExponential
    case 1: {                                               // gaussian
      const double h = sqrt(sum);
      return var * exp(-h * h);
    }
    case 3: {  // separableExponential
      double s = 0.;
      for (int i = 0; i < dim; i++) s += fabs(xt[i]);
      return var * exp(-s);
    }
    case 5: {  // matern32
      const double h = sqrt(sum);
      return var * (1. + sqrt(3.) * h) * exp(-sqrt(3.) * h);
    }
    case 6: {  // matern52
      const double h = sqrt(sum);
      return var * (1. + sqrt(5.) * h + 5. / 3. * h * h) * exp(-sqrt(5.) * h);
    }
    case 7: {  // dampedOscillation
      const double h = sqrt(sum);
      if (dim == 3) return var * exp(-h) * cos(h / sqrt(3.));
      return var * exp(-h) * cos(h);
    }
    case 9: {  // cauchy
      const double h = sqrt(sum);
      return var * pow(1. + pow(h, 2.), -3.);
    }
    case 10: {  // generalizedCauchy
      const double h = sqrt(sum);
      return var * pow(1. + pow(h, c.p0), -c.p1);
    }
    case 11: {  // cubic
      const double h = sqrt(sum);
      if (h > 1.) return 0.;
      return var * (1. - 7. * pow(h, 2.) + 8.75 * pow(h, 3.) - 3.5 * pow(h, 5.) + 0.75 * pow(h, 7.));
    }
    case 4: {  // matern (covariance.hh:536-556), K_nu from bessel_k instead of GSL
      const double h = sqrt(sum);
      if (h < 1e-10) return var;
      return var * c.p1 / c.p2 * pow(c.p0 * h, c.p3) * bessel_k(c.p3, c.p0 * h);
    }
    case 12:  // whiteNoise
      for (int i = 0; i < dim; i++)
        if (fabs(xt[i]) > 1e-10) return 0.;
      return var;
    default: return 0.;
  }
}

// GeometryMatrix::transform (covariance.hh:18-138)
__device__ __forceinline__ void geo_apply(const CovParams& c, const double* x, double* xt) {
  if (c.aniso == 0) {
    for (int i = 0; i < c.dim; i++) xt[i] = c.geo[0] * x[i];
  } else if (c.aniso == 1) {
    for (int i = 0; i < c.dim; i++) xt[i] = c.geo[i] * x[i];
  } else {
    for (int i = 0; i < c.dim; i++) {
      double s = 0.;
      for (int k = 0; k < c.dim; k++) s += c.geo[i * c.dim + k] * x[k];
      xt[i] = s;
    }
  }
}

// SmoothstepSigmoid over ClampingSigmoid (covariance.hh:204-287)
__device__ __forceinline__ double sigmoid_smoothstep(double one, double zero, double x, int rec) {
  const double ax = fabs(x);
  const double x1 = ax < one ? 1. : (ax > zero ? 0. : (zero - ax) / (zero - one));
  const double x2 = 2. * x1 - 1.;
  double normalization = 1., addition = 1., output = 1.;
  for (int i = 1; i <= rec; i++) {
    output *= 2. * i;
    addition *= 1 - x2 * x2;
    output += addition;
    output /= 2. * i + 1.;
    normalization *= 2. * i / (2. * i + 1.);
  }
  output *= x2 / normalization;
  output += 1.;
  output /= 2.;
  return output;
}

// SmoothSigmoid (covariance.hh:147-195)
__device__ __forceinline__ double sigmoid_smooth(double one, double zero, double x) {
  const double ax = fabs(x);
  if (ax < one) return 1.;
  if (ax > zero) return 0.;
  const double x1 = (zero - ax) / (zero - one), x2 = (ax - one) / (zero - one);
  const double t1 = x1 > 0. ? exp(-1. / x1) : 0., t2 = x2 > 0. ? exp(-1. / x2) : 0.;
  return t1 / (t1 + t2);
}

__device__ __forceinline__ double sigmoid_of(const CovParams& c, double one, double zero, double x) {
  return c.sig ? sigmoid_smooth(one, zero, x) : sigmoid_smoothstep(one, zero, x, c.rec);
}

// computeMatrixEntriesWithMerge (matrix.hh:652-775) at torus cell jj: the 2^d mirrored
// copies of the covariance, each damped by the sigmoid, plus the remainder times the
// covariance at half the torus (radialPlus)
__device__ __noinline__ double cov_merge(const CovParams& c, const int* jj) {
  double tc[3] = {0, 0, 0}, mc[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
  for (int i = 0; i < c.dim; i++) tc[i] = (double)(unsigned int)jj[i] * c.h[i];
  double cst = 0.;
  if (c.plus) {
    for (int i = 0; i < c.dim; i++) mc[i] = c.ext[i] * c.factor / 2.;
    geo_apply(c, mc, xt);
    cst = cov_eval(c, xt);
  }
  const double eps = 1e-10;
  const double sqrtDim = sqrt((double)c.dim);
  double value = 0., remainder = 1.;
  for (int m = 0; m < (1 << c.dim); m++) {
    for (int i = 0; i < c.dim; i++) mc[i] = ((m >> i) & 1) ? c.ext[i] * c.factor - tc[i] : tc[i];
    double damp = 1.;
    if (c.radial && sqrtDim < c.factor / 2.) {
      double radius = 0.;
      for (int i = 0; i < c.dim; i++) radius += (mc[i] * mc[i]) / (c.ext[i] * c.ext[i]);
      radius = sqrt(radius);
      damp = sigmoid_of(c, c.sstart * sqrtDim - eps, c.factor - (c.factor - c.send) * sqrtDim + eps, radius);
    } else {
      for (int i = 0; i < c.dim; i++)
        damp *= sigmoid_of(c, c.ext[i] * c.sstart - eps, c.ext[i] * c.send + eps, mc[i]);
    }
    if (damp < eps) continue;
    remainder -= damp;
    geo_apply(c, mc, xt);
    value += cov_eval(c, xt) * damp;
  }
  return value + cst * remainder;
}

// integral of the sigmoid (one edge 1, zero edge beta) from 1 to b > 1: zero beyond beta;
// below it a polynomial (smoothstep, exact with 16 Gauss-Legendre nodes up to 15
// recursions) or the smooth sigmoid (32 panels of 16 nodes)
__device__ __noinline__ double fold_integral(const CovParams& c, double b) {
  const double hi = b < c.fold_beta ? b : c.fold_beta;
  if (hi <= 1.) return 0.;
  const int panels = c.sig ? 32 : (c.rec <= 15 ? 1 : 8);
  const double wdt = (hi - 1.) / panels;
  double s = 0.;
  for (int p = 0; p < panels; p++) {
    const double a0 = 1. + p * wdt, mid = a0 + 0.5 * wdt;
    double q = 0.;
    for (int k = 0; k < kFoldNodes; k++) q += c.gl_w[k] * sigmoid_of(c, 1., c.fold_beta, mid + 0.5 * wdt * c.gl_x[k]);
    s += 0.5 * wdt * q;
  }
  return s;
}

// computeMatrixEntriesWithFold (matrix.hh:791-890): classical coordinates, and beyond the
// normalized radius 1 the radius r is replaced by 1 + integral_1^r sigmoid
__device__ __noinline__ double cov_fold(const CovParams& c, const int* jj) {
  double x[3] = {0, 0, 0}, xt[3] = {0, 0, 0};
  double norm = 0.;
  for (int i = 0; i < c.dim; i++) {
    double v = (double)(unsigned int)jj[i] * c.h[i];
    if (v > c.half[i]) v -= c.wrap[i];
    x[i] = v;
    norm += (v * v) / (c.ext[i] * c.ext[i]);
  }
  norm = sqrt(norm / (double)c.dim);
  if (norm > 1.) {
    const double val = fold_integral(c, norm) + 1.;
    for (int i = 0; i < c.dim; i++) x[i] *= val / norm;
  }
  geo_apply(c, x, xt);
  return cov_eval(c, xt);
}

// signed integral over [a, b] of the cofold integrand sigmoid(0, beta - alpha, beta - t):
// the smoothstep is a polynomial (exact with 16 Gauss-Legendre nodes up to 15 recursions),
// the smooth sigmoid takes 32 panels of 16 nodes
__device__ __noinline__ double cofold_integral(const CovParams& c, double alpha, double beta, double a, double b) {
  const int panels = c.sig ? 32 : (c.rec <= 15 ? 1 : 8);
  const double wdt = (b - a) / panels;
  double s = 0.;
  for (int p = 0; p < panels; p++) {
    const double mid = a + (p + 0.5) * wdt;
    double q = 0.;
    for (int k = 0; k < kFoldNodes; k++)
      q += c.gl_w[k] * sigmoid_of(c, 0., beta - alpha, beta - (mid + 0.5 * wdt * c.gl_x[k]));
    s += 0.5 * wdt * q;
  }
  return s;
}

// classical coordinates of torus cell jj (computeMatrixEntriesWithMirroring, matrix.hh:615-638)
__device__ __forceinline__ void classical_coord(const CovParams& c, const int* jj, double* x) {
  for (int i = 0; i < c.dim; i++) {
    double v = (double)(unsigned int)jj[i] * c.h[i];
    if (v > c.half[i]) v -= c.wrap[i];
    x[i] = v;
  }
}

// cofold norm: largest |coordinate| / extension over the axes (matrix.hh:928-931)
__device__ __forceinline__ double cofold_norm(const CovParams& c, const double* x) {
  double norm = 0.;
  for (int i = 0; i < c.dim; i++) {
    const double r = __ddiv_rn(fabs(x[i]), c.ext[i]);
    if (r > norm) norm = r;
  }
  return norm;
}

// covariance of the classically wrapped coordinates x
__device__ __forceinline__ double cov_classical(const CovParams& c, const double* x) {
  double xt[3] = {0, 0, 0};
  if (c.aniso == 0) {
    for (int i = 0; i < c.dim; i++) xt[i] = c.geo[0] * x[i];
  } else if (c.aniso == 1) {
    for (int i = 0; i < c.dim; i++) xt[i] = c.geo[i] * x[i];
  } else {
    for (int i = 0; i < c.dim; i++) {
      double s = 0.;
      for (int k = 0; k < c.dim; k++) s += c.geo[i * c.dim + k] * x[k];
      xt[i] = s;
    }
  }
  return cov_eval(c, xt);
}

// modifyMatrixEntriesWithCofold (matrix.hh:983-1001): beyond norm 1 the values below alpha
// become the offset, those in [alpha, beta) the offset plus the integral of the sigmoid
__device__ __noinline__ double cov_cofold(const CovParams& c, const int* jj) {
  double x[3] = {0, 0, 0};
  classical_coord(c, jj, x);
  const double v = cov_classical(c, x);
  if (c.cof[0] == 0. || !(cofold_norm(c, x) > 1.)) return v;
  const double alpha = c.cof[1], beta = c.cof[2], offset = c.cof[3];
  if (v < alpha) return offset;
  if (v < beta) return cofold_integral(c, alpha, beta, alpha, v) + offset;
  return v;
}

// covariance at torus cell (j0, j1, j2) with the classical mirroring (or merge / fold / cofold)
__device__ __forceinline__ double cov_at(const CovParams& c, int j0, int j1, int j2) {
  const int jj[3] = {j0, j1, j2};
  if (c.per == 1) return cov_merge(c, jj);
  if (c.per == 2) return cov_fold(c, jj);
  if (c.per == 3) return cov_cofold(c, jj);
  double x[3] = {0, 0, 0};
  classical_coord(c, jj, x);
  return cov_classical(c, x);
}

// row p of the torus (dims 1..d-1 flattened), element j along dim 0
struct CovRowLoad {
  CovParams c;
  int rowmod;  // rows enumerate (j1, j2) with j1 = p % rowmod (T1 for the full torus,
               // T1/2+1 when only the non-mirrored rows of an even torus are needed)
  template <typename T>
  __device__ __forceinline__ T real(long long p, int j) const {
    const int j1 = c.dim > 1 ? (int)(p % rowmod) : 0;
    const int j2 = c.dim > 2 ? (int)(p / rowmod) : 0;
    return (T)cov_at(c, j, j1, j2);
  }
  template <typename T>
  __device__ __forceinline__ cx<T> load(long long p, int j, long long) const {
    return mk<T>(real<T>(p, j), (T)0);
  }
};

// covariance values computed by the caller (a user covariance functor evaluated on the
// host, matrix.hh:223-265 "custom-iso"/"custom-aniso") read in place of cov_at: `v` holds
// the matrix cells with dimension 0 fastest, `rowlen` values per row (T0, or T0/2+1 for
// the DCT matrix, whose row j > T0/2 reads the mirrored cell T0 - j)
struct ValRowLoad {
  const double* v;
  int T0;
  int rowlen;
  int mirror;
  unsigned long long n;
  template <typename T>
  __device__ __forceinline__ T real(long long p, int j) const {
    const int jj = (mirror && j > T0 / 2) ? T0 - j : j;
    const unsigned long long i = (unsigned long long)p * (unsigned long long)rowlen + (unsigned long long)jj;
    return in_bounds((long long)i, (long long)n) ? (T)v[i] : (T)0;
  }
  template <typename T>
  __device__ __forceinline__ cx<T> load(long long p, int j, long long) const {
    return mk<T>(real<T>(p, j), (T)0);
  }
};

// ---------------------------------------------------------------------------
// counter-based normal noise: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC 2011) + Box-Muller.  One call yields the
// normals of two frequencies: k and k + T/2 along the last axis (the pair shares the
// counter of its first member).  The 2x32 variant serves the DFT backend.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

__device__ __forceinline__ uint2 philox2x32_10(uint2 ctr, uint32_t key) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t lo = ctr.x * 0xD256D193u;
    const uint32_t hi = __umulhi(ctr.x, 0xD256D193u);
    ctr = make_uint2(hi ^ key ^ ctr.y, lo);
    key += 0x9E3779B9u;
  }
  return ctr;
}

// Box-Muller of two 32-bit words: u1 in (0,1), u2 in [0,1)
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, float& r1, float& r2) {
  const float u1 = ((float)a + 0.5f) * 2.3283064365386963e-10f;
  const float rad = sqrtf(-1.3862943611198906f * __log2f(u1));  // -2 ln u1
  float s, c;
  __sincosf(6.283185307179586f * ((float)b * 2.3283064365386963e-10f) - 3.141592653589793f, &s, &c);
  r1 = rad * c;
  r2 = rad * s;
}
__device__ __forceinline__ void box_muller(uint32_t a, uint32_t b, double& r1, double& r2) {
  const double u1 = ((double)a + 0.5) * 2.3283064365386963e-10;
  const double rad = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * ((double)b * 2.3283064365386963e-10) - 1.0, &s, &c);
  r1 = rad * c;
  r2 = rad * s;
}

// counter of the frequency pair whose first member has stored index si; `epoch` (0 for
// single calls) distinguishes the realizations of repeated launches of a captured graph
__device__ __forceinline__ uint4 pair_counter(uint64_t si, uint32_t epoch) {
  return make_uint4((uint32_t)si, (uint32_t)(si >> 32), 0x70616972u, epoch);
}

// SplitMix64 finaliser (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014): the output function of the SplitMix64 sequence
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// 128 random bits for the frequency pair whose first member has stored index si
__device__ __forceinline__ uint4 pair_bits(uint64_t seed, uint64_t si, uint32_t epoch) {
#ifdef PF_NOISE_SPLITMIX
  const uint64_t s = mix64(seed ^ 0x5851f42d4c957f2dull);
  const uint64_t a = mix64(s + (2 * si) * 0x9e3779b97f4a7c15ull);
  const uint64_t b = mix64(s + (2 * si + 1) * 0x9e3779b97f4a7c15ull);
  return make_uint4((uint32_t)a, (uint32_t)(a >> 32), (uint32_t)b, (uint32_t)(b >> 32));
#else
  return philox4x32_10(pair_counter(si, epoch), make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
#endif
}

template <typename T>
__device__ __forceinline__ void normal_pair(uint64_t seed, uint64_t idx, T& r1, T& r2) {
  const uint2 c = philox2x32_10(make_uint2((uint32_t)idx, (uint32_t)(idx >> 32) ^ (uint32_t)(seed >> 32)),
                                (uint32_t)seed);
  box_muller(c.x, c.y, r1, r2);
}

// ---------------------------------------------------------------------------
// noise x sqrt(eigenvalue) in the R2C half spectrum (R2CFieldBackend::set,
// r2cfieldbackend.hh:305-325 fed by generateField, matrix.hh:375-404)
// ---------------------------------------------------------------------------
struct R2CNoise {
  int dim;
  int ext[3];
  int T0c;
  int transposed;
  int dct;            // eigenvalue layout: 1 = DCT prod(T/2+1), 0 = half spectrum, 2 = full spectrum
  int D0, D1;         // DCT cells of dims 0 and 1
  const void* sq;     // sqrt(lambda), float or double per the pass precision
  const double* noise;  // reference draw order, or null for the counter-based generator
  uint64_t seed;
  const unsigned* epoch;  // device word mixed into the counters (null: 0)
  unsigned nsq, nnoise;   // buffer sizes (eigenvalues, noise doubles)
  int Tl;                 // extended cells of the last dimension (the pass axis)
  // The pass transforms along the last axis: p enumerates the other frequencies
  // (k0 fastest), j is the last-axis frequency.
  // pencils of the pass: k0 = p (fastest), k1 = the outer block index (3D)
  __device__ __forceinline__ void decode(int p, int io, int& k0, int& k1) const {
    k0 = p;
    k1 = dim == 3 ? io : 0;
  }
  __device__ __forceinline__ unsigned stored(int k0, int k1, int kl) const {
    if (dim == 2) return (unsigned)k0 + (unsigned)T0c * (unsigned)kl;
    if (transposed) return (unsigned)k0 + (unsigned)T0c * ((unsigned)kl + (unsigned)ext[2] * (unsigned)k1);
    return (unsigned)k0 + (unsigned)T0c * ((unsigned)k1 + (unsigned)ext[1] * (unsigned)kl);
  }
  __device__ __forceinline__ unsigned lam_index(int k0, int k1, int kl) const {
    const int a1 = dim == 3 ? k1 : kl, a2 = dim == 3 ? kl : 0;
    if (dct == 1) {
      const int m1 = a1 <= ext[1] / 2 ? a1 : ext[1] - a1;
      const int m2 = a2 <= ext[2] / 2 ? a2 : ext[2] - a2;
      return (unsigned)k0 + (unsigned)D0 * ((unsigned)m1 + (unsigned)D1 * (unsigned)m2);
    }
    if (dct == 2)  // full DFT spectrum (dftmatrixbackend.hh:303-307)
      return (unsigned)k0 + (unsigned)ext[0] * ((unsigned)a1 + (unsigned)ext[1] * (unsigned)a2);
    return (unsigned)k0 + (unsigned)T0c * ((unsigned)a1 + (unsigned)ext[1] * (unsigned)a2);
  }
  template <typename T>
  __device__ __forceinline__ cx<T> scale(int k0, int k1, int kl, T r1, T r2) const {
    const unsigned li = lam_index(k0, k1, kl);
    if (!in_bounds32(li, nsq)) return mk<T>(0, 0);
    const T lam = ((const T*)sq)[li];
    const int a1 = dim == 3 ? k1 : kl, a2 = dim == 3 ? kl : 0;
    const bool selfconj = (k0 == 0 || 2 * k0 == ext[0]) && (a1 == 0 || 2 * a1 == ext[1]) &&
                          (dim < 3 || a2 == 0 || 2 * a2 == ext[2]);
    if (selfconj) return mk<T>(lam * r1, (T)0);
    // FP64 keeps the reference's lambda / sqrt(2) (r2cfieldbackend.hh:322-323)
    const T s = sizeof(T) == 8 ? lam / (T)1.41421356237309504880168872420969808
                               : lam * (T)0.70710678118654752440084436210484903928;
    return mk<T>(s * r1, s * r2);
  }
  // reference draw order noise (parity mode) or the counter-based pair definition
  template <typename T>
  __device__ __forceinline__ cx<T> load(long long pl, int j, long long io) const {
    int k0, k1;
    decode((int)pl, (int)io, k0, k1);
    const int L = Tl;
    T r1, r2;
    if (noise) {
      const unsigned si = stored(k0, k1, j);
      if (!in_bounds32(2 * si + 1, nnoise)) return mk<T>(0, 0);
      r1 = (T)noise[2 * si];
      r2 = (T)noise[2 * si + 1];
    } else {
      const int h = L / 2;
      const bool second = (L % 2 == 0) && j >= h;
      const unsigned si = stored(k0, k1, second ? j - h : j);
      const uint4 c = pair_bits(seed, si, epoch ? __ldg(epoch) : 0u);
      if (second)
        box_muller(c.z, c.w, r1, r2);
      else
        box_muller(c.x, c.y, r1, r2);
    }
    return scale<T>(k0, k1, j, r1, r2);
  }
  // elements j and j + L/2 from one generator call (L even, no noise buffer)
  template <typename T>
  __device__ __forceinline__ void load2(int pl, int j, int io, cx<T>& v0, cx<T>& v1) const {
    int k0, k1;
    decode(pl, io, k0, k1);
    const int h = Tl / 2;
    T r1, r2, r3, r4;
    if (noise) {
      const unsigned s0 = stored(k0, k1, j), s1 = stored(k0, k1, j + h);
      if (!in_bounds32(2 * s0 + 1, nnoise) || !in_bounds32(2 * s1 + 1, nnoise)) return;
      r1 = (T)noise[2 * s0];
      r2 = (T)noise[2 * s0 + 1];
      r3 = (T)noise[2 * s1];
      r4 = (T)noise[2 * s1 + 1];
    } else {
      const uint4 c = pair_bits(seed, stored(k0, k1, j), epoch ? __ldg(epoch) : 0u);
      box_muller(c.x, c.y, r1, r2);
      box_muller(c.z, c.w, r3, r4);
    }
    v0 = scale<T>(k0, k1, j, r1, r2);
    v1 = scale<T>(k0, k1, j + h, r3, r4);
  }
};

// full-torus complex noise of the DFT backend (dftfieldbackend.hh:276-280); the pass
// runs along the slowest dimension d-1 first (contiguous when dim == 1)
struct DFTNoise {
  int dim;
  int ext[3];
  int Ts[3];
  int transposed;
  int mat;  // 0 DCT (mirrored lookup), 2 DFT (full layout, stored order)
  const void* sq;
  const double* noise;
  uint64_t seed;
  unsigned nsq, nnoise;
  template <typename T>
  __device__ __forceinline__ cx<T> load(long long p, int j, long long) const {
    int k[3] = {0, 0, 0};
    if (dim == 1) {
      k[0] = j;
    } else if (dim == 2) {
      k[0] = (int)p;
      k[1] = j;
    } else {
      k[0] = (int)(p % ext[0]);
      k[1] = (int)(p / ext[0]);
      k[2] = j;
    }
    int a[3] = {k[0], k[1], k[2]};
    if (transposed) {
      const int x = dim - 1, y = dim - 2;
      const int t = a[x];
      a[x] = a[y];
      a[y] = t;
    }
    const uint64_t si = (uint64_t)a[0] + (uint64_t)Ts[0] * ((uint64_t)a[1] + (uint64_t)Ts[1] * (uint64_t)a[2]);
    uint64_t li;
    if (mat == 0) {
      int m[3];
      int D[3];
      for (int i = 0; i < 3; i++) {
        D[i] = ext[i] / 2 + 1;
        m[i] = k[i] <= ext[i] / 2 ? k[i] : ext[i] - k[i];
      }
      li = (uint64_t)m[0] + (uint64_t)D[0] * ((uint64_t)m[1] + (uint64_t)D[1] * (uint64_t)m[2]);
    } else {
      li = (uint64_t)k[0] + (uint64_t)ext[0] * ((uint64_t)k[1] + (uint64_t)ext[1] * (uint64_t)k[2]);
    }
    if (!in_bounds32((unsigned)li, nsq)) return mk<T>(0, 0);
    const T lam = ((const T*)sq)[li];
    T r1, r2;
    if (noise) {
      if (!in_bounds32((unsigned)(2 * si + 1), nnoise)) return mk<T>(0, 0);
      r1 = (T)noise[2 * si];
      r2 = (T)noise[2 * si + 1];
    } else {
      normal_pair<T>(seed, si, r1, r2);
    }
    return mk<T>(lam * r1, lam * r2);
  }
};

// Noise of one even/odd symmetry type of the DCT/DST field backend, extended to the whole
// torus so that complex backward transforms along every axis reproduce the mixed
// REDFT00/RODFT00 transform of the reference (dctdstfieldbackend.hh:149-165, 326-438):
//  - stored value at DCT index m (m_i <= T_i/2): 2^{-d/2} sqrt(lambda(m)) r 2^{b/2}, b = number
//    of even axes with m_i on the border (0 or T_i/2), and 0 if an odd axis is on its border
//    (DCTDSTFieldBackend::set, 418-438); r is draw type*D + flat(m) of the reference order;
//  - torus frequency k maps to m_i = min(k_i, T_i - k_i), with the sign -1 on odd axes for
//    k_i > T_i/2: then sum_k x(k) e^{+2 pi i k.x/T} = i^{#odd} * (REDFT00 x RODFT00 ...)(x),
//    since sum over an odd axis gives 2i sum sin(pi m x / (T/2)) = i RODFT00;
//  - the loader multiplies by i^{-#odd}, so the real part of the transform is the reference's
//    field of this type.
// Pencils of the first pass run along the last axis: p enumerates (k0, k1), j is k_last.
struct DctDstNoise {
  int dim;
  int ext[3];
  int D[3];
  int type;  // bit i set: axis i odd (RODFT00)
  int transposed;  // draws in the transposed cell order (fftw.transposed): dims d-1, d-2 swapped
  const void* sq;
  const double* noise;
  uint64_t seed;
  unsigned nsq, nnoise;
  unsigned Dtot;
  template <typename T>
  __device__ __forceinline__ cx<T> load(long long p, int j, long long) const {
    int k[3] = {0, 0, 0};
    if (dim == 1) {
      k[0] = j;
    } else if (dim == 2) {
      k[0] = (int)p;
      k[1] = j;
    } else {
      k[0] = (int)(p % ext[0]);
      k[1] = (int)(p / ext[0]);
      k[2] = j;
    }
    int m[3] = {0, 0, 0};
    int sign = 1, border = 0, nodd = 0;
    for (int i = 0; i < dim; i++) {
      const int h = ext[i] / 2;
      m[i] = k[i] <= h ? k[i] : ext[i] - k[i];
      const bool edge = m[i] == 0 || m[i] == h;
      if ((type >> i) & 1) {
        if (edge) return mk<T>(0, 0);
        if (k[i] > h) sign = -sign;
        nodd++;
      } else if (edge) {
        border++;
      }
    }
    const unsigned li = (unsigned)m[0] + (unsigned)D[0] * ((unsigned)m[1] + (unsigned)D[1] * (unsigned)m[2]);
    if (!in_bounds32(li, nsq)) return mk<T>(0, 0);
    // draw order (matrix.hh:349-360): the field backend's local cells, whose last two
    // dimensions are swapped in the transposed layout (dctdstfieldbackend.hh:855-871)
    unsigned ci = li;
    if (transposed && dim == 3)
      ci = (unsigned)m[0] + (unsigned)D[0] * ((unsigned)m[2] + (unsigned)D[2] * (unsigned)m[1]);
    else if (transposed && dim == 2)
      ci = (unsigned)m[1] + (unsigned)D[1] * (unsigned)m[0];
    const unsigned ri = (unsigned)type * Dtot + ci;
    T r;
    if (noise) {
      if (!in_bounds32(ri, nnoise)) return mk<T>(0, 0);
      r = (T)noise[ri];
    } else {
      T r2;
      normal_pair<T>(seed, ri, r, r2);
    }
    T v = ((const T*)sq)[li] * r * (T)sign;
    // 2^{-d/2} 2^{b/2}
    const int e = border - dim;
    v *= (e & 1) ? (T)0.70710678118654752440084436210484903928 : (T)1;
    v = ldexp(v, (e + (e & 1)) / 2);
    switch (nodd & 3) {
      case 0: return mk<T>(v, 0);
      case 1: return mk<T>(0, -v);
      case 2: return mk<T>(-v, 0);
      default: return mk<T>(0, v);
    }
  }
};

// eigenvalue factor lookup for the fused matvec pass (fieldBackend.mult,
// r2cfieldbackend.hh:337-341 with matrixBackend.eval, matrix.hh:1482-1495)
struct MultMid {
  static constexpr bool active = true;
  int dim;
  int ext[3];
  int C0;        // cells of dim 0 in the frequency array (T0/2+1 for R2C, T0 for DFT)
  int LC0;       // cells of dim 0 in the eigenvalue array (layouts 1 and 2)
  int layout;    // 0 DCT, 1 natural half spectrum, 2 natural full spectrum
  int D0, D1;
  int axis;      // axis of the fused pass (dim-1)
  const void* fac;  // factor per stored eigenvalue (precision of the pass)
  unsigned nfac;
  // pencils: 1D one row; 2D k0 = p; 3D k0 = p, k1 = the outer block index
  template <typename T>
  __device__ __forceinline__ cx<T> operator()(long long p, int j, long long io, cx<T> v) const {
    int k0, k1 = 0, k2 = 0;
    if (dim == 1) {
      k0 = j;
    } else if (dim == 2) {
      k0 = (int)p;
      k1 = j;
    } else {
      k0 = (int)p;
      k1 = (int)io;
      k2 = j;
    }
    unsigned li;
    if (layout == 0) {
      const int m0 = k0 <= ext[0] / 2 ? k0 : ext[0] - k0;
      const int m1 = k1 <= ext[1] / 2 ? k1 : ext[1] - k1;
      const int m2 = k2 <= ext[2] / 2 ? k2 : ext[2] - k2;
      li = (unsigned)m0 + (unsigned)D0 * ((unsigned)m1 + (unsigned)D1 * (unsigned)m2);
    } else {
      li = (unsigned)k0 + (unsigned)LC0 * ((unsigned)k1 + (unsigned)ext[1] * (unsigned)k2);
    }
    if (!in_bounds32(li, nfac)) return mk<T>(0, 0);
    const T f = ((const T*)fac)[li];
    return mk<T>(v.x * f, v.y * f);
  }
};

// ---------------------------------------------------------------------------
// eigenvalue scan (matrix.hh:266-317) over the transformed spectrum
// ---------------------------------------------------------------------------
struct ScanOut {
  unsigned int small, zero, negative, pad;
  unsigned long long minkey;
};

__device__ __forceinline__ unsigned long long dkey(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// key of an ordered key back to the double (inverse of dkey)
__device__ __forceinline__ double dkey_value(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// Statistics of modifyMatrixEntriesWithCofold (matrix.hh:913-945) over the matrix cells
// C0 x C1 x C2 (the T/2+1 cells per axis of the DCT matrix, the torus otherwise):
// keys[0] = min key of the classical values with norm <= 1 (the constrained cells),
// keys[1] = max key of those with norm > 1 within ext/T of half the torus on some axis.
__global__ void __launch_bounds__(kThreads) k_cofold_stats(CovParams c, int C0, int C1, int C2,
                                                           unsigned long long* keys) {
  unsigned long long mn = ~0ull, mx = 0ull;
  const uint64_t n = (uint64_t)C0 * C1 * C2;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i / (uint64_t)C0;
    const int jj[3] = {(int)(i % (uint64_t)C0), (int)(r % (uint64_t)C1), (int)(r / (uint64_t)C1)};
    double x[3] = {0, 0, 0};
    classical_coord(c, jj, x);
    const double v = cov_classical(c, x);
    if (cofold_norm(c, x) <= 1.) {
      const unsigned long long k = dkey(v);
      mn = k < mn ? k : mn;
    } else {
      bool border = false;
      for (int a = 0; a < c.dim; a++)
        if (c.half[a] - fabs(x[a]) < __ddiv_rn(c.ext[a], (double)(unsigned int)c.T[a])) border = true;
      if (border) {
        const unsigned long long k = dkey(v);
        mx = k > mx ? k : mx;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long a = __shfl_xor_sync(0xffffffffu, mn, o), b = __shfl_xor_sync(0xffffffffu, mx, o);
    mn = a < mn ? a : mn;
    mx = b > mx ? b : mx;
  }
  if ((threadIdx.x & 31) == 0) {
    if (mn != ~0ull) atomicMin(&keys[0], mn);
    if (mx != 0ull) atomicMax(&keys[1], mx);
  }
}

// alpha = max border value, beta = min(max_factor * alpha, min constrained value),
// offset = beta - integral_alpha^beta sigmoid (matrix.hh:947-972); cof = {active, alpha,
// beta, offset}; inactive (identity) when either set of cells is empty
__global__ void k_cofold_finish(CovParams c, double max_factor, const unsigned long long* keys, double* cof) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (keys[0] == ~0ull || keys[1] == 0ull) {
    cof[0] = 0.;
    return;
  }
  const double minc = dkey_value(keys[0]), alpha = dkey_value(keys[1]);
  const double mf = max_factor * alpha;
  const double beta = minc < mf ? minc : mf;
  cof[0] = 1.;
  cof[1] = alpha;
  cof[2] = beta;
  cof[3] = beta - cofold_integral(c, alpha, beta, alpha, beta);
}

struct ScanArgs {
  const double2* spec;  // complex spectrum, natural layout, cells C[0..2]
  int C[3];
  int Ts[3];            // stored layout cells (swapped when transposed)
  int transposed;
  int dim;
  int faithful;         // reference real-view scan (R2C only)
  uint64_t count;
  double N;
  double threshold;
  double* lam;          // out: eigenvalues, natural layout
  double* sq64;
  float* sq32;
  float* lam32;
  ScanOut* out;
};

__device__ __forceinline__ void scan_one(double v, double thr, unsigned int& sm, unsigned int& ze,
                                         unsigned int& ne, double& mn) {
  if (v < mn) mn = v;
  if (v < 1e-6) {
    if (v < thr) {
      if (v > -thr)
        ze++;
      else
        ne++;
    } else
      sm++;
  }
}

__global__ void __launch_bounds__(kThreads) k_scan(const ScanArgs a) {
  unsigned int sm = 0, ze = 0, ne = 0;
  double mn = 1.7976931348623157e308;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.count; i += stride) {
    const double2 z = a.spec[i];
    double re = z.x / a.N, im = z.y / a.N;
    if (a.faithful) {
      // position of this entry in the reference's stored (possibly transposed) order
      const uint64_t k0 = i % a.C[0];
      const uint64_t r = i / a.C[0];
      const uint64_t k1 = r % a.C[1];
      const uint64_t k2 = r / a.C[1];
      uint64_t si;
      if (a.transposed && a.dim == 3)
        si = k0 + (uint64_t)a.C[0] * (k2 + (uint64_t)a.C[2] * k1);
      else
        si = i;
      if (2 * si < a.count) {
        scan_one(re, a.threshold, sm, ze, ne, mn);
        if (re < 0.) re = 0.;
      }
      if (2 * si + 1 < a.count) scan_one(im, a.threshold, sm, ze, ne, mn);
    } else {
      scan_one(re, a.threshold, sm, ze, ne, mn);
      if (re < 0.) re = 0.;
    }
    a.lam[i] = re;
    const double s = sqrt(re);
    a.sq64[i] = s;
    a.sq32[i] = (float)s;
    a.lam32[i] = (float)re;
  }
  // block reduction
  __shared__ unsigned int rs[3][kThreads / 32];
  __shared__ double rm[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    sm += __shfl_down_sync(0xffffffffu, sm, o);
    ze += __shfl_down_sync(0xffffffffu, ze, o);
    ne += __shfl_down_sync(0xffffffffu, ne, o);
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    rs[0][w] = sm;
    rs[1][w] = ze;
    rs[2][w] = ne;
    rm[w] = mn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kThreads / 32; k++) {
      sm += rs[0][k];
      ze += rs[1][k];
      ne += rs[2][k];
      mn = fmin(mn, rm[k]);
    }
    if (sm) atomicAdd(&a.out->small, sm);
    if (ze) atomicAdd(&a.out->zero, ze);
    if (ne) atomicAdd(&a.out->negative, ne);
    atomicMin(&a.out->minkey, dkey(mn));
  }
}

// DFT-matrix spectrum scan: get() is the real part and set() clears both parts
// (dftmatrixbackend.hh:322-338); same statistics as above.
// (covered by k_scan with faithful = 0 over the full complex torus.)

// factor arrays for the matvecs: lambda/N, sqrt(lambda)/N, 1/(lambda N), pinv(lambda)/N
template <typename T>
__global__ void k_factors(const double* __restrict__ lam, uint64_t n, double invN, int op, T* out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double l = lam[i];
    double f;
    if (op == 0)
      f = l * invN;
    else if (op == 1)
      f = sqrt(l) * invN;
    else if (op == 2)
      f = (1. / l) * invN;
    else  // pseudo-inverse: clamped (zero) eigenvalues are left out of the preconditioner
      f = l > 0. ? (1. / l) * invN : 0.;
    out[i] = (T)f;
  }
}

template <typename S>
__global__ void k_transform(S* v, uint64_t n, int kind, double lam) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = apply_mutator<S>(kind, (S)lam, v[i]);
}

}  // namespace pf
