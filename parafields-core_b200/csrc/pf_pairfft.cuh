// pf_pairfft.cuh -- FP32 pencil passes on Blackwell's paired FP32 instructions.
//
// Every thread transforms the same butterfly column of TWO pencils (A, B) at once.  The
// pair's values live in "P2" form, re = (Re A, Re B) and im = (Im A, Im B), so each complex
// add/subtract of a Stockham stage is one sm_100 FADD2/FFMA2 for both pencils and a
// twiddle multiply is five (__fadd2_rn / __fmul2_rn / __ffma2_rn, PTX add/mul/fma.rn.f32x2):
// half the issue slots of scalar butterflies, which is what bounds these passes.
//
// Layout and schedule (L a power of two, 64..2048, 256 threads, Q = 2048/L pairs per CTA):
//  - a thread owns 8 P2 values of its pair; stage 1 (radix 8) runs on the values the
//    loader produced, stages 2.. exchange through ONE padded shared buffer of 16-byte slots
//    (Re A, Re B, Im A, Im B), slot(q, j) = q*PLQ + j + j/8, read-all / barrier / write-all;
//  - the last stage writes its outputs straight to global memory (pruned to Lout);
//  - per-stage twiddle tables are stored by (r-1)*Ns + k (k fastest), pre-broadcast as
//    (wx, wx, wy, wy), so a warp's twiddle loads are conflict-free LDS.128;
//  - CTAs are persistent: the tables are copied to shared memory once per CTA;
//  - bounds violations are accumulated per thread and reported by one atomic at the end.
#pragma once

#include <cuda.h>

#include "pf_cg.cuh"
#include "pf_fastfft.cuh"

namespace pf {

constexpr int kP2Threads = 256;
// resident CTAs per SM the register allocation is sized for (per kernel family).  The
// strided pass is held to 64 registers (4 CTAs per SM): alone it runs as fast as with 3,
// and in the two-stream batch its CTAs fit beside the other stream's kernels (256^3
// Matern-3/2 batch: 0.388 against 0.401 ms per realization).  At 64 registers the
// complex-to-real pass spills and runs slower alone (0.088 against 0.077 ms) and in the
// batch, so it keeps 3.  The fused matvec pass spills a few words at 64 registers but waits
// on its gathers, and the extra warps win (128^3 C^-1: 0.066 against 0.075 ms).
#ifndef PF_P2_MIN_NOISE
#define PF_P2_MIN_NOISE 4
#endif
#ifndef PF_P2_MIN_C2C
#define PF_P2_MIN_C2C 4
#endif
#ifndef PF_P2_MIN_C2R
#define PF_P2_MIN_C2R 3
#endif
#ifndef PF_P2_MIN_MID
#define PF_P2_MIN_MID 4
#endif

struct P2 {
  float2 re, im;
};

__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ P2 padd(const P2& a, const P2& b) { return {f2add(a.re, b.re), f2add(a.im, b.im)}; }
__device__ __forceinline__ P2 psub(const P2& a, const P2& b) { return {f2sub(a.re, b.re), f2sub(a.im, b.im)}; }
__device__ __forceinline__ P2 p2_of(float4 s) { return {make_float2(s.x, s.y), make_float2(s.z, s.w)}; }
__device__ __forceinline__ float4 slot_of(const P2& a) { return make_float4(a.re.x, a.re.y, a.im.x, a.im.y); }
// P2 from the complex values of pencil A and pencil B
__device__ __forceinline__ P2 p2_ab(float2 a, float2 b) { return {make_float2(a.x, b.x), make_float2(a.y, b.y)}; }

// a * w for a twiddle pre-broadcast as (wx, wx, wy, wy)
__device__ __forceinline__ P2 ptw(const P2& a, float4 w) {
  const float2 wx = make_float2(w.x, w.y), wy = make_float2(w.z, w.w);
  return {f2sub(f2mul(a.re, wx), f2mul(a.im, wy)), f2fma(a.re, wy, f2mul(a.im, wx))};
}

// out[q] = sum_r v[r] exp(S 2 pi i r q / R), R = 2, 4, 8 (same conventions as Dft<T, R>)
template <int S>
__device__ __forceinline__ void pdft2(P2& v0, P2& v1) {
  const P2 a = v0;
  v0 = padd(a, v1);
  v1 = psub(a, v1);
}

template <int S>
__device__ __forceinline__ void pdft4(P2& v0, P2& v1, P2& v2, P2& v3) {
  const P2 a = padd(v0, v2), b = psub(v0, v2), c = padd(v1, v3), d = psub(v1, v3);
  v0 = padd(a, c);
  v2 = psub(a, c);
  if (S > 0) {  // X1 = b + i d, X3 = b - i d
    v1 = {f2sub(b.re, d.im), f2add(b.im, d.re)};
    v3 = {f2add(b.re, d.im), f2sub(b.im, d.re)};
  } else {  // X1 = b - i d, X3 = b + i d
    v1 = {f2add(b.re, d.im), f2sub(b.im, d.re)};
    v3 = {f2sub(b.re, d.im), f2add(b.im, d.re)};
  }
}

template <int S>
__device__ __forceinline__ void pdft8(P2* v) {
  P2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  P2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  pdft4<S>(e0, e1, e2, e3);
  pdft4<S>(o0, o1, o2, o3);
  const float2 h = make_float2(0.70710678118654752f, 0.70710678118654752f);
  const float2 nh = make_float2(-0.70710678118654752f, -0.70710678118654752f);
  v[0] = padd(e0, o0);
  v[4] = psub(e0, o0);
  // q = 2: o2 * (S i)
  if (S > 0) {
    v[2] = {f2sub(e2.re, o2.im), f2add(e2.im, o2.re)};
    v[6] = {f2add(e2.re, o2.im), f2sub(e2.im, o2.re)};
  } else {
    v[2] = {f2add(e2.re, o2.im), f2sub(e2.im, o2.re)};
    v[6] = {f2sub(e2.re, o2.im), f2add(e2.im, o2.re)};
  }
  // q = 1: o1 * W8 = h (o1.re - S o1.im, o1.im + S o1.re)
  const float2 t1r = S > 0 ? f2sub(o1.re, o1.im) : f2add(o1.re, o1.im);
  const float2 t1i = S > 0 ? f2add(o1.im, o1.re) : f2sub(o1.im, o1.re);
  v[1] = {f2fma(h, t1r, e1.re), f2fma(h, t1i, e1.im)};
  v[5] = {f2fma(nh, t1r, e1.re), f2fma(nh, t1i, e1.im)};
  // q = 3: o3 * W8^3 = -h (o3.re + S o3.im, o3.im - S o3.re)
  const float2 u = S > 0 ? f2add(o3.re, o3.im) : f2sub(o3.re, o3.im);
  const float2 w = S > 0 ? f2sub(o3.im, o3.re) : f2add(o3.im, o3.re);
  v[3] = {f2fma(nh, u, e3.re), f2fma(nh, w, e3.im)};
  v[7] = {f2fma(h, u, e3.re), f2fma(h, w, e3.im)};
}

template <int R, int S>
__device__ __forceinline__ void pdft(P2* v) {
  if constexpr (R == 8) {
    pdft8<S>(v);
  } else if constexpr (R == 4) {
    pdft4<S>(v[0], v[1], v[2], v[3]);
  } else {
    static_assert(R == 2, "power-of-two radices only");
    pdft2<S>(v[0], v[1]);
  }
}

// ---------------------------------------------------------------------------
// compile-time geometry of a pair pass
// ---------------------------------------------------------------------------
template <int L>
struct P2Geom {
  static_assert(L >= 64 && L <= 2048 && (L & (L - 1)) == 0, "power-of-two length 64..2048");
  static constexpr int TP = L / 8;                   // threads per pair
  static constexpr int Q = kP2Threads / TP;          // pairs per CTA
  static constexpr int NP = 2 * Q;                   // pencils per tile
  // padded slots per pair: L + L/8 rounded so that the Q pairs of a warp phase fall in
  // distinct 16-byte bank groups (residue 8/Q mod 8 for Q <= 8, odd beyond)
  static constexpr int base = L + L / 8;
  static constexpr int want = Q >= 8 ? 1 : (8 / Q) % 8;
  static constexpr int PLQ = base + ((want - base % 8) + 8) % 8;
  // twiddle entries of stages 2.. ((R-1) * Ns each)
  template <int Ns = 8>
  static constexpr int tw_entries() {
    if constexpr (Ns >= L)
      return 0;
    else
      return (pick_radix(L / Ns) - 1) * Ns + tw_entries<Ns * pick_radix(L / Ns)>();
  }
  static constexpr int NTW = tw_entries();
};

__device__ __forceinline__ int p2_slot(int PLQ, int q, int j) { return q * PLQ + j + (j >> 3); }

// stages 2.. of the transform: v holds the thread's 8 values of stage Ns's input
// (after stage 1 they are in buf).  Out(j, P2) receives the final outputs.
template <int L, int S, int Ns, int TWOFF, class Out>
__device__ __forceinline__ void p2_stages(P2 (&v)[8], float4* buf, const float4* tw, int u, int q,
                                          const Out& out) {
  using G = P2Geom<L>;
  constexpr int R = pick_radix(L / Ns);
  constexpr int NB = 8 / R;
  constexpr int NBF = L / R;
  constexpr bool LAST = Ns * R == L;
  __syncthreads();
  // TP, NBF and Ns are multiples of 8, so slot(j + 8m) = slot(j) + 9m: one runtime slot
  // per thread, the rest compile-time offsets
  static_assert(G::TP % 8 == 0 && NBF % 8 == 0 && Ns % 8 == 0, "slot offsets need multiples of 8");
  const float4* rd = buf + p2_slot(G::PLQ, q, u);
#pragma unroll
  for (int i = 0; i < NB; i++) {
#pragma unroll
    for (int r = 0; r < R; r++) v[i * R + r] = p2_of(rd[(i * G::TP + r * NBF) / 8 * 9]);
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NB; i++) {
    const int t = u + i * G::TP;
    const int k = t % Ns;
#pragma unroll
    for (int r = 1; r < R; r++) v[i * R + r] = ptw(v[i * R + r], tw[TWOFF + (r - 1) * Ns + k]);
    pdft<R, S>(&v[i * R]);
    if constexpr (LAST) {
#pragma unroll
      for (int r = 0; r < R; r++) out(t + r * Ns, v[i * R + r]);
    } else {
      float4* wr = buf + p2_slot(G::PLQ, q, (t / Ns) * Ns * R + k);
#pragma unroll
      for (int r = 0; r < R; r++) wr[r * Ns / 8 * 9] = slot_of(v[i * R + r]);
    }
  }
  if constexpr (!LAST) p2_stages<L, S, Ns * R, TWOFF + (R - 1) * Ns>(v, buf, tw, u, q, out);
}

// whole transform from the stage-1 inputs v[r] = element u + r*L/8
template <int L, int S, class Out>
__device__ __forceinline__ void p2_transform(P2 (&v)[8], float4* buf, const float4* tw, int u, int q,
                                             const Out& out) {
  using G = P2Geom<L>;
  pdft8<S>(v);
  float4* wr = buf + p2_slot(G::PLQ, q, u * 8);  // u*8 + r stays within one group of 8
#pragma unroll
  for (int r = 0; r < 8; r++) wr[r] = slot_of(v[r]);
  p2_stages<L, S, 8, 0>(v, buf, tw, u, q, out);
}

__device__ __forceinline__ void p2_copy_table(float4* dst, const float4* __restrict__ src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
}

// bit 1: an index outside its buffer (access skipped); bit 2: a bounded wait gave up
__device__ __forceinline__ void p2_report(unsigned bad) {
  if (bad) atomicOr(&g_bounds_error, bad);
}

// ---------------------------------------------------------------------------
// pair loaders / storers over the plan's arrays (element (p, j, o) at
// p*rowstride + j*jstride + o*ostride, complex float)
// ---------------------------------------------------------------------------
// pencils p and p+1 adjacent (rowstride 1, even strides, 16-byte aligned base)
struct P2ArrLoad {
  const float4* ptr;  // pairs of complex
  unsigned jstride, ostride;  // in complex elements (even)
  unsigned n;                 // complex elements in the buffer
  int Lin;
  int np;
  // per-tile part of the loads of pencils (p, p+1) at outer index o, elements j < Lin
  struct Tile {
    unsigned base;
    bool two, ok;
  };
  __device__ __forceinline__ Tile tile(int p, int o, unsigned& bad) const {
    Tile t;
    t.base = (unsigned)p + (unsigned)o * ostride;
    t.two = p + 1 < np;
    const unsigned long long top = (unsigned long long)t.base + (unsigned long long)(Lin - 1) * jstride + 1u;
    t.ok = p < np && Lin > 0 && top < (unsigned long long)n;
    bad |= (unsigned)(p < np && Lin > 0 && !t.ok);
    return t;
  }
  __device__ __forceinline__ P2 load_t(const Tile& t, int j) const {
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t.ok && j < Lin) s = ptr[(t.base + (unsigned)j * jstride) >> 1];
    if (!t.two) {
      s.z = 0.f;
      s.w = 0.f;
    }
    return {make_float2(s.x, s.z), make_float2(s.y, s.w)};
  }
};

struct P2ArrStore {
  float4* ptr;
  unsigned jstride, ostride;
  unsigned n;
  int np;
  // per-tile part of the stores of pencils (p, p+1) at outer index o, elements j < Lout:
  // base index, whether pencil p+1 exists, and one bounds check for the whole tile
  struct Tile {
    unsigned base;
    bool two, ok;
  };
  __device__ __forceinline__ Tile tile(int p, int o, int Lout, unsigned& bad) const {
    Tile t;
    t.base = (unsigned)p + (unsigned)o * ostride;
    t.two = p + 1 < np;
    const unsigned long long top =
        (unsigned long long)t.base + (unsigned long long)(Lout - 1) * jstride + (t.two ? 1u : 0u);
    t.ok = p < np && Lout > 0 && top < (unsigned long long)n;
    bad |= (unsigned)(p < np && Lout > 0 && !t.ok);
    return t;
  }
  __device__ __forceinline__ void store_t(const Tile& t, int j, const P2& v) const {
    if (!t.ok) return;
    const unsigned i = t.base + (unsigned)j * jstride;
    if (t.two)
      ptr[i >> 1] = make_float4(v.re.x, v.im.x, v.re.y, v.im.y);
    else
      reinterpret_cast<float2*>(ptr)[i] = make_float2(v.re.x, v.im.x);
  }
};

// rows p and p+1 of a complex array (element k of row p at p*rowstride + k)
struct P2RowLoad {
  const float2* ptr;
  unsigned rowstride;
  unsigned n;
  int Lin;  // valid elements per row
  int np;
  __device__ __forceinline__ float2 one(int p, int k, unsigned& bad) const {
    const unsigned i = (unsigned)p * rowstride + (unsigned)k;
    const bool want = p < np && k < Lin;
    const bool ok = want && i < n;
    bad |= (unsigned)(want && !ok);
    return ok ? ptr[i] : make_float2(0.f, 0.f);
  }
};

// ---------------------------------------------------------------------------
// Generation pass 1: counter-based (or buffered) noise x sqrt(lambda) on the R2C half
// spectrum, backward transform along the last axis, pruned store (R2CNoise semantics,
// r2cfieldbackend.hh:305-325 fed by matrix.hh:375-404).  Pencils are k0 (fastest) per
// outer block k1 (3D); one Philox call per pencil serves elements j and j + L/2.
// ---------------------------------------------------------------------------
struct PhiloxKeys {
  uint32_t kx[10], ky[10];
};

__device__ __forceinline__ uint4 philox_rk(uint4 c, const PhiloxKeys& k) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ k.kx[r], (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k.ky[r],
                   (uint32_t)p0);
  }
  return c;
}

// Box-Muller (u1 = (a + 1/2) 2^-32 in (0, 1], u2 from the top 24 bits of b), fast
// intrinsics; the radius uses x * rsqrt(x) with x clamped away from 0
__device__ __forceinline__ float2 box_muller_fast(uint32_t a, uint32_t b) {
  const float u1 = fmaf(__uint2float_rn(a), 2.3283064365386963e-10f, 1.1641532182693481e-10f);
  const float x = fmaxf(-1.3862943611198906f * __log2f(u1), 1e-30f);  // -2 ln u1
  const float rad = x * rsqrtf(x);
  const float u2 = __uint_as_float(0x3f800000u | (b >> 9)) - 1.0f;  // [0, 1)
  float s, c;
  __sincosf(fmaf(6.283185307179586f, u2, -3.141592653589793f), &s, &c);
  return make_float2(rad * c, rad * s);
}

// MUFU approximations without the denormal-input handling of the intrinsics; every
// argument below is a normal number (u1 >= 2^-33, x >= 1e-30, |angle| <= pi and not tiny
// unless zero), so the results equal __log2f / rsqrtf / __sinf / __cosf
__device__ __forceinline__ float lg2_ftz(float x) {
  float y;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ void sincos_ftz(float x, float* s, float* c) {
  asm("sin.approx.ftz.f32 %0, %1;" : "=f"(*s) : "f"(x));
  asm("cos.approx.ftz.f32 %0, %1;" : "=f"(*c) : "f"(x));
}

// Box-Muller for pencils A and B at once: (a, b) of pencil A and (c, d) of pencil B give
// the normal pairs (re, im) of both in the pair layout re = (Re A, Re B), im = (Im A, Im B);
// the same operations and rounding as box_muller_fast, the products issued as FMUL2/FFMA2
__device__ __forceinline__ P2 box_muller_pair(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  const float2 u1 = f2fma(make_float2(__uint2float_rn(a), __uint2float_rn(c)),
                          make_float2(2.3283064365386963e-10f, 2.3283064365386963e-10f),
                          make_float2(1.1641532182693481e-10f, 1.1641532182693481e-10f));
  const float2 x2 = f2mul(make_float2(lg2_ftz(u1.x), lg2_ftz(u1.y)),
                          make_float2(-1.3862943611198906f, -1.3862943611198906f));
  const float2 x = make_float2(fmaxf(x2.x, 1e-30f), fmaxf(x2.y, 1e-30f));
  const float2 rad = f2mul(x, make_float2(rsqrt_ftz(x.x), rsqrt_ftz(x.y)));
  const float2 u2 = f2add(make_float2(__uint_as_float(0x3f800000u | (b >> 9)), __uint_as_float(0x3f800000u | (d >> 9))),
                          make_float2(-1.0f, -1.0f));
  const float2 ang = f2fma(make_float2(6.283185307179586f, 6.283185307179586f), u2,
                           make_float2(-3.141592653589793f, -3.141592653589793f));
  float sA, cA, sB, cB;
  sincos_ftz(ang.x, &sA, &cA);
  sincos_ftz(ang.y, &sB, &cB);
  return {f2mul(rad, make_float2(cA, cB)), f2mul(rad, make_float2(sA, sB))};
}

// The seeded noise of the R2C field backend written out in the reference's draw order
// (rand1, rand2 per stored frequency): the same counters, Philox4x32-10 words and
// Box-Muller definitions as the generation passes (paired FP32 form for FP32 plans, the FP64
// form for FP64 plans), so that a host implementation fed these values reproduces a seeded
// realization.  One thread per stored frequency k (last-axis index kl < T/2 when the last
// extent is even: it also writes the partner kl + T/2 from the same counter).
struct NoiseExport {
  int dim, T0c, ext1, ext2, Tl;
  int transposed, fp64;
  uint64_t seed;
  uint32_t epoch;
  unsigned long long n;  // doubles in `out`
  __device__ __forceinline__ unsigned stored(int k0, int k1, int kl) const {
    if (dim == 2) return (unsigned)k0 + (unsigned)T0c * (unsigned)kl;
    if (transposed) return (unsigned)k0 + (unsigned)T0c * ((unsigned)kl + (unsigned)ext2 * (unsigned)k1);
    return (unsigned)k0 + (unsigned)T0c * ((unsigned)k1 + (unsigned)ext1 * (unsigned)kl);
  }
};

__global__ void k_export_noise(NoiseExport e, double* __restrict__ out) {
  const bool paired = e.Tl % 2 == 0;
  const int kls = paired ? e.Tl / 2 : e.Tl;
  const int n1 = e.dim == 3 ? e.ext1 : 1;
  const long long total = (long long)e.T0c * n1 * kls;
  const uint2 key = make_uint2((uint32_t)e.seed, (uint32_t)(e.seed >> 32));
  unsigned bad = 0;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int k0 = (int)(t % e.T0c);
    const long long rest = t / e.T0c;
    const int k1 = (int)(rest % n1);
    const int kl = (int)(rest / n1);
    const unsigned s0 = e.stored(k0, k1, kl);
    const uint4 c = philox4x32_10(pair_counter(s0, e.epoch), key);
    double r[4];
    if (e.fp64) {
      box_muller(c.x, c.y, r[0], r[1]);
      box_muller(c.z, c.w, r[2], r[3]);
    } else {
      const float2 a = box_muller_fast(c.x, c.y), b = box_muller_fast(c.z, c.w);
      r[0] = a.x;
      r[1] = a.y;
      r[2] = b.x;
      r[3] = b.y;
    }
    const unsigned long long i0 = 2ull * s0;
    if (i0 + 1 < e.n) {
      out[i0] = r[0];
      out[i0 + 1] = r[1];
    } else {
      bad = 1;
    }
    if (paired) {
      const unsigned long long i1 = 2ull * e.stored(k0, k1, kl + kls);
      if (i1 + 1 < e.n) {
        out[i1] = r[2];
        out[i1 + 1] = r[3];
      } else {
        bad = 1;
      }
    }
  }
  if (bad) atomicOr(&g_bounds_error, 1u);
}

template <int DIM, int LAYOUT, bool TRANSP>
struct P2Noise {
  // LAYOUT: 1 = DCT prod(T/2+1) eigenvalues (mirrored lookup), 0 = R2C half spectrum,
  // 2 = full DFT spectrum (dftmatrixbackend.hh:303-307)
  int ext0, ext1, ext2;
  int T0c, D0, D1;
  const float* sq;
  const double* noise;
  unsigned nsq, nnoise;
  int np;
  const unsigned* epoch;  // device word mixed into the counters (null: 0)
  PhiloxKeys keys;
  __device__ __forceinline__ unsigned stored(int k0, int k1, int kl) const {
    if (DIM == 2) return (unsigned)k0 + (unsigned)T0c * (unsigned)kl;
    if (TRANSP) return (unsigned)k0 + (unsigned)T0c * ((unsigned)kl + (unsigned)ext2 * (unsigned)k1);
    return (unsigned)k0 + (unsigned)T0c * ((unsigned)k1 + (unsigned)ext1 * (unsigned)kl);
  }
  __device__ __forceinline__ unsigned lam_index(int k0, int k1, int kl) const {
    const int a1 = DIM == 3 ? k1 : kl, a2 = DIM == 3 ? kl : 0;
    if (LAYOUT == 1) {
      const int m1 = a1 <= ext1 / 2 ? a1 : ext1 - a1;
      const int m2 = DIM == 3 ? (a2 <= ext2 / 2 ? a2 : ext2 - a2) : 0;
      return (unsigned)k0 + (unsigned)D0 * ((unsigned)m1 + (unsigned)D1 * (unsigned)m2);
    }
    if (LAYOUT == 2) return (unsigned)k0 + (unsigned)ext0 * ((unsigned)a1 + (unsigned)ext1 * (unsigned)a2);
    return (unsigned)k0 + (unsigned)T0c * ((unsigned)a1 + (unsigned)ext1 * (unsigned)a2);
  }
  // (lambda A, lambda B) and the self-conjugate rule for both pencils at last-axis kl
  __device__ __forceinline__ P2 scale(int k0, int k1, int kl, float2 rA, float2 rB, unsigned& bad) const {
    const unsigned li = lam_index(k0, k1, kl);
    const bool vb = k0 + 1 < np;
    const bool okA = li < nsq, okB = !vb || li + 1 < nsq;
    bad |= (unsigned)(!okA || !okB);
    const float lA = okA ? sq[li] : 0.f;
    const float lB = (vb && okB) ? sq[li + 1] : 0.f;
    const int a1 = DIM == 3 ? k1 : kl, a2 = DIM == 3 ? kl : 0;
    const bool sc12 = (a1 == 0 || 2 * a1 == ext1) && (DIM < 3 || a2 == 0 || 2 * a2 == ext2);
    const bool scA = sc12 && (k0 == 0 || 2 * k0 == ext0);
    const bool scB = sc12 && (2 * (k0 + 1) == ext0);
    const float h = 0.70710678118654752f;
    const float sA = scA ? lA : lA * h, sB = scB ? lB : lB * h;
    P2 o;
    o.re = f2mul(make_float2(sA, sB), make_float2(rA.x, rB.x));
    o.im = make_float2(scA ? 0.f : sA * rA.y, scB ? 0.f : sB * rB.y);
    return o;
  }
  // Per-tile part of the counter-noise lookups (the pass axis is the last torus axis, so its
  // length is the transform length L): for elements j < L/2 and j + L/2 of pencils
  // (k0, k0+1) at outer index k1, the stored index is si0 + sstride * kl, the eigenvalue
  // index li0 + lstride * m(kl) with m(kl) = kl, or min(kl, L - kl) for the DCT layout, and
  // the self-conjugate rule reduces to (row part) && j == 0.  One bounds check covers the
  // tile.
  struct Tile {
    unsigned si0, sstride, li0, lstride, ep;
    bool vb, ok, scA, scB;
  };
  template <int L>
  __device__ __forceinline__ Tile tile(int p, int o, unsigned& bad) const {
    Tile t;
    const int k0 = p, k1 = DIM == 3 ? o : 0;
    if (DIM == 2) {
      t.si0 = (unsigned)k0;
      t.sstride = (unsigned)T0c;
    } else if (TRANSP) {
      t.si0 = (unsigned)k0 + (unsigned)T0c * (unsigned)ext2 * (unsigned)k1;
      t.sstride = (unsigned)T0c;
    } else {
      t.si0 = (unsigned)k0 + (unsigned)T0c * (unsigned)k1;
      t.sstride = (unsigned)T0c * (unsigned)ext1;
    }
    if (LAYOUT == 1) {
      const int m1 = k1 <= ext1 / 2 ? k1 : ext1 - k1;
      t.li0 = (unsigned)k0 + (DIM == 3 ? (unsigned)D0 * (unsigned)m1 : 0u);
      t.lstride = DIM == 3 ? (unsigned)D0 * (unsigned)D1 : (unsigned)D0;
    } else if (LAYOUT == 2) {
      t.li0 = (unsigned)k0 + (DIM == 3 ? (unsigned)ext0 * (unsigned)k1 : 0u);
      t.lstride = DIM == 3 ? (unsigned)ext0 * (unsigned)ext1 : (unsigned)ext0;
    } else {
      t.li0 = (unsigned)k0 + (DIM == 3 ? (unsigned)T0c * (unsigned)k1 : 0u);
      t.lstride = DIM == 3 ? (unsigned)T0c * (unsigned)ext1 : (unsigned)T0c;
    }
    t.vb = k0 + 1 < np;
    const unsigned mmax = LAYOUT == 1 ? (unsigned)(L / 2) : (unsigned)(L - 1);
    const unsigned long long top = (unsigned long long)t.li0 + (unsigned long long)t.lstride * mmax + (t.vb ? 1u : 0u);
    t.ok = p < np && top < (unsigned long long)nsq;
    bad |= (unsigned)(p < np && !t.ok);
    const bool sc1 = DIM < 3 || k1 == 0 || 2 * k1 == ext1;
    t.scA = sc1 && (k0 == 0 || 2 * k0 == ext0);
    t.scB = sc1 && 2 * (k0 + 1) == ext0;
    t.ep = epoch ? __ldg(epoch) : 0u;
    return t;
  }
  // normals z (pair layout) times (lambda A, lambda B) of eigenvalue index li, with the
  // self-conjugate rule (factor 1 and zero imaginary part) at the rows' first element
  __device__ __forceinline__ P2 scale_t(const Tile& t, unsigned li, bool first, const P2& z) const {
    const float lA = sq[li];
    const float lB = t.vb ? sq[li + 1] : 0.f;
    const bool scA = t.scA && first, scB = t.scB && first;
    const float h = 0.70710678118654752f;
    const float2 s = f2mul(make_float2(lA, lB), make_float2(scA ? 1.f : h, scB ? 1.f : h));
    P2 o;
    o.re = f2mul(s, z.re);
    o.im = f2mul(s, z.im);
    if (scA) o.im.x = 0.f;
    if (scB) o.im.y = 0.f;
    return o;
  }
  // counter noise of elements j < L/2 and j + L/2 of the tile's pencil pair
  template <int L>
  __device__ __forceinline__ void load2t(const Tile& t, int j, P2& x0, P2& x1) const {
    if (!t.ok) {
      x0 = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      x1 = x0;
      return;
    }
    constexpr int h = L / 2;
    const unsigned si = t.si0 + t.sstride * (unsigned)j;
    const uint4 cA = philox_rk(make_uint4(si, 0u, 0x70616972u, t.ep), keys);
    const uint4 cB = philox_rk(make_uint4(si + 1u, 0u, 0x70616972u, t.ep), keys);
    const P2 z0 = box_muller_pair(cA.x, cA.y, cB.x, cB.y), z1 = box_muller_pair(cA.z, cA.w, cB.z, cB.w);
    const unsigned m1 = LAYOUT == 1 ? (unsigned)(h - j) : (unsigned)(j + h);
    x0 = scale_t(t, t.li0 + t.lstride * (unsigned)j, j == 0, z0);
    x1 = scale_t(t, t.li0 + t.lstride * m1, j == 0, z1);
  }
  // elements j and j + L/2 of pencils (p, p+1); pencil = k0, outer = k1
  template <int L>
  __device__ __forceinline__ void load2(int p, int j, int o, P2& x0, P2& x1, unsigned& bad) const {
    const int k0 = p, k1 = DIM == 3 ? o : 0;
    constexpr int h = L / 2;
    if (p >= np) {  // pair beyond the last pencil: zero input, no lookups
      x0 = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      x1 = x0;
      return;
    }
    float2 a0, a1, b0, b1;  // normals: pencil A at j, j+h; pencil B at j, j+h
    if (noise) {
      const unsigned s0 = stored(k0, k1, j), s1 = stored(k0, k1, j + h);
      const bool vb = k0 + 1 < np;
      const unsigned top = vb ? 2u * s0 + 3u : 2u * s0 + 1u, top1 = vb ? 2u * s1 + 3u : 2u * s1 + 1u;
      const bool ok = top < nnoise && top1 < nnoise;
      bad |= (unsigned)!ok;
      double2 n00 = make_double2(0, 0), n01 = n00, n10 = n00, n11 = n00;
      if (ok) {
        const double2* nz2 = reinterpret_cast<const double2*>(noise);
        n00 = nz2[s0];
        n10 = nz2[s1];
        if (vb) {
          n01 = nz2[s0 + 1];
          n11 = nz2[s1 + 1];
        }
      }
      a0 = make_float2((float)n00.x, (float)n00.y);
      a1 = make_float2((float)n10.x, (float)n10.y);
      b0 = make_float2((float)n01.x, (float)n01.y);
      b1 = make_float2((float)n11.x, (float)n11.y);
    } else {
      const unsigned si = stored(k0, k1, j);
      const unsigned ep = epoch ? __ldg(epoch) : 0u;
      const uint4 cA = philox_rk(make_uint4(si, 0u, 0x70616972u, ep), keys);
      const uint4 cB = philox_rk(make_uint4(si + 1u, 0u, 0x70616972u, ep), keys);
      a0 = box_muller_fast(cA.x, cA.y);
      a1 = box_muller_fast(cA.z, cA.w);
      b0 = box_muller_fast(cB.x, cB.y);
      b1 = box_muller_fast(cB.z, cB.w);
    }
    x0 = scale(k0, k1, j, a0, b0, bad);
    x1 = scale(k0, k1, j + h, a1, b1, bad);
  }
};

// Tile order of the persistent passes.  With a counter (zeroed in the stream before the
// launch) every CTA takes its next tile index from it, so CTAs on SMs that run faster take
// more tiles and the launch ends when the work does (the noise pass alone: 0.263 against 0.284
// ms with the static order on the 256^3 workload).  Thread 0 fetches the index of the next
// tile while the current one is transformed; the other threads read it after the barrier at
// the end of the tile (every tile body passes barriers after the previous read of *s).
// Without a counter the CTAs stride over the tiles by the grid size.
__device__ __forceinline__ long long tile_first(unsigned long long* ctr, long long* s) {
  if (!ctr) return blockIdx.x;
  if (threadIdx.x == 0) *s = (long long)atomicAdd(ctr, 1ull);
  __syncthreads();
  return *s;
}
__device__ __forceinline__ unsigned long long tile_prefetch(unsigned long long* ctr) {
  return (ctr && threadIdx.x == 0) ? atomicAdd(ctr, 1ull) : 0ull;
}
__device__ __forceinline__ long long tile_next(unsigned long long* ctr, long long* s, long long tile,
                                               unsigned long long nxt) {
  if (!ctr) return tile + gridDim.x;
  if (threadIdx.x == 0) *s = (long long)nxt;
  __syncthreads();
  return *s;
}

template <int L, class Ld>
__global__ void __launch_bounds__(kP2Threads, PF_P2_MIN_NOISE)
    kp2_noise(const float4* __restrict__ twg, long long ntiles, int tpo, int Lout, Ld ld, P2ArrStore st,
              unsigned long long* ctr) {
  __shared__ long long s_tile;
  using G = P2Geom<L>;
  extern __shared__ __align__(16) float4 p2_smem[];
  float4* buf = p2_smem;
  float4* tw = p2_smem + G::Q * G::PLQ;
  p2_copy_table(tw, twg, G::NTW);
  __syncthreads();
  const int q = threadIdx.x % G::Q, u = threadIdx.x / G::Q;
  unsigned bad = 0;
  for (long long tile = tile_first(ctr, &s_tile); tile < ntiles;) {
    const unsigned long long nxt = tile_prefetch(ctr);
    const int o = (int)(tile / tpo);
    const int p = (int)(tile - (long long)o * tpo) * G::NP + 2 * q;
    P2 v[8];
    if (ld.noise) {  // noise buffer in the reference's draw order
#pragma unroll
      for (int r = 0; r < 4; r++) ld.template load2<L>(p, u + r * G::TP, o, v[r], v[r + 4], bad);
    } else {  // counter-based noise: index arithmetic and bounds check once per tile
      const auto t = ld.template tile<L>(p, o, bad);
#pragma unroll
      for (int r = 0; r < 4; r++) ld.template load2t<L>(t, u + r * G::TP, v[r], v[r + 4]);
    }
    const P2ArrStore::Tile so = st.tile(p, o, Lout, bad);
    p2_transform<L, +1>(v, buf, tw, u, q, [&](int j, const P2& x) {
      if (j < Lout) st.store_t(so, j, x);
    });
    tile = tile_next(ctr, &s_tile, tile, nxt);
  }
  p2_report(bad);
}

// ---------------------------------------------------------------------------
// Generation pass 1 for last-axis lengths L = 3 M (M a power of two, 64..512): the
// length-L backward transform split as
//   X[3 k1 + k2] = sum_n1 W_M^(n1 k1) [ W_L^(n1 k2) sum_n2 x[n1 + M n2] W_3^(n2 k2) ],
// i.e. a radix-3 step with twiddles, then three paired M-point transforms per pencil
// pair (one per k2).  A tile holds PP pencil pairs: their noise is first generated into
// shared memory (the exchange buffer, PP L slots), then every thread reads the three inputs
// of its radix-3 butterflies, and thread slot q transforms sub-pencil k2 = q % 3 of pair
// q / 3.  The block has exactly 3 PP M/8 threads.
// ---------------------------------------------------------------------------
template <int M>
struct P2Geom3 {
  using G = P2Geom<M>;
  static constexpr int L = 3 * M;
  static constexpr int PP = kP2Threads / (3 * G::TP);  // pencil pairs per tile
  static constexpr int NT = PP * 3 * G::TP;            // threads per CTA
  static constexpr int QS = 3 * PP;                    // sub-pencil slots
  static_assert(PP >= 1 && QS <= G::Q, "sub-pencil slots fit the exchange buffer");
  static_assert(PP * L <= G::Q * G::PLQ, "the tile's noise fits the exchange buffer");
};

// Radix-3 step and M-point transforms of a tile staged in the exchange buffer (pair g's
// element n at buf[g L + n]): thread slot q transforms sub-pencil k2 = q % 3 of pair q / 3;
// Out(j, value) receives output j = 3 k1 + k2.  Sign S of the transform (W = exp(S 2 pi i / .)).
// output k2 of the radix-3 butterfly of (a, b, c) (elements n1, n1 + M, n1 + 2M), times the
// twiddle w = W_L^(n1 k2) (unused for k2 = 0)
template <int S>
__device__ __forceinline__ P2 p2_radix3_point(const P2& a, const P2& b, const P2& c, int k2, float4 w) {
  const P2 sm = padd(b, c);
  if (k2 == 0) return padd(a, sm);
  // W_3^(k2) = -1/2 + i S sin(2 pi k2 / 3): + sqrt(3)/2 for (S, k2) = (+, 1) and (-, 2)
  const float sq3 = (k2 == 1) == (S > 0) ? 0.86602540378443865f : -0.86602540378443865f;
  const float2 hf = make_float2(-0.5f, -0.5f), s3 = make_float2(sq3, sq3), ns3 = make_float2(-sq3, -sq3);
  const P2 df = psub(b, c);
  // a - (b + c) / 2 + i s3 (b - c)
  const P2 y = {f2fma(hf, sm.re, f2fma(ns3, df.im, a.re)), f2fma(hf, sm.im, f2fma(s3, df.re, a.im))};
  return ptw(y, w);
}

template <int M, int S, class Out>
__device__ __forceinline__ void p2_radix3_transform(float4* buf, const float4* tw, const float4* tw3, int u, int q,
                                                    const Out& out) {
  using G = P2Geom<M>;
  constexpr int L = 3 * M;
  const int pq = q / 3, k2 = q - 3 * (q / 3);
  P2 v[8];
  const float4* xs = buf + pq * L;
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const int n1 = u + r * G::TP;
    v[r] = p2_radix3_point<S>(p2_of(xs[n1]), p2_of(xs[n1 + M]), p2_of(xs[n1 + 2 * M]), k2,
                              k2 ? tw3[(k2 - 1) * M + n1] : make_float4(1.f, 1.f, 0.f, 0.f));
  }
  __syncthreads();  // every thread has read the staged tile before the transform writes the buffer
  p2_transform<M, S>(v, buf, tw, u, q, [&](int k1, const P2& x) { out(3 * k1 + k2, x); });
}

template <int M, class Ld>
__global__ void __launch_bounds__(kP2Threads, PF_P2_MIN_NOISE)
    kp2_noise3(const float4* __restrict__ twg, long long ntiles, int tpo, int Lout, Ld ld, P2ArrStore st,
               unsigned long long* ctr) {
  __shared__ long long s_tile;
  using G = P2Geom<M>;
  using G3 = P2Geom3<M>;
  constexpr int L = G3::L;
  extern __shared__ __align__(16) float4 p2_smem[];
  float4* buf = p2_smem;  // exchange buffer; also the tile's noise, pair g at buf[g L + n]
  float4* tw = p2_smem + G::Q * G::PLQ;
  const float4* tw3 = tw + G::NTW;  // exp(+2 pi i n1 k2 / L) at (k2 - 1) M + n1, k2 = 1, 2
  p2_copy_table(tw, twg, G::NTW + 2 * M);
  __syncthreads();
  const int tid = threadIdx.x;
  const int q = tid % G3::QS, u = tid / G3::QS;  // transform: sub-pencil slot, column
  const int pq = q / 3;
  const int gp = tid / (3 * G::TP), gi = tid - gp * (3 * G::TP);  // generation: pair, index
  unsigned bad = 0;
  for (long long tile = tile_first(ctr, &s_tile); tile < ntiles;) {
    const unsigned long long nxt = tile_prefetch(ctr);
    const int o = (int)(tile / tpo);
    const int p0 = (int)(tile - (long long)o * tpo) * (2 * G3::PP);
    {  // noise x[n] of pair gp, elements j and j + L/2 per call
      const int p = p0 + 2 * gp;
      float4* xs = buf + gp * L;
      if (ld.noise) {
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const int j = gi + r * (3 * G::TP);
          P2 x0, x1;
          ld.template load2<L>(p, j, o, x0, x1, bad);
          xs[j] = slot_of(x0);
          xs[j + L / 2] = slot_of(x1);
        }
      } else {
        const auto t = ld.template tile<L>(p, o, bad);
#pragma unroll
        for (int r = 0; r < 4; r++) {
          const int j = gi + r * (3 * G::TP);
          P2 x0, x1;
          ld.template load2t<L>(t, j, x0, x1);
          xs[j] = slot_of(x0);
          xs[j + L / 2] = slot_of(x1);
        }
      }
    }
    __syncthreads();
    const P2ArrStore::Tile so = st.tile(p0 + 2 * pq, o, Lout, bad);
    p2_radix3_transform<M, +1>(buf, tw, tw3, u, q, [&](int j, const P2& x) {
      if (j < Lout) st.store_t(so, j, x);
    });
    tile = tile_next(ctr, &s_tile, tile, nxt);
  }
  p2_report(bad);
}

// Strided complex pass of length L = 3 M (pencils p, p+1 adjacent): every thread loads the
// three inputs of its radix-3 butterflies itself, then the paired M-point transforms run as
// in kp2_noise3.
template <int M, int S>
__global__ void __launch_bounds__(kP2Threads, PF_P2_MIN_C2C)
    kp2_c2c3(const float4* __restrict__ twg, long long ntiles, int tpo, int Lout, P2ArrLoad ld, P2ArrStore st,
             unsigned long long* ctr) {
  __shared__ long long s_tile;
  using G = P2Geom<M>;
  using G3 = P2Geom3<M>;
  extern __shared__ __align__(16) float4 p2_smem[];
  float4* buf = p2_smem;
  float4* tw = p2_smem + G::Q * G::PLQ;
  const float4* tw3 = tw + G::NTW;
  p2_copy_table(tw, twg, G::NTW + 2 * M);
  __syncthreads();
  const int tid = threadIdx.x;
  const int q = tid % G3::QS, u = tid / G3::QS;
  const int pq = q / 3, k2 = q - 3 * (q / 3);
  unsigned bad = 0;
  for (long long tile = tile_first(ctr, &s_tile); tile < ntiles;) {
    const unsigned long long nxt = tile_prefetch(ctr);
    const int o = (int)(tile / tpo);
    const int p0 = (int)(tile - (long long)o * tpo) * (2 * G3::PP);
    // the three inputs of each radix-3 butterfly straight from global memory (the three
    // threads of a pencil pair that share them read the same addresses, served by L1)
    const P2ArrLoad::Tile lt = ld.tile(p0 + 2 * pq, o, bad);
    P2 v[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int n1 = u + r * G::TP;
      v[r] = p2_radix3_point<S>(ld.load_t(lt, n1), ld.load_t(lt, n1 + M), ld.load_t(lt, n1 + 2 * M), k2,
                                k2 ? tw3[(k2 - 1) * M + n1] : make_float4(1.f, 1.f, 0.f, 0.f));
    }
    const P2ArrStore::Tile so = st.tile(p0 + 2 * pq, o, Lout, bad);
    p2_transform<M, S>(v, buf, tw, u, q, [&](int k1, const P2& x) {
      const int j = 3 * k1 + k2;
      if (j < Lout) st.store_t(so, j, x);
    });
    tile = tile_next(ctr, &s_tile, tile, nxt);
  }
  p2_report(bad);
}

// ---------------------------------------------------------------------------
// Strided complex pass (pencils p, p+1 adjacent), e.g. the middle generation pass.
// ---------------------------------------------------------------------------
template <int L, int S>
__global__ void __launch_bounds__(kP2Threads, PF_P2_MIN_C2C)
    kp2_c2c(const float4* __restrict__ twg, long long ntiles, int tpo, int Lout, P2ArrLoad ld, P2ArrStore st,
            unsigned long long* ctr) {
  __shared__ long long s_tile;
  using G = P2Geom<L>;
  extern __shared__ __align__(16) float4 p2_smem[];
  float4* buf = p2_smem;
  float4* tw = p2_smem + G::Q * G::PLQ;
  p2_copy_table(tw, twg, G::NTW);
  __syncthreads();
  const int q = threadIdx.x % G::Q, u = threadIdx.x / G::Q;
  unsigned bad = 0;
  for (long long tile = tile_first(ctr, &s_tile); tile < ntiles;) {
    const unsigned long long nxt = tile_prefetch(ctr);
    const int o = (int)(tile / tpo);
    const int p = (int)(tile - (long long)o * tpo) * G::NP + 2 * q;
    P2 v[8];
    const P2ArrLoad::Tile lt = ld.tile(p, o, bad);
#pragma unroll
    for (int r = 0; r < 8; r++) v[r] = ld.load_t(lt, u + r * G::TP);
    const P2ArrStore::Tile so = st.tile(p, o, Lout, bad);
    p2_transform<L, S>(v, buf, tw, u, q, [&](int j, const P2& x) {
      if (j < Lout) st.store_t(so, j, x);
    });
    tile = tile_next(ctr, &s_tile, tile, nxt);
  }
  p2_report(bad);
}

// ---------------------------------------------------------------------------
// Strided complex pass with its tiles staged by the tensor memory accelerator.  A tile
// (NP adjacent pencils x L rows, 32 KB for every L) is one or more 2D bulk tensor copies
// from HBM into shared memory (cp.async.bulk.tensor, completion counted on an mbarrier);
// two tile buffers alternate over the persistent loop, so the copy of the CTA's next tile
// runs while the current one is transformed.  No register or LSU work moves the inputs;
// the transform and the stores are those of kp2_c2c.  Columns beyond the last pencil and
// rows beyond the array read as zero (TMA out-of-bounds fill), rows j >= Lin of a tile are
// zeroed on the shared-memory read.  Every mbarrier wait is bounded: a wait that gives up
// sets bit 2 of the error word and the CTA leaves the loop (all threads together).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
constexpr uint32_t kTmaWaitLimit = 1u << 22;  // try_wait rounds before a wait gives up
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < kTmaWaitLimit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
// 2D tile copy global -> shared (no multicast), completion on `bar`
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

template <int L>
struct P2Tma {
  static constexpr int BOXR = L < 256 ? L : 256;              // rows per copy (box limit 256)
  static constexpr unsigned TILE_BYTES = (unsigned)L * P2Geom<L>::NP * 8u;  // 32 KB
  static constexpr size_t smem_bytes() {
    return 2 * (size_t)TILE_BYTES + (size_t)(P2Geom<L>::Q * P2Geom<L>::PLQ + P2Geom<L>::NTW) * 16 + 2 * 8;
  }
};

template <int L, int S>
__global__ void __launch_bounds__(kP2Threads, 2)
    kp2_c2c_tma(const __grid_constant__ CUtensorMap src, const float4* __restrict__ twg, long long ntiles, int tpo,
                int rows_per_outer, int Lin, int Lout, P2ArrStore st) {
  using G = P2Geom<L>;
  using M = P2Tma<L>;
  extern __shared__ __align__(128) float4 p2_tma_smem[];
  float4* tb0 = p2_tma_smem;
  float4* tb1 = p2_tma_smem + M::TILE_BYTES / 16;
  float4* buf = p2_tma_smem + 2 * (M::TILE_BYTES / 16);
  float4* tw = buf + G::Q * G::PLQ;
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + G::NTW);
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  p2_copy_table(tw, twg, G::NTW);
  __syncthreads();
  const int q = tid % G::Q, u = tid / G::Q;
  unsigned bad = 0;
  auto issue = [&](long long t, int slot) {
    const int o = (int)(t / tpo);
    const int p0 = (int)(t - (long long)o * tpo) * G::NP;
    float4* dst = slot ? tb1 : tb0;
    fence_proxy_async();  // the buffer's previous contents were read through the generic proxy
    mbar_expect_tx(&bar[slot], M::TILE_BYTES);
#pragma unroll
    for (int c = 0; c < L / M::BOXR; c++)
      tma_load_2d(dst + c * (M::BOXR * G::NP / 2), &src, &bar[slot], p0, o * rows_per_outer + c * M::BOXR);
  };
  long long tile = blockIdx.x;
  if (tid == 0 && tile < ntiles) issue(tile, 0);
  int k = 0;
  bool pending_next = false;
  for (; tile < ntiles; tile += gridDim.x, k++) {
    const int slot = k & 1;
    const long long next = tile + gridDim.x;
    pending_next = next < ntiles;
    // the other buffer was last read before a barrier of the previous tile's transform
    if (tid == 0 && pending_next) issue(next, slot ^ 1);
    const bool ok = mbar_wait_bounded(&bar[slot], (uint32_t)(k >> 1) & 1u);
    if (!__syncthreads_and(ok)) {
      bad |= 2u;
      break;
    }
    pending_next = false;
    const int o = (int)(tile / tpo);
    const int p = (int)(tile - (long long)o * tpo) * G::NP + 2 * q;
    const float4* t4 = slot ? tb1 : tb0;
    P2 v[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int j = u + r * G::TP;
      const float4 sv = j < Lin ? t4[j * (G::NP / 2) + q] : make_float4(0.f, 0.f, 0.f, 0.f);
      v[r] = {make_float2(sv.x, sv.z), make_float2(sv.y, sv.w)};
    }
    const P2ArrStore::Tile so = st.tile(p, o, Lout, bad);
    p2_transform<L, S>(v, buf, tw, u, q, [&](int j, const P2& x) {
      if (j < Lout) st.store_t(so, j, x);
    });
  }
  if ((bad & 2u) && tid == 0 && pending_next)  // a copy issued before the failed wait: bounded wait for it
    mbar_wait_bounded(&bar[(k & 1) ^ 1], (uint32_t)((k + 1) >> 1) & 1u);
  p2_report(bad);
}

// ---------------------------------------------------------------------------
// Fused strided pass of the matvec: forward transform, a per-element operator (Mid, e.g.
// the eigenvalue factor) and the backward transform of the same pencils, the spectrum
// staying in shared memory between the two (tables of both directions in shared memory).
// ---------------------------------------------------------------------------
template <int L, class Mid>
__global__ void __launch_bounds__(kP2Threads, PF_P2_MIN_MID)
    kp2_c2c_mid(const float4* __restrict__ twf, const float4* __restrict__ twb, long long ntiles, int tpo,
                int Lout, P2ArrLoad ld, Mid mid, P2ArrStore st, unsigned long long* ctr) {
  __shared__ long long s_tile;
  using G = P2Geom<L>;
  extern __shared__ __align__(16) float4 p2_smem[];
  float4* buf = p2_smem;
  float4* tf = p2_smem + G::Q * G::PLQ;
  float4* tb = tf + G::NTW;
  p2_copy_table(tf, twf, G::NTW);
  p2_copy_table(tb, twb, G::NTW);
  __syncthreads();
  const int q = threadIdx.x % G::Q, u = threadIdx.x / G::Q;
  unsigned bad = 0;
  for (long long tile = tile_first(ctr, &s_tile); tile < ntiles;) {
    const unsigned long long nxt = tile_prefetch(ctr);
    const int o = (int)(tile / tpo);
    const int p = (int)(tile - (long long)o * tpo) * G::NP + 2 * q;
    P2 v[8];
    const P2ArrLoad::Tile lt = ld.tile(p, o, bad);
#pragma unroll
    for (int r = 0; r < 8; r++) v[r] = ld.load_t(lt, u + r * G::TP);
    // forward transform; its outputs land in the exchange buffer (its last stage has read
    // the buffer and passed a barrier before the first output is written)
    p2_transform<L, -1>(v, buf, tf, u, q, [&](int j, const P2& x) { buf[p2_slot(G::PLQ, q, j)] = slot_of(x); });
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int j = u + r * G::TP;
      const P2 x = p2_of(buf[p2_slot(G::PLQ, q, j)]);
      cx<float> a = mk<float>(0.f, 0.f), b = a;  // pencils beyond the last one stay zero
      if (p < ld.np) a = mid.template operator()<float>(p, j, o, mk<float>(x.re.x, x.im.x));
      if (p + 1 < ld.np) b = mid.template operator()<float>(p + 1, j, o, mk<float>(x.re.y, x.im.y));
      v[r] = {make_float2(a.x, b.x), make_float2(a.y, b.y)};
    }
    __syncthreads();
    const P2ArrStore::Tile so = st.tile(p, o, Lout, bad);
    p2_transform<L, +1>(v, buf, tb, u, q, [&](int j, const P2& x) {
      if (j < Lout) st.store_t(so, j, x);
    });
    tile = tile_next(ctr, &s_tile, tile, nxt);
  }
  p2_report(bad);
}

// ---------------------------------------------------------------------------
// Complex-to-real rows (2L reals from L+1 complex, FFTW c2r semantics: Im of the DC
// and Nyquist inputs ignored), rows p and p+1 per pair, threads along the row.
// Store(p, m, x0, x1) receives reals 2m and 2m+1 of row p.
// ---------------------------------------------------------------------------
template <int L, class St>
__global__ void __launch_bounds__(kP2Threads, PF_P2_MIN_C2R)
    kp2_c2r(const float4* __restrict__ twg, long long ntiles, int Lout, P2RowLoad ld, St st) {
  using G = P2Geom<L>;
  extern __shared__ __align__(16) float4 p2_smem[];
  float4* buf = p2_smem;
  float4* tw = p2_smem + G::Q * G::PLQ;
  const float4* twT = tw + G::NTW;  // exp(+2 pi i m / 2L), m < L
  p2_copy_table(tw, twg, G::NTW + L);
  __syncthreads();
  const int u = threadIdx.x % G::TP, q = threadIdx.x / G::TP;
  unsigned bad = 0;
  [[maybe_unused]] double acc = 0.;  // St::kDot: this thread's share of the dot product
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int p = (int)tile * G::NP + 2 * q;
    P2 v[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int m = u + r * G::TP;
      float2 xa = ld.one(p, m, bad), xb = ld.one(p + 1, m, bad);
      float2 ya = ld.one(p, L - m, bad), yb = ld.one(p + 1, L - m, bad);
      if (m == 0) {
        xa.y = 0.f;
        xb.y = 0.f;
        ya.y = 0.f;
        yb.y = 0.f;
      }
      const P2 X = p2_ab(xa, xb), Y = p2_ab(ya, yb);
      // s = X + conj(Y), d = X - conj(Y), t = d w, Z = s + i t
      const P2 s = {f2add(X.re, Y.re), f2sub(X.im, Y.im)};
      const P2 d = {f2sub(X.re, Y.re), f2add(X.im, Y.im)};
      const P2 t = ptw(d, twT[m]);
      v[r] = {f2sub(s.re, t.im), f2add(s.im, t.re)};
    }
    p2_transform<L, +1>(v, buf, tw, u, q, [&](int m, const P2& z) {
      if (2 * m < Lout) {
        st.store(p, m, z, bad);
        if constexpr (St::kDot) acc += st.dot(p, m, z);
      }
    });
  }
  if constexpr (St::kDot) {  // a . out over the stored values, finished by the last block
    __shared__ double shd[32];
    acc = block_sum(acc, shd);
    if (cg_last_block(acc, st.part, st.cnt)) {
      const double t = cg_sum_partials(st.part, shd);
      if (threadIdx.x == 0) {
        *st.sdst = t;
        *st.cnt = 0u;
      }
    }
  }
  p2_report(bad);
}

// ---------------------------------------------------------------------------
// Complex-to-real rows with the rows staged by bulk copies.  A tile's NP rows are adjacent
// in memory (row stride `rowstride` complex, 16-byte multiple), so one cp.async.bulk per
// tile moves them into shared memory, completion counted on an mbarrier; two tile buffers
// alternate over the persistent loop, so the next tile's copy runs while the current one
// is transformed, and each input element is read from HBM once (the scalar kernel reads X[m]
// and X[L-m] as separate loads).  Rows beyond the last row read as zero; a copy whose rows
// would leave the buffer is not issued (bit 1 of the error word, zero rows).  Every wait is
// bounded: a wait that gives up sets bit 2 and the CTA leaves the loop (all threads together).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"((uint64_t)__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

template <int L>
struct P2Bulk {
  // shared memory of kp2_c2r_bulk for rows of `rowstride` complex
  static size_t smem_bytes(unsigned rowstride) {
    using G = P2Geom<L>;
    return 2 * (size_t)G::NP * rowstride * 8 + (size_t)(G::Q * G::PLQ + G::NTW + L) * 16 + 2 * 8;
  }
};

template <int L, class St>
__global__ void __launch_bounds__(kP2Threads, 2)
    kp2_c2r_bulk(const float4* __restrict__ twg, long long ntiles, int Lout, P2RowLoad ld, St st) {
  using G = P2Geom<L>;
  extern __shared__ __align__(128) float4 p2_bulk_smem[];
  const unsigned rs = ld.rowstride;
  const unsigned tile_f2 = (unsigned)G::NP * rs;  // complex per tile buffer (rs even: 16-byte multiple)
  float2* tb0 = reinterpret_cast<float2*>(p2_bulk_smem);
  float2* tb1 = tb0 + tile_f2;
  float4* buf = reinterpret_cast<float4*>(tb1 + tile_f2);
  float4* tw = buf + G::Q * G::PLQ;
  const float4* twT = tw + G::NTW;  // exp(+2 pi i m / 2L), m < L
  uint64_t* bar = reinterpret_cast<uint64_t*>(tw + G::NTW + L);
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  p2_copy_table(tw, twg, G::NTW + L);
  __syncthreads();
  const int u = tid % G::TP, q = tid / G::TP;
  unsigned bad = 0;
  auto issue = [&](long long t, int slot) {
    const long long p0 = t * G::NP;
    const long long nrows = ld.np - p0 < G::NP ? ld.np - p0 : G::NP;
    const unsigned long long top = (unsigned long long)(p0 + nrows) * rs;
    const bool ok = nrows > 0 && top <= (unsigned long long)ld.n;
    bad |= (unsigned)(nrows > 0 && !ok);
    const uint32_t bytes = ok ? (uint32_t)(nrows * rs * 8) : 0u;
    float2* dst = slot ? tb1 : tb0;
    fence_proxy_async();  // the buffer's previous contents were read through the generic proxy
    mbar_expect_tx(&bar[slot], bytes);
    if (bytes) bulk_load(dst, ld.ptr + (unsigned long long)p0 * rs, bytes, &bar[slot]);
  };
  long long tile = blockIdx.x;
  if (tid == 0 && tile < ntiles) issue(tile, 0);
  int k = 0;
  bool pending_next = false;
  for (; tile < ntiles; tile += gridDim.x, k++) {
    const int slot = k & 1;
    const long long next = tile + gridDim.x;
    pending_next = next < ntiles;
    // the other buffer was last read before a barrier of the previous tile's transform
    if (tid == 0 && pending_next) issue(next, slot ^ 1);
    const bool ok = mbar_wait_bounded(&bar[slot], (uint32_t)(k >> 1) & 1u);
    if (!__syncthreads_and(ok)) {
      bad |= 2u;
      break;
    }
    pending_next = false;
    const long long p0 = tile * G::NP;
    const int p = (int)p0 + 2 * q;
    const float2* ra = (slot ? tb1 : tb0) + (unsigned)(2 * q) * rs;
    const float2* rb = ra + rs;
    const bool va = p < ld.np, vb = p + 1 < ld.np;
    const float2 z2 = make_float2(0.f, 0.f);
    P2 v[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int m = u + r * G::TP;
      const bool im = m < ld.Lin, iy = L - m < ld.Lin;
      float2 xa = va && im ? ra[m] : z2, xb = vb && im ? rb[m] : z2;
      float2 ya = va && iy ? ra[L - m] : z2, yb = vb && iy ? rb[L - m] : z2;
      if (m == 0) {
        xa.y = 0.f;
        xb.y = 0.f;
        ya.y = 0.f;
        yb.y = 0.f;
      }
      const P2 X = p2_ab(xa, xb), Y = p2_ab(ya, yb);
      // s = X + conj(Y), d = X - conj(Y), t = d w, Z = s + i t
      const P2 s = {f2add(X.re, Y.re), f2sub(X.im, Y.im)};
      const P2 d = {f2sub(X.re, Y.re), f2add(X.im, Y.im)};
      const P2 t = ptw(d, twT[m]);
      v[r] = {f2sub(s.re, t.im), f2add(s.im, t.re)};
    }
    p2_transform<L, +1>(v, buf, tw, u, q, [&](int m, const P2& z) {
      if (2 * m < Lout) st.store(p, m, z, bad);
    });
  }
  if ((bad & 2u) && tid == 0 && pending_next)  // a copy issued before the failed wait: bounded wait for it
    mbar_wait_bounded(&bar[(k & 1) ^ 1], (uint32_t)((k + 1) >> 1) & 1u);
  p2_report(bad);
}

// Complex-to-real rows of length L = 3 M (2L reals from L+1 complex, FFTW c2r semantics as
// kp2_c2r): the rows' pre-processed values Z[m] = (X[m] + conj X[L-m]) + i w^m (X[m] -
// conj X[L-m]) of the tile's row pairs are staged in the exchange buffer, then the radix-3
// step and the paired M-point transforms run as in kp2_noise3; output j holds reals 2j, 2j+1.
template <int M, class St>
__global__ void __launch_bounds__(kP2Threads, PF_P2_MIN_C2R)
    kp2_c2r3(const float4* __restrict__ twg, long long ntiles, int Lout, P2RowLoad ld, St st) {
  using G = P2Geom<M>;
  using G3 = P2Geom3<M>;
  constexpr int L = G3::L;
  extern __shared__ __align__(16) float4 p2_smem[];
  float4* buf = p2_smem;
  float4* tw = p2_smem + G::Q * G::PLQ;
  const float4* tw3 = tw + G::NTW;          // radix-3 twiddles, 2M entries
  const float4* twT = tw3 + 2 * M;          // exp(+2 pi i m / 2L), m < L
  p2_copy_table(tw, twg, G::NTW + 2 * M + L);
  __syncthreads();
  const int tid = threadIdx.x;
  const int q = tid % G3::QS, u = tid / G3::QS;
  const int pq = q / 3;
  const int gp = tid / (3 * G::TP), gi = tid - gp * (3 * G::TP);
  unsigned bad = 0;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int p0 = (int)tile * (2 * G3::PP);
    {
      const int p = p0 + 2 * gp;
      float4* zs = buf + gp * L;
#pragma unroll
      for (int r = 0; r < 8; r++) {
        const int m = gi + r * (3 * G::TP);
        float2 xa = ld.one(p, m, bad), xb = ld.one(p + 1, m, bad);
        float2 ya = ld.one(p, L - m, bad), yb = ld.one(p + 1, L - m, bad);
        if (m == 0) {
          xa.y = 0.f;
          xb.y = 0.f;
          ya.y = 0.f;
          yb.y = 0.f;
        }
        const P2 X = p2_ab(xa, xb), Y = p2_ab(ya, yb);
        const P2 sv = {f2add(X.re, Y.re), f2sub(X.im, Y.im)};
        const P2 dv = {f2sub(X.re, Y.re), f2add(X.im, Y.im)};
        const P2 t = ptw(dv, twT[m]);
        zs[m] = slot_of(P2{f2sub(sv.re, t.im), f2add(sv.im, t.re)});
      }
    }
    __syncthreads();
    const int p = p0 + 2 * pq;
    p2_radix3_transform<M, +1>(buf, tw, tw3, u, q, [&](int j, const P2& z) {
      if (2 * j < Lout) st.store(p, j, z, bad);
    });
  }
  p2_report(bad);
}

// field rows of n0 reals (row p at p * n0) of type O (FP32 fields, or the FP64 vectors of
// the matvec and the CG), value transform applied in FP32
template <typename O>
struct P2FieldStoreT {
  using O2 = typename std::conditional<sizeof(O) == 8, double2, float2>::type;
  static constexpr bool kDot = false;
  O* out;
  int n0;
  int transform;
  float boxcox;
  unsigned n;
  int np;
  int Lout;
  int vec;  // out is aligned for pairs (8 bytes FP32, 16 bytes FP64) and n0 is even
  __device__ __forceinline__ void row(int p, int m, float a, float b, unsigned& bad) const {
    if (p >= np) return;
    if (transform) {
      a = apply_mutator<float>(transform, boxcox, a);
      b = apply_mutator<float>(transform, boxcox, b);
    }
    const unsigned i = (unsigned)p * (unsigned)n0 + 2u * (unsigned)m;
    const bool two = 2 * m + 1 < Lout;
    const bool ok = i + (two ? 1u : 0u) < n;
    bad |= (unsigned)!ok;
    if (!ok) return;
    if (two && vec) {
      O2 v;
      v.x = (O)a;
      v.y = (O)b;
      *reinterpret_cast<O2*>(out + i) = v;
    } else {
      out[i] = (O)a;
      if (two) out[i + 1] = (O)b;
    }
  }
  __device__ __forceinline__ void store(int p, int m, const P2& z, unsigned& bad) const {
    row(p, m, z.re.x, z.im.x, bad);
    row(p + 1, m, z.re.y, z.im.y, bad);
  }
};
using P2FieldStore = P2FieldStoreT<float>;

// FP64 rows of the matvec's output that also accumulate dv . out over the stored values
// (the CG's d . A d); kp2_c2r finishes the sum with the last-block reduction into *sdst.
// Every output element is stored exactly once, so every product enters once; the order of
// the sum is fixed by the kernel's static tile order.
struct P2FieldDotStore : P2FieldStoreT<double> {
  static constexpr bool kDot = true;
  const double* dv;
  double* part;   // one partial per CTA
  unsigned* cnt;  // ticket, 0 between kernels
  double* sdst;
  __device__ __forceinline__ double dot1(int p, int m, float a, float b) const {
    if (p >= np) return 0.;
    const unsigned i = (unsigned)p * (unsigned)n0 + 2u * (unsigned)m;
    const bool two = 2 * m + 1 < Lout;
    if (i + (two ? 1u : 0u) >= n) return 0.;
    double r = dv[i] * (double)a;
    if (two) r += dv[i + 1] * (double)b;
    return r;
  }
  __device__ __forceinline__ double dot(int p, int m, const P2& z) const {
    return dot1(p, m, z.re.x, z.im.x) + dot1(p + 1, m, z.re.y, z.im.y);
  }
};

// ---------------------------------------------------------------------------
// Real-to-complex rows (L+1 complex from 2L reals, FFTW r2c semantics), the forward
// transform of the matvec (r2cfieldbackend.hh:210-239 after fieldToExtendedField): rows p and
// p+1 per pair, threads along the row.  The 2L reals x of a row (the n0 field values, zero
// beyond) are transformed as the L complex z[m] = x[2m] + i x[2m+1]; with Z the forward
// length-L transform of z (in shared memory after the last stage),
//   X[k] = E - i w^k O,  E = (Z[k] + conj Z[L-k]) / 2,  O = (Z[k] - conj Z[L-k]) / 2,
// w = exp(-2 pi i / 2L), for k = 0..L (Z[L] = Z[0]).
// ---------------------------------------------------------------------------
// rows p and p+1 of n0 reals of type S (row p at p * n0)
template <typename S>
struct P2RealRowLoad {
  using S2 = typename std::conditional<sizeof(S) == 8, double2, float2>::type;
  const S* x;
  int n0;
  unsigned n;
  int np;
  int vec;  // x is aligned for pairs (8 bytes FP32, 16 bytes FP64) and n0 is even
  // (x[2m], x[2m+1]) of row p, zero beyond the row and beyond the last row
  __device__ __forceinline__ float2 pair(int p, int m, unsigned& bad) const {
    float2 z = make_float2(0.f, 0.f);
    if (p >= np || 2 * m >= n0) return z;
    const unsigned i = (unsigned)p * (unsigned)n0 + 2u * (unsigned)m;
    const bool two = 2 * m + 1 < n0;
    const bool ok = i + (two ? 1u : 0u) < n;
    bad |= (unsigned)!ok;
    if (!ok) return z;
    if (two && vec) {
      const S2 v = *reinterpret_cast<const S2*>(x + i);
      return make_float2((float)v.x, (float)v.y);
    }
    z.x = (float)x[i];
    if (two) z.y = (float)x[i + 1];
    return z;
  }
};

// FP64 rows of the CG's search direction, updated on the way into the matvec: d = z + beta d
// (beta = s[S_BETA]; no update once a residual-mode inner solve stopped, s[S_DONE] != 0),
// written back to d and returned in FP32 as P2RealRowLoad does.  Each element is loaded by
// exactly one thread of kp2_r2c, so the write-back has one writer.
struct P2DirRowLoad {
  const double* z;
  double* d;
  const double* s;
  int n0;
  unsigned n;
  int np;
  int vec;  // z and d 16-byte aligned and n0 even
  __device__ __forceinline__ float2 pair(int p, int m, unsigned& bad) const {
    float2 out = make_float2(0.f, 0.f);
    if (p >= np || 2 * m >= n0) return out;
    const unsigned i = (unsigned)p * (unsigned)n0 + 2u * (unsigned)m;
    const bool two = 2 * m + 1 < n0;
    const bool ok = i + (two ? 1u : 0u) < n;
    bad |= (unsigned)!ok;
    if (!ok) return out;
    const bool upd = s[S_DONE] == 0.;
    const double beta = s[S_BETA];
    if (two && vec) {
      const double2 zz = *reinterpret_cast<const double2*>(z + i);
      double2 dd = *reinterpret_cast<const double2*>(d + i);
      if (upd) {
        dd.x = zz.x + beta * dd.x;
        dd.y = zz.y + beta * dd.y;
        *reinterpret_cast<double2*>(d + i) = dd;
      }
      return make_float2((float)dd.x, (float)dd.y);
    }
    double a = d[i];
    if (upd) d[i] = a = z[i] + beta * a;
    out.x = (float)a;
    if (two) {
      double b = d[i + 1];
      if (upd) d[i + 1] = b = z[i + 1] + beta * b;
      out.y = (float)b;
    }
    return out;
  }
};

// complex rows p, p+1 (element k of row p at p * rowstride + k), elements k < Lout
struct P2RowStore {
  float2* ptr;
  unsigned rowstride;
  unsigned n;
  int np;
  int Lout;
  __device__ __forceinline__ void one(int p, int k, float2 v, unsigned& bad) const {
    if (p >= np || k >= Lout) return;
    const unsigned i = (unsigned)p * rowstride + (unsigned)k;
    const bool ok = i < n;
    bad |= (unsigned)!ok;
    if (ok) ptr[i] = v;
  }
};

template <int L, class Ld>
__global__ void __launch_bounds__(kP2Threads, PF_P2_MIN_C2R)
    kp2_r2c(const float4* __restrict__ twg, long long ntiles, Ld ld, P2RowStore st) {
  using G = P2Geom<L>;
  extern __shared__ __align__(16) float4 p2_smem[];
  float4* buf = p2_smem;
  float4* tw = p2_smem + G::Q * G::PLQ;
  const float4* twT = tw + G::NTW;  // exp(+2 pi i m / 2L), m < L
  p2_copy_table(tw, twg, G::NTW + L);
  __syncthreads();
  const int u = threadIdx.x % G::TP, q = threadIdx.x / G::TP;
  unsigned bad = 0;
  for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int p = (int)tile * G::NP + 2 * q;
    P2 v[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int m = u + r * G::TP;
      v[r] = p2_ab(ld.pair(p, m, bad), ld.pair(p + 1, m, bad));
    }
    // forward transform; Z lands in the exchange buffer (its last stage has read the buffer
    // and passed a barrier before the first output is written)
    p2_transform<L, -1>(v, buf, tw, u, q, [&](int j, const P2& x) { buf[p2_slot(G::PLQ, q, j)] = slot_of(x); });
    __syncthreads();
    const float2 half = make_float2(0.5f, 0.5f);
#pragma unroll
    for (int r = 0; r < 8; r++) {
      const int k = u + r * G::TP;
      const P2 A = p2_of(buf[p2_slot(G::PLQ, q, k)]);
      const P2 B = p2_of(buf[p2_slot(G::PLQ, q, (L - k) & (L - 1))]);
      // E = (A + conj B) / 2, O = (A - conj B) / 2
      const P2 E = {f2mul(half, f2add(A.re, B.re)), f2mul(half, f2sub(A.im, B.im))};
      const P2 O = {f2mul(half, f2sub(A.re, B.re)), f2mul(half, f2add(A.im, B.im))};
      // twT[k] = (c, s) = exp(+2 pi i k / 2L); X = (Er + c Oi - s Or, Ei - c Or - s Oi)
      const float4 w = twT[k];
      const float2 c = make_float2(w.x, w.y), sn = make_float2(w.z, w.w);
      const float2 xr = f2add(E.re, f2sub(f2mul(c, O.im), f2mul(sn, O.re)));
      const float2 xi = f2sub(E.im, f2fma(c, O.re, f2mul(sn, O.im)));
      st.one(p, k, make_float2(xr.x, xi.x), bad);
      st.one(p + 1, k, make_float2(xr.y, xi.y), bad);
      if (k == 0) {  // Nyquist X[L] = Re Z[0] - Im Z[0] (real)
        st.one(p, L, make_float2(A.re.x - A.im.x, 0.f), bad);
        st.one(p + 1, L, make_float2(A.re.y - A.im.y, 0.f), bad);
      }
    }
    __syncthreads();  // the buffer is read before the next tile's transform writes it
  }
  p2_report(bad);
}

}  // namespace pf
