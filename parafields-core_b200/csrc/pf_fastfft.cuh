// pf_fastfft.cuh -- compile-time specialised pencil passes for the common lengths.
//
// Same job as k_pass / k_r2c / k_c2r (one HBM read and one HBM write per pass, the
// whole 1D transform of B pencils in shared memory), specialised for B200:
//  - L, B and the directions are template parameters; the Stockham radix schedule
//    (8, then 4 / 2, then 3 / 5 / 7) unrolls at compile time;
//  - element (b, j) of a tile lives at row j + j/8 (one padding row every 8 rows) so
//    the stride-8 stores of a radix-8 first stage hit distinct banks;
//  - the first stage runs in registers on the values the loader (or the noise
//    generator) produced, and the last stage writes its outputs straight to global
//    memory, so a 3-stage transform touches shared memory 4 times per element;
//  - each thread keeps one pencil b = threadIdx.x % B; B = 8 * threads / L, so every
//    stage processes exactly one radix-8 butterfly column per thread;
//  - passes over work arrays prefetch the next tile with cp.async (software
//    pipelining across tiles in persistent CTAs).
#pragma once

#include "pf_kernels.cuh"

namespace pf {

constexpr int pick_radix(int m) {
  return (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5 : (m % 7 == 0) ? 7 : m;
}

// one radix-8 butterfly column per thread and stage: B = 8 * threads / L, rounded down to
// a power of two so that B divides the thread count (lengths with a factor 3)
constexpr int pow2_floor_c(int x) { return x >= 2 ? 2 * pow2_floor_c(x / 2) : 1; }
template <typename T, int L>
constexpr int fast_B() {
  return (8 * kThreads / L) >= 16 ? 16 : ((8 * kThreads / L) >= 1 ? pow2_floor_c(8 * kThreads / L) : 1);
}

// rows of one padded tile buffer holding `rows` logical rows
constexpr int padded_rows(int rows) { return rows + rows / 8 + 1; }

template <int B>
__device__ __forceinline__ int sidx(int j, int b) {
  return (j + (j >> 3)) * B + b;
}

// shared bytes of each kernel family (buffers + twiddle tables)
template <typename T, int L>
constexpr size_t fast_smem_pass() {
  return (size_t)(2 * padded_rows(L) * fast_B<T, L>() + L) * sizeof(cx<T>);
}
template <typename T, int L>
constexpr size_t fast_smem_pipe() {
  return (size_t)(3 * padded_rows(L) * fast_B<T, L>() + L) * sizeof(cx<T>);
}
template <typename T, int L>
constexpr size_t fast_smem_real() {
  return (size_t)(2 * padded_rows(L + 1) * fast_B<T, L>() + 2 * L) * sizeof(cx<T>);
}
template <typename T, int L>
constexpr size_t fast_smem_real_pipe() {
  return (size_t)(3 * padded_rows(L + 1) * fast_B<T, L>() + 2 * L) * sizeof(cx<T>);
}

template <typename T>
constexpr int fast_minblocks() {
  return sizeof(T) == 4 ? 3 : 2;
}

template <typename T, int SIGN>
__device__ __forceinline__ cx<T> tw_s(const cx<T>* tw, int m) {
  cx<T> w = tw[m];
  if (SIGN > 0) w.y = -w.y;
  return w;
}

template <typename T, int R, int SIGN, int L>
__device__ __forceinline__ void dft_r(cx<T>* v, const cx<T>* tw) {
  if constexpr (R == 2 || R == 3 || R == 4 || R == 5 || R == 8) {
    Dft<T, R>::run(v, SIGN, nullptr, L);
  } else {  // generic odd prime radix from the shared twiddle table
    cx<T> o[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
      cx<T> s = v[0];
#pragma unroll
      for (int r = 1; r < R; r++) s = cadd<T>(s, cmul<T>(v[r], tw_s<T, SIGN>(tw, ((r * q) % R) * (L / R))));
      o[q] = s;
    }
#pragma unroll
    for (int q = 0; q < R; q++) v[q] = o[q];
  }
}

// Stockham stage Ns (smem -> smem).  Outputs of butterfly t go to base + r*Ns.
template <typename T, int L, int B, int SIGN, int Ns>
__device__ __forceinline__ void fstage(const cx<T>* src, cx<T>* dst, const cx<T>* tw) {
  constexpr int R = pick_radix(L / Ns);
  constexpr int NBF = L / R;
  constexpr int TWS = L / (Ns * R);
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  for (int t = threadIdx.x / B; t < NBF; t += TSTEP) {
    const int k = t % Ns;
    cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      cx<T> a = src[sidx<B>(t + r * NBF, b)];
      if constexpr (Ns > 1) {
        if (r > 0) a = cmul<T>(a, tw_s<T, SIGN>(tw, r * k * TWS));
      }
      v[r] = a;
    }
    dft_r<T, R, SIGN, L>(v, tw);
    const int base = (t / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) dst[sidx<B>(base + r * Ns, b)] = v[r];
  }
}

// last stage: outputs j = t + r*Ns go straight to out(j, value)
template <typename T, int L, int B, int SIGN, int Ns, class Out>
__device__ __forceinline__ void fstage_last(const cx<T>* src, const cx<T>* tw, const Out& out) {
  constexpr int R = pick_radix(L / Ns);
  static_assert(Ns * R == L, "not the last stage");
  constexpr int NBF = L / R;
  constexpr int TWS = L / (Ns * R);
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  for (int t = threadIdx.x / B; t < NBF; t += TSTEP) {
    cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      cx<T> a = src[sidx<B>(t + r * NBF, b)];
      if constexpr (Ns > 1) {
        if (r > 0) a = cmul<T>(a, tw_s<T, SIGN>(tw, r * t * TWS));
      }
      v[r] = a;
    }
    dft_r<T, R, SIGN, L>(v, tw);
#pragma unroll
    for (int r = 0; r < R; r++) out(t + r * Ns, v[r]);
  }
}

// middle stages from Ns up to (excluding) the last one, ping-ponging src/dst
template <typename T, int L, int B, int SIGN, int Ns>
__device__ __forceinline__ void fstages_mid(cx<T>*& src, cx<T>*& dst, const cx<T>* tw) {
  if constexpr (Ns * pick_radix(L / Ns) < L) {
    fstage<T, L, B, SIGN, Ns>(src, dst, tw);
    __syncthreads();
    cx<T>* t = src;
    src = dst;
    dst = t;
    fstages_mid<T, L, B, SIGN, Ns * pick_radix(L / Ns)>(src, dst, tw);
  }
}

// Ns of the last stage
template <int L, int Ns = 1>
constexpr int last_ns() {
  if constexpr (Ns * pick_radix(L / Ns) < L)
    return last_ns<L, Ns * pick_radix(L / Ns)>();
  else
    return Ns;
}

// all stages smem -> smem (result in src)
template <typename T, int L, int B, int SIGN>
__device__ __forceinline__ void fstages_all(cx<T>*& src, cx<T>*& dst, const cx<T>* tw) {
  fstages_mid<T, L, B, SIGN, 1>(src, dst, tw);
  fstage<T, L, B, SIGN, last_ns<L>()>(src, dst, tw);
  __syncthreads();
  cx<T>* t = src;
  src = dst;
  dst = t;
}

// first stage (Ns = 1) on register values v[r] = element t + r*L/R1; result to dst
template <typename T, int L, int B, int SIGN>
__device__ __forceinline__ void fstage_first_regs(cx<T>* v, int t, cx<T>* dst, const cx<T>* tw) {
  constexpr int R = pick_radix(L);
  dft_r<T, R, SIGN, L>(v, tw);
  const int b = threadIdx.x % B;
#pragma unroll
  for (int r = 0; r < R; r++) dst[sidx<B>(t * R + r, b)] = v[r];
}

// the stages after a register first stage (src holds its output), ending in global
template <typename T, int L, int B, int SIGN, class Out>
__device__ __forceinline__ void fstages_rest_store(cx<T>*& src, cx<T>*& dst, const cx<T>* tw, const Out& out) {
  constexpr int R1 = pick_radix(L);
  fstages_mid<T, L, B, SIGN, R1>(src, dst, tw);
  fstage_last<T, L, B, SIGN, last_ns<L>()>(src, tw, out);
}

// the stages after a register first stage, ending in shared memory (result in src)
template <typename T, int L, int B, int SIGN>
__device__ __forceinline__ void fstages_rest_smem(cx<T>*& src, cx<T>*& dst, const cx<T>* tw) {
  constexpr int R1 = pick_radix(L);
  if constexpr (R1 < L) {
    fstages_mid<T, L, B, SIGN, R1>(src, dst, tw);
    fstage<T, L, B, SIGN, last_ns<L>()>(src, dst, tw);
    __syncthreads();
    cx<T>* t = src;
    src = dst;
    dst = t;
  }
}

// ---------------------------------------------------------------------------
// Complex pass with a functor loader.  Tile = B consecutive pencils (rows when
// CONTIG).  Optional fused elementwise Mid between a SIGN and a SIGN2 transform.
// PAIR loaders produce elements j and j + L/2 together (load2).
// ---------------------------------------------------------------------------
template <typename T, int L, int B, int SIGN, int SIGN2, bool CONTIG, bool PAIR, class Ld, class Mid, class St>
__global__ void __launch_bounds__(kThreads, fast_minblocks<T>())
    k_fpass(const PassArgs a, const cx<T>* __restrict__ twg, Ld ld, Mid mid, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PR = padded_rows(L);
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* b1 = b0 + PR * B;
  cx<T>* tw = b1 + PR * B;
  for (int i = threadIdx.x; i < L; i += kThreads) tw[i] = __ldg(twg + i);
  int p0, io;
  const int np = (int)a.npencil;
  if (CONTIG) {
    p0 = blockIdx.x * B;
    io = 0;
  } else {
    const int tpo = (np + B - 1) / B;
    io = blockIdx.x / tpo;
    p0 = (blockIdx.x - io * tpo) * B;
  }
  constexpr int R1 = pick_radix(L);
  constexpr int NBF1 = L / R1;
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  const int p = p0 + b;
  const bool live = p < np;
  __syncthreads();  // twiddles
  for (int t = threadIdx.x / B; t < NBF1; t += TSTEP) {
    cx<T> v[R1];
    if constexpr (PAIR) {
      static_assert(R1 % 2 == 0, "paired loads need an even first radix");
#pragma unroll
      for (int r = 0; r < R1 / 2; r++) {
        cx<T> x0 = mk<T>(0, 0), x1 = mk<T>(0, 0);
        if (live) ld.template load2<T>(p, t + r * NBF1, io, x0, x1);
        v[r] = x0;
        v[r + R1 / 2] = x1;
      }
    } else {
#pragma unroll
      for (int r = 0; r < R1; r++) v[r] = live ? ld.template load<T>(p, t + r * NBF1, io) : mk<T>(0, 0);
    }
    fstage_first_regs<T, L, B, SIGN>(v, t, b0, tw);
  }
  __syncthreads();
  cx<T>* src = b0;
  cx<T>* dst = b1;
  const int Lout = a.Lout;
  auto out = [&](int j, cx<T> v) {
    if (live && j < Lout) st.template store<T>(p, j, io, v);
  };
  if constexpr (Mid::active) {
    fstages_rest_smem<T, L, B, SIGN>(src, dst, tw);
    if (live)
      for (int j = threadIdx.x / B; j < L; j += TSTEP)
        src[sidx<B>(j, b)] = mid.template operator()<T>(p, j, io, src[sidx<B>(j, b)]);
    __syncthreads();
    fstages_mid<T, L, B, SIGN2, 1>(src, dst, tw);
    fstage_last<T, L, B, SIGN2, last_ns<L>()>(src, tw, out);
  } else {
    fstages_rest_store<T, L, B, SIGN>(src, dst, tw, out);
  }
}

// Real-to-complex rows (2L reals -> L+1 complex, half-length algorithm of k_r2c).
template <typename T, int L, int B, class Ld, class St>
__global__ void __launch_bounds__(kThreads, fast_minblocks<T>())
    k_fr2c(const PassArgs a, const cx<T>* __restrict__ twg, const cx<T>* __restrict__ twTg, Ld ld, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PR = padded_rows(L + 1);
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* b1 = b0 + PR * B;
  cx<T>* tw = b1 + PR * B;
  cx<T>* twT = tw + L;
  for (int i = threadIdx.x; i < L; i += kThreads) {
    tw[i] = __ldg(twg + i);
    twT[i] = __ldg(twTg + i);
  }
  const int np = (int)a.npencil;
  const int p0 = blockIdx.x * B;
  constexpr int R1 = pick_radix(L);
  constexpr int NBF1 = L / R1;
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  const int p = p0 + b;
  const bool live = p < np;
  __syncthreads();
  for (int t = threadIdx.x / B; t < NBF1; t += TSTEP) {
    cx<T> v[R1];
#pragma unroll
    for (int r = 0; r < R1; r++) {
      const int m = t + r * NBF1;
      v[r] = live ? mk<T>(ld.template real<T>(p, 2 * m), ld.template real<T>(p, 2 * m + 1)) : mk<T>(0, 0);
    }
    fstage_first_regs<T, L, B, -1>(v, t, b0, tw);
  }
  __syncthreads();
  cx<T>* src = b0;
  cx<T>* dst = b1;
  fstages_rest_smem<T, L, B, -1>(src, dst, tw);
  if (live)
    for (int k = threadIdx.x / B; k <= L && k < a.Lout; k += TSTEP) {
      const cx<T> zk = src[sidx<B>(k == L ? 0 : k, b)];
      const cx<T> zm = conjg<T>(src[sidx<B>(k == 0 ? 0 : L - k, b)]);
      const cx<T> e = cscale<T>(cadd<T>(zk, zm), (T)0.5);
      const cx<T> o = cscale<T>(csub<T>(zk, zm), (T)0.5);
      const cx<T> oi = mk<T>(o.y, -o.x);
      const cx<T> w = (k == L) ? mk<T>(-1, 0) : twT[k];
      st.template store<T>(p, k, 0, cadd<T>(e, cmul<T>(oi, w)));
    }
}

// Complex-to-real rows with a functor loader (FFTW c2r semantics, see k_c2r).
template <typename T, int L, int B, class Ld, class St>
__global__ void __launch_bounds__(kThreads, fast_minblocks<T>())
    k_fc2r(const PassArgs a, const cx<T>* __restrict__ twg, const cx<T>* __restrict__ twTg, Ld ld, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PR = padded_rows(L + 1);
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* b1 = b0 + PR * B;
  cx<T>* tw = b1 + PR * B;
  cx<T>* twT = tw + L;
  for (int i = threadIdx.x; i < L; i += kThreads) {
    tw[i] = __ldg(twg + i);
    twT[i] = __ldg(twTg + i);
  }
  const int np = (int)a.npencil;
  const int p0 = blockIdx.x * B;
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  const int p = p0 + b;
  const bool live = p < np;
  for (int k = threadIdx.x / B; k <= L; k += TSTEP) {
    cx<T> v = live ? ld.template load<T>(p, k, 0) : mk<T>(0, 0);
    if (k == 0 || k == L) v.y = 0;
    b1[sidx<B>(k, b)] = v;
  }
  __syncthreads();
  for (int k = threadIdx.x / B; k < L; k += TSTEP) {
    const cx<T> xk = b1[sidx<B>(k, b)];
    const cx<T> xm = conjg<T>(b1[sidx<B>(L - k, b)]);
    const cx<T> s = cadd<T>(xk, xm);
    const cx<T> d = csub<T>(xk, xm);
    const cx<T> t = cmul<T>(d, conjg<T>(twT[k]));
    b0[sidx<B>(k, b)] = mk<T>(s.x - t.y, s.y + t.x);
  }
  __syncthreads();
  cx<T>* src = b0;
  cx<T>* dst = b1;
  const int Lout = a.Lout;
  auto out = [&](int m, cx<T> v) {
    if (!live) return;
    if (2 * m < Lout) st.template real<T>(p, 2 * m, v.x);
    if (2 * m + 1 < Lout) st.template real<T>(p, 2 * m + 1, v.y);
  };
  fstages_mid<T, L, B, +1, 1>(src, dst, tw);
  fstage_last<T, L, B, +1, last_ns<L>()>(src, tw, out);
}

// ---------------------------------------------------------------------------
// software-pipelined persistent passes over work arrays: while a CTA transforms tile
// i, the asynchronous copies (cp.async, global -> shared without registers) of tile
// i + 1 are in flight, so the HBM latency hides behind the butterflies.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

// copies element (p, j, o) of an ArrLoad array into shared (zero outside Lin / np)
template <typename T>
__device__ __forceinline__ void tile_copy(const ArrLoad<cx<T>>& ld, cx<T>* dst, int p, int np, int j, int o) {
  const unsigned i = (unsigned)p * ld.rowstride + (unsigned)j * ld.jstride + (unsigned)o * ld.ostride;
  const bool ok = p < np && j < ld.Lin && in_bounds32(i, ld.n);
  if (sizeof(cx<T>) == 16)
    cp_async16(dst, ok ? (const void*)(ld.ptr + i) : (const void*)ld.ptr, ok ? 16 : 0);
  else
    cp_async8(dst, ok ? (const void*)(ld.ptr + i) : (const void*)ld.ptr, ok ? 8 : 0);
}

// Strided complex pass (pencils p of outer block o), persistent over tiles.
template <typename T, int L, int B, int SIGN, int SIGN2, class Mid, class St>
__global__ void __launch_bounds__(kThreads, fast_minblocks<T>())
    k_fpass_pipe(const PassArgs a, const cx<T>* __restrict__ twg, ArrLoad<cx<T>> ld, Mid mid, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PR = padded_rows(L);
  cx<T>* in0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* in1 = in0 + PR * B;
  cx<T>* work = in1 + PR * B;
  cx<T>* tw = work + PR * B;
  for (int i = threadIdx.x; i < L; i += kThreads) tw[i] = __ldg(twg + i);
  const int np = (int)a.npencil;
  const int tpo = (np + B - 1) / B;
  const long long ntiles = (long long)tpo * a.nouter;
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  const int jt = threadIdx.x / B;
  long long t = blockIdx.x;
  if (t < ntiles) {
    const int o = (int)(t / tpo), p = (int)(t - (long long)o * tpo) * B + b;
#pragma unroll 4
    for (int j = jt; j < L; j += TSTEP) tile_copy<T>(ld, in0 + sidx<B>(j, b), p, np, j, o);
  }
  cp_async_commit();
  for (int it = 0; t < ntiles; it++, t += gridDim.x) {
    cx<T>* cur = (it & 1) ? in1 : in0;
    cx<T>* nxt = (it & 1) ? in0 : in1;
    const long long tn = t + gridDim.x;
    if (tn < ntiles) {
      const int o = (int)(tn / tpo), p = (int)(tn - (long long)o * tpo) * B + b;
#pragma unroll 4
      for (int j = jt; j < L; j += TSTEP) tile_copy<T>(ld, nxt + sidx<B>(j, b), p, np, j, o);
    }
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const int o = (int)(t / tpo);
    const int p = (int)(t - (long long)o * tpo) * B + b;
    const bool live = p < np;
    const int Lout = a.Lout;
    auto out = [&](int j, cx<T> v) {
      if (live && j < Lout) st.template store<T>(p, j, o, v);
    };
    cx<T>* src = cur;
    cx<T>* dst = work;
    if constexpr (Mid::active) {
      fstages_all<T, L, B, SIGN>(src, dst, tw);
      if (live)
        for (int j = jt; j < L; j += TSTEP) src[sidx<B>(j, b)] = mid.template operator()<T>(p, j, o, src[sidx<B>(j, b)]);
      __syncthreads();
      fstages_mid<T, L, B, SIGN2, 1>(src, dst, tw);
      fstage_last<T, L, B, SIGN2, last_ns<L>()>(src, tw, out);
    } else {
      fstages_mid<T, L, B, SIGN, 1>(src, dst, tw);
      fstage_last<T, L, B, SIGN, last_ns<L>()>(src, tw, out);
    }
    __syncthreads();
  }
}

// Complex-to-real rows (2L reals from L+1 complex), persistent over row tiles.
template <typename T, int L, int B, class St>
__global__ void __launch_bounds__(kThreads, fast_minblocks<T>())
    k_fc2r_pipe(const PassArgs a, const cx<T>* __restrict__ twg, const cx<T>* __restrict__ twTg,
                ArrLoad<cx<T>> ld, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int PR = padded_rows(L + 1);
  cx<T>* in0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* in1 = in0 + PR * B;
  cx<T>* work = in1 + PR * B;
  cx<T>* tw = work + PR * B;
  cx<T>* twT = tw + L;
  for (int i = threadIdx.x; i < L; i += kThreads) {
    tw[i] = __ldg(twg + i);
    twT[i] = __ldg(twTg + i);
  }
  const int np = (int)a.npencil;
  const long long ntiles = (np + B - 1) / B;
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  const int jt = threadIdx.x / B;
  long long t = blockIdx.x;
  if (t < ntiles) {
    const int p = (int)t * B + b;
#pragma unroll 4
    for (int k = jt; k <= L; k += TSTEP) tile_copy<T>(ld, in0 + sidx<B>(k, b), p, np, k, 0);
  }
  cp_async_commit();
  for (int it = 0; t < ntiles; it++, t += gridDim.x) {
    cx<T>* cur = (it & 1) ? in1 : in0;
    cx<T>* nxt = (it & 1) ? in0 : in1;
    const long long tn = t + gridDim.x;
    if (tn < ntiles) {
      const int p = (int)tn * B + b;
#pragma unroll 4
      for (int k = jt; k <= L; k += TSTEP) tile_copy<T>(ld, nxt + sidx<B>(k, b), p, np, k, 0);
    }
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const int p = (int)t * B + b;
    const bool live = p < np;
    for (int k = jt; k < L; k += TSTEP) {
      cx<T> xk = cur[sidx<B>(k, b)];
      cx<T> xm = cur[sidx<B>(L - k, b)];
      if (k == 0) {
        xk.y = 0;
        xm.y = 0;
      }
      xm = conjg<T>(xm);
      const cx<T> s = cadd<T>(xk, xm);
      const cx<T> d = csub<T>(xk, xm);
      const cx<T> tt = cmul<T>(d, conjg<T>(twT[k]));
      work[sidx<B>(k, b)] = mk<T>(s.x - tt.y, s.y + tt.x);
    }
    __syncthreads();
    const int Lout = a.Lout;
    auto out = [&](int m, cx<T> v) {
      if (!live) return;
      if (2 * m < Lout) st.template real<T>(p, 2 * m, v.x);
      if (2 * m + 1 < Lout) st.template real<T>(p, 2 * m + 1, v.y);
    };
    cx<T>* src = work;
    cx<T>* dst = cur;
    fstages_mid<T, L, B, +1, 1>(src, dst, tw);
    fstage_last<T, L, B, +1, last_ns<L>()>(src, tw, out);
    __syncthreads();
  }
}

}  // namespace pf
