// pf_fastfft.cuh -- compile-time specialised pencil passes for the common lengths.
//
// Same structure as k_pass / k_r2c / k_c2r (one HBM read and one HBM write per pass,
// the whole 1D transform of B pencils in shared memory), but the length L, the tile
// width B and the transform directions are template parameters: the radix schedule
// (8, then 4 / 2, then 3 / 5 / 7) is unrolled at compile time, every index division
// becomes a shift or a multiply, the twiddle table is staged once per CTA in shared
// memory, and each thread keeps a fixed pencil b = threadIdx.x % B so the load/store
// functors' per-pencil work is done once.  Shared layout: element (b, j) at j*B + b,
// so B consecutive pencils of a strided axis (or B rows of a contiguous one) are read
// and written as B-wide segments.
#pragma once

#include "pf_kernels.cuh"

namespace pf {

constexpr int pick_radix(int m) {
  return (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 2 == 0) ? 2 : (m % 3 == 0) ? 3 : (m % 5 == 0) ? 5 : (m % 7 == 0) ? 7 : m;
}

// pencils per tile: two buffers of L*B complex within PF_TILE_BYTES (default 32 KB)
#ifndef PF_TILE_BYTES
#define PF_TILE_BYTES 32768
#endif
template <typename T, int L>
constexpr int fast_B() {
  constexpr int b = PF_TILE_BYTES / (2 * L * (int)sizeof(cx<T>));
  return b >= 16 ? 16 : (b >= 8 ? 8 : (b >= 4 ? 4 : (b >= 2 ? 2 : 1)));
}

template <typename T, int SIGN>
__device__ __forceinline__ cx<T> tw_s(const cx<T>* tw, int m) {
  cx<T> w = tw[m];
  if (SIGN > 0) w.y = -w.y;
  return w;
}

// one radix-R butterfly column: V adjacent pencils share the index arithmetic and
// the twiddle factors; for FP32 the V = 2 pencils move as one 128-bit access
template <typename T, int V>
struct PencilVec {
  static __device__ __forceinline__ void ld(const cx<T>* p, cx<T>* v) {
#pragma unroll
    for (int i = 0; i < V; i++) v[i] = p[i];
  }
  static __device__ __forceinline__ void st(cx<T>* p, const cx<T>* v) {
#pragma unroll
    for (int i = 0; i < V; i++) p[i] = v[i];
  }
};
template <>
struct PencilVec<float, 2> {
  static __device__ __forceinline__ void ld(const float2* p, float2* v) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = make_float2(q.x, q.y);
    v[1] = make_float2(q.z, q.w);
  }
  static __device__ __forceinline__ void st(float2* p, const float2* v) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
  }
};

// pencils per butterfly column (2 = 128-bit shared accesses for FP32); 1 measured
// faster on B200 (the wider column raises register use and lowers occupancy)
template <typename T, int B>
constexpr int fast_V() {
  return 1;
}

template <typename T, int L, int B, int SIGN, int Ns>
__device__ __forceinline__ void fstages(cx<T>*& src, cx<T>*& dst, const cx<T>* tw) {
  if constexpr (Ns < L) {
    constexpr int R = pick_radix(L / Ns);
    constexpr int NBF = L / R;
    constexpr int TWS = L / (Ns * R);
    constexpr int V = fast_V<T, B>();
    constexpr int BV = B / V;
    constexpr int TSTEP = kThreads / BV;
    const int bv = (threadIdx.x % BV) * V;
    for (int t = threadIdx.x / BV; t < NBF; t += TSTEP) {
      const int k = t % Ns;
      cx<T> v[V][R];
#pragma unroll
      for (int r = 0; r < R; r++) {
        cx<T> a[V];
        PencilVec<T, V>::ld(src + (t + r * NBF) * B + bv, a);
        if constexpr (Ns > 1) {
          if (r > 0) {
            const cx<T> w = tw_s<T, SIGN>(tw, r * k * TWS);
#pragma unroll
            for (int i = 0; i < V; i++) a[i] = cmul<T>(a[i], w);
          }
        }
#pragma unroll
        for (int i = 0; i < V; i++) v[i][r] = a[i];
      }
#pragma unroll
      for (int i = 0; i < V; i++) {
        if constexpr (R == 2 || R == 3 || R == 4 || R == 5 || R == 8) {
          Dft<T, R>::run(v[i], SIGN, nullptr, L);
        } else {
          // generic odd prime radix from the shared twiddle table
          cx<T> o[R];
#pragma unroll
          for (int q = 0; q < R; q++) {
            cx<T> s = v[i][0];
#pragma unroll
            for (int r = 1; r < R; r++)
              s = cadd<T>(s, cmul<T>(v[i][r], tw_s<T, SIGN>(tw, ((r * q) % R) * (L / R))));
            o[q] = s;
          }
#pragma unroll
          for (int q = 0; q < R; q++) v[i][q] = o[q];
        }
      }
      const int base = (t / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) {
        cx<T> a[V];
#pragma unroll
        for (int i = 0; i < V; i++) a[i] = v[i][r];
        PencilVec<T, V>::st(dst + (base + r * Ns) * B + bv, a);
      }
    }
    __syncthreads();
    cx<T>* tmp = src;
    src = dst;
    dst = tmp;
    fstages<T, L, B, SIGN, Ns * R>(src, dst, tw);
  }
}

template <typename T>
constexpr int fast_minblocks() {
  return sizeof(T) == 4 ? 3 : 2;
}

// Complex pass.  Tile = B consecutive pencils (rows when CONTIG).  Optional fused
// elementwise Mid between a SIGN and a SIGN2 transform.  Ld may provide
// load2(p, j, io, v0, v1) producing elements j and j + L/2 together (PAIR).
template <typename T, int L, int B, int SIGN, int SIGN2, bool CONTIG, bool PAIR, class Ld, class Mid, class St>
__global__ void __launch_bounds__(kThreads, fast_minblocks<T>())
    k_fpass(const PassArgs a, const cx<T>* __restrict__ twg, Ld ld, Mid mid, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* b1 = b0 + L * B;
  cx<T>* tw = b1 + L * B;
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
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  const int jt = threadIdx.x / B;
  const int p = p0 + b;
  const bool live = p < np;
  if constexpr (PAIR) {
#pragma unroll
    for (int j = jt; j < L / 2; j += TSTEP) {
      cx<T> v0 = mk<T>(0, 0), v1 = mk<T>(0, 0);
      if (live) ld.template load2<T>(p, j, io, v0, v1);
      b0[j * B + b] = v0;
      b0[(j + L / 2) * B + b] = v1;
    }
  } else {
#pragma unroll
    for (int j = jt; j < L; j += TSTEP) b0[j * B + b] = live ? ld.template load<T>(p, j, io) : mk<T>(0, 0);
  }
  __syncthreads();
  cx<T>* src = b0;
  cx<T>* dst = b1;
  fstages<T, L, B, SIGN, 1>(src, dst, tw);
  if constexpr (Mid::active) {
    if (live)
      for (int j = jt; j < L; j += TSTEP) src[j * B + b] = mid.template operator()<T>(p, j, io, src[j * B + b]);
    __syncthreads();
    fstages<T, L, B, SIGN2, 1>(src, dst, tw);
  }
  if (live) {
#pragma unroll 8
    for (int j = jt; j < a.Lout; j += TSTEP) st.template store<T>(p, j, io, src[j * B + b]);
  }
}

// Real-data passes along contiguous rows of 2L reals (see k_r2c / k_c2r for the
// half-length algorithm); shared: two (L+1)*B buffers, then tables tw (L) and twT (L).
template <typename T, int L, int B, class Ld, class St>
__global__ void __launch_bounds__(kThreads, fast_minblocks<T>())
    k_fr2c(const PassArgs a, const cx<T>* __restrict__ twg, const cx<T>* __restrict__ twTg, Ld ld, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* b1 = b0 + (L + 1) * B;
  cx<T>* tw = b1 + (L + 1) * B;
  cx<T>* twT = tw + L;
  for (int i = threadIdx.x; i < L; i += kThreads) {
    tw[i] = __ldg(twg + i);
    twT[i] = __ldg(twTg + i);
  }
  const int np = (int)a.npencil;
  const int p0 = blockIdx.x * B;
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  const int jt = threadIdx.x / B;
  const int p = p0 + b;
  const bool live = p < np;
#pragma unroll
  for (int m = jt; m < L; m += TSTEP) {
    cx<T> z = mk<T>(0, 0);
    if (live) z = mk<T>(ld.template real<T>(p, 2 * m), ld.template real<T>(p, 2 * m + 1));
    b0[m * B + b] = z;
  }
  __syncthreads();
  cx<T>* src = b0;
  cx<T>* dst = b1;
  fstages<T, L, B, -1, 1>(src, dst, tw);
  cx<T>* X = dst;
  for (int k = jt; k <= L; k += TSTEP) {
    const cx<T> zk = src[(k == L ? 0 : k) * B + b];
    const cx<T> zm = conjg<T>(src[(k == 0 ? 0 : L - k) * B + b]);
    const cx<T> e = cscale<T>(cadd<T>(zk, zm), (T)0.5);
    const cx<T> o = cscale<T>(csub<T>(zk, zm), (T)0.5);
    const cx<T> oi = mk<T>(o.y, -o.x);
    const cx<T> w = (k == L) ? mk<T>(-1, 0) : twT[k];
    X[k * B + b] = cadd<T>(e, cmul<T>(oi, w));
  }
  __syncthreads();
  if (live)
    for (int k = jt; k < a.Lout; k += TSTEP) st.template store<T>(p, k, 0, X[k * B + b]);
}

template <typename T, int L, int B, class Ld, class St>
__global__ void __launch_bounds__(kThreads, fast_minblocks<T>())
    k_fc2r(const PassArgs a, const cx<T>* __restrict__ twg, const cx<T>* __restrict__ twTg, Ld ld, St st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cx<T>* b0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* b1 = b0 + (L + 1) * B;
  cx<T>* tw = b1 + (L + 1) * B;
  cx<T>* twT = tw + L;
  for (int i = threadIdx.x; i < L; i += kThreads) {
    tw[i] = __ldg(twg + i);
    twT[i] = __ldg(twTg + i);
  }
  const int np = (int)a.npencil;
  const int p0 = blockIdx.x * B;
  constexpr int TSTEP = kThreads / B;
  const int b = threadIdx.x % B;
  const int jt = threadIdx.x / B;
  const int p = p0 + b;
  const bool live = p < np;
#pragma unroll
  for (int k = jt; k <= L; k += TSTEP) {
    cx<T> v = live ? ld.template load<T>(p, k, 0) : mk<T>(0, 0);
    if (k == 0 || k == L) v.y = 0;
    b1[k * B + b] = v;
  }
  __syncthreads();
  for (int k = jt; k < L; k += TSTEP) {
    const cx<T> xk = b1[k * B + b];
    const cx<T> xm = conjg<T>(b1[(L - k) * B + b]);
    const cx<T> s = cadd<T>(xk, xm);
    const cx<T> d = csub<T>(xk, xm);
    const cx<T> t = cmul<T>(d, conjg<T>(twT[k]));
    b0[k * B + b] = mk<T>(s.x - t.y, s.y + t.x);
  }
  __syncthreads();
  cx<T>* src = b0;
  cx<T>* dst = b1;
  fstages<T, L, B, +1, 1>(src, dst, tw);
  if (live)
    for (int j = jt; j < a.Lout; j += TSTEP) {
      const cx<T> v = src[(j >> 1) * B + b];
      st.template real<T>(p, j, (j & 1) ? v.y : v.x);
    }
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
  const long long i = (long long)p * ld.rowstride + (long long)j * ld.jstride + (long long)o * ld.ostride;
  const bool ok = p < np && j < ld.Lin && in_bounds(i, ld.n);
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
  cx<T>* in0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* in1 = in0 + L * B;
  cx<T>* work = in1 + L * B;
  cx<T>* tw = work + L * B;
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
    for (int j = jt; j < L; j += TSTEP) tile_copy<T>(ld, in0 + j * B + b, p, np, j, o);
  }
  cp_async_commit();
  for (int it = 0; t < ntiles; it++, t += gridDim.x) {
    cx<T>* cur = (it & 1) ? in1 : in0;
    cx<T>* nxt = (it & 1) ? in0 : in1;
    const long long tn = t + gridDim.x;
    if (tn < ntiles) {
      const int o = (int)(tn / tpo), p = (int)(tn - (long long)o * tpo) * B + b;
#pragma unroll 4
      for (int j = jt; j < L; j += TSTEP) tile_copy<T>(ld, nxt + j * B + b, p, np, j, o);
    }
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const int o = (int)(t / tpo);
    const int p = (int)(t - (long long)o * tpo) * B + b;
    cx<T>* src = cur;
    cx<T>* dst = work;
    fstages<T, L, B, SIGN, 1>(src, dst, tw);
    if constexpr (Mid::active) {
      if (p < np)
        for (int j = jt; j < L; j += TSTEP) src[j * B + b] = mid.template operator()<T>(p, j, o, src[j * B + b]);
      __syncthreads();
      fstages<T, L, B, SIGN2, 1>(src, dst, tw);
    }
    if (p < np) {
#pragma unroll 8
      for (int j = jt; j < a.Lout; j += TSTEP) st.template store<T>(p, j, o, src[j * B + b]);
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
  constexpr int LP = L + 1;
  cx<T>* in0 = reinterpret_cast<cx<T>*>(smem_raw);
  cx<T>* in1 = in0 + LP * B;
  cx<T>* work = in1 + LP * B;
  cx<T>* tw = work + LP * B;
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
    for (int k = jt; k <= L; k += TSTEP) tile_copy<T>(ld, in0 + k * B + b, p, np, k, 0);
  }
  cp_async_commit();
  for (int it = 0; t < ntiles; it++, t += gridDim.x) {
    cx<T>* cur = (it & 1) ? in1 : in0;
    cx<T>* nxt = (it & 1) ? in0 : in1;
    const long long tn = t + gridDim.x;
    if (tn < ntiles) {
      const int p = (int)tn * B + b;
#pragma unroll 4
      for (int k = jt; k <= L; k += TSTEP) tile_copy<T>(ld, nxt + k * B + b, p, np, k, 0);
    }
    cp_async_commit();
    cp_async_wait1();
    __syncthreads();
    const int p = (int)t * B + b;
    for (int k = jt; k < L; k += TSTEP) {
      cx<T> xk = cur[k * B + b];
      cx<T> xm = cur[(L - k) * B + b];
      if (k == 0) {
        xk.y = 0;
        xm.y = 0;
      }
      xm = conjg<T>(xm);
      const cx<T> s = cadd<T>(xk, xm);
      const cx<T> d = csub<T>(xk, xm);
      const cx<T> tt = cmul<T>(d, conjg<T>(twT[k]));
      work[k * B + b] = mk<T>(s.x - tt.y, s.y + tt.x);
    }
    __syncthreads();
    cx<T>* src = work;
    cx<T>* dst = cur;
    fstages<T, L, B, +1, 1>(src, dst, tw);
    if (p < np) {
#pragma unroll 8
      for (int j = jt; j < a.Lout; j += TSTEP) {
        const cx<T> v = src[(j >> 1) * B + b];
        st.template real<T>(p, j, (j & 1) ? v.y : v.x);
      }
    }
    __syncthreads();
  }
}

}  // namespace pf
