// pf_cg.cuh -- FP64 vector kernels of the CG inverse (Matrix::innerCG,
// include/parafields/matrix.hh:1315-1432).  Every dot product is reduced in two
// deterministic stages (fixed grid, fixed tree) so repeated solves give identical
// results; the scalars alpha/beta stay on the device.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pf {

// device and pinned-host scratch of one plan's CG
struct CgScratch {
  double *Ax = nullptr, *r = nullptr, *z = nullptr, *d = nullptr, *Ad = nullptr, *e = nullptr, *ri = nullptr;
  double *part = nullptr, *s = nullptr;
  unsigned* cnt = nullptr;  // ticket of the last-block reductions (0 between kernels)
  double* hs = nullptr;  // pinned copy of the scalars
  uint64_t n = 0;
};

constexpr int kCgThreads = 256;
// 8 x 148 SMs (64 warps per SM, one load in flight per thread: enough to stream the FP64
// vectors; 2 per SM ran the dot products at about a third of HBM bandwidth); fixed, so the
// reduction order is fixed
constexpr int kCgBlocks = 1184;

// scalar slots
enum CgSlot {
  S_SP = 0,     // (P r) . r of the current iteration
  S_DEN = 1,    // d . A d
  S_OLD = 2,    // energy before the update
  S_VAL = 3,    // energy after the update
  S_SPNEW = 4,  // (P r) . r of the next iteration
  S_BETA = 5,
  S_FIRST = 6,
  S_RR = 7,     // r . r
  S_BB = 8,     // b . b
  S_NZ = 9,     // count of |b_i| > 1e-10
  S_DONE = 10,  // residual-mode inner solve: 0 running, 1 converged, 2 NaN residual
  S_ITERS = 11, // residual-mode inner solve: iterations counted until it stopped
  S_THR = 12,   // residual-mode inner solve: stop once r . r <= S_THR
  S_COUNT = 16
};

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); k++) r += sh[k];
  __syncthreads();
  return r;
}

// Reductions finished inside the kernel: every block stores its partial, and the last block
// to take a ticket on `cnt` (which it resets to 0 for the next kernel of the stream) sums the
// partials in the fixed order of k_finish below, so the result is the same, bit for bit, as
// with the separate finishing kernel.
__device__ __forceinline__ bool cg_last_block(double v, double* part, unsigned* cnt) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    part[blockIdx.x] = v;
    __threadfence();  // the partial is visible before the ticket is taken
    last = atomicAdd(cnt, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  return last;
}
__device__ __forceinline__ double cg_sum_partials(const double* part, double* sh) {
  __threadfence();
  double v = 0.;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) v += __ldcg(part + i);
  return block_sum(v, sh);
}

// s[slot] = sum a_i * b_i; with beta set, then beta = SPNEW / SP and SP <- SPNEW
// (matrix.hh:1409-1417), nothing of which once a residual-mode inner solve stopped
__global__ void __launch_bounds__(kCgThreads) k_dot_fin(const double* __restrict__ a, const double* __restrict__ b,
                                                        uint64_t n, double* part, unsigned* cnt, double* s, int slot,
                                                        int beta) {
  __shared__ double sh[32];
  double v = 0.;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v += a[i] * b[i];
  v = block_sum(v, sh);
  if (!cg_last_block(v, part, cnt)) return;
  const double t = cg_sum_partials(part, sh);
  if (threadIdx.x == 0) {
    s[slot] = t;
    if (beta && s[S_DONE] == 0.) {
      s[S_BETA] = s[S_SPNEW] / s[S_SP];
      s[S_SP] = s[S_SPNEW];
    }
    *cnt = 0u;
  }
}

// part[2 blk] = d . Ad, part[2 blk + 1] = x . (0.5 Ax - b)  (matrix.hh:1373-1386)
__global__ void __launch_bounds__(kCgThreads) k_cg_pre(const double* __restrict__ x, const double* __restrict__ Ax,
                                                       const double* __restrict__ b, const double* __restrict__ d,
                                                       const double* __restrict__ Ad, uint64_t n, double* part) {
  __shared__ double sh[32];
  double s0 = 0., s1 = 0.;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    s0 += d[i] * Ad[i];
    s1 += x[i] * (0.5 * Ax[i] - b[i]);
  }
  s0 = block_sum(s0, sh);
  s1 = block_sum(s1, sh);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0;
    part[2 * blockIdx.x + 1] = s1;
  }
}

// x += alpha d; Ax += alpha Ad; r = b - Ax; part[blk] = x . (0.5 Ax - b)
// (matrix.hh:1390-1402), alpha = s[SP] / s[DEN]
__global__ void __launch_bounds__(kCgThreads) k_cg_update(double* __restrict__ x, double* __restrict__ Ax,
                                                          const double* __restrict__ d, const double* __restrict__ Ad,
                                                          const double* __restrict__ b, double* __restrict__ r,
                                                          uint64_t n, const double* s, double* part) {
  __shared__ double sh[32];
  const double alpha = s[S_SP] / s[S_DEN];
  double v = 0.;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double xi = x[i] + alpha * d[i];
    const double ai = Ax[i] + alpha * Ad[i];
    x[i] = xi;
    Ax[i] = ai;
    r[i] = b[i] - ai;
    v += xi * (0.5 * ai - b[i]);
  }
  v = block_sum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// sums `nout` (1 or 2) interleaved partial arrays of `nblk` blocks in a fixed order
// into s[slot0] (and s[slot1])
__global__ void k_finish(const double* part, int nblk, int nout, double* s, int slot0, int slot1) {
  __shared__ double sh[32];
  for (int k = 0; k < nout; k++) {
    double v = 0.;
    for (int i = threadIdx.x; i < nblk; i += blockDim.x) v += part[(size_t)i * nout + k];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) s[k == 0 ? slot0 : slot1] = v;
  }
}

// d = z + beta d
__global__ void __launch_bounds__(kCgThreads) k_cg_dir(double* __restrict__ d, const double* __restrict__ z, uint64_t n,
                                                       const double* s) {
  if (s[S_DONE] != 0.) return;
  const double beta = s[S_BETA];
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    d[i] = z[i] + beta * d[i];
}

// r = b - Ax
__global__ void k_sub(const double* __restrict__ b, const double* __restrict__ Ax, double* __restrict__ r, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - Ax[i];
}

// residual-mode PCG update: x += alpha d, r -= alpha Ad (alpha = SP / DEN), r . r into S_RR,
// then the stopping test by the last block: count the iteration, stop on r . r <= S_THR
// (S_DONE = 1) or a NaN residual (S_DONE = 2).  Nothing once the inner solve stopped: the
// host reads S_DONE only every few iterations, and the iterations launched after the stop
// leave x and r unchanged.
__global__ void __launch_bounds__(kCgThreads) k_pcg_update_fin(double* __restrict__ x, double* __restrict__ r,
                                                               const double* __restrict__ d,
                                                               const double* __restrict__ Ad, uint64_t n, double* s,
                                                               double* part, unsigned* cnt) {
  __shared__ double sh[32];
  if (s[S_DONE] != 0.) return;  // every block: no partial, no ticket
  const double alpha = s[S_SP] / s[S_DEN];
  double v = 0.;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    x[i] += alpha * d[i];
    const double ri = r[i] - alpha * Ad[i];
    r[i] = ri;
    v += ri * ri;
  }
  v = block_sum(v, sh);
  if (!cg_last_block(v, part, cnt)) return;
  const double rr = cg_sum_partials(part, sh);
  if (threadIdx.x == 0) {
    s[S_RR] = rr;
    s[S_ITERS] += 1.;
    if (!(rr == rr))
      s[S_DONE] = 2.;
    else if (rr <= s[S_THR])
      s[S_DONE] = 1.;
    *cnt = 0u;
  }
}

// start of a residual-mode inner solve: stop threshold on r . r, counters cleared
__global__ void k_pcg_start(double* s, double thr) {
  s[S_DONE] = 0.;
  s[S_ITERS] = 0.;
  s[S_THR] = thr;
}

__global__ void k_axpy(double* __restrict__ y, const double* __restrict__ x, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    y[i] += x[i];
}

// count of |b_i| > 1e-10 (multiplyInverse's zero-field shortcut, matrix.hh:193-198)
__global__ void __launch_bounds__(kCgThreads) k_nonzero(const double* __restrict__ b, uint64_t n, double* part) {
  __shared__ double sh[32];
  double c = 0.;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    c += fabs(b[i]) > 1e-10 ? 1. : 0.;
  c = block_sum(c, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = c;
}

}  // namespace pf
