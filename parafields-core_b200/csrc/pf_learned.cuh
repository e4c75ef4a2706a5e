// pf_learned.cuh -- kernels of the learned boundary correction of the torus-inverse
// preconditioner (inference, loss, backward pass, Adam).
//
// The residual-mode CG preconditions the domain-restricted covariance A = R C R^T with the
// torus inverse P0 = R C^+ R^T (one zero-padded FFT round trip).  P0 is exact for the
// circulant but the restriction couples the domain to the padding within a few
// correlation lengths of the faces, which is where P0 A departs from I.  The learned part
// rescales that spectral inverse with a positive diagonal that depends on the distance to
// the faces:
//     M r = D P0 D r,   D = diag(d),   d(x) = exp(psi(t_0(x)) + ... + psi(t_{dim-1}(x))),
// t_i(x) = (distance of cell x to the nearer face along axis i) * h_i / l_i, with l_i the
// correlation length along axis i, and psi a 1 -> H -> 1 tanh network shared by the axes
// (so it transfers across sizes and correlation lengths).  M is symmetric positive definite
// for every parameter value, so plain preconditioned CG stays valid.
//
// Training fits M to (b, x = A^-1 b) pairs produced by plain CG, with e_i = M b_i - x_i
// measured either in the solution norm or in the residual norm (A e_i = A M b_i - b_i, which
// weighs every eigen-direction of A M alike, as the CG convergence does):
//     L_sol = (1/count) sum_i ||e_i||^2 / ||x_i||^2,   L_res = (1/count) sum_i ||A e_i||^2 / ||b_i||^2,
//     dL/dd = sum_i c_i (g_i * v_i + b_i * P0(d * g_i)),
// with v_i = P0(d * b_i), g_i = e_i, c_i = 2/(count ||x_i||^2) (solution norm) or g_i = A A e_i,
// c_i = 2/(count ||b_i||^2) (residual norm; P0 and A are symmetric); d = exp(sum psi) gives
// dL/dpsi_i[m] = sum over the cells with coordinate m on axis i of d * dL/dd.
// Parameters: theta = [w1(H), b1(H), w2(H), b2], psi(t) = sum_h w2_h tanh(w1_h t + b1_h) + b2.
// Every reduction has a fixed order (deterministic training).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pf {

constexpr int kLpThreads = 256;

__device__ __forceinline__ double lp_psi(const double* th, int H, double t) {
  double s = th[3 * H];
  for (int h = 0; h < H; h++) s += th[2 * H + h] * tanh(th[h] * t + th[H + h]);
  return s;
}

// profile entries: psi at every feature value (axes back to back)
__global__ void k_lp_profile(const double* __restrict__ th, int H, const double* __restrict__ feat, int nf,
                             double* __restrict__ prof) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nf) prof[j] = lp_psi(th, H, feat[j]);
}

// d(x) = exp(prof_0[x0] + prof_1[x1] + prof_2[x2]) over the axes in use
__global__ void k_lp_scale(const double* __restrict__ prof, int dim, int n0, int n1, int n2,
                           double* __restrict__ d) {
  const uint64_t n = (uint64_t)n0 * n1 * n2;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const int x0 = (int)(i % n0);
    const uint64_t r = i / n0;
    const int x1 = (int)(r % n1), x2 = (int)(r / n1);
    double s = prof[x0];
    if (dim > 1) s += prof[n0 + x1];
    if (dim > 2) s += prof[n0 + n1 + x2];
    d[i] = exp(s);
  }
}

__global__ void k_lp_mul(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out,
                         uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = a[i] * b[i];
}

// e = d * v - x; per-block partial sums of e.e and x.x (fixed grid: deterministic)
__global__ void __launch_bounds__(kLpThreads) k_lp_err(const double* __restrict__ d, const double* __restrict__ v,
                                                       const double* __restrict__ x, double* __restrict__ e,
                                                       uint64_t n, double* __restrict__ part) {
  __shared__ double s0[kLpThreads], s1[kLpThreads];
  double a = 0., b = 0.;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double ei = d[i] * v[i] - x[i];
    e[i] = ei;
    a += ei * ei;
    b += x[i] * x[i];
  }
  s0[threadIdx.x] = a;
  s1[threadIdx.x] = b;
  __syncthreads();
  for (int w = kLpThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0[0];
    part[2 * blockIdx.x + 1] = s1[0];
  }
}

// per-block partial sums of a.a and c.c (fixed grid: deterministic)
__global__ void __launch_bounds__(kLpThreads) k_lp_sq2(const double* __restrict__ a, const double* __restrict__ c,
                                                       uint64_t n, double* __restrict__ part) {
  __shared__ double s0[kLpThreads], s1[kLpThreads];
  double x = 0., y = 0.;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    x += a[i] * a[i];
    y += c[i] * c[i];
  }
  s0[threadIdx.x] = x;
  s1[threadIdx.x] = y;
  __syncthreads();
  for (int w = kLpThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s0[threadIdx.x] += s0[threadIdx.x + w];
      s1[threadIdx.x] += s1[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = s0[0];
    part[2 * blockIdx.x + 1] = s1[0];
  }
}

// acc[0] += (e.e)/(x.x) / count; acc[1] = 2/((x.x) count) for the backward pass
__global__ void k_lp_err_finish(const double* __restrict__ part, int nblk, double inv_count, double* acc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double a = 0., b = 0.;
  for (int k = 0; k < nblk; k++) {
    a += part[2 * k];
    b += part[2 * k + 1];
  }
  acc[0] += b > 0 ? a / b * inv_count : 0.;
  acc[1] = b > 0 ? 2.0 * inv_count / b : 0.;
}

// g = acc[1] * (e * v + b * w) * d   (dL/dpsi per cell before the plane sums)
__global__ void k_lp_cellgrad(const double* __restrict__ e, const double* __restrict__ v, const double* __restrict__ b,
                              const double* __restrict__ w, const double* __restrict__ d, const double* __restrict__ acc,
                              uint64_t n, double* __restrict__ g) {
  const double c = acc[1];
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    g[i] = c * (e[i] * v[i] + b[i] * w[i]) * d[i];
}

// gprof[j] (+)= sum of g over the plane of profile entry j (block j; fixed order)
__global__ void __launch_bounds__(kLpThreads) k_lp_planesum(const double* __restrict__ g, int dim, int n0, int n1,
                                                            int n2, int accumulate, double* __restrict__ gprof) {
  __shared__ double sh[kLpThreads];
  const int j = blockIdx.x;
  int axis, m;
  if (j < n0) {
    axis = 0;
    m = j;
  } else if (j < n0 + n1) {
    axis = 1;
    m = j - n0;
  } else {
    axis = 2;
    m = j - n0 - n1;
  }
  double s = 0.;
  if (axis < dim) {
    const uint64_t plane = (uint64_t)n0 * n1 * n2 / (axis == 0 ? n0 : axis == 1 ? n1 : n2);
    for (uint64_t k = threadIdx.x; k < plane; k += blockDim.x) {
      uint64_t i;
      if (axis == 0) {
        i = (uint64_t)m + (uint64_t)n0 * k;
      } else if (axis == 1) {
        const uint64_t x0 = k % n0, x2 = k / n0;
        i = x0 + (uint64_t)n0 * (m + (uint64_t)n1 * x2);
      } else {
        i = k + (uint64_t)n0 * n1 * m;
      }
      s += g[i];
    }
  }
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int w = kLpThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) gprof[j] = (accumulate ? gprof[j] : 0.) + sh[0];
}

// dL/dtheta from dL/dpsi at every profile entry (one thread per parameter, fixed order)
__global__ void k_lp_mlp_grad(const double* __restrict__ th, int H, const double* __restrict__ feat,
                              const double* __restrict__ gprof, int nf, double* __restrict__ grad) {
  const int p = threadIdx.x;
  if (p > 3 * H) return;
  double s = 0.;
  for (int j = 0; j < nf; j++) {
    const double gj = gprof[j];
    if (gj == 0.) continue;
    const double t = feat[j];
    double dpsi;
    if (p == 3 * H) {
      dpsi = 1.;
    } else {
      const int h = p % H;
      const double a = tanh(th[h] * t + th[H + h]);
      if (p < H)
        dpsi = th[2 * H + h] * (1. - a * a) * t;
      else if (p < 2 * H)
        dpsi = th[2 * H + h] * (1. - a * a);
      else
        dpsi = a;
    }
    s += gj * dpsi;
  }
  grad[p] = s;
}

// Adam (Kingma and Ba, ICLR 2015) with bias correction, step t >= 1
__global__ void k_lp_adam(double* __restrict__ th, const double* __restrict__ grad, double* __restrict__ m,
                          double* __restrict__ v, int n, double lr, double b1, double b2, double eps, int t) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double g = grad[p];
  m[p] = b1 * m[p] + (1. - b1) * g;
  v[p] = b2 * v[p] + (1. - b2) * g * g;
  const double mh = m[p] / (1. - pow(b1, (double)t)), vh = v[p] / (1. - pow(b2, (double)t));
  th[p] -= lr * mh / (sqrt(vh) + eps);
}

}  // namespace pf
