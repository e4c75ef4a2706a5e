// pf_capi.cu -- C ABI of the single-GPU circulant-embedding path (include/parafields_b200.h).
//
// One translation unit: the plan object, the pass schedules of each Matrix operation
// and the device-side CG.  All kernels live in pf_kernels.cuh / pf_fft.cuh /
// pf_cg.cuh; nothing here runs arithmetic on the host except the tiny CG scalars.
#include <cuda_runtime.h>

#include <algorithm>
#include <complex>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <tuple>
#include <mutex>
#include <thread>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/parafields_b200.h"
#include "pf_cg.cuh"
#include "pf_kernels.cuh"
#include "pf_fastfft.cuh"
#include "pf_pairfft.cuh"
#include "pf_learned.cuh"
#include "../include/parafields_b200/fieldio.hh"

using namespace pf;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static pf_status fail(pf_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return st;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return fail(e_ == cudaErrorMemoryAllocation ? PF_ERR_OOM : PF_ERR_CUDA, "%s: %s (%s:%d)", \
                  #call, cudaGetErrorString(e_), __FILE__, __LINE__);                    \
  } while (0)

#define TRY(...)                   \
  do {                             \
    pf_status s_ = (__VA_ARGS__);  \
    if (s_ != PF_OK) return s_;    \
  } while (0)

// ---------------------------------------------------------------------------
// resolved geometry (RandomFieldTraits::update, fieldtraits.hh:217-314, and the
// default Matrix selection of RandomField, randomfield.hh:153-164)
// ---------------------------------------------------------------------------
struct Geom {
  int dim;
  int n[3], T[3], Ts[3];
  double h[3], ext[3];
  int factor;
  int mb, fb, transposed;
  int T0c;
  uint64_t domain, N, Nc, D, S, noise;
  int C[3];  // cells of the transformed spectrum array (natural layout)
};

static pf_status resolve(const pf_field_desc* d, Geom* g) {
  memset(g, 0, sizeof(*g));
  if (d->dim < 1 || d->dim > 3) return fail(PF_ERR_CONFIG, "dimension must be 1, 2 or 3");
  g->dim = d->dim;
  g->factor = d->periodic ? 1 : d->embedding_factor;
  if (g->factor < 1) return fail(PF_ERR_CONFIG, "embedding.factor must be positive");
  for (int i = 0; i < 3; i++) {
    g->n[i] = 1;
    g->T[i] = 1;
    g->h[i] = 1.;
    g->ext[i] = 1.;
  }
  for (int i = 0; i < d->dim; i++) {
    if (d->cells[i] < 1) return fail(PF_ERR_CONFIG, "grid.cells must be positive");
    g->n[i] = d->cells[i];
    g->ext[i] = d->extensions[i];
    g->h[i] = d->extensions[i] / (double)d->cells[i];
    g->T[i] = g->factor * d->cells[i];
  }
  int mb = d->matrix_backend, fb = d->field_backend;
  if (mb < 0)
    mb = d->dim == 1 ? PF_MATRIX_DFT
                     : ((d->anisotropy == PF_ANISO_NONE || d->anisotropy == PF_ANISO_AXIPARALLEL) ? PF_MATRIX_DCT
                                                                                                 : PF_MATRIX_R2C);
  if (fb < 0) fb = d->dim == 1 ? PF_FIELD_DFT : PF_FIELD_R2C;
  if (mb > 2 || fb > 2) return fail(PF_ERR_CONFIG, "unknown backend");
  if (d->dim == 1 && (mb != PF_MATRIX_DFT || fb != PF_FIELD_DFT))
    return fail(PF_ERR_CONFIG, "dim 1 requires DFTMatrixBackend and DFTFieldBackend");
  if (fb == PF_FIELD_DFT && mb == PF_MATRIX_R2C)
    return fail(PF_ERR_CONFIG, "R2CMatrixBackend cannot serve DFTFieldBackend");
  // matrix.hh:342-347: the DCT/DST field backend needs the DCT matrix backend
  if (fb == PF_FIELD_DCTDST && mb != PF_MATRIX_DCT) return fail(PF_ERR_CONFIG, "DCTDSTFieldBackend requires DCTMatrixBackend");
  for (int i = 0; i < d->dim; i++)
    if (mb == PF_MATRIX_DCT && (g->T[i] % 2))
      return fail(PF_ERR_CONFIG, "DCTMatrixBackend requires an even number of extended cells per dimension");
  if ((mb == PF_MATRIX_R2C || fb == PF_FIELD_R2C) && (g->T[0] % 2))
    return fail(PF_ERR_CONFIG, "the R2C backends need an even number of extended cells in dimension 0");
  g->mb = mb;
  g->fb = fb;
  int t = d->transposed < 0 ? (d->dim > 1) : (d->transposed != 0);
  if (d->dim == 1) t = 0;
  if (d->dim == 2 && (mb == PF_MATRIX_R2C || fb == PF_FIELD_R2C)) t = 0;
  g->transposed = t;
  for (int i = 0; i < 3; i++) g->Ts[i] = g->T[i];
  if (t) std::swap(g->Ts[d->dim - 1], g->Ts[d->dim - 2]);
  g->T0c = g->T[0] / 2 + 1;
  g->domain = 1;
  g->N = 1;
  g->D = 1;
  for (int i = 0; i < d->dim; i++) {
    g->domain *= (uint64_t)g->n[i];
    g->N *= (uint64_t)g->T[i];
    g->D *= (uint64_t)(g->T[i] / 2 + 1);
  }
  g->Nc = g->N / (uint64_t)g->T[0] * (uint64_t)g->T0c;
  g->S = mb == PF_MATRIX_DCT ? g->D : (mb == PF_MATRIX_R2C ? g->Nc : g->N);
  // draws per realization: (rand1, rand2) per stored frequency, or one draw per DCT cell and
  // symmetry type for DCTDSTFieldBackend (matrix.hh:349-366)
  g->noise = fb == PF_FIELD_R2C ? 2 * g->Nc : (fb == PF_FIELD_DCTDST ? (g->D << d->dim) : 2 * g->N);
  for (int i = 0; i < 3; i++) g->C[i] = 1;
  for (int i = 0; i < d->dim; i++)
    g->C[i] = mb == PF_MATRIX_DCT ? g->T[i] / 2 + 1 : (mb == PF_MATRIX_R2C ? (i == 0 ? g->T0c : g->T[i]) : g->T[i]);
  if (g->N > 0xffffffffull) return fail(PF_ERR_CONFIG, "extended domain exceeds 2^32 cells");
  const int c = d->covariance;
  if (c < 0 || c > PF_COV_CUSTOM) return fail(PF_ERR_CONFIG, "covariance structure not known");
  if (c == PF_COV_CUSTOM && d->periodization != PF_PERIODIZATION_CLASSICAL)
    return fail(PF_ERR_CONFIG, "custom covariance values take embedding.periodization = classical only");
  if (c == PF_COV_GAMMA_EXPONENTIAL && (d->exp_gamma < 0. || d->exp_gamma > 2.))
    return fail(PF_ERR_CONFIG, "exponent gamma has to be between 0 and 2");
  if (c == PF_COV_MATERN && d->matern_nu < 0.) return fail(PF_ERR_CONFIG, "matern nu has to be positive");
  if (c == PF_COV_GENERALIZED_CAUCHY) {
    if (d->cauchy_alpha <= 0. || d->cauchy_alpha > 2.)
      return fail(PF_ERR_CONFIG, "generalized Cauchy alpha has to be in range (0,2]");
    if (d->cauchy_beta <= 0.) return fail(PF_ERR_CONFIG, "generalized Cauchy beta has to be positive");
  }
  if (c == PF_COV_CUBIC && d->dim == 3) return fail(PF_ERR_CONFIG, "cubic covariance only applicable in 1D or 2D");
  if (d->anisotropy < 0 || d->anisotropy > 2)
    return fail(PF_ERR_CONFIG, "stochastic.anisotropy must be \"none\", \"axiparallel\" or \"geometric\"");
  if (d->periodization < 0 || d->periodization > 3)
    return fail(PF_ERR_CONFIG,
                "stochastic.periodization must be \"classical\", \"merge\", \"fold\", or \"cofold\"");
  if (d->periodization != PF_PERIODIZATION_CLASSICAL &&
      (d->sigmoid < 0 || d->sigmoid > 1))
    return fail(PF_ERR_CONFIG, "embedding.sigmoid must be \"smooth\" or \"smoothstep\"");
  if (d->periodization == PF_PERIODIZATION_COFOLD && d->cofold_recursions < 0)
    return fail(PF_ERR_CONFIG, "embedding.cofoldRecursions must be non-negative");
  if (d->periodization == PF_PERIODIZATION_MERGE || d->periodization == PF_PERIODIZATION_FOLD) {
    if (d->sigmoid_combine < 0 || d->sigmoid_combine > 2)
      return fail(PF_ERR_CONFIG, "sigmoidCombine must be tensor, radial or radialPlus");
    const int rq = d->periodization == PF_PERIODIZATION_MERGE ? d->merge_recursions : d->fold_recursions;
    if (rq == 99 && c != PF_COV_MATERN && c != PF_COV_GAMMA_EXPONENTIAL &&
        c != PF_COV_GENERALIZED_CAUCHY && c != PF_COV_EXPONENTIAL && c != PF_COV_MATERN32 &&
        c != PF_COV_MATERN52 && c != PF_COV_CAUCHY)
      return fail(PF_ERR_CONFIG, "magic recursions value 99 not implemented for choice of covariance");
  }
  if (d->precision != PF_PREC_F64 && d->precision != PF_PREC_F32) return fail(PF_ERR_CONFIG, "unknown precision");
  return PF_OK;
}

// radix schedule for a pencil length (largest radices first)
static bool make_radices(int L, Radices* r) {
  r->n = 0;
  int x = L;
  while (x % 8 == 0) r->r[r->n++] = 8, x /= 8;
  while (x % 4 == 0) r->r[r->n++] = 4, x /= 4;
  while (x % 2 == 0) r->r[r->n++] = 2, x /= 2;
  static const int odd[] = {3, 5, 7, 11, 13};
  for (int p : odd)
    while (x % p == 0) r->r[r->n++] = p, x /= p;
  return x == 1 && r->n < 20;
}

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------
struct ProfRec {
  const char* name;
  cudaEvent_t e0, e1;
  double bytes;
};

struct pf_learned;

struct pf_plan {
  pf_field_desc desc;
  Geom g;
  cudaStream_t stream = nullptr, own = nullptr;
  int device = 0;
  // spectrum (natural layout, g.S entries)
  bool have_spec = false;
  pf_eig_stats stats{};
  double* lam64 = nullptr;
  double* sq64 = nullptr;
  float* sq32 = nullptr;
  float* lam32 = nullptr;
  void* fac[2][4] = {{nullptr, nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr, nullptr}};
  ScanOut* scan = nullptr;
  double* cof = nullptr;  // cofold: 2 keys, then {active, alpha, beta, offset}
  // workspaces
  void* ws[3] = {nullptr, nullptr, nullptr};
  size_t ws_bytes[3] = {0, 0, 0};
  double* noise_dev = nullptr;
  size_t noise_cap = 0;
  void* io_dev = nullptr;
  size_t io_cap = 0;
  void* io2_dev = nullptr;
  size_t io2_cap = 0;
  // DFT backend spare field (matrix.hh:411-420)
  bool spare_valid = false;
  void* spare = nullptr;
  size_t spare_cap = 0;
  // CG scratch
  CgScratch cg;
  // profiling
  bool prof = false;
  std::vector<ProfRec> recs;
  std::vector<cudaEvent_t> evpool;
  uint64_t launches = 0;
  uint64_t bytes_held = 0;
  // device word mixed into the noise counters (ensembles replaying a captured graph)
  const unsigned* epoch = nullptr;
  // ws[0..1] are lent by an ensemble for one spectrum build (not freed by the plan)
  bool borrowed_ws = false;
  // learned preconditioner of the residual-mode CG (pf_plan_set_preconditioner), not owned
  pf_learned* learned = nullptr;
  // autotuned choices per generation pass (0 noise, 1 middle c2c, 2 c2r): kernel family
  // (0: paired FP32 where eligible, 1: scalar) and resident CTAs per SM of persistent
  // kernels (0: as many as fit); grid_cap is the value of the pass being launched
  int tune_variant[3] = {0, 0, 0};
  int tune_grid[3] = {0, 0, 0};
  int grid_cap = 0;
  // pipelined batches: two streams, each with its own pair of generation workspaces
  cudaStream_t lane[2] = {nullptr, nullptr};
  cudaEvent_t lane_ev[3] = {nullptr, nullptr, nullptr};
  void* ws_b[2] = {nullptr, nullptr};
  size_t ws_b_bytes[2] = {0, 0};
  // batched CG solves: solver lanes, each a plan that shares this plan's spectrum and
  // factor arrays (shared = true: it frees only its own workspaces, scratch and stream)
  bool shared = false;
  std::vector<pf_plan*> lanes;
  // pf_generate_batch to device memory: 0 = realizations alternate over two streams,
  // 1 = stage pipeline (noise passes on one stream, the remaining passes on the other)
  int batch_mode = 0;
  cudaEvent_t stage_ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // 3D generation: the middle and the complex-to-real passes run over this many groups of
  // output planes in turn, so that the intermediate between them (one group, held in a
  // buffer reused by every group) stays in L2 instead of crossing HBM twice; 1 = one group
  int gen_chunks = 1;
  // tile counters of the dynamically ordered paired passes: [kind (0 noise, 1 strided)]
  // [slot], the slot being the batch lane of the realization (0 outside batches), so that
  // kernels that run at the same time never share a counter
  unsigned long long* tile_ctr = nullptr;
  int ctr_slot = 0;
  // residual-mode CG: the next matvec's input d is first updated to z + beta d inside its
  // first pass (set around one matvec call by the CG driver; cg_dir_fusable says when)
  const double* cg_dir_z = nullptr;
  const double* cg_dir_s = nullptr;
  // residual-mode CG: the same matvec's last pass also sums cg_dot_d . out into *cg_dot_dst
  const double* cg_dot_d = nullptr;
  double* cg_dot_dst = nullptr;
};

static pf_status dalloc(pf_plan* P, void** p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(PF_ERR_OOM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
  }
  P->bytes_held += bytes;
  return PF_OK;
}

static void dfree(pf_plan* P, void** p, size_t bytes) {
  if (*p) {
    cudaFree(*p);
    P->bytes_held -= bytes;
    *p = nullptr;
  }
}

static pf_status ensure(pf_plan* P, void** p, size_t* cap, size_t bytes) {
  if (*cap >= bytes && *p) return PF_OK;
  dfree(P, p, *cap);
  *cap = 0;
  TRY(dalloc(P, p, bytes));
  *cap = bytes;
  return PF_OK;
}

static pf_status workspace(pf_plan* P, int i, size_t bytes, void** out) {
  TRY(ensure(P, &P->ws[i], &P->ws_bytes[i], bytes));
  *out = P->ws[i];
  return PF_OK;
}

// Process-wide cache of the constant tables (twiddles, Bluestein chirps, paired-pass
// twiddles): key (device, length, kind) -> device buffer.  Tables are immutable and shared
// by every plan on the device; they live until the process exits.
static std::mutex g_tab_mu;
static std::map<std::tuple<int, int, int>, void*> g_tab;

static void* tab_find(int dev, int L, int kind) {
  std::lock_guard<std::mutex> lk(g_tab_mu);
  auto it = g_tab.find(std::make_tuple(dev, L, kind));
  return it == g_tab.end() ? nullptr : it->second;
}

static pf_status tab_put(int dev, int L, int kind, const void* host, size_t bytes, void** out) {
  void* d = nullptr;
  if (cudaMalloc(&d, bytes) != cudaSuccess) return fail(PF_ERR_OOM, "table of %zu bytes", bytes);
  if (cudaMemcpy(d, host, bytes, cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(d);
    return fail(PF_ERR_CUDA, "table upload failed");
  }
  std::lock_guard<std::mutex> lk(g_tab_mu);
  auto key = std::make_tuple(dev, L, kind);
  auto it = g_tab.find(key);
  if (it != g_tab.end()) {  // another thread built it meanwhile
    cudaFree(d);
    *out = it->second;
  } else {
    g_tab[key] = d;
    *out = d;
  }
  return PF_OK;
}

template <typename T>
static pf_status twiddles(pf_plan* P, int L, const cx<T>** out) {
  if (void* c = tab_find(P->device, L, (int)sizeof(T))) {
    *out = (const cx<T>*)c;
    return PF_OK;
  }
  std::vector<cx<T>> h(L);
  for (int m = 0; m < L; m++) {
    long double a = 2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)L;
    h[m].x = (T)cosl(a);
    h[m].y = (T)-sinl(a);
  }
  void* d = nullptr;
  TRY(tab_put(P->device, L, (int)sizeof(T), h.data(), sizeof(cx<T>) * (size_t)L, &d));
  *out = (const cx<T>*)d;
  return PF_OK;
}

// Bluestein tables of a length-L transform (layout and definitions in pf_fft.cuh, Blue):
// one device buffer chirp | bhat | twM, cached in the twiddle map under key (L, 1000+size)
template <typename T>
static pf_status blue_tables(pf_plan* P, int L, Blue* out) {
  int M = 1;
  while (M < 2 * L - 1) M <<= 1;
  out->M = M;
  const int kind = 1000 + (int)sizeof(T);
  void* d = tab_find(P->device, L, kind);
  if (!d) {
    typedef std::complex<double> C;
    const double pi = 3.141592653589793238462643383279502884;
    std::vector<C> chirp(L), f(M, C(0, 0)), w(M / 2);
    for (int j = 0; j < L; j++) {
      const long long q = ((long long)j * j) % (2LL * L);  // exact phase index
      chirp[j] = std::polar(1.0, -pi * (double)q / (double)L);
    }
    for (int m = 0; m < M / 2; m++) w[m] = std::polar(1.0, -2.0 * pi * (double)m / (double)M);
    int lg = 0;
    while ((1 << lg) < M) lg++;
    auto rev = [&](int i) {
      int r = 0;
      for (int k = 0; k < lg; k++) r |= ((i >> k) & 1) << (lg - 1 - k);
      return r;
    };
    // b = conj(chirp) placed circularly, loaded in bit-reversed order for an in-place DIT
    for (int n = 0; n < L; n++) {
      f[rev(n)] = std::conj(chirp[n]);
      if (n > 0) f[rev(M - n)] = std::conj(chirp[n]);
    }
    for (int len = 2; len <= M; len <<= 1) {
      const int step = M / len;
      for (int i = 0; i < M; i += len)
        for (int k = 0; k < len / 2; k++) {
          const C u = f[i + k], v = f[i + k + len / 2] * w[k * step];
          f[i + k] = u + v;
          f[i + k + len / 2] = u - v;
        }
    }
    std::vector<cx<T>> h((size_t)L + M + M / 2);
    for (int j = 0; j < L; j++) h[j] = cx<T>{(T)chirp[j].real(), (T)chirp[j].imag()};
    for (int m = 0; m < M; m++) {
      const C v = f[rev(m)] / (double)M;
      h[L + m] = cx<T>{(T)v.real(), (T)v.imag()};
    }
    for (int m = 0; m < M / 2; m++) h[L + M + m] = cx<T>{(T)w[m].real(), (T)w[m].imag()};
    TRY(tab_put(P->device, L, kind, h.data(), h.size() * sizeof(cx<T>), &d));
  }
  const cx<T>* base = (const cx<T>*)d;
  out->chirp = base;
  out->bhat = base + L;
  out->twM = base + L + M;
  return PF_OK;
}

// Stockham radices of L, or Bluestein tables (one pencil per tile) when L has a prime
// factor above 13
template <typename T>
static pf_status schedule(pf_plan* P, int L, PassArgs* a) {
  a->blue = Blue{0, nullptr, nullptr, nullptr};
  if (make_radices(L, &a->rad)) return PF_OK;
  if (L > 4096) return fail(PF_ERR_CONFIG, "transform length %d above 4096 has a prime factor above 13", L);
  a->rad.n = 0;
  return blue_tables<T>(P, L, &a->blue);
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
static pf_status prof_begin(pf_plan* P, const char* name, double bytes, ProfRec* rec) {
  rec->name = name;
  rec->bytes = bytes;
  rec->e0 = rec->e1 = nullptr;
  if (!P->prof) return PF_OK;
  for (int k = 0; k < 2; k++) {
    cudaEvent_t e;
    if (!P->evpool.empty()) {
      e = P->evpool.back();
      P->evpool.pop_back();
    } else {
      CK(cudaEventCreate(&e));
    }
    (k ? rec->e1 : rec->e0) = e;
  }
  CK(cudaEventRecord(rec->e0, P->stream));
  return PF_OK;
}

static pf_status prof_end(pf_plan* P, ProfRec* rec) {
  P->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(PF_ERR_CUDA, "launch of %s failed: %s", rec->name, cudaGetErrorString(e));
  if (!P->prof) return PF_OK;
  CK(cudaEventRecord(rec->e1, P->stream));
  P->recs.push_back(*rec);
  return PF_OK;
}

static int pow2_floor(int x) {
  int p = 1;
  while (p * 2 <= x) p *= 2;
  return p;
}

// pencils per tile: two shared buffers of B pencils within ~64 KB
static void tile_params(int L, int elem, bool contig, PassArgs* a) {
  const int pitch = contig ? L + 1 : L;
  int per = 2 * pitch * elem;
  int B = std::max(1, pow2_floor(std::max(1, 65536 / per)));
  B = std::min(B, 16);
  if (!contig && B < 4 && per * 4 <= 160 * 1024) B = 4;
  if (!contig && B < 2 && per * 2 <= 200 * 1024) B = 2;
  a->B = B;
  a->pitch = pitch;
}

static size_t smem_of(const PassArgs& a, bool contig, int elem) {
  return (size_t)2 * a.B * (contig ? a.pitch : a.L) * elem;
}

template <typename K>
static pf_status set_smem(K kernel, size_t smem) {
  // the 48 KB a CTA gets without the attribute include the kernel's static shared memory
  if (smem > 40 * 1024) CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return PF_OK;
}

// complex pencil pass along a strided axis or along contiguous rows
template <typename T, bool CONTIG, class Ld, class Mid, class St>
static pf_status run_pass(pf_plan* P, const char* name, int L, int Lout, long long npencil, long long nouter,
                          int sign, int sign2, Ld ld, Mid mid, St st, double bytes) {
  PassArgs a{};
  a.L = L;
  a.Lout = Lout;
  a.npencil = npencil;
  a.nouter = nouter;
  a.sign = sign;
  a.sign2 = sign2;
  TRY(schedule<T>(P, L, &a));
  tile_params(L, (int)sizeof(cx<T>), CONTIG, &a);
  if (a.blue.M) {
    // Bluestein: one row per tile, or up to 8 interleaved strided pencils (coalesced row
    // segments) while two CTAs still fit on an SM
    a.B = 1;
    if (!CONTIG)
      while (a.B < 8 && (size_t)2 * a.B * (L + a.blue.M) * sizeof(cx<T>) <= 110 * 1024) a.B *= 2;
  }
  const cx<T>* tw = nullptr;
  TRY(twiddles<T>(P, L, &tw));
  // Bluestein: the tile buffer plus the M-element scratch (per pencil) in place of the
  // second buffer
  const size_t smem = a.blue.M ? ((size_t)(CONTIG ? a.pitch : L) + a.blue.M) * a.B * sizeof(cx<T>)
                               : smem_of(a, CONTIG, (int)sizeof(cx<T>));
  if (smem > 227 * 1024) return fail(PF_ERR_CONFIG, "pencil of length %d does not fit in shared memory", L);
  auto kern = k_pass<T, CONTIG, Ld, Mid, St>;
  TRY(set_smem(kern, smem));
  long long grid = CONTIG ? (npencil + a.B - 1) / a.B : ((npencil + a.B - 1) / a.B) * nouter;
  if (grid <= 0) return PF_OK;
  ProfRec rec;
  TRY(prof_begin(P, name, bytes, &rec));
  kern<<<(unsigned)grid, kThreads, smem, P->stream>>>(a, tw, ld, mid, st);
  return prof_end(P, &rec);
}

// real-data passes along dimension 0: rows of T0 = 2L reals <-> L+1 complex
template <typename T, bool R2C, class Ld, class St>
static pf_status run_real_pass(pf_plan* P, const char* name, int T0, int Lout, long long rows, Ld ld, St st,
                               double bytes) {
  PassArgs a{};
  a.L = T0 / 2;
  a.Lout = Lout;
  a.npencil = rows;
  a.nouter = 1;
  a.sign = R2C ? -1 : 1;
  TRY(schedule<T>(P, a.L, &a));
  tile_params(a.L, (int)sizeof(cx<T>), true, &a);
  if (a.blue.M) a.B = 1;
  const cx<T>* tw = nullptr;
  const cx<T>* twT = nullptr;
  TRY(twiddles<T>(P, a.L, &tw));
  TRY(twiddles<T>(P, T0, &twT));
  const size_t smem = smem_of(a, true, (int)sizeof(cx<T>)) + (size_t)a.blue.M * sizeof(cx<T>);
  if (smem > 227 * 1024) return fail(PF_ERR_CONFIG, "row of length %d does not fit in shared memory", T0);
  long long grid = (rows + a.B - 1) / a.B;
  if (grid <= 0) return PF_OK;
  ProfRec rec;
  if constexpr (R2C) {
    auto kern = k_r2c<T, Ld, St>;
    TRY(set_smem(kern, smem));
    TRY(prof_begin(P, name, bytes, &rec));
    kern<<<(unsigned)grid, kThreads, smem, P->stream>>>(a, tw, twT, ld, st);
  } else {
    auto kern = k_c2r<T, Ld, St>;
    TRY(set_smem(kern, smem));
    TRY(prof_begin(P, name, bytes, &rec));
    kern<<<(unsigned)grid, kThreads, smem, P->stream>>>(a, tw, twT, ld, st);
  }
  return prof_end(P, &rec);
}

// bytes from p to the end of the workspace holding it: the bound every access is checked
// against (0 for a pointer outside the workspaces)
static size_t cap_of(const pf_plan* P, const void* p) {
  for (int i = 0; i < 3; i++) {
    const char* b = (const char*)P->ws[i];
    if (b && (const char*)p >= b && (const char*)p < b + P->ws_bytes[i]) return P->ws_bytes[i] - ((const char*)p - b);
  }
  return 0;
}

// compile-time specialised passes for the common lengths; other lengths fall back to
// the runtime-radix kernels above
static int sm_count(pf_plan* P) {
  static int cached[128] = {0};
  const int d = P->device < 128 ? P->device : 0;
  if (!cached[d]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, P->device);
    cached[d] = n > 0 ? n : 148;
  }
  return cached[d];
}

// persistent grid: resident CTAs per SM x SMs, at most one CTA per tile
template <typename K>
static pf_status persistent_grid(pf_plan* P, K kern, size_t smem, long long ntiles, unsigned* grid) {
  int per = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, kThreads, smem));
  if (per < 1) per = 1;
  if (P->grid_cap > 0 && P->grid_cap < per) per = P->grid_cap;
  long long g = (long long)per * sm_count(P);
  if (g > ntiles) g = ntiles;
  *grid = (unsigned)(g > 0 ? g : 1);
  return PF_OK;
}

template <typename T, int SIGN, int SIGN2, class Mid, class St, int L>
static pf_status launch_fpass_pipe(pf_plan* P, const char* name, int Lout, long long npencil, long long nouter,
                                   ArrLoad<cx<T>> ld, Mid mid, St st, double bytes) {
  constexpr int B = fast_B<T, L>();
  PassArgs a{};
  a.L = L;
  a.Lout = Lout;
  a.B = B;
  a.npencil = npencil;
  a.nouter = nouter;
  const cx<T>* tw = nullptr;
  TRY(twiddles<T>(P, L, &tw));
  const size_t smem = fast_smem_pipe<T, L>();
  auto kern = k_fpass_pipe<T, L, B, SIGN, SIGN2, Mid, St>;
  TRY(set_smem(kern, smem));
  const long long ntiles = (npencil + B - 1) / B * nouter;
  if (ntiles <= 0) return PF_OK;
  if (npencil > 0x7fffffffLL) return fail(PF_ERR_CONFIG, "pass %s too large", name);
  unsigned grid = 1;
  TRY(persistent_grid(P, kern, smem, ntiles, &grid));
  ProfRec rec;
  TRY(prof_begin(P, name, bytes, &rec));
  kern<<<grid, kThreads, smem, P->stream>>>(a, tw, ld, mid, st);
  return prof_end(P, &rec);
}

template <typename T, int SIGN, int SIGN2, bool CONTIG, bool PAIR, class Ld, class Mid, class St, int L>
static pf_status launch_fpass(pf_plan* P, const char* name, int Lout, long long npencil, long long nouter, Ld ld,
                              Mid mid, St st, double bytes) {
  if constexpr (!CONTIG && !PAIR && std::is_same<Ld, ArrLoad<cx<T>>>::value)
    return launch_fpass_pipe<T, SIGN, SIGN2, Mid, St, L>(P, name, Lout, npencil, nouter, ld, mid, st, bytes);
  constexpr int B = fast_B<T, L>();
  PassArgs a{};
  a.L = L;
  a.Lout = Lout;
  a.B = B;
  a.npencil = npencil;
  a.nouter = nouter;
  a.sign = SIGN;
  a.sign2 = SIGN2;
  const cx<T>* tw = nullptr;
  TRY(twiddles<T>(P, L, &tw));
  const size_t smem = fast_smem_pass<T, L>();
  auto kern = k_fpass<T, L, B, SIGN, SIGN2, CONTIG, PAIR, Ld, Mid, St>;
  TRY(set_smem(kern, smem));
  const long long tiles = (npencil + B - 1) / B;
  const long long grid = CONTIG ? tiles : tiles * nouter;
  if (grid <= 0) return PF_OK;
  if (grid > 0x7fffffffLL || npencil > 0x7fffffffLL) return fail(PF_ERR_CONFIG, "pass %s too large", name);
  ProfRec rec;
  TRY(prof_begin(P, name, bytes, &rec));
  kern<<<(unsigned)grid, kThreads, smem, P->stream>>>(a, tw, ld, mid, st);
  return prof_end(P, &rec);
}

#define PF_FAST_LENGTHS(X) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024) X(1536) X(2048)

template <typename T, int SIGN, int SIGN2, bool CONTIG, bool PAIR, class Ld, class Mid, class St>
static pf_status run_fpass(pf_plan* P, const char* name, int L, int Lout, long long npencil, long long nouter, Ld ld,
                           Mid mid, St st, double bytes) {
  switch (L) {
#define PF_CASE(LL) \
  case LL:          \
    return launch_fpass<T, SIGN, SIGN2, CONTIG, PAIR, Ld, Mid, St, LL>(P, name, Lout, npencil, nouter, ld, mid, st, bytes);
    PF_FAST_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
      return run_pass<T, CONTIG>(P, name, L, Lout, npencil, nouter, SIGN, SIGN2, ld, mid, st, bytes);
  }
}

template <typename T, bool R2C, class Ld, class St, int L>
static pf_status launch_freal(pf_plan* P, const char* name, int Lout, long long rows, Ld ld, St st, double bytes) {
  constexpr int B = fast_B<T, L>();
  PassArgs a{};
  a.L = L;
  a.Lout = Lout;
  a.B = B;
  a.npencil = rows;
  a.nouter = 1;
  const cx<T>* tw = nullptr;
  const cx<T>* twT = nullptr;
  TRY(twiddles<T>(P, L, &tw));
  TRY(twiddles<T>(P, 2 * L, &twT));
  if constexpr (!R2C && std::is_same<Ld, ArrLoad<cx<T>>>::value) {
    const size_t smemp = fast_smem_real_pipe<T, L>();
    auto kern = k_fc2r_pipe<T, L, B, St>;
    TRY(set_smem(kern, smemp));
    const long long ntiles = (rows + B - 1) / B;
    if (ntiles <= 0) return PF_OK;
    if (rows > 0x7fffffffLL) return fail(PF_ERR_CONFIG, "pass %s too large", name);
    unsigned grid = 1;
    TRY(persistent_grid(P, kern, smemp, ntiles, &grid));
    ProfRec rec;
    TRY(prof_begin(P, name, bytes, &rec));
    kern<<<grid, kThreads, smemp, P->stream>>>(a, tw, twT, ld, st);
    return prof_end(P, &rec);
  }
  const size_t smem = fast_smem_real<T, L>();
  const long long grid = (rows + B - 1) / B;
  if (grid <= 0) return PF_OK;
  if (grid > 0x7fffffffLL || rows > 0x7fffffffLL) return fail(PF_ERR_CONFIG, "pass %s too large", name);
  ProfRec rec;
  if constexpr (R2C) {
    auto kern = k_fr2c<T, L, B, Ld, St>;
    TRY(set_smem(kern, smem));
    TRY(prof_begin(P, name, bytes, &rec));
    kern<<<(unsigned)grid, kThreads, smem, P->stream>>>(a, tw, twT, ld, st);
  } else {
    auto kern = k_fc2r<T, L, B, Ld, St>;
    TRY(set_smem(kern, smem));
    TRY(prof_begin(P, name, bytes, &rec));
    kern<<<(unsigned)grid, kThreads, smem, P->stream>>>(a, tw, twT, ld, st);
  }
  return prof_end(P, &rec);
}

template <typename T, bool R2C, class Ld, class St>
static pf_status run_freal(pf_plan* P, const char* name, int T0, int Lout, long long rows, Ld ld, St st,
                           double bytes) {
  switch (T0 / 2) {
#define PF_CASE(LL) \
  case LL:          \
    return launch_freal<T, R2C, Ld, St, LL>(P, name, Lout, rows, ld, st, bytes);
    PF_FAST_LENGTHS(PF_CASE)
#undef PF_CASE
    default:
      return run_real_pass<T, R2C>(P, name, T0, Lout, rows, ld, st, bytes);
  }
}

// row pitch of the half-spectrum work arrays: T0/2+1 rounded up to 8 complex, so every
// B-wide segment of a strided pass starts on a 64-byte boundary
static int half_pitch(const Geom& g) { return (g.T0c + 7) / 8 * 8; }

template <typename S>
static ArrLoad<S> arr_load(const pf_plan* P, const void* p, long long jstride, long long ostride, long long rowstride,
                           int Lin) {
  ArrLoad<S> l;
  l.ptr = (const S*)p;
  l.n = (unsigned)std::min<size_t>(cap_of(P, p) / sizeof(S), 0xffffffffu);
  l.jstride = jstride;
  l.ostride = ostride;
  l.rowstride = rowstride;
  l.Lin = Lin;
  return l;
}

template <typename S>
static ArrStore<S> arr_store(const pf_plan* P, void* p, long long jstride, long long ostride, long long rowstride) {
  ArrStore<S> s;
  s.ptr = (S*)p;
  s.n = (unsigned)std::min<size_t>(cap_of(P, p) / sizeof(S), 0xffffffffu);
  s.jstride = jstride;
  s.ostride = ostride;
  s.rowstride = rowstride;
  return s;
}

static unsigned grid_for(uint64_t n) {
  uint64_t g = (n + kThreads - 1) / kThreads;
  if (g > 148ull * 16) g = 148ull * 16;
  if (g == 0) g = 1;
  return (unsigned)g;
}

// ---------------------------------------------------------------------------
// spectrum: fillTransformedMatrix (matrix.hh:223-318)
// ---------------------------------------------------------------------------
// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on P_n from the
// asymptotic initial guesses), for the fold integrals
static void gauss_legendre(int n, double* x, double* w) {
  const double pi = 3.141592653589793238462643383279502884;
  for (int i = 0; i < n; i++) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5)), dp = 1.;
    for (int it = 0; it < 100; it++) {
      double p0 = 1., p1 = z;
      for (int k = 2; k <= n; k++) {
        const double p2 = ((2. * k - 1.) * z * p1 - (k - 1.) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1.);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = z;
    w[i] = 2. / ((1. - z * z) * dp * dp);
  }
}

static CovParams cov_params(const pf_field_desc* d, const Geom& g) {
  CovParams c{};
  c.dim = g.dim;
  c.cov = d->covariance;
  c.aniso = d->anisotropy;
  for (int i = 0; i < 3; i++) {
    c.T[i] = g.T[i];
    c.h[i] = g.h[i];
    c.half[i] = 0.5 * g.ext[i] * (double)g.factor;
    c.wrap[i] = g.ext[i] * (double)g.factor;
  }
  const double* cl = d->corr_length;
  if (d->anisotropy == PF_ANISO_NONE) {
    c.geo[0] = 1. / cl[0];  // covariance.hh:33-37
  } else if (d->anisotropy == PF_ANISO_AXIPARALLEL) {
    for (int i = 0; i < g.dim; i++) c.geo[i] = 1. / cl[i];  // covariance.hh:62-67
  } else {  // cofactor inverse, covariance.hh:94-128
    double* m = c.geo;
    if (g.dim == 3) {
      m[0] = cl[4] * cl[8] - cl[5] * cl[7];
      m[1] = cl[2] * cl[7] - cl[1] * cl[8];
      m[2] = cl[1] * cl[5] - cl[2] * cl[4];
      m[3] = cl[5] * cl[6] - cl[3] * cl[8];
      m[4] = cl[0] * cl[8] - cl[2] * cl[6];
      m[5] = cl[2] * cl[3] - cl[0] * cl[5];
      m[6] = cl[3] * cl[7] - cl[4] * cl[6];
      m[7] = cl[1] * cl[6] - cl[0] * cl[7];
      m[8] = cl[0] * cl[4] - cl[1] * cl[3];
      const double det = cl[0] * (cl[4] * cl[8] - cl[5] * cl[7]) - cl[1] * (cl[3] * cl[8] - cl[5] * cl[6]) +
                         cl[2] * (cl[3] * cl[7] - cl[4] * cl[6]);
      for (int i = 0; i < 9; i++) m[i] /= det;
    } else if (g.dim == 2) {
      m[0] = cl[3];
      m[1] = -cl[1];
      m[2] = -cl[2];
      m[3] = cl[0];
      const double det = cl[0] * cl[3] - cl[1] * cl[2];
      for (int i = 0; i < 4; i++) m[i] /= det;
    } else {
      m[0] = 1. / cl[0];
    }
  }
  c.variance = d->variance;
  if (d->covariance == PF_COV_GAMMA_EXPONENTIAL) c.p0 = d->exp_gamma;
  if (d->covariance == PF_COV_GENERALIZED_CAUCHY) {
    c.p0 = d->cauchy_alpha;
    c.p1 = d->cauchy_beta;
  }
  if (d->covariance == PF_COV_MATERN) {  // covariance.hh:515-520
    c.p0 = std::sqrt(2. * d->matern_nu);
    c.p1 = std::pow(2., 1. - d->matern_nu);
    c.p2 = std::tgamma(d->matern_nu);
    c.p3 = d->matern_nu;
  }
  c.per = d->periodization;
  c.sig = d->sigmoid;
  c.radial = d->sigmoid_combine != PF_COMBINE_TENSOR;
  c.plus = d->sigmoid_combine == PF_COMBINE_RADIAL_PLUS;
  c.factor = (double)g.factor;
  c.sstart = d->sigmoid_start;
  c.send = d->sigmoid_end < 0 ? (double)g.factor - 1. : d->sigmoid_end;
  for (int i = 0; i < 3; i++) c.ext[i] = g.ext[i];
  int rec = d->periodization == PF_PERIODIZATION_FOLD ? d->fold_recursions : d->merge_recursions;
  if (d->periodization == PF_PERIODIZATION_COFOLD) rec = d->cofold_recursions;  // no magic value
  c.fold_beta = d->fold_max_factor * 0.5 * (double)g.factor / std::sqrt((double)g.dim);  // matrix.hh:839-842
  gauss_legendre(kFoldNodes, c.gl_x, c.gl_w);
  if (rec == 99) {  // matrix.hh:693-717, 803-827
    const double hd = (double)g.dim / 2.;
    switch (d->covariance) {
      case PF_COV_MATERN: rec = (int)std::floor(d->matern_nu * 2. + hd); break;
      case PF_COV_GAMMA_EXPONENTIAL: rec = (int)std::floor(d->exp_gamma + hd); break;
      case PF_COV_GENERALIZED_CAUCHY: rec = (int)std::floor(d->cauchy_alpha + hd); break;
      case PF_COV_EXPONENTIAL: rec = 2; break;
      case PF_COV_MATERN32: rec = 4; break;
      case PF_COV_MATERN52: rec = 6; break;
      case PF_COV_CAUCHY: rec = 3; break;
      default: rec = 0;
    }
  }
  c.rec = rec;
  return c;
}

static pf_status spectrum_alloc(pf_plan* P) {
  const uint64_t S = P->g.S;
  if (!P->lam64) {
    TRY(dalloc(P, (void**)&P->lam64, S * 8));
    TRY(dalloc(P, (void**)&P->sq64, S * 8));
    TRY(dalloc(P, (void**)&P->sq32, S * 4));
    TRY(dalloc(P, (void**)&P->lam32, S * 4));
    TRY(dalloc(P, (void**)&P->scan, sizeof(ScanOut)));
  }
  return PF_OK;
}

// vals != NULL: the matrix cells were computed by the caller (device array, dimension 0
// fastest: prod(T_i/2+1) values for the DCT matrix, prod(T_i) otherwise) and replace the
// covariance evaluation of the first pass; periodization is then the caller's
static pf_status build_spectrum(pf_plan* P, const double* vals = nullptr) {
  const Geom& g = P->g;
  const pf_field_desc* d = &P->desc;
  for (pf_plan* l : P->lanes) pf_plan_destroy(l);  // they share the factor arrays freed below
  P->lanes.clear();
  if (!vals && d->covariance == PF_COV_CUSTOM)  // matrix.hh:227-230
    return fail(PF_ERR_STATE, "you need to call fillMatrix with your covariance class as parameter");
  TRY(spectrum_alloc(P));
  for (int a = 0; a < 2; a++)
    for (int o = 0; o < 4; o++)
      if (P->fac[a][o]) {
        cudaFree(P->fac[a][o]);
        P->bytes_held -= g.S * (a == 0 ? 8 : 4);
        P->fac[a][o] = nullptr;
      }
  CovRowLoad cl;
  cl.c = cov_params(d, g);
  const int dim = g.dim;
  if (d->periodization == PF_PERIODIZATION_COFOLD && !vals) {
    // statistics of the classical values over the matrix cells, then alpha, beta and the
    // offset on the device; the spectrum passes below apply the value map
    if (!P->cof) TRY(dalloc(P, (void**)&P->cof, 6 * sizeof(double)));
    static const unsigned long long init[2] = {~0ull, 0ull};
    CK(cudaMemcpyAsync(P->cof, init, sizeof(init), cudaMemcpyHostToDevice, P->stream));
    int C[3] = {1, 1, 1};
    for (int i = 0; i < dim; i++) C[i] = g.mb == PF_MATRIX_DCT ? g.T[i] / 2 + 1 : g.T[i];
    CovParams sc = cl.c;
    sc.per = 0;
    unsigned long long* keys = (unsigned long long*)P->cof;
    ProfRec rec;
    TRY(prof_begin(P, "spec_cofold_stats", 0.0, &rec));
    k_cofold_stats<<<grid_for((uint64_t)C[0] * C[1] * C[2]), kThreads, 0, P->stream>>>(sc, C[0], C[1], C[2], keys);
    k_cofold_finish<<<1, 32, 0, P->stream>>>(sc, d->cofold_max_factor, keys, P->cof + 2);
    TRY(prof_end(P, &rec));
    cl.c.cof = P->cof + 2;
  }
  void *A = nullptr, *Bw = nullptr;
  double2* spec = nullptr;
  const uint64_t full = g.mb == PF_MATRIX_DFT ? g.N : g.Nc;
  TRY(workspace(P, 0, full * sizeof(double2), &A));
  TRY(workspace(P, 1, full * sizeof(double2), &Bw));
  cl.rowmod = g.T[1];
  if (g.mb == PF_MATRIX_DCT) {
    // Even torus in every dimension (DCT-I, dctmatrixbackend.hh:240-272): the covariance is
    // evaluated only on the prod(T_i/2+1) non-mirrored cells; each later pass reads its
    // axis through the mirror j -> T - j and keeps the T/2+1 outputs the DCT-I needs.
    const int T0c = g.T0c;
    const int D1 = dim >= 2 ? g.T[1] / 2 + 1 : 1, D2 = dim >= 3 ? g.T[2] / 2 + 1 : 1;
    const long long rows = (long long)D1 * D2;
    cl.rowmod = D1;
    if (vals)
      TRY((run_freal<double, true>(P, "spec_r2c_vals", g.T[0], T0c, rows,
                                   ValRowLoad{vals, g.T[0], T0c, 1, (unsigned long long)g.D},
                                   arr_store<double2>(P, A, 1, 0, T0c), rows * T0c * 24.0)));
    else
      TRY((run_freal<double, true>(P, "spec_r2c_cov", g.T[0], T0c, rows, cl, arr_store<double2>(P, A, 1, 0, T0c),
                                   rows * T0c * 16.0)));
    spec = (double2*)A;
    if (dim >= 2) {
      MirrorLoad<double2> ml{(const double2*)A, (unsigned)T0c, (unsigned)((long long)T0c * D1), 1u,
                             (unsigned)std::min<size_t>(cap_of(P, A) / sizeof(double2), 0xffffffffu), g.T[1]};
      TRY((run_fpass<double, -1, -1, false, false>(P, "spec_c2c_d1", g.T[1], D1, T0c, D2, ml, NoMid(),
                                                   arr_store<double2>(P, Bw, T0c, (long long)T0c * D1, 1),
                                                   (double)T0c * D2 * (D1 + D1) * 16.0)));
      spec = (double2*)Bw;
      if (dim == 3) {
        const long long inner = (long long)T0c * D1;
        MirrorLoad<double2> m2{(const double2*)Bw, (unsigned)inner, 0u, 1u,
                               (unsigned)std::min<size_t>(cap_of(P, Bw) / sizeof(double2), 0xffffffffu), g.T[2]};
        TRY((run_fpass<double, -1, -1, false, false>(P, "spec_c2c_d2", g.T[2], D2, inner, 1, m2, NoMid(),
                                                     arr_store<double2>(P, A, inner, 0, 1),
                                                     (double)inner * (D2 + D2) * 16.0)));
        spec = (double2*)A;
      }
    }
  } else if (g.mb == PF_MATRIX_R2C) {
    const bool dct = false;
    const int T0c = g.T0c;
    const long long rows = (long long)(g.N / (uint64_t)g.T[0]);
    // dimension 0: covariance evaluation fused into the R2C load
    if (vals)
      TRY((run_freal<double, true>(P, "spec_r2c_vals", g.T[0], T0c, rows,
                                   ValRowLoad{vals, g.T[0], g.T[0], 0, (unsigned long long)g.N},
                                   arr_store<double2>(P, A, 1, 0, T0c), rows * (T0c * 16.0 + g.T[0] * 8.0))));
    else
      TRY((run_freal<double, true>(P, "spec_r2c_cov", g.T[0], T0c, rows, cl, arr_store<double2>(P, A, 1, 0, T0c),
                                   rows * T0c * 16.0)));
    spec = (double2*)A;
    if (dim >= 2) {
      const int L1 = g.T[1], L1o = dct ? g.T[1] / 2 + 1 : g.T[1];
      const long long outer = dim == 3 ? g.T[2] : 1;
      TRY((run_fpass<double, -1, -1, false, false>(P, "spec_c2c_d1", L1, L1o, T0c, outer,
                                                   arr_load<double2>(P, A, T0c, (long long)T0c * L1, 1, L1), NoMid(),
                                                   arr_store<double2>(P, Bw, T0c, (long long)T0c * L1o, 1),
                                                   (double)T0c * outer * (L1 + L1o) * 16.0)));
      spec = (double2*)Bw;
      if (dim == 3) {
        const int L2 = g.T[2], L2o = dct ? g.T[2] / 2 + 1 : g.T[2];
        const long long inner = (long long)T0c * L1o;
        TRY((run_fpass<double, -1, -1, false, false>(P, "spec_c2c_d2", L2, L2o, inner, 1,
                                                     arr_load<double2>(P, Bw, inner, 0, 1, L2), NoMid(),
                                                     arr_store<double2>(P, A, inner, 0, 1),
                                                     (double)inner * (L2 + L2o) * 16.0)));
        spec = (double2*)A;
      }
    }
  } else {  // DFT matrix: complex torus, every axis complex (dftmatrixbackend.hh:209-238)
    const long long rows = (long long)(g.N / (uint64_t)g.T[0]);
    if (vals)
      TRY((run_pass<double, true>(P, "spec_c2c_d0", g.T[0], g.T[0], rows, 1, -1, -1,
                                  ValRowLoad{vals, g.T[0], g.T[0], 0, (unsigned long long)g.N}, NoMid(),
                                  arr_store<double2>(P, A, 1, 0, g.T[0]), rows * g.T[0] * 24.0)));
    else
      TRY((run_pass<double, true>(P, "spec_c2c_d0", g.T[0], g.T[0], rows, 1, -1, -1, cl, NoMid(),
                                  arr_store<double2>(P, A, 1, 0, g.T[0]), rows * g.T[0] * 16.0)));
    spec = (double2*)A;
    void* src = A;
    void* dst = Bw;
    long long inner = g.T[0];
    for (int ax = 1; ax < dim; ax++) {
      const int L = g.T[ax];
      long long outer = (long long)(g.N / (uint64_t)inner / (uint64_t)L);
      TRY((run_pass<double, false>(P, ax == 1 ? "spec_c2c_d1" : "spec_c2c_d2", L, L, inner, outer, -1, -1,
                                   arr_load<double2>(P, src, inner, inner * L, 1, L), NoMid(),
                                   arr_store<double2>(P, dst, inner, inner * L, 1), (double)g.N * 32.0)));
      spec = (double2*)dst;
      std::swap(src, dst);
      inner *= L;
    }
  }
  // eigenvalue scan, clamp, square roots
  static const ScanOut scan_init = {0u, 0u, 0u, 0u, ~0ull};  // min key starts at the largest key
  CK(cudaMemcpyAsync(P->scan, &scan_init, sizeof(ScanOut), cudaMemcpyHostToDevice, P->stream));
  ScanArgs sa{};
  sa.spec = spec;
  for (int i = 0; i < 3; i++) {
    sa.C[i] = g.C[i];
    sa.Ts[i] = g.Ts[i];
  }
  sa.transposed = g.transposed;
  sa.dim = dim;
  sa.faithful = (g.mb == PF_MATRIX_R2C && d->eigen_check == PF_EIGCHECK_REFERENCE) ? 1 : 0;
  sa.count = g.S;
  sa.N = (double)(unsigned int)g.N;
  sa.threshold = d->threshold;
  sa.lam = P->lam64;
  sa.sq64 = P->sq64;
  sa.sq32 = P->sq32;
  sa.lam32 = P->lam32;
  sa.out = P->scan;
  {
    ProfRec rec;
    TRY(prof_begin(P, "spec_scan", g.S * (16.0 + 24.0), &rec));
    k_scan<<<grid_for(g.S), kThreads, 0, P->stream>>>(sa);
    TRY(prof_end(P, &rec));
  }
  ScanOut so;
  CK(cudaMemcpyAsync(&so, P->scan, sizeof(so), cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  P->stats.small = so.small;
  P->stats.zero = so.zero;
  P->stats.negative = so.negative;
  P->stats.pad_ = 0;
  unsigned long long k = so.minkey;
  unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double mn;
  memcpy(&mn, &b, 8);
  P->stats.smallest = mn;
  // release the FP64 spectrum workspaces: they are the largest buffers of the plan
  // (borrowed ones belong to the caller: an ensemble lends one pair to all its fields)
  if (P->borrowed_ws) {
    P->ws[0] = P->ws[1] = nullptr;
    P->ws_bytes[0] = P->ws_bytes[1] = 0;
    P->borrowed_ws = false;
  } else {
    dfree(P, &P->ws[0], P->ws_bytes[0]);
    P->ws_bytes[0] = 0;
    dfree(P, &P->ws[1], P->ws_bytes[1]);
    P->ws_bytes[1] = 0;
  }
  if (P->stats.negative > 0 && !d->approximate) {
    P->have_spec = false;
    return fail(PF_ERR_NEG_EIGEN, "negative eigenvalues in covariance matrix");
  }
  P->have_spec = true;
  return PF_OK;
}

// reads and clears the kernels' bounds-violation flag (synchronizes the stream)
static pf_status check_bounds(pf_plan* P, pf_status st) {
  unsigned int flag = 0;
  CK(cudaMemcpyFromSymbolAsync(&flag, g_bounds_error, sizeof(flag), 0, cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  if (flag) {
    const unsigned int zero = 0;
    CK(cudaMemcpyToSymbolAsync(g_bounds_error, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, P->stream));
    CK(cudaStreamSynchronize(P->stream));
    if (flag & 2u) return fail(PF_ERR_TIMEOUT, "a kernel's bounded wait for its tile copies gave up");
    return fail(PF_ERR_CUDA, "internal error: a kernel computed an index outside its buffer (access skipped)");
  }
  return st;
}

static pf_status ensure_spectrum(pf_plan* P) {
  if (P->have_spec) return PF_OK;
  return build_spectrum(P);
}

template <typename T>
static pf_status factor_array(pf_plan* P, int op, const T** out) {
  const int a = sizeof(T) == 8 ? 0 : 1;
  if (!P->fac[a][op]) {
    TRY(dalloc(P, &P->fac[a][op], P->g.S * sizeof(T)));
    ProfRec rec;
    TRY(prof_begin(P, "factors", P->g.S * (8.0 + sizeof(T)), &rec));
    k_factors<T><<<grid_for(P->g.S), kThreads, 0, P->stream>>>(P->lam64, P->g.S, 1.0 / (double)P->g.N, op,
                                                               (T*)P->fac[a][op]);
    TRY(prof_end(P, &rec));
  }
  *out = (const T*)P->fac[a][op];
  return PF_OK;
}

#include "pf_pair_host.inc"

// ---------------------------------------------------------------------------
// generation: generateField (matrix.hh:330-421)
// ---------------------------------------------------------------------------
// stages: bit 0 the noise pass (noise, scaling, backward transform along the last axis into
// workspace 0), bit 1 the remaining passes (workspace 0 -> field); both for one realization
template <typename T, typename S>
static pf_status gen_r2c(pf_plan* P, const double* noise_dev, uint64_t seed, S* out, int transform, int stages = 3) {
  const Geom& g = P->g;
  const int T0c = g.T0c, P0 = half_pitch(g);
  R2CNoise nz{};
  nz.dim = g.dim;
  for (int i = 0; i < 3; i++) nz.ext[i] = g.T[i];
  nz.T0c = T0c;
  nz.transposed = g.transposed;
  nz.dct = g.mb == PF_MATRIX_DCT ? 1 : (g.mb == PF_MATRIX_DFT ? 2 : 0);
  nz.D0 = g.T[0] / 2 + 1;
  nz.D1 = g.T[1] / 2 + 1;
  nz.sq = sizeof(T) == 8 ? (const void*)P->sq64 : (const void*)P->sq32;
  nz.noise = noise_dev;
  nz.seed = seed;
  nz.epoch = P->epoch;
  nz.nsq = (long long)g.S;
  nz.nnoise = (long long)g.noise;
  nz.Tl = g.T[g.dim - 1];
  const double e = sizeof(cx<T>);
  const double noise_b = noise_dev ? 16.0 : 0.0;
  const double lam_b = sizeof(T);
  const int last = g.dim - 1;
  const int Tl = g.T[last];
  void* W1 = nullptr;
  if (g.dim == 2) {
    TRY(workspace(P, 0, sizeof(cx<T>) * (size_t)P0 * g.n[1], &W1));
  } else {
    TRY(workspace(P, 0, sizeof(cx<T>) * (size_t)P0 * g.T[1] * g.n[2], &W1));
  }
  // backward along the last dimension first, noise scaling fused into the load and the
  // output pruned to the domain extent n_last (pencils: k0 x k1)
  const long long outer = g.dim == 3 ? g.T[1] : 1;
  const long long jst = g.dim == 3 ? (long long)P0 * g.T[1] : P0;
  // compulsory bytes: the spectrum read once (mirrored and repeated reads of a stored
  // eigenvalue hit L2), the noise buffer if any, the kept output planes written once
  const double b1 = (double)g.S * lam_b + (double)T0c * outer * (Tl * noise_b + (double)g.n[last] * e);
  constexpr bool F32 = std::is_same<T, float>::value && std::is_same<S, float>::value;
  struct CapReset {
    pf_plan* P;
    ~CapReset() { P->grid_cap = 0; }
  } cap_reset{P};
  P->grid_cap = P->tune_grid[0];
  if (!(stages & 1)) {
  } else if (F32 && P->tune_variant[0] == 0 && (p2_length(Tl) || p2_length3(Tl)) && p2_view_ok(W1, jst, P0, outer))
    TRY(p2_noise(P, "gen_noise_last", Tl, g.n[last], T0c, outer, nz, p2_store(P, W1, jst, P0, T0c), b1));
  else if (Tl % 2 == 0)
    TRY((run_fpass<T, +1, +1, false, true>(P, "gen_noise_last", Tl, g.n[last], T0c, outer, nz, NoMid(),
                                           arr_store<cx<T>>(P, W1, jst, P0, 1), b1)));
  else
    TRY((run_fpass<T, +1, +1, false, false>(P, "gen_noise_last", Tl, g.n[last], T0c, outer, nz, NoMid(),
                                            arr_store<cx<T>>(P, W1, jst, P0, 1), b1)));
  if (!(stages & 2)) return PF_OK;
  // the complex-to-real rows of `nrows` (pencil index j1 + n1 * plane) from `src` into
  // the field rows starting at `dst`
  auto c2r_rows = [&](const void* src, S* dst, long long nrows) -> pf_status {
    const double b3 = (double)nrows * (T0c * e + g.n[0] * sizeof(S));
    P->grid_cap = P->tune_grid[2];
    const size_t left = (size_t)(g.domain - (size_t)(dst - out));
    if constexpr (F32) {
      if (P->tune_variant[2] != 1 && g.T[0] % 2 == 0 && (p2_length(g.T[0] / 2) || p2_length3(g.T[0] / 2))) {
        P2RowLoad rl;
        rl.ptr = (const float2*)src;
        rl.rowstride = (unsigned)P0;
        rl.n = (unsigned)std::min<size_t>(cap_of(P, src) / sizeof(float2), 0xffffffffu);
        rl.Lin = T0c;
        rl.np = (int)nrows;
        P2FieldStore ps;
        ps.out = (float*)dst;
        ps.n0 = g.n[0];
        ps.transform = transform;
        ps.boxcox = (float)P->desc.boxcox_lambda;
        ps.n = (unsigned)left;
        ps.np = (int)nrows;
        ps.Lout = g.n[0];
        ps.vec = (g.n[0] % 2 == 0 && ((uintptr_t)dst & 7u) == 0) ? 1 : 0;
        if (P->tune_variant[2] == 2 && p2_bulk_ok(rl, g.T[0] / 2))  // rows staged by bulk copies
          return p2_c2r_bulk(P, "gen_c2r_d0_bulk", g.T[0] / 2, g.n[0], nrows, rl, ps, b3);
        return p2_c2r(P, "gen_c2r_d0", g.T[0] / 2, g.n[0], nrows, rl, ps, b3);
      }
    }
    FieldRowStore<S> fr{dst, g.n[0], transform, P->desc.boxcox_lambda, (unsigned)left};
    return run_freal<T, false>(P, "gen_c2r_d0", g.T[0], g.n[0], nrows,
                               arr_load<cx<T>>(P, src, 1, 0, P0, T0c), fr, b3);
  };
  if (g.dim == 2) return c2r_rows(W1, out, g.n[1]);
  // 3D: the middle pass (along axis 1, output pruned to n1) and the complex-to-real rows
  // run over groups of output planes (axis-2 index) in turn; the middle pass's output for
  // one group lives in workspace 1, which every group reuses (small groups keep it in L2)
  const int n2 = g.n[2];
  const int groups = std::max(1, std::min(P->gen_chunks, n2));
  const int gp = (n2 + groups - 1) / groups;  // planes per group
  void* W2 = nullptr;
  TRY(workspace(P, 1, sizeof(cx<T>) * (size_t)P0 * g.n[1] * gp, &W2));
  const long long w1_plane = (long long)P0 * g.T[1], w2_plane = (long long)P0 * g.n[1];
  for (int z0 = 0; z0 < n2; z0 += gp) {
    const int nz = std::min(gp, n2 - z0);
    void* src = (char*)W1 + sizeof(cx<T>) * (size_t)w1_plane * z0;
    const double b2 = (double)T0c * nz * (g.T[1] + g.n[1]) * e;
    P->grid_cap = P->tune_grid[1];
    const bool p2ok = F32 && (p2_length(g.T[1]) || p2_length3(g.T[1])) && p2_view_ok(src, P0, w1_plane, nz) &&
                      p2_view_ok(W2, P0, w2_plane, nz);
    const P2ArrLoad l1 = p2_load(P, src, P0, w1_plane, g.T[1], T0c);
    if (p2ok && P->tune_variant[1] == 2 && p2_length(g.T[1]) && p2_tma_ok(P, l1, nz))  // tiles staged by TMA
      TRY(p2_c2c_tma<+1>(P, "gen_c2c_d1_tma", g.T[1], g.n[1], T0c, nz, l1, p2_store(P, W2, P0, w2_plane, T0c), b2));
    else if (p2ok && P->tune_variant[1] != 1)
      TRY(p2_c2c<+1>(P, "gen_c2c_d1", g.T[1], g.n[1], T0c, nz, l1, p2_store(P, W2, P0, w2_plane, T0c), b2));
    else
      TRY((run_fpass<T, +1, +1, false, false>(P, "gen_c2c_d1", g.T[1], g.n[1], T0c, nz,
                                              arr_load<cx<T>>(P, src, P0, w1_plane, 1, g.T[1]), NoMid(),
                                              arr_store<cx<T>>(P, W2, P0, w2_plane, 1), b2)));
    TRY(c2r_rows(W2, out + (size_t)g.n[0] * g.n[1] * z0, (long long)g.n[1] * nz));
  }
  return PF_OK;
}

// DFT field backend: complex noise on the whole torus, backward c2c on every axis,
// Re -> field, Im -> spare field (dftfieldbackend.hh:186-280, 380-446)
template <typename T, typename S>
static pf_status gen_dft(pf_plan* P, const double* noise_dev, uint64_t seed, S* out, S* spare, int transform) {
  const Geom& g = P->g;
  DFTNoise nz{};
  nz.dim = g.dim;
  for (int i = 0; i < 3; i++) {
    nz.ext[i] = g.T[i];
    nz.Ts[i] = g.Ts[i];
  }
  nz.transposed = g.transposed;
  nz.mat = g.mb == PF_MATRIX_DCT ? 0 : 2;
  nz.sq = sizeof(T) == 8 ? (const void*)P->sq64 : (const void*)P->sq32;
  nz.noise = noise_dev;
  nz.seed = seed;
  nz.nsq = (long long)g.S;
  nz.nnoise = (long long)g.noise;
  SplitStore<S> ss{out, spare, g.n[0], transform, P->desc.boxcox_lambda, (unsigned)g.domain};
  const double e = sizeof(cx<T>);
  if (g.dim == 1) {
    return run_pass<T, true>(P, "gen_dft_d0", g.T[0], g.n[0], 1, 1, +1, +1, nz, NoMid(), ss,
                             (double)g.T[0] * (16.0 + sizeof(T)) + 2.0 * g.n[0] * sizeof(S));
  }
  void *W1 = nullptr, *W2 = nullptr;
  const int last = g.dim - 1;
  const long long inner = (long long)(g.N / (uint64_t)g.T[last]);
  TRY(workspace(P, 0, sizeof(cx<T>) * (size_t)inner * g.n[last], &W1));
  TRY(run_pass<T, false>(P, "gen_dft_noise", g.T[last], g.n[last], inner, 1, +1, +1, nz, NoMid(),
                         arr_store<cx<T>>(P, W1, inner, 0, 1), (double)inner * (g.T[last] * 16.0 + g.n[last] * e)));
  void* cur = W1;
  if (g.dim == 3) {
    TRY(workspace(P, 1, sizeof(cx<T>) * (size_t)g.T[0] * g.n[1] * g.n[2], &W2));
    TRY((run_pass<T, false>(P, "gen_dft_d1", g.T[1], g.n[1], g.T[0], g.n[2], +1, +1,
                            arr_load<cx<T>>(P, W1, g.T[0], (long long)g.T[0] * g.T[1], 1, g.T[1]), NoMid(),
                            arr_store<cx<T>>(P, W2, g.T[0], (long long)g.T[0] * g.n[1], 1),
                            (double)g.T[0] * g.n[2] * (g.T[1] + g.n[1]) * e)));
    cur = W2;
  }
  const long long rows = g.dim == 3 ? (long long)g.n[1] * g.n[2] : g.n[1];
  return run_pass<T, true>(P, "gen_dft_d0", g.T[0], g.n[0], rows, 1, +1, +1,
                           arr_load<cx<T>>(P, cur, 1, 0, g.T[0], g.T[0]), NoMid(), ss,
                           (double)rows * (g.T[0] * e + 2.0 * g.n[0] * sizeof(S)));
}

// DCT/DST field backend (matrix.hh:342-367, dctdstfieldbackend.hh): for each of the 2^d
// even/odd symmetry types, the scaled noise extended to the whole torus (DctDstNoise),
// complex backward transforms along every axis and the real part added into the field
template <typename T, typename S>
static pf_status gen_dctdst(pf_plan* P, const double* noise_dev, uint64_t seed, S* out, int transform) {
  const Geom& g = P->g;
  DctDstNoise nz{};
  nz.dim = g.dim;
  for (int i = 0; i < 3; i++) {
    nz.ext[i] = g.T[i];
    nz.D[i] = i < g.dim ? g.T[i] / 2 + 1 : 1;
  }
  nz.sq = sizeof(T) == 8 ? (const void*)P->sq64 : (const void*)P->sq32;
  nz.noise = noise_dev;
  nz.seed = seed;
  nz.nsq = (unsigned)g.S;
  nz.nnoise = (unsigned)g.noise;
  nz.Dtot = (unsigned)g.D;
  nz.transposed = g.transposed;
  const double e = sizeof(cx<T>);
  const int last = g.dim - 1;
  const long long inner = (long long)(g.N / (uint64_t)g.T[last]);
  for (int type = 0; type < (1 << g.dim); type++) {
    nz.type = type;
    AccStore<S> as{out, g.n[0], type != 0, (unsigned)g.domain};
    if (g.dim == 1) {
      TRY(run_pass<T, true>(P, "gen_dctdst_d0", g.T[0], g.n[0], 1, 1, +1, +1, nz, NoMid(), as,
                            (double)g.T[0] * (8.0 + sizeof(T)) + 2.0 * g.n[0] * sizeof(S)));
      continue;
    }
    void *W1 = nullptr, *W2 = nullptr;
    TRY(workspace(P, 0, sizeof(cx<T>) * (size_t)inner * g.n[last], &W1));
    TRY(run_pass<T, false>(P, "gen_dctdst_noise", g.T[last], g.n[last], inner, 1, +1, +1, nz, NoMid(),
                           arr_store<cx<T>>(P, W1, inner, 0, 1),
                           (double)inner * (g.T[last] * (8.0 + sizeof(T)) + g.n[last] * e)));
    void* cur = W1;
    if (g.dim == 3) {
      TRY(workspace(P, 1, sizeof(cx<T>) * (size_t)g.T[0] * g.n[1] * g.n[2], &W2));
      TRY((run_pass<T, false>(P, "gen_dctdst_d1", g.T[1], g.n[1], g.T[0], g.n[2], +1, +1,
                              arr_load<cx<T>>(P, W1, g.T[0], (long long)g.T[0] * g.T[1], 1, g.T[1]), NoMid(),
                              arr_store<cx<T>>(P, W2, g.T[0], (long long)g.T[0] * g.n[1], 1),
                              (double)g.T[0] * g.n[2] * (g.T[1] + g.n[1]) * e)));
      cur = W2;
    }
    const long long rows = g.dim == 3 ? (long long)g.n[1] * g.n[2] : g.n[1];
    TRY(run_pass<T, true>(P, "gen_dctdst_d0", g.T[0], g.n[0], rows, 1, +1, +1,
                          arr_load<cx<T>>(P, cur, 1, 0, g.T[0], g.T[0]), NoMid(), as,
                          (double)rows * (g.T[0] * e + 2.0 * g.n[0] * sizeof(S))));
  }
  if (transform) {  // the value transform acts on the summed field (randomfield.hh:641-651)
    ProfRec rec;
    TRY(prof_begin(P, "transform", g.domain * 2.0 * sizeof(S), &rec));
    k_transform<S><<<grid_for(g.domain), kThreads, 0, P->stream>>>(out, g.domain, transform, P->desc.boxcox_lambda);
    TRY(prof_end(P, &rec));
  }
  return PF_OK;
}

// ---------------------------------------------------------------------------
// matvecs: multiplyExtended / Root / InverseExtended (matrix.hh:1443-1646)
// ---------------------------------------------------------------------------
template <typename T>
static MultMid mult_mid(pf_plan* P, const T* fac) {
  const Geom& g = P->g;
  MultMid m{};
  m.dim = g.dim;
  for (int i = 0; i < 3; i++) m.ext[i] = g.T[i];
  m.C0 = g.fb == PF_FIELD_DFT ? g.T[0] : g.T0c;  // column count of the r2c schedule's half spectrum
  m.layout = g.mb == PF_MATRIX_DCT ? 0 : (g.mb == PF_MATRIX_R2C ? 1 : 2);
  m.LC0 = g.mb == PF_MATRIX_R2C ? g.T0c : g.T[0];
  m.D0 = g.T[0] / 2 + 1;
  m.D1 = g.T[1] / 2 + 1;
  m.axis = g.dim - 1;
  m.fac = fac;
  m.nfac = (long long)g.S;
  return m;
}

template <typename T, typename S>
static pf_status matvec_r2c(pf_plan* P, int op, const S* in, S* out) {
  const Geom& g = P->g;
  const T* fac = nullptr;
  TRY(factor_array<T>(P, op, &fac));
  MultMid mid = mult_mid<T>(P, fac);
  const int T0c = g.T0c, P0 = half_pitch(g);
  const double e = sizeof(cx<T>);
  const double lb = sizeof(T);
  FieldRowLoad<S> fl{in, g.n[0], (unsigned)g.domain};
  FieldRowStore<S> fs{out, g.n[0], 0, 0.0, (unsigned)g.domain};
  // the real-to-complex and complex-to-real rows along dim 0 take the paired kernels where
  // T0/2 is a power of two in [128, 2048] (FP32 transforms)
  const bool p2rows = std::is_same<T, float>::value && g.T[0] % 2 == 0 && p2_length(g.T[0] / 2);
  const int pair_ok = (g.n[0] % 2 == 0) ? 1 : 0;
  auto fwd_rows = [&](void* X, long long nrows) -> pf_status {
    const double b = (double)nrows * (g.n[0] * sizeof(S) + T0c * e);
    if (P->cg_dir_z) {  // CG direction update fused into this pass (FP32 transforms, FP64 vectors)
      if constexpr (std::is_same<T, float>::value && std::is_same<S, double>::value) {
        if (p2rows) {
          const bool al = ((uintptr_t)in % 16) == 0 && ((uintptr_t)P->cg_dir_z % 16) == 0;
          P2DirRowLoad dl{P->cg_dir_z, const_cast<double*>(in), P->cg_dir_s, g.n[0], (unsigned)g.domain,
                          (int)nrows, pair_ok && al ? 1 : 0};
          P2RowStore rs{(float2*)X, (unsigned)P0, (unsigned)std::min<size_t>(cap_of(P, X) / sizeof(float2), 0xffffffffu),
                        (int)nrows, T0c};
          return p2_r2c(P, "mv_r2c_d0", g.T[0] / 2, nrows, dl, rs, b + (double)nrows * g.n[0] * 16.0);
        }
      }
      return fail(PF_ERR_STATE, "internal error: fused direction update on a matvec without paired rows");
    }
    if constexpr (std::is_same<T, float>::value) {
      if (p2rows) {
        P2RealRowLoad<S> rl{in, g.n[0], (unsigned)g.domain, (int)nrows,
                            pair_ok && ((uintptr_t)in % (2 * sizeof(S))) == 0 ? 1 : 0};
        P2RowStore rs{(float2*)X, (unsigned)P0, (unsigned)std::min<size_t>(cap_of(P, X) / sizeof(float2), 0xffffffffu),
                      (int)nrows, T0c};
        return p2_r2c(P, "mv_r2c_d0", g.T[0] / 2, nrows, rl, rs, b);
      }
    }
    return run_freal<T, true>(P, "mv_r2c_d0", g.T[0], T0c, nrows, fl, arr_store<cx<T>>(P, X, 1, 0, P0), b);
  };
  auto inv_rows = [&](void* X, long long nrows) -> pf_status {
    const double b = (double)nrows * (T0c * e + g.n[0] * sizeof(S));
    if (P->cg_dot_d) {  // CG: d . (A d) summed in this pass (FP32 transforms, FP64 vectors)
      if constexpr (std::is_same<T, float>::value && std::is_same<S, double>::value) {
        if (p2rows) {
          P2RowLoad rl;
          rl.ptr = (const float2*)X;
          rl.rowstride = (unsigned)P0;
          rl.n = (unsigned)std::min<size_t>(cap_of(P, X) / sizeof(float2), 0xffffffffu);
          rl.Lin = T0c;
          rl.np = (int)nrows;
          P2FieldDotStore ps;
          ps.out = out;
          ps.n0 = g.n[0];
          ps.transform = 0;
          ps.boxcox = 0.f;
          ps.n = (unsigned)g.domain;
          ps.np = (int)nrows;
          ps.Lout = g.n[0];
          ps.vec = pair_ok && ((uintptr_t)out % 16) == 0 ? 1 : 0;
          ps.dv = P->cg_dot_d;
          ps.part = P->cg.part;  // 2 kCgBlocks doubles: more than any persistent grid's CTAs
          ps.cnt = P->cg.cnt;
          ps.sdst = P->cg_dot_dst;
          return p2_c2r(P, "mv_c2r_d0", g.T[0] / 2, g.n[0], nrows, rl, ps, b + (double)nrows * g.n[0] * 8.0);
        }
      }
      return fail(PF_ERR_STATE, "internal error: fused dot product on a matvec without paired rows");
    }
    if constexpr (std::is_same<T, float>::value) {
      if (p2rows) {
        P2RowLoad rl;
        rl.ptr = (const float2*)X;
        rl.rowstride = (unsigned)P0;
        rl.n = (unsigned)std::min<size_t>(cap_of(P, X) / sizeof(float2), 0xffffffffu);
        rl.Lin = T0c;
        rl.np = (int)nrows;
        P2FieldStoreT<S> ps{out, g.n[0], 0, 0.f, (unsigned)g.domain, (int)nrows, g.n[0],
                            pair_ok && ((uintptr_t)out % (2 * sizeof(S))) == 0 ? 1 : 0};
        return p2_c2r(P, "mv_c2r_d0", g.T[0] / 2, g.n[0], nrows, rl, ps, b);
      }
    }
    return run_freal<T, false>(P, "mv_c2r_d0", g.T[0], g.n[0], nrows, arr_load<cx<T>>(P, X, 1, 0, P0, T0c), fs, b);
  };
  if (g.dim == 2) {
    void* X1 = nullptr;
    TRY(workspace(P, 2, sizeof(cx<T>) * (size_t)P0 * g.n[1], &X1));
    TRY(fwd_rows(X1, g.n[1]));
    const double bf1 = (double)T0c * (2.0 * g.n[1] * e + g.T[1] * lb);
    if (std::is_same<T, float>::value && p2_length(g.T[1]) && p2_view_ok(X1, P0, 0, 1))
      TRY(p2_c2c_mid(P, "mv_fused_d1", g.T[1], g.n[1], T0c, 1, p2_load(P, X1, P0, 0, g.n[1], T0c), mid,
                     p2_store(P, X1, P0, 0, T0c), bf1));
    else
      TRY((run_fpass<T, -1, +1, false, false>(P, "mv_fused_d1", g.T[1], g.n[1], T0c, 1,
                                              arr_load<cx<T>>(P, X1, P0, 0, 1, g.n[1]), mid,
                                              arr_store<cx<T>>(P, X1, P0, 0, 1), bf1)));
    return inv_rows(X1, g.n[1]);
  }
  void *X1 = nullptr, *X2 = nullptr;
  TRY(workspace(P, 1, sizeof(cx<T>) * (size_t)P0 * g.n[1] * g.n[2], &X1));
  TRY(workspace(P, 2, sizeof(cx<T>) * (size_t)P0 * g.T[1] * g.n[2], &X2));
  const long long rows = (long long)g.n[1] * g.n[2];
  const long long s2 = (long long)P0 * g.T[1];
  TRY(fwd_rows(X1, rows));
  // the strided passes along dim 1 take the paired kernels where the torus length and the
  // views allow (FP32 transforms), as in generation
  const long long w1o = (long long)P0 * g.n[1];
  const bool p2d1 = std::is_same<T, float>::value && p2_length(g.T[1]) && p2_view_ok(X1, P0, w1o, g.n[2]) &&
                    p2_view_ok(X2, P0, s2, g.n[2]);
  const double bd1 = (double)T0c * g.n[2] * (g.n[1] + g.T[1]) * e;
  if (p2d1)
    TRY(p2_c2c<-1>(P, "mv_c2c_d1", g.T[1], g.T[1], T0c, g.n[2], p2_load(P, X1, P0, w1o, g.n[1], T0c),
                   p2_store(P, X2, P0, s2, T0c), bd1));
  else
    TRY((run_fpass<T, -1, -1, false, false>(P, "mv_c2c_d1", g.T[1], g.T[1], T0c, g.n[2],
                                            arr_load<cx<T>>(P, X1, P0, w1o, 1, g.n[1]), NoMid(),
                                            arr_store<cx<T>>(P, X2, P0, s2, 1), bd1)));
  // forward along dim 2, eigenvalue factor, backward along dim 2 (pencils k0 x k1)
  const double bf2 = (double)T0c * g.T[1] * (2.0 * g.n[2] * e + g.T[2] * lb);
  if (std::is_same<T, float>::value && p2_length(g.T[2]) && p2_view_ok(X2, s2, P0, g.T[1]))
    TRY(p2_c2c_mid(P, "mv_fused_d2", g.T[2], g.n[2], T0c, g.T[1], p2_load(P, X2, s2, P0, g.n[2], T0c), mid,
                   p2_store(P, X2, s2, P0, T0c), bf2));
  else
    TRY((run_fpass<T, -1, +1, false, false>(P, "mv_fused_d2", g.T[2], g.n[2], T0c, g.T[1],
                                            arr_load<cx<T>>(P, X2, s2, P0, 1, g.n[2]), mid,
                                            arr_store<cx<T>>(P, X2, s2, P0, 1), bf2)));
  if (p2d1)
    TRY(p2_c2c<+1>(P, "mv_c2c_d1i", g.T[1], g.n[1], T0c, g.n[2], p2_load(P, X2, P0, s2, g.T[1], T0c),
                   p2_store(P, X1, P0, w1o, T0c), bd1));
  else
    TRY((run_fpass<T, +1, +1, false, false>(P, "mv_c2c_d1i", g.T[1], g.n[1], T0c, g.n[2],
                                            arr_load<cx<T>>(P, X2, P0, s2, 1, g.T[1]), NoMid(),
                                            arr_store<cx<T>>(P, X1, P0, w1o, 1), bd1)));
  return inv_rows(X1, rows);
}

// DFT field backend matvec: complex embedding, c2c on every axis, Re extraction
template <typename T, typename S>
static pf_status matvec_dft(pf_plan* P, int op, const S* in, S* out) {
  const Geom& g = P->g;
  const T* fac = nullptr;
  TRY(factor_array<T>(P, op, &fac));
  MultMid mid = mult_mid<T>(P, fac);
  const double e = sizeof(cx<T>);
  FieldComplexLoad<S> fl{in, g.n[0], (unsigned)g.domain};
  SplitStore<S> ss{out, nullptr, g.n[0], 0, 0.0, (unsigned)g.domain};
  if (g.dim == 1)
    return run_pass<T, true>(P, "mv_dft_fused_d0", g.T[0], g.n[0], 1, 1, -1, +1, fl, mid, ss,
                             (double)g.T[0] * sizeof(T) + 2.0 * g.n[0] * sizeof(S));
  const long long rows = (long long)(g.domain / (uint64_t)g.n[0]);
  void *X1 = nullptr, *X2 = nullptr;
  if (g.dim == 2) {
    TRY(workspace(P, 2, sizeof(cx<T>) * (size_t)g.T[0] * g.n[1], &X1));
    TRY((run_pass<T, true>(P, "mv_dft_d0", g.T[0], g.T[0], rows, 1, -1, -1, fl, NoMid(),
                           arr_store<cx<T>>(P, X1, 1, 0, g.T[0]), (double)rows * (g.n[0] * sizeof(S) + g.T[0] * e))));
    TRY((run_pass<T, false>(P, "mv_dft_fused_d1", g.T[1], g.n[1], g.T[0], 1, -1, +1,
                            arr_load<cx<T>>(P, X1, g.T[0], 0, 1, g.n[1]), mid, arr_store<cx<T>>(P, X1, g.T[0], 0, 1),
                            (double)g.T[0] * 2.0 * g.n[1] * e)));
    return run_pass<T, true>(P, "mv_dft_d0i", g.T[0], g.n[0], rows, 1, +1, +1,
                             arr_load<cx<T>>(P, X1, 1, 0, g.T[0], g.T[0]), NoMid(), ss,
                             (double)rows * (g.T[0] * e + g.n[0] * sizeof(S)));
  }
  const long long in1 = (long long)g.T[0] * g.T[1];
  TRY(workspace(P, 1, sizeof(cx<T>) * (size_t)g.T[0] * g.n[1] * g.n[2], &X1));
  TRY(workspace(P, 2, sizeof(cx<T>) * (size_t)in1 * g.n[2], &X2));
  TRY((run_pass<T, true>(P, "mv_dft_d0", g.T[0], g.T[0], rows, 1, -1, -1, fl, NoMid(),
                         arr_store<cx<T>>(P, X1, 1, 0, g.T[0]), (double)rows * (g.n[0] * sizeof(S) + g.T[0] * e))));
  TRY((run_pass<T, false>(P, "mv_dft_d1", g.T[1], g.T[1], g.T[0], g.n[2], -1, -1,
                          arr_load<cx<T>>(P, X1, g.T[0], (long long)g.T[0] * g.n[1], 1, g.n[1]), NoMid(),
                          arr_store<cx<T>>(P, X2, g.T[0], in1, 1), (double)g.T[0] * g.n[2] * (g.n[1] + g.T[1]) * e)));
  TRY((run_pass<T, false>(P, "mv_dft_fused_d2", g.T[2], g.n[2], g.T[0], g.T[1], -1, +1,
                          arr_load<cx<T>>(P, X2, in1, g.T[0], 1, g.n[2]), mid, arr_store<cx<T>>(P, X2, in1, g.T[0], 1),
                          (double)in1 * 2.0 * g.n[2] * e)));
  TRY((run_pass<T, false>(P, "mv_dft_d1i", g.T[1], g.n[1], g.T[0], g.n[2], +1, +1,
                          arr_load<cx<T>>(P, X2, g.T[0], in1, 1, g.T[1]), NoMid(),
                          arr_store<cx<T>>(P, X1, g.T[0], (long long)g.T[0] * g.n[1], 1),
                          (double)g.T[0] * g.n[2] * (g.n[1] + g.T[1]) * e)));
  return run_pass<T, true>(P, "mv_dft_d0i", g.T[0], g.n[0], rows, 1, +1, +1,
                           arr_load<cx<T>>(P, X1, 1, 0, g.T[0], g.T[0]), NoMid(), ss,
                           (double)rows * (g.T[0] * e + g.n[0] * sizeof(S)));
}

// The DCT/DST field backend's products (matrix.hh:1449-1473) split the zero-padded input
// into its 2^d even/odd components (setComponent, dctdstfieldbackend.hh:444-460: value /
// 2^(d - border), zero on an odd axis's border), multiply each by the eigenvalues through
// its REDFT00/RODFT00 transforms and add the restrictions.  The circulant covariance maps
// each symmetry class to itself and the components sum to the zero-padded input, so the
// result is the circulant product (C_ext x)/N restricted to the domain: the r2c schedule
// computes it in one pass set instead of 2^d.
template <typename T, typename S>
static pf_status matvec_dev(pf_plan* P, int op, const S* in, S* out) {
  if (P->g.fb == PF_FIELD_R2C || P->g.fb == PF_FIELD_DCTDST) return matvec_r2c<T, S>(P, op, in, out);
  return matvec_dft<T, S>(P, op, in, out);
}

// internal operation: torus pseudo-inverse (clamped eigenvalues dropped), used as the
// preconditioner of the residual-mode CG
constexpr int kOpInvPinv = 3;

// whether the FP32 matvec of plan P takes the paired real-to-complex rows, into which the
// residual-mode CG folds its direction update (P2DirRowLoad)
static bool cg_dir_fusable(const pf_plan* P, bool fp32) {
  const Geom& g = P->g;
  return fp32 && (g.fb == PF_FIELD_R2C || g.fb == PF_FIELD_DCTDST) && g.T[0] % 2 == 0 && p2_length(g.T[0] / 2);
}

// CG helpers use FP64 vectors with FP64 or FP32 transforms
static pf_status cg_matvec(pf_plan* P, int op, bool fp32, const double* in, double* out) {
  if (fp32) return matvec_dev<float, double>(P, op, in, out);
  return matvec_dev<double, double>(P, op, in, out);
}

static pf_status learned_apply(pf_learned* Lp, bool fp32, const double* r, double* z);

#include "pf_cg_host.inc"
#include "pf_learned.inc"

static pf_status stage_noise(pf_plan* P, const double* noise, int noise_mem, const double** dev) {
  *dev = nullptr;
  if (!noise) return PF_OK;
  if (noise_mem == PF_MEM_DEVICE) {
    *dev = noise;
    return PF_OK;
  }
  TRY(ensure(P, (void**)&P->noise_dev, &P->noise_cap, P->g.noise * 8));
  CK(cudaMemcpyAsync(P->noise_dev, noise, P->g.noise * 8, cudaMemcpyHostToDevice, P->stream));
  *dev = P->noise_dev;
  return PF_OK;
}

template <typename S>
static pf_status generate_typed(pf_plan* P, const double* nd, uint64_t seed, S* out_dev, int transform) {
  const bool f64 = sizeof(S) == 8;
  if (P->g.fb == PF_FIELD_DCTDST)
    return f64 ? gen_dctdst<double, S>(P, nd, seed, out_dev, transform)
               : gen_dctdst<float, S>(P, nd, seed, out_dev, transform);
  if (P->g.fb == PF_FIELD_R2C)
    return f64 ? gen_r2c<double, S>(P, nd, seed, out_dev, transform) : gen_r2c<float, S>(P, nd, seed, out_dev, transform);
  TRY(ensure(P, &P->spare, &P->spare_cap, P->g.domain * sizeof(S)));
  TRY(f64 ? gen_dft<double, S>(P, nd, seed, out_dev, (S*)P->spare, transform)
          : gen_dft<float, S>(P, nd, seed, out_dev, (S*)P->spare, transform));
  P->spare_valid = true;
  return PF_OK;
}

// Stage pipeline of pf_generate_batch (device output, R2C field backend): the noise pass of
// realization r (issue-bound: integer multiplies and paired FP32 arithmetic) runs on one
// stream while the memory-bound remaining passes of realization r-1 run on the other.  The
// noise passes alternate between two intermediate buffers; events order every buffer's
// reuse after the passes that read it.
static pf_status generate_stage_pipeline(pf_plan* P, uint64_t seed, int32_t count, void* out, int tr) {
  if (!P->lane[0])
    for (int l = 0; l < 2; l++) CK(cudaStreamCreateWithFlags(&P->lane[l], cudaStreamNonBlocking));
  if (!P->lane_ev[0])
    for (int l = 0; l < 3; l++) CK(cudaEventCreateWithFlags(&P->lane_ev[l], cudaEventDisableTiming));
  if (!P->stage_ev[0])
    for (int l = 0; l < 4; l++) CK(cudaEventCreateWithFlags(&P->stage_ev[l], cudaEventDisableTiming));
  const bool f64 = P->desc.precision == PF_PREC_F64;
  const size_t bytes = P->g.domain * (f64 ? 8 : 4);
  cudaStream_t caller = P->stream;
  CK(cudaEventRecord(P->lane_ev[0], caller));
  for (int l = 0; l < 2; l++) CK(cudaStreamWaitEvent(P->lane[l], P->lane_ev[0], 0));
  cudaEvent_t* noise_done = P->stage_ev;      // [slot]: the noise pass wrote the buffer
  cudaEvent_t* buffer_free = P->stage_ev + 2;  // [slot]: the remaining passes read it
  pf_status st = PF_OK;
  for (int32_t r = 0; r < count && st == PF_OK; r++) {
    const int slot = r & 1;
    auto run = [&](int stages) {
      if (slot) {
        std::swap(P->ws[0], P->ws_b[0]);
        std::swap(P->ws_bytes[0], P->ws_b_bytes[0]);
      }
      P->ctr_slot = slot;
      void* dst = (char*)out + (size_t)r * bytes;
      const pf_status s2 = f64 ? gen_r2c<double, double>(P, nullptr, seed + r, (double*)dst, tr, stages)
                               : gen_r2c<float, float>(P, nullptr, seed + r, (float*)dst, tr, stages);
      if (slot) {
        std::swap(P->ws[0], P->ws_b[0]);
        std::swap(P->ws_bytes[0], P->ws_b_bytes[0]);
      }
      P->ctr_slot = 0;
      return s2;
    };
    P->stream = P->lane[0];
    if (r >= 2 && cudaStreamWaitEvent(P->lane[0], buffer_free[slot], 0) != cudaSuccess)
      st = fail(PF_ERR_CUDA, "stream wait failed");
    if (st == PF_OK) st = run(1);
    if (st == PF_OK && cudaEventRecord(noise_done[slot], P->lane[0]) != cudaSuccess)
      st = fail(PF_ERR_CUDA, "event record failed");
    P->stream = P->lane[1];
    if (st == PF_OK && cudaStreamWaitEvent(P->lane[1], noise_done[slot], 0) != cudaSuccess)
      st = fail(PF_ERR_CUDA, "stream wait failed");
    if (st == PF_OK) st = run(2);
    if (st == PF_OK && cudaEventRecord(buffer_free[slot], P->lane[1]) != cudaSuccess)
      st = fail(PF_ERR_CUDA, "event record failed");
    P->stream = caller;
  }
  P->stream = caller;
  for (int l = 0; l < 2; l++) {
    CK(cudaEventRecord(P->lane_ev[1 + l], P->lane[l]));
    CK(cudaStreamWaitEvent(caller, P->lane_ev[1 + l], 0));
  }
  P->spare_valid = false;
  return st;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void pf_field_desc_init(pf_field_desc* d) {
  if (!d) return;
  memset(d, 0, sizeof(*d));
  d->dim = 2;
  for (int i = 0; i < 3; i++) {
    d->cells[i] = 1;
    d->extensions[i] = 1.0;
  }
  d->embedding_factor = 2;
  d->covariance = PF_COV_EXPONENTIAL;
  d->variance = 1.0;
  d->anisotropy = PF_ANISO_NONE;
  d->corr_length[0] = 1.0;
  d->matern_nu = 0.5;
  d->exp_gamma = 1.0;
  d->cauchy_alpha = 1.0;
  d->cauchy_beta = 1.0;
  d->threshold = 1e-14;
  d->transposed = -1;
  d->matrix_backend = PF_MATRIX_DEFAULT;
  d->field_backend = PF_FIELD_DEFAULT;
  d->precision = PF_PREC_F64;
  d->eigen_check = PF_EIGCHECK_CORRECTED;
  d->cg_iterations = 100;
  d->transform = PF_TRANSFORM_NONE;
  d->periodization = PF_PERIODIZATION_CLASSICAL;
  d->sigmoid = PF_SIGMOID_SMOOTHSTEP;
  d->sigmoid_combine = PF_COMBINE_RADIAL_PLUS;
  d->merge_recursions = 99;
  d->sigmoid_start = 1.0;
  d->sigmoid_end = -1.0;
  d->fold_max_factor = 1.0;
  d->fold_recursions = 99;
  d->cofold_max_factor = 5.0;
  d->cofold_recursions = 1;
}

pf_status pf_plan_create(const pf_field_desc* desc, pf_plan** plan) {
  if (!desc || !plan) return fail(PF_ERR_ARG, "null argument");
  *plan = nullptr;
  Geom g;
  TRY(resolve(desc, &g));
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(PF_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
  }
  pf_plan* P = new pf_plan();
  P->desc = *desc;
  P->g = g;
  cudaGetDevice(&P->device);
  e = cudaStreamCreateWithFlags(&P->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete P;
    return fail(PF_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  P->stream = P->own;
  *plan = P;
  return PF_OK;
}

void pf_plan_destroy(pf_plan* P) {
  if (!P) return;
  cudaStreamSynchronize(P->stream);
  for (pf_plan* l : P->lanes) pf_plan_destroy(l);
  P->lanes.clear();
  if (P->shared) {  // a solver lane: the spectrum and factor arrays belong to its parent
    P->lam64 = nullptr;
    P->sq64 = nullptr;
    P->sq32 = nullptr;
    P->lam32 = nullptr;
    P->scan = nullptr;
    P->cof = nullptr;
    for (int a = 0; a < 2; a++)
      for (int o = 0; o < 4; o++) P->fac[a][o] = nullptr;
  }
  void** bufs[] = {(void**)&P->lam64, (void**)&P->sq64, (void**)&P->sq32, (void**)&P->lam32, (void**)&P->scan,
                   (void**)&P->cof, &P->ws[0], &P->ws[1], &P->ws[2], (void**)&P->noise_dev, &P->io_dev, &P->io2_dev, &P->spare,
                   (void**)&P->tile_ctr};
  for (void** b : bufs)
    if (*b) cudaFree(*b), *b = nullptr;
  for (int a = 0; a < 2; a++)
    for (int o = 0; o < 4; o++)
      if (P->fac[a][o]) cudaFree(P->fac[a][o]);
  cg_free(P);
  for (auto& r : P->recs) {
    cudaEventDestroy(r.e0);
    cudaEventDestroy(r.e1);
  }
  for (auto e : P->evpool) cudaEventDestroy(e);
  for (int l = 0; l < 2; l++) {
    if (P->ws_b[l]) cudaFree(P->ws_b[l]);
    if (P->lane[l]) cudaStreamDestroy(P->lane[l]);
  }
  for (int l = 0; l < 3; l++)
    if (P->lane_ev[l]) cudaEventDestroy(P->lane_ev[l]);
  for (int l = 0; l < 4; l++)
    if (P->stage_ev[l]) cudaEventDestroy(P->stage_ev[l]);
  if (P->own) cudaStreamDestroy(P->own);
  delete P;
}

pf_status pf_plan_set_stream(pf_plan* P, void* stream) {
  if (!P) return fail(PF_ERR_ARG, "null plan");
  P->stream = stream ? (cudaStream_t)stream : P->own;
  return PF_OK;
}

pf_status pf_plan_get_info(const pf_plan* P, pf_plan_info* info) {
  if (!P || !info) return fail(PF_ERR_ARG, "null argument");
  memset(info, 0, sizeof(*info));
  const Geom& g = P->g;
  info->dim = g.dim;
  for (int i = 0; i < 3; i++) {
    info->cells[i] = g.n[i];
    info->ext_cells[i] = g.T[i];
  }
  info->matrix_backend = g.mb;
  info->field_backend = g.fb;
  info->transposed = g.transposed;
  info->precision = P->desc.precision;
  info->domain_size = g.domain;
  info->ext_size = g.N;
  info->spectrum_size = g.S;
  info->noise_size = g.noise;
  info->device_bytes = P->bytes_held;
  return PF_OK;
}

pf_status pf_spectrum_build(pf_plan* P, pf_eig_stats* stats) {
  if (!P) return fail(PF_ERR_ARG, "null plan");
  P->spare_valid = false;
  pf_status st = build_spectrum(P);
  if (stats) *stats = P->stats;
  return check_bounds(P, st);
}

pf_status pf_spectrum_build_values(pf_plan* P, const double* values, uint64_t count, int32_t mem,
                                   pf_eig_stats* stats) {
  if (!P || !values) return fail(PF_ERR_ARG, "null argument");
  const Geom& g = P->g;
  const uint64_t need = g.mb == PF_MATRIX_DCT ? g.D : g.N;
  if (count != need)
    return fail(PF_ERR_ARG, "covariance values: %llu given, the matrix has %llu cells", (unsigned long long)count,
                (unsigned long long)need);
  P->spare_valid = false;
  const double* dv = values;
  double* staged = nullptr;
  if (mem != PF_MEM_DEVICE) {
    TRY(dalloc(P, (void**)&staged, need * 8));
    const cudaError_t e = cudaMemcpyAsync(staged, values, need * 8, cudaMemcpyHostToDevice, P->stream);
    if (e != cudaSuccess) {
      dfree(P, (void**)&staged, need * 8);
      return fail(PF_ERR_CUDA, "copy of the covariance values: %s", cudaGetErrorString(e));
    }
    dv = staged;
  }
  pf_status st = build_spectrum(P, dv);
  if (staged) {
    cudaStreamSynchronize(P->stream);
    dfree(P, (void**)&staged, need * 8);
  }
  if (stats) *stats = P->stats;
  return check_bounds(P, st);
}

pf_status pf_spectrum_copy(pf_plan* P, double* out, uint64_t count) {
  if (!P || !out) return fail(PF_ERR_ARG, "null argument");
  if (!P->have_spec) return fail(PF_ERR_STATE, "spectrum not built");
  const Geom& g = P->g;
  if (count != g.S) return fail(PF_ERR_ARG, "spectrum has %llu entries", (unsigned long long)g.S);
  std::vector<double> nat(g.S);
  CK(cudaMemcpyAsync(nat.data(), P->lam64, g.S * 8, cudaMemcpyDeviceToHost, P->stream));
  CK(cudaStreamSynchronize(P->stream));
  // natural -> the reference's storage order (swap the last two dims when transposed)
  const int c0 = g.C[0], c1 = g.C[1], c2 = g.C[2];
  if (!g.transposed) {
    memcpy(out, nat.data(), g.S * 8);
  } else if (g.dim == 3) {
    for (int k2 = 0; k2 < c2; k2++)
      for (int k1 = 0; k1 < c1; k1++)
        for (int k0 = 0; k0 < c0; k0++)
          out[(size_t)k0 + (size_t)c0 * ((size_t)k2 + (size_t)c2 * k1)] =
              nat[(size_t)k0 + (size_t)c0 * ((size_t)k1 + (size_t)c1 * k2)];
  } else {
    for (int k1 = 0; k1 < c1; k1++)
      for (int k0 = 0; k0 < c0; k0++) out[(size_t)k1 + (size_t)c1 * k0] = nat[(size_t)k0 + (size_t)c0 * k1];
  }
  return PF_OK;
}

pf_status pf_generate(pf_plan* P, const double* noise, int32_t noise_mem, uint64_t seed, void* out, int32_t out_mem,
                      int32_t apply_transform) {
  if (!P || !out) return fail(PF_ERR_ARG, "null argument");
  TRY(ensure_spectrum(P));
  const size_t es = P->desc.precision == PF_PREC_F64 ? 8 : 4;
  const size_t bytes = P->g.domain * es;
  void* dst = out;
  if (out_mem != PF_MEM_DEVICE) {
    TRY(ensure(P, &P->io_dev, &P->io_cap, bytes));
    dst = P->io_dev;
  }
  if (P->spare_valid) {  // matrix.hh:416-419: hand out the cached second field
    CK(cudaMemcpyAsync(dst, P->spare, bytes, cudaMemcpyDeviceToDevice, P->stream));
    P->spare_valid = false;
  } else {
    const double* nd = nullptr;
    TRY(stage_noise(P, noise, noise_mem, &nd));
    const int tr = apply_transform ? P->desc.transform : 0;
    if (es == 8)
      TRY(generate_typed<double>(P, nd, seed, (double*)dst, tr));
    else
      TRY(generate_typed<float>(P, nd, seed, (float*)dst, tr));
  }
  if (out_mem != PF_MEM_DEVICE) CK(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, P->stream));
  return check_bounds(P, PF_OK);
}

pf_status pf_generate_batch(pf_plan* P, uint64_t seed, int32_t count, void* out, int32_t out_mem,
                            int32_t apply_transform) {
  if (!P || !out || count < 0) return fail(PF_ERR_ARG, "bad argument");
  TRY(ensure_spectrum(P));
  const size_t es = P->desc.precision == PF_PREC_F64 ? 8 : 4;
  const size_t bytes = P->g.domain * es;
  const int tr = apply_transform ? P->desc.transform : 0;
  if (P->g.fb == PF_FIELD_R2C && count >= 2 && P->batch_mode == 1 && out_mem == PF_MEM_DEVICE)
    return check_bounds(P, generate_stage_pipeline(P, seed, count, out, tr));
  if (P->g.fb == PF_FIELD_R2C && count >= 2) {
    // Realizations are independent: alternate them over two streams, each with its own
    // workspaces, so that one realization's issue-bound noise pass overlaps the other's
    // memory-bound passes (and, for host output, the other's copy to the host, which runs
    // asynchronously when `out` is pinned).  The caller's stream waits for both at the end.
    if (!P->lane[0])
      for (int l = 0; l < 2; l++)
        CK(cudaStreamCreateWithFlags(&P->lane[l], cudaStreamNonBlocking));
    if (!P->lane_ev[0])
      for (int l = 0; l < 3; l++) CK(cudaEventCreateWithFlags(&P->lane_ev[l], cudaEventDisableTiming));
    cudaStream_t caller = P->stream;
    CK(cudaEventRecord(P->lane_ev[0], caller));
    for (int l = 0; l < 2; l++) CK(cudaStreamWaitEvent(P->lane[l], P->lane_ev[0], 0));
    const bool host = out_mem != PF_MEM_DEVICE;
    if (host) {  // one device staging buffer per stream
      TRY(ensure(P, &P->io_dev, &P->io_cap, bytes));
      TRY(ensure(P, &P->io2_dev, &P->io2_cap, bytes));
    }
    pf_status st = PF_OK;
    for (int32_t r = 0; r < count && st == PF_OK; r++) {
      const int slot = r & 1;
      void* dst = host ? (slot ? P->io2_dev : P->io_dev) : (char*)out + (size_t)r * bytes;
      if (slot)
        for (int i = 0; i < 2; i++) {
          std::swap(P->ws[i], P->ws_b[i]);
          std::swap(P->ws_bytes[i], P->ws_b_bytes[i]);
        }
      P->stream = P->lane[slot];
      P->ctr_slot = slot;
      st = es == 8 ? gen_r2c<double, double>(P, nullptr, seed + r, (double*)dst, tr)
                   : gen_r2c<float, float>(P, nullptr, seed + r, (float*)dst, tr);
      P->ctr_slot = 0;
      if (st == PF_OK && host &&
          cudaMemcpyAsync((char*)out + (size_t)r * bytes, dst, bytes, cudaMemcpyDeviceToHost, P->lane[slot]) !=
              cudaSuccess)
        st = fail(PF_ERR_CUDA, "copy of realization %d to the host failed", (int)r);
      P->stream = caller;
      if (slot)
        for (int i = 0; i < 2; i++) {
          std::swap(P->ws[i], P->ws_b[i]);
          std::swap(P->ws_bytes[i], P->ws_b_bytes[i]);
        }
    }
    for (int l = 0; l < 2; l++) {
      CK(cudaEventRecord(P->lane_ev[1 + l], P->lane[l]));
      CK(cudaStreamWaitEvent(caller, P->lane_ev[1 + l], 0));
    }
    P->spare_valid = false;
    return check_bounds(P, st);
  }
  for (int32_t r = 0; r < count; r++) {
    void* dst = (char*)out + (size_t)r * bytes;
    if (out_mem != PF_MEM_DEVICE) {
      TRY(ensure(P, &P->io_dev, &P->io_cap, bytes));
      dst = P->io_dev;
    }
    if (es == 8) {
      if (P->g.fb == PF_FIELD_R2C)
        TRY((gen_r2c<double, double>(P, nullptr, seed + r, (double*)dst, tr)));
      else
        TRY((generate_typed<double>(P, nullptr, seed + r, (double*)dst, tr)));
    } else {
      if (P->g.fb == PF_FIELD_R2C)
        TRY((gen_r2c<float, float>(P, nullptr, seed + r, (float*)dst, tr)));
      else
        TRY((generate_typed<float>(P, nullptr, seed + r, (float*)dst, tr)));
    }
    P->spare_valid = false;
    if (out_mem != PF_MEM_DEVICE)
      CK(cudaMemcpyAsync((char*)out + (size_t)r * bytes, dst, bytes, cudaMemcpyDeviceToHost, P->stream));
  }
  return check_bounds(P, PF_OK);
}

pf_status pf_matvec(pf_plan* P, int32_t op, int32_t precision, const void* in, void* out, int32_t mem) {
  if (!P || !in || !out) return fail(PF_ERR_ARG, "null argument");
  if (op < 0 || op > 2) return fail(PF_ERR_ARG, "unknown operation");
  TRY(ensure_spectrum(P));
  const size_t es = precision == PF_PREC_F64 ? 8 : 4;
  const size_t bytes = P->g.domain * es;
  const void* src = in;
  void* dst = out;
  if (mem != PF_MEM_DEVICE) {
    TRY(ensure(P, &P->io_dev, &P->io_cap, bytes));
    TRY(ensure(P, &P->io2_dev, &P->io2_cap, bytes));
    CK(cudaMemcpyAsync(P->io_dev, in, bytes, cudaMemcpyHostToDevice, P->stream));
    src = P->io_dev;
    dst = P->io2_dev;
  }
  if (precision == PF_PREC_F64)
    TRY((matvec_dev<double, double>(P, op, (const double*)src, (double*)dst)));
  else
    TRY((matvec_dev<float, float>(P, op, (const float*)src, (float*)dst)));
  if (mem != PF_MEM_DEVICE) CK(cudaMemcpyAsync(out, dst, bytes, cudaMemcpyDeviceToHost, P->stream));
  return check_bounds(P, PF_OK);
}

pf_status pf_multiply_inverse(pf_plan* P, const double* b, double* x, int32_t mem, const pf_cg_opts* opts,
                              pf_cg_report* report) {
  if (!P || !b || !x) return fail(PF_ERR_ARG, "null argument");
  TRY(ensure_spectrum(P));
  pf_cg_opts o;
  if (opts)
    o = *opts;
  else {
    memset(&o, 0, sizeof(o));
    o.mode = PF_CG_REFERENCE;
    o.precondition = 1;
  }
  const size_t bytes = P->g.domain * 8;
  const double* bd = b;
  double* xd = x;
  if (mem != PF_MEM_DEVICE) {
    TRY(ensure(P, &P->io_dev, &P->io_cap, bytes));
    TRY(ensure(P, &P->io2_dev, &P->io2_cap, bytes));
    CK(cudaMemcpyAsync(P->io_dev, b, bytes, cudaMemcpyHostToDevice, P->stream));
    bd = (const double*)P->io_dev;
    xd = (double*)P->io2_dev;
  }
  pf_cg_report rep{};
  pf_status st = cg_solve(P, bd, xd, o, &rep);
  if (st == PF_ERR_NOT_CONVERGED && P->learned && o.mode == PF_CG_RESIDUAL && o.precondition) {
    // plain CG is the fallback of the learned preconditioner: solve again with P0 alone
    pf_learned* keep = P->learned;
    P->learned = nullptr;
    const int used = rep.iterations;
    st = cg_solve(P, bd, xd, o, &rep);
    rep.iterations += used;
    P->learned = keep;
  }
  if (report) *report = rep;
  if (st != PF_OK && st != PF_ERR_NOT_CONVERGED) return check_bounds(P, st);
  if (mem != PF_MEM_DEVICE) CK(cudaMemcpyAsync(x, xd, bytes, cudaMemcpyDeviceToHost, P->stream));
  return check_bounds(P, st);
}

pf_status pf_multiply_inverse_batch(pf_plan* P, const double* B, double* X, int32_t count, int32_t mem,
                                    const pf_cg_opts* opts, pf_cg_report* reports, int32_t lanes) {
  if (!P || (count > 0 && (!B || !X)) || count < 0) return fail(PF_ERR_ARG, "bad argument");
  if (count == 0) return PF_OK;
  TRY(ensure_spectrum(P));
  pf_cg_opts o;
  if (opts)
    o = *opts;
  else {
    memset(&o, 0, sizeof(o));
    o.mode = PF_CG_REFERENCE;
    o.precondition = 1;
  }
  return check_bounds(P, cg_solve_batch(P, B, X, count, mem, o, reports, lanes));
}

pf_status pf_export_noise(pf_plan* P, uint64_t seed, uint32_t epoch, double* out, int32_t mem) {
  if (!P || !out) return fail(PF_ERR_ARG, "null argument");
  const Geom& g = P->g;
  if (g.fb != PF_FIELD_R2C) return fail(PF_ERR_CONFIG, "noise export serves the R2C field backend");
  NoiseExport e{};
  e.dim = g.dim;
  e.T0c = g.T0c;
  e.ext1 = g.T[1];
  e.ext2 = g.T[2];
  e.Tl = g.T[g.dim - 1];
  e.transposed = g.transposed;
  e.fp64 = P->desc.precision == PF_PREC_F64;
  e.seed = seed;
  e.epoch = epoch;
  e.n = g.noise;
  double* dst = out;
  if (mem != PF_MEM_DEVICE) {
    TRY(ensure(P, (void**)&P->noise_dev, &P->noise_cap, g.noise * 8));
    dst = P->noise_dev;
  }
  k_export_noise<<<grid_for(g.Nc), kThreads, 0, P->stream>>>(e, dst);
  P->launches++;
  CK(cudaGetLastError());
  if (mem != PF_MEM_DEVICE) CK(cudaMemcpyAsync(out, dst, g.noise * 8, cudaMemcpyDeviceToHost, P->stream));
  return check_bounds(P, PF_OK);
}

pf_status pf_apply_transform(pf_plan* P, int32_t precision, void* data, uint64_t count, int32_t mem) {
  if (!P || !data) return fail(PF_ERR_ARG, "null argument");
  const size_t es = precision == PF_PREC_F64 ? 8 : 4;
  void* d = data;
  if (mem != PF_MEM_DEVICE) {
    TRY(ensure(P, &P->io_dev, &P->io_cap, count * es));
    CK(cudaMemcpyAsync(P->io_dev, data, count * es, cudaMemcpyHostToDevice, P->stream));
    d = P->io_dev;
  }
  ProfRec rec;
  TRY(prof_begin(P, "transform", count * 2.0 * es, &rec));
  if (es == 8)
    k_transform<double><<<grid_for(count), kThreads, 0, P->stream>>>((double*)d, count, P->desc.transform,
                                                                    P->desc.boxcox_lambda);
  else
    k_transform<float><<<grid_for(count), kThreads, 0, P->stream>>>((float*)d, count, P->desc.transform,
                                                                   P->desc.boxcox_lambda);
  TRY(prof_end(P, &rec));
  if (mem != PF_MEM_DEVICE) CK(cudaMemcpyAsync(data, d, count * es, cudaMemcpyDeviceToHost, P->stream));
  return check_bounds(P, PF_OK);
}

pf_status pf_profile_enable(pf_plan* P, int32_t enable) {
  if (!P) return fail(PF_ERR_ARG, "null plan");
  CK(cudaStreamSynchronize(P->stream));
  for (auto& r : P->recs) {
    P->evpool.push_back(r.e0);
    P->evpool.push_back(r.e1);
  }
  P->recs.clear();
  P->prof = enable != 0;
  return PF_OK;
}

pf_status pf_profile_read(pf_plan* P, pf_kernel_time* out, int32_t cap, int32_t* count) {
  if (!P || !count) return fail(PF_ERR_ARG, "null argument");
  CK(cudaStreamSynchronize(P->stream));
  std::vector<std::string> order;
  std::map<std::string, pf_kernel_time> agg;
  for (auto& r : P->recs) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, r.e0, r.e1));
    auto it = agg.find(r.name);
    if (it == agg.end()) {
      pf_kernel_time k{};
      snprintf(k.name, sizeof(k.name), "%s", r.name);
      it = agg.emplace(r.name, k).first;
      order.push_back(r.name);
    }
    it->second.launches++;
    it->second.total_ms += ms;
    it->second.bytes += r.bytes;
  }
  int n = 0;
  for (auto& nm : order) {
    if (n < cap && out) out[n] = agg[nm];
    n++;
  }
  *count = n;
  return PF_OK;
}

uint64_t pf_launch_count(const pf_plan* P) { return P ? P->launches : 0; }

const char* pf_last_error_string(void) { return g_err.c_str(); }

const char* pf_version(void) { return "parafields-b200 0.1 (sm_100a)"; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Matrix-vector product without any device allocation
//
// Some callers cannot allocate device memory at the moment they need a product with
// the covariance: code running inside another framework's memory pool (which may
// own all of the GPU's memory), and solvers that reserve their memory once at start-up
// and treat a later cudaMalloc as an error because it synchronizes the device.  For
// them this variant of the 2D matvec keeps its scratch (the half-spectrum torus and the
// twiddle tables) in one fixed array that is part of the library image, so a call
// allocates nothing.
//
// The array is a file-scope __device__ symbol: every GPU that loads the library holds
// it until the process exits.  Its host-side name is only a stand-in, so the device
// address is fetched with cudaGetSymbolAddress once per device, on the first call made
// with that device current; make that first call before any stream capture starts.
// All calls share the array and every call rewrites the parts it reads, so nothing in
// it has to start at zero; calls that overlap on the GPU (other streams, other plans,
// other threads) race on it and must be serialized by the caller.
// ---------------------------------------------------------------------------
constexpr size_t kStaticScratchElems = size_t(1) << 18;  // complex doubles: 4 MiB
static __device__ __align__(256) double2 g_static_scratch[kStaticScratchElems];

static std::mutex g_static_mutex;
static double2* g_static_addr[128] = {nullptr};

static pf_status static_scratch_address(int plan_device, double2** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev != plan_device)
    return fail(PF_ERR_ARG, "pf_matvec_static: the plan's device (%d) must be the current device (%d)", plan_device,
                dev);
  if (dev < 0 || dev >= 128) return fail(PF_ERR_ARG, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_static_mutex);
  if (!g_static_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return fail(PF_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
    g_static_addr[dev] = (double2*)p;
  }
  *out = g_static_addr[dev];
  return PF_OK;
}

// exp(-2 pi i m / L), m < L, into tw
__global__ void k_static_twiddles(double2* tw, int L) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < L; m += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)m / (double)L, &s, &c);
    tw[m] = make_double2(c, s);
  }
}

// eigenvalue factor computed from the FP64 spectrum on the fly (no factor array)
struct StaticMid {
  static constexpr bool active = true;
  int T0, T1, C0, layout, D0;
  int op;
  double N;
  const double* lam;
  long long nlam;
  template <typename T>
  __device__ __forceinline__ cx<T> operator()(long long p, int j, long long, cx<T> v) const {
    const int k0 = (int)p, k1 = j;
    long long li;
    if (layout == 0) {
      const int m1 = k1 <= T1 / 2 ? k1 : T1 - k1;
      li = (long long)k0 + (long long)D0 * m1;
    } else {
      li = (long long)k0 + (long long)C0 * k1;
    }
    if (!in_bounds(li, nlam)) return mk<T>(0, 0);
    const double l = lam[li];
    const double f = op == 0 ? l / N : (op == 1 ? sqrt(l) / N : (1. / l) / N);
    return mk<T>((T)(v.x * f), (T)(v.y * f));
  }
};

extern "C" pf_status pf_matvec_static(pf_plan* P, int32_t op, const double* in, double* out) {
  if (!P || !in || !out) return fail(PF_ERR_ARG, "null argument");
  if (op < 0 || op > 2) return fail(PF_ERR_ARG, "unknown operation");
  const Geom& g = P->g;
  if (g.dim != 2 || g.fb != PF_FIELD_R2C)
    return fail(PF_ERR_CONFIG, "pf_matvec_static serves 2D plans with the R2C field backend");
  if (!P->have_spec) return fail(PF_ERR_STATE, "spectrum not built: call pf_spectrum_build first");
  // the kernels only reach device memory of the plan's GPU: anything else is refused
  // here instead of faulting inside a kernel
  for (const void* p : {(const void*)in, (const void*)out}) {
    cudaPointerAttributes at{};
    const cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(PF_ERR_ARG, "pf_matvec_static: in/out must be device pointers (%s)", cudaGetErrorString(e));
    }
    if ((at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged) || at.device != P->device)
      return fail(PF_ERR_ARG, "pf_matvec_static: in/out must be device memory of the plan's GPU %d", P->device);
  }
  const int T0 = g.T[0], T1 = g.T[1], L0 = T0 / 2, T0c = g.T0c, n0 = g.n[0], n1 = g.n[1];
  const size_t nX = (size_t)T0c * n1;
  const size_t need = nX + (size_t)L0 + (size_t)T0 + (size_t)T1;
  if (need > kStaticScratchElems)
    return fail(PF_ERR_ARG, "field too large for the static scratch: needs %zu complex doubles, limit %zu", need,
                kStaticScratchElems);
  double2* base = nullptr;
  TRY(static_scratch_address(P->device, &base));
  double2* X = base;
  double2* twL = X + nX;
  double2* twT = twL + L0;
  double2* tw1 = twT + T0;
  k_static_twiddles<<<8, 256, 0, P->stream>>>(twL, L0);
  k_static_twiddles<<<8, 256, 0, P->stream>>>(twT, T0);
  k_static_twiddles<<<8, 256, 0, P->stream>>>(tw1, T1);
  P->launches += 3;
  CK(cudaGetLastError());
  ArrStore<double2> xs{X, 1u, 0u, (unsigned)T0c, (unsigned)nX};
  ArrLoad<double2> xl0{X, 1u, 0u, (unsigned)T0c, (unsigned)nX, T0c};
  FieldRowLoad<double> fl{in, n0, (unsigned)g.domain};
  FieldRowStore<double> fs{out, n0, 0, 0.0, (unsigned)g.domain};
  // dimension 0 forward (r2c with zero padding)
  PassArgs a{};
  a.L = L0;
  a.Lout = T0c;
  a.npencil = n1;
  a.nouter = 1;
  a.sign = -1;
  if (!make_radices(L0, &a.rad)) return fail(PF_ERR_CONFIG, "length %d has a prime factor above 13", T0);
  tile_params(L0, 16, true, &a);
  size_t smem = smem_of(a, true, 16);
  if (smem > 227 * 1024) return fail(PF_ERR_CONFIG, "row of length %d does not fit in shared memory", T0);
  {
    auto kern = k_r2c<double, FieldRowLoad<double>, ArrStore<double2>>;
    TRY(set_smem(kern, smem));
    kern<<<(unsigned)((n1 + a.B - 1) / a.B), kThreads, smem, P->stream>>>(a, twL, twT, fl, xs);
  }
  // dimension 1: forward, eigenvalue factor, backward, in place
  StaticMid mid{T0, T1, g.mb == PF_MATRIX_R2C ? T0c : T0, g.mb == PF_MATRIX_DCT ? 0 : 1, T0 / 2 + 1, op,
                (double)g.N, P->lam64, (long long)g.S};
  PassArgs b{};
  b.L = T1;
  b.Lout = n1;
  b.npencil = T0c;
  b.nouter = 1;
  b.sign = -1;
  b.sign2 = +1;
  if (!make_radices(T1, &b.rad)) return fail(PF_ERR_CONFIG, "length %d has a prime factor above 13", T1);
  tile_params(T1, 16, false, &b);
  smem = smem_of(b, false, 16);
  if (smem > 227 * 1024) return fail(PF_ERR_CONFIG, "pencil of length %d does not fit in shared memory", T1);
  {
    ArrLoad<double2> xl1{X, (unsigned)T0c, 0u, 1u, (unsigned)nX, n1};
    ArrStore<double2> xs1{X, (unsigned)T0c, 0u, 1u, (unsigned)nX};
    auto kern = k_pass<double, false, ArrLoad<double2>, StaticMid, ArrStore<double2>>;
    TRY(set_smem(kern, smem));
    kern<<<(unsigned)((T0c + b.B - 1) / b.B), kThreads, smem, P->stream>>>(b, tw1, xl1, mid, xs1);
  }
  // dimension 0 backward (c2r) with extraction of the domain
  a.sign = +1;
  a.Lout = n0;
  smem = smem_of(a, true, 16);
  {
    auto kern = k_c2r<double, ArrLoad<double2>, FieldRowStore<double>>;
    TRY(set_smem(kern, smem));
    kern<<<(unsigned)((n1 + a.B - 1) / a.B), kThreads, smem, P->stream>>>(a, twL, twT, xl0, fs);
  }
  P->launches += 3;
  CK(cudaGetLastError());
  return PF_OK;
}

#include "pf_ensemble.inc"
#include "pf_tune.inc"
#include "pf_peaks.inc"
#include "pf_io.inc"
