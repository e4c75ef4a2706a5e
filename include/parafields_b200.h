/*
 * parafields_b200.h -- C ABI of the single-GPU (B200, sm_100a) circulant-embedding
 * path of parafields-core.
 *
 * The reference exposes this path as the C++ template class
 *   parafields::Matrix<Traits, MatrixBackend, FieldBackend>   (include/parafields/matrix.hh:55-133)
 * plugged into RandomField<GridTraits, IsoMatrix, AnisoMatrix> (include/parafields/randomfield.hh:42-47).
 * Its per-element backend concept (set/eval/mult called inside host loops,
 * matrix.hh:378-404) cannot be honoured by a GPU, so the drop-in sits at the Matrix level:
 * every entry point below replaces one Matrix member (cited per function), and the
 * C++ facade in parafields-core_b200/include/parafields_b200/ maps the reference's
 * Dune::ParameterTree keys and RandomField methods onto these calls.
 *
 * Conventions (all identical to the reference, single MPI rank):
 *  - multi-dimensional arrays are stored with dimension 0 fastest
 *    (fieldtraits.hh:400-430, indicesToIndex / indexToIndices);
 *  - extended (torus) cells T_i = embedding_factor * cells_i (fieldtraits.hh:269-272);
 *  - every forward transform divides by N = prod T_i, backward transforms are
 *    unnormalised (r2cmatrixbackend.hh:279-282, r2cfieldbackend.hh:233-236), so
 *    pf_matvec(PF_OP_MUL) returns (C_ext x)/N restricted to the domain, exactly as
 *    Matrix::operator* does (matrix.hh:142-151, 1443-1501);
 *  - spectra and noise use the reference's storage order, including the 3D
 *    "transposed" frequency layout (fftw.transposed, fieldtraits.hh:229-267).
 *
 * Errors: every function returns a pf_status; pf_last_error_string() gives the
 * message of the last failure on the calling thread.  PF_ERR_NEG_EIGEN carries the
 * text of the reference's NegativeEigenvalueError (matrix.hh:307-315).
 *
 * Threading: one plan is used by one host thread at a time (the reference's Matrix
 * is not thread-safe either, matrix.hh:87-90); distinct plans are independent.
 */
#ifndef PARAFIELDS_B200_H
#define PARAFIELDS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum pf_status {
  PF_OK = 0,
  PF_ERR_NEG_EIGEN = 1,     /* NegativeEigenvalueError, exceptions.hh:8-15 */
  PF_ERR_CONFIG = 2,        /* std::runtime_error for an invalid configuration */
  PF_ERR_OOM = 3,           /* device or pinned-host allocation failed */
  PF_ERR_CUDA = 4,          /* a CUDA runtime call failed */
  PF_ERR_NOT_CONVERGED = 5, /* CG hit its iteration cap without the requested residual */
  PF_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up */
  PF_ERR_STATE = 7,         /* call order violated (e.g. spectrum missing) */
  PF_ERR_ARG = 8,           /* null pointer / size mismatch */
  PF_ERR_IO = 9             /* a field file is missing, unreadable or not of the expected shape */
} pf_status;

/* stochastic.covariance (matrix.hh:232-260) */
typedef enum pf_covariance {
  PF_COV_EXPONENTIAL = 0,
  PF_COV_GAUSSIAN = 1,
  PF_COV_SPHERICAL = 2,
  PF_COV_SEPARABLE_EXPONENTIAL = 3,
  PF_COV_MATERN = 4,
  PF_COV_MATERN32 = 5,
  PF_COV_MATERN52 = 6,
  PF_COV_DAMPED_OSCILLATION = 7,
  PF_COV_GAMMA_EXPONENTIAL = 8,
  PF_COV_CAUCHY = 9,
  PF_COV_GENERALIZED_CAUCHY = 10,
  PF_COV_CUBIC = 11,
  PF_COV_WHITE_NOISE = 12,
  /* "custom-iso" / "custom-aniso": the matrix comes from the caller's covariance values,
   * pf_spectrum_build_values (matrix.hh:223-230) */
  PF_COV_CUSTOM = 13
} pf_covariance;

/* stochastic.anisotropy (matrix.hh:479-493) */
typedef enum pf_anisotropy {
  PF_ANISO_NONE = 0,        /* ScaledIdentityMatrix, covariance.hh:18-44 */
  PF_ANISO_AXIPARALLEL = 1, /* DiagonalMatrix, covariance.hh:49-74 */
  PF_ANISO_GEOMETRIC = 2    /* GeneralMatrix, covariance.hh:79-138 */
} pf_anisotropy;

/* Matrix backends (matrix.hh:1652-1735 give the defaults) */
typedef enum pf_matrix_backend {
  PF_MATRIX_DEFAULT = -1,
  PF_MATRIX_DCT = 0, /* DCTMatrixBackend, backends/dctmatrixbackend.hh */
  PF_MATRIX_R2C = 1, /* R2CMatrixBackend, backends/r2cmatrixbackend.hh */
  PF_MATRIX_DFT = 2  /* DFTMatrixBackend, backends/dftmatrixbackend.hh */
} pf_matrix_backend;

/* Field backends */
typedef enum pf_field_backend {
  PF_FIELD_DEFAULT = -1,
  PF_FIELD_R2C = 0,   /* R2CFieldBackend, backends/r2cfieldbackend.hh */
  PF_FIELD_DFT = 1,   /* DFTFieldBackend, backends/dftfieldbackend.hh */
  PF_FIELD_DCTDST = 2 /* DCTDSTFieldBackend, backends/dctdstfieldbackend.hh */
} pf_field_backend;

/* randomField.transform (mutators.hh:126-163) */
typedef enum pf_transform {
  PF_TRANSFORM_NONE = 0,
  PF_TRANSFORM_LOGNORMAL = 1,
  PF_TRANSFORM_FOLDEDNORMAL = 2,
  PF_TRANSFORM_SIGN = 3,
  PF_TRANSFORM_BOXCOX = 4
} pf_transform;

/* Arithmetic of the per-realization path (spectrum, CG reductions and residuals
 * are always FP64). */
typedef enum pf_precision { PF_PREC_F64 = 0, PF_PREC_F32 = 1 } pf_precision;

/* Eigenvalue scan after the spectrum transform (matrix.hh:266-317).
 * CORRECTED scans every stored eigenvalue.  REFERENCE reproduces the reference
 * exactly, including the R2C real-view scan that only inspects the first N_c/2
 * complex entries (r2cmatrixbackend.hh:164-170 with get/set 378-400). */
typedef enum pf_eigen_check { PF_EIGCHECK_CORRECTED = 0, PF_EIGCHECK_REFERENCE = 1 } pf_eigen_check;

/* Matrix-vector product kinds (matrix.hh:1443-1646) */
typedef enum pf_op {
  PF_OP_MUL = 0,    /* multiplyExtended: eigenvalue lambda */
  PF_OP_ROOT = 1,   /* multiplyRootExtended: sqrt(lambda) */
  PF_OP_INVEXT = 2  /* multiplyInverseExtended: 1/lambda (torus inverse) */
} pf_op;

/* Where a caller buffer lives. */
typedef enum pf_mem { PF_MEM_HOST = 0, PF_MEM_DEVICE = 1 } pf_mem;

/* Field / covariance configuration: one field per Dune::ParameterTree key the
 * reference reads on this path (fieldtraits.hh:175-186, 229; matrix.hh:268-269,
 * 479-480, 515-519; covariance.hh:33-128, 395-396, 515-516, 711-713;
 * mutators.hh:139-154). */
typedef struct pf_field_desc {
  int32_t dim;               /* 1, 2 or 3 */
  int32_t cells[3];          /* grid.cells */
  double extensions[3];      /* grid.extensions */
  int32_t embedding_factor;  /* embedding.factor (default 2) */
  int32_t periodic;          /* randomField.periodic: forces embedding factor 1 */
  int32_t covariance;        /* pf_covariance, stochastic.covariance */
  double variance;           /* stochastic.variance */
  int32_t anisotropy;        /* pf_anisotropy, stochastic.anisotropy */
  double corr_length[9];     /* stochastic.corrLength: scalar, dim-vector or dim x dim row-major */
  double matern_nu;          /* stochastic.maternNu */
  double exp_gamma;          /* stochastic.expGamma */
  double cauchy_alpha;       /* stochastic.cauchyAlpha */
  double cauchy_beta;        /* stochastic.cauchyBeta */
  int32_t approximate;       /* embedding.approximate (default false) */
  double threshold;          /* embedding.threshold (default 1e-14) */
  int32_t transposed;        /* fftw.transposed: -1 = reference default */
  int32_t matrix_backend;    /* pf_matrix_backend */
  int32_t field_backend;     /* pf_field_backend */
  int32_t precision;         /* pf_precision of realizations and FP32 matvecs */
  int32_t eigen_check;       /* pf_eigen_check */
  int32_t cg_iterations;     /* randomField.cgIterations (default 100) */
  int32_t transform;         /* pf_transform, randomField.transform */
  double boxcox_lambda;      /* transform.boxCoxLambda */
  /* smooth periodization (matrix.hh:510-602, 652-890): */
  int32_t periodization;     /* pf_periodization, embedding.periodization */
  int32_t sigmoid;           /* pf_sigmoid, embedding.sigmoid */
  int32_t sigmoid_combine;   /* pf_sigmoid_combine, stochastic.sigmoidCombine */
  int32_t merge_recursions;  /* embedding.mergeRecursions (99: the covariance's default) */
  double sigmoid_start;      /* embedding.sigmoidStart (default 1) */
  double sigmoid_end;        /* embedding.sigmoidEnd (negative: default factor - 1) */
  double fold_max_factor;    /* embedding.foldMaxFactor (default 1) */
  int32_t fold_recursions;   /* embedding.foldRecursions (99: the covariance's default) */
  int32_t cofold_recursions; /* embedding.cofoldRecursions (default 1) */
  double cofold_max_factor;  /* embedding.cofoldMaxFactor (default 5) */
} pf_field_desc;

/* embedding.periodization: classical mirroring, sigmoid merging of the 2^d mirrored copies,
 * folding of the distances beyond the domain, or cofolding of the covariance values beyond
 * the domain (cofold: DCT matrix backend, i.e. anisotropy none / axiparallel) */
typedef enum pf_periodization {
  PF_PERIODIZATION_CLASSICAL = 0,
  PF_PERIODIZATION_MERGE = 1,
  PF_PERIODIZATION_FOLD = 2,
  PF_PERIODIZATION_COFOLD = 3
} pf_periodization;
/* embedding.sigmoid (covariance.hh:147-287) */
typedef enum pf_sigmoid { PF_SIGMOID_SMOOTHSTEP = 0, PF_SIGMOID_SMOOTH = 1 } pf_sigmoid;
/* stochastic.sigmoidCombine (matrix.hh:668-677) */
typedef enum pf_sigmoid_combine {
  PF_COMBINE_RADIAL_PLUS = 0,
  PF_COMBINE_RADIAL = 1,
  PF_COMBINE_TENSOR = 2
} pf_sigmoid_combine;

/* Eigenvalue statistics of matrix.hh:270-299 (counts and minimum). */
typedef struct pf_eig_stats {
  uint32_t small;    /* threshold <= value < 1e-6 */
  uint32_t zero;     /* |value| < threshold */
  uint32_t negative; /* value <= -threshold */
  uint32_t pad_;
  double smallest;   /* minimum scanned value */
} pf_eig_stats;

/* Sizes the plan resolved from the descriptor (fieldtraits.hh:217-314). */
typedef struct pf_plan_info {
  int32_t dim;
  int32_t cells[3];
  int32_t ext_cells[3];     /* T_i */
  int32_t matrix_backend;   /* resolved pf_matrix_backend */
  int32_t field_backend;    /* resolved pf_field_backend */
  int32_t transposed;       /* resolved fftw.transposed */
  int32_t precision;
  uint64_t domain_size;     /* prod cells_i */
  uint64_t ext_size;        /* N = prod T_i */
  uint64_t spectrum_size;   /* stored eigenvalues: D (DCT), N_c (R2C), N (DFT) */
  uint64_t noise_size;      /* doubles consumed per realization (reference draw order) */
  uint64_t device_bytes;    /* device memory held by the plan */
} pf_plan_info;

/* CG options and report for pf_multiply_inverse (matrix.hh:189-206, 1315-1432). */
typedef enum pf_cg_mode {
  PF_CG_REFERENCE = 0, /* the reference's energy-stagnation rule and iteration cap */
  PF_CG_RESIDUAL = 1   /* stop at ||b - A x|| / ||b|| <= tol with an FP64 true residual */
} pf_cg_mode;

typedef struct pf_cg_opts {
  int32_t mode;            /* pf_cg_mode */
  int32_t max_iterations;  /* 0 = desc.cg_iterations (reference) or 1000 (residual mode) */
  double tolerance;        /* relative residual target for PF_CG_RESIDUAL (e.g. 1e-8) */
  int32_t inner_fp32;      /* 1: inner CG matvecs in FP32 with FP64 refinement */
  int32_t precondition;    /* 1: torus-inverse preconditioner (reference default) */
} pf_cg_opts;

typedef struct pf_cg_report {
  int32_t iterations;        /* total inner CG iterations */
  int32_t refinements;       /* outer FP64 residual recomputations */
  double relative_residual;  /* final ||b - A x|| / ||b|| (FP64 matvec) */
} pf_cg_report;

typedef struct pf_plan pf_plan;

/* Fills the descriptor with the reference's defaults (embedding.factor 2,
 * threshold 1e-14, cgIterations 100, transposed default, FP64, isotropic
 * exponential with unit variance and extensions). */
void pf_field_desc_init(pf_field_desc* desc);

/* Replaces the Matrix constructor + update() (matrix.hh:98-133) together with the
 * size computation of RandomFieldTraits::update (fieldtraits.hh:217-314) and the
 * default backend selection of RandomField (randomfield.hh:153-164). Allocates the
 * plan's device buffers; no transform runs here (the spectrum is lazy, as in the
 * reference, matrix.hh:333-334). */
pf_status pf_plan_create(const pf_field_desc* desc, pf_plan** plan);
void pf_plan_destroy(pf_plan* plan);

/* Launches all work of the plan on `stream` (a cudaStream_t; NULL = the plan's own). */
pf_status pf_plan_set_stream(pf_plan* plan, void* stream);
pf_status pf_plan_get_info(const pf_plan* plan, pf_plan_info* info);

/* Matrix::fillTransformedMatrix(covariance string) (matrix.hh:223-318): FP64
 * covariance evaluation on the torus (matrix.hh:615-638), FP64 spectrum transform
 * with the /N scaling, eigenvalue scan, clamp, and the NegativeEigenvalueError
 * rule (PF_ERR_NEG_EIGEN unless desc.approximate). `stats` may be NULL. */
pf_status pf_spectrum_build(pf_plan* plan, pf_eig_stats* stats);

/* Matrix::fillTransformedMatrix(Covariance&&) with a covariance functor of the caller's
 * own (matrix.hh:223-265, the "custom-iso"/"custom-aniso" covariances that
 * RandomField::fillMatrix passes in, randomfield.hh:430-451): the caller evaluates its
 * functor on the host at the matrix cells and hands over the values; the rest is
 * pf_spectrum_build (FP64 transform with the /N scaling, eigenvalue scan, clamp,
 * NegativeEigenvalueError rule).  `values` (memory `mem`) holds one value per matrix
 * cell, dimension 0 fastest, in the natural (untransposed) order: prod(T_i/2+1) cells
 * (index i_d in [0, T_d/2]) for the DCT matrix backend, prod(T_i) for R2C and DFT; cell
 * index i_d stands for the coordinate i_d * h_d, minus T_d * h_d beyond half the torus
 * (matrix.hh:615-638).  PF_ERR_ARG when `count` differs from that cell count. */
pf_status pf_spectrum_build_values(pf_plan* plan, const double* values, uint64_t count, int32_t mem,
                                   pf_eig_stats* stats);

/* Copies the finalized eigenvalues (FP64) in the reference's storage layout
 * (DCT: prod(T_i/2+1); R2C: N_c real parts; DFT: N real parts). */
pf_status pf_spectrum_copy(pf_plan* plan, double* out, uint64_t count);

/* Matrix::generateField (matrix.hh:330-421) for one realization.
 * noise != NULL: `noise` holds info.noise_size standard-normal doubles in the
 * reference's draw order (rand1, rand2 per stored frequency, matrix.hh:378-404),
 * in memory `noise_mem`.  noise == NULL: the noise is drawn on the device from a
 * counter-based generator keyed by `seed`.
 * `out` receives prod(cells) values (double for PF_PREC_F64, float for PF_PREC_F32)
 * in memory `out_mem`, with the descriptor's value transform applied when
 * `apply_transform` is nonzero (RandomField::evaluate, randomfield.hh:641-651).
 * With the DFT field backend the second (imaginary) field is cached in the plan
 * and returned by the next call without consuming noise (matrix.hh:411-420). */
pf_status pf_generate(pf_plan* plan, const double* noise, int32_t noise_mem, uint64_t seed,
                      void* out, int32_t out_mem, int32_t apply_transform);

/* The noise a seeded pf_generate call of this plan draws (seed, and the epoch an ensemble
 * mixes in: 0 for plans, the call number for ensemble fields), written as info.noise_size
 * doubles in the reference's draw order (rand1, rand2 per stored frequency,
 * matrix.hh:378-404) into `out` (memory `mem`).  Fed to pf_generate as a noise buffer, or to
 * a host implementation of the reference, it reproduces the seeded realization (to the
 * rounding of the plan's precision).  No counterpart in the reference, whose noise comes from
 * host generators.  R2C field backend only (PF_ERR_CONFIG otherwise). */
pf_status pf_export_noise(pf_plan* plan, uint64_t seed, uint32_t epoch, double* out, int32_t mem);

/* `count` realizations keyed by seed, seed+1, ... written back to back into `out` (which must
 * hold count * prod(cells) values).  For the R2C field backend the realizations run on two
 * streams: alternating, or (device output, chosen by pf_plan_autotune when faster) as a
 * stage pipeline with the noise pass of one realization beside the remaining passes of the
 * previous one. */
pf_status pf_generate_batch(pf_plan* plan, uint64_t seed, int32_t count, void* out,
                            int32_t out_mem, int32_t apply_transform);

/* Ensembles: many independent fields, each with its own size and covariance, generated
 * together.  In the reference every field is its own RandomField and generate() call
 * (randomfield.hh:512-558, matrix.hh:330-421); here one handle plans them all, builds
 * every FP64 spectrum once, captures the realization passes of all fields into one CUDA
 * graph (branches on several streams) and replays that graph with one launch per call.
 * All descriptors must share a precision and use the R2C field backend.  Field i of call
 * c (c = 1, 2, ...) is the counter-based realization keyed by seed + i with the call
 * number mixed into the counters, so calls draw new, reproducible realizations. */
typedef struct pf_ensemble pf_ensemble;
pf_status pf_ensemble_create(const pf_field_desc* descs, int32_t count, uint64_t seed,
                             pf_ensemble** ensemble);
void pf_ensemble_destroy(pf_ensemble* ensemble);
/* count, total cells, and offsets[count + 1] (field i at [offsets[i], offsets[i+1])) */
pf_status pf_ensemble_info(const pf_ensemble* ensemble, int32_t* count, uint64_t* total_cells,
                           uint64_t* offsets);
/* fillTransformedMatrix for every field; `stats` (count entries) and `failed` may be NULL.
 * Returns PF_ERR_NEG_EIGEN if any field without embedding.approximate has negative
 * eigenvalues (the other fields are still built). */
pf_status pf_ensemble_spectra(pf_ensemble* ensemble, pf_eig_stats* stats, int32_t* failed);
/* One realization of every field, concatenated into `out` (memory `out_mem`; NULL keeps
 * them in the device buffer of pf_ensemble_device_output).  The first call captures the
 * graph; every call is one graph launch.  Synchronous. */
pf_status pf_ensemble_generate(pf_ensemble* ensemble, void* out, int32_t out_mem);
/* Measured planning (pf_plan_autotune) of every field's realization passes, after
 * pf_ensemble_spectra; fields of one geometry share one timing through the wisdom table.
 * `timed` (may be NULL) receives the number of fields that were timed.  A graph captured
 * earlier is dropped and recaptured with the tuned kernels by the next generate call. */
pf_status pf_ensemble_autotune(pf_ensemble* ensemble, int32_t repetitions, int32_t* timed);
/* Replays the captured graph on `stream` (a cudaStream_t used as given; 0 is the legacy
 * default stream) without waiting. */
pf_status pf_ensemble_launch(pf_ensemble* ensemble, void* stream);
const void* pf_ensemble_device_output(const pf_ensemble* ensemble);
/* kernel launches inside one replay of the graph */
uint64_t pf_ensemble_launches_per_replay(const pf_ensemble* ensemble);

/* Matrix::operator* / multiplyRoot (matrix.hh:142-176, 1443-1573) and the torus
 * inverse multiplyInverseExtended (matrix.hh:1587-1646).  `in` and `out` hold
 * prod(cells) values of type `precision` (PF_PREC_F64: double, PF_PREC_F32: float);
 * in == out is allowed. */
pf_status pf_matvec(pf_plan* plan, int32_t op, int32_t precision, const void* in, void* out,
                    int32_t mem);

/* FP64 matrix-vector product (as pf_matvec with PF_PREC_F64) that allocates no memory.
 * No counterpart in the reference: it exists for callers that may not call cudaMalloc
 * when they need the product -- code living inside another framework's memory pool, and
 * solvers that reserve all device memory at start-up and cannot afford the device
 * synchronization of a later allocation.
 * Limits: 2D plans with the R2C field backend (PF_ERR_CONFIG otherwise), spectrum already
 * built (PF_ERR_STATE otherwise); `in`/`out` are device pointers of prod(cells) doubles on
 * the plan's GPU, which must be the current device (PF_ERR_ARG otherwise); the scratch
 * (T0/2+1)*n1 + T0/2 + T0 + T1 complex doubles must fit in the library's fixed
 * 2^18-element (4 MiB) device array (PF_ERR_ARG otherwise); torus lengths with a prime
 * factor above 13 (no Bluestein transform on this path) and rows whose transform tile
 * exceeds 227 KiB of shared memory return PF_ERR_CONFIG (pf_matvec serves both).
 * The array lives in every GPU that loads the library until the process exits; the first
 * call on a device looks up its address (make that call before any stream capture).
 * Calls share the array: calls that overlap on the GPU race and must be serialized.
 * Asynchronous on the plan's stream. */
pf_status pf_matvec_static(pf_plan* plan, int32_t op, const double* in, double* out);

/* Matrix::multiplyInverse (matrix.hh:189-206): zero-input shortcut, torus-inverse
 * initial guess, then the preconditioned CG of innerCG (matrix.hh:1315-1432).
 * FP64 vectors; `opts` NULL = reference mode. */
pf_status pf_multiply_inverse(pf_plan* plan, const double* b, double* x, int32_t mem,
                              const pf_cg_opts* opts, pf_cg_report* report);

/* Matrix::multiplyInverse (matrix.hh:189-206) for `count` right-hand sides stored back to
 * back in B (prod(cells) doubles each, memory `mem`), solutions into X, one report per
 * right-hand side in `reports` (may be NULL).  Each solve is the computation of
 * pf_multiply_inverse on that right-hand side; up to `lanes` (1..8) solves run at once,
 * each on its own stream with its own workspaces (about 14 domain-sized FP64 vectors of
 * device memory per lane) sharing the plan's spectrum, so one solve's reductions and
 * host synchronizations overlap the others' transforms.  With a learned preconditioner
 * attached the solves run one at a time.  Synchronous. */
pf_status pf_multiply_inverse_batch(pf_plan* plan, const double* B, double* X, int32_t count, int32_t mem,
                                    const pf_cg_opts* opts, pf_cg_report* reports, int32_t lanes);

/* Learned boundary correction of the CG preconditioner.  No counterpart in the reference
 * (its innerCG preconditions with the torus inverse only, matrix.hh:1315-1432).  The
 * residual-mode CG preconditions the domain-restricted covariance with the torus inverse
 * P0 (zero-padded FFT round trip); the learned part rescales it as M = D P0 D, D a positive
 * diagonal d(x) = exp(sum_i psi(t_i(x))), t_i the distance of cell x to the nearer face
 * along axis i in correlation lengths and psi a 1-H-1 tanh network.  M is symmetric
 * positive definite for all parameters, so plain PCG stays valid and remains the judge
 * through its FP64 true residual.  Training (Adam, on the GPU) fits M b ~ x on pairs
 * (b, x = A^-1 b) produced by plain CG (loss: pf_learned_set_loss).  A residual-mode solve
 * that does not converge with the learned preconditioner is repeated with P0 alone.
 * The object refers to its plan: destroy it before the plan. */
typedef struct pf_learned pf_learned;
pf_status pf_learned_create(pf_plan* plan, int32_t hidden, uint64_t seed, pf_learned** learned);
void pf_learned_destroy(pf_learned* learned);
int32_t pf_learned_param_count(const pf_learned* learned);           /* 3 * hidden + 1 */
pf_status pf_learned_get_params(const pf_learned* learned, double* params);  /* host */
pf_status pf_learned_set_params(pf_learned* learned, const double* params);  /* host */
/* loss and gradient (host array of param_count, may be NULL) over `count` pairs stored
 * back to back (prod(cells) doubles each) in memory `mem`; fp32 selects FP32 transforms */
pf_status pf_learned_loss_grad(pf_learned* learned, const double* B, const double* X, int32_t count,
                               int32_t mem, int32_t fp32, double* loss, double* grad);
/* `epochs` full-batch Adam steps; *loss_out (may be NULL) = loss after training */
pf_status pf_learned_train(pf_learned* learned, const double* B, const double* X, int32_t count,
                           int32_t mem, int32_t epochs, double lr, int32_t fp32, double* loss_out);
/* Training loss: residual_norm = 0 (default) uses ||M b - x||^2 / ||x||^2; 1 uses
 * ||A (M b - x)||^2 / ||b||^2.  The residual norm is not invariant to a scalar factor of M
 * (PCG is): where ||A P0 b - b|| > ||b||, as on the 48^3 and 128^3 exponential test cases,
 * it drives D toward 0 (loss -> 1) and the trained M is useless for CG. */
pf_status pf_learned_set_loss(pf_learned* learned, int32_t residual_norm);
/* z = D P0 D r (FP64 transforms) */
pf_status pf_learned_apply(pf_learned* learned, const double* r, double* z, int32_t mem);
/* Attaches `learned` (NULL detaches) as the preconditioner of PF_CG_RESIDUAL solves of `plan`. */
pf_status pf_plan_set_preconditioner(pf_plan* plan, pf_learned* learned);

/* Measured planning, the counterpart of fftw.measure / fftw.useWisdom (r2cfieldbackend.hh:
 * 212-230, fieldtraits.hh:175-186): times every candidate of each realization pass of the
 * plan (paired-FP32 or scalar kernels x resident CTAs per SM of the persistent kernels,
 * `repetitions` realizations each, default 3) and keeps the fastest per pass (a pass whose
 * paired and scalar kernels come within 10% is decided on a batch); then, on batches of 4
 * realizations, the plane groups of the last two 3D passes and the batch mode of
 * pf_generate_batch.  Choices go to
 * a process-wide wisdom table keyed by the pass geometry; a plan whose passes are all in it
 * takes them without timing (*timed = 0).  Clears the plan's profiling records.  R2C field
 * backend only (other plans: no-op). */
pf_status pf_plan_autotune(pf_plan* plan, int32_t repetitions, int32_t* timed);
/* Wisdom as text, one line "pass L pencils outer precision variant ctas_per_sm" per entry
 * (pass 0..2 the realization passes; pass 3 holds the batch mode of pf_generate_batch in
 * `variant` -- 0 realizations alternating over two streams, 1 the stage pipeline -- and, for
 * 3D plans, in `ctas_per_sm` the number of plane groups over which the last two passes run
 * in turn, each group's intermediate reusing one buffer that stays in L2; 0 or 1 = one
 * group); *needed = bytes including the terminating NUL. */
pf_status pf_wisdom_export(char* buf, uint64_t cap, uint64_t* needed);
pf_status pf_wisdom_import(const char* text);
void pf_wisdom_forget(void);

/* ValueTransform::apply (mutators.hh:35-163) over `count` values of `precision`. */
pf_status pf_apply_transform(pf_plan* plan, int32_t precision, void* data, uint64_t count,
                             int32_t mem);

/* Per-kernel device timing: when enabled, every launch of the plan is bracketed by
 * CUDA events on the plan's stream and accumulated per kernel name. */
pf_status pf_profile_enable(pf_plan* plan, int32_t enable);
/* Writes up to `cap` entries; returns the number of kernels seen in *count. */
typedef struct pf_kernel_time {
  char name[48];
  uint64_t launches;
  double total_ms;
  double bytes;  /* algorithmic bytes moved by all launches (reads + writes) */
} pf_kernel_time;
pf_status pf_profile_read(pf_plan* plan, pf_kernel_time* out, int32_t cap, int32_t* count);

/* StochasticPart::writeToFile (stochastic.hh:273-294, io.hh:170-349): the field in `data`
 * (host or device memory per `mem`, FP64 or FP32 per `precision`, dimension 0 fastest) to
 * "<base>.stoch.h5" (dataset /stochastic, IEEE F64LE, dimensions the cells in reverse order)
 * and "<base>.xdmf".  The HDF5 file is written without libhdf5 (version 0 superblock,
 * symbol-table root group, contiguous dataset). */
pf_status pf_field_write(const char* base, int32_t dim, const int32_t* cells, const double* extensions,
                         const void* data, int32_t precision, int32_t mem);
/* StochasticPart(traits, fileName) (stochastic.hh:80-110): "<base>.stoch.h5" into `data`
 * (host or device, FP64 or FP32); PF_ERR_IO when the file is missing ("File is missing: ...")
 * or its dataset does not hold the cells. */
pf_status pf_field_read(const char* base, int32_t dim, const int32_t* cells, void* data, int32_t precision,
                        int32_t mem);

/* CUDA-core arithmetic peaks of `device` (B200 extension, no reference counterpart): FP32
 * FFMA, paired FP32 FFMA2 and FP64 DFMA throughput from an in-register FMA microbenchmark
 * (best of 3 timed launches after one warm-up), the denominators of compute fractions. */
typedef struct pf_peaks {
  double fp32_ffma_tflops;
  double fp32_ffma2_tflops;
  double fp64_dfma_tflops;
  double sm_clock_mhz; /* the device's nominal maximum SM clock */
  int32_t sms;
  int32_t pad_;
} pf_peaks;
pf_status pf_measure_peaks(int32_t device, pf_peaks* out);

/* Number of kernel launches issued by this plan since creation. */
uint64_t pf_launch_count(const pf_plan* plan);

const char* pf_last_error_string(void);
const char* pf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PARAFIELDS_B200_H */
