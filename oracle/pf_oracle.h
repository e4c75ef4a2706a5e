/*
 * pf_oracle.h -- FP64 CPU restatement of parafields-core's circulant-embedding path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline legs of bench.py may load this library; the product path
 * (libpfcuda.so) never links or calls it.
 *
 * Parity status: the reference cannot be built here (FFTW3/FFTW3-MPI, MPI and
 * dune-common are absent) and its own tests hold no golden vectors
 * (test/fieldtest.cc:8-57 only call generate()), so parity with the reference
 * binary is UNPINNED.  The FFTW conventions the reference relies on (unnormalised
 * backward transforms, R2C half-spectrum along parafields dimension 0, c2r
 * ignoring the imaginary part of the DC/Nyquist entries, REDFT00 = DCT-I) are
 * pinned against scipy.fft (pocketfft) by tests/test_oracle_fft.py.
 *
 * All arrays use the reference's order: dimension 0 fastest.
 */
#ifndef PF_ORACLE_H
#define PF_ORACLE_H

#include <stdint.h>

#include "../include/parafields_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Resolved geometry of a descriptor (fieldtraits.hh:217-314). */
typedef struct oc_geom {
  int dim;
  int n[3];        /* cells */
  int T[3];        /* extended cells */
  int Ts[3];       /* extended cells in the stored frequency layout (swapped when transposed) */
  double h[3];     /* meshsize */
  double ext[3];
  int factor;
  int matrix_backend;
  int field_backend;
  int transposed;
  uint64_t domain;   /* prod n */
  uint64_t N;        /* prod T */
  uint64_t Nc;       /* (T0/2+1) prod_{i>0} T_i */
  uint64_t D;        /* prod (T_i/2+1) */
  uint64_t spectrum; /* stored eigenvalue count */
  uint64_t noise;    /* doubles per realization */
} oc_geom;

int oc_resolve(const pf_field_desc* d, oc_geom* g, char* err, int errlen);

/* One covariance functor (covariance.hh:296-823) at transformed coordinate x. */
double oc_covariance(const pf_field_desc* d, const double* x);
/* Modified Bessel function K_nu(x) (stands in for gsl_sf_bessel_Knu). */
double oc_bessel_k(double nu, double x);
/* Geometry transform (covariance.hh:18-138). */
void oc_geometry(const pf_field_desc* d, const double* x, double* xt);

/* Complex FFT (unnormalised, sign -1 forward / +1 backward) of arbitrary length,
 * interleaved re/im. */
void oc_fft(int n, double* data, int sign);
/* Along one axis of a multi-dim complex array (dimension 0 fastest). */
void oc_fft_axis(double* data, int ndim, const int* shape, int axis, int sign);
/* FFTW-semantics real transforms on natural layout (dimension 0 halved). */
void oc_r2c(int ndim, const int* T, const double* in, double* out);
void oc_c2r(int ndim, const int* T, const double* in, double* out);
/* REDFT00 (DCT-I) along every axis, in place, shape m_i. */
void oc_dct1(int ndim, const int* m, double* data);

/* Untransformed matrix entries exactly as computeMatrixEntriesWithMirroring fills
 * them (matrix.hh:615-638), in the backend's pre-transform layout:
 * DCT prod(T_i/2+1); R2C padded 2(T0/2+1) x T1 x T2; DFT prod T_i. */
int oc_fill_matrix(const pf_field_desc* d, double* out, uint64_t count);

/* fillTransformedMatrix (matrix.hh:223-318). `lambda` receives g.spectrum FP64
 * eigenvalues in the reference's storage layout.  Returns PF_OK or
 * PF_ERR_NEG_EIGEN (lambda and stats are filled in both cases). */
int oc_spectrum(const pf_field_desc* d, double* lambda, pf_eig_stats* stats);

/* generateField (matrix.hh:330-421) from noise in the reference's draw order.
 * field receives prod(cells) values; spare (may be NULL) receives the DFT
 * backend's second field. */
int oc_generate(const pf_field_desc* d, const double* lambda, const double* noise,
                double* field, double* spare);

/* multiplyExtended / multiplyRootExtended / multiplyInverseExtended. */
int oc_matvec(const pf_field_desc* d, const double* lambda, int op, const double* in,
              double* out);

/* multiplyInverse (matrix.hh:189-206) with innerCG (matrix.hh:1315-1432);
 * returns the CG iteration count through *iterations. */
int oc_multiply_inverse(const pf_field_desc* d, const double* lambda, const double* b,
                        double* x, int* iterations);

/* ValueTransform::apply (mutators.hh:35-163). */
void oc_transform(int kind, double boxcox_lambda, double* v, uint64_t n);

/* Stored frequency (reference layout index) -> eigenvalue lookup
 * (dctmatrixbackend.hh:346-355, r2cmatrixbackend.hh:337-362). */
double oc_eval_stored(const pf_field_desc* d, const oc_geom* g, const double* lambda,
                      uint64_t stored_index);

int oc_num_threads(void);
void oc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
