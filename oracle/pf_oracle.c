/*
 * pf_oracle.c -- FP64 CPU restatement of parafields-core's circulant-embedding path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline); the product
 * library never links it.  Parity with the reference binary is UNPINNED: the
 * reference needs FFTW3-MPI, MPI and dune-common, none of which exist here, and its
 * tests hold no golden vectors.  The FFT conventions are pinned against scipy.fft.
 *
 * Every function cites the reference lines it restates.  The FFT is this file's own
 * (Stockham autosort after Govindaraju et al., "High Performance Discrete Fourier
 * Transforms on Graphics Processors", SC 2008, plus Bluestein's chirp-z algorithm for
 * lengths with a prime factor above 61); it stands in for FFTW 3.3.8, the version CI
 * installs (.github/workflows/ci.yml:24-27).
 */
#include "pf_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_D 3.14159265358979323846264338327950288

int oc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------- */
/* configuration resolution: fieldtraits.hh:169-314, randomfield.hh:153-164    */
/* ------------------------------------------------------------------------- */

int oc_resolve(const pf_field_desc* d, oc_geom* g, char* err, int errlen) {
  memset(g, 0, sizeof(*g));
#define FAIL(msg)                                   \
  do {                                              \
    if (err) snprintf(err, (size_t)errlen, "%s", msg); \
    return PF_ERR_CONFIG;                           \
  } while (0)
  if (d->dim < 1 || d->dim > 3) FAIL("dimension must be 1, 2 or 3");
  g->dim = d->dim;
  g->factor = d->embedding_factor;
  if (d->periodic) g->factor = 1; /* fieldtraits.hh:199-205 */
  if (g->factor < 1) FAIL("embedding.factor must be positive");
  for (int i = 0; i < 3; i++) {
    g->n[i] = 1;
    g->T[i] = 1;
    g->ext[i] = 1.0;
    g->h[i] = 1.0;
  }
  for (int i = 0; i < d->dim; i++) {
    if (d->cells[i] < 1) FAIL("grid.cells must be positive");
    g->n[i] = d->cells[i];
    g->ext[i] = d->extensions[i];
    g->h[i] = d->extensions[i] / (double)d->cells[i]; /* fieldtraits.hh:270 */
    g->T[i] = g->factor * d->cells[i];                /* fieldtraits.hh:271 */
  }
  int mb = d->matrix_backend;
  if (mb < 0) {
    if (d->dim == 1)
      mb = PF_MATRIX_DFT;
    else if (d->anisotropy == PF_ANISO_NONE || d->anisotropy == PF_ANISO_AXIPARALLEL)
      mb = PF_MATRIX_DCT;
    else
      mb = PF_MATRIX_R2C;
  }
  int fb = d->field_backend;
  if (fb < 0) fb = (d->dim == 1) ? PF_FIELD_DFT : PF_FIELD_R2C; /* matrix.hh:1674-1691 */
  if (mb > 2 || fb > 2) FAIL("unknown backend");
  if (d->dim == 1 && (mb != PF_MATRIX_DFT || fb != PF_FIELD_DFT))
    FAIL("dim 1 requires DFTMatrixBackend and DFTFieldBackend");
  if (fb == PF_FIELD_DFT && mb == PF_MATRIX_R2C)
    FAIL("R2CMatrixBackend cannot serve DFTFieldBackend");
  if (fb == PF_FIELD_DCTDST) FAIL("DCTDSTFieldBackend is not supported");
  /* REDFT00 of T/2+1 points is the spectrum of a period-T torus only for even T */
  for (int i = 0; i < d->dim; i++)
    if (mb == PF_MATRIX_DCT && (g->T[i] % 2) != 0)
      FAIL("DCTMatrixBackend requires an even number of extended cells per dimension");
  g->matrix_backend = mb;
  g->field_backend = fb;
  int t = d->transposed < 0 ? (d->dim > 1) : (d->transposed != 0); /* fieldtraits.hh:229 */
  if (d->dim == 1) t = 0;
  if (d->dim == 2 && (mb == PF_MATRIX_R2C || fb == PF_FIELD_R2C)) t = 0; /* fieldtraits.hh:245-265 */
  g->transposed = t;
  for (int i = 0; i < 3; i++) g->Ts[i] = g->T[i];
  if (t) {
    int a = d->dim - 1, b = d->dim - 2, tmp = g->Ts[a];
    g->Ts[a] = g->Ts[b];
    g->Ts[b] = tmp;
  }
  g->domain = 1;
  g->N = 1;
  g->D = 1;
  for (int i = 0; i < d->dim; i++) {
    g->domain *= (uint64_t)g->n[i];
    g->N *= (uint64_t)g->T[i];
    g->D *= (uint64_t)(g->T[i] / 2 + 1);
  }
  g->Nc = g->N / (uint64_t)g->T[0] * (uint64_t)(g->T[0] / 2 + 1);
  g->spectrum = mb == PF_MATRIX_DCT ? g->D : (mb == PF_MATRIX_R2C ? g->Nc : g->N);
  g->noise = fb == PF_FIELD_R2C ? 2 * g->Nc : 2 * g->N;
  /* covariance parameter checks (covariance.hh:398-399, 521-522, 715-720) */
  if (d->covariance < 0 || d->covariance > PF_COV_WHITE_NOISE) FAIL("covariance structure not known");
  if (d->covariance == PF_COV_GAMMA_EXPONENTIAL && (d->exp_gamma < 0. || d->exp_gamma > 2.))
    FAIL("exponent gamma has to be between 0 and 2");
  if (d->covariance == PF_COV_MATERN && d->matern_nu < 0.) FAIL("matern nu has to be positive");
  if (d->covariance == PF_COV_GENERALIZED_CAUCHY) {
    if (d->cauchy_alpha <= 0. || d->cauchy_alpha > 2.)
      FAIL("generalized Cauchy alpha has to be in range (0,2]");
    if (d->cauchy_beta <= 0.) FAIL("generalized Cauchy beta has to be positive");
  }
  if (d->covariance == PF_COV_CUBIC && d->dim == 3) FAIL("cubic covariance only applicable in 1D or 2D");
  if (d->anisotropy < 0 || d->anisotropy > 2)
    FAIL("stochastic.anisotropy must be \"none\", \"axiparallel\" or \"geometric\"");
  /* matrix.hh:515-579 */
  if (d->periodization < 0 || d->periodization > 3)
    FAIL("stochastic.periodization must be \"classical\", \"merge\", \"fold\", or \"cofold\"");
  if (d->periodization != PF_PERIODIZATION_CLASSICAL) {
    if (d->sigmoid < 0 || d->sigmoid > 1) FAIL("embedding.sigmoid must be \"smooth\" or \"smoothstep\"");
    if (d->periodization != PF_PERIODIZATION_COFOLD && (d->sigmoid_combine < 0 || d->sigmoid_combine > 2))
      FAIL("sigmoidCombine must be tensor, radial or radialPlus");
    if (d->periodization == PF_PERIODIZATION_COFOLD && d->cofold_recursions < 0)
      FAIL("embedding.cofoldRecursions must be non-negative");
  }
#undef FAIL
  return PF_OK;
}

/* ------------------------------------------------------------------------- */
/* geometry + covariance: covariance.hh:18-138, 296-823                        */
/* ------------------------------------------------------------------------- */

void oc_geometry(const pf_field_desc* d, const double* x, double* xt) {
  const int dim = d->dim;
  if (d->anisotropy == PF_ANISO_NONE) { /* covariance.hh:33-43 */
    double v = 1. / d->corr_length[0];
    for (int i = 0; i < dim; i++) xt[i] = v * x[i];
  } else if (d->anisotropy == PF_ANISO_AXIPARALLEL) { /* covariance.hh:62-73 */
    for (int i = 0; i < dim; i++) xt[i] = (1. / d->corr_length[i]) * x[i];
  } else { /* covariance.hh:94-137 */
    double m[9];
    const double* c = d->corr_length;
    if (dim == 3) {
      m[0] = c[4] * c[8] - c[5] * c[7];
      m[1] = c[2] * c[7] - c[1] * c[8];
      m[2] = c[1] * c[5] - c[2] * c[4];
      m[3] = c[5] * c[6] - c[3] * c[8];
      m[4] = c[0] * c[8] - c[2] * c[6];
      m[5] = c[2] * c[3] - c[0] * c[5];
      m[6] = c[3] * c[7] - c[4] * c[6];
      m[7] = c[1] * c[6] - c[0] * c[7];
      m[8] = c[0] * c[4] - c[1] * c[3];
      double det = c[0] * (c[4] * c[8] - c[5] * c[7]) - c[1] * (c[3] * c[8] - c[5] * c[6]) +
                   c[2] * (c[3] * c[7] - c[4] * c[6]);
      for (int i = 0; i < 9; i++) m[i] /= det;
    } else if (dim == 2) {
      m[0] = c[3];
      m[1] = -c[1];
      m[2] = -c[2];
      m[3] = c[0];
      double det = c[0] * c[3] - c[1] * c[2];
      for (int i = 0; i < 4; i++) m[i] /= det;
    } else {
      m[0] = 1. / c[0];
    }
    for (int i = 0; i < dim; i++) {
      double s = 0.;
      for (int j = 0; j < dim; j++) s += m[i * dim + j] * x[j];
      xt[i] = s;
    }
  }
}

/* Modified Bessel function of the second kind K_nu(x), nu >= 0, x > 0.
 * Temme's series (N. M. Temme, J. Comput. Phys. 19, 324-337, 1975) for x <= 2 and
 * Steed's continued fraction CF2 (I. J. Thompson and A. R. Barnett, J. Comput. Phys.
 * 64, 490-509, 1986) for x > 2 give K_mu and K_mu+1 with |mu| <= 1/2; the upward
 * recurrence K_{m+1} = K_{m-1} + (2m/x) K_m reaches nu.  1/Gamma(1+z) enters through
 * its Taylor series (Abramowitz & Stegun 6.1.34; coefficients from the definition). */
static const double RGAMMA_SERIES[24] = {1.0, 0.5772156649015328606065, -0.655878071520253881077, -0.042002635034095235529,
    0.1665386113822914895017, -0.04219773455554433674821, -0.009621971527876973562115,
    0.007218943246663099542395, -0.001165167591859065112114, -0.0002152416741149509728157,
    0.0001280502823881161861532, -0.00002013485478078823865569, -0.000001250493482142670657345,
    0.000001133027231981695882374, -2.05633841697760710345e-7, 6.116095104481415817862e-9,
    5.002007644469222930056e-9, -1.181274570487020144588e-9, 1.043426711691100510492e-10,
    7.78226343990507125405e-12, -3.696805618642205708188e-12, 5.100370287454475979015e-13,
    -2.058326053566506783222e-14, -5.34812253942301798237e-15};

double oc_bessel_k(double nu, double x) {
  const int nl = (int)(nu + 0.5);
  const double mu = nu - nl, mu2 = mu * mu;
  double kmu, kmu1;
  if (x <= 2.0) {
    const double x2 = 0.5 * x;
    const double pimu = PI_D * mu;
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
    kmu = sqrt(PI_D / (2.0 * x)) * exp(-x) / s;
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

static double h_eff_of(int dim, const double* x) {
  double sum = 0.;
  for (int i = 0; i < dim; i++) sum += x[i] * x[i];
  return sqrt(sum);
}

double oc_covariance(const pf_field_desc* d, const double* x) {
  const int dim = d->dim;
  const double var = d->variance;
  switch (d->covariance) {
    case PF_COV_SPHERICAL: { /* covariance.hh:310-340 */
      double h = h_eff_of(dim, x);
      if (h > 1.) return 0.;
      if (dim == 3) return var * (1. - 1.5 * h + 0.5 * pow(h, 3));
      if (dim == 2) return var * (1. - 2. / PI_D * (h * sqrt(1. - pow(h, 2)) + asin(h)));
      return var * (1. - h);
    }
    case PF_COV_EXPONENTIAL: /* covariance.hh:365-374 */
      return var * exp(-h_eff_of(dim, x));
    case PF_COV_GAMMA_EXPONENTIAL: /* covariance.hh:413-422 */
      return var * exp(-pow(h_eff_of(dim, x), d->exp_gamma));
    case PF_COV_GAUSSIAN: { /* covariance.hh:447-456 */
      double h = h_eff_of(dim, x);
      return var * exp(-h * h);
    }
    case PF_COV_SEPARABLE_EXPONENTIAL: { /* covariance.hh:479-488 */
      double s = 0.;
      for (int i = 0; i < dim; i++) s += fabs(x[i]);
      return var * exp(-s);
    }
    case PF_COV_MATERN32: { /* covariance.hh:580-590 */
      double h = h_eff_of(dim, x);
      return var * (1. + sqrt(3.) * h) * exp(-sqrt(3.) * h);
    }
    case PF_COV_MATERN52: { /* covariance.hh:614-624 */
      double h = h_eff_of(dim, x);
      return var * (1. + sqrt(5.) * h + 5. / 3. * h * h) * exp(-sqrt(5.) * h);
    }
    case PF_COV_DAMPED_OSCILLATION: { /* covariance.hh:647-659 */
      double h = h_eff_of(dim, x);
      if (dim == 3) return var * exp(-h) * cos(h / sqrt(3.));
      return var * exp(-h) * cos(h);
    }
    case PF_COV_CAUCHY: { /* covariance.hh:681-690 */
      double h = h_eff_of(dim, x);
      return var * pow(1. + pow(h, 2), -3);
    }
    case PF_COV_GENERALIZED_CAUCHY: { /* covariance.hh:734-743 */
      double h = h_eff_of(dim, x);
      return var * pow(1. + pow(h, d->cauchy_alpha), -d->cauchy_beta);
    }
    case PF_COV_CUBIC: { /* covariance.hh:767-786 */
      double h = h_eff_of(dim, x);
      if (h > 1.) return 0.;
      return var * (1. - 7. * pow(h, 2) + 8.75 * pow(h, 3) - 3.5 * pow(h, 5) + 0.75 * pow(h, 7));
    }
    case PF_COV_MATERN: { /* covariance.hh:515-556 with GSL's K_nu replaced by oc_bessel_k */
      const double nu = d->matern_nu;
      const double sqrtTwoNu = sqrt(2. * nu), twoToOneMinusNu = pow(2., 1. - nu), gammaNu = tgamma(nu);
      const double h = h_eff_of(dim, x);
      if (h < 1e-10) return var;
      return var * twoToOneMinusNu / gammaNu * pow(sqrtTwoNu * h, nu) * oc_bessel_k(nu, sqrtTwoNu * h);
    }
    case PF_COV_WHITE_NOISE: /* covariance.hh:813-822 */
      for (int i = 0; i < dim; i++)
        if (fabs(x[i]) > 1e-10) return 0.;
      return var;
    default:
      return NAN;
  }
}

/* ------------------------------------------------------------------------- */
/* FFT (own implementation)                                                    */
/* ------------------------------------------------------------------------- */

typedef struct fftplan {
  int n;
  int nf;
  int fac[48];
  double* tw; /* 2n doubles: exp(-2 pi i k / n) */
  int blue;
  int m;
  double* chirp;   /* 2n: exp(-pi i k^2 / n) */
  double* bminus;  /* 2m: FFT_m(conj chirp) */
  double* bplus;   /* 2m: FFT_m(chirp) */
  struct fftplan* sub;
} fftplan;

static void plan_free(fftplan* p) {
  if (!p) return;
  free(p->tw);
  free(p->chirp);
  free(p->bminus);
  free(p->bplus);
  plan_free(p->sub);
  free(p);
}

static void exec_plan(const fftplan* p, double* x, double* work, int sign);

static fftplan* plan_make(int n) {
  fftplan* p = (fftplan*)calloc(1, sizeof(fftplan));
  p->n = n;
  int r = n;
  static const int pref[] = {4, 2, 3, 5, 7};
  for (int q = 0; q < 5; q++)
    while (r % pref[q] == 0) {
      p->fac[p->nf++] = pref[q];
      r /= pref[q];
    }
  for (int f = 11; f <= 61 && r > 1; f += 2)
    while (r % f == 0) {
      p->fac[p->nf++] = f;
      r /= f;
    }
  p->tw = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  for (int k = 0; k < n; k++) {
    double a = 2.0 * PI_D * (double)k / (double)n;
    p->tw[2 * k] = cos(a);
    p->tw[2 * k + 1] = -sin(a);
  }
  if (r > 1) { /* Bluestein for the whole length */
    p->blue = 1;
    p->nf = 0;
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->chirp = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    for (long long k = 0; k < n; k++) {
      long long k2 = (k * k) % (2LL * n);
      double a = PI_D * (double)k2 / (double)n;
      p->chirp[2 * k] = cos(a);
      p->chirp[2 * k + 1] = -sin(a);
    }
    p->sub = plan_make(m);
    p->bminus = (double*)calloc(2 * (size_t)m, sizeof(double));
    p->bplus = (double*)calloc(2 * (size_t)m, sizeof(double));
    for (int k = 0; k < n; k++) {
      double cr = p->chirp[2 * k], ci = p->chirp[2 * k + 1];
      p->bminus[2 * k] = cr;
      p->bminus[2 * k + 1] = -ci;
      p->bplus[2 * k] = cr;
      p->bplus[2 * k + 1] = ci;
      if (k > 0) {
        p->bminus[2 * (m - k)] = cr;
        p->bminus[2 * (m - k) + 1] = -ci;
        p->bplus[2 * (m - k)] = cr;
        p->bplus[2 * (m - k) + 1] = ci;
      }
    }
    double* w = (double*)malloc(sizeof(double) * 2 * (size_t)m);
    exec_plan(p->sub, p->bminus, w, -1);
    exec_plan(p->sub, p->bplus, w, -1);
    free(w);
  }
  return p;
}

/* twiddle exp(sign 2 pi i idx / n) from the table */
static inline void twid(const fftplan* p, long long idx, int sign, double* wr, double* wi) {
  int k = (int)(idx % p->n);
  *wr = p->tw[2 * k];
  *wi = sign < 0 ? p->tw[2 * k + 1] : -p->tw[2 * k + 1];
}

static void exec_stockham(const fftplan* p, double* x, double* work, int sign) {
  const int n = p->n;
  double* src = x;
  double* dst = work;
  int Ns = 1;
  double vr[64], vi[64], orr[64], oi[64];
  for (int s = 0; s < p->nf; s++) {
    const int R = p->fac[s];
    const int nR = n / R;
    const long long twstep = (long long)n / ((long long)Ns * R);
    for (int j = 0; j < nR; j++) {
      const int k = j % Ns;
      for (int r = 0; r < R; r++) {
        double ar = src[2 * (j + r * nR)], ai = src[2 * (j + r * nR) + 1];
        if (k) {
          double wr, wi;
          twid(p, (long long)r * k * twstep, sign, &wr, &wi);
          double tr = ar * wr - ai * wi;
          ai = ar * wi + ai * wr;
          ar = tr;
        }
        vr[r] = ar;
        vi[r] = ai;
      }
      /* DFT of length R: out[q] = sum_r v[r] exp(sign 2 pi i r q / R) */
      if (R == 2) {
        orr[0] = vr[0] + vr[1];
        oi[0] = vi[0] + vi[1];
        orr[1] = vr[0] - vr[1];
        oi[1] = vi[0] - vi[1];
      } else if (R == 4) {
        double ar = vr[0] + vr[2], ai = vi[0] + vi[2];
        double br = vr[0] - vr[2], bi = vi[0] - vi[2];
        double cr = vr[1] + vr[3], ci = vi[1] + vi[3];
        double dr = vr[1] - vr[3], di = vi[1] - vi[3];
        /* multiply d by (sign i) */
        double er = sign < 0 ? di : -di, ei = sign < 0 ? -dr : dr;
        orr[0] = ar + cr;
        oi[0] = ai + ci;
        orr[2] = ar - cr;
        oi[2] = ai - ci;
        orr[1] = br + er;
        oi[1] = bi + ei;
        orr[3] = br - er;
        oi[3] = bi - ei;
      } else {
        const long long step = n / R;
        for (int q = 0; q < R; q++) {
          double sr = 0., si = 0.;
          for (int r = 0; r < R; r++) {
            double wr, wi;
            twid(p, (long long)((r * q) % R) * step, sign, &wr, &wi);
            sr += vr[r] * wr - vi[r] * wi;
            si += vr[r] * wi + vi[r] * wr;
          }
          orr[q] = sr;
          oi[q] = si;
        }
      }
      const int base = (j / Ns) * Ns * R + k;
      for (int r = 0; r < R; r++) {
        dst[2 * (base + r * Ns)] = orr[r];
        dst[2 * (base + r * Ns) + 1] = oi[r];
      }
    }
    double* t = src;
    src = dst;
    dst = t;
    Ns *= R;
  }
  if (src != x) memcpy(x, src, sizeof(double) * 2 * (size_t)n);
}

/* work must hold 2*max(n, 2m) doubles for Bluestein plans */
static void exec_plan(const fftplan* p, double* x, double* work, int sign) {
  if (p->n == 1) return;
  if (!p->blue) {
    exec_stockham(p, x, work, sign);
    return;
  }
  const int n = p->n, m = p->m;
  double* a = work;          /* 2m */
  double* w2 = work + 2 * m; /* 2m */
  memset(a, 0, sizeof(double) * 2 * (size_t)m);
  for (int k = 0; k < n; k++) {
    double cr = p->chirp[2 * k], ci = sign < 0 ? p->chirp[2 * k + 1] : -p->chirp[2 * k + 1];
    double xr = x[2 * k], xi = x[2 * k + 1];
    a[2 * k] = xr * cr - xi * ci;
    a[2 * k + 1] = xr * ci + xi * cr;
  }
  exec_plan(p->sub, a, w2, -1);
  const double* B = sign < 0 ? p->bminus : p->bplus;
  for (int k = 0; k < m; k++) {
    double ar = a[2 * k], ai = a[2 * k + 1], br = B[2 * k], bi = B[2 * k + 1];
    a[2 * k] = ar * br - ai * bi;
    a[2 * k + 1] = ar * bi + ai * br;
  }
  exec_plan(p->sub, a, w2, +1);
  const double inv = 1.0 / (double)m;
  for (int k = 0; k < n; k++) {
    double cr = p->chirp[2 * k], ci = sign < 0 ? p->chirp[2 * k + 1] : -p->chirp[2 * k + 1];
    double yr = a[2 * k] * inv, yi = a[2 * k + 1] * inv;
    x[2 * k] = yr * cr - yi * ci;
    x[2 * k + 1] = yr * ci + yi * cr;
  }
}

static size_t plan_work(const fftplan* p) {
  size_t w = 2 * (size_t)p->n;
  if (p->blue) w = 4 * (size_t)p->m + 2 * (size_t)p->m;
  return w;
}

void oc_fft(int n, double* data, int sign) {
  fftplan* p = plan_make(n);
  double* w = (double*)malloc(sizeof(double) * plan_work(p));
  exec_plan(p, data, w, sign);
  free(w);
  plan_free(p);
}

void oc_fft_axis(double* data, int ndim, const int* shape, int axis, int sign) {
  size_t inner = 1, outer = 1;
  for (int i = 0; i < axis; i++) inner *= (size_t)shape[i];
  for (int i = axis + 1; i < ndim; i++) outer *= (size_t)shape[i];
  const int L = shape[axis];
  if (L == 1) return;
  fftplan* p = plan_make(L);
  const size_t wsz = plan_work(p);
  const long long total = (long long)(inner * outer);
#pragma omp parallel
  {
    double* buf = (double*)malloc(sizeof(double) * 2 * (size_t)L);
    double* w = (double*)malloc(sizeof(double) * wsz);
#pragma omp for schedule(static)
    for (long long t = 0; t < total; t++) {
      size_t ii = (size_t)t % inner, io = (size_t)t / inner;
      double* base = data + 2 * (ii + inner * (size_t)L * io);
      if (inner == 1) {
        exec_plan(p, base, w, sign);
      } else {
        for (int j = 0; j < L; j++) {
          buf[2 * j] = base[2 * inner * j];
          buf[2 * j + 1] = base[2 * inner * j + 1];
        }
        exec_plan(p, buf, w, sign);
        for (int j = 0; j < L; j++) {
          base[2 * inner * j] = buf[2 * j];
          base[2 * inner * j + 1] = buf[2 * j + 1];
        }
      }
    }
    free(buf);
    free(w);
  }
  plan_free(p);
}

/* R2C, FFTW semantics: out has shape (T0/2+1, T1, T2), complex interleaved. */
void oc_r2c(int ndim, const int* T, const double* in, double* out) {
  const int T0 = T[0], T0c = T[0] / 2 + 1;
  long long rows = 1;
  for (int i = 1; i < ndim; i++) rows *= T[i];
  fftplan* p = plan_make(T0);
  const size_t wsz = plan_work(p);
#pragma omp parallel
  {
    double* buf = (double*)malloc(sizeof(double) * 2 * (size_t)T0);
    double* w = (double*)malloc(sizeof(double) * wsz);
#pragma omp for schedule(static)
    for (long long r = 0; r < rows; r++) {
      for (int j = 0; j < T0; j++) {
        buf[2 * j] = in[(size_t)r * T0 + j];
        buf[2 * j + 1] = 0.;
      }
      exec_plan(p, buf, w, -1);
      memcpy(out + 2 * (size_t)r * T0c, buf, sizeof(double) * 2 * (size_t)T0c);
    }
    free(buf);
    free(w);
  }
  plan_free(p);
  int shp[3] = {T0c, ndim > 1 ? T[1] : 1, ndim > 2 ? T[2] : 1};
  for (int a = 1; a < ndim; a++) oc_fft_axis(out, ndim, shp, a, -1);
}

/* C2R, FFTW semantics: complex backward transforms along dims ndim-1..1, then a 1D
 * c2r along dim 0 that ignores Im at DC and (even T0) Nyquist. `in` is not modified. */
void oc_c2r(int ndim, const int* T, const double* in, double* out) {
  const int T0 = T[0], T0c = T[0] / 2 + 1;
  long long rows = 1;
  for (int i = 1; i < ndim; i++) rows *= T[i];
  double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)rows * T0c);
  memcpy(tmp, in, sizeof(double) * 2 * (size_t)rows * T0c);
  int shp[3] = {T0c, ndim > 1 ? T[1] : 1, ndim > 2 ? T[2] : 1};
  for (int a = ndim - 1; a >= 1; a--) oc_fft_axis(tmp, ndim, shp, a, +1);
  fftplan* p = plan_make(T0);
  const size_t wsz = plan_work(p);
#pragma omp parallel
  {
    double* buf = (double*)malloc(sizeof(double) * 2 * (size_t)T0);
    double* w = (double*)malloc(sizeof(double) * wsz);
#pragma omp for schedule(static)
    for (long long r = 0; r < rows; r++) {
      const double* X = tmp + 2 * (size_t)r * T0c;
      for (int k = 0; k < T0; k++) {
        if (k < T0c) {
          buf[2 * k] = X[2 * k];
          buf[2 * k + 1] = (k == 0 || (T0 % 2 == 0 && k == T0 / 2)) ? 0. : X[2 * k + 1];
        } else {
          buf[2 * k] = X[2 * (T0 - k)];
          buf[2 * k + 1] = -X[2 * (T0 - k) + 1];
        }
      }
      exec_plan(p, buf, w, +1);
      for (int j = 0; j < T0; j++) out[(size_t)r * T0 + j] = buf[2 * j];
    }
    free(buf);
    free(w);
  }
  plan_free(p);
  free(tmp);
}

/* REDFT00 along every axis (dctmatrixbackend.hh:252-266): DFT of the even extension. */
void oc_dct1(int ndim, const int* m, double* data) {
  for (int a = 0; a < ndim; a++) {
    size_t inner = 1, outer = 1;
    for (int i = 0; i < a; i++) inner *= (size_t)m[i];
    for (int i = a + 1; i < ndim; i++) outer *= (size_t)m[i];
    const int L = m[a];
    if (L < 2) continue;
    const int E = 2 * (L - 1);
    fftplan* p = plan_make(E);
    const size_t wsz = plan_work(p);
    const long long total = (long long)(inner * outer);
#pragma omp parallel
    {
      double* buf = (double*)malloc(sizeof(double) * 2 * (size_t)E);
      double* w = (double*)malloc(sizeof(double) * wsz);
#pragma omp for schedule(static)
      for (long long t = 0; t < total; t++) {
        size_t ii = (size_t)t % inner, io = (size_t)t / inner;
        double* base = data + ii + inner * (size_t)L * io;
        for (int j = 0; j < E; j++) {
          int s = j < L ? j : E - j;
          buf[2 * j] = base[inner * (size_t)s];
          buf[2 * j + 1] = 0.;
        }
        exec_plan(p, buf, w, -1);
        for (int k = 0; k < L; k++) base[inner * (size_t)k] = buf[2 * k];
      }
      free(buf);
      free(w);
    }
    plan_free(p);
  }
}

/* ------------------------------------------------------------------------- */
/* matrix fill: computeMatrixEntriesWithMirroring, matrix.hh:615-638           */
/* ------------------------------------------------------------------------- */

static void fill_cells(const oc_geom* g, int* cells) {
  for (int i = 0; i < 3; i++) cells[i] = 1;
  for (int i = 0; i < g->dim; i++) {
    if (g->matrix_backend == PF_MATRIX_DCT)
      cells[i] = g->T[i] / 2 + 1; /* dctmatrixbackend.hh:776-787 */
    else if (g->matrix_backend == PF_MATRIX_R2C)
      cells[i] = i == 0 ? 2 * (g->T[0] / 2 + 1) : g->T[i]; /* r2cmatrixbackend.hh:459-462 */
    else
      cells[i] = g->T[i];
  }
}

/* ClampingSigmoid / SmoothstepSigmoid / SmoothSigmoid (covariance.hh:147-287) */
static double oc_sigmoid(int kind, double oneEdge, double zeroEdge, double x, unsigned int recursions) {
  if (kind == PF_SIGMOID_SMOOTH) {
    if (fabs(x) < oneEdge) return 1.;
    if (fabs(x) > zeroEdge) return 0.;
    const double x1 = (zeroEdge - fabs(x)) / (zeroEdge - oneEdge);
    const double x2 = (fabs(x) - oneEdge) / (zeroEdge - oneEdge);
    const double th1 = x1 > 0. ? exp(-1. / x1) : 0.;
    const double th2 = x2 > 0. ? exp(-1. / x2) : 0.;
    return th1 / (th1 + th2);
  }
  double x1;
  if (fabs(x) < oneEdge)
    x1 = 1.;
  else if (fabs(x) > zeroEdge)
    x1 = 0.;
  else
    x1 = (zeroEdge - fabs(x)) / (zeroEdge - oneEdge);
  const double x2 = 2. * x1 - 1.;
  double normalization = 1., addition = 1., output = 1.;
  for (unsigned int i = 1; i <= recursions; i++) {
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

/* mergeRecursions / foldRecursions default 99 (matrix.hh:693-717, 803-827) */
static unsigned int oc_merge_recursions(const pf_field_desc* d) {
  const int r = d->periodization == PF_PERIODIZATION_FOLD ? d->fold_recursions : d->merge_recursions;
  if (r != 99) return (unsigned int)r;
  switch (d->covariance) {
    case PF_COV_MATERN: return (unsigned int)floor(d->matern_nu * 2. + d->dim / 2.);
    case PF_COV_GAMMA_EXPONENTIAL: return (unsigned int)floor(d->exp_gamma + d->dim / 2.);
    case PF_COV_GENERALIZED_CAUCHY: return (unsigned int)floor(d->cauchy_alpha + d->dim / 2.);
    case PF_COV_EXPONENTIAL: return 2;
    case PF_COV_MATERN32: return 4;
    case PF_COV_MATERN52: return 6;
    case PF_COV_CAUCHY: return 3;
    default: return 0;
  }
}

/* computeMatrixEntriesWithMerge (matrix.hh:652-775) at true coordinates tc */
static double oc_merge_value(const pf_field_desc* d, const oc_geom* g, const double* tc) {
  const int dim = g->dim;
  const unsigned int factor = (unsigned int)g->factor;
  const double start = d->sigmoid_start;
  const double end = d->sigmoid_end < 0 ? (double)factor - 1. : d->sigmoid_end;
  const unsigned int rec = oc_merge_recursions(d);
  const int radial = d->sigmoid_combine != PF_COMBINE_TENSOR;
  double constValue = 0.;
  if (d->sigmoid_combine == PF_COMBINE_RADIAL_PLUS) {
    double half[3] = {0, 0, 0}, th[3] = {0, 0, 0};
    for (int i = 0; i < dim; i++) half[i] = g->ext[i] * factor / 2.;
    oc_geometry(d, half, th);
    constValue = oc_covariance(d, th);
  }
  const double eps = 1e-10;
  const double sqrtDim = sqrt((double)dim);
  double value = 0., remainder = 1.;
  for (unsigned int j = 0; j < (1u << dim); j++) {
    double mirror[3] = {0, 0, 0}, trans[3] = {0, 0, 0};
    for (int i = 0; i < dim; i++) mirror[i] = (j & (1u << i)) ? g->ext[i] * factor - tc[i] : tc[i];
    double dampening = 1.;
    if (radial && sqrtDim < factor / 2.) {
      double radius = 0.;
      for (int i = 0; i < dim; i++) radius += (mirror[i] * mirror[i]) / (g->ext[i] * g->ext[i]);
      radius = sqrt(radius);
      dampening = oc_sigmoid(d->sigmoid, start * sqrtDim - eps, factor - (factor - end) * sqrtDim + eps, radius, rec);
    } else {
      for (int i = 0; i < dim; i++)
        dampening *= oc_sigmoid(d->sigmoid, g->ext[i] * start - eps, g->ext[i] * end + eps, mirror[i], rec);
    }
    if (dampening < eps) continue;
    remainder -= dampening;
    oc_geometry(d, mirror, trans);
    value += oc_covariance(d, trans) * dampening;
  }
  return value + constValue * remainder;
}

/* adaptive Simpson quadrature of the fold sigmoid (in place of GSL's qng) */
static double oc_fold_sig(const pf_field_desc* d, double beta, unsigned int rec, double x) {
  return oc_sigmoid(d->sigmoid, 1., beta, x, rec);
}
static double oc_simpson(const pf_field_desc* d, double beta, unsigned int rec, double a, double b, double fa,
                         double fm, double fb, double whole, int depth) {
  const double m = 0.5 * (a + b), lm = 0.5 * (a + m), rm = 0.5 * (m + b);
  const double flm = oc_fold_sig(d, beta, rec, lm), frm = oc_fold_sig(d, beta, rec, rm);
  const double left = (m - a) / 6. * (fa + 4. * flm + fm), right = (b - m) / 6. * (fm + 4. * frm + fb);
  if (depth <= 0 || fabs(left + right - whole) <= 1e-15 * 15.) return left + right + (left + right - whole) / 15.;
  return oc_simpson(d, beta, rec, a, m, fa, flm, fm, left, depth - 1) +
         oc_simpson(d, beta, rec, m, b, fm, frm, fb, right, depth - 1);
}

/* computeMatrixEntriesWithFold (matrix.hh:791-890) at classical coordinates coord */
static double oc_fold_value(const pf_field_desc* d, const oc_geom* g, double* coord) {
  const int dim = g->dim;
  const double beta = d->fold_max_factor * 0.5 * g->factor / sqrt((double)dim);
  const unsigned int rec = oc_merge_recursions(d);
  double norm = 0.;
  for (int i = 0; i < dim; i++) norm += (coord[i] * coord[i]) / (g->ext[i] * g->ext[i]);
  norm = sqrt(norm / (double)dim);
  if (norm > 1.) {
    const double hi = norm < beta ? norm : beta;
    double val = 0.;
    if (hi > 1.) {
      const double fa = oc_fold_sig(d, beta, rec, 1.), fb = oc_fold_sig(d, beta, rec, hi);
      const double fm = oc_fold_sig(d, beta, rec, 0.5 * (1. + hi));
      val = oc_simpson(d, beta, rec, 1., hi, fa, fm, fb, (hi - 1.) / 6. * (fa + 4. * fm + fb), 40);
    }
    val += 1.;
    for (int i = 0; i < dim; i++) coord[i] *= val / norm;
  }
  double tc[3] = {0, 0, 0};
  oc_geometry(d, coord, tc);
  return oc_covariance(d, tc);
}

/* integrand of the cofold integral: sigmoid(0, beta - alpha, beta - t) (matrix.hh:956-962) */
static double oc_cofold_sig(const pf_field_desc* d, double alpha, double beta, double t) {
  return oc_sigmoid(d->sigmoid, 0., beta - alpha, beta - t, (unsigned int)d->cofold_recursions);
}
static double oc_cofold_simpson(const pf_field_desc* d, double alpha, double beta, double a, double b, double fa,
                                double fm, double fb, double whole, int depth) {
  const double m = 0.5 * (a + b), lm = 0.5 * (a + m), rm = 0.5 * (m + b);
  const double flm = oc_cofold_sig(d, alpha, beta, lm), frm = oc_cofold_sig(d, alpha, beta, rm);
  const double left = (m - a) / 6. * (fa + 4. * flm + fm), right = (b - m) / 6. * (fm + 4. * frm + fb);
  if (depth <= 0 || fabs(left + right - whole) <= 15. * 1e-15 * fabs(b - a))
    return left + right + (left + right - whole) / 15.;
  return oc_cofold_simpson(d, alpha, beta, a, m, fa, flm, fm, left, depth - 1) +
         oc_cofold_simpson(d, alpha, beta, m, b, fm, frm, fb, right, depth - 1);
}
/* signed integral over [a, b] by adaptive Simpson quadrature (in place of GSL's qng) */
static double oc_cofold_integral(const pf_field_desc* d, double alpha, double beta, double a, double b) {
  if (a == b) return 0.;
  const double fa = oc_cofold_sig(d, alpha, beta, a), fb = oc_cofold_sig(d, alpha, beta, b);
  const double fm = oc_cofold_sig(d, alpha, beta, 0.5 * (a + b));
  return oc_cofold_simpson(d, alpha, beta, a, b, fa, fm, fb, (b - a) / 6. * (fa + 4. * fm + fb), 30);
}

/* classical coordinates and the cofold norm max_i |coord_i| / ext_i of matrix cell idx
 * (matrix.hh:917-931) */
static double oc_cofold_coord(const oc_geom* g, const int* cells, uint64_t idx, double* coord) {
  const double fac = (double)g->factor;
  uint64_t r = idx;
  double norm = 0.;
  for (int i = 0; i < g->dim; i++) {
    const unsigned int ii = (unsigned int)(r % (uint64_t)cells[i]);
    r /= (uint64_t)cells[i];
    coord[i] = (double)ii * g->h[i];
    if (coord[i] > 0.5 * g->ext[i] * fac) coord[i] -= g->ext[i] * fac;
  }
  for (int i = 0; i < g->dim; i++)
    if (fabs(coord[i]) / g->ext[i] > norm) norm = fabs(coord[i]) / g->ext[i];
  return norm;
}

/* modifyMatrixEntriesWithCofold (matrix.hh:905-1013) on the classically filled matrix */
static void oc_cofold_modify(const pf_field_desc* d, const oc_geom* g, const int* cells, double* m,
                             uint64_t total) {
  const double fac = (double)g->factor;
  double minConstrained = 1.7976931348623157e308, maxBorder = -1.7976931348623157e308;
  for (uint64_t idx = 0; idx < total; idx++) {
    double coord[3] = {0, 0, 0};
    const double norm = oc_cofold_coord(g, cells, idx, coord);
    const double val = m[idx];
    if (norm <= 1.) {
      if (val < minConstrained) minConstrained = val;
    } else {
      for (int i = 0; i < g->dim; i++)
        if (val > maxBorder && 0.5 * g->ext[i] * fac - fabs(coord[i]) < g->ext[i] / (double)g->T[i])
          maxBorder = val;
    }
  }
  const double alpha = maxBorder;
  const double mf = d->cofold_max_factor * maxBorder;
  const double beta = minConstrained < mf ? minConstrained : mf;
  const double offset = beta - oc_cofold_integral(d, alpha, beta, alpha, beta);
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < (long long)total; idx++) {
    double coord[3] = {0, 0, 0};
    if (oc_cofold_coord(g, cells, (uint64_t)idx, coord) > 1.) {
      const double x = m[idx];
      if (x < alpha)
        m[idx] = offset;
      else if (x < beta)
        m[idx] = oc_cofold_integral(d, alpha, beta, alpha, x) + offset;
    }
  }
}

int oc_fill_matrix(const pf_field_desc* d, double* out, uint64_t count) {
  oc_geom g;
  int st = oc_resolve(d, &g, NULL, 0);
  if (st) return st;
  int cells[3];
  fill_cells(&g, cells);
  const uint64_t total = (uint64_t)cells[0] * cells[1] * cells[2];
  if (count != total) return PF_ERR_ARG;
  const double fac = (double)g.factor;
#pragma omp parallel for schedule(static)
  for (long long idx = 0; idx < (long long)total; idx++) {
    long long r = idx;
    double coord[3] = {0, 0, 0}, tc[3] = {0, 0, 0};
    if (d->periodization == PF_PERIODIZATION_MERGE) {
      for (int i = 0; i < g.dim; i++) {
        unsigned int ii = (unsigned int)(r % cells[i]);
        r /= cells[i];
        coord[i] = (double)ii * g.h[i];
      }
      out[idx] = oc_merge_value(d, &g, coord);
      continue;
    }
    for (int i = 0; i < g.dim; i++) {
      unsigned int ii = (unsigned int)(r % cells[i]);
      r /= cells[i];
      coord[i] = (double)ii * g.h[i];
      if (coord[i] > 0.5 * g.ext[i] * fac) coord[i] -= g.ext[i] * fac;
    }
    if (d->periodization == PF_PERIODIZATION_FOLD) {
      out[idx] = oc_fold_value(d, &g, coord);
      continue;
    }
    oc_geometry(d, coord, tc);
    out[idx] = oc_covariance(d, tc);
  }
  if (d->periodization == PF_PERIODIZATION_COFOLD) oc_cofold_modify(d, &g, cells, out, total);
  return PF_OK;
}

/* ------------------------------------------------------------------------- */
/* layouts                                                                     */
/* ------------------------------------------------------------------------- */

/* stored index of natural multi-index k (cells c natural); swaps the last two dims
 * when transposed (FFTW_MPI_TRANSPOSED_OUT, r2cfieldbackend.hh:190-199) */
static inline uint64_t stored_index(const oc_geom* g, const int* c, const int* k) {
  int kk[3] = {k[0], k[1], k[2]}, cc[3] = {c[0], c[1], c[2]};
  if (g->transposed) {
    int a = g->dim - 1, b = g->dim - 2, t;
    t = kk[a];
    kk[a] = kk[b];
    kk[b] = t;
    t = cc[a];
    cc[a] = cc[b];
    cc[b] = t;
  }
  return (uint64_t)kk[0] + (uint64_t)cc[0] * ((uint64_t)kk[1] + (uint64_t)cc[1] * (uint64_t)kk[2]);
}

double oc_eval_stored(const pf_field_desc* d, const oc_geom* g, const double* lambda,
                      uint64_t si) {
  (void)d;
  /* stored multi-index in the field backend's (possibly swapped) frequency layout */
  int fc[3] = {1, 1, 1};
  for (int i = 0; i < g->dim; i++) fc[i] = g->Ts[i];
  if (g->field_backend == PF_FIELD_R2C) fc[0] = g->T[0] / 2 + 1;
  int a[3] = {0, 0, 0};
  uint64_t r = si;
  for (int i = 0; i < g->dim; i++) {
    a[i] = (int)(r % (uint64_t)fc[i]);
    r /= (uint64_t)fc[i];
  }
  if (g->matrix_backend == PF_MATRIX_DCT) { /* dctmatrixbackend.hh:346-355 */
    int ec[3] = {1, 1, 1};
    for (int i = 0; i < g->dim; i++) {
      ec[i] = g->Ts[i] / 2 + 1;
      if (a[i] >= ec[i]) a[i] = g->Ts[i] - a[i];
    }
    return lambda[(uint64_t)a[0] + (uint64_t)ec[0] * ((uint64_t)a[1] + (uint64_t)ec[1] * (uint64_t)a[2])];
  }
  if (g->matrix_backend == PF_MATRIX_R2C) /* sameLayout: r2cmatrixbackend.hh:337 */
    return lambda[si];
  /* DFT matrix: dftmatrixbackend.hh:303-307 */
  return lambda[(uint64_t)a[0] + (uint64_t)g->Ts[0] * ((uint64_t)a[1] + (uint64_t)g->Ts[1] * (uint64_t)a[2])];
}

/* ------------------------------------------------------------------------- */
/* spectrum: fillTransformedMatrix, matrix.hh:223-318                          */
/* ------------------------------------------------------------------------- */

static void scan_values(double* v, uint64_t count, uint64_t stride, double threshold,
                        pf_eig_stats* s, double* also_zero) {
  /* matrix.hh:270-291, sequential order */
  unsigned int small = 0, neg = 0, zero = 0;
  double smallest = 1.7976931348623157e308;
  for (uint64_t i = 0; i < count; i++) {
    double value = v[i * stride];
    if (value < smallest) smallest = value;
    if (value < 1e-6) {
      if (value < threshold) {
        if (value > -threshold)
          zero++;
        else
          neg++;
      } else
        small++;
    }
    if (value < 0.) {
      v[i * stride] = 0.;
      if (also_zero) also_zero[i * stride] = 0.;
    }
  }
  s->small = small;
  s->negative = neg;
  s->zero = zero;
  s->pad_ = 0;
  s->smallest = smallest;
}

int oc_spectrum(const pf_field_desc* d, double* lambda, pf_eig_stats* stats) {
  oc_geom g;
  int st = oc_resolve(d, &g, NULL, 0);
  if (st) return st;
  int cells[3];
  fill_cells(&g, cells);
  const uint64_t fillN = (uint64_t)cells[0] * cells[1] * cells[2];
  double* m = (double*)malloc(sizeof(double) * fillN);
  oc_fill_matrix(d, m, fillN);
  const double N = (double)(unsigned int)g.N;
  pf_eig_stats s;
  memset(&s, 0, sizeof(s));
  int Tn[3] = {g.T[0], g.T[1], g.T[2]};
  if (g.matrix_backend == PF_MATRIX_DCT) {
    int mm[3] = {cells[0], cells[1], cells[2]};
    oc_dct1(g.dim, mm, m);
    for (uint64_t i = 0; i < fillN; i++) m[i] /= N; /* dctmatrixbackend.hh:268-269 */
    /* stored (possibly transposed) layout */
    int k[3];
    for (k[2] = 0; k[2] < mm[2]; k[2]++)
      for (k[1] = 0; k[1] < mm[1]; k[1]++)
        for (k[0] = 0; k[0] < mm[0]; k[0]++) {
          uint64_t nat = (uint64_t)k[0] + (uint64_t)mm[0] * ((uint64_t)k[1] + (uint64_t)mm[1] * k[2]);
          lambda[stored_index(&g, mm, k)] = m[nat];
        }
    scan_values(lambda, g.D, 1, d->threshold, &s, NULL);
  } else if (g.matrix_backend == PF_MATRIX_R2C) {
    /* compact the padded real rows into a plain torus */
    const int T0 = g.T[0], T0p = cells[0];
    const uint64_t rows = g.N / (uint64_t)T0;
    double* torus = (double*)malloc(sizeof(double) * g.N);
    for (uint64_t r = 0; r < rows; r++) memcpy(torus + r * T0, m + r * T0p, sizeof(double) * T0);
    double* X = (double*)malloc(sizeof(double) * 2 * g.Nc);
    oc_r2c(g.dim, Tn, torus, X);
    free(torus);
    for (uint64_t i = 0; i < 2 * g.Nc; i++) X[i] /= N; /* r2cmatrixbackend.hh:279-282 */
    double* S = (double*)malloc(sizeof(double) * 2 * g.Nc); /* stored layout */
    int c[3] = {T0 / 2 + 1, g.T[1], g.T[2]};
    if (g.dim < 3) c[2] = 1;
    if (g.dim < 2) c[1] = 1;
    int k[3];
    for (k[2] = 0; k[2] < c[2]; k[2]++)
      for (k[1] = 0; k[1] < c[1]; k[1]++)
        for (k[0] = 0; k[0] < c[0]; k[0]++) {
          uint64_t nat = (uint64_t)k[0] + (uint64_t)c[0] * ((uint64_t)k[1] + (uint64_t)c[1] * k[2]);
          uint64_t si = stored_index(&g, c, k);
          S[2 * si] = X[2 * nat];
          S[2 * si + 1] = X[2 * nat + 1];
        }
    if (d->eigen_check == PF_EIGCHECK_REFERENCE)
      scan_values(S, g.Nc, 1, d->threshold, &s, NULL); /* real view of the first N_c doubles */
    else
      scan_values(S, g.Nc, 2, d->threshold, &s, NULL);
    for (uint64_t i = 0; i < g.Nc; i++) lambda[i] = S[2 * i]; /* finalize, 412-421 */
    free(X);
    free(S);
  } else { /* DFT matrix */
    double* X = (double*)malloc(sizeof(double) * 2 * g.N);
    for (uint64_t i = 0; i < g.N; i++) {
      X[2 * i] = m[i];
      X[2 * i + 1] = 0.;
    }
    for (int a = 0; a < g.dim; a++) oc_fft_axis(X, g.dim, Tn, a, -1);
    for (uint64_t i = 0; i < 2 * g.N; i++) X[i] /= N; /* dftmatrixbackend.hh:232-235 */
    double* S = (double*)malloc(sizeof(double) * 2 * g.N);
    int k[3];
    for (k[2] = 0; k[2] < Tn[2]; k[2]++)
      for (k[1] = 0; k[1] < Tn[1]; k[1]++)
        for (k[0] = 0; k[0] < Tn[0]; k[0]++) {
          uint64_t nat = (uint64_t)k[0] + (uint64_t)Tn[0] * ((uint64_t)k[1] + (uint64_t)Tn[1] * k[2]);
          uint64_t si = stored_index(&g, Tn, k);
          S[2 * si] = X[2 * nat];
          S[2 * si + 1] = X[2 * nat + 1];
        }
    /* get() is the real part, set() zeroes both parts (dftmatrixbackend.hh:322-338) */
    double* im = (double*)malloc(sizeof(double) * g.N);
    for (uint64_t i = 0; i < g.N; i++) {
      lambda[i] = S[2 * i];
      im[i] = S[2 * i + 1];
    }
    scan_values(lambda, g.N, 1, d->threshold, &s, im);
    free(im);
    free(X);
    free(S);
  }
  free(m);
  if (stats) *stats = s;
  if (s.negative > 0 && !d->approximate) return PF_ERR_NEG_EIGEN; /* matrix.hh:307-315 */
  return PF_OK;
}

/* ------------------------------------------------------------------------- */
/* generation: generateField, matrix.hh:330-421                                 */
/* ------------------------------------------------------------------------- */

int oc_generate(const pf_field_desc* d, const double* lambda, const double* noise,
                double* field, double* spare) {
  oc_geom g;
  int st = oc_resolve(d, &g, NULL, 0);
  if (st) return st;
  const int dim = g.dim;
  int Tn[3] = {g.T[0], g.T[1], g.T[2]};
  if (g.field_backend == PF_FIELD_R2C) {
    int c[3] = {g.T[0] / 2 + 1, g.T[1], g.T[2]};
    double* X = (double*)malloc(sizeof(double) * 2 * g.Nc);
    const double sqrtTwo = sqrt(2.);
#pragma omp parallel for schedule(static)
    for (long long nat = 0; nat < (long long)g.Nc; nat++) {
      int k[3];
      long long r = nat;
      for (int i = 0; i < 3; i++) {
        k[i] = (int)(r % c[i]);
        r /= c[i];
      }
      uint64_t si = stored_index(&g, c, k);
      double lam = sqrt(oc_eval_stored(d, &g, lambda, si));
      double r1 = noise[2 * si], r2 = noise[2 * si + 1];
      int allMultiple = 1; /* r2cfieldbackend.hh:309-316 */
      for (int i = 0; i < dim; i++)
        if ((2 * (long long)k[i]) % g.T[i] != 0) allMultiple = 0;
      if (allMultiple) {
        X[2 * nat] = lam * r1;
        X[2 * nat + 1] = 0;
      } else {
        X[2 * nat] = lam / sqrtTwo * r1;
        X[2 * nat + 1] = lam / sqrtTwo * r2;
      }
    }
    double* torus = (double*)malloc(sizeof(double) * g.N);
    oc_c2r(dim, Tn, X, torus);
    free(X);
    /* extendedFieldToField, r2cfieldbackend.hh:433-441 */
#pragma omp parallel for schedule(static)
    for (long long idx = 0; idx < (long long)g.domain; idx++) {
      long long r = idx;
      int j[3] = {0, 0, 0};
      for (int i = 0; i < dim; i++) {
        j[i] = (int)(r % g.n[i]);
        r /= g.n[i];
      }
      field[idx] = torus[(uint64_t)j[0] + (uint64_t)g.T[0] * ((uint64_t)j[1] + (uint64_t)g.T[1] * j[2])];
    }
    free(torus);
    if (spare) memset(spare, 0, sizeof(double) * g.domain);
    return PF_OK;
  }
  /* DFT field backend: dftfieldbackend.hh:276-280, c2c backward, two fields */
  double* X = (double*)malloc(sizeof(double) * 2 * g.N);
#pragma omp parallel for schedule(static)
  for (long long nat = 0; nat < (long long)g.N; nat++) {
    int k[3];
    long long r = nat;
    for (int i = 0; i < 3; i++) {
      k[i] = (int)(r % Tn[i]);
      r /= Tn[i];
    }
    uint64_t si = stored_index(&g, Tn, k);
    double lam = sqrt(oc_eval_stored(d, &g, lambda, si));
    X[2 * nat] = lam * noise[2 * si];
    X[2 * nat + 1] = lam * noise[2 * si + 1];
  }
  for (int a = dim - 1; a >= 0; a--) oc_fft_axis(X, dim, Tn, a, +1);
  for (uint64_t idx = 0; idx < g.domain; idx++) {
    uint64_t r = idx;
    int j[3] = {0, 0, 0};
    for (int i = 0; i < dim; i++) {
      j[i] = (int)(r % (uint64_t)g.n[i]);
      r /= (uint64_t)g.n[i];
    }
    uint64_t e = (uint64_t)j[0] + (uint64_t)g.T[0] * ((uint64_t)j[1] + (uint64_t)g.T[1] * j[2]);
    field[idx] = X[2 * e];
    if (spare) spare[idx] = X[2 * e + 1];
  }
  free(X);
  return PF_OK;
}

/* ------------------------------------------------------------------------- */
/* matvecs: multiplyExtended / Root / InverseExtended, matrix.hh:1443-1646     */
/* ------------------------------------------------------------------------- */

static int matvec_geom(const pf_field_desc* d, const oc_geom* g, const double* lambda, int op,
                       const double* in, double* out) {
  const int dim = g->dim;
  int Tn[3] = {g->T[0], g->T[1], g->T[2]};
  const double N = (double)(unsigned int)g->N;
  if (g->field_backend == PF_FIELD_R2C) {
    double* torus = (double*)calloc(g->N, sizeof(double)); /* fieldToExtendedField */
    for (uint64_t idx = 0; idx < g->domain; idx++) {
      uint64_t r = idx;
      int j[3] = {0, 0, 0};
      for (int i = 0; i < dim; i++) {
        j[i] = (int)(r % (uint64_t)g->n[i]);
        r /= (uint64_t)g->n[i];
      }
      torus[(uint64_t)j[0] + (uint64_t)g->T[0] * ((uint64_t)j[1] + (uint64_t)g->T[1] * j[2])] = in[idx];
    }
    double* X = (double*)malloc(sizeof(double) * 2 * g->Nc);
    oc_r2c(dim, Tn, torus, X);
    int c[3] = {g->T[0] / 2 + 1, g->T[1], g->T[2]};
#pragma omp parallel for schedule(static)
    for (long long nat = 0; nat < (long long)g->Nc; nat++) {
      int k[3];
      long long r = nat;
      for (int i = 0; i < 3; i++) {
        k[i] = (int)(r % c[i]);
        r /= c[i];
      }
      double ev = oc_eval_stored(d, g, lambda, stored_index(g, c, k));
      double f = op == PF_OP_MUL ? ev : (op == PF_OP_ROOT ? sqrt(ev) : 1. / ev);
      X[2 * nat] = (X[2 * nat] / N) * f;
      X[2 * nat + 1] = (X[2 * nat + 1] / N) * f;
    }
    oc_c2r(dim, Tn, X, torus);
    for (uint64_t idx = 0; idx < g->domain; idx++) {
      uint64_t r = idx;
      int j[3] = {0, 0, 0};
      for (int i = 0; i < dim; i++) {
        j[i] = (int)(r % (uint64_t)g->n[i]);
        r /= (uint64_t)g->n[i];
      }
      out[idx] = torus[(uint64_t)j[0] + (uint64_t)g->T[0] * ((uint64_t)j[1] + (uint64_t)g->T[1] * j[2])];
    }
    free(X);
    free(torus);
    return PF_OK;
  }
  double* X = (double*)calloc(2 * g->N, sizeof(double));
  for (uint64_t idx = 0; idx < g->domain; idx++) {
    uint64_t r = idx;
    int j[3] = {0, 0, 0};
    for (int i = 0; i < dim; i++) {
      j[i] = (int)(r % (uint64_t)g->n[i]);
      r /= (uint64_t)g->n[i];
    }
    X[2 * ((uint64_t)j[0] + (uint64_t)g->T[0] * ((uint64_t)j[1] + (uint64_t)g->T[1] * j[2]))] = in[idx];
  }
  for (int a = 0; a < dim; a++) oc_fft_axis(X, dim, Tn, a, -1);
#pragma omp parallel for schedule(static)
  for (long long nat = 0; nat < (long long)g->N; nat++) {
    int k[3];
    long long r = nat;
    for (int i = 0; i < 3; i++) {
      k[i] = (int)(r % Tn[i]);
      r /= Tn[i];
    }
    double ev = oc_eval_stored(d, g, lambda, stored_index(g, Tn, k));
    double f = op == PF_OP_MUL ? ev : (op == PF_OP_ROOT ? sqrt(ev) : 1. / ev);
    X[2 * nat] = (X[2 * nat] / N) * f;
    X[2 * nat + 1] = (X[2 * nat + 1] / N) * f;
  }
  for (int a = dim - 1; a >= 0; a--) oc_fft_axis(X, dim, Tn, a, +1);
  for (uint64_t idx = 0; idx < g->domain; idx++) {
    uint64_t r = idx;
    int j[3] = {0, 0, 0};
    for (int i = 0; i < dim; i++) {
      j[i] = (int)(r % (uint64_t)g->n[i]);
      r /= (uint64_t)g->n[i];
    }
    out[idx] = X[2 * ((uint64_t)j[0] + (uint64_t)g->T[0] * ((uint64_t)j[1] + (uint64_t)g->T[1] * j[2]))];
  }
  free(X);
  return PF_OK;
}

int oc_matvec(const pf_field_desc* d, const double* lambda, int op, const double* in,
              double* out) {
  oc_geom g;
  int st = oc_resolve(d, &g, NULL, 0);
  if (st) return st;
  return matvec_geom(d, &g, lambda, op, in, out);
}

/* ------------------------------------------------------------------------- */
/* CG: multiplyInverse + innerCG, matrix.hh:189-206, 1315-1432                 */
/* ------------------------------------------------------------------------- */

int oc_multiply_inverse(const pf_field_desc* d, const double* lambda, const double* b,
                        double* x, int* iterations) {
  oc_geom g;
  int st = oc_resolve(d, &g, NULL, 0);
  if (st) return st;
  const uint64_t n = g.domain;
  if (iterations) *iterations = 0;
  int fieldZero = 1;
  for (uint64_t i = 0; i < n; i++)
    if (fabs(b[i]) > 1e-10) fieldZero = 0;
  if (fieldZero) {
    memcpy(x, b, sizeof(double) * n);
    return PF_OK;
  }
  matvec_geom(d, &g, lambda, PF_OP_INVEXT, b, x); /* initial guess */
  double* Aiter = (double*)malloc(sizeof(double) * n);
  double* res = (double*)malloc(sizeof(double) * n);
  double* pres = (double*)malloc(sizeof(double) * n);
  double* dir = (double*)malloc(sizeof(double) * n);
  double* Ad = (double*)malloc(sizeof(double) * n);
  /* matrix.hh:1329 multiplies the right-hand side too; the product is unused */
  matvec_geom(d, &g, lambda, PF_OP_MUL, x, Aiter);
  for (uint64_t i = 0; i < n; i++) res[i] = b[i] - Aiter[i];
  matvec_geom(d, &g, lambda, PF_OP_INVEXT, res, pres);
  memcpy(dir, pres, sizeof(double) * n);
  int converged = 0;
  double sp = 0.;
  for (uint64_t i = 0; i < n; i++) sp += pres[i] * res[i];
  double sp2 = 0.;
  for (uint64_t i = 0; i < n; i++) sp2 += res[i] * res[i];
  if (sqrt(fabs(sp2)) < 1e-6) converged = 1;
  double first = 0.;
  for (uint64_t i = 0; i < n; i++) first += x[i] * (0.5 * Aiter[i] - b[i]);
  int count = 0;
  const int maxit = d->cg_iterations;
  while (!converged && count < maxit) {
    matvec_geom(d, &g, lambda, PF_OP_MUL, dir, Ad);
    double den = 0.;
    for (uint64_t i = 0; i < n; i++) den += dir[i] * Ad[i];
    double alpha = sp / den;
    double oldv = 0.;
    for (uint64_t i = 0; i < n; i++) oldv += x[i] * (0.5 * Aiter[i] - b[i]);
    for (uint64_t i = 0; i < n; i++) {
      x[i] += alpha * dir[i];
      Aiter[i] += alpha * Ad[i];
    }
    double value = 0.;
    for (uint64_t i = 0; i < n; i++) value += x[i] * (0.5 * Aiter[i] - b[i]);
    for (uint64_t i = 0; i < n; i++) res[i] = b[i] - Aiter[i];
    matvec_geom(d, &g, lambda, PF_OP_INVEXT, res, pres);
    double beta = 1. / sp;
    sp = 0.;
    for (uint64_t i = 0; i < n; i++) sp += pres[i] * res[i];
    beta *= sp;
    for (uint64_t i = 0; i < n; i++) dir[i] = pres[i] + beta * dir[i];
    if (value != first)
      if (fabs(value - oldv) / fabs(value - first) < 1e-16) converged = 1;
    count++;
  }
  if (iterations) *iterations = count;
  free(Aiter);
  free(res);
  free(pres);
  free(dir);
  free(Ad);
  return PF_OK;
}

/* ------------------------------------------------------------------------- */
/* value transforms: mutators.hh:35-118                                        */
/* ------------------------------------------------------------------------- */

void oc_transform(int kind, double lam, double* v, uint64_t n) {
  for (uint64_t i = 0; i < n; i++) {
    switch (kind) {
      case PF_TRANSFORM_LOGNORMAL:
        v[i] = exp(v[i]);
        break;
      case PF_TRANSFORM_FOLDEDNORMAL:
        v[i] = fabs(v[i]);
        break;
      case PF_TRANSFORM_SIGN:
        v[i] = v[i] < 0. ? -1. : 1.;
        break;
      case PF_TRANSFORM_BOXCOX:
        v[i] = pow(v[i] * lam + 1, -lam);
        break;
      default:
        break;
    }
  }
}
