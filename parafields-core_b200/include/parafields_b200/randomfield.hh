// randomfield.hh -- C++ mirror of parafields-core's RandomField / Matrix API for the
// circulant-embedding path, running on the B200 library through the C ABI in
// include/parafields_b200.h.
//
//   parafields_b200::ParameterTree config;   // same keys as Dune::ParameterTree configs
//   config["grid.cells"] = "512 512"; ...
//   parafields_b200::RandomField<2> field(config);
//   field.generate(seed);                    // randomfield.hh:512-529
//   field.timesMatrix();                     // randomfield.hh:1181-1202
//
// Noise: generate(seed) draws from std::default_random_engine + std::normal_distribution
// in the reference's order (CppRNGBackend, backends/cpprngbackend.hh:16-59, used when GSL
// is absent), so a reference build without GSL and this facade produce the same field
// for the same seed up to floating-point rounding.  generateWithRNG accepts any object
// with RF sample(), exactly like randomfield.hh:541-558.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/parafields_b200.h"
#include "fieldio.hh"
#include "parametertree.hh"

namespace parafields_b200 {

// exceptions.hh:8-15
class NegativeEigenvalueError : public std::runtime_error {
 public:
  explicit NegativeEigenvalueError(const std::string& what) : std::runtime_error(what) {}
};

inline void check(pf_status st) {
  if (st == PF_OK) return;
  const std::string msg = pf_last_error_string();
  if (st == PF_ERR_NEG_EIGEN) throw NegativeEigenvalueError{msg};
  throw std::runtime_error{msg};
}

// fftw.measure / fftw.useWisdom (r2cfieldbackend.hh:75-96, 212-216): with fftw.measure the
// realization passes of a plan are planned by measurement (pf_plan_autotune) once its
// spectrum exists; with fftw.useWisdom the planning choices are read from this file when a
// plan is made and written back when it is destroyed.  The file holds the library's own
// wisdom text (pf_wisdom_export), so it is not the reference's FFTW wisdom file.
inline const char* wisdomFileName() { return "wisdom-R2CField-b200.txt"; }

struct PlanningKeys {
  bool measure = false;
  bool useWisdom = false;
  template <typename Config>
  static PlanningKeys fromConfig(const Config& config) {
    PlanningKeys k;
    k.measure = config.template get<bool>("fftw.measure", false);
    k.useWisdom = config.template get<bool>("fftw.useWisdom", false);
    return k;
  }
  void importWisdom() const {
    if (!useWisdom) return;
    std::ifstream f(wisdomFileName());
    if (!f) return;  // no file yet: FFTW's import_wisdom_from_filename ignores it too
    std::stringstream ss;
    ss << f.rdbuf();
    check(pf_wisdom_import(ss.str().c_str()));
  }
  void exportWisdom() const noexcept {
    if (!useWisdom) return;
    uint64_t need = 0;
    if (pf_wisdom_export(nullptr, 0, &need) != PF_OK || need == 0) return;
    std::string buf(need, '\0');
    if (pf_wisdom_export(&buf[0], need, &need) != PF_OK) return;
    std::ofstream f(wisdomFileName(), std::ofstream::trunc);
    f << buf.c_str();
  }
  // after the spectrum was built
  void plan(pf_plan* p) const {
    if (measure) check(pf_plan_autotune(p, 0, nullptr));
  }
};

// Configuration keys of the path -> descriptor (fieldtraits.hh:175-186, 229;
// matrix.hh:232-260, 268-269, 479-493, 515-602; covariance.hh:33-128, 395-396, 515-516,
// 711-713; mutators.hh:139-154).  Additional keys: gpu.precision (double|float, default
// from RF) and gpu.eigenCheck (corrected|reference).
template <unsigned dim, typename RF, typename Config>
pf_field_desc descFromConfig(const Config& config) {
  pf_field_desc d;
  pf_field_desc_init(&d);
  d.dim = (int32_t)dim;
  const auto cells = config.template get<std::array<unsigned, dim>>("grid.cells");
  const auto ext = config.template get<std::array<double, dim>>("grid.extensions");
  for (unsigned i = 0; i < dim; i++) {
    d.cells[i] = (int32_t)cells[i];
    d.extensions[i] = ext[i];
  }
  d.variance = config.template get<double>("stochastic.variance");
  const std::string cov = config.template get<std::string>("stochastic.covariance");
  static const char* names[] = {"exponential", "gaussian", "spherical", "separableExponential", "matern",
                                "matern32", "matern52", "dampedOscillation", "gammaExponential", "cauchy",
                                "generalizedCauchy", "cubic", "whiteNoise"};
  d.covariance = -1;
  for (int i = 0; i < 13; i++)
    if (cov == names[i]) d.covariance = i;
  if (cov == "custom-iso" || cov == "custom-aniso") d.covariance = PF_COV_CUSTOM;
  if (d.covariance < 0) throw std::runtime_error{"covariance structure " + cov + " not known"};
  if (d.covariance == PF_COV_MATERN) d.matern_nu = config.template get<double>("stochastic.maternNu");
  if (d.covariance == PF_COV_GAMMA_EXPONENTIAL) d.exp_gamma = config.template get<double>("stochastic.expGamma");
  if (d.covariance == PF_COV_GENERALIZED_CAUCHY) {
    d.cauchy_alpha = config.template get<double>("stochastic.cauchyAlpha");
    d.cauchy_beta = config.template get<double>("stochastic.cauchyBeta");
  }
  const std::string aniso = config.template get<std::string>("stochastic.anisotropy", std::string("none"));
  if (aniso == "none") {
    d.anisotropy = PF_ANISO_NONE;
    d.corr_length[0] = config.template get<double>("stochastic.corrLength");
  } else if (aniso == "axiparallel") {
    d.anisotropy = PF_ANISO_AXIPARALLEL;
    const auto c = config.template get<std::array<double, dim>>("stochastic.corrLength");
    for (unsigned i = 0; i < dim; i++) d.corr_length[i] = c[i];
  } else if (aniso == "geometric") {
    d.anisotropy = PF_ANISO_GEOMETRIC;
    const auto c = config.template get<std::array<double, dim * dim>>("stochastic.corrLength");
    for (unsigned i = 0; i < dim * dim; i++) d.corr_length[i] = c[i];
  } else {
    throw std::runtime_error{"stochastic.anisotropy must be \"none\", \"axiparallel\" or \"geometric\""};
  }
  d.periodic = config.template get<bool>("randomField.periodic", false);
  d.approximate = config.template get<bool>("embedding.approximate", false);
  d.cg_iterations = (int32_t)config.template get<unsigned>("randomField.cgIterations", 100u);
  d.embedding_factor = (int32_t)config.template get<unsigned>("embedding.factor", 2u);
  d.threshold = config.template get<double>("embedding.threshold", 1e-14);
  if (config.hasKey("fftw.transposed")) d.transposed = config.template get<bool>("fftw.transposed") ? 1 : 0;
  const std::string per = config.template get<std::string>("embedding.periodization", std::string("classical"));
  if (per == "merge" || per == "fold" || per == "cofold") {
    d.periodization = per == "merge" ? PF_PERIODIZATION_MERGE
                                     : (per == "fold" ? PF_PERIODIZATION_FOLD : PF_PERIODIZATION_COFOLD);
    d.fold_max_factor = config.template get<double>("embedding.foldMaxFactor", 1.);
    d.fold_recursions = (int32_t)config.template get<unsigned>("embedding.foldRecursions", 99u);
    d.cofold_max_factor = config.template get<double>("embedding.cofoldMaxFactor", 5.);
    d.cofold_recursions = (int32_t)config.template get<double>("embedding.cofoldRecursions", 1.);
    const std::string sig = config.template get<std::string>("embedding.sigmoid", std::string("smoothstep"));
    if (sig == "smooth")
      d.sigmoid = PF_SIGMOID_SMOOTH;
    else if (sig == "smoothstep")
      d.sigmoid = PF_SIGMOID_SMOOTHSTEP;
    else
      throw std::runtime_error{"embedding.sigmoid must be \"smooth\" or \"smoothstep\""};
    const std::string comb = config.template get<std::string>("stochastic.sigmoidCombine", std::string("radialPlus"));
    if (comb == "radialPlus")
      d.sigmoid_combine = PF_COMBINE_RADIAL_PLUS;
    else if (comb == "radial")
      d.sigmoid_combine = PF_COMBINE_RADIAL;
    else if (comb == "tensor")
      d.sigmoid_combine = PF_COMBINE_TENSOR;
    else
      throw std::runtime_error{"sigmoidCombine must be tensor, radial or radialPlus"};
    d.sigmoid_start = config.template get<double>("embedding.sigmoidStart", 1.);
    d.sigmoid_end = config.template get<double>("embedding.sigmoidEnd", (double)d.embedding_factor - 1.);
    d.merge_recursions = (int32_t)config.template get<unsigned>("embedding.mergeRecursions", 99u);
  } else if (per != "classical") {
    throw std::runtime_error{
        "stochastic.periodization must be \"classical\", \"merge\", \"fold\", or \"cofold\""};
  }
  const std::string optim = config.template get<std::string>("embedding.optim", std::string("none"));
  if (optim != "none") throw std::runtime_error{"optimization requires dune-nonlinopt"};
  const std::string tr = config.template get<std::string>("randomField.transform", std::string("none"));
  if (tr == "none")
    d.transform = PF_TRANSFORM_NONE;
  else if (tr == "logNormal")
    d.transform = PF_TRANSFORM_LOGNORMAL;
  else if (tr == "foldedNormal")
    d.transform = PF_TRANSFORM_FOLDEDNORMAL;
  else if (tr == "sign")
    d.transform = PF_TRANSFORM_SIGN;
  else if (tr == "boxCox") {
    d.transform = PF_TRANSFORM_BOXCOX;
    d.boxcox_lambda = config.template get<double>("transform.boxCoxLambda");
  } else
    throw std::runtime_error{"transform type not known"};
  const std::string prec =
      config.template get<std::string>("gpu.precision", std::string(sizeof(RF) == 4 ? "float" : "double"));
  d.precision = prec == "float" ? PF_PREC_F32 : PF_PREC_F64;
  const std::string eig = config.template get<std::string>("gpu.eigenCheck", std::string("corrected"));
  d.eigen_check = eig == "reference" ? PF_EIGCHECK_REFERENCE : PF_EIGCHECK_CORRECTED;
  return d;
}

// std::default_random_engine + std::normal_distribution (cpprngbackend.hh:16-59)
template <typename RF>
class CppRNGBackend {
  std::default_random_engine generator;
  std::normal_distribution<RF> normalDist{0., 1.};

 public:
  void seed(unsigned int s) { generator.seed(s); }
  RF sample() { return normalDist(generator); }
};

// ValueTransform (mutators.hh:126-163)
template <typename RF>
class ValueTransform {
  int kind = PF_TRANSFORM_NONE;
  RF lambda = 0;

 public:
  ValueTransform() = default;
  ValueTransform(int k, RF l) : kind(k), lambda(l) {}
  void apply(RF& v) const {
    switch (kind) {
      case PF_TRANSFORM_LOGNORMAL: v = std::exp(v); break;
      case PF_TRANSFORM_FOLDEDNORMAL: v = std::abs(v); break;
      case PF_TRANSFORM_SIGN: v = v < 0. ? -1. : 1.; break;
      case PF_TRANSFORM_BOXCOX: v = std::pow(v * lambda + 1, -lambda); break;
      default: break;
    }
  }
};

// Covariance values of a caller-supplied functor on the matrix cells of a plan, in the
// layout pf_spectrum_build_values takes: computeMatrixEntriesWithMirroring
// (matrix.hh:615-638) with the ScaledIdentityMatrix geometry that fillTransformedMatrix
// applies to user functors (matrix.hh:262-264, covariance.hh:18-44), i.e. coordinate
// i_d * h_d (minus T_d * h_d beyond half the torus) divided by stochastic.corrLength and
// value covariance(variance, transformed coordinate).  The DCT matrix keeps the
// prod(T_d/2+1) non-mirrored cells, the R2C and DFT matrices every torus cell.
template <unsigned dim, typename RF, typename Covariance>
std::vector<double> customCovarianceValues(const pf_plan_info& info, const std::array<double, dim>& extensions,
                                           double variance, double corrLength, Covariance&& covariance) {
  std::array<std::size_t, 3> m{1, 1, 1};
  std::array<double, 3> h{1., 1., 1.}, period{1., 1., 1.};
  for (unsigned i = 0; i < dim; i++) {
    const unsigned T = (unsigned)info.ext_cells[i];
    m[i] = info.matrix_backend == PF_MATRIX_DCT ? T / 2 + 1 : T;
    h[i] = extensions[i] / (double)info.cells[i];
    period[i] = h[i] * (double)T;  // extensions * embedding factor
  }
  std::vector<double> values(m[0] * m[1] * m[2]);
  std::array<RF, dim> coord, trans;
  std::size_t k = 0;
  for (std::size_t i2 = 0; i2 < m[2]; i2++)
    for (std::size_t i1 = 0; i1 < m[1]; i1++)
      for (std::size_t i0 = 0; i0 < m[0]; i0++, k++) {
        const std::size_t idx[3] = {i0, i1, i2};
        for (unsigned i = 0; i < dim; i++) {
          coord[i] = (RF)((double)idx[i] * h[i]);
          if (coord[i] > (RF)(0.5 * period[i])) coord[i] -= (RF)period[i];
          trans[i] = (RF)(1. / corrLength) * coord[i];
        }
        values[k] = (double)covariance((RF)variance, trans);
      }
  return values;
}

// The plan of one field configuration (matrix.hh:55-206) on the GPU, as the facade's
// RandomField below uses it.  parafields_b200/gpumatrix.hh holds the adapter that fills
// the reference's own IsoMatrix/AnisoMatrix template slot.
template <typename RF>
class GpuPlan {
  pf_plan* plan_ = nullptr;
  pf_plan_info info_{};
  pf_field_desc desc_{};
  bool spare_pending_ = false;
  bool custom_ = false;
  PlanningKeys planning_{};
  bool planned_ = false;  // fftw.measure: the passes were planned for this matrix
  bool hasValues_ = false;  // custom covariance: the spectrum was built from values

  // fftw.measure once the matrix can be built (the built-in covariances build it lazily on
  // first use; a custom covariance needs fillTransformedMatrix with its functor first)
  void plan() {
    if (planned_ || !planning_.measure || (custom_ && !hasValues_)) return;
    planning_.plan(plan_);
    planned_ = true;
  }

 public:
  GpuPlan(const pf_field_desc& d, bool customCovariance = false, PlanningKeys planning = PlanningKeys{})
      : desc_(d), custom_(customCovariance), planning_(planning) {
    if ((d.precision == PF_PREC_F64) != (sizeof(RF) == 8))
      throw std::runtime_error{"gpu.precision must match the field's value type"};
    planning_.importWisdom();
    check(pf_plan_create(&d, &plan_));
    check(pf_plan_get_info(plan_, &info_));
  }
  ~GpuPlan() {
    planning_.exportWisdom();
    pf_plan_destroy(plan_);
  }
  GpuPlan(const GpuPlan&) = delete;
  GpuPlan& operator=(const GpuPlan&) = delete;

  const pf_plan_info& info() const { return info_; }
  pf_plan* plan() const { return plan_; }

  // fillTransformedMatrix(string) (matrix.hh:223-318)
  pf_eig_stats fillTransformedMatrix() {
    if (custom_) throw std::runtime_error{"you need to call fillMatrix with your covariance class as parameter"};
    pf_eig_stats s{};
    check(pf_spectrum_build(plan_, &s));
    planned_ = false;
    plan();
    spare_pending_ = false;
    return s;
  }

  // fillTransformedMatrix(Covariance&&) with a user functor (matrix.hh:223-265): evaluated
  // on the host at the matrix cells, transformed and checked on the GPU
  template <unsigned dim, typename Covariance>
  pf_eig_stats fillTransformedMatrix(const std::array<double, dim>& extensions, Covariance&& covariance) {
    const std::vector<double> v = customCovarianceValues<dim, RF>(info_, extensions, desc_.variance,
                                                                  desc_.corr_length[0], covariance);
    pf_eig_stats s{};
    check(pf_spectrum_build_values(plan_, v.data(), v.size(), PF_MEM_HOST, &s));
    hasValues_ = true;
    planned_ = false;
    plan();
    spare_pending_ = false;
    return s;
  }

  // generateField (matrix.hh:330-421): the noise is drawn on the host in the reference's
  // order, then scaled and transformed on the GPU; the DFT backend's second field is
  // returned by the next call without drawing noise (matrix.hh:411-420)
  template <typename RNG>
  void generateField(RNG& rng, std::vector<RF>& data) {
    plan();
    data.resize(info_.domain_size);
    std::vector<double> noise;
    if (!spare_pending_) {
      noise.resize(info_.noise_size);
      for (auto& v : noise) v = (double)rng.sample();
    }
    check(pf_generate(plan_, noise.empty() ? nullptr : noise.data(), PF_MEM_HOST, 0, data.data(), PF_MEM_HOST, 0));
    spare_pending_ = info_.field_backend == PF_FIELD_DFT && !spare_pending_;
  }

  // operator* / multiplyRoot / multiplyInverseExtended (matrix.hh:142-176, 1587-1646)
  void multiply(int op, const std::vector<RF>& in, std::vector<RF>& out) const {
    out.resize(in.size());
    check(pf_matvec(plan_, op, sizeof(RF) == 8 ? PF_PREC_F64 : PF_PREC_F32, in.data(), out.data(), PF_MEM_HOST));
  }

  // multiplyInverse (matrix.hh:189-206); FP64 CG vectors
  pf_cg_report multiplyInverse(const std::vector<RF>& in, std::vector<RF>& out, const pf_cg_opts* opts = nullptr) {
    std::vector<double> b(in.begin(), in.end()), x(in.size());
    pf_cg_report rep{};
    pf_status st = pf_multiply_inverse(plan_, b.data(), x.data(), PF_MEM_HOST, opts, &rep);
    if (st != PF_ERR_NOT_CONVERGED) check(st);
    out.assign(x.begin(), x.end());
    return rep;
  }

  // generateUncorrelatedField (matrix.hh:433-445): host white noise, seed + rank
  void generateUncorrelatedField(unsigned int seed, std::vector<RF>& data) const {
    std::default_random_engine generator(seed);
    std::normal_distribution<RF> normalDist(0., 1.);
    data.resize(info_.domain_size);
    for (auto& v : data) v = normalDist(generator);
  }

  // setVarianceAsField (matrix.hh:456-462)
  void setVarianceAsField(std::vector<RF>& data) const { data.assign(info_.domain_size, (RF)desc_.variance); }
};

// RandomField (randomfield.hh:42-1389) restricted to its stochastic part: the trend
// part, file I/O and MPI redistribution are not part of this path.
template <unsigned dim, typename RF = double>
class RandomField {
  ParameterTree config_;
  pf_field_desc desc_;
  ValueTransform<RF> transform_;
  std::shared_ptr<GpuPlan<RF>> matrix_;
  std::vector<RF> data_;
  bool cacheInvMatvec_, cacheInvRootMatvec_;
  bool invMatvecValid_ = true, invRootMatvecValid_ = true;
  std::vector<RF> invMatvecPart_, invRootMatvecPart_;
  std::array<unsigned, dim> cells_;
  std::array<double, dim> ext_;
  std::array<unsigned, dim> dataCells_;  // resolution of data_ and the cached parts
  bool custom_ = false;

  void ensureMatrix() const {}

  // StochasticPart::refine (stochastic.hh:597-672): each cell value copied to its 2^d children
  std::vector<RF> refined(const std::vector<RF>& old) const {
    static_assert(dim == 2 || dim == 3, "refine is implemented for dim 2 and 3, as in the reference");
    std::array<unsigned, 3> n{1, 1, 1}, o{1, 1, 1};
    for (unsigned i = 0; i < dim; i++) {
      n[i] = cells_[i];
      o[i] = dataCells_[i];
    }
    std::vector<RF> out((std::size_t)n[0] * n[1] * n[2]);
    for (unsigned z = 0; z < n[2]; z++)
      for (unsigned y = 0; y < n[1]; y++)
        for (unsigned x = 0; x < n[0]; x++)
          out[x + (std::size_t)n[0] * (y + (std::size_t)n[1] * z)] =
              old[x / 2 + (std::size_t)o[0] * (y / 2 + (std::size_t)o[1] * (dim == 3 ? z / 2 : 0))];
    return out;
  }

  // StochasticPart::coarsen (stochastic.hh:679-755): mean of the 2^d children, summed in the
  // reference's order
  std::vector<RF> coarsened(const std::vector<RF>& old) const {
    static_assert(dim == 2 || dim == 3, "coarsen is implemented for dim 2 and 3, as in the reference");
    std::array<unsigned, 3> n{1, 1, 1}, o{1, 1, 1};
    for (unsigned i = 0; i < dim; i++) {
      n[i] = cells_[i];
      o[i] = dataCells_[i];
    }
    std::vector<RF> out((std::size_t)n[0] * n[1] * n[2]);
    const std::size_t sx = 1, sy = o[0], sz = (std::size_t)o[0] * o[1];
    for (unsigned z = 0; z < n[2]; z++)
      for (unsigned y = 0; y < n[1]; y++)
        for (unsigned x = 0; x < n[0]; x++) {
          const std::size_t b = 2 * x + sy * (2 * y + (std::size_t)o[1] * (dim == 3 ? 2 * z : 0));
          RF v = 0.;
          v += old[b];
          v += old[b + sx];
          v += old[b + sy];
          v += old[b + sy + sx];
          if (dim == 3) {
            v += old[b + sz];
            v += old[b + sz + sx];
            v += old[b + sz + sy];
            v += old[b + sz + sy + sx];
          }
          out[x + (std::size_t)n[0] * (y + (std::size_t)n[1] * z)] = v / (RF)(1u << dim);
        }
    return out;
  }

  // RandomFieldTraits::refine / coarsen (fieldtraits.hh:321-348) + Matrix::update
  void resizeMatrix(unsigned mul, unsigned div) {
    for (unsigned i = 0; i < dim; i++) {
      cells_[i] = cells_[i] * mul / div;
      desc_.cells[i] = (int32_t)cells_[i];
    }
    matrix_ = std::make_shared<GpuPlan<RF>>(desc_, custom_, PlanningKeys::fromConfig(config_));
  }

  // RandomField::refine / coarsen (randomfield.hh:880-1018), using the cached matrix-vector
  // products when they are valid
  void changeLevel(bool up) {
    if (dataCells_ == cells_) return;  // StochasticPart: level unchanged
    const RF scale = std::pow(RF(0.5), up ? -RF(dim) : RF(dim));
    auto level = [&](const std::vector<RF>& v) { return up ? refined(v) : coarsened(v); };
    if (cacheInvMatvec_ && invMatvecValid_) {
      invMatvecPart_ = level(invMatvecPart_);
      matrix_->multiply(PF_OP_MUL, invMatvecPart_, data_);
      for (auto& v : data_) v *= scale;
      for (auto& v : invMatvecPart_) v *= scale;
      if (cacheInvRootMatvec_) {
        matrix_->multiply(PF_OP_ROOT, invMatvecPart_, invRootMatvecPart_);
        for (auto& v : invRootMatvecPart_) v *= scale;
        invRootMatvecValid_ = true;
      }
    } else if (cacheInvRootMatvec_ && invRootMatvecValid_) {
      invRootMatvecPart_ = level(invRootMatvecPart_);
      matrix_->multiply(PF_OP_ROOT, invRootMatvecPart_, data_);
      for (auto& v : data_) v *= scale;
      for (auto& v : invRootMatvecPart_) v *= scale;
      if (cacheInvMatvec_) {
        invMatvecPart_ = data_;
        invMatvecValid_ = false;
      }
    } else {
      data_ = level(data_);
      if (cacheInvMatvec_) invMatvecPart_ = level(invMatvecPart_);
      if (cacheInvRootMatvec_) invRootMatvecPart_ = level(invRootMatvecPart_);
    }
    dataCells_ = cells_;
  }

  static ParameterTree configFromFile(const std::string& fileName) {
    ParameterTree c;
    c.readIniFile(fileName + ".field");
    return c;
  }

 public:
  // randomfield.hh:135-172 (with a file name: stochastic.hh:80-110, the field is read from
  // "<fileName>.stoch.h5"; the cached products are then invalid)
  RandomField(const ParameterTree& config, const std::string& fileName) : RandomField(config) {
    if (fileName.empty()) return;
    const std::vector<double> v = readStochastic(fileName, dim, cells_.data());
    data_.assign(v.begin(), v.end());
    invMatvecValid_ = invRootMatvecValid_ = false;
  }
  // randomfield.hh:192-230: configuration from "<fileName>.field", field from
  // "<fileName>.stoch.h5"
  explicit RandomField(const std::string& fileName) : RandomField(configFromFile(fileName), fileName) {}

  // randomfield.hh:706-713 (trend components are not part of this path): the field to
  // "<fileName>.stoch.h5" and "<fileName>.xdmf", the configuration to "<fileName>.field"
  void writeToFile(const std::string& fileName) const {
    if (dataCells_ != cells_) throw std::runtime_error{"writeToFile: call refine() or coarsen() first"};
    writeStochastic(fileName, dim, cells_.data(), data_.data());
    writeXdmf(fileName, dim, cells_.data(), ext_.data());
    std::ofstream file(fileName + ".field", std::ofstream::trunc);
    if (!file) throw std::runtime_error{"cannot create " + fileName + ".field"};
    config_.report(file);
  }

  explicit RandomField(const ParameterTree& config)
      : config_(config),
        desc_(descFromConfig<dim, RF>(config)),
        cacheInvMatvec_(config.get<bool>("randomField.cacheInvMatvec", false)),
        cacheInvRootMatvec_(config.get<bool>("randomField.cacheInvRootMatvec", false)) {
    transform_ = ValueTransform<RF>(desc_.transform, (RF)desc_.boxcox_lambda);
    const std::string cov = config.get<std::string>("stochastic.covariance");
    custom_ = cov == "custom-iso" || cov == "custom-aniso";
    matrix_ = std::make_shared<GpuPlan<RF>>(desc_, custom_, PlanningKeys::fromConfig(config));
    cells_ = config.get<std::array<unsigned, dim>>("grid.cells");
    dataCells_ = cells_;
    ext_ = config.get<std::array<double, dim>>("grid.extensions");
    data_.assign(matrix_->info().domain_size, RF(0));
    if (cacheInvMatvec_) invMatvecPart_ = data_;
    if (cacheInvRootMatvec_) invRootMatvecPart_ = data_;
  }

  GpuPlan<RF>& matrix() { return *matrix_; }

  // randomfield.hh:430-451: the matrix of a "custom-iso" / "custom-aniso" field from the
  // caller's covariance functor, RF operator()(RF variance, const std::array<RF, dim>& x);
  // classical periodization (the built-in covariances also support merge/fold/cofold)
  template <typename Covariance>
  void fillMatrix(Covariance&& covariance) {
    if (desc_.periodization != PF_PERIODIZATION_CLASSICAL)
      throw std::runtime_error{"custom covariance functors support embedding.periodization = classical only"};
    matrix_->template fillTransformedMatrix<dim>(ext_, covariance);
  }

  // randomfield.hh:880-887 / 955-961: double (halve) the resolution of the matrix
  void refineMatrix() { resizeMatrix(2, 1); }
  void coarsenMatrix() { resizeMatrix(1, 2); }
  // randomfield.hh:897-945 / 971-1018: bring the field (and cached products) to the
  // matrix's resolution
  void refine() { changeLevel(true); }
  void coarsen() { changeLevel(false); }
  const std::vector<RF>& dataVector() const { return data_; }
  std::vector<RF>& dataVector() { return data_; }

  // randomfield.hh:512-529 (seed += rank; one rank here)
  void generate(unsigned int seed) {
    CppRNGBackend<RF> rng;
    rng.seed(seed);
    generateWithRNG(rng);
  }

  // randomfield.hh:541-558
  template <typename RNG>
  void generateWithRNG(RNG& rng) {
    matrix_->generateField(rng, data_);
    invMatvecValid_ = false;
    invRootMatvecValid_ = false;
  }

  // randomfield.hh:593-612
  void generateUncorrelated(unsigned int seed) {
    matrix_->generateUncorrelatedField(seed, data_);
    invMatvecValid_ = false;
    invRootMatvecValid_ = false;
  }

  // randomfield.hh:641-651 with StochasticPart::evaluate (stochastic.hh:480-574) and
  // coordsToIndices (fieldtraits.hh:443-451); a point on the upper boundary belongs to
  // the last cell
  void evaluate(const std::array<double, dim>& location, RF& output) const {
    std::size_t index = 0, stride = 1;
    for (unsigned i = 0; i < dim; i++) {
      unsigned c = (unsigned)(location[i] * (cells_[i] + 1e-6) / ext_[i]);
      if (c >= cells_[i]) c = cells_[i] - 1;
      index += c * stride;
      stride *= cells_[i];
    }
    output = data_[index];
    transform_.apply(output);
  }

  // randomfield.hh:664-695
  void bulkEvaluate(std::vector<RF>& output, std::array<unsigned, dim>& sizes) const {
    sizes = cells_;
    output = data_;
    for (auto& v : output) transform_.apply(v);
  }

  // randomfield.hh:1181-1202
  void timesMatrix() {
    if (cacheInvMatvec_) {
      invMatvecPart_ = data_;
      invMatvecValid_ = true;
    }
    if (cacheInvRootMatvec_) {
      matrix_->multiply(PF_OP_ROOT, data_, invRootMatvecPart_);
      invRootMatvecValid_ = true;
    }
    std::vector<RF> out;
    matrix_->multiply(PF_OP_MUL, data_, out);
    data_.swap(out);
  }

  // randomfield.hh:1211-1238
  void timesInverseMatrix() {
    if (cacheInvMatvec_ && invMatvecValid_) {
      if (cacheInvRootMatvec_) {
        matrix_->multiply(PF_OP_ROOT, invMatvecPart_, invRootMatvecPart_);
        invRootMatvecValid_ = true;
      }
      data_ = invMatvecPart_;
      invMatvecValid_ = false;
    } else {
      std::vector<RF> out;
      matrix_->multiplyInverse(data_, out);
      data_.swap(out);
      if (cacheInvMatvec_) invMatvecValid_ = false;
      if (cacheInvRootMatvec_) invRootMatvecValid_ = false;
    }
  }

  // randomfield.hh:1250-1268
  void timesMatrixRoot() {
    if (cacheInvMatvec_ && cacheInvRootMatvec_) {
      invMatvecPart_ = invRootMatvecPart_;
      invMatvecValid_ = invRootMatvecValid_;
    }
    if (cacheInvRootMatvec_) {
      invRootMatvecPart_ = data_;
      invRootMatvecValid_ = true;
    }
    std::vector<RF> out;
    matrix_->multiply(PF_OP_ROOT, data_, out);
    data_.swap(out);
  }

  // randomfield.hh:1278-1310
  void timesInvMatRoot() {
    if (cacheInvRootMatvec_ && invRootMatvecValid_) {
      data_ = invRootMatvecPart_;
      invRootMatvecValid_ = false;
      if (cacheInvMatvec_) {
        invRootMatvecPart_ = invMatvecPart_;
        invRootMatvecValid_ = invMatvecValid_;
        invMatvecValid_ = false;
      }
    } else {
      std::vector<RF> out;
      matrix_->multiplyInverse(data_, out);
      data_.swap(out);
      if (cacheInvRootMatvec_) {
        invRootMatvecPart_ = data_;
        invRootMatvecValid_ = true;
      }
      matrix_->multiply(PF_OP_ROOT, data_, out);
      data_.swap(out);
      if (cacheInvMatvec_) invMatvecValid_ = false;
    }
  }

  // vector-space operations of the stochastic part (randomfield.hh:1027-1342)
  RandomField& operator+=(const RandomField& o) {
    for (std::size_t i = 0; i < data_.size(); i++) data_[i] += o.data_[i];
    invMatvecValid_ = invRootMatvecValid_ = false;
    return *this;
  }
  RandomField& operator-=(const RandomField& o) {
    for (std::size_t i = 0; i < data_.size(); i++) data_[i] -= o.data_[i];
    invMatvecValid_ = invRootMatvecValid_ = false;
    return *this;
  }
  RandomField& operator*=(RF a) {
    for (auto& v : data_) v *= a;
    if (cacheInvMatvec_)
      for (auto& v : invMatvecPart_) v *= a;
    if (cacheInvRootMatvec_)
      for (auto& v : invRootMatvecPart_) v *= a;
    return *this;
  }
  RandomField& axpy(const RandomField& o, RF a) {
    for (std::size_t i = 0; i < data_.size(); i++) data_[i] += a * o.data_[i];
    invMatvecValid_ = invRootMatvecValid_ = false;
    return *this;
  }
  RF operator*(const RandomField& o) const {
    RF s = 0;
    for (std::size_t i = 0; i < data_.size(); i++) s += data_[i] * o.data_[i];
    return s;
  }
  RF oneNorm() const {
    RF s = 0;
    for (auto v : data_) s += std::abs(v);
    return s;
  }
  RF twoNorm() const { return std::sqrt(*this * *this); }
  RF infNorm() const {
    RF m = 0;
    for (auto v : data_) m = std::max(m, std::abs(v));
    return m;
  }
  void zero() {
    std::fill(data_.begin(), data_.end(), RF(0));
    invMatvecValid_ = invRootMatvecValid_ = false;
  }
};

}  // namespace parafields_b200
