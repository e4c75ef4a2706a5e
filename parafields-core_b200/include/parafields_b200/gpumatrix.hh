// gpumatrix.hh -- the B200 matrix in the reference's own plug-in slot.
//
// parafields-core picks its covariance matrix at compile time through template template
// parameters (include/parafields/randomfield.hh:42-47):
//
//   using Field = parafields::RandomField<GridTraits, parafields_b200::GpuMatrix,
//                                         parafields_b200::GpuMatrix>;
//
// RandomField instantiates IsoMatrix<Traits> / AnisoMatrix<Traits> with its
// RandomFieldTraits (randomfield.hh:153-164, 208-218) and calls the members that
// parafields::Matrix defines (matrix.hh:63-206, 223-265, 330-462).  GpuMatrix<Traits>
// defines the same members and forwards them to the C ABI of libpfcuda.so
// (include/parafields_b200.h); the spectrum, the realizations and the products live on
// the GPU, the StochasticPart's dataVector stays the host vector the reference uses.
//
// Access: RandomFieldTraits befriends IsoMatrix<ThisType>, AnisoMatrix<ThisType> and
// their MatrixBackendType / FieldBackendType (fieldtraits.hh:104-107), and StochasticPart
// befriends Traits::IsoMatrixType / AnisoMatrixType (stochastic.hh:37-38), so GpuMatrix
// reads the traits' configuration and writes dataVector / evalValid as Matrix does.
#pragma once

#include <array>
#include <cmath>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../../../include/parafields_b200.h"
#include "randomfield.hh"

namespace parafields {
template <typename Traits>
class StochasticPart;  // stochastic.hh:21-27
}

namespace parafields_b200 {

// The matrix "backend" of the GPU matrix: the plan's device buffers (spectrum in the
// layout of the DCT, R2C or DFT matrix backend).  It exists so that
// Matrix::MatrixBackendType names a class, as RandomFieldTraits befriends it.
template <typename Traits>
class GpuMatrixBackend {
 public:
  explicit GpuMatrixBackend(const std::shared_ptr<Traits>&) {}
};

// The field "backend": the plan's device work tori (R2C, DFT or DCT/DST field backend).
template <typename Traits>
class GpuFieldBackend {
 public:
  explicit GpuFieldBackend(const std::shared_ptr<Traits>&) {}
};

template <typename Traits>
class GpuMatrix {
 public:
  using MatrixBackendType = GpuMatrixBackend<Traits>;  // matrix.hh:63-66
  using FieldBackendType = GpuFieldBackend<Traits>;
  using StochasticPartType = parafields::StochasticPart<Traits>;

 private:
  using RF = typename Traits::RF;
  enum { dim = Traits::dim };

  const std::shared_ptr<Traits> traits;
  MatrixBackendType matrixBackend;
  FieldBackendType fieldBackend;
  std::string covariance;
  RF variance = 0;
  mutable pf_plan* plan = nullptr;
  mutable pf_plan_info info{};
  mutable bool valid = false;       // matrixBackend.valid(): spectrum built for this level
  mutable bool sparePending = false;  // DFT field backend: second field cached (matrix.hh:411-420)
  PlanningKeys planning;             // fftw.measure / fftw.useWisdom

  void release() {
    if (plan) {
      planning.exportWisdom();
      pf_plan_destroy(plan);
    }
    plan = nullptr;
  }

  static constexpr int32_t precision() { return sizeof(RF) == 8 ? PF_PREC_F64 : PF_PREC_F32; }

  // (traits' config + current level) -> descriptor; the traits' cells change with
  // refine / coarsen (fieldtraits.hh:321-348) while the configuration keeps grid.cells
  pf_field_desc descriptor() const {
    pf_field_desc d = descFromConfig<dim, RF>((*traits).config);
    for (unsigned i = 0; i < dim; i++) d.cells[i] = (int32_t)(*traits).cells[i];
    return d;
  }

  // matrix-vector products on the host vector of a StochasticPart, in place
  void product(int32_t op, std::vector<RF>& v) const {
    check(pf_matvec(plan, op, precision(), v.data(), v.data(), PF_MEM_HOST));
  }

 public:
  // Matrix(const std::shared_ptr<Traits>&) (matrix.hh:98-105)
  explicit GpuMatrix(const std::shared_ptr<Traits>& traits_)
      : traits(traits_), matrixBackend(traits_), fieldBackend(traits_) {
    update();
  }
  ~GpuMatrix() { release(); }
  GpuMatrix(const GpuMatrix&) = delete;
  GpuMatrix& operator=(const GpuMatrix&) = delete;

  // update() (matrix.hh:117-131): called after construction and after the traits were
  // refined or coarsened; the plan is rebuilt for the traits' current cells and its
  // spectrum is built lazily, as the reference's backends are
  void update() {
    release();
    covariance = (*traits).covariance;
    variance = (*traits).variance;
    const pf_field_desc d = descriptor();
    planning = PlanningKeys::fromConfig((*traits).config);
    planning.importWisdom();
    check(pf_plan_create(&d, &plan));
    check(pf_plan_get_info(plan, &info));
    valid = false;
    sparePending = false;
  }

  // operator* (matrix.hh:142-151): multiplyExtended, i.e. (C_ext x)/N on the domain
  StochasticPartType operator*(const StochasticPartType& input) const {
    StochasticPartType output(input);
    ensureSpectrum();
    product(PF_OP_MUL, output.dataVector);
    output.evalValid = false;
    return output;
  }

  // multiplyRoot (matrix.hh:165-174)
  StochasticPartType multiplyRoot(const StochasticPartType& input) const {
    StochasticPartType output(input);
    ensureSpectrum();
    product(PF_OP_ROOT, output.dataVector);
    output.evalValid = false;
    return output;
  }

  // multiplyInverse (matrix.hh:189-206): zero-field shortcut, torus-inverse initial
  // guess and innerCG with the reference's stopping rules, all inside pf_multiply_inverse
  StochasticPartType multiplyInverse(const StochasticPartType& input) const {
    StochasticPartType output(input);
    bool fieldZero = true;
    for (std::size_t i = 0; i < (std::size_t)input.localDomainSize; i++)
      if (std::abs(input.dataVector[i]) > 1e-10) fieldZero = false;
    if (fieldZero) return output;
    ensureSpectrum();
    std::vector<double> b(input.dataVector.begin(), input.dataVector.begin() + input.localDomainSize);
    std::vector<double> x(b.size());
    pf_cg_report rep{};
    check(pf_multiply_inverse(plan, b.data(), x.data(), PF_MEM_HOST, nullptr, &rep));
    for (std::size_t i = 0; i < x.size(); i++) output.dataVector[i] = (RF)x[i];
    output.evalValid = false;
    return output;
  }

  // fillTransformedMatrix (matrix.hh:223-318): a covariance name builds the spectrum on
  // the GPU; any other argument is the caller's covariance functor, evaluated on the host
  // at the matrix cells with the ScaledIdentityMatrix geometry (matrix.hh:262-264) and
  // handed to the GPU for the transform and the eigenvalue check
  template <typename Covariance>
  void fillTransformedMatrix(Covariance&& cov) const {
    pf_eig_stats stats{};
    if constexpr (std::is_same<std::decay_t<Covariance>, std::string>::value) {
      if (cov == "custom-iso" || cov == "custom-aniso")
        throw std::runtime_error{"you need to call fillMatrix with your covariance class as parameter"};
      check(pf_spectrum_build(plan, &stats));
    } else {
      std::array<double, dim> ext;
      for (unsigned i = 0; i < dim; i++) ext[i] = (double)(*traits).extensions[i];
      const double corr = (*traits).config.template get<double>("stochastic.corrLength");
      const std::vector<double> v = customCovarianceValues<dim, RF>(info, ext, (double)variance, corr, cov);
      check(pf_spectrum_build_values(plan, v.data(), v.size(), PF_MEM_HOST, &stats));
    }
    planning.plan(plan);
    valid = true;
    sparePending = false;
  }

  // generateField (matrix.hh:330-421): the noise is drawn from rng.sample() on the host
  // in the reference's order (two draws per stored frequency, or one per DCT cell and
  // symmetry type), then scaled, transformed and extracted on the GPU.  With the DFT
  // field backend every second call returns the cached imaginary part without drawing.
  template <typename RNG>
  void generateField(RNG& rngBackend, StochasticPartType& stochasticPart) const {
    if (!valid) fillTransformedMatrix(covariance);
    std::vector<double> noise;
    if (!sparePending) {
      noise.resize(info.noise_size);
      for (auto& v : noise) v = (double)rngBackend.sample();
    }
    check(pf_generate(plan, noise.empty() ? nullptr : noise.data(), PF_MEM_HOST, 0,
                      stochasticPart.dataVector.data(), PF_MEM_HOST, 0));
    sparePending = info.field_backend == PF_FIELD_DFT && !sparePending;
    stochasticPart.evalValid = false;
  }

  // generateUncorrelatedField (matrix.hh:433-445): host white noise, seed + rank
  void generateUncorrelatedField(unsigned int seed, StochasticPartType& stochasticPart) const {
    seed += (unsigned int)(*traits).rank;
    std::default_random_engine generator(seed);
    std::normal_distribution<RF> normalDist(0., 1.);
    for (std::size_t index = 0; index < (std::size_t)stochasticPart.localDomainSize; index++)
      stochasticPart.dataVector[index] = normalDist(generator);
    stochasticPart.evalValid = false;
  }

  // setVarianceAsField (matrix.hh:456-462)
  void setVarianceAsField(StochasticPartType& stochasticPart) const {
    for (std::size_t index = 0; index < (std::size_t)stochasticPart.localDomainSize; index++)
      stochasticPart.dataVector[index] = variance;
    stochasticPart.evalValid = false;
  }

 private:
  void ensureSpectrum() const {
    if (!valid) fillTransformedMatrix(covariance);
  }
};

}  // namespace parafields_b200
