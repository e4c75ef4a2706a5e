// Compile and run test of parafields_b200::GpuMatrix in the reference's template slot.
//
// The reference's RandomFieldTraits, StochasticPart and RandomField need dune-common and
// MPI, which this image lacks, so this file declares stand-ins with the same names,
// member names, friend declarations and call forms that GpuMatrix relies on
// (fieldtraits.hh:60-150: friend IsoMatrix<ThisType>, friend
// IsoMatrix<ThisType>::MatrixBackendType / FieldBackendType, private members config,
// cells, extensions, variance, covariance, rank; stochastic.hh:21-60: friend
// Traits::IsoMatrixType, private dataVector / evalValid / localDomainSize;
// randomfield.hh:153-164, 430-451, 512-558, 1181-1268: IsoMatrix<Traits>(traits),
// .template fillTransformedMatrix<Covariance>(...), generateField(rng, stochasticPart),
// (*matrix) * part, multiplyRoot, multiplyInverse, update() after refinement).
// GpuMatrix compiles against them exactly as it would inside a reference build.
//
//   slot_main run <ini> <seed> <outdir>      generate / timesMatrix / timesMatrixRoot /
//                                            timesInverseMatrix / refineMatrix+generate
//   slot_main custom <ini> <seed> <outdir>   fillMatrix(user functor) + generate
//   slot_main noise <count> <seed> <outdir>   the first <count> samples of the seeded
//                                            CppRNGBackend stream that generate() draws
#include <array>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <memory>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "parafields_b200/parametertree.hh"

namespace Dune {
using ParameterTree = parafields_b200::ParameterTree;
}

namespace parafields {

template <typename GridTraits, template <typename> class IsoMatrix, template <typename> class AnisoMatrix>
class RandomField;
template <typename Traits>
class StochasticPart;

// stand-in for RandomFieldTraits (fieldtraits.hh:60-150), single rank
template <typename GridTraits, template <typename> class IsoMatrix, template <typename> class AnisoMatrix>
class RandomFieldTraits {
  using ThisType = RandomFieldTraits<GridTraits, IsoMatrix, AnisoMatrix>;

 public:
  enum { dim = GridTraits::dim };
  using RF = typename GridTraits::RangeField;
  using IsoMatrixType = IsoMatrix<ThisType>;
  using AnisoMatrixType = AnisoMatrix<ThisType>;
  using Index = unsigned int;
  using Indices = std::array<Index, dim>;

 private:
  friend StochasticPart<ThisType>;
  friend IsoMatrix<ThisType>;
  friend AnisoMatrix<ThisType>;
  friend typename IsoMatrix<ThisType>::MatrixBackendType;
  friend typename IsoMatrix<ThisType>::FieldBackendType;
  friend typename AnisoMatrix<ThisType>::MatrixBackendType;
  friend typename AnisoMatrix<ThisType>::FieldBackendType;
  friend RandomField<GridTraits, IsoMatrix, AnisoMatrix>;

  int rank = 0, commSize = 1;
  const Dune::ParameterTree& config;
  const std::array<RF, dim> extensions;
  const RF variance;
  const std::string covariance;
  unsigned int level = 0;
  Indices cells;
  Index localDomainSize = 1;

 public:
  explicit RandomFieldTraits(const Dune::ParameterTree& config_)
      : config(config_),
        extensions(config.get<std::array<RF, dim>>("grid.extensions")),
        variance(config.get<RF>("stochastic.variance")),
        covariance(config.get<std::string>("stochastic.covariance")),
        cells(config.get<Indices>("grid.cells")) {
    update();
  }
  void update() {
    localDomainSize = 1;
    for (unsigned i = 0; i < dim; i++) localDomainSize *= cells[i];
  }
  // fieldtraits.hh:321-333: twice the cells per dimension
  void refine() {
    for (unsigned i = 0; i < dim; i++) cells[i] *= 2;
    level++;
    update();
  }
};

// stand-in for StochasticPart (stochastic.hh:21-60): the members the matrix touches
template <typename Traits>
class StochasticPart {
  using RF = typename Traits::RF;
  friend typename Traits::IsoMatrixType;
  friend typename Traits::AnisoMatrixType;
  template <typename G, template <typename> class I, template <typename> class A>
  friend class RandomField;

  std::shared_ptr<Traits> traits;
  typename Traits::Index localDomainSize;
  mutable std::vector<RF> dataVector;
  mutable bool evalValid = false;

 public:
  explicit StochasticPart(const std::shared_ptr<Traits>& t) : traits(t) { update(); }
  void update() {
    localDomainSize = (*traits).localDomainSize;
    dataVector.assign(localDomainSize, RF(0));
    evalValid = false;
  }
};

// std::default_random_engine + std::normal_distribution, seeded with seed + rank
template <typename Traits>
class CppRNGBackend {
  std::default_random_engine generator;
  std::normal_distribution<typename Traits::RF> normalDist{0., 1.};

 public:
  explicit CppRNGBackend(unsigned int seed) : generator(seed) {}
  typename Traits::RF sample() { return normalDist(generator); }
};

// stand-in for RandomField: the call forms of randomfield.hh
template <typename GridTraits, template <typename> class IsoMatrix, template <typename> class AnisoMatrix>
class RandomField {
 public:
  using Traits = RandomFieldTraits<GridTraits, IsoMatrix, AnisoMatrix>;

 private:
  std::shared_ptr<Traits> traits;
  std::shared_ptr<IsoMatrix<Traits>> isoMatrix;
  std::shared_ptr<AnisoMatrix<Traits>> anisoMatrix;
  bool useAnisoMatrix;
  StochasticPart<Traits> stochasticPart;

 public:
  explicit RandomField(const Dune::ParameterTree& config)
      : traits(new Traits(config)), stochasticPart(traits) {
    const std::string aniso = config.get<std::string>("stochastic.anisotropy", std::string("none"));
    const std::string cov = config.get<std::string>("stochastic.covariance");
    if ((aniso == "none" || aniso == "axiparallel") && cov != "custom-aniso") {
      isoMatrix = std::shared_ptr<IsoMatrix<Traits>>(new IsoMatrix<Traits>(traits));
      useAnisoMatrix = false;
    } else {
      anisoMatrix = std::shared_ptr<AnisoMatrix<Traits>>(new AnisoMatrix<Traits>(traits));
      useAnisoMatrix = true;
    }
  }
  template <typename Covariance>
  void fillMatrix(Covariance&& covariance) {
    if (useAnisoMatrix)
      (*anisoMatrix).template fillTransformedMatrix<Covariance>(std::forward<Covariance>(covariance));
    else
      (*isoMatrix).template fillTransformedMatrix<Covariance>(std::forward<Covariance>(covariance));
  }
  void generate(unsigned int seed) {
    CppRNGBackend<Traits> rng(seed + (unsigned)(*traits).rank);
    if (useAnisoMatrix)
      (*anisoMatrix).generateField(rng, stochasticPart);
    else
      (*isoMatrix).generateField(rng, stochasticPart);
  }
  void timesMatrix() {
    stochasticPart = useAnisoMatrix ? (*anisoMatrix) * stochasticPart : (*isoMatrix) * stochasticPart;
  }
  void timesMatrixRoot() {
    stochasticPart = useAnisoMatrix ? (*anisoMatrix).multiplyRoot(stochasticPart)
                                    : (*isoMatrix).multiplyRoot(stochasticPart);
  }
  void timesInverseMatrix() {
    stochasticPart = useAnisoMatrix ? (*anisoMatrix).multiplyInverse(stochasticPart)
                                    : (*isoMatrix).multiplyInverse(stochasticPart);
  }
  void generateUncorrelated(unsigned int seed) {
    if (useAnisoMatrix)
      (*anisoMatrix).generateUncorrelatedField(seed, stochasticPart);
    else
      (*isoMatrix).generateUncorrelatedField(seed, stochasticPart);
  }
  void refineMatrix() {
    (*traits).refine();
    if (useAnisoMatrix)
      (*anisoMatrix).update();
    else
      (*isoMatrix).update();
    stochasticPart.update();
  }
  const std::vector<typename Traits::RF>& data() const { return stochasticPart.dataVector; }
};

}  // namespace parafields

#include "parafields_b200/gpumatrix.hh"

template <unsigned d>
struct GridTraits {
  enum { dim = d };
  using RangeField = double;
};

// a user covariance functor with the signature of the reference's built-in ones
// (covariance.hh:355-372): sigma^2 exp(-|x|)
struct UserExponential {
  template <typename RF, long unsigned int dim>
  RF operator()(const RF variance, const std::array<RF, dim>& x) const {
    RF sum = 0.;
    for (unsigned int i = 0; i < dim; i++) sum += x[i] * x[i];
    return variance * std::exp(-std::sqrt(sum));
  }
};

static void dump(const std::string& path, const std::vector<double>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

template <unsigned dim>
static int run(const std::string& mode, const Dune::ParameterTree& cfg, unsigned seed, const std::string& out) {
  using Field = parafields::RandomField<GridTraits<dim>, parafields_b200::GpuMatrix, parafields_b200::GpuMatrix>;
  Field field(cfg);
  if (mode == "custom") field.fillMatrix(UserExponential());
  field.generate(seed);
  dump(out + "/field.bin", field.data());
  if (mode == "custom") return 0;
  field.timesMatrix();
  dump(out + "/cx.bin", field.data());
  field.timesMatrixRoot();
  dump(out + "/rcx.bin", field.data());
  field.timesInverseMatrix();
  dump(out + "/inv.bin", field.data());
  field.refineMatrix();
  field.generate(seed);
  dump(out + "/refined_field.bin", field.data());
  std::printf("slot ok\n");
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  Dune::ParameterTree cfg;
  try {
    if (std::string(argv[1]) == "noise") {
      using T = parafields::RandomFieldTraits<GridTraits<2>, parafields_b200::GpuMatrix, parafields_b200::GpuMatrix>;
      parafields::CppRNGBackend<T> rng((unsigned)std::stoul(argv[3]));
      std::vector<double> v(std::stoull(argv[2]));
      for (auto& x : v) x = rng.sample();
      dump(std::string(argv[4]) + "/noise.bin", v);
      return 0;
    }
    cfg.readIniFile(argv[2]);
    std::istringstream in(cfg.raw("grid.cells"));
    unsigned dim = 0, x;
    while (in >> x) dim++;
    const unsigned seed = (unsigned)std::stoul(argv[3]);
    if (dim == 2) return run<2>(argv[1], cfg, seed, argv[4]);
    if (dim == 3) return run<3>(argv[1], cfg, seed, argv[4]);
    return 5;
  } catch (const parafields_b200::NegativeEigenvalueError& e) {
    std::printf("NegativeEigenvalueError: %s\n", e.what());
    return 3;
  } catch (const std::exception& e) {
    std::printf("error: %s\n", e.what());
    return 4;
  }
}
