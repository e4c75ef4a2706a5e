// Test driver of the C++ facade (parafields_b200::RandomField).
//   facade_main config <ini>                 prints the descriptor built from the keys
//   facade_main run <ini> <seed> <outdir>    generate / timesMatrix / timesInverseMatrix,
//                                            writing noise, fields and products as raw doubles
//   facade_main refine <ini> <seed> <outdir> refine / coarsen, without and with a cached
//                                            inverse product (randomField.cacheInvMatvec)
//   facade_main io <ini> <seed> <outdir>     writeToFile, then RandomField(fileName) and
//                                            RandomField(config, fileName) read it back
#include <cstdio>
#include <fstream>
#include <iostream>

#include "parafields_b200/randomfield.hh"

using namespace parafields_b200;

static void dump(const std::string& path, const std::vector<double>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(double)));
}

template <unsigned dim>
static int run(const ParameterTree& cfg, unsigned seed, const std::string& out) {
  RandomField<dim> field(cfg);
  field.generate(seed);
  // the noise generate() drew: the same CppRNGBackend stream
  CppRNGBackend<double> rng;
  rng.seed(seed);
  std::vector<double> noise(field.matrix().info().noise_size);
  for (auto& v : noise) v = rng.sample();
  dump(out + "/noise.bin", noise);
  dump(out + "/field.bin", field.dataVector());
  std::vector<double> bulk;
  std::array<unsigned, dim> sizes;
  field.bulkEvaluate(bulk, sizes);
  dump(out + "/bulk.bin", bulk);
  std::array<double, dim> loc;
  for (unsigned i = 0; i < dim; i++) loc[i] = 0.5 * cfg.get<std::array<double, dim>>("grid.extensions")[i];
  double mid = 0;
  field.evaluate(loc, mid);
  dump(out + "/mid.bin", {mid});
  field.timesMatrix();
  dump(out + "/cx.bin", field.dataVector());
  field.timesInverseMatrix();
  dump(out + "/cinvcx.bin", field.dataVector());
  field.generateUncorrelated(seed);
  dump(out + "/white.bin", field.dataVector());
  return 0;
}

template <unsigned dim>
static int io_run(const ParameterTree& cfg, unsigned seed, const std::string& out) {
  RandomField<dim> field(cfg);
  field.generate(seed);
  field.writeToFile(out + "/saved");
  RandomField<dim> again(out + "/saved");
  RandomField<dim> again2(cfg, out + "/saved");
  if (again.dataVector() != field.dataVector() || again2.dataVector() != field.dataVector()) return 3;
  // the product of the read field equals the product of the original
  field.timesMatrix();
  again.timesMatrix();
  dump(out + "/a.bin", field.dataVector());
  dump(out + "/b.bin", again.dataVector());
  std::printf("io ok\n");
  return 0;
}

template <unsigned dim>
static int refine_run(const ParameterTree& cfg, unsigned seed, const std::string& out) {
  if constexpr (dim == 1) {
    return 5;
  } else {
    RandomField<dim> field(cfg);
    field.generate(seed);
    dump(out + "/field.bin", field.dataVector());
    field.refineMatrix();
    field.refine();
    dump(out + "/refined.bin", field.dataVector());
    field.coarsenMatrix();
    field.coarsen();
    dump(out + "/back.bin", field.dataVector());
    // with the inverse product cached: timesMatrix keeps x, refine recomputes C_fine refine(x)
    ParameterTree c2 = cfg;
    c2["randomField.cacheInvMatvec"] = "true";
    RandomField<dim> cached(c2);
    cached.generate(seed);
    cached.timesMatrix();
    cached.refineMatrix();
    cached.refine();
    dump(out + "/cached_refined.bin", cached.dataVector());
    return 0;
  }
}

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  ParameterTree cfg;
  try {
    cfg.readIniFile(argv[2]);
    const std::string mode = argv[1];
    const std::string cells = cfg.raw("grid.cells");
    unsigned dim = 0;
    {
      std::istringstream in(cells);
      unsigned x;
      while (in >> x) dim++;
    }
    if (mode == "config") {
      pf_field_desc d = dim == 1 ? descFromConfig<1, double>(cfg)
                                 : (dim == 2 ? descFromConfig<2, double>(cfg) : descFromConfig<3, double>(cfg));
      std::printf("dim=%d cells=%d,%d,%d ext=%g,%g,%g factor=%d periodic=%d cov=%d var=%g aniso=%d corr=%g,%g,%g,%g "
                  "approx=%d thr=%g transposed=%d prec=%d eig=%d cg=%d transform=%d boxcox=%g gamma=%g\n",
                  d.dim, d.cells[0], d.cells[1], d.cells[2], d.extensions[0], d.extensions[1], d.extensions[2],
                  d.embedding_factor, d.periodic, d.covariance, d.variance, d.anisotropy, d.corr_length[0],
                  d.corr_length[1], d.corr_length[2], d.corr_length[3], d.approximate, d.threshold, d.transposed,
                  d.precision, d.eigen_check, d.cg_iterations, d.transform, d.boxcox_lambda, d.exp_gamma);
      std::printf("per=%d sig=%d comb=%d mrec=%d sstart=%g send=%g fmf=%g frec=%d cmf=%g crec=%d\n", d.periodization,
                  d.sigmoid, d.sigmoid_combine, d.merge_recursions, d.sigmoid_start, d.sigmoid_end, d.fold_max_factor,
                  d.fold_recursions, d.cofold_max_factor, d.cofold_recursions);
      return 0;
    }
    const unsigned seed = (unsigned)std::stoul(argv[3]);
    if (mode == "refine") return dim == 2 ? refine_run<2>(cfg, seed, argv[4]) : refine_run<3>(cfg, seed, argv[4]);
    if (mode == "io")
      return dim == 1 ? io_run<1>(cfg, seed, argv[4]) : (dim == 2 ? io_run<2>(cfg, seed, argv[4]) : io_run<3>(cfg, seed, argv[4]));
    if (dim == 1) return run<1>(cfg, seed, argv[4]);
    if (dim == 2) return run<2>(cfg, seed, argv[4]);
    return run<3>(cfg, seed, argv[4]);
  } catch (const NegativeEigenvalueError& e) {
    std::printf("NegativeEigenvalueError: %s\n", e.what());
    return 3;
  } catch (const std::exception& e) {
    std::printf("error: %s\n", e.what());
    return 4;
  }
}
