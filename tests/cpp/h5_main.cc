// CPU checks of the header-only field files: writes a field with fieldio.hh / h5lite.hh and
// reads it back; the test also parses the file independently.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <sstream>
#include <string>
#include <vector>

#include "parafields_b200/fieldio.hh"
#include "parafields_b200/parametertree.hh"

using namespace parafields_b200;

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string mode = argv[1], base = argv[2];
  if (mode == "write") {  // write <base> dim c0 c1 c2 e0 e1 e2 [f32]
    const int dim = std::atoi(argv[3]);
    unsigned cells[3] = {1, 1, 1};
    double ext[3] = {1, 1, 1};
    size_t n = 1;
    for (int i = 0; i < dim; i++) {
      cells[i] = (unsigned)std::atoi(argv[4 + i]);
      ext[i] = std::atof(argv[4 + dim + i]);
      n *= cells[i];
    }
    const bool f32 = argc > 4 + 2 * dim && std::string(argv[4 + 2 * dim]) == "f32";
    std::vector<double> d(n);
    std::vector<float> f(n);
    for (size_t i = 0; i < n; i++) {
      d[i] = std::sin(0.37 * (double)i) * 1.5 + 1e-3 * (double)i;
      f[i] = (float)d[i];
    }
    if (f32)
      writeStochastic(base, dim, cells, f.data());
    else
      writeStochastic(base, dim, cells, d.data());
    writeXdmf(base, dim, cells, ext);
    const std::vector<double> back = readStochastic(base, dim, cells);
    for (size_t i = 0; i < n; i++)
      if (back[i] != (f32 ? (double)f[i] : d[i])) {
        std::printf("mismatch at %zu\n", i);
        return 1;
      }
    std::printf("ok %zu\n", n);
    return 0;
  }
  if (mode == "read") {  // read <base> dim c0 c1 c2 -> values, one per line
    const int dim = std::atoi(argv[3]);
    unsigned cells[3] = {1, 1, 1};
    for (int i = 0; i < dim; i++) cells[i] = (unsigned)std::atoi(argv[4 + i]);
    try {
      const std::vector<double> v = readStochastic(base, dim, cells);
      for (double x : v) std::printf("%.17g\n", x);
    } catch (const std::exception& e) {
      std::printf("error: %s\n", e.what());
      return 1;
    }
    return 0;
  }
  if (mode == "report") {  // report <ini> -> the report, then the report parsed again
    ParameterTree c;
    c.readIniFile(base);
    std::ostringstream a;
    c.report(a);
    ParameterTree d;
    d.parseIni(a.str());
    std::ostringstream b;
    d.report(b);
    std::printf("%s", a.str().c_str());
    return a.str() == b.str() ? 0 : 1;
  }
  return 2;
}
