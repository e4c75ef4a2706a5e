// fieldio.hh -- the files of StochasticPart::writeToFile (stochastic.hh:273-294): the field
// as dataset /stochastic of "<name>.stoch.h5" (h5lite.hh) and the XDMF description
// "<name>.xdmf" that points visualisation tools at it (writeToXDMF, io.hh:306-349, for
// dimensions 1 to 3).
#pragma once

#include <cstdint>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "h5lite.hh"

namespace parafields_b200 {

// XDMF 2.0 structured grid over the cells (dimension 0 fastest), spacing extension / cells
// per axis (the 1D and 2D files repeat axis 0's spacing to fill three entries, and list
// the spacings in axis order), one cell-centred attribute read from the HDF5 dataset
inline void writeXdmf(const std::string& fileName, int dim, const unsigned* cells, const double* ext) {
  if (dim < 1 || dim > 3) throw std::runtime_error{"XDMF output is written for dimensions 1 to 3"};
  std::ofstream file(fileName + ".xdmf", std::ofstream::trunc);
  if (!file) throw std::runtime_error{"cannot create " + fileName + ".xdmf"};
  std::string rev;
  for (int i = 0; i < dim; i++) rev += std::to_string(cells[dim - 1 - i]) + " ";
  file << "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n<Xdmf Version=\"2.0\">\n <Domain>\n";
  file << "  <Grid Name=\"StructuredGrid\">\n   <Topology TopologyType=\"3DRectMesh\" NumberOfElements=\"" << rev
       << "\"/>\n   <Geometry GeometryType=\"origin_dxdydz\">\n    <DataItem Dimensions=\"3\">\n     0. 0. 0.\n"
       << "    </DataItem>\n    <DataItem Dimensions=\"3\">\n     ";
  for (int i = 0; i < 3 - dim; i++) file << ext[0] / cells[0] << " ";
  for (int i = 0; i < dim; i++) file << ext[i] / cells[i] << " ";
  file << "\n    </DataItem>\n   </Geometry>\n   <Attribute Name=\"" << fileName << "\" Center=\"Cell\">\n"
       << "    <DataItem Dimensions=\"" << rev << "\" Format=\"HDF\">\n     " << fileName << ".stoch.h5:/stochastic\n"
       << "    </DataItem>\n   </Attribute>\n  </Grid>\n </Domain>\n</Xdmf>" << std::endl;
}

// "<fileName>.stoch.h5": the field (dimension 0 fastest) as an IEEE F64LE dataset whose
// dimensions are the cells in reverse order (io.hh:203-225)
template <typename T>
void writeStochastic(const std::string& fileName, int dim, const unsigned* cells, const T* data) {
  std::vector<uint64_t> dims;
  for (int i = dim - 1; i >= 0; i--) dims.push_back(cells[i]);
  h5lite::write(fileName + ".stoch.h5", "stochastic", dims, data, 8);
}

// reads "<fileName>.stoch.h5" (stochastic.hh:86-103); the dataset must hold the cells
inline std::vector<double> readStochastic(const std::string& fileName, int dim, const unsigned* cells) {
  const std::string path = fileName + ".stoch.h5";
  {
    std::ifstream test(path);
    if (!test.good()) throw std::runtime_error{"File is missing: " + path};
  }
  std::vector<uint64_t> dims;
  std::vector<double> v = h5lite::read(path, "stochastic", &dims);
  bool match = (int)dims.size() == dim;
  for (int i = 0; match && i < dim; i++) match = dims[dim - 1 - i] == cells[i];
  if (!match) throw std::runtime_error{"field file " + path + " does not hold the configured cells"};
  return v;
}

}  // namespace parafields_b200
