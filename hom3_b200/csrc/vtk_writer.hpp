// vtk_writer.hpp -- legacy VTK output of a solver domain (host only).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace h3c {

// the cells to write, in the caller's (container) numbering
struct VtkDomain {
  std::string path;        // full file name
  int nd = 2;
  int64_t n_cells = 0;
  int64_t ld = 0;          // leading dimension of x_center
  const double* x_center;  // [nd][ld]
  const double* length;    // [n_cells]
};

// one stream of io::Vtk: dims components of int (Ind) or float (Num) values,
// stored [dims][n_cells]; names: one per component, or a base name that gets
// "_k" suffixes when dims > 1 (vtk.hpp:109-115)
struct VtkStream {
  std::vector<std::string> names;
  int dims = 1;
  bool is_int = false;
  std::vector<int64_t> ints;
  std::vector<double> nums;
};

int write_vtk_file(const VtkDomain& d, const std::vector<VtkStream>& streams, std::string* err);

}  // namespace h3c
