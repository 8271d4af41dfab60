// grid_build.hpp -- the built grid shared by the host builder (grid_build.cpp)
// and the device builder (grid_build_device.cu).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/h3c.h"

namespace gridb {

struct Cell {
  int level;
  long long i[3];
};

struct BuiltGrid {
  int nd = 2;
  long long n_int = 0, n_tot = 0, nsub = 0;
  std::vector<int64_t> nbr;      // [2nd][n_tot]
  std::vector<double> xc;        // [nd][n_tot]
  std::vector<double> len;       // [n_tot]
  std::vector<int32_t> bc;       // [n_tot]
  std::vector<int64_t> sub;      // [2^(nd-1)][nsub]
  std::vector<Cell> cells;       // interior + ghost cells (ghost: level/coords of its position)
  std::vector<h3c_bc> bcs;       // placeholders (conditions are given to h3c_set_grid)
};

// the message h3c_last_error(NULL) reports (defined with the solver's errors)
void set_global_error(const std::string& msg);

}  // namespace gridb

struct h3c_built_grid_s : gridb::BuiltGrid {};
