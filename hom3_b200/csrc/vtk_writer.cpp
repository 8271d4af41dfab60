// vtk_writer.cpp -- host-side output of a solver's domain in hom3's legacy VTK
// format: Solver::write_domain (src/solver/fv/solver.hpp:328-376) through
// io::Vtk<nd, io::format::binary> (src/io/vtk.hpp:156-450).
//
// File layout (vtk.hpp:177-183, 239-338): an ASCII header, then POINTS (the
// unique cell vertices sorted by x, then y, then z; 2D points get z = 0),
// CELLS (2^nd vertex ids per cell, vertex order of child_rel_pos,
// grid/grid.hpp:41-59), CELL_TYPES (pixel 8 / voxel 11) and CELL_DATA: one
// SCALARS block per stream component.  Binary values are big-endian float32
// (Num) and int32 (Ind); an invalid Ind is written as -1 (vtk.hpp:363, 382-385).
// Cells are written in container order: internal cells, then ghosts.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "vtk_writer.hpp"

namespace h3c {
namespace {

// misc/math.hpp:291-292 (FloatingPoint::AlmostEquals: within 4 units in the last place)
bool almost_equal(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return false;
  auto biased = [](double x) {
    int64_t i;
    std::memcpy(&i, &x, sizeof i);
    const uint64_t u = (uint64_t)i;
    const uint64_t sign = 1ull << 63;
    return (u & sign) ? ~u + 1 : u | sign;
  };
  const uint64_t x = biased(a), y = biased(b);
  return (x >= y ? x - y : y - x) <= 4;
}

struct Out {
  FILE* f = nullptr;
  bool ok = true;
  void text(const std::string& s) { ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size(); }
  void be32(uint32_t u) {
    const unsigned char b[4] = {(unsigned char)(u >> 24), (unsigned char)(u >> 16), (unsigned char)(u >> 8),
                                (unsigned char)u};
    ok = ok && std::fwrite(b, 1, 4, f) == 4;
  }
  void num(double x) {  // static_cast<float>, byte-swapped (vtk.hpp:364, 375-378, 415-441)
    const float v = (float)x;
    uint32_t u;
    std::memcpy(&u, &v, 4);
    be32(u);
  }
  void id(int64_t x, int64_t invalid = INT64_MAX) {  // interpret_id (vtk.hpp:363, 382-385)
    be32((uint32_t)(int32_t)(x == invalid ? -1 : (int32_t)x));
  }
  void newline() { text("\n"); }
};

}  // namespace

int write_vtk_file(const VtkDomain& D, const std::vector<VtkStream>& streams, std::string* err) {
  const int nd = D.nd;
  const int64_t n = D.n_cells;
  const int nvert = 1 << nd;
  // cell vertices: x_c + h/2 child_rel_pos(v) (grid/grid.hpp:414-434, solver.hpp:761-775)
  std::vector<double> verts((size_t)n * nvert * 3, 0.0);
  for (int64_t c = 0; c < n; ++c) {
    const double hh = 0.5 * D.length[c];
    for (int v = 0; v < nvert; ++v)
      for (int d = 0; d < nd; ++d) {
        const int rel = ((v >> d) & 1) ? 1 : -1;
        verts[((size_t)c * nvert + v) * 3 + d] = D.x_center[d * D.ld + c] + hh * rel;
      }
  }
  // unique vertices in the order of vertex_cmp (x major, then y, then z; vtk.hpp:264-294)
  std::vector<int64_t> order((size_t)n * nvert);
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int64_t)i;
  auto key = [&](int64_t i, int d) { return verts[(size_t)i * 3 + d]; };
  auto less = [&](int64_t a, int64_t b) {
    for (int d = 0; d < nd; ++d) {
      const double x = key(a, d), y = key(b, d);
      if (almost_equal(x, y)) continue;
      return x < y;
    }
    return false;
  };
  std::stable_sort(order.begin(), order.end(), less);
  std::vector<int64_t> uid(order.size());
  std::vector<int64_t> uniq;
  for (size_t k = 0; k < order.size(); ++k) {
    const int64_t i = order[k];
    bool same = !uniq.empty();
    if (same)
      for (int d = 0; d < nd; ++d) same = same && almost_equal(key(i, d), key(uniq.back(), d));
    if (!same) uniq.push_back(i);
    uid[i] = (int64_t)uniq.size() - 1;
  }

  Out o;
  o.f = std::fopen(D.path.c_str(), "wb");
  if (!o.f) {
    if (err) *err = "cannot open " + D.path;
    return -1;
  }
  // header (vtk.hpp:177-183, 407-411)
  o.text("# vtk DataFile Version 2.0\n");
  o.text("HOM3 legacy vtk Output \n");
  o.text("BINARY\n");
  o.text("DATASET UNSTRUCTURED_GRID\n");
  // points (vtk.hpp:296-304)
  o.text("POINTS " + std::to_string(uniq.size()) + " FLOAT\n");
  for (const int64_t i : uniq) {
    for (int d = 0; d < nd; ++d) o.num(key(i, d));
    if (nd == 2) o.num(0.0);
  }
  o.newline();
  // cells (vtk.hpp:306-326)
  o.text("CELLS " + std::to_string(n) + " " + std::to_string(n * (nvert + 1)) + "\n");
  for (int64_t c = 0; c < n; ++c) {
    o.id(nvert);
    for (int v = 0; v < nvert; ++v) o.id(uid[(size_t)c * nvert + v]);
  }
  o.newline();
  // cell types (vtk.hpp:328-331): pixel 8, voxel 11
  o.text("CELL_TYPES " + std::to_string(n) + "\n");
  for (int64_t c = 0; c < n; ++c) o.id(nd == 2 ? 8 : 11);
  o.newline();
  // cell data (vtk.hpp:333-337, 201-237)
  o.text("CELL_DATA " + std::to_string(n) + "\n");
  for (const VtkStream& s : streams) {
    for (int k = 0; k < s.dims; ++k) {
      const std::string name = s.names.size() == (size_t)s.dims ? s.names[k]
                               : s.dims > 1 ? s.names[0] + "_" + std::to_string(k)
                                            : s.names[0];
      o.text("SCALARS " + name + (s.is_int ? " int" : " float") + "\n");
      o.text("LOOKUP_TABLE default\n");
      for (int64_t c = 0; c < n; ++c) {
        if (s.is_int) o.id(s.ints[(size_t)k * n + c]);
        else o.num(s.nums[(size_t)k * n + c]);
      }
      o.newline();
    }
  }
  const bool ok = o.ok && std::fclose(o.f) == 0;
  if (!ok && err) *err = "write error on " + D.path;
  return ok ? 0 : -1;
}

}  // namespace h3c
