// hom3_b200.hpp -- C++ host layer over the C ABI (h3c.h), mirroring the
// surface of hom3's finite-volume Solver (src/solver/fv/solver.hpp:60-221)
// and its driver helpers (src/solver/fv/utilities.hpp:14-113), so a hom3
// driver reads the same:
//
//   hom3_b200::Grid grid{nd, rootMin, rootMax, level};          // grid::helpers::cube::properties
//   hom3_b200::Solver s{grid, props};                            // Solver(SolverIdx, io::Properties)
//   s.set_initial_condition([](const double* x, double* q) {..});
//   s.append_bcs(hom3_b200::cube_conditions(grid, cond));        // solver::fv::append_bcs
//   hom3_b200::run_solver(s, maxNoTimeSteps);                    // solver::fv::run_solver
//
// Errors: hom3 terminates the process (TERMINATE, misc/error.hpp:27-38); this
// layer throws hom3_b200::Error with the library's message instead.
#pragma once
#include <array>
#include <cmath>
#include <functional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "h3c.h"

namespace hom3_b200 {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, h3c_solver s = nullptr) {
  if (rc == H3C_OK) return;
  char buf[512];
  h3c_last_error(s, buf, sizeof(buf));
  throw Error(rc, std::string("h3c error ") + std::to_string(rc) + ": " + buf);
}

// Properties: the io::Properties keys hom3 reads on this path.
struct Properties {
  int physics = H3C_EULER, flux = H3C_FLUX_AUSM, time_integration = H3C_EULER_FORWARD, precision = H3C_FP64;
  double timeEnd = 1.0, CFL = 0.2, CFL_viscous = 0.4, gamma = 1.4, Rspecific = 287.058, T0 = 273.15,
         rho0 = 1.225, Minfty = 0.1, ReInfty = 100.0, Pr0 = 0.72, Sutherland0 = 110.4, diffusivity = 1.0,
         T_ref = 273.15;
  int domain_kind = 0;  // "initialDomain": 0 all, 1 sdf > 0, 2 sdf < 0
  h3c_sdf domain{};
  int reconstruction = H3C_RECON_NONE;  // EXTENSION: H3C_RECON_MUSCL
  double limiter_k = 1.0;               // Venkatakrishnan K
};

// Root cell + MinLevel generator (grid/helpers.hpp:163-179); refine: EXTENSION.
struct Grid {
  int nd;
  std::array<double, 3> xmin{}, xmax{};
  int level;
  std::vector<std::pair<std::array<double, 4>, int>> refine;  // {cx, cy, cz, r}, level
  h3c_grid_desc desc(const Properties& p, const std::vector<h3c_sdf>& geoms) const {
    h3c_grid_desc d{};
    d.nd = nd;
    for (int i = 0; i < 3; ++i) { d.xmin[i] = xmin[i]; d.xmax[i] = xmax[i]; }
    d.min_level = level;
    d.n_refine = (int)refine.size();
    for (size_t k = 0; k < refine.size() && k < 4; ++k) {
      for (int i = 0; i < 3; ++i) d.refine_center[k][i] = refine[k].first[i];
      d.refine_radius[k] = refine[k].first[3];
      d.refine_level[k] = refine[k].second;
    }
    d.domain_kind = p.domain_kind;
    d.domain = p.domain;
    d.n_bcs = (int)geoms.size();
    for (size_t i = 0; i < geoms.size() && i < 16; ++i) d.bc_geom[i] = geoms[i];
    return d;
  }
  double cell_length_at_level(int l) const {
    double L = 0;
    for (int i = 0; i < nd; ++i) L = std::max(L, xmax[i] - xmin[i]);
    return L / std::pow(2, l);
  }
};

// A boundary: geometry (signed distance) + condition (bc::Interface, boundary_condition.hpp:22-58).
struct Boundary {
  h3c_sdf geometry;
  h3c_bc condition;
};

inline h3c_bc condition(int kind, std::vector<double> v = {}) {
  h3c_bc c{};
  c.kind = kind;
  for (size_t i = 0; i < v.size() && i < 8; ++i) c.v[i] = v[i];
  return c;
}

// The 2nd cube faces with one condition each, in hom3's order (grid/helpers.hpp:112-160).
inline std::vector<Boundary> cube_boundaries(const Grid& g, const std::vector<h3c_bc>& conds) {
  h3c_sdf faces[6];
  const h3c_grid_desc d = g.desc(Properties{}, {});
  const int n = h3c_cube_boundaries(&d, faces);
  if (n < 0 || (int)conds.size() != n) throw Error(H3C_E_INVALID, "cube_boundaries: one condition per face");
  std::vector<Boundary> r;
  for (int i = 0; i < n; ++i) r.push_back({faces[i], conds[i]});
  return r;
}
inline std::vector<Boundary> cube_boundaries(const Grid& g, const h3c_bc& c) {
  return cube_boundaries(g, std::vector<h3c_bc>(2 * g.nd, c));
}

class Solver {
 public:
  using InitialCondition = std::function<void(const double* x, double* q)>;

  Solver(const Grid& grid, const Properties& p) : grid_(grid), props_(p) {
    h3c_desc d{};
    d.nd = grid.nd; d.physics = p.physics; d.flux = p.flux; d.time_integration = p.time_integration;
    d.precision = p.precision; d.time_end = p.timeEnd; d.cfl = p.CFL; d.cfl_viscous = p.CFL_viscous;
    d.gamma = p.gamma; d.Rspecific = p.Rspecific; d.T0 = p.T0; d.rho0 = p.rho0; d.Minfty = p.Minfty;
    d.ReInfty = p.ReInfty; d.Pr0 = p.Pr0; d.Sutherland0 = p.Sutherland0; d.diffusivity = p.diffusivity;
    d.T_ref = p.T_ref;
    d.reconstruction = p.reconstruction;
    d.limiter_k = p.limiter_k;
    nv_ = p.physics == H3C_HEAT ? 1 : grid.nd + 2;
    check(h3c_create(&d, &s_));
  }
  ~Solver() { if (s_) h3c_destroy(s_); }
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;

  // ---- input: solver.hpp:153-169 ----
  void set_initial_condition(InitialCondition ic) { ic_ = std::move(ic); }
  void append_bc(const Boundary& b) { bcs_.push_back(b); }
  void append_bcs(const std::vector<Boundary>& bs) { for (auto& b : bs) append_bc(b); }

  // ---- initialize: solver.hpp:133-138 (grid from the library's builder) ----
  void initialize() {
    std::vector<h3c_sdf> geoms;
    std::vector<h3c_bc> conds;
    for (auto& b : bcs_) { geoms.push_back(b.geometry); conds.push_back(b.condition); }
    const h3c_grid_desc gd = grid_.desc(props_, geoms);
    h3c_built_grid bg = nullptr;
    check(h3c_grid_build(&gd, &bg));
    h3c_grid v{};
    h3c_grid_view(bg, &v);
    v.n_bcs = (int)conds.size();
    v.bcs = conds.data();
    n_cells_ = v.n_cells;
    first_ghost_ = v.first_ghost;
    x_.assign(v.x_center, v.x_center + grid_.nd * v.n_cells);
    len_.assign(v.length, v.length + v.n_cells);
    const int rc = h3c_set_grid(s_, &v);
    h3c_grid_free(bg);
    check(rc, s_);
    // impose_initial_condition: 2^nd Gauss-point cell average (quadrature.hpp:43-74)
    lhs_.assign((size_t)nv_ * n_cells_, 0.0);
    if (ic_) {
      const double gp = 1 / std::sqrt(3);
      const int nd = grid_.nd;
      for (long long c = 0; c < first_ghost_; ++c) {
        const double l = len_[c];
        std::array<double, 5> sum{};
        for (int k = 0; k < (1 << nd); ++k) {
          double x[3] = {0, 0, 0};
          for (int d = 0; d < nd; ++d)
            x[d] = x_[d * n_cells_ + c] + 0.5 * l * ((((k >> d) & 1) ? 1.0 : -1.0) * gp);
          std::array<double, 5> q{};
          ic_(x, q.data());
          for (int v2 = 0; v2 < nv_; ++v2) sum[v2] = k == 0 ? q[v2] : sum[v2] + q[v2];
        }
        double vol = l;
        for (int d = 1; d < nd; ++d) vol = l * vol;
        for (int v2 = 0; v2 < nv_; ++v2) lhs_[v2 * n_cells_ + c] = sum[v2] * vol / (double)(1 << nd) / vol;
      }
    }
    check(h3c_set_state(s_, 0, lhs_.data(), n_cells_), s_);
    check(h3c_reset_time(s_), s_);
  }

  // ---- solver interface: solver.hpp:100-145 ----
  void solve() { check(h3c_solve(s_, 1), s_); }
  void solve(long long n) { check(h3c_solve(s_, n), s_); }
  double dt() const { double v; check(h3c_dt(s_, &v), s_); return v; }
  void dt(double forced) { check(h3c_force_dt(s_, forced), s_); }
  double min_dt() const { double v; check(h3c_min_dt(s_, &v), s_); return v; }
  double time() const { double v; check(h3c_time(s_, &v), s_); return v; }
  long long step() const { int64_t v; check(h3c_step(s_, &v), s_); return v; }
  double final_time() const { return props_.timeEnd; }

  // ---- data: Q<tag>() (solver.hpp:189-221), lhs = 0 / rhs = 1 ----
  const std::vector<double>& Q(int which = 0) {
    lhs_.resize((size_t)nv_ * n_cells_);
    check(h3c_get_state(s_, which, lhs_.data(), n_cells_), s_);
    return lhs_;
  }
  long long n_cells() const { return n_cells_; }
  long long first_ghost() const { return first_ghost_; }
  int nvars() const { return nv_; }
  const std::vector<double>& x_center() const { return x_; }
  h3c_solver handle() const { return s_; }

 private:
  Grid grid_;
  Properties props_;
  h3c_solver s_ = nullptr;
  int nv_ = 4;
  InitialCondition ic_;
  std::vector<Boundary> bcs_;
  long long n_cells_ = 0, first_ghost_ = 0;
  std::vector<double> x_, len_, lhs_;
};

// ---- driver helpers: utilities.hpp:61-113 ----
inline bool solver_finished(long long maxNoSteps, const Solver& s) {
  return s.time() >= s.final_time() || s.step() >= maxNoSteps;
}
inline bool solution_diverged(const Solver& s) {
  double dt = 0;
  const int rc = h3c_dt(s.handle(), &dt);
  if (rc == H3C_E_NONFINITE) return true;  // dt out of range or a cell failed the state check
  check(rc, s.handle());
  return dt < 1e-300 || dt > 1e300;
}
// run_solver without the VTK output: initialize, step until finished, and
// throw where hom3 would TERMINATE("Solution diverged!").
inline void run_solver(Solver& s, long long maxNoTimeSteps) {
  s.initialize();
  while (!solver_finished(maxNoTimeSteps, s)) {
    s.solve();
    if (solution_diverged(s)) throw Error(H3C_E_NONFINITE, "Solution diverged!");
  }
}

}  // namespace hom3_b200
