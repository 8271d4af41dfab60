// h3o.hpp -- CPU oracle for the hom3 finite-volume hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is a plain C++17 restatement of the
// algorithm in gnzlbg/hom3 (header-only C++14, uncompilable here: it needs
// Eigen3, Boost, MPI and HDF5).  It exists so that tests, the smoke check and
// the CPU baseline leg of the benchmark have something to compare the CUDA
// path against.  Nothing in the shipped library links, loads or calls it.
//
// Pinning: the tree / neighbour layer is pinned against hom3's own golden
// tables (src/containers/hierarchical/tests/hierarchical_container_test.cpp
// :43-49, :58-110, :112-173, :190-280), reproduced as fixtures under
// tests/golden.  hom3's solver tests are run-to-completion smoke tests with no
// numeric assertions (src/solver/fv/euler/tests/euler_fv_solver_test.cpp,
// cns/tests/cns_fv_solver_test.cpp, heat/tests/heat_fv_solver_test.cpp), so
// the finite-volume arithmetic below is pinned only by known-answer properties
// (free-stream preservation, conservation, exact Riemann solution, analytic
// vortex) -- FV parity is "unpinned by hom3's tests".
//
// Every function cites the hom3 file:line it restates (paths relative to the
// hom3 source tree).  Where hom3 relies on Eigen's reduction order or
// libc++'s unstable std::sort the restatement picks a fixed order and says so.
//
// Extensions that hom3 does not have are marked "EXTENSION (not in hom3)".
#pragma once
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <limits>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

namespace h3o {

using Ind = int64_t;
using SInd = int32_t;
constexpr Ind INV = std::numeric_limits<Ind>::max();    // misc/constants.hpp:42-43
constexpr SInd SINV = std::numeric_limits<SInd>::max();
constexpr double PI = 3.141592653589793238462643383279502884;  // misc/constants.hpp:67

// Forward-mode dual number (value, derivative) for the derivative build of the
// oracle (Solver<Dual>): every operation propagates d(x) by the chain rule;
// comparisons look at values only, so branches are those of the double build.
struct Dual {
  double v = 0, d = 0;
  Dual() {}
  Dual(double x) : v(x) {}
  Dual(double x, double y) : v(x), d(y) {}
};
inline Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
inline Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
inline Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
inline Dual operator/(Dual a, Dual b) { return {a.v / b.v, (a.d * b.v - a.v * b.d) / (b.v * b.v)}; }
inline Dual operator-(Dual a) { return {-a.v, -a.d}; }
inline Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
inline Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
inline Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
inline Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
inline Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
inline Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
inline Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
inline Dual operator/(double a, Dual b) { return {a / b.v, -a * b.d / (b.v * b.v)}; }
inline Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
#define H3O_DUAL_CMP(op)                                                  \
  inline bool operator op(Dual a, Dual b) { return a.v op b.v; }         \
  inline bool operator op(Dual a, double b) { return a.v op b; }         \
  inline bool operator op(double a, Dual b) { return a op b.v; }
H3O_DUAL_CMP(<) H3O_DUAL_CMP(>) H3O_DUAL_CMP(<=) H3O_DUAL_CMP(>=) H3O_DUAL_CMP(==) H3O_DUAL_CMP(!=)
#undef H3O_DUAL_CMP
inline Dual sqrt(Dual a) { const double r = std::sqrt(a.v); return {r, a.d / (2 * r)}; }
inline Dual abs(Dual a) { return a.v < 0 ? -a : a; }
inline Dual pow(Dual a, double e) { const double r = std::pow(a.v, e); return {r, e * std::pow(a.v, e - 1) * a.d}; }
inline double value(double x) { return x; }
inline double value(Dual x) { return x.v; }

// ---------------------------------------------------------------------------
// Stencils: grid/grid.hpp:41-81, containers/hierarchical/implementation.hpp:46-65
// ---------------------------------------------------------------------------
static const int child_rel_pos_2d[4][2] = {{-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
static const int child_rel_pos_3d[8][3] = {{-1, -1, -1}, {1, -1, -1}, {-1, 1, -1}, {1, 1, -1},
                                           {-1, -1, 1},  {1, -1, 1},  {-1, 1, 1},  {1, 1, 1}};
static const int nghbr_rel_pos_3d[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0},
                                           {0, 1, 0},  {0, 0, -1}, {0, 0, 1}};
constexpr SInd SI = SINV;
static const SInd rel_sibling[8][6] = {
    {SI, 1, SI, 2, SI, 4}, {0, SI, SI, 3, SI, 5}, {SI, 3, 0, SI, SI, 6}, {2, SI, 1, SI, SI, 7},
    {SI, 5, SI, 6, 0, SI}, {4, SI, SI, 7, 1, SI}, {SI, 7, 4, SI, 2, SI}, {6, SI, 5, SI, 3, SI}};
static const int opposite_pos[6] = {1, 0, 3, 2, 5, 4};

inline int child_rel(int nd, int c, int d) {
  return nd == 2 ? child_rel_pos_2d[c][d] : child_rel_pos_3d[c][d];
}

// ---------------------------------------------------------------------------
// Tree: containers/hierarchical/implementation.hpp + grid/grid.hpp
// ---------------------------------------------------------------------------
struct Tree {
  int nd;
  double rootLength;
  double rootCoords[3] = {0, 0, 0};
  std::vector<Ind> parent, firstChild;
  std::vector<std::vector<Ind>> node2cell;  // per solver (hierarchical/implementation.hpp:207-218)

  // RootCell ctor: grid/grid.hpp:108-132 (length starts at machine epsilon)
  Tree(int nd_, const double* xmin, const double* xmax, int maxSolvers) : nd(nd_) {
    rootLength = std::numeric_limits<double>::epsilon();
    for (int d = 0; d < nd; ++d) {
      const double lengthD = xmax[d] - xmin[d];
      rootLength = std::max(rootLength, lengthD);
      rootCoords[d] = xmin[d] + 0.5 * lengthD;
    }
    parent.push_back(INV);  // initialize_root_node_
    firstChild.push_back(INV);
    node2cell.assign(maxSolvers, std::vector<Ind>(1, INV));
  }
  Ind size() const { return (Ind)parent.size(); }
  int nchild() const { return 1 << nd; }
  int npos() const { return 2 * nd; }
  bool is_root(Ind n) const { return parent[n] == INV; }
  bool is_leaf(Ind n) const { return firstChild[n] == INV; }
  // child(): hierarchical/implementation.hpp:256-259.  For a leaf hom3 adds pos to the
  // invalid id (overflow); the intended meaning (no child) is used here.
  Ind child(Ind n, int pos) const { return firstChild[n] == INV ? INV : firstChild[n] + pos; }
  // position_in_parent: hierarchical/implementation.hpp:271-280
  int pos_in_parent(Ind n) const { return (int)(n - firstChild[parent[n]]); }
  // level: hierarchical/implementation.hpp:427-441
  int level(Ind n) const {
    int l = 0;
    n = parent[n];
    while (n != INV) { n = parent[n]; ++l; }
    return l;
  }
  // refine_node: hierarchical/implementation.hpp:320-364 (compact tree -> children appended)
  Ind refine(Ind n) {
    const Ind first = size();
    firstChild[n] = first;
    for (int c = 0; c < nchild(); ++c) {
      parent.push_back(n);
      firstChild.push_back(INV);
      for (auto& m : node2cell) m.push_back(INV);
    }
    return first;
  }
  // MinLevel::generate_mesh: grid/generation.hpp:45-59.  The node range is
  // fixed at the start of each pass (Range{node_begin, node_end}).
  void min_level(int L) {
    bool done = false;
    while (!done) {
      done = true;
      const Ind end = size();
      for (Ind n = 0; n < end; ++n) {
        if (is_leaf(n) && level(n) != L) { refine(n); done = false; }
      }
    }
  }
  // find_samelvl_neighbor: hierarchical/implementation.hpp:457-543
  Ind find_samelvl_neighbor(Ind n, int pos) const {
    if (is_root(n)) return INV;
    std::vector<int> traversed;
    Ind cur = n;
    while (true) {
      const Ind p = parent[cur];
      const int pip = pos_in_parent(cur);
      if (rel_sibling[pip][pos] != SINV) break;
      if (is_root(p)) return INV;
      traversed.push_back(pip);
      cur = p;
    }
    cur = child(parent[cur], rel_sibling[pos_in_parent(cur)][pos]);
    for (auto it = traversed.rbegin(); it != traversed.rend(); ++it) {
      const int ncp = rel_sibling[*it][opposite_pos[pos]];
      const Ind nxt = child(cur, ncp);
      if (nxt == INV) return INV;
      cur = nxt;
    }
    return cur;
  }
  // cell_length_at_level / cell_length: grid/grid.hpp:344-351
  double length_at_level(int l) const { return rootLength / std::pow(2, l); }
  double length(Ind n) const { return length_at_level(level(n)); }
  // cell_coordinates: grid/grid.hpp:358-374 (recursive from the root)
  void coords(Ind n, double* x) const {
    if (level(n) != 0) {
      const Ind p = parent[n];
      const int pip = pos_in_parent(n);
      const double rel = 0.25 * length(p);
      double xp[3];
      coords(p, xp);
      for (int d = 0; d < nd; ++d) x[d] = xp[d] + (double)child_rel(nd, pip, d) * rel;
    } else {
      for (int d = 0; d < nd; ++d) x[d] = rootCoords[d];
    }
  }
  // neighbor_coordinates: grid/grid.hpp:379-390
  void neighbor_coords(Ind n, int pos, double* x) const {
    double xn[3];
    coords(n, xn);
    const double l = length(n);
    for (int d = 0; d < nd; ++d) x[d] = xn[d] + (double)nghbr_rel_pos_3d[pos][d] * l;
  }
  std::vector<Ind> leaf_nodes() const {
    std::vector<Ind> r;
    for (Ind n = 0; n < size(); ++n)
      if (is_leaf(n)) r.push_back(n);
    return r;
  }

  // EXTENSION (not in hom3): refine leaves whose cell box intersects a sphere
  // until they reach `maxLevel`, then enforce the 2:1 face balance that
  // find_samelvl_neighbor's documentation requires (hierarchical/implementation.hpp:456).
  void refine_sphere(const double* c, double r, int maxLevel);
  void balance_2to1();
};

// ---------------------------------------------------------------------------
// Signed distance functions: geometry/implicit.hpp:39-132
// Convention: > 0 outside, < 0 inside.
// ---------------------------------------------------------------------------
enum SdfKind { SDF_NONE = 0, SDF_EDGE = 1, SDF_SQUARE = 2, SDF_SPHERE = 3 };
struct Sdf {
  int kind = SDF_NONE;
  int inverted = 0;
  double p[6] = {0, 0, 0, 0, 0, 0};
  double operator()(int nd, const double* x) const {
    double r = 0;
    if (kind == SDF_EDGE) {  // implicit.hpp:91-103: normal . (x - point)
      for (int d = 0; d < nd; ++d) r += p[3 + d] * (x[d] - p[d]);
    } else if (kind == SDF_SQUARE) {  // implicit.hpp:52-85
      double dist[3];
      for (int d = 0; d < nd; ++d) dist[d] = p[d] - 0.5 * p[3 + d] - x[d];
      for (int d = 0; d < nd; ++d)
        if (x[d] > p[d]) dist[d] = x[d] - (p[d] + 0.5 * p[3 + d]);
      int npos = 0;
      for (int d = 0; d < nd; ++d) npos += dist[d] > 0;
      if (npos == nd) {
        double s = 0;
        for (int d = 0; d < nd; ++d) s += dist[d] * dist[d];
        r = std::sqrt(s);
      } else if (npos < 2) {
        r = dist[0];
        for (int d = 1; d < nd; ++d) r = std::max(r, dist[d]);
      } else {  // nd == 3, two positive: distance to an edge
        if (dist[0] < 0) r = std::sqrt(std::pow(dist[1], 2) + std::pow(dist[2], 2));
        else if (dist[1] < 0) r = std::sqrt(std::pow(dist[0], 2) + std::pow(dist[2], 2));
        else r = std::sqrt(std::pow(dist[0], 2) + std::pow(dist[1], 2));
      }
    } else if (kind == SDF_SPHERE) {  // implicit.hpp:39-46
      double s = 0;
      for (int d = 0; d < nd; ++d) s += (x[d] - p[d]) * (x[d] - p[d]);
      r = std::sqrt(s) - p[3];
    }
    return inverted ? -1. * r : r;  // adaptors::Inverted, implicit.hpp:119-127
  }
};

// is_cut_by: grid/grid.hpp:601-626 (cell vertices from child_rel_pos)
inline bool is_cut_by(int nd, const double* xc, double len, const Sdf& sdf) {
  const double h = 0.5 * len;
  bool allPos = true, allNeg = true;
  for (int v = 0; v < (1 << nd); ++v) {
    double x[3];
    for (int d = 0; d < nd; ++d) x[d] = xc[d] + h * (double)child_rel(nd, v, d);
    const double s = sdf(nd, x);
    allPos = allPos && (s > 0);
    allNeg = allNeg && (s < 0);
  }
  return !(allPos || allNeg);
}

// make_boundaries: grid/helpers.hpp:112-160 (left,right,bottom,top,front,back)
inline std::vector<Sdf> cube_boundaries(int nd, const Tree& t) {
  const double length = t.rootLength;
  const double eps = length * 1e-15;
  const double x_max = t.rootCoords[0] + 0.5 * length - eps;
  const double x_min = t.rootCoords[0] - 0.5 * length + eps;
  const double off = x_min + 0.5 * length;
  std::vector<Sdf> r;
  for (int d = 0; d < nd; ++d) {
    for (int side = 0; side < 2; ++side) {
      Sdf s;
      s.kind = SDF_EDGE;
      for (int k = 0; k < nd; ++k) { s.p[k] = off; s.p[3 + k] = 0.0; }
      s.p[d] = side == 0 ? x_min : x_max;
      s.p[3 + d] = side == 0 ? +1.0 : -1.0;  // edge::n(neg)=+1, n(pos)=-1
      r.push_back(s);
    }
  }
  return r;
}

// ---------------------------------------------------------------------------
// Physical parameters: euler/quantities.hpp:23-189, cns/quantities.hpp:23-115,
// heat/quantities.hpp:13-56
// ---------------------------------------------------------------------------
enum PhysicsKind { PHYS_EULER = 0, PHYS_CNS = 1, PHYS_HEAT = 2, PHYS_ADVECTION = 3 /* advection/physics.hpp:21-149 */ };
enum FluxKind { FLUX_AUSM = 0, FLUX_LLF = 1, FLUX_UPWIND = 2 /* advection/tags.hpp:14-15 */ };
// Advection velocity fields u(x) (the "velocity" property, advection/physics.hpp:36-37)
enum VelocityKind {
  VEL_CONSTANT = 0,  // vel = {u_0, u_1, u_2}
  VEL_ROTATION = 1,  // advection_fv_solver_test.cpp:69-85 (radial_velocity); vel = {u_mag, c_0, c_1}
};
enum TimeKind { TI_EULER_FORWARD = 0, TI_RK2 = 1, TI_SSPRK3 = 2 /* EXTENSION: Shu-Osher SSP-RK3 */ };
enum ReconKind { RECON_NONE = 0, RECON_MUSCL = 1 /* EXTENSION: LSQ + MUSCL + Venkatakrishnan */ };

struct Params {
  int physics = PHYS_EULER, flux = FLUX_AUSM, ti = TI_EULER_FORWARD;
  int recon = RECON_NONE;
  double limiter_k = 1.0;  // Venkatakrishnan: eps^2 = (limiter_k h)^3
  double cfl = 0.2, cfl_viscous = 0.4;
  double gamma = 1.4, Rspecific = 287.058, T0 = 273.15, rho0 = 1.225, Minfty = 0.1;
  double ReInfty = 100, Pr0 = 0.72, Sutherland0 = 110.4;
  double diffusivity = 1.0, T_ref = 273.15;
  int vel_kind = VEL_CONSTANT;  // advection velocity field
  double vel[4] = {0, 0, 0, 0};
  double time_end = 1.0;
  // derived
  double gm1 = 0.4, sOverTref = 0, sOverTrefP1 = 1, Re0 = 1;
  double T_inf = 1, rho_inf = 1, u_inf = 0, p_inf = 1, mu_inf = 1;
  void derive() {
    gm1 = gamma - 1.;
    T_inf = 1.0 / (1 + 0.5 * gm1 * (Minfty * Minfty));  // euler/quantities.hpp:132-133
    rho_inf = std::pow(T_inf, 1. / gm1);               // :136-137
    u_inf = Minfty * std::sqrt(T_inf);                 // :140-141
    p_inf = std::pow(T_inf, gamma / gm1) / gamma;      // :144-145
    sOverTref = Sutherland0 / T0;                      // cns/quantities.hpp:28
    sOverTrefP1 = sOverTref + 1.0;                     // :29
    mu_inf = sutherland(T_inf);                        // :74-75
    Re0 = ReInfty * mu_inf / (rho_inf * u_inf);        // :30
  }
  // cns/quantities.hpp:113-115
  double sutherland(double T) const { return std::pow(T, 1.5) * sOverTrefP1 / (T + sOverTref); }
};

// ---------------------------------------------------------------------------
// Boundary / coupling conditions (kinds shared by all physics)
// ---------------------------------------------------------------------------
enum BcKind {
  BC_EULER_NEUMANN = 0,        // euler/boundary_conditions.hpp:17-43 (constant surface flux)
  BC_EULER_DIRICHLET = 1,      // :47-67 (constant surface state)
  BC_EULER_VORTEX = 2,         // :71-93
  BC_CNS_INFLOW = 3,           // cns/boundary_conditions.hpp:28-65
  BC_CNS_OUTFLOW = 4,          // :72-105
  BC_CNS_ADIABATIC_NOSLIP = 5, // :117-150
  BC_CNS_ADIABATIC_SLIP = 6,   // :157-193
  BC_CNS_ISOTHERMAL_NOSLIP = 7,// :200-238
  BC_HEAT_DIRICHLET = 8,       // heat/boundary_conditions.hpp:15-37
  BC_HEAT_NEUMANN = 9,         // :40-63
  BC_CPL_EULER_EULER = 10,     // euler/coupling_conditions.hpp:17-35
  BC_CPL_CNS_HEAT = 11,        // cns/coupling_conditions.hpp:22-43 (CNS side)
  BC_CPL_HEAT_CNS = 12,        // heat/coupling_conditions.hpp:18-38 (heat side)
  BC_CPL_HEAT_HEAT = 13,       // heat/coupling_conditions.hpp:41-61
  BC_PERIODIC = 14,            // EXTENSION (not in hom3): copy of the cell on the opposite face
  BC_ADV_DIRICHLET = 15,       // advection/boundary_conditions.hpp:15-37 (constant surface value)
  BC_ADV_NEUMANN = 16,         // :40-63 (constant surface flux)
  BC_ADV_CHARACTERISTIC = 17,  // :66-94
};

struct Bc {
  int kind = BC_EULER_NEUMANN;
  Sdf geom;
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int partner = -1;  // solver index of the coupled solver
};

// Initial conditions (cell averages by 2^nd Gauss points)
enum IcKind {
  IC_CONSTANT_PV = 0,   // constant primitive state (tests' constant_ic lambdas)
  IC_SHOCK_TUBE = 1,    // euler/initial_conditions.hpp:51-90
  IC_VORTEX = 2,        // euler/initial_conditions.hpp:14-39 (2D)
  IC_EXPLOSION = 3,     // euler_fv_solver_test.cpp:222-245
  IC_CONSTANT_CV = 4,   // constant conservative state (heat: T)
  IC_RIEMANN3D_PERTURBED = 5,  // EXTENSION (not in hom3): 3D Riemann + Fourier modes
  IC_VORTEX_PARAM = 6,  // EXTENSION (not in hom3): vortex with centre/strength params
  IC_TAYLOR_GREEN = 7,  // EXTENSION (not in hom3): 3D Taylor-Green vortex
  IC_DISC = 8,          // advection_fv_solver_test.cpp:106-115: q_in inside a disc, q_out outside
};

template <class T> struct World;

// ---------------------------------------------------------------------------
// Solver: solver/fv/solver.hpp:60-994 with the physics of euler/, cns/, heat/
// ---------------------------------------------------------------------------
template <class T> struct Solver {
  using State = std::array<T, 5>;
  using ICState = std::array<double, 5>;  // initial conditions are evaluated in double
  World<T>* w = nullptr;
  int idx = 0;
  int nd = 2, nv = 4;
  Params P;
  std::vector<Bc> bcs;
  // domain predicate: 0 all, 1 sdf > 0, 2 sdf < 0
  int domain_kind = 0;
  Sdf domain;
  int ic_kind = IC_CONSTANT_PV;
  double ic[80] = {0};
  // Container columns: container.hpp:58-66
  std::vector<T> Q[3][5];  // lhs, rhs, and the second SSP-RK3 stage
  std::vector<Ind> nbr[6];
  std::vector<double> xc[3];
  std::vector<double> len;
  std::vector<double> vel_[3];  // advection velocity u(x_center) of every cell, ghosts included
  std::vector<SInd> bc_idx;
  std::vector<Ind> node;
  Ind firstGC = INV;
  // EXTENSION (not in hom3): coarse/fine sub-face groups of 2:1 balanced
  // trees.  nbr < -1 encodes group k = -nbr - 2 whose 2^(nd-1) finer cells are
  // subs[k * 2^(nd-1) + j], j in increasing child position.
  std::vector<Ind> subs;
  // EXTENSION: interior cell paired with each periodic ghost (index g - firstGC)
  std::vector<Ind> periodic_partner;
  // numerical data: solver.hpp:406-416
  T dt_ = 0;
  double time_ = 0, tEnd_ = 0;
  Ind step_ = 0;
  T forced_dt_ = 0;
  Ind forced_step_ = INV;

  Ind size() const { return (Ind)len.size(); }
  Ind n_internal() const { return firstGC == INV ? size() : firstGC; }
  int rho_i() const { return nd; }
  int E_i() const { return nd + 1; }
  T& q(int t, Ind c, int v) { return Q[t][v][c]; }
  const T& q(int t, Ind c, int v) const { return Q[t][v][c]; }
  bool is_ghost(Ind c) const { return node[c] == INV; }

  Ind push_cell() {
    for (int t = 0; t < 3; ++t)
      for (int v = 0; v < nv; ++v) Q[t][v].push_back(T(std::numeric_limits<double>::quiet_NaN()));
    for (int p = 0; p < 2 * nd; ++p) nbr[p].push_back(INV);
    for (int d = 0; d < nd; ++d) xc[d].push_back(std::numeric_limits<double>::quiet_NaN());
    len.push_back(std::numeric_limits<double>::quiet_NaN());
    bc_idx.push_back(SINV);
    node.push_back(INV);
    return size() - 1;
  }

  // ---- primitive helpers: euler/physics.hpp:83-149 ----
  T rho(int t, Ind c) const { return q(t, c, nd); }
  T rho_u(int t, Ind c, int d) const { return q(t, c, d); }
  T rho_E(int t, Ind c) const { return q(t, c, nd + 1); }
  T u(int t, Ind c, int d) const { return rho_u(t, c, d) / rho(t, c); }
  T u_mag2(int t, Ind c) const {  // squaredNorm; summation order fixed left to right
    T s = u(t, c, 0) * u(t, c, 0);
    for (int d = 1; d < nd; ++d) s = s + u(t, c, d) * u(t, c, d);
    return s;
  }
  T p(int t, Ind c) const { return P.gm1 * (rho_E(t, c) - 0.5 * rho(t, c) * u_mag2(t, c)); }
  T a(int t, Ind c) const { using std::sqrt; return sqrt(P.gamma * p(t, c) / rho(t, c)); }
  T Temp(int t, Ind c) const {  // euler T: euler/physics.hpp:144-145; heat T: heat/physics.hpp:51-58
    if (P.physics == PHYS_HEAT) return q(t, c, 0);
    return P.gamma * p(t, c) / rho(t, c);
  }
  // cv / pv: euler/quantities.hpp:153-189
  template <class S> S cv(const S& pvs) const {
    S c{};
    c[nd] = pvs[nd];
    typename S::value_type velMag2 = 0;
    for (int d = 0; d < nd; ++d) {
      c[d] = pvs[nd] * pvs[d];
      velMag2 = velMag2 + pvs[d] * pvs[d];
    }
    c[nd + 1] = pvs[nd + 1] / (P.gamma - 1.0) + 0.5 * pvs[nd] * velMag2;
    return c;
  }
  State pv(const State& cvs) const {
    State r{};
    r[nd] = cvs[nd];
    T velMag2 = 0;
    for (int d = 0; d < nd; ++d) {
      r[d] = cvs[d] / cvs[nd];
      velMag2 = velMag2 + r[d] * r[d];
    }
    r[nd + 1] = (P.gamma - 1.0) * (cvs[nd + 1] - 0.5 * cvs[nd] * velMag2);
    return r;
  }
  State Qrow(int t, Ind c) const {
    State s{};
    for (int v = 0; v < nv; ++v) s[v] = q(t, c, v);
    return s;
  }
  void setQ(int t, Ind c, const State& s) {
    for (int v = 0; v < nv; ++v) q(t, c, v) = s[v];
  }

  // ---- numerical fluxes ----
  // Euler flux: euler/physics.hpp:98-113
  State euler_flux(int t, Ind c, int d) const {
    State f{};
    f[nd] = rho_u(t, c, d);
    for (int i = 0; i < nd; ++i) f[i] = rho_u(t, c, i) * u(t, c, d);
    f[d] = f[d] + p(t, c);
    f[nd + 1] = u(t, c, d) * (rho_E(t, c) + p(t, c));
    return f;
  }
  // m_int_, p_int_: euler/physics.hpp:297-310
  static T m_int(int s, T M) {
    using std::abs;
    const double sd = (double)s;
    return abs(M) > 1 ? T(0.5 * (M + sd * abs(M))) : T((sd * 0.25) * ((M + sd) * (M + sd)));
  }
  static T p_int(int s, T M) {
    using std::abs;
    const double sd = (double)s;
    return abs(M) > 1 ? T(0.5 * (M + sd * abs(M)) / M) : T(0.25 * ((M + sd) * (M + sd)) * (2. - sd * M));
  }
  // theta_: euler/physics.hpp:315-325
  State theta(int t, Ind c) const {
    State f{};
    f[nd] = rho(t, c);
    for (int i = 0; i < nd; ++i) f[i] = rho_u(t, c, i);
    f[nd + 1] = rho_E(t, c) + p(t, c);
    const T ac = a(t, c);
    for (int v = 0; v < nv; ++v) f[v] = f[v] * ac;
    return f;
  }
  // AUSM: euler/physics.hpp:276-293
  State ausm(int t, Ind l, Ind r, int d) const {
    const T ML = u(t, l, d) / a(t, l);
    const T MR = u(t, r, d) / a(t, r);
    const T m_i = m_int(+1, ML) + m_int(-1, MR);
    const T p_i = p_int(+1, ML) * p(t, l) + p_int(-1, MR) * p(t, r);
    State f = m_i >= 0 ? theta(t, l) : theta(t, r);
    for (int v = 0; v < nv; ++v) f[v] = f[v] * m_i;
    f[d] = f[d] + p_i;
    return f;
  }
  // LLF: euler/physics.hpp:262-267
  State llf(int t, Ind l, Ind r, int d, double dx, T dt) const {
    const State fl = euler_flux(t, l, d), fr = euler_flux(t, r, d);
    State f{};
    const T k = dx / dt;
    for (int v = 0; v < nv; ++v) f[v] = 0.5 * ((fl[v] + fr[v]) + k * (q(t, l, v) - q(t, r, v)));
    return f;
  }

  // slope: solver.hpp:596-623
  T slope(int t, Ind c, int v, int dir) const {
    const Ind m = nbr[2 * dir][c], pp = nbr[2 * dir + 1][c];
    if (m != INV && pp != INV) return (q(t, pp, v) - q(t, m, v)) / (2. * len[c]);
    if (m != INV) return slope(t, m, v, dir);
    if (pp != INV) return slope(t, pp, v, dir);
    // EXTENSION: a periodic ghost takes the slope of its paired interior cell
    if (bcs[bc_idx[c]].kind == BC_PERIODIC) return slope(t, periodic_partner[c - firstGC], v, dir);
    // ghost cell: BC slope of its boundary cell (boundary_condition.hpp:45-67)
    const Ind b = boundary_cell(c);
    const T s = slope(t, b, v, dir);
    const int k = bcs[bc_idx[c]].kind;
    const bool wall = k == BC_CNS_ADIABATIC_NOSLIP || k == BC_CNS_ISOTHERMAL_NOSLIP ||
                      k == BC_CPL_CNS_HEAT;  // cns/boundary_conditions.hpp:143-147, 230-234
    return (wall && v < nd) ? T(-s) : s;
  }
  // surface_slope: solver.hpp:656-678 (l,r are neighbours along `ndir`)
  T surface_slope(int t, Ind l, Ind r, int ndir, int v, int sdir) const {
    if (ndir == sdir) return (q(t, r, v) - q(t, l, v)) / len[r];
    return 0.5 * (slope(t, r, v, sdir) + slope(t, l, v, sdir));
  }
  // boundary_info: solver.hpp:298-313
  // the "velocity" function of the advection physics at x (advection/physics.hpp:35-37, 104-106)
  void velocity_field(const double* x, double* u) const {
    for (int d = 0; d < 3; ++d) u[d] = 0;
    if (P.vel_kind == VEL_CONSTANT) {
      for (int d = 0; d < nd; ++d) u[d] = P.vel[d];
      return;
    }
    // radial_velocity of advection_fv_solver_test.cpp:69-85 (2D), centre and magnitude as parameters
    const double u_mag = P.vel[0];
    const double c0 = P.vel[1], c1 = P.vel[2];
    const double radius = std::sqrt((x[0] - c0) * (x[0] - c0) + (x[1] - c1) * (x[1] - c1));
    const double angle = 0.5 * PI - std::acos((x[0] - c0) / radius);
    u[0] = std::abs(radius * u_mag * std::sin(angle + 0.5 * PI));
    u[1] = std::abs(radius * u_mag * std::cos(angle + 0.5 * PI));
    if (x[1] - c1 > 0.) u[0] *= -1;
    if (x[0] - c0 < 0.) u[1] *= -1;
  }
  void compute_velocity() {
    for (int d = 0; d < 3; ++d) vel_[d].assign(size(), 0.0);
    if (P.physics != PHYS_ADVECTION) return;
    for (Ind c = 0; c < size(); ++c) {
      double x[3] = {0, 0, 0}, u[3];
      for (int d = 0; d < nd; ++d) x[d] = xc[d][c];
      velocity_field(x, u);
      for (int d = 0; d < nd; ++d) vel_[d][c] = u[d];
    }
  }
  double velocity(Ind c, int d) const { return vel_[d][c]; }

  Ind boundary_cell(Ind g) const {
    for (int p = 0; p < 2 * nd; ++p)
      if (nbr[p][g] != INV) return nbr[p][g];
    return INV;
  }
  int boundary_pos(Ind g) const {  // position of the boundary cell w.r.t. the ghost
    for (int p = 0; p < 2 * nd; ++p)
      if (nbr[p][g] != INV) return p;
    return -1;
  }

  // CNS viscous flux: cns/physics.hpp:305-338 with the *_srfc helpers :221-293
  State viscous(int t, Ind l, Ind r, int dir) const {
    State f{};
    const T rho_s = 0.5 * (rho(t, l) + rho(t, r));
    auto rho_u_s = [&](int d) { return T(0.5 * (rho_u(t, l, d) + rho_u(t, r, d))); };
    const T rho_E_s = 0.5 * (rho_E(t, l) + rho_E(t, r));
    auto u_s = [&](int d) { return T(rho_u_s(d) / rho_s); };
    T umag2 = 0;
    for (int d = 0; d < nd; ++d) umag2 = umag2 + u_s(d) * u_s(d);
    const T p_s = P.gm1 * (rho_E_s - 0.5 * rho_s * umag2);
    auto grad_rho = [&](int d) { return surface_slope(t, l, r, dir, nd, d); };
    auto grad_rho_u = [&](int c, int d) { return surface_slope(t, l, r, dir, c, d); };
    auto grad_rho_E = [&](int d) { return surface_slope(t, l, r, dir, nd + 1, d); };
    auto grad_u = [&](int c, int d) {
      return T((grad_rho_u(c, d) * rho_s - grad_rho(d) * rho_u_s(c)) / (rho_s * rho_s));
    };
    // mu at the surface from averaged p and rho: cns/physics.hpp:311-314
    const T p_avg = 0.5 * (p(t, l) + p(t, r));
    const T r_avg = 0.5 * (rho(t, l) + rho(t, r));
    const T mu_s = sutherland(P.gamma * p_avg / r_avg);
    // grad_p_srfc: :282-293
    T grad_rho_umag2 = grad_rho(dir) * umag2;
    for (int d = 0; d < nd; ++d) grad_rho_umag2 = grad_rho_umag2 + rho_s * 2. * u_s(d) * grad_u(d, dir);
    const T gradP = P.gm1 * (grad_rho_E(dir) - 0.5 * grad_rho_umag2);
    const T gradRho = grad_rho(dir);
    // heat_flux: :101-105
    const T qf = -mu_s * P.gamma / (P.gm1 * P.Pr0 * rho_s) * (gradP - p_s / rho_s * gradRho);
    // shear_stress: :110-123, nabla_u(i,j) = grad_u(j, i)
    T nab[3][3];
    for (int i = 0; i < nd; ++i)
      for (int j = 0; j < nd; ++j) nab[i][j] = grad_u(j, i);
    T tr = nab[0][0];
    for (int i = 1; i < nd; ++i) tr = tr + nab[i][i];
    const T div_u = tr * 2. / 3.;
    T Eacc = 0;
    for (int k = 0; k < nd; ++k) {
      // tau(k, dir) = -mu * (nab(k,dir) + nab(dir,k) - div_u * I(k,dir))
      const T tkd = -mu_s * ((nab[k][dir] + nab[dir][k]) - div_u * (k == dir ? 1. : 0.));
      f[k] = 1. / P.Re0 * tkd;
      Eacc = Eacc + u_s(k) * tkd;
    }
    f[nd + 1] = 1. / P.Re0 * (Eacc + qf);
    return f;
  }
  T sutherland(T Tt) const { using std::pow; return pow(Tt, 1.5) * P.sOverTrefP1 / (Tt + P.sOverTref); }

  // ---- EXTENSION (not in hom3): second-order MUSCL reconstruction ----
  // Primitive variables w = (u_0..u_{nd-1}, rho, p) (velocity in the momentum
  // slots).  Per interior cell: least-squares gradient over the face
  // neighbours (same-level, coarser, the finer cells of a sub-face group and
  // ghosts at their mirrored centres), weights 1/|dx|^2, normal equations
  // solved by the adjugate; then Venkatakrishnan's limiter per variable,
  // psi = min(1, min over faces phi), eps^2 = (K h)^3.  Ghost cells carry no
  // gradient (first order on the ghost side) except periodic ghosts, which
  // take their paired cell's.  A face uses one point for both sides: on the
  // face plane (from the minus-side cell), transverse coordinates of the
  // smaller cell.  A face whose reconstructed density or pressure is not
  // positive on either side falls back to the cell values.
  std::vector<T> Wg[5][3];  // limited gradients [v][d] per cell
  using WState = std::array<T, 5>;
  WState prim_w(int t, Ind c) const {
    WState w{};
    for (int d = 0; d < nd; ++d) w[d] = u(t, c, d);
    w[nd] = rho(t, c);
    w[nd + 1] = p(t, c);
    return w;
  }
  // the face neighbours of interior cell c: f(n, d, side), side -1 / +1
  template <class F> void for_each_face(Ind c, F f) const {
    const int ns = 1 << (nd - 1);
    for (int d = 0; d < nd; ++d)
      for (int sd = 0; sd < 2; ++sd) {
        const Ind n = nbr[2 * d + sd][c];
        const int side = sd == 0 ? -1 : 1;
        if (n >= 0) f(n, d, side);
        else
          for (int j = 0; j < ns; ++j) f(subs[(-n - 2) * ns + j], d, side);
      }
  }
  // the face point of the face between L (minus side) and R along d
  void face_point(Ind L, Ind R, int d, double* xf) const {
    const Ind sm = len[R] < len[L] ? R : L;
    for (int k = 0; k < nd; ++k) xf[k] = xc[k][sm];
    xf[d] = xc[d][L] + 0.5 * len[L];
  }
  static T vk_phi(T a, T b, T e2) {
    return ((a * a + e2) * b + 2. * b * b * a) / (b * (a * a + 2. * b * b + a * b + e2));
  }
  void compute_gradients(int t) {
    const Ind n = n_internal();
    for (int v = 0; v < 5; ++v)
      for (int d = 0; d < 3; ++d) Wg[v][d].assign(size(), T(0));
#pragma omp parallel for schedule(static)
    for (Ind c = 0; c < n; ++c) {
      const WState wc = prim_w(t, c);
      T M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
      T b[5][3] = {};
      WState wmax = wc, wmin = wc;
      for_each_face(c, [&](Ind nb, int, int) {
        const WState wn = prim_w(t, nb);
        double dx[3];
        double r2 = 0;
        for (int k = 0; k < nd; ++k) {
          dx[k] = xc[k][nb] - xc[k][c];
          r2 = k == 0 ? dx[k] * dx[k] : r2 + dx[k] * dx[k];
        }
        const double wgt = 1.0 / r2;
        for (int i = 0; i < nd; ++i)
          for (int j = 0; j < nd; ++j) M[i][j] = M[i][j] + (wgt * dx[i]) * dx[j];
        for (int v = 0; v < nv; ++v) {
          const T dw = wn[v] - wc[v];
          for (int i = 0; i < nd; ++i) b[v][i] = b[v][i] + (wgt * dx[i]) * dw;
          wmax[v] = wn[v] > wmax[v] ? wn[v] : wmax[v];
          wmin[v] = wn[v] < wmin[v] ? wn[v] : wmin[v];
        }
      });
      // adjugate inverse of the symmetric normal matrix
      T inv[3][3];
      if (nd == 2) {
        const T id = 1.0 / (M[0][0] * M[1][1] - M[0][1] * M[1][0]);
        inv[0][0] = M[1][1] * id;
        inv[1][1] = M[0][0] * id;
        inv[0][1] = -M[0][1] * id;
        inv[1][0] = -M[1][0] * id;
      } else {
        const T c00 = M[1][1] * M[2][2] - M[1][2] * M[2][1];
        const T c01 = M[1][2] * M[2][0] - M[1][0] * M[2][2];
        const T c02 = M[1][0] * M[2][1] - M[1][1] * M[2][0];
        const T id = 1.0 / (M[0][0] * c00 + M[0][1] * c01 + M[0][2] * c02);
        inv[0][0] = c00 * id;
        inv[0][1] = (M[0][2] * M[2][1] - M[0][1] * M[2][2]) * id;
        inv[0][2] = (M[0][1] * M[1][2] - M[0][2] * M[1][1]) * id;
        inv[1][0] = c01 * id;
        inv[1][1] = (M[0][0] * M[2][2] - M[0][2] * M[2][0]) * id;
        inv[1][2] = (M[0][2] * M[1][0] - M[0][0] * M[1][2]) * id;
        inv[2][0] = c02 * id;
        inv[2][1] = (M[0][1] * M[2][0] - M[0][0] * M[2][1]) * id;
        inv[2][2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * id;
      }
      const double kh = P.limiter_k * len[c];
      const T e2 = kh * kh * kh;
      for (int v = 0; v < nv; ++v) {
        T G[3];
        for (int i = 0; i < nd; ++i) {
          T s = inv[i][0] * b[v][0];
          for (int j = 1; j < nd; ++j) s = s + inv[i][j] * b[v][j];
          G[i] = s;
        }
        const T dmax = wmax[v] - wc[v], dmin = wmin[v] - wc[v];
        T psi = 1.0;
        for_each_face(c, [&](Ind nb, int d, int side) {
          double xf[3];
          if (side < 0) face_point(nb, c, d, xf);
          else face_point(c, nb, d, xf);
          T d2 = G[0] * (xf[0] - xc[0][c]);
          for (int k = 1; k < nd; ++k) d2 = d2 + G[k] * (xf[k] - xc[k][c]);
          T phi = 1.0;
          if (d2 > 0) phi = vk_phi(dmax, d2, e2);
          else if (d2 < 0) phi = vk_phi(dmin, d2, e2);
          psi = phi < psi ? phi : psi;
        });
        for (int i = 0; i < nd; ++i) Wg[v][i][c] = psi * G[i];
      }
    }
    // periodic ghosts take their paired cell's gradient
    for (Ind g = firstGC; g < size(); ++g)
      if (bcs[bc_idx[g]].kind == BC_PERIODIC)
        for (int v = 0; v < nv; ++v)
          for (int d = 0; d < nd; ++d) Wg[v][d][g] = Wg[v][d][periodic_partner[g - firstGC]];
  }
  // reconstructed primitive state of cell X at the face point xf
  WState recon_w(int t, Ind X, const double* xf) const {
    WState w = prim_w(t, X);
    for (int v = 0; v < nv; ++v) {
      T s = w[v];
      for (int k = 0; k < nd; ++k) s = s + Wg[v][k][X] * (xf[k] - xc[k][X]);
      w[v] = s;
    }
    return w;
  }
  // AUSM (euler/physics.hpp:276-325) of two primitive states
  State ausm_w(const WState& wl, const WState& wr, int d) const {
    auto side = [&](const WState& w, State& th, T& pp, T& M) {
      using std::sqrt;
      const T rh = w[nd];
      pp = w[nd + 1];
      const T a_ = sqrt(P.gamma * pp / rh);
      M = w[d] / a_;
      T um2 = w[0] * w[0];
      for (int k = 1; k < nd; ++k) um2 = um2 + w[k] * w[k];
      for (int k = 0; k < nd; ++k) th[k] = (rh * w[k]) * a_;
      th[nd] = rh * a_;
      th[nd + 1] = ((pp / P.gm1 + 0.5 * rh * um2) + pp) * a_;
    };
    State tl{}, tr{};
    T pl, pr, ML, MR;
    side(wl, tl, pl, ML);
    side(wr, tr, pr, MR);
    const T m_i = m_int(+1, ML) + m_int(-1, MR);
    const T p_i = p_int(+1, ML) * pl + p_int(-1, MR) * pr;
    State f = m_i >= 0 ? tl : tr;
    for (int v = 0; v < nv; ++v) f[v] = f[v] * m_i;
    f[d] = f[d] + p_i;
    return f;
  }
  State muscl_flux(int t, Ind l, Ind r, int d) const {
    double xf[3];
    face_point(l, r, d, xf);
    WState wl = recon_w(t, l, xf), wr = recon_w(t, r, xf);
    if (!(wl[nd] > 0) || !(wl[nd + 1] > 0) || !(wr[nd] > 0) || !(wr[nd + 1] > 0)) {
      wl = prim_w(t, l);
      wr = prim_w(t, r);
    }
    return ausm_w(wl, wr, d);
  }

  // compute_num_flux dispatch (euler/physics.hpp:175-178, cns/physics.hpp:155-161, heat/physics.hpp:113-119)
  State face_flux(int t, Ind l, Ind r, int d, double dx, T dt) const {
    if (P.physics == PHYS_ADVECTION) {
      State f{};
      const T qL = q(t, l, 0), qR = q(t, r, 0);
      const double uL = velocity(l, d), uR = velocity(r, d);
      if (P.flux == FLUX_LLF) {  // advection/physics.hpp:120-130
        const double lambda_max = std::max(std::abs(uL), std::abs(uR));
        f[0] = 0.5 * (qL * uL + qR * uR + lambda_max * (qL - qR));
      } else {  // upwind: advection/physics.hpp:132-145 (hom3 negates u_L q_L when the face velocity is negative)
        const double u_srfc = 0.5 * (uL + uR);
        f[0] = uL * qL;
        if (u_srfc < 0) f[0] = f[0] * -1.;
      }
      return f;
    }
    if (P.physics == PHYS_HEAT) {
      State f{};
      f[0] = 1 / dx * (q(t, l, 0) - q(t, r, 0));
      return f;
    }
    if (P.recon == RECON_MUSCL) return muscl_flux(t, l, r, d);
    State f = P.flux == FLUX_LLF ? llf(t, l, r, d, dx, dt) : ausm(t, l, r, d);
    if (P.physics == PHYS_CNS) {
      const State fv = viscous(t, l, r, d);
      for (int v = 0; v < nv; ++v) f[v] = f[v] + fv[v];
    }
    return f;
  }
  // num_flux: solver.hpp:440-460
  State num_flux(int t, Ind c) const {
    State res{};
    const double dx = len[c];
    const int ns = 1 << (nd - 1);
    const double wgt = nd == 2 ? 0.5 : 0.25;
    for (int d = 0; d < nd; ++d) {
      const Ind m = nbr[2 * d][c], pp = nbr[2 * d + 1][c];
      State fm{}, fp{};
      if (m >= 0) {
        fm = face_flux(t, m, c, d, dx, dt_);
      } else {  // EXTENSION: finer cells on the minus side
        for (int j = 0; j < ns; ++j) {
          const State f = face_flux(t, subs[(-m - 2) * ns + j], c, d, dx, dt_);
          for (int v = 0; v < nv; ++v) fm[v] = j == 0 ? f[v] : T(fm[v] + f[v]);
        }
        for (int v = 0; v < nv; ++v) fm[v] = wgt * fm[v];
      }
      if (pp >= 0) {
        fp = face_flux(t, c, pp, d, dx, dt_);
      } else {  // EXTENSION: finer cells on the plus side
        for (int j = 0; j < ns; ++j) {
          const State f = face_flux(t, c, subs[(-pp - 2) * ns + j], d, dx, dt_);
          for (int v = 0; v < nv; ++v) fp[v] = j == 0 ? f[v] : T(fp[v] + f[v]);
        }
        for (int v = 0; v < nv; ++v) fp[v] = wgt * fp[v];
      }
      for (int v = 0; v < nv; ++v) res[v] = res[v] + (fm[v] - fp[v]);
    }
    const T k = dt_ / dx;
    for (int v = 0; v < nv; ++v) res[v] = k * res[v];
    return res;
  }
  // compute_dt per cell: euler/physics.hpp:182-196, cns/physics.hpp:167-187, heat/physics.hpp:82-85
  T cell_dt(Ind c) const {
    using std::abs;
    const double h = len[c];
    if (P.physics == PHYS_HEAT) return P.cfl * 0.5 * std::pow(h, 2.);
    if (P.physics == PHYS_ADVECTION) {  // advection/physics.hpp:78-87
      double u_max = std::numeric_limits<double>::lowest();
      for (int d = 0; d < nd; ++d) u_max = std::max(u_max, std::abs(velocity(c, d)));
      return T(P.cfl * h / u_max);
    }
    const T a_ = a(0, c);
    T S = std::numeric_limits<double>::lowest();
    for (int d = 0; d < nd; ++d) {
      const T cand = abs(u(0, c, d)) + a_;
      S = (S < cand) ? cand : S;  // std::max
    }
    const T dt_inv = P.cfl * h / S;
    if (P.physics != PHYS_CNS) return dt_inv;
    const T S_coeff = sutherland(Temp(0, c)) / (rho(0, c) * h);
    const T a1 = S_coeff / P.Re0, a2 = S_coeff / (P.Re0 * P.Pr0 * P.gm1);
    const T S_visc = (a1 < a2) ? a2 : a1;
    const T dt_v = P.cfl_viscous * h / (2 * S_visc);
    return (dt_v < dt_inv) ? dt_v : dt_inv;  // std::min
  }
  // compute_dt: solver.hpp:511-517
  T compute_dt() const {
    T dt = std::numeric_limits<double>::max();
    const Ind n = n_internal();
#pragma omp parallel
    {
      T loc = std::numeric_limits<double>::max();
#pragma omp for schedule(static) nowait
      for (Ind c = 0; c < n; ++c) {
        const T cd = cell_dt(c);
        loc = (cd < loc) ? cd : loc;  // std::min(dt, cd): NaN never wins
      }
#pragma omp critical
      dt = (loc < dt) ? loc : dt;
    }
    return dt;
  }
  // set_dt: solver.hpp:541-551
  void set_dt() {
    if (time_ + dt_ < tEnd_) {
      if (step_ == forced_step_) dt_ = forced_dt_;
      else dt_ = compute_dt();
    } else {
      dt_ = tEnd_ - time_;
    }
  }
  void force_dt(T dt) { forced_step_ = step_; forced_dt_ = dt; }  // :522-525

  // ---- boundary conditions ----
  void isentropic_vortex(const double* x, double t, ICState& out) const;
  Ind partner_cell(Ind g) const;  // coupling.hpp:24-39
  void apply_bc(int t, int b, Ind g0, Ind g1);
  // apply_bcs: solver.hpp:561-586 (segment discovery by find_if, as in hom3)
  void apply_bcs(int t) {
    Ind first = 0;
    while (first < size() && bc_idx[first] == SINV) ++first;
    if (first == size()) return;
    SInd bcIdx = bc_idx[first];
    Ind last = 0;
    while (last < size() && bc_idx[last] != bcIdx) ++last;
    for (int k = 0; k < (int)bcs.size(); ++k) {
      ++bcIdx;
      const Ind fg = last;
      last = fg;
      while (last < size() && bc_idx[last] != bcIdx) ++last;
      apply_bc(t, k, fg, last);
    }
  }

  // evolve: solver.hpp:470-494
  void evolve() {
    const Ind n = n_internal();
    if (P.ti == TI_EULER_FORWARD) {
      if (P.recon == RECON_MUSCL) compute_gradients(0);
#pragma omp parallel for schedule(static)
      for (Ind c = 0; c < n; ++c) {
        const State nf = num_flux(0, c);
        for (int v = 0; v < nv; ++v) q(1, c, v) = q(0, c, v) + nf[v] + 0.0;  // source term is zero
      }
#pragma omp parallel for schedule(static)
      for (Ind c = 0; c < n; ++c)
        for (int v = 0; v < nv; ++v) q(0, c, v) = q(1, c, v);
    } else if (P.ti == TI_RK2) {
      if (P.recon == RECON_MUSCL) compute_gradients(0);
#pragma omp parallel for schedule(static)
      for (Ind c = 0; c < n; ++c) {
        const State nf = num_flux(0, c);
        for (int v = 0; v < nv; ++v) q(1, c, v) = q(0, c, v) + nf[v];
      }
      apply_bcs(1);
      if (P.recon == RECON_MUSCL) compute_gradients(1);
#pragma omp parallel for schedule(static)
      for (Ind c = 0; c < n; ++c) {
        const State nf = num_flux(1, c);
        for (int v = 0; v < nv; ++v) q(0, c, v) = 0.5 * ((q(0, c, v) + q(1, c, v)) + nf[v]);
      }
    } else {  // EXTENSION (not in hom3): SSP-RK3 in Shu-Osher form
      if (P.recon == RECON_MUSCL) compute_gradients(0);
#pragma omp parallel for schedule(static)
      for (Ind c = 0; c < n; ++c) {
        const State nf = num_flux(0, c);
        for (int v = 0; v < nv; ++v) q(1, c, v) = q(0, c, v) + nf[v];
      }
      apply_bcs(1);
      if (P.recon == RECON_MUSCL) compute_gradients(1);
#pragma omp parallel for schedule(static)
      for (Ind c = 0; c < n; ++c) {
        const State nf = num_flux(1, c);
        for (int v = 0; v < nv; ++v) q(2, c, v) = 0.75 * q(0, c, v) + 0.25 * (q(1, c, v) + nf[v]);
      }
      apply_bcs(2);
      if (P.recon == RECON_MUSCL) compute_gradients(2);
#pragma omp parallel for schedule(static)
      for (Ind c = 0; c < n; ++c) {
        const State nf = num_flux(2, c);
        for (int v = 0; v < nv; ++v) q(0, c, v) = (1.0 / 3.0) * q(0, c, v) + (2.0 / 3.0) * (q(2, c, v) + nf[v]);
      }
    }
  }
  // solve: solver.hpp:140-145
  void solve() {
    apply_bcs(0);
    set_dt();
    evolve();
    time_ += value(dt_);
    ++step_;
  }

  bool in_domain(const double* x) const {
    if (domain_kind == 0) return true;
    const double s = domain(nd, x);
    return domain_kind == 1 ? (s > 0.) : (s < 0.);
  }
  void eval_ic(const double* x, ICState& out) const;
  void initialize();
};

// ---------------------------------------------------------------------------
// World: one grid shared by several solvers (coupled tests)
// ---------------------------------------------------------------------------
template <class T> struct World {
  std::unique_ptr<Tree> tree;
  std::vector<std::unique_ptr<Solver<T>>> solvers;
  int nd = 2;
};

// isentropic_vortex: euler/initial_conditions.hpp:14-39 (hard-coded
// beta=5, gamma=1.4, x0=(-5,-5), u=v=1 in hom3).
template <class T>
void Solver<T>::isentropic_vortex(const double* x, double t, ICState& out) const {
  double beta = 5, gamma = 1.4, x00 = -5.0, x01 = -5.0, uu = 1, vv = 1;
  if (ic_kind == IC_VORTEX_PARAM) { beta = ic[0]; x00 = ic[1]; x01 = ic[2]; uu = ic[3]; vv = ic[4]; }
  const double x_t = x[0] - uu * t, y_t = x[1] - vv * t;
  const double r = std::sqrt(std::pow(x_t - x00, 2) + std::pow(y_t - x01, 2));
  const double eT1mr2 = std::exp(1 - std::pow(r, 2));
  const double eT21mr2 = std::exp(2 * (1 - std::pow(r, 2)));
  ICState pvars{};
  pvars[0] = uu - beta * eT1mr2 * (y_t - x01) / (2 * PI);
  pvars[1] = vv + beta * eT1mr2 * (x_t - x00) / (2 * PI);
  pvars[2] = std::pow((1 - ((gamma - 1) * std::pow(beta, 2) * eT21mr2) / (16 * gamma * std::pow(PI, 2))),
                      1 / (gamma - 1));
  pvars[3] = std::pow(pvars[2], gamma);
  // cv<nd>(pvars, 1.4): euler/quantities.hpp:153-166 with gamma = 1.4
  ICState c{};
  c[2] = pvars[2];
  double vm2 = 0;
  for (int d = 0; d < 2; ++d) { c[d] = pvars[2] * pvars[d]; vm2 += pvars[d] * pvars[d]; }
  c[3] = pvars[3] / (1.4 - 1.0) + 0.5 * pvars[2] * vm2;
  out = c;
}

template <class T> void Solver<T>::eval_ic(const double* x, ICState& out) const {
  ICState pvars{};
  if (ic_kind == IC_CONSTANT_PV) {
    for (int v = 0; v < nv; ++v) pvars[v] = ic[v];
    out = cv(pvars);
  } else if (ic_kind == IC_CONSTANT_CV) {
    for (int v = 0; v < nv; ++v) out[v] = ic[v];
  } else if (ic_kind == IC_SHOCK_TUBE) {
    // ic = {dir, angle, x0, rhoL, umagL, pL, rhoR, umagR, pR}: euler/initial_conditions.hpp:51-90
    const int dir = (int)ic[0];
    const double angle = ic[1], x0 = ic[2];
    const double alpha = angle * (2 * PI) / 360;
    double x_rot[3] = {0, 0, 0};
    x_rot[0] = std::cos(alpha) * x[0] - std::sin(alpha) * x[1];
    x_rot[1] = std::sin(alpha) * x[0] + std::cos(alpha) * x[1];
    double uL[3] = {0, 0, 0}, uR[3] = {0, 0, 0};
    uL[0] = ic[4] * std::cos(alpha); uL[1] = ic[4] * std::sin(alpha);
    uR[0] = ic[7] * std::cos(alpha); uR[1] = ic[7] * std::sin(alpha);
    const bool approx0 = std::abs(alpha - 0.0) <= 4 * std::numeric_limits<double>::epsilon();
    const double pos = approx0 ? x0 : x0 * std::sqrt(2.);
    if (x_rot[dir] < pos) {
      pvars[nd] = ic[3];
      for (int d = 0; d < nd; ++d) pvars[d] = uL[d];
      pvars[nd + 1] = ic[5];
    } else {
      pvars[nd] = ic[6];
      for (int d = 0; d < nd; ++d) pvars[d] = uR[d];
      pvars[nd + 1] = ic[8];
    }
    // shock_tube converts with gamma = 1.4 hard-coded (euler/initial_conditions.hpp:58)
    ICState c{};
    c[nd] = pvars[nd];
    double vm2 = 0;
    for (int d = 0; d < nd; ++d) { c[d] = pvars[nd] * pvars[d]; vm2 += pvars[d] * pvars[d]; }
    c[nd + 1] = pvars[nd + 1] / (1.4 - 1.0) + 0.5 * pvars[nd] * vm2;
    out = c;
  } else if (ic_kind == IC_VORTEX || ic_kind == IC_VORTEX_PARAM) {
    isentropic_vortex(x, 0.0, out);
  } else if (ic_kind == IC_EXPLOSION) {
    // ic = {cx, cy, cz, R, rho_in, p_in, rho_out, p_out}: euler_fv_solver_test.cpp:222-245
    double s = 0;
    for (int d = 0; d < nd; ++d) s += (x[d] - ic[d]) * (x[d] - ic[d]);
    const bool inside = std::sqrt(s) < ic[3];
    for (int d = 0; d < nd; ++d) pvars[d] = 0;
    pvars[nd] = inside ? ic[4] : ic[6];
    pvars[nd + 1] = inside ? ic[5] : ic[7];
    out = cv(pvars);
  } else if (ic_kind == IC_DISC) {
    // ic = {c_0, c_1, c_2, R, q_in, q_out}: advection_fv_solver_test.cpp:106-115
    double s2 = 0;
    for (int d = 0; d < nd; ++d) s2 += (x[d] - ic[d]) * (x[d] - ic[d]);
    out[0] = std::sqrt(s2) - ic[3] > 0. ? ic[5] : ic[4];
  } else if (ic_kind == IC_TAYLOR_GREEN) {
    // EXTENSION (not in hom3): ic = {U, rho0, p0}; u = U sin x cos y cos z,
    // v = -U cos x sin y cos z, w = 0, p = p0 + rho0 U^2/16 (cos 2x + cos 2y)(cos 2z + 2),
    // rho = rho0 p / p0 (isothermal start)
    const double U = ic[0], r0 = ic[1], p0 = ic[2];
    const double z = nd == 3 ? x[2] : 0.0;
    pvars[0] = U * std::sin(x[0]) * std::cos(x[1]) * std::cos(z);
    pvars[1] = -U * std::cos(x[0]) * std::sin(x[1]) * std::cos(z);
    if (nd == 3) pvars[2] = 0.0;
    const double p = p0 + r0 * U * U / 16.0 * (std::cos(2 * x[0]) + std::cos(2 * x[1])) * (std::cos(2 * z) + 2.0);
    pvars[nd] = r0 * p / p0;
    pvars[nd + 1] = p;
    out = cv(pvars);
  } else if (ic_kind == IC_RIEMANN3D_PERTURBED) {
    // EXTENSION (not in hom3).  ic = {x0, rhoL, pL, rhoR, pR, amp, nmodes,
    // then per mode (kx, ky, kz, phase) starting at ic[8]} -- at most 16 modes.
    const int nm = (int)ic[6];
    double pert = 0;
    for (int m = 0; m < nm; ++m) {
      const double* k = ic + 8 + 4 * m;
      double arg = k[3];
      for (int d = 0; d < nd; ++d) arg += 2 * PI * k[d] * x[d];
      pert += std::sin(arg);
    }
    const double f = 1.0 + ic[5] * pert / (nm > 0 ? nm : 1);
    const bool left = x[0] < ic[0];
    for (int d = 0; d < nd; ++d) pvars[d] = 0;
    pvars[nd] = (left ? ic[1] : ic[3]) * f;
    pvars[nd + 1] = (left ? ic[2] : ic[4]) * f;
    out = cv(pvars);
  }
}

// local_bndry_ids: coupling.hpp:24-39 -- the partner is the other solver's
// cell at the grid node that neighbours the boundary node at the ghost's position.
template <class T> Ind Solver<T>::partner_cell(Ind g) const {
  const Ind b = boundary_cell(g);
  const int bpos = boundary_pos(g);
  const int gpos = opposite_pos[bpos];
  const Ind bn = node[b];
  const Ind on = w->tree->find_samelvl_neighbor(bn, gpos);
  const int other = bcs[bc_idx[g]].partner;
  return on == INV ? INV : w->tree->node2cell[other][on];
}

template <class T> void Solver<T>::apply_bc(int t, int k, Ind g0, Ind g1) {
  const Bc& B = bcs[k];
  for (Ind g = g0; g < g1; ++g) {
    const Ind b = boundary_cell(g);
    switch (B.kind) {
      case BC_EULER_NEUMANN: {  // euler/boundary_conditions.hpp:17-43
        double dx2 = 0;
        for (int d = 0; d < nd; ++d) dx2 += (xc[d][b] - xc[d][g]) * (xc[d][b] - xc[d][g]);
        const double dx = std::sqrt(dx2);  // cell_dx: solver.hpp:590-592
        for (int v = 0; v < nv; ++v) q(t, g, v) = q(t, b, v) - dx * B.v[v];
        break;
      }
      case BC_EULER_DIRICHLET:  // :279-288
        for (int v = 0; v < nv; ++v) q(t, g, v) = 2.0 * B.v[v] - q(t, b, v);
        break;
      case BC_EULER_VORTEX: {  // :304-316 (also overwrites the boundary cell)
        double xg[3], xb[3];
        for (int d = 0; d < nd; ++d) { xg[d] = xc[d][g]; xb[d] = xc[d][b]; }
        ICState sg, sb;
        isentropic_vortex(xg, time_, sg);
        isentropic_vortex(xb, time_, sb);
        for (int v = 0; v < nv; ++v) { q(t, g, v) = sg[v]; q(t, b, v) = sb[v]; }
        break;
      }
      case BC_CNS_INFLOW: {  // cns/boundary_conditions.hpp:37-61; v = surface pv (u.., rho, p)
        const State bp = pv(Qrow(t, b));
        State gp{};
        for (int d = 0; d < nd; ++d) gp[d] = 2.0 * B.v[d] - bp[d];
        gp[nd] = 2.0 * B.v[nd] - bp[nd];
        gp[nd + 1] = bp[nd + 1] - 0 * 0;
        setQ(t, g, cv(gp));
        break;
      }
      case BC_CNS_OUTFLOW: {  // :81-101; v = surface pv, only p (v[nd+1]) is used
        const State bp = pv(Qrow(t, b));
        State gp{};
        for (int d = 0; d < nd; ++d) gp[d] = bp[d] - 0 * 0;
        gp[nd] = bp[nd] - 0 * 0;
        gp[nd + 1] = 2.0 * B.v[nd + 1] - bp[nd + 1];
        setQ(t, g, cv(gp));
        break;
      }
      case BC_CNS_ADIABATIC_NOSLIP: {  // :124-141
        const State bp = pv(Qrow(t, b));
        State gp{};
        for (int d = 0; d < nd; ++d) gp[d] = 2.0 * 0 - bp[d];
        gp[nd] = bp[nd] - 0 * 0;
        gp[nd + 1] = bp[nd + 1] - 0 * 0;
        setQ(t, g, cv(gp));
        break;
      }
      case BC_CNS_ADIABATIC_SLIP: {  // :164-190
        const int bpos = boundary_pos(g);
        const int ndir = bpos / 2;
        const State bp = pv(Qrow(t, b));
        State gp{};
        for (int d = 0; d < nd; ++d) gp[d] = bp[d] - 0 * 0;
        gp[ndir] = 2.0 * 0 - bp[ndir];
        gp[nd] = bp[nd] - 0 * 0;
        gp[nd + 1] = bp[nd + 1] - 0 * 0;
        setQ(t, g, cv(gp));
        break;
      }
      case BC_CNS_ISOTHERMAL_NOSLIP:  // :209-228; v = {T_srfc}
      case BC_CPL_CNS_HEAT: {         // cns/coupling_conditions.hpp:22-43
        const State bp = pv(Qrow(t, b));
        T Ts;
        if (B.kind == BC_CNS_ISOTHERMAL_NOSLIP) {
          Ts = B.v[0];
        } else {
          const Ind o = partner_cell(g);
          const T Tf = Temp(0, b);  // fluid T from lhs
          const T Tsol = w->solvers[B.partner]->Temp(0, o);  // solid T from lhs
          // EXTENSION: conductivity ratio kappa = k_solid / k_fluid in v[0] (0: hom3's mean)
          const double kap = B.v[0];
          Ts = (kap == 0.0 || kap == 1.0) ? T(0.5 * (Tf + Tsol)) : T((Tf + kap * Tsol) / (1.0 + kap));
        }
        State gp{};
        for (int d = 0; d < nd; ++d) gp[d] = 2.0 * 0 - bp[d];
        const T p_srfc = bp[nd + 1];
        const T rho_srfc = p_srfc * P.gamma / Ts;
        gp[nd] = 2.0 * rho_srfc - bp[nd];
        gp[nd + 1] = bp[nd + 1] - 0 * 0;
        setQ(t, g, cv(gp));
        break;
      }
      case BC_HEAT_DIRICHLET:  // heat/boundary_conditions.hpp:15-37; v = {T}
        q(t, g, 0) = 2.0 * B.v[0] - q(t, b, 0);
        break;
      case BC_HEAT_NEUMANN: {  // :40-63
        double dx2 = 0;
        for (int d = 0; d < nd; ++d) dx2 += (xc[d][b] - xc[d][g]) * (xc[d][b] - xc[d][g]);
        q(t, g, 0) = q(t, b, 0) - std::sqrt(dx2) * B.v[0];
        break;
      }
      case BC_CPL_HEAT_CNS:    // heat/coupling_conditions.hpp:18-38
      case BC_CPL_HEAT_HEAT: { // :41-61
        const Ind o = partner_cell(g);
        const T Tthis = Temp(0, b);
        const T Tother = w->solvers[B.partner]->Temp(0, o);
        const double kap = B.kind == BC_CPL_HEAT_CNS ? B.v[0] : 0.0;  // EXTENSION: k_solid / k_fluid
        const T Ts = B.kind == BC_CPL_HEAT_CNS
                         ? ((kap == 0.0 || kap == 1.0) ? T(0.5 * (Tother + Tthis)) : T((Tother + kap * Tthis) / (1.0 + kap)))
                         : T(0.5 * (Tthis + Tother));
        q(t, g, 0) = 2.0 * Ts - q(t, b, 0);
        break;
      }
      case BC_PERIODIC: {  // EXTENSION
        const Ind o = periodic_partner[g - firstGC];
        for (int v = 0; v < nv; ++v) q(t, g, v) = q(t, o, v);
        break;
      }
      case BC_ADV_DIRICHLET:  // advection/boundary_conditions.hpp:25-32; v = {q_srfc}
        q(t, g, 0) = 2.0 * B.v[0] - q(t, b, 0);
        break;
      case BC_ADV_NEUMANN: {  // :50-58; v = {surface flux}, distance of the cell centres
        double dx2 = 0;
        for (int d = 0; d < nd; ++d) dx2 += (xc[d][b] - xc[d][g]) * (xc[d][b] - xc[d][g]);
        q(t, g, 0) = q(t, b, 0) - std::sqrt(dx2) * B.v[0];
        break;
      }
      case BC_ADV_CHARACTERISTIC: {  // :71-91
        const int pos = opposite_pos[boundary_pos(g)];  // the ghost's position w.r.t. its boundary cell
        const int dir = pos / 2;
        const double v = velocity(b, dir);
        if ((v > 0. && pos % 2 == 0) || (v < 0. && pos % 2 == 1)) {
          q(t, g, 0) = 2.0 * q(t, b, 0) - q(t, b, 0);  // dirichlet(q_b, q_b)
        } else {
          double dx2 = 0;
          for (int d = 0; d < nd; ++d) dx2 += (xc[d][b] - xc[d][g]) * (xc[d][b] - xc[d][g]);
          q(t, g, 0) = q(t, b, 0) - std::sqrt(dx2) * 0.0;  // neumann(q_b, 0, dx)
        }
        break;
      }
      case BC_CPL_EULER_EULER: {  // euler/coupling_conditions.hpp:17-35
        const Ind o = partner_cell(g);
        const Solver<T>& os = *w->solvers[B.partner];
        for (int v = 0; v < nv; ++v) q(t, g, v) = os.q(t, o, v);
        break;
      }
      default:
        throw std::runtime_error("unknown bc kind");
    }
  }
}

// initialize: solver.hpp:133-138 with create_local_cells (876-930),
// create_ghost_cells (935-977), sort_gc (811-834), impose_initial_condition
// (980-992) and quadrature::integrate (quadrature.hpp:43-74).
template <class T> void Solver<T>::initialize() {
  Tree& tr = *w->tree;
  dt_ = 0; time_ = 0; tEnd_ = P.time_end; step_ = 0; forced_dt_ = 0; forced_step_ = INV;
  // 1) one cell per leaf inside the initial domain
  for (Ind n : tr.leaf_nodes()) {
    double x[3];
    tr.coords(n, x);
    if (!in_domain(x)) continue;
    const Ind c = push_cell();
    node[c] = n;
    tr.node2cell[idx][n] = c;
    for (int d = 0; d < nd; ++d) xc[d][c] = x[d];
    len[c] = tr.length(n);
  }
  // 2) same-level neighbours (solver.hpp:899-908)
  bool uniform = true;
  for (Ind c = 1; c < size(); ++c) uniform = uniform && len[c] == len[0];
  for (Ind c = 0; c < size(); ++c) {
    for (int p = 0; p < 2 * nd; ++p) {
      const Ind nn = tr.find_samelvl_neighbor(node[c], p);
      nbr[p][c] = nn != INV ? tr.node2cell[idx][nn] : INV;
      if (uniform || nbr[p][c] != INV) continue;
      // EXTENSION (not in hom3): coarse/fine faces of a refined tree
      if (nn != INV && !tr.is_leaf(nn)) {
        const int dir = p / 2;
        std::vector<Ind> grp;
        for (int ch = 0; ch < tr.nchild(); ++ch) {
          const int bit = (child_rel(nd, ch, dir) > 0) ? 1 : 0;
          if (bit != ((p & 1) ? 0 : 1)) continue;
          const Ind cn = tr.child(nn, ch);
          if (!tr.is_leaf(cn) || tr.node2cell[idx][cn] == INV) { grp.clear(); break; }
          grp.push_back(tr.node2cell[idx][cn]);
        }
        if (!grp.empty()) {
          nbr[p][c] = -2 - (Ind)(subs.size() >> (nd - 1));
          subs.insert(subs.end(), grp.begin(), grp.end());
        }
      } else if (nn == INV && !tr.is_root(node[c])) {
        const Ind pn = tr.find_samelvl_neighbor(tr.parent[node[c]], p);
        if (pn != INV && tr.is_leaf(pn) && tr.node2cell[idx][pn] != INV) nbr[p][c] = tr.node2cell[idx][pn];
      }
    }
  }
  firstGC = size();
  // 3) ghost cells, BC by BC, over the cells cut by each boundary
  const Ind nLeaf = size();
  for (int b = 0; b < (int)bcs.size(); ++b) {
    for (Ind c = 0; c < nLeaf; ++c) {
      double x[3];
      for (int d = 0; d < nd; ++d) x[d] = xc[d][c];
      if (!is_cut_by(nd, x, tr.length(node[c]), bcs[b].geom)) continue;
      std::vector<int> missing;
      for (int p = 0; p < 2 * nd; ++p)
        if (nbr[p][c] == INV) missing.push_back(p);
      for (int p : missing) {
        double xn[3];
        tr.neighbor_coords(node[c], p, xn);
        if (!(bcs[b].geom(nd, xn) < 0.)) continue;
        // create_ghost_cell: solver.hpp:843-861
        const Ind g = push_cell();
        node[g] = INV;
        nbr[p][c] = g;
        nbr[opposite_pos[p]][g] = c;
        for (int d = 0; d < nd; ++d)
          xc[d][g] = xc[d][c] + len[c] * (double)nghbr_rel_pos_3d[p][d];
        len[g] = len[c];
        bc_idx[g] = b;
      }
    }
  }
  // 4) sort ghosts by bc id.  hom3 uses std::sort (unstable); ghosts are
  // created in bc order already, so a stable sort keeps creation order.  The
  // order of ghosts inside one bc segment does not change any value.
  {
    const Ind first = firstGC;
    std::vector<Ind> perm(size() - first);
    std::iota(perm.begin(), perm.end(), first);
    std::stable_sort(perm.begin(), perm.end(), [&](Ind a, Ind b) { return bc_idx[a] < bc_idx[b]; });
    auto permute = [&](auto& col) {
      auto tmp = col;
      for (Ind i = 0; i < (Ind)perm.size(); ++i) col[first + i] = tmp[perm[i]];
    };
    for (int p = 0; p < 2 * nd; ++p) permute(nbr[p]);
    for (int d = 0; d < nd; ++d) permute(xc[d]);
    permute(len); permute(bc_idx); permute(node);
    for (Ind g = first; g < size(); ++g)
      for (int p = 0; p < 2 * nd; ++p)
        if (nbr[p][g] != INV) nbr[opposite_pos[p]][nbr[p][g]] = g;
  }
  // EXTENSION: periodic partners -- the interior cell at the ghost's position
  // wrapped into the root cell
  {
    periodic_partner.assign(size() - firstGC, INV);
    bool any = false;
    for (auto& b : bcs) any = any || b.kind == BC_PERIODIC;
    if (any) {
      const double L = tr.rootLength;
      double lo[3];
      for (int d = 0; d < nd; ++d) lo[d] = tr.rootCoords[d] - 0.5 * L;
      auto key = [&](const double* x, double h) {
        long long k = 0;
        for (int d = 0; d < nd; ++d) {
          double w = x[d] - lo[d];
          w = w - L * std::floor(w / L);
          k = k * 4194304LL + (long long)std::floor(w / h);
        }
        return k;
      };
      std::unordered_map<long long, Ind> cellAt;
      for (Ind c = 0; c < firstGC; ++c) {
        double x[3];
        for (int d = 0; d < nd; ++d) x[d] = xc[d][c];
        cellAt[key(x, len[c]) * 32 + tr.level(node[c])] = c;
      }
      for (Ind g = firstGC; g < size(); ++g) {
        if (bcs[bc_idx[g]].kind != BC_PERIODIC) continue;
        double x[3];
        for (int d = 0; d < nd; ++d) x[d] = xc[d][g];
        const Ind b = boundary_cell(g);
        auto it = cellAt.find(key(x, len[g]) * 32 + tr.level(node[b]));
        if (it == cellAt.end()) throw std::runtime_error("periodic ghost without partner");
        periodic_partner[g - firstGC] = it->second;
      }
    }
  }
  compute_velocity();
  // 5) initial condition: cell average by 2^nd Gauss points
  const double gp = 1 / std::sqrt(3);
  for (Ind c = 0; c < firstGC; ++c) {
    const double l = tr.length(node[c]);
    ICState sum{};
    for (int k = 0; k < (1 << nd); ++k) {
      double x[3];
      for (int d = 0; d < nd; ++d) x[d] = xc[d][c] + 0.5 * l * ((double)child_rel(nd, k, d) * gp);
      ICState f{};
      eval_ic(x, f);
      for (int v = 0; v < nv; ++v) sum[v] = k == 0 ? f[v] : sum[v] + f[v];
    }
    double vol = l;
    for (int d = 1; d < nd; ++d) vol = l * vol;
    for (int v = 0; v < nv; ++v) q(0, c, v) = sum[v] * vol / (double)(1 << nd) / vol;
  }
  set_dt();
}

// EXTENSION (not in hom3): sphere refinement + 2:1 balance
inline void Tree::refine_sphere(const double* c, double r, int maxLevel) {
  bool done = false;
  while (!done) {
    done = true;
    const Ind end = size();
    for (Ind n = 0; n < end; ++n) {
      if (!is_leaf(n) || level(n) >= maxLevel) continue;
      double x[3];
      coords(n, x);
      const double h = 0.5 * length(n);
      double s = 0;  // squared distance from sphere centre to the cell box
      for (int d = 0; d < nd; ++d) {
        const double lo = x[d] - h, hi = x[d] + h;
        const double q = std::max(lo - c[d], std::max(0.0, c[d] - hi));
        s += q * q;
      }
      if (s < r * r) { refine(n); done = false; }
    }
  }
  balance_2to1();
}

inline void Tree::balance_2to1() {
  // A leaf must not have a face neighbour region refined more than one level
  // deeper.  Iterate: refine any leaf whose same-level neighbour exists and
  // has a child that is not a leaf.
  bool done = false;
  while (!done) {
    done = true;
    const Ind end = size();
    for (Ind n = 0; n < end; ++n) {
      if (!is_leaf(n)) continue;
      bool need = false;
      for (int p = 0; p < 2 * nd && !need; ++p) {
        const Ind m = find_samelvl_neighbor(n, p);
        if (m == INV || is_leaf(m)) continue;
        for (int k = 0; k < nchild(); ++k)
          if (!is_leaf(child(m, k))) { need = true; break; }
      }
      if (need) { refine(n); done = false; }
    }
  }
}

}  // namespace h3o
