// hom3's solver test cases, written against the C++ layer (include/hom3_b200.hpp)
// the way hom3 writes them against its own Solver
// (src/solver/fv/euler/tests/euler_fv_solver_test.cpp:85-286,
//  src/solver/fv/heat/tests/heat_fv_solver_test.cpp:81-105).
// hom3's versions only check that the run reaches timeEnd without diverging;
// these also check the state: a constant state must be preserved exactly and
// density / pressure / temperature stay positive and finite.
// Prints one line per case: "<name> <steps> <time> <ok>".
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <exception>
#include <string>

#include "hom3_b200.hpp"

using namespace hom3_b200;

static Properties euler_properties(double timeEnd) {  // euler_fv_solver_test.cpp:47-79
  Properties p;
  p.physics = H3C_EULER;
  p.flux = H3C_FLUX_AUSM;
  p.time_integration = H3C_EULER_FORWARD;
  p.timeEnd = timeEnd;
  p.gamma = 1.4;
  p.Minfty = 0.1;
  p.CFL = 0.2;
  return p;
}

static void cv(int nd, const double* pv, double* q) {  // euler/quantities.hpp:153-166
  const double rho = pv[nd];
  double vm2 = 0;
  for (int d = 0; d < nd; ++d) { q[d] = rho * pv[d]; vm2 += pv[d] * pv[d]; }
  q[nd] = rho;
  q[nd + 1] = pv[nd + 1] / (1.4 - 1.0) + 0.5 * rho * vm2;
}

static bool physical(Solver& s, int nd) {
  const auto& q = s.Q(0);
  const long long n = s.n_cells();
  for (long long c = 0; c < s.first_ghost(); ++c) {
    const double rho = q[nd * n + c];
    double um2 = 0;
    for (int d = 0; d < nd; ++d) um2 += (q[d * n + c] / rho) * (q[d * n + c] / rho);
    const double p = 0.4 * (q[(nd + 1) * n + c] - 0.5 * rho * um2);
    if (!(rho > 0 && p > 0 && std::isfinite(rho) && std::isfinite(p))) return false;
  }
  return true;
}

static void report(const char* name, Solver& s, bool ok) {
  std::printf("%s %lld %.17g %d\n", name, s.step(), s.time(), ok ? 1 : 0);
}

static int run_cases(int level);

int main(int argc, char** argv) {
  try {
    return run_cases(argc > 1 ? std::atoi(argv[1]) : 5);
  } catch (const std::exception& e) {  // hom3 would TERMINATE; report and fail
    std::printf("error %s\n", e.what());
    return 1;
  }
}

static int run_cases(int level) {
  const Grid cube3{3, {0, 0, 0}, {1, 1, 1}, level};
  // constant_ic: euler_fv_solver_test.cpp:85-112 -- "The solution is the initial condition for all t"
  {
    Solver s{cube3, euler_properties(0.25)};
    s.set_initial_condition([](const double*, double* q) {
      const double pv[5] = {0.5, 0.5, 0.5, 1.0, 1.0};
      cv(3, pv, q);
    });
    s.append_bcs(cube_boundaries(cube3, condition(H3C_BC_EULER_NEUMANN)));
    s.initialize();
    const std::vector<double> q0 = s.Q(0);
    run_solver(s, 10000);
    const auto& q1 = s.Q(0);
    bool same = true;
    for (int v = 0; v < 5; ++v)
      for (long long c = 0; c < s.first_ghost(); ++c) same = same && q1[v * s.n_cells() + c] == q0[v * s.n_cells() + c];
    report("euler_constant_ic", s, same && s.time() >= 0.25);
  }
  // sod_shock_tube_ic (:126-156) and problem123_ic (:171-201)
  for (int k = 0; k < 2; ++k) {
    const double x0 = k == 0 ? 0.3 : 0.5;
    const double L[3] = {k == 0 ? 1.0 : 1.0, k == 0 ? 0.75 : -2.0, k == 0 ? 1.0 : 0.4};
    const double R[3] = {k == 0 ? 0.125 : 1.0, k == 0 ? 0.0 : 2.0, k == 0 ? 0.1 : 0.4};
    Solver s{cube3, euler_properties(k == 0 ? 0.2 : 0.15)};
    s.set_initial_condition([=](const double* x, double* q) {  // ic::shock_tube, euler/initial_conditions.hpp:51-90
      const double* S = x[0] < x0 ? L : R;
      const double pv[5] = {S[1], 0.0, 0.0, S[0], S[2]};
      cv(3, pv, q);
    });
    s.append_bcs(cube_boundaries(cube3, condition(H3C_BC_EULER_NEUMANN)));
    run_solver(s, 10000);
    report(k == 0 ? "euler_sod_shock_tube_ic" : "euler_problem123_ic", s, physical(s, 3));
  }
  // explosion_ic (euler_fv_solver_test.cpp:212-255)
  {
    Solver s{cube3, euler_properties(0.25)};
    s.set_initial_condition([](const double* x, double* q) {
      const double r = std::sqrt((x[0] - 0.5) * (x[0] - 0.5) + (x[1] - 0.5) * (x[1] - 0.5) + (x[2] - 0.5) * (x[2] - 0.5));
      const double pv[5] = {0, 0, 0, r < 0.2 ? 1.0 : 0.125, r < 0.2 ? 1.0 : 0.1};
      cv(3, pv, q);
    });
    s.append_bcs(cube_boundaries(cube3, condition(H3C_BC_EULER_NEUMANN)));
    run_solver(s, 10000);
    report("euler_explosion_ic", s, physical(s, 3));
  }
  // isentropic_vortex_ic (:258-286): 2D on [-8,8]^2
  {
    const Grid sq{2, {-8, -8, 0}, {8, 8, 0}, level};
    Solver s{sq, euler_properties(2.0)};
    s.set_initial_condition([](const double* x, double* q) {  // ic::isentropic_vortex at t = 0
      const double PI = 3.141592653589793238462643383279502884, beta = 5, gamma = 1.4;
      const double r = std::sqrt((x[0] + 5) * (x[0] + 5) + (x[1] + 5) * (x[1] + 5));
      const double e1 = std::exp(1 - r * r), e2 = std::exp(2 * (1 - r * r));
      const double u = 1 - beta * e1 * (x[1] + 5) / (2 * PI), v = 1 + beta * e1 * (x[0] + 5) / (2 * PI);
      const double rho = std::pow(1 - ((gamma - 1) * beta * beta * e2) / (16 * gamma * PI * PI), 1 / (gamma - 1));
      const double pv[4] = {u, v, rho, std::pow(rho, gamma)};
      cv(2, pv, q);
    });
    s.append_bcs(cube_boundaries(sq, condition(H3C_BC_EULER_VORTEX)));
    run_solver(s, 10000);
    report("euler_isentropic_vortex_ic", s, physical(s, 2));
  }
  // heat one_dimensional_dirichlet: heat_fv_solver_test.cpp:81-105
  {
    const Grid g{3, {0, 0, 0}, {1, 1, 1}, level > 4 ? 4 : level};
    Properties p;
    p.physics = H3C_HEAT;
    p.CFL = 0.5;
    p.timeEnd = 0.25;
    Solver s{g, p};
    s.set_initial_condition([](const double*, double* q) { q[0] = 0.0; });
    const h3c_bc d = condition(H3C_BC_HEAT_DIRICHLET, {1.0}), nbc = condition(H3C_BC_HEAT_NEUMANN, {0.0});
    s.append_bcs(cube_boundaries(g, {d, d, nbc, nbc, nbc, nbc}));
    run_solver(s, 1000);
    const auto& q = s.Q(0);
    bool ok = true;
    for (long long c = 0; c < s.first_ghost(); ++c) ok = ok && q[c] >= -1e-12 && q[c] <= 1.0 + 1e-12;
    report("heat_one_dimensional_dirichlet", s, ok);
  }
  return 0;
}
