// h3o_capi.cpp -- C entry points of the CPU oracle, for ctypes.
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, by __graft_entry__.smoke() and
// by the CPU-baseline / reference legs of bench.py.  Never linked into the
// shipped library.
#include <cstring>

#include "h3o.hpp"
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace h3o;
using W = World<double>;

extern "C" {

typedef struct {
  int kind, inverted;
  double p[6];
} h3o_sdf;

typedef struct {
  int kind;
  h3o_sdf geom;
  double v[8];
  int partner;
} h3o_bc;

typedef struct {
  int physics, flux, time_integration;
  double cfl, cfl_viscous, gamma, Rspecific, T0, rho0, Minfty, ReInfty, Pr0, Sutherland0,
      diffusivity, T_ref, time_end;
  int domain_kind;
  h3o_sdf domain;
  int ic_kind;
  double ic[80];
  int n_bcs;
  const h3o_bc* bcs;
  int recon;         // EXTENSION: 0 none (hom3), 1 MUSCL (LSQ gradients, Venkatakrishnan limiter)
  double limiter_k;  // Venkatakrishnan constant K
  int vel_kind;      // advection velocity field (VelocityKind)
  double vel[4];
} h3o_solver_desc;

static Sdf to_sdf(const h3o_sdf& s) {
  Sdf r;
  r.kind = s.kind;
  r.inverted = s.inverted;
  for (int i = 0; i < 6; ++i) r.p[i] = s.p[i];
  return r;
}

void* h3o_world_create(int nd, const double* xmin, const double* xmax, int max_solvers) {
  auto* w = new W();
  w->nd = nd;
  w->tree.reset(new Tree(nd, xmin, xmax, max_solvers));
  return w;
}
void h3o_world_destroy(void* w) { delete (W*)w; }
int h3o_world_min_level(void* w, int level) {
  ((W*)w)->tree->min_level(level);
  return 0;
}
int h3o_world_refine_sphere(void* w, const double* c, double r, int max_level) {
  ((W*)w)->tree->refine_sphere(c, r, max_level);
  return 0;
}
int64_t h3o_grid_nnodes(void* w) { return ((W*)w)->tree->size(); }
int64_t h3o_grid_neighbor(void* w, int64_t n, int pos) {
  return ((W*)w)->tree->find_samelvl_neighbor(n, pos);
}
int64_t h3o_grid_child(void* w, int64_t n, int pos) { return ((W*)w)->tree->child(n, pos); }
int h3o_grid_is_leaf(void* w, int64_t n) { return ((W*)w)->tree->is_leaf(n); }
int h3o_grid_level(void* w, int64_t n) { return ((W*)w)->tree->level(n); }
int h3o_grid_pos_in_parent(void* w, int64_t n) { return ((W*)w)->tree->pos_in_parent(n); }
void h3o_grid_coords(void* w, int64_t n, double* x) { ((W*)w)->tree->coords(n, x); }
double h3o_grid_length(void* w, int64_t n) { return ((W*)w)->tree->length(n); }
double h3o_grid_root_length(void* w) { return ((W*)w)->tree->rootLength; }
int h3o_cube_boundaries(void* w, h3o_sdf* out) {
  W* ww = (W*)w;
  auto b = cube_boundaries(ww->nd, *ww->tree);
  for (size_t i = 0; i < b.size(); ++i) {
    out[i].kind = b[i].kind;
    out[i].inverted = b[i].inverted;
    for (int k = 0; k < 6; ++k) out[i].p[k] = b[i].p[k];
  }
  return (int)b.size();
}
double h3o_sdf_eval(int nd, const h3o_sdf* s, const double* x) { return to_sdf(*s)(nd, x); }

int h3o_add_solver(void* w, const h3o_solver_desc* d) {
  W* ww = (W*)w;
  auto s = std::make_unique<Solver<double>>();
  s->w = ww;
  s->idx = (int)ww->solvers.size();
  s->nd = ww->nd;
  Params& P = s->P;
  P.physics = d->physics;
  P.flux = d->flux;
  P.ti = d->time_integration;
  P.cfl = d->cfl; P.cfl_viscous = d->cfl_viscous; P.gamma = d->gamma; P.Rspecific = d->Rspecific;
  P.T0 = d->T0; P.rho0 = d->rho0; P.Minfty = d->Minfty; P.ReInfty = d->ReInfty; P.Pr0 = d->Pr0;
  P.Sutherland0 = d->Sutherland0; P.diffusivity = d->diffusivity; P.T_ref = d->T_ref;
  P.time_end = d->time_end;
  P.recon = d->recon;
  P.limiter_k = d->limiter_k;
  P.vel_kind = d->vel_kind;
  for (int i = 0; i < 4; ++i) P.vel[i] = d->vel[i];
  P.derive();
  s->nv = (P.physics == PHYS_HEAT || P.physics == PHYS_ADVECTION) ? 1 : ww->nd + 2;
  s->domain_kind = d->domain_kind;
  s->domain = to_sdf(d->domain);
  s->ic_kind = d->ic_kind;
  std::memcpy(s->ic, d->ic, sizeof(s->ic));
  for (int i = 0; i < d->n_bcs; ++i) {
    Bc b;
    b.kind = d->bcs[i].kind;
    b.geom = to_sdf(d->bcs[i].geom);
    std::memcpy(b.v, d->bcs[i].v, sizeof(b.v));
    b.partner = d->bcs[i].partner;
    s->bcs.push_back(b);
  }
  if ((int)ww->tree->node2cell.size() <= s->idx) return -1;
  ww->solvers.push_back(std::move(s));
  return (int)ww->solvers.size() - 1;
}

static Solver<double>& S(void* w, int s) { return *((W*)w)->solvers[s]; }

// advection velocity of every cell (ghosts included), [nd][n_cells]
void h3o_velocity(void* w, int s, double* out) {
  const Solver<double>& so = S(w, s);
  const int64_t n = so.size();
  for (int d = 0; d < so.nd; ++d)
    for (int64_t c = 0; c < n; ++c) out[d * n + c] = so.vel_[d].empty() ? 0.0 : so.vel_[d][c];
}

int h3o_initialize(void* w, int s) {
  try {
    S(w, s).initialize();
  } catch (...) {
    return -1;
  }
  return 0;
}
int h3o_solve(void* w, int s, int nsteps) {
  for (int i = 0; i < nsteps; ++i) S(w, s).solve();
  return 0;
}
int h3o_nv(void* w, int s) { return S(w, s).nv; }
int64_t h3o_ncells(void* w, int s) { return S(w, s).size(); }
int64_t h3o_first_ghost(void* w, int s) { return S(w, s).firstGC; }
void h3o_get_state(void* w, int s, int which, double* out) {
  auto& so = S(w, s);
  const int64_t n = so.size();
  for (int v = 0; v < so.nv; ++v) std::memcpy(out + v * n, so.Q[which][v].data(), n * sizeof(double));
}
void h3o_set_state(void* w, int s, int which, const double* in) {
  auto& so = S(w, s);
  const int64_t n = so.size();
  for (int v = 0; v < so.nv; ++v) std::memcpy(so.Q[which][v].data(), in + v * n, n * sizeof(double));
}
void h3o_get_tables(void* w, int s, int64_t* nbrs, double* xc, double* len, int32_t* bc,
                    int64_t* node) {
  auto& so = S(w, s);
  const int64_t n = so.size();
  for (int p = 0; p < 2 * so.nd; ++p) std::memcpy(nbrs + p * n, so.nbr[p].data(), n * 8);
  for (int d = 0; d < so.nd; ++d) std::memcpy(xc + d * n, so.xc[d].data(), n * 8);
  std::memcpy(len, so.len.data(), n * 8);
  std::memcpy(bc, so.bc_idx.data(), n * 4);
  if (node) std::memcpy(node, so.node.data(), n * 8);
}
int64_t h3o_nsubfaces(void* w, int s) {
  auto& so = S(w, s);
  return (int64_t)so.subs.size() >> (so.nd - 1);
}
void h3o_subfaces(void* w, int s, int64_t* out) {
  auto& so = S(w, s);
  std::memcpy(out, so.subs.data(), so.subs.size() * 8);
}
int h3o_partner_cells(void* w, int s, int64_t* out) {
  auto& so = S(w, s);
  for (int64_t g = so.firstGC; g < so.size(); ++g) {
    const int k = so.bcs[so.bc_idx[g]].kind;
    const bool cpl = k == BC_CPL_EULER_EULER || k == BC_CPL_CNS_HEAT || k == BC_CPL_HEAT_CNS ||
                     k == BC_CPL_HEAT_HEAT;
    out[g - so.firstGC] = cpl ? so.partner_cell(g) : k == BC_PERIODIC ? so.periodic_partner[g - so.firstGC] : INV;
  }
  return 0;
}
double h3o_dt(void* w, int s) { return S(w, s).dt_; }
double h3o_time(void* w, int s) { return S(w, s).time_; }
int64_t h3o_step(void* w, int s) { return S(w, s).step_; }
double h3o_min_dt(void* w, int s) { return S(w, s).compute_dt(); }
void h3o_force_dt(void* w, int s, double dt) { S(w, s).force_dt(dt); }
void h3o_apply_bcs(void* w, int s, int which) { S(w, s).apply_bcs(which); }
void h3o_quantities(void* w, int s, double* out) {
  const Params& P = S(w, s).P;
  out[0] = P.T_inf; out[1] = P.rho_inf; out[2] = P.u_inf; out[3] = P.p_inf; out[4] = P.mu_inf;
  out[5] = P.Re0; out[6] = P.gm1; out[7] = P.sOverTref;
}
// coupling::apply (CNS-heat): coupling.hpp:52-63
void h3o_couple_cht(void* w, int cns, int heat, double Tr0) {
  auto& c = S(w, cns);
  auto& h = S(w, heat);
  const double scaling = Tr0 * c.P.Pr0 * c.P.Re0;
  const double min_dt_cns = c.compute_dt();
  const double min_dt_heat = h.compute_dt() / scaling;
  const double dt = std::min(min_dt_cns, min_dt_heat);
  c.force_dt(dt);
  h.force_dt(dt * scaling);
}
// coupling::apply (equal solvers): coupling.hpp:66-73
void h3o_couple_equal(void* w, int a, int b) {
  const double da = S(w, a).compute_dt(), db = S(w, b).compute_dt();
  const double dt = std::min(da, db);
  S(w, a).force_dt(dt);
  S(w, b).force_dt(dt);
}
typedef struct {
  int physics, flux, ti, nd, n_bcs;
  double cfl, cfl_viscous, gamma, Rspecific, T0, rho0, Minfty, ReInfty, Pr0, Sutherland0, time_end;
  int bc_kind[16];
  double bc_v[16][8];
  int recon;
  double limiter_k;
} h3o_info;

void h3o_solver_info(void* w, int s, h3o_info* o) {
  auto& so = S(w, s);
  const Params& P = so.P;
  o->physics = P.physics; o->flux = P.flux; o->ti = P.ti; o->nd = so.nd;
  o->n_bcs = (int)so.bcs.size();
  o->cfl = P.cfl; o->cfl_viscous = P.cfl_viscous; o->gamma = P.gamma; o->Rspecific = P.Rspecific;
  o->T0 = P.T0; o->rho0 = P.rho0; o->Minfty = P.Minfty; o->ReInfty = P.ReInfty; o->Pr0 = P.Pr0;
  o->Sutherland0 = P.Sutherland0; o->time_end = P.time_end;
  o->recon = P.recon;
  o->limiter_k = P.limiter_k;
  for (int k = 0; k < (int)so.bcs.size() && k < 16; ++k) {
    o->bc_kind[k] = so.bcs[k].kind;
    for (int j = 0; j < 8; ++j) o->bc_v[k][j] = so.bcs[k].v[j];
  }
}

// ---- forward-mode derivative build (Solver<Dual>): same grid and physics, the
// state carries a direction; steps run with frozen time steps ----
using WD = World<Dual>;
// a derivative twin of solver s of world w: same tree, description and initial state
void* h3o_dual_clone(void* w, int s) {
  W* src = (W*)w;
  const Solver<double>& so = *src->solvers[s];
  auto* wd = new WD();
  wd->nd = src->nd;
  wd->tree.reset(new Tree(*src->tree));
  wd->tree->node2cell.assign(1, std::vector<Ind>(wd->tree->size(), INV));
  auto d = std::make_unique<Solver<Dual>>();
  d->w = wd;
  d->idx = 0;
  d->nd = so.nd;
  d->nv = so.nv;
  d->P = so.P;
  d->bcs = so.bcs;
  d->domain_kind = so.domain_kind;
  d->domain = so.domain;
  d->ic_kind = so.ic_kind;
  std::memcpy(d->ic, so.ic, sizeof(d->ic));
  wd->solvers.push_back(std::move(d));
  return wd;
}
void h3o_dual_world_destroy(void* w) { delete (WD*)w; }
int h3o_dual_initialize(void* w) {
  try { ((WD*)w)->solvers[0]->initialize(); } catch (...) { return -1; }
  return 0;
}
void h3o_dual_set_state(void* w, const double* val, const double* dot) {
  auto& so = *((WD*)w)->solvers[0];
  const int64_t n = so.size();
  for (int v = 0; v < so.nv; ++v)
    for (int64_t c = 0; c < n; ++c) so.Q[0][v][c] = Dual(val[v * n + c], dot[v * n + c]);
}
void h3o_dual_get_state(void* w, double* val, double* dot) {
  auto& so = *((WD*)w)->solvers[0];
  const int64_t n = so.size();
  for (int v = 0; v < so.nv; ++v)
    for (int64_t c = 0; c < n; ++c) { val[v * n + c] = so.Q[0][v][c].v; dot[v * n + c] = so.Q[0][v][c].d; }
}
void h3o_dual_solve_dt(void* w, int nsteps, const double* dts) {
  auto& so = *((WD*)w)->solvers[0];
  for (int i = 0; i < nsteps; ++i) {
    so.force_dt(Dual(dts[i]));
    so.solve();
  }
}
int64_t h3o_dual_ncells(void* w) { return ((WD*)w)->solvers[0]->size(); }

int h3o_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void h3o_set_num_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}
}
