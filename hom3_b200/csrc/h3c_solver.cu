// h3c_solver.cu -- host side of the C ABI declared in include/h3c.h.
//
// Takes hom3's cell container (caller numbering), renumbers interior cells
// along a Morton curve, uploads int32 SoA neighbour tables and per-ghost
// boundary tables, and drives the step kernels of fv_kernels.cuh on the
// solver's stream.  The step scalars (dt, time, step, forced dt) live on the
// device so a run of steps never waits for the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include "vtk_writer.hpp"
#include "grid_build.hpp"

#include <nvtx3/nvToolsExt.h>

#include "../../include/h3c.h"
#include "fv_kernels.cuh"
#include "adjoint_kernels.cuh"
#include "muscl_kernels.cuh"
#include "muscl_adjoint.cuh"
#include "cns_adjoint.cuh"
#include "stage_halo.hpp"
#include "stage_warp.hpp"

using namespace h3c;

namespace {
std::string g_last_error;  // errors not tied to a solver (NULL handle)

constexpr long long kForcedNone = std::numeric_limits<long long>::max();

// An NVTX range over a host call (visible to nsys / ncu range filters; a no-op without a tool attached).
struct Range {
  explicit Range(const char* name) { nvtxRangePushA(name); }
  ~Range() { nvtxRangePop(); }
};

// An instantiated graph of solver steps and the lhs buffer its capture started from.
struct StepGraph {
  cudaGraphExec_t exec = nullptr;
  const double* q0 = nullptr;
};
}  // namespace

namespace gridb {
void set_global_error(const std::string& msg) { g_last_error = msg; }
}  // namespace gridb

struct h3c_solver_s {
  h3c_desc desc{};
  int nd = 2, nv = 4;
  PhysConst pc{};
  double Re0 = 1, Pr0 = 1;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  // grid
  bool has_grid = false;
  long long n_int = 0, n_tot = 0, ng = 0, ld = 0, nsub = 0;
  long long n_caller = 0;  // cells in the caller's numbering (all instances)
  int n_inst = 1, sc_count = 1;
  long long ntiles = 0;
  int persist_blocks = 0;  // AUSM stage grid: 0 = one block per tile, else a persistent grid
  int* d_blk_inst = nullptr;
  long long* d_inst_end = nullptr;
  int* d_ginst = nullptr;
  int* d_nbr = nullptr;
  unsigned char* d_lvl = nullptr;
  int* d_sub = nullptr;
  double lens[kMaxLevels] = {0};
  int nlev = 0;
  int* d_gbndry = nullptr;
  unsigned char *d_gpos = nullptr, *d_gapply = nullptr, *d_gown = nullptr;
  double* d_gdx = nullptr;
  int* d_gpartner = nullptr;
  double* d_xc = nullptr;
  double* d_vel = nullptr;  // advection velocity [nd][ld], internal numbering, ghosts included
  bool vel_set = false;
  int n_bcs = 0;
  std::vector<h3c_bc> bcs;
  std::vector<BcParam> h_bcs;
  BcParam* d_bcs = nullptr;
  h3c_solver partner = nullptr;
  const double* partner_override = nullptr;  // partner state the coupling conditions read (adjoint recompute)
  // state
  double* d_q[3] = {nullptr, nullptr, nullptr};  // lhs, rhs, second SSP-RK3 stage
  double* d_slopes = nullptr;
  double* d_stage = nullptr;  // host<->device staging in caller numbering
  long long stage_cap = 0;
  double* d_adj = nullptr;  // adjoint workspace (checkpoints, stage states, cotangents), kept between calls
  size_t adj_cap = 0;
  long long* d_dev2caller = nullptr;
  std::vector<long long> dev2caller, caller2dev;
  Scalars* d_sc = nullptr;
  Scalars* h_sc = nullptr;  // pinned host copy of instance 0's scalars (the per-step dt read-back)
  bool unfused_dt = false;  // a condition rewrites interior cells (vortex)
  bool ghost_unapplied = false;  // some ghost gets no condition (hom3's find_if segments)
  bool needs_partner = false, needs_periodic = false;  // coupling / periodic conditions present
  bool partner_set = false, periodic_set = false;
  bool tile = true;  // Euler stages use the shared-memory tile kernel
  bool cns_adj_dual = false;  // CNS adjoint faces by dual numbers instead of the hand-written reverse
  int halo_cap = 0;           // cap on the Euler halo entries held in shared memory (0: none)
  int euler_kernel = 1;       // Euler/AUSM stage: 0 halo-staged tile, 1 per-lane tile, 2 per cell, 3 warp-tiled,
                              // 4 per-lane tile of 512 cells (3D, one grid)
  int warp_bps = 0;           // resident blocks per SM of the warp-tiled kernel (0: unavailable)
  // halo-staged Euler/AUSM stage (h3c_stage_halo.cu): tables, launch size
  bool halo = true;     // option: use it when its tables exist
  bool halo_ok = false; // tables built for the current grid
  unsigned short* d_lnb = nullptr;
  int *d_hids = nullptr, *d_hoff = nullptr, *d_goff = nullptr;
  unsigned short* d_grp = nullptr;
  int hmax = 0, halo_bps = 0;
  size_t halo_smem = 0;
  double halo_mean = 0;
  int halo_maxh = 0;
  // CNS tile kernel (h3c_stage_cns.cu): its tables reuse d_lnb / d_hids / d_hoff
  bool cns_ok = false;
  int* d_h1end = nullptr;
  unsigned short* d_hnb = nullptr;
  double* d_gsl = nullptr;  // ghost slopes [nd * nv][ngl]
  long long ngl = 0;
  int h1max = 0, cns_bps = 0;
  size_t cns_smem = 0;
  // Captured step graphs replayed by h3c_solve: runs of kGraphSteps steps
  // (graph8) and single steps (graph1), one of each per lhs buffer the
  // capture started from (forward Euler alternates the two buffers).
  StepGraph graph8[2], graph1[2];
  long long graph_per_step = 0;  // kernel launches one captured step holds
  bool plain_done = false;  // a step ran outside capture (kernel attributes are set)
  int stage_next = 0;       // the next part of a step run by parts (h3c_solve_stage); 0 between steps
  // coupled conjugate-heat steps (h3c_cht_solve) captured with the heat partner
  cudaGraphExec_t cpl_graph = nullptr;
  h3c_solver cpl_with = nullptr;
  const double *cpl_q0 = nullptr, *cpl_q0_other = nullptr;
  double cpl_scaling = 0.0;
  long long cpl_launches = 0;
  long long graph_launches = 0;
  bool graphs = true;
  std::string err;
  // launch accounting and optional per-kernel CUDA-event timing (h3c_profile)
  long long launches = 0;
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof_rec;

  int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    err = buf;
    return code;
  }
  int cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return H3C_OK;
    return fail(e == cudaErrorMemoryAllocation ? H3C_E_NOMEM : H3C_E_CUDA, "%s: %s", what,
                cudaGetErrorString(e));
  }
};

#define H3C_CUDA(s, call)                          \
  do {                                             \
    int rc__ = (s)->cuda((call), #call);           \
    if (rc__ != H3C_OK) return rc__;               \
  } while (0)

namespace {

template <class T> void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

void drop_cpl_graph(h3c_solver s) {
  if (s->cpl_graph) cudaGraphExecDestroy(s->cpl_graph);
  s->cpl_graph = nullptr;
  s->cpl_with = nullptr;
}

void drop_graph(h3c_solver s) {
  for (int k = 0; k < 2; ++k)
    for (StepGraph* g : {&s->graph8[k], &s->graph1[k]}) {
      if (g->exec) cudaGraphExecDestroy(g->exec);
      *g = StepGraph{};
    }
  s->plain_done = false;  // the next capture follows a plain step of the current configuration
  // a coupled graph holds this solver's and its partner's buffers
  drop_cpl_graph(s);
  if (s->partner && s->partner->cpl_with == s) drop_cpl_graph(s->partner);
}

void free_grid(h3c_solver s) {
  drop_graph(s);
  s->stage_next = 0;
  dfree(s->d_nbr); dfree(s->d_lvl); dfree(s->d_sub); dfree(s->d_gbndry); dfree(s->d_gpos);
  dfree(s->d_gapply); dfree(s->d_gown); dfree(s->d_gdx); dfree(s->d_gpartner); dfree(s->d_xc);
  dfree(s->d_bcs); dfree(s->d_q[0]); dfree(s->d_q[1]); dfree(s->d_q[2]); dfree(s->d_slopes); dfree(s->d_stage);
  dfree(s->d_dev2caller);
  dfree(s->d_vel);
  s->vel_set = false;
  dfree(s->d_blk_inst); dfree(s->d_inst_end); dfree(s->d_ginst);
  dfree(s->d_lnb); dfree(s->d_hids); dfree(s->d_hoff); dfree(s->d_goff); dfree(s->d_grp);
  dfree(s->d_h1end); dfree(s->d_hnb); dfree(s->d_gsl);
  s->halo_ok = false;
  s->cns_ok = false;
  dfree(s->d_adj);
  s->adj_cap = 0;
  s->stage_cap = 0;
  s->has_grid = false;
}

Geometry geometry(const h3c_solver s) {
  Geometry g;
  g.nbr = s->d_nbr;
  g.lvl = s->d_lvl;
  g.sub = s->d_sub;
  g.nsub = s->nsub;
  g.n_int = s->n_int;
  g.n_tot = s->n_tot;
  g.ld = s->ld;
  for (int i = 0; i < kMaxLevels; ++i) g.len[i] = s->lens[i];
  g.blk_inst = s->n_inst > 1 ? s->d_blk_inst : nullptr;
  g.inst_end = s->n_inst > 1 ? s->d_inst_end : nullptr;
  g.ntiles = s->ntiles;
  g.vel = s->d_vel;
  return g;
}

GhostTables ghosts(const h3c_solver s) {
  GhostTables t;
  t.bndry = s->d_gbndry;
  t.pos = s->d_gpos;
  t.bc_apply = s->d_gapply;
  t.bc_own = s->d_gown;
  t.dx = s->d_gdx;
  t.partner = s->d_gpartner;
  t.xc = s->d_xc;
  t.ginst = s->n_inst > 1 ? s->d_ginst : nullptr;
  t.ng = s->ng;
  t.bcs = s->d_bcs;
  return t;
}

unsigned blocks(long long n) { return (unsigned)std::max<long long>(1, (n + kBlock - 1) / kBlock); }

int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
  }
  return sms;
}

// kernel kinds reported by h3c_profile_read
enum { K_BC = 0, K_CFL = 1, K_SCALAR = 2, K_STAGE1 = 3, K_STAGE2 = 4, K_SLOPES = 5, K_COPY = 6, K_OTHER = 7, K_NKINDS = 8 };

cudaEvent_t take_event(h3c_solver s) {
  cudaEvent_t e;
  if (!s->ev_pool.empty()) {
    e = s->ev_pool.back();
    s->ev_pool.pop_back();
  } else {
    cudaEventCreate(&e);
  }
  return e;
}

// Counts one kernel launch of `kind` and, when profiling, brackets it with
// events on the solver's stream.
struct Launch {
  h3c_solver s;
  int kind;
  cudaEvent_t a = nullptr, b = nullptr;
  Launch(h3c_solver s_, int k) : s(s_), kind(k) {
    s->launches++;
    if (s->prof) {
      a = take_event(s);
      b = take_event(s);
      cudaEventRecord(a, s->stream);
    }
  }
  ~Launch() {
    if (s->prof) {
      cudaEventRecord(b, s->stream);
      s->prof_rec.push_back({kind, {a, b}});
    }
  }
};

// ---- kernel dispatch -------------------------------------------------------
template <int ND, int PHYS>
void launch_bc_t(h3c_solver s, double* q, const double* qlhs) {
  PartnerView pv{nullptr, 0};
  if (s->partner) pv = PartnerView{s->partner_override ? s->partner_override : s->partner->d_q[0], s->partner->ld};
  Launch L(s, K_BC);
  k_bc<ND, PHYS><<<blocks(s->ng), kBlock, 0, s->stream>>>(q, qlhs, geometry(s), ghosts(s), s->pc, s->d_sc, pv);
}
// conditions applied to q; coupling conditions read temperatures from qlhs
void launch_bc_ptr(h3c_solver s, double* q, const double* qlhs) {
  if (s->ng == 0) return;
  if (s->nd == 2) {
    if (s->desc.physics == H3C_EULER) launch_bc_t<2, EULER>(s, q, qlhs);
    else if (s->desc.physics == H3C_CNS) launch_bc_t<2, CNS>(s, q, qlhs);
    else if (s->desc.physics == H3C_ADVECTION) launch_bc_t<2, ADVECTION>(s, q, qlhs);
    else launch_bc_t<2, HEAT>(s, q, qlhs);
  } else {
    if (s->desc.physics == H3C_EULER) launch_bc_t<3, EULER>(s, q, qlhs);
    else if (s->desc.physics == H3C_CNS) launch_bc_t<3, CNS>(s, q, qlhs);
    else if (s->desc.physics == H3C_ADVECTION) launch_bc_t<3, ADVECTION>(s, q, qlhs);
    else launch_bc_t<3, HEAT>(s, q, qlhs);
  }
}
void launch_bc(h3c_solver s, int which) { launch_bc_ptr(s, s->d_q[which], s->d_q[0]); }

template <int ND, int PHYS>
void launch_cfl_t(h3c_solver s, long long* slot) {
  Launch L(s, K_CFL);
  k_cfl<ND, PHYS><<<blocks(s->n_int), kBlock, 0, s->stream>>>(s->d_q[0], geometry(s), s->pc, slot, s->d_sc);
}
void launch_cfl(h3c_solver s, long long* slot) {
  if (s->desc.physics == H3C_ADVECTION && !s->vel_set) return;  // no velocity yet: no time step
  {
    Launch L(s, K_SCALAR);
    k_reset_slot<<<blocks(s->n_inst), kBlock, 0, s->stream>>>(slot, s->n_inst);
  }
  if (s->nd == 2) {
    if (s->desc.physics == H3C_EULER) launch_cfl_t<2, EULER>(s, slot);
    else if (s->desc.physics == H3C_CNS) launch_cfl_t<2, CNS>(s, slot);
    else if (s->desc.physics == H3C_ADVECTION) launch_cfl_t<2, ADVECTION>(s, slot);
    else launch_cfl_t<2, HEAT>(s, slot);
  } else {
    if (s->desc.physics == H3C_EULER) launch_cfl_t<3, EULER>(s, slot);
    else if (s->desc.physics == H3C_CNS) launch_cfl_t<3, CNS>(s, slot);
    else if (s->desc.physics == H3C_ADVECTION) launch_cfl_t<3, ADVECTION>(s, slot);
    else launch_cfl_t<3, HEAT>(s, slot);
  }
}

void launch_slopes_ptr(h3c_solver s, const double* q) {
  Launch L(s, K_SLOPES);
  if (s->nd == 2)
    k_slopes<2><<<blocks(s->n_tot), kBlock, 0, s->stream>>>(q, geometry(s), ghosts(s), s->d_slopes);
  else
    k_slopes<3><<<blocks(s->n_tot), kBlock, 0, s->stream>>>(q, geometry(s), ghosts(s), s->d_slopes);
}

void launch_slopes(h3c_solver s, int which) {
  Launch L(s, K_SLOPES);
  if (s->nd == 2)
    k_slopes<2><<<blocks(s->n_tot), kBlock, 0, s->stream>>>(s->d_q[which], geometry(s), ghosts(s), s->d_slopes);
  else
    k_slopes<3><<<blocks(s->n_tot), kBlock, 0, s->stream>>>(s->d_q[which], geometry(s), ghosts(s), s->d_slopes);
}

// EXTENSION: limited least-squares gradients of the stage input (MUSCL)
void launch_grad(h3c_solver s, const double* q) {
  Launch L(s, K_SLOPES);
  const double K = s->desc.limiter_k;
  if (s->nd == 2) {
    if (s->nsub > 0) k_muscl_grad<2, true><<<blocks(s->n_int), kBlock, 0, s->stream>>>(q, s->d_xc, geometry(s), s->pc, K, s->d_slopes);
    else k_muscl_grad<2, false><<<blocks(s->n_int), kBlock, 0, s->stream>>>(q, s->d_xc, geometry(s), s->pc, K, s->d_slopes);
    if (s->needs_periodic) k_muscl_ghosts<2><<<blocks(s->ng), kBlock, 0, s->stream>>>(s->d_slopes, geometry(s), ghosts(s));
  } else {
    if (s->nsub > 0) k_muscl_grad<3, true><<<blocks(s->n_int), kBlock, 0, s->stream>>>(q, s->d_xc, geometry(s), s->pc, K, s->d_slopes);
    else k_muscl_grad<3, false><<<blocks(s->n_int), kBlock, 0, s->stream>>>(q, s->d_xc, geometry(s), s->pc, K, s->d_slopes);
    if (s->needs_periodic) k_muscl_ghosts<3><<<blocks(s->ng), kBlock, 0, s->stream>>>(s->d_slopes, geometry(s), ghosts(s));
  }
}

template <int ND, int PHYS, int FLUX, class R, int MODE, bool HANG, bool FUSE>
void stage_t(h3c_solver s, const double* qin, double* out) {
  Launch L(s, MODE == 0 ? K_STAGE1 : K_STAGE2);
  if (PHYS == EULER && FLUX == AUSM && s->desc.reconstruction == H3C_RECON_MUSCL) {
    k_stage_muscl<ND, R, MODE, HANG, FUSE><<<blocks(s->n_int), kBlock, 0, s->stream>>>(
        qin, out, s->d_slopes, s->d_xc, geometry(s), s->pc, s->d_sc, &s->d_sc->dtmin_ord);
    return;
  }
  if (PHYS == CNS && s->tile && s->halo && s->cns_ok) {
    int grid = s->persist_blocks > 0 ? s->persist_blocks : s->cns_bps * num_sms();
    grid = (int)std::max<long long>(1, std::min<long long>(grid, s->ntiles));
    const CnsHaloGeom ch{HaloGeom{s->d_lnb, s->d_hids, s->d_hoff, s->d_grp, s->d_goff, s->hmax}, s->d_h1end, s->d_hnb,
                         s->d_gsl, s->ngl, s->h1max};
    if (s->ng > 0) s->launches++;  // the ghost-slope pass
    cns_halo_stage(ND, std::is_same<R, float>::value, MODE, FUSE, qin, out, geometry(s), ghosts(s), ch, s->pc,
                   s->d_sc, &s->d_sc->dtmin_ord, &s->d_sc->status, grid, s->cns_smem, s->stream, s->d_gsl);
    return;
  }
  if (PHYS == EULER && FLUX == AUSM && s->tile && s->euler_kernel == 3 && s->warp_bps > 0) {
    warp_stage(ND, std::is_same<R, float>::value, MODE, HANG, FUSE, qin, out, geometry(s), s->pc, s->d_sc,
               &s->d_sc->dtmin_ord, s->stream);
    return;
  }
  if (PHYS == EULER && FLUX == AUSM && s->tile && (s->euler_kernel == 2 || s->euler_kernel == 3)) {  // per cell
    k_stage_ausm_cell<ND, R, MODE, HANG, FUSE><<<blocks(s->n_int), kBlock, 0, s->stream>>>(
        qin, out, geometry(s), s->pc, s->d_sc, &s->d_sc->dtmin_ord);
    return;
  }
  if (PHYS == EULER && FLUX == AUSM && s->tile && s->halo && s->halo_ok && s->euler_kernel == 0) {
    int grid = s->persist_blocks > 0 ? s->persist_blocks : s->halo_bps * num_sms();
    grid = (int)std::max<long long>(1, std::min<long long>(grid, s->ntiles));
    HaloGeom hg{s->d_lnb, s->d_hids, s->d_hoff, s->d_grp, s->d_goff, s->hmax};
    halo_stage(ND, std::is_same<R, float>::value, MODE, HANG, FUSE, qin, out, geometry(s), hg, s->pc, s->d_sc,
               &s->d_sc->dtmin_ord, &s->d_sc->status, grid, s->halo_smem, s->stream);
    return;
  }
  if constexpr (ND == 3) {
    if (PHYS == EULER && FLUX == AUSM && s->tile && s->euler_kernel == 4 && s->n_inst == 1) {
      // 512-cell tiles (8x8x8 Morton bricks), two blocks of 512 threads per SM
      constexpr int TB = 512;
      constexpr size_t smem = ausm_smem_bytes<R, ND, TB>();
      static bool attr = false;  // one opt-in per instantiation (dynamic smem above 48 KB)
      if (!attr) {
        cudaFuncSetAttribute(k_stage_ausm<ND, R, MODE, HANG, FUSE, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        attr = true;
      }
      Geometry g = geometry(s);
      g.ntiles = (s->n_int + TB - 1) / TB;
      const long long grid = s->persist_blocks > 0 ? std::min<long long>(s->persist_blocks, g.ntiles) : g.ntiles;
      k_stage_ausm<ND, R, MODE, HANG, FUSE, TB><<<(unsigned)std::max<long long>(1, grid), TB, smem, s->stream>>>(
          qin, out, g, s->pc, s->d_sc, &s->d_sc->dtmin_ord);
      return;
    }
  }
  if (PHYS == EULER && FLUX == AUSM && s->tile) {
    constexpr size_t smem = ausm_smem_bytes<R, ND>();
    static bool attr = false;  // one opt-in per instantiation (dynamic smem above 48 KB)
    if (!attr) {
      cudaFuncSetAttribute(k_stage_ausm<ND, R, MODE, HANG, FUSE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      attr = true;
    }
    const long long grid = s->persist_blocks > 0 ? std::min<long long>(s->persist_blocks, s->ntiles) : s->ntiles;
    k_stage_ausm<ND, R, MODE, HANG, FUSE><<<(unsigned)std::max<long long>(1, grid), kBlock, smem, s->stream>>>(
        qin, out, geometry(s), s->pc, s->d_sc, &s->d_sc->dtmin_ord);
    return;
  }
  if (PHYS == EULER && s->tile) {
    constexpr size_t smem = tile_smem_bytes<R, ND>();
    static bool attr = false;  // one opt-in per instantiation (dynamic smem above 48 KB)
    if (!attr) {
      cudaFuncSetAttribute(k_stage_tile<ND, FLUX, R, MODE, HANG, FUSE>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      attr = true;
    }
    k_stage_tile<ND, FLUX, R, MODE, HANG, FUSE><<<blocks(s->n_int), kBlock, smem, s->stream>>>(
        qin, out, geometry(s), s->pc, s->d_sc, &s->d_sc->dtmin_ord);
    return;
  }
  k_stage<ND, PHYS, FLUX, R, MODE, HANG, FUSE><<<blocks(s->n_int), kBlock, 0, s->stream>>>(
      qin, out, s->d_slopes, geometry(s), s->pc, s->d_sc, &s->d_sc->dtmin_ord);
}
// Euler adjoint stage in the tile kernel (one block per Morton tile)
template <int ND, bool HANG>
static void adj_ausm_t(h3c_solver s, const double* qin, const double* lamin, double* gout, const double* extra,
                       const double* extra2, double alpha, double beta, double gam, double gam2) {
  constexpr size_t smem = adj_ausm_smem_bytes<ND>();
  static bool attr = false;  // one opt-in per instantiation (dynamic smem above 48 KB)
  if (!attr) {
    cudaFuncSetAttribute(k_adj_ausm<ND, HANG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr = true;
  }
  k_adj_ausm<ND, HANG><<<(unsigned)std::max<long long>(1, s->ntiles), kBlock, smem, s->stream>>>(
      qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2, geometry(s), ghosts(s), s->pc, s->d_sc);
}

template <int ND, int PHYS, int FLUX, class R, int MODE, bool HANG>
void stage_f(h3c_solver s, const double* qin, double* out, bool fuse) {
  if (fuse) stage_t<ND, PHYS, FLUX, R, MODE, HANG, true>(s, qin, out);
  else stage_t<ND, PHYS, FLUX, R, MODE, HANG, false>(s, qin, out);
}
template <int ND, int PHYS, int FLUX, class R, int MODE>
void stage_h(h3c_solver s, const double* qin, double* out, bool fuse) {
  if (PHYS != CNS && s->nsub > 0) stage_f<ND, PHYS, FLUX, R, MODE, PHYS != CNS>(s, qin, out, fuse);
  else stage_f<ND, PHYS, FLUX, R, MODE, false>(s, qin, out, fuse);
}
template <int ND, int PHYS, int FLUX, class R>
void stage_m(h3c_solver s, int mode, const double* qin, double* out, bool fuse) {
  if (mode == 0) stage_h<ND, PHYS, FLUX, R, 0>(s, qin, out, fuse);
  else if (mode == 2) stage_h<ND, PHYS, FLUX, R, 2>(s, qin, out, fuse);
  else if (mode == 3) stage_h<ND, PHYS, FLUX, R, 3>(s, qin, out, fuse);
  else stage_h<ND, PHYS, FLUX, R, 4>(s, qin, out, fuse);
}
template <int ND>
void stage_nd(h3c_solver s, int mode, const double* qin, double* out, bool fuse) {
  const bool mixed = s->desc.precision == H3C_MIXED;
  switch (s->desc.physics) {
    case H3C_EULER:
      if (s->desc.flux == H3C_FLUX_LLF) {
        if (mixed) stage_m<ND, EULER, LLF, float>(s, mode, qin, out, fuse);
        else stage_m<ND, EULER, LLF, double>(s, mode, qin, out, fuse);
      } else {
        if (mixed) stage_m<ND, EULER, AUSM, float>(s, mode, qin, out, fuse);
        else stage_m<ND, EULER, AUSM, double>(s, mode, qin, out, fuse);
      }
      break;
    case H3C_CNS:
      if (mixed) stage_m<ND, CNS, AUSM, float>(s, mode, qin, out, fuse);
      else stage_m<ND, CNS, AUSM, double>(s, mode, qin, out, fuse);
      break;
    case H3C_ADVECTION:
      if (s->desc.flux == H3C_FLUX_LLF) stage_m<ND, ADVECTION, LLF, double>(s, mode, qin, out, fuse);
      else stage_m<ND, ADVECTION, UPWIND, double>(s, mode, qin, out, fuse);
      break;
    default:
      stage_m<ND, HEAT, AUSM, double>(s, mode, qin, out, fuse);
  }
}
void launch_stage(h3c_solver s, int mode, const double* qin, double* out, bool fuse) {
  if (s->nd == 2) stage_nd<2>(s, mode, qin, out, fuse);
  else stage_nd<3>(s, mode, qin, out, fuse);
}

__global__ void k_init_time(Scalars* sc0, double tEnd, int n_inst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  Scalars* sc = sc0 + i;
  sc->dt = 0;
  sc->time = 0;
  sc->tEnd = tEnd;
  sc->forced_dt = 0;
  sc->step = 0;
  sc->forced_step = 0x7fffffffffffffffLL;
  sc->dtmin_ord = kOrdMax;
  sc->mindt_ord = kOrdMax;
  sc->status = 0;
}
__global__ void k_force_dt(Scalars* sc, double dt) {
  sc->forced_step = sc->step;
  sc->forced_dt = dt;
}
// coupling::apply(Tr0, cns, heat): coupling.hpp:52-63
__global__ void k_couple_cht(Scalars* cns, Scalars* heat, double scaling) {
  const double min_dt_cns = ord_to_dbl(cns->mindt_ord);
  const double min_dt_heat = ord_to_dbl(heat->mindt_ord) / scaling;
  const double dt = (min_dt_heat < min_dt_cns) ? min_dt_heat : min_dt_cns;  // std::min
  cns->forced_step = cns->step;
  cns->forced_dt = dt;
  heat->forced_step = heat->step;
  heat->forced_dt = dt * scaling;
}
// coupling::apply(s1, s2): coupling.hpp:66-73
__global__ void k_couple_equal(Scalars* a, Scalars* b) {
  const double da = ord_to_dbl(a->mindt_ord), db = ord_to_dbl(b->mindt_ord);
  const double dt = (db < da) ? db : da;
  a->forced_step = a->step;
  a->forced_dt = dt;
  b->forced_step = b->step;
  b->forced_dt = dt;
}

// Morton key of an interior cell's lower corner in units of the finest cell
// (x in the lowest bit: hom3's child positions, grid/grid.hpp:41-59).
uint64_t morton(const long long* ix, int nd) {
  uint64_t k = 0;
  const int bits = nd == 2 ? 31 : 21;
  for (int b = 0; b < bits; ++b)
    for (int d = 0; d < nd; ++d) k |= (uint64_t)((ix[d] >> b) & 1) << (b * nd + d);
  return k;
}

int valid_cell(long long v, long long n) { return v >= 0 && v < n; }

}  // namespace

// ============================================================================
extern "C" {

int h3c_last_error(h3c_solver s, char* buf, size_t n) {
  const std::string& e = s ? s->err : g_last_error;
  if (buf && n) {
    std::strncpy(buf, e.c_str(), n - 1);
    buf[n - 1] = 0;
  }
  return (int)e.size();
}

int h3c_create(const h3c_desc* d, h3c_solver* out) {
  if (!d || !out) { g_last_error = "h3c_create: null argument"; return H3C_E_INVALID; }
  if (d->nd != 2 && d->nd != 3) { g_last_error = "h3c_create: nd must be 2 or 3"; return H3C_E_INVALID; }
  if (d->physics < 0 || d->physics > 3 || d->flux < 0 || d->flux > 2 || d->time_integration < 0 ||
      d->time_integration > 2 || d->precision < 0 || d->precision > 1 || d->reconstruction < 0 ||
      d->reconstruction > 1) {
    g_last_error = "h3c_create: unknown physics / flux / time integration / precision";
    return H3C_E_INVALID;
  }
  if (d->reconstruction == H3C_RECON_MUSCL && (d->physics != H3C_EULER || d->flux != H3C_FLUX_AUSM)) {
    g_last_error = "h3c_create: MUSCL reconstruction is implemented for Euler with the AUSM flux";
    return H3C_E_INVALID;
  }
  if (d->physics == H3C_CNS && d->flux != H3C_FLUX_AUSM) {
    g_last_error = "h3c_create: CNS supports the standard flux (AUSM + three-point) only";
    return H3C_E_INVALID;
  }
  if ((d->physics == H3C_ADVECTION) != (d->flux == H3C_FLUX_UPWIND) &&
      !(d->physics == H3C_ADVECTION && d->flux == H3C_FLUX_LLF)) {
    g_last_error = "h3c_create: advection takes the upwind or LLF flux (advection/tags.hpp:14-15); "
                   "the upwind flux is advection's";
    return H3C_E_INVALID;
  }
  auto s = std::make_unique<h3c_solver_s>();
  s->desc = *d;
  s->nd = d->nd;
  s->nv = (d->physics == H3C_HEAT || d->physics == H3C_ADVECTION) ? 1 : d->nd + 2;
  // quantities: euler/quantities.hpp:131-145, cns/quantities.hpp:28-30, 74-75
  const double gamma = d->gamma, gm1 = gamma - 1.;
  const double T_inf = 1.0 / (1 + 0.5 * gm1 * (d->Minfty * d->Minfty));
  const double rho_inf = std::pow(T_inf, 1. / gm1);
  const double u_inf = d->Minfty * std::sqrt(T_inf);
  const double sOverTref = d->T0 > 0 ? d->Sutherland0 / d->T0 : 0.0;
  const double sOverTrefP1 = sOverTref + 1.0;
  const double mu_inf = std::pow(T_inf, 1.5) * sOverTrefP1 / (T_inf + sOverTref);
  s->Re0 = d->physics == H3C_CNS ? d->ReInfty * mu_inf / (rho_inf * u_inf) : 1.0;
  s->Pr0 = d->Pr0;
  s->pc = PhysConst{gamma, gm1, d->cfl, d->cfl_viscous, s->Re0, d->Pr0, sOverTref, sOverTrefP1};
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    g_last_error = std::string("h3c_create: cudaStreamCreate: ") + cudaGetErrorString(e);
    return H3C_E_CUDA;
  }
  e = cudaMalloc(&s->d_sc, sizeof(Scalars));
  if (e != cudaSuccess) {
    cudaStreamDestroy(s->stream);
    g_last_error = std::string("h3c_create: cudaMalloc: ") + cudaGetErrorString(e);
    return H3C_E_NOMEM;
  }
  // a direct DMA target for the step scalars (a pageable one is staged by the driver)
  if (cudaMallocHost(&s->h_sc, sizeof(Scalars)) != cudaSuccess) {
    cudaGetLastError();
    s->h_sc = nullptr;
  }
  k_init_time<<<1, 1, 0, s->stream>>>(s->d_sc, d->time_end, 1);
  *out = s.release();
  return H3C_OK;
}

int h3c_destroy(h3c_solver s) {
  if (!s) return H3C_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  free_grid(s);
  dfree(s->d_sc);
  if (s->h_sc) cudaFreeHost(s->h_sc);
  for (auto& r : s->prof_rec) { cudaEventDestroy(r.second.first); cudaEventDestroy(r.second.second); }
  for (auto e : s->ev_pool) cudaEventDestroy(e);
  if (s->stream && s->own_stream) cudaStreamDestroy(s->stream);
  delete s;
  return H3C_OK;
}

// Per-instance table preparation shared by h3c_set_grid / h3c_set_grids.
struct InstanceTables {
  long long n = 0, fg = 0, ld = 0, nsub = 0;
  std::vector<long long> order;          // interior cells in Morton order (caller numbering)
  std::vector<int> gb, gbp;              // ghost -> boundary cell, boundary position
  std::vector<unsigned char> apply, own; // per ghost, local bc indices (255: none)
};

static int prepare_instance(h3c_solver s, int k, const h3c_grid* gr, InstanceTables& T) {
  const int nd = s->nd, np = 2 * nd;
  const long long n = gr->n_cells, fg = gr->first_ghost, ld = gr->ld;
  if (n <= 0 || fg <= 0 || fg > n || ld < n || !gr->neighbors || !gr->x_center || !gr->length || !gr->bc_idx)
    return s->fail(H3C_E_INVALID, "h3c_set_grid: instance %d: bad sizes or null tables", k);
  if (n >= (1LL << 31)) return s->fail(H3C_E_INVALID, "h3c_set_grid: more than 2^31 cells");
  if (gr->n_bcs < 0 || gr->n_bcs > kMaxBcs || (gr->n_bcs > 0 && !gr->bcs))
    return s->fail(H3C_E_INVALID, "h3c_set_grid: n_bcs must be in [0, %d]", kMaxBcs);
  const long long nsub = gr->subface_cells ? gr->n_subfaces : 0;
  if (nsub > 0 && s->desc.physics == H3C_CNS)
    return s->fail(H3C_E_INVALID, "h3c_set_grid: coarse/fine faces are not supported for CNS");
  const int nsubc = 1 << (nd - 1);
  auto nb = [&](int p, long long c) { return gr->neighbors[p * ld + c]; };
  auto is_group = [&](long long v) { return nsub > 0 && v <= -2 && (-v - 2) < nsub; };
  for (long long c = 0; c < fg; ++c) {
    for (int p = 0; p < np; ++p) {
      const long long v = nb(p, c);
      if (!valid_cell(v, n) && !is_group(v))
        return s->fail(H3C_E_INVALID, "h3c_set_grid: internal cell %lld has no neighbour at position %d", c, p);
    }
    if (!(gr->length[c] > 0)) return s->fail(H3C_E_INVALID, "h3c_set_grid: cell %lld has length <= 0", c);
  }
  T.gb.assign(n - fg, 0);
  T.gbp.assign(n - fg, 0);
  for (long long g = fg; g < n; ++g) {
    int cnt = 0, first = -1;
    for (int p = 0; p < np; ++p)
      if (valid_cell(nb(p, g), n)) { ++cnt; if (first < 0) first = p; }
    if (cnt != 1)
      return s->fail(H3C_E_INVALID, "h3c_set_grid: ghost %lld has %d neighbours (expected 1)", g, cnt);
    const long long b = nb(first, g);
    if (b >= fg) return s->fail(H3C_E_INVALID, "h3c_set_grid: ghost %lld is linked to ghost %lld", g, b);
    T.gb[g - fg] = (int)b;
    T.gbp[g - fg] = first;
    const int bc = gr->bc_idx[g];
    if (bc < 0 || bc >= gr->n_bcs)
      return s->fail(H3C_E_INVALID, "h3c_set_grid: ghost %lld has bc index %d (n_bcs %d)", g, bc, gr->n_bcs);
  }
  for (long long q = 0; q < nsub; ++q)
    for (int j = 0; j < nsubc; ++j) {
      const long long v = gr->subface_cells[j * nsub + q];
      if (!valid_cell(v, n)) return s->fail(H3C_E_INVALID, "h3c_set_grid: sub-face %lld has an invalid cell", q);
    }
  // Morton order of interior cells (lower corners in units of the finest cell)
  double xmin[3] = {1e300, 1e300, 1e300};
  double hmin = 1e300;
  for (long long c = 0; c < fg; ++c) hmin = std::min(hmin, gr->length[c]);
  for (long long c = 0; c < fg; ++c)
    for (int d = 0; d < nd; ++d) xmin[d] = std::min(xmin[d], gr->x_center[d * ld + c] - 0.5 * gr->length[c]);
  std::vector<std::pair<uint64_t, long long>> keys(fg);
  for (long long c = 0; c < fg; ++c) {
    long long ix[3] = {0, 0, 0};
    for (int d = 0; d < nd; ++d)
      ix[d] = std::llround((gr->x_center[d * ld + c] - 0.5 * gr->length[c] - xmin[d]) / hmin);
    keys[c] = {morton(ix, nd), c};
  }
  std::stable_sort(keys.begin(), keys.end(),
                   [](const std::pair<uint64_t, long long>& a, const std::pair<uint64_t, long long>& b) {
                     return a.first < b.first;
                   });
  T.order.resize(fg);
  for (long long c = 0; c < fg; ++c) T.order[c] = keys[c].second;
  // hom3's bc segment discovery (solver.hpp:561-586)
  T.apply.assign(n - fg, 255);
  T.own.assign(n - fg, 0);
  auto valid_bc = [&](long long c) { return gr->bc_idx[c] >= 0 && gr->bc_idx[c] < gr->n_bcs; };
  long long first = 0;
  while (first < n && !valid_bc(first)) ++first;
  if (first < n) {
    int bcIdx = gr->bc_idx[first];
    long long last = 0;
    while (last < n && gr->bc_idx[last] != bcIdx) ++last;
    for (int q = 0; q < gr->n_bcs; ++q) {
      ++bcIdx;
      const long long f0 = last;
      last = f0;
      while (last < n && gr->bc_idx[last] != bcIdx) ++last;
      for (long long c = std::max(f0, fg); c < last; ++c) T.apply[c - fg] = (unsigned char)q;
    }
  }
  for (long long g = fg; g < n; ++g) T.own[g - fg] = (unsigned char)gr->bc_idx[g];
  T.n = n;
  T.fg = fg;
  T.ld = ld;
  T.nsub = nsub;
  return H3C_OK;
}

// Every index the stage, condition and CFL kernels read through, checked on
// the device after upload (the tables are renumbered on the host, so this
// checks that step): neighbour entries of interior cells (not the padding
// between the instances of a batch, dev2caller < 0) are cells or
// sub-face groups, group members and ghosts' boundary cells are cells, level
// bytes index the length table, halo-list entries (their cell bits,
// hid_mask) are cells.  bad[0] counts violations; the kernels never index
// through an unchecked table.
__global__ void k_check_tables(const int* __restrict__ nbr, const int* __restrict__ sub,
                               const int* __restrict__ gbndry, const unsigned char* __restrict__ lvl,
                               const int* __restrict__ hids, int hid_mask, long long nhids,
                               const long long* __restrict__ dev2caller, long long n_int, long long n_tot,
                               long long ld, long long nsub, int np, int nsubc, long long ng, int nlev,
                               unsigned long long* bad) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long b = 0;
  if (i < n_int && dev2caller[i] >= 0) {
    for (int p = 0; p < np; ++p) {
      const long long v = nbr[p * ld + i];
      b += !((v >= 0 && v < n_tot) || (v <= -2 && -v - 2 < nsub));
    }
    b += lvl[i] >= nlev;
  }
  if (i < nsub)
    for (int j = 0; j < nsubc; ++j) b += !(sub[j * nsub + i] >= 0 && sub[j * nsub + i] < n_tot);
  if (i < ng) b += !(gbndry[i] >= 0 && gbndry[i] < n_int);
  if (i < nhids) {
    const int h = hids[i] & hid_mask;
    b += !(hids[i] >= 0 && h < n_tot);
  }
  if (b) atomicAdd(bad, b);
}

static int set_grids(h3c_solver s, int ninst, const h3c_grid* grids) {
  if (!s || !grids || ninst < 1) return H3C_E_INVALID;
  Range r("h3c_set_grid");
  const int nd = s->nd, np = 2 * nd, nsubc = 1 << (nd - 1);
  std::vector<InstanceTables> T(ninst);
  for (int k = 0; k < ninst; ++k)
    if (int rc = prepare_instance(s, k, &grids[k], T[k])) return rc;
  // ---- merged conditions (identical conditions of different instances share one entry) ----
  std::vector<h3c_bc> ubcs;
  std::vector<std::vector<unsigned char>> bcmap(ninst);
  for (int k = 0; k < ninst; ++k) {
    for (int q = 0; q < grids[k].n_bcs; ++q) {
      const h3c_bc& b = grids[k].bcs[q];
      int found = -1;
      for (size_t u = 0; u < ubcs.size(); ++u)
        if (ubcs[u].kind == b.kind && std::memcmp(ubcs[u].v, b.v, sizeof(b.v)) == 0) { found = (int)u; break; }
      if (found < 0) {
        if ((int)ubcs.size() == kMaxBcs)
          return s->fail(H3C_E_INVALID, "h3c_set_grids: more than %d distinct conditions", kMaxBcs);
        ubcs.push_back(b);
        found = (int)ubcs.size() - 1;
      }
      bcmap[k].push_back((unsigned char)found);
    }
  }
  // ---- lengths -> level table ----
  std::vector<double> lens;
  for (int k = 0; k < ninst; ++k)
    for (long long c = 0; c < T[k].n; ++c) {
      const double l = grids[k].length[c];
      if (std::find(lens.begin(), lens.end(), l) == lens.end()) {
        if ((int)lens.size() == kMaxLevels)
          return s->fail(H3C_E_INVALID, "h3c_set_grid: more than %d distinct cell lengths", kMaxLevels);
        lens.push_back(l);
      }
    }
  std::sort(lens.begin(), lens.end(), std::greater<double>());
  // ---- device layout: interior ranges 256-aligned per instance, then all ghosts ----
  std::vector<long long> int_start(ninst), int_end(ninst), ghost_start(ninst), caller_off(ninst), sub_off(ninst);
  long long cur = 0, ncaller = 0, nsub = 0, ng = 0;
  for (int k = 0; k < ninst; ++k) {
    if (k > 0) cur = (cur + kBlock - 1) / kBlock * kBlock;
    int_start[k] = cur;
    cur += T[k].fg;
    int_end[k] = cur;
    caller_off[k] = ncaller;
    ncaller += T[k].n;
    sub_off[k] = nsub;
    nsub += T[k].nsub;
    ng += T[k].n - T[k].fg;
  }
  const long long n_int = cur;
  for (int k = 0; k < ninst; ++k) {
    ghost_start[k] = cur;
    cur += T[k].n - T[k].fg;
  }
  const long long n_tot = cur;
  if (n_tot >= (1LL << 31)) return s->fail(H3C_E_INVALID, "h3c_set_grids: more than 2^31 cells");
  std::vector<long long> dev2caller(n_tot, -1), caller2dev(ncaller, -1);
  for (int k = 0; k < ninst; ++k) {
    for (long long i = 0; i < T[k].fg; ++i) dev2caller[int_start[k] + i] = caller_off[k] + T[k].order[i];
    for (long long g = T[k].fg; g < T[k].n; ++g) dev2caller[ghost_start[k] + g - T[k].fg] = caller_off[k] + g;
  }
  for (long long i = 0; i < n_tot; ++i)
    if (dev2caller[i] >= 0) caller2dev[dev2caller[i]] = i;
  // ---- tables in device numbering ----
  free_grid(s);
  s->n_int = n_int;
  s->n_tot = n_tot;
  s->ng = ng;
  s->n_caller = ncaller;
  s->ld = (n_tot + 31) / 32 * 32;
  s->nsub = nsub;
  s->nlev = (int)lens.size();
  s->n_inst = ninst;
  s->ntiles = (n_int + kBlock - 1) / kBlock;
  for (int i = 0; i < kMaxLevels; ++i) s->lens[i] = i < s->nlev ? lens[i] : 0.0;
  const long long L = s->ld;
  std::vector<int> h_nbr(np * L, -1);
  std::vector<unsigned char> h_lvl(L, 0);
  std::vector<double> h_xc(nd * L, 0.0);
  std::vector<int> h_sub(nsubc * std::max<long long>(nsub, 1), 0);
  const long long ngm = std::max<long long>(1, ng);
  std::vector<int> h_gb(ngm, 0), h_ginst(ngm, 0);
  std::vector<unsigned char> h_gpos(ngm, 0), h_apply(ngm, 255), h_own(ngm, 0);
  std::vector<double> h_gdx(ngm, 0.0);
  std::vector<int> h_blk(std::max<long long>(1, s->ntiles), 0);
  s->ghost_unapplied = false;
  for (int k = 0; k < ninst; ++k) {
    const h3c_grid& gr = grids[k];
    const InstanceTables& I = T[k];
    const long long co = caller_off[k];
    auto to_dev = [&](long long v) -> int {
      if (valid_cell(v, I.n)) return (int)caller2dev[co + v];
      if (I.nsub > 0 && v <= -2 && (-v - 2) < I.nsub) return (int)(v - sub_off[k]);  // -2 - (local + offset)
      return -1;
    };
    for (long long c = 0; c < I.n; ++c) {
      const long long i = caller2dev[co + c];
      h_lvl[i] = (unsigned char)(std::find(lens.begin(), lens.end(), gr.length[c]) - lens.begin());
      for (int d = 0; d < nd; ++d) h_xc[d * L + i] = gr.x_center[d * I.ld + c];
      for (int p = 0; p < np; ++p) {
        const long long v = gr.neighbors[p * I.ld + c];
        if (c < I.fg || valid_cell(v, I.n)) h_nbr[p * L + i] = to_dev(v);
      }
    }
    for (long long q = 0; q < I.nsub; ++q)
      for (int j = 0; j < nsubc; ++j)
        h_sub[j * nsub + sub_off[k] + q] = (int)caller2dev[co + gr.subface_cells[j * I.nsub + q]];
    for (long long g = 0; g < I.n - I.fg; ++g) {
      const long long gi = ghost_start[k] - n_int + g;
      const long long b = I.gb[g];
      h_gb[gi] = (int)caller2dev[co + b];
      h_gpos[gi] = (unsigned char)(I.gbp[g] ^ 1);  // ghost position w.r.t. its boundary cell
      h_apply[gi] = I.apply[g] == 255 ? 255 : bcmap[k][I.apply[g]];
      if (I.apply[g] == 255) s->ghost_unapplied = true;
      h_own[gi] = bcmap[k][I.own[g]];
      h_ginst[gi] = k;
      double s2 = 0;
      for (int d = 0; d < nd; ++d) {
        const double dd = gr.x_center[d * I.ld + b] - gr.x_center[d * I.ld + I.fg + g];
        s2 += dd * dd;
      }
      h_gdx[gi] = std::sqrt(s2);
    }
    for (long long t = int_start[k] / kBlock; t * kBlock < int_end[k]; ++t) h_blk[t] = k;
  }
  // ---- tables of the halo-staged Euler/AUSM stage kernel ----
  HaloHost HH;
  CnsHaloHost CH;
  bool halo_tables = false, cns_tables = false;
  if (s->desc.physics == H3C_CNS && ninst == 1 && nsub == 0 && lens.size() == 1) {
    std::vector<long long> tend(s->ntiles);
    for (long long t = 0; t < s->ntiles; ++t) tend[t] = std::min((t + 1) * kBlock, n_int);
    cns_tables = halo_build_cns(nd, L, n_int, s->ntiles, tend, h_nbr.data(), CH);
  }
  if (s->desc.physics == H3C_EULER && s->desc.flux == H3C_FLUX_AUSM && s->desc.reconstruction != H3C_RECON_MUSCL) {
    std::vector<long long> tend(s->ntiles);
    for (long long t = 0; t < s->ntiles; ++t) tend[t] = std::min((t + 1) * kBlock, int_end[h_blk[t]]);
    halo_tables = halo_build(nd, L, s->ntiles, tend, h_nbr.data(), h_sub.data(), std::max<long long>(nsub, 1), HH);
  }
  s->bcs = ubcs;
  s->n_bcs = (int)ubcs.size();
  s->h_bcs.assign(std::max<size_t>(1, ubcs.size()), BcParam{});
  s->unfused_dt = false;
  s->needs_partner = s->needs_periodic = false;
  for (size_t q = 0; q < ubcs.size(); ++q) {
    BcParam& B = s->h_bcs[q];
    B.kind = ubcs[q].kind;
    if (B.kind < 0 || B.kind > H3C_BC_EXCHANGE)
      return s->fail(H3C_E_INVALID, "h3c_set_grid: bc kind %d", B.kind);
    const bool adv_kind = B.kind >= H3C_BC_ADV_DIRICHLET && B.kind <= H3C_BC_ADV_CHARACTERISTIC;
    if (adv_kind != (s->desc.physics == H3C_ADVECTION) && B.kind != H3C_BC_PERIODIC && B.kind != H3C_BC_EXCHANGE)
      return s->fail(H3C_E_INVALID, "h3c_set_grid: bc kind %d does not belong to this physics", B.kind);
    B.wall = (B.kind == H3C_BC_CNS_ADIABATIC_NOSLIP || B.kind == H3C_BC_CNS_ISOTHERMAL_NOSLIP ||
              B.kind == H3C_BC_CPL_CNS_HEAT);
    for (int j = 0; j < 8; ++j) B.v[j] = ubcs[q].v[j];
    if (B.kind == H3C_BC_EULER_VORTEX) {
      if (nd != 2 || s->desc.physics == H3C_HEAT)
        return s->fail(H3C_E_INVALID, "h3c_set_grid: the isentropic vortex condition is 2D Euler/CNS only "
                                      "(euler/initial_conditions.hpp:41-46)");
      s->unfused_dt = true;
    }
    if (B.kind >= H3C_BC_CPL_EULER_EULER && B.kind <= H3C_BC_CPL_HEAT_HEAT) s->needs_partner = true;
    if (B.kind == H3C_BC_PERIODIC) s->needs_periodic = true;
  }
  if (ninst > 1 && (s->needs_partner || s->needs_periodic))
    return s->fail(H3C_E_INVALID, "h3c_set_grids: coupling and periodic conditions need a single grid");
  for (const BcParam& B : s->h_bcs)
    if (B.kind == H3C_BC_EXCHANGE &&
        (s->desc.physics == H3C_CNS || s->desc.reconstruction == H3C_RECON_MUSCL))
      return s->fail(H3C_E_INVALID, "h3c_set_grid: exchange ghosts need a first-order flux without cell slopes "
                                    "(not CNS, not MUSCL): their slopes would be the neighbouring subdomain's");
  s->dev2caller = dev2caller;
  s->caller2dev = caller2dev;
  s->partner = nullptr;
  s->partner_set = s->periodic_set = false;
  // allocations
  H3C_CUDA(s, cudaMalloc(&s->d_nbr, sizeof(int) * np * L));
  H3C_CUDA(s, cudaMalloc(&s->d_lvl, L));
  H3C_CUDA(s, cudaMalloc(&s->d_sub, sizeof(int) * h_sub.size()));
  H3C_CUDA(s, cudaMalloc(&s->d_xc, sizeof(double) * nd * L));
  H3C_CUDA(s, cudaMalloc(&s->d_gbndry, sizeof(int) * ngm));
  H3C_CUDA(s, cudaMalloc(&s->d_gpos, ngm));
  H3C_CUDA(s, cudaMalloc(&s->d_gapply, ngm));
  H3C_CUDA(s, cudaMalloc(&s->d_gown, ngm));
  H3C_CUDA(s, cudaMalloc(&s->d_gdx, sizeof(double) * ngm));
  H3C_CUDA(s, cudaMalloc(&s->d_gpartner, sizeof(int) * ngm));
  H3C_CUDA(s, cudaMalloc(&s->d_bcs, sizeof(BcParam) * s->h_bcs.size()));
  H3C_CUDA(s, cudaMalloc(&s->d_q[0], sizeof(double) * s->nv * L));
  H3C_CUDA(s, cudaMalloc(&s->d_q[1], sizeof(double) * s->nv * L));
  if (s->desc.time_integration == H3C_SSPRK3) H3C_CUDA(s, cudaMalloc(&s->d_q[2], sizeof(double) * s->nv * L));
  if (s->desc.physics == H3C_CNS || s->desc.reconstruction == H3C_RECON_MUSCL)
    H3C_CUDA(s, cudaMalloc(&s->d_slopes, sizeof(double) * nd * s->nv * L));
  H3C_CUDA(s, cudaMalloc(&s->d_dev2caller, sizeof(long long) * n_tot));
  if (ninst > 1) {
    H3C_CUDA(s, cudaMalloc(&s->d_blk_inst, sizeof(int) * h_blk.size()));
    H3C_CUDA(s, cudaMalloc(&s->d_inst_end, sizeof(long long) * ninst));
    H3C_CUDA(s, cudaMalloc(&s->d_ginst, sizeof(int) * ngm));
    H3C_CUDA(s, cudaMemcpy(s->d_blk_inst, h_blk.data(), sizeof(int) * h_blk.size(), cudaMemcpyHostToDevice));
    H3C_CUDA(s, cudaMemcpy(s->d_inst_end, int_end.data(), sizeof(long long) * ninst, cudaMemcpyHostToDevice));
    H3C_CUDA(s, cudaMemcpy(s->d_ginst, h_ginst.data(), sizeof(int) * ngm, cudaMemcpyHostToDevice));
  }
  if (ninst != s->sc_count) {  // one Scalars per instance
    H3C_CUDA(s, cudaStreamSynchronize(s->stream));
    dfree(s->d_sc);
    H3C_CUDA(s, cudaMalloc(&s->d_sc, sizeof(Scalars) * ninst));
    s->sc_count = ninst;
  }
  H3C_CUDA(s, cudaMemcpy(s->d_nbr, h_nbr.data(), sizeof(int) * np * L, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_lvl, h_lvl.data(), L, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_sub, h_sub.data(), sizeof(int) * h_sub.size(), cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_xc, h_xc.data(), sizeof(double) * nd * L, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_gbndry, h_gb.data(), sizeof(int) * ngm, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_gpos, h_gpos.data(), ngm, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_gapply, h_apply.data(), ngm, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_gown, h_own.data(), ngm, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_gdx, h_gdx.data(), sizeof(double) * ngm, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemset(s->d_gpartner, 0xff, sizeof(int) * ngm));
  if (halo_tables) {
    const bool mixed = s->desc.precision == H3C_MIXED;
    // halo entries kept in shared memory: as many as let 3 blocks share an SM
    HH.hmax = halo_slots_for(nd, mixed, HH.max_halo, 3);
    if (s->halo_cap > 0) HH.hmax = std::min(HH.hmax, s->halo_cap);
    const size_t smem = halo_smem_bytes(nd, mixed, HH.hmax);
    const int bps = halo_prepare(nd, mixed, smem);
    if (bps > 0) {
      H3C_CUDA(s, cudaMalloc(&s->d_lnb, sizeof(unsigned short) * HH.lnb.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_hids, sizeof(int) * HH.ids.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_hoff, sizeof(int) * HH.off.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_grp, sizeof(unsigned short) * HH.grp.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_goff, sizeof(int) * HH.goff.size()));
      H3C_CUDA(s, cudaMemcpy(s->d_lnb, HH.lnb.data(), sizeof(unsigned short) * HH.lnb.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemcpy(s->d_hids, HH.ids.data(), sizeof(int) * HH.ids.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemcpy(s->d_hoff, HH.off.data(), sizeof(int) * HH.off.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemcpy(s->d_grp, HH.grp.data(), sizeof(unsigned short) * HH.grp.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemcpy(s->d_goff, HH.goff.data(), sizeof(int) * HH.goff.size(), cudaMemcpyHostToDevice));
      s->hmax = HH.hmax;
      s->halo_smem = smem;
      s->halo_bps = bps;
      s->halo_mean = HH.mean_halo;
      s->halo_maxh = HH.max_halo;
      s->halo_ok = true;
    }
  }
  if (s->desc.physics == H3C_EULER && s->desc.flux == H3C_FLUX_AUSM && s->desc.reconstruction != H3C_RECON_MUSCL)
    s->warp_bps = warp_prepare(nd, s->desc.precision == H3C_MIXED);
  if (cns_tables) {
    const bool mixed = s->desc.precision == H3C_MIXED;
    const size_t smem = cns_halo_smem_bytes(nd, mixed, CH.base.hmax, CH.h1max);
    const int bps = smem <= 227 * 1024 ? cns_halo_prepare(nd, mixed, smem) : 0;
    if (bps > 0) {
      const HaloHost& B = CH.base;
      s->ngl = std::max<long long>(1, (ng + 31) / 32 * 32);
      H3C_CUDA(s, cudaMalloc(&s->d_lnb, sizeof(unsigned short) * B.lnb.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_hids, sizeof(int) * B.ids.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_hoff, sizeof(int) * B.off.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_h1end, sizeof(int) * CH.h1end.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_hnb, sizeof(unsigned short) * CH.hnb.size()));
      H3C_CUDA(s, cudaMalloc(&s->d_gsl, sizeof(double) * nd * s->nv * s->ngl));
      H3C_CUDA(s, cudaMemcpy(s->d_lnb, B.lnb.data(), sizeof(unsigned short) * B.lnb.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemcpy(s->d_hids, B.ids.data(), sizeof(int) * B.ids.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemcpy(s->d_hoff, B.off.data(), sizeof(int) * B.off.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemcpy(s->d_h1end, CH.h1end.data(), sizeof(int) * CH.h1end.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemcpy(s->d_hnb, CH.hnb.data(), sizeof(unsigned short) * CH.hnb.size(), cudaMemcpyHostToDevice));
      H3C_CUDA(s, cudaMemset(s->d_gsl, 0, sizeof(double) * nd * s->nv * s->ngl));
      s->hmax = B.hmax;
      s->h1max = CH.h1max;
      s->cns_smem = smem;
      s->cns_bps = bps;
      s->halo_mean = B.mean_halo;
      s->halo_maxh = B.max_halo;
      s->cns_ok = true;
    }
  }
  H3C_CUDA(s, cudaMemcpy(s->d_bcs, s->h_bcs.data(), sizeof(BcParam) * s->h_bcs.size(), cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_dev2caller, dev2caller.data(), sizeof(long long) * n_tot, cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemset(s->d_q[0], 0, sizeof(double) * s->nv * L));
  H3C_CUDA(s, cudaMemset(s->d_q[1], 0, sizeof(double) * s->nv * L));
  if (s->d_q[2]) H3C_CUDA(s, cudaMemset(s->d_q[2], 0, sizeof(double) * s->nv * L));
  if (s->d_slopes) H3C_CUDA(s, cudaMemset(s->d_slopes, 0, sizeof(double) * nd * s->nv * L));
  // The uploads and clears above ran on the legacy default stream, which the
  // solver's non-blocking stream does not wait for (a pageable cudaMemcpy may
  // return before its DMA lands, a cudaMemset before it runs): finish them
  // before the stream's kernels read the tables.
  H3C_CUDA(s, cudaStreamSynchronize(cudaStreamLegacy));
  {
    unsigned long long* d_bad = nullptr;
    H3C_CUDA(s, cudaMalloc(&d_bad, sizeof(unsigned long long)));
    H3C_CUDA(s, cudaMemsetAsync(d_bad, 0, sizeof(unsigned long long), s->stream));
    const long long nh = (s->halo_ok || s->cns_ok) && s->d_hids ? HH.ids.size() + CH.base.ids.size() : 0;
    const long long span = std::max({n_int, nsub, ng, nh, 1LL});
    const int hid_mask = s->halo_ok ? kHaloCellMask : -1;  // Euler entries carry a direction
    k_check_tables<<<blocks(span), kBlock, 0, s->stream>>>(s->d_nbr, s->d_sub, s->d_gbndry, s->d_lvl, s->d_hids,
                                                           hid_mask, nh, s->d_dev2caller, n_int, n_tot, L, nsub,
                                                           np, nsubc, ng,
                                                           s->nlev, d_bad);
    unsigned long long bad = 0;
    const cudaError_t e = cudaMemcpyAsync(&bad, d_bad, sizeof(bad), cudaMemcpyDeviceToHost, s->stream);
    const cudaError_t e2 = cudaStreamSynchronize(s->stream);
    cudaFree(d_bad);
    H3C_CUDA(s, e);
    H3C_CUDA(s, e2);
    if (bad) return s->fail(H3C_E_INVALID, "h3c_set_grid: %llu device table entries out of range", bad);
  }
  k_init_time<<<blocks(ninst), kBlock, 0, s->stream>>>(s->d_sc, s->desc.time_end, ninst);
  H3C_CUDA(s, cudaGetLastError());
  s->has_grid = true;
  return H3C_OK;
}

int h3c_set_grid(h3c_solver s, const h3c_grid* gr) { return set_grids(s, 1, gr); }

int h3c_set_grids(h3c_solver s, int n, const h3c_grid* grids) { return set_grids(s, n, grids); }

// Coupling and periodic conditions read partner cells: refuse to launch them
// before the partner tables exist.
static int ready(h3c_solver s, const char* what) {
  if (!s->has_grid) return s->fail(H3C_E_STATE, "%s: no grid", what);
  if (s->needs_partner && !s->partner_set)
    return s->fail(H3C_E_STATE, "%s: coupling conditions without h3c_set_partner", what);
  if (s->needs_periodic && !s->periodic_set)
    return s->fail(H3C_E_STATE, "%s: periodic conditions without h3c_set_periodic", what);
  if (s->desc.physics == H3C_ADVECTION && !s->vel_set)
    return s->fail(H3C_E_STATE, "%s: advection without h3c_set_velocity", what);
  return H3C_OK;
}

static int ensure_stage(h3c_solver s, long long ld) {
  const long long need = (long long)s->nv * ld;
  if (need > s->stage_cap) {
    dfree(s->d_stage);
    H3C_CUDA(s, cudaMalloc(&s->d_stage, sizeof(double) * need));
    s->stage_cap = need;
  }
  return H3C_OK;
}

int h3c_set_state(h3c_solver s, int which, const double* q, int64_t ld) {
  if (!s || !q || (which != 0 && which != 1)) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_set_state: no grid");
  const long long nc = s->n_caller;
  if (ld < nc) return s->fail(H3C_E_INVALID, "h3c_set_state: ld < n_cells");
  int rc = ensure_stage(s, nc);
  if (rc) return rc;
  for (int v = 0; v < s->nv; ++v)  // q in host or device memory (unified addressing)
    H3C_CUDA(s, cudaMemcpyAsync(s->d_stage + v * nc, q + v * ld, sizeof(double) * nc, cudaMemcpyDefault,
                                s->stream));
  k_gather<<<blocks(s->n_tot), kBlock, 0, s->stream>>>(s->d_stage, nc, s->d_q[which], s->ld, s->d_dev2caller,
                                                       s->n_tot, s->nv);
  if (which == 0) launch_cfl(s, &s->d_sc->dtmin_ord);
  H3C_CUDA(s, cudaStreamSynchronize(s->stream));
  return s->cuda(cudaGetLastError(), "h3c_set_state");
}

int h3c_set_velocity(h3c_solver s, const double* u, int64_t ld) {
  if (!s || !u) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_set_velocity: no grid");
  if (s->desc.physics != H3C_ADVECTION) return s->fail(H3C_E_INVALID, "h3c_set_velocity: not an advection solver");
  const long long nc = s->n_caller;
  if (ld < nc) return s->fail(H3C_E_INVALID, "h3c_set_velocity: ld < n_cells");
  for (int d = 0; d < s->nd; ++d)
    for (long long c = 0; c < nc; ++c)
      if (!std::isfinite(u[d * ld + c])) return s->fail(H3C_E_INVALID, "h3c_set_velocity: non-finite velocity");
  if (!s->d_vel) H3C_CUDA(s, cudaMalloc(&s->d_vel, sizeof(double) * s->nd * s->ld));
  H3C_CUDA(s, cudaMemsetAsync(s->d_vel, 0, sizeof(double) * s->nd * s->ld, s->stream));
  double* tmp = nullptr;
  H3C_CUDA(s, cudaMalloc(&tmp, sizeof(double) * s->nd * nc));
  for (int d = 0; d < s->nd; ++d)
    cudaMemcpyAsync(tmp + d * nc, u + d * ld, sizeof(double) * nc, cudaMemcpyHostToDevice, s->stream);
  k_gather<<<blocks(s->n_tot), kBlock, 0, s->stream>>>(tmp, nc, s->d_vel, s->ld, s->d_dev2caller, s->n_tot, s->nd);
  const cudaError_t e = cudaStreamSynchronize(s->stream);
  cudaFree(tmp);
  if (e != cudaSuccess) return s->cuda(e, "h3c_set_velocity");
  s->vel_set = true;
  drop_graph(s);
  // the time step depends on the velocity: recompute the next step's dt from the current lhs
  launch_cfl(s, &s->d_sc->dtmin_ord);
  H3C_CUDA(s, cudaStreamSynchronize(s->stream));
  return s->cuda(cudaGetLastError(), "h3c_set_velocity");
}

int h3c_write_vtk(h3c_solver s, const char* fname, const h3c_grid* grid, const int64_t* node_ids) {
  if (!s || !fname || !grid) return H3C_E_INVALID;
  if (int rc = ready(s, "h3c_write_vtk")) return rc;
  if (s->n_inst != 1) return s->fail(H3C_E_INVALID, "h3c_write_vtk: single grids only");
  const long long n = s->n_caller;
  if (grid->n_cells != n || grid->first_ghost < 0 || grid->first_ghost > n || grid->ld < n || !grid->neighbors ||
      !grid->x_center || !grid->length || !grid->bc_idx)
    return s->fail(H3C_E_INVALID, "h3c_write_vtk: the grid is not the one given to h3c_set_grid");
  const int nd = s->nd, nv = s->nv, phys = s->desc.physics;
  // write_domain(solver) applies the conditions to lhs first (solver.hpp:328-333)
  launch_bc(s, 0);
  std::vector<double> q((size_t)nv * n);
  if (int rc = h3c_get_state(s, 0, q.data(), n)) return rc;
  // device columns in the caller's numbering (cell slopes for the vorticity, the advection velocity)
  auto download = [&](const double* src, int cols, std::vector<double>& out) -> int {
    double* tmp = nullptr;
    H3C_CUDA(s, cudaMalloc(&tmp, sizeof(double) * cols * n));
    k_scatter<<<blocks(s->n_tot), kBlock, 0, s->stream>>>(src, s->ld, tmp, n, s->d_dev2caller, s->n_tot, cols);
    out.resize((size_t)cols * n);
    cudaMemcpyAsync(out.data(), tmp, sizeof(double) * cols * n, cudaMemcpyDeviceToHost, s->stream);
    const cudaError_t e = cudaStreamSynchronize(s->stream);
    cudaFree(tmp);
    return s->cuda(e, "h3c_write_vtk");
  };
  std::vector<VtkStream> st;
  auto ints = [&](std::vector<std::string> names, int dims) -> VtkStream& {
    st.push_back(VtkStream{});
    st.back().names = std::move(names);
    st.back().dims = dims;
    st.back().is_int = true;
    st.back().ints.assign((size_t)dims * n, INT64_MAX);
    return st.back();
  };
  auto nums = [&](std::vector<std::string> names, int dims) -> VtkStream& {
    st.push_back(VtkStream{});
    st.back().names = std::move(names);
    st.back().dims = dims;
    st.back().nums.assign((size_t)dims * n, 0.0);
    return st.back();
  };
  // solver.hpp:351-370: cell id, grid node, same-level neighbours, ghost flag, bc index
  { auto& x = ints({"locallCellIds"}, 1); for (long long c = 0; c < n; ++c) x.ints[c] = c; }
  { auto& x = ints({"gridNodeIds"}, 1); if (node_ids) for (long long c = 0; c < n; ++c) x.ints[c] = node_ids[c]; }
  {
    auto& x = ints({"local_nghbrs"}, 2 * nd);
    for (int p = 0; p < 2 * nd; ++p)
      for (long long c = 0; c < n; ++c) {
        const int64_t v = grid->neighbors[p * grid->ld + c];
        x.ints[(size_t)p * n + c] = (v >= 0 && v < n) || v <= -2 ? v : INT64_MAX;  // <= -2: sub-face group
      }
  }
  { auto& x = ints({"ghost_cell"}, 1); for (long long c = grid->first_ghost; c < n; ++c) x.ints[c] = 1; }
  {
    // SInd bc index; an internal cell's invalid<SInd>() is a valid Ind and is written as is
    auto& x = ints({"bcIdx"}, 1);
    for (long long c = 0; c < n; ++c) {
      const int32_t b = grid->bc_idx[c];
      x.ints[c] = (b >= 0 && b < grid->n_bcs) ? b : INT32_MAX;
    }
  }
  // conservative variables (V::cv_names: euler/indices.hpp:20-30, heat/indices.hpp:16-22, advection/indices.hpp)
  {
    std::vector<std::string> names;
    if (phys == H3C_HEAT) names = {"T"};
    else if (phys == H3C_ADVECTION) names = {"q"};
    else {
      for (int d = 0; d < nd; ++d) names.push_back("rho_u" + std::to_string(d));
      names.push_back("rho");
      names.push_back("rho_E");
    }
    auto& x = nums(names, nv);
    x.nums = q;
  }
  // physics_output: euler/physics.hpp:207-226 (+ cns/physics.hpp:193-201), advection/physics.hpp:90-95
  if (phys == H3C_EULER || phys == H3C_CNS) {
    const double gamma = s->desc.gamma, gm1 = gamma - 1.0;
    std::vector<double> a(n), p(n), u((size_t)nd * n), M(n), e(n), T(n);
    for (long long c = 0; c < n; ++c) {
      const double rho = q[(size_t)nd * n + c], rhoE = q[(size_t)(nd + 1) * n + c];
      double um2 = 0;
      for (int d = 0; d < nd; ++d) {
        u[(size_t)d * n + c] = q[(size_t)d * n + c] / rho;
        um2 += u[(size_t)d * n + c] * u[(size_t)d * n + c];
      }
      p[c] = gm1 * (rhoE - 0.5 * rho * um2);
      a[c] = std::sqrt(gamma * p[c] / rho);
      M[c] = std::sqrt(um2) / a[c];
      e[c] = p[c] / gm1 / rho;
      T[c] = gamma * p[c] / rho;
    }
    nums({"a"}, 1).nums = a;
    nums({"p"}, 1).nums = p;
    nums({"u"}, nd).nums = u;
    nums({"M"}, 1).nums = M;
    nums({"e"}, 1).nums = e;
    nums({"T"}, 1).nums = T;
    if (phys == H3C_CNS) {
      std::vector<double> mu(n);
      for (long long c = 0; c < n; ++c)
        mu[c] = std::pow(T[c], 1.5) * s->pc.sOverTrefP1 / (T[c] + s->pc.sOverTref);  // cns/quantities.hpp:113-115
      nums({"mu"}, 1).nums = mu;
      // vorticity from slope_u (cns/physics.hpp:89-94, 126-138) on the cell slopes of the step
      launch_slopes_ptr(s, s->d_q[0]);
      std::vector<double> sl;
      if (int rc = download(s->d_slopes, nd * nv, sl)) return rc;
      auto slope = [&](long long c, int v, int sd) { return sl[(size_t)(sd * nv + v) * n + c]; };
      auto slope_u = [&](long long c, int dir, int sd) {
        const double rho = q[(size_t)nd * n + c];
        return (slope(c, dir, sd) * rho - slope(c, nd, sd) * q[(size_t)dir * n + c]) / std::pow(rho, 2.);
      };
      const int nw = nd == 2 ? 1 : 3;
      auto& w = nums({"vorticity"}, nw);
      for (long long c = 0; c < n; ++c) {
        if (nd == 2) {
          w.nums[c] = slope_u(c, 1, 0) - slope_u(c, 0, 1);
        } else {
          w.nums[c] = slope_u(c, 2, 1) - slope_u(c, 1, 2);
          w.nums[(size_t)n + c] = slope_u(c, 0, 2) - slope_u(c, 2, 0);
          w.nums[(size_t)2 * n + c] = slope_u(c, 1, 0) - slope_u(c, 0, 1);
        }
      }
    }
  } else if (phys == H3C_ADVECTION) {
    std::vector<double> vel;
    if (int rc = download(s->d_vel, nd, vel)) return rc;
    nums({"u"}, nd).nums = vel;
  }
  VtkDomain D;
  D.path = std::string(fname) + ".vtk";
  D.nd = nd;
  D.n_cells = n;
  D.ld = grid->ld;
  D.x_center = grid->x_center;
  D.length = grid->length;
  std::string err;
  if (write_vtk_file(D, st, &err)) return s->fail(H3C_E_INVALID, "h3c_write_vtk: %s", err.c_str());
  return H3C_OK;
}

int h3c_get_state(h3c_solver s, int which, double* q, int64_t ld) {
  if (!s || !q || (which != 0 && which != 1)) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_get_state: no grid");
  const long long nc = s->n_caller;
  if (ld < nc) return s->fail(H3C_E_INVALID, "h3c_get_state: ld < n_cells");
  int rc = ensure_stage(s, nc);
  if (rc) return rc;
  k_scatter<<<blocks(s->n_tot), kBlock, 0, s->stream>>>(s->d_q[which], s->ld, s->d_stage, nc, s->d_dev2caller,
                                                        s->n_tot, s->nv);
  for (int v = 0; v < s->nv; ++v)  // q in host or device memory (unified addressing)
    H3C_CUDA(s, cudaMemcpyAsync(q + v * ld, s->d_stage + v * nc, sizeof(double) * nc, cudaMemcpyDefault,
                                s->stream));
  H3C_CUDA(s, cudaStreamSynchronize(s->stream));
  return s->cuda(cudaGetLastError(), "h3c_get_state");
}

int h3c_state_device(h3c_solver s, int which, double** ptr, int64_t* ld) {
  if (!s || !ptr || !ld || (which != 0 && which != 1)) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_state_device: no grid");
  *ptr = s->d_q[which];
  *ld = s->ld;
  return H3C_OK;
}

int h3c_device_order(h3c_solver s, int64_t* perm) {
  if (!s || !perm) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_device_order: no grid");
  for (long long c = 0; c < s->n_caller; ++c) perm[c] = s->caller2dev[c];
  return H3C_OK;
}

int h3c_get_stream(h3c_solver s, void** stream) {
  if (!s || !stream) return H3C_E_INVALID;
  *stream = (void*)s->stream;
  return H3C_OK;
}

int h3c_sizes(h3c_solver s, int64_t* n_cells, int64_t* first_ghost, int* nv) {
  if (!s) return H3C_E_INVALID;
  if (n_cells) *n_cells = s->n_caller;
  if (first_ghost) *first_ghost = s->n_int;
  if (nv) *nv = s->nv;
  return H3C_OK;
}

int h3c_reset_time(h3c_solver s) {
  if (!s) return H3C_E_INVALID;
  if (s->ng < 0) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_reset_time: no grid");
  s->stage_next = 0;  // a step run by parts starts over
  k_init_time<<<blocks(s->n_inst), kBlock, 0, s->stream>>>(s->d_sc, s->desc.time_end, s->n_inst);
  launch_cfl(s, &s->d_sc->dtmin_ord);
  k_set_dt<<<blocks(s->n_inst), kBlock, 0, s->stream>>>(s->d_sc, 0, s->n_inst);
  return s->cuda(cudaGetLastError(), "h3c_reset_time");
}

int h3c_apply_bcs(h3c_solver s, int which) {
  if (!s || (which != 0 && which != 1)) return H3C_E_INVALID;
  if (int rc = ready(s, "h3c_apply_bcs")) return rc;
  launch_bc(s, which);
  return s->cuda(cudaGetLastError(), "h3c_apply_bcs");
}

// Solver::solve (solver.hpp:140-145): apply_bcs(lhs), set_dt, evolve, advance.
// Per-stage preparation of a stage input q: CNS cell slopes or MUSCL gradients.
static bool cns_tile_active(h3c_solver s) { return s->desc.physics == H3C_CNS && s->tile && s->halo && s->cns_ok; }

static void prepare_stage(h3c_solver s, const double* q, int which) {
  if (s->desc.physics == H3C_CNS) {
    if (!cns_tile_active(s)) launch_slopes(s, which);  // the tile kernel computes slopes itself
  }
  else if (s->desc.reconstruction == H3C_RECON_MUSCL) launch_grad(s, q);
}

// One solver step (solver.hpp:140-145) on the solver's buffers.  keep (may be
// null) receives copies of the ghost-filled stage inputs in consecutive
// nv * ld slots; dts (may be null) records the step's dt at index i.
// Stages per step of the time integration.
static int stage_count(const h3c_solver s) {
  const int ti = s->desc.time_integration;
  return ti == H3C_EULER_FORWARD ? 1 : ti == H3C_RUNGE_KUTTA_2 ? 2 : 3;
}

// Part k of one step (k = 0 .. stage_count - 1, in order): k = 0 applies the
// conditions to lhs and sets the step's dt; k > 0 applies the conditions to
// its stage input; every part then runs its stage; the last part advances
// time and step.  keep (optional) receives each stage's input; dts (optional)
// records the step's dt at index i.
static void enqueue_stage(h3c_solver s, int k, bool fuse, double* keep, double* dts, long long i) {
  const size_t Qb = sizeof(double) * s->nv * s->ld;
  const long long Q = s->nv * s->ld;
  const int ti = s->desc.time_integration;
  const int last = stage_count(s) - 1;
  if (k == 0) {
    launch_bc(s, 0);
    if (!fuse) launch_cfl(s, &s->d_sc->dtmin_ord);
    {
      Launch L(s, K_SCALAR);
      k_set_dt<<<blocks(s->n_inst), kBlock, 0, s->stream>>>(s->d_sc, 1, s->n_inst);
    }
    if (dts) {
      Launch L(s, K_SCALAR);
      k_record_dt<<<1, 1, 0, s->stream>>>(s->d_sc, dts, i);
    }
    if (keep) cudaMemcpyAsync(keep, s->d_q[0], Qb, cudaMemcpyDeviceToDevice, s->stream);
    prepare_stage(s, s->d_q[0], 0);
    if (ti == H3C_EULER_FORWARD) {
      // evolve(euler_forward): solver.hpp:470-479 (rhs = lhs + R; lhs = rhs as a buffer swap)
      launch_stage(s, 0, s->d_q[0], s->d_q[1], fuse);
      std::swap(s->d_q[0], s->d_q[1]);
    } else {
      // evolve(runge_kutta_2): solver.hpp:483-494, and the first SSP-RK3 stage
      launch_stage(s, 0, s->d_q[0], s->d_q[1], false);
    }
  } else if (k == 1) {
    launch_bc(s, 1);
    if (keep) cudaMemcpyAsync(keep + Q, s->d_q[1], Qb, cudaMemcpyDeviceToDevice, s->stream);
    if (ti == H3C_RUNGE_KUTTA_2) {
      prepare_stage(s, s->d_q[1], 1);
      launch_stage(s, 2, s->d_q[1], s->d_q[0], fuse);
    } else {
      // EXTENSION: SSP-RK3, conditions before every stage
      cudaMemcpyAsync(s->d_q[2], s->d_q[0], Qb, cudaMemcpyDeviceToDevice, s->stream);
      prepare_stage(s, s->d_q[1], 1);
      launch_stage(s, 3, s->d_q[1], s->d_q[2], false);
    }
  } else {
    launch_bc(s, 2);
    if (keep) cudaMemcpyAsync(keep + 2 * Q, s->d_q[2], Qb, cudaMemcpyDeviceToDevice, s->stream);
    prepare_stage(s, s->d_q[2], 2);
    launch_stage(s, 4, s->d_q[2], s->d_q[0], fuse);
  }
  if (k == last) {
    Launch L(s, K_SCALAR);
    k_advance<<<blocks(s->n_inst), kBlock, 0, s->stream>>>(s->d_sc, s->n_inst);
  }
}

static void enqueue_step(h3c_solver s, bool fuse, double* keep, double* dts, long long i) {
  for (int k = 0; k < stage_count(s); ++k) enqueue_stage(s, k, fuse, keep, dts, i);
}

static void enqueue_steps(h3c_solver s, int64_t nsteps) {
  const bool fuse = !s->unfused_dt;
  for (int64_t it = 0; it < nsteps; ++it) enqueue_step(s, fuse, nullptr, nullptr, 0);
}

// Steps per replayed graph: even, so forward Euler's buffer swap returns the
// state pointers to where the capture started.
constexpr int kGraphSteps = 8;

// Captures `n` steps starting from the current lhs buffer into `slot`
// (capturing runs nothing: the state and the buffer pointers stay as they
// were); false when the stream cannot be captured.
static bool capture_steps(h3c_solver s, int n, StepGraph* slot) {
  double* saved[3] = {s->d_q[0], s->d_q[1], s->d_q[2]};
  if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  const long long l0 = s->launches;
  enqueue_steps(s, n);
  const long long per_step = (s->launches - l0) / n;
  s->launches = l0;
  for (int j = 0; j < 3; ++j) s->d_q[j] = saved[j];
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s->stream, &g);
  if (e != cudaSuccess || !g) {
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    return false;
  }
  const cudaError_t ei = cudaGraphInstantiate(&slot->exec, g, 0);
  cudaGraphDestroy(g);
  if (ei != cudaSuccess) {
    cudaGetLastError();
    *slot = StepGraph{};
    return false;
  }
  slot->q0 = s->d_q[0];
  s->graph_per_step = per_step;
  return true;
}

// The graph of `n` steps for the current lhs buffer, captured on first use.
static StepGraph* graph_for(h3c_solver s, StepGraph* slots, int n) {
  for (int j = 0; j < 2; ++j)
    if (slots[j].exec && slots[j].q0 == s->d_q[0]) return &slots[j];
  for (int j = 0; j < 2; ++j)
    if (!slots[j].exec) return capture_steps(s, n, &slots[j]) ? &slots[j] : nullptr;
  return nullptr;
}

// Captures every step graph a later h3c_solve can replay, for both lhs
// buffers where forward Euler alternates them, so that no capture or
// instantiation falls inside a later run of steps whatever its length.
static void capture_all(h3c_solver s) {
  const bool fe = s->desc.time_integration == H3C_EULER_FORWARD;
  for (int side = 0; side < (fe ? 2 : 1); ++side) {
    if (side) std::swap(s->d_q[0], s->d_q[1]);
    graph_for(s, s->graph8, kGraphSteps);
    graph_for(s, s->graph1, 1);
    if (side) std::swap(s->d_q[0], s->d_q[1]);
  }
}

static bool launch_graph(h3c_solver s, const StepGraph* g, int n) {
  if (cudaGraphLaunch(g->exec, s->stream) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  s->launches += s->graph_per_step * n;
  // as enqueue_step does; kGraphSteps is even, so only single steps swap
  if (s->desc.time_integration == H3C_EULER_FORWARD && (n & 1)) std::swap(s->d_q[0], s->d_q[1]);
  return true;
}

int h3c_solve(h3c_solver s, int64_t nsteps) {
  if (!s || nsteps < 0) return H3C_E_INVALID;
  Range r("h3c_solve");
  if (int rc = ready(s, "h3c_solve")) return rc;
  if (s->stage_next != 0)
    return s->fail(H3C_E_STATE, "h3c_solve: a step run by parts is at part %d (h3c_solve_stage)", s->stage_next);
  // Steps replay captured graphs (no per-launch host cost) once one step has
  // run plainly (kernel attributes are set outside capture); coupled solvers
  // read their partner's current buffers and profiling brackets every
  // launch, so those take the plain path.
  const bool graphable = s->graphs && !s->prof && s->partner == nullptr;
  if (graphable && !s->plain_done && nsteps > 0) {
    enqueue_steps(s, 1);
    s->plain_done = true;
    --nsteps;
  }
  if (graphable && s->plain_done) {
    capture_all(s);
    for (StepGraph* g; nsteps >= kGraphSteps && (g = graph_for(s, s->graph8, kGraphSteps)) &&
                       launch_graph(s, g, kGraphSteps);)
      nsteps -= kGraphSteps;
    for (StepGraph* g; nsteps > 0 && (g = graph_for(s, s->graph1, 1)) && launch_graph(s, g, 1);) --nsteps;
  }
  if (nsteps > 0) {
    enqueue_steps(s, nsteps);
    s->plain_done = true;
  }
  return s->cuda(cudaGetLastError(), "h3c_solve");
}

int h3c_stages(h3c_solver s, int* n) {
  if (!s || !n) return H3C_E_INVALID;
  *n = stage_count(s);
  return H3C_OK;
}

int h3c_solve_stage(h3c_solver s, int k) {
  if (!s) return H3C_E_INVALID;
  static const char* names[3] = {"h3c_solve_stage 0", "h3c_solve_stage 1", "h3c_solve_stage 2"};
  Range r(names[k >= 0 && k < 3 ? k : 0]);
  if (int rc = ready(s, "h3c_solve_stage")) return rc;
  if (k != s->stage_next)
    return s->fail(H3C_E_STATE, "h3c_solve_stage: part %d requested, part %d is next", k, s->stage_next);
  enqueue_stage(s, k, !s->unfused_dt, nullptr, nullptr, 0);
  s->stage_next = k + 1 == stage_count(s) ? 0 : k + 1;
  return s->cuda(cudaGetLastError(), "h3c_solve_stage");
}

int h3c_stage_input(h3c_solver s, int k, double** ptr) {
  if (!s || !ptr || k < 0 || k >= stage_count(s)) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_stage_input: no grid");
  *ptr = s->d_q[k];  // lhs, rhs, third buffer: the inputs of parts 0, 1, 2
  return H3C_OK;
}

int h3c_dtmin_device(h3c_solver s, int64_t** ptr) {
  if (!s || !ptr) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_dtmin_device: no grid");
  static_assert(sizeof(long long) == sizeof(int64_t), "ordered bits");
  *ptr = reinterpret_cast<int64_t*>(&s->d_sc->dtmin_ord);
  return H3C_OK;
}

static int read_scalars(h3c_solver s, Scalars* out) {
  Scalars* dst = s->h_sc ? s->h_sc : out;
  H3C_CUDA(s, cudaMemcpyAsync(dst, s->d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream));
  H3C_CUDA(s, cudaStreamSynchronize(s->stream));
  if (dst != out) *out = *dst;
  return H3C_OK;
}

// The error the status bits of a step's scalars stand for (hom3 terminates
// the run instead: solution_diverged, utilities.hpp:74-76, 107-110, and the
// check_variables asserts, euler/physics.hpp:229-239).  The bits stay set
// until h3c_status or h3c_reset_time clears them, so every later read of
// dt / time / step reports the failure too.
static int status_error(h3c_solver s, const Scalars& sc, int inst = 0) {
  if (sc.status & kStatusTimeout)
    return s->fail(H3C_E_TIMEOUT, "instance %d: a bounded device wait for a tile's copies ran out", inst);
  if (!(sc.status & (kStatusState | kStatusDt))) return H3C_OK;
  std::string m = "instance " + std::to_string(inst) + ":";
  char buf[160];
  if (sc.status & kStatusDt) {
    std::snprintf(buf, sizeof(buf), " solution diverged: dt = %g is outside [1e-300, 1e300] at step %lld;", sc.dt,
                  (long long)sc.step);
    m += buf;
  }
  if (sc.status & kStatusState) {
    std::snprintf(buf, sizeof(buf), " a cell is not finite or (Euler/CNS) has a non-positive density, energy or "
                                    "pressure (hom3's check_variables) at step %lld;", (long long)sc.step);
    m += buf;
  }
  m.pop_back();
  return s->fail(H3C_E_NONFINITE, "%s", m.c_str());
}

int h3c_min_dt(h3c_solver s, double* dt) {
  if (!s || !dt) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_min_dt: no grid");
  if (s->desc.physics == H3C_ADVECTION && !s->vel_set)
    return s->fail(H3C_E_STATE, "h3c_min_dt: advection without h3c_set_velocity");
  launch_cfl(s, &s->d_sc->mindt_ord);
  Scalars sc;
  int rc = read_scalars(s, &sc);
  if (rc) return rc;
  *dt = ord_to_dbl(sc.mindt_ord);
  return status_error(s, sc);
}

int h3c_dt(h3c_solver s, double* dt) {
  if (!s || !dt) return H3C_E_INVALID;
  Scalars sc;
  int rc = read_scalars(s, &sc);
  if (rc) return rc;
  *dt = sc.dt;
  return status_error(s, sc);
}
int h3c_time(h3c_solver s, double* t) {
  if (!s || !t) return H3C_E_INVALID;
  Scalars sc;
  int rc = read_scalars(s, &sc);
  if (rc) return rc;
  *t = sc.time;
  return status_error(s, sc);
}
int h3c_step(h3c_solver s, int64_t* step) {
  if (!s || !step) return H3C_E_INVALID;
  Scalars sc;
  int rc = read_scalars(s, &sc);
  if (rc) return rc;
  *step = sc.step;
  return status_error(s, sc);
}
int h3c_force_dt(h3c_solver s, double dt) {
  if (!s) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_force_dt: no grid");
  k_force_dt<<<1, 1, 0, s->stream>>>(s->d_sc, dt);
  return s->cuda(cudaGetLastError(), "h3c_force_dt");
}
int h3c_status(h3c_solver s, int* flags) {
  if (!s || !flags) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_status: no grid");
  std::vector<Scalars> h(s->n_inst);
  H3C_CUDA(s, cudaMemcpyAsync(h.data(), s->d_sc, sizeof(Scalars) * s->n_inst, cudaMemcpyDeviceToHost, s->stream));
  H3C_CUDA(s, cudaStreamSynchronize(s->stream));
  int f = 0;
  for (int i = 0; i < s->n_inst; ++i) {
    f |= h[i].status;
    if (h[i].status) {
      const int zero = 0;
      H3C_CUDA(s, cudaMemcpy(&s->d_sc[i].status, &zero, sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  if (f) H3C_CUDA(s, cudaStreamSynchronize(cudaStreamLegacy));  // cleared before the stream's next kernels
  *flags = f;
  return H3C_OK;
}

int h3c_set_partner(h3c_solver s, h3c_solver partner, const int64_t* partner_cells) {
  if (!s || !partner || !partner_cells) return H3C_E_INVALID;
  if (!s->has_grid || !partner->has_grid) return s->fail(H3C_E_STATE, "h3c_set_partner: no grid");
  if (s->nd != partner->nd) return s->fail(H3C_E_INVALID, "h3c_set_partner: dimension mismatch");
  std::vector<int> h(std::max<long long>(1, s->ng), -1);
  for (long long i = 0; i < s->ng; ++i) {
    const long long o = partner_cells[i];
    if (o >= 0 && o < partner->n_caller) h[i] = (int)partner->caller2dev[o];
  }
  // every ghost of a coupling condition needs a partner cell
  std::vector<unsigned char> own(s->ng);
  if (s->ng) H3C_CUDA(s, cudaMemcpy(own.data(), s->d_gown, s->ng, cudaMemcpyDeviceToHost));
  for (long long i = 0; i < s->ng; ++i) {
    const int kind = s->h_bcs[own[i]].kind;
    const bool cpl = kind == H3C_BC_CPL_EULER_EULER || kind == H3C_BC_CPL_CNS_HEAT ||
                     kind == H3C_BC_CPL_HEAT_CNS || kind == H3C_BC_CPL_HEAT_HEAT;
    if (cpl && h[i] < 0) return s->fail(H3C_E_INVALID, "h3c_set_partner: coupled ghost %lld has no partner", i);
  }
  for (int k = 0; k < s->n_bcs; ++k) {
    s->h_bcs[k].partner_gamma = partner->desc.gamma;
    s->h_bcs[k].partner_physics = partner->desc.physics;
    s->h_bcs[k].partner_nd = partner->nd;
  }
  H3C_CUDA(s, cudaMemcpy(s->d_bcs, s->h_bcs.data(), sizeof(BcParam) * s->h_bcs.size(), cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaMemcpy(s->d_gpartner, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaStreamSynchronize(cudaStreamLegacy));  // the copies land before the stream's kernels read them
  s->partner = partner;
  s->partner_set = true;
  // coupled solvers run on one stream, so each sees the other's finished steps
  if (s->stream != partner->stream) {
    H3C_CUDA(s, cudaStreamSynchronize(s->stream));
    if (s->own_stream) cudaStreamDestroy(s->stream);
    s->stream = partner->stream;
    s->own_stream = false;
    // the partner keeps ownership of its stream; it must outlive this solver's use of it
  }
  return H3C_OK;
}

int h3c_set_periodic(h3c_solver s, const int64_t* partner_cells) {
  if (!s || !partner_cells) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_set_periodic: no grid");
  std::vector<int> h(std::max<long long>(1, s->ng), -1);
  std::vector<unsigned char> own(s->ng);
  if (s->ng) H3C_CUDA(s, cudaMemcpy(own.data(), s->d_gown, s->ng, cudaMemcpyDeviceToHost));
  for (long long i = 0; i < s->ng; ++i) {
    const long long o = partner_cells[i];
    if (o >= 0 && o < s->n_int) h[i] = (int)s->caller2dev[o];
    if (s->h_bcs[own[i]].kind == H3C_BC_PERIODIC && h[i] < 0)
      return s->fail(H3C_E_INVALID, "h3c_set_periodic: periodic ghost %lld has no interior partner", i);
  }
  H3C_CUDA(s, cudaMemcpy(s->d_gpartner, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
  H3C_CUDA(s, cudaStreamSynchronize(cudaStreamLegacy));  // the copy lands before the stream's kernels read it
  s->periodic_set = true;
  return H3C_OK;
}

int h3c_couple_cht(h3c_solver cns, h3c_solver heat, double Tr0) {
  if (!cns || !heat) return H3C_E_INVALID;
  if (!cns->has_grid || !heat->has_grid) return cns->fail(H3C_E_STATE, "h3c_couple_cht: no grid");
  if (cns->desc.physics != H3C_CNS || heat->desc.physics != H3C_HEAT)
    return cns->fail(H3C_E_INVALID, "h3c_couple_cht: expects (cns, heat)");
  if (cns->stream != heat->stream) return cns->fail(H3C_E_STATE, "h3c_couple_cht: solvers are not coupled");
  const double scaling = Tr0 * cns->Pr0 * cns->Re0;
  launch_cfl(cns, &cns->d_sc->mindt_ord);
  launch_cfl(heat, &heat->d_sc->mindt_ord);
  k_couple_cht<<<1, 1, 0, cns->stream>>>(cns->d_sc, heat->d_sc, scaling);
  return cns->cuda(cudaGetLastError(), "h3c_couple_cht");
}

// One coupled step: coupling::apply(Tr0, cns, heat), cns.solve(), heat.solve()
// (coupled_cns_heat_test.cpp:235-248), all on the shared stream.
static void enqueue_cht(h3c_solver cns, h3c_solver heat, double scaling, int64_t n) {
  for (int64_t i = 0; i < n; ++i) {
    launch_cfl(cns, &cns->d_sc->mindt_ord);
    launch_cfl(heat, &heat->d_sc->mindt_ord);
    {
      Launch L(cns, K_SCALAR);
      k_couple_cht<<<1, 1, 0, cns->stream>>>(cns->d_sc, heat->d_sc, scaling);
    }
    enqueue_steps(cns, 1);
    enqueue_steps(heat, 1);
  }
}

int h3c_cht_solve(h3c_solver cns, h3c_solver heat, double Tr0, int64_t nsteps) {
  Range r("h3c_cht_solve");
  if (!cns || !heat || nsteps < 0) return H3C_E_INVALID;
  if (int rc = ready(cns, "h3c_cht_solve")) return rc;
  if (int rc = ready(heat, "h3c_cht_solve")) return rc;
  if (cns->desc.physics != H3C_CNS || heat->desc.physics != H3C_HEAT)
    return cns->fail(H3C_E_INVALID, "h3c_cht_solve: expects (cns, heat)");
  if (cns->stream != heat->stream || cns->partner != heat || heat->partner != cns)
    return cns->fail(H3C_E_STATE, "h3c_cht_solve: solvers are not coupled with each other");
  const double scaling = Tr0 * cns->Pr0 * cns->Re0;
  const bool graphable = cns->graphs && heat->graphs && !cns->prof && !heat->prof;
  if (graphable && nsteps >= kGraphSteps) {
    if (cns->cpl_graph && (cns->cpl_with != heat || cns->cpl_q0 != cns->d_q[0] ||
                           cns->cpl_q0_other != heat->d_q[0] || cns->cpl_scaling != scaling))
      drop_cpl_graph(cns);
    if (!cns->cpl_graph) {
      enqueue_cht(cns, heat, scaling, 1);  // one plain step first (kernel attributes outside capture)
      nsteps -= 1;
      const long long lc = cns->launches, lh = heat->launches;
      cudaGraph_t g = nullptr;
      if (cudaStreamBeginCapture(cns->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        enqueue_cht(cns, heat, scaling, kGraphSteps);
        if (cudaStreamEndCapture(cns->stream, &g) == cudaSuccess && g &&
            cudaGraphInstantiate(&cns->cpl_graph, g, 0) == cudaSuccess) {
          cns->cpl_with = heat;
          cns->cpl_q0 = cns->d_q[0];
          cns->cpl_q0_other = heat->d_q[0];
          cns->cpl_scaling = scaling;
          cns->cpl_launches = (cns->launches - lc) + (heat->launches - lh);
        } else {
          cns->cpl_graph = nullptr;
        }
        if (g) cudaGraphDestroy(g);
      }
      cudaGetLastError();
      cns->launches = lc;  // captured launches are counted when the graph runs
      heat->launches = lh;
    }
    while (cns->cpl_graph && nsteps >= kGraphSteps) {
      H3C_CUDA(cns, cudaGraphLaunch(cns->cpl_graph, cns->stream));
      cns->launches += cns->cpl_launches;
      nsteps -= kGraphSteps;
    }
  }
  enqueue_cht(cns, heat, scaling, nsteps);
  return cns->cuda(cudaGetLastError(), "h3c_cht_solve");
}

int h3c_couple_equal(h3c_solver a, h3c_solver b) {
  if (!a || !b) return H3C_E_INVALID;
  if (!a->has_grid || !b->has_grid) return a->fail(H3C_E_STATE, "h3c_couple_equal: no grid");
  if (a->stream != b->stream) return a->fail(H3C_E_STATE, "h3c_couple_equal: solvers are not coupled");
  launch_cfl(a, &a->d_sc->mindt_ord);
  launch_cfl(b, &b->d_sc->mindt_ord);
  k_couple_equal<<<1, 1, 0, a->stream>>>(a->d_sc, b->d_sc);
  return a->cuda(cudaGetLastError(), "h3c_couple_equal");
}

__global__ void k_selftest_nr(const double* x, double* r, double* rs, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  r[i] = nr_rcp(x[i]);
  rs[i] = nr_rsqrt(x[i]);
}

int h3c_selftest_nr(const double* x, int64_t n, double* rcp, double* rsqrt) {
  if (!x || !rcp || !rsqrt || n <= 0 || n > (1LL << 24)) return H3C_E_INVALID;
  double *dx = nullptr, *dr = nullptr, *ds = nullptr;
  cudaError_t e = cudaMalloc(&dx, 3 * n * sizeof(double));
  if (e != cudaSuccess) { g_last_error = cudaGetErrorString(e); return H3C_E_NOMEM; }
  dr = dx + n;
  ds = dr + n;
  cudaMemcpy(dx, x, n * sizeof(double), cudaMemcpyHostToDevice);
  k_selftest_nr<<<blocks(n), kBlock>>>(dx, dr, ds, n);
  cudaMemcpy(rcp, dr, n * sizeof(double), cudaMemcpyDeviceToHost);
  e = cudaMemcpy(rsqrt, ds, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dx);
  if (e != cudaSuccess) { g_last_error = cudaGetErrorString(e); return H3C_E_CUDA; }
  return H3C_OK;
}

int h3c_set_option(h3c_solver s, int option, int value) {
  if (!s) return H3C_E_INVALID;
  switch (option) {
    case H3C_OPT_TILE_KERNEL: s->tile = value != 0; break;
    case H3C_OPT_GRAPHS: s->graphs = value != 0; break;
    case H3C_OPT_HALO_KERNEL: s->halo = value != 0; break;
    case H3C_OPT_EULER_KERNEL:
      if (value < 0 || value > 4)
        return s->fail(H3C_E_INVALID, "h3c_set_option: Euler kernel must be 0, 1, 2, 3 or 4");
      s->euler_kernel = value;
      break;
    case H3C_OPT_CNS_ADJOINT_DUAL: s->cns_adj_dual = value != 0; break;
    case H3C_OPT_HALO_SLOTS: {
      if (value < 0 || value % 32) return s->fail(H3C_E_INVALID, "h3c_set_option: halo slots must be a multiple of 32");
      s->halo_cap = value;
      if (s->halo_ok) {  // the Euler kernel's shared-memory size follows the cap
        const bool mixed = s->desc.precision == H3C_MIXED;
        int hm = halo_slots_for(s->nd, mixed, s->halo_maxh, 3);
        if (value > 0) hm = std::min(hm, value);
        const size_t smem = halo_smem_bytes(s->nd, mixed, hm);
        const int bps = halo_prepare(s->nd, mixed, smem);
        if (bps <= 0) return s->fail(H3C_E_INVALID, "h3c_set_option: %d halo slots do not fit", hm);
        s->hmax = hm;
        s->halo_smem = smem;
        s->halo_bps = bps;
      }
      break;
    }
    case H3C_OPT_PERSISTENT_BLOCKS:
      if (value < 0) return s->fail(H3C_E_INVALID, "h3c_set_option: persistent blocks must be >= 0");
      s->persist_blocks = value;
      break;
    default: return s->fail(H3C_E_INVALID, "h3c_set_option: unknown option %d", option);
  }
  drop_graph(s);
  return H3C_OK;
}

int h3c_kernel_info(h3c_solver s, int64_t* info, int n) {
  if (!s || !info || n < 0) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_kernel_info: no grid");
  const bool euler = s->desc.physics == H3C_EULER && s->desc.reconstruction != H3C_RECON_MUSCL;
  const bool cns = cns_tile_active(s);
  const bool halo = cns || (euler && s->desc.flux == H3C_FLUX_AUSM && s->tile && s->halo && s->halo_ok);
  const long long bps = cns ? s->cns_bps : s->halo_bps;
  const int64_t grid = halo ? std::max<long long>(1, std::min<long long>(s->persist_blocks > 0 ? s->persist_blocks
                                                                         : bps * num_sms(),
                                                                         s->ntiles))
                            : (s->persist_blocks > 0 ? std::min<long long>(s->persist_blocks, s->ntiles) : s->ntiles);
  const bool ausm_tile = euler && s->desc.flux == H3C_FLUX_AUSM && s->tile;
  const bool tile512 = ausm_tile && s->euler_kernel == 4 && s->nd == 3 && s->n_inst == 1;
  const bool warpk = ausm_tile && s->euler_kernel == 3 && s->warp_bps > 0;
  const bool cellk = ausm_tile && (s->euler_kernel == 2 || s->euler_kernel == 3) && !warpk;
  const bool halo_used = halo && (cns || s->euler_kernel == 0);
  const int64_t v[8] = {tile512 ? 5 : warpk ? 4 : cellk ? 3 : halo_used ? 2 : (euler && s->tile ? 1 : 0),
                        (s->halo_ok || s->cns_ok) ? s->hmax : 0,
                        s->halo_maxh, (int64_t)std::llround(1000.0 * s->halo_mean), bps, grid,
                        (int64_t)(cns ? s->cns_smem : s->halo_smem), s->ntiles};
  for (int i = 0; i < n && i < 8; ++i) info[i] = v[i];
  return H3C_OK;
}

int h3c_instances(h3c_solver s, double* dt, double* time, int64_t* step) {
  if (!s) return H3C_E_INVALID;
  if (!s->has_grid) return s->fail(H3C_E_STATE, "h3c_instances: no grid");
  std::vector<Scalars> h(s->n_inst);
  H3C_CUDA(s, cudaMemcpyAsync(h.data(), s->d_sc, sizeof(Scalars) * s->n_inst, cudaMemcpyDeviceToHost, s->stream));
  H3C_CUDA(s, cudaStreamSynchronize(s->stream));
  for (int i = 0; i < s->n_inst; ++i) {
    if (dt) dt[i] = h[i].dt;
    if (time) time[i] = h[i].time;
    if (step) step[i] = h[i].step;
  }
  for (int i = 0; i < s->n_inst; ++i)
    if (int rc = status_error(s, h[i], i)) return rc;
  return H3C_OK;
}

// Launch configurations h3c_autotune chooses from; the index is the choice
// it returns.  persist: blocks per SM of a persistent grid (0: the kernel's
// default grid).
struct TuneCand {
  bool tile;
  int euler_kernel;
  int persist;
};
constexpr TuneCand kTune[] = {
    {true, 1, 0}, {true, 1, 1}, {true, 1, 2}, {true, 1, 3}, {true, 1, 4},  // per-lane tile (CNS: its tile kernel)
    {false, 2, 0},                                                          // generic per-cell kernels
    {true, 2, 0},                                                           // per-cell AUSM kernel
    {true, 0, 1}, {true, 0, 2}, {true, 0, 3},                               // halo-staged tile kernel
    {true, 3, 0},                                                           // warp-tiled kernel
    {true, 4, 0},                                                           // per-lane tile of 512 cells
};
constexpr int kTuneN = sizeof(kTune) / sizeof(kTune[0]);

// Whether candidate i launches a kernel of its own for this solver (the
// others would repeat a configuration already timed).
static bool tune_applies(h3c_solver s, int i) {
  const TuneCand& c = kTune[i];
  if (!c.tile) return true;
  const bool euler_ausm = s->desc.physics == H3C_EULER && s->desc.flux == H3C_FLUX_AUSM &&
                          s->desc.reconstruction != H3C_RECON_MUSCL;
  if (euler_ausm)
    return (c.euler_kernel != 0 || (s->halo && s->halo_ok)) && (c.euler_kernel != 3 || s->warp_bps > 0) &&
           (c.euler_kernel != 4 || (s->nd == 3 && s->n_inst == 1));
  if (s->desc.physics == H3C_CNS && s->halo && s->cns_ok) return c.euler_kernel == 1;
  return i == 0;  // one tile configuration where the options change nothing else
}

// Times `nsteps` steps for each launch configuration that applies (stage
// kernel x persistent grid size) from the same saved state and keeps the fastest.
int h3c_autotune(h3c_solver s, int nsteps, int* choice, double* ms_out) {
  if (!s || nsteps < 1) return H3C_E_INVALID;
  if (int rc = ready(s, "h3c_autotune")) return rc;
  const int sms = num_sms();
  const size_t qbytes = sizeof(double) * s->nv * s->ld;
  double* save = nullptr;
  Scalars* save_sc = nullptr;
  H3C_CUDA(s, cudaMalloc(&save, 2 * qbytes));
  H3C_CUDA(s, cudaMalloc(&save_sc, sizeof(Scalars) * s->n_inst));
  double* const q0 = s->d_q[0];
  double* const q1 = s->d_q[1];
  cudaMemcpyAsync(save, q0, qbytes, cudaMemcpyDeviceToDevice, s->stream);
  cudaMemcpyAsync(save + s->nv * s->ld, q1, qbytes, cudaMemcpyDeviceToDevice, s->stream);
  cudaMemcpyAsync(save_sc, s->d_sc, sizeof(Scalars) * s->n_inst, cudaMemcpyDeviceToDevice, s->stream);
  auto restore = [&]() {
    s->d_q[0] = q0;  // forward Euler swaps the buffers
    s->d_q[1] = q1;
    cudaMemcpyAsync(q0, save, qbytes, cudaMemcpyDeviceToDevice, s->stream);
    cudaMemcpyAsync(q1, save + s->nv * s->ld, qbytes, cudaMemcpyDeviceToDevice, s->stream);
    cudaMemcpyAsync(s->d_sc, save_sc, sizeof(Scalars) * s->n_inst, cudaMemcpyDeviceToDevice, s->stream);
  };
  auto apply = [&](int i) {
    s->tile = kTune[i].tile;
    s->euler_kernel = kTune[i].euler_kernel;
    s->persist_blocks = kTune[i].persist * sms;
    drop_graph(s);
  };
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int best = 0;
  double best_ms = 1e300;
  const bool prof = s->prof;
  s->prof = false;
  for (int i = 0; i < kTuneN; ++i) {
    if (!tune_applies(s, i)) continue;
    restore();
    apply(i);
    h3c_solve(s, 2);  // warm-up: a plain step (kernel attributes), then the graph captures
    cudaEventRecord(a, s->stream);
    h3c_solve(s, nsteps);
    cudaEventRecord(b, s->stream);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best_ms) {
      best_ms = ms;
      best = i;
    }
  }
  s->prof = prof;
  restore();
  apply(best);
  cudaStreamSynchronize(s->stream);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(save);
  cudaFree(save_sc);
  if (choice) *choice = best;
  if (ms_out) *ms_out = best_ms / nsteps;
  return s->cuda(cudaGetLastError(), "h3c_autotune");
}

// ---- frozen-dt stepping and the discrete adjoint ----------------------------
static int adjoint_supported(h3c_solver s, const char* what, bool coupled = false) {
  if (int rc = ready(s, what)) return rc;
  if (s->n_inst != 1) return s->fail(H3C_E_INVALID, "%s: single grids only", what);
  const bool ok_phys = ((s->desc.physics == H3C_EULER || s->desc.physics == H3C_CNS) && s->desc.flux == H3C_FLUX_AUSM) ||
                       (s->desc.physics == H3C_EULER && s->desc.flux == H3C_FLUX_LLF) || s->desc.physics == H3C_HEAT;
  if (!ok_phys) return s->fail(H3C_E_INVALID, "%s: Euler (AUSM, LLF), CNS (AUSM) and heat only", what);
  if (s->desc.physics == H3C_CNS && s->nsub > 0)
    return s->fail(H3C_E_INVALID, "%s: CNS on coarse/fine faces has no adjoint", what);
  if (s->ghost_unapplied) return s->fail(H3C_E_INVALID, "%s: a ghost cell gets no condition", what);
  for (int k = 0; k < s->n_bcs; ++k) {
    const int kind = s->h_bcs[k].kind;
    const bool cns_kind = kind >= H3C_BC_CNS_INFLOW && kind <= H3C_BC_CNS_ISOTHERMAL_NOSLIP;
    const bool cpl = kind == H3C_BC_CPL_CNS_HEAT || kind == H3C_BC_CPL_HEAT_CNS;
    if (!(kind == H3C_BC_EULER_NEUMANN || kind == H3C_BC_EULER_DIRICHLET || kind == H3C_BC_HEAT_NEUMANN ||
          kind == H3C_BC_HEAT_DIRICHLET || kind == H3C_BC_PERIODIC || (cns_kind && s->desc.physics == H3C_CNS) ||
          (cpl && coupled)))
      return s->fail(H3C_E_INVALID, "%s: condition kind %d has no adjoint here", what, kind);
  }
  return H3C_OK;
}

// One step with the given time step on explicit buffers.  st[0] is the
// step's start state; the stage inputs (ghosts filled) are left in st[0..]
// (RK2: st[1]; SSP-RK3: st[1], st[2]) and the new state in out.  For forward
// Euler out must not alias st[0]; for the Runge-Kutta schemes out == st[0] is
// allowed (in-place last stage), otherwise st[0] is copied to out first.
static void frozen_step(h3c_solver s, double* const* st, double* out, const double* d_dts, long long i) {
  const size_t Qb = sizeof(double) * s->nv * s->ld;
  launch_bc_ptr(s, st[0], st[0]);
  {
    Launch L(s, K_SCALAR);
    k_set_dt_from<<<1, 1, 0, s->stream>>>(s->d_sc, d_dts, i);
  }
  const int ti = s->desc.time_integration;
  const bool cns = s->desc.physics == H3C_CNS;
  if (s->desc.reconstruction == H3C_RECON_MUSCL) launch_grad(s, st[0]);
  if (cns) launch_slopes_ptr(s, st[0]);
  if (ti == H3C_EULER_FORWARD) {
    launch_stage(s, 0, st[0], out, false);
  } else if (ti == H3C_RUNGE_KUTTA_2) {
    launch_stage(s, 0, st[0], st[1], false);
    launch_bc_ptr(s, st[1], st[0]);
    if (out != st[0]) cudaMemcpyAsync(out, st[0], Qb, cudaMemcpyDeviceToDevice, s->stream);
    if (s->desc.reconstruction == H3C_RECON_MUSCL) launch_grad(s, st[1]);
    if (cns) launch_slopes_ptr(s, st[1]);
    launch_stage(s, 2, st[1], out, false);
  } else {
    launch_stage(s, 0, st[0], st[1], false);
    launch_bc_ptr(s, st[1], st[0]);
    cudaMemcpyAsync(st[2], st[0], Qb, cudaMemcpyDeviceToDevice, s->stream);
    if (s->desc.reconstruction == H3C_RECON_MUSCL) launch_grad(s, st[1]);
    if (cns) launch_slopes_ptr(s, st[1]);
    launch_stage(s, 3, st[1], st[2], false);
    launch_bc_ptr(s, st[2], st[0]);
    if (out != st[0]) cudaMemcpyAsync(out, st[0], Qb, cudaMemcpyDeviceToDevice, s->stream);
    if (s->desc.reconstruction == H3C_RECON_MUSCL) launch_grad(s, st[2]);
    if (cns) launch_slopes_ptr(s, st[2]);
    launch_stage(s, 4, st[2], out, false);
  }
  {
    Launch L(s, K_SCALAR);
    k_advance<<<1, 1, 0, s->stream>>>(s->d_sc, 1);
  }
}

int h3c_solve_dt(h3c_solver s, int64_t nsteps, const double* dts) {
  Range r("h3c_solve_dt");
  if (!s || nsteps < 0 || (nsteps > 0 && !dts)) return H3C_E_INVALID;
  if (int rc = ready(s, "h3c_solve_dt")) return rc;
  if (s->n_inst != 1) return s->fail(H3C_E_INVALID, "h3c_solve_dt: single grids only");
  if (nsteps == 0) return H3C_OK;
  double* d_dts = nullptr;
  H3C_CUDA(s, cudaMalloc(&d_dts, sizeof(double) * nsteps));
  cudaMemcpyAsync(d_dts, dts, sizeof(double) * nsteps, cudaMemcpyHostToDevice, s->stream);
  for (int64_t i = 0; i < nsteps; ++i) {
    if (s->desc.time_integration == H3C_EULER_FORWARD) {
      double* st[1] = {s->d_q[0]};
      frozen_step(s, st, s->d_q[1], d_dts, i);
      std::swap(s->d_q[0], s->d_q[1]);
    } else {
      double* st[3] = {s->d_q[0], s->d_q[1], s->d_q[2]};
      frozen_step(s, st, s->d_q[0], d_dts, i);
    }
  }
  launch_cfl(s, &s->d_sc->dtmin_ord);  // the next h3c_solve computes dt from this state
  cudaStreamSynchronize(s->stream);
  cudaFree(d_dts);
  return s->cuda(cudaGetLastError(), "h3c_solve_dt");
}

// Backward sweep of the discrete adjoint.  Memory: nck checkpoints + the
// stage states of one segment + 3 work + 3 cotangent states.  The forward
// stores the stage states of the last segment as it goes, so that segment
// (all of them when every >= nsteps) needs no recomputation.
int h3c_adjoint(h3c_solver s, int64_t nsteps, int64_t every, const double* dJ_dqN, double* dJ_dq0, double* dts_out) {
  Range r("h3c_adjoint");
  if (!s || nsteps < 1 || every < 0 || !dJ_dqN || !dJ_dq0) return H3C_E_INVALID;
  if (int rc = adjoint_supported(s, "h3c_adjoint")) return rc;
  const long long L = s->ld, nv = s->nv, Q = nv * L;
  const int ti = s->desc.time_integration;
  const long long per = ti == H3C_EULER_FORWARD ? 1 : ti == H3C_RUNGE_KUTTA_2 ? 2 : 3;  // stages per step
  const bool muscl = s->desc.reconstruction == H3C_RECON_MUSCL;
  // MUSCL reverse: face and ghost cotangents, own terms, limiter terms (4 states), gradient and
  // normal-equation cotangents (2 x nd nv columns), extreme-neighbour owners (nv int columns)
  const bool cnsphys = s->desc.physics == H3C_CNS;
  // CNS reverse: face cotangents (at the MUSCL face slot) and slope cotangents (at the gradient slot)
  const long long extra_m = muscl ? 4 * Q + 2 * s->nd * Q + (Q + 1) / 2 + 1 : cnsphys ? 4 * Q + s->nd * Q : 0;
  auto need = [&](long long ev) {
    const long long nck = (nsteps + ev - 1) / ev;
    return sizeof(double) * ((size_t)Q * (nck + per * ev + 7) + nsteps + extra_m);
  };
  if (every > nsteps) every = nsteps;
  if (every == 0) {  // no recomputation if that fits in half of the free memory, else ~sqrt(N) segments
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    const size_t budget = fr / 2 + s->adj_cap;
    every = nsteps;
    if (need(every) > budget) every = std::max<long long>(1, (long long)std::sqrt((double)nsteps));
    while (every > 1 && need(every) > budget) --every;
  }
  const long long nck = (nsteps + every - 1) / every;
  const size_t bytes = need(every);
  if (bytes > s->adj_cap) {
    dfree(s->d_adj);
    s->adj_cap = 0;
    if (cudaMalloc(&s->d_adj, bytes) != cudaSuccess) {
      cudaGetLastError();
      s->d_adj = nullptr;
      return s->fail(H3C_E_NOMEM, "h3c_adjoint: %zu bytes of checkpoints do not fit (%lld checkpoints + %lld stage states)",
                     bytes, nck, per * every);
    }
    s->adj_cap = bytes;
  }
  double* ck = s->d_adj;
  double* seg = ck + Q * nck;
  double* work = seg + Q * per * every;
  double* lam = work + Q * 3;
  double* d_dts = lam + Q * 4;
  double* m_qface = d_dts + nsteps;  // MUSCL reverse buffers (unused otherwise)
  double* m_qghost = m_qface + Q;
  double* m_wself = m_qghost + Q;
  double* m_dl1 = m_wself + Q;
  double* m_gbar = m_dl1 + Q;
  double* m_bbar = m_gbar + s->nd * Q;
  int* m_owner = reinterpret_cast<int*>(m_bbar + s->nd * Q);
  const long long last0 = (nck - 1) * every;  // first step of the last segment
  // ---- forward: the solver's own step (CFL dt), checkpoints, dt record ----
  const bool fuse = !s->unfused_dt;
  for (int64_t i = 0; i < nsteps; ++i) {
    if (i % every == 0)
      cudaMemcpyAsync(ck + Q * (i / every), s->d_q[0], sizeof(double) * Q, cudaMemcpyDeviceToDevice, s->stream);
    enqueue_step(s, fuse, i >= last0 ? seg + Q * per * (i - last0) : nullptr, d_dts, i);
  }
  Scalars saved;
  cudaMemcpyAsync(&saved, s->d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, s->stream);
  // ---- cotangent of the final state (caller numbering -> internal) ----
  double* lamA = lam;          // lambda^{n+1}
  double* lamB = lam + Q;      // lambda^n
  double* lamC = lam + 2 * Q;  // last-stage input cotangent (RK2, SSP-RK3)
  double* lamD = lam + 3 * Q;  // first-stage output cotangent (SSP-RK3)
  cudaMemsetAsync(lam, 0, sizeof(double) * Q * 4, s->stream);
  if (int rc = ensure_stage(s, s->n_caller)) return rc;
  // host or device arrays (unified addressing)
  for (int v = 0; v < nv; ++v)
    cudaMemcpyAsync(s->d_stage + v * s->n_caller, dJ_dqN + v * s->n_caller, sizeof(double) * s->n_caller,
                    cudaMemcpyDefault, s->stream);
  k_gather<<<blocks(s->n_int), kBlock, 0, s->stream>>>(s->d_stage, s->n_caller, lamA, L, s->d_dev2caller, s->n_int, (int)nv);
  ++s->launches;
  auto adj = [&](const double* qin, const double* lamin, double* gout, double alpha, double beta,
                 const double* extra = nullptr, double gam = 0.0, const double* extra2 = nullptr,
                 double gam2 = 0.0) {
    const Geometry g = geometry(s);
    const GhostTables gt = ghosts(s);
    if (cnsphys) {
      launch_slopes_ptr(s, qin);  // the forward's cell slopes of this stage input
      Launch La(s, K_OTHER);
      const unsigned nb = (unsigned)blocks(s->n_int);
      if (s->nd == 2) {
        (s->cns_adj_dual ? k_adjc_face<2, false> : k_adjc_face<2, true>)<<<nb, kBlock, 0, s->stream>>>(
            qin, s->d_slopes, lamin, alpha, g, gt, s->pc, s->d_sc, nullptr, m_qface, m_gbar, nullptr);
        k_adjc_slopes<2><<<nb, kBlock, 0, s->stream>>>(qin, lamin, extra, extra2, beta, gam, gam2, g, gt, s->pc,
                                                       nullptr, m_qface, m_gbar, nullptr, gout);
      } else {
        (s->cns_adj_dual ? k_adjc_face<3, false> : k_adjc_face<3, true>)<<<nb, kBlock, 0, s->stream>>>(
            qin, s->d_slopes, lamin, alpha, g, gt, s->pc, s->d_sc, nullptr, m_qface, m_gbar, nullptr);
        k_adjc_slopes<3><<<nb, kBlock, 0, s->stream>>>(qin, lamin, extra, extra2, beta, gam, gam2, g, gt, s->pc,
                                                       nullptr, m_qface, m_gbar, nullptr, gout);
      }
      s->launches += 1;  // two kernels under one Launch record
      return;
    }
    if (muscl) {
      launch_grad(s, qin);  // the forward's limited gradients of this stage input
      Launch La(s, K_OTHER);
      const unsigned nb = (unsigned)blocks(s->n_int);
      const double K = s->desc.limiter_k;
#define H3C_ADJM(ND, HANG)                                                                                          \
  k_adjm_face<ND, HANG><<<nb, kBlock, 0, s->stream>>>(qin, s->d_slopes, s->d_xc, lamin, alpha, g, gt, s->pc, s->d_sc, \
                                                      m_qface, m_gbar);                                              \
  k_adjm_lim<ND, HANG><<<nb, kBlock, 0, s->stream>>>(qin, s->d_xc, m_gbar, g, gt, s->pc, K, m_bbar, m_dl1, m_owner,   \
                                                     m_wself, m_qghost);                                             \
  k_adjm_gather<ND, HANG><<<nb, kBlock, 0, s->stream>>>(qin, s->d_xc, lamin, extra, extra2, beta, gam, gam2, g, gt,    \
                                                        s->pc, m_bbar, m_dl1, m_owner, m_wself, m_qface, m_qghost,   \
                                                        gout)
      if (s->nd == 2) {
        if (s->nsub > 0) { H3C_ADJM(2, true); } else { H3C_ADJM(2, false); }
      } else {
        if (s->nsub > 0) { H3C_ADJM(3, true); } else { H3C_ADJM(3, false); }
      }
#undef H3C_ADJM
      s->launches += 2;  // three kernels under one Launch record
      return;
    }
    Launch La(s, K_OTHER);
    if (s->desc.physics == H3C_EULER && s->desc.flux == H3C_FLUX_LLF) {  // the per-cell gather
      if (s->nd == 2)
        k_adj_stage<2, EULER, LLF><<<blocks(s->n_int), kBlock, 0, s->stream>>>(qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2, nullptr, g, gt, s->pc, s->d_sc);
      else
        k_adj_stage<3, EULER, LLF><<<blocks(s->n_int), kBlock, 0, s->stream>>>(qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2, nullptr, g, gt, s->pc, s->d_sc);
      return;
    }
    if (s->desc.physics == H3C_EULER && s->tile) {
      if (s->nd == 2) {
        if (s->nsub > 0) adj_ausm_t<2, true>(s, qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2);
        else adj_ausm_t<2, false>(s, qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2);
      } else {
        if (s->nsub > 0) adj_ausm_t<3, true>(s, qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2);
        else adj_ausm_t<3, false>(s, qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2);
      }
      return;
    }
    if (s->nd == 2) {
      if (s->desc.physics == H3C_HEAT)
        k_adj_stage<2, HEAT><<<blocks(s->n_int), kBlock, 0, s->stream>>>(qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2, nullptr, g, gt, s->pc, s->d_sc);
      else
        k_adj_stage<2, EULER><<<blocks(s->n_int), kBlock, 0, s->stream>>>(qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2, nullptr, g, gt, s->pc, s->d_sc);
    } else {
      if (s->desc.physics == H3C_HEAT)
        k_adj_stage<3, HEAT><<<blocks(s->n_int), kBlock, 0, s->stream>>>(qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2, nullptr, g, gt, s->pc, s->d_sc);
      else
        k_adj_stage<3, EULER><<<blocks(s->n_int), kBlock, 0, s->stream>>>(qin, lamin, gout, extra, extra2, alpha, beta, gam, gam2, nullptr, g, gt, s->pc, s->d_sc);
    }
  };
  // ---- backward over segments; all but the last recompute their stage states from the checkpoint ----
  for (long long k = nck - 1; k >= 0; --k) {
    const long long i0 = k * every, i1 = std::min<long long>(nsteps, i0 + every);
    if (k != nck - 1) {
      double* cur = work;
      cudaMemcpyAsync(cur, ck + Q * k, sizeof(double) * Q, cudaMemcpyDeviceToDevice, s->stream);
      for (long long i = i0; i < i1; ++i) {
        double* s0 = seg + Q * per * (i - i0);
        cudaMemcpyAsync(s0, cur, sizeof(double) * Q, cudaMemcpyDeviceToDevice, s->stream);
        double* nxt = (cur == work) ? work + Q : work;
        double* st[3] = {s0, s0 + Q, s0 + 2 * Q};
        frozen_step(s, st, nxt, d_dts, i);
        cur = nxt;
      }
    }
    for (long long i = i1 - 1; i >= i0; --i) {
      double* s0 = seg + Q * per * (i - i0);
      {
        Launch L3(s, K_SCALAR);
        k_set_dt_from<<<1, 1, 0, s->stream>>>(s->d_sc, d_dts, i);
      }
      if (ti == H3C_EULER_FORWARD) {
        adj(s0, lamA, lamB, 1.0, 1.0);
      } else if (ti == H3C_RUNGE_KUTTA_2) {
        // lambda* = 0.5 lambda + VJP(q*; 0.5 lambda); lambda^n = 0.5 lambda + lambda* + VJP(q^n; lambda*)
        adj(s0 + Q, lamA, lamC, 0.5, 0.5);
        adj(s0, lamC, lamB, 1.0, 1.0, lamA, 0.5);
      } else {
        // q' = 1/3 q + 2/3 (q2 + R(q2)), q2 = 3/4 q + 1/4 (q1 + R(q1)), q1 = q + R(q):
        // l2 = 2/3 (l + VJP(q2; l)), l1 = 1/4 (l2 + VJP(q1; l2)), l^n = l1 + VJP(q; l1) + 1/3 l + 3/4 l2
        adj(s0 + 2 * Q, lamA, lamC, 2.0 / 3.0, 2.0 / 3.0);
        adj(s0 + Q, lamC, lamD, 0.25, 0.25);
        adj(s0, lamD, lamB, 1.0, 1.0, lamA, 1.0 / 3.0, lamC, 0.75);
      }
      std::swap(lamA, lamB);
    }
  }
  // ---- gradient (internal -> caller numbering), dt sequence ----
  cudaMemsetAsync(s->d_stage, 0, sizeof(double) * nv * s->n_caller, s->stream);
  k_scatter<<<blocks(s->n_int), kBlock, 0, s->stream>>>(lamA, L, s->d_stage, s->n_caller, s->d_dev2caller, s->n_int, (int)nv);
  ++s->launches;
  for (int v = 0; v < nv; ++v)
    cudaMemcpyAsync(dJ_dq0 + v * s->n_caller, s->d_stage + v * s->n_caller, sizeof(double) * s->n_caller,
                    cudaMemcpyDefault, s->stream);
  if (dts_out) cudaMemcpyAsync(dts_out, d_dts, sizeof(double) * nsteps, cudaMemcpyDefault, s->stream);
  // the solver is left at step N with the scalars of the forward run
  cudaStreamSynchronize(s->stream);
  cudaMemcpyAsync(s->d_sc, &saved, sizeof(Scalars), cudaMemcpyHostToDevice, s->stream);
  H3C_CUDA(s, cudaStreamSynchronize(s->stream));
  return s->cuda(cudaGetLastError(), "h3c_adjoint");
}

// ---- adjoint of the coupled conjugate-heat loop ----------------------------
// lam_f += xbar dT_f/dq at the fluid cell each heat interface ghost reads
// (T_f = gamma p / rho of the fluid state after its step)
__global__ void k_cht_heat_to_fluid(const double* __restrict__ xbar, GhostTables gth, const double* __restrict__ qf,
                                    long long ldf, int ndf, double gammaf, double* __restrict__ lamf) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gth.ng) return;
  const int b = gth.bc_apply[i];
  if (b == 255 || gth.bcs[b].kind != BC_CPL_HEAT_CNS) return;
  const int P = gth.partner[i];
  if (P < 0) return;
  const double xb = xbar[i];
  const double rho = qf[ndf * ldf + P], rinv = 1.0 / rho;
  double um2 = 0.0, u[3] = {0, 0, 0};
  for (int d = 0; d < ndf; ++d) {
    u[d] = qf[d * ldf + P] * rinv;
    um2 += u[d] * u[d];
  }
  const double gm1 = gammaf - 1.0;
  const double p = gm1 * (qf[(ndf + 1) * ldf + P] - 0.5 * rho * um2);
  for (int d = 0; d < ndf; ++d) atomicAdd(lamf + d * ldf + P, xb * (-gammaf * gm1 * u[d] * rinv));
  atomicAdd(lamf + ndf * ldf + P, xb * gammaf * (0.5 * gm1 * um2 - p * rinv) * rinv);
  atomicAdd(lamf + (ndf + 1) * ldf + P, xb * gammaf * gm1 * rinv);
}
// lam_s += tbar at the solid cell each fluid interface ghost reads
__global__ void k_cht_fluid_to_heat(const double* __restrict__ tbar, GhostTables gtf, double* __restrict__ lams) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gtf.ng) return;
  const int b = gtf.bc_apply[i];
  if (b == 255 || gtf.bcs[b].kind != BC_CPL_CNS_HEAT) return;
  const int Q = gtf.partner[i];
  if (Q < 0) return;
  atomicAdd(lams + Q, tbar[i]);
}

static void caller_to_internal(h3c_solver s, const double* src, double* dst) {
  for (int v = 0; v < s->nv; ++v)
    cudaMemcpyAsync(s->d_stage + v * s->n_caller, src + v * s->n_caller, sizeof(double) * s->n_caller,
                    cudaMemcpyDefault, s->stream);
  k_gather<<<blocks(s->n_int), kBlock, 0, s->stream>>>(s->d_stage, s->n_caller, dst, s->ld, s->d_dev2caller, s->n_int,
                                                       s->nv);
  ++s->launches;
}
static void internal_to_caller(h3c_solver s, const double* src, double* dst) {
  cudaMemsetAsync(s->d_stage, 0, sizeof(double) * s->nv * s->n_caller, s->stream);
  k_scatter<<<blocks(s->n_int), kBlock, 0, s->stream>>>(src, s->ld, s->d_stage, s->n_caller, s->d_dev2caller, s->n_int,
                                                        s->nv);
  ++s->launches;
  for (int v = 0; v < s->nv; ++v)
    cudaMemcpyAsync(dst + v * s->n_caller, s->d_stage + v * s->n_caller, sizeof(double) * s->n_caller,
                    cudaMemcpyDefault, s->stream);
}

int h3c_cht_adjoint(h3c_solver cns, h3c_solver heat, double Tr0, int64_t nsteps, int64_t every,
                    const double* dJ_dqN, const double* dJ_dTN, double* dJ_dq0, double* dJ_dT0, double* dts) {
  Range r("h3c_cht_adjoint");
  if (!cns || !heat || nsteps < 1 || every < 0 || !dJ_dqN || !dJ_dTN || !dJ_dq0 || !dJ_dT0) return H3C_E_INVALID;
  if (int rc = adjoint_supported(cns, "h3c_cht_adjoint", true)) return rc;
  if (int rc = adjoint_supported(heat, "h3c_cht_adjoint", true)) return rc;
  if (cns->desc.physics != H3C_CNS || heat->desc.physics != H3C_HEAT)
    return cns->fail(H3C_E_INVALID, "h3c_cht_adjoint: expects (cns, heat)");
  if (cns->stream != heat->stream || cns->partner != heat || heat->partner != cns)
    return cns->fail(H3C_E_STATE, "h3c_cht_adjoint: solvers are not coupled with each other");
  if (cns->desc.time_integration != H3C_EULER_FORWARD || heat->desc.time_integration != H3C_EULER_FORWARD)
    return cns->fail(H3C_E_INVALID, "h3c_cht_adjoint: forward Euler (the coupled loop's scheme) only");
  if (cns->unfused_dt || heat->unfused_dt) return cns->fail(H3C_E_INVALID, "h3c_cht_adjoint: unsupported condition");
  if (every == 0 || every > nsteps) every = std::min<int64_t>(nsteps, every == 0 ? 100 : every);
  const double scaling = Tr0 * cns->Pr0 * cns->Re0;
  const long long Qf = (long long)cns->nv * cns->ld, Qs = (long long)heat->nv * heat->ld;
  const long long nck = (nsteps + every - 1) / every;
  // workspace: checkpoints, stage inputs of one segment (+ the fluid state after it), work and cotangent states,
  // CNS reverse buffers, per-ghost cross cotangents, dt records
  const size_t nd = (size_t)Qf * (nck + (every + 1) + 2 + 3 + 1 + cns->nd) + (size_t)Qs * (nck + every + 2 + 2) +
                    (size_t)heat->ng + (size_t)cns->ng + 2 * (size_t)nsteps + 2 * (size_t)every + 8;
  double* ws = nullptr;
  if (cudaMalloc(&ws, sizeof(double) * nd) != cudaSuccess) {
    cudaGetLastError();
    return cns->fail(H3C_E_NOMEM, "h3c_cht_adjoint: %zu bytes of checkpoints do not fit", sizeof(double) * nd);
  }
  double* p = ws;
  auto take = [&](size_t n) { double* r = p; p += n; return r; };
  double* ckf = take(Qf * nck);
  double* cks = take(Qs * nck);
  double* segf = take(Qf * (every + 1));
  double* segs = take(Qs * every);
  double* wf = take(2 * Qf);
  double* wsd = take(2 * Qs);
  double* lf = take(3 * Qf);
  double* ls = take(2 * Qs);
  double* qface = take(Qf);
  double* sbar = take(cns->nd * Qf);
  double* xbar = take(std::max<long long>(1, heat->ng));
  double* tbar = take(std::max<long long>(1, cns->ng));
  double* dtf = take(nsteps);
  double* dth = take(nsteps);
  double* sdtf = take(every);  // one segment's time steps (the captured segment graphs read and write these)
  double* sdth = take(every);
  cudaStream_t st = cns->stream;
  // Full segments are captured once as CUDA graphs (forward and backward) and
  // replayed: their buffers are fixed and their time steps go through
  // sdtf / sdth.  An even segment length returns forward Euler's swapped
  // state buffers to where the capture started.
  const bool seg_graphs = cns->graphs && heat->graphs && !cns->prof && !heat->prof && every % 2 == 0;
  auto capture = [&](auto&& body, cudaGraphExec_t* exec, long long* launches) -> bool {
    const long long lc = cns->launches, lh = heat->launches;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    double* saved[4] = {cns->d_q[0], cns->d_q[1], heat->d_q[0], heat->d_q[1]};
    body();
    cns->d_q[0] = saved[0];  // the capture ran no step
    cns->d_q[1] = saved[1];
    heat->d_q[0] = saved[2];
    heat->d_q[1] = saved[3];
    *launches = (cns->launches - lc) + (heat->launches - lh);
    cns->launches = lc;
    heat->launches = lh;
    bool ok = cudaStreamEndCapture(st, &g) == cudaSuccess && g && cudaGraphInstantiate(exec, g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
      cudaGetLastError();
      *exec = nullptr;
    }
    return ok;
  };
  cudaGraphExec_t gfwd = nullptr, gbwd = nullptr;
  long long nl_fwd = 0, nl_bwd = 0;
  if (int rc = ensure_stage(cns, cns->n_caller)) { cudaFree(ws); return rc; }
  if (int rc = ensure_stage(heat, heat->n_caller)) { cudaFree(ws); return rc; }
  // ---- forward: the coupled loop (coupling::apply, cns step, heat step), checkpoints, dt records ----
  auto fwd_seg = [&](long long n) {
    for (long long j = 0; j < n; ++j) {
      launch_cfl(cns, &cns->d_sc->mindt_ord);
      launch_cfl(heat, &heat->d_sc->mindt_ord);
      {
        Launch L(cns, K_SCALAR);
        k_couple_cht<<<1, 1, 0, st>>>(cns->d_sc, heat->d_sc, scaling);
      }
      enqueue_step(cns, true, nullptr, sdtf, j);
      enqueue_step(heat, true, nullptr, sdth, j);
    }
  };
  for (long long k = 0; k < nck; ++k) {
    const long long i0 = k * every, i1 = std::min<long long>(nsteps, i0 + every);
    cudaMemcpyAsync(ckf + Qf * k, cns->d_q[0], sizeof(double) * Qf, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(cks + Qs * k, heat->d_q[0], sizeof(double) * Qs, cudaMemcpyDeviceToDevice, st);
    if (seg_graphs && i1 - i0 == every && (gfwd || capture([&] { fwd_seg(every); }, &gfwd, &nl_fwd))) {
      cudaGraphLaunch(gfwd, st);
      cns->launches += nl_fwd;
    } else {
      fwd_seg(i1 - i0);
    }
    cudaMemcpyAsync(dtf + i0, sdtf, sizeof(double) * (i1 - i0), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(dth + i0, sdth, sizeof(double) * (i1 - i0), cudaMemcpyDeviceToDevice, st);
  }
  Scalars savf, savs;
  cudaMemcpyAsync(&savf, cns->d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&savs, heat->d_sc, sizeof(Scalars), cudaMemcpyDeviceToHost, st);
  // ---- terminal cotangents ----
  double *lfA = lf, *lfB = lf + Qf, *lfT = lf + 2 * Qf, *lsA = ls, *lsB = ls + Qs;
  cudaMemsetAsync(lf, 0, sizeof(double) * 3 * Qf, st);
  cudaMemsetAsync(ls, 0, sizeof(double) * 2 * Qs, st);
  caller_to_internal(cns, dJ_dqN, lfA);
  caller_to_internal(heat, dJ_dTN, lsA);
  const Geometry gf = geometry(cns), gs = geometry(heat);
  const GhostTables gtf = ghosts(cns), gts = ghosts(heat);
  const unsigned nbf = (unsigned)blocks(cns->n_int), nbs = (unsigned)blocks(heat->n_int);
  // ---- backward over segments, each recomputed from its checkpoint ----
  // The segment body works on fixed buffers: the checkpoint is copied into
  // wf / wsd, the segment's time steps into sdtf / sdth, and the cotangents
  // stay in lf / ls (an even number of swaps per full segment).
  auto bwd_seg = [&](long long n) {
    double *curf = wf, *curs = wsd;
    for (long long j = 0; j < n; ++j) {
      double* sf0 = segf + Qf * j;
      double* ss0 = segs + Qs * j;
      cudaMemcpyAsync(sf0, curf, sizeof(double) * Qf, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(ss0, curs, sizeof(double) * Qs, cudaMemcpyDeviceToDevice, st);
      double* nxf = (curf == wf) ? wf + Qf : wf;
      double* nxs = (curs == wsd) ? wsd + Qs : wsd;
      cns->partner_override = ss0;  // the fluid's wall conditions read the solid before its step
      double* stf[1] = {sf0};
      frozen_step(cns, stf, nxf, sdtf, j);
      heat->partner_override = nxf;  // the solid's conditions read the fluid after its step
      double* sts[1] = {ss0};
      frozen_step(heat, sts, nxs, sdth, j);
      cns->partner_override = nullptr;
      heat->partner_override = nullptr;
      curf = nxf;
      curs = nxs;
    }
    cudaMemcpyAsync(segf + Qf * n, curf, sizeof(double) * Qf, cudaMemcpyDeviceToDevice, st);
    for (long long j = n - 1; j >= 0; --j) {
      double* sf0 = segf + Qf * j;
      double* sf1 = segf + Qf * (j + 1);  // fluid state after step j
      double* ss0 = segs + Qs * j;
      {
        Launch L(cns, K_SCALAR);
        k_set_dt_from<<<1, 1, 0, st>>>(cns->d_sc, sdtf, j);
        k_set_dt_from<<<1, 1, 0, st>>>(heat->d_sc, sdth, j);
        ++cns->launches;
      }
      // heat step: lam_s^i = (I + dR_s/dT_s)^T lam_s^{i+1}; its interface reads of T_f -> fluid cotangent
      cudaMemsetAsync(xbar, 0, sizeof(double) * std::max<long long>(1, heat->ng), st);
      {
        Launch L(heat, K_OTHER);
        if (heat->nd == 2)
          k_adj_stage<2, HEAT><<<nbs, kBlock, 0, st>>>(ss0, lsA, lsB, nullptr, nullptr, 1.0, 1.0, 0.0, 0.0, xbar, gs, gts,
                                                       heat->pc, heat->d_sc);
        else
          k_adj_stage<3, HEAT><<<nbs, kBlock, 0, st>>>(ss0, lsA, lsB, nullptr, nullptr, 1.0, 1.0, 0.0, 0.0, xbar, gs, gts,
                                                       heat->pc, heat->d_sc);
      }
      cudaMemcpyAsync(lfT, lfA, sizeof(double) * Qf, cudaMemcpyDeviceToDevice, st);
      k_cht_heat_to_fluid<<<blocks(std::max<long long>(1, heat->ng)), kBlock, 0, st>>>(xbar, gts, sf1, cns->ld, cns->nd,
                                                                                        cns->desc.gamma, lfT);
      ++heat->launches;
      // fluid step: lam_f^i = (I + dR_f/dq_f)^T lam~_f; its wall reads of T_s -> solid cotangent
      cudaMemsetAsync(tbar, 0, sizeof(double) * std::max<long long>(1, cns->ng), st);
      launch_slopes_ptr(cns, sf0);
      {
        Launch L(cns, K_OTHER);
        if (cns->nd == 2) {
          (cns->cns_adj_dual ? k_adjc_face<2, false> : k_adjc_face<2, true>)<<<nbf, kBlock, 0, st>>>(
              sf0, cns->d_slopes, lfT, 1.0, gf, gtf, cns->pc, cns->d_sc, ss0, qface, sbar, tbar);
          k_adjc_slopes<2><<<nbf, kBlock, 0, st>>>(sf0, lfT, nullptr, nullptr, 1.0, 0.0, 0.0, gf, gtf, cns->pc, ss0,
                                                   qface, sbar, tbar, lfB);
        } else {
          (cns->cns_adj_dual ? k_adjc_face<3, false> : k_adjc_face<3, true>)<<<nbf, kBlock, 0, st>>>(
              sf0, cns->d_slopes, lfT, 1.0, gf, gtf, cns->pc, cns->d_sc, ss0, qface, sbar, tbar);
          k_adjc_slopes<3><<<nbf, kBlock, 0, st>>>(sf0, lfT, nullptr, nullptr, 1.0, 0.0, 0.0, gf, gtf, cns->pc, ss0,
                                                   qface, sbar, tbar, lfB);
        }
        ++cns->launches;
      }
      k_cht_fluid_to_heat<<<blocks(std::max<long long>(1, cns->ng)), kBlock, 0, st>>>(tbar, gtf, lsB);
      ++cns->launches;
      std::swap(lfA, lfB);
      std::swap(lsA, lsB);
    }
  };
  for (long long k = nck - 1; k >= 0; --k) {
    const long long i0 = k * every, i1 = std::min<long long>(nsteps, i0 + every);
    cudaMemcpyAsync(wf, ckf + Qf * k, sizeof(double) * Qf, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(wsd, cks + Qs * k, sizeof(double) * Qs, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(sdtf, dtf + i0, sizeof(double) * (i1 - i0), cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(sdth, dth + i0, sizeof(double) * (i1 - i0), cudaMemcpyDeviceToDevice, st);
    if (seg_graphs && i1 - i0 == every) {
      double *a0 = lfA, *b0 = lfB, *c0 = lsA, *d0 = lsB;
      if (!gbwd && !capture([&] { bwd_seg(every); }, &gbwd, &nl_bwd)) {
        lfA = a0, lfB = b0, lsA = c0, lsB = d0;  // a failed capture ran nothing
        bwd_seg(every);
      } else {
        lfA = a0, lfB = b0, lsA = c0, lsB = d0;  // an even number of swaps: the same buffers
        cudaGraphLaunch(gbwd, st);
        cns->launches += nl_bwd;
      }
    } else {
      bwd_seg(i1 - i0);
    }
  }
  internal_to_caller(cns, lfA, dJ_dq0);
  internal_to_caller(heat, lsA, dJ_dT0);
  if (dts) {
    cudaMemcpyAsync(dts, dtf, sizeof(double) * nsteps, cudaMemcpyDefault, st);
    cudaMemcpyAsync(dts + nsteps, dth, sizeof(double) * nsteps, cudaMemcpyDefault, st);
  }
  cudaStreamSynchronize(st);
  // both solvers are left at step N with the scalars of the forward run
  cudaMemcpyAsync(cns->d_sc, &savf, sizeof(Scalars), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(heat->d_sc, &savs, sizeof(Scalars), cudaMemcpyHostToDevice, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (gfwd) cudaGraphExecDestroy(gfwd);
  if (gbwd) cudaGraphExecDestroy(gbwd);
  cudaFree(ws);
  if (e != cudaSuccess) return cns->cuda(e, "h3c_cht_adjoint");
  return cns->cuda(cudaGetLastError(), "h3c_cht_adjoint");
}

int h3c_launches(h3c_solver s, int64_t* n) {
  if (!s || !n) return H3C_E_INVALID;
  *n = s->launches;
  return H3C_OK;
}

int h3c_profile(h3c_solver s, int enable) {
  if (!s) return H3C_E_INVALID;
  s->prof = enable != 0;
  return H3C_OK;
}

int h3c_profile_read(h3c_solver s, double* ms, int64_t* count, int nkinds) {
  if (!s || !ms || !count || nkinds <= 0) return H3C_E_INVALID;
  H3C_CUDA(s, cudaStreamSynchronize(s->stream));
  for (int k = 0; k < nkinds; ++k) { ms[k] = 0; count[k] = 0; }
  for (auto& r : s->prof_rec) {
    float t = 0;
    H3C_CUDA(s, cudaEventElapsedTime(&t, r.second.first, r.second.second));
    if (r.first < nkinds) { ms[r.first] += t; count[r.first] += 1; }
    s->ev_pool.push_back(r.second.first);
    s->ev_pool.push_back(r.second.second);
  }
  s->prof_rec.clear();
  return H3C_OK;
}

}  // extern "C"
