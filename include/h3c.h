/* h3c.h -- C ABI of hom3_b200, the B200 (sm_100a) finite-volume hot path that
 * drops in for hom3's Solver::solve().
 *
 * hom3 (gnzlbg/hom3) is a header-only C++ library whose plugin interface is
 * compile-time (CRTP physics plugins, type-erased boundary conditions).  The
 * entry points below are what a hom3 maintainer binds from C++ to move the
 * step onto the GPU: the solver keeps building its grid and ghost cells on the
 * host (Solver::initialize, src/solver/fv/solver.hpp:133-138) and hands the
 * resulting cell tables to h3c_set_grid; Solver::solve() (solver.hpp:140-145)
 * becomes h3c_solve.  Every entry point names the hom3 interface it replaces.
 *
 * Conventions
 *  - Every function returns 0 on success or a negative H3C_E* code; the
 *    message is available from h3c_last_error().  Nothing here exits.
 *  - Cell numbering at this boundary is the caller's (hom3's container order:
 *    internal cells [0, first_ghost), ghost cells [first_ghost, n_cells)
 *    sorted by bc id, container.hpp:58-66, solver.hpp:811-834).  Internally
 *    cells are renumbered along a Morton space-filling curve.
 *  - State arrays are column-major (n x nv with leading dimension ld), the
 *    layout of hom3's lhs/rhs Eigen columns (container.hpp:59-60).
 *  - A solver owns all of its device memory and runs on its own CUDA stream;
 *    coupled solvers share one stream (h3c_set_partner).  One handle must not
 *    be used from two host threads at once.
 */
#ifndef H3C_H_
#define H3C_H_
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define H3C_ABI_VERSION 1

/* error codes */
#define H3C_OK 0
#define H3C_E_INVALID (-1)   /* invalid argument or inconsistent tables */
#define H3C_E_CUDA (-2)      /* CUDA runtime error */
#define H3C_E_NONFINITE (-3) /* dt or state became non-finite / non-positive */
#define H3C_E_STATE (-4)     /* call made in the wrong state (e.g. no grid yet) */
#define H3C_E_TIMEOUT (-5)   /* a bounded device wait ran out */
#define H3C_E_NOMEM (-6)     /* device allocation failed */

/* physics: euler/physics.hpp:25, cns/physics.hpp:27, heat/physics.hpp:21,
 * advection/physics.hpp:21-149 (one scalar q carried by a given velocity
 * field u(x), h3c_set_velocity) */
#define H3C_EULER 0
#define H3C_CNS 1
#define H3C_HEAT 2
#define H3C_ADVECTION 3
/* numerical flux tags: euler/tags.hpp:13-16 (AUSM, LLF); cns/tags.hpp:22
 * (standard = AUSM + three-point viscous, selected by H3C_CNS + AUSM);
 * heat/tags.hpp:13 (three_point, the only heat flux). */
#define H3C_FLUX_AUSM 0
#define H3C_FLUX_LLF 1
/* advection/tags.hpp:14-15: local Lax-Friedrichs (H3C_FLUX_LLF) or upwind.
 * hom3's upwind flux is u_L q_L, negated when the face velocity
 * (u_L + u_R)/2 is negative (advection/physics.hpp:132-145); reproduced. */
#define H3C_FLUX_UPWIND 2
/* time integration tags: solver/fv/tags.hpp:24-25 */
#define H3C_EULER_FORWARD 0
#define H3C_RUNGE_KUTTA_2 1
/* EXTENSION (not in hom3): three-stage strong-stability-preserving
 * Runge-Kutta in Shu-Osher form, q1 = q + dt R(q),
 * q2 = 3/4 q + 1/4 (q1 + dt R(q1)), q' = 1/3 q + 2/3 (q2 + dt R(q2)),
 * conditions applied before every stage. */
#define H3C_SSPRK3 2
/* reconstruction of the face states.  EXTENSION (not in hom3, which is
 * first order, solver.hpp:45-49): MUSCL on the primitive variables
 * (u, rho, p) with least-squares gradients over the face neighbours and
 * Venkatakrishnan's limiter, eps^2 = (limiter_k h)^3.  Euler with AUSM. */
#define H3C_RECON_NONE 0
#define H3C_RECON_MUSCL 1
/* arithmetic of the face fluxes (the state, residual and dt stay FP64) */
#define H3C_FP64 0
#define H3C_MIXED 1 /* FP32 reconstruction + face flux, FP64 update */

/* Boundary / coupling conditions.  Values v[] per kind:
 *  EULER_NEUMANN      surface flux per variable (euler/boundary_conditions.hpp:17-43)
 *  EULER_DIRICHLET    surface state per variable (:47-67)
 *  EULER_VORTEX       none; analytic isentropic vortex, overwrites the
 *                     boundary cell too (:71-93, euler/initial_conditions.hpp:14-39)
 *  CNS_INFLOW         surface primitive state (u_0..u_{nd-1}, rho, p); u and
 *                     rho imposed, zero normal pressure gradient (cns/boundary_conditions.hpp:28-65)
 *  CNS_OUTFLOW        same layout, only p is used (:72-105)
 *  CNS_ADIABATIC_NOSLIP / CNS_ADIABATIC_SLIP   none (:117-193)
 *  CNS_ISOTHERMAL_NOSLIP  v[0] = wall temperature (:200-238)
 *  HEAT_DIRICHLET     v[0] = surface temperature (heat/boundary_conditions.hpp:15-37)
 *  HEAT_NEUMANN       v[0] = surface heat flux (:40-63)
 *  ADV_DIRICHLET      v[0] = surface value (advection/boundary_conditions.hpp:15-37)
 *  ADV_NEUMANN        v[0] = surface flux (:40-63)
 *  ADV_CHARACTERISTIC none (:66-94; both of its branches give the boundary cell's value)
 *  CPL_*              coupling with the partner solver (h3c_set_partner):
 *                     euler/coupling_conditions.hpp:17-35, cns/coupling_conditions.hpp:22-43,
 *                     heat/coupling_conditions.hpp:18-61.  CPL_CNS_HEAT / CPL_HEAT_CNS:
 *                     EXTENSION v[0] = conductivity ratio kappa = k_solid / k_fluid, interface
 *                     temperature (T_fluid + kappa T_solid) / (1 + kappa) (flux continuity for
 *                     equal cells); 0 or 1 gives hom3's mean 0.5 (T_fluid + T_solid) */
#define H3C_BC_EULER_NEUMANN 0
#define H3C_BC_EULER_DIRICHLET 1
#define H3C_BC_EULER_VORTEX 2
#define H3C_BC_CNS_INFLOW 3
#define H3C_BC_CNS_OUTFLOW 4
#define H3C_BC_CNS_ADIABATIC_NOSLIP 5
#define H3C_BC_CNS_ADIABATIC_SLIP 6
#define H3C_BC_CNS_ISOTHERMAL_NOSLIP 7
#define H3C_BC_HEAT_DIRICHLET 8
#define H3C_BC_HEAT_NEUMANN 9
#define H3C_BC_CPL_EULER_EULER 10
#define H3C_BC_CPL_CNS_HEAT 11
#define H3C_BC_CPL_HEAT_CNS 12
#define H3C_BC_CPL_HEAT_HEAT 13
/* EXTENSION (not in hom3): periodic pairing of opposite cube faces; the
 * caller supplies the partner cell of each ghost through h3c_set_periodic. */
#define H3C_BC_PERIODIC 14
#define H3C_BC_ADV_DIRICHLET 15
#define H3C_BC_ADV_NEUMANN 16
#define H3C_BC_ADV_CHARACTERISTIC 17
/* EXTENSION (not in hom3, which has no domain decomposition): the ghost is a
 * cell of a neighbouring subdomain (another solver holding another part of
 * the same grid); the library leaves its state as the caller writes it
 * between the parts of a step (h3c_solve_stage).  Any physics. */
#define H3C_BC_EXCHANGE 18

typedef struct h3c_solver_s* h3c_solver;

/* Solver properties: the io::Properties keys hom3 reads on this path
 * (solver.hpp:88-95,870; euler/physics.hpp:39-42; euler/quantities.hpp:23-29;
 *  cns/physics.hpp:57-61; cns/quantities.hpp:23-30; heat/physics.hpp:36-39). */
typedef struct {
  int nd;               /* 2 or 3 */
  int physics;          /* H3C_EULER / H3C_CNS / H3C_HEAT / H3C_ADVECTION */
  int flux;             /* H3C_FLUX_* */
  int time_integration; /* H3C_EULER_FORWARD / H3C_RUNGE_KUTTA_2 / H3C_SSPRK3 */
  int precision;        /* H3C_FP64 / H3C_MIXED */
  double time_end;      /* "timeEnd" */
  double cfl;           /* "CFL" */
  double cfl_viscous;   /* "CFL_viscous" */
  double gamma;         /* "gamma" */
  double Rspecific;     /* "Rspecific" [J/(kg K)] */
  double T0;            /* "T0" [K] */
  double rho0;          /* "rho0" [kg/m^3] */
  double Minfty;        /* "Minfty" */
  double ReInfty;       /* "ReInfty" */
  double Pr0;           /* "Pr0" */
  double Sutherland0;   /* "Sutherland0" [K] */
  double diffusivity;   /* "diffusivity" [m^2/s] (heat; does not enter the step) */
  double T_ref;         /* "T_ref" [K] (heat; does not enter the step) */
  int reconstruction;   /* H3C_RECON_NONE (hom3) / H3C_RECON_MUSCL (EXTENSION) */
  double limiter_k;     /* Venkatakrishnan constant K of H3C_RECON_MUSCL */
} h3c_desc;

typedef struct {
  int kind;     /* H3C_BC_* */
  double v[8];  /* parameters, see above */
} h3c_bc;

/* The solver's cell container after Solver::initialize (container.hpp:58-66,
 * solver.hpp:876-977).  Column-major arrays with leading dimension ld >= n_cells. */
typedef struct {
  int64_t n_cells;           /* cells().size(): internal + ghost */
  int64_t first_ghost;       /* firstGC_ */
  int64_t ld;                /* leading dimension of neighbors / x_center */
  const int64_t* neighbors;  /* [2nd][ld]; no neighbour: any value outside [0, n_cells) */
  const double* x_center;    /* [nd][ld] cell centres */
  const double* length;      /* [n_cells] cell lengths */
  const int32_t* bc_idx;     /* [n_cells] bc index of ghosts; internal cells: any value < 0 or >= n_bcs */
  int n_bcs;                 /* number of appended boundary conditions, <= 64 */
  const h3c_bc* bcs;         /* [n_bcs] in append_bc order (solver.hpp:159-169) */
  /* EXTENSION (not in hom3, whose solver links same-level neighbours only,
   * solver.hpp:899-908): coarse/fine faces of 2:1 balanced trees.  A
   * neighbour entry v <= -2 names sub-face group k = -v - 2 whose 2^(nd-1)
   * finer cells are subface_cells[j * n_subfaces + k] (j in increasing child
   * position); a coarser neighbour is stored as a plain cell index.  Face
   * fluxes through a group are area-weighted by 2^-(nd-1).  Zero / NULL for
   * hom3 grids. */
  int64_t n_subfaces;
  const int64_t* subface_cells;
} h3c_grid;

/* ---- lifecycle: Solver(SolverIdx, io::Properties), solver.hpp:88-95 ---- */
int h3c_create(const h3c_desc* desc, h3c_solver* out);
int h3c_destroy(h3c_solver s);
/* Copies the message of the last error on this solver (or a global one when
 * s is NULL) into buf and returns its full length. */
int h3c_last_error(h3c_solver s, char* buf, size_t n);

/* ---- batches (no hom3 counterpart: hom3 steps one solver at a time) ----
 * h3c_set_grids: n independent grids (instances) of one solver description
 * advanced together: every stage is one launch over all instances' cells, each
 * instance keeps its own dt / time / step.  The caller numbering is the
 * concatenation of the instances' cells (instance k's cell c is caller cell
 * sum_{j<k} n_cells_j + c) for h3c_set_state / h3c_get_state / h3c_device_order.
 * Euler and heat only; no coupling or periodic conditions.  h3c_dt / h3c_time /
 * h3c_step / h3c_min_dt / h3c_force_dt refer to instance 0. */
int h3c_set_grids(h3c_solver s, int n, const h3c_grid* grids);
/* per-instance dt, time and step (arrays of n; any may be NULL) */
int h3c_instances(h3c_solver s, double* dt, double* time, int64_t* step);
/* Times nsteps steps for each launch configuration that applies to the
 * solver, from the same saved state, restores the state and keeps the
 * fastest (sets H3C_OPT_TILE_KERNEL, H3C_OPT_EULER_KERNEL and
 * H3C_OPT_PERSISTENT_BLOCKS); returns its index and its time per step (ms).
 * Index: 0-4 the per-lane tile kernel (CNS: the CNS tile kernel) with its
 * default grid or 1-4 persistent blocks per SM; 5 the generic per-cell
 * kernels; 6 the per-cell AUSM kernel; 7-9 the halo-staged tile kernel with
 * 1-3 persistent blocks per SM; 10 the warp-tiled kernel. */
int h3c_autotune(h3c_solver s, int nsteps, int* choice, double* ms_per_step);

/* ---- data: the tables create_local_cells/create_ghost_cells build
 * (solver.hpp:876-977) and the state columns lhs/rhs (container.hpp:59-60) ---- */
int h3c_set_grid(h3c_solver s, const h3c_grid* grid);
/* which: 0 = lhs, 1 = rhs.  Arrays in host or device memory, caller numbering, [nv][ld]. */
int h3c_set_state(h3c_solver s, int which, const double* q, int64_t ld);
int h3c_get_state(h3c_solver s, int which, double* q, int64_t ld);
/* ---- output: Solver::write_domain (solver.hpp:328-376) ----
 * Applies the conditions to lhs and writes fname + ".vtk" in hom3's legacy
 * binary VTK layout (io/vtk.hpp:156-450): the cells in container order as
 * pixels / voxels, then cell data locallCellIds, gridNodeIds, local_nghbrs_*,
 * ghost_cell, bcIdx, the conservative variables, and the physics output
 * (Euler: a, p, u_*, M, e, T; CNS: also mu and vorticity; advection: u_*).
 * grid: the tables given to h3c_set_grid; node_ids: each cell's grid node
 * (NULL writes -1).  Host only apart from the state download; single grids. */
int h3c_write_vtk(h3c_solver s, const char* fname, const h3c_grid* grid, const int64_t* node_ids);
/* Advection velocity of every cell, ghosts included: the physics' velocity
 * function evaluated at the cell centres (Physics::velocity,
 * advection/physics.hpp:104-106, which hom3 evaluates at x_center on every
 * use).  Host array [nd][ld], caller numbering.  Required before an
 * advection solver steps; the next time step is recomputed from it. */
int h3c_set_velocity(h3c_solver s, const double* u, int64_t ld);
/* Device-resident state in the internal (Morton) numbering: pointer, leading
 * dimension and the internal index of every caller cell (perm[caller] = internal). */
int h3c_state_device(h3c_solver s, int which, double** ptr, int64_t* ld);
int h3c_device_order(h3c_solver s, int64_t* perm);
int h3c_get_stream(h3c_solver s, void** stream);
int h3c_sizes(h3c_solver s, int64_t* n_cells, int64_t* first_ghost, int* nv);

/* ---- stepping: Solver::solve (solver.hpp:140-145), n times.  The step runs
 * on the solver's stream and returns without waiting for it. ---- */
int h3c_solve(h3c_solver s, int64_t nsteps);
/* Solver::initialize's final set_dt (solver.hpp:137, 541-551): computes dt
 * from the current lhs with time = 0, dt = 0. */
int h3c_reset_time(h3c_solver s);
/* Solver::apply_bcs on lhs (0) or rhs (1) (solver.hpp:561-586). */
int h3c_apply_bcs(h3c_solver s, int which);
/* Solver::min_dt (solver.hpp:109, 511-517): synchronous. */
int h3c_min_dt(h3c_solver s, double* dt);
/* Solver::dt() / dt(Num) (solver.hpp:112-115, 522-525). */
int h3c_dt(h3c_solver s, double* dt);
int h3c_force_dt(h3c_solver s, double dt);
int h3c_time(h3c_solver s, double* t);
int h3c_step(h3c_solver s, int64_t* step);
/* Failure detection.  hom3 ends a run when dt leaves [1e-300, 1e300]
 * (solution_diverged, utilities.hpp:74-76, 107-110) and asserts positive
 * density, energy and pressure in every cell (check_variables,
 * euler/physics.hpp:229-239; for heat and advection only a non-finite value
 * counts here, since hom3's own heat and advection tests leave T = 0 and
 * q < 0 in cells).
 * The device records both as status bits of each instance while it steps
 * (no extra synchronisation: the CFL reduction checks every cell it reads);
 * h3c_solve stays asynchronous, and the next call that reads the step
 * scalars -- h3c_dt, h3c_time, h3c_step, h3c_min_dt, h3c_instances --
 * returns H3C_E_NONFINITE (or H3C_E_TIMEOUT for a device wait that ran out)
 * with h3c_last_error saying which, after writing the value it read.  The
 * bits are sticky: h3c_status returns the OR over instances
 * (H3C_STATUS_DT | H3C_STATUS_STATE | H3C_STATUS_TIMEOUT) and clears them;
 * h3c_reset_time clears them too. */
#define H3C_STATUS_DT 1
#define H3C_STATUS_STATE 2
#define H3C_STATUS_TIMEOUT 4
int h3c_status(h3c_solver s, int* flags);

/* ---- stepping by parts (no hom3 counterpart: hom3 has no domain decomposition) ----
 * One grid split over several solvers (subdomains, one per GPU) needs, before
 * every stage, the neighbouring subdomains' cells in its H3C_BC_EXCHANGE
 * ghosts, and one time step for all.  h3c_stages: stages per step (forward
 * Euler 1, RK2 2, SSP-RK3 3).  h3c_solve_stage(s, k), k = 0 .. stages - 1 in
 * order, is part k of one h3c_solve step: part 0 applies the conditions to
 * lhs and sets the step's dt from the minimum cell time step; part k > 0
 * applies the conditions to its input; each part then runs its stage; the
 * last part also advances time and step.  h3c_stage_input(s, k, &p): device
 * pointer (internal numbering, [nv][ld], see h3c_device_order) of part k's
 * input state, into whose exchange ghosts the caller writes before part k.
 * h3c_dtmin_device(s, &p): the device int64 from which part 0 takes the
 * step's dt (the minimum cell time step of lhs as ordered bits: integer
 * order is time-step order); the caller replaces it by the minimum over the
 * subdomains before part 0.  h3c_solve refuses to run between parts. */
int h3c_stages(h3c_solver s, int* n);
int h3c_solve_stage(h3c_solver s, int k);
int h3c_stage_input(h3c_solver s, int k, double** ptr);
int h3c_dtmin_device(h3c_solver s, int64_t** ptr);

/* Fused multiply-add issue rates of the current device (no hom3 counterpart):
 * long register-only FMA chains, timed with CUDA events; FP64 and FP32 FMAs
 * per second (one FMA = two flops).  The roofline of an arithmetic-bound
 * stage kernel is set by the FP64 rate, which the copy and GEMM peaks do not
 * give.  Allocates and frees a few bytes of device memory. */
int h3c_fma_rates(double* fp64_per_s, double* fp32_per_s);

/* ---- instrumentation (no hom3 counterpart: hom3 has no timers) ----
 * h3c_launches: kernels this solver has launched since creation.
 * h3c_profile(s, 1): bracket every subsequent launch with CUDA events on the
 * solver's stream; h3c_profile_read sums the elapsed times per kernel kind
 * (0 boundary conditions, 1 CFL reduction, 2 scalar step bookkeeping,
 * 3 first stage / forward Euler, 4 second RK stage, 5 slopes, 7 adjoint stages) and resets. */
int h3c_launches(h3c_solver s, int64_t* n);
/* Execution options (no hom3 counterpart; results do not depend on them):
 * H3C_OPT_TILE_KERNEL  Euler stages and their adjoint in the shared-memory tile kernels (default 1)
 * H3C_OPT_GRAPHS       replay runs of steps from a captured CUDA graph (default 1)
 * H3C_OPT_HALO_KERNEL  the halo-staged tile kernels (each tile and its halo copied into shared
 *                      memory by bulk copies) may be used: the CNS stage and H3C_OPT_EULER_KERNEL 0
 *                      (default 1; 0: CNS steps in the per-cell kernel, Euler kernel 0 in the per-lane one) */
#define H3C_OPT_TILE_KERNEL 1
#define H3C_OPT_GRAPHS 2
#define H3C_OPT_HALO_KERNEL 3
/* H3C_OPT_PERSISTENT_BLOCKS  blocks of the Euler/AUSM stage launch, each looping over tiles
 *                            (0, the default: one block per tile for the per-lane tile kernel,
 *                            the resident blocks of all SMs for the halo-staged one) */
#define H3C_OPT_PERSISTENT_BLOCKS 4
/* H3C_OPT_CNS_ADJOINT_DUAL  the CNS adjoint's face derivatives by forward-mode dual numbers instead
 *                           of the hand-written reverse sweep (default 0; kept as a cross-check) */
#define H3C_OPT_CNS_ADJOINT_DUAL 5
/* H3C_OPT_HALO_SLOTS  at most this many halo entries per tile in shared memory (a multiple of 32;
 *                     0, the default: as many as let three blocks share an SM); entries beyond
 *                     are read from global memory where a face needs them */
#define H3C_OPT_HALO_SLOTS 6
/* H3C_OPT_EULER_KERNEL  the Euler/AUSM stage kernel (with the tile kernels on): 0 the halo-staged
 *                       tile kernel when its tables exist, 1 (the default) the per-lane tile kernel,
 *                       2 one thread per cell, faces from both sides, 3 one warp per 32 Morton cells
 *                       (each face state once per warp, each face between two of its cells once),
 *                       4 the per-lane tile kernel on 512-cell tiles (8x8x8 Morton bricks, 512-thread
 *                       blocks; 3D single grids, otherwise kernel 1) */
#define H3C_OPT_EULER_KERNEL 7
int h3c_set_option(h3c_solver s, int option, int value);
/* The Euler stage launch in use (no hom3 counterpart): info[0] kernel (0 per
 * cell, 1 per-lane tile, 2 halo-staged tile, 3 the per-cell AUSM kernel, 4 the warp-tiled AUSM
 * kernel, 5 the per-lane tile kernel on 512-cell tiles), [1] halo slots per tile, [2]
 * largest tile halo, [3] mean tile halo x 1000, [4] resident blocks per SM
 * of the halo-staged kernel, [5] blocks launched, [6] its dynamic shared
 * memory in bytes, [7] 256-cell tiles; the first n entries are written. */
int h3c_kernel_info(h3c_solver s, int64_t* info, int n);
/* Self-test of the device reciprocal / reciprocal square root the kernels
 * use in place of division (n <= 2^24 positive inputs, host arrays). */
int h3c_selftest_nr(const double* x, int64_t n, double* rcp, double* rsqrt);
int h3c_profile(h3c_solver s, int enable);
int h3c_profile_read(h3c_solver s, double* ms, int64_t* count, int nkinds);

/* ---- allocation-free time step (no counterpart in hom3) ----
 * For callers that cannot allocate device memory -- code running inside a
 * framework that owns all device memory through its own pool, or a step
 * controller that must not call cudaMalloc because it synchronises the device
 * and would serialise the caller's streams.  Computes the same minimum cell
 * time step as h3c_min_dt (hom3's compute_dt) from caller-owned device
 * buffers: q = interior-cell state [nv][ld], length = their cell lengths,
 * dt_out = one device double; asynchronous on `stream`.  Euler, CNS and heat
 * (advection, whose time step needs the velocity field, returns
 * H3C_E_INVALID).  Allocates nothing: its scratch is a fixed 128 KiB array
 * inside the library (held on every GPU that loads it until exit), so
 * n_cells <= 4,194,304; larger sizes return H3C_E_INVALID.  Errors set the
 * text of h3c_last_error(NULL, ...).  The first call on a device looks up
 * the array's address (make that first call before any stream capture); with
 * CUDA's default lazy module loading it also loads the library's device code,
 * which reserves device memory, so a caller whose pool takes all device
 * memory makes the first call at its own initialisation, before the pool
 * does (or sets CUDA_MODULE_LOADING=EAGER).  Calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller. */
int h3c_min_dt_noalloc(const h3c_desc* desc, const double* q, int64_t ld, int64_t n_cells,
                       const double* length, double* dt_out, void* stream);

/* ---- discrete adjoint (no hom3 counterpart) ----
 * h3c_solve_dt: nsteps steps with the given time steps (host array) instead
 * of the CFL time step -- the forward map the adjoint differentiates.
 * h3c_adjoint: runs nsteps steps from the current state (leaving the solver
 * at step N, like h3c_solve) with a checkpoint every `every` steps (0: the
 * library picks -- no recomputation when that fits in half of the free device
 * memory), then returns dJ/dq0 for J = <dJ_dqN, q_N> with the time steps
 * frozen at the forward values (returned in dts, may be NULL).  dJ_dqN,
 * dJ_dq0 and dts are [nv][n_cells] / [nsteps] arrays in caller numbering, in
 * host or device memory; ghost entries of dJ_dqN are ignored, of dJ_dq0 zero.
 * The last segment's stage states are kept from the forward run; the other
 * segments are recomputed from their checkpoints.  The workspace stays
 * allocated for the next call.  Euler with the AUSM (and MUSCL) or LLF flux,
 * CNS, and heat; Neumann / Dirichlet / periodic conditions (CNS also its wall,
 * inflow and outflow conditions). */
int h3c_solve_dt(h3c_solver s, int64_t nsteps, const double* dts);
int h3c_adjoint(h3c_solver s, int64_t nsteps, int64_t every, const double* dJ_dqN, double* dJ_dq0, double* dts);

/* Discrete adjoint of the coupled conjugate-heat loop (no hom3 counterpart):
 * nsteps of h3c_cht_solve's loop (forward Euler in both solvers) from the
 * current states, checkpoints every `every` steps (0: 100), then dJ/dq0 of
 * the fluid and dJ/dT0 of the solid for J = <dJ_dqN, q_N> + <dJ_dTN, T_N>,
 * the coupled time steps frozen at the forward values (dts, may be NULL:
 * [2][nsteps], fluid then solid).  Arrays in each solver's caller numbering,
 * host or device memory.  The interface conditions are differentiated in both
 * directions (the fluid wall reads the solid's temperature, the solid ghost
 * the fluid's). */
int h3c_cht_adjoint(h3c_solver cns, h3c_solver heat, double Tr0, int64_t nsteps, int64_t every,
                    const double* dJ_dqN, const double* dJ_dTN, double* dJ_dq0, double* dJ_dT0, double* dts);

/* ---- coupling: coupling.hpp:24-73 ----
 * partner_cells[g - first_ghost] = the partner solver's cell (caller
 * numbering of the partner) that local_bndry_ids (coupling.hpp:24-39) finds
 * for ghost g, or any negative value for ghosts of non-coupled conditions.
 * Both solvers then share the partner's stream. */
int h3c_set_partner(h3c_solver s, h3c_solver partner, const int64_t* partner_cells);
/* coupling::apply(Tr0, cns, heat), coupling.hpp:52-63 */
int h3c_couple_cht(h3c_solver cns, h3c_solver heat, double Tr0);
/* nsteps of the coupled loop of coupled_cns_heat_test.cpp:235-248 --
 * coupling::apply(Tr0, cns, heat), cns.solve(), heat.solve() per step -- on
 * the solvers' shared stream; runs of steps replay one captured CUDA graph
 * (the same kernels as the three calls per step). */
int h3c_cht_solve(h3c_solver cns, h3c_solver heat, double Tr0, int64_t nsteps);
/* coupling::apply(s1, s2), coupling.hpp:66-73 */
int h3c_couple_equal(h3c_solver a, h3c_solver b);
/* EXTENSION (not in hom3): partner cells (caller numbering, same solver) for
 * the ghosts of H3C_BC_PERIODIC conditions. */
int h3c_set_periodic(h3c_solver s, const int64_t* partner_cells);

/* ---- grid builder (the device grid layer): builds hom3-equivalent tables
 * for the MinLevel generator (grid/generation.hpp:39-60) and cube /
 * box boundaries (grid/helpers.hpp:112-160, geometry/implicit.hpp:39-205),
 * with leaves in Morton order.  EXTENSION (not in hom3): refinement of the
 * cells that intersect spheres, 2:1 balanced, with coarse/fine faces. ---- */
#define H3C_SDF_NONE 0
#define H3C_SDF_EDGE 1   /* p = point[3], normal[3] */
#define H3C_SDF_SQUARE 2 /* p = center[3], lengths[3] */
#define H3C_SDF_SPHERE 3 /* p = center[3], radius */
typedef struct {
  int kind;
  int inverted;
  double p[6];
} h3c_sdf;

typedef struct {
  int nd;
  double xmin[3], xmax[3]; /* root cell (grid/grid.hpp:106-139) */
  int min_level;           /* MinLevel "level" */
  int n_refine;            /* EXTENSION: spheres refined to refine_level */
  double refine_center[4][3];
  double refine_radius[4];
  int refine_level[4];
  int domain_kind;         /* 0 all leaves, 1 leaves with sdf > 0, 2 with sdf < 0 */
  h3c_sdf domain;          /* "initialDomain" predicate */
  int n_bcs;               /* boundaries in append order */
  h3c_sdf bc_geom[16];
} h3c_grid_desc;

typedef struct h3c_built_grid_s* h3c_built_grid;
int h3c_grid_build(const h3c_grid_desc* desc, h3c_built_grid* out);
/* The same tables built on the GPU (no hom3 counterpart): refinement, 2:1
 * balance, Morton ranking, neighbour / sub-face search and ghost creation as
 * data-parallel kernels and scans on the current device, then copied to the
 * host; bit-identical to h3c_grid_build's.  Free with h3c_grid_free. */
int h3c_grid_build_device(const h3c_grid_desc* desc, h3c_built_grid* out);
/* Table views valid until h3c_grid_free; the layout is that of h3c_grid. */
int h3c_grid_view(h3c_built_grid g, h3c_grid* view);
/* cube faces of the root cell in hom3's order left,right,bottom,top,front,back;
 * returns their number (2nd) or a negative error code */
int h3c_cube_boundaries(const h3c_grid_desc* desc, h3c_sdf* out);
int h3c_grid_free(h3c_built_grid g);

#ifdef __cplusplus
}
#endif
#endif /* H3C_H_ */
