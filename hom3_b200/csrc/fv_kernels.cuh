// fv_kernels.cuh -- sm_100a kernels of the finite-volume step.
//
// One thread per cell.  Cells are stored in Morton order (interior cells
// [0, n_int), ghosts after them), state as SoA FP64 columns q[v * ld + c].
// The arithmetic follows hom3's physics plugins operation by operation
// (citations per function, paths relative to hom3's src/), so the FP64 path
// reproduces hom3's per-step results to rounding (FMA contraction is the only
// difference).  R is the arithmetic type of the face flux: double for the
// drop-in path, float for the mixed path (state, residual accumulation, update
// and dt stay FP64).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace h3c {

constexpr int kBlock = 256;
constexpr int kMaxLevels = 32;
constexpr int kMaxBcs = 64;

enum Physics { EULER = 0, CNS = 1, HEAT = 2, ADVECTION = 3 };
enum Flux { AUSM = 0, LLF = 1, UPWIND = 2 };
// variables per cell: Euler/CNS (rho u_d, rho, rho E); heat T; advection q
template <int ND, int PHYS> __host__ __device__ constexpr int nvars() {
  return (PHYS == HEAT || PHYS == ADVECTION) ? 1 : ND + 2;
}
enum BcKind {
  BC_EULER_NEUMANN = 0, BC_EULER_DIRICHLET = 1, BC_EULER_VORTEX = 2, BC_CNS_INFLOW = 3,
  BC_CNS_OUTFLOW = 4, BC_CNS_ADIABATIC_NOSLIP = 5, BC_CNS_ADIABATIC_SLIP = 6,
  BC_CNS_ISOTHERMAL_NOSLIP = 7, BC_HEAT_DIRICHLET = 8, BC_HEAT_NEUMANN = 9,
  BC_CPL_EULER_EULER = 10, BC_CPL_CNS_HEAT = 11, BC_CPL_HEAT_CNS = 12, BC_CPL_HEAT_HEAT = 13,
  BC_PERIODIC = 14, BC_ADV_DIRICHLET = 15, BC_ADV_NEUMANN = 16, BC_ADV_CHARACTERISTIC = 17, BC_EXCHANGE = 18
};

// Device-resident step scalars (solver.hpp:406-416) and reduction slots.
struct Scalars {
  double dt, time, tEnd, forced_dt;
  long long step, forced_step;
  long long dtmin_ord;  // min of cell dt for the next set_dt (ordered bits)
  long long mindt_ord;  // min of cell dt for h3c_min_dt
  int status;           // kStatus* bits, sticky until h3c_status reads them
  int pad;
};

// Scalars::status bits
constexpr int kStatusDt = 1;      // set_dt produced dt outside [1e-300, 1e300] (utilities.hpp:74-76)
constexpr int kStatusState = 2;   // a cell violates check_variables (euler/physics.hpp:229-239)
constexpr int kStatusTimeout = 4; // a bounded device wait ran out

// Physical constants of one solver (euler/quantities.hpp, cns/quantities.hpp)
struct PhysConst {
  double gamma, gm1, cfl, cflv, Re0, Pr0, sOverTref, sOverTrefP1;
};

struct BcParam {
  int kind;
  int wall;          // tangential velocity slopes flip sign (cns walls)
  double v[8];
  double partner_gamma;
  int partner_physics;
  int partner_nd;
};

// The partner state a coupling / periodic condition reads at launch time.
struct PartnerView {
  const double* q;  // partner lhs (coupling); unused for periodic (own target state)
  long long ld;
};

struct Geometry {
  const int* __restrict__ nbr;            // [2nd][ld] (>=0 cell, -1 none, <=-2 sub-face group)
  const unsigned char* __restrict__ lvl;  // [ld] index into len[]
  const int* __restrict__ sub;            // [2^(nd-1)][nsub]
  long long nsub;
  long long n_int, n_tot, ld;
  double len[kMaxLevels];
  // Batches of independent grids: interior cells of instance k occupy
  // [start_k, inst_end[k]) with start_k a multiple of kBlock, so every
  // kBlock-cell tile belongs to one instance (blk_inst[tile]); the cells
  // between inst_end[k] and the next start are padding.  nullptr: one grid.
  const int* __restrict__ blk_inst;
  const long long* __restrict__ inst_end;
  long long ntiles;
  // advection velocity u(x_center) of every cell, ghosts included: [nd][ld] (nullptr otherwise)
  const double* __restrict__ vel;
};

__device__ __forceinline__ int tile_instance(const Geometry& g, long long tile) {
  return g.blk_inst ? g.blk_inst[tile] : 0;
}
__device__ __forceinline__ long long instance_end(const Geometry& g, int inst) {
  return g.blk_inst ? g.inst_end[inst] : g.n_int;
}
// the per-instance copy of a Scalars field (instances are consecutive Scalars)
template <class T> __device__ __forceinline__ T* per_instance(T* slot0, int inst) {
  return reinterpret_cast<T*>(reinterpret_cast<char*>(slot0) + (size_t)inst * sizeof(Scalars));
}

struct GhostTables {
  const int* __restrict__ bndry;          // [ng] boundary cell of each ghost
  const unsigned char* __restrict__ pos;  // [ng] position of the ghost w.r.t. its boundary cell
  const unsigned char* __restrict__ bc_apply;  // [ng] bc applied by apply_bcs (255: none)
  const unsigned char* __restrict__ bc_own;    // [ng] the ghost's own bc index
  const double* __restrict__ dx;          // [ng] |x_b - x_g| (cell_dx, solver.hpp:590-592)
  const int* __restrict__ partner;        // [ng] partner cell (internal numbering) or -1
  const double* __restrict__ xc;          // [nd][ld] cell centres (vortex bc)
  const int* __restrict__ ginst;          // [ng] instance of each ghost (nullptr: one grid)
  long long ng;
  const BcParam* bcs;                     // [n_bcs] device array
};

// ---------------------------------------------------------------------------
// ordered-bits min for doubles (NaN never wins, as std::min(dt, NaN) in hom3)
// ---------------------------------------------------------------------------
__device__ __forceinline__ long long dbl_to_ord(double x) {
  long long i = __double_as_longlong(x);
  return i >= 0 ? i : (i ^ 0x7fffffffffffffffLL);
}
__host__ __device__ inline double ord_to_dbl(long long o) {
  long long i = o >= 0 ? o : (o ^ 0x7fffffffffffffffLL);
#ifdef __CUDA_ARCH__
  return __longlong_as_double(i);
#else
  double d;
  memcpy(&d, &i, 8);
  return d;
#endif
}
constexpr long long kOrdMax = 0x7fefffffffffffffLL;  // bits of DBL_MAX

// Minimum of v over a block of at most TB threads (TB / 32 <= 32 warps),
// folded into *dst by one atomicMin (NaN never wins).  Every thread calls it.
template <int TB>
__device__ __forceinline__ void block_min_atomic_tb(long long v, long long* dst) {
  __shared__ long long red[TB / 32];
  for (int o = 16; o > 0; o >>= 1) {
    long long w = __shfl_down_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : kOrdMax;
    for (int o = 16; o > 0; o >>= 1) {
      long long w = __shfl_down_sync(0xffffffffu, v, o);
      v = w < v ? w : v;
    }
    if (lane == 0 && v < kOrdMax) atomicMin(dst, v);
  }
}
__device__ __forceinline__ void block_min_atomic(long long v, long long* dst) { block_min_atomic_tb<kBlock>(v, dst); }

// The same minimum without a block barrier, for kernels that have none: each
// warp folds its minimum into a shared slot; the last warp of the block to
// arrive (a shared counter) makes the one global atomicMin.  slot and cnt
// must hold kOrdMax and 0 before the first warp arrives (set at the kernel's
// start, before a barrier).  Every warp of the block must call it once.
__device__ __forceinline__ void block_min_atomic_nobar(long long v, long long* dst, long long* slot, unsigned* cnt) {
  for (int o = 16; o > 0; o >>= 1) {
    long long w = __shfl_down_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(slot, v);
    __threadfence_block();
    if (atomicAdd(cnt, 1u) == (blockDim.x >> 5) - 1) {
      __threadfence_block();
      const long long m = *(volatile long long*)slot;
      if (m < kOrdMax) atomicMin(dst, m);
    }
  }
}

// Records in the instance's status that some cell of this warp failed the
// state check (one atomic per warp that saw one; every lane must call).
__device__ __forceinline__ void flag_bad_state(bool bad, const Scalars* sc, int inst) {
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0)
    atomicOr(const_cast<int*>(&sc[inst].status), kStatusState);
}

// ---------------------------------------------------------------------------
// Reciprocal and reciprocal square root without division: hardware estimate
// refined by two Newton-Raphson iterations (y <- y + y(1 - xy) for 1/x,
// y <- y + y(1/2 - (x/2) y^2) for 1/sqrt(x)), each of which doubles the
// correct bits of the estimate.  Branch-free; valid for positive normal
// inputs, which is all a physical state produces (density, pressure, sound
// speed).  Tested against IEEE 1/x and 1/sqrt(x) within 2 ulp.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double nr_rcp(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}
__device__ __forceinline__ double nr_rsqrt(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double h = 0.5 * x;
  double r = fma(-h * y, y, 0.5);
  y = fma(y, r, y);
  r = fma(-h * y, y, 0.5);
  return fma(y, r, y);
}
__device__ __forceinline__ float nr_rcp(float x) { return __frcp_rn(x); }
__device__ __forceinline__ float nr_rsqrt(float x) { return rsqrtf(x); }

// Moves cell c's row of a [nv][ld] state towards L2 (a hint: no register is
// taken and nothing waits on it).  The in-place stages read their start
// state only at the update, after the face loops; issued at the start, the
// prefetch overlaps that read's DRAM latency with the face work.
template <int NV>
__device__ __forceinline__ void prefetch_row_l2(const double* q, long long ld, long long c) {
#pragma unroll
  for (int v = 0; v < NV; ++v) asm volatile("prefetch.global.L2 [%0];" ::"l"(q + v * ld + c));
}

// ---------------------------------------------------------------------------
// primitive variables: euler/physics.hpp:83-125.  u = rho u / rho,
// p = (gamma - 1)(rho E - rho |u|^2 / 2), a = sqrt(gamma p / rho), and the
// directional Mach numbers M_d = u_d / a the AUSM flux needs
// (euler/physics.hpp:279-280), computed once per cell.
// ---------------------------------------------------------------------------
template <class R, int ND> struct Prim {
  R q[ND + 2];
  R u[ND];
  R M[ND];
  R p, a;
};

template <class R, int ND>
__device__ __forceinline__ void make_prim(Prim<R, ND>& P, R gamma, R gm1) {
  const R rho = P.q[ND];
  const R rinv = nr_rcp(rho);
  R um2 = R(0);
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    P.u[d] = P.q[d] * rinv;
    um2 = d == 0 ? P.u[d] * P.u[d] : um2 + P.u[d] * P.u[d];
  }
  P.p = gm1 * (P.q[ND + 1] - R(0.5) * rho * um2);
  const R a2 = gamma * P.p * rinv;
  const R ainv = nr_rsqrt(a2);
  P.a = a2 * ainv;
#pragma unroll
  for (int d = 0; d < ND; ++d) P.M[d] = P.u[d] * ainv;
}

template <class R, int ND>
__device__ __forceinline__ void load_prim(Prim<R, ND>& P, const double* __restrict__ q, long long ld,
                                          int c, R gamma, R gm1) {
#pragma unroll
  for (int v = 0; v < ND + 2; ++v) P.q[v] = (R)__ldg(q + v * ld + c);
  make_prim<R, ND>(P, gamma, gm1);
}

// m_int_, p_int_: euler/physics.hpp:297-310.  For |M| > 1 the split values
// are exactly M or 0 (Mach) and 1 or 0 (pressure): 0.5 (M + s|M|) is M or 0
// and that over M is 1 or 0 without rounding, so no division is needed.
template <class R> __device__ __forceinline__ R m_int(R s, R M) {
  const R sup = (s * M > R(0)) ? M : R(0);
  return fabs(M) > R(1) ? sup : (s * R(0.25)) * ((M + s) * (M + s));
}
template <class R> __device__ __forceinline__ R p_int(R s, R M) {
  const R sup = (s * M > R(0)) ? R(1) : R(0);
  return fabs(M) > R(1) ? sup : (R(0.25) * ((M + s) * (M + s))) * (R(2) - s * M);
}

// AUSM (Liou-Steffen): euler/physics.hpp:276-293, theta_ :315-325
template <class R, int ND>
__device__ __forceinline__ void ausm(const Prim<R, ND>& L, const Prim<R, ND>& Rt, int d, R* f) {
  const R ML = L.M[d];
  const R MR = Rt.M[d];
  const R mi = m_int<R>(R(1), ML) + m_int<R>(R(-1), MR);
  const R pi = p_int<R>(R(1), ML) * L.p + p_int<R>(R(-1), MR) * Rt.p;
  const bool left = mi >= R(0);
  const R a = left ? L.a : Rt.a;
#pragma unroll
  for (int v = 0; v < ND + 1; ++v) f[v] = ((left ? L.q[v] : Rt.q[v]) * a) * mi;
  f[ND + 1] = (((left ? L.q[ND + 1] + L.p : Rt.q[ND + 1] + Rt.p)) * a) * mi;
#pragma unroll
  for (int v = 0; v < ND; ++v)
    if (v == d) f[v] = f[v] + pi;
}

// Euler flux: euler/physics.hpp:98-113; LLF: :262-267
template <class R, int ND>
__device__ __forceinline__ void llf(const Prim<R, ND>& L, const Prim<R, ND>& Rt, int d, R dx_dt, R* f) {
  R fl[ND + 2], fr[ND + 2];
  fl[ND] = L.q[d];
  fr[ND] = Rt.q[d];
#pragma unroll
  for (int i = 0; i < ND; ++i) {
    fl[i] = L.q[i] * L.u[d];
    fr[i] = Rt.q[i] * Rt.u[d];
  }
#pragma unroll
  for (int i = 0; i < ND; ++i)
    if (i == d) { fl[i] = fl[i] + L.p; fr[i] = fr[i] + Rt.p; }
  fl[ND + 1] = L.u[d] * (L.q[ND + 1] + L.p);
  fr[ND + 1] = Rt.u[d] * (Rt.q[ND + 1] + Rt.p);
#pragma unroll
  for (int v = 0; v < ND + 2; ++v) f[v] = R(0.5) * ((fl[v] + fr[v]) + dx_dt * (L.q[v] - Rt.q[v]));
}

// Sutherland's law: cns/quantities.hpp:113-115
template <class R> __device__ __forceinline__ R sutherland(R T, R sOverTref, R sOverTrefP1) {
  return (T * sqrt(T)) * sOverTrefP1 / (T + sOverTref);
}

// Three-point viscous flux: cns/physics.hpp:305-338 with the surface helpers
// :221-293 and surface_slope (solver.hpp:656-678).  sl/sr: cell slopes
// [sd][v] of the left / right cell.  hom3 divides by rho_s, rho_s^2, len_r,
// (T + S) and gm1 Pr0 rho_s face by face; here each divisor's reciprocal is
// taken once (nr_rcp: hardware estimate + Newton steps, within 2 ulp) and
// multiplied in, and T^1.5 is T * T * rsqrt(T) -- an arithmetic difference
// of a few ulp per flux, far inside the parity tolerance.
template <class R, int ND>
__device__ __forceinline__ void viscous(const Prim<R, ND>& L, const Prim<R, ND>& Rt, const R* sl,
                                        const R* sr, int d, R len_r, const PhysConst& pc, R* f) {
  constexpr int NV = ND + 2;
  const R gamma = (R)pc.gamma, gm1 = (R)pc.gm1;
  const R rho_s = R(0.5) * (L.q[ND] + Rt.q[ND]);
  const R rinv = nr_rcp(rho_s);
  R rho_u_s[ND], u_s[ND];
  R umag2 = R(0);
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    rho_u_s[k] = R(0.5) * (L.q[k] + Rt.q[k]);
    u_s[k] = rho_u_s[k] * rinv;
    umag2 = k == 0 ? u_s[k] * u_s[k] : umag2 + u_s[k] * u_s[k];
  }
  const R rho_E_s = R(0.5) * (L.q[ND + 1] + Rt.q[ND + 1]);
  const R p_s = gm1 * (rho_E_s - R(0.5) * rho_s * umag2);
  const R ilen = nr_rcp(len_r);
  auto gs = [&](int v, int sd) -> R {
    return sd == d ? (Rt.q[v] - L.q[v]) * ilen : R(0.5) * (sr[sd * NV + v] + sl[sd * NV + v]);
  };
  const R rinv2 = rinv * rinv;
  R gu[ND][ND];  // gu[c][sd] = d u_c / d x_sd at the surface
#pragma unroll
  for (int c = 0; c < ND; ++c)
#pragma unroll
    for (int sd = 0; sd < ND; ++sd) gu[c][sd] = (gs(c, sd) * rho_s - gs(ND, sd) * rho_u_s[c]) * rinv2;
  const R p_avg = R(0.5) * (L.p + Rt.p);
  // Sutherland's law (cns/quantities.hpp:113-115): T^1.5 (1 + S) / (T + S)
  const R T = gamma * p_avg * rinv;
  const R mu_s = (T * (T * nr_rsqrt(T))) * (R)pc.sOverTrefP1 * nr_rcp(T + (R)pc.sOverTref);
  R grad_rho_umag2 = gs(ND, d) * umag2;
#pragma unroll
  for (int k = 0; k < ND; ++k) grad_rho_umag2 = grad_rho_umag2 + rho_s * R(2) * u_s[k] * gu[k][d];
  const R gradP = gm1 * (gs(ND + 1, d) - R(0.5) * grad_rho_umag2);
  const R gradRho = gs(ND, d);
  const R cq = gamma / (gm1 * (R)pc.Pr0);  // a kernel constant: hoisted out of the face loops
  const R qf = -mu_s * cq * rinv * (gradP - p_s * rinv * gradRho);
  // nabla_u(i, j) = gu[j][i]; trace = sum gu[i][i]
  R tr = gu[0][0];
#pragma unroll
  for (int i = 1; i < ND; ++i) tr = tr + gu[i][i];
  const R div_u = tr * R(2.0 / 3.0);
  const R invRe = R(1) / (R)pc.Re0;  // a kernel constant
  R Eacc = R(0);
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    // nabla_u(k, d) + nabla_u(d, k) = gu[d][k] + gu[k][d]
    R t = gu[d][k] + gu[k][d];
    if (k == d) t = t - div_u;
    const R tkd = -mu_s * t;
    f[k] = invRe * tkd;
    Eacc = k == 0 ? u_s[k] * tkd : Eacc + u_s[k] * tkd;
  }
  f[ND] = R(0);
  f[ND + 1] = invRe * (Eacc + qf);
}

// ---------------------------------------------------------------------------
// per-cell time step: euler/physics.hpp:182-196, cns/physics.hpp:167-187,
// heat/physics.hpp:82-85, advection/physics.hpp:78-87 (u: the cell's velocity)
// bad (optional): the cell fails hom3's check_variables -- density, energy
// and pressure positive (euler/physics.hpp:229-239, shared by CNS).  For heat
// and advection only a non-finite value counts: hom3's own heat test starts
// from T = 0 (heat/physics.hpp:89-95 asks T > 0, in debug builds only) and
// its upwind advection test makes q negative (the flux is reproduced as
// written).  NaN fails every comparison, so it is bad too.
// ---------------------------------------------------------------------------
template <int ND, int PHYS>
__device__ __forceinline__ double cell_dt(const double* q, double h, const PhysConst& pc,
                                          const double* u = nullptr, bool* bad = nullptr) {
  if (PHYS == HEAT) {
    if (bad) *bad = !isfinite(q[0]);
    return pc.cfl * 0.5 * (h * h);
  }
  if (PHYS == ADVECTION) {
    if (bad) *bad = !isfinite(q[0]);
    double u_max = -1.7976931348623157e308;
#pragma unroll
    for (int d = 0; d < ND; ++d) u_max = fmax(u_max, fabs(u[d]));
    return pc.cfl * h / u_max;
  }
  Prim<double, ND> P;
#pragma unroll
  for (int v = 0; v < ND + 2; ++v) P.q[v] = q[v];
  make_prim<double, ND>(P, pc.gamma, pc.gm1);
  if (bad) *bad = !(P.q[ND] > 0.0 && P.q[ND + 1] > 0.0 && P.p > 0.0);
  double S = -1.7976931348623157e308;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const double cand = fabs(P.u[d]) + P.a;
    S = (S < cand) ? cand : S;
  }
  // cfl h / S with S's reciprocal by nr_rcp (within 2 ulp of the division)
  const double dt_inv = PHYS == CNS ? pc.cfl * h / S : (pc.cfl * h) * nr_rcp(S);
  if (PHYS != CNS) return dt_inv;
  const double T = pc.gamma * P.p / P.q[ND];
  const double S_coeff = sutherland<double>(T, pc.sOverTref, pc.sOverTrefP1) / (P.q[ND] * h);
  const double a1 = S_coeff / pc.Re0, a2 = S_coeff / (pc.Re0 * pc.Pr0 * pc.gm1);
  const double S_visc = (a1 < a2) ? a2 : a1;
  const double dt_v = pc.cflv * h / (2 * S_visc);
  return (dt_v < dt_inv) ? dt_v : dt_inv;
}

template <int ND, int PHYS>
__global__ void __launch_bounds__(kBlock) k_cfl(const double* __restrict__ q, Geometry g, PhysConst pc,
                                                long long* dst, const Scalars* sc) {
  constexpr int NV = nvars<ND, PHYS>();
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int inst = tile_instance(g, blockIdx.x);
  long long o = kOrdMax;
  bool bad = false;
  if (c < instance_end(g, inst)) {
    double qc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) qc[v] = __ldg(q + v * g.ld + c);
    double uc[ND];
    if (PHYS == ADVECTION) {
#pragma unroll
      for (int d = 0; d < ND; ++d) uc[d] = __ldg(g.vel + d * g.ld + c);
    }
    const double dt = cell_dt<ND, PHYS>(qc, g.len[g.lvl[c]], pc, uc, &bad);
    if (!isnan(dt)) o = dbl_to_ord(dt);
  }
  flag_bad_state(bad, sc, inst);
  block_min_atomic(o, per_instance(dst, inst));
}

#ifndef H3C_DEVICE_FUNCTIONS_ONLY  // non-template kernels: defined in one translation unit
// set_dt: solver.hpp:541-551 (dtmin_ord holds compute_dt of the current lhs)
__global__ void k_set_dt(Scalars* s0, int reset_after, int n_inst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  Scalars* s = s0 + i;
  double dt;
  if (s->time + s->dt < s->tEnd) {
    dt = (s->step == s->forced_step) ? s->forced_dt : ord_to_dbl(s->dtmin_ord);
  } else {
    dt = s->tEnd - s->time;
  }
  s->dt = dt;
  if (!(dt >= 1e-300 && dt <= 1e300)) s->status |= kStatusDt;  // utilities.hpp:74-76
  if (reset_after) s->dtmin_ord = kOrdMax;
}
// advance: solver.hpp:502-505
__global__ void k_advance(Scalars* s0, int n_inst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_inst) return;
  Scalars* s = s0 + i;
  s->time += s->dt;
  s->step += 1;
}
__global__ void k_reset_slot(long long* slot, int n_inst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_inst) *per_instance(slot, i) = kOrdMax;
}
#endif  // H3C_DEVICE_FUNCTIONS_ONLY

// ---------------------------------------------------------------------------
// isentropic vortex: euler/initial_conditions.hpp:14-39 (2D, hom3's fixed
// parameters: beta 5, gamma 1.4, centre (-5,-5), u = v = 1)
// ---------------------------------------------------------------------------
__device__ inline void isentropic_vortex(double x0, double x1, double t, double* out) {
  const double PI = 3.141592653589793238462643383279502884;
  const double beta = 5, gamma = 1.4, c0 = -5.0, c1 = -5.0, uu = 1, vv = 1;
  const double x_t = x0 - uu * t, y_t = x1 - vv * t;
  const double r = sqrt((x_t - c0) * (x_t - c0) + (y_t - c1) * (y_t - c1));
  const double eT1mr2 = exp(1 - r * r);
  const double eT21mr2 = exp(2 * (1 - r * r));
  const double pu = uu - beta * eT1mr2 * (y_t - c1) / (2 * PI);
  const double pv = vv + beta * eT1mr2 * (x_t - c0) / (2 * PI);
  const double rho = pow((1 - ((gamma - 1) * (beta * beta) * eT21mr2) / (16 * gamma * (PI * PI))), 1 / (gamma - 1));
  const double p = pow(rho, gamma);
  out[0] = rho * pu;
  out[1] = rho * pv;
  out[2] = rho;
  out[3] = p / (1.4 - 1.0) + 0.5 * rho * (pu * pu + pv * pv);
}

// ---------------------------------------------------------------------------
// boundary conditions: one thread per ghost.  apply_bcs (solver.hpp:561-586)
// with the conditions of euler/, cns/, heat/ boundary_conditions.hpp and the
// coupling conditions; bc_apply[] carries hom3's segment assignment.
// ---------------------------------------------------------------------------
// Temperature of a partner cell from the partner's lhs: euler/physics.hpp:144-145
// (gamma p / rho) for Euler/CNS, heat/physics.hpp:51-58 (T itself) for heat.
__device__ __forceinline__ double partner_T(const BcParam& B, const PartnerView& pv, int o) {
  if (B.partner_physics == HEAT) return pv.q[o];
  const int pnd = B.partner_nd;
  const double* pq = pv.q;
  const long long pld = pv.ld;
  const double rho = pq[pnd * pld + o];
  double um2 = 0;
  for (int d = 0; d < pnd; ++d) {
    const double u = pq[d * pld + o] / rho;
    um2 = d == 0 ? u * u : um2 + u * u;
  }
  const double p = (B.partner_gamma - 1.) * (pq[(pnd + 1) * pld + o] - 0.5 * rho * um2);
  return B.partner_gamma * p / rho;
}

// q: the state the condition is applied to (lhs or rhs); qlhs: the solver's
// lhs, which the coupling conditions read temperatures from in both cases.
template <int ND, int PHYS>
__global__ void __launch_bounds__(kBlock) k_bc(double* __restrict__ q, const double* __restrict__ qlhs,
                                               Geometry g, GhostTables gt, PhysConst pc,
                                               const Scalars* __restrict__ sc, PartnerView pv) {
  constexpr int NV = nvars<ND, PHYS>();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gt.ng) return;
  const int b = gt.bc_apply[i];
  if (b == 255) return;
  const BcParam& B = gt.bcs[b];
  if (B.kind == BC_EXCHANGE) return;  // written by the caller (another solver's cells)
  const long long gcell = g.n_int + i;
  const int bc = gt.bndry[i];
  const long long ld = g.ld;
  double qb[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) qb[v] = q[v * ld + bc];
  double out[NV];
  switch (B.kind) {
    case BC_EULER_NEUMANN:  // euler/boundary_conditions.hpp:17-43
    case BC_HEAT_NEUMANN:   // heat/boundary_conditions.hpp:40-63
#pragma unroll
      for (int v = 0; v < NV; ++v) out[v] = qb[v] - gt.dx[i] * B.v[v];
      break;
    case BC_EULER_DIRICHLET:  // euler/boundary_conditions.hpp:47-67
    case BC_HEAT_DIRICHLET:   // heat/boundary_conditions.hpp:15-37
#pragma unroll
      for (int v = 0; v < NV; ++v) out[v] = 2.0 * B.v[v] - qb[v];
      break;
    case BC_EULER_VORTEX: {  // euler/boundary_conditions.hpp:70-93
      double vg[4] = {0, 0, 0, 0}, vb[4] = {0, 0, 0, 0};
      if (ND == 2) {
        const double t = sc[gt.ginst ? gt.ginst[i] : 0].time;
        isentropic_vortex(gt.xc[gcell], gt.xc[ld + gcell], t, vg);
        isentropic_vortex(gt.xc[bc], gt.xc[ld + bc], t, vb);
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        out[v] = vg[v & 3];
        q[v * ld + bc] = vb[v & 3];  // also overwrites the boundary cell
      }
      break;
    }
    case BC_CPL_EULER_EULER: {  // euler/coupling_conditions.hpp:17-35
      const int o = gt.partner[i];
      if (o < 0 || pv.q == nullptr) return;  // host refuses to launch without partner tables
#pragma unroll
      for (int v = 0; v < NV; ++v) out[v] = pv.q[v * pv.ld + o];
      break;
    }
    case BC_PERIODIC: {  // EXTENSION (not in hom3): copy of the paired cell
      const int o = gt.partner[i];
      if (o < 0) return;
#pragma unroll
      for (int v = 0; v < NV; ++v) out[v] = q[v * ld + o];
      break;
    }
    case BC_ADV_NEUMANN:  // advection/boundary_conditions.hpp:50-58
      out[0] = qb[0] - gt.dx[i] * B.v[0];
      break;
    case BC_ADV_DIRICHLET:  // :25-32
      out[0] = 2.0 * B.v[0] - qb[0];
      break;
    case BC_ADV_CHARACTERISTIC: {  // :71-91
      // inflow (the boundary cell's velocity along the ghost's direction points into the domain):
      // dirichlet(q_b, q_b); otherwise neumann(q_b, 0, dx).  Both are q_b.
      const int pos = gt.pos[i];
      const double v = g.vel ? g.vel[(pos >> 1) * ld + bc] : 0.0;
      const bool inflow = (v > 0. && (pos & 1) == 0) || (v < 0. && (pos & 1) == 1);
      out[0] = inflow ? 2.0 * qb[0] - qb[0] : qb[0] - gt.dx[i] * 0.0;
      break;
    }
    case BC_CPL_HEAT_CNS:     // heat/coupling_conditions.hpp:24-37
    case BC_CPL_HEAT_HEAT: {  // :47-60
      if (gt.partner[i] < 0 || pv.q == nullptr) return;
      const double Tother = partner_T(B, pv, gt.partner[i]);
      const double Tthis = qlhs[bc];
      const double kap = B.kind == BC_CPL_HEAT_CNS ? B.v[0] : 0.0;  // EXTENSION: k_solid / k_fluid
      const double Ts = B.kind == BC_CPL_HEAT_CNS
                            ? ((kap == 0.0 || kap == 1.0) ? 0.5 * (Tother + Tthis) : (Tother + kap * Tthis) / (1.0 + kap))
                            : 0.5 * (Tthis + Tother);
      out[0] = 2.0 * Ts - qb[0];
      break;
    }
    default: {
      if (NV == 1) { out[0] = qb[0]; break; }
      const double gamma = pc.gamma;
      // pv of the boundary cell: euler/quantities.hpp:173-186
      double bp[ND + 2], gp[ND + 2];
      bp[ND] = qb[ND];
      double vm2 = 0;
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        bp[d] = qb[d] / qb[ND];
        vm2 = d == 0 ? bp[d] * bp[d] : vm2 + bp[d] * bp[d];
      }
      bp[ND + 1] = (gamma - 1.0) * (qb[ND + 1] - 0.5 * qb[ND] * vm2);
#pragma unroll
      for (int v = 0; v < ND + 2; ++v) gp[v] = bp[v];
      if (B.kind == BC_CNS_INFLOW) {  // cns/boundary_conditions.hpp:37-61
#pragma unroll
        for (int d = 0; d < ND; ++d) gp[d] = 2.0 * B.v[d] - bp[d];
        gp[ND] = 2.0 * B.v[ND] - bp[ND];
      } else if (B.kind == BC_CNS_OUTFLOW) {  // :81-101
        gp[ND + 1] = 2.0 * B.v[ND + 1] - bp[ND + 1];
      } else if (B.kind == BC_CNS_ADIABATIC_NOSLIP) {  // :124-141
#pragma unroll
        for (int d = 0; d < ND; ++d) gp[d] = 0.0 - bp[d];
      } else if (B.kind == BC_CNS_ADIABATIC_SLIP) {  // :164-190
        const int ndir = gt.pos[i] >> 1;  // floor(boundary position w.r.t. the ghost / 2)
#pragma unroll
        for (int d = 0; d < ND; ++d)
          if (d == ndir) gp[d] = 0.0 - bp[d];
      } else if (B.kind == BC_CNS_ISOTHERMAL_NOSLIP || B.kind == BC_CPL_CNS_HEAT) {  // :209-228
        double Ts = B.v[0];
        if (B.kind == BC_CPL_CNS_HEAT) {  // cns/coupling_conditions.hpp:28-42
          if (gt.partner[i] < 0 || pv.q == nullptr) return;
          double ql[ND + 2];
#pragma unroll
          for (int v = 0; v < ND + 2; ++v) ql[v] = qlhs[v * ld + bc];
          double um2 = 0;
#pragma unroll
          for (int d = 0; d < ND; ++d) {
            const double u = ql[d] / ql[ND];
            um2 = d == 0 ? u * u : um2 + u * u;
          }
          const double pf = pc.gm1 * (ql[ND + 1] - 0.5 * ql[ND] * um2);
          const double Tf = gamma * pf / ql[ND];
          const double Tsol = partner_T(B, pv, gt.partner[i]);
          // EXTENSION: conductivity ratio kappa = k_solid / k_fluid in v[0] (0: hom3's mean)
          const double kap = B.v[0];
          Ts = (kap == 0.0 || kap == 1.0) ? 0.5 * (Tf + Tsol) : (Tf + kap * Tsol) / (1.0 + kap);
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) gp[d] = 0.0 - bp[d];
        const double rho_srfc = bp[ND + 1] * gamma / Ts;
        gp[ND] = 2.0 * rho_srfc - bp[ND];
      }
      // cv: euler/quantities.hpp:153-166
      out[ND] = gp[ND];
      double gm2 = 0;
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        out[d] = gp[ND] * gp[d];
        gm2 = d == 0 ? gp[d] * gp[d] : gm2 + gp[d] * gp[d];
      }
      out[ND + 1] = gp[ND + 1] / (gamma - 1.0) + 0.5 * gp[ND] * gm2;
      break;
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) q[v * ld + gcell] = out[v];
}

// ---------------------------------------------------------------------------
// cell slopes for the viscous flux: slope (solver.hpp:596-623) of every cell,
// ghosts included, stored as sl[(sd * NV + v) * ld + c].  Interior cells
// have both neighbours; a ghost takes its boundary cell's central slope, with
// the wall conditions' sign flip of tangential velocity slopes
// (boundary_condition.hpp:63-67, cns/boundary_conditions.hpp:143-147,230-234).
// ---------------------------------------------------------------------------
template <int ND>
__global__ void __launch_bounds__(kBlock) k_slopes(const double* __restrict__ q, Geometry g, GhostTables gt,
                                                   double* __restrict__ sl) {
  constexpr int NV = ND + 2;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n_tot) return;
  const long long ld = g.ld;
  long long b = c;
  int dg = -1;
  bool wall = false;
  if (c >= g.n_int) {
    const long long i = c - g.n_int;
    const BcParam& B = gt.bcs[gt.bc_own[i]];
    b = B.kind == BC_PERIODIC ? gt.partner[i] : gt.bndry[i];
    if (b < 0) return;
    dg = gt.pos[i] >> 1;
    wall = B.wall != 0;
  }
  const double h2 = 2. * g.len[g.lvl[b]];
#pragma unroll
  for (int sd = 0; sd < ND; ++sd) {
    const int m = g.nbr[(2 * sd) * ld + b];
    const int p = g.nbr[(2 * sd + 1) * ld + b];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = (__ldg(q + v * ld + p) - __ldg(q + v * ld + m)) / h2;
      if (wall && v < ND && sd != dg) s = -s;
      sl[(sd * NV + v) * ld + c] = s;
    }
  }
}

// Explicit stage update from q0 (the step's start state, in `out` for the
// in-place stages), the stage input qc and r = dt/dx R(qc):
//   MODE 0: qc + r (FE, first stage of RK2 / SSP-RK3)
//   MODE 2: 0.5 ((q0 + qc) + r) (RK2 second stage, solver.hpp:483-494)
//   MODE 3: 3/4 q0 + 1/4 (qc + r), MODE 4: 1/3 q0 + 2/3 (qc + r) (EXTENSION: SSP-RK3)
template <int MODE> __device__ __forceinline__ double rk_combine(double q0, double qc, double r) {
  if (MODE == 0) return qc + r;
  if (MODE == 2) return 0.5 * ((q0 + qc) + r);
  if (MODE == 3) return 0.75 * q0 + 0.25 * (qc + r);
  return (1.0 / 3.0) * q0 + (2.0 / 3.0) * (qc + r);
}

// ---------------------------------------------------------------------------
// Stage kernel: num_flux (solver.hpp:440-460) + the explicit update of evolve
// (solver.hpp:470-494).
//   out = rk_combine<MODE>(out, qin, dt/dx R(qin)); MODE 2, 3 and 4 read the
//   start state from `out` (in place).
// FUSE: also reduce the next step's cell dt of `out` into *dtmin (the
// compute_dt of the next set_dt; valid when no condition rewrites interior cells).
// HANG: the grid has coarse/fine faces (EXTENSION, not in hom3).
// ---------------------------------------------------------------------------
template <int ND, int PHYS, int FLUX, class R, int MODE, bool HANG, bool FUSE>
__global__ void __launch_bounds__(kBlock) k_stage(const double* __restrict__ qin, double* out,
                                                  const double* __restrict__ sl, Geometry g, PhysConst pc,
                                                  const Scalars* __restrict__ sc, long long* dtmin) {
  constexpr int NV = nvars<ND, PHYS>();
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int inst = tile_instance(g, blockIdx.x);
  const bool live = c < instance_end(g, inst);
  long long ord = kOrdMax;
  bool bad = false;
  if (live) {
    const long long ld = g.ld;
    const double dt = sc[inst].dt;
    const double dx = g.len[g.lvl[c]];
    double qc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) qc[v] = __ldg(qin + v * ld + c);
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;

    if (PHYS == ADVECTION) {
      // advection/physics.hpp:120-145 on the cells' velocities along d: local Lax-Friedrichs,
      // or hom3's upwind flux u_L q_L, negated when the face velocity (u_L + u_R) / 2 is negative
      auto adv_flux = [&](double qL, double qR, double uL, double uR) {
        if (FLUX == LLF) {
          const double lambda_max = fmax(fabs(uL), fabs(uR));
          return 0.5 * (qL * uL + qR * uR + lambda_max * (qL - qR));
        }
        const double u_srfc = 0.5 * (uL + uR);
        const double f = uL * qL;
        return u_srfc < 0 ? f * -1. : f;
      };
      if (!HANG) {
        // all neighbour indices first, then all neighbour states and velocities: the loads of
        // every face are in flight together
        int nm[ND], np_[ND];
        double uc[ND], qm[ND], qp[ND], um[ND], up[ND];
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          nm[d] = __ldg(g.nbr + (2 * d) * ld + c);
          np_[d] = __ldg(g.nbr + (2 * d + 1) * ld + c);
          uc[d] = __ldg(g.vel + d * ld + c);
        }
#pragma unroll
        for (int d = 0; d < ND; ++d) {
          qm[d] = __ldg(qin + nm[d]);
          um[d] = __ldg(g.vel + d * ld + nm[d]);
          qp[d] = __ldg(qin + np_[d]);
          up[d] = __ldg(g.vel + d * ld + np_[d]);
        }
#pragma unroll
        for (int d = 0; d < ND; ++d)
          acc[0] = acc[0] + (adv_flux(qm[d], qc[0], um[d], uc[d]) - adv_flux(qc[0], qp[d], uc[d], up[d]));
      }
#pragma unroll
      for (int d = 0; d < ND && HANG; ++d) {
        const double uc = __ldg(g.vel + d * ld + c);
        const int m = g.nbr[(2 * d) * ld + c], p = g.nbr[(2 * d + 1) * ld + c];
        double fm, fp;
        if (!HANG || m >= 0) {
          fm = adv_flux(__ldg(qin + m), qc[0], __ldg(g.vel + d * ld + m), uc);
        } else {
          const long long k = -m - 2;
          double ws = 0;
#pragma unroll
          for (int j = 0; j < (1 << (ND - 1)); ++j) {
            const int n = g.sub[j * g.nsub + k];
            const double f = adv_flux(__ldg(qin + n), qc[0], __ldg(g.vel + d * ld + n), uc);
            ws = j == 0 ? f : ws + f;
          }
          fm = (ND == 2 ? 0.5 : 0.25) * ws;
        }
        if (!HANG || p >= 0) {
          fp = adv_flux(qc[0], __ldg(qin + p), uc, __ldg(g.vel + d * ld + p));
        } else {
          const long long k = -p - 2;
          double ws = 0;
#pragma unroll
          for (int j = 0; j < (1 << (ND - 1)); ++j) {
            const int n = g.sub[j * g.nsub + k];
            const double f = adv_flux(qc[0], __ldg(qin + n), uc, __ldg(g.vel + d * ld + n));
            ws = j == 0 ? f : ws + f;
          }
          fp = (ND == 2 ? 0.5 : 0.25) * ws;
        }
        acc[0] = acc[0] + (fm - fp);
      }
    } else if (PHYS == HEAT) {
      // three_point: heat/physics.hpp:113-119, (1/dx)(T_l - T_r)
      const double idx = 1 / dx;
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const int m = g.nbr[(2 * d) * ld + c], p = g.nbr[(2 * d + 1) * ld + c];
        double fm, fp;
        if (!HANG || m >= 0) {
          fm = idx * (__ldg(qin + m) - qc[0]);
        } else {
          const long long k = -m - 2;
          double ws = 0;
#pragma unroll
          for (int j = 0; j < (1 << (ND - 1)); ++j) {
            const double f = idx * (__ldg(qin + g.sub[j * g.nsub + k]) - qc[0]);
            ws = j == 0 ? f : ws + f;
          }
          fm = (ND == 2 ? 0.5 : 0.25) * ws;
        }
        if (!HANG || p >= 0) {
          fp = idx * (qc[0] - __ldg(qin + p));
        } else {
          const long long k = -p - 2;
          double ws = 0;
#pragma unroll
          for (int j = 0; j < (1 << (ND - 1)); ++j) {
            const double f = idx * (qc[0] - __ldg(qin + g.sub[j * g.nsub + k]));
            ws = j == 0 ? f : ws + f;
          }
          fp = (ND == 2 ? 0.5 : 0.25) * ws;
        }
        acc[0] = acc[0] + (fm - fp);
      }
    } else {
      const R gamma = (R)pc.gamma, gm1 = (R)pc.gm1;
      Prim<R, ND> Pc;
#pragma unroll
      for (int v = 0; v < ND + 2; ++v) Pc.q[v] = (R)qc[v];
      make_prim<R, ND>(Pc, gamma, gm1);
      const R dx_dt = (R)(dx / dt);
      R slc[PHYS == CNS ? ND * (ND + 2) : 1];
      if (PHYS == CNS) {
#pragma unroll
        for (int k = 0; k < ND * (ND + 2); ++k) slc[k] = (R)__ldg(sl + k * ld + c);
      }
      // flux of the face (l = a, r = b) with a or b the centre cell
      auto face = [&](const Prim<R, ND>& L, const Prim<R, ND>& Rt, const R* sL, const R* sR, R len_r, int d,
                      R* f) {
        if (FLUX == LLF) llf<R, ND>(L, Rt, d, dx_dt, f);
        else ausm<R, ND>(L, Rt, d, f);
        if (PHYS == CNS) {
          R fv[ND + 2];
          viscous<R, ND>(L, Rt, sL, sR, d, len_r, pc, fv);
#pragma unroll
          for (int v = 0; v < ND + 2; ++v) f[v] = f[v] + fv[v];
        }
      };
      auto load_nb = [&](int n, Prim<R, ND>& P, R* sn) {
        load_prim<R, ND>(P, qin, ld, n, gamma, gm1);
        if (PHYS == CNS) {
#pragma unroll
          for (int k = 0; k < ND * (ND + 2); ++k) sn[k] = (R)__ldg(sl + k * ld + n);
        }
      };
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const int m = g.nbr[(2 * d) * ld + c], p = g.nbr[(2 * d + 1) * ld + c];
        double fm[NV], fp[NV];
        {
          if (!HANG || m >= 0) {
            Prim<R, ND> Pn;
            R sn[PHYS == CNS ? ND * (ND + 2) : 1];
            load_nb(m, Pn, sn);
            R f[ND + 2];
            face(Pn, Pc, sn, slc, (R)dx, d, f);
#pragma unroll
            for (int v = 0; v < NV; ++v) fm[v] = (double)f[v];
          } else {
            const long long k = -m - 2;
#pragma unroll
            for (int j = 0; j < (1 << (ND - 1)); ++j) {
              const int n = g.sub[j * g.nsub + k];
              Prim<R, ND> Pn;
              R sn[PHYS == CNS ? ND * (ND + 2) : 1];
              load_nb(n, Pn, sn);
              R f[ND + 2];
              face(Pn, Pc, sn, slc, (R)dx, d, f);
#pragma unroll
              for (int v = 0; v < NV; ++v) fm[v] = j == 0 ? (double)f[v] : fm[v] + (double)f[v];
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) fm[v] = (ND == 2 ? 0.5 : 0.25) * fm[v];
          }
        }
        {
          if (!HANG || p >= 0) {
            Prim<R, ND> Pn;
            R sn[PHYS == CNS ? ND * (ND + 2) : 1];
            load_nb(p, Pn, sn);
            R f[ND + 2];
            face(Pc, Pn, slc, sn, (R)g.len[g.lvl[p]], d, f);
#pragma unroll
            for (int v = 0; v < NV; ++v) fp[v] = (double)f[v];
          } else {
            const long long k = -p - 2;
#pragma unroll
            for (int j = 0; j < (1 << (ND - 1)); ++j) {
              const int n = g.sub[j * g.nsub + k];
              Prim<R, ND> Pn;
              R sn[PHYS == CNS ? ND * (ND + 2) : 1];
              load_nb(n, Pn, sn);
              R f[ND + 2];
              face(Pc, Pn, slc, sn, (R)g.len[g.lvl[n]], d, f);
#pragma unroll
              for (int v = 0; v < NV; ++v) fp[v] = j == 0 ? (double)f[v] : fp[v] + (double)f[v];
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) fp[v] = (ND == 2 ? 0.5 : 0.25) * fp[v];
          }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fm[v] - fp[v]);
      }
    }
    const double k = dt / dx;
    double o[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = rk_combine<MODE>(MODE == 0 ? 0.0 : out[v * ld + c], qc[v], k * acc[v]);
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v * ld + c] = o[v];
    if (FUSE) {
      double uc[ND];
      if (PHYS == ADVECTION) {
#pragma unroll
        for (int d = 0; d < ND; ++d) uc[d] = __ldg(g.vel + d * ld + c);
      }
      const double cd = cell_dt<ND, PHYS>(o, dx, pc, uc, &bad);
      if (!isnan(cd)) ord = dbl_to_ord(cd);
    }
  }
  if (FUSE) {
    flag_bad_state(bad, sc, inst);
    block_min_atomic(ord, per_instance(dtmin, inst));
  }
}

// ---------------------------------------------------------------------------
// Tile stage kernel (Euler).  A block owns kBlock consecutive cells of the
// Morton order, which form a compact brick of the grid.  Primitive variables
// are computed once per cell into shared memory, each cell evaluates the flux
// of its plus face in every direction once, and a cell takes its minus-face
// flux from the neighbour's plus-face result when that neighbour is in the
// tile and links back to it (same-level face) -- the same F(l, r) evaluation
// hom3's num_flux performs twice (solver.hpp:446-453), so results are
// bit-identical to k_stage.  Faces leaving the tile, and coarse/fine faces,
// are evaluated directly.
// Shared memory (dynamic): prim [ND+4][kBlock] of R, plus-face flux
// [ND][ND+2][kBlock] of double.
// ---------------------------------------------------------------------------
template <class R, int ND>
__host__ __device__ constexpr size_t tile_smem_bytes() {
  return sizeof(R) * (3 * ND + 4) * kBlock + sizeof(double) * ND * (ND + 2) * kBlock + sizeof(int) * ND * kBlock;
}

template <int ND, int FLUX, class R, int MODE, bool HANG, bool FUSE>
__global__ void __launch_bounds__(kBlock, 3) k_stage_tile(const double* __restrict__ qin, double* out, Geometry g,
                                                       PhysConst pc, const Scalars* __restrict__ sc,
                                                       long long* dtmin) {
  constexpr int NV = ND + 2;
  constexpr int NP = 3 * ND + 4;  // rows: q[ND+2], u[ND], p, a, M[ND]
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sprim = reinterpret_cast<R*>(smem_raw);
  const long long c0 = (long long)blockIdx.x * kBlock;
  const int tid = threadIdx.x;
  const long long c = c0 + tid;
  const int inst = tile_instance(g, blockIdx.x);
  const long long iend = instance_end(g, inst);
  const bool live = c < iend;
  const long long ld = g.ld;
  const R gamma = (R)pc.gamma, gm1 = (R)pc.gm1;
  const double dt = sc[inst].dt;
  const double dx = live ? g.len[g.lvl[c]] : 1.0;
  const R dx_dt = (R)(dx / dt);

  // ---- phase A: own state and primitives -> shared memory ----
  double qc[NV];
  Prim<R, ND> Pc;
  if (live) {
#pragma unroll
    for (int v = 0; v < NV; ++v) qc[v] = __ldg(qin + v * ld + c);
#pragma unroll
    for (int v = 0; v < NV; ++v) Pc.q[v] = (R)qc[v];
    make_prim<R, ND>(Pc, gamma, gm1);
#pragma unroll
    for (int v = 0; v < NV; ++v) sprim[v * kBlock + tid] = Pc.q[v];
#pragma unroll
    for (int d = 0; d < ND; ++d) sprim[(NV + d) * kBlock + tid] = Pc.u[d];
    sprim[(NV + ND) * kBlock + tid] = Pc.p;
    sprim[(NV + ND + 1) * kBlock + tid] = Pc.a;
#pragma unroll
    for (int d = 0; d < ND; ++d) sprim[(NV + ND + 2 + d) * kBlock + tid] = Pc.M[d];
  }
  __syncthreads();

  const long long tile_end = min(c0 + (long long)kBlock, iend);
  auto in_tile = [&](long long n) { return n >= c0 && n < tile_end; };
  auto prim_of = [&](long long n, Prim<R, ND>& P) {
    if (in_tile(n)) {
      const int t = (int)(n - c0);
#pragma unroll
      for (int v = 0; v < NV; ++v) P.q[v] = sprim[v * kBlock + t];
#pragma unroll
      for (int d = 0; d < ND; ++d) P.u[d] = sprim[(NV + d) * kBlock + t];
      P.p = sprim[(NV + ND) * kBlock + t];
      P.a = sprim[(NV + ND + 1) * kBlock + t];
#pragma unroll
      for (int d = 0; d < ND; ++d) P.M[d] = sprim[(NV + ND + 2 + d) * kBlock + t];
    } else {
      load_prim<R, ND>(P, qin, ld, (int)n, gamma, gm1);
    }
  };
  auto flux = [&](const Prim<R, ND>& L, const Prim<R, ND>& Rt, int d, R* f) {
    if (FLUX == LLF) llf<R, ND>(L, Rt, d, dx_dt, f);
    else ausm<R, ND>(L, Rt, d, f);
  };
  constexpr int NS = 1 << (ND - 1);
  constexpr double W = ND == 2 ? 0.5 : 0.25;
  double* sf = reinterpret_cast<double*>(smem_raw + sizeof(R) * NP * kBlock);  // [ND][NV][kBlock]
  int* snp = reinterpret_cast<int*>(sf + ND * NV * kBlock);                     // [ND][kBlock] plus neighbours

  // ---- phase B: plus-face fluxes ----
  int nbm[ND];
  if (live) {
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const int p = g.nbr[(2 * d + 1) * ld + c];
      nbm[d] = g.nbr[(2 * d) * ld + c];
      snp[d * kBlock + tid] = p;
      double fp[NV];
      if (!HANG || p >= 0) {
        Prim<R, ND> Pn;
        prim_of(p, Pn);
        R f[NV];
        flux(Pc, Pn, d, f);
#pragma unroll
        for (int v = 0; v < NV; ++v) fp[v] = (double)f[v];
      } else {
        const long long k = -p - 2;
#pragma unroll
        for (int j = 0; j < NS; ++j) {
          Prim<R, ND> Pn;
          prim_of(g.sub[j * g.nsub + k], Pn);
          R f[NV];
          flux(Pc, Pn, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fp[v] = j == 0 ? (double)f[v] : fp[v] + (double)f[v];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) fp[v] = __dmul_rn(W, fp[v]);  // rounded: no FMA with the sums below
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) sf[(d * NV + v) * kBlock + tid] = fp[v];
    }
  }
  __syncthreads();

  // ---- phase C: minus faces, residual, update ----
  long long ord = kOrdMax;
  bool bad = false;
  if (live) {
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const int m = nbm[d];
      double fm[NV];
      if (!HANG || m >= 0) {
        if (in_tile(m) && snp[d * kBlock + (int)(m - c0)] == (int)c) {
          const int t = (int)(m - c0);
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = sf[(d * NV + v) * kBlock + t];
        } else {
          Prim<R, ND> Pn;
          prim_of(m, Pn);
          R f[NV];
          flux(Pn, Pc, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = (double)f[v];
        }
      } else {
        const long long k = -m - 2;
#pragma unroll
        for (int j = 0; j < NS; ++j) {
          Prim<R, ND> Pn;
          prim_of(g.sub[j * g.nsub + k], Pn);
          R f[NV];
          flux(Pn, Pc, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = j == 0 ? (double)f[v] : fm[v] + (double)f[v];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) fm[v] = __dmul_rn(W, fm[v]);
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fm[v] - sf[(d * NV + v) * kBlock + tid]);
    }
    const double k = dt / dx;
    double o[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = rk_combine<MODE>(MODE == 0 ? 0.0 : out[v * ld + c], qc[v], k * acc[v]);
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v * ld + c] = o[v];
    if (FUSE) {
      const double cd = cell_dt<ND, EULER>(o, dx, pc, nullptr, &bad);
      if (!isnan(cd)) ord = dbl_to_ord(cd);
    }
  }
  if (FUSE) {
    flag_bad_state(bad, sc, inst);
    block_min_atomic(ord, per_instance(dtmin, inst));
  }
}

// ---------------------------------------------------------------------------
// AUSM tile kernel.  Same tiling as k_stage_tile, specialised for the AUSM
// flux: each cell publishes its face state -- theta = a (rho u, rho, rho E + p)
// (theta_, euler/physics.hpp:315-325), p and the Mach numbers M_d -- so a
// face flux is m_i theta_{up} + p_i e_d (euler/physics.hpp:276-293) from
// 7 shared loads.  All of the cell's own global loads are issued first.
// Shared memory: face state [2ND+4][kBlock] of R, plus-face flux
// [ND][ND+2][kBlock] of double, plus neighbours [ND][kBlock] of int.
// ---------------------------------------------------------------------------
template <class R, int ND, int TB = kBlock>
__host__ __device__ constexpr size_t ausm_smem_bytes() {
  return sizeof(R) * (2 * ND + 3) * TB + sizeof(double) * ND * (ND + 2) * TB + sizeof(int) * ND * TB;
}

template <class R, int ND> struct FaceState {
  R th[ND + 2];
  R p;
  R M;  // Mach number along the face direction
};

template <class R, int ND>
__device__ __forceinline__ void ausm_face(const FaceState<R, ND>& L, const FaceState<R, ND>& Rt, int d, R* f) {
  const R mi = m_int<R>(R(1), L.M) + m_int<R>(R(-1), Rt.M);
  const R pi = p_int<R>(R(1), L.M) * L.p + p_int<R>(R(-1), Rt.M) * Rt.p;
  const bool left = mi >= R(0);
#pragma unroll
  for (int v = 0; v < ND + 2; ++v) f[v] = (left ? L.th[v] : Rt.th[v]) * mi;
#pragma unroll
  for (int v = 0; v < ND; ++v)
    if (v == d) f[v] = f[v] + pi;
}

template <class R, int ND>
__device__ __forceinline__ void face_state_global(FaceState<R, ND>& F, const double* __restrict__ q, long long ld,
                                                  int n, int d, R gamma, R gm1) {
  Prim<R, ND> P;
  load_prim<R, ND>(P, q, ld, n, gamma, gm1);
#pragma unroll
  for (int v = 0; v < ND + 1; ++v) F.th[v] = P.q[v] * P.a;
  F.th[ND + 1] = (P.q[ND + 1] + P.p) * P.a;
  F.p = P.p;
  F.M = P.M[d];
}

#ifndef H3C_AUSM_MINB
#define H3C_AUSM_MINB 4  // blocks per SM the AUSM tile kernel is register-budgeted for
#endif
// Persistent: block b processes tiles b, b + gridDim.x, ... (the grid size is
// a launch choice the batch autotuner makes; one block per tile by default).
// TB: cells per tile = threads per block.  kBlock (256: an 8x8x4 Morton brick
// in 3D), or 512 (8x8x8) for one grid: g.ntiles then counts 512-cell tiles,
// and the same 32 warps per SM come as two blocks instead of four.
template <int ND, class R, int MODE, bool HANG, bool FUSE, int TB = kBlock>
__global__ void __launch_bounds__(TB, H3C_AUSM_MINB * kBlock / TB) k_stage_ausm(const double* __restrict__ qin,
                                                                              double* out, Geometry g, PhysConst pc,
                                                                              const Scalars* __restrict__ sc,
                                                                              long long* dtmin) {
  constexpr int NV = ND + 2;
  constexpr int NS = 1 << (ND - 1);
  constexpr double W = ND == 2 ? 0.5 : 0.25;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* sfs = reinterpret_cast<R*>(smem_raw);                                   // [NV + 1 + ND][TB]
  double* sf = reinterpret_cast<double*>(smem_raw + sizeof(R) * (2 * ND + 3) * TB);  // [ND][NV][TB]
  int* snp = reinterpret_cast<int*>(sf + ND * NV * TB);                  // [ND][TB]
  const int tid = threadIdx.x;
  const long long ld = g.ld;
  const R gamma = (R)pc.gamma, gm1 = (R)pc.gm1;

  for (long long tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
    const long long c0 = tile * TB;
    const long long c = c0 + tid;
    const int inst = tile_instance(g, tile);
    const long long tile_end = min(c0 + (long long)TB, instance_end(g, inst));
    const bool live = c < tile_end;
    if (MODE != 0 && live) prefetch_row_l2<NV>(out, ld, c);  // the in-place start state, read at the update

    // ---- own loads first: state, neighbours, level ----
    double qc[NV];
    int nbp[ND], nbm[ND];
    if (live) {
#pragma unroll
      for (int v = 0; v < NV; ++v) qc[v] = __ldg(qin + v * ld + c);
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        nbm[d] = __ldg(g.nbr + (2 * d) * ld + c);
        nbp[d] = __ldg(g.nbr + (2 * d + 1) * ld + c);
      }
    }
    // ---- face state of the cell -> shared memory ----
    if (live) {
      Prim<R, ND> Pc;
#pragma unroll
      for (int v = 0; v < NV; ++v) Pc.q[v] = (R)qc[v];
      make_prim<R, ND>(Pc, gamma, gm1);
#pragma unroll
      for (int v = 0; v < ND + 1; ++v) sfs[v * TB + tid] = Pc.q[v] * Pc.a;
      sfs[(ND + 1) * TB + tid] = (Pc.q[ND + 1] + Pc.p) * Pc.a;
      sfs[NV * TB + tid] = Pc.p;
#pragma unroll
      for (int d = 0; d < ND; ++d) sfs[(NV + 1 + d) * TB + tid] = Pc.M[d];
#pragma unroll
      for (int d = 0; d < ND; ++d) snp[d * TB + tid] = nbp[d];
    }
    __syncthreads();

    auto in_tile = [&](long long n) { return n >= c0 && n < tile_end; };
    auto fstate = [&](long long n, int d, FaceState<R, ND>& F) {
      if (in_tile(n)) {
        const int t = (int)(n - c0);
#pragma unroll
        for (int v = 0; v < NV; ++v) F.th[v] = sfs[v * TB + t];
        F.p = sfs[NV * TB + t];
        F.M = sfs[(NV + 1 + d) * TB + t];
      } else {
        face_state_global<R, ND>(F, qin, ld, (int)n, d, gamma, gm1);
      }
    };
    auto own = [&](int d, FaceState<R, ND>& F) {
#pragma unroll
      for (int v = 0; v < NV; ++v) F.th[v] = sfs[v * TB + tid];
      F.p = sfs[NV * TB + tid];
      F.M = sfs[(NV + 1 + d) * TB + tid];
    };

    // ---- plus faces ----
    if (live) {
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        FaceState<R, ND> Fc;
        own(d, Fc);
        const int p = nbp[d];
        double fp[NV];
        if (!HANG || p >= 0) {
          FaceState<R, ND> Fn;
          fstate(p, d, Fn);
          R f[NV];
          ausm_face<R, ND>(Fc, Fn, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fp[v] = (double)f[v];
        } else {
          const long long k = -p - 2;
#pragma unroll
          for (int j = 0; j < NS; ++j) {
            FaceState<R, ND> Fn;
            fstate(__ldg(g.sub + j * g.nsub + k), d, Fn);
            R f[NV];
            ausm_face<R, ND>(Fc, Fn, d, f);
#pragma unroll
            for (int v = 0; v < NV; ++v) fp[v] = j == 0 ? (double)f[v] : fp[v] + (double)f[v];
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) fp[v] = __dmul_rn(W, fp[v]);  // rounded: no FMA with the sums below
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) sf[(d * NV + v) * TB + tid] = fp[v];
      }
    }
    __syncthreads();

    // ---- minus faces, residual, update ----
    long long ord = kOrdMax;
  bool bad = false;
    if (live) {
      double acc[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] = 0.0;
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const int m = nbm[d];
        double fm[NV];
        if (in_tile(m) && snp[d * TB + (int)(m - c0)] == (int)c) {
          const int t = (int)(m - c0);
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = sf[(d * NV + v) * TB + t];
        } else if (!HANG || m >= 0) {
          FaceState<R, ND> Fc, Fn;
          own(d, Fc);
          fstate(m, d, Fn);
          R f[NV];
          ausm_face<R, ND>(Fn, Fc, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = (double)f[v];
        } else {
          FaceState<R, ND> Fc;
          own(d, Fc);
          const long long k = -m - 2;
#pragma unroll
          for (int j = 0; j < NS; ++j) {
            FaceState<R, ND> Fn;
            fstate(__ldg(g.sub + j * g.nsub + k), d, Fn);
            R f[NV];
            ausm_face<R, ND>(Fn, Fc, d, f);
#pragma unroll
            for (int v = 0; v < NV; ++v) fm[v] = j == 0 ? (double)f[v] : fm[v] + (double)f[v];
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = __dmul_rn(W, fm[v]);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fm[v] - sf[(d * NV + v) * TB + tid]);
      }
      double qo[NV];
      if (MODE != 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) qo[v] = out[v * ld + c];
      }
      // the cell's own state and length read again (L1/L2) rather than held
      // in registers across the face loops: fewer spills at 64 registers
      const double dt = sc[inst].dt;
      const double dxc = g.len[g.lvl[c]];
      const double k = dt / dxc;
      double o[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) o[v] = rk_combine<MODE>(MODE == 0 ? 0.0 : qo[v], __ldg(qin + v * ld + c), k * acc[v]);
#pragma unroll
      for (int v = 0; v < NV; ++v) out[v * ld + c] = o[v];
      if (FUSE) {
        const double cd = cell_dt<ND, EULER>(o, dxc, pc, nullptr, &bad);
        if (!isnan(cd)) ord = dbl_to_ord(cd);
      }
    }
    if (FUSE) {
    flag_bad_state(bad, sc, inst);
    block_min_atomic_tb<TB>(ord, per_instance(dtmin, inst));
  }
    __syncthreads();  // shared memory is rewritten by the next tile
  }
}

// ---------------------------------------------------------------------------
// AUSM stage, one thread per cell without shared memory: every face of the
// cell is evaluated by the cell itself (each interior face twice, once from
// each side, as hom3's num_flux does: solver.hpp:446-453), the neighbours'
// face states recomputed from their state.  No barrier and no divergence
// between border and interior cells: a warp's lanes all run the same code.
// The face flux is the tile kernels' F(l, r) (face_state_global +
// ausm_face), summed per direction in hom3's order.
// ---------------------------------------------------------------------------
#ifndef H3C_CELL_MINB
#define H3C_CELL_MINB 3  // blocks per SM the per-cell AUSM kernel is register-budgeted for
#endif
template <int ND, class R, int MODE, bool HANG, bool FUSE>
__global__ void __launch_bounds__(kBlock, H3C_CELL_MINB) k_stage_ausm_cell(const double* __restrict__ qin, double* out,
                                                                          Geometry g, PhysConst pc,
                                                                          const Scalars* __restrict__ sc,
                                                                          long long* dtmin) {
  constexpr int NV = ND + 2, NS = 1 << (ND - 1);
  constexpr double W = ND == 2 ? 0.5 : 0.25;
  const int tid = threadIdx.x;
  const long long c = (long long)blockIdx.x * blockDim.x + tid;
  const int inst = tile_instance(g, blockIdx.x);
  const bool live = c < instance_end(g, inst);
  const long long ld = g.ld;
  const R gamma = (R)pc.gamma, gm1 = (R)pc.gm1;
  if (MODE != 0 && live) prefetch_row_l2<NV>(out, ld, c);  // the in-place start state, read at the update
  // The cell's own face state (theta, p, Mach number along each direction),
  // kept in the thread's column of shared memory rather than in registers
  // across the direction loop: at three blocks per SM the loop spills otherwise.
  __shared__ R own[NV + 1 + ND][kBlock];
  __shared__ long long min_slot;
  __shared__ unsigned min_cnt;
  if (FUSE) {
    if (tid == 0) {
      min_slot = kOrdMax;
      min_cnt = 0;
    }
    __syncthreads();  // every warp is at the start: the only barrier
  }
  long long ord = kOrdMax;
  bool bad = false;
  if (live) {
    {
      Prim<R, ND> P;
#pragma unroll
      for (int v = 0; v < NV; ++v) P.q[v] = (R)__ldg(qin + v * ld + c);
      make_prim<R, ND>(P, gamma, gm1);
#pragma unroll
      for (int v = 0; v < ND + 1; ++v) own[v][tid] = P.q[v] * P.a;
      own[ND + 1][tid] = (P.q[ND + 1] + P.p) * P.a;
      own[NV][tid] = P.p;
#pragma unroll
      for (int d = 0; d < ND; ++d) own[NV + 1 + d][tid] = P.M[d];
    }
    auto neighbour_fs = [&](int d, FaceState<R, ND>& F, const double* qn) {
      Prim<R, ND> P;
#pragma unroll
      for (int v = 0; v < NV; ++v) P.q[v] = (R)qn[v];
      make_prim<R, ND>(P, gamma, gm1);
#pragma unroll
      for (int v = 0; v < ND + 1; ++v) F.th[v] = P.q[v] * P.a;
      F.th[ND + 1] = (P.q[ND + 1] + P.p) * P.a;
      F.p = P.p;
      F.M = P.M[d];
    };
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
    // Directions whose faces are all plain run in the unrolled loop; a
    // direction with a coarse/fine group on either side is deferred to a
    // second, rolled loop after it, so that the group path's registers are
    // not live across the common path (which would spill it).
    unsigned deferred = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const int m = __ldg(g.nbr + 2 * d * ld + c), p = __ldg(g.nbr + (2 * d + 1) * ld + c);
      if (HANG && (m < 0 || p < 0)) {
        deferred |= 1u << d;
        continue;
      }
      FaceState<R, ND> Fc;
#pragma unroll
      for (int v = 0; v < NV; ++v) Fc.th[v] = own[v][tid];
      Fc.p = own[NV][tid];
      Fc.M = own[NV + 1 + d][tid];
      // both neighbours' states along d, loaded together
      double qm[NV], qp[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        qm[v] = __ldg(qin + v * ld + m);
        qp[v] = __ldg(qin + v * ld + p);
      }
      FaceState<R, ND> Fm, Fp;
      neighbour_fs(d, Fm, qm);
      neighbour_fs(d, Fp, qp);
      R f[NV];
      double fm[NV];
      ausm_face<R, ND>(Fm, Fc, d, f);
#pragma unroll
      for (int v = 0; v < NV; ++v) fm[v] = (double)f[v];
      ausm_face<R, ND>(Fc, Fp, d, f);
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fm[v] - (double)f[v]);
    }
    if (HANG && deferred) {
      // coarse/fine faces: W times the sum over the group's fine cells
#pragma unroll 1
      for (int d = 0; d < ND; ++d) {
        if (!((deferred >> d) & 1u)) continue;
        FaceState<R, ND> Fc;
#pragma unroll
        for (int v = 0; v < NV; ++v) Fc.th[v] = own[v][tid];
        Fc.p = own[NV][tid];
        Fc.M = own[NV + 1 + d][tid];
        double fo[2][NV];
#pragma unroll 1
        for (int side = 0; side < 2; ++side) {
          const int n = __ldg(g.nbr + (2 * d + side) * ld + c);
          const int cnt = n >= 0 ? 1 : NS;
          const long long kk = -(long long)n - 2;
          double sum[NV];
#pragma unroll 1
          for (int j = 0; j < cnt; ++j) {
            FaceState<R, ND> Fn;
            face_state_global<R, ND>(Fn, qin, ld, n >= 0 ? n : __ldg(g.sub + j * g.nsub + kk), d, gamma, gm1);
            R f[NV];
            if (side == 0) ausm_face<R, ND>(Fn, Fc, d, f);
            else ausm_face<R, ND>(Fc, Fn, d, f);
#pragma unroll
            for (int v = 0; v < NV; ++v) sum[v] = j == 0 ? (double)f[v] : sum[v] + (double)f[v];
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) fo[side][v] = n < 0 ? __dmul_rn(W, sum[v]) : sum[v];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fo[0][v] - fo[1][v]);
      }
    }
    const double dx = g.len[g.lvl[c]];
    const double k = sc[inst].dt * nr_rcp(dx);
    double qc[NV], qo[NV];  // the stage input and the in-place stages' start state, read only now
#pragma unroll
    for (int v = 0; v < NV; ++v) qc[v] = __ldg(qin + v * ld + c);
    if (MODE != 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) qo[v] = out[v * ld + c];
    }
    double o[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = rk_combine<MODE>(MODE == 0 ? 0.0 : qo[v], qc[v], k * acc[v]);
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v * ld + c] = o[v];
    if (FUSE) {
      const double cd = cell_dt<ND, EULER>(o, dx, pc, nullptr, &bad);
      if (!isnan(cd)) ord = dbl_to_ord(cd);
    }
  }
  if (FUSE) {
    flag_bad_state(bad, sc, inst);
    block_min_atomic_nobar(ord, per_instance(dtmin, inst), &min_slot, &min_cnt);
  }
}

#ifndef H3C_DEVICE_FUNCTIONS_ONLY  // non-template kernels: defined in one translation unit
// gather / scatter between the caller's numbering and the internal one
__global__ void k_gather(const double* __restrict__ src, long long src_ld, double* __restrict__ dst,
                         long long dst_ld, const long long* __restrict__ dev_to_caller, long long n, int nv) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const long long s = dev_to_caller[c];
  if (s < 0) return;  // padding between batch instances
  for (int v = 0; v < nv; ++v) dst[v * dst_ld + c] = src[v * src_ld + s];
}
__global__ void k_scatter(const double* __restrict__ src, long long src_ld, double* __restrict__ dst,
                          long long dst_ld, const long long* __restrict__ dev_to_caller, long long n, int nv) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  const long long s = dev_to_caller[c];
  if (s < 0) return;  // padding between batch instances
  for (int v = 0; v < nv; ++v) dst[v * dst_ld + s] = src[v * src_ld + c];
}
#endif  // H3C_DEVICE_FUNCTIONS_ONLY

}  // namespace h3c
