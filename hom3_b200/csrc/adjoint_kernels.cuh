// adjoint_kernels.cuh -- discrete adjoint of the explicit stage (no hom3
// counterpart: hom3 has no adjoint).
//
// A stage maps q -> q + k R(q), k = dt / h per cell, R the num_flux sum of
// face fluxes (solver.hpp:440-460).  Its vector-Jacobian product for a
// cotangent lambda is gathered per cell: every face (L, R) of the cell adds
// w^T dF/dq_cell with w = k_R' lambda_R - k_L' lambda_L (the face enters the
// left residual with a minus sign, the right one with a plus; k' carries the
// 2^-(nd-1) area weight on the coarse side of a coarse/fine face).  Ghost
// states depend on their boundary cell through the condition (Neumann: I,
// Dirichlet: -I), periodic ghosts are their paired interior cell.  The AUSM
// flux is differentiated by hand in reverse mode; its upwind choice (sign of
// the interface Mach number) and the |M| > 1 branches of the split functions
// are frozen at the forward values.  The time step is frozen too.
#pragma once
#include "fv_kernels.cuh"

#ifndef H3C_ADJ_MINB
#define H3C_ADJ_MINB 2  // resident blocks per SM the adjoint stage is compiled for
#endif

namespace h3c {

// derivatives of the split functions (euler/physics.hpp:297-310), |M| > 1 branches frozen
__device__ __forceinline__ double dm_int(double s, double M) {
  if (fabs(M) > 1.0) return (s * M > 0.0) ? 1.0 : 0.0;
  return s * 0.5 * (M + s);
}
__device__ __forceinline__ double dp_int(double s, double M) {
  if (fabs(M) > 1.0) return 0.0;
  return 0.5 * (M + s) * (2.0 - s * M) - s * 0.25 * (M + s) * (M + s);
}
__device__ __forceinline__ double m_int_d(double s, double M) {
  if (fabs(M) > 1.0) return (s * M > 0.0) ? M : 0.0;
  return (s * 0.25) * ((M + s) * (M + s));
}
__device__ __forceinline__ double p_int_d(double s, double M) {
  if (fabs(M) > 1.0) return (s * M > 0.0) ? 1.0 : 0.0;
  return (0.25 * ((M + s) * (M + s))) * (2.0 - s * M);
}

// a[d] for a direction d known only at run time, by selects (no local-memory indexing)
template <int N> __device__ __forceinline__ double pick(const double* a, int d) {
  double r = a[0];
#pragma unroll
  for (int k = 1; k < N; ++k) r = d == k ? a[k] : r;
  return r;
}

// primitive state of one side, all directions (Newton reciprocals as in make_prim)
template <int ND> struct SideAD {
  double q[ND + 2];
  double rinv, u[ND], um2, p, a, ainv, M[ND];
};

template <int ND>
__device__ __forceinline__ void side_forward(SideAD<ND>& S, double gamma, double gm1) {
  S.rinv = nr_rcp(S.q[ND]);
  S.um2 = 0.0;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    S.u[k] = S.q[k] * S.rinv;
    S.um2 = k == 0 ? S.u[k] * S.u[k] : S.um2 + S.u[k] * S.u[k];
  }
  S.p = gm1 * (S.q[ND + 1] - 0.5 * S.q[ND] * S.um2);
  const double a2 = gamma * S.p * S.rinv;
  S.ainv = nr_rsqrt(a2);
  S.a = a2 * S.ainv;
#pragma unroll
  for (int k = 0; k < ND; ++k) S.M[k] = S.u[k] * S.ainv;
}

// reverse through p(q), a(q), M_d(q) of one side; adds to g[ND + 2]
template <int ND>
__device__ __forceinline__ void side_reverse(const SideAD<ND>& S, int d, double gamma, double gm1, double Mbar,
                                             double abar, double pbar, double* g) {
  double ubar[ND];
#pragma unroll
  for (int k = 0; k < ND; ++k) ubar[k] = k == d ? Mbar * S.ainv : 0.0;
  abar -= Mbar * pick<ND>(S.M, d) * S.ainv;
  const double a2bar = 0.5 * abar * S.ainv;
  pbar += a2bar * gamma * S.rinv;
  double rinvbar = a2bar * gamma * S.p;
  g[ND + 1] += gm1 * pbar;
  g[ND] -= 0.5 * gm1 * S.um2 * pbar;
  const double um2bar = -0.5 * gm1 * S.q[ND] * pbar;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    ubar[k] += 2.0 * S.u[k] * um2bar;
    g[k] += S.rinv * ubar[k];
    rinvbar += S.q[k] * ubar[k];
  }
  g[ND] -= S.rinv * S.rinv * rinvbar;
}

// gL += w^T dF/dq_L, gR += w^T dF/dq_R for the AUSM flux F(q_L, q_R) along d
template <int ND>
__device__ __forceinline__ void ausm_vjp(const SideAD<ND>& SL, const SideAD<ND>& SR, int d, const double* w,
                                         double gamma, double gm1, double* gL, double* gR) {
  constexpr int NV = ND + 2;
  const double ML = pick<ND>(SL.M, d), MR = pick<ND>(SR.M, d);
  const double mi = m_int_d(1.0, ML) + m_int_d(-1.0, MR);
  const bool left = mi >= 0.0;
  const SideAD<ND>& Su = left ? SL : SR;
  // F_v = mi theta_v + [v == d] pi, theta = a (q_0 .. q_ND, q_E + p) of the upwind side
  double wq = 0.0;
#pragma unroll
  for (int v = 0; v < NV - 1; ++v) wq += w[v] * Su.q[v];
  wq += w[NV - 1] * (Su.q[NV - 1] + Su.p);
  const double mbar = Su.a * wq;
  const double pibar = pick<ND>(w, d);
  const double MLbar = dm_int(1.0, ML) * mbar + dp_int(1.0, ML) * SL.p * pibar;
  const double MRbar = dm_int(-1.0, MR) * mbar + dp_int(-1.0, MR) * SR.p * pibar;
  double pLbar = p_int_d(1.0, ML) * pibar;
  double pRbar = p_int_d(-1.0, MR) * pibar;
  const double abar_u = mi * wq;
  const double am = Su.a * mi;
  double aLbar = 0.0, aRbar = 0.0;
  if (left) {
#pragma unroll
    for (int v = 0; v < NV; ++v) gL[v] += am * w[v];
    pLbar += am * w[NV - 1];
    aLbar = abar_u;
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) gR[v] += am * w[v];
    pRbar += am * w[NV - 1];
    aRbar = abar_u;
  }
  side_reverse<ND>(SL, d, gamma, gm1, MLbar, aLbar, pLbar, gL);
  side_reverse<ND>(SR, d, gamma, gm1, MRbar, aRbar, pRbar, gR);
}

// gL += w^T dF/dq_L, gR += w^T dF/dq_R for the local Lax-Friedrichs flux
// F = 1/2 (f(q_L) + f(q_R) + dx/dt (q_L - q_R)) along d (euler/physics.hpp:
// 98-113, 262-267).  The physical flux f is differentiated exactly; the
// dissipation term's cotangent wdiss = 1/2 sum over the two residuals of
// (dx/dt of the cell that evaluated the face) x (its part of w) is passed in,
// since each cell evaluates its faces with its own length.
template <int ND>
__device__ __forceinline__ void euler_flux_vjp(const SideAD<ND>& S, int d, const double* w, double gm1, double gamma,
                                               double* g) {
  // f_k = m_d u_k + p [k == d], f_rho = m_d, f_E = u_d (E + p)
  const double ud = pick<ND>(S.u, d);
  const double H = (S.q[ND + 1] + S.p) * S.rinv;
  const double wd = pick<ND>(w, d);
  double wu = 0.0;  // sum_k w_k u_k
#pragma unroll
  for (int k = 0; k < ND; ++k) wu += w[k] * S.u[k];
  const double wpm = wd + w[ND + 1] * ud;  // cotangent of p through f_d and f_E
#pragma unroll
  for (int j = 0; j < ND; ++j) {
    double gj = ud * w[j] - gm1 * S.u[j] * wpm;  // u_d w_j + dp/dm_j (w_d + w_E u_d)
    if (j == d) gj += wu + w[ND] + w[ND + 1] * H;
    g[j] += gj;
  }
  g[ND] += -ud * wu + 0.5 * gm1 * S.um2 * wpm - w[ND + 1] * ud * H;
  g[ND + 1] += gm1 * wd + gamma * ud * w[ND + 1];
}

template <int ND>
__device__ __forceinline__ void llf_vjp(const SideAD<ND>& SL, const SideAD<ND>& SR, int d, const double* w,
                                        const double* wdiss, double gamma, double gm1, double* gL, double* gR) {
  constexpr int NV = ND + 2;
  double hw[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) hw[v] = 0.5 * w[v];
  euler_flux_vjp<ND>(SL, d, hw, gm1, gamma, gL);
  euler_flux_vjp<ND>(SR, d, hw, gm1, gamma, gR);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    gL[v] += wdiss[v];
    gR[v] -= wdiss[v];
  }
}

// Per-cell adjoint of one stage:
//   gout_c = beta lam_c + [VJP of (q -> alpha k R(q)) with cotangent lam]_c
//            + gamma_e extra_c + gamma_e2 extra2_c
// q is the stage input with its ghosts filled by the conditions.
template <int ND, int PHYS, int FLUX = AUSM>
__global__ void __launch_bounds__(kBlock, H3C_ADJ_MINB) k_adj_stage(const double* __restrict__ q, const double* __restrict__ lam,
                                                      double* __restrict__ gout, const double* __restrict__ extra,
                                                      const double* __restrict__ extra2, double alpha, double beta,
                                                      double gamma_e, double gamma_e2, double* __restrict__ xbar,
                                                      Geometry g,
                                                      GhostTables gt, PhysConst pc, const Scalars* __restrict__ sc) {
  constexpr int NV = nvars<ND, PHYS>();
  constexpr int NS = 1 << (ND - 1);
  constexpr double W = ND == 2 ? 0.5 : 0.25;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n_int) return;
  const long long ld = g.ld;
  const double dt = sc->dt;
  const double hc = g.len[g.lvl[c]];
  const double kc = alpha * dt / hc;
  double lc[NV], acc[NV];
  SideAD<ND> Sc;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    lc[v] = lam[v * ld + c];
    acc[v] = 0.0;
  }
  if (PHYS == HEAT) {
    Sc.q[0] = q[c];
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) Sc.q[v] = q[v * ld + c];
    side_forward<ND>(Sc, pc.gamma, pc.gm1);
  }
  // resolve a neighbour entry: interior cell (its own residual) or ghost (condition Jacobian)
  // returns the residual-owning cell for the cotangent and the Jacobian sign of the ghost
  auto face = [&](int nb_cell, bool c_is_left, double kc_face, double kn_face, int d) {
    // nb_cell: neighbour index (interior or ghost)
    double w[NV];
    double jac = 0.0;  // ghost: dq_ghost/dq_c = jac I; interior: 0
    double xjac = 0.0;  // conjugate heat ghost: dT_ghost / dT_partner
    long long gi = -1;
    long long own = nb_cell;
    double kn = kn_face;
    if (nb_cell >= g.n_int) {
      const long long i = nb_cell - g.n_int;
      const int b = gt.bc_apply[i];
      own = -1;
      kn = 0.0;
      if (b != 255) {
        const int kind = gt.bcs[b].kind;
        if (kind == BC_PERIODIC) {
          // the ghost is a copy of its paired cell, whose residual holds the same face
          own = gt.partner[i];
          if (own >= 0) kn = alpha * dt / g.len[g.lvl[own]];
        } else if (kind == BC_CPL_HEAT_CNS || kind == BC_CPL_HEAT_HEAT) {
          // T_g = 2 T_s - T_b, T_s = (T_other + kappa T_b) / (1 + kappa) (kappa = 1: the mean)
          const double kap0 = kind == BC_CPL_HEAT_CNS ? gt.bcs[b].v[0] : 1.0;
          const double kap = kap0 == 0.0 ? 1.0 : kap0;
          jac = 2.0 * kap / (1.0 + kap) - 1.0;
          xjac = 2.0 / (1.0 + kap);
          gi = i;
        } else {
          jac = (kind == BC_EULER_DIRICHLET || kind == BC_HEAT_DIRICHLET) ? -1.0 : 1.0;
        }
      }
    }
    double ln[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) ln[v] = own >= 0 ? lam[v * ld + own] : 0.0;
    // w = k_R lambda_R - k_L lambda_L
#pragma unroll
    for (int v = 0; v < NV; ++v) w[v] = c_is_left ? (kn * ln[v] - kc_face * lc[v]) : (kc_face * lc[v] - kn * ln[v]);
    double gc[NV], gn[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) { gc[v] = 0.0; gn[v] = 0.0; }
    if (PHYS == HEAT) {
      // F = (T_L - T_R) / dx_owner (heat/physics.hpp:113-119): the two residuals use their own dx
      const double hn = own >= 0 ? g.len[g.lvl[own]] : hc;
      const double wl = c_is_left ? -kc_face * lc[0] / hc : kc_face * lc[0] / hc;  // c's residual term
      const double wn = own >= 0 ? (c_is_left ? kn * ln[0] / hn : -kn * ln[0] / hn) : 0.0;
      // d/dT_c of (+-F): c is L -> +1, c is R -> -1 ; ghost chain: d/dT_g -> opposite sign times jac
      const double sgn = c_is_left ? 1.0 : -1.0;
      gc[0] = (wl + wn) * sgn;
      if (own < 0) gc[0] += wl * (-sgn) * jac;
      if (gi >= 0 && xbar) xbar[gi] = wl * (-sgn) * xjac;  // cotangent of the partner temperature
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] += gc[v];
      return;
    }
    SideAD<ND> Sn;
#pragma unroll
    for (int v = 0; v < NV; ++v) Sn.q[v] = q[v * ld + nb_cell];
    side_forward<ND>(Sn, pc.gamma, pc.gm1);
    if (FLUX == LLF) {
      // c's residual evaluates the face with dx_c / dt, the neighbour's with its own length
      const double cdx = hc / dt, ndx = own >= 0 ? g.len[g.lvl[own]] / dt : 0.0;
      double wdiss[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double wc = c_is_left ? -kc_face * lc[v] : kc_face * lc[v];
        const double wn = c_is_left ? kn * ln[v] : -kn * ln[v];
        wdiss[v] = 0.5 * (cdx * wc + ndx * wn);
      }
      if (c_is_left) llf_vjp<ND>(Sc, Sn, d, w, wdiss, pc.gamma, pc.gm1, gc, gn);
      else llf_vjp<ND>(Sn, Sc, d, w, wdiss, pc.gamma, pc.gm1, gn, gc);
    } else if (c_is_left) {
      ausm_vjp<ND>(Sc, Sn, d, w, pc.gamma, pc.gm1, gc, gn);
    } else {
      ausm_vjp<ND>(Sn, Sc, d, w, pc.gamma, pc.gm1, gn, gc);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] += gc[v] + jac * gn[v];
  };
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const int m = g.nbr[(2 * d) * ld + c];
    const int p = g.nbr[(2 * d + 1) * ld + c];
    // minus side: c is the right cell of F(m, c)
    if (m >= 0) {
      const bool coarser = m < g.n_int && g.len[g.lvl[m]] > hc;
      const double km = m < g.n_int ? alpha * dt / g.len[g.lvl[m]] : 0.0;
      face(m, false, kc, coarser ? W * km : km, d);
    } else {
      const long long k = -m - 2;
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        const int f = g.sub[j * g.nsub + k];
        face(f, false, W * kc, alpha * dt / g.len[g.lvl[f]], d);
      }
    }
    // plus side: c is the left cell of F(c, p)
    if (p >= 0) {
      const bool coarser = p < g.n_int && g.len[g.lvl[p]] > hc;
      const double kp = p < g.n_int ? alpha * dt / g.len[g.lvl[p]] : 0.0;
      face(p, true, kc, coarser ? W * kp : kp, d);
    } else {
      const long long k = -p - 2;
#pragma unroll
      for (int j = 0; j < NS; ++j) {
        const int f = g.sub[j * g.nsub + k];
        face(f, true, W * kc, alpha * dt / g.len[g.lvl[f]], d);
      }
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double o = beta * lc[v] + acc[v];
    if (extra) o += gamma_e * extra[v * ld + c];
    if (extra2) o += gamma_e2 * extra2[v * ld + c];
    gout[v * ld + c] = o;
  }
}

// ---------------------------------------------------------------------------
// Euler adjoint stage on the forward's Morton tiles.  The per-cell gather
// above evaluates the reverse of every face twice, once from each side, and
// its warps diverge between in-tile, border, ghost and coarse/fine faces.
// Here every cell publishes its primitive side state and its weighted
// cotangent k lambda in shared memory, then
//   (1) every cell reverses its plus faces (one uniform call per direction:
//       the neighbour comes from shared memory in the tile, else from global
//       memory or its ghost condition) and, where the right cell is in the
//       tile and points back (same level), stores that cell's half in the
//       cell's minus-face slot;
//   (2) the minus faces left over (tile border, ghost, coarse/fine) are
//       compacted into a list that the block's threads work through;
//   (3) every cell sums its plus faces and its minus-face slots in a fixed
//       order: the result is deterministic.
// Same result as k_adj_stage<ND, EULER> up to the order of the face sums.
// Shared memory: side state [ND + 6][kBlock] (q, 1/rho, p, a, 1/a), k lambda
// [ND + 2][kBlock], minus-face slots [ND][ND + 2][kBlock] of double, plus and
// minus neighbours [2][ND][kBlock] of int, the work list [ND kBlock] of
// ushort and the scan's warp totals.
// ---------------------------------------------------------------------------
template <int ND> __host__ __device__ constexpr size_t adj_ausm_smem_bytes() {
  return sizeof(double) * ((ND + 6) + (ND + 2) + ND * (ND + 2)) * kBlock + sizeof(int) * 2 * ND * kBlock +
         sizeof(unsigned short) * ND * kBlock + sizeof(int) * (kBlock / 32 + 1);
}

// side state of a cell from its published q, 1/rho, p, a, 1/a (the operations of side_forward)
template <int ND> __device__ __forceinline__ void side_from_shared(SideAD<ND>& S, const double* ss, int t) {
  constexpr int NV = ND + 2;
#pragma unroll
  for (int v = 0; v < NV; ++v) S.q[v] = ss[v * kBlock + t];
  S.rinv = ss[NV * kBlock + t];
  S.p = ss[(NV + 1) * kBlock + t];
  S.a = ss[(NV + 2) * kBlock + t];
  S.ainv = ss[(NV + 3) * kBlock + t];
  S.um2 = 0.0;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    S.u[k] = S.q[k] * S.rinv;
    S.um2 = k == 0 ? S.u[k] * S.u[k] : S.um2 + S.u[k] * S.u[k];
  }
#pragma unroll
  for (int k = 0; k < ND; ++k) S.M[k] = S.u[k] * S.ainv;
}

// Neighbour nb of a face read from global memory: its side state, the
// weighted cotangent kn lambda of the cell whose residual holds the face on
// its side (0 for a ghost, the paired cell for a periodic ghost) and the
// ghost's condition Jacobian dq_ghost / dq_c = jac I (0 for interior cells).
template <int ND>
__device__ __forceinline__ void adj_neighbour(int nb, double kn_face, const double* __restrict__ q,
                                              const double* __restrict__ lam, double alpha, double dt,
                                              const Geometry& g, const GhostTables& gt, const PhysConst& pc,
                                              SideAD<ND>& Sn, double* kln, double& jac) {
  constexpr int NV = ND + 2;
  const long long ld = g.ld;
  jac = 0.0;
  long long own = nb;
  double kn = kn_face;
  if (nb >= g.n_int) {
    const long long i = nb - g.n_int;
    const int b = gt.bc_apply[i];
    own = -1;
    kn = 0.0;
    if (b != 255) {
      const int kind = gt.bcs[b].kind;
      if (kind == BC_PERIODIC) {
        own = gt.partner[i];
        if (own >= 0) kn = alpha * dt / g.len[g.lvl[own]];
      } else {
        jac = kind == BC_EULER_DIRICHLET ? -1.0 : 1.0;
      }
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    Sn.q[v] = __ldg(q + v * ld + nb);
    kln[v] = own >= 0 ? kn * __ldg(lam + v * ld + own) : 0.0;
  }
  side_forward<ND>(Sn, pc.gamma, pc.gm1);
}

#ifndef H3C_ADJT_MINB
#define H3C_ADJT_MINB 2  // resident blocks per SM the tile adjoint is compiled for
#endif
// gout_c = beta lam_c + [VJP of (q -> alpha k R(q)) with cotangent lam]_c + gamma_e extra_c + gamma_e2 extra2_c
template <int ND, bool HANG>
__global__ void __launch_bounds__(kBlock, H3C_ADJT_MINB)
    k_adj_ausm(const double* __restrict__ q, const double* __restrict__ lam, double* __restrict__ gout,
               const double* __restrict__ extra, const double* __restrict__ extra2, double alpha, double beta,
               double gamma_e, double gamma_e2, Geometry g, GhostTables gt, PhysConst pc,
               const Scalars* __restrict__ sc) {
  constexpr int NV = ND + 2;
  constexpr int NS = 1 << (ND - 1);
  constexpr double W = ND == 2 ? 0.5 : 0.25;
  constexpr int NW = kBlock / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* ss = reinterpret_cast<double*>(smem_raw);  // [ND + 6][kBlock]
  double* skl = ss + (ND + 6) * kBlock;              // [NV][kBlock]
  double* sg = skl + NV * kBlock;                    // [ND][NV][kBlock] minus-face slots
  int* snp = reinterpret_cast<int*>(sg + ND * NV * kBlock);  // [ND][kBlock]
  int* snm = snp + ND * kBlock;                               // [ND][kBlock]
  unsigned short* sitem = reinterpret_cast<unsigned short*>(snm + ND * kBlock);  // [ND kBlock]
  int* swarp = reinterpret_cast<int*>(sitem + ND * kBlock);                      // [NW + 1]
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const long long ld = g.ld;
  const long long c0 = (long long)blockIdx.x * kBlock;
  const long long c = c0 + tid;
  const long long tile_end = min(c0 + (long long)kBlock, g.n_int);
  const bool live = c < tile_end;
  const double dt = sc->dt;
  auto in_tile = [&](long long n) { return n >= c0 && n < tile_end; };

  // ---- own loads, side state and k lambda -> shared memory ----
  double hc = 1.0, kc = 0.0;
  SideAD<ND> Sc;
  if (live) {
#pragma unroll
    for (int v = 0; v < NV; ++v) Sc.q[v] = __ldg(q + v * ld + c);
    hc = g.len[g.lvl[c]];
    kc = alpha * dt / hc;
    side_forward<ND>(Sc, pc.gamma, pc.gm1);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      ss[v * kBlock + tid] = Sc.q[v];
      skl[v * kBlock + tid] = kc * __ldg(lam + v * ld + c);
    }
    ss[NV * kBlock + tid] = Sc.rinv;
    ss[(NV + 1) * kBlock + tid] = Sc.p;
    ss[(NV + 2) * kBlock + tid] = Sc.a;
    ss[(NV + 3) * kBlock + tid] = Sc.ainv;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      snm[d * kBlock + tid] = __ldg(g.nbr + (2 * d) * ld + c);
      snp[d * kBlock + tid] = __ldg(g.nbr + (2 * d + 1) * ld + c);
    }
  }
  __syncthreads();

  // ---- (1) plus faces: c is the left cell of F(c, p) ----
  double acc[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) acc[v] = 0.0;
  if (live) {
#pragma unroll 1
    for (int d = 0; d < ND; ++d) {
      const int p = snp[d * kBlock + tid];
      double gc[NV], gn[NV], w[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) { gc[v] = 0.0; gn[v] = 0.0; }
      if (HANG && p < 0) {
        // c is the coarse cell of a coarse/fine face: its residual takes W times each sub-face
        const long long k = -p - 2;
#pragma unroll 1
        for (int j = 0; j < NS; ++j) {
          const int f = __ldg(g.sub + j * g.nsub + k);
          SideAD<ND> Sn;
          double jac;
          adj_neighbour<ND>(f, alpha * dt / g.len[g.lvl[f]], q, lam, alpha, dt, g, gt, pc, Sn, w, jac);
#pragma unroll
          for (int v = 0; v < NV; ++v) w[v] = w[v] - W * skl[v * kBlock + tid];
          ausm_vjp<ND>(Sc, Sn, d, w, pc.gamma, pc.gm1, gc, gn);
        }
      } else {
        SideAD<ND> Sn;
        double jac = 0.0;
        bool give = false;
        int t = 0;
        if (in_tile(p)) {
          t = (int)(p - c0);
          side_from_shared<ND>(Sn, ss, t);
          give = snm[d * kBlock + t] == (int)c;
          // not pointing back: p is the coarse cell of a coarse/fine face
          const double f = give ? 1.0 : (g.len[g.lvl[p]] > hc ? W : 1.0);
#pragma unroll
          for (int v = 0; v < NV; ++v) w[v] = f * skl[v * kBlock + t];
        } else {
          const bool coarser = p < g.n_int && g.len[g.lvl[p]] > hc;
          const double kp = p < g.n_int ? alpha * dt / g.len[g.lvl[p]] : 0.0;
          adj_neighbour<ND>(p, coarser ? W * kp : kp, q, lam, alpha, dt, g, gt, pc, Sn, w, jac);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) w[v] = w[v] - skl[v * kBlock + tid];
        ausm_vjp<ND>(Sc, Sn, d, w, pc.gamma, pc.gm1, gc, gn);
#pragma unroll
        for (int v = 0; v < NV; ++v) gc[v] += jac * gn[v];
        if (give) {
#pragma unroll
          for (int v = 0; v < NV; ++v) sg[(d * NV + v) * kBlock + t] = gn[v];
        }
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] += gc[v];
    }
  }

  // ---- (2) minus faces no in-tile left cell covers -> work list ----
  int need = 0;
  if (live) {
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const int m = snm[d * kBlock + tid];
      const bool covered = in_tile(m) && snp[d * kBlock + (int)(m - c0)] == (int)c;
      if (!covered) need |= 1 << d;
    }
  }
  int cnt = __popc(need), incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) swarp[wid] = incl;
  __syncthreads();
  if (tid == 0) {
    int run = 0;
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      const int x = swarp[k];
      swarp[k] = run;
      run += x;
    }
    swarp[NW] = run;
  }
  __syncthreads();
  {
    int pos = swarp[wid] + incl - cnt;
#pragma unroll
    for (int d = 0; d < ND; ++d)
      if (need & (1 << d)) sitem[pos++] = (unsigned short)((tid << 2) | d);
  }
  const int total = swarp[NW];
  __syncthreads();
  for (int k = tid; k < total; k += kBlock) {
    const int it = sitem[k];
    const int t = it >> 2, d = it & 3;
    const long long cc = c0 + t;
    const int m = snm[d * kBlock + t];
    const double hx = g.len[g.lvl[cc]];
    SideAD<ND> Sx;
    side_from_shared<ND>(Sx, ss, t);
    double gx[NV], gn[NV], w[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) { gx[v] = 0.0; gn[v] = 0.0; }
    if (HANG && m < 0) {
      const long long k2 = -m - 2;
#pragma unroll 1
      for (int j = 0; j < NS; ++j) {
        const int f = __ldg(g.sub + j * g.nsub + k2);
        SideAD<ND> Sn;
        double jac;
        adj_neighbour<ND>(f, alpha * dt / g.len[g.lvl[f]], q, lam, alpha, dt, g, gt, pc, Sn, w, jac);
#pragma unroll
        for (int v = 0; v < NV; ++v) w[v] = W * skl[v * kBlock + t] - w[v];
        ausm_vjp<ND>(Sn, Sx, d, w, pc.gamma, pc.gm1, gn, gx);
      }
    } else {
      const bool coarser = m < g.n_int && g.len[g.lvl[m]] > hx;
      const double km = m < g.n_int ? alpha * dt / g.len[g.lvl[m]] : 0.0;
      SideAD<ND> Sn;
      double jac;
      adj_neighbour<ND>(m, coarser ? W * km : km, q, lam, alpha, dt, g, gt, pc, Sn, w, jac);
#pragma unroll
      for (int v = 0; v < NV; ++v) w[v] = skl[v * kBlock + t] - w[v];
      ausm_vjp<ND>(Sn, Sx, d, w, pc.gamma, pc.gm1, gn, gx);
#pragma unroll
      for (int v = 0; v < NV; ++v) gx[v] += jac * gn[v];
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) sg[(d * NV + v) * kBlock + t] = gx[v];
  }
  __syncthreads();

  // ---- (3) sum: plus faces, then the minus-face slots ----
  if (live) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double o = beta * __ldg(lam + v * ld + c) + acc[v];
#pragma unroll
      for (int d = 0; d < ND; ++d) o += sg[(d * NV + v) * kBlock + tid];
      if (extra) o += gamma_e * extra[v * ld + c];
      if (extra2) o += gamma_e2 * extra2[v * ld + c];
      gout[v * ld + c] = o;
    }
  }
}

// frozen time step of step i
__global__ void k_set_dt_from(Scalars* sc, const double* dts, long long i) { sc->dt = dts[i]; }
__global__ void k_record_dt(const Scalars* sc, double* dts, long long i) { dts[i] = sc->dt; }

}  // namespace h3c
