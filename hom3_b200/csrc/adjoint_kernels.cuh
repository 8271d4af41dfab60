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
  abar -= Mbar * S.M[d] * S.ainv;
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
  const double ML = SL.M[d], MR = SR.M[d];
  const double mi = m_int_d(1.0, ML) + m_int_d(-1.0, MR);
  const bool left = mi >= 0.0;
  const SideAD<ND>& Su = left ? SL : SR;
  // F_v = mi theta_v + [v == d] pi, theta = a (q_0 .. q_ND, q_E + p) of the upwind side
  double wq = 0.0;
#pragma unroll
  for (int v = 0; v < NV - 1; ++v) wq += w[v] * Su.q[v];
  wq += w[NV - 1] * (Su.q[NV - 1] + Su.p);
  const double mbar = Su.a * wq;
  const double pibar = w[d];
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

// Per-cell adjoint of one stage:
//   gout_c = beta lam_c + [VJP of (q -> alpha k R(q)) with cotangent lam]_c
//            + gamma_e extra_c + gamma_e2 extra2_c
// q is the stage input with its ghosts filled by the conditions.
template <int ND, int PHYS>
__global__ void __launch_bounds__(kBlock, H3C_ADJ_MINB) k_adj_stage(const double* __restrict__ q, const double* __restrict__ lam,
                                                      double* __restrict__ gout, const double* __restrict__ extra,
                                                      const double* __restrict__ extra2, double alpha, double beta,
                                                      double gamma_e, double gamma_e2, double* __restrict__ xbar,
                                                      Geometry g,
                                                      GhostTables gt, PhysConst pc, const Scalars* __restrict__ sc) {
  constexpr int NV = PHYS == HEAT ? 1 : ND + 2;
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
    if (c_is_left) ausm_vjp<ND>(Sc, Sn, d, w, pc.gamma, pc.gm1, gc, gn);
    else ausm_vjp<ND>(Sn, Sc, d, w, pc.gamma, pc.gm1, gn, gc);
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

// frozen time step of step i
__global__ void k_set_dt_from(Scalars* sc, const double* dts, long long i) { sc->dt = dts[i]; }
__global__ void k_record_dt(const Scalars* sc, double* dts, long long i) { dts[i] = sc->dt; }

}  // namespace h3c
