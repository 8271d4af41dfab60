// cns_adjoint.cuh -- discrete adjoint of the compressible Navier-Stokes stage
// (AUSM + three-point viscous flux with cell slopes).  No hom3 counterpart.
//
// The face flux F(q_L, q_R, s_L, s_R) (s: the cells' slopes in the directions
// across the face) is differentiated in forward mode with DN<kAdjDirs> dual
// numbers run through the library's own make_prim / ausm / viscous
// templates, a few directions per pass, and contracted with the face weight
// w = k_R lambda_R - k_L lambda_L.  Ghost states are differentiated the same
// way through cns_ghost (the formulas of k_bc's CNS branch).  The AUSM
// upwind / |M| > 1 branches are frozen at the forward values.  The face
// direction is a template constant in every dual evaluation: with a run-time
// direction, the dual viscous flux's indexing of its velocity-gradient array
// came out wrong in this build (values right, derivatives not), while the
// same code with the direction known at compile time differentiates exactly.
//
//  k_adjc_face    per cell: own-side cotangents of the state and of the slopes;
//                 non-periodic ghost sides through the ghost Jacobian.  By
//                 default the face flux is reversed by hand (ausm_vjp +
//                 viscous_vjp: one forward and one reverse sweep per face);
//                 the dual-number evaluation stays as a cross-check.
//  k_adjc_slopes  per cell: the slope stencils (central differences) gathered
//                 from the neighbours, ghosts through their Jacobian; writes
//                 beta lam + VJP + extras.
#pragma once
#include "dual.cuh"
#include "muscl_adjoint.cuh"  // stencil_owner

namespace h3c {

#ifndef H3C_ADJ_DIRS
#define H3C_ADJ_DIRS 2  // measured fastest on the 512 x 128 fluid: fewer registers spill
#endif
constexpr int kAdjDirs = H3C_ADJ_DIRS;  // dual directions per pass

template <int K> __device__ __forceinline__ DN<K> nr_rcp(const DN<K>& a) {
  DN<K> r(nr_rcp(a.v));
  const double s = -r.v * r.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * s;
  return r;
}
template <int K> __device__ __forceinline__ DN<K> nr_rsqrt(const DN<K>& a) {
  DN<K> r(nr_rsqrt(a.v));
  const double s = -0.5 * r.v * r.v * r.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * s;
  return r;
}

// Ghost state of a condition from its boundary cell's state qb (and, for a
// conjugate wall, the solid's temperature Tsol): the formulas of k_bc for
// EULER_NEUMANN / EULER_DIRICHLET and the CNS conditions.  Forward Euler: the
// fluid temperature of the conjugate wall is read from qb (lhs).
template <class T, int ND>
__device__ __forceinline__ void cns_ghost(const T* qb, const BcParam& B, int ndir, double gdx, T Tsol,
                                          const PhysConst& pc, T* out) {
  constexpr int NV = ND + 2;
  if (B.kind == BC_EULER_NEUMANN) {
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = qb[v] - gdx * B.v[v];
    return;
  }
  if (B.kind == BC_EULER_DIRICHLET) {
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = 2.0 * B.v[v] - qb[v];
    return;
  }
  const double gamma = pc.gamma;
  T bp[NV], gp[NV];
  bp[ND] = qb[ND];
  T vm2(0.0);
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    bp[d] = qb[d] / qb[ND];
    vm2 = d == 0 ? bp[d] * bp[d] : vm2 + bp[d] * bp[d];
  }
  bp[ND + 1] = (gamma - 1.0) * (qb[ND + 1] - 0.5 * qb[ND] * vm2);
#pragma unroll
  for (int v = 0; v < NV; ++v) gp[v] = bp[v];
  if (B.kind == BC_CNS_INFLOW) {
#pragma unroll
    for (int d = 0; d < ND; ++d) gp[d] = 2.0 * B.v[d] - bp[d];
    gp[ND] = 2.0 * B.v[ND] - bp[ND];
  } else if (B.kind == BC_CNS_OUTFLOW) {
    gp[ND + 1] = 2.0 * B.v[ND + 1] - bp[ND + 1];
  } else if (B.kind == BC_CNS_ADIABATIC_NOSLIP) {
#pragma unroll
    for (int d = 0; d < ND; ++d) gp[d] = 0.0 - bp[d];
  } else if (B.kind == BC_CNS_ADIABATIC_SLIP) {
#pragma unroll
    for (int d = 0; d < ND; ++d)
      if (d == ndir) gp[d] = 0.0 - bp[d];
  } else if (B.kind == BC_CNS_ISOTHERMAL_NOSLIP || B.kind == BC_CPL_CNS_HEAT) {
    T Ts(B.v[0]);
    if (B.kind == BC_CPL_CNS_HEAT) {
      T um2(0.0);
#pragma unroll
      for (int d = 0; d < ND; ++d) {
        const T u = qb[d] / qb[ND];
        um2 = d == 0 ? u * u : um2 + u * u;
      }
      const T pf = pc.gm1 * (qb[ND + 1] - 0.5 * qb[ND] * um2);
      const T Tf = gamma * pf / qb[ND];
      const double kap = B.v[0];
      Ts = (kap == 0.0 || kap == 1.0) ? 0.5 * (Tf + Tsol) : (Tf + kap * Tsol) / (1.0 + kap);
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) gp[d] = 0.0 - bp[d];
    const T rho_srfc = bp[ND + 1] * gamma / Ts;
    gp[ND] = 2.0 * rho_srfc - bp[ND];
  }
  out[ND] = gp[ND];
  T gm2(0.0);
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    out[d] = gp[ND] * gp[d];
    gm2 = d == 0 ? gp[d] * gp[d] : gm2 + gp[d] * gp[d];
  }
  out[ND + 1] = gp[ND + 1] / (gamma - 1.0) + 0.5 * gp[ND] * gm2;
}

// qbar_b += (dq_g/dq_b)^T gbar; returns (dq_g/dTsol)^T gbar (conjugate walls)
template <int ND>
__device__ __forceinline__ double ghost_vjp(const double* qb, const BcParam& B, int ndir, double gdx, double Tsol,
                                            const PhysConst& pc, const double* gbar, double* qbar_b) {
  constexpr int NV = ND + 2;
  DN<NV + 1> x[NV], T, out[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    x[v] = DN<NV + 1>(qb[v]);
    x[v].d[v] = 1.0;
  }
  T = DN<NV + 1>(Tsol);
  T.d[NV] = 1.0;
  cns_ghost<DN<NV + 1>, ND>(x, B, ndir, gdx, T, pc, out);
  double tb = 0.0;
#pragma unroll
  for (int u = 0; u < NV; ++u) {
#pragma unroll
    for (int v = 0; v < NV; ++v) qbar_b[v] += gbar[u] * out[u].d[v];
    tb += gbar[u] * out[u].d[NV];
  }
  return tb;
}

// the CNS face flux (AUSM + viscous) of face (L, R) along D on dual numbers
template <int ND, int K, int D>
__device__ __forceinline__ void cns_face_dual(const DN<K>* qL, const DN<K>* qR, const DN<K>* sL, const DN<K>* sR,
                                              double len_r, const PhysConst& pc, DN<K>* f) {
  constexpr int NV = ND + 2;
  const DN<K> gamma(pc.gamma), gm1(pc.gm1);
  Prim<DN<K>, ND> PL, PR;
#pragma unroll
  for (int v = 0; v < NV; ++v) { PL.q[v] = qL[v]; PR.q[v] = qR[v]; }
  make_prim<DN<K>, ND>(PL, gamma, gm1);
  make_prim<DN<K>, ND>(PR, gamma, gm1);
  ausm<DN<K>, ND>(PL, PR, D, f);
  DN<K> fv[NV];
  viscous<DN<K>, ND>(PL, PR, sL, sR, D, DN<K>(len_r), pc, fv);
#pragma unroll
  for (int v = 0; v < NV; ++v) f[v] = f[v] + fv[v];
}

// Reverse of the three-point viscous flux of face (L, R) along D
// (viscous(): cns/physics.hpp:305-338 with surface_slope, solver.hpp:656-678):
// for the cotangent w of F, adds w^T dF/dq to gL, gR (the pressures' share
// through side_reverse) and w^T dF/ds to sLb, sRb for the transverse slopes
// the flux reads (sd != D).  Every quotient and Sutherland's law
// (cns/quantities.hpp:113-115) are differentiated exactly; the divisors'
// reciprocals are taken once (nr_rcp / nr_rsqrt), as the forward flux does.
template <int ND, int D>
__device__ __forceinline__ void viscous_vjp(const SideAD<ND>& L, const SideAD<ND>& R, const double* sL,
                                            const double* sR, double len_r, const PhysConst& pc, const double* w,
                                            double* gL, double* gR, double* sLb, double* sRb) {
  constexpr int NV = ND + 2;
  const double gamma = pc.gamma, gm1 = pc.gm1;
  // ---- forward ----
  const double rho_s = 0.5 * (L.q[ND] + R.q[ND]);
  const double rinv = nr_rcp(rho_s), rinv2 = rinv * rinv;
  const double ilen = nr_rcp(len_r);
  double rus[ND], us[ND];
  double umag2 = 0.0;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    rus[k] = 0.5 * (L.q[k] + R.q[k]);
    us[k] = rus[k] * rinv;
    umag2 = k == 0 ? us[k] * us[k] : umag2 + us[k] * us[k];
  }
  const double rEs = 0.5 * (L.q[ND + 1] + R.q[ND + 1]);
  const double p_s = gm1 * (rEs - 0.5 * rho_s * umag2);
  double G[NV][ND];  // G[v][sd]: the surface derivative gs(v, sd)
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int sd = 0; sd < ND; ++sd)
      G[v][sd] = sd == D ? (R.q[v] - L.q[v]) * ilen : 0.5 * (sR[sd * NV + v] + sL[sd * NV + v]);
  double gu[ND][ND];
#pragma unroll
  for (int c = 0; c < ND; ++c)
#pragma unroll
    for (int sd = 0; sd < ND; ++sd) gu[c][sd] = (G[c][sd] * rho_s - G[ND][sd] * rus[c]) * rinv2;
  const double p_avg = 0.5 * (L.p + R.p);
  const double T = gamma * p_avg * rinv;
  const double iTS = nr_rcp(T + pc.sOverTref);
  const double mu = (T * (T * nr_rsqrt(T))) * pc.sOverTrefP1 * iTS;
  const double cA = gamma / (gm1 * pc.Pr0);
  const double A = -mu * cA * rinv;  // qf = A (gradP - p_s / rho_s gradRho)
  double grum = G[ND][D] * umag2;
#pragma unroll
  for (int k = 0; k < ND; ++k) grum = grum + rho_s * 2.0 * us[k] * gu[k][D];
  const double gradP = gm1 * (G[ND + 1][D] - 0.5 * grum);
  const double gradRho = G[ND][D];
  const double Bv = gradP - p_s * rinv * gradRho;
  double tr = gu[0][0];
#pragma unroll
  for (int i = 1; i < ND; ++i) tr = tr + gu[i][i];
  const double divu = tr * (2.0 / 3.0);
  const double invRe = 1.0 / pc.Re0;
  double t[ND];
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    t[k] = gu[D][k] + gu[k][D];
    if (k == D) t[k] = t[k] - divu;
  }
  // ---- reverse ----
  const double Eaccb = invRe * w[ND + 1];  // f_E = invRe (sum_k u_k tau_kd + qf)
  const double qfb = invRe * w[ND + 1];
  double usb[ND], rusb[ND], gub[ND][ND], Gb[NV][ND];
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    usb[k] = 0.0;
    rusb[k] = 0.0;
#pragma unroll
    for (int j = 0; j < ND; ++j) gub[k][j] = 0.0;
  }
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int sd = 0; sd < ND; ++sd) Gb[v][sd] = 0.0;
  double mub = 0.0, rho_sb = 0.0, divb = 0.0;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    const double tkd = -mu * t[k];
    const double tkdb = invRe * w[k] + us[k] * Eaccb;
    usb[k] += tkd * Eaccb;
    mub += -t[k] * tkdb;
    const double tb = -mu * tkdb;
    gub[D][k] += tb;
    gub[k][D] += tb;
    if (k == D) divb -= tb;
  }
  const double trb = divb * (2.0 / 3.0);
#pragma unroll
  for (int i = 0; i < ND; ++i) gub[i][i] += trb;
  // qf = A Bv
  const double Ab = qfb * Bv, Bb = qfb * A;
  mub += Ab * (-cA * rinv);
  rho_sb += Ab * (mu * cA * rinv2);
  const double gradPb = Bb;
  const double p_sb = -Bb * gradRho * rinv;
  Gb[ND][D] += -Bb * p_s * rinv;
  rho_sb += Bb * p_s * gradRho * rinv2;
  Gb[ND + 1][D] += gm1 * gradPb;
  const double grumb = -0.5 * gm1 * gradPb;
  Gb[ND][D] += grumb * umag2;
  double umag2b = grumb * G[ND][D];
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    rho_sb += grumb * 2.0 * us[k] * gu[k][D];
    usb[k] += grumb * 2.0 * rho_s * gu[k][D];
    gub[k][D] += grumb * 2.0 * rho_s * us[k];
  }
  // mu(T) = T^1.5 (1 + S) / (T + S): dmu/dT = mu (1.5 / T - 1 / (T + S))
  const double Tb = mub * mu * (1.5 * nr_rcp(T) - iTS);
  const double p_avgb = Tb * gamma * rinv;
  rho_sb -= Tb * T * rinv;
  // gu = (G rho_s - G_rho rus) / rho_s^2
#pragma unroll
  for (int c = 0; c < ND; ++c)
#pragma unroll
    for (int sd = 0; sd < ND; ++sd) {
      const double gq = gub[c][sd] * rinv2;
      Gb[c][sd] += gq * rho_s;
      Gb[ND][sd] -= gq * rus[c];
      rusb[c] -= gq * G[ND][sd];
      rho_sb += gq * G[c][sd] - 2.0 * rho_s * gq * gu[c][sd];
    }
  // G: normal differences of the states, transverse means of the slopes
#pragma unroll
  for (int v = 0; v < NV; ++v)
#pragma unroll
    for (int sd = 0; sd < ND; ++sd) {
      if (sd == D) {
        gR[v] += Gb[v][sd] * ilen;
        gL[v] -= Gb[v][sd] * ilen;
      } else {
        sRb[sd * NV + v] += 0.5 * Gb[v][sd];
        sLb[sd * NV + v] += 0.5 * Gb[v][sd];
      }
    }
  // p_s = gm1 (rEs - rho_s umag2 / 2)
  const double rEsb = gm1 * p_sb;
  rho_sb += -0.5 * gm1 * umag2 * p_sb;
  umag2b += -0.5 * gm1 * rho_s * p_sb;
  gL[ND + 1] += 0.5 * rEsb;
  gR[ND + 1] += 0.5 * rEsb;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    usb[k] += 2.0 * us[k] * umag2b;
    rusb[k] += usb[k] * rinv;
    rho_sb -= usb[k] * us[k] * rinv;
    gL[k] += 0.5 * rusb[k];
    gR[k] += 0.5 * rusb[k];
  }
  gL[ND] += 0.5 * rho_sb;
  gR[ND] += 0.5 * rho_sb;
  // the cells' pressures through make_prim
  side_reverse<ND>(L, D, gamma, gm1, 0.0, 0.0, 0.5 * p_avgb, gL);
  side_reverse<ND>(R, D, gamma, gm1, 0.0, 0.0, 0.5 * p_avgb, gR);
}

// the two faces of cell c along direction D, reversed by hand: AUSM
// (ausm_vjp) plus the viscous flux (viscous_vjp), one forward and one reverse
// sweep per face giving the cotangents of both cells' states and slopes
template <int ND, int D>
__device__ __forceinline__ void adjc_faces_rev(long long c, const double* __restrict__ q, const double* __restrict__ sl,
                                               const double* __restrict__ lam, double alpha, double dt,
                                               const Geometry& g, const GhostTables& gt, const PhysConst& pc,
                                               const double* __restrict__ psol, const SideAD<ND>& Sc,
                                               const double* slc, const double* lc, double hc, double* qb, double* sb,
                                               double* __restrict__ tbar) {
  constexpr int NV = ND + 2;
  const long long ld = g.ld;
  const double kc = alpha * dt / hc;
#pragma unroll 1
  for (int sd2 = 0; sd2 < 2; ++sd2) {
    const int side = sd2 == 0 ? -1 : 1;
    const int n = g.nbr[(2 * D + sd2) * ld + c];
    double jac = 0.0;
    const int own = stencil_owner(g, gt, n, &jac);
    const double kn = own >= 0 ? alpha * dt / g.len[g.lvl[own]] : 0.0;
    double w[NV];
    SideAD<ND> Sn;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double ln = own >= 0 ? lam[v * ld + own] : 0.0;
      w[v] = side > 0 ? (kn * ln - kc * lc[v]) : (kc * lc[v] - kn * ln);
      Sn.q[v] = q[v * ld + n];
    }
    side_forward<ND>(Sn, pc.gamma, pc.gm1);
    double sln[ND * NV];
#pragma unroll
    for (int k = 0; k < ND * NV; ++k) sln[k] = sl[k * ld + n];
    const bool cL = side > 0;  // c is the left cell of the face
    const double len_r = cL ? g.len[g.lvl[n]] : hc;
    double gc[NV], gn[NV], sbc[ND * NV], sbn[ND * NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) gc[v] = gn[v] = 0.0;
#pragma unroll
    for (int k = 0; k < ND * NV; ++k) sbc[k] = sbn[k] = 0.0;
    if (cL) {
      ausm_vjp<ND>(Sc, Sn, D, w, pc.gamma, pc.gm1, gc, gn);
      viscous_vjp<ND, D>(Sc, Sn, slc, sln, len_r, pc, w, gc, gn, sbc, sbn);
    } else {
      ausm_vjp<ND>(Sn, Sc, D, w, pc.gamma, pc.gm1, gn, gc);
      viscous_vjp<ND, D>(Sn, Sc, sln, slc, len_r, pc, w, gn, gc, sbn, sbc);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) qb[v] += gc[v];
#pragma unroll
    for (int k = 0; k < ND * NV; ++k) sb[k] += sbc[k];
    if (own == -1) {  // a non-periodic ghost: its state and slopes come from c
      const long long i = n - g.n_int;
      const BcParam& B = gt.bcs[gt.bc_apply[i]];
      const double Tsol = (B.kind == BC_CPL_CNS_HEAT && psol && gt.partner[i] >= 0) ? psol[gt.partner[i]] : 0.0;
      double qcv[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) qcv[v] = Sc.q[v];
      const double tb = ghost_vjp<ND>(qcv, B, gt.pos[i] >> 1, gt.dx[i], Tsol, pc, gn, qb);
      if (tbar && B.kind == BC_CPL_CNS_HEAT) tbar[i] = tb;
      const BcParam& Bo = gt.bcs[gt.bc_own[i]];
#pragma unroll
      for (int s2 = 0; s2 < ND; ++s2) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const double sign = (Bo.wall && v < ND && s2 != D) ? -1.0 : 1.0;
          sb[s2 * NV + v] += sign * sbn[s2 * NV + v];
        }
      }
    }
  }
}

// the two faces of cell c along direction D (see k_adjc_face)
template <int ND, int D>
__device__ __forceinline__ void adjc_faces(long long c, const double* __restrict__ q, const double* __restrict__ sl,
                                           const double* __restrict__ lam, double alpha, double dt, const Geometry& g,
                                           const GhostTables& gt, const PhysConst& pc,
                                           const double* __restrict__ psol, const double* qc, const double* lc,
                                           double hc, double* qb, double* sb, double* __restrict__ tbar) {
  constexpr int NV = ND + 2;
  constexpr int NT = (ND - 1) * NV;      // transverse slopes per side
  constexpr int NDIR = 2 * NV + 2 * NT;  // dual directions of one face
  constexpr int K = kAdjDirs;
  const long long ld = g.ld;
  const double kc = alpha * dt / hc;
#pragma unroll 1
  for (int sd2 = 0; sd2 < 2; ++sd2) {
    const int side = sd2 == 0 ? -1 : 1;
    const int n = g.nbr[(2 * D + sd2) * ld + c];
    double jac = 0.0;
    const int own = stencil_owner(g, gt, n, &jac);
    const double kn = own >= 0 ? alpha * dt / g.len[g.lvl[own]] : 0.0;
    double w[NV], qn[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double ln = own >= 0 ? lam[v * ld + own] : 0.0;
      w[v] = side > 0 ? (kn * ln - kc * lc[v]) : (kc * lc[v] - kn * ln);
      qn[v] = q[v * ld + n];
    }
    const bool cL = side > 0;  // c is the left cell of the face
    const double len_r = cL ? g.len[g.lvl[n]] : hc;
    double nb[NV], nsb[ND * NV];  // cotangents of the neighbour side (ghosts only)
#pragma unroll
    for (int v = 0; v < NV; ++v) nb[v] = 0.0;
#pragma unroll
    for (int k = 0; k < ND * NV; ++k) nsb[k] = 0.0;
    // The neighbour side's derivatives are needed only when the neighbour is a
    // non-periodic ghost (its state comes from c); an interior or periodic
    // neighbour takes its own.  Directions in use, in order: own state, [the
    // neighbour's state,] own transverse slopes[, the neighbour's].
    const bool all = own == -1;
    const int ndir = all ? NDIR : NV + NT;
#pragma unroll 1
    for (int j0 = 0; j0 < ndir; j0 += K) {
      DN<K> aq[NV], bq[NV], as[ND * NV], bs[ND * NV], f[NV];  // a: cell c, b: neighbour
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        aq[v] = DN<K>(qc[v]);
        bq[v] = DN<K>(qn[v]);
        const int ja = v - j0, jb = all ? NV + v - j0 : -1;
        if (ja >= 0 && ja < K) aq[v].d[ja] = 1.0;
        if (jb >= 0 && jb < K) bq[v].d[jb] = 1.0;
      }
      int t = 0;
#pragma unroll
      for (int s2 = 0; s2 < ND; ++s2) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          as[s2 * NV + v] = DN<K>(sl[(s2 * NV + v) * ld + c]);
          bs[s2 * NV + v] = DN<K>(sl[(s2 * NV + v) * ld + n]);
          if (s2 != D) {
            const int ja = (all ? 2 * NV : NV) + t - j0, jb = all ? 2 * NV + NT + t - j0 : -1;
            if (ja >= 0 && ja < K) as[s2 * NV + v].d[ja] = 1.0;
            if (jb >= 0 && jb < K) bs[s2 * NV + v].d[jb] = 1.0;
            ++t;
          }
        }
      }
      if (cL) cns_face_dual<ND, K, D>(aq, bq, as, bs, len_r, pc, f);
      else cns_face_dual<ND, K, D>(bq, aq, bs, as, len_r, pc, f);
#pragma unroll
      for (int jj = 0; jj < K; ++jj) {
        const int jl = j0 + jj;
        if (jl >= ndir) break;
        const int j = all ? jl : (jl < NV ? jl : jl + NV);  // the direction's index in the full list
        double gj = 0.0;
#pragma unroll
        for (int v = 0; v < NV; ++v) gj += w[v] * f[v].d[jj];
        if (j < NV) {
          qb[j] += gj;
        } else if (j < 2 * NV) {
          nb[j - NV] += gj;
        } else {
          const int tt = j < 2 * NV + NT ? j - 2 * NV : j - 2 * NV - NT;
          const int s2i = tt / NV, v = tt % NV;
          const int s2 = s2i < D ? s2i : s2i + 1;  // transverse directions skip D
          if (j < 2 * NV + NT) sb[s2 * NV + v] += gj;
          else nsb[s2 * NV + v] += gj;
        }
      }
    }
    if (own == -1) {  // a non-periodic ghost: its state and slopes come from c
      const long long i = n - g.n_int;
      const BcParam& B = gt.bcs[gt.bc_apply[i]];
      const double Tsol = (B.kind == BC_CPL_CNS_HEAT && psol && gt.partner[i] >= 0) ? psol[gt.partner[i]] : 0.0;
      const double tb = ghost_vjp<ND>(qc, B, gt.pos[i] >> 1, gt.dx[i], Tsol, pc, nb, qb);
      if (tbar && B.kind == BC_CPL_CNS_HEAT) tbar[i] = tb;
      const BcParam& Bo = gt.bcs[gt.bc_own[i]];
#pragma unroll
      for (int s2 = 0; s2 < ND; ++s2) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const double sign = (Bo.wall && v < ND && s2 != D) ? -1.0 : 1.0;
          sb[s2 * NV + v] += sign * nsb[s2 * NV + v];
        }
      }
    }
  }
}

// Face pass.  q: stage input (ghosts filled), sl: its slopes (k_slopes layout
// [(sd * NV + v) * ld + c]); psol: the conjugate partner's state (heat lhs) or
// nullptr.  Writes qface [NV][ld], sbar [ND * NV][ld] and, per conjugate
// ghost, tbar (the cotangent of the solid temperature it reads).
// REV: the hand-written reverse (adjc_faces_rev, one sweep per face);
// otherwise the forward-mode dual evaluation (adjc_faces), kept as a check.
template <int ND, bool REV = true>
__global__ void __launch_bounds__(kBlock) k_adjc_face(const double* __restrict__ q, const double* __restrict__ sl,
                                                      const double* __restrict__ lam, double alpha, Geometry g,
                                                      GhostTables gt, PhysConst pc, const Scalars* __restrict__ sc,
                                                      const double* __restrict__ psol, double* __restrict__ qface,
                                                      double* __restrict__ sbar, double* __restrict__ tbar) {
  constexpr int NV = ND + 2;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n_int) return;
  const long long ld = g.ld;
  const double dt = sc->dt;
  const double hc = g.len[g.lvl[c]];
  double qc[NV], lc[NV], qb[NV], sb[ND * NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) { qc[v] = q[v * ld + c]; lc[v] = lam[v * ld + c]; qb[v] = 0.0; }
#pragma unroll
  for (int k = 0; k < ND * NV; ++k) sb[k] = 0.0;
  if (REV) {
    SideAD<ND> Sc;
#pragma unroll
    for (int v = 0; v < NV; ++v) Sc.q[v] = qc[v];
    side_forward<ND>(Sc, pc.gamma, pc.gm1);
    double slc[ND * NV];
#pragma unroll
    for (int k = 0; k < ND * NV; ++k) slc[k] = sl[k * ld + c];
    adjc_faces_rev<ND, 0>(c, q, sl, lam, alpha, dt, g, gt, pc, psol, Sc, slc, lc, hc, qb, sb, tbar);
    adjc_faces_rev<ND, 1>(c, q, sl, lam, alpha, dt, g, gt, pc, psol, Sc, slc, lc, hc, qb, sb, tbar);
    if constexpr (ND == 3)
      adjc_faces_rev<ND, ND - 1>(c, q, sl, lam, alpha, dt, g, gt, pc, psol, Sc, slc, lc, hc, qb, sb, tbar);
  } else {
    adjc_faces<ND, 0>(c, q, sl, lam, alpha, dt, g, gt, pc, psol, qc, lc, hc, qb, sb, tbar);
    adjc_faces<ND, 1>(c, q, sl, lam, alpha, dt, g, gt, pc, psol, qc, lc, hc, qb, sb, tbar);
    if constexpr (ND == 3) adjc_faces<ND, ND - 1>(c, q, sl, lam, alpha, dt, g, gt, pc, psol, qc, lc, hc, qb, sb, tbar);
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) qface[v * ld + c] = qb[v];
#pragma unroll
  for (int k = 0; k < ND * NV; ++k) sbar[k * ld + c] = sb[k];
}

// Slope stencils: s_X[sd][v] = (q_{p(X)} - q_{m(X)}) / (2 h_X) for every cell X.
template <int ND>
__global__ void __launch_bounds__(kBlock) k_adjc_slopes(const double* __restrict__ q, const double* __restrict__ lam,
                                                        const double* __restrict__ extra,
                                                        const double* __restrict__ extra2, double beta,
                                                        double gamma_e, double gamma_e2, Geometry g, GhostTables gt,
                                                        PhysConst pc, const double* __restrict__ psol,
                                                        const double* __restrict__ qface,
                                                        const double* __restrict__ sbar, double* __restrict__ tbar,
                                                        double* __restrict__ gout) {
  constexpr int NV = ND + 2;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n_int) return;
  const long long ld = g.ld;
  const double hc = g.len[g.lvl[c]];
  double qb[NV], qc[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) { qb[v] = qface[v * ld + c]; qc[v] = q[v * ld + c]; }
#pragma unroll 1
  for (int sd = 0; sd < ND; ++sd) {
#pragma unroll 1
    for (int s2 = 0; s2 < 2; ++s2) {
      const int n = g.nbr[(2 * sd + s2) * ld + c];
      double jac = 0.0;
      const int X = stencil_owner(g, gt, n, &jac);
      // c is X's plus neighbour when X is c's minus neighbour, and vice versa
      const double sgn = s2 == 0 ? 1.0 : -1.0;
      if (X >= 0) {
        const double f = sgn / (2.0 * g.len[g.lvl[X]]);
#pragma unroll
        for (int v = 0; v < NV; ++v) qb[v] += f * sbar[(sd * NV + v) * ld + X];
      } else if (X == -1) {  // c's own slope reads the ghost's state
        const long long i = n - g.n_int;
        const BcParam& B = gt.bcs[gt.bc_apply[i]];
        double gb[NV];
        const double f = -sgn / (2.0 * hc);  // the ghost is c's plus neighbour (+) or minus neighbour (-)
#pragma unroll
        for (int v = 0; v < NV; ++v) gb[v] = f * sbar[(sd * NV + v) * ld + c];
        const double Tsol = (B.kind == BC_CPL_CNS_HEAT && psol && gt.partner[i] >= 0) ? psol[gt.partner[i]] : 0.0;
        const double tb = ghost_vjp<ND>(qc, B, gt.pos[i] >> 1, gt.dx[i], Tsol, pc, gb, qb);
        if (tbar && B.kind == BC_CPL_CNS_HEAT) tbar[i] += tb;
      }
    }
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double o = beta * lam[v * ld + c] + qb[v];
    if (extra) o += gamma_e * extra[v * ld + c];
    if (extra2) o += gamma_e2 * extra2[v * ld + c];
    gout[v * ld + c] = o;
  }
}

}  // namespace h3c
