// muscl_adjoint.cuh -- EXTENSION (no hom3 counterpart): discrete adjoint of
// the MUSCL stage of muscl_kernels.cuh.  The reconstruction is differentiated
// exactly where it is smooth; its switches are frozen at the forward values:
// the AUSM upwind side and |M| > 1 branches, the limiter's minimising face and
// its d2 > 0 / d2 < 0 branch, the neighbour that attains the largest /
// smallest value, and the positivity fallback of a face.
//
// Cotangents are gathered, never scattered (deterministic, no atomics):
//  k_adjm_face   per cell, every face: AUSM reverse on the reconstructed
//                states with the face weight w = k_R lambda_R - k_L lambda_L
//                (the face appears in both residuals); the cell's own side
//                gives the cotangent of its primitive state and of its
//                limited gradient; non-periodic ghost sides go straight to
//                the boundary cell through the condition (I or -I).
//  k_adjm_lim    per cell X: limiter and least-squares reverse -> gradient
//                cotangent b of the normal equations, the limiter's
//                sensitivity to the extreme neighbour, X's own terms.
//  k_adjm_gather per cell c: collects b and the limiter terms of every cell
//                whose stencil holds c, maps primitive to conservative
//                cotangents and writes beta lam + VJP + extras.
#pragma once
#include "adjoint_kernels.cuh"
#include "muscl_kernels.cuh"

namespace h3c {

// q-space cotangent of w = (u, rho, p)(q) at state w: qbar = (dw/dq)^T wbar
template <int ND>
__device__ __forceinline__ void prim_transpose(const double* w, const double* wbar, double gm1, double* qbar) {
  const double rinv = nr_rcp(w[ND]);
  double um2 = 0.0, uub = 0.0;
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    um2 += w[k] * w[k];
    uub += wbar[k] * w[k];
    qbar[k] = wbar[k] * rinv - gm1 * w[k] * wbar[ND + 1];
  }
  qbar[ND] = wbar[ND] - uub * rinv + 0.5 * gm1 * um2 * wbar[ND + 1];
  qbar[ND + 1] = gm1 * wbar[ND + 1];
}

// reverse of one side's a, M_d (and, for the upwind side, theta) of the AUSM
// flux on primitive states; adds to wb
template <int ND>
__device__ __forceinline__ void ausmw_side_reverse(const double* w, int d, double gamma, double Mbar, double abar,
                                                   double pbar, double* wb) {
  const double rho = w[ND], p = w[ND + 1];
  const double rinv = nr_rcp(rho);
  const double a2 = gamma * p * rinv;
  const double ainv = nr_rsqrt(a2);
  const double M = w[d] * ainv;
  wb[d] += Mbar * ainv;
  abar -= Mbar * M * ainv;
  const double a2bar = 0.5 * abar * ainv;
  wb[ND + 1] += pbar + a2bar * gamma * rinv;
  wb[ND] -= a2bar * gamma * p * rinv * rinv;
}

// wbL += (dF/dwL)^T wv, wbR += (dF/dwR)^T wv for the AUSM flux of two primitive states along d
template <int ND>
__device__ __forceinline__ void ausmw_vjp(const double* wL, const double* wR, int d, const double* wv, double gamma,
                                          double igm1, double* wbL, double* wbR) {
  constexpr int NV = ND + 2;
  auto mach = [&](const double* w, double& a, double& M) {
    const double a2 = gamma * w[ND + 1] * nr_rcp(w[ND]);
    const double ainv = nr_rsqrt(a2);
    a = a2 * ainv;
    M = w[d] * ainv;
  };
  double aL, ML, aR, MR;
  mach(wL, aL, ML);
  mach(wR, aR, MR);
  const double mi = m_int_d(1.0, ML) + m_int_d(-1.0, MR);
  const bool left = mi >= 0.0;
  const double* wu = left ? wL : wR;
  const double au = left ? aL : aR;
  // conservative components of the upwind side: rho u_k, rho, E + p
  const double rho = wu[ND], p = wu[ND + 1];
  double um2 = 0.0;
#pragma unroll
  for (int k = 0; k < ND; ++k) um2 += wu[k] * wu[k];
  const double Ep = p * igm1 + 0.5 * rho * um2 + p;
  double wq = wv[ND] * rho + wv[NV - 1] * Ep;
#pragma unroll
  for (int k = 0; k < ND; ++k) wq += wv[k] * rho * wu[k];
  const double mbar = au * wq;
  const double pibar = wv[d];
  const double MLbar = dm_int(1.0, ML) * mbar + dp_int(1.0, ML) * wL[ND + 1] * pibar;
  const double MRbar = dm_int(-1.0, MR) * mbar + dp_int(-1.0, MR) * wR[ND + 1] * pibar;
  double pLbar = p_int_d(1.0, ML) * pibar, pRbar = p_int_d(-1.0, MR) * pibar;
  double aLbar = 0.0, aRbar = 0.0;
  // theta = a (rho u, rho, E + p) of the upwind side, times mi
  const double am = au * mi;
  double* wbu = left ? wbL : wbR;
  double Ebar = am * wv[NV - 1];
#pragma unroll
  for (int k = 0; k < ND; ++k) {
    const double qb = am * wv[k];  // rho u_k
    wbu[k] += rho * qb;
    wbu[ND] += wu[k] * qb;
  }
  wbu[ND] += am * wv[ND];
  // E = p / (gamma - 1) + rho |u|^2 / 2, plus the explicit + p
#pragma unroll
  for (int k = 0; k < ND; ++k) wbu[k] += rho * wu[k] * Ebar;
  wbu[ND] += 0.5 * um2 * Ebar;
  if (left) {
    pLbar += (igm1 + 1.0) * Ebar;
    aLbar = mi * wq;
  } else {
    pRbar += (igm1 + 1.0) * Ebar;
    aRbar = mi * wq;
  }
  ausmw_side_reverse<ND>(wL, d, gamma, MLbar, aLbar, pLbar, wbL);
  ausmw_side_reverse<ND>(wR, d, gamma, MRbar, aRbar, pRbar, wbR);
}

// the cell that owns a neighbour's cotangent: interior -> itself, periodic
// ghost -> its paired cell, other ghosts -> -1 (the boundary cell's condition)
__device__ __forceinline__ int stencil_owner(const Geometry& g, const GhostTables& gt, int n, double* jac) {
  *jac = 0.0;
  if (n < g.n_int) return n;
  const long long i = n - g.n_int;
  const int b = gt.bc_apply[i];
  if (b == 255) return -2;
  const int kind = gt.bcs[b].kind;
  if (kind == BC_PERIODIC) return gt.partner[i];
  *jac = (kind == BC_EULER_DIRICHLET) ? -1.0 : 1.0;
  return -1;
}

// ---- face pass ----
template <int ND, bool HANG>
__global__ void __launch_bounds__(kBlock) k_adjm_face(const double* __restrict__ q, const double* __restrict__ grad,
                                                      const double* __restrict__ xc, const double* __restrict__ lam,
                                                      double alpha, Geometry g, GhostTables gt, PhysConst pc,
                                                      const Scalars* __restrict__ sc, double* __restrict__ qbar_face,
                                                      double* __restrict__ gbar) {
  constexpr int NV = ND + 2;
  constexpr double W = ND == 2 ? 0.5 : 0.25;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n_int) return;
  const long long ld = g.ld;
  const double gm1 = pc.gm1, gamma = pc.gamma, igm1 = 1.0 / pc.gm1;
  const double dt = sc->dt;
  const double hc = g.len[g.lvl[c]];
  const double kc = alpha * dt / hc;
  double wc[NV], lc[NV], xcc[ND], wbc[NV], gb[NV * ND], qbg[NV];
  prim_w<ND>(q, ld, c, gm1, wc);
#pragma unroll
  for (int v = 0; v < NV; ++v) { lc[v] = lam[v * ld + c]; wbc[v] = 0.0; qbg[v] = 0.0; }
#pragma unroll
  for (int k = 0; k < NV * ND; ++k) gb[k] = 0.0;
#pragma unroll
  for (int k = 0; k < ND; ++k) xcc[k] = __ldg(xc + k * ld + c);
  for_each_face<ND, HANG>(g, c, [&](int n, int d, int side) {
    // weights of the face in the two residuals
    const int mside = g.nbr[(side < 0 ? 2 * d : 2 * d + 1) * ld + c];
    const bool group = HANG && mside < 0;  // c is the coarse side of a sub-face group
    const double kc_face = group ? W * kc : kc;
    double jac = 0.0;
    const int own = stencil_owner(g, gt, n, &jac);
    double kn = 0.0;
    if (own >= 0) {
      kn = alpha * dt / g.len[g.lvl[own]];
      if (n < g.n_int && g.len[g.lvl[n]] > hc) kn *= W;  // n is the coarse side
    }
    double ln[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) ln[v] = own >= 0 ? lam[v * ld + own] : 0.0;
    double wv[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) wv[v] = side > 0 ? (kn * ln[v] - kc_face * lc[v]) : (kc_face * lc[v] - kn * ln[v]);
    // the forward face states
    const int L = side < 0 ? n : (int)c, Rr = side < 0 ? (int)c : n;
    double xf[ND];
    face_point<ND>(g, xc, L, Rr, d, xf);
    double wn[NV], xn[ND], wcf[NV], wnf[NV];
    prim_w<ND>(q, ld, n, gm1, wn);
#pragma unroll
    for (int k = 0; k < ND; ++k) xn[k] = __ldg(xc + k * ld + n);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = wc[v];
#pragma unroll
      for (int k = 0; k < ND; ++k) s = s + __ldg(grad + (v * ND + k) * ld + c) * (xf[k] - xcc[k]);
      wcf[v] = s;
      double t = wn[v];
#pragma unroll
      for (int k = 0; k < ND; ++k) t = t + __ldg(grad + (v * ND + k) * ld + n) * (xf[k] - xn[k]);
      wnf[v] = t;
    }
    const bool fallback = !(wcf[ND] > 0) || !(wcf[ND + 1] > 0) || !(wnf[ND] > 0) || !(wnf[ND + 1] > 0);
    if (fallback) {
#pragma unroll
      for (int v = 0; v < NV; ++v) { wcf[v] = wc[v]; wnf[v] = wn[v]; }
    }
    double bc_[NV], bn[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) { bc_[v] = 0.0; bn[v] = 0.0; }
    if (side > 0) ausmw_vjp<ND>(wcf, wnf, d, wv, gamma, igm1, bc_, bn);
    else ausmw_vjp<ND>(wnf, wcf, d, wv, gamma, igm1, bn, bc_);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      wbc[v] += bc_[v];
      if (!fallback) {
#pragma unroll
        for (int k = 0; k < ND; ++k) gb[v * ND + k] += bc_[v] * (xf[k] - xcc[k]);
      }
    }
    if (own == -1) {  // ghost through its condition (its gradient is zero)
      double qg[NV];
      prim_transpose<ND>(wn, bn, gm1, qg);
#pragma unroll
      for (int v = 0; v < NV; ++v) qbg[v] += jac * qg[v];
    }
  });
  double qb[NV];
  prim_transpose<ND>(wc, wbc, gm1, qb);
#pragma unroll
  for (int v = 0; v < NV; ++v) qbar_face[v * ld + c] = qb[v] + qbg[v];
#pragma unroll
  for (int k = 0; k < NV * ND; ++k) gbar[k * ld + c] = gb[k];
}

// ---- limiter and least-squares reverse ----
template <int ND, bool HANG>
__global__ void __launch_bounds__(kBlock) k_adjm_lim(const double* __restrict__ q, const double* __restrict__ xc,
                                                     const double* __restrict__ gbar, Geometry g, GhostTables gt,
                                                     PhysConst pc, double limiter_k, double* __restrict__ bbar,
                                                     double* __restrict__ dl1, int* __restrict__ owner,
                                                     double* __restrict__ wself, double* __restrict__ qghost) {
  constexpr int NV = ND + 2;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n_int) return;
  const long long ld = g.ld;
  const double gm1 = pc.gm1;
  double wc[NV], wmax[NV], wmin[NV], xcc[ND];
  int imax[NV], imin[NV];
  prim_w<ND>(q, ld, c, gm1, wc);
#pragma unroll
  for (int v = 0; v < NV; ++v) { wmax[v] = wc[v]; wmin[v] = wc[v]; imax[v] = -1; imin[v] = -1; }
#pragma unroll
  for (int k = 0; k < ND; ++k) xcc[k] = __ldg(xc + k * ld + c);
  double M[ND][ND], b[NV][ND];
#pragma unroll
  for (int i = 0; i < ND; ++i) {
#pragma unroll
    for (int j = 0; j < ND; ++j) M[i][j] = 0.0;
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
#pragma unroll
    for (int i = 0; i < ND; ++i) b[v][i] = 0.0;
  }
  for_each_face<ND, HANG>(g, c, [&](int n, int, int) {
    double wn[NV], dx[ND];
    prim_w<ND>(q, ld, n, gm1, wn);
    double r2 = 0.0;
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      dx[k] = __ldg(xc + k * ld + n) - xcc[k];
      r2 = k == 0 ? dx[k] * dx[k] : r2 + dx[k] * dx[k];
    }
    const double wgt = nr_rcp(r2);
#pragma unroll
    for (int i = 0; i < ND; ++i) {
#pragma unroll
      for (int j = 0; j < ND; ++j) M[i][j] = M[i][j] + (wgt * dx[i]) * dx[j];
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double dw = wn[v] - wc[v];
#pragma unroll
      for (int i = 0; i < ND; ++i) b[v][i] = b[v][i] + (wgt * dx[i]) * dw;
      if (wn[v] > wmax[v]) { wmax[v] = wn[v]; imax[v] = n; }
      if (wn[v] < wmin[v]) { wmin[v] = wn[v]; imin[v] = n; }
    }
  });
  double inv[ND][ND];
  if (ND == 2) {
    const double id = nr_rcp(M[0][0] * M[1][1] - M[0][1] * M[1][0]);
    inv[0][0] = M[1][1] * id;
    inv[1][1] = M[0][0] * id;
    inv[0][1] = -M[0][1] * id;
    inv[1][0] = -M[1][0] * id;
  } else {
    const int i2 = ND - 1;
    const double c00 = M[1][1] * M[i2][i2] - M[1][i2] * M[i2][1];
    const double c01 = M[1][i2] * M[i2][0] - M[1][0] * M[i2][i2];
    const double c02 = M[1][0] * M[i2][1] - M[1][1] * M[i2][0];
    const double id = nr_rcp(M[0][0] * c00 + M[0][1] * c01 + M[0][i2] * c02);
    inv[0][0] = c00 * id;
    inv[0][1] = (M[0][i2] * M[i2][1] - M[0][1] * M[i2][i2]) * id;
    inv[0][i2] = (M[0][1] * M[1][i2] - M[0][i2] * M[1][1]) * id;
    inv[1][0] = c01 * id;
    inv[1][1] = (M[0][0] * M[i2][i2] - M[0][i2] * M[i2][0]) * id;
    inv[1][i2] = (M[0][i2] * M[1][0] - M[0][0] * M[1][i2]) * id;
    inv[i2][0] = c02 * id;
    inv[i2][1] = (M[0][1] * M[i2][0] - M[0][0] * M[i2][1]) * id;
    inv[i2][i2] = (M[0][0] * M[1][1] - M[0][1] * M[1][0]) * id;
  }
  const double kh = limiter_k * g.len[g.lvl[c]];
  const double e2 = kh * kh * kh;
  double G[NV][ND], psi[NV], d2s[NV], rf[NV][ND];
  int branch[NV];  // 0: psi = 1, 1: from the largest neighbour, -1: from the smallest
#pragma unroll
  for (int v = 0; v < NV; ++v) {
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double s = inv[i][0] * b[v][0];
#pragma unroll
      for (int j = 1; j < ND; ++j) s = s + inv[i][j] * b[v][j];
      G[v][i] = s;
      rf[v][i] = 0.0;
    }
    psi[v] = 1.0;
    d2s[v] = 0.0;
    branch[v] = 0;
    wmax[v] = wmax[v] - wc[v];
    wmin[v] = wmin[v] - wc[v];
  }
  for_each_face<ND, HANG>(g, c, [&](int n, int d, int side) {
    double xf[ND];
    if (side < 0) face_point<ND>(g, xc, n, (int)c, d, xf);
    else face_point<ND>(g, xc, (int)c, n, d, xf);
#pragma unroll
    for (int k = 0; k < ND; ++k) xf[k] = xf[k] - xcc[k];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double d2 = G[v][0] * xf[0];
#pragma unroll
      for (int k = 1; k < ND; ++k) d2 = d2 + G[v][k] * xf[k];
      double phi = 1.0;
      int br = 0;
      if (d2 > 0) { phi = vk_phi(wmax[v], d2, e2); br = 1; }
      else if (d2 < 0) { phi = vk_phi(wmin[v], d2, e2); br = -1; }
      if (phi < psi[v]) {
        psi[v] = phi;
        branch[v] = br;
        d2s[v] = d2;
#pragma unroll
        for (int k = 0; k < ND; ++k) rf[v][k] = xf[k];
      }
    }
  });
  // reverse: limited gradient psi G
  double wb[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) wb[v] = 0.0;
  double qgh[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) qgh[v] = 0.0;
  double bb[NV][ND];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double Gb[ND], psib = 0.0;
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      const double gk = gbar[(v * ND + k) * ld + c];
      Gb[k] = psi[v] * gk;
      psib += gk * G[v][k];
    }
    double l1b = 0.0;
    int own = -2;
    if (branch[v] != 0) {
      const double a = branch[v] > 0 ? wmax[v] : wmin[v];
      const double bq = d2s[v];
      const double N = (a * a + e2) * bq + 2. * bq * bq * a;
      const double D = bq * (a * a + 2. * bq * bq + a * bq + e2);
      const double Di = nr_rcp(D);
      const double phi = N * Di;
      const double Na = 2. * a * bq + 2. * bq * bq, Nb = a * a + e2 + 4. * a * bq;
      const double Da = bq * (2. * a + bq), Db = (a * a + 2. * bq * bq + a * bq + e2) + bq * (4. * bq + a);
      const double pa = (Na - phi * Da) * Di, pb = (Nb - phi * Db) * Di;
#pragma unroll
      for (int k = 0; k < ND; ++k) Gb[k] += psib * pb * rf[v][k];
      const int ext = branch[v] > 0 ? imax[v] : imin[v];
      if (ext >= 0) {  // the extreme is a neighbour (not the cell itself)
        l1b = psib * pa;
        wb[v] -= l1b;
        double jac = 0.0;
        own = stencil_owner(g, gt, ext, &jac);
        if (own == -1) {  // ghost through its condition
          double wg[NV], e[NV], qg[NV];
          prim_w<ND>(q, ld, ext, gm1, wg);
#pragma unroll
          for (int u = 0; u < NV; ++u) e[u] = u == v ? l1b : 0.0;
          prim_transpose<ND>(wg, e, gm1, qg);
#pragma unroll
          for (int u = 0; u < NV; ++u) qgh[u] += jac * qg[u];
        }
      }
    }
    dl1[v * ld + c] = l1b;
    owner[v * ld + c] = own;
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double s = inv[i][0] * Gb[0];
#pragma unroll
      for (int j = 1; j < ND; ++j) s = s + inv[i][j] * Gb[j];
      bb[v][i] = s;
      bbar[(v * ND + i) * ld + c] = s;
    }
  }
  // b_v = sum_n wgt dx (w_n - w_c): the cell's own term and its non-periodic ghosts
  for_each_face<ND, HANG>(g, c, [&](int n, int, int) {
    double dx[ND];
    double r2 = 0.0;
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      dx[k] = __ldg(xc + k * ld + n) - xcc[k];
      r2 = k == 0 ? dx[k] * dx[k] : r2 + dx[k] * dx[k];
    }
    const double wgt = nr_rcp(r2);
    double t[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = dx[0] * bb[v][0];
#pragma unroll
      for (int k = 1; k < ND; ++k) s += dx[k] * bb[v][k];
      t[v] = wgt * s;
      wb[v] -= t[v];
    }
    double jac = 0.0;
    if (stencil_owner(g, gt, n, &jac) == -1) {
      double wg[NV], qg[NV];
      prim_w<ND>(q, ld, n, gm1, wg);
      prim_transpose<ND>(wg, t, gm1, qg);
#pragma unroll
      for (int u = 0; u < NV; ++u) qgh[u] += jac * qg[u];
    }
  });
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    wself[v * ld + c] = wb[v];
    qghost[v * ld + c] = qgh[v];
  }
}

// ---- gather and combination ----
template <int ND, bool HANG>
__global__ void __launch_bounds__(kBlock) k_adjm_gather(const double* __restrict__ q, const double* __restrict__ xc,
                                                        const double* __restrict__ lam, const double* __restrict__ extra,
                                                        const double* __restrict__ extra2, double beta, double gamma_e,
                                                        double gamma_e2, Geometry g, GhostTables gt, PhysConst pc,
                                                        const double* __restrict__ bbar, const double* __restrict__ dl1,
                                                        const int* __restrict__ owner,
                                                        const double* __restrict__ wself,
                                                        const double* __restrict__ qbar_face,
                                                        const double* __restrict__ qghost, double* __restrict__ gout) {
  constexpr int NV = ND + 2;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= g.n_int) return;
  const long long ld = g.ld;
  double wb[NV], xcc[ND], wc[NV];
  prim_w<ND>(q, ld, c, pc.gm1, wc);
#pragma unroll
  for (int v = 0; v < NV; ++v) wb[v] = wself[v * ld + c];
#pragma unroll
  for (int k = 0; k < ND; ++k) xcc[k] = __ldg(xc + k * ld + c);
  // every cell X whose stencil holds c: c's face neighbours (periodic ghosts stand for their paired cell)
  for_each_face<ND, HANG>(g, c, [&](int n, int, int) {
    double jac = 0.0;
    const int X = stencil_owner(g, gt, n, &jac);
    if (X < 0) return;
    double dx[ND];
    double r2 = 0.0;
#pragma unroll
    for (int k = 0; k < ND; ++k) {
      dx[k] = xcc[k] - __ldg(xc + k * ld + n);  // from X (or its image) to c
      r2 = k == 0 ? dx[k] * dx[k] : r2 + dx[k] * dx[k];
    }
    const double wgt = nr_rcp(r2);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = dx[0] * bbar[(v * ND) * ld + X];
#pragma unroll
      for (int k = 1; k < ND; ++k) s += dx[k] * bbar[(v * ND + k) * ld + X];
      wb[v] += wgt * s;
      if (owner[v * ld + X] == (int)c) wb[v] += dl1[v * ld + X];
    }
  });
  double qb[NV];
  prim_transpose<ND>(wc, wb, pc.gm1, qb);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double o = beta * lam[v * ld + c] + qb[v] + qbar_face[v * ld + c] + qghost[v * ld + c];
    if (extra) o += gamma_e * extra[v * ld + c];
    if (extra2) o += gamma_e2 * extra2[v * ld + c];
    gout[v * ld + c] = o;
  }
}

}  // namespace h3c
