// muscl_kernels.cuh -- EXTENSION (not in hom3, whose finite-volume scheme is
// first order, solver.hpp:45-49): second-order MUSCL reconstruction of the
// primitive variables w = (u_0..u_{nd-1}, rho, p) for the Euler/AUSM stage.
//
//  * k_muscl_grad: per interior cell, the least-squares gradient over the face
//    neighbours (same-level and coarser cells, the finer cells of a sub-face
//    group, ghosts at their mirrored centres) with weights 1/|dx|^2, the
//    normal equations solved by the adjugate, then Venkatakrishnan's limiter
//    per variable: psi = min(1, min over faces phi(D, d2)), D the largest /
//    smallest neighbour difference, d2 the unlimited change to the face point,
//    phi(a, b) = ((a^2 + e) b + 2 b^2 a) / (b (a^2 + 2 b^2 + a b + e)),
//    e = (K h)^3.  Stores psi_v G_v.
//  * k_muscl_ghosts: periodic ghosts take their paired cell's gradient; other
//    ghosts keep a zero gradient (first order on the ghost side).
//  * k_stage_muscl: per cell, every face evaluates AUSM on the reconstructed
//    states w + psi G . (x_f - x) of both sides at one face point (on the face
//    plane, transverse coordinates of the smaller cell), falling back to the
//    cell values when a reconstructed density or pressure is not positive.
//    Both cells of a face compute the same F(l, r), so the update conserves.
#pragma once
#include "fv_kernels.cuh"

namespace h3c {

template <int ND>
__device__ __forceinline__ void prim_w(const double* __restrict__ q, long long ld, long long c, double gm1,
                                       double* w) {
  const double rho = __ldg(q + ND * ld + c);
  const double rinv = nr_rcp(rho);
  double um2 = 0.0;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    w[d] = __ldg(q + d * ld + c) * rinv;
    um2 = d == 0 ? w[d] * w[d] : um2 + w[d] * w[d];
  }
  w[ND] = rho;
  w[ND + 1] = gm1 * (__ldg(q + (ND + 1) * ld + c) - 0.5 * rho * um2);
}

// the face neighbours of interior cell c: f(n, d, side), side -1 (minus) / +1 (plus)
template <int ND, bool HANG, class F>
__device__ __forceinline__ void for_each_face(const Geometry& g, long long c, F&& f) {
#pragma unroll
  for (int d = 0; d < ND; ++d) {
#pragma unroll
    for (int sd = 0; sd < 2; ++sd) {
      const int n = g.nbr[(2 * d + sd) * g.ld + c];
      const int side = sd == 0 ? -1 : 1;
      if (!HANG || n >= 0) {
        f(n, d, side);
      } else {
        const long long k = -n - 2;
#pragma unroll
        for (int j = 0; j < (1 << (ND - 1)); ++j) f(g.sub[j * g.nsub + k], d, side);
      }
    }
  }
}

// face point of the face between L (minus side) and R along d
template <int ND>
__device__ __forceinline__ void face_point(const Geometry& g, const double* __restrict__ xc, int L, int R, int d,
                                           double* xf) {
  const double hL = g.len[g.lvl[L]], hR = g.len[g.lvl[R]];
  const int sm = hR < hL ? R : L;
#pragma unroll
  for (int k = 0; k < ND; ++k) xf[k] = __ldg(xc + k * g.ld + sm);
  xf[d] = __ldg(xc + d * g.ld + L) + 0.5 * hL;
}

__device__ __forceinline__ double vk_phi(double a, double b, double e2) {
  return ((a * a + e2) * b + 2. * b * b * a) * nr_rcp(b * (a * a + 2. * b * b + a * b + e2));
}

template <int ND, bool HANG>
__global__ void __launch_bounds__(kBlock) k_muscl_grad(const double* __restrict__ q, const double* __restrict__ xc,
                                                       Geometry g, PhysConst pc, double limiter_k,
                                                       double* __restrict__ grad) {
  constexpr int NV = ND + 2;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= instance_end(g, tile_instance(g, blockIdx.x))) return;  // also skips padding between instances
  const long long ld = g.ld;
  const double gm1 = pc.gm1;
  double wc[NV], wmax[NV], wmin[NV];
  prim_w<ND>(q, ld, c, gm1, wc);
#pragma unroll
  for (int v = 0; v < NV; ++v) { wmax[v] = wc[v]; wmin[v] = wc[v]; }
  double xcc[ND];
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
    double wn[NV];
    prim_w<ND>(q, ld, n, gm1, wn);
    double dx[ND];
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
      wmax[v] = wn[v] > wmax[v] ? wn[v] : wmax[v];
      wmin[v] = wn[v] < wmin[v] ? wn[v] : wmin[v];
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
    const int i2 = ND - 1;  // == 2; keeps the indices in range for ND == 2
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
  double G[NV][ND], psi[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
#pragma unroll
    for (int i = 0; i < ND; ++i) {
      double s = inv[i][0] * b[v][0];
#pragma unroll
      for (int j = 1; j < ND; ++j) s = s + inv[i][j] * b[v][j];
      G[v][i] = s;
    }
    psi[v] = 1.0;
    wmax[v] = wmax[v] - wc[v];  // largest / smallest neighbour difference
    wmin[v] = wmin[v] - wc[v];
  }
  // one pass over the faces for all variables: the face offset is loaded once
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
      if (d2 > 0) phi = vk_phi(wmax[v], d2, e2);
      else if (d2 < 0) phi = vk_phi(wmin[v], d2, e2);
      psi[v] = phi < psi[v] ? phi : psi[v];
    }
  });
#pragma unroll
  for (int v = 0; v < NV; ++v) {
#pragma unroll
    for (int i = 0; i < ND; ++i) grad[(v * ND + i) * ld + c] = psi[v] * G[v][i];
  }
}

template <int ND>
__global__ void __launch_bounds__(kBlock) k_muscl_ghosts(double* __restrict__ grad, Geometry g, GhostTables gt) {
  constexpr int NV = ND + 2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gt.ng) return;
  if (gt.bcs[gt.bc_own[i]].kind != BC_PERIODIC) return;
  const int o = gt.partner[i];
  if (o < 0) return;
  const long long gc = g.n_int + i;
#pragma unroll
  for (int k = 0; k < NV * ND; ++k) grad[k * g.ld + gc] = grad[k * g.ld + o];
}

// primitive face state -> the AUSM operand (Prim of fv_kernels.cuh)
template <class R, int ND>
__device__ __forceinline__ void prim_from_w(const double* w, R gamma, R igm1, Prim<R, ND>& P) {
  const R rho = (R)w[ND];
  R um2 = R(0);
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    P.u[d] = (R)w[d];
    P.q[d] = rho * P.u[d];
    um2 = d == 0 ? P.u[d] * P.u[d] : um2 + P.u[d] * P.u[d];
  }
  P.q[ND] = rho;
  P.p = (R)w[ND + 1];
  P.q[ND + 1] = P.p * igm1 + R(0.5) * rho * um2;
  const R a2 = gamma * P.p * nr_rcp(rho);
  const R ainv = nr_rsqrt(a2);
  P.a = a2 * ainv;
#pragma unroll
  for (int d = 0; d < ND; ++d) P.M[d] = P.u[d] * ainv;
}

template <int ND, class R, int MODE, bool HANG, bool FUSE>
__global__ void __launch_bounds__(kBlock) k_stage_muscl(const double* __restrict__ qin, double* out,
                                                        const double* __restrict__ grad,
                                                        const double* __restrict__ xc, Geometry g, PhysConst pc,
                                                        const Scalars* __restrict__ sc, long long* dtmin) {
  constexpr int NV = ND + 2;
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int inst = tile_instance(g, blockIdx.x);
  const bool live = c < instance_end(g, inst);
  long long ord = kOrdMax;
  bool bad = false;
  if (live) {
    const long long ld = g.ld;
    const double dt = sc[inst].dt;
    const double dx = g.len[g.lvl[c]];
    const double gm1 = pc.gm1;
    const R gamma = (R)pc.gamma, igm1 = R(1) / (R)pc.gm1;
    double qc[NV], wc[NV], Gc[NV * ND], xcc[ND];
#pragma unroll
    for (int v = 0; v < NV; ++v) qc[v] = __ldg(qin + v * ld + c);
    prim_w<ND>(qin, ld, c, gm1, wc);
#pragma unroll
    for (int k = 0; k < NV * ND; ++k) Gc[k] = __ldg(grad + k * ld + c);
#pragma unroll
    for (int k = 0; k < ND; ++k) xcc[k] = __ldg(xc + k * ld + c);
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
    // flux of the face between c and n along d (side: where n lies), into f
    auto face = [&](int n, int d, int side, double* fo) {
      const int L = side < 0 ? n : (int)c, Rr = side < 0 ? (int)c : n;
      double xf[ND];
      face_point<ND>(g, xc, L, Rr, d, xf);
      double wn[NV], xn[ND];
      prim_w<ND>(qin, ld, n, gm1, wn);
#pragma unroll
      for (int k = 0; k < ND; ++k) xn[k] = __ldg(xc + k * ld + n);
      double wcf[NV], wnf[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double s = wc[v];
#pragma unroll
        for (int k = 0; k < ND; ++k) s = s + Gc[v * ND + k] * (xf[k] - xcc[k]);
        wcf[v] = s;
        double t = wn[v];
#pragma unroll
        for (int k = 0; k < ND; ++k) t = t + __ldg(grad + (v * ND + k) * ld + n) * (xf[k] - xn[k]);
        wnf[v] = t;
      }
      if (!(wcf[ND] > 0) || !(wcf[ND + 1] > 0) || !(wnf[ND] > 0) || !(wnf[ND + 1] > 0)) {
#pragma unroll
        for (int v = 0; v < NV; ++v) { wcf[v] = wc[v]; wnf[v] = wn[v]; }
      }
      Prim<R, ND> Pc, Pn;
      prim_from_w<R, ND>(wcf, gamma, igm1, Pc);
      prim_from_w<R, ND>(wnf, gamma, igm1, Pn);
      R f[NV];
      if (side < 0) ausm<R, ND>(Pn, Pc, d, f);
      else ausm<R, ND>(Pc, Pn, d, f);
#pragma unroll
      for (int v = 0; v < NV; ++v) fo[v] = (double)f[v];
    };
    // one side of direction d: a neighbour or a sub-face group (area-weighted sum)
    auto side_flux = [&](int n, int d, int side, double* fo) {
      if (!HANG || n >= 0) {
        face(n, d, side, fo);
        return;
      }
      const long long kg = -n - 2;
#pragma unroll
      for (int j = 0; j < (1 << (ND - 1)); ++j) {
        double f[NV];
        face(g.sub[j * g.nsub + kg], d, side, f);
#pragma unroll
        for (int v = 0; v < NV; ++v) fo[v] = j == 0 ? f[v] : fo[v] + f[v];
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) fo[v] = (ND == 2 ? 0.5 : 0.25) * fo[v];
    };
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      double fm[NV], fp[NV];
      side_flux(g.nbr[(2 * d) * ld + c], d, -1, fm);
      side_flux(g.nbr[(2 * d + 1) * ld + c], d, 1, fp);
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fm[v] - fp[v]);
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

}  // namespace h3c
