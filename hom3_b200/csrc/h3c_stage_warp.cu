// h3c_stage_warp.cu -- the warp-tiled Euler/AUSM stage kernel.
//
// One thread per interior cell, one warp per 32 consecutive Morton cells (a
// 4x4x2 brick of a uniform 3D region, 8x4 in 2D).  hom3's num_flux
// (src/solver/fv/solver.hpp:440-460) evaluates every face from both of its
// cells; the per-cell kernel does the same and recomputes each neighbour's
// face state (its primitive variables) once per face.  Here a warp
//   1. computes the face state of each of its cells once (shared memory),
//   2. lists the faces whose neighbour lies outside the warp (a ballot per
//      face position gives each a slot) and computes those neighbours' face
//      states, one entry per lane, with the loads of two entries in flight,
//   3. lists the minus faces that no plus face of the warp covers (the
//      neighbour is outside the warp, or a coarser cell of it) and evaluates
//      them, one face per lane,
//   4. per direction evaluates each cell's plus face once and hands it to
//      the neighbour whose minus face it is (shared memory),
// then sums the faces per direction in hom3's order and updates the cell as
// the other stage kernels do (rk_combine, fused next-step CFL minimum).
// The face flux is the tile kernels' F(l, r) (ausm_face of the two face
// states), so the result is theirs up to the compiler's FMA placement.
// Coarse/fine sub-face groups, and faces beyond the per-warp caps of
// stage_warp.hpp, are evaluated by their own cell from global memory.
#include <cuda_runtime.h>

#include <algorithm>

#define H3C_DEVICE_FUNCTIONS_ONLY
#include "fv_kernels.cuh"
#include "stage_warp.hpp"

namespace h3c {

namespace {

#ifndef H3C_WARP_MINB
#define H3C_WARP_MINB 3  // blocks per SM the kernel is register-budgeted for
#endif

// Per-warp shared memory.  own: the warp's cells' face states (theta, p and
// the Mach number along every direction); halo: face states of the cells
// outside the warp (theta, p, Mach number along the entry's direction);
// plus: the plus-face fluxes of the current direction; minus: the listed
// minus faces' fluxes.
template <class R, int ND> struct WarpSmem {
  static constexpr int NV = ND + 2;
  R own[NV + 1 + ND][32];
  R halo[NV + 2][kWarpHalo];
  double plus[NV][32];
  double minus[NV][kWarpMinus];
  int halo_cell[kWarpHalo];
  unsigned char halo_dir[kWarpHalo];
  int minus_item[kWarpMinus];  // left state (lane, or 32 + halo entry) | right lane << 8 | direction << 16
};

template <class R, int ND>
__device__ __forceinline__ void own_state(const WarpSmem<R, ND>& S, int lane, int d, FaceState<R, ND>& F) {
  constexpr int NV = ND + 2;
#pragma unroll
  for (int v = 0; v < NV; ++v) F.th[v] = S.own[v][lane];
  F.p = S.own[NV][lane];
  F.M = S.own[NV + 1 + d][lane];
}

template <class R, int ND>
__device__ __forceinline__ void halo_state(const WarpSmem<R, ND>& S, int h, FaceState<R, ND>& F) {
  constexpr int NV = ND + 2;
#pragma unroll
  for (int v = 0; v < NV; ++v) F.th[v] = S.halo[v][h];
  F.p = S.halo[NV][h];
  F.M = S.halo[NV + 1][h];
}

template <class R, int ND>
__device__ __forceinline__ void face_state_of(const double* qn, int d, R gamma, R gm1, FaceState<R, ND>& F) {
  constexpr int NV = ND + 2;
  Prim<R, ND> P;
#pragma unroll
  for (int v = 0; v < NV; ++v) P.q[v] = (R)qn[v];
  make_prim<R, ND>(P, gamma, gm1);
#pragma unroll
  for (int v = 0; v < ND + 1; ++v) F.th[v] = P.q[v] * P.a;
  F.th[ND + 1] = (P.q[ND + 1] + P.p) * P.a;
  F.p = P.p;
  F.M = P.M[0];  // the Mach number along d, selected without indexing (d is not a constant here)
#pragma unroll
  for (int e = 1; e < ND; ++e) F.M = d == e ? P.M[e] : F.M;
}

template <int ND, class R, int MODE, bool HANG, bool FUSE>
__global__ void __launch_bounds__(kBlock, H3C_WARP_MINB)
    k_stage_ausm_warp(const double* __restrict__ qin, double* out, Geometry g, PhysConst pc,
                      const Scalars* __restrict__ sc, long long* dtmin) {
  constexpr int NV = ND + 2, NS = 1 << (ND - 1);
  constexpr double W = ND == 2 ? 0.5 : 0.25;
  extern __shared__ __align__(16) unsigned char warp_smem_raw[];
  const int lane = threadIdx.x & 31;
  WarpSmem<R, ND>& S = reinterpret_cast<WarpSmem<R, ND>*>(warp_smem_raw)[threadIdx.x >> 5];
  __shared__ long long min_slot;
  __shared__ unsigned min_cnt;
  if (FUSE) {
    if (threadIdx.x == 0) {
      min_slot = kOrdMax;
      min_cnt = 0;
    }
    __syncthreads();  // the only block barrier
  }
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long w0 = c - lane;
  const int inst = tile_instance(g, blockIdx.x);
  const long long iend = instance_end(g, inst);
  const bool live = c < iend;
  const long long wend = w0 + 32 < iend ? w0 + 32 : iend;  // the warp's cells: [w0, wend)
  if (MODE != 0 && live) prefetch_row_l2<NV>(out, g.ld, c);  // the in-place start state, read at the update
  const unsigned below = (1u << lane) - 1u;
  const long long ld = g.ld;
  const R gamma = (R)pc.gamma, gm1 = (R)pc.gm1;
  auto in_warp = [&](int n) { return n >= w0 && n < wend; };

  // ---- 1. own state and face state ----
  // (the own state is read again at the update rather than held in registers
  // across the face lists)
  int nb[2 * ND];
#pragma unroll
  for (int p = 0; p < 2 * ND; ++p) nb[p] = live ? __ldg(g.nbr + p * ld + c) : -1;
  if (live) {
    Prim<R, ND> P;
#pragma unroll
    for (int v = 0; v < NV; ++v) P.q[v] = (R)__ldg(qin + v * ld + c);
    make_prim<R, ND>(P, gamma, gm1);
#pragma unroll
    for (int v = 0; v < ND + 1; ++v) S.own[v][lane] = P.q[v] * P.a;
    S.own[ND + 1][lane] = (P.q[ND + 1] + P.p) * P.a;
    S.own[NV][lane] = P.p;
#pragma unroll
    for (int d = 0; d < ND; ++d) S.own[NV + 1 + d][lane] = P.M[d];
  }

  // ---- 2. faces whose neighbour lies outside the warp: one halo entry each ----
  int hs[2 * ND];
  int nh = 0;
#pragma unroll
  for (int s = 0; s < 2 * ND; ++s) {
    const int n = nb[s];
    const bool need = n >= 0 && !in_warp(n);
    const unsigned m = __ballot_sync(0xffffffffu, need);
    const int slot = nh + __popc(m & below);
    hs[s] = need && slot < kWarpHalo ? slot : -1;
    if (hs[s] >= 0) {
      S.halo_cell[slot] = n;
      S.halo_dir[slot] = (unsigned char)(s >> 1);
    }
    nh += __popc(m);
  }
  nh = nh < kWarpHalo ? nh : kWarpHalo;
  __syncwarp();
  {
    static_assert(kWarpHalo == 64, "two halo entries per lane");
    const int ia = lane, ib = lane + 32;
    double qa[NV], qb[NV];
    const int na = ia < nh ? S.halo_cell[ia] : 0, nbb = ib < nh ? S.halo_cell[ib] : 0;
    if (ia < nh) {
#pragma unroll
      for (int v = 0; v < NV; ++v) qa[v] = __ldg(qin + v * ld + na);
    }
    if (ib < nh) {
#pragma unroll
      for (int v = 0; v < NV; ++v) qb[v] = __ldg(qin + v * ld + nbb);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int i = k == 0 ? ia : ib;
      if (i < nh) {
        FaceState<R, ND> F;
        face_state_of<R, ND>(k == 0 ? qa : qb, S.halo_dir[i], gamma, gm1, F);
#pragma unroll
        for (int v = 0; v < NV; ++v) S.halo[v][i] = F.th[v];
        S.halo[NV][i] = F.p;
        S.halo[NV + 1][i] = F.M;
      }
    }
  }

  // ---- 3. minus faces no plus face of the warp covers ----
  // shared[d]: the minus neighbour is a cell of the warp whose plus
  // neighbour is this cell (same level), so its plus face is this face.
  bool shared[ND];
  int ms[ND];
  int nm = 0;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const int m = nb[2 * d];
    const bool inw = m >= 0 && in_warp(m);
    const int src = inw ? (int)(m - w0) : lane;
    const int mp = __shfl_sync(0xffffffffu, nb[2 * d + 1], src);
    shared[d] = live && inw && (long long)mp == c;
    const int loc = inw ? src : (hs[2 * d] >= 0 ? 32 + hs[2 * d] : -1);
    const bool need = live && !shared[d] && m >= 0 && loc >= 0;
    const unsigned mk = __ballot_sync(0xffffffffu, need);
    const int slot = nm + __popc(mk & below);
    ms[d] = need && slot < kWarpMinus ? slot : -1;
    if (ms[d] >= 0) S.minus_item[slot] = loc | (lane << 8) | (d << 16);
    nm += __popc(mk);
  }
  nm = nm < kWarpMinus ? nm : kWarpMinus;
  __syncwarp();  // own and halo face states, and the minus list, are visible to the warp
  if (lane < nm) {
    static_assert(kWarpMinus == 32, "one minus face per lane");
    const int it = S.minus_item[lane];
    const int loc = it & 0xff, rl = (it >> 8) & 0xff, d = it >> 16;
    FaceState<R, ND> L, Rt;
    if (loc < 32) own_state<R, ND>(S, loc, d, L);
    else halo_state<R, ND>(S, loc - 32, L);
    own_state<R, ND>(S, rl, d, Rt);
    R f[NV];
    ausm_face<R, ND>(L, Rt, d, f);
#pragma unroll
    for (int v = 0; v < NV; ++v) S.minus[v][lane] = (double)f[v];
  }

  // a neighbour's face state along d wherever it is: the warp, the halo, or global memory
  auto state_of = [&](int n, int slot, int d, FaceState<R, ND>& F) {
    if (in_warp(n)) {
      own_state<R, ND>(S, (int)(n - w0), d, F);
    } else if (slot >= 0) {
      halo_state<R, ND>(S, slot, F);
    } else {
      face_state_global<R, ND>(F, qin, ld, n, d, gamma, gm1);
    }
  };

  // ---- 4. per direction: plus faces once, minus faces from the warp or the list ----
  double acc[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) acc[v] = 0.0;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const int m = nb[2 * d], p = nb[2 * d + 1];
    double fp[NV], fm[NV];
    if (live) {
      FaceState<R, ND> Fc;
      own_state<R, ND>(S, lane, d, Fc);
      if (!HANG || p >= 0) {
        FaceState<R, ND> Fp;
        state_of(p, hs[2 * d + 1], d, Fp);
        R f[NV];
        ausm_face<R, ND>(Fc, Fp, d, f);
#pragma unroll
        for (int v = 0; v < NV; ++v) fp[v] = (double)f[v];
      } else {  // coarse/fine face: W times the sum over the group's fine cells
        const long long k = -(long long)p - 2;
#pragma unroll 1
        for (int j = 0; j < NS; ++j) {
          FaceState<R, ND> Fn;
          face_state_global<R, ND>(Fn, qin, ld, __ldg(g.sub + j * g.nsub + k), d, gamma, gm1);
          R f[NV];
          ausm_face<R, ND>(Fc, Fn, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fp[v] = j == 0 ? (double)f[v] : fp[v] + (double)f[v];
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) fp[v] = __dmul_rn(W, fp[v]);
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) S.plus[v][lane] = fp[v];
    }
    __syncwarp();  // the plus faces of this direction are visible
    if (live) {
      if (shared[d]) {
#pragma unroll
        for (int v = 0; v < NV; ++v) fm[v] = S.plus[v][m - w0];
      } else if (ms[d] >= 0) {
#pragma unroll
        for (int v = 0; v < NV; ++v) fm[v] = S.minus[v][ms[d]];
      } else {
        FaceState<R, ND> Fc;
        own_state<R, ND>(S, lane, d, Fc);
        if (!HANG || m >= 0) {
          FaceState<R, ND> Fm;
          state_of(m, hs[2 * d], d, Fm);
          R f[NV];
          ausm_face<R, ND>(Fm, Fc, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = (double)f[v];
        } else {
          const long long k = -(long long)m - 2;
#pragma unroll 1
          for (int j = 0; j < NS; ++j) {
            FaceState<R, ND> Fn;
            face_state_global<R, ND>(Fn, qin, ld, __ldg(g.sub + j * g.nsub + k), d, gamma, gm1);
            R f[NV];
            ausm_face<R, ND>(Fn, Fc, d, f);
#pragma unroll
            for (int v = 0; v < NV; ++v) fm[v] = j == 0 ? (double)f[v] : fm[v] + (double)f[v];
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = __dmul_rn(W, fm[v]);
        }
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fm[v] - fp[v]);
    }
    __syncwarp();  // the next direction rewrites the plus faces
  }

  // ---- update and the fused CFL minimum ----
  long long ord = kOrdMax;
  bool bad = false;
  if (live) {
    const double dx = g.len[g.lvl[c]];
    const double k = sc[inst].dt * nr_rcp(dx);
    double qo[NV];
    if (MODE != 0) {
#pragma unroll
      for (int v = 0; v < NV; ++v) qo[v] = out[v * ld + c];
    }
    double o[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = rk_combine<MODE>(MODE == 0 ? 0.0 : qo[v], __ldg(qin + v * ld + c), k * acc[v]);
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

template <class R, int ND>
constexpr size_t smem_for() {
  return sizeof(WarpSmem<R, ND>) * (kBlock / 32);
}

template <int ND, class R, int MODE, bool HANG, bool FUSE>
int prepare_one() {
  auto k = k_stage_ausm_warp<ND, R, MODE, HANG, FUSE>;
  constexpr size_t smem = smem_for<R, ND>();
  if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kBlock, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}
template <int ND, class R, int MODE, bool HANG>
int prepare_f() {
  return std::min(prepare_one<ND, R, MODE, HANG, false>(), prepare_one<ND, R, MODE, HANG, true>());
}
template <int ND, class R, int MODE>
int prepare_h() {
  return std::min(prepare_f<ND, R, MODE, false>(), prepare_f<ND, R, MODE, true>());
}
template <int ND, class R>
int prepare_m() {
  return std::min(std::min(prepare_h<ND, R, 0>(), prepare_h<ND, R, 2>()),
                  std::min(prepare_h<ND, R, 3>(), prepare_h<ND, R, 4>()));
}

template <int ND, class R, int MODE, bool HANG>
void launch_f(bool fuse, const double* qin, double* out, const Geometry& g, const PhysConst& pc, const Scalars* sc,
              long long* dtmin, cudaStream_t st) {
  constexpr size_t smem = smem_for<R, ND>();
  const unsigned grid = (unsigned)std::max<long long>(1, (g.n_int + kBlock - 1) / kBlock);
  if (fuse) k_stage_ausm_warp<ND, R, MODE, HANG, true><<<grid, kBlock, smem, st>>>(qin, out, g, pc, sc, dtmin);
  else k_stage_ausm_warp<ND, R, MODE, HANG, false><<<grid, kBlock, smem, st>>>(qin, out, g, pc, sc, dtmin);
}
template <int ND, class R, int MODE>
void launch_h(bool hang, bool fuse, const double* qin, double* out, const Geometry& g, const PhysConst& pc,
              const Scalars* sc, long long* dtmin, cudaStream_t st) {
  if (hang) launch_f<ND, R, MODE, true>(fuse, qin, out, g, pc, sc, dtmin, st);
  else launch_f<ND, R, MODE, false>(fuse, qin, out, g, pc, sc, dtmin, st);
}
template <int ND, class R>
void launch_m(int mode, bool hang, bool fuse, const double* qin, double* out, const Geometry& g, const PhysConst& pc,
              const Scalars* sc, long long* dtmin, cudaStream_t st) {
  switch (mode) {
    case 0: launch_h<ND, R, 0>(hang, fuse, qin, out, g, pc, sc, dtmin, st); break;
    case 2: launch_h<ND, R, 2>(hang, fuse, qin, out, g, pc, sc, dtmin, st); break;
    case 3: launch_h<ND, R, 3>(hang, fuse, qin, out, g, pc, sc, dtmin, st); break;
    default: launch_h<ND, R, 4>(hang, fuse, qin, out, g, pc, sc, dtmin, st); break;
  }
}

}  // namespace

size_t warp_smem_bytes(int nd, bool mixed) {
  if (nd == 2) return mixed ? smem_for<float, 2>() : smem_for<double, 2>();
  return mixed ? smem_for<float, 3>() : smem_for<double, 3>();
}

int warp_prepare(int nd, bool mixed) {
  if (nd == 2) return mixed ? prepare_m<2, float>() : prepare_m<2, double>();
  return mixed ? prepare_m<3, float>() : prepare_m<3, double>();
}

void warp_stage(int nd, bool mixed, int mode, bool hang, bool fuse, const double* qin, double* out,
                const Geometry& g, const PhysConst& pc, const Scalars* sc, long long* dtmin, cudaStream_t st) {
  if (nd == 2) {
    if (mixed) launch_m<2, float>(mode, hang, fuse, qin, out, g, pc, sc, dtmin, st);
    else launch_m<2, double>(mode, hang, fuse, qin, out, g, pc, sc, dtmin, st);
  } else {
    if (mixed) launch_m<3, float>(mode, hang, fuse, qin, out, g, pc, sc, dtmin, st);
    else launch_m<3, double>(mode, hang, fuse, qin, out, g, pc, sc, dtmin, st);
  }
}

}  // namespace h3c
