// h3c_stage_halo.cu -- the Euler/AUSM stage on Morton tiles staged into shared
// memory by bulk copies, and the host tables it reads.
//
// hom3's step evaluates, for every cell, the 2 nd face fluxes of num_flux
// (src/solver/fv/solver.hpp:440-460) with the AUSM flux
// (src/solver/fv/euler/physics.hpp:276-325) and applies the explicit update of
// evolve (solver.hpp:470-494).  Here one block owns a 256-cell tile of the
// Morton order at a time (persistent blocks take tiles round-robin):
//
//  1. copies: one thread issues cp.async.bulk copies of the tile's state
//     columns, neighbour-slot columns and level bytes into shared memory
//     (completion counted on an mbarrier); every thread issues 8-byte
//     cp.async copies of the state of its share of the tile's halo cells
//     (the cells outside the tile that the tile's faces read, listed at
//     set-up).  The next tile's copies are issued as soon as the current
//     tile's copies have been turned into face states, so they are in flight
//     while the current tile's fluxes are computed.
//  2. face states: theta = a (rho u, rho, rho E + p), p and the Mach numbers
//     of every tile and halo cell, computed once into shared memory
//     (theta_, euler/physics.hpp:315-325).
//  3. fluxes, direction by direction: each cell evaluates its plus face and
//     publishes it; a cell takes its minus face from the tile neighbour that
//     published it (a same-level face, linked both ways), or evaluates it
//     itself (tile border, coarse/fine face).  Every face flux is the same
//     F(l, r) evaluation hom3 performs, and each cell sums
//     F(minus) - F(plus) direction by direction in hom3's order, so results
//     are bit-identical to the per-cell evaluation.
//  4. update and the fused CFL minimum of the next step.
//
// No branch of a warp reads global memory for a neighbour: the per-lane
// divergent neighbour loads of the register-tiled kernel (k_stage_ausm) are
// replaced by the cooperative, coalesced halo copies of step 1.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <thread>
#include <vector>

#define H3C_DEVICE_FUNCTIONS_ONLY
#include "fv_kernels.cuh"
#include "stage_halo.hpp"
#include "async_copy.cuh"

namespace h3c {

template <class R, int ND>
__host__ __device__ constexpr size_t halo_layout_bytes(int hmax) {
  // mbarrier (16) | landing [nv][256 + hmax] f64, later the published plus fluxes [2][nv][256] f64 |
  // tile face states [nv + 1 + nd][256] R | halo face states [nv + 2][hmax] R |
  // neighbour slots [2nd][256] u16 | levels [256] u8
  return 16 +
         (8 * (size_t)(ND + 2) * (kHaloTile + hmax) > 16 * (size_t)(ND + 2) * kHaloTile
              ? 8 * (size_t)(ND + 2) * (kHaloTile + hmax)
              : 16 * (size_t)(ND + 2) * kHaloTile) +
         sizeof(R) * (size_t)(2 * ND + 3) * kHaloTile + sizeof(R) * (size_t)(ND + 4) * hmax +
         2 * (size_t)(2 * ND) * kHaloTile + (size_t)kHaloTile;
}

// Face state of a cell from its state q: theta = a (rho u, rho, rho E + p),
// p and the Mach numbers, the arithmetic of k_stage_ausm's face states.
template <class R, int ND>
__device__ __forceinline__ void face_state_of(const double* q, R gamma, R gm1, R* th, R& p, R* M) {
  Prim<R, ND> P;
#pragma unroll
  for (int v = 0; v < ND + 2; ++v) P.q[v] = (R)q[v];
  make_prim<R, ND>(P, gamma, gm1);
#pragma unroll
  for (int v = 0; v < ND + 1; ++v) th[v] = P.q[v] * P.a;
  th[ND + 1] = (P.q[ND + 1] + P.p) * P.a;
  p = P.p;
#pragma unroll
  for (int d = 0; d < ND; ++d) M[d] = P.M[d];
}

template <int ND, class R, int MODE, bool HANG, bool FUSE>
__global__ void __launch_bounds__(kHaloTile, 3)
    k_stage_halo(const double* __restrict__ qin, double* out, Geometry g, HaloGeom hg, PhysConst pc,
                 const Scalars* __restrict__ sc, long long* dtmin, int* status) {
  constexpr int NV = ND + 2, NP = 2 * ND, NS = 1 << (ND - 1), TB = kHaloTile;
  constexpr int KH = kHaloMaxSlots / kHaloTile;  // halo entries one thread copies, at most
  constexpr int NFT = 2 * ND + 3;                // tile face-state rows: th[nv], p, M[nd]
  constexpr double W = ND == 2 ? 0.5 : 0.25;
  const int HM = hg.hmax;  // halo entries held in shared memory; later ones are read from global memory
  const int S = TB + HM;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem);
  double* land = reinterpret_cast<double*>(smem + 16);  // [NV][S]; after the face states: fluxes [2][NV][TB]
  const size_t uni = (size_t)NV * S > (size_t)2 * NV * TB ? (size_t)NV * S : (size_t)2 * NV * TB;
  R* fst = reinterpret_cast<R*>(land + uni);            // [NFT][TB]
  R* fsh = fst + (size_t)NFT * TB;                      // [NV + 2][HM]
  unsigned short* ln = reinterpret_cast<unsigned short*>(fsh + (size_t)(NV + 2) * HM);  // [NP][TB]
  unsigned char* ll = reinterpret_cast<unsigned char*>(ln + NP * TB);                  // [TB]
  double* fx = land;
  __shared__ double slen[kMaxLevels];
  const int tid = threadIdx.x;
  const long long ld = g.ld;
  const R gamma = (R)pc.gamma, gm1 = (R)pc.gm1;

  long long tile = blockIdx.x;
  if (tile >= g.ntiles) return;
  if (tid < kMaxLevels) slen[tid] = g.len[tid];
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();

  // the halo entries of tile t this thread copies; returns the tile's entry count and its offset
  auto fetch_ids = [&](long long t, int* hid, int& o0) -> int {
    o0 = __ldg(hg.halo_off + t);
    const int nh = __ldg(hg.halo_off + t + 1) - o0;
#pragma unroll
    for (int k = 0; k < KH; ++k) {
      const int h = tid + k * TB;
      hid[k] = (h < nh && h < HM) ? __ldg(hg.halo_ids + o0 + h) : 0;
    }
    return nh;
  };
  // the copies of tile t: its state, neighbour slots and levels by bulk copy,
  // the state of its first HM halo entries by 8-byte asynchronous copies
  auto issue = [&](long long t, const int* hid, int nh) {
    if (tid == 0) {
      const long long c0 = t * TB;
      const long long te = min(c0 + TB, instance_end(g, tile_instance(g, t)));
      const unsigned ncp = (unsigned)((te - c0 + 15) & ~15LL);  // whole 16-cell groups: 16-byte multiples
      fence_proxy_async();
      mbar_expect_tx(bar, ncp * (8u * NV + 2u * NP + 1u));
#pragma unroll
      for (int v = 0; v < NV; ++v) bulk_g2s(land + (size_t)v * S, qin + v * ld + c0, ncp * 8u, bar);
#pragma unroll
      for (int p = 0; p < NP; ++p) bulk_g2s(ln + p * TB, hg.lnb + p * ld + c0, ncp * 2u, bar);
      bulk_g2s(ll, g.lvl + c0, ncp, bar);
    }
#pragma unroll
    for (int k = 0; k < KH; ++k) {
      const int h = tid + k * TB;
      if (h < nh && h < HM) {
        const long long n = hid[k] & kHaloCellMask;
#pragma unroll
        for (int v = 0; v < NV; ++v) cp_async8(land + (size_t)v * S + TB + h, qin + v * ld + n);
      }
    }
    cp_async_commit();
  };

  int hid[KH], hid_n[KH];
  int o0 = 0, o0_n = 0;
  int nh = fetch_ids(tile, hid, o0);

  for (int it = 0; tile < g.ntiles; tile += gridDim.x, ++it) {
    issue(tile, hid, nh);
    const long long next = tile + gridDim.x;
    int nh_n = 0;
    if (next < g.ntiles) nh_n = fetch_ids(next, hid_n, o0_n);  // consumed by the next iteration's copies
    const long long c0 = tile * TB, c = c0 + tid;
    const int inst = tile_instance(g, tile);
    const long long te = min(c0 + (long long)TB, instance_end(g, inst));
    const bool live = c < te;
    const int gbase = HANG ? __ldg(hg.grp_off + tile) : 0;
    double qo[NV];
    if (MODE != 0 && live) {
#pragma unroll
      for (int v = 0; v < NV; ++v) qo[v] = out[v * ld + c];
    }

    // ---- this tile's copies ----
    const bool ok = mbar_wait_bounded(bar, (unsigned)(it & 1));
    cp_async_wait_all();
    if (!__syncthreads_and(ok)) {
      if (tid == 0) atomicOr(status, kStatusTimeout);
      return;
    }

    // ---- face states: the own cell's (also kept in registers), the halo entries' along their direction ----
    // (the cell's own state is read again from global memory at the update,
    // not held in registers across the face loops)
    R thc[NV], pcell = R(0), Mc[ND];
    if (live) {
      double qc[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) qc[v] = land[(size_t)v * S + tid];
      face_state_of<R, ND>(qc, gamma, gm1, thc, pcell, Mc);
#pragma unroll
      for (int v = 0; v < NV; ++v) fst[v * TB + tid] = thc[v];
      fst[NV * TB + tid] = pcell;
#pragma unroll
      for (int d = 0; d < ND; ++d) fst[(NV + 1 + d) * TB + tid] = Mc[d];
    }
#pragma unroll
    for (int k = 0; k < KH; ++k) {
      const int h = tid + k * TB;
      if (h < nh && h < HM) {
        double qh[NV];
        R th[NV], ph, Mh[ND];
#pragma unroll
        for (int v = 0; v < NV; ++v) qh[v] = land[(size_t)v * S + TB + h];
        face_state_of<R, ND>(qh, gamma, gm1, th, ph, Mh);
        const int dir = hid[k] >> kHaloDirShift;
        R Md = Mh[0];
#pragma unroll
        for (int d = 1; d < ND; ++d) Md = dir == d ? Mh[d] : Md;
#pragma unroll
        for (int v = 0; v < NV; ++v) fsh[v * HM + h] = th[v];
        fsh[NV * HM + h] = ph;
        fsh[(NV + 1) * HM + h] = Md;
      }
    }
    __syncthreads();  // face states complete; the landing area becomes the flux buffers

    // the face state of slot s along d: a tile cell, a shared halo entry, or an overflow entry read from global memory
    auto load_fs = [&](int s, int d, FaceState<R, ND>& F) {
      if (s < TB) {
#pragma unroll
        for (int v = 0; v < NV; ++v) F.th[v] = fst[v * TB + s];
        F.p = fst[NV * TB + s];
        F.M = fst[(NV + 1 + d) * TB + s];
      } else if (s - TB < HM) {
        const int h = s - TB;
#pragma unroll
        for (int v = 0; v < NV; ++v) F.th[v] = fsh[v * HM + h];
        F.p = fsh[NV * HM + h];
        F.M = fsh[(NV + 1) * HM + h];
      } else {
        const int n = __ldg(hg.halo_ids + o0 + (s - TB)) & kHaloCellMask;
        face_state_global<R, ND>(F, qin, ld, n, d, gamma, gm1);
      }
    };

    // ---- fluxes, direction by direction ----
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      double* X = fx + (d & 1) * NV * TB;
      FaceState<R, ND> Fc;
#pragma unroll
      for (int v = 0; v < NV; ++v) Fc.th[v] = thc[v];
      Fc.p = pcell;
      Fc.M = Mc[d];
      if (live) {
        const int p = ln[(2 * d + 1) * TB + tid];
        double fp[NV];
        if (!HANG || !(p & kGroupBit)) {
          FaceState<R, ND> Fn;
          load_fs(p, d, Fn);
          R f[NV];
          ausm_face<R, ND>(Fc, Fn, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fp[v] = (double)f[v];
        } else {
          const unsigned short* gsl = hg.grp + (size_t)(gbase + (p & ~kGroupBit)) * NS;
#pragma unroll
          for (int j = 0; j < NS; ++j) {
            FaceState<R, ND> Fn;
            load_fs(__ldg(gsl + j), d, Fn);
            R f[NV];
            ausm_face<R, ND>(Fc, Fn, d, f);
#pragma unroll
            for (int v = 0; v < NV; ++v) fp[v] = j == 0 ? (double)f[v] : fp[v] + (double)f[v];
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) fp[v] = __dmul_rn(W, fp[v]);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) X[v * TB + tid] = fp[v];
      }
      __syncthreads();  // plus fluxes of direction d published
      if (live) {
        const int m = ln[(2 * d) * TB + tid];
        double fm[NV];
        if (m < TB && ln[(2 * d + 1) * TB + m] == tid) {
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = X[v * TB + m];
        } else if (!HANG || !(m & kGroupBit)) {
          FaceState<R, ND> Fn;
          load_fs(m, d, Fn);
          R f[NV];
          ausm_face<R, ND>(Fn, Fc, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = (double)f[v];
        } else {
          const unsigned short* gsl = hg.grp + (size_t)(gbase + (m & ~kGroupBit)) * NS;
#pragma unroll
          for (int j = 0; j < NS; ++j) {
            FaceState<R, ND> Fn;
            load_fs(__ldg(gsl + j), d, Fn);
            R f[NV];
            ausm_face<R, ND>(Fn, Fc, d, f);
#pragma unroll
            for (int v = 0; v < NV; ++v) fm[v] = j == 0 ? (double)f[v] : fm[v] + (double)f[v];
          }
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = __dmul_rn(W, fm[v]);
        }
        // the own plus flux as published (a rounded value: no FMA with this sum, as in the per-lane kernel)
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fm[v] - X[v * TB + tid]);
      }
      // the buffer X is written again two directions later, after the next barrier
    }

    // ---- update and the next step's CFL minimum ----
    long long ord = kOrdMax;
    bool bad = false;
    if (live) {
      const double dx = slen[ll[tid]];
      const double dt = sc[inst].dt;
      const double k = dt / dx;
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
      block_min_atomic(ord, per_instance(dtmin, inst));
    }
    __syncthreads();  // the shared buffers are rewritten by the next tile's copies
    nh = nh_n;
    o0 = o0_n;
#pragma unroll
    for (int k = 0; k < KH; ++k) hid[k] = hid_n[k];
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
bool halo_build(int nd, long long ld, long long ntiles, const std::vector<long long>& tile_end, const int* nbr,
                const int* sub, long long nsub, HaloHost& H) {
  const int NP = 2 * nd, NS = 1 << (nd - 1), TB = kHaloTile;
  if (ld >= (1LL << kHaloDirShift)) return false;  // cell ids share their word with the direction
  H.lnb.assign((size_t)NP * ld, 0);
  std::vector<std::vector<int>> halo(ntiles);
  std::vector<std::vector<unsigned short>> grp(ntiles);
  std::atomic<bool> ok{true};
  auto work = [&](long long t0, long long t1) {
    std::vector<long long> tmp;  // (cell << 2) | direction
    for (long long t = t0; t < t1 && ok.load(std::memory_order_relaxed); ++t) {
      const long long c0 = t * TB, ce = tile_end[t];
      auto outside = [&](long long v) { return v < c0 || v >= ce; };
      tmp.clear();
      for (long long c = c0; c < ce; ++c)
        for (int p = 0; p < NP; ++p) {
          const long long v = nbr[p * ld + c];
          const int dir = p >> 1;
          if (v >= 0) {
            if (outside(v)) tmp.push_back((v << 2) | dir);
          } else if (v <= -2) {
            const long long k = -v - 2;
            for (int j = 0; j < NS; ++j) {
              const long long sv = sub[j * nsub + k];
              if (outside(sv)) tmp.push_back((sv << 2) | dir);
            }
          }
        }
      std::sort(tmp.begin(), tmp.end());
      tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
      if ((long long)tmp.size() + TB >= kGroupBit) {  // slots are 15-bit
        ok = false;
        break;
      }
      auto slot = [&](long long v, int dir) -> unsigned short {
        if (!outside(v)) return (unsigned short)(v - c0);
        return (unsigned short)(TB + (std::lower_bound(tmp.begin(), tmp.end(), (v << 2) | dir) - tmp.begin()));
      };
      std::vector<unsigned short>& G = grp[t];
      for (long long c = c0; c < ce; ++c)
        for (int p = 0; p < NP; ++p) {
          const long long v = nbr[p * ld + c];
          const int dir = p >> 1;
          unsigned short e = 0;
          if (v >= 0) {
            e = slot(v, dir);
          } else if (v <= -2) {
            const long long k = -v - 2;
            const size_t gi = G.size() / NS;
            if (gi >= kGroupBit) {
              ok = false;
              break;
            }
            e = (unsigned short)(kGroupBit | gi);
            for (int j = 0; j < NS; ++j) G.push_back(slot(sub[j * nsub + k], dir));
          }
          H.lnb[(size_t)p * ld + c] = e;
        }
      std::vector<int>& hl = halo[t];
      hl.resize(tmp.size());
      for (size_t i = 0; i < tmp.size(); ++i) hl[i] = (int)((tmp[i] >> 2) | ((tmp[i] & 3) << kHaloDirShift));
    }
  };
  const int nthr = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 16));
  std::vector<std::thread> pool;
  const long long per = (ntiles + nthr - 1) / nthr;
  for (int i = 0; i < nthr; ++i) {
    const long long a = i * per, b = std::min(ntiles, a + per);
    if (a < b) pool.emplace_back(work, a, b);
  }
  for (auto& th : pool) th.join();
  if (!ok) return false;
  H.off.assign(ntiles + 1, 0);
  H.goff.assign(ntiles + 1, 0);
  size_t nids = 0, ngrp = 0;
  int mx = 0;
  for (long long t = 0; t < ntiles; ++t) {
    nids += halo[t].size();
    ngrp += grp[t].size() / NS;
    mx = std::max(mx, (int)halo[t].size());
    H.off[t + 1] = (int)nids;
    H.goff[t + 1] = (int)ngrp;
  }
  H.ids.resize(std::max<size_t>(nids, 1));
  H.grp.resize(std::max<size_t>(ngrp * NS, 1));
  for (long long t = 0; t < ntiles; ++t) {
    std::copy(halo[t].begin(), halo[t].end(), H.ids.begin() + H.off[t]);
    std::copy(grp[t].begin(), grp[t].end(), H.grp.begin() + (size_t)H.goff[t] * NS);
  }
  H.max_halo = mx;
  H.mean_halo = ntiles ? (double)nids / ntiles : 0.0;
  H.hmax = std::max(32, (mx + 31) / 32 * 32);  // the caller may hold fewer in shared memory (halo_slots_for)
  return true;
}

int halo_slots_for(int nd, bool mixed, int max_halo, int blocks_per_sm) {
  // shared memory of an SM (228 KB) less 1 KB reserved per block and the static arrays
  const size_t budget = (size_t)233472 / blocks_per_sm - 1024 - 512;
  int hm = std::min(kHaloMaxSlots, std::max(32, (max_halo + 31) / 32 * 32));
  while (hm > 32 && halo_smem_bytes(nd, mixed, hm) > budget) hm -= 32;
  return hm;
}

size_t halo_smem_bytes(int nd, bool mixed, int hmax) {
  if (nd == 2) return mixed ? halo_layout_bytes<float, 2>(hmax) : halo_layout_bytes<double, 2>(hmax);
  return mixed ? halo_layout_bytes<float, 3>(hmax) : halo_layout_bytes<double, 3>(hmax);
}

namespace {

template <int ND, class R, int MODE, bool HANG, bool FUSE>
int prepare_one(size_t smem) {
  auto k = k_stage_halo<ND, R, MODE, HANG, FUSE>;
  // the opt-in limit (less the kernel's static arrays), not this grid's size: several solvers
  // share the kernel and its attribute
  int dev = 0, optin = 0;
  cudaFuncAttributes fa{};
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaFuncGetAttributes(&fa, k) != cudaSuccess || (size_t)optin < smem + fa.sharedSizeBytes ||
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes) !=
          cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kHaloTile, smem) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nb;
}
template <int ND, class R, int MODE, bool HANG>
int prepare_f(size_t smem) {
  return std::min(prepare_one<ND, R, MODE, HANG, false>(smem), prepare_one<ND, R, MODE, HANG, true>(smem));
}
template <int ND, class R, int MODE>
int prepare_h(size_t smem) {
  return std::min(prepare_f<ND, R, MODE, false>(smem), prepare_f<ND, R, MODE, true>(smem));
}
template <int ND, class R>
int prepare_m(size_t smem) {
  return std::min(std::min(prepare_h<ND, R, 0>(smem), prepare_h<ND, R, 2>(smem)),
                  std::min(prepare_h<ND, R, 3>(smem), prepare_h<ND, R, 4>(smem)));
}

template <int ND, class R, int MODE, bool HANG, bool FUSE>
void launch_one(const double* qin, double* out, const Geometry& g, const HaloGeom& h, const PhysConst& pc,
                const Scalars* sc, long long* dtmin, int* status, int grid, size_t smem, cudaStream_t st) {
  k_stage_halo<ND, R, MODE, HANG, FUSE><<<grid, kHaloTile, smem, st>>>(qin, out, g, h, pc, sc, dtmin, status);
}
template <int ND, class R, int MODE, bool HANG>
void launch_f(bool fuse, const double* qin, double* out, const Geometry& g, const HaloGeom& h, const PhysConst& pc,
              const Scalars* sc, long long* dtmin, int* status, int grid, size_t smem, cudaStream_t st) {
  if (fuse) launch_one<ND, R, MODE, HANG, true>(qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
  else launch_one<ND, R, MODE, HANG, false>(qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
}
template <int ND, class R, int MODE>
void launch_h(bool hang, bool fuse, const double* qin, double* out, const Geometry& g, const HaloGeom& h,
              const PhysConst& pc, const Scalars* sc, long long* dtmin, int* status, int grid, size_t smem,
              cudaStream_t st) {
  if (hang) launch_f<ND, R, MODE, true>(fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
  else launch_f<ND, R, MODE, false>(fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
}
template <int ND, class R>
void launch_m(int mode, bool hang, bool fuse, const double* qin, double* out, const Geometry& g, const HaloGeom& h,
              const PhysConst& pc, const Scalars* sc, long long* dtmin, int* status, int grid, size_t smem,
              cudaStream_t st) {
  switch (mode) {
    case 0: launch_h<ND, R, 0>(hang, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st); break;
    case 2: launch_h<ND, R, 2>(hang, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st); break;
    case 3: launch_h<ND, R, 3>(hang, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st); break;
    default: launch_h<ND, R, 4>(hang, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st); break;
  }
}

}  // namespace

int halo_prepare(int nd, bool mixed, size_t smem) {
  if (nd == 2) return mixed ? prepare_m<2, float>(smem) : prepare_m<2, double>(smem);
  return mixed ? prepare_m<3, float>(smem) : prepare_m<3, double>(smem);
}

void halo_stage(int nd, bool mixed, int mode, bool hang, bool fuse, const double* qin, double* out,
                const Geometry& g, const HaloGeom& h, const PhysConst& pc, const Scalars* sc, long long* dtmin,
                int* status, int grid, size_t smem, cudaStream_t st) {
  if (nd == 2) {
    if (mixed) launch_m<2, float>(mode, hang, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
    else launch_m<2, double>(mode, hang, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
  } else {
    if (mixed) launch_m<3, float>(mode, hang, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
    else launch_m<3, double>(mode, hang, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
  }
}

}  // namespace h3c
