// h3c_stage_cns.cu -- the compressible Navier-Stokes stage on Morton tiles
// staged into shared memory, and its host tables.
//
// hom3's CNS flux is AUSM plus a three-point viscous flux
// (src/solver/fv/cns/physics.hpp:155-161, 305-338) whose transverse
// derivatives average the central slopes of the two face cells
// (surface_slope / slope, src/solver/fv/solver.hpp:596-678).  The per-cell
// kernel evaluates every face twice and reads slopes that a separate pass
// wrote for every cell.  Here a block owns a 256-cell tile at a time:
//
//  1. copies (as in h3c_stage_halo.cu): the tile's state and neighbour slots
//     by cp.async.bulk, the halo cells' state by cp.async: the first layer
//     (the tile's face neighbours) and the second (the cells the first
//     layer's slopes read: edge-diagonal neighbours of the tile);
//  2. primitive variables and slopes of the tile and first-layer cells,
//     computed once into shared memory (a ghost's slopes -- its boundary or
//     periodic partner cell's, with the walls' sign rule -- from a ghost-only
//     slope pass run before the stage);
//  3. fluxes direction by direction, each face once (the plus face is
//     published for the neighbour's minus face, as in the Euler tile kernel);
//     every face is the same F(l, r) evaluation and each cell sums
//     F(minus) - F(plus) in hom3's order, so the results are bit-identical to
//     the per-cell kernel;
//  4. the update and the fused CFL minimum.
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

// Slopes of the ghost cells: the ghost branch of k_slopes (a ghost takes its
// boundary cell's central slope, a periodic ghost its partner's, with the
// walls' sign flip of tangential velocity slopes: boundary_condition.hpp:63-67,
// cns/boundary_conditions.hpp:143-147, 230-234), same arithmetic.
template <int ND>
__global__ void __launch_bounds__(kBlock) k_ghost_slopes(const double* __restrict__ q, Geometry g, GhostTables gt,
                                                         double* __restrict__ gsl, long long ngl) {
  constexpr int NV = ND + 2;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gt.ng) return;
  const long long ld = g.ld;
  const BcParam& B = gt.bcs[gt.bc_own[i]];
  const long long b = B.kind == BC_PERIODIC ? gt.partner[i] : gt.bndry[i];
  if (b < 0) return;
  const int dg = gt.pos[i] >> 1;
  const bool wall = B.wall != 0;
  const double h2 = 2. * g.len[g.lvl[b]];
#pragma unroll
  for (int sd = 0; sd < ND; ++sd) {
    const int m = g.nbr[(2 * sd) * ld + b];
    const int p = g.nbr[(2 * sd + 1) * ld + b];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double s = (__ldg(q + v * ld + p) - __ldg(q + v * ld + m)) / h2;
      if (wall && v < ND && sd != dg) s = -s;
      gsl[(sd * NV + v) * ngl + i] = s;
    }
  }
}

// The slopes a face reads: the transverse slopes of momentum and density
// (cns/physics.hpp:305-338 reads no energy slope), [sd][v] for v <= nd.
template <int ND> constexpr int kCnsSlopeVars = ND + 1;

// Shared memory of one block.  In FP64 the copies land in the primitive
// rows themselves (the tile and first-layer cells' states are the first nv
// rows of the primitives) and only the second layer has a landing area of
// its own; in FP32 (R = float) the FP64 states land in a separate area.
//   mbarrier (16) | [FP32: landing [nv][S] f64] | primitives [nv + nd + 2][S1] R |
//   [FP64: second-layer landing [nv][S - S1] f64] | slopes [nd (nd + 1)][S1] R |
//   plus fluxes [nv][256] f64 | neighbour slots [2][2nd][256] u16
template <class R, int ND>
__host__ __device__ constexpr bool cns_land_in_prims() {
  return sizeof(R) == sizeof(double);
}
template <class R, int ND>
__host__ __device__ constexpr size_t cns_layout_bytes(int hmax, int h1max) {
  return 16 + (cns_land_in_prims<R, ND>() ? 8 * (size_t)(ND + 2) * (hmax - h1max) : 8 * (size_t)(ND + 2) * (kHaloTile + hmax)) +
         sizeof(R) * (size_t)(2 * ND + 4 + ND * kCnsSlopeVars<ND>) * (kHaloTile + h1max) + 8 * (size_t)(ND + 2) * kHaloTile +
         2 * 2 * (size_t)(2 * ND) * kHaloTile;
}

#ifndef H3C_CNS_MINB
#define H3C_CNS_MINB 2  // blocks per SM the CNS tile kernel is register-budgeted for
#endif

template <int ND, class R, int MODE, bool FUSE>
__global__ void __launch_bounds__(kHaloTile, H3C_CNS_MINB)
    k_stage_cns_halo(const double* __restrict__ qin, double* out, Geometry g, CnsHaloGeom ch, PhysConst pc,
                     const Scalars* __restrict__ sc, long long* dtmin, int* status) {
  constexpr int NV = ND + 2, NP = 2 * ND, TB = kHaloTile;
  constexpr int NPR = NV + ND + 2;  // q[nv], M[nd], p, a
  constexpr int SV = kCnsSlopeVars<ND>;
  constexpr int NSL = ND * SV;      // slopes [sd][v], v <= nd
  constexpr int KH = kHaloMaxSlots / kHaloTile;
  constexpr bool LIP = cns_land_in_prims<R, ND>();
  const HaloGeom& hg = ch.h;
  const int S = TB + hg.hmax, S1 = TB + ch.h1max, S2 = S - S1;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem);
  double* land = reinterpret_cast<double*>(smem + 16);                           // FP32: [NV][S]
  R* pr = reinterpret_cast<R*>(land + (LIP ? 0 : (size_t)NV * S));              // [NPR][S1]
  double* land2 = reinterpret_cast<double*>(pr + (size_t)NPR * S1);             // FP64: [NV][S2]
  R* sl = reinterpret_cast<R*>(land2 + (LIP ? (size_t)NV * S2 : 0));             // [NSL][S1]
  double* fx = reinterpret_cast<double*>(sl + (size_t)NSL * S1);                  // [NV][TB]
  unsigned short* ln = reinterpret_cast<unsigned short*>(fx + NV * TB);           // [2][NP][TB]
  const int tid = threadIdx.x;
  const long long ld = g.ld;
  const R gamma = (R)pc.gamma, gm1 = (R)pc.gm1;
  const double h = g.len[0];  // single-level grid
  const double h2 = 2. * h;
  const R hr = (R)h;

  // where the state of slot s (tile, first or second layer) lands
  auto qslot = [&](int v, int s) -> double* {
    if (LIP) return s < S1 ? reinterpret_cast<double*>(pr) + (size_t)v * S1 + s : land2 + (size_t)v * S2 + (s - S1);
    return land + (size_t)v * S + s;
  };

  long long tile = blockIdx.x;
  if (tile >= g.ntiles) return;
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncthreads();

  // halo cells (layer 1 then layer 2) of tile t this thread copies
  auto fetch_ids = [&](long long t, int* hid, int& o0, int& nh1) -> int {
    o0 = __ldg(hg.halo_off + t);
    const int nh = __ldg(hg.halo_off + t + 1) - o0;
    nh1 = __ldg(ch.h1end + t) - o0;
#pragma unroll
    for (int k = 0; k < KH; ++k) {
      const int hh = tid + k * TB;
      hid[k] = hh < nh ? __ldg(hg.halo_ids + o0 + hh) : 0;
    }
    return nh;
  };
  auto issue = [&](long long t, int buf, const int* hid, int nh) {
    if (tid == 0) {
      const long long c0 = t * TB;
      const long long te = min(c0 + TB, instance_end(g, tile_instance(g, t)));
      const unsigned ncp = (unsigned)((te - c0 + 15) & ~15LL);
      fence_proxy_async();
      mbar_expect_tx(bar, ncp * (8u * NV + 2u * NP));
#pragma unroll
      for (int v = 0; v < NV; ++v) bulk_g2s(qslot(v, 0), qin + v * ld + c0, ncp * 8u, bar);
#pragma unroll
      for (int p = 0; p < NP; ++p) bulk_g2s(ln + (buf * NP + p) * TB, hg.lnb + p * ld + c0, ncp * 2u, bar);
    }
#pragma unroll
    for (int k = 0; k < KH; ++k) {
      const int hh = tid + k * TB;
      if (hh < nh) {
        const long long n = hid[k];
#pragma unroll
        for (int v = 0; v < NV; ++v) cp_async8(qslot(v, TB + hh), qin + v * ld + n);
      }
    }
    cp_async_commit();
  };
  // primitive variables of a state (make_prim, euler/physics.hpp:83-125) into slot s;
  // in FP64 the state rows already hold q
  auto store_prim = [&](const double* q, int s) {
    Prim<R, ND> P;
#pragma unroll
    for (int v = 0; v < NV; ++v) P.q[v] = (R)q[v];
    make_prim<R, ND>(P, gamma, gm1);
    if (!LIP) {
#pragma unroll
      for (int v = 0; v < NV; ++v) pr[v * S1 + s] = P.q[v];
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) pr[(NV + d) * S1 + s] = P.M[d];
    pr[(NV + ND) * S1 + s] = P.p;
    pr[(NV + ND + 1) * S1 + s] = P.a;
  };
  auto load_prim_s = [&](int s, int d, Prim<R, ND>& P) {
#pragma unroll
    for (int v = 0; v < NV; ++v) P.q[v] = pr[v * S1 + s];
#pragma unroll
    for (int e = 0; e < ND; ++e) P.M[e] = e == d ? pr[(NV + e) * S1 + s] : R(0);
#pragma unroll
    for (int e = 0; e < ND; ++e) P.u[e] = R(0);  // not read by the AUSM and viscous fluxes
    P.p = pr[(NV + ND) * S1 + s];
    P.a = pr[(NV + ND + 1) * S1 + s];
  };
  // the transverse slopes (sd != d, v <= nd) the viscous flux of direction d
  // reads, in the [sd][v] layout (v < nv) the viscous flux indexes
  auto load_slopes = [&](int s, int d, R* out_) {
#pragma unroll
    for (int sd = 0; sd < ND; ++sd)
#pragma unroll
      for (int v = 0; v < NV; ++v)
        out_[sd * NV + v] = (sd != d && v < SV) ? sl[(sd * SV + v) * S1 + s] : R(0);
  };
  // central slopes of slot s from its face-neighbour slots m, p along sd
  auto store_slopes = [&](int s, int sd, int m, int p) {
#pragma unroll
    for (int v = 0; v < SV; ++v) sl[(sd * SV + v) * S1 + s] = (R)((*qslot(v, p) - *qslot(v, m)) / h2);
  };
  // the face flux F(l, r): AUSM + three-point viscous (cns/physics.hpp:155-161)
  auto face = [&](const Prim<R, ND>& L, const Prim<R, ND>& Rt, const R* sL, const R* sR, int d, R* f) {
    ausm<R, ND>(L, Rt, d, f);
    R fv[NV];
    viscous<R, ND>(L, Rt, sL, sR, d, hr, pc, fv);
#pragma unroll
    for (int v = 0; v < NV; ++v) f[v] = f[v] + fv[v];
  };

  int hid[KH];
  int o0, nh1;
  int nh = fetch_ids(tile, hid, o0, nh1);
  issue(tile, 0, hid, nh);

  for (int it = 0; tile < g.ntiles; tile += gridDim.x, ++it) {
    const int buf = LIP ? 0 : (it & 1);
    const long long next = tile + gridDim.x;
    const long long c0 = tile * TB, c = c0 + tid;
    const int inst = tile_instance(g, tile);
    const long long te = min(c0 + (long long)TB, instance_end(g, inst));
    const bool live = c < te;
    if (MODE != 0 && live) prefetch_row_l2<NV>(out, ld, c);  // the in-place start state, read at the update

    const bool ok = mbar_wait_bounded(bar, (unsigned)(it & 1));
    cp_async_wait_all();
    if (!__syncthreads_and(ok)) {
      if (tid == 0) atomicOr(status, kStatusTimeout);
      return;
    }

    // ---- primitives and slopes of the own cell and the layer-1 cells ----
    const unsigned short* L = ln + buf * NP * TB;
    if (live) {
      double qc[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) qc[v] = *qslot(v, tid);
      store_prim(qc, tid);
#pragma unroll
      for (int sd = 0; sd < ND; ++sd) store_slopes(tid, sd, L[(2 * sd) * TB + tid], L[(2 * sd + 1) * TB + tid]);
    }
#pragma unroll
    for (int k = 0; k < KH; ++k) {
      const int hh = tid + k * TB;
      if (hh < nh1) {
        const int s = TB + hh;
        double qh[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) qh[v] = *qslot(v, s);
        store_prim(qh, s);
        const long long n = hid[k];
        if (n >= g.n_int) {  // a ghost: the ghost-slope pass
#pragma unroll
          for (int sd = 0; sd < ND; ++sd)
#pragma unroll
            for (int v = 0; v < SV; ++v)
              sl[(sd * SV + v) * S1 + s] = (R)__ldg(ch.gsl + (sd * NV + v) * ch.ngl + (n - g.n_int));
        } else {
#pragma unroll
          for (int sd = 0; sd < ND; ++sd) {
            const unsigned short m = __ldg(ch.hnb + (size_t)(o0 + hh) * NP + 2 * sd);
            const unsigned short p = __ldg(ch.hnb + (size_t)(o0 + hh) * NP + 2 * sd + 1);
            if (m != 0xffff) store_slopes(s, sd, m, p);
          }
        }
      }
    }
    __syncthreads();  // primitives and slopes complete

    int hid_n[KH], o0_n = 0, nh1_n = 0, nh_n = 0;
    if (!LIP) {  // FP32: the next tile lands in its own area while this one's fluxes run
      if (next < g.ntiles) {
        nh_n = fetch_ids(next, hid_n, o0_n, nh1_n);
        issue(next, buf ^ 1, hid_n, nh_n);
      }
    }

    // ---- fluxes, direction by direction ----
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      if (live) {
        Prim<R, ND> Pc, Pn;
        load_prim_s(tid, d, Pc);
        const int p = L[(2 * d + 1) * TB + tid];
        load_prim_s(p, d, Pn);
        R slc[ND * NV], sn[ND * NV];
        load_slopes(tid, d, slc);
        load_slopes(p, d, sn);
        R f[NV];
        face(Pc, Pn, slc, sn, d, f);
#pragma unroll
        for (int v = 0; v < NV; ++v) fx[v * TB + tid] = (double)f[v];
      }
      __syncthreads();  // this direction's plus faces are published
      if (live) {
        const int m = L[(2 * d) * TB + tid];
        double fm[NV];
        if (m < TB && L[(2 * d + 1) * TB + m] == tid) {
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = fx[v * TB + m];
        } else {
          Prim<R, ND> Pc, Pn;
          load_prim_s(tid, d, Pc);
          load_prim_s(m, d, Pn);
          R slc[ND * NV], sn[ND * NV];
          load_slopes(tid, d, slc);
          load_slopes(m, d, sn);
          R f[NV];
          face(Pn, Pc, sn, slc, d, f);
#pragma unroll
          for (int v = 0; v < NV; ++v) fm[v] = (double)f[v];
        }
        // the own plus flux as published (a rounded value: no FMA with this sum, as in the per-cell kernel)
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = acc[v] + (fm[v] - fx[v * TB + tid]);
      }
      __syncthreads();  // the next direction rewrites the plus faces
    }

    // ---- update and the next step's CFL minimum ----
    long long ord = kOrdMax;
    bool bad = false;
    if (live) {
      const double dt = sc[inst].dt;
      const double k = dt / h;
      double qc[NV], qo[NV];  // FP32: the landing area already holds the next tile
#pragma unroll
      for (int v = 0; v < NV; ++v) qc[v] = LIP ? *qslot(v, tid) : __ldg(qin + v * ld + c);
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
        const double cd = cell_dt<ND, CNS>(o, h, pc, nullptr, &bad);
        if (!isnan(cd)) ord = dbl_to_ord(cd);
      }
    }
    if (FUSE) {
      flag_bad_state(bad, sc, inst);
      block_min_atomic(ord, per_instance(dtmin, inst));
    }
    if (LIP) {  // FP64: the next tile lands where this one's primitives were
      __syncthreads();
      if (next < g.ntiles) {
        nh = fetch_ids(next, hid, o0, nh1);
        issue(next, 0, hid, nh);
      }
    } else {
      nh = nh_n;
      o0 = o0_n;
      nh1 = nh1_n;
#pragma unroll
      for (int k = 0; k < KH; ++k) hid[k] = hid_n[k];
    }
  }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
bool halo_build_cns(int nd, long long ld, long long n_int, long long ntiles, const std::vector<long long>& tile_end,
                    const int* nbr, CnsHaloHost& H) {
  const int NP = 2 * nd, TB = kHaloTile;
  H.base.lnb.assign((size_t)NP * ld, 0);
  std::vector<std::vector<int>> l1s(ntiles), l2s(ntiles);
  std::vector<std::vector<unsigned short>> hns(ntiles);
  std::atomic<bool> ok{true};
  auto work = [&](long long t0, long long t1) {
    std::vector<int> l1, l2;
    std::vector<unsigned char> need;
    for (long long t = t0; t < t1 && ok.load(std::memory_order_relaxed); ++t) {
      const long long c0 = t * TB, ce = tile_end[t];
      auto outside = [&](long long v) { return v < c0 || v >= ce; };
      l1.clear();
      for (long long c = c0; c < ce; ++c)
        for (int p = 0; p < NP; ++p) {
          const long long v = nbr[p * ld + c];
          if (v < 0) {  // CNS grids have no coarse/fine faces: every neighbour is a cell
            ok = false;
            return;
          }
          if (outside(v)) l1.push_back((int)v);
        }
      std::sort(l1.begin(), l1.end());
      l1.erase(std::unique(l1.begin(), l1.end()), l1.end());
      auto idx1 = [&](long long v) { return (long long)(std::lower_bound(l1.begin(), l1.end(), (int)v) - l1.begin()); };
      // slope directions each layer-1 cell needs: every direction but the ones it is a face neighbour across
      need.assign(l1.size(), 0);
      for (long long c = c0; c < ce; ++c)
        for (int p = 0; p < NP; ++p) {
          const long long v = nbr[p * ld + c];
          if (outside(v)) need[idx1(v)] |= (unsigned char)(((1 << nd) - 1) & ~(1 << (p >> 1)));
        }
      auto in_l1 = [&](long long v) { return std::binary_search(l1.begin(), l1.end(), (int)v); };
      l2.clear();
      for (size_t i = 0; i < l1.size(); ++i) {
        if (l1[i] >= n_int) continue;  // ghost: slopes from the ghost pass
        for (int sd = 0; sd < nd; ++sd) {
          if (!((need[i] >> sd) & 1)) continue;
          for (int side = 0; side < 2; ++side) {
            const long long v = nbr[(2 * sd + side) * ld + l1[i]];
            if (v < 0) {
              ok = false;
              return;
            }
            if (outside(v) && !in_l1(v)) l2.push_back((int)v);
          }
        }
      }
      std::sort(l2.begin(), l2.end());
      l2.erase(std::unique(l2.begin(), l2.end()), l2.end());
      if ((int)(l1.size() + l2.size()) > kHaloMaxSlots) {
        ok = false;
        return;
      }
      auto slot = [&](long long v) -> unsigned short {
        if (!outside(v)) return (unsigned short)(v - c0);
        auto it1 = std::lower_bound(l1.begin(), l1.end(), (int)v);
        if (it1 != l1.end() && *it1 == v) return (unsigned short)(TB + (it1 - l1.begin()));
        return (unsigned short)(TB + l1.size() + (std::lower_bound(l2.begin(), l2.end(), (int)v) - l2.begin()));
      };
      for (long long c = c0; c < ce; ++c)
        for (int p = 0; p < NP; ++p) H.base.lnb[(size_t)p * ld + c] = slot(nbr[p * ld + c]);
      std::vector<unsigned short>& hn = hns[t];
      hn.assign(l1.size() * NP, 0xffff);
      for (size_t i = 0; i < l1.size(); ++i) {
        if (l1[i] >= n_int) continue;
        for (int p = 0; p < NP; ++p)
          if ((need[i] >> (p >> 1)) & 1) hn[i * NP + p] = slot(nbr[p * ld + l1[i]]);
      }
      l1s[t] = l1;
      l2s[t] = l2;
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
  HaloHost& B = H.base;
  B.off.assign(ntiles + 1, 0);
  B.goff.assign(ntiles + 1, 0);
  H.h1end.assign(std::max<long long>(ntiles, 1), 0);
  size_t nids = 0;
  int mx = 0, mx1 = 0;
  for (long long t = 0; t < ntiles; ++t) {
    const int n1 = (int)l1s[t].size(), n2 = (int)l2s[t].size();
    H.h1end[t] = (int)(nids + n1);
    nids += n1 + n2;
    B.off[t + 1] = (int)nids;
    mx = std::max(mx, n1 + n2);
    mx1 = std::max(mx1, n1);
  }
  B.ids.resize(std::max<size_t>(nids, 1));
  H.hnb.assign(std::max<size_t>(nids, 1) * NP, 0xffff);
  for (long long t = 0; t < ntiles; ++t) {
    std::copy(l1s[t].begin(), l1s[t].end(), B.ids.begin() + B.off[t]);
    std::copy(l2s[t].begin(), l2s[t].end(), B.ids.begin() + B.off[t] + l1s[t].size());
    std::copy(hns[t].begin(), hns[t].end(), H.hnb.begin() + (size_t)B.off[t] * NP);
  }
  B.grp.assign(1, 0);
  B.max_halo = mx;
  B.mean_halo = ntiles ? (double)nids / ntiles : 0.0;
  B.hmax = std::max(32, (mx + 31) / 32 * 32);
  H.h1max = std::max(32, (mx1 + 31) / 32 * 32);
  return true;
}

size_t cns_halo_smem_bytes(int nd, bool mixed, int hmax, int h1max) {
  if (nd == 2) return mixed ? cns_layout_bytes<float, 2>(hmax, h1max) : cns_layout_bytes<double, 2>(hmax, h1max);
  return mixed ? cns_layout_bytes<float, 3>(hmax, h1max) : cns_layout_bytes<double, 3>(hmax, h1max);
}

namespace {

template <int ND, class R, int MODE, bool FUSE>
int cprep_one(size_t smem) {
  auto k = k_stage_cns_halo<ND, R, MODE, FUSE>;
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
template <int ND, class R, int MODE>
int cprep_f(size_t smem) {
  return std::min(cprep_one<ND, R, MODE, false>(smem), cprep_one<ND, R, MODE, true>(smem));
}
template <int ND, class R>
int cprep_m(size_t smem) {
  return std::min(std::min(cprep_f<ND, R, 0>(smem), cprep_f<ND, R, 2>(smem)),
                  std::min(cprep_f<ND, R, 3>(smem), cprep_f<ND, R, 4>(smem)));
}

template <int ND, class R, int MODE>
void claunch_f(bool fuse, const double* qin, double* out, const Geometry& g, const CnsHaloGeom& h,
               const PhysConst& pc, const Scalars* sc, long long* dtmin, int* status, int grid, size_t smem,
               cudaStream_t st) {
  if (fuse) k_stage_cns_halo<ND, R, MODE, true><<<grid, kHaloTile, smem, st>>>(qin, out, g, h, pc, sc, dtmin, status);
  else k_stage_cns_halo<ND, R, MODE, false><<<grid, kHaloTile, smem, st>>>(qin, out, g, h, pc, sc, dtmin, status);
}
template <int ND, class R>
void claunch_m(int mode, bool fuse, const double* qin, double* out, const Geometry& g, const CnsHaloGeom& h,
               const PhysConst& pc, const Scalars* sc, long long* dtmin, int* status, int grid, size_t smem,
               cudaStream_t st) {
  switch (mode) {
    case 0: claunch_f<ND, R, 0>(fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st); break;
    case 2: claunch_f<ND, R, 2>(fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st); break;
    case 3: claunch_f<ND, R, 3>(fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st); break;
    default: claunch_f<ND, R, 4>(fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st); break;
  }
}

}  // namespace

int cns_halo_prepare(int nd, bool mixed, size_t smem) {
  if (nd == 2) return mixed ? cprep_m<2, float>(smem) : cprep_m<2, double>(smem);
  return mixed ? cprep_m<3, float>(smem) : cprep_m<3, double>(smem);
}

void cns_halo_stage(int nd, bool mixed, int mode, bool fuse, const double* qin, double* out, const Geometry& g,
                    const GhostTables& gt, const CnsHaloGeom& h, const PhysConst& pc, const Scalars* sc,
                    long long* dtmin, int* status, int grid, size_t smem, cudaStream_t st, double* gsl) {
  if (gt.ng > 0) {
    const unsigned nb = (unsigned)((gt.ng + kBlock - 1) / kBlock);
    if (nd == 2) k_ghost_slopes<2><<<nb, kBlock, 0, st>>>(qin, g, gt, gsl, h.ngl);
    else k_ghost_slopes<3><<<nb, kBlock, 0, st>>>(qin, g, gt, gsl, h.ngl);
  }
  if (nd == 2) {
    if (mixed) claunch_m<2, float>(mode, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
    else claunch_m<2, double>(mode, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
  } else {
    if (mixed) claunch_m<3, float>(mode, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
    else claunch_m<3, double>(mode, fuse, qin, out, g, h, pc, sc, dtmin, status, grid, smem, st);
  }
}

}  // namespace h3c
