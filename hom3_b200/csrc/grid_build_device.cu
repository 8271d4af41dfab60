// grid_build_device.cu -- the tables of h3c_grid_build (grid_build.cpp)
// computed on the GPU (no hom3 counterpart: hom3 walks its pointer tree on
// the host, hierarchical/implementation.hpp:457-543, and creates ghosts cell by cell,
// solver.hpp:935-977).
//
// The tree lives in dense per-level maps indexed by the Morton code of the
// node's integer coordinates (code ABSENT, INTERNAL, LEAF before ranking, the
// leaf's id after).  Every step of the host builder is data-parallel apart
// from its counters, which are deterministic orders and become scans:
//  * sphere refinement, level by level (a leaf's test depends on the leaf only);
//  * 2:1 face balance in passes, each computing every leaf's need from the
//    state at the start of the pass, then refining (the host's passes);
//  * leaf ids in Morton order of the finest-level corner: a flag at
//    code << nd (maxl - level) in the finest map, exclusive scan;
//  * sub-face groups numbered in (cell, face) order: scan of per-face flags;
//  * ghosts boundary by boundary, numbered in (cell, face) order within a
//    boundary: scan of per-cell counts, one boundary after the other (a
//    ghost fills its face, so later boundaries see it).
// The floating-point expressions are the host's, with products and sums
// rounded separately (__dmul_rn / __dadd_rn): no FMA contraction can move a
// signed distance across zero, so the tables are bit-identical.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "../../include/h3c.h"
#include "grid_build.hpp"

namespace {

constexpr int kB = 256;
constexpr int32_t ABSENT = -1, INTERNAL = -2, LEAF = -3;
__constant__ int kRelD[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

struct DRoot {
  int nd;
  double length, centre[3];
};

struct Spheres {
  int n;
  double c[4][3], r[4];
  int level[4];
};

__device__ __forceinline__ double level_length(double L, int l) { return scalbn(L, -l); }  // L / 2^l, exact

// sdf_eval of grid_build.cpp (geometry/implicit.hpp:39-132) without contraction
__device__ double dsdf(int nd, const h3c_sdf& s, const double* x) {
  double r = 0;
  if (s.kind == H3C_SDF_EDGE) {
    for (int d = 0; d < nd; ++d) r = __dadd_rn(r, __dmul_rn(s.p[3 + d], __dadd_rn(x[d], -s.p[d])));
  } else if (s.kind == H3C_SDF_SQUARE) {
    double dist[3];
    for (int d = 0; d < nd; ++d) dist[d] = __dadd_rn(__dadd_rn(s.p[d], -__dmul_rn(0.5, s.p[3 + d])), -x[d]);
    for (int d = 0; d < nd; ++d)
      if (x[d] > s.p[d]) dist[d] = __dadd_rn(x[d], -__dadd_rn(s.p[d], __dmul_rn(0.5, s.p[3 + d])));
    int npos = 0;
    for (int d = 0; d < nd; ++d) npos += dist[d] > 0;
    if (npos == nd) {
      double q = 0;
      for (int d = 0; d < nd; ++d) q = __dadd_rn(q, __dmul_rn(dist[d], dist[d]));
      r = sqrt(q);
    } else if (npos < 2) {
      r = dist[0];
      for (int d = 1; d < nd; ++d) r = fmax(r, dist[d]);
    } else {
      if (dist[0] < 0) r = sqrt(__dadd_rn(__dmul_rn(dist[1], dist[1]), __dmul_rn(dist[2], dist[2])));
      else if (dist[1] < 0) r = sqrt(__dadd_rn(__dmul_rn(dist[0], dist[0]), __dmul_rn(dist[2], dist[2])));
      else r = sqrt(__dadd_rn(__dmul_rn(dist[0], dist[0]), __dmul_rn(dist[1], dist[1])));
    }
  } else if (s.kind == H3C_SDF_SPHERE) {
    double q = 0;
    for (int d = 0; d < nd; ++d) {
      const double t = __dadd_rn(x[d], -s.p[d]);
      q = __dadd_rn(q, __dmul_rn(t, t));
    }
    r = __dadd_rn(sqrt(q), -s.p[3]);
  }
  return s.inverted ? -1. * r : r;
}

// integer coordinates of Morton code m at a level
__device__ __forceinline__ void demorton(unsigned long long m, int nd, int level, long long* i) {
  i[0] = i[1] = i[2] = 0;
  for (int b = 0; b < level; ++b)
    for (int d = 0; d < nd; ++d) i[d] |= (long long)((m >> (b * nd + d)) & 1ull) << b;
}
__device__ __forceinline__ unsigned long long dmorton(const long long* i, int nd, int level) {
  unsigned long long k = 0;
  for (int b = 0; b < level; ++b)
    for (int d = 0; d < nd; ++d) k |= (unsigned long long)((i[d] >> b) & 1) << (b * nd + d);
  return k;
}

// cell centre accumulated level by level (grid/grid.hpp:358-374, centre() of grid_build.cpp)
__device__ void dcentre(const DRoot& r, int level, const long long* i, double* x) {
  for (int d = 0; d < r.nd; ++d) x[d] = r.centre[d];
  for (int k = 1; k <= level; ++k) {
    const double rel = __dmul_rn(0.25, level_length(r.length, k - 1));
    for (int d = 0; d < r.nd; ++d) {
      const int bit = (int)((i[d] >> (level - k)) & 1);
      x[d] = __dadd_rn(x[d], bit ? rel : -rel);
    }
  }
}

__device__ __forceinline__ bool dinside(int nd, int l, const long long* i) {
  for (int d = 0; d < nd; ++d)
    if (i[d] < 0 || i[d] >= (1LL << l)) return false;
  return true;
}

unsigned nblk(long long n) { return (unsigned)std::max<long long>(1, (n + kB - 1) / kB); }

// ---- exclusive scan of int32 (in place), total returned -------------------
constexpr int kScanB = 1024;  // elements per block (256 threads x 4)

__global__ void k_scan_block(int32_t* a, long long n, int32_t* sums) {
  __shared__ int32_t warp_tot[kB / 32];
  const int t = threadIdx.x;
  const long long base = (long long)blockIdx.x * kScanB + 4 * t;
  int32_t v[4], run = 0;
  for (int k = 0; k < 4; ++k) {
    v[k] = base + k < n ? a[base + k] : 0;
    const int32_t x = v[k];
    v[k] = run;
    run += x;
  }
  int32_t incl = run;
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t y = __shfl_up_sync(0xffffffffu, incl, o);
    if ((t & 31) >= o) incl += y;
  }
  if ((t & 31) == 31) warp_tot[t >> 5] = incl;
  __syncthreads();
  int32_t woff = 0;
  for (int w = 0; w < (t >> 5); ++w) woff += warp_tot[w];
  const int32_t off = woff + incl - run;
  for (int k = 0; k < 4; ++k)
    if (base + k < n) a[base + k] = v[k] + off;
  if (t == kB - 1) sums[blockIdx.x] = woff + incl;
}
__global__ void k_scan_add(int32_t* a, long long n, const int32_t* sums) {
  const long long base = (long long)blockIdx.x * kScanB + 4 * threadIdx.x;
  const int32_t add = sums[blockIdx.x];
  for (int k = 0; k < 4; ++k)
    if (base + k < n) a[base + k] += add;
}

// exclusive scan of a[0, n) on the device; returns the total (-1 on a CUDA error)
long long scan_exclusive(int32_t* a, long long n) {
  if (n <= 0) return 0;
  const long long nb = (n + kScanB - 1) / kScanB;
  int32_t* sums = nullptr;
  if (cudaMalloc(&sums, sizeof(int32_t) * (nb + 1)) != cudaSuccess) return -1;
  k_scan_block<<<(unsigned)nb, kB>>>(a, n, sums);
  long long total;
  if (nb > 1) {
    total = scan_exclusive(sums, nb);
    k_scan_add<<<(unsigned)nb, kB>>>(a, n, sums);
  } else {
    int32_t t = 0;
    cudaMemcpy(&t, sums, sizeof t, cudaMemcpyDeviceToHost);
    total = t;
  }
  cudaFree(sums);
  return cudaGetLastError() == cudaSuccess ? total : -1;
}

}  // namespace

namespace {

// level l of the maps starts at off[l]; 2^(nd l) nodes
struct Maps {
  int32_t* m = nullptr;
  unsigned char* need = nullptr;
  long long off[30] = {0};
};

__global__ void k_fill_level(int32_t* m, long long n, int32_t v) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) m[k] = v;
}

// refine_all's sphere test (grid_build.cpp): the leaf's box intersects a
// sphere whose refinement level is above the leaf's
__global__ void k_refine_sphere(int32_t* ml, int32_t* mchild, long long n, int l, int nd, DRoot r, Spheres sp) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n || ml[m] != LEAF) return;
  long long i[3];
  demorton((unsigned long long)m, nd, l, i);
  double x[3];
  dcentre(r, l, i, x);
  const double h = __dmul_rn(0.5, level_length(r.length, l));
  bool hit = false;
  for (int k = 0; k < sp.n && !hit; ++k) {
    if (l >= sp.level[k]) continue;
    double s = 0;
    for (int d = 0; d < nd; ++d) {
      const double lo = __dadd_rn(x[d], -h), hi = __dadd_rn(x[d], h);
      const double q = fmax(__dadd_rn(lo, -sp.c[k][d]), fmax(0.0, __dadd_rn(sp.c[k][d], -hi)));
      s = __dadd_rn(s, __dmul_rn(q, q));
    }
    hit = s < __dmul_rn(sp.r[k], sp.r[k]);
  }
  if (!hit) return;
  ml[m] = INTERNAL;
  for (int ch = 0; ch < (1 << nd); ++ch) mchild[((unsigned long long)m << nd) | ch] = LEAF;
}

// 2:1 face balance: a leaf whose same-size face neighbour is refined and has a refined child
__global__ void k_balance_need(const int32_t* ml, const int32_t* mchild, unsigned char* need, long long n, int l,
                               int nd) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n) return;
  need[m] = 0;
  if (ml[m] != LEAF) return;
  long long i[3];
  demorton((unsigned long long)m, nd, l, i);
  for (int p = 0; p < 2 * nd; ++p) {
    long long j[3] = {i[0], i[1], i[2]};
    j[p >> 1] += kRelD[p][p >> 1];
    if (!dinside(nd, l, j)) continue;
    const unsigned long long mj = dmorton(j, nd, l);
    if (ml[mj] != INTERNAL) continue;
    for (int ch = 0; ch < (1 << nd); ++ch)
      if (mchild[(mj << nd) | ch] == INTERNAL) { need[m] = 1; return; }
  }
}
__global__ void k_balance_apply(int32_t* ml, int32_t* mchild, const unsigned char* need, long long n, int nd,
                                int* changed) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n || !need[m]) return;
  ml[m] = INTERNAL;
  for (int ch = 0; ch < (1 << nd); ++ch) mchild[((unsigned long long)m << nd) | ch] = LEAF;
  *changed = 1;
}

// leaves whose centre is in the initial domain flag their finest-level corner
__global__ void k_leaf_flags(const int32_t* ml, long long n, int l, int nd, int maxl, DRoot r, int domain_kind,
                             h3c_sdf dom, int32_t* fine) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n || ml[m] != LEAF) return;
  if (domain_kind != 0) {
    long long i[3];
    demorton((unsigned long long)m, nd, l, i);
    double x[3];
    dcentre(r, l, i, x);
    const double s = dsdf(nd, dom, x);
    if (!(domain_kind == 1 ? (s > 0.) : (s < 0.))) return;
  }
  fine[(unsigned long long)m << (nd * (maxl - l))] = 1;
}
// leaf ids (the scanned flags); leaves outside the domain become ABSENT
__global__ void k_leaf_ids(int32_t* ml, long long n, int l, int nd, int maxl, const int32_t* flags,
                           const int32_t* rank, int* cell_level, long long* cell_code) {
  const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= n || ml[m] != LEAF) return;
  const unsigned long long f = (unsigned long long)m << (nd * (maxl - l));
  if (!flags[f]) { ml[m] = ABSENT; return; }
  const int32_t id = rank[f];
  ml[m] = id;
  cell_level[id] = l;
  cell_code[id] = m;
}
// centres and lengths of the interior cells
__global__ void k_cells(const int* cell_level, const long long* cell_code, long long n_int, int nd, DRoot r,
                        double* xc, long long ldx, double* len) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_int) return;
  long long i[3];
  demorton((unsigned long long)cell_code[k], nd, cell_level[k], i);
  double x[3];
  dcentre(r, cell_level[k], i, x);
  for (int d = 0; d < nd; ++d) xc[d * ldx + k] = x[d];
  len[k] = level_length(r.length, cell_level[k]);
}

}  // namespace

namespace {

struct MapView {
  const int32_t* m;
  long long off[30];
  __device__ __forceinline__ int32_t at(int l, unsigned long long code) const { return m[off[l] + code]; }
};

// Neighbours of the interior cells (grid_build.cpp "neighbours"): same-level
// leaf; a refined node whose face children are all leaves (flag a sub-face
// group; pass 2 numbers it); else the coarser leaf covering the position.
// nb = -1: none.  grp[k np + p] = 1 for a group.
__global__ void k_neighbours(MapView mv, const int* cell_level, const long long* cell_code, long long n_int, int nd,
                             long long* nb, int32_t* grp) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_int) return;
  const int np = 2 * nd, l = cell_level[k];
  long long i[3];
  demorton((unsigned long long)cell_code[k], nd, l, i);
  for (int p = 0; p < np; ++p) {
    const int dir = p >> 1;
    long long v_nb = -1;
    int32_t g = 0;
    long long j[3] = {i[0], i[1], i[2]};
    j[dir] += kRelD[p][dir];
    if (dinside(nd, l, j)) {
      const unsigned long long mj = dmorton(j, nd, l);
      const int32_t v = mv.at(l, mj);
      if (v >= 0) {
        v_nb = v;
      } else if (v == INTERNAL) {
        bool ok = true;
        for (int ch = 0; ch < (1 << nd) && ok; ++ch) {
          if (((ch >> dir) & 1) != ((p & 1) ? 0 : 1)) continue;
          ok = mv.at(l + 1, (mj << nd) | ch) >= 0;
        }
        g = ok ? 1 : 0;
      } else if (l > 0) {
        long long pj[3] = {j[0] >> 1, j[1] >> 1, j[2] >> 1};
        const int32_t pv = mv.at(l - 1, dmorton(pj, nd, l - 1));
        if (pv >= 0) v_nb = pv;
      }
    }
    nb[(long long)p * n_int + k] = v_nb;
    grp[k * np + p] = g;
  }
}
// pass 2: group ids (scanned flags) -> nb = -2 - id and the group's finer cells
__global__ void k_subfaces(MapView mv, const int* cell_level, const long long* cell_code, long long n_int, int nd,
                           const int32_t* grp_flag, const int32_t* grp_id, long long nsub, long long* nb,
                           long long* sub) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_int) return;
  const int np = 2 * nd, l = cell_level[k];
  long long i[3];
  demorton((unsigned long long)cell_code[k], nd, l, i);
  for (int p = 0; p < np; ++p) {
    if (!grp_flag[k * np + p]) continue;
    const int dir = p >> 1;
    const long long q = grp_id[k * np + p];
    nb[(long long)p * n_int + k] = -2 - q;
    long long j[3] = {i[0], i[1], i[2]};
    j[dir] += kRelD[p][dir];
    const unsigned long long mj = dmorton(j, nd, l);
    int t = 0;
    for (int ch = 0; ch < (1 << nd); ++ch) {
      if (((ch >> dir) & 1) != ((p & 1) ? 0 : 1)) continue;
      sub[(long long)t * nsub + q] = mv.at(l + 1, (mj << nd) | ch);
      ++t;
    }
  }
}

// Ghosts of boundary b (solver.hpp:935-977): a cell cut by the boundary (its
// 2^nd vertices not all on one side) gets a ghost at every still-missing face
// position whose neighbour centre has a negative signed distance.
__global__ void k_ghost_count(const double* xc, const double* len, const long long* nb, long long n_int, int nd,
                              h3c_sdf geom, int32_t* cnt, unsigned char* mask) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_int) return;
  const double l = len[k];
  double x[3] = {0, 0, 0};
  for (int d = 0; d < nd; ++d) x[d] = xc[d * n_int + k];
  bool allPos = true, allNeg = true;
  for (int v = 0; v < (1 << nd); ++v) {
    double xv[3];
    for (int d = 0; d < nd; ++d) xv[d] = __dadd_rn(x[d], __dmul_rn(__dmul_rn(0.5, l), ((v >> d) & 1) ? 1.0 : -1.0));
    const double s = dsdf(nd, geom, xv);
    allPos = allPos && s > 0;
    allNeg = allNeg && s < 0;
  }
  unsigned char mk = 0;
  if (!(allPos || allNeg)) {
    for (int p = 0; p < 2 * nd; ++p) {
      if (nb[(long long)p * n_int + k] != -1) continue;
      double xn[3];
      for (int d = 0; d < nd; ++d) xn[d] = __dadd_rn(x[d], __dmul_rn((double)kRelD[p][d], l));
      if (dsdf(nd, geom, xn) < 0.) mk |= (unsigned char)(1 << p);
    }
  }
  mask[k] = mk;
  cnt[k] = __popc(mk);
}
// ghost g = base + off[k] + t gets global index n_int + g; its centre is g_xc[3 g + d]
__global__ void k_ghost_fill(const double* xc, const double* len, long long* nb, long long n_int, int nd, int b,
                             const unsigned char* mask, const int32_t* off, long long base, long long gcap,
                             long long* g_back, int* g_pos, double* g_xc, double* g_len, int32_t* g_bc) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_int || !mask[k]) return;
  long long g = base + off[k];
  const double l = len[k];
  for (int p = 0; p < 2 * nd; ++p) {
    if (!(mask[k] & (1 << p))) continue;
    if (g >= gcap) return;  // capacity checked on the host before the launch
    nb[(long long)p * n_int + k] = n_int + g;
    g_back[g] = k;
    g_pos[g] = p;
    for (int d = 0; d < nd; ++d) g_xc[g * 3 + d] = __dadd_rn(xc[d * n_int + k], __dmul_rn(l, (double)kRelD[p][d]));
    g_len[g] = l;
    g_bc[g] = b;
    ++g;
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
namespace {

struct DevBuf {
  std::vector<void*> ptrs;
  ~DevBuf() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <class T> T* alloc(long long n) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * (size_t)std::max<long long>(n, 1)) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return (T*)p;
  }
  template <class T> bool grow(T*& p, long long n_old, long long n_new) {
    T* q = alloc<T>(n_new);
    if (!q) return false;
    if (n_old > 0 && cudaMemcpy(q, p, sizeof(T) * n_old, cudaMemcpyDeviceToDevice) != cudaSuccess) return false;
    for (auto& x : ptrs)
      if (x == (void*)p) { cudaFree(x); x = nullptr; }
    p = q;
    return true;
  }
};

int fail(const std::string& m, int code = H3C_E_INVALID) {
  gridb::set_global_error("h3c_grid_build_device: " + m);
  return code;
}

}  // namespace

extern "C" int h3c_grid_build_device(const h3c_grid_desc* d, h3c_built_grid* out) {
  if (!d || !out) return H3C_E_INVALID;
  const int nd = d->nd;
  if (nd != 2 && nd != 3) return fail("nd must be 2 or 3");
  if (d->min_level < 0 || d->n_refine < 0 || d->n_refine > 4 || d->n_bcs < 0 || d->n_bcs > 16)
    return fail("bad level / refine / bc counts");
  int maxl = d->min_level;
  for (int k = 0; k < d->n_refine; ++k) maxl = std::max(maxl, d->refine_level[k]);
  if ((long long)nd * maxl > 28) return fail("grid too large for dense level maps");
  // root cell: make_root of grid_build.cpp
  DRoot root;
  root.nd = nd;
  root.length = std::numeric_limits<double>::epsilon();
  for (int k = 0; k < 3; ++k) root.centre[k] = 0;
  for (int k = 0; k < nd; ++k) {
    const double lk = d->xmax[k] - d->xmin[k];
    root.length = std::max(root.length, lk);
    root.centre[k] = d->xmin[k] + 0.5 * lk;
  }
  Spheres sp;
  sp.n = d->n_refine;
  for (int k = 0; k < 4; ++k) {
    for (int j = 0; j < 3; ++j) sp.c[k][j] = d->refine_center[k][j];
    sp.r[k] = d->refine_radius[k];
    sp.level[k] = d->refine_level[k];
  }
  DevBuf B;
  MapView mv;
  long long total = 0;
  for (int l = 0; l <= maxl; ++l) {
    mv.off[l] = total;
    total += 1LL << (nd * l);
  }
  int32_t* maps = B.alloc<int32_t>(total);
  unsigned char* need = B.alloc<unsigned char>(total);
  int* changed = B.alloc<int>(1);
  if (!maps || !need || !changed) return fail("out of device memory", H3C_E_NOMEM);
  mv.m = maps;
  auto lvl = [&](int l) { return maps + mv.off[l]; };
  auto cnt = [&](int l) { return 1LL << (nd * l); };
  // ---- MinLevel leaves, sphere refinement level by level ----
  for (int l = 0; l <= maxl; ++l)
    k_fill_level<<<nblk(cnt(l)), kB>>>(lvl(l), cnt(l), l < d->min_level ? INTERNAL : l == d->min_level ? LEAF : ABSENT);
  if (d->n_refine > 0) {
    for (int l = d->min_level; l < maxl; ++l)
      k_refine_sphere<<<nblk(cnt(l)), kB>>>(lvl(l), lvl(l + 1), cnt(l), l, nd, root, sp);
    // 2:1 face balance, pass by pass
    for (int pass = 0; pass < 64; ++pass) {
      for (int l = 0; l < maxl; ++l)
        k_balance_need<<<nblk(cnt(l)), kB>>>(lvl(l), lvl(l + 1), need + mv.off[l], cnt(l), l, nd);
      cudaMemset(changed, 0, sizeof(int));
      for (int l = 0; l < maxl; ++l)
        k_balance_apply<<<nblk(cnt(l)), kB>>>(lvl(l), lvl(l + 1), need + mv.off[l], cnt(l), nd, changed);
      int h = 0;
      if (cudaMemcpy(&h, changed, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess) return fail("CUDA error", H3C_E_CUDA);
      if (!h) break;
    }
  }
  // ---- leaf ids in Morton order of the finest-level corner, inside the initial domain ----
  const long long nfine = cnt(maxl);
  int32_t* flags = B.alloc<int32_t>(nfine);
  int32_t* rank = B.alloc<int32_t>(nfine);
  if (!flags || !rank) return fail("out of device memory", H3C_E_NOMEM);
  cudaMemset(flags, 0, sizeof(int32_t) * nfine);
  for (int l = 0; l <= maxl; ++l)
    k_leaf_flags<<<nblk(cnt(l)), kB>>>(lvl(l), cnt(l), l, nd, maxl, root, d->domain_kind, d->domain, flags);
  cudaMemcpy(rank, flags, sizeof(int32_t) * nfine, cudaMemcpyDeviceToDevice);
  const long long n_int = scan_exclusive(rank, nfine);
  if (n_int < 0) return fail("CUDA error in the leaf scan", H3C_E_CUDA);
  int* cell_level = B.alloc<int>(n_int);
  long long* cell_code = B.alloc<long long>(n_int);
  double* xc = B.alloc<double>((long long)nd * n_int);
  double* len = B.alloc<double>(n_int);
  if (!cell_level || !cell_code || !xc || !len) return fail("out of device memory", H3C_E_NOMEM);
  for (int l = 0; l <= maxl; ++l)
    k_leaf_ids<<<nblk(cnt(l)), kB>>>(lvl(l), cnt(l), l, nd, maxl, flags, rank, cell_level, cell_code);
  k_cells<<<nblk(n_int), kB>>>(cell_level, cell_code, n_int, nd, root, xc, n_int, len);
  // ---- neighbours and sub-face groups ----
  const int np = 2 * nd, nsubc = 1 << (nd - 1);
  long long* nb = B.alloc<long long>((long long)np * n_int);
  int32_t* grp = B.alloc<int32_t>((long long)np * n_int);
  int32_t* grp_id = B.alloc<int32_t>((long long)np * n_int);
  if (!nb || !grp || !grp_id) return fail("out of device memory", H3C_E_NOMEM);
  k_neighbours<<<nblk(n_int), kB>>>(mv, cell_level, cell_code, n_int, nd, nb, grp);
  cudaMemcpy(grp_id, grp, sizeof(int32_t) * np * n_int, cudaMemcpyDeviceToDevice);
  const long long nsub = scan_exclusive(grp_id, (long long)np * n_int);
  if (nsub < 0) return fail("CUDA error in the sub-face scan", H3C_E_CUDA);
  long long* sub = B.alloc<long long>(nsubc * nsub);
  if (!sub) return fail("out of device memory", H3C_E_NOMEM);
  if (nsub > 0) k_subfaces<<<nblk(n_int), kB>>>(mv, cell_level, cell_code, n_int, nd, grp, grp_id, nsub, nb, sub);
  // ---- ghosts, boundary by boundary ----
  int32_t* gcnt = B.alloc<int32_t>(n_int);
  unsigned char* gmask = B.alloc<unsigned char>(n_int);
  long long gcap = std::max<long long>(1024, n_int / 8);
  long long* g_back = B.alloc<long long>(gcap);
  int* g_pos = B.alloc<int>(gcap);
  double* g_xc = B.alloc<double>(3 * gcap);
  double* g_len = B.alloc<double>(gcap);
  int32_t* g_bc = B.alloc<int32_t>(gcap);
  if (!gcnt || !gmask || !g_back || !g_pos || !g_xc || !g_len || !g_bc) return fail("out of device memory", H3C_E_NOMEM);
  long long ng = 0;
  for (int b = 0; b < d->n_bcs; ++b) {
    k_ghost_count<<<nblk(n_int), kB>>>(xc, len, nb, n_int, nd, d->bc_geom[b], gcnt, gmask);
    const long long nb_b = scan_exclusive(gcnt, n_int);
    if (nb_b < 0) return fail("CUDA error in the ghost scan", H3C_E_CUDA);
    if (ng + nb_b > gcap) {
      long long cap = gcap;
      while (ng + nb_b > cap) cap *= 2;
      if (!B.grow(g_back, ng, cap) || !B.grow(g_pos, ng, cap) || !B.grow(g_xc, 3 * ng, 3 * cap) ||
          !B.grow(g_len, ng, cap) || !B.grow(g_bc, ng, cap))
        return fail("out of device memory", H3C_E_NOMEM);
      gcap = cap;
    }
    if (nb_b > 0)
      k_ghost_fill<<<nblk(n_int), kB>>>(xc, len, nb, n_int, nd, b, gmask, gcnt, ng, gcap, g_back, g_pos, g_xc, g_len,
                                        g_bc);
    ng += nb_b;
  }
  if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess)
    return fail("CUDA error", H3C_E_CUDA);
  // ---- tables back to the host, in the layout of h3c_grid_build ----
  std::vector<long long> h_nb((size_t)np * n_int), h_sub((size_t)nsubc * nsub), h_code(n_int), h_back(ng);
  std::vector<int> h_level(n_int), h_pos(ng);
  std::vector<double> h_xc((size_t)nd * n_int), h_len(n_int), h_gxc((size_t)3 * ng), h_glen(ng);
  std::vector<int32_t> h_gbc(ng);
  auto down = [&](void* dst, const void* src, size_t bytes) {
    return bytes == 0 || cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
  };
  if (!down(h_nb.data(), nb, sizeof(long long) * h_nb.size()) || !down(h_sub.data(), sub, sizeof(long long) * h_sub.size()) ||
      !down(h_code.data(), cell_code, sizeof(long long) * n_int) || !down(h_level.data(), cell_level, sizeof(int) * n_int) ||
      !down(h_xc.data(), xc, sizeof(double) * h_xc.size()) || !down(h_len.data(), len, sizeof(double) * n_int) ||
      !down(h_back.data(), g_back, sizeof(long long) * ng) || !down(h_pos.data(), g_pos, sizeof(int) * ng) ||
      !down(h_gxc.data(), g_xc, sizeof(double) * 3 * ng) || !down(h_glen.data(), g_len, sizeof(double) * ng) ||
      !down(h_gbc.data(), g_bc, sizeof(int32_t) * ng))
    return fail("CUDA error in the download", H3C_E_CUDA);
  auto g = std::make_unique<h3c_built_grid_s>();
  const long long n_tot = n_int + ng;
  g->nd = nd;
  g->n_int = n_int;
  g->n_tot = n_tot;
  g->nsub = nsub;
  const int64_t INV = std::numeric_limits<int64_t>::max();
  g->nbr.assign((size_t)np * n_tot, INV);
  for (int p = 0; p < np; ++p)
    for (long long k = 0; k < n_int; ++k) {
      const long long v = h_nb[(size_t)p * n_int + k];
      g->nbr[(size_t)p * n_tot + k] = v == -1 ? INV : v;
    }
  for (long long q = 0; q < ng; ++q) g->nbr[(size_t)(h_pos[q] ^ 1) * n_tot + n_int + q] = h_back[q];
  g->xc.assign((size_t)nd * n_tot, 0.0);
  for (int dd = 0; dd < nd; ++dd) {
    for (long long k = 0; k < n_int; ++k) g->xc[(size_t)dd * n_tot + k] = h_xc[(size_t)dd * n_int + k];
    for (long long q = 0; q < ng; ++q) g->xc[(size_t)dd * n_tot + n_int + q] = h_gxc[(size_t)3 * q + dd];
  }
  g->len.resize(n_tot);
  g->bc.resize(n_tot);
  for (long long k = 0; k < n_int; ++k) {
    g->len[k] = h_len[k];
    g->bc[k] = std::numeric_limits<int32_t>::max();
  }
  for (long long q = 0; q < ng; ++q) {
    g->len[n_int + q] = h_glen[q];
    g->bc[n_int + q] = h_gbc[q];
  }
  g->sub = std::vector<int64_t>(h_sub.begin(), h_sub.end());
  g->cells.resize(n_tot);
  for (long long k = 0; k < n_int; ++k) {
    gridb::Cell c{h_level[k], {0, 0, 0}};
    for (int b = 0; b < h_level[k]; ++b)
      for (int dd = 0; dd < nd; ++dd) c.i[dd] |= (long long)((h_code[k] >> (b * nd + dd)) & 1) << b;
    g->cells[k] = c;
  }
  for (long long q = 0; q < ng; ++q) {
    gridb::Cell c = g->cells[h_back[q]];
    c.i[h_pos[q] >> 1] += (h_pos[q] & 1) ? 1 : -1;
    g->cells[n_int + q] = c;
  }
  g->bcs.assign(std::max(1, d->n_bcs), h3c_bc{});
  *out = g.release();
  return H3C_OK;
}
