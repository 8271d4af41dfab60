// grid_build.cpp -- host grid builder of hom3_b200 (the "device grid layer").
//
// Produces the cell tables hom3's Solver::initialize builds
// (solver.hpp:876-977) without hom3's pointer tree: leaves are addressed by
// (level, integer coordinates) in dense per-level lookup arrays, neighbours
// are found by coordinate arithmetic instead of up/down tree walks
// (hierarchical/implementation.hpp:457-543), and interior cells come out in Morton order,
// which for a MinLevel grid is also hom3's leaf order.  Conventions that must
// match hom3 to give identical tables:
//  * cell centres are accumulated from the root centre level by level with
//    +-0.25 * parent length, as cell_coordinates does (grid/grid.hpp:358-374);
//  * lengths are root_length / 2^level (grid/grid.hpp:344-351);
//  * cut test on the 2^nd cell vertices (grid/grid.hpp:601-626), ghosts at
//    missing neighbour positions with negative signed distance, created
//    boundary by boundary and cell by cell (solver.hpp:935-977);
//  * signed distances of geometry/implicit.hpp:39-132 and the cube faces of
//    grid/helpers.hpp:112-160.
// EXTENSION (not in hom3): sphere refinement with 2:1 face balance and
// coarse/fine sub-face groups.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "../../include/h3c.h"
#include "grid_build.hpp"

namespace {

using gridb::BuiltGrid;
using gridb::Cell;
void fail_msg(const char* m) { gridb::set_global_error(m); }

double sdf_eval(int nd, const h3c_sdf& s, const double* x) {
  double r = 0;
  if (s.kind == H3C_SDF_EDGE) {
    for (int d = 0; d < nd; ++d) r += s.p[3 + d] * (x[d] - s.p[d]);
  } else if (s.kind == H3C_SDF_SQUARE) {
    double dist[3];
    for (int d = 0; d < nd; ++d) dist[d] = s.p[d] - 0.5 * s.p[3 + d] - x[d];
    for (int d = 0; d < nd; ++d)
      if (x[d] > s.p[d]) dist[d] = x[d] - (s.p[d] + 0.5 * s.p[3 + d]);
    int npos = 0;
    for (int d = 0; d < nd; ++d) npos += dist[d] > 0;
    if (npos == nd) {
      double q = 0;
      for (int d = 0; d < nd; ++d) q += dist[d] * dist[d];
      r = std::sqrt(q);
    } else if (npos < 2) {
      r = dist[0];
      for (int d = 1; d < nd; ++d) r = std::max(r, dist[d]);
    } else {
      if (dist[0] < 0) r = std::sqrt(dist[1] * dist[1] + dist[2] * dist[2]);
      else if (dist[1] < 0) r = std::sqrt(dist[0] * dist[0] + dist[2] * dist[2]);
      else r = std::sqrt(dist[0] * dist[0] + dist[1] * dist[1]);
    }
  } else if (s.kind == H3C_SDF_SPHERE) {
    double q = 0;
    for (int d = 0; d < nd; ++d) q += (x[d] - s.p[d]) * (x[d] - s.p[d]);
    r = std::sqrt(q) - s.p[3];
  }
  return s.inverted ? -1. * r : r;
}

struct Root {
  int nd;
  double length, centre[3], xmin[3];
};

Root make_root(const h3c_grid_desc& d) {
  Root r;
  r.nd = d.nd;
  r.length = std::numeric_limits<double>::epsilon();
  for (int k = 0; k < d.nd; ++k) {
    const double lk = d.xmax[k] - d.xmin[k];
    r.length = std::max(r.length, lk);
    r.centre[k] = d.xmin[k] + 0.5 * lk;
  }
  for (int k = 0; k < d.nd; ++k) r.xmin[k] = r.centre[k] - 0.5 * r.length;
  return r;
}

double level_length(const Root& r, int l) { return r.length / std::pow(2, l); }

void centre(const Root& r, const Cell& c, double* x) {
  for (int d = 0; d < r.nd; ++d) x[d] = r.centre[d];
  for (int k = 1; k <= c.level; ++k) {
    const double rel = 0.25 * level_length(r, k - 1);
    for (int d = 0; d < r.nd; ++d) {
      const int bit = (int)((c.i[d] >> (c.level - k)) & 1);
      x[d] = x[d] + (bit ? 1.0 : -1.0) * rel;
    }
  }
}

uint64_t morton(const long long* ix, int nd, int bits) {
  uint64_t k = 0;
  for (int b = 0; b < bits; ++b)
    for (int d = 0; d < nd; ++d) k |= (uint64_t)((ix[d] >> b) & 1) << (b * nd + d);
  return k;
}

// Dense per-level maps: code < -1 internal node, -1 absent, >= 0 leaf id.
struct Levels {
  int nd, maxl;
  std::vector<std::vector<int32_t>> m;
  static constexpr int32_t ABSENT = -1, INTERNAL = -2;
  bool init(int nd_, int maxl_) {
    nd = nd_;
    maxl = maxl_;
    if ((long long)nd * maxl > 28) return false;
    m.resize(maxl + 1);
    for (int l = 0; l <= maxl; ++l) m[l].assign((size_t)1 << (nd * l), ABSENT);
    return true;
  }
  int32_t& at(int l, const long long* i) { return m[l][morton(i, nd, l)]; }
  bool inside(int l, const long long* i) const {
    for (int d = 0; d < nd; ++d)
      if (i[d] < 0 || i[d] >= (1LL << l)) return false;
    return true;
  }
};

const int kRel[6][3] = {{-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

}  // namespace

extern "C" {

int h3c_cube_boundaries(const h3c_grid_desc* d, h3c_sdf* out) {
  if (!d || !out || (d->nd != 2 && d->nd != 3)) return H3C_E_INVALID;
  const Root r = make_root(*d);
  const double eps = r.length * 1e-15;
  const double x_max = r.centre[0] + 0.5 * r.length - eps;
  const double x_min = r.centre[0] - 0.5 * r.length + eps;
  const double off = x_min + 0.5 * r.length;
  int k = 0;
  for (int dd = 0; dd < d->nd; ++dd)
    for (int side = 0; side < 2; ++side) {
      h3c_sdf s;
      std::memset(&s, 0, sizeof(s));
      s.kind = H3C_SDF_EDGE;
      for (int j = 0; j < d->nd; ++j) s.p[j] = off;
      s.p[dd] = side == 0 ? x_min : x_max;
      s.p[3 + dd] = side == 0 ? 1.0 : -1.0;
      out[k++] = s;
    }
  return k;
}

int h3c_grid_build(const h3c_grid_desc* d, h3c_built_grid* out) {
  if (!d || !out) return H3C_E_INVALID;
  const int nd = d->nd;
  if (nd != 2 && nd != 3) { fail_msg("h3c_grid_build: nd must be 2 or 3"); return H3C_E_INVALID; }
  if (d->min_level < 0 || d->n_refine < 0 || d->n_refine > 4 || d->n_bcs < 0 || d->n_bcs > 16) {
    fail_msg("h3c_grid_build: bad level / refine / bc counts");
    return H3C_E_INVALID;
  }
  const Root root = make_root(*d);
  int maxl = d->min_level;
  for (int k = 0; k < d->n_refine; ++k) maxl = std::max(maxl, d->refine_level[k]);
  Levels L;
  if (!L.init(nd, maxl)) { fail_msg("h3c_grid_build: grid too large for dense level maps"); return H3C_E_INVALID; }
  // ---- leaves: MinLevel (grid/generation.hpp:39-60), then sphere refinement ----
  std::vector<Cell> leaves;
  {
    const long long n = 1LL << (nd * d->min_level);
    leaves.reserve(n);
    for (long long m = 0; m < n; ++m) {
      Cell c{d->min_level, {0, 0, 0}};
      for (int b = 0; b < d->min_level; ++b)
        for (int dd = 0; dd < nd; ++dd) c.i[dd] |= ((m >> (b * nd + dd)) & 1LL) << b;
      leaves.push_back(c);
    }
  }
  auto refine_all = [&](auto pred) {
    bool changed = true;
    while (changed) {
      changed = false;
      std::vector<Cell> next;
      next.reserve(leaves.size());
      for (const Cell& c : leaves) {
        if (c.level < maxl && pred(c)) {
          changed = true;
          for (int ch = 0; ch < (1 << nd); ++ch) {
            Cell k{c.level + 1, {0, 0, 0}};
            for (int dd = 0; dd < nd; ++dd) k.i[dd] = 2 * c.i[dd] + ((ch >> dd) & 1);
            next.push_back(k);
          }
        } else {
          next.push_back(c);
        }
      }
      leaves.swap(next);
    }
  };
  if (d->n_refine > 0) {
    refine_all([&](const Cell& c) {
      double x[3];
      centre(root, c, x);
      const double h = 0.5 * level_length(root, c.level);
      for (int k = 0; k < d->n_refine; ++k) {
        if (c.level >= d->refine_level[k]) continue;
        double s = 0;
        for (int dd = 0; dd < nd; ++dd) {
          const double lo = x[dd] - h, hi = x[dd] + h;
          const double q = std::max(lo - d->refine_center[k][dd], std::max(0.0, d->refine_center[k][dd] - hi));
          s += q * q;
        }
        if (s < d->refine_radius[k] * d->refine_radius[k]) return true;
      }
      return false;
    });
    // 2:1 face balance: refine a leaf when a face neighbour of its size has
    // children that are themselves refined.
    auto mark = [&]() {
      for (auto& m : L.m) std::fill(m.begin(), m.end(), Levels::ABSENT);
      for (size_t k = 0; k < leaves.size(); ++k) {
        Cell c = leaves[k];
        L.at(c.level, c.i) = (int32_t)k;
        while (c.level > 0) {
          for (int dd = 0; dd < nd; ++dd) c.i[dd] >>= 1;
          c.level -= 1;
          L.at(c.level, c.i) = Levels::INTERNAL;
        }
      }
    };
    bool changed = true;
    while (changed) {
      mark();
      changed = false;
      std::vector<char> need(leaves.size(), 0);
      for (size_t k = 0; k < leaves.size(); ++k) {
        const Cell& c = leaves[k];
        for (int p = 0; p < 2 * nd && !need[k]; ++p) {
          long long j[3] = {c.i[0], c.i[1], c.i[2]};
          j[p >> 1] += kRel[p][p >> 1];
          if (!L.inside(c.level, j) || L.at(c.level, j) != Levels::INTERNAL) continue;
          for (int ch = 0; ch < (1 << nd); ++ch) {
            long long cj[3];
            for (int dd = 0; dd < nd; ++dd) cj[dd] = 2 * j[dd] + ((ch >> dd) & 1);
            if (c.level + 1 <= maxl && L.at(c.level + 1, cj) == Levels::INTERNAL) { need[k] = 1; break; }
          }
        }
      }
      std::vector<Cell> next;
      for (size_t k = 0; k < leaves.size(); ++k) {
        if (!need[k]) { next.push_back(leaves[k]); continue; }
        changed = true;
        const Cell& c = leaves[k];
        for (int ch = 0; ch < (1 << nd); ++ch) {
          Cell kc{c.level + 1, {0, 0, 0}};
          for (int dd = 0; dd < nd; ++dd) kc.i[dd] = 2 * c.i[dd] + ((ch >> dd) & 1);
          next.push_back(kc);
        }
      }
      leaves.swap(next);
    }
  }
  // ---- Morton order of leaves (finest-level corner keys) ----
  {
    std::vector<std::pair<uint64_t, size_t>> keys(leaves.size());
    for (size_t k = 0; k < leaves.size(); ++k) {
      long long ix[3];
      for (int dd = 0; dd < nd; ++dd) ix[dd] = leaves[k].i[dd] << (maxl - leaves[k].level);
      keys[k] = {morton(ix, nd, maxl), k};
    }
    std::sort(keys.begin(), keys.end());
    std::vector<Cell> sorted(leaves.size());
    for (size_t k = 0; k < keys.size(); ++k) sorted[k] = leaves[keys[k].second];
    leaves.swap(sorted);
  }
  // ---- initial domain (solver.hpp:882-892) ----
  auto in_domain = [&](const double* x) {
    if (d->domain_kind == 0) return true;
    const double s = sdf_eval(nd, d->domain, x);
    return d->domain_kind == 1 ? (s > 0.) : (s < 0.);
  };
  auto g = std::make_unique<h3c_built_grid_s>();
  g->nd = nd;
  std::vector<double> xs;
  for (const Cell& c : leaves) {
    double x[3];
    centre(root, c, x);
    if (!in_domain(x)) continue;
    g->cells.push_back(c);
    for (int dd = 0; dd < nd; ++dd) xs.push_back(x[dd]);
  }
  const long long n_int = (long long)g->cells.size();
  // lookup: leaf id of cells in the domain, INTERNAL for refined nodes
  for (auto& m : L.m) std::fill(m.begin(), m.end(), Levels::ABSENT);
  for (long long k = 0; k < n_int; ++k) {
    Cell c = g->cells[k];
    L.at(c.level, c.i) = (int32_t)k;
  }
  for (const Cell& c0 : leaves) {
    Cell c = c0;
    while (c.level > 0) {
      for (int dd = 0; dd < nd; ++dd) c.i[dd] >>= 1;
      c.level -= 1;
      L.at(c.level, c.i) = Levels::INTERNAL;
    }
  }
  // ---- neighbours ----
  const int np = 2 * nd, nsubc = 1 << (nd - 1);
  std::vector<std::vector<int64_t>> nb(np, std::vector<int64_t>(n_int, -1));
  std::vector<int64_t> subs;  // flattened groups of nsubc
  for (long long k = 0; k < n_int; ++k) {
    const Cell& c = g->cells[k];
    for (int p = 0; p < np; ++p) {
      const int dir = p >> 1;
      long long j[3] = {c.i[0], c.i[1], c.i[2]};
      j[dir] += kRel[p][dir];
      if (!L.inside(c.level, j)) continue;
      const int32_t v = L.at(c.level, j);
      if (v >= 0) { nb[p][k] = v; continue; }
      if (v == Levels::INTERNAL) {
        // finer neighbours: the children of (level, j) that touch this face,
        // in increasing child position
        std::vector<int64_t> grp;
        bool ok = true;
        for (int ch = 0; ch < (1 << nd); ++ch) {
          if (((ch >> dir) & 1) != ((p & 1) ? 0 : 1)) continue;
          long long cj[3];
          for (int dd = 0; dd < nd; ++dd) cj[dd] = 2 * j[dd] + ((ch >> dd) & 1);
          const int32_t cv = L.at(c.level + 1, cj);
          if (cv < 0) { ok = false; break; }
          grp.push_back(cv);
        }
        if (ok) {
          nb[p][k] = -2 - (int64_t)(subs.size() / nsubc);
          subs.insert(subs.end(), grp.begin(), grp.end());
        }
        continue;
      }
      // coarser neighbour: the parent-level cell covering the position
      if (c.level > 0) {
        long long pj[3];
        for (int dd = 0; dd < nd; ++dd) pj[dd] = j[dd] >> 1;
        const int32_t pv = L.at(c.level - 1, pj);
        if (pv >= 0) nb[p][k] = pv;
      }
    }
  }
  // ---- ghost cells, boundary by boundary (solver.hpp:935-977) ----
  std::vector<int32_t> bcs(n_int, -1);
  for (int b = 0; b < d->n_bcs; ++b) {
    const h3c_sdf& geom = d->bc_geom[b];
    for (long long k = 0; k < n_int; ++k) {
      const Cell c = g->cells[k];
      const double l = level_length(root, c.level);
      double x[3] = {0, 0, 0};  // copy: xs grows below
      for (int dd = 0; dd < nd; ++dd) x[dd] = xs[k * nd + dd];
      bool allPos = true, allNeg = true;
      for (int v = 0; v < (1 << nd); ++v) {
        double xv[3];
        for (int dd = 0; dd < nd; ++dd) xv[dd] = x[dd] + 0.5 * l * (((v >> dd) & 1) ? 1.0 : -1.0);
        const double s = sdf_eval(nd, geom, xv);
        allPos = allPos && s > 0;
        allNeg = allNeg && s < 0;
      }
      if (allPos || allNeg) continue;
      int missing[6], nm = 0;
      for (int p = 0; p < np; ++p)
        if (nb[p][k] == -1) missing[nm++] = p;
      for (int t = 0; t < nm; ++t) {
        const int p = missing[t];
        double xn[3];
        for (int dd = 0; dd < nd; ++dd) xn[dd] = x[dd] + (double)kRel[p][dd] * l;
        if (!(sdf_eval(nd, geom, xn) < 0.)) continue;
        const long long gi = (long long)g->cells.size();
        Cell gc = c;
        gc.i[p >> 1] += kRel[p][p >> 1];
        g->cells.push_back(gc);
        for (int q = 0; q < np; ++q) nb[q].push_back(-1);
        nb[p][k] = gi;
        nb[p ^ 1][gi] = k;
        for (int dd = 0; dd < nd; ++dd) xs.push_back(x[dd] + l * (double)kRel[p][dd]);
        bcs.push_back(b);
      }
    }
  }
  const long long n_tot = (long long)g->cells.size();
  g->n_int = n_int;
  g->n_tot = n_tot;
  g->nsub = (long long)subs.size() / nsubc;
  g->nbr.assign((size_t)np * n_tot, -1);
  for (int p = 0; p < np; ++p)
    for (long long k = 0; k < n_tot; ++k) g->nbr[p * n_tot + k] = nb[p][k] == -1 ? std::numeric_limits<int64_t>::max() : nb[p][k];
  g->xc.assign((size_t)nd * n_tot, 0.0);
  for (long long k = 0; k < n_tot; ++k)
    for (int dd = 0; dd < nd; ++dd) g->xc[dd * n_tot + k] = xs[k * nd + dd];
  g->len.resize(n_tot);
  for (long long k = 0; k < n_tot; ++k) g->len[k] = level_length(root, g->cells[k].level);
  g->bc.resize(n_tot);
  for (long long k = 0; k < n_tot; ++k) g->bc[k] = k < n_int ? std::numeric_limits<int32_t>::max() : bcs[k];
  g->sub.assign((size_t)nsubc * std::max<long long>(g->nsub, 0), 0);
  for (long long q = 0; q < g->nsub; ++q)
    for (int j = 0; j < nsubc; ++j) g->sub[j * g->nsub + q] = subs[q * nsubc + j];
  g->bcs.assign(std::max(1, d->n_bcs), h3c_bc{});
  *out = g.release();
  return H3C_OK;
}

int h3c_grid_view(h3c_built_grid g, h3c_grid* v) {
  if (!g || !v) return H3C_E_INVALID;
  std::memset(v, 0, sizeof(*v));
  v->n_cells = g->n_tot;
  v->first_ghost = g->n_int;
  v->ld = g->n_tot;
  v->neighbors = g->nbr.data();
  v->x_center = g->xc.data();
  v->length = g->len.data();
  v->bc_idx = g->bc.data();
  v->n_bcs = 0;
  v->bcs = nullptr;
  v->n_subfaces = g->nsub;
  v->subface_cells = g->nsub > 0 ? g->sub.data() : nullptr;
  return H3C_OK;
}

int h3c_grid_free(h3c_built_grid g) {
  delete g;
  return H3C_OK;
}

}  // extern "C"
