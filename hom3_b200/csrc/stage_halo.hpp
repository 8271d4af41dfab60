// stage_halo.hpp -- host interface of the halo-staged Euler/AUSM stage kernel
// (h3c_stage_halo.cu), shared with the solver's host code (h3c_solver.cu).
//
// The kernel replaces hom3's num_flux + evolve loop (src/solver/fv/
// solver.hpp:440-460, 470-494) for Euler with the AUSM flux.  It works on
// 256-cell tiles of the Morton order.  Per tile, set-up time tables list
//   * the tile's halo: every (cell, direction) pair such that a face of a
//     tile cell along that direction reads a cell outside the tile
//     (same-level neighbours, ghosts and the fine cells of coarse/fine
//     sub-face groups), sorted, and
//   * for every cell and face position the shared-memory slot the face's
//     neighbour lives in (0..255: a tile cell, 256 + h: halo cell h) or, with
//     kGroupBit set, the index of the face's sub-face group in the tile's
//     group list (whose entries are the slots of the group's fine cells).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "fv_kernels.cuh"

namespace h3c {

constexpr int kHaloTile = 256;              // cells per tile = threads per block
constexpr int kHaloMaxSlots = 1024;         // halo entries a tile may hold in shared memory
constexpr unsigned short kGroupBit = 0x8000;
// Euler halo entries are (cell, direction) pairs: the id word carries the
// cell in its low 29 bits and the face direction it is read across above
// them (the CNS tables list plain cell ids).
constexpr int kHaloDirShift = 29;
constexpr int kHaloCellMask = (1 << kHaloDirShift) - 1;

// Device tables of the halo-staged kernel.
struct HaloGeom {
  const unsigned short* __restrict__ lnb;  // [2nd][ld] neighbour slot (or kGroupBit | group) per cell
  const int* __restrict__ halo_ids;        // halo cells of all tiles, concatenated
  const int* __restrict__ halo_off;        // [ntiles + 1] offsets into halo_ids
  const unsigned short* __restrict__ grp;  // [groups][2^(nd-1)] slots of each group's fine cells
  const int* __restrict__ grp_off;         // [ntiles + 1] first group of each tile
  int hmax;                                // halo slots reserved per tile (multiple of 32)
};

// Host copies of the tables before upload.
struct HaloHost {
  std::vector<unsigned short> lnb, grp;
  std::vector<int> ids, off, goff;
  int hmax = 0;
  int max_halo = 0;      // largest halo of any tile
  double mean_halo = 0;  // halo cells per tile, mean
};

// Builds the tables from the device-numbered neighbour table nbr [2nd][ld]
// (>= 0 cell, <= -2 sub-face group -2 - k of sub [2^(nd-1)][nsub]) for the
// tiles of [0, n_int); tile_end[t] is the end of tile t's cells (tiles never
// span two batch instances).  Returns false when a tile's slots overflow 15
// bits or the cells 29 bits (the caller then keeps the per-lane tile kernel).
// Halo ids carry the direction in bits 29-30.
bool halo_build(int nd, long long ld, long long ntiles, const std::vector<long long>& tile_end, const int* nbr,
                const int* sub, long long nsub, HaloHost& H);

// Dynamic shared memory of one block for nd / precision / halo slots.
size_t halo_smem_bytes(int nd, bool mixed, int hmax);
// The halo entries a tile keeps in shared memory so that blocks_per_sm
// blocks fit on an SM (at most the largest tile halo, rounded up to 32);
// a tile's entries beyond it are read from global memory where used.
int halo_slots_for(int nd, bool mixed, int max_halo, int blocks_per_sm);

// Opts every instantiation for nd / precision into `smem` bytes of dynamic
// shared memory and returns the resident blocks per SM at that size (0 when
// the kernel cannot be launched with it).  Call outside stream capture.
int halo_prepare(int nd, bool mixed, size_t smem);

// One stage: out = rk_combine<mode>(out, qin, dt/dx R(qin)) over the tiles,
// with the fused next-step CFL minimum into dtmin when fuse.  grid blocks
// take the tiles round-robin.  status receives bit 2 when a bounded wait for
// a tile's copies runs out.
void halo_stage(int nd, bool mixed, int mode, bool hang, bool fuse, const double* qin, double* out,
                const Geometry& g, const HaloGeom& h, const PhysConst& pc, const Scalars* sc, long long* dtmin,
                int* status, int grid, size_t smem, cudaStream_t st);

// ---------------------------------------------------------------------------
// CNS (AUSM + three-point viscous flux) on the same tiles (h3c_stage_cns.cu).
// The viscous flux reads the transverse slopes of both face cells, so the
// tables add, per tile, a second halo layer: the cells the slopes of the
// first layer read (the tile's edge-diagonal neighbours, and ghosts next to
// first-layer boundary cells).  Ghost cells' slopes (a boundary or periodic
// partner cell's slope, with the walls' sign rule) come from a ghost-only
// slope pass.  Single-level grids only (hom3's CNS has no coarse/fine faces).
// ---------------------------------------------------------------------------
struct CnsHaloGeom {
  HaloGeom h;                                // lnb, halo ids (layer 1 then layer 2 per tile), offsets, slots
  const int* __restrict__ h1end;             // [ntiles] end of tile t's layer 1 in halo_ids
  const unsigned short* __restrict__ hnb;    // [halo_ids entries][2nd] slots of a layer-1 cell's face
                                             // neighbours (0xffff: that slope is not needed)
  const double* __restrict__ gsl;            // [nd * nv][ngl] slopes of the ghost cells
  long long ngl;                             // leading dimension of gsl
  int h1max;                                 // layer-1 slots reserved per tile (multiple of 32)
};

struct CnsHaloHost {
  HaloHost base;                             // lnb, ids, off; grp unused
  std::vector<int> h1end;
  std::vector<unsigned short> hnb;
  int h1max = 0;
};

bool halo_build_cns(int nd, long long ld, long long n_int, long long ntiles, const std::vector<long long>& tile_end,
                    const int* nbr, CnsHaloHost& H);
size_t cns_halo_smem_bytes(int nd, bool mixed, int hmax, int h1max);
int cns_halo_prepare(int nd, bool mixed, size_t smem);
// the ghost-slope pass and the stage; h = the grid's (single) cell length
void cns_halo_stage(int nd, bool mixed, int mode, bool fuse, const double* qin, double* out, const Geometry& g,
                    const GhostTables& gt, const CnsHaloGeom& h, const PhysConst& pc, const Scalars* sc,
                    long long* dtmin, int* status, int grid, size_t smem, cudaStream_t st, double* gsl);

}  // namespace h3c
