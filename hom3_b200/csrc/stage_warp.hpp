// stage_warp.hpp -- host interface of the warp-tiled Euler/AUSM stage kernel
// (h3c_stage_warp.cu), shared with the solver's host code (h3c_solver.cu).
//
// The kernel replaces hom3's num_flux + evolve loop (src/solver/fv/
// solver.hpp:440-460, 470-494) for Euler with the AUSM flux, one thread per
// cell and one warp per 32 consecutive Morton cells: each cell's face state
// is computed once, the face state of a cell outside the warp once per face
// that reads it, and a face between two cells of the warp once.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "fv_kernels.cuh"

namespace h3c {

// Halo entries (faces whose neighbour lies outside the warp) and minus faces
// that no plus face of the warp covers, kept in shared memory per warp; the
// faces beyond either cap are evaluated from global memory by their cell.
constexpr int kWarpHalo = 64;
constexpr int kWarpMinus = 32;

// Dynamic shared memory of one 256-thread block for nd / precision.
size_t warp_smem_bytes(int nd, bool mixed);

// Opts every instantiation for nd / precision into its dynamic shared memory
// and returns the resident blocks per SM (0 when it cannot launch).  Call
// outside stream capture.
int warp_prepare(int nd, bool mixed);

// One stage: out = rk_combine<mode>(out, qin, dt/dx R(qin)) over the interior
// cells (one thread per cell), with the fused next-step CFL minimum into
// dtmin when fuse.
void warp_stage(int nd, bool mixed, int mode, bool hang, bool fuse, const double* qin, double* out,
                const Geometry& g, const PhysConst& pc, const Scalars* sc, long long* dtmin, cudaStream_t st);

}  // namespace h3c
