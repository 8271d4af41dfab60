// h3c_noalloc.cu -- the CFL time step of a state without any device allocation.
//
// Some callers cannot allocate device memory: a host code that runs inside a
// framework owning all of the GPU's memory through its own pool, or a time
// step controller that must not call cudaMalloc because cudaMalloc
// synchronises the device and would serialise the caller's streams.  For
// them h3c_min_dt_noalloc computes the same minimum of the per-cell time
// step as h3c_min_dt (hom3's Solver::min_dt / compute_dt,
// src/solver/fv/solver.hpp:109, 511-517) from device buffers the caller owns,
// using as scratch a fixed array compiled into this library.
//
// The scratch array holds one partial minimum per 256-cell block, so a call
// accepts at most kNoAllocMaxCells cells.  Every GPU that loads the library
// holds the array until the process exits.  All calls share it and it keeps
// the last call's contents (each call writes every partial it reads, so
// nothing needs clearing); calls whose kernels overlap on the GPU -- on two
// streams, or from two host threads -- race on it and must be serialised by
// the caller.  Euler, CNS and heat are covered; advection (whose time step
// needs the per-cell velocity field) is rejected.
//
// The first call on a device looks up the array's address.  Under CUDA's
// default lazy module loading that first call (or the first kernel launch of
// this library) also loads the library's device code, which reserves device
// memory for the code and the array; a caller whose pool will own all device
// memory makes the first call during its own initialisation, before the pool
// takes the memory (or sets CUDA_MODULE_LOADING=EAGER).  After that, calls
// reserve nothing.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/h3c.h"
#define H3C_DEVICE_FUNCTIONS_ONLY
#include "fv_kernels.cuh"

namespace gridb {
void set_global_error(const std::string& msg);  // h3c_last_error(NULL, ...) text
}

namespace {

constexpr int kNoAllocMaxBlocks = 16384;  // 128 KiB of partial minima
constexpr long long kNoAllocMaxCells = (long long)kNoAllocMaxBlocks * h3c::kBlock;  // 4,194,304
constexpr int kMaxDevices = 64;

// File-scope device scratch.  In host code this name only stands in for the
// symbol; the device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) long long g_noalloc_scratch[kNoAllocMaxBlocks];

long long* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Per-block minimum of the cell time step, written to partials[blockIdx.x].
template <int ND, int PHYS>
__global__ void __launch_bounds__(h3c::kBlock) k_cfl_partials(const double* __restrict__ q, long long ld,
                                                               const double* __restrict__ len, long long n,
                                                               h3c::PhysConst pc, long long* partials) {
  using namespace h3c;
  constexpr int NV = nvars<ND, PHYS>();
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long v = kOrdMax;
  if (c < n) {
    double qc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) qc[k] = q[k * ld + c];
    const double dt = cell_dt<ND, PHYS>(qc, len[c], pc);
    if (!isnan(dt)) v = dbl_to_ord(dt);
  }
  __shared__ long long red[kBlock / 32];
  for (int o = 16; o > 0; o >>= 1) {
    const long long w = __shfl_down_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long m = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = red[w] < m ? red[w] : m;
    partials[blockIdx.x] = m;
  }
}

// One block folds the partials and writes the time step.
__global__ void k_cfl_fold(const long long* __restrict__ partials, int nblocks, double* dt_out) {
  using namespace h3c;
  long long v = kOrdMax;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) v = partials[i] < v ? partials[i] : v;
  __shared__ long long red[kBlock / 32];
  for (int o = 16; o > 0; o >>= 1) {
    const long long w = __shfl_down_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long m = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = red[w] < m ? red[w] : m;
    *dt_out = ord_to_dbl(m);
  }
}

// Device address of the scratch array on the current device, looked up once
// per device (with that device current).
int scratch_address(long long** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return H3C_E_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return H3C_E_INVALID;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    long long* p = nullptr;
    e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return H3C_E_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return H3C_OK;
}

}  // namespace

extern "C" int h3c_min_dt_noalloc(const h3c_desc* desc, const double* q, int64_t ld, int64_t n_cells,
                                  const double* length, double* dt_out, void* stream) {
  using namespace h3c;
  auto fail = [](int code, const std::string& m) {
    gridb::set_global_error("h3c_min_dt_noalloc: " + m);
    return code;
  };
  if (!desc || !q || !length || !dt_out) return fail(H3C_E_INVALID, "null argument");
  if (desc->nd != 2 && desc->nd != 3) return fail(H3C_E_INVALID, "nd must be 2 or 3");
  if (desc->physics < 0 || desc->physics > 2)
    return fail(H3C_E_INVALID, "physics must be Euler, CNS or heat (advection is not covered)");
  if (n_cells < 1 || n_cells > kNoAllocMaxCells)
    return fail(H3C_E_INVALID, "n_cells must be in [1, " + std::to_string(kNoAllocMaxCells) +
                                   "]: the fixed scratch array holds one partial minimum per 256 cells");
  if (ld < n_cells) return fail(H3C_E_INVALID, "ld < n_cells");
  long long* scratch = nullptr;
  if (int rc = scratch_address(&scratch))
    return fail(rc, "cudaGetSymbolAddress of the scratch array failed on the current device");
  // physical constants: euler/quantities.hpp:131-145, cns/quantities.hpp:28-30, 74-75
  const double gamma = desc->gamma, gm1 = gamma - 1.;
  const double T_inf = 1.0 / (1 + 0.5 * gm1 * (desc->Minfty * desc->Minfty));
  const double rho_inf = std::pow(T_inf, 1. / gm1);
  const double u_inf = desc->Minfty * std::sqrt(T_inf);
  const double sOverTref = desc->T0 > 0 ? desc->Sutherland0 / desc->T0 : 0.0;
  const double sOverTrefP1 = sOverTref + 1.0;
  const double mu_inf = std::pow(T_inf, 1.5) * sOverTrefP1 / (T_inf + sOverTref);
  const double Re0 = desc->physics == H3C_CNS ? desc->ReInfty * mu_inf / (rho_inf * u_inf) : 1.0;
  const PhysConst pc{gamma, gm1, desc->cfl, desc->cfl_viscous, Re0, desc->Pr0, sOverTref, sOverTrefP1};
  const int nblocks = (int)((n_cells + kBlock - 1) / kBlock);
  cudaStream_t st = (cudaStream_t)stream;
  if (desc->nd == 2) {
    if (desc->physics == H3C_EULER) k_cfl_partials<2, EULER><<<nblocks, kBlock, 0, st>>>(q, ld, length, n_cells, pc, scratch);
    else if (desc->physics == H3C_CNS) k_cfl_partials<2, CNS><<<nblocks, kBlock, 0, st>>>(q, ld, length, n_cells, pc, scratch);
    else k_cfl_partials<2, HEAT><<<nblocks, kBlock, 0, st>>>(q, ld, length, n_cells, pc, scratch);
  } else {
    if (desc->physics == H3C_EULER) k_cfl_partials<3, EULER><<<nblocks, kBlock, 0, st>>>(q, ld, length, n_cells, pc, scratch);
    else if (desc->physics == H3C_CNS) k_cfl_partials<3, CNS><<<nblocks, kBlock, 0, st>>>(q, ld, length, n_cells, pc, scratch);
    else k_cfl_partials<3, HEAT><<<nblocks, kBlock, 0, st>>>(q, ld, length, n_cells, pc, scratch);
  }
  k_cfl_fold<<<1, kBlock, 0, st>>>(scratch, nblocks, dt_out);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? H3C_OK : fail(H3C_E_CUDA, cudaGetErrorString(e));
}
