// h3c_rates.cu -- arithmetic issue rates of the GPU the library runs on.
//
// The stage kernels do FP64 arithmetic (Newton reciprocals and square roots,
// the AUSM splits, the viscous flux) on every face; whether a kernel is bound
// by that arithmetic or by memory needs the device's FP64 rate, which the
// copy and GEMM peaks do not give.  These kernels run long chains of
// independent fused multiply-adds in registers (no memory traffic) and time
// them with CUDA events.
#include <cuda_runtime.h>

#include <string>

#include "../../include/h3c.h"

namespace gridb {
void set_global_error(const std::string& msg);
}

namespace {

constexpr int kChains = 8;    // independent accumulators per thread
constexpr int kIters = 4096;  // FMAs per chain

template <class T>
__global__ void k_fma_rate(T* out, T b, T c) {
  T a[kChains];
#pragma unroll
  for (int k = 0; k < kChains; ++k) a[k] = (T)(threadIdx.x + k);
#pragma unroll 4
  for (int i = 0; i < kIters; ++i)
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = fma(a[k], b, c);
  T s = 0;
#pragma unroll
  for (int k = 0; k < kChains; ++k) s += a[k];
  if (s == (T)-1.2345) out[0] = s;  // keeps the chains live; never true for these inputs
}

template <class T>
int rate(double* per_s) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  T* out = nullptr;
  if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return H3C_E_NOMEM;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  const int blocks = sms * 8, threads = 256;
  k_fma_rate<T><<<blocks, threads>>>(out, (T)0.999999, (T)1e-7);  // warm-up
  cudaEventRecord(a);
  k_fma_rate<T><<<blocks, threads>>>(out, (T)0.999999, (T)1e-7);
  cudaEventRecord(b);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    gridb::set_global_error(cudaGetErrorString(e));
    return H3C_E_CUDA;
  }
  *per_s = (double)blocks * threads * kChains * kIters / (ms * 1e-3);
  return H3C_OK;
}

}  // namespace

int h3c_fma_rates(double* fp64_per_s, double* fp32_per_s) {
  if (!fp64_per_s || !fp32_per_s) return H3C_E_INVALID;
  if (int rc = rate<double>(fp64_per_s)) return rc;
  return rate<float>(fp32_per_s);
}
