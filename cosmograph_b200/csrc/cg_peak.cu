// cg_peak.cu -- the FP64 arithmetic peak of the current GPU, measured, for
// the compute roofline of the substep kernels (no counterpart in the
// reference).
//
// Every thread runs eight independent FMA chains; the grid fills every SM
// several times over, so the FP64 pipes stay busy and the latency of one
// chain is hidden by the others.  Timed with CUDA events around one launch
// after a warm-up launch.
#include <cuda_runtime.h>

#include <string>

#include "cosmograph_b200.h"
#include "cg_internal.h"

namespace {

__global__ void fma_chains_kernel(double* out, int iters, double b, double c) {
  double a[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) a[q] = 1.0 + 1e-3 * (threadIdx.x + q);
#pragma unroll 1
  for (int n = 0; n < iters; ++n) {
#pragma unroll
    for (int u = 0; u < 16; ++u)
#pragma unroll
      for (int q = 0; q < 8; ++q) a[q] = fma(a[q], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) s += a[q];
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains alive; never true for these inputs
}

}  // namespace

extern "C" int cg_fp64_peak(double* flops_per_s) {
  if (!flops_per_s) {
    cg::set_global_error("null pointer");
    return CG_ERR_INVALID;
  }
  int dev = 0, sms = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double* out = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(double) * 65536);
  if (e == cudaSuccess) e = cudaEventCreate(&t0);
  if (e == cudaSuccess) e = cudaEventCreate(&t1);
  const int threads = 256, blocks = sms * 8, iters = 2048;
  float ms = 0.0f;
  if (e == cudaSuccess) {
    fma_chains_kernel<<<blocks, threads>>>(out, iters / 8, 0.999999, 1e-7);  // warm-up
    cudaEventRecord(t0);
    fma_chains_kernel<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(t1);
    e = cudaEventSynchronize(t1);
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  cudaFree(out);
  if (e != cudaSuccess) {
    cg::set_global_error((std::string("cg_fp64_peak: ") + cudaGetErrorString(e)).c_str());
    return CG_ERR_CUDA;
  }
  // 2 flops per FMA, 16 x 8 FMAs per thread and iteration
  const double flops = 2.0 * 16.0 * 8.0 * (double)iters * (double)threads * (double)blocks;
  *flops_per_s = flops / (ms * 1e-3);
  return CG_OK;
}
