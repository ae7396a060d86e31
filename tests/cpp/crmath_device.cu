// crmath_device.cu -- evaluates the correctly rounded exp / expm1 / log1p of
// cosmograph_b200/csrc/cg_crmath.h on the GPU and, for comparison, the same
// code compiled for the host.  Test infrastructure, built by
// tests/test_crmath.py with nvcc (host part without FP contraction).
#include <cuda_runtime.h>

#include <cstddef>

#include "cg_crmath.h"

namespace {
__global__ void eval_kernel(int fn, const double* x, double* y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = x[i];
    y[i] = fn == 0 ? cg::crm::exp(v) : fn == 1 ? cg::crm::expm1(v) : cg::crm::log1p(v);
  }
}
}  // namespace

// fn: 0 exp, 1 expm1, 2 log1p.  Returns 0, or the CUDA error code.
extern "C" int crm_eval_device(int fn, const double* hx, double* hy, size_t n) {
  double *dx = nullptr, *dy = nullptr;
  cudaError_t e = cudaMalloc(&dx, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&dy, n * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(dx, hx, n * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    eval_kernel<<<592, 256>>>(fn, dx, dy, n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(hy, dy, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dy);
  return (int)e;
}

extern "C" void crm_eval_host(int fn, const double* x, double* y, size_t n) {
  for (size_t i = 0; i < n; ++i) y[i] = fn == 0 ? cg::crm::exp(x[i]) : fn == 1 ? cg::crm::expm1(x[i]) : cg::crm::log1p(x[i]);
}
