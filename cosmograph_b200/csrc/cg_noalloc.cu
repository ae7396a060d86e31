// cg_noalloc.cu -- cg_conformal_average_noalloc: the volume-weighted grid
// average without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: programs that hand all
// device memory to their own pool or run under a fixed memory budget, and
// code that must not trigger the implicit device synchronisation a
// cudaMalloc/cudaFree can cause.  This entry point keeps its scratch (the
// per-block partial sums of the reduction) in a fixed array compiled into
// the library instead.  The array exists once per GPU for the life of the
// process, whether or not the entry point is ever called, and every call on
// that GPU shares it.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "cosmograph_b200.h"
#include "cg_internal.h"

namespace {

constexpr int kMaxBlocks = CG_NOALLOC_MAX_BLOCKS;
constexpr size_t kMaxPoints = CG_NOALLOC_MAX_POINTS;
constexpr int kMaxDevices = 64;

// Two partial sums per reduction block: 2 * 1024 doubles = 16 KiB per GPU.
__device__ __align__(256) double g_scratch[2 * kMaxBlocks];

std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};  // device address of g_scratch, per device

// Host code cannot use g_scratch directly: in host code the name refers to a
// host-side stand-in, not device memory.  Look up the device address once
// per device, with that device current.
int scratch_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cg::set_global_error((std::string("cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
    return CG_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    cg::set_global_error("device index beyond the supported range");
    return CG_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) {
      cg::set_global_error((std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e)).c_str());
      return CG_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return CG_OK;
}

}  // namespace

extern "C" int cg_conformal_average_noalloc(const double* d_field, const double* d_phi, size_t n,
                                            double phi_frw, double* d_out, void* stream) {
  if (!d_field || !d_phi || !d_out) {
    cg::set_global_error("null pointer");
    return CG_ERR_INVALID;
  }
  if (n == 0 || n > kMaxPoints) {
    cg::set_global_error(("n must be in 1.." + std::to_string(kMaxPoints) +
                          " (the fixed scratch of cg_conformal_average_noalloc)").c_str());
    return CG_ERR_INVALID;
  }
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != CG_OK) return rc;
  const int nblk = (int)((n + 255) / 256 < (size_t)kMaxBlocks ? (n + 255) / 256 : (size_t)kMaxBlocks);
  // every block rewrites its own partial sums, so nothing has to be cleared
  cudaError_t e = cg::launch_conformal_average(d_field, d_phi, (int)n, phi_frw, scratch, nblk, d_out,
                                               static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) {
    cg::set_global_error((std::string("kernel launch: ") + cudaGetErrorString(e)).c_str());
    return CG_ERR_CUDA;
  }
  return CG_OK;
}
