// cg_mixed_inst.cu -- instantiation and launchers of the FP32-mixed kernels.
#include "cg_internal.h"
#include "cg_mixed.cuh"

namespace cg {
namespace mixed {

namespace {
dim3 grid3(int nx, int ny, int nz) { return dim3((nz + kBZ - 1) / kBZ, (ny + kBY - 1) / kBY, (nx + kBX - 1) / kBX); }

template <int O, int M>
cudaError_t go(const MixedBox& b, const Bg& bg, int stage, cudaStream_t st) {
  Ptrs P{};
  P.p = b.P;
  P.f = b.F;
  P.newp = b.P;
  P.status = b.status;
  switch (stage) {
    case 1: P.in = b.X; P.prev = nullptr; P.out = b.Y; P.fp_in = b.FP0; P.fp_out = b.FP1; break;
    case 2: P.in = b.Y; P.prev = b.X; P.out = b.X; P.fp_in = b.FP1; P.fp_out = b.FP0; break;
    case 3: P.in = b.X; P.prev = b.Y; P.out = b.Y; P.fp_in = b.FP0; P.fp_out = b.FP1; break;
    default: P.in = b.Y; P.prev = b.X; P.out = b.X; P.fp_in = b.FP1; P.fp_out = b.FP0; break;
  }
  constexpr size_t smem = sizeof(float) * S_NSLOT * kThreads;
  mixed_kernel<O, M><<<grid3(b.nx, b.ny, b.nz), dim3(kBZ, kBY, kBX), smem, st>>>(
      b.nx, b.ny, b.nz, b.lapse, b.normalize, (float)(1.0 / b.dx), b.dt, bg, P, stage);
  return cudaGetLastError();
}
template <int O>
cudaError_t go_m(const MixedBox& b, const Bg& bg, int stage, cudaStream_t st) {
  return b.matter == kDust ? go<O, kDust>(b, bg, stage, st) : go<O, kVacuum>(b, bg, stage, st);
}
}  // namespace

cudaError_t launch_stage(const MixedBox& b, const Bg& bg, int stage, cudaStream_t st) {
  switch (b.order) {
    case 2: return go_m<2>(b, bg, stage, st);
    case 4: return go_m<4>(b, bg, stage, st);
    case 6: return go_m<6>(b, bg, stage, st);
    case 8: return go_m<8>(b, bg, stage, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_init(const MixedBox& b, const Bg& bg, cudaStream_t st) {
  const dim3 g = grid3(b.nx, b.ny, b.nz), blk(kBZ, kBY, kBX);
  if (b.matter == kDust)
    mixed_init_kernel<kDust><<<g, blk, 0, st>>>(b.nx, b.ny, b.nz, b.normalize, bg, b.P, b.X, b.FP0);
  else
    mixed_init_kernel<kVacuum><<<g, blk, 0, st>>>(b.nx, b.ny, b.nz, b.normalize, bg, b.P, b.X, b.FP0);
  return cudaGetLastError();
}

}  // namespace mixed
}  // namespace cg
