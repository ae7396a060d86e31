// cg_mixed_inst.cu -- instantiation and launchers of the FP32-mixed kernels.
#include <cstring>

#include "cg_internal.h"
#include "cg_mixed.cuh"

namespace cg {
namespace mixed {

namespace {
dim3 grid3(int nx, int ny, int nz) { return dim3((nz + kBZ - 1) / kBZ, (ny + kBY - 1) / kBY, (nx + kBX - 1) / kBX); }

template <int M>
constexpr size_t smem_bytes() {
  return sizeof(float) * NSlot<M>::value * kThreads;
}

// dynamic shared memory above the 48 KB default (the scalar slots) needs
// the kernel's attribute raised once
template <class K>
cudaError_t allow_smem(K kernel, size_t smem, bool& done) {
  if (done || smem <= 48 * 1024) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) done = true;
  return e;
}

template <int O, int M, bool KO>
cudaError_t go(const MixedBox& b, const Bg& bg, int stage, cudaStream_t st) {
  Ptrs P{};
  P.p = b.P;
  P.f = b.F;
  P.newp = b.P;
  P.status = b.status;
  P.kavg = b.kavg;
  switch (stage) {
    case 1: P.in = b.X; P.prev = nullptr; P.out = b.Y; P.fp_in = b.FP0; P.fp_out = b.FP1; break;
    case 2: P.in = b.Y; P.prev = b.X; P.out = b.X; P.fp_in = b.FP1; P.fp_out = b.FP0; break;
    case 3: P.in = b.X; P.prev = b.Y; P.out = b.Y; P.fp_in = b.FP0; P.fp_out = b.FP1; break;
    default: P.in = b.Y; P.prev = b.X; P.out = b.X; P.fp_in = b.FP1; P.fp_out = b.FP0; break;
  }
  constexpr size_t smem = smem_bytes<M>();
  static bool done = false;
  cudaError_t e = allow_smem(mixed_kernel<O, M, KO>, smem, done);
  if (e != cudaSuccess) return e;
  const CUtensorMap& map = (stage == 1 || stage == 3) ? b.mapX : b.mapY;  // the substep's input
  mixed_kernel<O, M, KO><<<grid3(b.nx - 2 * b.xg, b.ny, b.nz), dim3(kBZ, kBY, kBX), smem, st>>>(
      b.nx, b.ny, b.nz, b.lapse, b.normalize, (float)(1.0 / b.dx), b.dt, bg, P, stage, map, b.tma, b.xg / kBX);
  return cudaGetLastError();
}
template <int O, bool KO>
cudaError_t go_mk(const MixedBox& b, const Bg& bg, int stage, cudaStream_t st) {
  switch (b.matter) {
    case kDust: return go<O, kDust, KO>(b, bg, stage, st);
    case kScalar: return go<O, kScalar, KO>(b, bg, stage, st);
    default: return go<O, kVacuum, KO>(b, bg, stage, st);
  }
}
// Kreiss-Oliger dissipation exists for stencil orders 2 and 8 (utils/math.h:36-72)
template <int O>
cudaError_t go_m(const MixedBox& b, const Bg& bg, int stage, cudaStream_t st) {
  if constexpr (O == 2 || O == 8) {
    if (b.ko != 0.0) return go_mk<O, true>(b, bg, stage, st);
  }
  return go_mk<O, false>(b, bg, stage, st);
}

template <int O, int M>
cudaError_t go_group(const GroupBox* table, const GroupBg& gb, int stage, int grid, cudaStream_t st) {
  constexpr size_t smem = smem_bytes<M>();
  static bool done = false;
  cudaError_t e = allow_smem(mixed_group_kernel<O, M>, smem, done);
  if (e != cudaSuccess) return e;
  const int g = grid > 0 ? grid : gb.total;
  mixed_group_kernel<O, M><<<g, dim3(kBZ, kBY, kBX), smem, st>>>(table, gb, stage);
  return cudaGetLastError();
}
template <int O>
cudaError_t go_group_m(const GroupBox* table, const GroupBg& gb, int matter, int stage, int grid, cudaStream_t st) {
  switch (matter) {
    case kDust: return go_group<O, kDust>(table, gb, stage, grid, st);
    case kScalar: return go_group<O, kScalar>(table, gb, stage, grid, st);
    default: return go_group<O, kVacuum>(table, gb, stage, grid, st);
  }
}
template <int O, int M>
int ctas() {
  constexpr size_t smem = smem_bytes<M>();
  static bool done = false;
  if (allow_smem(mixed_group_kernel<O, M>, smem, done) != cudaSuccess) return 1;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mixed_group_kernel<O, M>, kThreads, smem) != cudaSuccess)
    return 1;
  return n > 0 ? n : 1;
}
template <int O>
int ctas_m(int matter) {
  switch (matter) {
    case kDust: return ctas<O, kDust>();
    case kScalar: return ctas<O, kScalar>();
    default: return ctas<O, kVacuum>();
  }
}
template <int O>
bool encode_maps(MixedBox& b) {
  using G = TileG<O>;
  return tma_host::encode(&b.mapX, b.X, sizeof(float), b.nx, b.ny, b.nz, b.nfields, G::TZ, G::TY, G::TX) &&
         tma_host::encode(&b.mapY, b.Y, sizeof(float), b.nx, b.ny, b.nz, b.nfields, G::TZ, G::TY, G::TX);
}
}  // namespace

void make_tile_maps(MixedBox& b) {
  std::memset(&b.mapX, 0, sizeof(b.mapX));
  std::memset(&b.mapY, 0, sizeof(b.mapY));
  b.maps = b.tma = 0;
  // row strides must be multiples of 16 bytes; the bases are cudaMalloc'd
  if (b.nz % 4 != 0 || !b.X || !b.Y) return;
  bool ok = false;
  switch (b.order) {
    case 2: ok = encode_maps<2>(b); break;
    case 4: ok = encode_maps<4>(b); break;
    case 6: ok = encode_maps<6>(b); break;
    case 8: ok = encode_maps<8>(b); break;
    default: break;
  }
  b.maps = b.tma = ok ? 1 : 0;
}

cudaError_t launch_group(const GroupBox* table, const GroupBg& gb, int order, int matter, int stage, int grid,
                         cudaStream_t st) {
  switch (order) {
    case 2: return go_group_m<2>(table, gb, matter, stage, grid, st);
    case 4: return go_group_m<4>(table, gb, matter, stage, grid, st);
    case 6: return go_group_m<6>(table, gb, matter, stage, grid, st);
    case 8: return go_group_m<8>(table, gb, matter, stage, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

int group_ctas_per_sm(int order, int matter) {
  switch (order) {
    case 2: return ctas_m<2>(matter);
    case 4: return ctas_m<4>(matter);
    case 6: return ctas_m<6>(matter);
    default: return ctas_m<8>(matter);
  }
}

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
  switch (b.matter) {
    case kDust: mixed_init_kernel<kDust><<<g, blk, 0, st>>>(b.nx, b.ny, b.nz, b.normalize, bg, b.P, b.X, b.FP0); break;
    case kScalar: mixed_init_kernel<kScalar><<<g, blk, 0, st>>>(b.nx, b.ny, b.nz, b.normalize, bg, b.P, b.X, b.FP0); break;
    default: mixed_init_kernel<kVacuum><<<g, blk, 0, st>>>(b.nx, b.ny, b.nz, b.normalize, bg, b.P, b.X, b.FP0); break;
  }
  return cudaGetLastError();
}

}  // namespace mixed
}  // namespace cg
