// cg_stage_inst.cu -- instantiates the substep and step-initialisation kernels.
//
// Compiled twice: with -DCG_VARIANT_NS=exact and --fmad=false (the parity
// build: every product and sum rounds separately, as in the reference's
// strict build), and with -DCG_VARIANT_NS=fast and --fmad=true.
#include "cg_internal.h"
#include "cg_stage.cuh"

#ifndef CG_VARIANT_NS
#error "CG_VARIANT_NS must be defined (exact or fast)"
#endif

// Built a second time with -DCG_Z4C_UNIT=1: the Z4c-damping instantiations of
// the substep and constraint kernels (launch_stage_z4c, launch_constraints_z4c)
// in a translation unit of their own, so that the two compile in parallel.
#ifndef CG_Z4C_UNIT
#define CG_Z4C_UNIT 0
#endif
// Built with -DCG_SHIFT_UNIT=1 (parity build only): the shift instantiations
// of the substep kernel (launch_stage_shift), Kreiss-Oliger compiled in.
#ifndef CG_SHIFT_UNIT
#define CG_SHIFT_UNIT 0
#endif
#define CG_AUX_UNIT (CG_Z4C_UNIT || CG_SHIFT_UNIT)

namespace cg {
namespace CG_VARIANT_NS {

constexpr bool kZ4cUnit = CG_Z4C_UNIT != 0;
constexpr bool kShiftUnit = CG_SHIFT_UNIT != 0;

#if !CG_AUX_UNIT
// BSSN::stepInit (bssn.cc:219-226) on the device: the first substep's input
// is the normalised copy of _p (RK4Register::stepInit + set_DIFFgamma_Aij_norm);
// for dust also the flux primitives of that input (Dust::stepInit ->
// populateDerivedFields, dust.cc:65-72 and :121-133).
template <int MATTER>
__global__ void __launch_bounds__(128) init_kernel(BoxGeom geo, Physics ph, StageBg bg, const double* P,
                                                   double* X, double* FP0) {
  constexpr int NFLD = NF<MATTER>::value;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= geo.nz || j >= geo.ny) return;
  const int c = (i * geo.ny + j) * geo.nz + k;
  const int N = geo.pts;
  double v[NFLD];
#pragma unroll
  for (int f = 0; f < NFLD; ++f) v[f] = P[(size_t)f * N + c];
  if (ph.normalize) {
    double g[6], A[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) { g[m] = v[F_G11 + m]; A[m] = v[F_A11 + m]; }
    normalize_point(g, A);
#pragma unroll
    for (int m = 0; m < 6; ++m) { v[F_G11 + m] = g[m]; v[F_A11 + m] = A[m]; }
  }
#pragma unroll
  for (int f = 0; f < NFLD; ++f) X[(size_t)f * N + c] = v[f];
  if (MATTER == kDust) {
    double g[6], gi[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) g[m] = v[F_G11 + m];
    inv_metric(g, gi);
    const double S[3] = {v[F_S1], v[F_S2], v[F_S3]};
    const double phi = v[F_PHI] + bg.phi_FRW;
    double e[2];
    {
      const double x[2] = {-4.0 * phi, 6.0 * phi};
      xexp_n<2>(x, e);
    }
    const DustPrim dp = dust_prim(gi, e[0], e[1], v[F_D], S);
    const double al = v[F_ALPHA] + 1.0;
    FP0[(size_t)P_AD * N + c] = al * v[F_D];
#pragma unroll
    for (int m = 0; m < 3; ++m) FP0[(size_t)(P_AS1 + m) * N + c] = al * S[m];
#pragma unroll
    for (int m = 0; m < 3; ++m) FP0[(size_t)(P_V1 + m) * N + c] = dp.v[m];
  }
}

#endif  // !CG_AUX_UNIT

namespace {
dim3 block_dims() { return dim3(32, 4, 1); }
dim3 grid_dims(const BoxDev& b) {
  return dim3((b.nz + 31) / 32, (b.ny + 3) / 4, b.nx);
}
dim3 stage_block() { return dim3(kBZ, kBY, kBX); }
// bricks of the points a substep updates: x-slab boxes skip their ghost planes
dim3 stage_grid(const BoxDev& b) {
  return dim3((b.nz + kBZ - 1) / kBZ, (b.ny + kBY - 1) / kBY, (b.nx - 2 * b.xg + kBX - 1) / kBX);
}

template <int O, int M>
cudaError_t go_stage(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st) {
  StagePtrs P{};
  P.kavg = b.kavg;
  P.p = b.P;
  P.f = b.F;
  P.status = b.status;
  switch (stage) {
    case 1: P.in = b.X; P.prev = nullptr; P.out = b.Y; P.fp_in = b.FP0; P.fp_out = b.FP1; break;
    case 2: P.in = b.Y; P.prev = b.X; P.out = b.X; P.fp_in = b.FP1; P.fp_out = b.FP0; break;
    case 3: P.in = b.X; P.prev = b.Y; P.out = b.Y; P.fp_in = b.FP0; P.fp_out = b.FP1; break;
    default: P.in = b.Y; P.prev = b.X; P.out = b.P; P.norm = b.X; P.fp_in = b.FP1; P.fp_out = b.FP0; break;
  }
  BoxGeom geo{b.nx, b.ny, b.nz, b.pts, b.xg / kBX};
  const CUtensorMap& map = (stage == 1 || stage == 3) ? b.mapX : b.mapY;  // the substep's input
  FluxMaps fm;
  const CUtensorMap* fsrc = (stage == 1 || stage == 3) ? b.fmap0 : b.fmap1;
  for (int a = 0; a < 3; ++a) fm.m[a] = fsrc[a];
  constexpr bool Z = kZ4cUnit;
  constexpr size_t smem = stage_smem<O, M, kEvolve, Z>();
  if constexpr (kShiftUnit) {
    // one instantiation per order and matter; the dissipation is switched at run time
    static bool configured_shift = false;
    if (!configured_shift) {
      cudaError_t e = cudaFuncSetAttribute(stage_kernel<O, M, kEvolve, true, false, true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      configured_shift = true;
    }
    stage_kernel<O, M, kEvolve, true, false, true><<<stage_grid(b), stage_block(), smem, st>>>(
        geo, b.ph, bg, P, stage, map, b.tma, fm, b.fmaps);
    return cudaGetLastError();
  }
  if constexpr (O == 2 || O == 8) {
    if (b.ph.ko_coeff != 0.0) {  // Kreiss-Oliger dissipation: its own instantiation
      static bool configured_ko = false;
      if (!configured_ko) {
        cudaError_t e = cudaFuncSetAttribute(stage_kernel<O, M, kEvolve, true, Z>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        configured_ko = true;
      }
      stage_kernel<O, M, kEvolve, true, Z><<<stage_grid(b), stage_block(), smem, st>>>(geo, b.ph, bg, P, stage, map,
                                                                                       b.tma, fm, b.fmaps);
      return cudaGetLastError();
    }
  }
  static bool configured = false;  // per instantiation
  if (!configured) {
    cudaError_t e =
        cudaFuncSetAttribute(stage_kernel<O, M, kEvolve, false, Z>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  stage_kernel<O, M, kEvolve, false, Z><<<stage_grid(b), stage_block(), smem, st>>>(geo, b.ph, bg, P, stage, map,
                                                                                    b.tma, fm, b.fmaps);
  return cudaGetLastError();
}

#if !CG_SHIFT_UNIT
template <int O, int M>
cudaError_t go_constraints(const BoxDev& b, const StageBg& bg, double* cvals, double* cpart, cudaStream_t st) {
  StagePtrs P{};
  P.in = b.X;
  P.p = b.P;
  P.fp_in = b.FP0;
  P.status = b.status;
  P.kavg = b.kavg;
  P.cvals = cvals;
  P.cpart = cpart;
  BoxGeom geo{b.nx, b.ny, b.nz, b.pts, b.xg / kBX};
  constexpr bool Z = kZ4cUnit;
  constexpr size_t smem = stage_smem<O, M, kConstraints, Z>();
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel<O, M, kConstraints, false, Z>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  FluxMaps fm{};
  stage_kernel<O, M, kConstraints, false, Z><<<stage_grid(b), stage_block(), smem, st>>>(geo, b.ph, bg, P, 1, b.mapX,
                                                                                         b.tma, fm, 0);
  return cudaGetLastError();
}

template <int O>
cudaError_t go_constraints_m(const BoxDev& b, const StageBg& bg, double* cvals, double* cpart, cudaStream_t st) {
  switch (b.matter) {
    case kDust: return go_constraints<O, kDust>(b, bg, cvals, cpart, st);
    case kScalar: return go_constraints<O, kScalar>(b, bg, cvals, cpart, st);
    case kStaticMatter: return go_constraints<O, kStaticMatter>(b, bg, cvals, cpart, st);
    default: return go_constraints<O, kVacuum>(b, bg, cvals, cpart, st);
  }
}
#endif  // !CG_SHIFT_UNIT

#if !CG_AUX_UNIT
template <int O, int M>
cudaError_t go_group(const GroupBox* table, const GroupBg& gb, int stage, int grid, cudaStream_t st) {
  constexpr size_t smem = stage_smem<O, M, kEvolve>();
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(stage_group_kernel<O, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const int g = grid > 0 ? grid : gb.total;
  stage_group_kernel<O, M><<<g, stage_block(), smem, st>>>(table, gb, stage);
  return cudaGetLastError();
}

template <int O, int M>
int ctas_per_sm() {
  constexpr size_t smem = stage_smem<O, M, kEvolve>();
  if (cudaFuncSetAttribute(stage_group_kernel<O, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return 1;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, stage_group_kernel<O, M>, kThreads, smem) != cudaSuccess)
    return 1;
  return n > 0 ? n : 1;
}

template <int O>
cudaError_t go_group_m(const GroupBox* table, const GroupBg& gb, int matter, int stage, int grid, cudaStream_t st) {
  switch (matter) {
    case kDust: return go_group<O, kDust>(table, gb, stage, grid, st);
    case kScalar: return go_group<O, kScalar>(table, gb, stage, grid, st);
    case kStaticMatter: return go_group<O, kStaticMatter>(table, gb, stage, grid, st);
    default: return go_group<O, kVacuum>(table, gb, stage, grid, st);
  }
}
template <int O>
int ctas_m(int matter) {
  switch (matter) {
    case kDust: return ctas_per_sm<O, kDust>();
    case kScalar: return ctas_per_sm<O, kScalar>();
    case kStaticMatter: return ctas_per_sm<O, kStaticMatter>();
    default: return ctas_per_sm<O, kVacuum>();
  }
}

#endif  // !CG_AUX_UNIT

template <int O>
cudaError_t go_stage_m(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st) {
  switch (b.matter) {
    case kDust: return go_stage<O, kDust>(b, bg, stage, st);
    case kScalar: return go_stage<O, kScalar>(b, bg, stage, st);
#if !CG_SHIFT_UNIT  // static matter has no shift (cg_create rejects it)
    case kStaticMatter: return go_stage<O, kStaticMatter>(b, bg, stage, st);
#endif
    default: return go_stage<O, kVacuum>(b, bg, stage, st);
  }
}
#if !CG_AUX_UNIT
template <int O>
bool encode_maps(BoxDev& b) {
  using G = TileG<O>;
  b.fmaps = 0;
  if (!(tma_host::encode(&b.mapX, b.X, sizeof(double), b.nx, b.ny, b.nz, b.nfields, G::TZ, G::TY, G::TX) &&
        tma_host::encode(&b.mapY, b.Y, sizeof(double), b.nx, b.ny, b.nz, b.nfields, G::TZ, G::TY, G::TX)))
    return false;
  if (b.FP0 && b.FP1) {  // dust: x, y, z boxes of the flux primitives
    constexpr int R = O / 2;
    const int box[3][3] = {{kBZ, kBY, kBX + 2 * R}, {kBZ, kBY + 2 * R, kBX}, {G::TZ, kBY, kBX}};
    bool ok = true;
    for (int a = 0; a < 3; ++a) {
      ok = ok && tma_host::encode(&b.fmap0[a], b.FP0, sizeof(double), b.nx, b.ny, b.nz, P_N, box[a][0], box[a][1],
                                  box[a][2]);
      ok = ok && tma_host::encode(&b.fmap1[a], b.FP1, sizeof(double), b.nx, b.ny, b.nz, P_N, box[a][0], box[a][1],
                                  box[a][2]);
    }
    b.fmaps = ok ? 1 : 0;
  }
  return true;
}
#endif  // !CG_AUX_UNIT
}  // namespace

#if !CG_AUX_UNIT
void make_tile_maps(BoxDev& b) {
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

#endif  // !CG_AUX_UNIT

#if !CG_AUX_UNIT && !CG_REFERENCE_ORDER
// the shift is built into the parity build only; cg_create accepts it with CG_PREC_FP64 alone
cudaError_t launch_stage_shift(const BoxDev&, const StageBg&, int, cudaStream_t) { return cudaErrorNotSupported; }
#endif

#if CG_Z4C_UNIT
cudaError_t launch_stage_z4c(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st) {
#elif CG_SHIFT_UNIT
cudaError_t launch_stage_shift(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st) {
#else
cudaError_t launch_stage(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st) {
  if (b.z4c) return launch_stage_z4c(b, bg, stage, st);
  if (b.shift) return launch_stage_shift(b, bg, stage, st);
#endif
  switch (b.order) {
    case 2: return go_stage_m<2>(b, bg, stage, st);
    case 4: return go_stage_m<4>(b, bg, stage, st);
    case 6: return go_stage_m<6>(b, bg, stage, st);
    case 8: return go_stage_m<8>(b, bg, stage, st);
    default: return cudaErrorInvalidValue;
  }
}

#if !CG_SHIFT_UNIT  // shift boxes take the constraint statistics of the plain kernels
#if CG_Z4C_UNIT
cudaError_t launch_constraints_z4c(const BoxDev& b, const StageBg& bg, double* cvals, double* cpart, cudaStream_t st) {
#else
cudaError_t launch_constraints(const BoxDev& b, const StageBg& bg, double* cvals, double* cpart, cudaStream_t st) {
  if (b.z4c) return launch_constraints_z4c(b, bg, cvals, cpart, st);
#endif
  switch (b.order) {
    case 2: return go_constraints_m<2>(b, bg, cvals, cpart, st);
    case 4: return go_constraints_m<4>(b, bg, cvals, cpart, st);
    case 6: return go_constraints_m<6>(b, bg, cvals, cpart, st);
    case 8: return go_constraints_m<8>(b, bg, cvals, cpart, st);
    default: return cudaErrorInvalidValue;
  }
}
#endif  // !CG_SHIFT_UNIT

#if !CG_AUX_UNIT
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

int constraint_blocks(const BoxDev& b) {
  const dim3 g = stage_grid(b);
  return (int)(g.x * g.y * g.z);
}

cudaError_t launch_init(const BoxDev& b, const StageBg& bg, cudaStream_t st) {
  BoxGeom geo{b.nx, b.ny, b.nz, b.pts, b.xg / kBX};
  switch (b.matter) {
    case kDust: init_kernel<kDust><<<grid_dims(b), block_dims(), 0, st>>>(geo, b.ph, bg, b.P, b.X, b.FP0); break;
    case kScalar: init_kernel<kScalar><<<grid_dims(b), block_dims(), 0, st>>>(geo, b.ph, bg, b.P, b.X, b.FP0); break;
    case kStaticMatter: init_kernel<kStaticMatter><<<grid_dims(b), block_dims(), 0, st>>>(geo, b.ph, bg, b.P, b.X, b.FP0); break;
    default: init_kernel<kVacuum><<<grid_dims(b), block_dims(), 0, st>>>(geo, b.ph, bg, b.P, b.X, b.FP0); break;
  }
  const int extra = (b.z4c ? 1 : 0) + (b.shift ? 7 : 0);
  if (extra) {  // theta and the shift fields: not normalised, copied as they are
    const size_t pts = (size_t)b.pts, f0 = (size_t)(b.nfields - extra);
    cudaError_t e = cudaMemcpyAsync(b.X + f0 * pts, b.P + f0 * pts, (size_t)extra * pts * sizeof(double),
                                    cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

#endif  // !CG_AUX_UNIT

}  // namespace CG_VARIANT_NS
}  // namespace cg
