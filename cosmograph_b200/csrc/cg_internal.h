// cg_internal.h -- host-side declarations shared by the CUDA translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "cg_group.h"
#include "cg_types.h"

namespace cg {

// Device storage of one periodic box.  Every register block holds
// nfields arrays of pts doubles (field f at offset f*pts), x-major with z
// fastest like the reference's CosmoArray (utils/Array.h:47-61).
struct BoxDev {
  CUtensorMap mapX, mapY;  // TMA maps of X and Y (4-D {nz, ny, nx, field}); valid when maps != 0
  int maps;                // the maps are encoded
  int tma;                 // interior tiles are copied by TMA (maps != 0 and the option on)
  int nx, ny, nz, pts, nfields, order, matter;
  int xg;  // ghost planes on each x face (0: periodic box)
  int z4c;  // Z4c damping: theta is field nfields - 1 (stage_kernel<..., Z4C = true>)
  int shift;  // the shift: beta1..3, auxB1..3, expN are the last 7 fields (stage_kernel<..., SHIFT = true>)
  CUtensorMap fmap0[3], fmap1[3];  // TMA maps of the flux primitives FP0 / FP1 (x, y, z boxes)
  int fmaps;                       // those maps are encoded
  Physics ph;
  double* P;    // the reference's _p register (state at the start of a step)
  double* F;    // the reference's _f register (RK accumulator)
  double* X;    // substep inputs a^1 (normalised), a^3 and, after a step, the next a^1
  double* Y;    // substep inputs a^2, a^4
  double* FP0;  // dust flux primitives (P_N arrays) of a^1, a^3
  double* FP1;  // dust flux primitives of a^2, a^4
  unsigned* status;
  const double* kavg;  // device K_avg for the lapses that use it, else null
};

// Device storage of one box evolved in the FP32-mixed form: FP64 _p and _f,
// FP32 perturbation substep inputs and dust flux primitives.
struct MixedBox {
  CUtensorMap mapX, mapY;  // TMA maps of X and Y (4-D {nz, ny, nx, field}); valid when maps != 0
  int maps;                // the maps are encoded
  int tma;                 // interior tiles are copied by TMA (maps != 0 and the option on)
  int nx, ny, nz, pts, nfields, order, matter, lapse, normalize;
  int xg;  // ghost planes on each x face (0: periodic box)
  double dx, dt;
  double ko;     // Kreiss-Oliger coefficient (0: none)
  double* kavg;  // device K_avg - Kbar of the substep input (lapses with K_avg), else null
  double* P;
  double* F;
  float* X;
  float* Y;
  float* FP0;
  float* FP1;
  unsigned* status;
};
namespace mixed {
struct Bg;
struct GroupBox;
struct GroupBg;
cudaError_t launch_stage(const MixedBox& b, const Bg& bg, int stage, cudaStream_t st);
cudaError_t launch_init(const MixedBox& b, const Bg& bg, cudaStream_t st);
// encode b.mapX / b.mapY and set b.maps = b.tma = 1 when the box allows TMA tile copies
void make_tile_maps(MixedBox& b);
// one launch for substep `stage` of every box of a mixed group (as launch_group)
cudaError_t launch_group(const GroupBox* table, const GroupBg& gb, int order, int matter, int stage, int grid,
                         cudaStream_t st);
int group_ctas_per_sm(int order, int matter);
}  // namespace mixed

// Kernel variants: identical source, compiled without (exact) or with (fast)
// FMA contraction.
enum Variant : int { kExact = 0, kFast = 1 };

namespace tma_host {
// 4-D tensor map {nz, ny, nx, nfields} of elem-byte floats (4 or 8) at base,
// box {bz, by, bx, 1}; false (map zeroed) when the layout or the driver does
// not allow it
bool encode(CUtensorMap* map, void* base, int elem, int nx, int ny, int nz, int nfields, int bz, int by, int bx);
}  // namespace tma_host

namespace exact {
// encode b.mapX / b.mapY and set b.maps = b.tma = 1 when the box allows TMA tile copies
void make_tile_maps(BoxDev& b);
cudaError_t launch_stage(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st);
cudaError_t launch_init(const BoxDev& b, const StageBg& bg, cudaStream_t st);
// constraint statistics pass 1 on the first-substep input X: per-point values
// (10 arrays of pts) into cvals, 27 partial results per CTA into cpart
cudaError_t launch_constraints(const BoxDev& b, const StageBg& bg, double* cvals, double* cpart, cudaStream_t st);
int constraint_blocks(const BoxDev& b);
// the Z4c instantiations (cg_stage_inst.cu built with -DCG_Z4C_UNIT=1)
cudaError_t launch_stage_z4c(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st);
cudaError_t launch_constraints_z4c(const BoxDev& b, const StageBg& bg, double* cvals, double* cpart, cudaStream_t st);
// the shift instantiations (cg_stage_inst.cu built with -DCG_SHIFT_UNIT=1; the
// parity build only)
cudaError_t launch_stage_shift(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st);
}  // namespace exact
namespace fast {
void make_tile_maps(BoxDev& b);
cudaError_t launch_stage(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st);
cudaError_t launch_init(const BoxDev& b, const StageBg& bg, cudaStream_t st);
cudaError_t launch_stage_z4c(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st);
cudaError_t launch_constraints_z4c(const BoxDev& b, const StageBg& bg, double* cvals, double* cpart, cudaStream_t st);
cudaError_t launch_stage_shift(const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st);
}  // namespace fast

// One launch for substep `stage` of every box of an FP64 group (table: device
// copy of the group's GroupBox entries in launch order).  grid <= 0: one CTA
// per brick; otherwise a persistent grid of that many CTAs.
namespace exact {
cudaError_t launch_group(const GroupBox* table, const GroupBg& gb, int order, int matter, int stage, int grid,
                         cudaStream_t st);
int group_ctas_per_sm(int order, int matter);
}  // namespace exact
namespace fast {
cudaError_t launch_group(const GroupBox* table, const GroupBg& gb, int order, int matter, int stage, int grid,
                         cudaStream_t st);
int group_ctas_per_sm(int order, int matter);
}  // namespace fast
inline cudaError_t launch_group(int v, const GroupBox* table, const GroupBg& gb, int order, int matter, int stage,
                                int grid, cudaStream_t st) {
  return v == kFast ? fast::launch_group(table, gb, order, matter, stage, grid, st)
                    : exact::launch_group(table, gb, order, matter, stage, grid, st);
}
inline int group_ctas_per_sm(int v, int order, int matter) {
  return v == kFast ? fast::group_ctas_per_sm(order, matter) : exact::group_ctas_per_sm(order, matter);
}

// Volume-weighted average (utils/math.h:1403-1415) of n values of `field`,
// weights exp(6 (phi + phi_frw)); `partial` holds 2*nblk doubles of scratch,
// the result lands in out[0] (device).  Defined in cg_abi.cu.
cudaError_t launch_conformal_average(const double* field, const double* phi, int n, double phi_frw,
                                     double* partial, int nblk, double* out, cudaStream_t st);

// GPU initial data (cg_ics.cu)
struct GridSpec {
  int nx, ny, nz, order;
  double dx;
};
namespace ics {
size_t grf_scratch_doubles(const GridSpec& s);
int grf_dust(const GridSpec& s, double* P, double* scratch, const double* delta_host, uint64_t seed, double rms,
             double ns, double kc, double rho_L, cudaStream_t st, std::string& err);
int grf_scalar(const GridSpec& s, double* P, double* scratch, const double* dphi_host, uint64_t seed, double rms,
               double phi0, double mass, double kc, cudaStream_t st, std::string& err);
}  // namespace ics

// Message returned by cg_last_error(NULL) on this host thread.
void set_global_error(const char* msg);

inline cudaError_t launch_stage(int v, const BoxDev& b, const StageBg& bg, int stage, cudaStream_t st) {
  return v == kFast ? fast::launch_stage(b, bg, stage, st) : exact::launch_stage(b, bg, stage, st);
}
inline cudaError_t launch_init(int v, const BoxDev& b, const StageBg& bg, cudaStream_t st) {
  return v == kFast ? fast::launch_init(b, bg, st) : exact::launch_init(b, bg, st);
}

}  // namespace cg
