// cg_group.h -- launch groups: boxes of the same order, matter model and
// arithmetic advanced by one launch per substep (host and device types).
#pragma once

#include <cuda.h>

#include "cg_types.h"

namespace cg {

// One FP64 box of a launch group: geometry, numerics and register blocks, its
// brick counts along x, y, z and the index of its first brick in the launch's
// work list.  Device table, written once when the group is formed.
struct GroupBox {
  CUtensorMap mapX, mapY;  // TMA maps of X and Y (valid when tma != 0)
  int tma;
  int nx, ny, nz, pts;
  Physics ph;
  const double* kavg;
  double *P, *F, *X, *Y, *FP0, *FP1;
  unsigned* status;
  int nbx, nby, nbz;
  int first;
};
// TMA maps of a member's dust flux primitives (FP0, FP1; the x, y and z boxes
// of the divergence), stored after the GroupBox entries in the same device
// table (entry q at (GroupFluxMaps*)(table + nboxes) + q).
struct GroupFluxMaps {
  CUtensorMap fp0[3], fp1[3];
  int valid;
};
static_assert(sizeof(GroupBox) % alignof(GroupFluxMaps) == 0, "the flux maps after the GroupBox entries stay aligned");
constexpr int kMaxGroupBoxes = 64;
// Per-substep values of every box of an FP64 group (kernel parameter, by value).
struct GroupBg {
  int nboxes, total;
  StageBg bg[kMaxGroupBoxes];
};

}  // namespace cg
