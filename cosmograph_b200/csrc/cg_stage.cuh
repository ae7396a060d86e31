// cg_stage.cuh -- the fused RK4 substep kernel for one periodic box (FP64).
//
// One launch performs, for every grid point, what the reference does in a
// whole substep of its sim drivers (sims/dust.cc:119-157, sims/scalar.cc:
// 275-317, components/bssn/bssn.cc:327-339):
//   sources      BSSN::clearSrc + Dust::addBSSNSrc + Lambda::addBSSNSource, or
//                Scalar::addBSSNSource (computed on chip, never stored)
//   BSSN RHS     BSSN::RKEvolve -> set_bd_values + ev_* (bssn.cc:231-831)
//   matter RHS   Dust::RKEvolve (flux divergence, dust.cc:160-224) or
//                Scalar::RKEvolvePt (scalar.cc:85-199)
//   register     RK4Register::K{n}Finalize for every field (RK4Register.h:175-222)
//   next inputs  the dust flux primitives of the substep's output, and at the
//                last substep the normalised copy of the new state that the
//                next step's first substep reads (BSSN::stepInit, bssn.cc:219-226)
//
// Register roles (each a block of nfields arrays of pts doubles):
//   in    a^n, the substep input (read with stencils)
//   prev  a^{n-1}, read at the centre point only: the reference's dust sources
//         at substep n>1 pair W, sqrt(gamma), g_ij from the previous substep's
//         populateDerivedFields with the current D, S_i (dust.cc:226-264)
//   p, f  the reference's _p and _f registers
//   out   a^{n+1} (n<4) or the new _p (n=4)
// At n=4, norm receives the next step's first-substep input.
//
// Kernel shape.  A CTA owns a 4x4x8 (x,y,z) brick, one point per thread.
// Phase 1 walks the stencil fields one at a time (a rolled loop, so the whole
// CTA touches one field's halo region at a time and it stays in L1), computes
// that field's derivatives at the thread's point and parks them in the
// thread's column of a shared-memory slot array.  Phase 2 (the algebra of
// set_bd_values and ev_*) reads the derivatives back from shared memory as it
// needs them, so few values are live in registers at once.  Bricks whose
// stencils never cross the periodic boundary use plain strided addressing;
// the others wrap every tap.
#pragma once

#include "cg_group.h"
#include "cg_point.cuh"
#include "cg_tile.cuh"
#include "cg_tma.cuh"
#include "cosmograph_b200.h"

namespace cg {

struct StagePtrs {
  const double* in;
  const double* prev;
  const double* p;
  double* f;
  double* out;
  double* norm;
  const double* fp_in;   // P_N flux-primitive arrays of a^n
  double* fp_out;        // flux primitives of the output state
  unsigned* status;      // error flags (bit 0: NaN in DIFFphi, bit 1: non-finite field)
  const double* kavg;    // device-side K_avg of a^n, or null (bssn.cc:168)
  double* cvals;         // constraint mode: per-point value and scaled value of H, M, G, A, S (10 arrays),
                         // then the Ricci scalar and DIFFr (arrays 10, 11)
  double* cpart;         // constraint mode: kCPart partial results per CTA
};

struct BoxGeom {
  int nx, ny, nz;
  int pts;
  int bx0;  // first x brick of the launch (x-slab boxes skip their ghost planes)
};

constexpr unsigned kStatusNaN = 1u;
constexpr unsigned kStatusNonFinite = 2u;
constexpr unsigned kStatusTileTimeout64 = CG_STATUS_TILE_TIMEOUT;  // a TMA tile copy was late or lost

template <int MATTER>
struct NF {
  static constexpr int value = MATTER == kDust ? 22 : (MATTER == kScalar ? 23 : (MATTER == kStaticMatter ? 19 : 18));
};

// CTA brick and field tiles (cg_tile.cuh)
using Brick = tile::Brick64;
constexpr int kBX = Brick::BX, kBY = Brick::BY, kBZ = Brick::BZ, kThreads = Brick::THREADS;
// A tile starts at an even z (z0 - ZO, ZO = r rounded up to even) and its row
// pitch is even, so that rows and TMA boxes start on 16-byte boundaries.
template <int O>
struct TileShape {
  static constexpr int R = O / 2, ZO = (R + 1) / 2 * 2, PITCH = (ZO - R + kBZ + 2 * R + 1) / 2 * 2;
};
template <int O>
using TileG = tile::Geom<O, Brick, TileShape<O>::PITCH, TileShape<O>::ZO>;

// Per-thread shared-memory slots (one column of kThreads doubles per slot).
enum : int {
  S_DG = 0,           // d_I g_q           18  (later reused for Gamma_{I q})
  S_T1 = 18,          // g^{kl} d_k d_l g_q  6
  S_DPHI = 24,        // d_I phi            3
  S_DDPHI = 27,       // d_I d_J phi        6
  S_DA = 33,          // d_I alpha          3
  S_DDA = 36,         // d_I d_J alpha      6
  S_DK = 42,          // d_I K              3
  S_DGAM = 45,        // d_J Gamma^K       9  (index 3*K + J)
  S_SRC = 54,         // sources           11
  S_G = 65,           // Gamma^I_q         18
  S_MAT = 83,         // dust: 4 divergences; scalar: 15 first derivatives
};
// Phase 1 writes no slot in [S_SRC, S_MAT): that region holds the field tile
// and its row offsets until phase 2 starts.
constexpr int kTileSlot = S_SRC, kTileSlots = S_MAT - S_SRC;
// Z4C: Z4c damping (USE_Z4c_DAMPING): the first derivatives of theta in
// three more slots after the matter slots
template <int MATTER, bool Z4C = false>
struct Slots {
  static constexpr int dth = S_MAT + (MATTER == kDust ? 4 : (MATTER == kScalar ? 15 : 0));
  static constexpr int value = dth + (Z4C ? 3 : 0);
};

// What a launch of the point kernel does with the geometry it computes.
enum Mode : int { kEvolve = 0, kConstraints = 1 };
// constraint mode: d_d A_q after the matter slots (18)
template <int MATTER, bool Z4C = false>
struct SlotsC {
  static constexpr int dA = Slots<MATTER, Z4C>::value;
  static constexpr int value = dA + 18;
};
// A second tile buffer after the slot array lets the TMA copy of the next
// field overlap the derivatives of the current one.  Evolve mode, dust and
// vacuum: two CTAs per SM still fit in shared memory (with Z4c's three more
// slots they would not: one buffer).
template <int O, int MATTER, int MODE, bool Z4C = false>
struct TileBuffers {
  static constexpr bool kTwo = MODE == kEvolve && MATTER != kScalar && !Z4C;
  // dust also stages the x and z boxes of its flux primitives here (5 arrays
  // each, flux_from_tiles)
  static constexpr size_t kTile = TileG<O>::SIZE * sizeof(double);
  static constexpr size_t kFluxX = 5 * (kBX + O) * kBY * kBZ * sizeof(double);
  static constexpr size_t kFluxZ = 5 * kBX * kBY * TileG<O>::TZ * sizeof(double);
  static constexpr size_t kNeed =
      MATTER == kDust ? (kTile > kFluxX ? (kTile > kFluxZ ? kTile : kFluxZ) : (kFluxX > kFluxZ ? kFluxX : kFluxZ))
                      : kTile;
  static constexpr size_t kBytes = (kNeed + 127) / 128 * 128;
};
// dynamic shared memory of a substep launch
template <int O, int MATTER, int MODE, bool Z4C = false>
constexpr size_t stage_smem() {
  return sizeof(double) * kThreads * (MODE == kConstraints ? SlotsC<MATTER, Z4C>::value : Slots<MATTER, Z4C>::value) +
         (TileBuffers<O, MATTER, MODE, Z4C>::kTwo ? TileBuffers<O, MATTER, MODE, Z4C>::kBytes : 0);
}
// two CTAs per SM (228 KB, 1 KB reserved per CTA, up to 1 KB of static shared memory)
static_assert(2 * (stage_smem<8, kDust, kEvolve>() + 2048) <= 228 * 1024, "two dust CTAs fit on an SM");
static_assert(2 * (stage_smem<8, kScalar, kEvolve, true>() + 2048) <= 228 * 1024, "two Z4c CTAs fit on an SM");
// per-block partial results of the constraint pass (see constraint_reduce)
constexpr int kCPart = 27;

// Register roles of substep n, the same for every box (X/Y ping-pong).
__device__ __forceinline__ StagePtrs group_ptrs(const GroupBox& b, int stage) {
  StagePtrs p{};
  p.p = b.P;
  p.f = b.F;
  p.status = b.status;
  p.kavg = b.kavg;
  switch (stage) {
    case 1: p.in = b.X; p.prev = nullptr; p.out = b.Y; p.fp_in = b.FP0; p.fp_out = b.FP1; break;
    case 2: p.in = b.Y; p.prev = b.X; p.out = b.X; p.fp_in = b.FP1; p.fp_out = b.FP0; break;
    case 3: p.in = b.X; p.prev = b.Y; p.out = b.Y; p.fp_in = b.FP0; p.fp_out = b.FP1; break;
    default: p.in = b.Y; p.prev = b.X; p.out = b.P; p.norm = b.X; p.fp_in = b.FP1; p.fp_out = b.FP0; break;
  }
  return p;
}

namespace CG_VARIANT_NS {

// Stencil taps of one point.  WRAP=false: the brick lies at least r points
// from every face, taps are plain offsets.  WRAP=true: periodic wrap.
template <bool WRAP>
struct Taps {
  int i, j, k, nx, ny, nz, sx, sy, c;
  __device__ __forceinline__ int at(int di, int dj, int dk) const {
    if (!WRAP) return c + di * sx + dj * sy + dk;
    return (wrap(i + di, nx) * ny + wrap(j + dj, ny)) * nz + wrap(k + dk, nz);
  }
  __device__ __forceinline__ int ax(int a, int n) const {
    return at(a == 0 ? n : 0, a == 1 ? n : 0, a == 2 ? n : 0);
  }
  __device__ __forceinline__ int pl(int a, int n, int b, int m) const {
    return at((a == 0 ? n : 0) + (b == 0 ? m : 0), (a == 1 ? n : 0) + (b == 1 ? m : 0),
              (a == 2 ? n : 0) + (b == 2 ? m : 0));
  }
};

// first derivative (utils/math.h:74-100, 231-263, 412-450, 554-586)
template <int O, class T>
__device__ __forceinline__ double d1(const T& t, int a, const Physics& ph) {
  auto V = [&](int n) { return t.ax(a, n); };
  double s;
  if (O == 2) {
    s = (-1.0 / 2.0 * V(-1) + 1.0 / 2.0 * V(1));
  } else if (O == 4) {
    s = (+1.0 / 12.0 * V(-2) - 2.0 / 3.0 * V(-1) + 2.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2));
  } else if (O == 6) {
    s = (-1.0 / 60.0 * V(-3) + 3.0 / 20.0 * V(-2) - 3.0 / 4.0 * V(-1) + 3.0 / 4.0 * V(1) -
         3.0 / 20.0 * V(2) + 1.0 / 60.0 * V(3));
  } else {
    s = ((1.0 / 280.0 * V(-4) - 1.0 / 280.0 * V(4)) - (4.0 / 105.0 * V(-3) - 4.0 / 105.0 * V(3)) +
         (1.0 / 5.0 * V(-2) - 1.0 / 5.0 * V(2)) - (4.0 / 5.0 * V(-1) - 4.0 / 5.0 * V(1)));
  }
  return divdx(s, ph);
}

// second derivative along one axis (utils/math.h:857-885, 958-993, 995-1036, 1038-1085)
template <int O, class T>
__device__ __forceinline__ double d2(const T& t, int a, const Physics& ph) {
  auto V = [&](int n) { return t.ax(a, n); };
  double s;
  if (O == 2) {
    s = (V(-1) - 2.0 * V(0) + V(1));
  } else if (O == 4) {
    s = (-1.0 / 12.0 * V(-2) + 4.0 / 3.0 * V(-1) - 5.0 / 2.0 * V(0) + 4.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2));
  } else if (O == 6) {
    s = (1.0 / 90.0 * V(-3) - 3.0 / 20.0 * V(-2) + 3.0 / 2.0 * V(-1) - 49.0 / 18.0 * V(0) + 3.0 / 2.0 * V(1) -
         3.0 / 20.0 * V(2) + 1.0 / 90.0 * V(3));
  } else {
    s = (-1.0 / 560.0 * V(-4) + 8.0 / 315.0 * V(-3) - 1.0 / 5.0 * V(-2) + 8.0 / 5.0 * V(-1) -
         205.0 / 72.0 * V(0) + 8.0 / 5.0 * V(1) - 1.0 / 5.0 * V(2) + 8.0 / 315.0 * V(3) - 1.0 / 560.0 * V(4));
  }
  return divdx(divdx(s, ph), ph);
}

// mixed second derivative on axes a < b (utils/math.h:676-855)
template <int O, class T>
__device__ __forceinline__ double dm(const T& t, int a, int b, const Physics& ph) {
  auto P = [&](int n) { return -t.pl(a, n, b, -n) + t.pl(a, n, b, n) + t.pl(a, -n, b, -n) - t.pl(a, -n, b, n); };
  double s;
  if (O == 2) {
    s = P(1) / 4.0;
  } else if (O == 4) {
    s = (P(1) - 1.0 / 16.0 * P(2)) / 3.0;
  } else if (O == 6) {
    s = (135.0 * P(1) - 27.0 / 2.0 * P(2) + P(3)) / 360.0;
  } else {
    s = (2.0 / 5.0 * P(1) - 1.0 / 20.0 * P(2) + 2.0 / 315.0 * P(3) - 1.0 / 2240.0 * P(4));
  }
  return divdx(divdx(s, ph), ph);
}

// taps of one stored field read from global memory through the index taps T
// (the shift's derivatives and upwinded advection)
template <class T>
struct GlobalTaps {
  const double* f;
  T t;
  __device__ __forceinline__ double ax(int a, int n) const { return __ldg(f + t.ax(a, n)); }
  __device__ __forceinline__ double pl(int a, int n, int b, int m) const { return __ldg(f + t.pl(a, n, b, m)); }
};

// upwind_derivative (utils/math.h:1247-1252): c times the lopsided derivative
// on the side c points to, lop_{forward,backward}_derivative plus the
// matching dissipation stencil (math.h:166-230, 265-339, 888-956, 1087-1131,
// 1220-1230).  The reference defines both as zero at orders 6 and 8.
template <int O, class T>
__device__ __forceinline__ double upwind(const T& t, int a, double c, const Physics& ph) {
  auto V = [&](int n) { return t.ax(a, n); };
  if constexpr (O == 2) {
    if (c > 0) {
      const double lop = divdx((-1.0 / 2.0 * V(2) + 2.0 * V(1) - 3.0 / 2.0 * V(0)), ph);
      const double dd = divdx(divdx((2.0 * V(0) - 5.0 * V(1) + 4.0 * V(2) - 1.0 * V(3)), ph), ph);
      return c * (lop + -1.0 / 2.0 * ph.dx * dd);
    }
    const double lop = divdx((+1.0 / 2.0 * V(-2) - 2.0 * V(-1) + 3.0 / 2.0 * V(0)), ph);
    const double dd = divdx(divdx((2.0 * V(0) - 5.0 * V(-1) + 4.0 * V(-2) - 1.0 * V(-3)), ph), ph);
    return c * (lop + +1.0 / 2.0 * ph.dx * dd);
  } else if constexpr (O == 4) {
    if (c > 0)
      return c * (divdx((+1.0 / 12.0 * V(3) - 1.0 / 2.0 * V(2) + 3.0 / 2.0 * V(1) - 5.0 / 6.0 * V(0) -
                         1.0 / 4.0 * V(-1)), ph) + 0.0);
    return c * (divdx((-1.0 / 12.0 * V(-3) + 1.0 / 2.0 * V(-2) - 3.0 / 2.0 * V(-1) + 5.0 / 6.0 * V(0) +
                       1.0 / 4.0 * V(1)), ph) + 0.0);
  } else {
    return c * (0.0 + 0.0);
  }
}

// derivative of the product of two stored arrays (dust fluxes (alpha*D)*v^i,
// dust.cc:121-133, and their divergence :203-224)
template <int O, class T>
__device__ __forceinline__ double d1p(const double* __restrict__ fa, const double* __restrict__ fb, const T& t,
                                      int a, const Physics& ph) {
  auto V = [&](int n) {
    const int q = t.ax(a, n);
    return __ldg(fa + q) * __ldg(fb + q);
  };
  double s;
  if (O == 2) {
    s = (-1.0 / 2.0 * V(-1) + 1.0 / 2.0 * V(1));
  } else if (O == 4) {
    s = (+1.0 / 12.0 * V(-2) - 2.0 / 3.0 * V(-1) + 2.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2));
  } else if (O == 6) {
    s = (-1.0 / 60.0 * V(-3) + 3.0 / 20.0 * V(-2) - 3.0 / 4.0 * V(-1) + 3.0 / 4.0 * V(1) -
         3.0 / 20.0 * V(2) + 1.0 / 60.0 * V(3));
  } else {
    s = ((1.0 / 280.0 * V(-4) - 1.0 / 280.0 * V(4)) - (4.0 / 105.0 * V(-3) - 4.0 / 105.0 * V(3)) +
         (1.0 / 5.0 * V(-2) - 1.0 / 5.0 * V(2)) - (4.0 / 5.0 * V(-1) - 4.0 / 5.0 * V(1)));
  }
  return divdx(s, ph);
}

// Fields copied into tiles in phase 1, in order: (constraint mode) A_q with
// first derivatives; the metric components, phi and alpha with first and
// second derivatives; K and Gamma^i with first derivatives; (scalar) phi, Pi,
// psi_i with first derivatives.  With Z4c, theta (stored after the matter
// fields) with first derivatives after Gamma^i.
template <int MATTER, int MODE, bool Z4C = false>
struct Phase1 {
  static constexpr int NA = MODE == kConstraints ? 6 : 0;
  static constexpr int NZ = Z4C ? 1 : 0;
  static constexpr int NS = MATTER == kScalar ? 5 : 0;
  static constexpr int N = NA + 8 + 4 + NZ + NS;
  __device__ __forceinline__ static int field(int it) {
    if (it < NA) return F_A11 + it;
    it -= NA;
    if (it < 8) return it < 6 ? F_G11 + it : (it == 6 ? F_PHI : F_ALPHA);
    it -= 8;
    if (it < 4) return it == 0 ? F_K : F_GAM1 + it - 1;
    it -= 4;
    if (it < NZ) return NF<MATTER>::value;  // theta
    it -= NZ;
    return F_SPHI + it;
  }
};

// Phase 1: every derivative the point needs, parked in shared memory.  One
// field at a time is copied into the tile (the next one is fetched into
// registers, or into L2 on the TMA path, meanwhile); all threads of the CTA
// take part.
//
// The copies: by TMA when tmap is set (a brick whose halo lies inside the
// box), else by the threads' own loads with periodic wrap.  Returns false (the
// same value in every thread) when a TMA copy did not complete within
// ph.tma_wait cycles; the status word then carries kStatusTileTimeout64.  A
// late copy is still waited for (tma::wait_drain), so that no copy is in
// flight when a buffer is reused or the CTA leaves; after a copy that never
// lands the CTA issues no more.
template <int O, int MATTER, int MODE, bool Z4C>
__device__ __forceinline__ void field_derivatives(int it, const tile::Taps<TileG<O>, double>& t, const Physics& ph,
                                                  const double gi[6], double* sl);

//
// bar[0] (and bar[1] with two buffers) are the buffers' mbarriers; bit b of
// phase is the parity bar[b] completes next.
template <int O, int MATTER, int MODE, bool Z4C = false>
__device__ __forceinline__ bool derivatives(const double* __restrict__ a, int N, const Physics& ph, const double gi[6],
                                            double* sl, double* tl, double* tl2, const int* rowoff, int tid, int x0,
                                            int y0, int z0, int nz, int cc, const CUtensorMap* tmap, uint64_t* bar,
                                            unsigned& phase, unsigned* status) {
  using PF = Phase1<MATTER, MODE, Z4C>;
  using G = TileG<O>;
  constexpr bool TWO = TileBuffers<O, MATTER, MODE, Z4C>::kTwo;
  constexpr unsigned kBytes = (unsigned)(G::SIZE * sizeof(double));
  // TMA: field it into buffer it % 2 (one buffer: 0), field it + 1 into L2;
  // thread 0 copies, every thread notes the buffer's copy as pending
  unsigned pending = 0;
  auto issue = [&](int it) {
    const int b = TWO ? (it & 1) : 0;
    if (tid == 0) {
      tma::arrive_expect_tx(bar + b, kBytes);
      tma::load_4d(b ? tl2 : tl, tmap, z0 - G::ZO, y0 - G::R, x0 - G::R, PF::field(it), bar + b);
      if (it + 1 < PF::N) tma::prefetch_4d(tmap, z0 - G::ZO, y0 - G::R, x0 - G::R, PF::field(it + 1));
    }
    pending |= 1u << b;
  };
  // ok: every copy landed within ph.tma_wait cycles; lost: one never landed
  // (the CTA then issues no more copies, waits for the ones in flight and
  // returns with the status flagged)
  bool ok = true, lost = false;
  auto wait = [&](int b) {
    if (!(pending & (1u << b))) return;
    const int w = tma::wait_drain(bar + b, (phase >> b) & 1u, ph.tma_wait);
    ok = ok && w == 0;
    pending &= ~(1u << b);
    if (w == 2) lost = true;
    else phase ^= 1u << b;
  };
  const bool by_tma = tmap != nullptr;
  tile::Loader<G, Brick, double> ld;
  tile::AsyncLoader<G, Brick> ald;
  if (by_tma) {
    if (TWO) {
      tma::fence_proxy_async();  // this thread's shared-memory accesses come before the copy's writes
      __syncthreads();
      issue(0);
    }
  } else if (TWO) {
    // two buffers: cp.async copies of field it + 1 run while field it is differentiated
    ald.init(tid, z0, nz);
    ald.issue(tl, a + (size_t)PF::field(0) * N, rowoff);
  } else {
    ld.init(tid, z0, nz);
    ld.fetch(a + (size_t)PF::field(0) * N, rowoff);
  }
  // one loop (and one copy of the derivative code) for both kinds of copy
#pragma unroll 1
  for (int it = 0; it < PF::N; ++it) {
    int b = 0;
    if (by_tma) {
      tma::fence_proxy_async();
      lost = __syncthreads_or(lost);  // the buffer the next copy writes has been read
      if (!lost) {
        if (!TWO) issue(it);
        else if (it + 1 < PF::N) issue(it + 1);
      }
      b = TWO ? (it & 1) : 0;
      wait(b);
    } else if (TWO) {
      __syncthreads();  // the buffer the next copies write has been read
      if (it + 1 < PF::N) {
        ald.issue((it + 1) & 1 ? tl2 : tl, a + (size_t)PF::field(it + 1) * N, rowoff);
        tile::cp_async_wait<1>();  // this thread's copies of field it have landed
      } else {
        tile::cp_async_wait<0>();
      }
      __syncthreads();  // and every other thread's
      b = it & 1;
    } else {
      __syncthreads();  // the previous tile has been read
      ld.store(tl);
      __syncthreads();
      if (it + 1 < PF::N) ld.fetch(a + (size_t)PF::field(it + 1) * N, rowoff);
    }
    field_derivatives<O, MATTER, MODE, Z4C>(it, tile::Taps<G, double>{b ? tl2 : tl, cc}, ph, gi, sl);
  }
  if (by_tma) {
    wait(0);  // after a lost copy: the other buffer's copy in flight
    wait(1);
    ok = __syncthreads_and(ok && !lost);
    if (!ok && tid == 0) atomicOr(status, kStatusTileTimeout64);
  }
  return ok;
}

// the derivatives of phase-1 field `it` from its tile, into the slots
template <int O, int MATTER, int MODE, bool Z4C>
__device__ __forceinline__ void field_derivatives(int it, const tile::Taps<TileG<O>, double>& t, const Physics& ph,
                                                  const double gi[6], double* sl) {
  using PF = Phase1<MATTER, MODE, Z4C>;
  {
    if (it < PF::NA) {
      // d_d A_q for the momentum constraint (BSSN_MI, bssn_macros.h:498-500)
      const int q = it;
      sl[(SlotsC<MATTER, Z4C>::dA + 3 * q + 0) * kThreads] = d1<O>(t, 0, ph);
      sl[(SlotsC<MATTER, Z4C>::dA + 3 * q + 1) * kThreads] = d1<O>(t, 1, ph);
      sl[(SlotsC<MATTER, Z4C>::dA + 3 * q + 2) * kThreads] = d1<O>(t, 2, ph);
    } else if (it < PF::NA + 8) {
      // calculate_dgamma / calculate_ddgamma / calculate_dalpha_dphi
      // (bssn.cc:480-521).  For g_q the second derivatives are contracted at
      // once with the inverse metric (BSSN_CALCULATE_RICCI_UNITARY_TERM1,
      // bssn_macros.h:248-249, summed over (k,l) in the reference's order).
      const int q = it - PF::NA;
      const double g1 = d1<O>(t, 0, ph), g2 = d1<O>(t, 1, ph), g3 = d1<O>(t, 2, ph);
      const double h11 = d2<O>(t, 0, ph), h22 = d2<O>(t, 1, ph), h33 = d2<O>(t, 2, ph);
      const double h12 = dm<O>(t, 0, 1, ph), h13 = dm<O>(t, 0, 2, ph), h23 = dm<O>(t, 1, 2, ph);
      if (q < 6) {
        sl[(S_DG + 0 * 6 + q) * kThreads] = g1;
        sl[(S_DG + 1 * 6 + q) * kThreads] = g2;
        sl[(S_DG + 2 * 6 + q) * kThreads] = g3;
        double s = gi[0] * h11;
        s = s + gi[1] * h12;
        s = s + gi[2] * h13;
        s = s + gi[1] * h12;
        s = s + gi[3] * h22;
        s = s + gi[4] * h23;
        s = s + gi[2] * h13;
        s = s + gi[4] * h23;
        s = s + gi[5] * h33;
        sl[(S_T1 + q) * kThreads] = s;
      } else {
        const int b1 = q == 6 ? S_DPHI : S_DA, b2 = q == 6 ? S_DDPHI : S_DDA;
        sl[(b1 + 0) * kThreads] = g1;
        sl[(b1 + 1) * kThreads] = g2;
        sl[(b1 + 2) * kThreads] = g3;
        sl[(b2 + 0) * kThreads] = h11;
        sl[(b2 + 1) * kThreads] = h12;
        sl[(b2 + 2) * kThreads] = h13;
        sl[(b2 + 3) * kThreads] = h22;
        sl[(b2 + 4) * kThreads] = h23;
        sl[(b2 + 5) * kThreads] = h33;
      }
    } else if (it < PF::NA + 12) {
      // K and Gamma^K: first derivatives (calculate_dK, bssn.cc:529-535; the
      // d_J Gamma^K of BSSN_CALCULATE_RICCI_UNITARY_TERM2, bssn_macros.h:251-252)
      const int q = it - PF::NA - 8;
      const int b = q == 0 ? S_DK : S_DGAM + 3 * (q - 1);
      sl[(b + 0) * kThreads] = d1<O>(t, 0, ph);
      sl[(b + 1) * kThreads] = d1<O>(t, 1, ph);
      sl[(b + 2) * kThreads] = d1<O>(t, 2, ph);
    } else if (Z4C && it == PF::NA + 12) {
      // calculate_dtheta (bssn.cc:537-544)
      constexpr int b = Slots<MATTER, Z4C>::dth;
      sl[(b + 0) * kThreads] = d1<O>(t, 0, ph);
      sl[(b + 1) * kThreads] = d1<O>(t, 1, ph);
      sl[(b + 2) * kThreads] = d1<O>(t, 2, ph);
    } else {
      // Scalar::getScalarData derivatives (scalar.cc:109-127): d_d of phi, Pi, psi1..3
      const int m = it - PF::NA - 12 - PF::NZ;
      sl[(S_MAT + 3 * m + 0) * kThreads] = d1<O>(t, 0, ph);
      sl[(S_MAT + 3 * m + 1) * kThreads] = d1<O>(t, 1, ph);
      sl[(S_MAT + 3 * m + 2) * kThreads] = d1<O>(t, 2, ph);
    }
  }
}

// Dust flux divergences d_i(alpha D v^i), d_i(alpha S_m v^i) (dust.cc:203-224)
// from the stored flux primitives, taps read from global memory.
template <int O, class T>
__device__ __forceinline__ void flux_divergences(const T& t, const double* __restrict__ fp, int N, const Physics& ph,
                                                 double* sl, int m0 = 0, int m1 = 4) {
  const double* v1 = fp + (size_t)P_V1 * N;
  const double* v2 = fp + (size_t)P_V2 * N;
  const double* v3 = fp + (size_t)P_V3 * N;
#pragma unroll 1
  for (int m = m0; m < m1; ++m) {
    const double* u = fp + (size_t)(P_AD + m) * N;
    sl[(S_MAT + m) * kThreads] = d1p<O>(u, v1, t, 0, ph) + d1p<O>(u, v2, t, 1, ph) + d1p<O>(u, v3, t, 2, ph);
  }
}

// TMA boxes of the dust flux primitives for their divergence: for axis a the
// brick extended by r along a only (x: (4+2r) x 2 x 16, y: 4 x (2+2r) x 16,
// z: 4 x 2 x the tile row of the field tiles, starting at an aligned z).
template <int O>
struct FluxBox {
  static constexpr int R = O / 2;
  static constexpr int XB = (kBX + 2 * R) * kBY * kBZ;
  static constexpr int YB = kBX * (kBY + 2 * R) * kBZ;
  static constexpr int ZP = TileG<O>::TZ, ZB = kBX * kBY * ZP;
};
struct FluxMaps {
  CUtensorMap m[3];  // x, y and z boxes of the substep input's 7 flux-primitive arrays
};

// divergence term along one axis from box tiles: u (4 arrays, the m-th at
// u + m*len) and v^a (at u + 4*len); the product at each tap as d1p forms it
template <int O>
__device__ __forceinline__ double d1p_tile(const double* u, const double* v, int c, int s, const Physics& ph) {
  auto V = [&](int n) { return u[c + n * s] * v[c + n * s]; };
  double r;
  if (O == 2) {
    r = (-1.0 / 2.0 * V(-1) + 1.0 / 2.0 * V(1));
  } else if (O == 4) {
    r = (+1.0 / 12.0 * V(-2) - 2.0 / 3.0 * V(-1) + 2.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2));
  } else if (O == 6) {
    r = (-1.0 / 60.0 * V(-3) + 3.0 / 20.0 * V(-2) - 3.0 / 4.0 * V(-1) + 3.0 / 4.0 * V(1) -
         3.0 / 20.0 * V(2) + 1.0 / 60.0 * V(3));
  } else {
    r = ((1.0 / 280.0 * V(-4) - 1.0 / 280.0 * V(4)) - (4.0 / 105.0 * V(-3) - 4.0 / 105.0 * V(3)) +
         (1.0 / 5.0 * V(-2) - 1.0 / 5.0 * V(2)) - (4.0 / 5.0 * V(-1) - 4.0 / 5.0 * V(1)));
  }
  return divdx(r, ph);
}

// Dust flux divergences of a brick inside the box from TMA boxes: x boxes
// into tl2, y boxes into tl, then z boxes into tl2; the sum over axes in the
// order of flux_divergences.  All threads of the CTA take part.
// (tx, ty, tz): the thread's point in the brick; it computes the divergences
// m0 <= m < m1 (alpha*D, alpha*S_1..3)
template <int O>
__device__ __forceinline__ bool flux_from_tiles(const FluxMaps* fm, double* tl, double* tl2, int tid, int x0, int y0,
                                                int z0, const Physics& ph, double* sl, uint64_t* bar,
                                                unsigned& phase, int tx, int ty, int tz, int m0 = 0, int m1 = 4) {
  using FB = FluxBox<O>;
  constexpr int R = FB::R;
  // every staging area fits its buffer: x and z boxes in the second tile
  // buffer, y boxes in the first (the phase-2-only slot columns)
  static_assert(5 * FB::XB * sizeof(double) <= TileBuffers<O, kDust, kEvolve>::kBytes, "x boxes fit");
  static_assert(5 * FB::ZB * sizeof(double) <= TileBuffers<O, kDust, kEvolve>::kBytes, "z boxes fit");
  static_assert(5 * FB::YB * sizeof(double) <= (size_t)kTileSlots * kThreads * sizeof(double), "y boxes fit");
  // as in derivatives: bounded waits that let late copies land; after a lost
  // copy no more copies, the ones in flight waited for
  bool ok = true, lost = false;
  unsigned pending = 0;
  auto wait = [&](int b) {
    if (!(pending & (1u << b))) return;
    const int w = tma::wait_drain(bar + b, (phase >> b) & 1u, ph.tma_wait);
    ok = ok && w == 0;
    pending &= ~(1u << b);
    if (w == 2) lost = true;
    else phase ^= 1u << b;
  };
  auto load5 = [&](int a, double* dst, uint64_t* b, int len) {
    tma::arrive_expect_tx(b, (unsigned)(5 * len * sizeof(double)));
    const int cx = x0 - (a == 0 ? R : 0), cy = y0 - (a == 1 ? R : 0);
    const int cz = z0 - (a == 2 ? TileG<O>::ZO : 0);
    for (int q = 0; q < 5; ++q)  // alpha*D, alpha*S_1..3, then v^a
      tma::load_4d(dst + (size_t)q * len, &fm->m[a], cz, cy, cx, q < 4 ? P_AD + q : P_V1 + a, b);
  };
  tma::fence_proxy_async();
  __syncthreads();  // the field tiles have been read
  if (tid == 0) {
    load5(0, tl2, bar + 1, FB::XB);
    load5(1, tl, bar, FB::YB);
  }
  pending = 3u;
  wait(1);
  {
    const int c = ((tx + R) * kBY + ty) * kBZ + tz;
#pragma unroll 1
    for (int m = m0; m < m1; ++m)
      sl[(S_MAT + m) * kThreads] = d1p_tile<O>(tl2 + (size_t)m * FB::XB, tl2 + (size_t)4 * FB::XB, c, kBY * kBZ, ph);
  }
  tma::fence_proxy_async();
  lost = __syncthreads_or(lost);  // the x boxes have been read
  if (!lost) {
    if (tid == 0) load5(2, tl2, bar + 1, FB::ZB);
    pending |= 2u;
  }
  wait(0);
  {
    const int c = (tx * (kBY + 2 * R) + ty + R) * kBZ + tz;
#pragma unroll 1
    for (int m = m0; m < m1; ++m)
      sl[(S_MAT + m) * kThreads] =
          sl[(S_MAT + m) * kThreads] + d1p_tile<O>(tl + (size_t)m * FB::YB, tl + (size_t)4 * FB::YB, c, kBZ, ph);
  }
  wait(1);
  {
    const int c = (tx * kBY + ty) * FB::ZP + tz + TileG<O>::ZO;
#pragma unroll 1
    for (int m = m0; m < m1; ++m)
      sl[(S_MAT + m) * kThreads] =
          sl[(S_MAT + m) * kThreads] + d1p_tile<O>(tl2 + (size_t)m * FB::ZB, tl2 + (size_t)4 * FB::ZB, c, 1, ph);
  }
  return __syncthreads_and(ok && !lost);
}

// Kreiss-Oliger dissipation of one field at (i, j, k) (utils/math.h:36-72;
// the reference defines it for stencil orders 2 and 8 only): the sixth
// (order 2: fourth) undivided difference along each axis, taps from global
// memory, plain offsets when the taps stay inside the box.
template <int O>
__device__ __forceinline__ double ko_dissipation(const double* __restrict__ f, int i, int j, int k, int nx, int ny, int nz,
                                              bool inside, const Physics& ph) {
  const double c = ph.ko_coeff;
  auto at = [&](int a, int n) {
    int ii = i + (a == 0 ? n : 0), jj = j + (a == 1 ? n : 0), kk = k + (a == 2 ? n : 0);
    if (!inside) {
      ii = wrap(ii, nx);
      jj = wrap(jj, ny);
      kk = wrap(kk, nz);
    }
    return __ldg(f + ((size_t)ii * ny + jj) * nz + kk);
  };
  auto X = [&](int n) { return at(0, n); };
  auto Y = [&](int n) { return at(1, n); };
  auto Z = [&](int n) { return at(2, n); };
  if (O == 2) {
    const double st = (1.0 * X(-2) + 1.0 * Y(-2) + 1.0 * Z(-2) - 4.0 * X(-1) - 4.0 * Y(-1) - 4.0 * Z(-1) +
                       6.0 * X(0) + 6.0 * Y(0) + 6.0 * Z(0) - 4.0 * X(1) - 4.0 * Y(1) - 4.0 * Z(1) + 1.0 * X(2) +
                       1.0 * Y(2) + 1.0 * Z(2)) /
                      ph.ko_pden;
    return c * ph.ko_pnum / 64.0 * st;
  }
  const double st = (1.0 * X(-5) + 1.0 * Y(-5) + 1.0 * Z(-5) - 10.0 * X(-4) - 10.0 * Y(-4) - 10.0 * Z(-4) +
                     45.0 * X(-3) + 45.0 * Y(-3) + 45.0 * Z(-3) - 120.0 * X(-2) - 120.0 * Y(-2) - 120.0 * Z(-2) +
                     210.0 * X(-1) + 210.0 * Y(-1) + 210.0 * Z(-1) - 252.0 * X(0) - 252.0 * Y(0) - 252.0 * Z(0) +
                     210.0 * X(1) + 210.0 * Y(1) + 210.0 * Z(1) - 120.0 * X(2) - 120.0 * Y(2) - 120.0 * Z(2) +
                     45.0 * X(3) + 45.0 * Y(3) + 45.0 * Z(3) - 10.0 * X(4) - 10.0 * Y(4) - 10.0 * Z(4) +
                     1.0 * X(5) + 1.0 * Y(5) + 1.0 * Z(5)) /
                    ph.ko_pden;
  return -c * ph.ko_pnum / 1024.0 * st;
}

// Deterministic CTA reduction of Q values per thread: the first NSUM are
// summed, the rest maximised; warp shuffles, then the warps in order.  Thread
// 0 writes the Q results of this CTA to part[cta * Q].
template <int Q, int NSUM>
__device__ __forceinline__ void cta_reduce(double (&q)[Q], double* part, int cta) {
  __shared__ double red[kThreads / 32][Q];
  const int tid = threadIdx.x + kBZ * (threadIdx.y + kBY * threadIdx.z);
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int m = 0; m < Q; ++m) {
    double x = q[m];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = m < NSUM ? x + y : fmax(x, y);
    }
    if (lane == 0) red[warp][m] = x;
  }
  __syncthreads();
  if (tid == 0) {
#pragma unroll 1
    for (int m = 0; m < Q; ++m) {
      double x = red[0][m];
      for (int w = 1; w < kThreads / 32; ++w) x = m < NSUM ? x + red[w][m] : fmax(x, red[w][m]);
      part[(size_t)cta * Q + m] = x;
    }
  }
}

// The fused substep for the brick at brick coordinates (cx, cy, cz) of one
// box; cta numbers the CTA's partial results in constraint mode.  KO: the
// Kreiss-Oliger terms are compiled in (a separate instantiation, so that the
// common case carries none of their code).  Z4C: Z4c damping (the field theta
// after the matter fields, bssn.cc:834-848 and the theta terms of ev_*; the
// reference's USE_Z4c_DAMPING), also a separate instantiation.
template <int O, int MATTER, int MODE, bool KO = false, bool Z4C = false, bool SHIFT = false>
__device__ __forceinline__ void stage_body(const BoxGeom& geo, const Physics& ph, StageBg bg, const StagePtrs& P,
                                           int stage, int cx, int cy, int cz, int cta, const CUtensorMap* tmap,
                                           uint64_t* bar, unsigned& phase, bool& tma_ok,
                                           const FluxMaps* fmaps = nullptr) {
  constexpr int F_THETA = NF<MATTER>::value;
  // the shift fields beta1..3, auxB1..3, expN follow the matter fields (and theta)
  constexpr int F_BETA = NF<MATTER>::value + (Z4C ? 1 : 0), F_AUXB = F_BETA + 3, F_EXPN = F_BETA + 6;
  constexpr int NFLD = NF<MATTER>::value + (Z4C ? 1 : 0) + (SHIFT ? 7 : 0);
  static_assert(!SHIFT || MODE == kEvolve, "constraint statistics do not read the shift");
  constexpr int NSLOT = MODE == kConstraints ? SlotsC<MATTER, Z4C>::value : Slots<MATTER, Z4C>::value;
  // Z4c damping amplitudes (cosmo_macros.h:94-100)
  constexpr double k1 = Z4C ? 0.5 : 0.0, k2 = Z4C ? 0.1 : 0.0;
  static_assert(NSLOT >= S_MAT, "the tile region lies inside the slot array");
  static_assert(TileG<O>::SIZE * sizeof(double) + TileG<O>::ROWS * sizeof(int) <=
                    (size_t)kTileSlots * kThreads * sizeof(double),
                "tile and row offsets fit the phase-2-only slots");
  constexpr int R = O / 2;
  extern __shared__ __align__(128) double smem[];  // 128-byte aligned: TMA destinations
  const int tid = threadIdx.x + kBZ * (threadIdx.y + kBY * threadIdx.z);
  double* sl = smem + tid;  // this thread's slot column
  auto S = [&](int s) -> double& { return sl[s * kThreads]; };

  const int k0 = cz * kBZ + threadIdx.x;
  const int j0 = cy * kBY + threadIdx.y;
  const int i0 = cx * kBX + threadIdx.z;
  const bool live = i0 < geo.nx && j0 < geo.ny && k0 < geo.nz;
  // every thread takes part in the tile copies of phase 1 (and, in constraint
  // mode, in the CTA reduction); threads past the box edge compute a valid
  // point and write nothing
  const int k = min(k0, geo.nz - 1), j = min(j0, geo.ny - 1), i = min(i0, geo.nx - 1);
  if (P.kavg) bg.K_avg = *P.kavg;
  const int N = geo.pts;
  const int c = (i * geo.ny + j) * geo.nz + k;
  const double* __restrict__ a = P.in;
  auto C = [&](int f) { return a[(size_t)f * N + c]; };
  // The epilogue's register reads (_p, _f) are issued long after this point;
  // warm L2 with them now.  Those reads and every epilogue write are
  // single-use streams (ld/st .cs, evict first), which leaves L2 to the
  // neighbouring bricks' tile rows.
  if (MODE == kEvolve) {
#pragma unroll 1
    for (int f = 0; f < NFLD; ++f) {
      asm volatile("prefetch.global.L2 [%0];" :: "l"(P.p + (size_t)f * N + c));
      if (stage > 1) asm volatile("prefetch.global.L2 [%0];" :: "l"(P.f + (size_t)f * N + c));
    }
  }

  // ---- centre values (set_local_vals, bssn.cc:430-435) ----------------------
  double g[6], gi[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) g[q] = C(F_G11 + q);
  inv_metric(g, gi);

  // ---- phase 1: derivatives into shared memory ---------------------------------
  const int x0 = cx * kBX, y0 = cy * kBY, z0 = cz * kBZ;
  bool flux_tiles = false;  // the dust flux divergences came from TMA boxes
  {
    using G = TileG<O>;
    double* tl = smem + kTileSlot * kThreads;
    int* rowoff = reinterpret_cast<int*>(tl + G::SIZE);
    // TMA when the brick's halo lies inside the box (no wrap)
    const bool by_tma = tmap && tma_ok && x0 >= G::R && x0 + kBX + G::R <= geo.nx && y0 >= G::R &&
                        y0 + kBY + G::R <= geo.ny && z0 >= G::ZO && z0 + kBZ + G::R <= geo.nz;
    if (!by_tma) {
      tile::row_offsets<G, Brick>(x0, y0, geo.nx, geo.ny, geo.nz, tid, rowoff);
      __syncthreads();  // every warp reads every row offset
    }
    // after a copy timed out the CTA copies by threads (the barrier's phase is unknown)
    double* tl2 = TileBuffers<O, MATTER, MODE, Z4C>::kTwo ? smem + NSLOT * kThreads : nullptr;
    tma_ok = derivatives<O, MATTER, MODE, Z4C>(a, N, ph, gi, sl, tl, tl2, rowoff, tid, x0, y0, z0, geo.nz,
                                          tile::centre<G>(threadIdx.z, threadIdx.y, threadIdx.x),
                                          by_tma ? tmap : nullptr, bar, phase, P.status) &&
             tma_ok;
    if constexpr (MATTER == kDust && MODE == kEvolve && TileBuffers<O, MATTER, MODE, Z4C>::kTwo) {
      flux_tiles = fmaps && by_tma && tma_ok;
      if (flux_tiles) {
        tma_ok = flux_from_tiles<O>(fmaps, tl, tl2, tid, x0, y0, z0, ph, sl, bar, phase, threadIdx.z, threadIdx.y,
                                    threadIdx.x);
        if (!tma_ok && tid == 0) atomicOr(P.status, kStatusTileTimeout64);
      }
    }
    __syncthreads();  // the tile region becomes slots again
  }
  if (MODE == kEvolve && !live) return;  // no CTA-wide synchronisation after this point
  if (!flux_tiles) {
    const bool interior = x0 >= R && x0 + kBX + R <= geo.nx && y0 >= R && y0 + kBY + R <= geo.ny && z0 >= R &&
                          z0 + kBZ + R <= geo.nz;
    // the dust flux divergences of bricks that did not take them from TMA
    // boxes: taps from global memory
    if (MATTER == kDust) {
      if (interior) flux_divergences<O>(Taps<false>{i, j, k, geo.nx, geo.ny, geo.nz, geo.ny * geo.nz, geo.nz, c},
                                        P.fp_in, N, ph, sl);
      else flux_divergences<O>(Taps<true>{i, j, k, geo.nx, geo.ny, geo.nz, geo.ny * geo.nz, geo.nz, c}, P.fp_in, N,
                               ph, sl);
    }
  }

  // ---- phase 2: the algebra of set_bd_values (bssn.cc:361-421) ----------------
  const double phi = C(F_PHI) + bg.phi_FRW;
  const double Kd = C(F_K);
  const double K = Kd + bg.K_FRW;
  const double alphad = C(F_ALPHA);
  const double alpha = alphad + 1.0;
  // Z4c's theta and its derivatives (0 without Z4c, as the reference's
  // zero-initialised BSSNData leaves them)
  const double theta = Z4C ? C(F_THETA) : 0.0;
  double dth[3] = {0.0, 0.0, 0.0};
  if constexpr (Z4C) {
#pragma unroll
    for (int d = 0; d < 3; ++d) dth[d] = S(Slots<MATTER, Z4C>::dth + d);
  }
  double gm[6];
  gm[0] = g[0] + 1.0; gm[1] = g[1]; gm[2] = g[2];
  gm[3] = g[3] + 1.0; gm[4] = g[4]; gm[5] = g[5] + 1.0;
  // the shift (set_local_vals and calculate_dbeta, bssn.cc:430-435, 548-559):
  // beta^i and db[j][i] = d_j beta^i, centred stencils on global taps (0
  // without the shift, as the reference's zero-initialised BSSNData leaves
  // them); up(f, j) = upwind_derivative of field f along axis j with beta^j
  double beta[3] = {0.0, 0.0, 0.0};
  double db[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  const Taps<true> tg{i, j, k, geo.nx, geo.ny, geo.nz, geo.ny * geo.nz, geo.nz, c};
  auto gtap = [&](int fld) { return GlobalTaps<Taps<true>>{a + (size_t)fld * N, tg}; };
  auto up = [&](int fld, int d) { return upwind<O>(gtap(fld), d, beta[d], ph); };
  // second derivative d_x d_y of field fld (double_derivative, utils/math.h:1319-1336)
  auto ddf = [&](int x, int y, int fld) {
    return x == y ? d2<O>(gtap(fld), x, ph) : dm<O>(gtap(fld), x < y ? x : y, x < y ? y : x, ph);
  };
  if constexpr (SHIFT) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      beta[q] = C(F_BETA + q);
#pragma unroll
      for (int d = 0; d < 3; ++d) db[d][q] = d1<O>(gtap(F_BETA + q), d, ph);
    }
  }
  const double divb = (db[0][0] + db[1][1]) + db[2][2];
  // every e^x this point's substep takes, in one batch: of phi and, for dust
  // after the first substep, of the previous substep's phi (the lagged
  // sources); static matter takes e^{-6 phi} in the sixth place
  double phip = phi;
  if (MATTER == kDust && stage > 1) phip = __ldcs(&P.prev[(size_t)F_PHI * N + c]) + bg.phi_FRW_prev;
  // (without dust the previous substep's phi is not needed: five values, six
  // with static matter)
  // The parity build evaluates the batch through this thread's slots of the
  // Christoffel symbols (free until they are formed): arguments in S_G,
  // results in S_G + NX, the fast evaluation in a rolled loop (one copy of its
  // code, which stays in the instruction cache), the accurate phase for the
  // undecided ones after it; the same correctly rounded values as xexp_n.
  constexpr int NX = MATTER == kDust ? 8 : (MATTER == kStaticMatter ? 6 : 5);
  static_assert(2 * NX <= 18, "the batch fits the Christoffel slots");
  double ex[8];
  {
    double xa[NX];
#pragma unroll
    for (int q = 0; q < NX; ++q)
      xa[q] = q < 5 ? (q == 0 ? -4.0 : q == 1 ? 4.0 : q == 2 ? 6.0 : q == 3 ? 5.0 : -5.0) * phi
                    : (MATTER == kStaticMatter ? -6.0 * phi : (q == 5 ? -4.0 : q == 6 ? 4.0 : 6.0) * phip);
    if constexpr (kReferenceOrder) {
#pragma unroll
      for (int q = 0; q < NX; ++q) S(S_G + q) = xa[q];
      unsigned bad = 0;
#pragma unroll 1
      for (int q = 0; q < NX; ++q) {
        double y;
        if (!crm::exp_fast(S(S_G + q), y)) bad |= 1u << q;
        S(S_G + NX + q) = y;
      }
#pragma unroll 1
      while (bad) {
        const int q = __ffs(bad) - 1;
        bad &= bad - 1;
        S(S_G + NX + q) = crm::exp_full(S(S_G + q));
      }
#pragma unroll
      for (int q = 0; q < NX; ++q) ex[q] = S(S_G + NX + q);
    } else {
      double ey[NX];
      xexp_n<NX>(xa, ey);
#pragma unroll
      for (int q = 0; q < NX; ++q) ex[q] = ey[q];
    }
  }
  if constexpr (NX < 8) {  // without dust the previous substep's phi is this one's
    if constexpr (NX == 5) ex[5] = ex[0];
    ex[6] = ex[1];
    ex[7] = ex[2];
  }
  const double em4phi = ex[0], e4phi = ex[1], e6phi = ex[2], e5phi = ex[3], em5phi = ex[4];
  const double em4phip = ex[5], e4phip = ex[6], e6phip = ex[7];

  // -- sources and matter centre quantities --
  double rhs_m[5] = {0, 0, 0, 0, 0};
  if (MATTER == kDust) {
    const double D = C(F_D);
    const double Sv[3] = {C(F_S1), C(F_S2), C(F_S3)};
    double Wl, detgl, gph[6];
    if (stage == 1) {
      // the stepInit populate used this same state (sims/dust.cc:56-62)
      const DustPrim dp = dust_prim(gi, em4phi, e6phi, D, Sv);
      Wl = dp.W;
      const double e4 = e4phi;
      detgl = e6phi;
#pragma unroll
      for (int m = 0; m < 6; ++m) gph[m] = e4 * gm[m];
    } else {
      const double* pv = P.prev;
      double gp[6], gip[6];
#pragma unroll
      for (int m = 0; m < 6; ++m) gp[m] = __ldcs(&pv[(size_t)(F_G11 + m) * N + c]);
      const double Dp = __ldcs(&pv[(size_t)F_D * N + c]);
      const double Sp[3] = {__ldcs(&pv[(size_t)F_S1 * N + c]), __ldcs(&pv[(size_t)F_S2 * N + c]), __ldcs(&pv[(size_t)F_S3 * N + c])};
      inv_metric(gp, gip);
      const DustPrim dp = dust_prim(gip, em4phip, e6phip, Dp, Sp);
      Wl = dp.W;
      const double e4 = e4phip;
      detgl = e6phip;
      gph[0] = e4 * (gp[0] + 1.0); gph[1] = e4 * gp[1]; gph[2] = e4 * gp[2];
      gph[3] = e4 * (gp[3] + 1.0); gph[4] = e4 * gp[4]; gph[5] = e4 * (gp[5] + 1.0);
    }
    double q[Q_N];
    dust_sources(Wl, detgl, gph, D, Sv, ph.lambda, q);
#pragma unroll
    for (int m = 0; m < Q_N; ++m) S(S_SRC + m) = q[m];
    // momentum source S_m^src (dust.cc:135-146) with the current W, v
    const DustPrim cur = dust_prim(gi, em4phi, e6phi, D, Sv);
    const double e4 = e4phi;
    rhs_m[0] = S(S_MAT + 0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double dp = S(S_DPHI + d);
      auto DG = [&](int qq) { return S(S_DG + 6 * d + qq); };
      const double src =
          1.0 / 2.0 * alpha * cur.W * D * e4 *
              (cur.v[0] * cur.v[0] * (4.0 * gm[0] * dp + DG(0)) + cur.v[1] * cur.v[1] * (4.0 * gm[3] * dp + DG(3)) +
               cur.v[2] * cur.v[2] * (4.0 * gm[5] * dp + DG(5)) +
               2.0 * (cur.v[0] * cur.v[1] * (4.0 * gm[1] * dp + DG(1)) + cur.v[0] * cur.v[2] * (4.0 * gm[2] * dp + DG(2)) +
                      cur.v[1] * cur.v[2] * (4.0 * gm[4] * dp + DG(4)))) -
          cur.W * D * S(S_DA + d);
      rhs_m[1 + d] = S(S_MAT + 1 + d) + src;
    }
  } else if (MATTER == kScalar) {
    // Scalar::addBSSNSource (scalar.cc:201-260) and RKEvolvePt (:85-199)
    const double sphi = C(F_SPHI), sPi = C(F_SPI);
    const double psi[3] = {C(F_SPSI1), C(F_SPSI1 + 1), C(F_SPSI1 + 2)};
    auto SD = [&](int m, int d) { return S(S_MAT + 3 * m + d); };  // d_d of scalar field m
    // with the shift, dt_phi = beta^i d_i phi - alpha Pi and n^mu d_mu phi =
    // (dt_phi - beta^i d_i phi) / alpha, term by term (scalar.cc:132-140, 224-229)
    double dtphi = (-alpha * sPi), nmu_num = dtphi;
    if constexpr (SHIFT) {
      double u = beta[0] * SD(0, 0) + beta[1] * SD(0, 1);
      u = u + beta[2] * SD(0, 2);
      dtphi = u - alpha * sPi;
      nmu_num = dtphi - beta[0] * SD(0, 0);
      nmu_num = nmu_num - beta[1] * SD(0, 1);
      nmu_num = nmu_num - beta[2] * SD(0, 2);
    }
    const double nmu = (nmu_num) / alpha;
    const double dd = (gi[0] * SD(0, 0) * SD(0, 0) + gi[3] * SD(0, 1) * SD(0, 1) + gi[5] * SD(0, 2) * SD(0, 2) +
                       2.0 * (gi[1] * SD(0, 0) * SD(0, 1) + gi[2] * SD(0, 0) * SD(0, 2) + gi[4] * SD(0, 1) * SD(0, 2)));
    const double V = pot_V(ph, sphi);
    S(S_SRC + Q_R) = 0.5 * nmu * nmu + 0.5 * em4phi * dd + V;
    S(S_SRC + Q_S) = 3.0 / 2.0 * nmu * nmu - 0.5 * em4phi * dd - 3.0 * V;
#pragma unroll
    for (int m = 0; m < 3; ++m) S(S_SRC + Q_S1 + m) = -nmu * SD(0, m);
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = I; J < 3; ++J) S(S_SRC + Q_STF11 + sym(I, J)) = SD(0, I) * SD(0, J) - gm[sym(I, J)] / 3.0 * dd;
    double inner = 0.0;
#pragma unroll
    for (int X = 0; X < 3; ++X)
#pragma unroll
      for (int Y = 0; Y < 3; ++Y) {
        const double u = gi[sym(X, Y)] * (alpha * SD(2 + Y, X) + psi[X] * S(S_DA + Y));
        inner = (X == 0 && Y == 0) ? u : inner + u;
      }
    double gt[3];
#pragma unroll
    for (int I = 0; I < 3; ++I)
      gt[I] = (C(F_GAM1 + I) - 2.0 * (gi[sym(I, 0)] * S(S_DPHI + 0) + gi[sym(I, 1)] * S(S_DPHI + 1) +
                                      gi[sym(I, 2)] * S(S_DPHI + 2)));
    rhs_m[0] = dtphi;
    const double piv = alpha * ((gt[0]) * psi[0] * em4phi + (gt[1]) * psi[1] * em4phi + (gt[2]) * psi[2] * em4phi +
                                K * sPi + pot_dV(ph, sphi));
    if constexpr (SHIFT) {
      double u = beta[0] * SD(1, 0) + beta[1] * SD(1, 1);
      u = u + beta[2] * SD(1, 2);
      rhs_m[1] = (u - em4phi * (inner)) + piv;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        double w = beta[0] * SD(2 + m, 0) + beta[1] * SD(2 + m, 1);
        w = w + beta[2] * SD(2 + m, 2);
        w = w + psi[0] * db[m][0];
        w = w + psi[1] * db[m][1];
        w = w + psi[2] * db[m][2];
        w = w - alpha * SD(1, m);
        rhs_m[2 + m] = w - sPi * S(S_DA + m);
      }
    } else {
      rhs_m[1] = (-em4phi * (inner) + piv);
#pragma unroll
      for (int m = 0; m < 3; ++m) rhs_m[2 + m] = (-alpha * SD(1, m) - sPi * S(S_DA + m));
    }
  } else if (MATTER == kStaticMatter) {
    // BSSN::clearSrc, Static::addBSSNSrc (components/static/static.cc:19-36)
    // and Lambda::addBSSNSource: the fixed density sources DIFFr only
#pragma unroll
    for (int m = 0; m < Q_N; ++m) S(S_SRC + m) = 0.0;
    const double phid = C(F_PHI);
    double r = 0.0;
    r += ex[5] * C(F_DIFFD) + bg.rho_FRW * xexpm1(-6.0 * phid);
    r += ph.lambda;
    S(S_SRC + Q_R) = r;
    S(S_SRC + Q_S) = 0.0 + -3.0 * ph.lambda;
  } else {
#pragma unroll
    for (int m = 0; m < Q_N; ++m) S(S_SRC + m) = 0.0;
  }

  // -- Christoffels (bssn.cc:577-590, bssn_macros.h:221-229) --
  // Gamma^I_q go to their own slots; the lowered Gamma_{I q} then replace
  // d_I g_q, which nothing reads afterwards.
  // the pair (J, K) in a rolled loop (slot addresses at run time, one copy of
  // the code), the three brackets shared by the three I
#pragma unroll 1
  for (int q = 0; q < 6; ++q) {
    const int J = q < 3 ? 0 : (q < 5 ? 1 : 2), Kx = q < 3 ? q : (q < 5 ? q - 2 : 2);  // sym(J, Kx) = q
    auto dg = [&](int d, int qq) { return S(S_DG + 6 * d + qq); };
    const double b0 = dg(J, sym(Kx, 0)) + dg(Kx, sym(J, 0)) - dg(0, q);
    const double b1 = dg(J, sym(Kx, 1)) + dg(Kx, sym(J, 1)) - dg(1, q);
    const double b2 = dg(J, sym(Kx, 2)) + dg(Kx, sym(J, 2)) - dg(2, q);
#pragma unroll
    for (int I = 0; I < 3; ++I) {
      double u = gi[sym(I, 0)] * (b0);
      u = u + gi[sym(I, 1)] * (b1);
      u = u + gi[sym(I, 2)] * (b2);
      S(S_G + 6 * I + q) = 0.5 * (u);
    }
  }
  {
    double GLv[3][6];
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = 0; J < 3; ++J)
#pragma unroll
        for (int Kx = J; Kx < 3; ++Kx) {
          auto dg = [&](int d, int qq) { return S(S_DG + 6 * d + qq); };
          GLv[I][sym(J, Kx)] = 0.5 * (dg(J, sym(Kx, I)) + dg(Kx, sym(J, I)) - dg(I, sym(J, Kx)));
        }
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int qq = 0; qq < 6; ++qq) S(S_DG + 6 * I + qq) = GLv[I][qq];
  }
  auto G = [&](int I, int qq) { return S(S_G + 6 * I + qq); };
  auto GL = [&](int I, int qq) { return S(S_DG + 6 * I + qq); };
  double Gd[3];
#pragma unroll
  for (int I = 0; I < 3; ++I)
    Gd[I] = G(I, 0) * gi[0] + G(I, 3) * gi[3] + G(I, 5) * gi[5] + 2.0 * (G(I, 1) * gi[1] + G(I, 2) * gi[2] + G(I, 4) * gi[4]);

  // -- D_i D_j phi (bssn.cc:592-602) and (D_i D_j alpha)^TF (:604-626) --
  double dphi[3], da[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { dphi[d] = S(S_DPHI + d); da[d] = S(S_DA + d); }
  double DDa[6];
  double gld[3];
#pragma unroll
  for (int I = 0; I < 3; ++I) gld[I] = gi[sym(I, 0)] * dphi[0] + gi[sym(I, 1)] * dphi[1] + gi[sym(I, 2)] * dphi[2];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int qq = sym(I, J);
      S(S_DDPHI + qq) = S(S_DDPHI + qq) - (G(0, qq) * dphi[0] + G(1, qq) * dphi[1] + G(2, qq) * dphi[2]);
      double t = 0.0;
#pragma unroll
      for (int L = 0; L < 3; ++L) {
        const double u = G(L, qq) + 2.0 * ((L == I ? 1.0 : 0.0) * dphi[J] + (L == J ? 1.0 : 0.0) * dphi[I] - gm[qq] * gld[L]);
        t = L == 0 ? u * da[L] : t + u * da[L];
      }
      DDa[qq] = S(S_DDA + qq) - (t);
    }
  double DDaTR = gi[0] * DDa[0] + gi[3] * DDa[3] + gi[5] * DDa[5] + 2.0 * (gi[1] * DDa[1] + gi[2] * DDa[2] + gi[4] * DDa[4]);
#pragma unroll
  for (int m = 0; m < 6; ++m) S(S_DDA + m) = DDa[m] - (1.0 / 3.0) * gm[m] * DDaTR;
  DDaTR *= em4phi;

  // -- Ricci (bssn.cc:629-674, bssn_macros.h:248-277) --
  auto DDphi = [&](int qq) { return S(S_DDPHI + qq); };
  const double expression =
      (gi[0] * (DDphi(0) + 2.0 * dphi[0] * dphi[0]) + gi[3] * (DDphi(3) + 2.0 * dphi[1] * dphi[1]) +
       gi[5] * (DDphi(5) + 2.0 * dphi[2] * dphi[2]) +
       2.0 * (gi[1] * (DDphi(1) + 2.0 * dphi[0] * dphi[1]) + gi[2] * (DDphi(2) + 2.0 * dphi[0] * dphi[2]) +
              gi[4] * (DDphi(4) + 2.0 * dphi[1] * dphi[2])));
  // BSSN_CALCULATE_RICCI_UNITARY_TERM4 summed over (K,L,M) in the reference's
  // order, all six components at once so each Gamma is read once per term
  // Ricci term 4 (BSSN_CALCULATE_RICCI_UNITARY_TERM4, bssn_macros.h:248-277):
  // sum_{K,L,M} g^{LM} (G^K_{LI} G_{J,KM} + G^K_{LJ} G_{I,KM}
  // + (G^K_{IM} G_{K,LJ} + G^K_{JM} G_{K,LI}) / 2), contracted through the
  // raised symbols H^K_{MX} = sum_L g^{LM} G^K_{LX}:
  // t4_IJ = sum_{K,M} (H^K_{MI} G_{J,KM} + H^K_{MJ} G_{I,KM})
  //       + sum_{K,L} (H^K_{LI} G_{K,LJ} + H^K_{LJ} G_{K,LI}) / 2.
  // A third of the reference's multiplications, in a different summation
  // order: the FMA build uses it.  The parity build (kReferenceOrder) sums
  // the reference's terms in the reference's order, so that its rounding is
  // the reference's.
  double t4[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  if constexpr (kReferenceOrder) {
    // the parity build: the reference's 27 terms per component, summed over
    // (K, L, M) with M fastest, each term formed as the macro forms it; the
    // six components advance together, so the symbols of one K are loaded
    // once for all of them.  K is a rolled loop: its body (54 terms) stays
    // in the instruction cache for the second and third pass, where the
    // unrolled 162 terms did not (the slot addresses take K at run time; the
    // sum starts from +0, which changes no value)
#pragma unroll 1
    for (int Kx = 0; Kx < 3; ++Kx)
#pragma unroll
      for (int L = 0; L < 3; ++L)
#pragma unroll
        for (int M = 0; M < 3; ++M)
#pragma unroll
          for (int I = 0; I < 3; ++I)
#pragma unroll
            for (int J = I; J < 3; ++J) {
              const double u =
                  gi[sym(L, M)] * (G(Kx, sym(L, I)) * GL(J, sym(Kx, M)) + G(Kx, sym(L, J)) * GL(I, sym(Kx, M)) +
                                   0.5 * (G(Kx, sym(I, M)) * GL(Kx, sym(L, J)) + G(Kx, sym(J, M)) * GL(Kx, sym(L, I))));
              t4[sym(I, J)] = t4[sym(I, J)] + u;
            }
  } else {
#pragma unroll
  for (int Kx = 0; Kx < 3; ++Kx) {
    double Hm[3][3];  // H^K_{MX} = sum_L g^{LM} G^K_{LX}
#pragma unroll
    for (int M = 0; M < 3; ++M)
#pragma unroll
      for (int X = 0; X < 3; ++X)
        Hm[M][X] = gi[sym(0, M)] * G(Kx, sym(0, X)) + gi[sym(1, M)] * G(Kx, sym(1, X)) + gi[sym(2, M)] * G(Kx, sym(2, X));
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = I; J < 3; ++J) {
        double u = 0.0, w = 0.0;
#pragma unroll
        for (int M = 0; M < 3; ++M) {
          u = u + (Hm[M][I] * GL(J, sym(Kx, M)) + Hm[M][J] * GL(I, sym(Kx, M)));
          w = w + (Hm[M][I] * GL(Kx, sym(M, J)) + Hm[M][J] * GL(Kx, sym(M, I)));
        }
        t4[sym(I, J)] = t4[sym(I, J)] + (u + 0.5 * w);
      }
  }
  }
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int ij = sym(I, J);
      auto dGam = [&](int Jx, int Kx) { return S(S_DGAM + 3 * Kx + Jx); };
      const double t2a = gm[sym(0, I)] * dGam(J, 0) + gm[sym(1, I)] * dGam(J, 1) + gm[sym(2, I)] * dGam(J, 2);
      const double t2b = gm[sym(0, J)] * dGam(I, 0) + gm[sym(1, J)] * dGam(I, 1) + gm[sym(2, J)] * dGam(I, 2);
      const double t3a = Gd[0] * GL(I, sym(J, 0)) + Gd[1] * GL(I, sym(J, 1)) + Gd[2] * GL(I, sym(J, 2));
      const double t3b = Gd[0] * GL(J, sym(I, 0)) + Gd[1] * GL(J, sym(I, 1)) + Gd[2] * GL(J, sym(I, 2));
      const double U = (-0.5 * (S(S_T1 + ij)) + 0.5 * (t2a + t2b) + 0.5 * (t3a + t3b) + t4[ij]);
      S(S_T1 + ij) = U - 2.0 * (DDphi(ij) - 2.0 * dphi[I] * dphi[J] + gm[ij] * (expression));
    }
  auto Ric = [&](int qq) { return S(S_T1 + qq); };  // full Ricci R_ij (bssn.cc:650-655)
  const double ricci = em4phi * (Ric(0) * gi[0] + Ric(3) * gi[3] + Ric(5) * gi[5] +
                                 2.0 * (Ric(1) * gi[1] + Ric(2) * gi[2] + Ric(4) * gi[4]));

  // -- A^ij, A_ij A^ij (calculate_Acont, bssn.cc:463-472) --
  double A[6], Ac[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) A[q] = C(F_A11 + q);
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      double t = gi[sym(I, 0)] * gi[sym(J, 0)] * A[sym(0, 0)];
      t = t + gi[sym(I, 1)] * gi[sym(J, 0)] * A[sym(1, 0)];
      t = t + gi[sym(I, 2)] * gi[sym(J, 0)] * A[sym(2, 0)];
      t = t + gi[sym(I, 0)] * gi[sym(J, 1)] * A[sym(0, 1)];
      t = t + gi[sym(I, 1)] * gi[sym(J, 1)] * A[sym(1, 1)];
      t = t + gi[sym(I, 2)] * gi[sym(J, 1)] * A[sym(2, 1)];
      t = t + gi[sym(I, 0)] * gi[sym(J, 2)] * A[sym(0, 2)];
      t = t + gi[sym(I, 1)] * gi[sym(J, 2)] * A[sym(1, 2)];
      t = t + gi[sym(I, 2)] * gi[sym(J, 2)] * A[sym(2, 2)];
      Ac[sym(I, J)] = t;
    }
  const double AijAij = Ac[0] * A[0] + Ac[3] * A[3] + Ac[5] * A[5] + 2.0 * (Ac[1] * A[1] + Ac[2] * A[2] + Ac[4] * A[4]);
  const double r = S(S_SRC + Q_R) + bg.rho_FRW;
  // Hamiltonian constraint, bssn.cc:1073-1084 (theta = 0)
  const double H = -e5phi / 8.0 * (ricci + 2.0 / 3.0 * ((K + 2.0 * theta) * (K + 2.0 * theta)) - AijAij - 16.0 * kPi * r);

  if constexpr (MODE == kConstraints) {
    // BSSN::setConstraintCalcs per point (bssn.cc:983-1006)
    double v[5], sc[5];
    v[0] = H;  // hamiltonianConstraintCalc / Scale, bssn.cc:1073-1100
    sc[0] = (e5phi / 8.0) * sqrt(ricci * ricci + AijAij * AijAij +
                                          (2.0 / 3.0 * ((K + 2.0 * theta) * (K + 2.0 * theta))) *
                                              (2.0 / 3.0 * ((K + 2.0 * theta) * (K + 2.0 * theta))) +
                                          (16.0 * kPi * r) * (16.0 * kPi * r));
    {  // momentum, BSSN_MI / BSSN_MI_SCALE (bssn_macros.h:487-527)
      const double e6 = e6phi;
      double mv[3], ms[3];
#pragma unroll
      for (int I = 0; I < 3; ++I) {
        double t6 = 0.0;
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
          for (int X = 0; X < 3; ++X) {
            const double u = gi[sym(X, d)] * A[sym(X, I)] * dphi[d];
            t6 = (d == 0 && X == 0) ? u : t6 + u;
          }
        double tD = 0.0;
#pragma unroll
        for (int X = 0; X < 3; ++X)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double u = gi[sym(X, d)] * S(SlotsC<MATTER, Z4C>::dA + 3 * sym(X, I) + d);
            tD = (X == 0 && d == 0) ? u : tD + u;
          }
        tD = tD - Gd[0] * A[sym(0, I)] - Gd[1] * A[sym(1, I)] - Gd[2] * A[sym(2, I)];
#pragma unroll
        for (int X = 0; X < 3; ++X)
#pragma unroll
          for (int Y = 0; Y < 3; ++Y) tD = tD - GL(Y, sym(X, I)) * Ac[sym(Y, X)];
        const double sI = S(S_SRC + Q_S1 + I);
        mv[I] = e6 * (-2.0 / 3.0 * S(S_DK + I) - 8 * kPi * (sI) - 2.0 / 3.0 * 2.0 * dth[I] + 6.0 * (t6) + (tD));
        ms[I] = e6 * (fabs(2.0 / 3.0 * S(S_DK + I)) + fabs(8 * kPi * (sI)) + fabs(2.0 / 3.0 * 2.0 * dth[I]) +
                      6.0 * fabs(t6) + fabs(tD));
      }
      v[1] = sqrt(mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2]);
      sc[1] = sqrt(ms[0] * ms[0] + ms[1] * ms[1] + ms[2] * ms[2]);
    }
    {  // christoffel constraint, BSSN_GI_CALC / BSSN_GI_SCALE (bssn_macros.h:530-536)
      double gv[3], gs[3];
#pragma unroll
      for (int I = 0; I < 3; ++I) {
        const double Gam = C(F_GAM1 + I);
        gv[I] = Gam - gi[0] * G(I, 0) - gi[3] * G(I, 3) - gi[5] * G(I, 5) -
                2.0 * (gi[1] * G(I, 1) + gi[2] * G(I, 2) + gi[4] * G(I, 4));
        gs[I] = fabs(Gam) + fabs(gi[0] * G(I, 0) - gi[3] * G(I, 3) - gi[5] * G(I, 5) -
                                 2.0 * (gi[1] * G(I, 1) + gi[2] * G(I, 2) + gi[4] * G(I, 4)));
      }
      v[2] = sqrt(gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2]);
      sc[2] = sqrt(gs[0] * gs[0] + gs[1] * gs[1] + gs[2] * gs[2]);
    }
    // AijTFConstraintCalc / Scale (bssn.cc:1182-1192)
    v[3] = gi[0] * A[0] + gi[3] * A[3] + gi[5] * A[5] + 2.0 * (gi[1] * A[1] + gi[2] * A[2] + gi[4] * A[4]);
    sc[3] = fabs(gi[0] * A[0]) + fabs(gi[3] * A[3]) + fabs(gi[5] * A[5]) +
            2.0 * (fabs(gi[1] * A[1]) + fabs(gi[2] * A[2]) + fabs(gi[4] * A[4]));
    // unitDetConstraintCalc / Scale (bssn.cc:1199-1219)
    v[4] = fabs(g[0] + g[3] + g[5] - g[1] * g[1] - g[2] * g[2] - g[4] * g[4] + g[0] * g[3] + g[0] * g[5] +
                g[3] * g[5] - g[4] * g[4] * g[0] - g[2] * g[2] * g[3] - g[1] * g[1] * g[5] +
                2.0 * g[1] * g[2] * g[4] + g[0] * g[3] * g[5]);
    sc[4] = (fabs(g[0]) + fabs(g[3]) + fabs(g[5]) + g[1] * g[1] + g[2] * g[2] + g[4] * g[4] + fabs(g[0] * g[3]) +
             fabs(g[0] * g[5]) + fabs(g[3] * g[5]) + g[4] * g[4] * g[0] + g[2] * g[2] * g[3] +
             g[1] * g[1] * g[5] + 2.0 * fabs(g[1] * g[2] * g[4]) + fabs(g[0] * g[3] * g[5]));
    double q[kCPart];
    const double dx = ph.dx;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
      const double sd = v[m] / sc[m];
      q[m] = live ? v[m] : 0.0;
      q[5 + m] = live ? sc[m] : 0.0;
      q[10 + m] = live ? sd : 0.0;
      q[17 + m] = live ? fabs(v[m]) : 0.0;
      q[22 + m] = live ? fabs(sd) : 0.0;
      if (live) {
        P.cvals[(size_t)(2 * m) * N + c] = v[m];
        P.cvals[(size_t)(2 * m + 1) * N + c] = sd;
      }
    }
    if (live) {
      // ricci_a (bssn.cc:663) and DIFFr_a at this point, for io_bssn_dump_statistics
      P.cvals[(size_t)10 * N + c] = ricci;
      P.cvals[(size_t)11 * N + c] = S(S_SRC + Q_R);
    }
    q[15] = live ? v[0] * v[0] * dx * dx * dx : 0.0;
    q[16] = live ? v[1] * v[1] * dx * dx * dx : 0.0;
    cta_reduce<kCPart, 17>(q, P.cpart, cta);
    return;
  }

  // ---- evolution equations and K{n}Finalize, field by field --------------------
  const double dt = ph.dt;
  double outv[NFLD];
  const bool renorm = ph.normalize != 0;
  // Kreiss-Oliger terms of the 18 BSSN fields (subtracted from their RHS,
  // bssn.cc:748-831), parked in the slots of the lowered Christoffels, which
  // nothing reads after the Ricci tensor
  constexpr int RKO = O == 8 ? 5 : 2;
  const bool ko_on = KO && (O == 2 || O == 8) && ph.ko_coeff != 0.0;
  if constexpr (KO) {
    if (ko_on) {
      const bool inside = x0 >= RKO && x0 + kBX + RKO <= geo.nx && y0 >= RKO && y0 + kBY + RKO <= geo.ny &&
                          z0 >= RKO && z0 + kBZ + RKO <= geo.nz;
#pragma unroll 1
      for (int f = 0; f < F_NBSSN; ++f)
        S(S_DG + f) = ko_dissipation<O>(a + (size_t)f * N, i, j, k, geo.nx, geo.ny, geo.nz, inside, ph);
    }
  }
  auto ko = [&](int fld) -> double { return ko_on ? S(S_DG + fld) : 0.0; };
  // Each right-hand side is parked in a slot free in the epilogue (the
  // lowered Christoffels for the 18 BSSN fields, after the field's
  // dissipation value there has been read; d_J Gamma^K and D_i D_j phi for the
  // rest), and one rolled loop below updates the registers of every field.
  static_assert(NFLD <= F_NBSSN + 9 + 6, "every right-hand side has a slot");
  auto cvslot = [](int fld) { return fld < F_NBSSN ? S_DG + fld : (fld < F_NBSSN + 9 ? S_DGAM + fld - F_NBSSN : S_DDPHI + fld - F_NBSSN - 9); };
  auto finalize = [&](int fld, double cv) { S(cvslot(fld)) = cv; };

  // ev_DIFFgammaIJ (bssn.cc:748-753, BSSN_DT_DIFFGAMMAIJ bssn_macros.h:292-307)
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int m = sym(I, J);
      double v = (-2.0 * alpha * A[m]);
      if constexpr (SHIFT) {
        // advection and the Lie-derivative terms of the shift, term by term
#pragma unroll
        for (int d = 0; d < 3; ++d) v = v + up(F_G11 + m, d);
#pragma unroll
        for (int X = 0; X < 3; ++X) v = v + gm[sym(I, X)] * db[J][X];
#pragma unroll
        for (int X = 0; X < 3; ++X) v = v + gm[sym(J, X)] * db[I][X];
        v = v - (2.0 / 3.0) * gm[m] * (divb);
      }
      finalize(F_G11 + m, v + 0.5 * ph.a_adj_amp * dt * H * g[m] - ko(F_G11 + m));
    }
  // ev_AIJ (bssn.cc:755-760, BSSN_DT_AIJ bssn_macros.h:334-337); with the
  // shift the A_ij and Gamma^i right-hand sides are kept for the
  // AijDriverShift and Gamma-driver gauges
  double rhsA[6], rhsG[3];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int qq = sym(I, J);
      double aa = 0.0;
#pragma unroll
      for (int X = 0; X < 3; ++X)
#pragma unroll
        for (int Y = 0; Y < 3; ++Y) {
          const double u = gi[sym(X, Y)] * A[sym(X, I)] * A[sym(Y, J)];
          aa = (X == 0 && Y == 0) ? u : aa + u;
        }
      const double RTF = Ric(qq) - (1.0 / 3.0) * e4phi * gm[qq] * ricci;
      double dtA = (em4phi * (alpha * (RTF - 8.0 * kPi * S(S_SRC + Q_STF11 + qq)) - S(S_DDA + qq)) +
                    alpha * (((K + 2.0 * theta) * A[qq]) - 2.0 * (aa)));
      if constexpr (SHIFT) {  // BSSN_DT_AIJ with the shift (bssn_macros.h:319-332)
#pragma unroll
        for (int d = 0; d < 3; ++d) dtA = dtA + up(F_A11 + qq, d);
#pragma unroll
        for (int X = 0; X < 3; ++X) dtA = dtA + A[sym(I, X)] * db[J][X];
#pragma unroll
        for (int X = 0; X < 3; ++X) dtA = dtA + A[sym(J, X)] * db[I][X];
        dtA = dtA - (2.0 / 3.0) * A[qq] * (divb);
      }
      const double evA = dtA - 1.0 * ph.a_adj_amp * dt * A[qq] * H - ko(F_A11 + qq);
      if constexpr (SHIFT) rhsA[qq] = evA;
      finalize(F_A11 + qq, evA);
    }
  // ev_GammaI (bssn.cc:762-764, BSSN_DT_GAMMAI_NOSHIFT bssn_macros.h:342-361)
  const double sq[3] = {S(S_SRC + Q_S1), S(S_SRC + Q_S2), S(S_SRC + Q_S3)};
#pragma unroll
  for (int I = 0; I < 3; ++I) {
    auto Gs = [&](int qq) { return S(S_G + 6 * I + qq); };
    const double so = (Gs(0) * Ac[0] + Gs(3) * Ac[3] + Gs(5) * Ac[5] + 2.0 * (Gs(1) * Ac[1] + Gs(2) * Ac[2] + Gs(4) * Ac[4]) +
                       6.0 * (Ac[sym(I, 0)] * dphi[0] + Ac[sym(I, 1)] * dphi[1] + Ac[sym(I, 2)] * dphi[2]));
    const double ns =
        (-2.0 * (Ac[sym(I, 0)] * da[0] + Ac[sym(I, 1)] * da[1] + Ac[sym(I, 2)] * da[2]) +
         2.0 * alpha *
             (+so -
              (1.0 / 3.0) * (2.0 * (gi[sym(I, 0)] * S(S_DK + 0) + gi[sym(I, 1)] * S(S_DK + 1) + gi[sym(I, 2)] * S(S_DK + 2)) +
                             gi[sym(I, 0)] * dth[0] + gi[sym(I, 1)] * dth[1] + gi[sym(I, 2)] * dth[2]) -
              2.0 * alpha * k1 * (C(F_GAM1 + I) - Gd[I]) -
              8.0 * kPi * (gi[sym(I, 0)] * sq[0] + gi[sym(I, 1)] * sq[1] + gi[sym(I, 2)] * sq[2])));
    if constexpr (SHIFT) {
      // BSSN_DT_GAMMAI_SHIFT (bssn_macros.h:363-382), term by term
      double sh = up(F_GAM1 + I, 0);
      sh = sh + up(F_GAM1 + I, 1);
      sh = sh + up(F_GAM1 + I, 2);
      sh = sh - Gd[0] * db[0][I];
      sh = sh - Gd[1] * db[1][I];
      sh = sh - Gd[2] * db[2][I];
      sh = sh + (2.0 / 3.0) * Gd[I] * (divb);
      double t = 0.0;  // gamma^{IJ} d_K d_J beta^K, J slow, K fast
#pragma unroll
      for (int Jx = 0; Jx < 3; ++Jx)
#pragma unroll
        for (int Kx = 0; Kx < 3; ++Kx) {
          const double u = gi[sym(I, Jx)] * ddf(Kx, Jx, F_BETA + Kx);
          t = (Jx == 0 && Kx == 0) ? u : t + u;
        }
      sh = sh + (1.0 / 3.0) * (t);
      const double w = (gi[0] * ddf(0, 0, F_BETA + I) + gi[3] * ddf(1, 1, F_BETA + I) + gi[5] * ddf(2, 2, F_BETA + I) +
                        2.0 * (gi[1] * ddf(0, 1, F_BETA + I) + gi[2] * ddf(0, 2, F_BETA + I) +
                               gi[4] * ddf(1, 2, F_BETA + I)));
      sh = sh + (w);
      rhsG[I] = (ns + sh) - ko(F_GAM1 + I);
      finalize(F_GAM1 + I, rhsG[I]);
    } else {
      finalize(F_GAM1 + I, ns + 0.0 - ko(F_GAM1 + I));
    }
  }
  // ev_DIFFK (bssn.cc:766-795)
  {
    double v = (-DDaTR + alpha * (1.0 / 3.0 * (Kd + 2.0 * theta) * (Kd + 2.0 * theta + 2.0 * bg.K_FRW) + AijAij) +
                4.0 * kPi * alpha * (S(S_SRC + Q_R) + S(S_SRC + Q_S)) + 4.0 * kPi * alphad * (bg.rho_FRW + bg.S_FRW));
    if constexpr (SHIFT) {
#pragma unroll
      for (int d = 0; d < 3; ++d) v = v + up(F_K, d);
    }
    if (ph.k_damping_amp != 0.0) v = v - 1.0 * ph.k_damping_amp * H * em5phi;
    if constexpr (Z4C) v = v + k1 * (1.0 - k2) * theta;
    finalize(F_K, v - ko(F_K));
  }
  // ev_DIFFphi (bssn.cc:797-820)
  {
    double v = (0.1 * ph.a_adj_amp * dt * H - 1.0 / 6.0 * (alpha * (Kd + 2.0 * theta) + alphad * bg.K_FRW - (divb)));
    if constexpr (SHIFT) {
#pragma unroll
      for (int d = 0; d < 3; ++d) v = v + up(F_PHI, d);
    }
    finalize(F_PHI, v - ko(F_PHI));
  }
  // ev_DIFFalpha (bssn.cc:822-831)
  if constexpr (SHIFT) {
    double v = ev_lapse_shift(ph, bg, alpha, K, Kd, phi, beta, da);
#pragma unroll
    for (int d = 0; d < 3; ++d) v = v + up(F_ALPHA, d);
    finalize(F_ALPHA, v - ko(F_ALPHA));
  } else {
    finalize(F_ALPHA, ev_lapse(ph, bg, alpha, K, Kd, phi) - ko(F_ALPHA));
  }
  if constexpr (Z4C) {
    // ev_theta (bssn.cc:834-848)
    double kth = 0.0;
    if constexpr (KO) {
      if (ko_on) {
        const bool inside = x0 >= RKO && x0 + kBX + RKO <= geo.nx && y0 >= RKO && y0 + kBY + RKO <= geo.ny &&
                            z0 >= RKO && z0 + kBZ + RKO <= geo.nz;
        kth = ko_dissipation<O>(a + (size_t)F_THETA * N, i, j, k, geo.nx, geo.ny, geo.nz, inside, ph);
      }
    }
    finalize(F_THETA, (0.5 * alpha * (ricci + 2.0 / 3.0 * ((K + 2.0 * theta) * (K + 2.0 * theta)) - AijAij -
                                      16.0 * kPi * (r)) -
                       alpha * k1 * (2.0 + k2) * theta) -
                          kth);
  }
  if constexpr (SHIFT) {
    // ev_beta^i: the shift gauge minus the dissipation (bssn.cc:853-869,
    // BSSNGaugeHandler.cc:113-146, 156-211, 226-273)
#pragma unroll
    for (int I = 0; I < 3; ++I) {
      double v = 0.0;
      switch (ph.shift) {
        case kShiftGammaDriver: v = C(F_AUXB + I); break;
        case kShiftDampedWave: {
          // the reference's y and z shifts both read Gamma3
          const double GamI = C(F_GAM1 + (I == 0 ? 0 : 2));
          v = beta[0] * db[0][I] + beta[1] * db[1][I];
          v = v + beta[2] * db[2][I];
          v = v - ph.dw_mu_s * alpha * beta[I];
          double X = -gi[sym(I, 0)] * da[0];
          X = X - gi[sym(I, 1)] * da[1];
          X = X - gi[sym(I, 2)] * da[2];
          X = X + alpha * (GamI - 2.0 * (gi[sym(I, 0)] * dphi[0] + gi[sym(I, 1)] * dphi[1] + gi[sym(I, 2)] * dphi[2]));
          v = v + alpha * (-ph.dw_mu_l * (12.0 * phi * ph.dw_p - log(alpha)) * beta[I] + em4phi * (X));
          break;
        }
        case kShiftAwA: v = ph.gauge_wave_dir == I + 1 ? -2.0 * K * alpha : 0.0; break;
        case kShiftAijDriver:
          v = -ph.k_driver_coeff * (fabs(rhsA[sym(I, 0)] + A[sym(I, 0)]) + fabs(rhsA[sym(I, 1)] + A[sym(I, 1)]) +
                                    fabs(rhsA[sym(I, 2)] + A[sym(I, 2)]));
          break;
        default: break;
      }
      double kb = 0.0;
      if (ko_on) {
        const bool inside = x0 >= RKO && x0 + kBX + RKO <= geo.nx && y0 >= RKO && y0 + kBY + RKO <= geo.ny &&
                            z0 >= RKO && z0 + kBZ + RKO <= geo.nz;
        kb = ko_dissipation<O>(a + (size_t)(F_BETA + I) * N, i, j, k, geo.nx, geo.ny, geo.nz, inside, ph);
      }
      finalize(F_BETA + I, v - kb);
    }
    // ev_auxB^i (bssn.cc:879-892)
#pragma unroll
    for (int I = 0; I < 3; ++I) finalize(F_AUXB + I, 0.75 * rhsG[I] - ph.gd_eta * C(F_AUXB + I));
    // ev_expN (bssn.cc:871-875)
    {
      double v = beta[0] * d1<O>(gtap(F_EXPN), 0, ph) + beta[1] * d1<O>(gtap(F_EXPN), 1, ph);
      v = v + beta[2] * d1<O>(gtap(F_EXPN), 2, ph);
      finalize(F_EXPN, v - alpha * K / 3.0);
    }
  }
  if (MATTER == kDust) {
#pragma unroll
    for (int m = 0; m < 4; ++m) finalize(F_D + m, rhs_m[m]);
  } else if (MATTER == kScalar) {
#pragma unroll
    for (int m = 0; m < 5; ++m) finalize(F_SPHI + m, rhs_m[m]);
  } else if (MATTER == kStaticMatter) {
    // the fixed density is no register of the reference: every output keeps it
    const double pv = __ldcs(&P.p[(size_t)F_DIFFD * N + c]);
    __stcs(&P.out[(size_t)F_DIFFD * N + c], pv);
    if (stage == 4) __stcs(&P.norm[(size_t)F_DIFFD * N + c], pv);
    S(cvslot(F_DIFFD)) = pv;
  }

  // RK4Register::K{n}Finalize (RK4Register.h:180-230) of every field, one
  // rolled loop (one copy of the code) with the next field's registers
  // loaded while this one is updated; the substep's divisors chosen once:
  // f = f + dt cv / 6 (substep 1, from f = 0), / 3 (2, 3); a = p + dt cv / 2
  // (1, 2), / 1 (3); p = f + (dt cv / 6 + p) (4).  IEEE division rounds the
  // same for a divisor held in a register, and 0 + x = x, so the values are
  // those of the four separate forms.  The new values replace the
  // right-hand sides in the slots.
  {
    const double fdiv = stage == 1 ? 6.0 : 3.0, odiv = stage == 3 ? 1.0 : 2.0;
    auto skip = [](int fld) { return MATTER == kStaticMatter && fld == F_DIFFD; };
    double pv = __ldcs(&P.p[c]);
    double fv = stage == 1 ? 0.0 : __ldcs(&P.f[c]);
#pragma unroll 1
    for (int fld = 0; fld < NFLD; ++fld) {
      const double pcur = pv, fcur = fv;
      if (fld + 1 < NFLD) {
        pv = __ldcs(&P.p[(size_t)(fld + 1) * N + c]);
        fv = stage == 1 ? 0.0 : __ldcs(&P.f[(size_t)(fld + 1) * N + c]);
      }
      if (skip(fld)) continue;
      const double t = dt * S(cvslot(fld));
      double o;
      if (stage == 4) {
        o = fcur + (t / 6.0 + pcur);
      } else {
        __stcs(&P.f[(size_t)fld * N + c], fcur + t / fdiv);
        o = pcur + t / odiv;
      }
      __stcs(&P.out[(size_t)fld * N + c], o);
      // at the last substep the new state is also the next step's first
      // input, except gamma and A, which are renormalised below
      if (stage == 4 && !(renorm && fld < F_K && fld != F_PHI)) __stcs(&P.norm[(size_t)fld * N + c], o);
      S(cvslot(fld)) = o;
    }
  }
#pragma unroll
  for (int f = 0; f < NFLD; ++f) outv[f] = S(cvslot(f));

  // ---- the next substep's inputs -----------------------------------------------
  if (stage == 4) {
    // failure detection (sims/sim.cc:179-183 counts NaNs of DIFFphi)
    bool bad_any = false;
#pragma unroll
    for (int f = 0; f < NFLD; ++f) bad_any |= !isfinite(outv[f]);
    if (bad_any) {
      if (isnan(outv[F_PHI])) atomicOr(P.status, kStatusNaN);
      atomicOr(P.status, kStatusNonFinite);
    }
    // next step's first-substep input: normalised gamma/A (bssn.cc:224-225)
    if (renorm) {
      double gn[6], An[6];
#pragma unroll
      for (int m = 0; m < 6; ++m) { gn[m] = outv[F_G11 + m]; An[m] = outv[F_A11 + m]; }
      normalize_point(gn, An);
#pragma unroll
      for (int m = 0; m < 6; ++m) {
        outv[F_G11 + m] = gn[m];
        outv[F_A11 + m] = An[m];
        __stcs(&P.norm[(size_t)(F_G11 + m) * N + c], gn[m]);
        __stcs(&P.norm[(size_t)(F_A11 + m) * N + c], An[m]);
      }
    }
  }
  if (MATTER == kDust) {
    // flux primitives of the output state for the next substep's divergence
    double go[6], gio[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) go[m] = outv[F_G11 + m];
    inv_metric(go, gio);
    const double So[3] = {outv[F_S1], outv[F_S2], outv[F_S3]};
    const double phio = outv[F_PHI] + bg.phi_FRW_next;
    double eo[2];
    {
      const double xo[2] = {-4.0 * phio, 6.0 * phio};
      xexp_n<2>(xo, eo);
    }
    const DustPrim dp = dust_prim(gio, eo[0], eo[1], outv[F_D], So);
    const double alo = outv[F_ALPHA] + 1.0;
    double* fo = P.fp_out;
    __stcs(&fo[(size_t)P_AD * N + c], alo * outv[F_D]);
#pragma unroll
    for (int m = 0; m < 3; ++m) __stcs(&fo[(size_t)(P_AS1 + m) * N + c], alo * So[m]);
#pragma unroll
    for (int m = 0; m < 3; ++m) __stcs(&fo[(size_t)(P_V1 + m) * N + c], dp.v[m]);
  }
}

// the two TMA barriers of a CTA: initialised once, before any copy
__device__ __forceinline__ void init_tile_barriers(uint64_t* bar, bool use) {
  if (use && threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
    tma::bar_init(bar, 1);
    tma::bar_init(bar + 1, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

// One box: one CTA per brick.  tmap: the TMA map of this substep's input
// (use_tma = 0: every tile is copied by the threads).
template <int O, int MATTER, int MODE, bool KO = false, bool Z4C = false, bool SHIFT = false>
__global__ void __launch_bounds__(kThreads, 2)
stage_kernel(BoxGeom geo, Physics ph, StageBg bg, StagePtrs P, int stage, const __grid_constant__ CUtensorMap tmap,
             int use_tma, const __grid_constant__ FluxMaps fmaps, int use_fmaps) {
  __shared__ __align__(8) uint64_t bar[2];
  init_tile_barriers(bar, use_tma != 0);
  unsigned phase = 0;
  bool tma_ok = true;
  stage_body<O, MATTER, MODE, KO, Z4C, SHIFT>(geo, ph, bg, P, stage, blockIdx.z + geo.bx0, blockIdx.y, blockIdx.x,
                                  blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
                                  use_tma ? &tmap : nullptr, bar, phase, tma_ok,
                                  use_tma && use_fmaps ? &fmaps : nullptr);
}

// A group of boxes of the same order and matter model, one launch per
// substep: the bricks of all boxes form one work list (boxes[] in launch
// order, box b's bricks at [first, first + bricks)); each CTA takes work
// items blockIdx.x, blockIdx.x + gridDim.x, ... (a persistent launch when the
// grid is smaller than the list).
template <int O, int MATTER>
__global__ void __launch_bounds__(kThreads, 2)
stage_group_kernel(const GroupBox* __restrict__ boxes, GroupBg gb, int stage) {
  __shared__ GroupBox sb;
  __shared__ StagePtrs sp;
  __shared__ StageBg sbg;
  __shared__ const CUtensorMap* stm;
  __shared__ const FluxMaps* sfm;
  __shared__ __align__(8) uint64_t bar[2];
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0;
  init_tile_barriers(bar, true);
  unsigned phase = 0;
  bool tma_ok = true;
  for (int w = blockIdx.x; w < gb.total; w += gridDim.x) {
    __syncthreads();  // the previous brick is finished with the slots, the tile and sb
    if (lead) {
      int lo = 0, hi = gb.nboxes - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (boxes[mid].first <= w) lo = mid; else hi = mid - 1;
      }
      sb = boxes[lo];
      sp = group_ptrs(sb, stage);
      sbg = gb.bg[lo];
      // the map is read from global memory (a TMA map cannot live in shared memory)
      stm = boxes[lo].tma ? (stage == 1 || stage == 3 ? &boxes[lo].mapX : &boxes[lo].mapY) : nullptr;
      if (stm) tma::acquire_map(stm);  // the host wrote the map into the table
      sfm = nullptr;
      if (MATTER == kDust && stm) {  // the flux-primitive boxes, after the GroupBox entries
        const GroupFluxMaps& fx = reinterpret_cast<const GroupFluxMaps*>(boxes + gb.nboxes)[lo];
        if (fx.valid) {
          sfm = reinterpret_cast<const FluxMaps*>(stage == 1 || stage == 3 ? fx.fp0 : fx.fp1);
          for (int a = 0; a < 3; ++a) tma::acquire_map(&sfm->m[a]);
        }
      }
    }
    __syncthreads();
    const int l = w - sb.first;
    const int cz = l % sb.nbz, cy = (l / sb.nbz) % sb.nby, cx = l / (sb.nbz * sb.nby);
    const BoxGeom geo{sb.nx, sb.ny, sb.nz, sb.pts, 0};
    stage_body<O, MATTER, kEvolve>(geo, sb.ph, sbg, sp, stage, cx, cy, cz, 0, stm, bar, phase, tma_ok, sfm);
  }
}

}  // namespace CG_VARIANT_NS
}  // namespace cg
