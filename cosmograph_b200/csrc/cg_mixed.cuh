// cg_mixed.cuh -- the FP32-mixed RK4 substep kernel (BSSN + dust or vacuum).
//
// Same fused substep as cg_stage.cuh (sources, BSSN and dust right-hand
// sides, RK4Register::K{n}Finalize, next-substep inputs) with a different
// split of precision:
//   * the substep inputs a^n are stored as FP32 perturbations
//       delta_f = a_f - abar_f
//     about a spatially uniform background abar (one value per field and
//     substep) that the host integrates in FP64 with the same RK4 stages;
//   * stencils and the right-hand side are evaluated in FP32 in perturbation
//     form: the kernel computes RHS(abar + delta) - RHS(abar), and the host
//     adds RHS(abar) in FP64.  Every term of the BSSN and dust equations is
//     already first order in the perturbation except the zeroth-order parts
//     of dK/dt, dphi/dt, dalpha/dt and the dust density source; those are
//     expanded explicitly (e.g. alpha K^2 - abar Kbar^2 =
//     abar (2 Kbar + dK) dK + dalpha K^2) so no FP32 cancellation occurs;
//   * the RK registers _p and _f and the register update stay FP64.
// The equations are the reference's (components/bssn/bssn.cc:361-831,
// bssn_macros.h:221-385, components/dust_fluid/dust.cc:109-264) with a
// trivial FRW reference (the dust driver's FRW(0,0), bssn.cc:25), every
// lapse gauge of BSSNGaugeHandler (the K_avg of the ConformalFLRW, Anharmonic
// and 1+log lapses enters as its perturbation, reduced from the FP32 inputs),
// Kreiss-Oliger dissipation (orders 2 and 8), a_adj_amp = k_damping_amp = 0.
#pragma once

#include "cg_group.h"
#include "cosmograph_b200.h"
#include "cg_tile.cuh"
#include "cg_tma.cuh"
#include "cg_types.h"

namespace cg {
namespace mixed {

using Brick = tile::Brick32;
constexpr int kBX = Brick::BX, kBY = Brick::BY, kBZ = Brick::BZ, kThreads = Brick::THREADS;
// FP32 tiles with a 24-float row pitch (conflict-free taps, cg_tile.cuh)
// whose column 0 is z0 - 4: a TMA box {24, TY, TX} starts at an aligned z
// for every stencil order
template <int O>
using TileG = tile::Geom<O, Brick, 24, 4>;
constexpr unsigned kStatusTileTimeout = CG_STATUS_TILE_TIMEOUT;  // a TMA tile copy was late or lost

struct Ptrs {
  const float* in;     // delta of a^n
  const float* prev;   // delta of a^{n-1} (substeps 2-4)
  const double* p;     // _p (FP64, full values)
  double* f;           // _f (FP64)
  double* newp;        // substep 4: the new _p (same block as p)
  float* out;          // delta of a^{n+1}, or of the next step's a^1 at substep 4
  const float* fp_in;  // dust flux primitives of a^n (FP32)
  float* fp_out;       // flux primitives of the output state
  unsigned* status;
  const double* kavg;  // K_avg - Kbar of the substep input (lapses with K_avg), else null
};

// Uniform background of one substep (FP64).  A uniform state keeps every
// field but K, phi, alpha and, for matter, D or the scalar phi and Pi at
// zero, so only those five are stored, at index bgi(field) (field 18 is D or
// the scalar phi, field 19 is S1 or Pi).
constexpr int kBgN = 5;
struct Bg {
  double in[kBgN];    // abar of a^n
  double prev[kBgN];  // abar of a^{n-1}
  double out[kBgN];   // abar of the substep output
  double rhs[kBgN];   // RHS(abar of a^n), added to the kernel's perturbation RHS
  double e6l;         // exp(-6 phibar) of the state whose W, sqrt(gamma) the sources lag on
  double lambda;      // rho_Lambda
  double pot_const, pot_mass;  // scalar potential V = pot_const or m^2 phi^2 / 2
  int potential;
  double gd_c;                 // 1+log lapse coefficient
  double dw_mu_l, dw_p, dw_u;  // damped-wave lapse: mu_L, p and mu_L (12 p phibar - ln abar) - Kbar
  double ko_scale;             // Kreiss-Oliger: c / (64 dx) (order 2) or -c / (1024 dx) (order 8)
  long long tma_wait;          // cycles a CTA waits for a TMA tile copy before it flags a timeout
  // constraint damping (a_adj_amp, k_damping_amp): the background's
  // Hamiltonian constraint Hbar = -e^{5 phibar} / 8 * Hcbar, Hcbar =
  // 2/3 Kbar^2 - 16 pi rhobar, and a_adj_amp dt, k_damping_amp / 8
  double Hbar, Hcbar, e5phib, a_adj_dt, k_damp8;
  int damping;                 // either amplitude is nonzero
};
__host__ __device__ constexpr int bgi(int f) {
  return f == F_K ? 0 : (f == F_PHI ? 1 : (f == F_ALPHA ? 2 : (f == 18 ? 3 : (f == 19 ? 4 : -1))));
}
__host__ __device__ inline double bgv(const double* a, int f) { return bgi(f) < 0 ? 0.0 : a[bgi(f)]; }

// One box of a mixed launch group (device table) and the per-substep
// backgrounds of a group (kernel parameter); as the FP64 GroupBox / GroupBg.
struct GroupBox {
  CUtensorMap mapX, mapY;  // TMA maps of the FP32 inputs (valid when tma != 0)
  int nx, ny, nz, pts, lapse, normalize;
  float idx;
  double dt;
  double *P, *F;
  float *X, *Y, *FP0, *FP1;
  unsigned* status;
  const double* kavg;
  int nbx, nby, nbz;
  int first;
  int tma;
};
struct GroupBg {
  int nboxes, total;
  Bg bg[kMaxGroupBoxes];
};

// per-thread FP32 slots (same meaning as the FP64 kernel's)
enum : int {
  S_DG = 0, S_T1 = 18, S_DPHI = 24, S_DDPHI = 27, S_DA = 33, S_DDA = 36, S_DK = 42,
  S_DGAM = 45, S_SRC = 54, S_G = 65, S_MAT = 83, S_NSLOT = 87
};
// slots per thread: dust 4 flux divergences, scalar 15 first derivatives
template <int MATTER>
struct NSlot {
  static constexpr int value = S_MAT + (MATTER == kDust ? 4 : (MATTER == kScalar ? 15 : 0));
};
// phase 1 writes no slot in [S_SRC, S_MAT): the field tile lives there
constexpr int kTileSlot = S_SRC, kTileSlots = S_MAT - S_SRC;

__device__ __forceinline__ int wrapf(int v, int n) {
  v = v < 0 ? v + n : v;
  return v >= n ? v - n : v;
}

template <bool WRAP>
struct Taps {
  int i, j, k, nx, ny, nz, sx, sy, c;
  __device__ __forceinline__ int at(int di, int dj, int dk) const {
    if (!WRAP) return c + di * sx + dj * sy + dk;
    return (wrapf(i + di, nx) * ny + wrapf(j + dj, ny)) * nz + wrapf(k + dk, nz);
  }
  __device__ __forceinline__ int ax(int a, int n) const {
    return at(a == 0 ? n : 0, a == 1 ? n : 0, a == 2 ? n : 0);
  }
  __device__ __forceinline__ int pl(int a, int n, int b, int m) const {
    return at((a == 0 ? n : 0) + (b == 0 ? m : 0), (a == 1 ? n : 0) + (b == 1 ? m : 0),
              (a == 2 ? n : 0) + (b == 2 ? m : 0));
  }
};

// taps of one field read from global memory through index taps T
template <class T>
struct GTaps {
  const float* f;
  T t;
  __device__ __forceinline__ float ax(int a, int n) const { return __ldg(f + t.ax(a, n)); }
};

// FP32 centred stencils (utils/math.h:74-1085 coefficients)
template <int O, class T>
__device__ __forceinline__ float d1(const T& t, int a, float idx) {
  auto V = [&](int n) { return t.ax(a, n); };
  float s;
  if (O == 2) s = 0.5f * (V(1) - V(-1));
  else if (O == 4) s = (2.0f / 3.0f) * (V(1) - V(-1)) - (1.0f / 12.0f) * (V(2) - V(-2));
  else if (O == 6) s = 0.75f * (V(1) - V(-1)) - 0.15f * (V(2) - V(-2)) + (1.0f / 60.0f) * (V(3) - V(-3));
  else s = 0.8f * (V(1) - V(-1)) - 0.2f * (V(2) - V(-2)) + (4.0f / 105.0f) * (V(3) - V(-3)) - (1.0f / 280.0f) * (V(4) - V(-4));
  return s * idx;
}
template <int O, class T>
__device__ __forceinline__ float d2(const T& t, int a, float idx2) {
  auto V = [&](int n) { return t.ax(a, n); };
  float s;
  if (O == 2) s = (V(1) + V(-1)) - 2.0f * V(0);
  else if (O == 4) s = (4.0f / 3.0f) * (V(1) + V(-1)) - (1.0f / 12.0f) * (V(2) + V(-2)) - 2.5f * V(0);
  else if (O == 6) s = 1.5f * (V(1) + V(-1)) - 0.15f * (V(2) + V(-2)) + (1.0f / 90.0f) * (V(3) + V(-3)) - (49.0f / 18.0f) * V(0);
  else s = 1.6f * (V(1) + V(-1)) - 0.2f * (V(2) + V(-2)) + (8.0f / 315.0f) * (V(3) + V(-3)) - (1.0f / 560.0f) * (V(4) + V(-4)) - (205.0f / 72.0f) * V(0);
  return s * idx2;
}
template <int O, class T>
__device__ __forceinline__ float dm(const T& t, int a, int b, float idx2) {
  auto P = [&](int n) { return (t.pl(a, n, b, n) + t.pl(a, -n, b, -n)) - (t.pl(a, n, b, -n) + t.pl(a, -n, b, n)); };
  float s;
  if (O == 2) s = 0.25f * P(1);
  else if (O == 4) s = (1.0f / 3.0f) * P(1) - (1.0f / 48.0f) * P(2);
  else if (O == 6) s = 0.375f * P(1) - 0.0375f * P(2) + (1.0f / 360.0f) * P(3);
  else s = 0.4f * P(1) - 0.05f * P(2) + (2.0f / 315.0f) * P(3) - (1.0f / 2240.0f) * P(4);
  return s * idx2;
}
template <int O, class T>
__device__ __forceinline__ float d1p(const float* __restrict__ fa, const float* __restrict__ fb, const T& t, int a,
                                     float idx) {
  auto V = [&](int n) {
    const int q = t.ax(a, n);
    return __ldg(fa + q) * __ldg(fb + q);
  };
  float s;
  if (O == 2) s = 0.5f * (V(1) - V(-1));
  else if (O == 4) s = (2.0f / 3.0f) * (V(1) - V(-1)) - (1.0f / 12.0f) * (V(2) - V(-2));
  else if (O == 6) s = 0.75f * (V(1) - V(-1)) - 0.15f * (V(2) - V(-2)) + (1.0f / 60.0f) * (V(3) - V(-3));
  else s = 0.8f * (V(1) - V(-1)) - 0.2f * (V(2) - V(-2)) + (4.0f / 105.0f) * (V(3) - V(-3)) - (1.0f / 280.0f) * (V(4) - V(-4));
  return s * idx;
}

__device__ __forceinline__ void inv_metricf(const float g[6], float gi[6]) {
  gi[0] = 1.0f + g[3] + g[5] - g[4] * g[4] + g[3] * g[5];
  gi[3] = 1.0f + g[0] + g[5] - g[2] * g[2] + g[0] * g[5];
  gi[5] = 1.0f + g[0] + g[3] - g[1] * g[1] + g[0] * g[3];
  gi[1] = g[2] * g[4] - g[1] * (1.0f + g[5]);
  gi[2] = g[1] * g[4] - g[2] * (1.0f + g[3]);
  gi[4] = g[1] * g[2] - g[4] * (1.0f + g[0]);
}

// W - 1 (as w2/(W+1), no cancellation) and v^i of Dust::getDustData (dust.cc:177-200)
struct DustF {
  float W, Wm1, w2, v[3];
};
__device__ __forceinline__ DustF dust_primf(const float gi[6], float em4, float e6, float D, const float S[3]) {
  DustF d;
  d.w2 = em4 * (gi[0] * S[0] * S[0] + gi[3] * S[1] * S[1] + gi[5] * S[2] * S[2] +
                2.0f * (gi[1] * S[0] * S[1] + gi[2] * S[0] * S[2] + gi[4] * S[1] * S[2])) / (D * D);
  d.W = sqrtf(1.0f + d.w2);
  d.Wm1 = d.w2 / (d.W + 1.0f);
  const float c = em4 / e6;
  d.v[0] = c * (gi[0] * S[0] + gi[1] * S[1] + gi[2] * S[2]);
  d.v[1] = c * (gi[1] * S[0] + gi[3] * S[1] + gi[4] * S[2]);
  d.v[2] = c * (gi[2] * S[0] + gi[4] * S[1] + gi[5] * S[2]);
  return d;
}

// Phase 1 (as in the FP64 kernel): the metric components, phi and alpha with
// first and second derivatives, one field tile at a time, the next field
// fetched into registers meanwhile.  The fields with first derivatives only
// (K, Gamma^i, the scalar field) read their taps from global memory after
// the tiles (mixed_body).
__device__ __forceinline__ int phase1_field(int it) {
  return it < 6 ? F_G11 + it
                : (it == 6 ? F_PHI : (it == 7 ? F_ALPHA : (it == 8 ? F_K : (it < 12 ? F_GAM1 + it - 9 : F_SPHI + it - 12))));
}

// first and second derivatives of phase-1 field `it` from its tile
template <int O, class T>
__device__ __forceinline__ void field_derivatives(int it, const T& t, float idx, float idx2, const float gi[6],
                                                  float* sl) {
  {
    if (it < 8) {
      const float g1 = d1<O>(t, 0, idx), g2 = d1<O>(t, 1, idx), g3 = d1<O>(t, 2, idx);
      const float h11 = d2<O>(t, 0, idx2), h22 = d2<O>(t, 1, idx2), h33 = d2<O>(t, 2, idx2);
      const float h12 = dm<O>(t, 0, 1, idx2), h13 = dm<O>(t, 0, 2, idx2), h23 = dm<O>(t, 1, 2, idx2);
      if (it < 6) {
        sl[(S_DG + 0 * 6 + it) * kThreads] = g1;
        sl[(S_DG + 1 * 6 + it) * kThreads] = g2;
        sl[(S_DG + 2 * 6 + it) * kThreads] = g3;
        sl[(S_T1 + it) * kThreads] =
            gi[0] * h11 + gi[3] * h22 + gi[5] * h33 + 2.0f * (gi[1] * h12 + gi[2] * h13 + gi[4] * h23);
      } else {
        const int b1 = it == 6 ? S_DPHI : S_DA, b2 = it == 6 ? S_DDPHI : S_DDA;
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
    }
  }
}

// The tile copies: by TMA (tmap != null, a brick whose halo lies inside the
// box) or by the threads' own loads with periodic wrap.  Returns false (the
// same value in every thread) when a TMA copy did not complete within
// tma_wait cycles; the status word then carries kStatusTileTimeout.  A late
// copy is still waited for (tma::wait_drain), so that none is in flight when
// the tile is reused or the CTA leaves; after a copy that never lands the CTA
// issues no more.
template <int O, int MATTER>
__device__ __forceinline__ bool derivatives(const float* __restrict__ a, int N, float idx, float idx2,
                                            const float gi[6], float* sl, float* tl, const int* rowoff, int tid,
                                            int x0, int y0, int z0, int nz, int cc, const CUtensorMap* tmap,
                                            uint64_t* bar, unsigned& phase, unsigned* status, long long tma_wait) {
  using G = TileG<O>;
  const tile::Taps<G, float> t{tl, cc};
  constexpr int NIT = 8;  // fields with second derivatives; first-derivative-only fields use global taps
  const bool by_tma = tmap != nullptr;
  bool ok = true, lost = false;
  tile::Loader<G, Brick, float> ld;
  if (!by_tma) {
    ld.init(tid, z0, nz);
    ld.fetch(a + (size_t)phase1_field(0) * N, rowoff);
  }
  // one loop (and one copy of the derivative code) for both kinds of copy
#pragma unroll 1
  for (int it = 0; it < NIT; ++it) {
    if (by_tma) {
      tma::fence_proxy_async();        // this thread's shared-memory accesses come before the copy's writes
      lost = __syncthreads_or(lost);   // the previous tile has been read
      if (!lost) {
        if (tid == 0) {
          tma::arrive_expect_tx(bar, (unsigned)(G::SIZE * sizeof(float)));
          tma::load_4d(tl, tmap, z0 - G::ZO, y0 - G::R, x0 - G::R, phase1_field(it), bar);
          // the next field's tile into L2 while this one is used
          if (it + 1 < NIT) tma::prefetch_4d(tmap, z0 - G::ZO, y0 - G::R, x0 - G::R, phase1_field(it + 1));
        }
        const int w = tma::wait_drain(bar, phase, tma_wait);
        ok = ok && w == 0;
        if (w == 2) lost = true;
        else phase ^= 1u;
      }
    } else {
      __syncthreads();
      ld.store(tl);
      __syncthreads();
      if (it + 1 < NIT) ld.fetch(a + (size_t)phase1_field(it + 1) * N, rowoff);
    }
    field_derivatives<O>(it, t, idx, idx2, gi, sl);
  }
  if (by_tma) {
    ok = __syncthreads_and(ok && !lost);
    if (!ok && tid == 0) atomicOr(status, kStatusTileTimeout);
  }
  return ok;
}

// dust flux divergences from the stored FP32 flux primitives (global taps)
template <int O, class T>
__device__ __forceinline__ void flux_divergences(const T& t, const float* __restrict__ fp, int N, float idx,
                                                 float* sl) {
  const float* v1 = fp + (size_t)P_V1 * N;
  const float* v2 = fp + (size_t)P_V2 * N;
  const float* v3 = fp + (size_t)P_V3 * N;
#pragma unroll 1
  for (int m = 0; m < 4; ++m) {
    const float* u = fp + (size_t)(P_AD + m) * N;
    sl[(S_MAT + m) * kThreads] = d1p<O>(u, v1, t, 0, idx) + d1p<O>(u, v2, t, 1, idx) + d1p<O>(u, v3, t, 2, idx);
  }
}

// dalpha/dt(abar + delta) - dalpha/dt(abar) for the lapse gauges of
// BSSNGaugeHandler.cc:16-275 with a trivial FRW reference (K_FRW = 0, so the
// conformal-synchronous lapse is static); dKa = K_avg - Kbar.  The host adds
// dalpha/dt(abar), in which K_avg = Kbar.
__device__ __forceinline__ float lapse_drhs(int lapse, const Bg& bg, float alb, float dal, float alpha, float Kb,
                                            float dK, float dphi, float dKa) {
  switch (lapse) {
    case kHarmonic: return -(alb * dK + dal * (Kb + dK));
    case kConformalFLRW: return -(1.0f / 3.0f) * (alb * dKa + dal * (Kb + dKa));
    case kAnharmonic: return alpha * alpha * (dK - dKa);
    case kOnePlusLog: return -2.0f * (float)bg.gd_c * alpha * (dK - dKa);
    case kAwAGaugeWave: return -(alpha * alpha * dK + (2.0f * alb + dal) * dal * Kb);
    case kAwAShiftedWave: return -dK;
    case kDampedWave: {
      const float du = (float)bg.dw_mu_l * (12.0f * (float)bg.dw_p * dphi - log1pf(dal / alb)) - dK;
      return alpha * alpha * du + (2.0f * alb + dal) * dal * (float)bg.dw_u;
    }
    default: return 0.0f;
  }
}

// Kreiss-Oliger dissipation of one FP32 perturbation (the stencil of a
// constant is zero, so it is the dissipation of the full field): the sixth
// (order 2: fourth) undivided difference along each axis from global taps,
// times bg.ko_scale (utils/math.h:36-72, as the FP64 kernel's ko_dissipation).
template <int O>
__device__ __forceinline__ float ko_f(const float* __restrict__ f, const Taps<true>& t, float scale) {
  float s = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    auto V = [&](int n) { return __ldg(f + t.ax(a, n)); };
    if (O == 2) s += (V(-2) + V(2)) - 4.0f * (V(-1) + V(1)) + 6.0f * V(0);
    else
      s += (V(-5) + V(5)) - 10.0f * (V(-4) + V(4)) + 45.0f * (V(-3) + V(3)) - 120.0f * (V(-2) + V(2)) +
           210.0f * (V(-1) + V(1)) - 252.0f * V(0);
  }
  return scale * s;
}

// The FP32-mixed substep for the brick at brick coordinates (cx, cy, cz).
// KO: Kreiss-Oliger dissipation compiled in (orders 2 and 8 only).
template <int O, int MATTER, bool KO = false>
__device__ __forceinline__ void mixed_body(int nx, int ny, int nz, int lapse, int normalize, float idx, double dt,
                                           const Bg& bg, const Ptrs& P, int stage, int cx, int cy, int cz,
                                           const CUtensorMap* tmap, uint64_t* bar, unsigned& phase,
                                           bool& tma_ok) {
  constexpr int NFLD = MATTER == kDust ? 22 : (MATTER == kScalar ? 23 : 18);
  constexpr int R = O / 2;
  constexpr float kPif = 3.14159265358979f;
  extern __shared__ __align__(128) float smf[];  // 128-byte aligned: TMA destinations
  const int tid = threadIdx.x + kBZ * (threadIdx.y + kBY * threadIdx.z);
  float* sl = smf + tid;
  auto S = [&](int s) -> float& { return sl[s * kThreads]; };
  const int k0 = cz * kBZ + threadIdx.x;
  const int j0 = cy * kBY + threadIdx.y;
  const int i0 = cx * kBX + threadIdx.z;
  // every thread takes part in the tile copies; threads past the box edge
  // compute a valid point and leave after phase 1
  const bool live = i0 < nx && j0 < ny && k0 < nz;
  const int k = min(k0, nz - 1), j = min(j0, ny - 1), i = min(i0, nx - 1);
  const int N = nx * ny * nz;
  const int c = (i * ny + j) * nz + k;
  const float* __restrict__ a = P.in;
  auto D_ = [&](int f) { return a[(size_t)f * N + c]; };  // delta at the centre
  // warm L2 with the epilogue's FP64 register reads; those reads and the
  // epilogue writes are single-use streams (ld/st .cs), as in the FP64 kernel
#pragma unroll 1
  for (int f = 0; f < NFLD; ++f) {
    asm volatile("prefetch.global.L2 [%0];" :: "l"(P.p + (size_t)f * N + c));
    if (stage > 1) asm volatile("prefetch.global.L2 [%0];" :: "l"(P.f + (size_t)f * N + c));
  }

  float g[6], gi[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) g[q] = D_(F_G11 + q);
  inv_metricf(g, gi);

  const int x0 = cx * kBX, y0 = cy * kBY, z0 = cz * kBZ;
  const float idx2 = idx * idx;
  {
    static_assert(TileG<O>::SIZE * sizeof(float) + TileG<O>::ROWS * sizeof(int) <=
                      (size_t)kTileSlots * kThreads * sizeof(float),
                  "tile and row offsets fit the phase-2-only slots");
    using G = TileG<O>;
    float* tl = smf + kTileSlot * kThreads;
    int* rowoff = reinterpret_cast<int*>(tl + G::SIZE);
    // TMA when the brick's halo lies inside the box (no wrap)
    const bool by_tma = tmap && tma_ok && x0 >= G::R && x0 + kBX + G::R <= nx && y0 >= G::R && y0 + kBY + G::R <= ny &&
                        z0 >= G::ZO && z0 + kBZ + G::R <= nz;
    if (!by_tma) {
      tile::row_offsets<G, Brick>(x0, y0, nx, ny, nz, tid, rowoff);
      __syncthreads();  // every warp reads every row offset
    }
    // after a copy timed out the CTA copies by threads (the barrier's phase is unknown)
    tma_ok = derivatives<O, MATTER>(a, N, idx, idx2, gi, sl, tl, rowoff, tid, x0, y0, z0, nz,
                                    tile::centre<G>(threadIdx.z, threadIdx.y, threadIdx.x), by_tma ? tmap : nullptr,
                                    bar, phase, P.status, bg.tma_wait) && tma_ok;
    __syncthreads();
  }
  if (!live) return;
  {
    const bool interior =
        x0 >= R && x0 + kBX + R <= nx && y0 >= R && y0 + kBY + R <= ny && z0 >= R && z0 + kBZ + R <= nz;
    auto gpass = [&](auto t) {
      constexpr int NG = MATTER == kScalar ? 9 : 4;  // K, Gamma^i (and phi_s, Pi, psi_i)
#pragma unroll 1
      for (int q = 0; q < NG; ++q) {
        const int fld = q == 0 ? F_K : (q < 4 ? F_GAM1 + q - 1 : F_SPHI + q - 4);
        const int b = q == 0 ? S_DK : (q < 4 ? S_DGAM + 3 * (q - 1) : S_MAT + 3 * (q - 4));
        const GTaps<decltype(t)> gt{a + (size_t)fld * N, t};
        S(b + 0) = d1<O>(gt, 0, idx);
        S(b + 1) = d1<O>(gt, 1, idx);
        S(b + 2) = d1<O>(gt, 2, idx);
      }
      if (MATTER == kDust) flux_divergences<O>(t, P.fp_in, N, idx, sl);
    };
    if (interior) gpass(Taps<false>{i, j, k, nx, ny, nz, ny * nz, nz, c});
    else gpass(Taps<true>{i, j, k, nx, ny, nz, ny * nz, nz, c});
  }

  // ---- centre values: perturbations and full values -------------------------
  const float dphi0 = D_(F_PHI), dK = D_(F_K), dal = D_(F_ALPHA);
  const float phib = (float)bgv(bg.in, F_PHI), Kb = (float)bgv(bg.in, F_K), alb = (float)(1.0 + bgv(bg.in, F_ALPHA));
  const float phi = phib + dphi0, K = Kb + dK, alpha = alb + dal;
  float gm[6];
  gm[0] = g[0] + 1.0f; gm[1] = g[1]; gm[2] = g[2];
  gm[3] = g[3] + 1.0f; gm[4] = g[4]; gm[5] = g[5] + 1.0f;
  const float em4phi = __expf(-4.0f * phi);

  // ---- dust sources in perturbation form ---------------------------------------
  float rhs_m[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
  float dr = 0.f, Sdust = 0.f, rS_full = 0.f;  // delta rho, S (second order), full rho + S
  if (MATTER == kDust) {
    const float Db = (float)bgv(bg.in, F_D);
    const float D = Db + D_(F_D);
    const float Sv[3] = {D_(F_S1), D_(F_S2), D_(F_S3)};
    // lagged W, sqrt(gamma), g_ij (Dust::addBSSNSrc, dust.cc:226-264)
    float gl[6], gil[6], dphil, phil, Dl, Sl[3];
    if (stage == 1) {
#pragma unroll
      for (int m = 0; m < 6; ++m) { gl[m] = g[m]; gil[m] = gi[m]; }
      dphil = dphi0; phil = phi; Dl = D;
      Sl[0] = Sv[0]; Sl[1] = Sv[1]; Sl[2] = Sv[2];
    } else {
      const float* pv = P.prev;
#pragma unroll
      for (int m = 0; m < 6; ++m) gl[m] = __ldcs(&pv[(size_t)(F_G11 + m) * N + c]);
      inv_metricf(gl, gil);
      dphil = __ldcs(&pv[(size_t)F_PHI * N + c]);
      phil = (float)bgv(bg.prev, F_PHI) + dphil;
      Dl = (float)bgv(bg.prev, F_D) + __ldcs(&pv[(size_t)F_D * N + c]);
      Sl[0] = __ldcs(&pv[(size_t)F_S1 * N + c]); Sl[1] = __ldcs(&pv[(size_t)F_S2 * N + c]); Sl[2] = __ldcs(&pv[(size_t)F_S3 * N + c]);
    }
    const float em4l = __expf(-4.0f * phil), e6l = __expf(6.0f * phil), e4l = __expf(4.0f * phil);
    const DustF dl = dust_primf(gil, em4l, e6l, Dl, Sl);
    const float e6bl = (float)bg.e6l;  // exp(-6 phibar_lag)
    // rho = W D / sqrt(gamma); rhobar = Dbar exp(-6 phibar_lag)
    dr = e6bl * (dl.W * D * expm1f(-6.0f * dphil) + dl.Wm1 * D + D_(F_D));
    const float inv_detg = 1.0f / e6l;
    Sdust = D * inv_detg * dl.w2 / dl.W;
    rS_full = (float)(bgv(bg.in, F_D) * bg.e6l) + dr + Sdust - 2.0f * (float)bg.lambda;
    S(S_SRC + Q_R) = dr;
    S(S_SRC + Q_S) = Sdust;
#pragma unroll
    for (int m = 0; m < 3; ++m) S(S_SRC + Q_S1 + m) = Sv[m] * inv_detg;
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = I; J < 3; ++J)
        S(S_SRC + Q_STF11 + sym(I, J)) = Sv[I] * Sv[J] / (dl.W * D) * inv_detg - (1.0f / 3.0f) * (e4l * (gl[sym(I, J)] + (I == J ? 1.0f : 0.0f))) * Sdust;
    // dust RHS: divergence + momentum source with the current W, v (dust.cc:135-146)
    const DustF cur = dust_primf(gi, em4phi, __expf(6.0f * phi), D, Sv);
    const float e4 = __expf(4.0f * phi);
    rhs_m[0] = S(S_MAT + 0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const float dp = S(S_DPHI + d);
      auto DG = [&](int qq) { return S(S_DG + 6 * d + qq); };
      const float src =
          0.5f * alpha * cur.W * D * e4 *
              (cur.v[0] * cur.v[0] * (4.0f * gm[0] * dp + DG(0)) + cur.v[1] * cur.v[1] * (4.0f * gm[3] * dp + DG(3)) +
               cur.v[2] * cur.v[2] * (4.0f * gm[5] * dp + DG(5)) +
               2.0f * (cur.v[0] * cur.v[1] * (4.0f * gm[1] * dp + DG(1)) + cur.v[0] * cur.v[2] * (4.0f * gm[2] * dp + DG(2)) +
                       cur.v[1] * cur.v[2] * (4.0f * gm[4] * dp + DG(4)))) -
          cur.W * D * S(S_DA + d);
      rhs_m[1 + d] = S(S_MAT + 1 + d) + src;
    }
  } else if (MATTER == kScalar) {
    // Scalar::addBSSNSource and RKEvolvePt (scalar.cc:85-260) in perturbation
    // form about the uniform phi_s, Pi (psi_i has no background); with
    // n^mu d_mu phi = -Pi the sources are rho = Pi^2/2 + e^{-4phi} dd/2 + V,
    // S = 3 Pi^2/2 - e^{-4phi} dd/2 - 3V, S_i = Pi d_i phi_s,
    // S_ij^TF = d_i phi_s d_j phi_s - gamma_ij dd/3, dd = g^ij d_i phi_s d_j phi_s.
    const float sphib = (float)bgv(bg.in, F_SPHI), Pib = (float)bgv(bg.in, F_SPI);
    const float dsphi = D_(F_SPHI), dPi = D_(F_SPI);
    const float sphi = sphib + dsphi, Pi = Pib + dPi;
    const float psi[3] = {D_(F_SPSI1), D_(F_SPSI1 + 1), D_(F_SPSI1 + 2)};
    auto SD = [&](int m, int d) { return S(S_MAT + 3 * m + d); };  // d_d of scalar field m
    const float dd = gi[0] * SD(0, 0) * SD(0, 0) + gi[3] * SD(0, 1) * SD(0, 1) + gi[5] * SD(0, 2) * SD(0, 2) +
                     2.0f * (gi[1] * SD(0, 0) * SD(0, 1) + gi[2] * SD(0, 0) * SD(0, 2) + gi[4] * SD(0, 1) * SD(0, 2));
    const bool quad = bg.potential == kPotQuadratic;
    const float m2 = (float)(bg.pot_mass * bg.pot_mass);
    const float V = quad ? 0.5f * m2 * sphi * sphi : (float)bg.pot_const;
    const float dV = quad ? 0.5f * m2 * (2.0f * sphib + dsphi) * dsphi : 0.0f;  // V - Vbar
    const float dPi2 = (2.0f * Pib + dPi) * dPi;                              // Pi^2 - Pibar^2
    dr = 2.0f * dPi2 - 2.0f * dV;  // delta(rho + S); the dd terms cancel
    Sdust = 0.0f;
    rS_full = 2.0f * Pi * Pi - 2.0f * V;
    S(S_SRC + Q_R) = 0.5f * dPi2 + 0.5f * em4phi * dd + dV;
#pragma unroll
    for (int m = 0; m < 3; ++m) S(S_SRC + Q_S1 + m) = Pi * SD(0, m);
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = I; J < 3; ++J) S(S_SRC + Q_STF11 + sym(I, J)) = SD(0, I) * SD(0, J) - gm[sym(I, J)] * (1.0f / 3.0f) * dd;
    float inner = 0.0f;
#pragma unroll
    for (int X = 0; X < 3; ++X)
#pragma unroll
      for (int Y = 0; Y < 3; ++Y) inner += gi[sym(X, Y)] * (alpha * SD(2 + Y, X) + psi[X] * S(S_DA + Y));
    float gtpsi = 0.0f;
#pragma unroll
    for (int I = 0; I < 3; ++I)
      gtpsi += (D_(F_GAM1 + I) - 2.0f * (gi[sym(I, 0)] * S(S_DPHI + 0) + gi[sym(I, 1)] * S(S_DPHI + 1) +
                                         gi[sym(I, 2)] * S(S_DPHI + 2))) * psi[I];
    // alpha (K Pi + V') - alphabar (Kbar Pibar + V'bar), expanded
    const float ddV = quad ? m2 * dsphi : 0.0f;
    const float X = K * Pi + (quad ? m2 * sphi : 0.0f);
    const float dX = Kb * dPi + dK * Pi + ddV;
    rhs_m[0] = -(alb * dPi + dal * Pi);
    rhs_m[1] = -em4phi * inner + alpha * gtpsi * em4phi + (alb * dX + dal * X);
#pragma unroll
    for (int m = 0; m < 3; ++m) rhs_m[2 + m] = -alpha * SD(1, m) - Pi * S(S_DA + m);
  } else {
#pragma unroll
    for (int m = 0; m < Q_N; ++m) S(S_SRC + m) = 0.f;
  }

  // ---- Christoffels, D_iD_j phi, (D_iD_j alpha)^TF, Ricci (first order) ---------
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = 0; J < 3; ++J)
#pragma unroll
      for (int Kx = J; Kx < 3; ++Kx) {
        auto dg = [&](int d, int qq) { return S(S_DG + 6 * d + qq); };
        S(S_G + 6 * I + sym(J, Kx)) =
            0.5f * (gi[sym(I, 0)] * (dg(J, sym(Kx, 0)) + dg(Kx, sym(J, 0)) - dg(0, sym(J, Kx))) +
                    gi[sym(I, 1)] * (dg(J, sym(Kx, 1)) + dg(Kx, sym(J, 1)) - dg(1, sym(J, Kx))) +
                    gi[sym(I, 2)] * (dg(J, sym(Kx, 2)) + dg(Kx, sym(J, 2)) - dg(2, sym(J, Kx))));
      }
  {
    float GLv[3][6];
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = 0; J < 3; ++J)
#pragma unroll
        for (int Kx = J; Kx < 3; ++Kx) {
          auto dg = [&](int d, int qq) { return S(S_DG + 6 * d + qq); };
          GLv[I][sym(J, Kx)] = 0.5f * (dg(J, sym(Kx, I)) + dg(Kx, sym(J, I)) - dg(I, sym(J, Kx)));
        }
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int qq = 0; qq < 6; ++qq) S(S_DG + 6 * I + qq) = GLv[I][qq];
  }
  auto G = [&](int I, int qq) { return S(S_G + 6 * I + qq); };
  auto GL = [&](int I, int qq) { return S(S_DG + 6 * I + qq); };
  float Gd[3];
#pragma unroll
  for (int I = 0; I < 3; ++I)
    Gd[I] = G(I, 0) * gi[0] + G(I, 3) * gi[3] + G(I, 5) * gi[5] + 2.0f * (G(I, 1) * gi[1] + G(I, 2) * gi[2] + G(I, 4) * gi[4]);
  float dphi[3], da[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { dphi[d] = S(S_DPHI + d); da[d] = S(S_DA + d); }
  float DDa[6], gld[3];
#pragma unroll
  for (int I = 0; I < 3; ++I) gld[I] = gi[sym(I, 0)] * dphi[0] + gi[sym(I, 1)] * dphi[1] + gi[sym(I, 2)] * dphi[2];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int qq = sym(I, J);
      S(S_DDPHI + qq) = S(S_DDPHI + qq) - (G(0, qq) * dphi[0] + G(1, qq) * dphi[1] + G(2, qq) * dphi[2]);
      float t = 0.f;
#pragma unroll
      for (int L = 0; L < 3; ++L)
        t += (G(L, qq) + 2.0f * ((L == I ? dphi[J] : 0.f) + (L == J ? dphi[I] : 0.f) - gm[qq] * gld[L])) * da[L];
      DDa[qq] = S(S_DDA + qq) - t;
    }
  float DDaTR = gi[0] * DDa[0] + gi[3] * DDa[3] + gi[5] * DDa[5] + 2.0f * (gi[1] * DDa[1] + gi[2] * DDa[2] + gi[4] * DDa[4]);
#pragma unroll
  for (int m = 0; m < 6; ++m) S(S_DDA + m) = DDa[m] - (1.0f / 3.0f) * gm[m] * DDaTR;
  DDaTR *= em4phi;
  auto DDphi = [&](int qq) { return S(S_DDPHI + qq); };
  const float expression =
      gi[0] * (DDphi(0) + 2.0f * dphi[0] * dphi[0]) + gi[3] * (DDphi(3) + 2.0f * dphi[1] * dphi[1]) +
      gi[5] * (DDphi(5) + 2.0f * dphi[2] * dphi[2]) +
      2.0f * (gi[1] * (DDphi(1) + 2.0f * dphi[0] * dphi[1]) + gi[2] * (DDphi(2) + 2.0f * dphi[0] * dphi[2]) +
              gi[4] * (DDphi(4) + 2.0f * dphi[1] * dphi[2]));
  // Ricci term 4 (bssn_macros.h:248-277), sum_{K,L,M} g^{LM} (G^K_{LI} G_{J,KM}
  // + G^K_{LJ} G_{I,KM} + (G^K_{IM} G_{K,LJ} + G^K_{JM} G_{K,LI}) / 2), with the
  // L index raised first: H^K_{MX} = sum_L g^{LM} G^K_{LX}, so that
  // t4_IJ = sum_{K,M} (H^K_{MI} G_{J,KM} + H^K_{MJ} G_{I,KM})
  //       + sum_{K,L} (H^K_{LI} G_{K,LJ} + H^K_{LJ} G_{K,LI}) / 2
  // (about a third of the multiplications; the FP64 kernel keeps the
  // reference's order).
  float t4[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
  for (int Kx = 0; Kx < 3; ++Kx) {
    float H[3][3];  // H[M][X]
#pragma unroll
    for (int M = 0; M < 3; ++M)
#pragma unroll
      for (int X = 0; X < 3; ++X)
        H[M][X] = gi[sym(0, M)] * G(Kx, sym(0, X)) + gi[sym(1, M)] * G(Kx, sym(1, X)) + gi[sym(2, M)] * G(Kx, sym(2, X));
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = I; J < 3; ++J) {
        float u = 0.f, w = 0.f;
#pragma unroll
        for (int M = 0; M < 3; ++M) {
          u += H[M][I] * GL(J, sym(Kx, M)) + H[M][J] * GL(I, sym(Kx, M));
          w += H[M][I] * GL(Kx, sym(M, J)) + H[M][J] * GL(Kx, sym(M, I));
        }
        t4[sym(I, J)] += u + 0.5f * w;
      }
  }
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int ij = sym(I, J);
      auto dGam = [&](int Jx, int Kx) { return S(S_DGAM + 3 * Kx + Jx); };
      const float t2 = gm[sym(0, I)] * dGam(J, 0) + gm[sym(1, I)] * dGam(J, 1) + gm[sym(2, I)] * dGam(J, 2) +
                       gm[sym(0, J)] * dGam(I, 0) + gm[sym(1, J)] * dGam(I, 1) + gm[sym(2, J)] * dGam(I, 2);
      const float t3 = Gd[0] * (GL(I, sym(J, 0)) + GL(J, sym(I, 0))) + Gd[1] * (GL(I, sym(J, 1)) + GL(J, sym(I, 1))) +
                       Gd[2] * (GL(I, sym(J, 2)) + GL(J, sym(I, 2)));
      const float U = -0.5f * S(S_T1 + ij) + 0.5f * t2 + 0.5f * t3 + t4[ij];
      S(S_T1 + ij) = U - 2.0f * (DDphi(ij) - 2.0f * dphi[I] * dphi[J] + gm[ij] * expression);
    }
  auto Ric = [&](int qq) { return S(S_T1 + qq); };
  const float ricci = em4phi * (Ric(0) * gi[0] + Ric(3) * gi[3] + Ric(5) * gi[5] + 2.0f * (Ric(1) * gi[1] + Ric(2) * gi[2] + Ric(4) * gi[4]));
  const float e4phi = __expf(4.0f * phi);
  float A[6], Ac[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) A[q] = D_(F_A11 + q);
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      float t = 0.f;
#pragma unroll
      for (int X = 0; X < 3; ++X)
#pragma unroll
        for (int Y = 0; Y < 3; ++Y) t += gi[sym(I, X)] * gi[sym(J, Y)] * A[sym(X, Y)];
      Ac[sym(I, J)] = t;
    }
  const float AijAij = Ac[0] * A[0] + Ac[3] * A[3] + Ac[5] * A[5] + 2.0f * (Ac[1] * A[1] + Ac[2] * A[2] + Ac[4] * A[4]);

  // ---- perturbation right-hand sides + FP64 register update ----------------------
  double outv[NFLD];
  const Taps<true> tko{i, j, k, nx, ny, nz, ny * nz, nz, c};
  // the RK4 register update (RK4Register.h:180-230) with the substep's
  // divisors chosen once, one code path per field (as the FP64 kernel's)
  const double fdiv = stage == 1 ? 6.0 : 3.0, odiv = stage == 3 ? 1.0 : 2.0;
  auto finalize = [&](int fld, float drhs) {
    if constexpr (KO) {
      if (fld < F_D) drhs -= ko_f<O>(a + (size_t)fld * N, tko, (float)bg.ko_scale);
    }
    const double cv = bgv(bg.rhs, fld) + (double)drhs;
    const double pv = __ldcs(&P.p[(size_t)fld * N + c]);
    const double fv = stage == 1 ? 0.0 : __ldcs(&P.f[(size_t)fld * N + c]);
    const double t = dt * cv;
    double o;
    if (stage == 4) {
      o = fv + (t / 6.0 + pv);
      __stcs(&P.newp[(size_t)fld * N + c], o);
    } else {
      __stcs(&P.f[(size_t)fld * N + c], fv + t / fdiv);
      o = pv + t / odiv;
    }
    outv[fld] = o;
  };
  // constraint damping (bssn.cc:748-820): H in perturbation form,
  // H - Hbar = -(e^{5 phibar}/8) (expm1(5 dphi) Hcbar + e^{5 dphi} dHc) with
  // dHc = ricci + 2/3 (2 Kbar + dK) dK - A_ij A^ij - 16 pi drho
  float Hd = 0.f, dH = 0.f, dHc = 0.f;
  if (bg.damping) {
    dHc = ricci + (2.0f / 3.0f) * (2.0f * Kb + dK) * dK - AijAij - 16.0f * kPif * S(S_SRC + Q_R);
    dH = -(float)(bg.e5phib * (1.0 / 8.0)) * (expm1f(5.0f * dphi0) * (float)bg.Hcbar + __expf(5.0f * dphi0) * dHc);
    Hd = (float)bg.Hbar + dH;
  }
  const float adt = (float)bg.a_adj_dt;
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    float v = -2.0f * alpha * A[m];
    if (bg.damping) v += 0.5f * adt * Hd * g[m];
    finalize(F_G11 + m, v);
  }
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int qq = sym(I, J);
      float aa = 0.f;
#pragma unroll
      for (int X = 0; X < 3; ++X)
#pragma unroll
        for (int Y = 0; Y < 3; ++Y) aa += gi[sym(X, Y)] * A[sym(X, I)] * A[sym(Y, J)];
      const float RTF = Ric(qq) - (1.0f / 3.0f) * e4phi * gm[qq] * ricci;
      float v = em4phi * (alpha * (RTF - 8.0f * kPif * S(S_SRC + Q_STF11 + qq)) - S(S_DDA + qq)) +
                alpha * (K * A[qq] - 2.0f * aa);
      if (bg.damping) v -= adt * A[qq] * Hd;
      finalize(F_A11 + qq, v);
    }
#pragma unroll
  for (int I = 0; I < 3; ++I) {
    const float so = G(I, 0) * Ac[0] + G(I, 3) * Ac[3] + G(I, 5) * Ac[5] + 2.0f * (G(I, 1) * Ac[1] + G(I, 2) * Ac[2] + G(I, 4) * Ac[4]) +
                     6.0f * (Ac[sym(I, 0)] * dphi[0] + Ac[sym(I, 1)] * dphi[1] + Ac[sym(I, 2)] * dphi[2]);
    const float gdK = gi[sym(I, 0)] * S(S_DK + 0) + gi[sym(I, 1)] * S(S_DK + 1) + gi[sym(I, 2)] * S(S_DK + 2);
    const float gS = gi[sym(I, 0)] * S(S_SRC + Q_S1) + gi[sym(I, 1)] * S(S_SRC + Q_S2) + gi[sym(I, 2)] * S(S_SRC + Q_S3);
    finalize(F_GAM1 + I, -2.0f * (Ac[sym(I, 0)] * da[0] + Ac[sym(I, 1)] * da[1] + Ac[sym(I, 2)] * da[2]) +
                             2.0f * alpha * (so - (2.0f / 3.0f) * gdK - 8.0f * kPif * gS));
  }
  // zeroth-order equations in explicit perturbation form
  const float dRK = -DDaTR + (alb * (2.0f * Kb + dK) * dK + dal * K * K) * (1.0f / 3.0f) + alpha * AijAij +
                    4.0f * kPif * (alb * (dr + Sdust) + dal * rS_full);
  finalize(F_K, bg.damping ? dRK + (float)bg.k_damp8 * dHc : dRK);
  finalize(F_PHI, bg.damping ? -(1.0f / 6.0f) * (alb * dK + dal * K) + 0.1f * adt * dH
                             : -(1.0f / 6.0f) * (alb * dK + dal * K));
  finalize(F_ALPHA, lapse_drhs(lapse, bg, alb, dal, alpha, Kb, dK, dphi0, P.kavg ? (float)__ldg(P.kavg) : 0.0f));
  if (MATTER == kDust) {
#pragma unroll
    for (int m = 0; m < 4; ++m) finalize(F_D + m, rhs_m[m]);
  } else if (MATTER == kScalar) {
#pragma unroll
    for (int m = 0; m < 5; ++m) finalize(F_SPHI + m, rhs_m[m]);
  }

  if (stage == 4) {
    bool bad_any = false;
#pragma unroll
    for (int f = 0; f < NFLD; ++f) bad_any |= !isfinite(outv[f]);
    if (bad_any) {
      if (isnan(outv[F_PHI])) atomicOr(P.status, 1u);
      atomicOr(P.status, 2u);
    }
    // the next step's first-substep input is the normalised new state (bssn.cc:224-225)
    if (normalize) {
    double gn[6], An[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) { gn[m] = outv[F_G11 + m]; An[m] = outv[F_A11 + m]; }
    {
      double omd = -1.0 * (gn[0] + gn[3] + gn[5] - gn[1] * gn[1] - gn[2] * gn[2] - gn[4] * gn[4] + gn[0] * gn[3] +
                           gn[0] * gn[5] + gn[3] * gn[5] - gn[4] * gn[4] * gn[0] - gn[2] * gn[2] * gn[3] -
                           gn[1] * gn[1] * gn[5] + 2.0 * gn[1] * gn[2] * gn[4] + gn[0] * gn[3] * gn[5]);
      const double tt = -1.0 * expm1(log1p(-1.0 * omd) / 3.0);
      const double inv = 1.0 / (1.0 - tt);
      gn[0] = (gn[0] + tt) * inv; gn[3] = (gn[3] + tt) * inv; gn[5] = (gn[5] + tt) * inv;
      gn[1] *= inv; gn[2] *= inv; gn[4] *= inv;
      double gin[6];
      gin[0] = 1.0 + gn[3] + gn[5] - gn[4] * gn[4] + gn[3] * gn[5];
      gin[3] = 1.0 + gn[0] + gn[5] - gn[2] * gn[2] + gn[0] * gn[5];
      gin[5] = 1.0 + gn[0] + gn[3] - gn[1] * gn[1] + gn[0] * gn[3];
      gin[1] = gn[2] * gn[4] - gn[1] * (1.0 + gn[5]);
      gin[2] = gn[1] * gn[4] - gn[2] * (1.0 + gn[3]);
      gin[4] = gn[1] * gn[2] - gn[4] * (1.0 + gn[0]);
      const double trA = gin[0] * An[0] + gin[3] * An[3] + gin[5] * An[5] + 2.0 * (gin[1] * An[1] + gin[2] * An[2] + gin[4] * An[4]);
      An[0] = (An[0] - 1.0 / 3.0 * (1.0 + gn[0]) * trA) * inv;
      An[3] = (An[3] - 1.0 / 3.0 * (1.0 + gn[3]) * trA) * inv;
      An[5] = (An[5] - 1.0 / 3.0 * (1.0 + gn[5]) * trA) * inv;
      An[1] = (An[1] - 1.0 / 3.0 * gn[1] * trA) * inv;
      An[2] = (An[2] - 1.0 / 3.0 * gn[2] * trA) * inv;
      An[4] = (An[4] - 1.0 / 3.0 * gn[4] * trA) * inv;
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) { outv[F_G11 + m] = gn[m]; outv[F_A11 + m] = An[m]; }
    }
  }
#pragma unroll
  for (int f = 0; f < NFLD; ++f) __stcs(&P.out[(size_t)f * N + c], (float)(outv[f] - bgv(bg.out, f)));
  if (MATTER == kDust) {
    float go[6], gio[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) go[m] = (float)outv[F_G11 + m];
    inv_metricf(go, gio);
    const float So[3] = {(float)outv[F_S1], (float)outv[F_S2], (float)outv[F_S3]};
    const float phio = (float)outv[F_PHI];
    const float Do = (float)outv[F_D];
    const DustF dp = dust_primf(gio, __expf(-4.0f * phio), __expf(6.0f * phio), Do, So);
    const float alo = (float)(outv[F_ALPHA] + 1.0);
    float* fo = P.fp_out;
    __stcs(&fo[(size_t)P_AD * N + c], alo * Do);
#pragma unroll
    for (int m = 0; m < 3; ++m) __stcs(&fo[(size_t)(P_AS1 + m) * N + c], alo * So[m]);
#pragma unroll
    for (int m = 0; m < 3; ++m) __stcs(&fo[(size_t)(P_V1 + m) * N + c], dp.v[m]);
  }
}

// the TMA barrier of a CTA: initialised once, before any copy
__device__ __forceinline__ void init_tile_barrier(uint64_t* bar, bool use) {
  if (use && threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
    tma::bar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
}

// One box: one CTA per updated brick.  tmap: the TMA map of this substep's
// input (use_tma = 0: every tile is copied by the threads).
template <int O, int MATTER, bool KO>
__global__ void __launch_bounds__(kThreads, 4)
mixed_kernel(int nx, int ny, int nz, int lapse, int normalize, float idx, double dt, Bg bg, Ptrs P, int stage,
             const __grid_constant__ CUtensorMap tmap, int use_tma, int bx0) {
  __shared__ __align__(8) uint64_t bar;
  init_tile_barrier(&bar, use_tma != 0);
  unsigned phase = 0;
  bool tma_ok = true;
  // bx0: first x brick (x-slab boxes skip their ghost planes)
  mixed_body<O, MATTER, KO>(nx, ny, nz, lapse, normalize, idx, dt, bg, P, stage, blockIdx.z + bx0, blockIdx.y, blockIdx.x,
                        use_tma ? &tmap : nullptr, &bar, phase, tma_ok);
}

// Register roles of substep n (X/Y ping-pong, as in the single-box launcher).
__device__ __forceinline__ Ptrs group_ptrs(const GroupBox& b, int stage) {
  Ptrs p{};
  p.p = b.P;
  p.f = b.F;
  p.newp = b.P;
  p.status = b.status;
  p.kavg = b.kavg;
  switch (stage) {
    case 1: p.in = b.X; p.prev = nullptr; p.out = b.Y; p.fp_in = b.FP0; p.fp_out = b.FP1; break;
    case 2: p.in = b.Y; p.prev = b.X; p.out = b.X; p.fp_in = b.FP1; p.fp_out = b.FP0; break;
    case 3: p.in = b.X; p.prev = b.Y; p.out = b.Y; p.fp_in = b.FP0; p.fp_out = b.FP1; break;
    default: p.in = b.Y; p.prev = b.X; p.out = b.X; p.fp_in = b.FP1; p.fp_out = b.FP0; break;
  }
  return p;
}

// A group of mixed boxes, one launch per substep over the work list of all
// their bricks (see the FP64 stage_group_kernel).
template <int O, int MATTER>
__global__ void __launch_bounds__(kThreads, 4)
mixed_group_kernel(const GroupBox* __restrict__ boxes, GroupBg gb, int stage) {
  __shared__ GroupBox sb;
  __shared__ Ptrs sp;
  __shared__ Bg sbg;
  __shared__ const CUtensorMap* stm;
  __shared__ __align__(8) uint64_t bar;
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0;
  init_tile_barrier(&bar, true);
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
    }
    __syncthreads();
    const int l = w - sb.first;
    const int cz = l % sb.nbz, cy = (l / sb.nbz) % sb.nby, cx = l / (sb.nbz * sb.nby);
    mixed_body<O, MATTER>(sb.nx, sb.ny, sb.nz, sb.lapse, sb.normalize, sb.idx, sb.dt, sbg, sp, stage, cx, cy, cz, stm,
                          &bar, phase, tma_ok);
  }
}

// first-substep input of a step: normalised _p minus the background, FP32;
// dust flux primitives of that state
template <int MATTER>
__global__ void __launch_bounds__(kThreads) mixed_init_kernel(int nx, int ny, int nz, int normalize, Bg bg,
                                                              const double* Pp, float* X, float* FP0) {
  constexpr int NFLD = MATTER == kDust ? 22 : (MATTER == kScalar ? 23 : 18);
  const int k = blockIdx.x * kBZ + threadIdx.x;
  const int j = blockIdx.y * kBY + threadIdx.y;
  const int i = blockIdx.z * kBX + threadIdx.z;
  if (i >= nx || j >= ny || k >= nz) return;
  const int N = nx * ny * nz;
  const int c = (i * ny + j) * nz + k;
  double v[NFLD];
#pragma unroll
  for (int f = 0; f < NFLD; ++f) v[f] = Pp[(size_t)f * N + c];
  double gn[6], An[6];
#pragma unroll
  for (int m = 0; m < 6; ++m) { gn[m] = v[F_G11 + m]; An[m] = v[F_A11 + m]; }
  if (normalize) {
    double omd = -1.0 * (gn[0] + gn[3] + gn[5] - gn[1] * gn[1] - gn[2] * gn[2] - gn[4] * gn[4] + gn[0] * gn[3] +
                         gn[0] * gn[5] + gn[3] * gn[5] - gn[4] * gn[4] * gn[0] - gn[2] * gn[2] * gn[3] -
                         gn[1] * gn[1] * gn[5] + 2.0 * gn[1] * gn[2] * gn[4] + gn[0] * gn[3] * gn[5]);
    const double tt = -1.0 * expm1(log1p(-1.0 * omd) / 3.0);
    const double inv = 1.0 / (1.0 - tt);
    gn[0] = (gn[0] + tt) * inv; gn[3] = (gn[3] + tt) * inv; gn[5] = (gn[5] + tt) * inv;
    gn[1] *= inv; gn[2] *= inv; gn[4] *= inv;
    double gin[6];
    gin[0] = 1.0 + gn[3] + gn[5] - gn[4] * gn[4] + gn[3] * gn[5];
    gin[3] = 1.0 + gn[0] + gn[5] - gn[2] * gn[2] + gn[0] * gn[5];
    gin[5] = 1.0 + gn[0] + gn[3] - gn[1] * gn[1] + gn[0] * gn[3];
    gin[1] = gn[2] * gn[4] - gn[1] * (1.0 + gn[5]);
    gin[2] = gn[1] * gn[4] - gn[2] * (1.0 + gn[3]);
    gin[4] = gn[1] * gn[2] - gn[4] * (1.0 + gn[0]);
    const double trA = gin[0] * An[0] + gin[3] * An[3] + gin[5] * An[5] + 2.0 * (gin[1] * An[1] + gin[2] * An[2] + gin[4] * An[4]);
    An[0] = (An[0] - 1.0 / 3.0 * (1.0 + gn[0]) * trA) * inv;
    An[3] = (An[3] - 1.0 / 3.0 * (1.0 + gn[3]) * trA) * inv;
    An[5] = (An[5] - 1.0 / 3.0 * (1.0 + gn[5]) * trA) * inv;
    An[1] = (An[1] - 1.0 / 3.0 * gn[1] * trA) * inv;
    An[2] = (An[2] - 1.0 / 3.0 * gn[2] * trA) * inv;
    An[4] = (An[4] - 1.0 / 3.0 * gn[4] * trA) * inv;
  }
#pragma unroll
  for (int m = 0; m < 6; ++m) { v[F_G11 + m] = gn[m]; v[F_A11 + m] = An[m]; }
#pragma unroll
  for (int f = 0; f < NFLD; ++f) X[(size_t)f * N + c] = (float)(v[f] - bgv(bg.in, f));
  if (MATTER == kDust) {
    float go[6], gio[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) go[m] = (float)v[F_G11 + m];
    inv_metricf(go, gio);
    const float So[3] = {(float)v[F_S1], (float)v[F_S2], (float)v[F_S3]};
    const float phio = (float)v[F_PHI];
    const DustF dp = dust_primf(gio, __expf(-4.0f * phio), __expf(6.0f * phio), (float)v[F_D], So);
    const float alo = (float)(v[F_ALPHA] + 1.0);
    FP0[(size_t)P_AD * N + c] = alo * (float)v[F_D];
#pragma unroll
    for (int m = 0; m < 3; ++m) FP0[(size_t)(P_AS1 + m) * N + c] = alo * So[m];
#pragma unroll
    for (int m = 0; m < 3; ++m) FP0[(size_t)(P_V1 + m) * N + c] = dp.v[m];
  }
}

}  // namespace mixed
}  // namespace cg
