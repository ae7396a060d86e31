// cg_point.cuh -- per-grid-point BSSN(+dust/+scalar) arithmetic, device side.
//
//
// This is the arithmetic of BSSN::set_bd_values and the ev_* evolution
// functions (components/bssn/bssn.cc:361-831, bssn_macros.h:221-385), the
// dust source and flux terms (components/dust_fluid/dust.cc:109-264) and the
// scalar-field terms (components/scalar/scalar.cc:132-260), evaluated for one
// point by one thread.  Operand order inside every expression follows the
// reference so that, compiled without FMA contraction, the FP64 kernel
// reproduces the reference's rounding (with e^x, expm1 and log1p correctly
// rounded, as an exact C library returns them).
//
// Finite differences use the reference's centred stencils of order 2/4/6/8
// (utils/math.h:74-1085): first derivatives on the 2r axis points, second
// derivatives on the 2r+1 axis points and mixed derivatives on the 4r
// in-plane diagonal points (i+-n, j+-n); r = ORDER/2.
//
// The functions live in namespace cg::CG_VARIANT_NS so that the translation
// units compiled with and without FMA contraction never share a symbol.
#pragma once

#include "cg_crmath.h"
#include "cg_types.h"

#ifndef CG_VARIANT_NS
#error "CG_VARIANT_NS must be defined (exact or fast)"
#endif

namespace cg {
namespace CG_VARIANT_NS {

// The parity build (compiled with -DCG_REFERENCE_ORDER=1 and without FMA
// contraction) evaluates every expression in the reference's operand order
// and takes e^x, expm1 and log1p correctly rounded (cg_crmath.h), the values
// any exact C library returns; the FMA build uses CUDA's functions.
#ifndef CG_REFERENCE_ORDER
#define CG_REFERENCE_ORDER 0
#endif
constexpr bool kReferenceOrder = CG_REFERENCE_ORDER != 0;

// e^x of N arguments at once (one copy of the accurate phase per batch)
template <int N>
__device__ __forceinline__ void xexp_n(const double (&x)[N], double (&y)[N]) {
  if constexpr (kReferenceOrder) {
    crm::exp_n<N>(x, y);
  } else {
#pragma unroll
    for (int n = 0; n < N; ++n) y[n] = ::exp(x[n]);
  }
}
__device__ __forceinline__ double xexp(double x) {
  if constexpr (kReferenceOrder) return crm::exp(x);
  else return ::exp(x);
}
__device__ __forceinline__ double xexpm1(double x) {
  if constexpr (kReferenceOrder) return crm::expm1(x);
  else return ::expm1(x);
}
__device__ __forceinline__ double xlog1p(double x) {
  if constexpr (kReferenceOrder) return crm::log1p(x);
  else return ::log1p(x);
}

__device__ __forceinline__ int wrap(int v, int n) {
  v = v < 0 ? v + n : v;
  return v >= n ? v - n : v;
}

// Periodic neighbourhood of one grid point; linear index within one field.
struct Site {
  int i, j, k, nx, ny, nz;
  __device__ __forceinline__ int at(int di, int dj, int dk) const {
    return (wrap(i + di, nx) * ny + wrap(j + dj, ny)) * nz + wrap(k + dk, nz);
  }
  __device__ __forceinline__ int ax(int a, int n) const {
    return at(a == 0 ? n : 0, a == 1 ? n : 0, a == 2 ? n : 0);
  }
  __device__ __forceinline__ int pl(int a, int n, int b, int m) const {
    int o[3] = {0, 0, 0};
    o[a] += n;
    o[b] += m;
    return at(o[0], o[1], o[2]);
  }
};

template <typename T>
__device__ __forceinline__ T ld(const T* __restrict__ p, int idx) {
  return __ldg(p + idx);
}

// x/dx, bit-identical to the reference's division (a multiply when dx is a
// power of two, where both round identically).
__device__ __forceinline__ double divdx(double x, const Physics& ph) {
  return ph.dx_pow2 ? x * ph.inv_dx : x / ph.dx;
}

// First derivative along axis a: utils/math.h:74-100, 231-263, 412-450, 554-586.
template <int O>
__device__ __forceinline__ double der1(const double* __restrict__ f, const Site& s, int a,
                                       const Physics& ph) {
  auto V = [&](int n) { return ld(f, s.ax(a, n)); };
  double t;
  if (O == 2) {
    t = (-1.0 / 2.0 * V(-1) + 1.0 / 2.0 * V(1));
  } else if (O == 4) {
    t = (+1.0 / 12.0 * V(-2) - 2.0 / 3.0 * V(-1) + 2.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2));
  } else if (O == 6) {
    t = (-1.0 / 60.0 * V(-3) + 3.0 / 20.0 * V(-2) - 3.0 / 4.0 * V(-1) + 3.0 / 4.0 * V(1) -
         3.0 / 20.0 * V(2) + 1.0 / 60.0 * V(3));
  } else {
    t = ((1.0 / 280.0 * V(-4) - 1.0 / 280.0 * V(4)) - (4.0 / 105.0 * V(-3) - 4.0 / 105.0 * V(3)) +
         (1.0 / 5.0 * V(-2) - 1.0 / 5.0 * V(2)) - (4.0 / 5.0 * V(-1) - 4.0 / 5.0 * V(1)));
  }
  return divdx(t, ph);
}

// Second derivative along axis a: utils/math.h:857-885, 958-993, 995-1036, 1038-1085.
template <int O>
__device__ __forceinline__ double der2(const double* __restrict__ f, const Site& s, int a,
                                       const Physics& ph) {
  auto V = [&](int n) { return ld(f, s.ax(a, n)); };
  double t;
  if (O == 2) {
    t = (V(-1) - 2.0 * V(0) + V(1));
  } else if (O == 4) {
    t = (-1.0 / 12.0 * V(-2) + 4.0 / 3.0 * V(-1) - 5.0 / 2.0 * V(0) + 4.0 / 3.0 * V(1) -
         1.0 / 12.0 * V(2));
  } else if (O == 6) {
    t = (1.0 / 90.0 * V(-3) - 3.0 / 20.0 * V(-2) + 3.0 / 2.0 * V(-1) - 49.0 / 18.0 * V(0) +
         3.0 / 2.0 * V(1) - 3.0 / 20.0 * V(2) + 1.0 / 90.0 * V(3));
  } else {
    t = (-1.0 / 560.0 * V(-4) + 8.0 / 315.0 * V(-3) - 1.0 / 5.0 * V(-2) + 8.0 / 5.0 * V(-1) -
         205.0 / 72.0 * V(0) + 8.0 / 5.0 * V(1) - 1.0 / 5.0 * V(2) + 8.0 / 315.0 * V(3) -
         1.0 / 560.0 * V(4));
  }
  return divdx(divdx(t, ph), ph);
}

// Mixed second derivative on axes a < b: utils/math.h:676-855.
template <int O>
__device__ __forceinline__ double derm(const double* __restrict__ f, const Site& s, int a, int b,
                                       const Physics& ph) {
  auto P = [&](int n) {
    return -ld(f, s.pl(a, n, b, -n)) + ld(f, s.pl(a, n, b, n)) + ld(f, s.pl(a, -n, b, -n)) -
           ld(f, s.pl(a, -n, b, n));
  };
  double t;
  if (O == 2) {
    t = P(1) / 4.0;
  } else if (O == 4) {
    t = (P(1) - 1.0 / 16.0 * P(2)) / 3.0;
  } else if (O == 6) {
    t = (135.0 * P(1) - 27.0 / 2.0 * P(2) + P(3)) / 360.0;
  } else {
    t = (2.0 / 5.0 * P(1) - 1.0 / 20.0 * P(2) + 2.0 / 315.0 * P(3) - 1.0 / 2240.0 * P(4));
  }
  return divdx(divdx(t, ph), ph);
}

// utils/math.h:1319-1330
template <int O>
__device__ __forceinline__ double der2ab(const double* __restrict__ f, const Site& s, int a, int b,
                                        const Physics& ph) {
  if (a == b) return der2<O>(f, s, a, ph);
  return a < b ? derm<O>(f, s, a, b, ph) : derm<O>(f, s, b, a, ph);
}

// Inverse conformal metric assuming unit determinant, bssn.cc:447-455.
__device__ __forceinline__ void inv_metric(const double g[6], double gi[6]) {
  gi[0] = 1.0 + g[3] + g[5] - g[4] * g[4] + g[3] * g[5];
  gi[3] = 1.0 + g[0] + g[5] - g[2] * g[2] + g[0] * g[5];
  gi[5] = 1.0 + g[0] + g[3] - g[1] * g[1] + g[0] * g[3];
  gi[1] = g[2] * g[4] - g[1] * (1.0 + g[5]);
  gi[2] = g[1] * g[4] - g[2] * (1.0 + g[3]);
  gi[4] = g[1] * g[2] - g[4] * (1.0 + g[0]);
}

// BSSN::set_DIFFgamma_Aij_norm for one point, bssn.cc:69-118.
__device__ __forceinline__ void normalize_point(double g[6], double A[6]) {
  double omd = -1.0 * (g[0] + g[3] + g[5] - g[1] * g[1] - g[2] * g[2] - g[4] * g[4] + g[0] * g[3] +
                       g[0] * g[5] + g[3] * g[5] - g[4] * g[4] * g[0] - g[2] * g[2] * g[3] -
                       g[1] * g[1] * g[5] + 2.0 * g[1] * g[2] * g[4] + g[0] * g[3] * g[5]);
  double t = -1.0 * xexpm1(xlog1p(-1.0 * omd) / 3.0);
  g[0] = (g[0] + t) / (1.0 - t);
  g[3] = (g[3] + t) / (1.0 - t);
  g[5] = (g[5] + t) / (1.0 - t);
  g[1] = (g[1]) / (1.0 - t);
  g[2] = (g[2]) / (1.0 - t);
  g[4] = (g[4]) / (1.0 - t);
  double gi[6];
  inv_metric(g, gi);
  double trA = gi[0] * A[0] + gi[3] * A[3] + gi[5] * A[5] + 2.0 * (gi[1] * A[1] + gi[2] * A[2] + gi[4] * A[4]);
  A[0] = (A[0] - 1.0 / 3.0 * (1.0 + g[0]) * trA) / (1.0 - t);
  A[3] = (A[3] - 1.0 / 3.0 * (1.0 + g[3]) * trA) / (1.0 - t);
  A[5] = (A[5] - 1.0 / 3.0 * (1.0 + g[5]) * trA) / (1.0 - t);
  A[1] = (A[1] - 1.0 / 3.0 * g[1] * trA) / (1.0 - t);
  A[2] = (A[2] - 1.0 / 3.0 * g[2] * trA) / (1.0 - t);
  A[4] = (A[4] - 1.0 / 3.0 * g[4] * trA) / (1.0 - t);
}

// Dust primitives of one point (Dust::getDustData, dust.cc:177-200, and the
// products of populateDerivedFields, dust.cc:121-133).
struct DustPrim {
  double W, v[3];
};
// em4phi = exp(-4 phi), e6phi = exp(6 phi) of the point's phi
__device__ __forceinline__ DustPrim dust_prim(const double gi[6], double em4phi, double e6phi, double D,
                                              const double S[3]) {
  DustPrim d;
  const double giIJSISJ = em4phi * (gi[0] * S[0] * S[0] + gi[3] * S[1] * S[1] + gi[5] * S[2] * S[2] +
                                    2.0 * (gi[1] * S[0] * S[1] + gi[2] * S[0] * S[2] + gi[4] * S[1] * S[2]));
  d.W = sqrt(1.0 + giIJSISJ / D / D);
  d.v[0] = em4phi / e6phi * (gi[0] * S[0] + gi[1] * S[1] + gi[2] * S[2]);
  d.v[1] = em4phi / e6phi * (gi[1] * S[0] + gi[3] * S[1] + gi[4] * S[2]);
  d.v[2] = em4phi / e6phi * (gi[2] * S[0] + gi[4] * S[1] + gi[5] * S[2]);
  return d;
}

// BSSN sources from dust (Dust::addBSSNSrc, dust.cc:247-260) plus
// Lambda::addBSSNSource (lambda.cc:37-38), from the lagged derived values
// (W, det g, g_ij of the previous populate) and the current D, S_i.
__device__ __forceinline__ void dust_sources(double W, double detg, const double gphys[6], double D,
                                             const double S[3], double lambda, double q[Q_N]) {
  q[Q_R] = W * D / detg;
  const double Sd = D / detg * (W * W - 1.0) / W;
  q[Q_S] = Sd;
  for (int m = 0; m < 3; ++m) q[Q_S1 + m] = S[m] / detg;
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J)
      q[Q_STF11 + sym(I, J)] = S[I] * S[J] / W / D / detg - 1.0 / 3.0 * gphys[sym(I, J)] * Sd;
  q[Q_R] += lambda;
  q[Q_S] += -3.0 * lambda;
}

// lapse gauges, BSSNGaugeHandler.cc:16-275 (no shift)
__device__ __forceinline__ double ev_lapse(const Physics& ph, const StageBg& bg, double alpha,
                                           double K, double Kd, double phi) {
  switch (ph.lapse) {
    case kHarmonic: return -1.0 * alpha * (K);
    case kConformalFLRW: return -1.0 / 3.0 * alpha * bg.K_avg;
    case kConformalSync: return -1.0 / 3.0 * alpha * bg.K_FRW;
    case kAnharmonic: return 1.0 * (alpha * alpha) * (K - bg.K_avg);
    case kOnePlusLog: return -2.0 * alpha * (K - bg.K_avg) * ph.gd_c;
    case kAwAGaugeWave: return -1.0 * (alpha * alpha) * Kd;
    case kAwAShiftedWave: return -1.0 * Kd;
    case kDampedWave: return (alpha * alpha) * (ph.dw_mu_l * (12.0 * phi * ph.dw_p - log(alpha)) - K);
    default: return 0.0;
  }
}

// with the shift, the 1+log and damped-wave lapses add beta^i d_i alpha, term
// by term (BSSNGaugeHandler.cc:66-67, 152-153)
__device__ __forceinline__ double ev_lapse_shift(const Physics& ph, const StageBg& bg, double alpha, double K,
                                                 double Kd, double phi, const double beta[3], const double da[3]) {
  double v = ev_lapse(ph, bg, alpha, K, Kd, phi);
  if (ph.lapse == kOnePlusLog || ph.lapse == kDampedWave) {
    v = v + beta[0] * da[0];
    v = v + beta[1] * da[1];
    v = v + beta[2] * da[2];
  }
  return v;
}

__device__ __forceinline__ double pot_V(const Physics& ph, double phi) {
  return ph.potential == kPotQuadratic ? 0.5 * (ph.pot_mass * ph.pot_mass) * (phi * phi) : ph.pot_const;
}
__device__ __forceinline__ double pot_dV(const Physics& ph, double phi) {
  return ph.potential == kPotQuadratic ? (ph.pot_mass * ph.pot_mass) * phi : 0.0;
}

}  // namespace CG_VARIANT_NS
}  // namespace cg
