// cg_stage.cuh -- the fused RK4 substep kernel for one periodic box (FP64).
//
// One launch performs, for every grid point, what the reference does in a
// whole substep of its sim drivers (sims/dust.cc:119-157, sims/scalar.cc:
// 275-317, components/bssn/bssn.cc:327-339):
//   sources      BSSN::clearSrc + Dust::addBSSNSrc + Lambda::addBSSNSource, or
//                Scalar::addBSSNSource (computed in registers, never stored)
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
#pragma once

#include "cg_point.cuh"

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
};

struct BoxGeom {
  int nx, ny, nz;
  int pts;
};

constexpr unsigned kStatusNaN = 1u;
constexpr unsigned kStatusNonFinite = 2u;

template <int MATTER>
struct NF {
  static constexpr int value = MATTER == kDust ? 22 : (MATTER == kScalar ? 23 : 18);
};

namespace CG_VARIANT_NS {

// derivative along axis a of the product of two stored arrays (the dust fluxes
// alpha*D*v^i = (alpha*D)*v^i, dust.cc:121-133, and their divergence :203-224)
template <int O>
__device__ __forceinline__ double der1_prod(const double* __restrict__ fa, const double* __restrict__ fb,
                                            const Site& s, int a, const Physics& ph) {
  auto V = [&](int n) {
    const int q = s.ax(a, n);
    return ld(fa, q) * ld(fb, q);
  };
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

template <int O, int MATTER>
__global__ void __launch_bounds__(128)
stage_kernel(BoxGeom geo, Physics ph, StageBg bg, StagePtrs P, int stage) {
  constexpr int NFLD = NF<MATTER>::value;
  if (P.kavg) bg.K_avg = *P.kavg;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int i = blockIdx.z;
  if (k >= geo.nz || j >= geo.ny) return;
  const Site s{i, j, k, geo.nx, geo.ny, geo.nz};
  const int c = (i * geo.ny + j) * geo.nz + k;
  const int N = geo.pts;
  const double* __restrict__ a = P.in;
  auto F = [&](int f) { return a + (size_t)f * N; };

  // ---- centre values (set_local_vals, bssn.cc:430-435) -------------------
  double g[6], A[6], Gam[3];
#pragma unroll
  for (int q = 0; q < 6; ++q) g[q] = ld(F(F_G11 + q), c);
#pragma unroll
  for (int q = 0; q < 6; ++q) A[q] = ld(F(F_A11 + q), c);
#pragma unroll
  for (int q = 0; q < 3; ++q) Gam[q] = ld(F(F_GAM1 + q), c);
  const double phi_d = ld(F(F_PHI), c), Kd = ld(F(F_K), c), alphad = ld(F(F_ALPHA), c);

  double gi[6];
  inv_metric(g, gi);
  const double phi = phi_d + bg.phi_FRW;
  const double K = Kd + bg.K_FRW;
  double gm[6];
  gm[0] = g[0] + 1.0; gm[1] = g[1]; gm[2] = g[2];
  gm[3] = g[3] + 1.0; gm[4] = g[4]; gm[5] = g[5] + 1.0;
  const double alpha = alphad + 1.0;

  // ---- first derivatives -------------------------------------------------
  double dphi[3], da[3], dK[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) dphi[d] = der1<O>(F(F_PHI), s, d, ph);
#pragma unroll
  for (int d = 0; d < 3; ++d) da[d] = der1<O>(F(F_ALPHA), s, d, ph);
#pragma unroll
  for (int d = 0; d < 3; ++d) dK[d] = der1<O>(F(F_K), s, d, ph);
  double dg[3][6];  // d_I g_JK (calculate_dgamma, bssn.cc:480-483)
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int q = 0; q < 6; ++q) dg[I][q] = der1<O>(F(F_G11 + q), s, I, ph);

  // ---- matter: sources and RHS pieces that need only the centre ----------
  double q[Q_N];
  double rhs_m[5] = {0, 0, 0, 0, 0};
  double mat_c[5] = {0, 0, 0, 0, 0};  // matter centre values (dust D,S or scalar fields)
  if (MATTER == kDust) {
    const double D = ld(F(F_D), c);
    const double S[3] = {ld(F(F_S1), c), ld(F(F_S2), c), ld(F(F_S3), c)};
    mat_c[0] = D; mat_c[1] = S[0]; mat_c[2] = S[1]; mat_c[3] = S[2];
    // lagged derived fields (populateDerivedFields of the previous substep)
    double Wl, detgl, gphys[6];
    if (stage == 1) {
      const DustPrim dp = dust_prim(gi, phi, D, S);
      Wl = dp.W;
      const double e4phi = exp(4.0 * phi);
      detgl = exp(6.0 * phi);
#pragma unroll
      for (int m = 0; m < 6; ++m) gphys[m] = e4phi * gm[m];
    } else {
      const double* pv = P.prev;
      double gp[6];
#pragma unroll
      for (int m = 0; m < 6; ++m) gp[m] = pv[(size_t)(F_G11 + m) * N + c];
      const double phip = pv[(size_t)F_PHI * N + c] + bg.phi_FRW_prev;
      const double Dp = pv[(size_t)F_D * N + c];
      const double Sp[3] = {pv[(size_t)F_S1 * N + c], pv[(size_t)F_S2 * N + c], pv[(size_t)F_S3 * N + c]};
      double gip[6];
      inv_metric(gp, gip);
      const DustPrim dp = dust_prim(gip, phip, Dp, Sp);
      Wl = dp.W;
      const double e4phi = exp(4.0 * phip);
      detgl = exp(6.0 * phip);
      gphys[0] = e4phi * (gp[0] + 1.0); gphys[1] = e4phi * gp[1]; gphys[2] = e4phi * gp[2];
      gphys[3] = e4phi * (gp[3] + 1.0); gphys[4] = e4phi * gp[4]; gphys[5] = e4phi * (gp[5] + 1.0);
    }
    dust_sources(Wl, detgl, gphys, D, S, ph.lambda, q);
    // dust RHS: flux divergence (dust.cc:203-224) + momentum source (dust.cc:135-146)
    const DustPrim cur = dust_prim(gi, phi, D, S);
    const double* __restrict__ fp = P.fp_in;
    auto FP = [&](int m) { return fp + (size_t)m * N; };
    rhs_m[0] = der1_prod<O>(FP(P_AD), FP(P_V1), s, 0, ph) + der1_prod<O>(FP(P_AD), FP(P_V2), s, 1, ph) +
               der1_prod<O>(FP(P_AD), FP(P_V3), s, 2, ph);
    const double e4 = exp(4.0 * phi);
#pragma unroll
    for (int m = 0; m < 3; ++m) {
      const int d = m;  // momentum component S_{m+1}: derivative index of the source
      const double* dgd = dg[d];
      const double src =
          1.0 / 2.0 * alpha * cur.W * D * e4 *
              (cur.v[0] * cur.v[0] * (4.0 * gm[0] * dphi[d] + dgd[0]) + cur.v[1] * cur.v[1] * (4.0 * gm[3] * dphi[d] + dgd[3]) +
               cur.v[2] * cur.v[2] * (4.0 * gm[5] * dphi[d] + dgd[5]) +
               2.0 * (cur.v[0] * cur.v[1] * (4.0 * gm[1] * dphi[d] + dgd[1]) +
                      cur.v[0] * cur.v[2] * (4.0 * gm[2] * dphi[d] + dgd[2]) +
                      cur.v[1] * cur.v[2] * (4.0 * gm[4] * dphi[d] + dgd[4]))) -
          cur.W * D * da[d];
      rhs_m[1 + m] = der1_prod<O>(FP(P_AS1 + m), FP(P_V1), s, 0, ph) +
                     der1_prod<O>(FP(P_AS1 + m), FP(P_V2), s, 1, ph) +
                     der1_prod<O>(FP(P_AS1 + m), FP(P_V3), s, 2, ph) + src;
    }
  } else if (MATTER == kScalar) {
    // Scalar::getScalarData (scalar.cc:97-130) and addBSSNSource (:201-260)
    const double sphi = ld(F(F_SPHI), c), sPi = ld(F(F_SPI), c);
    const double psi[3] = {ld(F(F_SPSI1), c), ld(F(F_SPSI1 + 1), c), ld(F(F_SPSI1 + 2), c)};
    mat_c[0] = sphi; mat_c[1] = sPi; mat_c[2] = psi[0]; mat_c[3] = psi[1]; mat_c[4] = psi[2];
    double sdphi[3], sdPi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) sdphi[d] = der1<O>(F(F_SPHI), s, d, ph);
#pragma unroll
    for (int d = 0; d < 3; ++d) sdPi[d] = der1<O>(F(F_SPI), s, d, ph);
    const double nmu = ((-alpha * sPi)) / alpha;
    const double dd = (gi[0] * sdphi[0] * sdphi[0] + gi[3] * sdphi[1] * sdphi[1] + gi[5] * sdphi[2] * sdphi[2] +
                       2.0 * (gi[1] * sdphi[0] * sdphi[1] + gi[2] * sdphi[0] * sdphi[2] + gi[4] * sdphi[1] * sdphi[2]));
    const double V = pot_V(ph, sphi);
    const double em4 = exp(-4.0 * phi);
    q[Q_R] = 0.5 * nmu * nmu + 0.5 * em4 * dd + V;
    q[Q_S] = 3.0 / 2.0 * nmu * nmu - 0.5 * em4 * dd - 3.0 * V;
#pragma unroll
    for (int m = 0; m < 3; ++m) q[Q_S1 + m] = -nmu * sdphi[m];
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = I; J < 3; ++J) q[Q_STF11 + sym(I, J)] = sdphi[I] * sdphi[J] - gm[sym(I, J)] / 3.0 * dd;
    // scalar RHS (scalar.cc:132-199)
    double inner = 0.0;
#pragma unroll
    for (int X = 0; X < 3; ++X)
#pragma unroll
      for (int Y = 0; Y < 3; ++Y) {
        const double u = gi[sym(X, Y)] * (alpha * der1<O>(F(F_SPSI1 + Y), s, X, ph) + psi[X] * da[Y]);
        inner = (X == 0 && Y == 0) ? u : inner + u;
      }
    double gt[3];
#pragma unroll
    for (int I = 0; I < 3; ++I)
      gt[I] = (Gam[I] - 2.0 * (gi[sym(I, 0)] * dphi[0] + gi[sym(I, 1)] * dphi[1] + gi[sym(I, 2)] * dphi[2]));
    rhs_m[0] = (-alpha * sPi);
    rhs_m[1] = (-exp(-4.0 * phi) * (inner) +
                alpha * ((gt[0]) * psi[0] * exp(-4.0 * phi) + (gt[1]) * psi[1] * exp(-4.0 * phi) +
                         (gt[2]) * psi[2] * exp(-4.0 * phi) + K * sPi + pot_dV(ph, sphi)));
#pragma unroll
    for (int m = 0; m < 3; ++m) rhs_m[2 + m] = (-alpha * sdPi[m] - sPi * da[m]);
  } else {
#pragma unroll
    for (int m = 0; m < Q_N; ++m) q[m] = 0.0;
  }
  const double r = q[Q_R] + bg.rho_FRW;

  // ---- A^ij, A_ij A^ij (calculate_Acont, bssn.cc:463-472) ------------------
  double Ac[6];
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

  // ---- Christoffels (bssn.cc:577-590, bssn_macros.h:221-229) ---------------
  double G[3][6], GL[3][6], Gd[3];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = 0; J < 3; ++J)
#pragma unroll
      for (int Kx = J; Kx < 3; ++Kx) {
        double t = gi[sym(I, 0)] * (dg[J][sym(Kx, 0)] + dg[Kx][sym(J, 0)] - dg[0][sym(J, Kx)]);
        t = t + gi[sym(I, 1)] * (dg[J][sym(Kx, 1)] + dg[Kx][sym(J, 1)] - dg[1][sym(J, Kx)]);
        t = t + gi[sym(I, 2)] * (dg[J][sym(Kx, 2)] + dg[Kx][sym(J, 2)] - dg[2][sym(J, Kx)]);
        G[I][sym(J, Kx)] = 0.5 * (t);
        GL[I][sym(J, Kx)] = 0.5 * (dg[J][sym(Kx, I)] + dg[Kx][sym(J, I)] - dg[I][sym(J, Kx)]);
      }
#pragma unroll
  for (int I = 0; I < 3; ++I)
    Gd[I] = G[I][0] * gi[0] + G[I][3] * gi[3] + G[I][5] * gi[5] + 2.0 * (G[I][1] * gi[1] + G[I][2] * gi[2] + G[I][4] * gi[4]);

  // ---- D_i D_j phi (bssn.cc:592-602) and (D_i D_j alpha)^TF (:604-626) -----
  double DDphi[6], DDa[6];
  double gld[3];
#pragma unroll
  for (int I = 0; I < 3; ++I) gld[I] = gi[sym(I, 0)] * dphi[0] + gi[sym(I, 1)] * dphi[1] + gi[sym(I, 2)] * dphi[2];
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int qq = sym(I, J);
      DDphi[qq] = der2ab<O>(F(F_PHI), s, I, J, ph) - (G[0][qq] * dphi[0] + G[1][qq] * dphi[1] + G[2][qq] * dphi[2]);
      double t = 0.0;
#pragma unroll
      for (int L = 0; L < 3; ++L) {
        const double u = G[L][qq] + 2.0 * ((L == I ? 1.0 : 0.0) * dphi[J] + (L == J ? 1.0 : 0.0) * dphi[I] - gm[qq] * gld[L]);
        t = L == 0 ? u * da[L] : t + u * da[L];
      }
      DDa[qq] = der2ab<O>(F(F_ALPHA), s, I, J, ph) - (t);
    }
  double DDaTR = gi[0] * DDa[0] + gi[3] * DDa[3] + gi[5] * DDa[5] + 2.0 * (gi[1] * DDa[1] + gi[2] * DDa[2] + gi[4] * DDa[4]);
#pragma unroll
  for (int m = 0; m < 6; ++m) DDa[m] -= (1.0 / 3.0) * gm[m] * DDaTR;
  DDaTR *= exp(-4.0 * phi);

  // ---- Ricci (bssn.cc:629-674, bssn_macros.h:248-277) ------------------------
  double dGam[3][3];  // d_J Gamma^K
#pragma unroll
  for (int Kx = 0; Kx < 3; ++Kx)
#pragma unroll
    for (int J = 0; J < 3; ++J) dGam[J][Kx] = der1<O>(F(F_GAM1 + Kx), s, J, ph);
  double Ric[6];
  const double expression =
      (gi[0] * (DDphi[0] + 2.0 * dphi[0] * dphi[0]) + gi[3] * (DDphi[3] + 2.0 * dphi[1] * dphi[1]) +
       gi[5] * (DDphi[5] + 2.0 * dphi[2] * dphi[2]) +
       2.0 * (gi[1] * (DDphi[1] + 2.0 * dphi[0] * dphi[1]) + gi[2] * (DDphi[2] + 2.0 * dphi[0] * dphi[2]) +
              gi[4] * (DDphi[4] + 2.0 * dphi[1] * dphi[2])));
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      const int ij = sym(I, J);
      const double* fg = F(F_G11 + ij);
      double ddg[6];  // d_K d_L g_IJ (calculate_ddgamma, bssn.cc:491-494)
#pragma unroll
      for (int Kx = 0; Kx < 3; ++Kx)
#pragma unroll
        for (int L = Kx; L < 3; ++L) ddg[sym(Kx, L)] = der2ab<O>(fg, s, Kx, L, ph);
      double t1 = 0.0;
#pragma unroll
      for (int Kx = 0; Kx < 3; ++Kx)
#pragma unroll
        for (int L = 0; L < 3; ++L) {
          const double u = gi[sym(Kx, L)] * ddg[sym(Kx, L)];
          t1 = (Kx == 0 && L == 0) ? u : t1 + u;
        }
      const double t2a = gm[sym(0, I)] * dGam[J][0] + gm[sym(1, I)] * dGam[J][1] + gm[sym(2, I)] * dGam[J][2];
      const double t2b = gm[sym(0, J)] * dGam[I][0] + gm[sym(1, J)] * dGam[I][1] + gm[sym(2, J)] * dGam[I][2];
      const double t3a = Gd[0] * GL[I][sym(J, 0)] + Gd[1] * GL[I][sym(J, 1)] + Gd[2] * GL[I][sym(J, 2)];
      const double t3b = Gd[0] * GL[J][sym(I, 0)] + Gd[1] * GL[J][sym(I, 1)] + Gd[2] * GL[J][sym(I, 2)];
      double t4 = 0.0;
#pragma unroll
      for (int Kx = 0; Kx < 3; ++Kx)
#pragma unroll
        for (int L = 0; L < 3; ++L)
#pragma unroll
          for (int M = 0; M < 3; ++M) {
            const double u = gi[sym(L, M)] * (G[Kx][sym(L, I)] * GL[J][sym(Kx, M)] + G[Kx][sym(L, J)] * GL[I][sym(Kx, M)] +
                                              0.5 * (G[Kx][sym(I, M)] * GL[Kx][sym(L, J)] + G[Kx][sym(J, M)] * GL[Kx][sym(L, I)]));
            t4 = (Kx == 0 && L == 0 && M == 0) ? u : t4 + u;
          }
      const double U = (-0.5 * (t1) + 0.5 * (t2a + t2b) + 0.5 * (t3a + t3b) + t4);
      Ric[ij] = U - 2.0 * (DDphi[ij] - 2.0 * dphi[I] * dphi[J] + gm[ij] * (expression));
    }
  const double ricci = exp(-4.0 * phi) * (Ric[0] * gi[0] + Ric[3] * gi[3] + Ric[5] * gi[5] +
                                         2.0 * (Ric[1] * gi[1] + Ric[2] * gi[2] + Ric[4] * gi[4]));
  const double e4phi = exp(4.0 * phi);
  // Hamiltonian constraint, bssn.cc:1073-1084 (theta = 0)
  const double H = -exp(5.0 * phi) / 8.0 * (ricci + 2.0 / 3.0 * ((K + 2.0 * 0.0) * (K + 2.0 * 0.0)) - AijAij - 16.0 * kPi * r);

  // ---- evolution equations (bssn.cc:748-831, bssn_macros.h:292-385) --------
  double rhs[NFLD];
  const double dt = ph.dt;
#pragma unroll
  for (int m = 0; m < 6; ++m) rhs[F_G11 + m] = (-2.0 * alpha * A[m]) + 0.5 * ph.a_adj_amp * dt * H * g[m];
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
      const double RTF = Ric[qq] - (1.0 / 3.0) * e4phi * gm[qq] * ricci;
      const double dtA = (exp(-4.0 * phi) * (alpha * (RTF - 8.0 * kPi * q[Q_STF11 + qq]) - DDa[qq]) +
                          alpha * (((K + 2.0 * 0.0) * A[qq]) - 2.0 * (aa)));
      rhs[F_A11 + qq] = dtA - 1.0 * ph.a_adj_amp * dt * A[qq] * H;
    }
#pragma unroll
  for (int I = 0; I < 3; ++I) {
    const double so = (G[I][0] * Ac[0] + G[I][3] * Ac[3] + G[I][5] * Ac[5] + 2.0 * (G[I][1] * Ac[1] + G[I][2] * Ac[2] + G[I][4] * Ac[4]) +
                       6.0 * (Ac[sym(I, 0)] * dphi[0] + Ac[sym(I, 1)] * dphi[1] + Ac[sym(I, 2)] * dphi[2]));
    const double ns =
        (-2.0 * (Ac[sym(I, 0)] * da[0] + Ac[sym(I, 1)] * da[1] + Ac[sym(I, 2)] * da[2]) +
         2.0 * alpha *
             (+so -
              (1.0 / 3.0) * (2.0 * (gi[sym(I, 0)] * dK[0] + gi[sym(I, 1)] * dK[1] + gi[sym(I, 2)] * dK[2]) +
                             gi[sym(I, 0)] * 0.0 + gi[sym(I, 1)] * 0.0 + gi[sym(I, 2)] * 0.0) -
              2.0 * alpha * 0.0 * (Gam[I] - Gd[I]) -
              8.0 * kPi * (gi[sym(I, 0)] * q[Q_S1] + gi[sym(I, 1)] * q[Q_S2] + gi[sym(I, 2)] * q[Q_S3])));
    rhs[F_GAM1 + I] = ns + 0.0;
  }
  rhs[F_K] = (-DDaTR + alpha * (1.0 / 3.0 * (Kd + 2.0 * 0.0) * (Kd + 2.0 * 0.0 + 2.0 * bg.K_FRW) + AijAij) +
              4.0 * kPi * alpha * (q[Q_R] + q[Q_S]) + 4.0 * kPi * alphad * (bg.rho_FRW + bg.S_FRW) -
              1.0 * ph.k_damping_amp * H * exp(-5.0 * phi));
  rhs[F_PHI] = (0.1 * ph.a_adj_amp * dt * H - 1.0 / 6.0 * (alpha * (Kd + 2.0 * 0.0) + alphad * bg.K_FRW - (0.0 + 0.0 + 0.0)));
  rhs[F_ALPHA] = ev_lapse(ph, bg, alpha, K, Kd, phi);
  if (MATTER == kDust) {
#pragma unroll
    for (int m = 0; m < 4; ++m) rhs[F_D + m] = rhs_m[m];
  } else if (MATTER == kScalar) {
#pragma unroll
    for (int m = 0; m < 5; ++m) rhs[F_SPHI + m] = rhs_m[m];
  }

  // ---- RK4Register::K{n}Finalize (RK4Register.h:175-222) --------------------
  double outv[NFLD];
#pragma unroll
  for (int f = 0; f < NFLD; ++f) {
    const double pv = P.p[(size_t)f * N + c];
    const double cv = rhs[f];
    if (stage == 1) {
      P.f[(size_t)f * N + c] = dt * cv / 6.0;
      outv[f] = pv + dt * cv / 2.0;
    } else if (stage == 2) {
      const double fv = P.f[(size_t)f * N + c];
      P.f[(size_t)f * N + c] = fv + dt * cv / 3.0;
      outv[f] = pv + dt * cv / 2.0;
    } else if (stage == 3) {
      const double fv = P.f[(size_t)f * N + c];
      P.f[(size_t)f * N + c] = fv + dt * cv / 3.0;
      outv[f] = pv + dt * cv;
    } else {
      const double fv = P.f[(size_t)f * N + c];
      outv[f] = fv + (dt * cv / 6.0 + pv);
    }
    P.out[(size_t)f * N + c] = outv[f];
  }
  (void)mat_c;

  // ---- the next substep's inputs ---------------------------------------------
  if (stage == 4) {
    // failure detection (sims/sim.cc:179-183 counts NaNs of DIFFphi)
    bool bad_phi = isnan(outv[F_PHI]);
    bool bad_any = false;
#pragma unroll
    for (int f = 0; f < NFLD; ++f) bad_any |= !isfinite(outv[f]);
    if (bad_phi) atomicOr(P.status, kStatusNaN);
    if (bad_any) atomicOr(P.status, kStatusNonFinite);
    // next step's first-substep input: normalised gamma/A (bssn.cc:224-225)
    if (ph.normalize) {
      double gn[6], An[6];
#pragma unroll
      for (int m = 0; m < 6; ++m) { gn[m] = outv[F_G11 + m]; An[m] = outv[F_A11 + m]; }
      normalize_point(gn, An);
#pragma unroll
      for (int m = 0; m < 6; ++m) { outv[F_G11 + m] = gn[m]; outv[F_A11 + m] = An[m]; }
    }
#pragma unroll
    for (int f = 0; f < NFLD; ++f) P.norm[(size_t)f * N + c] = outv[f];
  }
  if (MATTER == kDust) {
    // flux primitives of the output state for the next substep's divergence
    double go[6], gio[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) go[m] = outv[F_G11 + m];
    inv_metric(go, gio);
    const double So[3] = {outv[F_S1], outv[F_S2], outv[F_S3]};
    const double phio = outv[F_PHI] + bg.phi_FRW_next;
    const DustPrim dp = dust_prim(gio, phio, outv[F_D], So);
    const double alo = outv[F_ALPHA] + 1.0;
    double* fo = P.fp_out;
    fo[(size_t)P_AD * N + c] = alo * outv[F_D];
#pragma unroll
    for (int m = 0; m < 3; ++m) fo[(size_t)(P_AS1 + m) * N + c] = alo * So[m];
#pragma unroll
    for (int m = 0; m < 3; ++m) fo[(size_t)(P_V1 + m) * N + c] = dp.v[m];
  }
}

}  // namespace CG_VARIANT_NS
}  // namespace cg
