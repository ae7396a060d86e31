// cg_types.h -- parameter structs and slot enums shared by host and device code.
#pragma once

#include <cstdint>

namespace cg {

constexpr double kPi = 3.14159265358979323846;  // cosmo_macros.h:106 (4*atan(1) == M_PI)

// symmetric-pair index: 11,12,13,22,23,33 -> 0..5
__host__ __device__ constexpr int sym(int a, int b) {
  return a <= b ? (a == 0 ? b : (a == 1 ? 2 + b : 5)) : (b == 0 ? a : (b == 1 ? 2 + a : 5));
}

// Field slots inside a register block (same order as the state files).
enum : int {
  F_G11 = 0, F_G12, F_G13, F_G22, F_G23, F_G33, F_PHI, F_A11, F_A12, F_A13,
  F_A22, F_A23, F_A33, F_K, F_GAM1, F_GAM2, F_GAM3, F_ALPHA, F_NBSSN = 18,
  F_D = 18, F_S1 = 19, F_S2 = 20, F_S3 = 21,
  F_SPHI = 18, F_SPI = 19, F_SPSI1 = 20,
  F_DIFFD = 18  // static matter: the fixed density, not evolved
};
// source slots (bssn_macros.h:101-112)
enum : int { Q_R = 0, Q_S, Q_S1, Q_S2, Q_S3, Q_STF11, Q_N = 11 };
// dust flux primitives stored per point for the next substep's flux divergence:
// alpha*D, alpha*S_1..3, v^1..3 (dust.cc:121-133 forms the products of these)
enum : int { P_AD = 0, P_AS1, P_AS2, P_AS3, P_V1, P_V2, P_V3, P_N = 7 };

enum Matter : int { kVacuum = 0, kDust = 1, kScalar = 2, kStaticMatter = 3 };
enum Lapse : int {
  kStatic = 0, kHarmonic, kConformalFLRW, kConformalSync, kAnharmonic, kOnePlusLog,
  kAwAGaugeWave, kAwAShiftedWave, kDampedWave
};
enum Potential : int { kPotConst = 0, kPotQuadratic = 1 };
enum Shift : int { kShiftNone = 0, kShiftStatic, kShiftGammaDriver, kShiftDampedWave, kShiftAwA, kShiftAijDriver };

// Per-box physics parameters shared by all stage kernels.
struct Physics {
  int matter, lapse, potential, normalize;
  double dx, inv_dx, dt;
  int dx_pow2;            // dx is a power of two: x/dx == x*inv_dx exactly
  double lambda;          // rho_Lambda
  double a_adj_amp, k_damping_amp, gd_c, dw_mu_l, dw_p;
  double pot_const, pot_mass;
  double ko_coeff;        // KO_damping_coefficient (orders 2 and 8)
  // pow(dx, 4) and pow(dx, 3) (order 2) or pow(dx, 10) and pow(dx, 9) (order
  // 8), from the host's pow as the reference's KO_dissipation_Q takes them
  double ko_pden, ko_pnum;
  int shift;              // Shift gauge (kShiftNone: no shift fields)
  int gauge_wave_dir;     // AwAShiftedWave direction, 1..3
  double gd_eta, dw_mu_s, k_driver_coeff;
  long long tma_wait;     // cycles a CTA waits for a TMA tile copy before it flags a timeout
};

// Background values for one substep (FRW stage values, grid averages).
struct StageBg {
  double phi_FRW, K_FRW, rho_FRW, S_FRW;  // FRW getters during this substep
  double K_avg;                           // conformal average of K (bssn.cc:168)
  double phi_FRW_prev;                    // FRW phi during the previous substep
  double phi_FRW_next;                    // FRW phi during the next substep
};

}  // namespace cg
