/*
 * cg_oracle.c -- CPU restatement of the CosmoGRaPH BSSN(+dust/+scalar) RK4
 * evolution path.  TEST INFRASTRUCTURE ONLY (see cg_oracle.h): it is the
 * checker the CUDA path is compared against, and the timed CPU "port"
 * baseline; nothing in the product calls it.
 *
 * Structure follows the reference one pass per method, as the reference's
 * OpenMP loops do, so that intermediate arrays (sources, dust fluxes) match
 * the reference's lifetimes exactly.  Operand order inside every expression
 * follows the reference expression cited next to it; build with
 * -ffp-contract=off for bit-level parity with the reference's strict build.
 */
#include "cg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* PI (cosmo_macros.h:106) is 4*atan(1), which equals M_PI exactly. */
#define CG_PI 3.14159265358979323846
#define PW2(x) ((x) * (x))

void cgo_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* with Z4c damping, theta follows these (its index is cgo_num_fields) */
int cgo_num_fields(int matter) {
  return matter == CGO_DUST ? 22 : matter == CGO_SCALAR ? 23 : matter == CGO_STATIC ? 19 : 18;
}

/* field slots, cg_state.h order */
enum {
  F_G11, F_G12, F_G13, F_G22, F_G23, F_G33, F_PHI, F_A11, F_A12, F_A13, F_A22,
  F_A23, F_A33, F_K, F_GAM1, F_GAM2, F_GAM3, F_ALPHA, F_NBSSN,
  F_D = 18, F_S1, F_S2, F_S3,
  F_SPHI = 18, F_SPI, F_SPSI1, F_SPSI2, F_SPSI3
};
/* source slots (bssn_macros.h:101-112) */
enum { Q_R, Q_S, Q_S1, Q_S2, Q_S3, Q_STF11, Q_STF12, Q_STF13, Q_STF22, Q_STF23, Q_STF33, Q_N };
/* dust derived arrays (components/dust_fluid/dust.h:37-46) */
enum {
  U_ADV1, U_ADV2, U_ADV3, U_AS1V1, U_AS1V2, U_AS1V3, U_AS2V1, U_AS2V2, U_AS2V3,
  U_AS3V1, U_AS3V2, U_AS3V3, U_S1SRC, U_S2SRC, U_S3SRC, U_DETG, U_G11, U_G12,
  U_G13, U_G22, U_G23, U_G33, U_W, U_N
};

/* symmetric index 11,12,13,22,23,33 -> 0..5 */
static const int SYM[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

typedef struct {
  const cgo_params *p;
  long nx, ny, nz, pts;
  int nf;
  double *reg_p, *reg_a, *reg_c, *reg_f; /* nf*pts each */
  double *src;                           /* Q_N*pts */
  double *dust;                          /* U_N*pts */
  /* FRW state */
  double frw_phi, frw_K, fl_rho[CGO_MAX_FLUIDS];
  double phi_K[4], K_K[4], fl_K[4][CGO_MAX_FLUIDS];
  double get_phi, get_K, get_rho, get_S;
  /* BSSN::setExtraFieldData outputs (bssn.cc:165-170) */
  double K_avg, avg_vol, rho_avg, K_min;
} sim_t;

static inline long wrap(long i, long n) {
  long m = i % n;
  return m < 0 ? m + n : m;
}
static inline long IDX(const sim_t *s, long i, long j, long k) {
  return (wrap(i, s->nx) * s->ny + wrap(j, s->ny)) * s->nz + wrap(k, s->nz);
}
/* field value at a periodic offset along axis d (0,1,2) by n */
static inline double at1(const sim_t *s, const double *f, long i, long j, long k, int d, int n) {
  return f[IDX(s, i + (d == 0) * n, j + (d == 1) * n, k + (d == 2) * n)];
}
/* value at offsets n along axis a and m along axis b */
static inline double at2(const sim_t *s, const double *f, long i, long j, long k, int a, int n,
                         int b, int m) {
  long o[3] = {0, 0, 0};
  o[a] += n;
  o[b] += m;
  return f[IDX(s, i + o[0], j + o[1], k + o[2])];
}

/* First derivative, utils/math.h:74-100 (O2), :231-263 (O4), :412-450 (O6),
 * :554-586 (O8).  d = 1,2,3 as in the reference. */
static double deriv(const sim_t *s, long i, long j, long k, int d, const double *f) {
  const double dx = s->p->dx;
  const int a = d - 1;
#define V(n) at1(s, f, i, j, k, a, n)
  switch (s->p->order) {
    case 2:
      return ((-1.0 / 2.0 * V(-1) + 1.0 / 2.0 * V(1)) / dx);
    case 4:
      return (+1.0 / 12.0 * V(-2) - 2.0 / 3.0 * V(-1) + 2.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2)) / dx;
    case 6:
      return (-1.0 / 60.0 * V(-3) + 3.0 / 20.0 * V(-2) - 3.0 / 4.0 * V(-1) + 3.0 / 4.0 * V(1) -
              3.0 / 20.0 * V(2) + 1.0 / 60.0 * V(3)) /
             dx;
    default:
      return ((1.0 / 280.0 * V(-4) - 1.0 / 280.0 * V(4)) - (4.0 / 105.0 * V(-3) - 4.0 / 105.0 * V(3)) +
              (1.0 / 5.0 * V(-2) - 1.0 / 5.0 * V(2)) - (4.0 / 5.0 * V(-1) - 4.0 / 5.0 * V(1))) /
             dx;
  }
#undef V
}

/* Second derivative along one axis, utils/math.h:857-885 (O2), :958-993 (O4),
 * :995-1036 (O6), :1038-1085 (O8). */
static double dderiv_diag(const sim_t *s, long i, long j, long k, int d, const double *f) {
  const double dx = s->p->dx;
  const int a = d - 1;
#define V(n) at1(s, f, i, j, k, a, n)
  switch (s->p->order) {
    case 2:
      return (V(-1) - 2.0 * V(0) + V(1)) / dx / dx;
    case 4:
      return (-1.0 / 12.0 * V(-2) + 4.0 / 3.0 * V(-1) - 5.0 / 2.0 * V(0) + 4.0 / 3.0 * V(1) -
              1.0 / 12.0 * V(2)) /
             dx / dx;
    case 6:
      return (1.0 / 90.0 * V(-3) - 3.0 / 20.0 * V(-2) + 3.0 / 2.0 * V(-1) - 49.0 / 18.0 * V(0) +
              3.0 / 2.0 * V(1) - 3.0 / 20.0 * V(2) + 1.0 / 90.0 * V(3)) /
             dx / dx;
    default:
      return (-1.0 / 560.0 * V(-4) + 8.0 / 315.0 * V(-3) - 1.0 / 5.0 * V(-2) + 8.0 / 5.0 * V(-1) -
              205.0 / 72.0 * V(0) + 8.0 / 5.0 * V(1) - 1.0 / 5.0 * V(2) + 8.0 / 315.0 * V(3) -
              1.0 / 560.0 * V(4)) /
             dx / dx;
  }
#undef V
}

/* Mixed second derivative on the diagonal points (i+-n, j+-n):
 * utils/math.h:676-701 (O2), :703-743 (O4), :745-794 (O6), :796-855 (O8). */
static double dderiv_mixed(const sim_t *s, long i, long j, long k, int d1, int d2,
                           const double *f) {
  const double dx = s->p->dx;
  const int a = (d1 < d2 ? d1 : d2) - 1, b = (d1 < d2 ? d2 : d1) - 1;
#define P(n)                                                                          \
  (-at2(s, f, i, j, k, a, n, b, -(n)) + at2(s, f, i, j, k, a, n, b, n) +              \
   at2(s, f, i, j, k, a, -(n), b, -(n)) - at2(s, f, i, j, k, a, -(n), b, n))
  switch (s->p->order) {
    case 2:
      return P(1) / 4.0 / dx / dx;
    case 4:
      return (P(1) - 1.0 / 16.0 * P(2)) / 3.0 / dx / dx;
    case 6:
      return (135.0 * P(1) - 27.0 / 2.0 * P(2) + P(3)) / 360.0 / dx / dx;
    default:
      return (2.0 / 5.0 * P(1) - 1.0 / 20.0 * P(2) + 2.0 / 315.0 * P(3) - 1.0 / 2240.0 * P(4)) / dx /
             dx;
  }
#undef P
}

/* utils/math.h:1319-1330 */
static double dderiv(const sim_t *s, long i, long j, long k, int d1, int d2, const double *f) {
  return d1 == d2 ? dderiv_diag(s, i, j, k, d1, f) : dderiv_mixed(s, i, j, k, d1, d2, f);
}

/* Kreiss-Oliger dissipation, utils/math.h:36-72 (orders 2 and 8 only). */
static double ko_diss(const sim_t *s, long i, long j, long k, const double *f) {
  const double c = s->p->ko_coeff, dx = s->p->dx;
  if (c == 0) return 0;
#define X(n) f[IDX(s, i + (n), j, k)]
#define Y(n) f[IDX(s, i, j + (n), k)]
#define Z(n) f[IDX(s, i, j, k + (n))]
  if (s->p->order == 2) {
    double st = (1.0 * X(-2) + 1.0 * Y(-2) + 1.0 * Z(-2) - 4.0 * X(-1) - 4.0 * Y(-1) - 4.0 * Z(-1) +
                 6.0 * X(0) + 6.0 * Y(0) + 6.0 * Z(0) - 4.0 * X(1) - 4.0 * Y(1) - 4.0 * Z(1) +
                 1.0 * X(2) + 1.0 * Y(2) + 1.0 * Z(2)) /
                pow(dx, 4.0);
    return c * pow(dx, 3.0) / 64.0 * st;
  }
  if (s->p->order == 8) {
    double st = (1.0 * X(-5) + 1.0 * Y(-5) + 1.0 * Z(-5) - 10.0 * X(-4) - 10.0 * Y(-4) -
                 10.0 * Z(-4) + 45.0 * X(-3) + 45.0 * Y(-3) + 45.0 * Z(-3) - 120.0 * X(-2) -
                 120.0 * Y(-2) - 120.0 * Z(-2) + 210.0 * X(-1) + 210.0 * Y(-1) + 210.0 * Z(-1) -
                 252.0 * X(0) - 252.0 * Y(0) - 252.0 * Z(0) + 210.0 * X(1) + 210.0 * Y(1) +
                 210.0 * Z(1) - 120.0 * X(2) - 120.0 * Y(2) - 120.0 * Z(2) + 45.0 * X(3) +
                 45.0 * Y(3) + 45.0 * Z(3) - 10.0 * X(4) - 10.0 * Y(4) - 10.0 * Z(4) + 1.0 * X(5) +
                 1.0 * Y(5) + 1.0 * Z(5)) /
                pow(dx, 10.0);
    return -c * pow(dx, 9.0) / 1024.0 * st;
  }
#undef X
#undef Y
#undef Z
  return 0.0;
}

/* The per-point workspace of BSSN::set_bd_values (bssn.cc:361-421). */
typedef struct {
  double g[6], phi_d, A[6], Kd, Gam[3], alphad; /* DIFF fields: 11,12,13,22,23,33 */
  double src[Q_N];
  double phi, K, gamma[6], r, S, alpha;
  double gi[6];
  double Acont[6], AijAij;
  double dg[3][6];      /* d_I g_JK */
  double ddg[6][6];     /* d_I d_J g_KL, first index sym(IJ) */
  double dphi[3], ddphi[6], da[3], dK[3];
  double G[3][6], GL[3][6], Gammad[3];
  double DDphi[6], DDaTF[6], DDaTR;
  double Uricci[6], ricci_t[6], ricci, ricciTF[6];
  double H;
  double theta, dtheta[3]; /* Z4c: theta and its first derivatives (0 without Z4c) */
} bd_t;

/* BSSN::set_bd_values, bssn.cc:361-421, on the "_a" register and sources */
static void set_bd(const sim_t *s, long i, long j, long k, bd_t *bd) {
  const long idx = IDX(s, i, j, k);
  const long N = s->pts;
  const double *a = s->reg_a;
  for (int q = 0; q < 6; ++q) bd->g[q] = a[(F_G11 + q) * N + idx];
  bd->phi_d = a[F_PHI * N + idx];
  for (int q = 0; q < 6; ++q) bd->A[q] = a[(F_A11 + q) * N + idx];
  bd->Kd = a[F_K * N + idx];
  for (int q = 0; q < 3; ++q) bd->Gam[q] = a[(F_GAM1 + q) * N + idx];
  bd->alphad = a[F_ALPHA * N + idx];
  for (int q = 0; q < Q_N; ++q) bd->src[q] = s->src[q * N + idx];
  /* Z4c: set_local_vals and calculate_dtheta (bssn.cc:430-435, 537-544) */
  const long fth = cgo_num_fields(s->p->matter);
  bd->theta = s->p->z4c ? a[fth * N + idx] : 0.0;
  for (int q = 0; q < 3; ++q) bd->dtheta[q] = s->p->z4c ? deriv(s, i, j, k, q + 1, a + fth * N) : 0.0;

  /* set_gammai_values, bssn.cc:447-455 */
  const double *g = bd->g;
  bd->gi[0] = 1.0 + g[3] + g[5] - PW2(g[4]) + g[3] * g[5];
  bd->gi[3] = 1.0 + g[0] + g[5] - PW2(g[2]) + g[0] * g[5];
  bd->gi[5] = 1.0 + g[0] + g[3] - PW2(g[1]) + g[0] * g[3];
  bd->gi[1] = g[2] * g[4] - g[1] * (1.0 + g[5]);
  bd->gi[2] = g[1] * g[4] - g[2] * (1.0 + g[3]);
  bd->gi[4] = g[1] * g[2] - g[4] * (1.0 + g[0]);

  /* bssn.cc:384-394 */
  bd->phi = bd->phi_d + s->get_phi;
  bd->K = bd->Kd + s->get_K;
  bd->gamma[0] = g[0] + 1.0;
  bd->gamma[1] = g[1];
  bd->gamma[2] = g[2];
  bd->gamma[3] = g[3] + 1.0;
  bd->gamma[4] = g[4];
  bd->gamma[5] = g[5] + 1.0;
  bd->r = bd->src[Q_R] + s->get_rho;
  bd->S = bd->src[Q_S] + s->get_S;
  bd->alpha = bd->alphad + 1.0;

  const double *gi = bd->gi, *A = bd->A;
  /* calculate_Acont, bssn.cc:463-472 with BSSN_CALCULATE_ACONT (bssn_macros.h:233-237) */
  for (int I = 0; I < 3; ++I)
    for (int J = I; J < 3; ++J) {
      double t = gi[SYM[I][0]] * gi[SYM[J][0]] * A[SYM[0][0]];
      t = t + gi[SYM[I][1]] * gi[SYM[J][0]] * A[SYM[1][0]];
      t = t + gi[SYM[I][2]] * gi[SYM[J][0]] * A[SYM[2][0]];
      t = t + gi[SYM[I][0]] * gi[SYM[J][1]] * A[SYM[0][1]];
      t = t + gi[SYM[I][1]] * gi[SYM[J][1]] * A[SYM[1][1]];
      t = t + gi[SYM[I][2]] * gi[SYM[J][1]] * A[SYM[2][1]];
      t = t + gi[SYM[I][0]] * gi[SYM[J][2]] * A[SYM[0][2]];
      t = t + gi[SYM[I][1]] * gi[SYM[J][2]] * A[SYM[1][2]];
      t = t + gi[SYM[I][2]] * gi[SYM[J][2]] * A[SYM[2][2]];
      bd->Acont[SYM[I][J]] = t;
    }
  const double *Ac = bd->Acont;
  bd->AijAij = Ac[0] * A[0] + Ac[3] * A[3] + Ac[5] * A[5] +
               2.0 * (Ac[1] * A[1] + Ac[2] * A[2] + Ac[4] * A[4]);

  /* calculate_dgamma, bssn.cc:480-483 */
  for (int I = 0; I < 3; ++I)
    for (int q = 0; q < 6; ++q) bd->dg[I][q] = deriv(s, i, j, k, I + 1, a + (F_G11 + q) * N);
  /* calculate_ddgamma, bssn.cc:491-494 */
  for (int I = 0; I < 3; ++I)
    for (int J = I; J < 3; ++J)
      for (int q = 0; q < 6; ++q)
        bd->ddg[SYM[I][J]][q] = dderiv(s, i, j, k, I + 1, J + 1, a + (F_G11 + q) * N);
  /* calculate_dalpha_dphi, bssn.cc:502-521 */
  const double *fphi = a + F_PHI * N, *falpha = a + F_ALPHA * N;
  for (int I = 0; I < 3; ++I) bd->dphi[I] = deriv(s, i, j, k, I + 1, fphi);
  for (int I = 0; I < 3; ++I)
    for (int J = I; J < 3; ++J) bd->ddphi[SYM[I][J]] = dderiv(s, i, j, k, I + 1, J + 1, fphi);
  for (int I = 0; I < 3; ++I) bd->da[I] = deriv(s, i, j, k, I + 1, falpha);
  /* calculate_dK, bssn.cc:529-535 */
  for (int I = 0; I < 3; ++I) bd->dK[I] = deriv(s, i, j, k, I + 1, a + F_K * N);

  /* calculate_conformal_christoffels, bssn.cc:577-590 with
   * BSSN_CALCULATE_CHRISTOFFEL(_LOWER), bssn_macros.h:221-229 */
  for (int I = 0; I < 3; ++I)
    for (int J = 0; J < 3; ++J)
      for (int K = J; K < 3; ++K) {
        double t = gi[SYM[I][0]] * (bd->dg[J][SYM[K][0]] + bd->dg[K][SYM[J][0]] - bd->dg[0][SYM[J][K]]);
        t = t + gi[SYM[I][1]] * (bd->dg[J][SYM[K][1]] + bd->dg[K][SYM[J][1]] - bd->dg[1][SYM[J][K]]);
        t = t + gi[SYM[I][2]] * (bd->dg[J][SYM[K][2]] + bd->dg[K][SYM[J][2]] - bd->dg[2][SYM[J][K]]);
        bd->G[I][SYM[J][K]] = 0.5 * (t);
      }
  for (int I = 0; I < 3; ++I)
    for (int J = 0; J < 3; ++J)
      for (int K = J; K < 3; ++K)
        bd->GL[I][SYM[J][K]] =
            0.5 * (bd->dg[J][SYM[K][I]] + bd->dg[K][SYM[J][I]] - bd->dg[I][SYM[J][K]]);
  for (int I = 0; I < 3; ++I)
    bd->Gammad[I] = bd->G[I][0] * gi[0] + bd->G[I][3] * gi[3] + bd->G[I][5] * gi[5] +
                    2.0 * (bd->G[I][1] * gi[1] + bd->G[I][2] * gi[2] + bd->G[I][4] * gi[4]);

  /* calculateDDphi, bssn.cc:592-602 */
  for (int I = 0; I < 3; ++I)
    for (int J = I; J < 3; ++J) {
      const int q = SYM[I][J];
      bd->DDphi[q] = bd->ddphi[q] - (bd->G[0][q] * bd->dphi[0] + bd->G[1][q] * bd->dphi[1] +
                                     bd->G[2][q] * bd->dphi[2]);
    }

  /* calculateDDalphaTF, bssn.cc:604-626 with BSSN_CALCULATE_DIDJALPHA
   * (bssn_macros.h:241-245) */
  double gildlphi[3];
  for (int I = 0; I < 3; ++I)
    gildlphi[I] = gi[SYM[I][0]] * bd->dphi[0] + gi[SYM[I][1]] * bd->dphi[1] + gi[SYM[I][2]] * bd->dphi[2];
  for (int I = 0; I < 3; ++I)
    for (int J = I; J < 3; ++J) {
      const int q = SYM[I][J];
      double t = 0.0;
      for (int L = 0; L < 3; ++L) {
        double u = bd->G[L][q] + 2.0 * ((L == I) * bd->dphi[J] + (L == J) * bd->dphi[I] -
                                        bd->gamma[q] * gildlphi[L]);
        t = L == 0 ? u * bd->da[L] : t + u * bd->da[L];
      }
      bd->DDaTF[q] = dderiv(s, i, j, k, I + 1, J + 1, falpha) - (t);
    }
  bd->DDaTR = gi[0] * bd->DDaTF[0] + gi[3] * bd->DDaTF[3] + gi[5] * bd->DDaTF[5] +
              2.0 * (gi[1] * bd->DDaTF[1] + gi[2] * bd->DDaTF[2] + gi[4] * bd->DDaTF[4]);
  for (int q = 0; q < 6; ++q) bd->DDaTF[q] -= (1.0 / 3.0) * bd->gamma[q] * bd->DDaTR;
  bd->DDaTR *= exp(-4.0 * bd->phi);

  /* calculateRicciTF, bssn.cc:629-674 with BSSN_CALCULATE_RICCI_UNITARY
   * (bssn_macros.h:248-277) */
  double dGam[3][3]; /* dGam[J][K] = d_J Gamma^K */
  for (int K = 0; K < 3; ++K)
    for (int J = 0; J < 3; ++J) dGam[J][K] = deriv(s, i, j, k, J + 1, a + (F_GAM1 + K) * N);
  for (int I = 0; I < 3; ++I)
    for (int J = I; J < 3; ++J) {
      const int ij = SYM[I][J];
      double t1 = 0.0;
      for (int K = 0; K < 3; ++K)
        for (int L = 0; L < 3; ++L) {
          double u = gi[SYM[K][L]] * bd->ddg[SYM[K][L]][ij];
          t1 = (K == 0 && L == 0) ? u : t1 + u;
        }
      double t2a = bd->gamma[SYM[0][I]] * dGam[J][0] + bd->gamma[SYM[1][I]] * dGam[J][1] +
                   bd->gamma[SYM[2][I]] * dGam[J][2];
      double t2b = bd->gamma[SYM[0][J]] * dGam[I][0] + bd->gamma[SYM[1][J]] * dGam[I][1] +
                   bd->gamma[SYM[2][J]] * dGam[I][2];
      double t3a = bd->Gammad[0] * bd->GL[I][SYM[J][0]] + bd->Gammad[1] * bd->GL[I][SYM[J][1]] +
                   bd->Gammad[2] * bd->GL[I][SYM[J][2]];
      double t3b = bd->Gammad[0] * bd->GL[J][SYM[I][0]] + bd->Gammad[1] * bd->GL[J][SYM[I][1]] +
                   bd->Gammad[2] * bd->GL[J][SYM[I][2]];
      double t4 = 0.0;
      for (int K = 0; K < 3; ++K)
        for (int L = 0; L < 3; ++L)
          for (int M = 0; M < 3; ++M) {
            double u = gi[SYM[L][M]] *
                       (bd->G[K][SYM[L][I]] * bd->GL[J][SYM[K][M]] + bd->G[K][SYM[L][J]] * bd->GL[I][SYM[K][M]] +
                        0.5 * (bd->G[K][SYM[I][M]] * bd->GL[K][SYM[L][J]] +
                               bd->G[K][SYM[J][M]] * bd->GL[K][SYM[L][I]]));
            t4 = (K == 0 && L == 0 && M == 0) ? u : t4 + u;
          }
      bd->Uricci[ij] = (-0.5 * (t1) + 0.5 * (t2a + t2b) + 0.5 * (t3a + t3b) + t4);
    }
  const double *dphi = bd->dphi;
  const double expression =
      (gi[0] * (bd->DDphi[0] + 2.0 * dphi[0] * dphi[0]) + gi[3] * (bd->DDphi[3] + 2.0 * dphi[1] * dphi[1]) +
       gi[5] * (bd->DDphi[5] + 2.0 * dphi[2] * dphi[2]) +
       2.0 * (gi[1] * (bd->DDphi[1] + 2.0 * dphi[0] * dphi[1]) + gi[2] * (bd->DDphi[2] + 2.0 * dphi[0] * dphi[2]) +
              gi[4] * (bd->DDphi[4] + 2.0 * dphi[1] * dphi[2])));
  for (int I = 0; I < 3; ++I)
    for (int J = I; J < 3; ++J) {
      const int q = SYM[I][J];
      bd->ricci_t[q] = bd->Uricci[q] - 2.0 * (bd->DDphi[q] - 2.0 * dphi[I] * dphi[J] + bd->gamma[q] * (expression));
    }
  const double *R = bd->ricci_t;
  bd->ricci = exp(-4.0 * bd->phi) *
              (R[0] * gi[0] + R[3] * gi[3] + R[5] * gi[5] + 2.0 * (R[1] * gi[1] + R[2] * gi[2] + R[4] * gi[4]));
  for (int q = 0; q < 6; ++q)
    bd->ricciTF[q] = R[q] - (1.0 / 3.0) * exp(4.0 * bd->phi) * bd->gamma[q] * bd->ricci;

  /* hamiltonianConstraintCalc, bssn.cc:1073-1084 */
  const double theta = bd->theta;
  bd->H = -exp(5.0 * bd->phi) / 8.0 *
          (bd->ricci + 2.0 / 3.0 * PW2(bd->K + 2.0 * theta) - bd->AijAij - 16.0 * CG_PI * bd->r);
}

/* BSSNGaugeHandler lapse functions, BSSNGaugeHandler.cc:16-275 */
static double ev_lapse(const sim_t *s, const bd_t *bd) {
  const cgo_params *p = s->p;
  switch (p->lapse) {
    case CGO_LAPSE_HARMONIC: return -1.0 * bd->alpha * (bd->K);
    case CGO_LAPSE_CONFORMAL_FLRW: return -1.0 / 3.0 * bd->alpha * s->K_avg;
    case CGO_LAPSE_CONFORMAL_SYNC: return -1.0 / 3.0 * bd->alpha * s->get_K;
    case CGO_LAPSE_ANHARMONIC: return 1.0 * PW2(bd->alpha) * (bd->K - s->K_avg);
    case CGO_LAPSE_ONE_PLUS_LOG:
      return -2.0 * bd->alpha * (bd->K - s->K_avg) * p->gd_c + 0.0 * bd->da[0] + 0.0 * bd->da[1] +
             0.0 * bd->da[2];
    case CGO_LAPSE_AWA_GAUGE_WAVE: return -1.0 * PW2(bd->alpha) * bd->Kd;
    case CGO_LAPSE_AWA_SHIFTED_WAVE: return -1.0 * bd->Kd;
    case CGO_LAPSE_DAMPED_WAVE:
      return PW2(bd->alpha) * (p->dw_mu_l * (12.0 * bd->phi * p->dw_p - log(bd->alpha)) - bd->K) +
             0.0 * bd->da[0] + 0.0 * bd->da[1] + 0.0 * bd->da[2];
    default: return 0.0;
  }
}

/* Z4c damping amplitudes (cosmo_macros.h:94-100): 0.5 and 0.1 with Z4c, else 0 */
static double z4c_k1(const sim_t *s) { return s->p->z4c ? 0.5 : 0.0; }
static double z4c_k2(const sim_t *s) { return s->p->z4c ? 0.1 : 0.0; }

/* The BSSN_RK_EVOLVE_PT evolution functions, bssn.cc:748-848 and
 * bssn_macros.h:292-385 (no shift); with Z4c also ev_theta (bssn.cc:834-848),
 * written to out[cgo_num_fields(matter)]. */
static void bssn_rhs(const sim_t *s, long i, long j, long k, const bd_t *bd, double *out) {
  const cgo_params *p = s->p;
  const long N = s->pts;
  const double *a = s->reg_a;
  const double dt = p->dt, theta = bd->theta, k1 = z4c_k1(s), k2 = z4c_k2(s);
  const double *gi = bd->gi, *A = bd->A;
  /* ev_DIFFgammaIJ, bssn.cc:748-753 */
  for (int q = 0; q < 6; ++q)
    out[F_G11 + q] = (-2.0 * bd->alpha * A[q]) + 0.5 * p->a_adj_amp * dt * bd->H * bd->g[q] -
                     ko_diss(s, i, j, k, a + (F_G11 + q) * N);
  /* ev_AIJ, bssn.cc:755-760 with BSSN_DT_AIJ (bssn_macros.h:334-337) */
  for (int I = 0; I < 3; ++I)
    for (int J = I; J < 3; ++J) {
      const int q = SYM[I][J];
      double aa = 0.0;
      for (int X = 0; X < 3; ++X)
        for (int Y = 0; Y < 3; ++Y) {
          double u = gi[SYM[X][Y]] * A[SYM[X][I]] * A[SYM[Y][J]];
          aa = (X == 0 && Y == 0) ? u : aa + u;
        }
      double dtA = (exp(-4.0 * bd->phi) *
                        (bd->alpha * (bd->ricciTF[q] - 8.0 * CG_PI * bd->src[Q_STF11 + q]) - bd->DDaTF[q]) +
                    bd->alpha * (((bd->K + 2.0 * theta) * A[q]) - 2.0 * (aa)));
      out[F_A11 + q] = dtA - 1.0 * p->a_adj_amp * dt * A[q] * bd->H - ko_diss(s, i, j, k, a + (F_A11 + q) * N);
    }
  /* ev_GammaI, bssn.cc:762-764 with BSSN_DT_GAMMAI_NOSHIFT (bssn_macros.h:348-361) */
  for (int I = 0; I < 3; ++I) {
    const double *Ac = bd->Acont;
    double so = (bd->G[I][0] * Ac[0] + bd->G[I][3] * Ac[3] + bd->G[I][5] * Ac[5] +
                 2.0 * (bd->G[I][1] * Ac[1] + bd->G[I][2] * Ac[2] + bd->G[I][4] * Ac[4]) +
                 6.0 * (Ac[SYM[I][0]] * bd->dphi[0] + Ac[SYM[I][1]] * bd->dphi[1] + Ac[SYM[I][2]] * bd->dphi[2]));
    double ns =
        (-2.0 * (Ac[SYM[I][0]] * bd->da[0] + Ac[SYM[I][1]] * bd->da[1] + Ac[SYM[I][2]] * bd->da[2]) +
         2.0 * bd->alpha *
             (+so -
              (1.0 / 3.0) * (2.0 * (gi[SYM[I][0]] * bd->dK[0] + gi[SYM[I][1]] * bd->dK[1] + gi[SYM[I][2]] * bd->dK[2]) +
                             gi[SYM[I][0]] * bd->dtheta[0] + gi[SYM[I][1]] * bd->dtheta[1] +
                             gi[SYM[I][2]] * bd->dtheta[2]) -
              2.0 * bd->alpha * k1 * (bd->Gam[I] - bd->Gammad[I]) -
              8.0 * CG_PI *
                  (gi[SYM[I][0]] * bd->src[Q_S1] + gi[SYM[I][1]] * bd->src[Q_S2] + gi[SYM[I][2]] * bd->src[Q_S3])));
    out[F_GAM1 + I] = (ns + 0.0) - ko_diss(s, i, j, k, a + (F_GAM1 + I) * N);
  }
  /* ev_DIFFK, bssn.cc:766-795 */
  out[F_K] = (-bd->DDaTR +
              bd->alpha * (1.0 / 3.0 * (bd->Kd + 2.0 * theta) * (bd->Kd + 2.0 * theta + 2.0 * s->get_K) + bd->AijAij) +
              4.0 * CG_PI * bd->alpha * (bd->src[Q_R] + bd->src[Q_S]) +
              4.0 * CG_PI * bd->alphad * (s->get_rho + s->get_S) -
              1.0 * p->k_damping_amp * bd->H * exp(-5.0 * bd->phi) + k1 * (1.0 - k2) * theta -
              ko_diss(s, i, j, k, a + F_K * N));
  /* ev_DIFFphi, bssn.cc:797-820 */
  out[F_PHI] = (0.1 * p->a_adj_amp * dt * bd->H -
                1.0 / 6.0 * (bd->alpha * (bd->Kd + 2.0 * theta) + bd->alphad * s->get_K - (0.0 + 0.0 + 0.0)) -
                ko_diss(s, i, j, k, a + F_PHI * N));
  /* ev_DIFFalpha, bssn.cc:822-831 */
  out[F_ALPHA] = ev_lapse(s, bd) - ko_diss(s, i, j, k, a + F_ALPHA * N);
  if (p->z4c) {
    /* ev_theta, bssn.cc:834-848 */
    const long fth = cgo_num_fields(p->matter);
    out[fth] = (0.5 * bd->alpha * (bd->ricci + 2.0 / 3.0 * PW2(bd->K + 2.0 * bd->theta) - bd->AijAij - 16.0 * CG_PI * (bd->r)) -
                bd->alpha * k1 * (2.0 + k2) * bd->theta) -
               ko_diss(s, i, j, k, a + fth * N);
  }
}

/* ------------------------------------------------------------------ */
/* Dust: components/dust_fluid/dust.cc                                 */
/* ------------------------------------------------------------------ */

/* Dust::populateDerivedFields, dust.cc:109-158 (with getDustData :177-200) */
static void dust_populate(sim_t *s) {
  const long N = s->pts;
  long ii;
#pragma omp parallel for schedule(static)
  for (ii = 0; ii < s->nx; ++ii) {
    bd_t bd;
    for (long j = 0; j < s->ny; ++j)
      for (long k = 0; k < s->nz; ++k) {
        const long idx = IDX(s, ii, j, k);
        set_bd(s, ii, j, k, &bd);
        const double D = s->reg_a[F_D * N + idx];
        const double S1 = s->reg_a[F_S1 * N + idx], S2 = s->reg_a[F_S2 * N + idx],
                     S3 = s->reg_a[F_S3 * N + idx];
        const double *gi = bd.gi;
        const double em4phi = exp(-4.0 * bd.phi);
        const double e6phi = exp(6.0 * bd.phi);
        const double giIJSISJ =
            em4phi * (gi[0] * S1 * S1 + gi[3] * S2 * S2 + gi[5] * S3 * S3 +
                      2.0 * (gi[1] * S1 * S2 + gi[2] * S1 * S3 + gi[4] * S2 * S3));
        const double W = sqrt(1.0 + giIJSISJ / D / D);
        const double v1 = em4phi / e6phi * (gi[0] * S1 + gi[1] * S2 + gi[2] * S3);
        const double v2 = em4phi / e6phi * (gi[1] * S1 + gi[3] * S2 + gi[4] * S3);
        const double v3 = em4phi / e6phi * (gi[2] * S1 + gi[4] * S2 + gi[5] * S3);
        double *u = s->dust;
        u[U_ADV1 * N + idx] = bd.alpha * D * v1;
        u[U_ADV2 * N + idx] = bd.alpha * D * v2;
        u[U_ADV3 * N + idx] = bd.alpha * D * v3;
        u[U_AS1V1 * N + idx] = bd.alpha * S1 * v1;
        u[U_AS1V2 * N + idx] = bd.alpha * S1 * v2;
        u[U_AS1V3 * N + idx] = bd.alpha * S1 * v3;
        u[U_AS2V1 * N + idx] = bd.alpha * S2 * v1;
        u[U_AS2V2 * N + idx] = bd.alpha * S2 * v2;
        u[U_AS2V3 * N + idx] = bd.alpha * S2 * v3;
        u[U_AS3V1 * N + idx] = bd.alpha * S3 * v1;
        u[U_AS3V2 * N + idx] = bd.alpha * S3 * v2;
        u[U_AS3V3 * N + idx] = bd.alpha * S3 * v3;
        const double *gm = bd.gamma;
        for (int d = 0; d < 3; ++d) {
          const double *dg = bd.dg[d];
          const double dp = bd.dphi[d];
          u[(U_S1SRC + d) * N + idx] =
              1.0 / 2.0 * bd.alpha * W * D * exp(4.0 * bd.phi) *
                  (v1 * v1 * (4.0 * gm[0] * dp + dg[0]) + v2 * v2 * (4.0 * gm[3] * dp + dg[3]) +
                   v3 * v3 * (4.0 * gm[5] * dp + dg[5]) +
                   2.0 * (v1 * v2 * (4.0 * gm[1] * dp + dg[1]) + v1 * v3 * (4.0 * gm[2] * dp + dg[2]) +
                          v2 * v3 * (4.0 * gm[4] * dp + dg[4]))) -
              W * D * bd.da[d];
        }
        const double e4phi = exp(4.0 * bd.phi);
        u[U_DETG * N + idx] = exp(6.0 * bd.phi);
        for (int q = 0; q < 6; ++q) u[(U_G11 + q) * N + idx] = e4phi * gm[q];
        u[U_W * N + idx] = W;
      }
  }
}

/* Dust::RKEvolve, dust.cc:160-174 (dt_D, dt_Si :203-224) */
static void dust_rkevolve(sim_t *s) {
  dust_populate(s);
  const long N = s->pts;
  const double *u = s->dust;
  long ii;
#pragma omp parallel for schedule(static)
  for (ii = 0; ii < s->nx; ++ii)
    for (long j = 0; j < s->ny; ++j)
      for (long k = 0; k < s->nz; ++k) {
        const long idx = IDX(s, ii, j, k);
        s->reg_c[F_D * N + idx] = deriv(s, ii, j, k, 1, u + U_ADV1 * N) + deriv(s, ii, j, k, 2, u + U_ADV2 * N) +
                                  deriv(s, ii, j, k, 3, u + U_ADV3 * N);
        for (int m = 0; m < 3; ++m) {
          const double *fl = u + (U_AS1V1 + 3 * m) * N;
          s->reg_c[(F_S1 + m) * N + idx] = deriv(s, ii, j, k, 1, fl) + deriv(s, ii, j, k, 2, fl + N) +
                                           deriv(s, ii, j, k, 3, fl + 2 * N) + u[(U_S1SRC + m) * N + idx];
        }
      }
}

/* BSSN::clearSrc (bssn.cc:310-319), Dust::addBSSNSrc (dust.cc:226-264),
 * Lambda::addBSSNSource (lambda.cc:26-43) */
static void dust_sources(sim_t *s) {
  const long N = s->pts;
  const double *u = s->dust, *a = s->reg_a;
  double *q = s->src;
  const double lam = s->p->lambda;
  long idx;
#pragma omp parallel for schedule(static)
  for (idx = 0; idx < N; ++idx) {
    const double W = u[U_W * N + idx], detg = u[U_DETG * N + idx];
    const double D = a[F_D * N + idx];
    const double S[3] = {a[F_S1 * N + idx], a[F_S2 * N + idx], a[F_S3 * N + idx]};
    double r = 0.0, Ssum = 0.0;
    r += W * D / detg;
    Ssum += D / detg * (W * W - 1.0) / W;
    q[Q_R * N + idx] = r;
    q[Q_S * N + idx] = Ssum;
    for (int m = 0; m < 3; ++m) q[(Q_S1 + m) * N + idx] = 0.0 + S[m] / detg;
    for (int I = 0; I < 3; ++I)
      for (int J = I; J < 3; ++J)
        q[(Q_STF11 + SYM[I][J]) * N + idx] =
            0.0 + (S[I] * S[J] / W / D / detg - 1.0 / 3.0 * u[(U_G11 + SYM[I][J]) * N + idx] * Ssum);
    q[Q_R * N + idx] += lam;
    q[Q_S * N + idx] += -3.0 * lam;
  }
}

/* BSSN::clearSrc, Static::addBSSNSrc (components/static/static.cc:19-36),
 * Lambda::addBSSNSource: the fixed density DIFFD (field 18) sources DIFFr
 * with the current DIFFphi and the FRW getters of this substep */
static void static_sources(sim_t *s) {
  const long N = s->pts;
  const double *a = s->reg_a;
  double *q = s->src;
  const double lam = s->p->lambda, phi_FRW = s->get_phi, rho_FRW = s->get_rho;
  long idx;
#pragma omp parallel for schedule(static)
  for (idx = 0; idx < N; ++idx) {
    for (int m = 0; m < Q_N; ++m) q[m * N + idx] = 0.0;
    const double phid = a[F_PHI * N + idx];
    q[Q_R * N + idx] += exp(-6.0 * (phid + phi_FRW)) * a[F_NBSSN * N + idx] + rho_FRW * expm1(-6.0 * phid);
    q[Q_R * N + idx] += lam;
    q[Q_S * N + idx] += -3.0 * lam;
  }
}

/* ------------------------------------------------------------------ */
/* Scalar: components/scalar/scalar.cc                                 */
/* ------------------------------------------------------------------ */

static double pot_V(const sim_t *s, double phi) {
  return s->p->potential == CGO_POT_QUADRATIC ? 0.5 * PW2(s->p->pot_mass) * PW2(phi) : s->p->pot_const;
}
static double pot_dV(const sim_t *s, double phi) {
  return s->p->potential == CGO_POT_QUADRATIC ? PW2(s->p->pot_mass) * phi : 0.0;
}

typedef struct {
  double phi, Pi, psi[3];
  double dphi[3], dPi[3], dpsi[3][3]; /* dpsi[d][m] = d_d psi_m */
} sd_t;

/* Scalar::getScalarData, scalar.cc:97-130 */
static void scalar_data(const sim_t *s, long i, long j, long k, sd_t *sd) {
  const long N = s->pts, idx = IDX(s, i, j, k);
  const double *a = s->reg_a;
  sd->phi = a[F_SPHI * N + idx];
  sd->Pi = a[F_SPI * N + idx];
  for (int m = 0; m < 3; ++m) sd->psi[m] = a[(F_SPSI1 + m) * N + idx];
  for (int d = 0; d < 3; ++d) sd->dphi[d] = deriv(s, i, j, k, d + 1, a + F_SPHI * N);
  for (int d = 0; d < 3; ++d) sd->dPi[d] = deriv(s, i, j, k, d + 1, a + F_SPI * N);
  for (int m = 0; m < 3; ++m)
    for (int d = 0; d < 3; ++d) sd->dpsi[d][m] = deriv(s, i, j, k, d + 1, a + (F_SPSI1 + m) * N);
}

/* Scalar::RKEvolvePt, scalar.cc:85-95 (dt_* :132-199) */
static void scalar_rhs(const sim_t *s, const bd_t *bd, const sd_t *sd, double *out) {
  const double *gi = bd->gi, *da = bd->da;
  const double al = bd->alpha;
  out[F_SPHI] = (-bd->alpha * sd->Pi);
  const double inner =
      gi[0] * (al * sd->dpsi[0][0] + sd->psi[0] * da[0]) + gi[1] * (al * sd->dpsi[0][1] + sd->psi[0] * da[1]) +
      gi[2] * (al * sd->dpsi[0][2] + sd->psi[0] * da[2]) + gi[1] * (al * sd->dpsi[1][0] + sd->psi[1] * da[0]) +
      gi[3] * (al * sd->dpsi[1][1] + sd->psi[1] * da[1]) + gi[4] * (al * sd->dpsi[1][2] + sd->psi[1] * da[2]) +
      gi[2] * (al * sd->dpsi[2][0] + sd->psi[2] * da[0]) + gi[4] * (al * sd->dpsi[2][1] + sd->psi[2] * da[1]) +
      gi[5] * (al * sd->dpsi[2][2] + sd->psi[2] * da[2]);
  double gterm[3];
  for (int I = 0; I < 3; ++I)
    gterm[I] = (bd->Gam[I] - 2.0 * (gi[SYM[I][0]] * bd->dphi[0] + gi[SYM[I][1]] * bd->dphi[1] +
                                    gi[SYM[I][2]] * bd->dphi[2]));
  out[F_SPI] = (-exp(-4.0 * bd->phi) * (inner) +
                bd->alpha * ((gterm[0]) * sd->psi[0] * exp(-4.0 * bd->phi) + (gterm[1]) * sd->psi[1] * exp(-4.0 * bd->phi) +
                             (gterm[2]) * sd->psi[2] * exp(-4.0 * bd->phi) + bd->K * sd->Pi + pot_dV(s, sd->phi)));
  for (int m = 0; m < 3; ++m) out[F_SPSI1 + m] = (-bd->alpha * sd->dPi[m] - sd->Pi * da[m]);
}

/* BSSN::clearSrc + Scalar::addBSSNSource, scalar.cc:201-260 */
static void scalar_sources(sim_t *s) {
  const long N = s->pts;
  double *q = s->src;
  long idx;
#pragma omp parallel for schedule(static)
  for (idx = 0; idx < N; ++idx)
    for (int m = 0; m < Q_N; ++m) q[m * N + idx] = 0.0;
  /* set_bd_values reads the sources; the scalar pass reads them while they
   * are zero, exactly as the reference does after clearSrc. */
  double *nq = (double *)malloc(sizeof(double) * Q_N * N);
  long ii;
#pragma omp parallel for schedule(static)
  for (ii = 0; ii < s->nx; ++ii) {
    bd_t bd;
    sd_t sd;
    for (long j = 0; j < s->ny; ++j)
      for (long k = 0; k < s->nz; ++k) {
        const long idx2 = IDX(s, ii, j, k);
        set_bd(s, ii, j, k, &bd);
        scalar_data(s, ii, j, k, &sd);
        const double *gi = bd.gi, *dp = sd.dphi;
        const double nmudmuphi = ((-bd.alpha * sd.Pi)) / bd.alpha;
        const double diphidiphi = (gi[0] * dp[0] * dp[0] + gi[3] * dp[1] * dp[1] + gi[5] * dp[2] * dp[2] +
                                   2.0 * (gi[1] * dp[0] * dp[1] + gi[2] * dp[0] * dp[2] + gi[4] * dp[1] * dp[2]));
        const double V = pot_V(s, sd.phi);
        nq[Q_R * N + idx2] = 0.0 + (0.5 * nmudmuphi * nmudmuphi + 0.5 * exp(-4.0 * bd.phi) * diphidiphi + V);
        nq[Q_S * N + idx2] =
            0.0 + (3.0 / 2.0 * nmudmuphi * nmudmuphi - 0.5 * exp(-4.0 * bd.phi) * diphidiphi - 3.0 * V);
        for (int m = 0; m < 3; ++m) nq[(Q_S1 + m) * N + idx2] = 0.0 + -nmudmuphi * dp[m];
        for (int I = 0; I < 3; ++I)
          for (int J = I; J < 3; ++J)
            nq[(Q_STF11 + SYM[I][J]) * N + idx2] =
                0.0 + (dp[I] * dp[J] - bd.gamma[SYM[I][J]] / 3.0 * diphidiphi);
      }
  }
  memcpy(q, nq, sizeof(double) * Q_N * N);
  free(nq);
}

/* ------------------------------------------------------------------ */
/* FRW reference integrator, utils/FRW.h                              */
/* ------------------------------------------------------------------ */
#define PI_L 3.141592653589793238462643383279502884L

static void frw_set_gets(sim_t *s, double phi, double K, const double *rho) {
  s->get_phi = phi;
  s->get_K = K;
  s->get_rho = 0.0;
  s->get_S = 0.0;
  for (int n = 0; n < s->p->nfluids; ++n) {
    s->get_rho += rho[n];
    s->get_S += 3.0 * rho[n] * s->p->fluid_w[n];
  }
}

/* FRW::P1_step / P2_step / P3_step / RK_total_step, utils/FRW.h:94-254 */
static void frw_stage(sim_t *s, int n, double h) {
  const int nf = s->p->nfluids;
  const double *w = s->p->fluid_w;
  double K_in = s->frw_K, rho_in[CGO_MAX_FLUIDS];
  if (n == 1) {
    for (int m = 0; m < nf; ++m) rho_in[m] = s->fl_rho[m];
  } else {
    const double c = n == 4 ? h : h / 2.0;
    const int prev = n - 2;
    K_in = s->frw_K + c * s->K_K[prev];
    for (int m = 0; m < nf; ++m) rho_in[m] = s->fl_rho[m] + c * s->fl_K[prev][m];
  }
  s->phi_K[n - 1] = -1.0 * K_in / 6.0;
  double K_source = 0.0;
  for (int m = 0; m < nf; ++m) K_source += 4.0 * PI_L * rho_in[m] * (1.0 + 3.0 * w[m]);
  s->K_K[n - 1] = 1.0 / 3.0 * K_in * K_in + K_source;
  for (int m = 0; m < nf; ++m) s->fl_K[n - 1][m] = K_in * rho_in[m] * (1.0 + w[m]);
  if (n < 4) {
    const double c = n == 3 ? h : h / 2.0;
    double rho[CGO_MAX_FLUIDS];
    for (int m = 0; m < nf; ++m) rho[m] = s->fl_rho[m] + c * s->fl_K[n - 1][m];
    frw_set_gets(s, s->frw_phi + c * s->phi_K[n - 1], s->frw_K + c * s->K_K[n - 1], rho);
  } else {
    s->frw_phi += h / 6.0 * (s->phi_K[0] + 2.0 * s->phi_K[1] + 2.0 * s->phi_K[2] + s->phi_K[3]);
    s->frw_K += h / 6.0 * (s->K_K[0] + 2.0 * s->K_K[1] + 2.0 * s->K_K[2] + s->K_K[3]);
    for (int m = 0; m < nf; ++m)
      s->fl_rho[m] += h / 6.0 * (s->fl_K[0][m] + 2.0 * s->fl_K[1][m] + 2.0 * s->fl_K[2][m] + s->fl_K[3][m]);
    frw_set_gets(s, s->frw_phi, s->frw_K, s->fl_rho);
  }
}

void cgo_frw_evolve(double *state, const double *w, int nfluids, double h, int steps) {
  cgo_params p;
  memset(&p, 0, sizeof(p));
  p.nfluids = nfluids;
  for (int m = 0; m < nfluids; ++m) p.fluid_w[m] = w[m];
  sim_t s;
  memset(&s, 0, sizeof(s));
  s.p = &p;
  s.frw_phi = state[0];
  s.frw_K = state[1];
  for (int m = 0; m < nfluids; ++m) s.fl_rho[m] = state[2 + m];
  for (int st = 0; st < steps; ++st)
    for (int n = 1; n <= 4; ++n) frw_stage(&s, n, h);
  state[0] = s.frw_phi;
  state[1] = s.frw_K;
  for (int m = 0; m < nfluids; ++m) state[2 + m] = s.fl_rho[m];
}

/* ------------------------------------------------------------------ */
/* Grid reductions, utils/math.h:1359-1522                             */
/* ------------------------------------------------------------------ */

/* BSSN::setExtraFieldData, bssn.cc:165-170 */
static void extra_field_data(sim_t *s) {
  const long N = s->pts;
  const double *K = s->reg_a + F_K * N, *phi = s->reg_a + F_PHI * N, *r = s->src + Q_R * N;
  const double pf = s->get_phi;
  double kmin = K[0], sK = 0.0, sP = 0.0, sR = 0.0, vol = 0.0;
  long idx;
#pragma omp parallel for reduction(min : kmin) reduction(+ : sK, sP, sR, vol)
  for (idx = 0; idx < N; ++idx) {
    const double e = exp(6.0 * (phi[idx] + pf));
    if (K[idx] < kmin) kmin = K[idx];
    sK += e * K[idx];
    sP += e * phi[idx];
    sR += e * r[idx];
    vol += e;
  }
  vol = vol / N;
  s->K_min = kmin;
  s->K_avg = sK / N / vol;
  s->avg_vol = exp(6.0 * (sP / N / vol));
  s->rho_avg = sR / N / vol;
}

/* ------------------------------------------------------------------ */
/* Driver: RK4Register semantics (utils/RK4Register.h:164-222)         */
/* ------------------------------------------------------------------ */

/* BSSN::set_DIFFgamma_Aij_norm, bssn.cc:61-119, in place on "_a" */
static void normalize_a(sim_t *s) {
  const long N = s->pts;
  double *a = s->reg_a;
  long idx;
#pragma omp parallel for schedule(static)
  for (idx = 0; idx < N; ++idx) {
    double *g11 = a + F_G11 * N + idx, *g12 = a + F_G12 * N + idx, *g13 = a + F_G13 * N + idx;
    double *g22 = a + F_G22 * N + idx, *g23 = a + F_G23 * N + idx, *g33 = a + F_G33 * N + idx;
    double omd = -1.0 * (*g11 + *g22 + *g33 - PW2(*g12) - PW2(*g13) - PW2(*g23) + *g11 * *g22 + *g11 * *g33 +
                         *g22 * *g33 - PW2(*g23) * *g11 - PW2(*g13) * *g22 - PW2(*g12) * *g33 +
                         2.0 * *g12 * *g13 * *g23 + *g11 * *g22 * *g33);
    double t = -1.0 * expm1(log1p(-1.0 * omd) / 3.0);
    *g11 = (*g11 + t) / (1.0 - t);
    *g22 = (*g22 + t) / (1.0 - t);
    *g33 = (*g33 + t) / (1.0 - t);
    *g12 = (*g12) / (1.0 - t);
    *g13 = (*g13) / (1.0 - t);
    *g23 = (*g23) / (1.0 - t);
    double gi11 = 1.0 + *g22 + *g33 - PW2(*g23) + *g22 * *g33;
    double gi22 = 1.0 + *g11 + *g33 - PW2(*g13) + *g11 * *g33;
    double gi33 = 1.0 + *g11 + *g22 - PW2(*g12) + *g11 * *g22;
    double gi12 = *g13 * *g23 - *g12 * (1.0 + *g33);
    double gi13 = *g12 * *g23 - *g13 * (1.0 + *g22);
    double gi23 = *g12 * *g13 - *g23 * (1.0 + *g11);
    double *A11 = a + F_A11 * N + idx, *A12 = a + F_A12 * N + idx, *A13 = a + F_A13 * N + idx;
    double *A22 = a + F_A22 * N + idx, *A23 = a + F_A23 * N + idx, *A33 = a + F_A33 * N + idx;
    double trA = gi11 * *A11 + gi22 * *A22 + gi33 * *A33 + 2.0 * (gi12 * *A12 + gi13 * *A13 + gi23 * *A23);
    *A11 = (*A11 - 1.0 / 3.0 * (1.0 + *g11) * trA) / (1.0 - t);
    *A22 = (*A22 - 1.0 / 3.0 * (1.0 + *g22) * trA) / (1.0 - t);
    *A33 = (*A33 - 1.0 / 3.0 * (1.0 + *g33) * trA) / (1.0 - t);
    *A12 = (*A12 - 1.0 / 3.0 * *g12 * trA) / (1.0 - t);
    *A13 = (*A13 - 1.0 / 3.0 * *g13 * trA) / (1.0 - t);
    *A23 = (*A23 - 1.0 / 3.0 * *g23 * trA) / (1.0 - t);
  }
}

static int sim_init(sim_t *s, const cgo_params *p) {
  if (!p || p->nx < 1 || p->ny < 1 || p->nz < 1) return -1;
  if (p->order != 2 && p->order != 4 && p->order != 6 && p->order != 8) return -2;
  if (p->matter < 0 || p->matter > 3) return -3;
  if (p->nfluids < 0 || p->nfluids > CGO_MAX_FLUIDS) return -4;
  memset(s, 0, sizeof(*s));
  s->p = p;
  s->nx = p->nx;
  s->ny = p->ny;
  s->nz = p->nz;
  s->pts = s->nx * s->ny * s->nz;
  s->nf = cgo_num_fields(p->matter) + (p->z4c ? 1 : 0);
  const size_t n = (size_t)s->nf * s->pts;
  s->reg_p = (double *)calloc(n, sizeof(double));
  s->reg_a = (double *)calloc(n, sizeof(double));
  s->reg_c = (double *)calloc(n, sizeof(double));
  s->reg_f = (double *)calloc(n, sizeof(double));
  s->src = (double *)calloc((size_t)Q_N * s->pts, sizeof(double));
  s->dust = p->matter == CGO_DUST ? (double *)calloc((size_t)U_N * s->pts, sizeof(double)) : NULL;
  if (!s->reg_p || !s->reg_a || !s->reg_c || !s->reg_f || !s->src || (p->matter == CGO_DUST && !s->dust))
    return -5;
  s->frw_phi = p->frw_phi;
  s->frw_K = p->frw_K;
  for (int m = 0; m < p->nfluids; ++m) s->fl_rho[m] = p->fluid_rho[m];
  frw_set_gets(s, s->frw_phi, s->frw_K, s->fl_rho);
  return 0;
}

static void sim_free(sim_t *s) {
  free(s->reg_p);
  free(s->reg_a);
  free(s->reg_c);
  free(s->reg_f);
  free(s->src);
  free(s->dust);
}

/* BSSN::RKEvolve (bssn.cc:231-243) for every field, plus the scalar's
 * fused point loop (sims/scalar.cc:104-108) */
static void evolve_substep(sim_t *s) {
  const long N = s->pts;
  long ii;
#pragma omp parallel for schedule(static)
  for (ii = 0; ii < s->nx; ++ii) {
    bd_t bd;
    sd_t sd;
    double out[24];
    for (long j = 0; j < s->ny; ++j)
      for (long k = 0; k < s->nz; ++k) {
        const long idx = IDX(s, ii, j, k);
        set_bd(s, ii, j, k, &bd);
        bssn_rhs(s, ii, j, k, &bd, out);
        int nf = F_NBSSN;
        if (s->p->matter == CGO_SCALAR) {
          scalar_data(s, ii, j, k, &sd);
          scalar_rhs(s, &bd, &sd, out);
          nf = 23;
        } else if (s->p->matter == CGO_STATIC) {
          out[F_NBSSN] = 0.0;  /* DIFFD is not evolved: the register update keeps it */
          nf = 19;
        }
        for (int f = 0; f < nf; ++f) s->reg_c[f * N + idx] = out[f];
        if (s->p->z4c) s->reg_c[(long)(s->nf - 1) * N + idx] = out[s->nf - 1];
      }
  }
  if (s->p->matter == CGO_DUST) dust_rkevolve(s);
}

static void step_init(sim_t *s) {
  const long n = (long)s->nf * s->pts;
  long q;
  /* RK4Register::stepInit, RK4Register.h:164-173 */
#pragma omp parallel for schedule(static)
  for (q = 0; q < n; ++q) {
    s->reg_a[q] = s->reg_p[q];
    s->reg_f[q] = 0;
  }
  extra_field_data(s);
  if (s->p->normalize_metric) normalize_a(s);
  if (s->p->matter == CGO_DUST) {
    dust_populate(s);
    dust_sources(s);
  } else if (s->p->matter == CGO_SCALAR) {
    scalar_sources(s);
  } else if (s->p->matter == CGO_STATIC) {
    static_sources(s);
  }
}

/* RK4Register::K1..K4Finalize (RK4Register.h:175-222) with the a<->c swap */
static void finalize(sim_t *s, int n) {
  const long cnt = (long)s->nf * s->pts;
  const double dt = s->p->dt;
  double *p = s->reg_p, *c = s->reg_c, *f = s->reg_f;
  long q;
#pragma omp parallel for schedule(static)
  for (q = 0; q < cnt; ++q) {
    if (n == 1) {
      f[q] += dt * c[q] / 6.0;
      c[q] = p[q] + dt * c[q] / 2.0;
    } else if (n == 2) {
      f[q] += dt * c[q] / 3.0;
      c[q] = p[q] + dt * c[q] / 2.0;
    } else if (n == 3) {
      f[q] += dt * c[q] / 3.0;
      c[q] = p[q] + dt * c[q];
    } else {
      f[q] += dt * c[q] / 6.0 + p[q];
      c[q] = f[q];
      p[q] = f[q];
    }
  }
  double *t = s->reg_a;
  s->reg_a = s->reg_c;
  s->reg_c = t;
}

static void run_step(sim_t *s) {
  for (int n = 1; n <= 4; ++n) {
    if (n > 1) {
      if (s->p->matter == CGO_DUST)
        dust_sources(s);
      else if (s->p->matter == CGO_SCALAR)
        scalar_sources(s);
      else if (s->p->matter == CGO_STATIC)
        static_sources(s);
    }
    evolve_substep(s);
    /* BSSN::K{n}Finalize, bssn.cc:267-305: FRW stage, registers, reductions */
    frw_stage(s, n, s->p->dt);
    finalize(s, n);
    extra_field_data(s);
  }
}

int cgo_evolve(const cgo_params *p, double *fields, int steps, double *frw_out) {
  sim_t s;
  int rc = sim_init(&s, p);
  if (rc) {
    sim_free(&s);
    return rc;
  }
  memcpy(s.reg_p, fields, sizeof(double) * s.nf * s.pts);
  for (int st = 0; st < steps; ++st) {
    step_init(&s);
    run_step(&s);
  }
  memcpy(fields, s.reg_p, sizeof(double) * s.nf * s.pts);
  if (frw_out) {
    frw_out[0] = s.frw_phi;
    frw_out[1] = s.frw_K;
    for (int m = 0; m < p->nfluids; ++m) frw_out[2 + m] = s.fl_rho[m];
  }
  sim_free(&s);
  return 0;
}

int cgo_rhs(const cgo_params *p, const double *fields, double *rhs_out) {
  sim_t s;
  int rc = sim_init(&s, p);
  if (rc) {
    sim_free(&s);
    return rc;
  }
  memcpy(s.reg_p, fields, sizeof(double) * s.nf * s.pts);
  step_init(&s);
  evolve_substep(&s);
  memcpy(rhs_out, s.reg_c, sizeof(double) * s.nf * s.pts);
  sim_free(&s);
  return 0;
}

/* BSSN::momentumConstraintCalc / Scale (bssn.cc:1102-1136, BSSN_MI and
 * BSSN_MI_SCALE, bssn_macros.h:487-527) */
static void momentum(const sim_t *s, long i, long j, long k, const bd_t *bd, int I, double *val, double *scale) {
  const long N = s->pts;
  const double *a = s->reg_a, *gi = bd->gi, *A = bd->A, *dp = bd->dphi;
  const double e6 = exp(6.0 * bd->phi);
  const double t6 = gi[SYM[0][0]] * A[SYM[0][I]] * dp[0] + gi[SYM[1][0]] * A[SYM[1][I]] * dp[0] +
                    gi[SYM[2][0]] * A[SYM[2][I]] * dp[0] + gi[SYM[0][1]] * A[SYM[0][I]] * dp[1] +
                    gi[SYM[1][1]] * A[SYM[1][I]] * dp[1] + gi[SYM[2][1]] * A[SYM[2][I]] * dp[1] +
                    gi[SYM[0][2]] * A[SYM[0][I]] * dp[2] + gi[SYM[1][2]] * A[SYM[1][I]] * dp[2] +
                    gi[SYM[2][2]] * A[SYM[2][I]] * dp[2];
  double dA[3][3]; /* dA[X][d] = d_d A_{X I} */
  for (int X = 0; X < 3; ++X)
    for (int d = 0; d < 3; ++d) dA[X][d] = deriv(s, i, j, k, d + 1, a + (F_A11 + SYM[X][I]) * N);
  double tD = 0.0;
  for (int X = 0; X < 3; ++X)
    for (int d = 0; d < 3; ++d) {
      double u = gi[SYM[X][d]] * dA[X][d];
      tD = (X == 0 && d == 0) ? u : tD + u;
    }
  tD = tD - bd->Gammad[0] * A[SYM[0][I]] - bd->Gammad[1] * A[SYM[1][I]] - bd->Gammad[2] * A[SYM[2][I]];
  for (int X = 0; X < 3; ++X)
    for (int Y = 0; Y < 3; ++Y) tD = tD - bd->GL[Y][SYM[X][I]] * bd->Acont[SYM[Y][X]];
  const double theta_d = bd->dtheta[I];
  *val = e6 * (-2.0 / 3.0 * bd->dK[I] - 8 * CG_PI * (bd->src[Q_S1 + I]) - 2.0 / 3.0 * 2.0 * theta_d + 6.0 * (t6) + (tD));
  *scale = e6 * (fabs(2.0 / 3.0 * bd->dK[I]) + fabs(8 * CG_PI * (bd->src[Q_S1 + I])) +
                 fabs(2.0 / 3.0 * 2.0 * theta_d) + 6.0 * fabs(t6) + fabs(tD));
}

/* io_bssn_dump_statistics (IO/io.cc:8-14, 386-403) after the step
 * initialisation: volume-weighted mean and standard deviation of DIFFphi,
 * DIFFK, DIFFr and ricci (conformal_average / conformal_standard_deviation,
 * utils/math.h:1403-1470, weights exp(6 (DIFFphi + phi_FRW))), then
 * volume_average (math.h:1382-1393).  ricci as set_bd_values computes it for
 * prepBSSNOutput (sims/sim.cc:214-225). */
int cgo_field_statistics(const cgo_params *p, const double *fields, double *out) {
  sim_t s;
  int rc = sim_init(&s, p);
  if (rc) {
    sim_free(&s);
    return rc;
  }
  memcpy(s.reg_p, fields, sizeof(double) * s.nf * s.pts);
  step_init(&s);
  const long N = s.pts;
  double *ricci = (double *)malloc(sizeof(double) * N);
  long ii;
#pragma omp parallel for schedule(static)
  for (ii = 0; ii < s.nx; ++ii) {
    bd_t bd;
    for (long j = 0; j < s.ny; ++j)
      for (long k = 0; k < s.nz; ++k) {
        set_bd(&s, ii, j, k, &bd);
        ricci[IDX(&s, ii, j, k)] = bd.ricci;
      }
  }
  const double *f[4] = {s.reg_a + F_PHI * N, s.reg_a + F_K * N, s.src + Q_R * N, ricci};
  const double *phi = s.reg_a + F_PHI * N;
  double vol = 0.0;
  for (long q = 0; q < N; ++q) vol += exp(6.0 * (phi[q] + s.frw_phi));
  vol /= N;
  for (int m = 0; m < 4; ++m) {
    double sum = 0.0;
    for (long q = 0; q < N; ++q) sum += exp(6.0 * (phi[q] + s.frw_phi)) * f[m][q];
    const double avg = sum / N / vol;
    double var = 0.0;
    for (long q = 0; q < N; ++q) var += exp(6.0 * (phi[q] + s.frw_phi)) * PW2(avg - f[m][q]);
    out[2 * m] = avg;
    out[2 * m + 1] = sqrt(var / (N - 1) / vol);
  }
  out[8] = vol;
  free(ricci);
  sim_free(&s);
  return 0;
}

int cgo_constraints(const cgo_params *p, const double *fields, double *Hv, double *Mv, double *Gv, double *Av,
                    double *Sv) {
  sim_t s;
  int rc = sim_init(&s, p);
  if (rc) {
    sim_free(&s);
    return rc;
  }
  memcpy(s.reg_p, fields, sizeof(double) * s.nf * s.pts);
  step_init(&s);
  const long N = s.pts;
  /* per-point values: 5 constraints x (val, scale, scaled) */
  double *pv = (double *)malloc(sizeof(double) * 15 * N);
  double H_L2 = 0, M_L2 = 0;
  double dx = p->dx;
  long ii;
#pragma omp parallel for schedule(static) reduction(+ : H_L2, M_L2)
  for (ii = 0; ii < s.nx; ++ii) {
    bd_t bd;
    for (long j = 0; j < s.ny; ++j)
      for (long k = 0; k < s.nz; ++k) {
        const long idx = IDX(&s, ii, j, k);
        set_bd(&s, ii, j, k, &bd);
        const double *gi = bd.gi, *A = bd.A, *g = bd.g;
        double v[5], sc[5];
        /* hamiltonianConstraintCalc/Scale, bssn.cc:1073-1100 */
        v[0] = bd.H;
        sc[0] = (exp(5.0 * bd.phi) / 8.0) *
                sqrt(PW2(bd.ricci) + PW2(bd.AijAij) + PW2(2.0 / 3.0 * PW2(bd.K + 2.0 * 0.0)) + PW2(16.0 * CG_PI * bd.r));
        /* momentum (vector magnitude), BSSN_COMPUTE_CONSTRAINT_STAT_VARS_VEC */
        double mv[3], ms[3];
        for (int I = 0; I < 3; ++I) momentum(&s, ii, j, k, &bd, I, &mv[I], &ms[I]);
        v[1] = sqrt(PW2(mv[0]) + PW2(mv[1]) + PW2(mv[2]));
        sc[1] = sqrt(PW2(ms[0]) + PW2(ms[1]) + PW2(ms[2]));
        /* christoffel constraint, BSSN_GI_CALC / BSSN_GI_SCALE (bssn_macros.h:530-536) */
        double gv[3], gs[3];
        for (int I = 0; I < 3; ++I) {
          const double *G = bd.G[I];
          gv[I] = bd.Gam[I] - gi[0] * G[0] - gi[3] * G[3] - gi[5] * G[5] - 2.0 * (gi[1] * G[1] + gi[2] * G[2] + gi[4] * G[4]);
          gs[I] = fabs(bd.Gam[I]) +
                  fabs(gi[0] * G[0] - gi[3] * G[3] - gi[5] * G[5] - 2.0 * (gi[1] * G[1] + gi[2] * G[2] + gi[4] * G[4]));
        }
        v[2] = sqrt(PW2(gv[0]) + PW2(gv[1]) + PW2(gv[2]));
        sc[2] = sqrt(PW2(gs[0]) + PW2(gs[1]) + PW2(gs[2]));
        /* AijTFConstraintCalc/Scale, bssn.cc:1182-1192 */
        v[3] = gi[0] * A[0] + gi[3] * A[3] + gi[5] * A[5] + 2.0 * (gi[1] * A[1] + gi[2] * A[2] + gi[4] * A[4]);
        sc[3] = fabs(gi[0] * A[0]) + fabs(gi[3] * A[3]) + fabs(gi[5] * A[5]) +
                2.0 * (fabs(gi[1] * A[1]) + fabs(gi[2] * A[2]) + fabs(gi[4] * A[4]));
        /* unitDetConstraintCalc/Scale, bssn.cc:1199-1219 */
        v[4] = fabs(g[0] + g[3] + g[5] - PW2(g[1]) - PW2(g[2]) - PW2(g[4]) + g[0] * g[3] + g[0] * g[5] + g[3] * g[5] -
                    PW2(g[4]) * g[0] - PW2(g[2]) * g[3] - PW2(g[1]) * g[5] + 2.0 * g[1] * g[2] * g[4] + g[0] * g[3] * g[5]);
        sc[4] = (fabs(g[0]) + fabs(g[3]) + fabs(g[5]) + PW2(g[1]) + PW2(g[2]) + PW2(g[4]) + fabs(g[0] * g[3]) +
                 fabs(g[0] * g[5]) + fabs(g[3] * g[5]) + PW2(g[4]) * g[0] + PW2(g[2]) * g[3] + PW2(g[1]) * g[5] +
                 2.0 * fabs(g[1] * g[2] * g[4]) + fabs(g[0] * g[3] * g[5]));
        for (int c = 0; c < 5; ++c) {
          pv[(3 * c + 0) * N + idx] = v[c];
          pv[(3 * c + 1) * N + idx] = sc[c];
          pv[(3 * c + 2) * N + idx] = v[c] / sc[c];
        }
        H_L2 += v[0] * v[0] * dx * dx * dx;
        M_L2 += v[1] * v[1] * dx * dx * dx;
      }
  }
  double *outs[5] = {Hv, Mv, Gv, Av, Sv};
  for (int c = 0; c < 5; ++c) {
    const double *val = pv + (3 * c) * N, *sca = pv + (3 * c + 1) * N, *scd = pv + (3 * c + 2) * N;
    double mean = 0, mean_scale = 0, mean_scaled = 0, mx = 0, mx_s = 0;
    long q;
#pragma omp parallel for reduction(+ : mean, mean_scale, mean_scaled) reduction(max : mx, mx_s)
    for (q = 0; q < N; ++q) {
      mean += val[q];
      mean_scale += sca[q];
      mean_scaled += scd[q];
      if (fabs(val[q]) > mx) mx = fabs(val[q]);
      if (fabs(scd[q]) > mx_s) mx_s = fabs(scd[q]);
    }
    mean /= N;
    mean_scaled /= N;
    double sd = 0, sd_s = 0;
#pragma omp parallel for reduction(+ : sd, sd_s)
    for (q = 0; q < N; ++q) {
      sd += PW2(val[q] - mean);
      sd_s += PW2(scd[q] - mean_scaled);
    }
    sd = sqrt(sd / (N - 1.0));
    sd_s = sqrt(sd_s / (N - 1.0));
    double *o = outs[c];
    o[0] = mean;
    o[1] = sd;
    o[2] = mx;
    o[3] = mean_scale;
    o[4] = mean_scaled;
    o[5] = sd_s;
    o[6] = mx_s;
  }
  Hv[7] = sqrt(H_L2);
  Mv[7] = sqrt(M_L2);
  free(pv);
  sim_free(&s);
  return 0;
}
