/*
 * cg_oracle.h -- CPU restatement of CosmoGRaPH's BSSN (+dust/+scalar) RK4
 * evolution path, in plain C with OpenMP.  TEST INFRASTRUCTURE: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker or the timed CPU baseline, never as the product path.
 *
 * Unlike the reference, grid size and stencil order are run-time parameters.
 * Every expression follows the reference's operand order so that, built
 * without FMA contraction, it reproduces the reference build bit for bit
 * except where libm calls differ.  Parity is pinned against the reference's
 * own sources (oracle/build_ref.py) through the fixtures in tests/golden/.
 */
#ifndef CG_ORACLE_H
#define CG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* matter models */
#define CGO_VACUUM 0
#define CGO_DUST 1
#define CGO_SCALAR 2
#define CGO_STATIC 3  /* the static sims' matter: a fixed density DIFFD (components/static/static.cc) */

/* lapse gauges (components/bssn/BSSNGaugeHandler.h:95-110) */
#define CGO_LAPSE_STATIC 0
#define CGO_LAPSE_HARMONIC 1
#define CGO_LAPSE_CONFORMAL_FLRW 2
#define CGO_LAPSE_CONFORMAL_SYNC 3
#define CGO_LAPSE_ANHARMONIC 4
#define CGO_LAPSE_ONE_PLUS_LOG 5
#define CGO_LAPSE_AWA_GAUGE_WAVE 6
#define CGO_LAPSE_AWA_SHIFTED_WAVE 7
#define CGO_LAPSE_DAMPED_WAVE 8

/* scalar potentials: the reference's constant potential
 * (components/scalar/scalar.cc:262-274) or V = m^2 phi^2 / 2 */
#define CGO_POT_CONST 0
#define CGO_POT_QUADRATIC 1

#define CGO_MAX_FLUIDS 4

typedef struct {
  int nx, ny, nz;
  int order;            /* 2, 4, 6, 8 */
  int matter;           /* CGO_VACUUM / CGO_DUST / CGO_SCALAR / CGO_STATIC */
  int lapse;            /* CGO_LAPSE_* */
  int normalize_metric; /* bssn.cc:19 default 1 */
  int potential;        /* CGO_POT_* */
  double dx, dt;
  double lambda;        /* rho_Lambda added by Lambda::addBSSNSource */
  double ko_coeff;      /* KO_damping_coefficient (bssn.cc:15) */
  double a_adj_amp;     /* bssn.cc:16 */
  double k_damping_amp; /* bssn.cc:17 */
  double gd_c;          /* BSSNGaugeHandler.h:142 */
  double dw_mu_l, dw_p; /* BSSNGaugeHandler.h:139-141 */
  double pot_const;     /* V for CGO_POT_CONST (COSMO_CONST = 3e-4) */
  double pot_mass;      /* m for CGO_POT_QUADRATIC */
  /* FRW reference background (utils/FRW.h) */
  double frw_phi, frw_K;
  int nfluids;
  double fluid_rho[CGO_MAX_FLUIDS], fluid_w[CGO_MAX_FLUIDS];
  int z4c;              /* USE_Z4c_DAMPING (cosmo_macros.h:91-100): the field theta
                           after the matter fields, damping amplitudes 0.5, 0.1 */
} cgo_params;

/* Number of fields of a matter model: 18, 22, 23, or 19 (static: the 18
 * BSSN fields and the fixed density DIFFD, which no substep changes). */
int cgo_num_fields(int matter);

/* Advance `steps` RK4 steps.  `fields` holds the "_p" register of every
 * evolved field (cg_state.h order), nfields*nx*ny*nz doubles, updated in
 * place.  frw_out (may be NULL) receives phi, K, then the fluid densities.
 * Returns 0, or a negative code on invalid parameters. */
int cgo_evolve(const cgo_params *p, double *fields, int steps, double *frw_out);

/* Step initialisation followed by the first substep's right-hand side:
 * rhs_out receives the "_c" register of every field (nfields*N^3). */
int cgo_rhs(const cgo_params *p, const double *fields, double *rhs_out);

/* io_bssn_dump_statistics columns (IO/io.cc:8-14, 386-403) after the step
 * initialisation: {avg, stdev} of DIFFphi, DIFFK, DIFFr, ricci (volume
 * weighted), then the volume average; out[9]. */
int cgo_field_statistics(const cgo_params *p, const double *fields, double *out);

/* Step initialisation, then the constraint statistics of
 * BSSN::setConstraintCalcs (bssn.cc:965-1071): H[8], M[8], G[7], A[7], S[7]. */
int cgo_constraints(const cgo_params *p, const double *fields, double *H,
                    double *M, double *G, double *A, double *S);

/* FRW reference integrator alone (utils/FRW.h:94-254): `steps` RK4 steps of
 * size h; state = {phi, K, rho_1..rho_n}; w = equations of state. */
void cgo_frw_evolve(double *state, const double *w, int nfluids, double h, int steps);

/* Threads used by the OpenMP loops (0 = library default). */
void cgo_set_threads(int n);

#ifdef __cplusplus
}
#endif

#endif
