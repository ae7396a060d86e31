/*
 * cosmograph_b200.h -- C ABI of the B200-native BSSN (+dust / +scalar) RK4
 * evolution path for periodic boxes.
 *
 * The reference (CosmoGRaPH, unigrid) exposes this path as C++ classes that
 * its sim drivers call in a fixed order; it has no FFI layer.  Each entry
 * point below names the reference interface it replaces.  The C++ facade in
 * cosmograph_b200/host/ (BSSN, Dust, Scalar, Lambda, RK4Register) keeps the
 * reference's method names on top of these calls.
 *
 * Conventions
 *   - Every call returns CG_OK (0) or a negative CG_ERR_* code; the message of
 *     the last failure is available from cg_last_error().  No C++ exception
 *     crosses this boundary.
 *   - Host buffers are borrowed for the duration of a call only; device memory
 *     belongs to the context.
 *   - Field arrays are FP64, x-major with z fastest, NP_INDEX(i,j,k) =
 *     (nz*ny)*i + nz*j + k (reference cosmo_macros.h:118), one array per field
 *     in the order of cg_field_name().
 *   - A context is used by one host thread at a time; work is queued on the
 *     context's CUDA stream.
 */
#ifndef COSMOGRAPH_B200_H
#define COSMOGRAPH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CG_ABI_VERSION 1

/* status codes */
#define CG_OK 0
#define CG_ERR_INVALID (-1)   /* bad argument or unsupported option      */
#define CG_ERR_CUDA (-2)      /* CUDA runtime error                      */
#define CG_ERR_MEMORY (-3)    /* device allocation failed                */
#define CG_ERR_STATE (-4)     /* call out of sequence                    */
#define CG_ERR_NAN (-10)      /* NaN detected in DIFFphi (the reference's
                                 `throw 10`, sims/sim.cc:179-183)          */

/* matter models (reference simulation_type, cosmo.cc:51-81) */
#define CG_MATTER_VACUUM 0
#define CG_MATTER_DUST 1
#define CG_MATTER_SCALAR 2
#define CG_MATTER_STATIC 3  /* the static sims' matter: a fixed density DIFFD that
                               sources DIFFr (components/static/static.cc:19-36,
                               sims/static.cc); Static or ConformalFLRW lapse    */

/* lapse gauges (reference BSSNGaugeHandler lapse map,
 * components/bssn/BSSNGaugeHandler.h:95-110) */
#define CG_LAPSE_STATIC 0
#define CG_LAPSE_HARMONIC 1
#define CG_LAPSE_CONFORMAL_FLRW 2
#define CG_LAPSE_CONFORMAL_SYNC 3
#define CG_LAPSE_ANHARMONIC 4
#define CG_LAPSE_ONE_PLUS_LOG 5
#define CG_LAPSE_AWA_GAUGE_WAVE 6
#define CG_LAPSE_AWA_SHIFTED_WAVE 7
#define CG_LAPSE_DAMPED_WAVE 8

/* arithmetic of the substep kernel */
#define CG_PREC_FP64 0      /* FP64, reference operand order, no FMA contraction */
#define CG_PREC_FP64_FMA 1  /* FP64 with FMA contraction                          */
#define CG_PREC_MIXED 2     /* FP32 perturbations about an FP64 uniform background,
                               FP32 stencils and right-hand side, FP64 RK registers
                               (vacuum, dust or scalar; every lapse; Kreiss-Oliger;
                               a_adj_amp / k_damping_amp; trivial FRW reference;
                               no Z4c or shift)                                     */

/* shift gauges (BSSNGaugeHandler.h:113-134); a box with a shift carries the
 * reference's USE_BSSN_SHIFT and USE_GAMMA_DRIVER fields */
#define CG_SHIFT_NONE 0             /* no shift fields                           */
#define CG_SHIFT_STATIC 1           /* "Static": beta^i fixed (advection stays)  */
#define CG_SHIFT_GAMMA_DRIVER 2     /* "GammaDriver": d_t beta^i = B^i           */
#define CG_SHIFT_DAMPED_WAVE 3      /* "DampedWave"                              */
#define CG_SHIFT_AWA_SHIFTED_WAVE 4 /* "AwAShiftedWave"                          */
#define CG_SHIFT_AIJ_DRIVER 5       /* "AijDriverShift"                          */

/* scalar potentials */
#define CG_POT_CONST 0      /* V = pot_const, dV = 0 (components/scalar/scalar.cc:262-274) */
#define CG_POT_QUADRATIC 1  /* V = m^2 phi^2 / 2                                            */

/* status flags (cg_status) */
#define CG_STATUS_NAN 1u        /* NaN in DIFFphi after a step          */
#define CG_STATUS_NONFINITE 2u  /* NaN or Inf in any evolved field      */
#define CG_STATUS_TILE_TIMEOUT 4u /* a TMA tile copy did not complete in
                                     about a second; the substep's output
                                     is not valid                        */

typedef struct cg_ctx cg_ctx;

/* One periodic box: the reference's compile-time switches
 * (cosmo_macros.h:12-84) and run-time config keys (components/bssn/bssn.cc:15-22,
 * cosmo.cc:41-42) as plain fields. */
typedef struct {
  int nx, ny, nz;          /* grid points per axis (each >= stencil_order/2 + 1) */
  int stencil_order;       /* 2, 4, 6 or 8 (STENCIL_ORDER)                       */
  int matter;              /* CG_MATTER_*                                        */
  int lapse;               /* CG_LAPSE_*                                         */
  int precision;           /* CG_PREC_*                                          */
  int normalize_metric;    /* config normalize_metric (default 1)                */
  int potential;           /* CG_POT_* (scalar matter only)                      */
  int x_ghost;             /* 0: periodic box.  g > 0: an x-slab of a larger
                              box; its first and last g planes are ghost planes
                              that the caller refreshes from the neighbouring
                              slabs before every substep (cg_substep_input);
                              kernels update the nx - 2g interior planes only.
                              Lapses with K_avg take it from the caller
                              (cg_set_kavg); FP32-mixed slabs of one box share
                              a background (cg_set_background); g a
                              multiple of 4, >= the stencil radius (and the
                              Kreiss-Oliger radius), nx - 2g a positive
                              multiple of 4.                                   */
  double dx, dt;           /* grid spacing and time step                          */
  double lambda;           /* rho_Lambda (Lambda::setLambda)                      */
  double ko_coeff;         /* KO_damping_coefficient (orders 2 and 8; FP64 only)   */
  double a_adj_amp;        /* config a_adj_amp                                    */
  double k_damping_amp;    /* config k_damping_amp                                */
  double gd_c;             /* config gd_c (OnePlusLog), default 1                 */
  double dw_mu_l, dw_p;    /* config dw_mu_l, dw_p (DampedWave)                   */
  double pot_const;        /* V for CG_POT_CONST (reference COSMO_CONST = 3e-4)    */
  double pot_mass;         /* m for CG_POT_QUADRATIC                              */
  double frw_phi, frw_K;   /* FRW reference background (utils/FRW.h:15-16)         */
  int nfluids;             /* FRW fluids (FRW::addFluid, utils/FRW.h:60-76), <= 4  */
  int z4c;                 /* 1: Z4c damping (the reference's USE_Z4c_DAMPING,
                              cosmo_macros.h:91-100, damping amplitudes 0.5 and
                              0.1): the constraint field theta is evolved and
                              stored after the matter fields (cg_num_fields + 1
                              fields); FP64 precisions only                    */
  double fluid_rho[4], fluid_w[4];
  int shift;               /* CG_SHIFT_*.  Not CG_SHIFT_NONE: the shift beta^i,
                              the Gamma-driver's B^i and expN (the reference
                              built with USE_BSSN_SHIFT and USE_GAMMA_DRIVER,
                              cosmo_macros.h:43-50) are evolved and stored
                              after the matter fields as beta1..3, auxB1..3,
                              expN (cg_num_fields + 7 fields), every field is
                              advected with upwinded stencils (the reference
                              defines them for orders 2 and 4; zero at 6 and
                              8).  CG_PREC_FP64 only; vacuum, dust or scalar;
                              no Z4c, no x-slab; >= 4 points per axis        */
  int gauge_wave_dir;      /* config gauge_wave_dir (AwAShiftedWave), default 1 */
  double gd_eta;           /* config gd_eta (B^i damping), default 0            */
  double dw_mu_s;          /* config dw_mu_s (DampedWave shift), default 0      */
  double k_driver_coeff;   /* config k_driver_coeff (AijDriverShift), 0.04      */
} cg_box_desc;

/* Fill a descriptor with the reference's defaults (Harmonic lapse, order 8,
 * dust, normalize_metric = 1, dx = 1/N, dt = 0.1 dx). */
void cg_box_desc_default(cg_box_desc *d, int n);

/* Create a context holding nboxes boxes (BSSN::BSSN + Dust::Dust / Scalar::Scalar
 * allocation, components/bssn/bssn.cc:13-44, components/dust_fluid/dust.cc:15-44).
 * Every field of every register starts at zero (BSSN::init, bssn.cc:126-144). */
int cg_create(const cg_box_desc *boxes, int nboxes, cg_ctx **out);

/* Release the context and its device memory. */
int cg_destroy(cg_ctx *ctx);

/* Queue all work on `stream` (a cudaStream_t; NULL = the context's own). */
int cg_set_stream(cg_ctx *ctx, void *stream);
int cg_get_stream(cg_ctx *ctx, void **stream);

/* Number of fields (18 vacuum, 22 dust, 23 scalar, 19 static) and their names
 * (BSSN_APPLY_TO_FIELDS order, bssn_macros.h:77-95, then D,S1,S2,S3,
 * phi,Pi,psi1,psi2,psi3, or the static density DIFFD, which no substep
 * changes). */
int cg_num_fields(int matter);
const char *cg_field_name(int matter, int field);

/* Copy the "_p" register of every field of one box from / to host memory;
 * count = nfields*nx*ny*nz doubles.  Replaces filling / reading
 * RK4Register::_array_p through BSSN::fields (bssn.cc:30-39). Synchronous. */
int cg_upload_state(cg_ctx *ctx, int box, const double *host, size_t count);
int cg_download_state(cg_ctx *ctx, int box, double *host, size_t count);

/* Same, asynchronous on the context's stream (host memory should be pinned). */
int cg_upload_state_async(cg_ctx *ctx, int box, const double *host, size_t count);
int cg_download_state_async(cg_ctx *ctx, int box, double *host, size_t count);

/* Download the box's "_p" registers into host_out and upload host_in as the
 * new "_p", asynchronously: the download follows the work queued so far on
 * the context's stream and runs field by field on a second stream, and each
 * field is uploaded (on the context's stream) as soon as it has been
 * downloaded, so the two directions overlap.  Both buffers pinned, count as
 * for cg_upload_state; work queued afterwards on the context's stream sees
 * the new state, and host_out is complete once that stream reaches it (e.g.
 * cg_synchronize).  No reference counterpart: streaming boxes through one
 * GPU (the reference evolves one box per process).
 *
 * When host_in was handed to cg_prefetch_state_async for this box before,
 * the exchange is staged instead: the state is copied on the device into a
 * staging buffer and downloaded from there on the second stream while later
 * work runs, and the prefetched input is copied on the device into the
 * registers.  host_out is then complete after cg_synchronize. */
int cg_exchange_state_async(cg_ctx *ctx, int box, double *host_out, const double *host_in, size_t count);

/* Start copying host_in (pinned, count as for cg_upload_state) into a device
 * staging buffer of the box at once, on a stream of its own, so that the copy
 * overlaps the work queued on the context's stream.  The next
 * cg_exchange_state_async of this box with the same host_in takes its input
 * from there.  host_in must stay unchanged until the context's stream has
 * passed that exchange.  The first call allocates the staging buffers (two
 * copies of the state).  No reference counterpart. */
int cg_prefetch_state_async(cg_ctx *ctx, int box, const double *host_in, size_t count);

/* One register of one field: reg = 'p', 'a' (current substep input), 'f'.
 * Replaces BSSN::fields["<name>_<reg>"] access (bssn.cc:30-39). Synchronous.
 * On a CG_PREC_MIXED box 'a' is held as an FP32 perturbation about a uniform
 * FP64 background: a download returns background + perturbation in FP64, an
 * upload is rejected (CG_ERR_INVALID). */
int cg_upload_field(cg_ctx *ctx, int box, int field, char reg, const double *host, size_t n);
int cg_download_field(cg_ctx *ctx, int box, int field, char reg, double *host, size_t n);

/* Device pointer of a register block of one box (nfields arrays of pts
 * doubles): reg = 'p' or 'f'.  For callers that keep their data on the GPU. */
int cg_device_register(cg_ctx *ctx, int box, char reg, double **dptr);

/* BSSN::stepInit (bssn.cc:219-226) + Dust::stepInit (dust.cc:65-72) +
 * Scalar::stepInit for every box: builds the first substep's input from _p. */
int cg_step_init(cg_ctx *ctx);

/* Substep n = 1..4 for every box: sources, BSSN and matter RHS and the
 * register update of RK4Register::K{n}Finalize in one fused kernel
 * (replaces BSSN::RKEvolve + Dust::RKEvolve / Scalar::RKEvolvePt +
 * BSSN::K{n}Finalize + Dust::K{n}Finalize, sims/dust.cc:114-161,
 * sims/scalar.cc:97-151).  Substeps must be called in order after
 * cg_step_init. */
int cg_rk_stage(cg_ctx *ctx, int n);

/* nsteps full RK4 steps for every box (stepInit + 4 substeps each; the
 * reference's DustSim::runStep minus output, sims/dust.cc:163-169).
 * Asynchronous: returns once the work is queued. */
int cg_step(cg_ctx *ctx, int nsteps);

/* Initial data on the GPU for a dust box: the reference's dust_ic_set_random
 * (components/dust_fluid/dust_ic.cc:23-140) in synchronous gauge from a
 * Gaussian random density contrast delta with P(k) ~ k^ns exp(-(k/cutoff)^2)
 * (k in units of the fundamental mode; cutoff <= 0: min(nx,ny,nz)/4), zero
 * mean and rms rms_delta, drawn from a counter-based generator seeded with
 * `seed`, or taken from `delta` (host, nx*ny*nz doubles) when it is not NULL.
 * Spectral inverse Laplacians on cuFFT (utils/Fourier.h:251-298), the box's
 * stencil order for derivatives, rho_Lambda = the box's lambda.  Writes the
 * _p register (every other field zero, FRW reference untouched) and resets
 * the box like cg_upload_state.  CG_ERR_INVALID if the density turns
 * negative somewhere.  Synchronous; allocates its scratch (about 11 doubles
 * per point) for the duration of the call. */
int cg_ic_grf_dust(cg_ctx *ctx, int box, const double *delta, uint64_t seed, double rms_delta, double ns,
                   double cutoff);

/* Initial data on the GPU for a scalar box (the GRF scalar configuration;
 * the host version is cosmograph_b200.ics.grf_scalar): phi = phi0 + a
 * Gaussian random fluctuation with P(k) ~ k^-3 for k <= cutoff (units of the
 * fundamental mode; cutoff <= 0: min(nx,ny,nz)/4), else 0, zero mean and rms
 * `rms`, drawn from the counter-based generator seeded with `seed`, or taken
 * from `dphi` (host, nx*ny*nz doubles) when it is not NULL; Pi = 0, psi_i =
 * d_i phi with the box's stencils (the relation of the reference's wave data,
 * components/scalar/scalar_ic.cc:43-48), DIFFK = -sqrt(24 pi rho) with
 * rho = mass^2 phi^2 / 2 + |d phi|^2 / 2, every other field zero.  Writes the
 * _p register and resets the box like cg_upload_state.  Synchronous;
 * allocates its scratch for the duration of the call. */
int cg_ic_grf_scalar(cg_ctx *ctx, int box, const double *dphi, uint64_t seed, double phi0, double rms, double mass,
                     double cutoff);

/* Launch options (cg_set_option).  No reference counterpart: the reference
 * evolves one box per process.
 *   CG_OPT_BATCH     1 (default): boxes of a context with the same precision,
 *                    stencil order and matter model (up to 64 per group) share
 *                    one launch per substep; 0: one launch per box.  Change it
 *                    between steps only.
 *   CG_OPT_GRAPH     1: cg_step records its launches as one CUDA graph and
 *                    replays it (the graph is kept and updated in place while
 *                    nsteps stays the same); 0 (default): direct launches.
 *   CG_OPT_AUTOTUNE  1 (default): before the first substep of a batched group,
 *                    time its launch shapes (launch order of the boxes, one CTA
 *                    per brick, a persistent grid of 1, 2 or 4 waves, or the
 *                    boxes' own launches) and keep the fastest.  Results do
 *                    not depend on the choice.
 *   CG_OPT_GROUP_GRID the launch shape of groups the autotuner has not set:
 *                    0 (default) one CTA per brick, n > 0 a persistent grid of
 *                    n CTAs, -1 one launch per box.
 *   CG_OPT_TMA       1 (default): the substep kernels copy the halo tiles of
 *                    bricks away from the periodic wrap with the tensor memory
 *                    accelerator (FP64 boxes with even nz, mixed boxes with nz
 *                    a multiple of 4); 0: every tile is copied by the CTA's
 *                    threads.  Results are identical.  Change it between
 *                    steps only.
 *   CG_OPT_TMA_WAIT  clock cycles a CTA waits for one TMA tile copy before it
 *                    raises CG_STATUS_TILE_TIMEOUT (0, the default: 2e9, about
 *                    a second).  A late copy is still waited for, up to 2e9
 *                    cycles more, before its buffer is reused or the CTA
 *                    leaves, so a small value tests the reporting path without
 *                    leaving copies in flight.  Change it between steps only. */
#define CG_OPT_BATCH 1
#define CG_OPT_GRAPH 2
#define CG_OPT_AUTOTUNE 3
#define CG_OPT_GROUP_GRID 4
#define CG_OPT_TMA 5
#define CG_OPT_TMA_WAIT 6
int cg_set_option(cg_ctx *ctx, int option, int value);

/* Launch groups of the context (formed on first use), and for group g:
 * info[0] boxes, [1] bricks, [2] CTAs per launch (0: one per brick, -1: one
 * launch per box),
 * [3] launch order (0: box index, 1: largest box first), [4] tuned (0/1),
 * [5] the first box of the launch order.  n >= 6. */
int cg_num_groups(cg_ctx *ctx, int *n);
int cg_group_info(cg_ctx *ctx, int group, int *info, int n);

/* Wait for queued work (and staged downloads); returns CG_ERR_NAN if a NaN
 * appeared in DIFFphi. */
int cg_synchronize(cg_ctx *ctx);

/* Sticky error flags (CG_STATUS_*), OR-reduced on the device. */
int cg_status(cg_ctx *ctx, uint32_t *flags);

/* FRW background state of a box: out[0] = phi, out[1] = K, out[2..] = fluid
 * densities (utils/FRW.h:79-83). */
int cg_frw_state(cg_ctx *ctx, int box, double *out, int n);

/* Steps completed by a box since creation or the last upload. */
int cg_step_count(cg_ctx *ctx, int box, int64_t *steps);

/* Device arrays that the next cg_rk_stage of a box reads with stencils: the
 * substep input (nfields arrays of nx*ny*nz values, field-major, x slowest;
 * double, or float perturbations for CG_PREC_MIXED) and, for dust, its flux
 * primitives (7 arrays of the same type: alpha*D, alpha*S_1..3, v^1..3; NULL
 * otherwise).  Valid after cg_step_init and after each cg_rk_stage, until the
 * next one.  For an x-slab box (x_ghost = g) the caller refreshes planes
 * [0, g) and [nx-g, nx) of every array from the neighbouring slabs' interior
 * planes before each substep (and, FP64, before cg_constraints /
 * cg_field_statistics).  No reference counterpart: the reference evolves one
 * box per process. */
int cg_substep_input(cg_ctx *ctx, int box, void **input, void **flux);

/* FP32-mixed x-slabs of one box share one uniform background: out[0..4] =
 * sums over the box's updated points of K, phi, alpha, field 18 (D or the
 * scalar phi) and field 19 (Pi) of "_p", out[5] = their count (n >= 6);
 * cg_set_background gives a mixed box the background means (K, phi, alpha,
 * field 18, field 19; NULL: its own means again) for the next step
 * initialisation.  Synchronous.  No reference counterpart. */
int cg_background_sums(cg_ctx *ctx, int box, double *out, int n);

/* x-slabs whose lapse uses the grid average of K (ConformalFLRW, Anharmonic,
 * OnePlusLog; BSSN::setExtraFieldData, bssn.cc:165-213) take the whole box's
 * K_avg = sum w K / sum w, w = exp(6 (DIFFphi + phi_FRW)).  Before each
 * substep: cg_kavg_sums queues this slab's two sums over its updated points
 * of the next substep's input into device memory and returns their address;
 * the caller adds up every slab's sums (e.g. an all-reduce on the context's
 * stream) and passes the device address of the totals to cg_set_kavg, which
 * queues K_avg for the next cg_rk_stage (which refuses to run without it).
 * FP64 boxes.  No reference counterpart. */
int cg_kavg_sums(cg_ctx *ctx, int box, double **dsums);
int cg_set_kavg(cg_ctx *ctx, int box, const double *dsums);
int cg_set_background(cg_ctx *ctx, int box, const double *means, int n);

/* Constraint statistics of one box between steps (after cg_step_init or a
 * whole step), BSSN::setConstraintCalcs (components/bssn/bssn.cc:965-1071)
 * on the first-substep input with its sources: Hamiltonian (H), momentum
 * magnitude (M), Christoffel (G), trace of A (A) and unit-determinant (S)
 * constraints; each array holds mean, stdev, max|.|, sum of scales, mean of
 * scaled, stdev of scaled, max|scaled| (BSSN_STORE_CONSTRAINT_STAT_VARS,
 * bssn_macros.h:553-560); H[7], M[7] are the L2 norms sqrt(sum C^2 dx^3).
 * FP64, fixed-order (deterministic) reductions; scratch owned by the context.
 * Synchronous. */
int cg_constraints(cg_ctx *ctx, int box, double *H, double *M, double *G, double *A, double *S);

/* Field statistics of one box between steps, the columns of the reference's
 * "<dump_file>.dat.gz" (io_bssn_dump_statistics, IO/io.cc:8-14, 386-403): out
 * = {avg, stdev} of DIFFphi, DIFFK, DIFFr (the density source) and the Ricci
 * scalar (ricci_a, bssn.cc:663), each volume-weighted by exp(6 (DIFFphi +
 * phi_FRW)) (conformal_average / conformal_standard_deviation, utils/math.h:
 * 1403-1470), then volume_average(DIFFphi) (math.h:1382-1393); n_out >= 9.
 * Same state and sources as cg_constraints.  Synchronous. */
int cg_field_statistics(cg_ctx *ctx, int box, double *out, int n_out);

/* Volume-weighted grid average of a device array, the reference's
 * conformal_average (utils/math.h:1403-1415) used by BSSN::setExtraFieldData
 * (components/bssn/bssn.cc:165-170):
 *   out = [sum exp(6(phi+phi_frw)) field / n] / [sum exp(6(phi+phi_frw)) / n]
 * over n points of d_field and d_phi (device pointers).  Uses scratch memory
 * owned by the context; synchronous, result in *out (host). */
int cg_conformal_average(cg_ctx *ctx, const double *d_field, const double *d_phi, size_t n,
                         double phi_frw, double *out);

/* cg_conformal_average without any device allocation.  No counterpart in the
 * reference: for callers that cannot let a library call cudaMalloc (their own
 * memory pool or a fixed memory budget, or no implicit device synchronisation
 * allowed).  The reduction's scratch is a fixed 16 KiB array compiled into the
 * library, held by every GPU that loads it until the process exits.
 *   - d_field, d_phi: n device values each; n <= CG_NOALLOC_MAX_POINTS, larger
 *     n is rejected with CG_ERR_INVALID (message via cg_last_error(NULL)).
 *   - d_out: one device double receiving the average; queued on `stream`
 *     (a cudaStream_t, NULL = legacy default stream), no host synchronisation.
 *   - The first call on a device looks up the scratch array's device address
 *     with that device current; make that first call before any stream
 *     capture begins.  The address is then kept per device index for the
 *     rest of the process: after a cudaDeviceReset of that device the kept
 *     address is stale, so do not call this entry point again in that
 *     process.
 *   - Only errors of this call's own launches are returned; an error left
 *     pending by earlier work on the calling thread is not cleared.
 *   - All calls on a GPU share the scratch: calls whose kernels overlap on the
 *     GPU (different streams, concurrent threads) race; serialise them. */
#define CG_NOALLOC_MAX_BLOCKS 1024
#define CG_NOALLOC_MAX_POINTS ((size_t)1 << 30)
int cg_conformal_average_noalloc(const double *d_field, const double *d_phi, size_t n, double phi_frw,
                                 double *d_out, void *stream);

/* The current GPU's FP64 arithmetic throughput in flop/s (an FMA counted as
 * two), measured with eight independent FMA chains per thread over a grid
 * of eight CTAs per SM, timed with CUDA events.  No counterpart in the
 * reference: the denominator of the substep kernels' compute roofline.
 * Synchronous; allocates 512 KiB for the duration of the call. */
int cg_fp64_peak(double *flops_per_s);

/* Message of the last failure on this context (or of cg_create, when ctx is NULL). */
const char *cg_last_error(cg_ctx *ctx);

/* ABI version (CG_ABI_VERSION). */
int cg_version(void);

#ifdef __cplusplus
}
#endif

#endif
