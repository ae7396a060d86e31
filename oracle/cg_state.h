/*
 * cg_state.h -- the raw state-file format shared by every oracle and by the
 * CUDA path's tests.  TEST INFRASTRUCTURE (oracle side).
 *
 * One file holds the "_p" register of every evolved field of one periodic box
 * (reference: RK4Register::_array_p, utils/RK4Register.h:27) as contiguous
 * little-endian FP64 arrays, x-major with z fastest, i.e. the reference's
 * NP_INDEX(i,j,k) = (NZ*NY)*i + NZ*j + k (cosmo_macros.h:118).  Field order is
 * the reference's field-list order: BSSN_APPLY_TO_FIELDS
 * (components/bssn/bssn_macros.h:77-95), then the dust registers D,S1,S2,S3
 * (components/dust_fluid/dust.h:32-35) or the scalar registers
 * phi,Pi,psi1,psi2,psi3 (components/scalar/scalar.h:35-39), or the static
 * sims' fixed density DIFFD (components/static/static.h:17).
 *
 * The header also carries dx, dt and the reference FRW background state
 * (utils/FRW.h:14-20) so that a CPU run and a GPU run start from identical
 * bytes.
 */
#ifndef CG_STATE_H
#define CG_STATE_H

#include <stdint.h>

#define CG_STATE_MAGIC "CGSTATE1"
#define CG_STATE_MAX_FLUIDS 4
#define CG_STATE_Z4C 1
#define CG_STATE_SHIFT 2

enum cg_state_matter { CG_STATE_VACUUM = 0, CG_STATE_DUST = 1, CG_STATE_SCALAR = 2, CG_STATE_STATIC = 3 };

typedef struct {
  char magic[8];          /* "CGSTATE1" */
  int32_t nx, ny, nz;     /* grid points per axis */
  int32_t nfields;        /* 18 (vacuum), 22 (dust), 23 (scalar) or 19 (static),
                             one more with Z4c, seven more with the shift */
  int32_t matter;         /* enum cg_state_matter */
  int32_t step;           /* RK4 steps completed */
  int32_t nfluids;        /* FRW fluids in use (0..CG_STATE_MAX_FLUIDS) */
  int32_t flags;          /* bit 0 (CG_STATE_Z4C): Z4c damping, the constraint
                             field theta is stored after the matter fields;
                             bit 1 (CG_STATE_SHIFT): the shift, seven fields
                             beta1..3, auxB1..3, expN stored after those */
  double dx, dt;
  double frw_phi, frw_K;  /* FRW reference background (utils/FRW.h:15-16) */
  double fluid_rho[CG_STATE_MAX_FLUIDS];
  double fluid_w[CG_STATE_MAX_FLUIDS];
  double lambda;          /* cosmological-constant density rho_Lambda */
  double reserved2[3];
} cg_state_header;        /* 168 bytes, followed by nfields*nx*ny*nz doubles */

#endif
