/*
 * ref_driver.cc -- TEST INFRASTRUCTURE: drives the reference's own, unmodified
 * BSSN / Dust / Scalar / Lambda classes (compiled from the reference sources
 * by oracle/build_ref.py into oracle/_ref/) on a state file written in the
 * cg_state.h format, so that the reference CPU implementation and the CUDA
 * path can be run from identical bytes.  Nothing in the product links or
 * calls this program; tests and bench.py's CPU-baseline leg run it as a
 * subprocess.
 *
 * The per-step call sequences replayed here are the reference's:
 *   dust   : DustSim::initDustStep + runDustStep   (sims/dust.cc:53-63, 114-161)
 *   scalar : ScalarSim::initScalarStep + runScalarStep (sims/scalar.cc:75-82, 97-151)
 *   vacuum : VacuumSim::initVacuumStep + runVacuumStep (sims/vacuum.cc:73-97)
 *   static : StaticSim::initStaticStep + runStaticStep (sims/static.cc:71-167),
 *            the fixed density DIFFD (Static, components/static/static.cc)
 *            read from and written back as field 18
 * minus output, NaN checks and ray sheets, which never touch the fields.
 * Built with -DUSE_Z4c_DAMPING=1 (build_ref.py flavours *_z4c) the driver
 * reads and writes theta after the matter fields; built with
 * -DUSE_BSSN_SHIFT=1 -DUSE_GAMMA_DRIVER=1 (flavours *_shift), beta1..3,
 * auxB1..3 and expN after those.
 *
 * Usage: cg_ref_<...> <mode> <config.txt> <state_in> <out> [steps]
 *   mode = evolve      : run <steps> RK4 steps, write the "_p" registers to <out>
 *          rhs         : run the step initialisation and the first substep's
 *                        RKEvolve, write every field's "_c" register (the RHS)
 *          constraints : step initialisation, then BSSN::setConstraintCalcs
 *                        (components/bssn/bssn.cc:965-1071); write the H, M,
 *                        G, A, S statistics as text to <out>, and the field
 *                        statistics of io_bssn_dump_statistics (IO/io.cc:8-14,
 *                        386-403: conformal average and standard deviation of
 *                        DIFFphi, DIFFK, DIFFr, ricci after the
 *                        set_bd_values sweep of prepBSSNOutput, sims/sim.cc:
 *                        214-225; volume average) as the row STATS
 * The last stdout line is "CGRESULT {json}" with the timing of the step loop.
 */
#include "cosmo_includes.h"
#include "cosmo_types.h"
#include "cosmo_globals.h"
#include "components/bssn/bssn.h"
#include "components/dust_fluid/dust.h"
#include "components/scalar/scalar.h"
#include "components/static/static.h"
#include "components/Lambda/lambda.h"
#include "utils/math.h"
#include "cg_state.h"

#include <time.h>
#include <unistd.h>
#include <vector>

cosmo::real_t dt, dx;
cosmo::TimerManager _timer;
cosmo::ConfigParser _config;

using namespace cosmo;

namespace {

const char *kBssnNames[18] = {
    "DIFFgamma11", "DIFFgamma12", "DIFFgamma13", "DIFFgamma22", "DIFFgamma23",
    "DIFFgamma33", "DIFFphi",     "A11",         "A12",         "A13",
    "A22",         "A23",         "A33",         "DIFFK",       "Gamma1",
    "Gamma2",      "Gamma3",      "DIFFalpha"};

double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

struct Sim {
  BSSN *bssn = nullptr;
  Dust *dust = nullptr;
  Scalar *scalar = nullptr;
  Static *stat = nullptr;
  Lambda *lambda = nullptr;
  int matter = CG_STATE_VACUUM;

  // pointers to the register arrays of every evolved field, in file order
  std::vector<arr_t *> reg(char r) {
    std::vector<arr_t *> out;
    for (int f = 0; f < 18; ++f)
      out.push_back(bssn->fields[std::string(kBssnNames[f]) + "_" + r]);
    auto pick = [r](cosmo::register_t &x) -> arr_t * {
      switch (r) {
        case 'p': return &x._array_p;
        case 'a': return &x._array_a;
        case 'c': return &x._array_c;
        default: return &x._array_f;
      }
    };
    if (matter == CG_STATE_DUST) {
      out.push_back(pick(dust->D));
      out.push_back(pick(dust->S1));
      out.push_back(pick(dust->S2));
      out.push_back(pick(dust->S3));
    } else if (matter == CG_STATE_SCALAR) {
      out.push_back(pick(scalar->phi));
      out.push_back(pick(scalar->Pi));
      out.push_back(pick(scalar->psi1));
      out.push_back(pick(scalar->psi2));
      out.push_back(pick(scalar->psi3));
    } else if (matter == CG_STATE_STATIC) {
      out.push_back(stat->fields["DIFFD_a"]);  // not a register: the same array for every role
    }
#if USE_Z4c_DAMPING
    out.push_back(bssn->fields[std::string("theta_") + r]);  // stored after the matter fields
#endif
#if USE_BSSN_SHIFT
    // then the shift, the Gamma-driver's auxB and expN (bssn_macros.h:73-75)
    for (const char *n : {"beta1", "beta2", "beta3"}) out.push_back(bssn->fields[std::string(n) + "_" + r]);
#if USE_GAMMA_DRIVER
    for (const char *n : {"auxB1", "auxB2", "auxB3"}) out.push_back(bssn->fields[std::string(n) + "_" + r]);
#endif
    out.push_back(bssn->fields[std::string("expN_") + r]);
#endif
    return out;
  }

  // sims/dust.cc:53-63, sims/scalar.cc:75-82, sims/vacuum.cc:73-78
  void init_step() {
    bssn->stepInit();
    if (matter == CG_STATE_DUST) {
      dust->stepInit(bssn);
      bssn->clearSrc();
      dust->addBSSNSrc(bssn);
      lambda->addBSSNSource(bssn);
    } else if (matter == CG_STATE_SCALAR) {
      scalar->stepInit();
      bssn->clearSrc();
      scalar->addBSSNSource(bssn);
    } else if (matter == CG_STATE_STATIC) {
      bssn->clearSrc();
      stat->addBSSNSrc(bssn->fields, bssn->frw);
      lambda->addBSSNSource(bssn);
    }
  }

  void evolve_substep() {
    if (matter == CG_STATE_SCALAR) {
      // sims/scalar.cc:104-108: one fused point loop
      idx_t i = 0, j = 0, k = 0;
      BSSNData b_data = {0};  // sims/scalar.cc:100 leaves this uninitialised; theta, beta and their derivatives are never written when Z4c and shift are off
#pragma omp parallel for firstprivate(j, k, b_data)
      LOOP3(i, j, k) {
        bssn->RKEvolvePt(i, j, k, &b_data);
        scalar->RKEvolvePt(&b_data);
      }
    } else {
      bssn->RKEvolve();
      if (matter == CG_STATE_DUST) dust->RKEvolve(bssn);
    }
  }

  void resource() {
    if (matter == CG_STATE_DUST) {
      bssn->clearSrc();
      dust->addBSSNSrc(bssn);
      lambda->addBSSNSource(bssn);
    } else if (matter == CG_STATE_SCALAR) {
      bssn->clearSrc();
      scalar->addBSSNSource(bssn);
    } else if (matter == CG_STATE_STATIC) {
      bssn->clearSrc();
      stat->addBSSNSrc(bssn->fields, bssn->frw);
      lambda->addBSSNSource(bssn);
    }
  }

  // sims/dust.cc:114-161, sims/scalar.cc:97-151, components/bssn/bssn.cc:327-339
  void run_step() {
    evolve_substep();
    bssn->K1Finalize();
    if (dust) dust->K1Finalize();
    if (scalar) scalar->K1Finalize();
    resource();
    evolve_substep();
    bssn->K2Finalize();
    if (dust) dust->K2Finalize();
    if (scalar) scalar->K2Finalize();
    resource();
    evolve_substep();
    bssn->K3Finalize();
    if (dust) dust->K3Finalize();
    if (scalar) scalar->K3Finalize();
    resource();
    evolve_substep();
    bssn->K4Finalize();
    if (dust) dust->K4Finalize();
    if (scalar) scalar->K4Finalize();
  }
};

void die(const char *msg) {
  fprintf(stderr, "cg_ref: %s\n", msg);
  fflush(stderr);
  _Exit(3);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 5) die("usage: <mode> <config> <state_in> <out> [steps]");
  std::string mode = argv[1];
  int steps = argc > 5 ? atoi(argv[5]) : 1;
  _config.parse(argv[2]);

  FILE *fin = fopen(argv[3], "rb");
  if (!fin) die("cannot open input state");
  cg_state_header h;
  if (fread(&h, sizeof(h), 1, fin) != 1) die("short header");
  if (memcmp(h.magic, CG_STATE_MAGIC, 8) != 0) die("bad magic");
  if (h.nx != NX || h.ny != NY || h.nz != NZ) die("grid size differs from the compiled N");
  if (((h.flags & CG_STATE_Z4C) != 0) != (USE_Z4c_DAMPING != 0))
    die("the state's Z4c flag differs from the build's USE_Z4c_DAMPING");
  if (((h.flags & CG_STATE_SHIFT) != 0) != (USE_BSSN_SHIFT != 0))
    die("the state's shift flag differs from the build's USE_BSSN_SHIFT");
  const long pts = (long)NX * NY * NZ;
  std::vector<double> buf((size_t)h.nfields * pts);
  if (fread(buf.data(), sizeof(double), buf.size(), fin) != buf.size()) die("short data");
  fclose(fin);

  dx = h.dx;
  dt = h.dt;

  Sim sim;
  sim.matter = h.matter;
  sim.bssn = new BSSN(&_config, nullptr);
  if (h.frw_phi != 0.0) sim.bssn->frw->set_phi(h.frw_phi);
  if (h.frw_K != 0.0) sim.bssn->frw->set_K(h.frw_K);
  for (int n = 0; n < h.nfluids; ++n) sim.bssn->frw->addFluid(h.fluid_rho[n], h.fluid_w[n]);
  if (h.matter == CG_STATE_DUST) {
    sim.dust = new Dust();
    sim.lambda = new Lambda();
    sim.lambda->setLambda(h.lambda);
  } else if (h.matter == CG_STATE_SCALAR) {
    sim.scalar = new Scalar();
  } else if (h.matter == CG_STATE_STATIC) {
    sim.stat = new Static();
    sim.stat->init();
    sim.lambda = new Lambda();
    sim.lambda->setLambda(h.lambda);
  }
  std::vector<arr_t *> P = sim.reg('p');
  if ((int)P.size() != h.nfields) die("field count differs from the matter model");
  for (int f = 0; f < h.nfields; ++f)
    memcpy(P[f]->_array, buf.data() + (size_t)f * pts, sizeof(double) * pts);

  double t0 = now_s();
  std::string extra;
  if (mode == "evolve") {
    for (int s = 0; s < steps; ++s) {
      const double ts = now_s();
      sim.init_step();
      sim.run_step();
      printf("CGSTEP %d %.6f\n", s, now_s() - ts);
      fflush(stdout);
    }
  } else if (mode == "rhs") {
    sim.init_step();
    sim.evolve_substep();
    P = sim.reg('c');
  } else if (mode == "constraints") {
    sim.init_step();
    real_t H[8] = {0}, M[8] = {0}, G[7] = {0}, A[7] = {0}, S[7] = {0};
    sim.bssn->setConstraintCalcs(H, M, G, A, S);
    FILE *fo = fopen(argv[4], "w");
    if (!fo) die("cannot open output");
    auto row = [fo](const char *n, real_t *v, int m) {
      fprintf(fo, "%s", n);
      for (int q = 0; q < m; ++q) fprintf(fo, " %.17g", v[q]);
      fprintf(fo, "\n");
    };
    row("H", H, 8);
    row("M", M, 8);
    row("G", G, 7);
    row("A", A, 7);
    row("S", S, 7);
    // CosmoSim::prepBSSNOutput: ricci_a at every point
    {
      idx_t i, j, k;
#pragma omp parallel for default(shared) private(i, j, k)
      LOOP3(i, j, k) {
        BSSNData b_data = {0};
        sim.bssn->set_bd_values(i, j, k, &b_data);
      }
    }
    map_t &F = sim.bssn->fields;
    const real_t phi_frw = sim.bssn->frw->get_phi();
    real_t st[9];
    const char *names[4] = {"DIFFphi_a", "DIFFK_a", "DIFFr_a", "ricci_a"};
    for (int q = 0; q < 4; ++q) {
      arr_t &f = *F[names[q]];
      st[2 * q] = conformal_average(f, *F["DIFFphi_a"], phi_frw);
      st[2 * q + 1] = conformal_standard_deviation(f, *F["DIFFphi_a"], phi_frw, st[2 * q]);
    }
    st[8] = volume_average(*F["DIFFphi_a"], phi_frw);
    row("STATS", st, 9);
    fclose(fo);
  } else {
    die("unknown mode");
  }
  double t1 = now_s();

  if (mode != "constraints") {
    FILE *fo = fopen(argv[4], "wb");
    if (!fo) die("cannot open output");
    cg_state_header ho = h;
    ho.step = h.step + (mode == "evolve" ? steps : 0);
    ho.frw_phi = sim.bssn->frw->get_phi();
    ho.frw_K = sim.bssn->frw->get_K();
    fwrite(&ho, sizeof(ho), 1, fo);
    for (int f = 0; f < h.nfields; ++f) fwrite(P[f]->_array, sizeof(double), pts, fo);
    fclose(fo);
  }
  printf("CGRESULT {\"mode\": \"%s\", \"steps\": %d, \"seconds\": %.6f, \"points\": %ld, "
         "\"threads\": %d}\n",
         mode.c_str(), mode == "evolve" ? steps : 0, t1 - t0, pts, omp_get_max_threads());
  fflush(stdout);
  // The reference's Dust/Scalar destructors call member destructors
  // explicitly (components/dust_fluid/dust.cc:46-52), which would double-free
  // at teardown; leave without running destructors.
  _Exit(0);
}
