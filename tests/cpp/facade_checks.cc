// Host-only checks of the C++ facade (no GPU call is made): configuration
// parsing, field map, FRW / Lambda set-up before the box exists, and the
// reference call-order rules that the facade enforces.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <string>

#include "cosmo_b200.hpp"

static int failures = 0;
#define EXPECT(cond)                                              \
  do {                                                            \
    if (!(cond)) {                                                \
      std::printf("FAIL %s:%d: %s\n", __FILE__, __LINE__, #cond); \
      ++failures;                                                 \
    }                                                             \
  } while (0)

template <class F>
static int thrown(F f) {
  try {
    f();
  } catch (int c) {
    return c;
  }
  return 12345;
}

int main(int argc, char** argv) {
  if (argc != 2) return 2;
  const std::string dir = argv[1];
  {
    std::ofstream o(dir + "/cfg.txt");
    o << "steps = 7\n  simulation_type   =   dust\nN = 24\nstencil_order = 4\nlapse = Harmonic\n"
         "dt_frac = 0.25\nH_LEN_FRAC = 1\nKO_damping_coefficient = 0.0\n";
  }
  cosmo::ConfigParser cfg(dir + "/cfg.txt");
  EXPECT(cfg["steps"] == "7");
  EXPECT(cfg["simulation_type"] == "dust");
  EXPECT(cfg("lapse", "Static") == "Harmonic");
  EXPECT(cfg("missing", "dflt") == "dflt");
  EXPECT(thrown([&] { (void)cfg["missing"]; }) == -1);
  EXPECT(thrown([&] { cosmo::ConfigParser bad(dir + "/nope.txt"); }) == -1);

  cosmo::BSSN bssn(&cfg);
  EXPECT(!bssn.created());
  EXPECT(bssn.desc().nx == 24 && bssn.desc().nz == 24);
  EXPECT(bssn.desc().stencil_order == 4);
  EXPECT(bssn.desc().lapse == CG_LAPSE_HARMONIC);
  EXPECT(bssn.desc().dx == 1.0 / 24.0);
  EXPECT(bssn.desc().dt == (double)(0.25L * (long double)(1.0 / 24.0)));
  EXPECT(bssn.num_fields() == 22);
  EXPECT(bssn.fields.count("DIFFphi_a") == 1 && bssn.fields.count("D_p") == 1 && bssn.fields.count("S3_f") == 1);
  EXPECT(bssn.fields.size() == 3 * 22);
  EXPECT(bssn.field_index("DIFFphi") == 6 && bssn.field_index("DIFFalpha") == 17 && bssn.field_index("D") == 18);
  EXPECT(thrown([&] { (void)bssn.field_index("phi"); }) == -1);

  // reference call order
  EXPECT(thrown([&] { bssn.RKEvolve(); }) == -1);
  EXPECT(thrown([&] { bssn.K1Finalize(); }) == -1);
  cosmo::Dust dust;
  EXPECT(thrown([&] { dust.K1Finalize(); }) == -1);
  EXPECT(thrown([&] { dust.RKEvolve(&bssn); }) == -1);  // before BSSN::RKEvolve
  EXPECT(dust.D != nullptr && dust.D->name == "D" && dust.S2->name == "S2");
  cosmo::Scalar scalar;
  EXPECT(thrown([&] { scalar.stepInit(&bssn); }) == -1);  // box is not a scalar box

  // FRW background and Lambda before the box is on the GPU
  bssn.frw->set_phi(0.125);
  bssn.frw->set_K(-3.0);
  bssn.frw->addFluid(0.5, 0.0);
  bssn.frw->addFluid(0.25, 1.0 / 3.0);
  EXPECT(bssn.frw->get_phi() == 0.125 && bssn.frw->get_K() == -3.0);
  EXPECT(bssn.frw->get_rho() == 0.75);
  EXPECT(std::fabs(bssn.frw->get_S() - 0.25) < 1e-15);
  cosmo::Lambda lam(1.0e-3);
  lam.addBSSNSource(&bssn);
  EXPECT(bssn.desc().lambda == 1.0e-3);

  // unknown options are configuration errors
  {
    std::ofstream o(dir + "/cfg2.txt");
    o << "steps = 1\nsimulation_type = dust\nlapse = NoSuchLapse\n";
  }
  cosmo::ConfigParser cfg2(dir + "/cfg2.txt");
  EXPECT(thrown([&] { cosmo::BSSN b2(&cfg2); }) == -1);
  {
    std::ofstream o(dir + "/cfg3.txt");
    o << "steps = 1\nsimulation_type = particles\n";
  }
  cosmo::ConfigParser cfg3(dir + "/cfg3.txt");
  EXPECT(thrown([&] { cosmo::BSSN b3(&cfg3); }) == 2);

  // the shift: the compile-time switch as the key BSSN_shift, the gauge as `shift`
  {
    std::ofstream o(dir + "/cfg4.txt");
    o << "simulation_type = scalar\nN = 8\nstencil_order = 4\nBSSN_shift = 1\nshift = GammaDriver\n"
         "gd_eta = 0.5\nZ4c_damping = 0\n";
  }
  cosmo::ConfigParser cfg4(dir + "/cfg4.txt");
  cosmo::BSSN b4(&cfg4);
  EXPECT(b4.desc().shift == CG_SHIFT_GAMMA_DRIVER && b4.desc().gd_eta == 0.5);
  EXPECT(b4.desc().gauge_wave_dir == 1 && b4.desc().k_driver_coeff == 0.04);
  EXPECT(b4.num_fields() == 23 + 7);
  EXPECT(b4.field_index("beta1") == 23 && b4.field_index("auxB3") == 28 && b4.field_index("expN") == 29);
  EXPECT(b4.fields.count("expN_p") == 1 && b4.fields.size() == 3 * 30);
  {
    std::ofstream o(dir + "/cfg5.txt");
    o << "simulation_type = dust\nN = 8\nshift = GammaDriver\n";
  }
  cosmo::ConfigParser cfg5(dir + "/cfg5.txt");
  EXPECT(thrown([&] { cosmo::BSSN b5(&cfg5); }) == -1);  // a shift gauge without the shift fields
  {
    std::ofstream o(dir + "/cfg6.txt");
    o << "simulation_type = dust\nN = 8\nBSSN_shift = 1\nshift = NoSuchShift\n";
  }
  cosmo::ConfigParser cfg6(dir + "/cfg6.txt");
  EXPECT(thrown([&] { cosmo::BSSN b6(&cfg6); }) == -1);

  std::printf(failures ? "facade checks: %d failures\n" : "facade checks: ok\n", failures);
  return failures ? 1 : 0;
}
