// cosmo_b200.hpp -- C++ host facade of the B200 BSSN evolution path.
//
// Keeps the component API that the reference's sim drivers use
// (components/bssn/bssn.h:22-80, components/dust_fluid/dust.h,
// components/scalar/scalar.h, components/Lambda/lambda.h,
// utils/RK4Register.h, utils/ConfigParser.h, sims/sim.h) on top of the C ABI
// in include/cosmograph_b200.h.  All field data stay on the GPU; the host
// objects hold a context handle, the box descriptor and sequence state.
//
// Mapping of the reference's per-substep calls onto the fused kernel:
//   BSSN::stepInit                    -> cg_step_init (includes Dust/Scalar::stepInit)
//   clearSrc / addBSSNSrc / addBSSNSource (dust, scalar, Lambda)
//                                     -> no device work: the sources are computed
//                                        inside the substep kernel; the calls are
//                                        checked for order only
//   BSSN::RKEvolve, Dust::RKEvolve    -> mark the substep's right-hand side as due
//   BSSN::K{n}Finalize                -> cg_rk_stage(n): sources, RHS and the RK4
//                                        register update of every field, one launch
//   Dust/Scalar::K{n}Finalize         -> order check (their registers were updated
//                                        by the same launch)
// Errors follow the reference: `throw int` (-1 configuration, initial data or
// a misuse of the API; 10 NaN, sims/sim.cc:179-183; 2 unknown simulation type,
// cosmo.cc:78-81).
#pragma once

#include <cstdint>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "cosmograph_b200.h"

namespace cosmo {

using real_t = double;
using idx_t = long long;

// "param = value" configuration file (utils/ConfigParser.h:9-24, ConfigParser.cc)
class ConfigParser {
 public:
  ConfigParser() = default;
  explicit ConfigParser(const std::string& fname) { parse(fname); }
  void parse(const std::string& fname);
  std::string getFileName() const { return fileName; }
  // required parameter: throws -1 when it is missing
  std::string operator[](const std::string& param) const;
  // optional parameter with a default
  std::string operator()(const std::string& param, const std::string& default_val) const;
  bool has(const std::string& param) const { return config.count(param) != 0; }
  void set(const std::string& param, const std::string& val) { config[param] = val; }

 private:
  std::map<std::string, std::string> config;
  std::string fileName;
};

// Output directory and log file (IO/IOData.h:24-70): an existing run directory
// is never overwritten; "<dir>.1", "<dir>.2", ... are used instead.
class IOData {
 public:
  explicit IOData(std::string output_dir);
  void log(const std::string& msg);
  const std::string& dir() const { return output_dir; }

 private:
  std::string output_dir;
  std::ofstream logfile;
};

class BSSN;

// One register of one field, resident on the GPU ('p', 'a' or 'f').
class DeviceArray {
 public:
  DeviceArray(BSSN* owner, int field, char reg, std::string name)
      : owner(owner), field(field), reg(reg), nm(std::move(name)) {}
  std::vector<double> values() const;          // synchronous copy to the host
  void download(double* host, size_t n) const;
  void upload(const double* host, size_t n);
  size_t size() const;
  const std::string& name() const { return nm; }

 private:
  BSSN* owner;
  int field;
  char reg;
  std::string nm;
};
using map_t = std::map<std::string, DeviceArray*>;

// The registers of one evolved field (utils/RK4Register.h:19-40).  The
// reference's _c register (RHS, then next-substep input) never reaches HBM:
// the substep kernel consumes it in registers.
struct RK4Register {
  std::string name;
  DeviceArray _array_p, _array_a, _array_f;
  RK4Register(BSSN* owner, int field, const std::string& nm)
      : name(nm), _array_p(owner, field, 'p', nm + "_p"), _array_a(owner, field, 'a', nm + "_a"),
        _array_f(owner, field, 'f', nm + "_f") {}
};

// FRW reference background (utils/FRW.h:79-83), read from the context.
class FRW {
 public:
  explicit FRW(BSSN* owner) : owner(owner) {}
  real_t get_phi() const;
  real_t get_K() const;
  real_t get_rho() const;  // sum of the fluids' densities
  real_t get_S() const;    // sum of 3 w rho
  // before the first device call only (initial data)
  void set_phi(real_t phi);
  void set_K(real_t K);
  void addFluid(real_t rho, real_t w);

 private:
  BSSN* owner;
};

// BSSN component (components/bssn/bssn.h:22-80).  Grid, matter model and
// numerics come from the configuration: N (or NX, NY, NZ), stencil_order,
// precision, simulation_type, lapse, normalize_metric, a_adj_amp,
// k_damping_amp, KO_damping_coefficient, gd_c, dw_mu_l, dw_p, dx / H_LEN_FRAC,
// dt_frac.  The context is created on the first call that needs the GPU, so
// initial data may still set the FRW background and Lambda before that.
class BSSN {
 public:
  explicit BSSN(ConfigParser* config);
  ~BSSN();
  BSSN(const BSSN&) = delete;
  BSSN& operator=(const BSSN&) = delete;

  void init();  // create the context (all registers zero, bssn.cc:126-144)
  void setDt(real_t dt);

  void stepInit();
  void RKEvolve();
  void K1Finalize() { finalize(1); }
  void K2Finalize() { finalize(2); }
  void K3Finalize() { finalize(3); }
  void K4Finalize() { finalize(4); }
  void clearSrc();
  void step();  // RKEvolve + K1..K4Finalize (bssn.cc:327-339); stepInit first

  // statistics of the current state (bssn.cc:965-1071): H[8], M[8], G/A/S[7]
  void setConstraintCalcs(real_t H[8], real_t M[8], real_t G[7], real_t A[7], real_t S[7]);
  // the columns of io_bssn_dump_statistics (IO/io.cc:8-14, 386-403): volume-
  // weighted mean and stdev of DIFFphi, DIFFK, DIFFr, ricci; volume average
  void fieldStatistics(real_t out[9]);

  // fields["DIFFphi_a"], fields["D_p"], ... (bssn.cc:30-39)
  map_t fields;
  std::unique_ptr<FRW> frw;
  real_t cur_t = 0.0;

  // initial data from a state file (the CGSTATE1 format of
  // cosmograph_b200.state: 168-byte header, then the _p register of every
  // field); sets the FRW background and Lambda from its header
  void loadState(const std::string& path);
  // write the _p register of every field in the same format
  void saveState(const std::string& path, int step);

  // plumbing for the facades
  cg_ctx* ctx();
  cg_box_desc& desc() { return d; }
  bool created() const { return c != nullptr; }
  int matter() const { return d.matter; }
  size_t points() const { return (size_t)d.nx * d.ny * d.nz; }
  int num_fields() const { return cg_num_fields(d.matter) + d.z4c + (d.shift != CG_SHIFT_NONE ? 7 : 0); }
  RK4Register* reg(const std::string& name);    // registers of one field
  int field_index(const std::string& name) const;
  void check(int rc, const char* what);
  bool nan_seen();
  int substep_done() const { return last_stage; }
  bool rhs_due() const { return rhs_pending; }
  void note_sources() { sources_set = true; }

 private:
  void finalize(int n);
  void ensure_fields();
  cg_box_desc d{};
  cg_ctx* c = nullptr;
  std::vector<std::unique_ptr<RK4Register>> regs;
  int last_stage = 0;        // 0 before stepInit, 1..4 after K{n}Finalize
  bool stepped_init = false;
  bool rhs_pending = false;
  bool sources_set = false;
};

// Dust component (components/dust_fluid/dust.h): conservative D, S_i.
class Dust {
 public:
  Dust() = default;
  void stepInit(BSSN* bssn);
  void RKEvolve(BSSN* bssn);
  void addBSSNSrc(BSSN* bssn);
  void K1Finalize() { finalize(1); }
  void K2Finalize() { finalize(2); }
  void K3Finalize() { finalize(3); }
  void K4Finalize() { finalize(4); }
  void setDt(real_t) {}
  // registers D, S1, S2, S3 (dust.h:32-35) once a BSSN is attached
  RK4Register* D = nullptr;
  RK4Register* S1 = nullptr;
  RK4Register* S2 = nullptr;
  RK4Register* S3 = nullptr;

 private:
  void attach(BSSN* bssn);
  void finalize(int n);
  BSSN* b = nullptr;
};

// Minimally coupled scalar field (components/scalar/scalar.h): phi, Pi, psi_i.
class Scalar {
 public:
  Scalar() = default;
  void stepInit(BSSN* bssn);
  void RKEvolve(BSSN* bssn);  // grid-wide form of RKEvolvePt
  void addBSSNSource(BSSN* bssn);
  void K1Finalize() { finalize(1); }
  void K2Finalize() { finalize(2); }
  void K3Finalize() { finalize(3); }
  void K4Finalize() { finalize(4); }
  void setDt(real_t) {}

 private:
  void finalize(int n);
  BSSN* b = nullptr;
};

// Static matter (components/static/static.h): a fixed density DIFFD (field
// 18 of the box) that sources DIFFr; the source is formed inside the substep
// kernel, this class keeps the reference's call sequence.
class Static {
 public:
  Static() = default;
  void init() {}
  void addBSSNSrc(BSSN* bssn);
};

// Cosmological constant (components/Lambda/lambda.h)
class Lambda {
 public:
  explicit Lambda(real_t rho_L = 0.0) : lambda(rho_L) {}
  void setLambda(real_t rho_L) { lambda = rho_L; }
  real_t getLambda() const { return lambda; }
  // the Lambda source is added inside the substep kernel from the box's
  // descriptor; this call checks that the two agree
  void addBSSNSource(BSSN* bssn);

 private:
  real_t lambda;
};

// Simulation drivers (sims/sim.h, sims/dust.h, sims/scalar.h, sims/vacuum.h)
class CosmoSim {
 public:
  explicit CosmoSim(ConfigParser* config);
  virtual ~CosmoSim();
  virtual void init() = 0;
  virtual void setICs() = 0;
  virtual void runStep() = 0;
  void simInit();
  void run();
  void runCommonStepTasks();
  void outputStateInformation();
  void outputCommon();     // snapshots, constraint and FRW time series at their intervals
  void outputSnapshots();  // 3-D / 2-D / 1-D field dumps (io_bssn_fields_snapshot)
  idx_t getStep() const { return step; }
  BSSN* bssn() { return bssnSim; }

 protected:
  void loadICs();
  ConfigParser* cfg;
  IOData* iodata = nullptr;
  BSSN* bssnSim = nullptr;
  idx_t step = 0;
  idx_t num_steps = 0;
  real_t t = 0.0;
  double rk_seconds = 0.0;
};

class DustSim : public CosmoSim {
 public:
  explicit DustSim(ConfigParser* config);
  ~DustSim() override;
  void init() override;
  void setICs() override;
  void runStep() override;
  void initDustStep();
  void runDustStep();

 private:
  Dust* dustSim = nullptr;
  Lambda* lambda = nullptr;
};

class ScalarSim : public CosmoSim {
 public:
  explicit ScalarSim(ConfigParser* config) : CosmoSim(config) {}
  ~ScalarSim() override;
  void init() override;
  void setICs() override;
  void runStep() override;
  void initScalarStep();
  void runScalarStep();

 private:
  Scalar* scalarSim = nullptr;
};

// sims/static.h: static matter, Static or ConformalFLRW lapse
class StaticSim : public CosmoSim {
 public:
  explicit StaticSim(ConfigParser* config);
  ~StaticSim() override;
  void init() override;
  void setICs() override;
  void runStep() override;
  void initStaticStep();
  void runStaticStep();

 private:
  Static* staticSim = nullptr;
  Lambda* lambda = nullptr;
};

class VacuumSim : public CosmoSim {
 public:
  explicit VacuumSim(ConfigParser* config) : CosmoSim(config) {}
  void init() override;
  void setICs() override;
  void runStep() override;
};

// The config-file driver (cosmo.cc:26-96): returns the process exit status.
int run_config_file(const std::string& fname);

}  // namespace cosmo
