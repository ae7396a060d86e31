// facade.cc -- the C++ component API (BSSN, Dust, Scalar, Lambda, sims) over
// the C ABI.  See cosmo_b200.hpp for the mapping onto the fused kernel.
#include "cosmo_b200.hpp"

#include <sys/stat.h>
#include <zlib.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>

namespace cosmo {

namespace {

[[noreturn]] void raise(int code, const std::string& msg) {
  std::cerr << "Error: " << msg << "\n";
  throw code;
}

std::string fmt15(double v) {
  char buf[40];
  std::snprintf(buf, sizeof(buf), "%.15g", v);
  return buf;
}

int lapse_code(const std::string& name) {
  static const std::map<std::string, int> m = {
      {"Static", CG_LAPSE_STATIC},           {"Harmonic", CG_LAPSE_HARMONIC},
      {"ConformalFLRW", CG_LAPSE_CONFORMAL_FLRW}, {"ConformalSync", CG_LAPSE_CONFORMAL_SYNC},
      {"Anharmonic", CG_LAPSE_ANHARMONIC},   {"OnePlusLog", CG_LAPSE_ONE_PLUS_LOG},
      {"AwAGaugeWave", CG_LAPSE_AWA_GAUGE_WAVE}, {"AwAShiftedWave", CG_LAPSE_AWA_SHIFTED_WAVE},
      {"DampedWave", CG_LAPSE_DAMPED_WAVE}};
  auto it = m.find(name);
  if (it == m.end()) raise(-1, "unknown lapse `" + name + "`");
  return it->second;
}

// shift gauges (BSSNGaugeHandler.h:113-134)
int shift_code(const std::string& name) {
  static const std::map<std::string, int> m = {
      {"Static", CG_SHIFT_STATIC}, {"GammaDriver", CG_SHIFT_GAMMA_DRIVER}, {"DampedWave", CG_SHIFT_DAMPED_WAVE},
      {"AwAShiftedWave", CG_SHIFT_AWA_SHIFTED_WAVE}, {"AijDriverShift", CG_SHIFT_AIJ_DRIVER}};
  auto it = m.find(name);
  if (it == m.end()) raise(-1, "Shift gauge not found: `" + name + "`");
  return it->second;
}

// names of the fields after the matter fields: theta (Z4c), then the shift's
const char* const kShiftNames[7] = {"beta1", "beta2", "beta3", "auxB1", "auxB2", "auxB3", "expN"};

int matter_code(const std::string& sim) {
  if (sim == "dust") return CG_MATTER_DUST;
  if (sim == "scalar") return CG_MATTER_SCALAR;
  if (sim == "vacuum") return CG_MATTER_VACUUM;
  if (sim == "static") return CG_MATTER_STATIC;
  raise(2, "simulation_type `" + sim + "` is not on this path (dust, scalar, vacuum, static)");
}

// state-file header (cosmograph_b200.state: "CGSTATE1", 168 bytes, little endian)
struct StateHeader {
  char magic[8];
  int32_t nx, ny, nz, nfields, matter, step, nfluids, reserved;
  double dx, dt, frw_phi, frw_K, fluid_rho[4], fluid_w[4], lambda, reserved2[3];
};
static_assert(sizeof(StateHeader) == 168, "state header is 168 bytes");

// append `value` + delimiter to <dir><name>.dat.gz (IO/io.cc:813-831 format)
void dump_value(IOData* io, double value, const std::string& name, const char* delim) {
  const std::string fn = io->dir() + name + ".dat.gz";
  gzFile f = gzopen(fn.c_str(), "ab");
  if (!f) {
    io->log("Error opening file: " + fn);
    return;
  }
  const std::string s = fmt15(value) + delim;
  gzwrite(f, s.data(), (unsigned)s.size());
  gzclose(f);
}

}  // namespace

// ---------------------------------------------------------------- ConfigParser
void ConfigParser::parse(const std::string& fname) {
  fileName = fname;
  std::ifstream fin(fname);
  if (!fin) raise(-1, "error opening " + fname + "! Make sure you have specified a valid config file.");
  std::string param, eq, val;
  // whitespace-separated "param = value" triples (ConfigParser.cc:37-42)
  while (fin >> param >> eq >> val) {
    std::cout << "config[" << param << "] = " << val << "\n";
    config[param] = val;
  }
}

std::string ConfigParser::operator[](const std::string& param) const {
  auto it = config.find(param);
  if (it == config.end())
    raise(-1, "param `" + param + "` is required, but was not set! Please set this in the configuration file, " +
                  fileName + ".");
  return it->second;
}

std::string ConfigParser::operator()(const std::string& param, const std::string& default_val) const {
  auto it = config.find(param);
  return it == config.end() ? default_val : it->second;
}

// ---------------------------------------------------------------------- IOData
IOData::IOData(std::string dir) {
  const std::string log_name = "log.txt";
  if (dir.empty()) dir = "output";
  if (dir.back() == '/') dir.pop_back();
  if (std::ifstream(dir + "/" + log_name)) {
    int s = 1;
    while (std::ifstream(dir + "." + std::to_string(s) + "/" + log_name)) ++s;
    std::cout << "Data files in output directory seem to already exist! Using '" << dir << "." << s
              << "' instead.\n";
    dir += "." + std::to_string(s);
  }
  mkdir(dir.c_str(), 0755);
  output_dir = dir + "/";
  logfile.open(output_dir + log_name);
  log("Log file open.");
}

void IOData::log(const std::string& msg) {
  std::cout << msg << "\n";
  if (logfile) logfile << msg << "\n" << std::flush;
}

// ----------------------------------------------------------------- DeviceArray
size_t DeviceArray::size() const { return owner->points(); }

void DeviceArray::download(double* host, size_t n) const {
  owner->check(cg_download_field(owner->ctx(), 0, field, reg, host, n), "download");
}

void DeviceArray::upload(const double* host, size_t n) {
  owner->check(cg_upload_field(owner->ctx(), 0, field, reg, host, n), "upload");
}

std::vector<double> DeviceArray::values() const {
  std::vector<double> v(size());
  download(v.data(), v.size());
  return v;
}

// ------------------------------------------------------------------------- FRW
namespace {
void frw_read(BSSN* b, double out[6]) {
  std::fill(out, out + 6, 0.0);
  b->check(cg_frw_state(b->ctx(), 0, out, 6), "frw state");
}
}  // namespace

real_t FRW::get_phi() const {
  if (!owner->created()) return owner->desc().frw_phi;
  double s[6];
  frw_read(owner, s);
  return s[0];
}
real_t FRW::get_K() const {
  if (!owner->created()) return owner->desc().frw_K;
  double s[6];
  frw_read(owner, s);
  return s[1];
}
real_t FRW::get_rho() const {
  const cg_box_desc& d = owner->desc();
  double s[6] = {0, 0, d.fluid_rho[0], d.fluid_rho[1], d.fluid_rho[2], d.fluid_rho[3]};
  if (owner->created()) frw_read(owner, s);
  double r = 0.0;
  for (int m = 0; m < d.nfluids; ++m) r += s[2 + m];
  return r;
}
real_t FRW::get_S() const {
  const cg_box_desc& d = owner->desc();
  double s[6] = {0, 0, d.fluid_rho[0], d.fluid_rho[1], d.fluid_rho[2], d.fluid_rho[3]};
  if (owner->created()) frw_read(owner, s);
  double S = 0.0;
  for (int m = 0; m < d.nfluids; ++m) S += 3.0 * s[2 + m] * d.fluid_w[m];
  return S;
}
void FRW::set_phi(real_t phi) {
  if (owner->created()) raise(-1, "the FRW background is fixed once the box is on the GPU");
  owner->desc().frw_phi = phi;
}
void FRW::set_K(real_t K) {
  if (owner->created()) raise(-1, "the FRW background is fixed once the box is on the GPU");
  owner->desc().frw_K = K;
}
void FRW::addFluid(real_t rho, real_t w) {
  cg_box_desc& d = owner->desc();
  if (owner->created()) raise(-1, "the FRW background is fixed once the box is on the GPU");
  if (d.nfluids >= 4) raise(-1, "at most 4 FRW fluids");
  d.fluid_rho[d.nfluids] = rho;
  d.fluid_w[d.nfluids] = w;
  d.nfluids++;
}

// ------------------------------------------------------------------------ BSSN
BSSN::BSSN(ConfigParser* config) {
  const ConfigParser& c = *config;
  const int n = std::stoi(c("N", "16"));
  cg_box_desc_default(&d, n);
  d.nx = std::stoi(c("NX", std::to_string(n)));
  d.ny = std::stoi(c("NY", std::to_string(n)));
  d.nz = std::stoi(c("NZ", std::to_string(n)));
  d.matter = matter_code(c("simulation_type", "vacuum"));
  d.stencil_order = std::stoi(c("stencil_order", "8"));
  const std::string prec = c("precision", "fp64");
  if (prec == "fp64") d.precision = CG_PREC_FP64;
  else if (prec == "fp64_fma") d.precision = CG_PREC_FP64_FMA;
  else if (prec == "mixed") d.precision = CG_PREC_MIXED;
  else raise(-1, "precision `" + prec + "` (fp64, fp64_fma or mixed)");
  d.lapse = lapse_code(c("lapse", "Static"));
  // the reference's compile-time USE_BSSN_SHIFT (with USE_GAMMA_DRIVER,
  // cosmo_macros.h:43-50) as the config key BSSN_shift; the gauge is `shift`
  // (BSSNGaugeHandler.h:200-223)
  const std::string shift = c("shift", "Static");
  const bool with_shift = std::stoi(c("BSSN_shift", "0")) != 0;
  if (!with_shift && shift != "Static") raise(-1, "a non-Static shift needs BSSN_shift = 1 (USE_BSSN_SHIFT)");
  d.shift = with_shift ? shift_code(shift) : CG_SHIFT_NONE;
  d.gauge_wave_dir = std::stoi(c("gauge_wave_dir", "1"));
  d.gd_eta = std::stod(c("gd_eta", "0.0"));
  d.dw_mu_s = std::stod(c("dw_mu_s", "0.0"));
  d.k_driver_coeff = std::stod(c("k_driver_coeff", "0.04"));
  d.normalize_metric = std::stoi(c("normalize_metric", "1"));
  // the reference's compile-time USE_Z4c_DAMPING (cosmo_macros.h:91-100) as a config key
  d.z4c = std::stoi(c("Z4c_damping", "0")) != 0 ? 1 : 0;
  d.ko_coeff = std::stod(c("KO_damping_coefficient", "0.0"));
  d.a_adj_amp = std::stod(c("a_adj_amp", "0.0"));
  d.k_damping_amp = std::stod(c("k_damping_amp", "0.0"));
  d.gd_c = std::stod(c("gd_c", "1.0"));
  d.dw_mu_l = std::stod(c("dw_mu_l", "0.0"));
  d.dw_p = std::stod(c("dw_p", "0.0"));
  const std::string pot = c("potential", "const");
  if (pot == "const") d.potential = CG_POT_CONST;
  else if (pot == "quadratic") d.potential = CG_POT_QUADRATIC;
  else raise(-1, "potential `" + pot + "` (const or quadratic)");
  d.pot_const = std::stod(c("pot_const", "3.0e-4"));
  d.pot_mass = std::stod(c("scalar_mass", "1.0"));
  // dx from the config or the box length (cosmo.cc:41-42); dt = dt_frac dx
  const long double len = std::stold(c("H_LEN_FRAC", "0.5"));
  const long double dx = c.has("dx") ? std::stold(c["dx"]) : len / (long double)d.nx;
  d.dx = (double)dx;
  d.dt = (double)(std::stold(c("dt_frac", "0.1")) * (long double)d.dx);
  frw = std::make_unique<FRW>(this);
  ensure_fields();
}

BSSN::~BSSN() {
  if (c) cg_destroy(c);
}

void BSSN::ensure_fields() {
  regs.clear();
  fields.clear();
  const int nb = cg_num_fields(d.matter), nf = num_fields();
  for (int f = 0; f < nf; ++f) {
    const std::string nm = f < nb ? cg_field_name(d.matter, f)
                                  : (d.z4c && f == nb ? "theta" : kShiftNames[f - nb - d.z4c]);
    regs.push_back(std::make_unique<RK4Register>(this, f, nm));
    RK4Register* r = regs.back().get();
    fields[nm + "_p"] = &r->_array_p;
    fields[nm + "_a"] = &r->_array_a;
    fields[nm + "_f"] = &r->_array_f;
  }
}

RK4Register* BSSN::reg(const std::string& name) {
  for (auto& r : regs)
    if (r->name == name) return r.get();
  raise(-1, "no field `" + name + "` in this box");
}

int BSSN::field_index(const std::string& name) const {
  for (int f = 0; f < cg_num_fields(d.matter); ++f)
    if (name == cg_field_name(d.matter, f)) return f;
  if (d.z4c && name == "theta") return cg_num_fields(d.matter);
  if (d.shift != CG_SHIFT_NONE)
    for (int q = 0; q < 7; ++q)
      if (name == kShiftNames[q]) return cg_num_fields(d.matter) + d.z4c + q;
  raise(-1, "no field `" + name + "` in this box");
}

void BSSN::check(int rc, const char* what) {
  if (rc == CG_OK) return;
  const char* m = cg_last_error(c);
  if (rc == CG_ERR_NAN) raise(10, std::string(what) + ": NAN detected!");
  raise(-1, std::string(what) + ": " + (m ? m : "error"));
}

cg_ctx* BSSN::ctx() {
  if (!c) init();
  return c;
}

void BSSN::init() {
  if (c) return;
  cg_ctx* h = nullptr;
  const int rc = cg_create(&d, 1, &h);
  if (rc != CG_OK) {
    const char* m = cg_last_error(nullptr);
    raise(-1, std::string("creating the box: ") + (m ? m : "error"));
  }
  c = h;
}

void BSSN::setDt(real_t dt) {
  if (c) raise(-1, "dt is fixed once the box is on the GPU");
  d.dt = dt;
}

void BSSN::stepInit() {
  check(cg_step_init(ctx()), "stepInit");
  last_stage = 0;
  stepped_init = true;
  rhs_pending = false;
  sources_set = false;
}

void BSSN::clearSrc() { sources_set = false; }

void BSSN::RKEvolve() {
  if (!stepped_init) raise(-1, "RKEvolve before stepInit");
  rhs_pending = true;
}

void BSSN::finalize(int n) {
  if (!stepped_init) raise(-1, "K" + std::to_string(n) + "Finalize before stepInit");
  if (!rhs_pending) raise(-1, "K" + std::to_string(n) + "Finalize without RKEvolve");
  if (last_stage != n - 1) raise(-1, "K" + std::to_string(n) + "Finalize out of order");
  check(cg_rk_stage(ctx(), n), "RK substep");
  rhs_pending = false;
  // after K4Finalize the next step's first-substep input is already built, so
  // substep 1 may follow directly; stepInit may also be repeated (the
  // reference calls it at the start of every step)
  last_stage = n == 4 ? 0 : n;
}

void BSSN::step() {
  RKEvolve();
  K1Finalize();
  RKEvolve();
  K2Finalize();
  RKEvolve();
  K3Finalize();
  RKEvolve();
  K4Finalize();
}

void BSSN::setConstraintCalcs(real_t H[8], real_t M[8], real_t G[7], real_t A[7], real_t S[7]) {
  check(cg_constraints(ctx(), 0, H, M, G, A, S), "setConstraintCalcs");
}

void BSSN::fieldStatistics(real_t out[9]) { check(cg_field_statistics(ctx(), 0, out, 9), "fieldStatistics"); }

bool BSSN::nan_seen() {
  if (!c) return false;
  const int rc = cg_synchronize(c);
  if (rc == CG_ERR_NAN) return true;
  check(rc, "synchronize");
  return false;
}

void BSSN::loadState(const std::string& path) {
  std::ifstream in(path, std::ios::binary);
  if (!in) raise(-1, "cannot open initial-data file " + path);
  StateHeader h{};
  in.read(reinterpret_cast<char*>(&h), sizeof(h));
  if (!in || std::memcmp(h.magic, "CGSTATE1", 8) != 0) raise(-1, path + " is not a CGSTATE1 state file");
  if (h.matter != d.matter)
    raise(-1, path + " holds matter model " + std::to_string(h.matter) + ", the simulation_type needs " +
                  std::to_string(d.matter));
  const int z4c = (h.reserved & 1) ? 1 : 0;  // the header's flags: theta after the matter fields
  if (z4c != d.z4c) raise(-1, path + (z4c ? " carries theta; set Z4c_damping = 1" : " carries no theta (Z4c_damping = 1)"));
  const int shift = (h.reserved & 2) ? 1 : 0;  // flag bit 1: the shift fields after those
  if (shift != (d.shift != CG_SHIFT_NONE ? 1 : 0))
    raise(-1, path + (shift ? " carries the shift; set BSSN_shift = 1" : " carries no shift (BSSN_shift = 1)"));
  if (h.nfields != cg_num_fields(h.matter) + z4c + 7 * shift || h.nfluids < 0 || h.nfluids > 4 || h.nx <= 0 || h.ny <= 0 ||
      h.nz <= 0)
    raise(-1, path + ": inconsistent header");
  if (c) raise(-1, "initial data must be loaded before the box is on the GPU");
  d.nx = h.nx;
  d.ny = h.ny;
  d.nz = h.nz;
  d.dx = h.dx;
  d.dt = h.dt;
  d.frw_phi = h.frw_phi;
  d.frw_K = h.frw_K;
  d.nfluids = h.nfluids;
  for (int m = 0; m < 4; ++m) {
    d.fluid_rho[m] = h.fluid_rho[m];
    d.fluid_w[m] = h.fluid_w[m];
  }
  d.lambda = h.lambda;
  const size_t count = (size_t)h.nfields * h.nx * h.ny * h.nz;
  std::vector<double> buf(count);
  in.read(reinterpret_cast<char*>(buf.data()), (std::streamsize)(count * sizeof(double)));
  if (!in) raise(-1, path + ": truncated field data");
  check(cg_upload_state(ctx(), 0, buf.data(), count), "upload initial data");
}

void BSSN::saveState(const std::string& path, int step) {
  StateHeader h{};
  std::memcpy(h.magic, "CGSTATE1", 8);
  h.nx = d.nx;
  h.ny = d.ny;
  h.nz = d.nz;
  h.nfields = num_fields();
  h.matter = d.matter;
  h.reserved = (d.z4c ? 1 : 0) | (d.shift != CG_SHIFT_NONE ? 2 : 0);  // flags: theta, then the shift fields
  h.step = step;
  h.dx = d.dx;
  h.dt = d.dt;
  double s[6];
  frw_read(this, s);
  h.frw_phi = s[0];
  h.frw_K = s[1];
  h.nfluids = d.nfluids;
  for (int m = 0; m < 4; ++m) {
    h.fluid_rho[m] = m < d.nfluids ? s[2 + m] : 0.0;
    h.fluid_w[m] = d.fluid_w[m];
  }
  h.lambda = d.lambda;
  const size_t count = (size_t)h.nfields * points();
  std::vector<double> buf(count);
  check(cg_download_state(ctx(), 0, buf.data(), count), "download state");
  std::ofstream out(path, std::ios::binary);
  out.write(reinterpret_cast<const char*>(&h), sizeof(h));
  out.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)(count * sizeof(double)));
  if (!out) raise(-1, "cannot write " + path);
}

// ------------------------------------------------------------- matter facades
void Dust::attach(BSSN* bssn) {
  if (!bssn) raise(-1, "Dust needs a BSSN instance");
  if (bssn->matter() != CG_MATTER_DUST) raise(-1, "the BSSN box was not created with dust");
  if (b == bssn) return;
  b = bssn;
  D = bssn->reg("D");
  S1 = bssn->reg("S1");
  S2 = bssn->reg("S2");
  S3 = bssn->reg("S3");
}

void Dust::stepInit(BSSN* bssn) {
  attach(bssn);
  if (!bssn->rhs_due() && bssn->substep_done() != 0) raise(-1, "Dust::stepInit inside a step");
}

void Dust::addBSSNSrc(BSSN* bssn) {
  attach(bssn);
  bssn->note_sources();
}

void Dust::RKEvolve(BSSN* bssn) {
  attach(bssn);
  if (!bssn->rhs_due()) raise(-1, "Dust::RKEvolve must follow BSSN::RKEvolve");
}

void Dust::finalize(int n) {
  if (!b) raise(-1, "Dust::K" + std::to_string(n) + "Finalize before the dust was attached");
  if (b->substep_done() != n % 4) raise(-1, "Dust::K" + std::to_string(n) + "Finalize before BSSN::K" +
                                             std::to_string(n) + "Finalize");
}

void Static::addBSSNSrc(BSSN* bssn) {
  if (!bssn || bssn->matter() != CG_MATTER_STATIC) raise(-1, "the BSSN box was not created with static matter");
  bssn->note_sources();
}

void Scalar::stepInit(BSSN* bssn) {
  if (!bssn || bssn->matter() != CG_MATTER_SCALAR) raise(-1, "the BSSN box was not created with a scalar field");
  b = bssn;
}

void Scalar::addBSSNSource(BSSN* bssn) {
  stepInit(bssn);
  bssn->note_sources();
}

void Scalar::RKEvolve(BSSN* bssn) {
  stepInit(bssn);
  if (!bssn->rhs_due()) raise(-1, "Scalar::RKEvolve must follow BSSN::RKEvolve");
}

void Scalar::finalize(int n) {
  if (!b) raise(-1, "Scalar::K" + std::to_string(n) + "Finalize before the field was attached");
  if (b->substep_done() != n % 4) raise(-1, "Scalar::K" + std::to_string(n) + "Finalize before BSSN::K" +
                                               std::to_string(n) + "Finalize");
}

void Lambda::addBSSNSource(BSSN* bssn) {
  if (!bssn) raise(-1, "Lambda needs a BSSN instance");
  if (bssn->desc().lambda != lambda) {
    if (bssn->created()) raise(-1, "rho_Lambda differs from the value the box was created with");
    bssn->desc().lambda = lambda;
  }
  bssn->note_sources();
}

// ----------------------------------------------------------------------- sims
CosmoSim::CosmoSim(ConfigParser* config) : cfg(config) {
  iodata = new IOData((*cfg)("output_dir", "output"));
  num_steps = std::stoll((*cfg)["steps"]);
}

CosmoSim::~CosmoSim() {
  delete bssnSim;
  delete iodata;
}

void CosmoSim::simInit() { bssnSim = new BSSN(cfg); }

void CosmoSim::loadICs() {
  if (!cfg->has("ic_file"))
    raise(-1, "set ic_file to a CGSTATE1 state file (written by cosmograph_b200.ics / BoxState.save)");
  const cg_box_desc before = bssnSim->desc();
  const bool keep_dx = cfg->has("dx") || cfg->has("dt_frac");
  bssnSim->loadState((*cfg)["ic_file"]);
  if (keep_dx) {
    // the configuration's dx / dt_frac win over the file's (cosmo.cc:41-42);
    // loadState already created the box, so they must agree
    if (bssnSim->desc().dx != before.dx || bssnSim->desc().dt != before.dt)
      raise(-1, "dx / dt_frac in the configuration differ from the initial-data file");
  }
  iodata->log("Loaded initial data from " + (*cfg)["ic_file"] + " (" + std::to_string(bssnSim->desc().nx) + "x" +
              std::to_string(bssnSim->desc().ny) + "x" + std::to_string(bssnSim->desc().nz) + ").");
}

void CosmoSim::runCommonStepTasks() {
  if (bssnSim->nan_seen()) {
    iodata->log("\nNAN detected!");
    throw 10;
  }
  if (step % 100 == 0) std::cout << "step " << step << " / " << num_steps << "\n" << std::flush;
}

// Field snapshots (io_bssn_fields_snapshot, IO/io.cc:106-158): for every
// field register named by a true "IO_3D_<name>" / "IO_2D_<name>" /
// "IO_1D_<name>" key, at the matching interval.  HDF5 is not available here:
// 3-D grids (all points) and 2-D grids (the first ny*nz points, the x = 0
// plane) are gz-compressed raw little-endian FP64 in the box's memory order
// (x-major, z fastest), named like the reference's files with ".f64.gz" for
// ".h5.gz"; 1-D strips are the reference's gz text rows (IO/io.cc:730-770).
void CosmoSim::outputSnapshots() {
  const std::string step_str = std::to_string(step);
  const cg_box_desc& d = bssnSim->desc();
  auto due = [&](const char* key) {
    const int iv = std::stoi((*cfg)(key, "0"));
    return iv > 0 && step % iv == 0;
  };
  const bool d3 = due("IO_3D_grid_interval"), d2 = due("IO_2D_grid_interval"), d1 = due("IO_1D_grid_interval");
  if (!d3 && !d2 && !d1) return;
  for (const auto& kv : bssnSim->fields) {
    const std::string& name = kv.first;
    const bool w3 = d3 && std::stoi((*cfg)("IO_3D_" + name, "0"));
    const bool w2 = d2 && std::stoi((*cfg)("IO_2D_" + name, "0"));
    const bool w1 = d1 && std::stoi((*cfg)("IO_1D_" + name, "0"));
    if (!w3 && !w2 && !w1) continue;
    const std::vector<double> v = kv.second->values();
    auto dump_raw = [&](const std::string& fn, size_t count) {
      gzFile f = gzopen(fn.c_str(), "wb");
      if (!f) {
        iodata->log("Error opening file: " + fn);
        return;
      }
      // gzwrite takes an unsigned byte count: write in pieces of at most
      // 1 GiB so that boxes above 4 GiB per field are written whole
      const char* p = reinterpret_cast<const char*>(v.data());
      size_t left = count * sizeof(double);
      bool ok = true;
      while (left > 0 && ok) {
        const unsigned piece = (unsigned)std::min<size_t>(left, (size_t)1 << 30);
        ok = gzwrite(f, p, piece) == (int)piece;
        p += piece;
        left -= piece;
      }
      if (gzclose(f) != Z_OK || !ok) iodata->log("Error writing file: " + fn);
    };
    if (w3) dump_raw(iodata->dir() + "3D_" + name + step_str + ".3d_grid.f64.gz", v.size());
    if (w2) dump_raw(iodata->dir() + "2D_" + name + step_str + ".2d_grid.f64.gz", (size_t)d.ny * d.nz);
    if (w1) {
      const int axis = std::stoi((*cfg)("IO_1D_" + name + "_axis", "1"));
      const long n1 = std::stol((*cfg)("IO_1D_" + name + "_xoffset", "0"));
      const long n2 = std::stol((*cfg)("IO_1D_" + name + "_yoffset", "0"));
      const std::string fn = iodata->dir() + "1D_" + name + ".strip.dat.gz";
      gzFile f = gzopen(fn.c_str(), "ab");
      if (!f) {
        iodata->log("Error opening file: " + fn);
        continue;
      }
      auto at = [&](long i, long j, long k) { return v[((size_t)i * d.ny + j) * d.nz + k]; };
      std::string row;
      const long len = axis == 1 ? d.nx : (axis == 2 ? d.ny : d.nz);
      for (long q = 0; q < len; ++q) {
        const double x = axis == 1 ? at(q, n1, n2) : (axis == 2 ? at(n1, q, n2) : at(n1, n2, q));
        row += fmt15(x) + "\t";
      }
      row += "\n";
      gzwrite(f, row.data(), (unsigned)row.size());
      gzclose(f);
    }
  }
}

void CosmoSim::outputCommon() {
  outputSnapshots();
  const int ci = std::stoi((*cfg)("IO_constraint_interval", "0"));
  if (ci > 0 && step % ci == 0) {
    real_t H[8] = {0}, M[8] = {0}, G[7] = {0}, A[7] = {0}, S[7] = {0};
    bssnSim->setConstraintCalcs(H, M, G, A, S);
    // columns of io_bssn_constraint_violation (IO/io.cc:241-277)
    dump_value(iodata, H[4], "H_violations", "\t");
    dump_value(iodata, H[5], "H_violations", "\t");
    dump_value(iodata, H[6], "H_violations", "\t");
    dump_value(iodata, H[2], "H_violations", "\t");
    dump_value(iodata, H[7], "H_violations", "\n");
    dump_value(iodata, M[4], "M_violations", "\t");
    dump_value(iodata, M[5], "M_violations", "\t");
    dump_value(iodata, M[6], "M_violations", "\t");
    dump_value(iodata, M[2], "M_violations", "\t");
    dump_value(iodata, M[7], "M_violations", "\n");
    const real_t* rest[3] = {G, A, S};
    const char* names[3] = {"G_violations", "A_violations", "S_violations"};
    for (int q = 0; q < 3; ++q) {
      dump_value(iodata, rest[q][4], names[q], "\t");
      dump_value(iodata, rest[q][5], names[q], "\t");
      dump_value(iodata, rest[q][6], names[q], "\t");
      dump_value(iodata, rest[q][2], names[q], "\n");
    }
  }
  const int si = std::stoi((*cfg)("IO_bssnstats_interval", "0"));
  if (si > 0 && step % si == 0) {
    // FRW columns of io_bssn_dump_statistics (IO/io.cc:354-376)
    const std::string fn = iodata->dir() + (*cfg)["dump_file"] + ".frwdat.gz";
    gzFile f = gzopen(fn.c_str(), "ab");
    if (!f) {
      iodata->log("Error opening file: " + fn);
    } else {
      std::string row;
      for (double v : {bssnSim->frw->get_phi(), bssnSim->frw->get_K(), bssnSim->frw->get_rho(),
                       bssnSim->frw->get_S()})
        row += fmt15(v) + "\t";
      row += "\n";
      gzwrite(f, row.data(), (unsigned)row.size());
      gzclose(f);
    }
    // field statistics (IO/io.cc:378-403): DETAILS of DIFFphi, DIFFK, DIFFr,
    // ricci, then the volume average
    const std::string fs = iodata->dir() + (*cfg)["dump_file"] + ".dat.gz";
    gzFile g = gzopen(fs.c_str(), "ab");
    if (!g) {
      iodata->log("Error opening file: " + fs);
    } else {
      real_t st[9];
      bssnSim->fieldStatistics(st);
      std::string row;
      for (double v : st) row += fmt15(v) + "\t";
      row += "\n";
      gzwrite(g, row.data(), (unsigned)row.size());
      gzclose(g);
    }
  }
}

void CosmoSim::outputStateInformation() {
  bssnSim->stepInit();
  iodata->log("---- Information from step " + std::to_string(step) + " of " + std::to_string(num_steps) + " ----");
  auto stats = [&](const char* name, double shift) {
    const std::vector<double> v = bssnSim->fields[std::string(name) + "_a"]->values();
    double s = 0.0, lo = v[0], hi = v[0];
    for (double x : v) {
      s += x;
      lo = std::min(lo, x);
      hi = std::max(hi, x);
    }
    return fmt15(s / (double)v.size() + shift) + " | " + fmt15(lo + shift) + " | " + fmt15(hi + shift);
  };
  iodata->log("Average | Min | Max conformal factor: " + stats("DIFFphi", bssnSim->frw->get_phi()));
  iodata->log("Average | Min | Max extrinsic curvature: " + stats("DIFFK", bssnSim->frw->get_K()));
  real_t H[8] = {0}, M[8] = {0}, G[7] = {0}, A[7] = {0}, S[7] = {0};
  bssnSim->setConstraintCalcs(H, M, G, A, S);
  iodata->log("Max. (Normed) Hamiltonian constraint violation: " + fmt15(H[2]) + " (" + fmt15(H[6]) + ")");
  iodata->log("Max. (Normed) Momentum constraint violation: " + fmt15(M[2]) + " (" + fmt15(M[6]) + ")");
  iodata->log("---- ---- ---- ----");
}

void CosmoSim::run() {
  iodata->log("Running simulation...");
  const bool stop_at_goal = std::stod((*cfg)("stop_at_expansion_goal", "0")) != 0.0;
  const double goal = std::stod((*cfg)("expansion_goal", "100.0"));
  double vol0 = 1.0;
  auto avg_vol = [&]() {
    // exp(6 <DIFFphi>) with exp(6 (DIFFphi + phi_FRW)) weights (bssn.cc:169)
    double* p = nullptr;
    bssnSim->check(cg_device_register(bssnSim->ctx(), 0, 'p', &p), "device register");
    const double* phi = p + (size_t)bssnSim->field_index("DIFFphi") * bssnSim->points();
    double avg = 0.0;
    bssnSim->check(cg_conformal_average(bssnSim->ctx(), phi, phi, bssnSim->points(), bssnSim->frw->get_phi(), &avg),
                   "conformal average");
    return std::exp(6.0 * avg);
  };
  // sims/sim.cc:103-122: steps 0..num_steps inclusive
  while (step <= num_steps) {
    runStep();
    t += bssnSim->desc().dt;
    if (stop_at_goal) {
      if (step == 0) {
        vol0 = avg_vol();
      } else if (std::pow(avg_vol() / vol0, 1.0 / 3.0) >= goal) {
        iodata->log("Target expasion reached, run ending.");
        break;
      }
    }
    ++step;
  }
  iodata->log("\nEnding simulation.");
  outputStateInformation();
  if (cfg->has("output_file")) bssnSim->saveState((*cfg)["output_file"], (int)step);
  iodata->log("RK_steps: " + fmt15(rk_seconds) + " s");
}

DustSim::DustSim(ConfigParser* config) : CosmoSim(config) {
  if ((*config)("shift", "") != "") {
    iodata->log("Error - non-zero shift not ok for this class!");
    throw -1;
  }
}

DustSim::~DustSim() {
  delete dustSim;
  delete lambda;
}

void DustSim::init() {
  simInit();
  iodata->log("Initializing 'dust' type simulation.");
  dustSim = new Dust();
  lambda = new Lambda();
}

void DustSim::setICs() {
  iodata->log("Setting dust initial conditions.");
  if (cfg->has("ic_file")) {
    loadICs();
  } else {
    // dust_ic_set_random (sims/dust.cc:40-51) built on the GPU from a seeded
    // Gaussian random density contrast: rms_delta, spectral index ns, cutoff
    // ic_spec_cut (modes; default N/4), rho_Lambda = Omega_L * 3 / (8 pi)
    const double omega_l = std::stod((*cfg)("Omega_L", "0.0"));
    bssnSim->desc().lambda = omega_l * 3.0 / (8.0 * 3.14159265358979323846);
    const uint64_t seed = std::stoull((*cfg)("seed", "9"));
    const double rms = std::stod((*cfg)("rms_delta", "1.0e-4"));
    const double ns = std::stod((*cfg)("ns", "0.96"));
    const double cut = std::stod((*cfg)("ic_spec_cut", "0"));
    iodata->log("Setting cosmological ICs (GPU): seed " + std::to_string(seed) + ", rms delta " + fmt15(rms));
    bssnSim->check(cg_ic_grf_dust(bssnSim->ctx(), 0, nullptr, seed, rms, ns, cut), "GRF initial data");
  }
  lambda->setLambda(bssnSim->desc().lambda);
  iodata->log("Finished setting ICs.");
}

void DustSim::initDustStep() {
  const auto t0 = std::chrono::steady_clock::now();
  bssnSim->stepInit();
  dustSim->stepInit(bssnSim);
  bssnSim->clearSrc();
  dustSim->addBSSNSrc(bssnSim);
  lambda->addBSSNSource(bssnSim);
  rk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void DustSim::runDustStep() {
  const auto t0 = std::chrono::steady_clock::now();
  // sims/dust.cc:114-161
  bssnSim->RKEvolve();
  dustSim->RKEvolve(bssnSim);
  bssnSim->K1Finalize();
  dustSim->K1Finalize();
  for (int n = 2; n <= 4; ++n) {
    bssnSim->clearSrc();
    dustSim->addBSSNSrc(bssnSim);
    lambda->addBSSNSource(bssnSim);
    bssnSim->RKEvolve();
    dustSim->RKEvolve(bssnSim);
    if (n == 2) {
      bssnSim->K2Finalize();
      dustSim->K2Finalize();
    } else if (n == 3) {
      bssnSim->K3Finalize();
      dustSim->K3Finalize();
    } else {
      bssnSim->K4Finalize();
      dustSim->K4Finalize();
    }
  }
  rk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void DustSim::runStep() {
  // sims/dust.cc:163-169
  initDustStep();
  runCommonStepTasks();
  outputCommon();
  if (step == 0) outputStateInformation();
  runDustStep();
}

ScalarSim::~ScalarSim() { delete scalarSim; }

void ScalarSim::init() {
  simInit();
  iodata->log("Running 'scalar' type simulation.");
  scalarSim = new Scalar();
}

void ScalarSim::setICs() {
  iodata->log("Setting initial conditions (ICs).");
  if (cfg->has("ic_file")) {
    loadICs();
  } else {
    // the GRF scalar configuration built on the GPU: phi = scalar_phi0 + a
    // k^-3 Gaussian random fluctuation of rms scalar_rms cut off at
    // ic_spec_cut modes (default N/4), Pi = 0, psi_i = d_i phi, K from the
    // local energy density with the run's scalar_mass
    const uint64_t seed = std::stoull((*cfg)("seed", "9"));
    const double phi0 = std::stod((*cfg)("scalar_phi0", "1.0e-2"));
    const double rms = std::stod((*cfg)("scalar_rms", "1.0e-5"));
    const double cut = std::stod((*cfg)("ic_spec_cut", "0"));
    const double mass = bssnSim->desc().pot_mass;
    iodata->log("Setting GRF scalar ICs (GPU): seed " + std::to_string(seed) + ", phi0 " + fmt15(phi0) + ", rms " +
                fmt15(rms));
    bssnSim->check(cg_ic_grf_scalar(bssnSim->ctx(), 0, nullptr, seed, phi0, rms, mass, cut), "GRF scalar initial data");
  }
  iodata->log("Finished setting ICs.");
}

void ScalarSim::initScalarStep() {
  const auto t0 = std::chrono::steady_clock::now();
  bssnSim->stepInit();
  scalarSim->stepInit(bssnSim);
  bssnSim->clearSrc();
  scalarSim->addBSSNSource(bssnSim);
  rk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void ScalarSim::runScalarStep() {
  const auto t0 = std::chrono::steady_clock::now();
  // sims/scalar.cc:97-151
  for (int n = 1; n <= 4; ++n) {
    if (n > 1) {
      bssnSim->clearSrc();
      scalarSim->addBSSNSource(bssnSim);
    }
    bssnSim->RKEvolve();
    scalarSim->RKEvolve(bssnSim);
    if (n == 1) {
      bssnSim->K1Finalize();
      scalarSim->K1Finalize();
    } else if (n == 2) {
      bssnSim->K2Finalize();
      scalarSim->K2Finalize();
    } else if (n == 3) {
      bssnSim->K3Finalize();
      scalarSim->K3Finalize();
    } else {
      bssnSim->K4Finalize();
      scalarSim->K4Finalize();
    }
  }
  rk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void ScalarSim::runStep() {
  // sims/scalar.cc:153-160
  runCommonStepTasks();
  initScalarStep();
  outputCommon();
  runScalarStep();
}

StaticSim::StaticSim(ConfigParser* config) : CosmoSim(config) {
  // sims/static.cc:11-17
  const std::string lapse = (*config)("lapse", "");
  if (lapse != "" && lapse != "Static" && lapse != "ConformalFLRW") {
    iodata->log("Error - not using a constant lapse gauge! You must use it for 'static' sims.");
    iodata->log("Please change this setting in the config file and re-run.");
    throw -1;
  }
}

StaticSim::~StaticSim() {
  delete staticSim;
  delete lambda;
}

void StaticSim::init() {
  simInit();
  iodata->log("Initializing 'static' type simulation.");
  staticSim = new Static();
  staticSim->init();
  lambda = new Lambda();
}

void StaticSim::setICs() {
  iodata->log("Setting static initial conditions (ICs).");
  loadICs();
  lambda->setLambda(bssnSim->desc().lambda);
  iodata->log("Finished setting ICs.");
}

void StaticSim::initStaticStep() {
  const auto t0 = std::chrono::steady_clock::now();
  // sims/static.cc:71-80
  bssnSim->stepInit();
  bssnSim->clearSrc();
  staticSim->addBSSNSrc(bssnSim);
  lambda->addBSSNSource(bssnSim);
  rk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void StaticSim::runStaticStep() {
  const auto t0 = std::chrono::steady_clock::now();
  // sims/static.cc:131-167 (without the ray sheets)
  for (int n = 1; n <= 4; ++n) {
    if (n > 1) {
      bssnSim->clearSrc();
      staticSim->addBSSNSrc(bssnSim);
      lambda->addBSSNSource(bssnSim);
    }
    bssnSim->RKEvolve();
    if (n == 1) bssnSim->K1Finalize();
    else if (n == 2) bssnSim->K2Finalize();
    else if (n == 3) bssnSim->K3Finalize();
    else bssnSim->K4Finalize();
  }
  rk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

void StaticSim::runStep() {
  // sims/static.cc:169-175
  initStaticStep();
  runCommonStepTasks();
  outputCommon();
  if (step == 0) outputStateInformation();
  runStaticStep();
}

void VacuumSim::init() {
  simInit();
  iodata->log("Running 'vacuum' type simulation.");
}

void VacuumSim::setICs() {
  loadICs();
  iodata->log("Finished setting ICs.");
}

void VacuumSim::runStep() {
  // sims/vacuum.cc:100-107
  runCommonStepTasks();
  const auto t0 = std::chrono::steady_clock::now();
  bssnSim->stepInit();
  rk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  outputCommon();
  const auto t1 = std::chrono::steady_clock::now();
  bssnSim->step();
  rk_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
}

// ---------------------------------------------------------------- the driver
int run_config_file(const std::string& fname) {
  try {
    ConfigParser config(fname);
    const std::string sim = config["simulation_type"];
    std::unique_ptr<CosmoSim> s;
    if (sim == "dust") s = std::make_unique<DustSim>(&config);
    else if (sim == "scalar") s = std::make_unique<ScalarSim>(&config);
    else if (sim == "vacuum") s = std::make_unique<VacuumSim>(&config);
    else if (sim == "static") s = std::make_unique<StaticSim>(&config);
    else {
      std::cerr << "Invalid simulation type specified. ";
      throw 2;
    }
    s->init();
    s->setICs();
    s->run();
  } catch (int code) {
    std::cerr << "cosmo_b200: stopped (code " << code << ")\n";
    return code == 0 ? EXIT_FAILURE : (code < 0 ? 1 : code);
  }
  return EXIT_SUCCESS;
}

}  // namespace cosmo
