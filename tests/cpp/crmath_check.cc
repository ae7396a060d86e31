// crmath_check.cc -- the correctly rounded exp / expm1 / log1p of
// cosmograph_b200/csrc/cg_crmath.h, compiled for the host, against 113-bit
// quad-precision evaluations (libquadmath) rounded once to double.
//
// Usage: crmath_check <exp|expm1|log1p> <count> <seed> [lo hi]
//   random arguments, uniform in [lo, hi] (default: the function's whole
//   useful range), plus the edge cases; prints one line:
//   "<fn> checked=N mismatches=M first=<x>"
// Usage: crmath_check eval <exp|expm1|log1p>   (reads doubles as hex bit
//   patterns from stdin, writes the results as hex bit patterns)
#include <quadmath.h>

#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "cg_crmath.h"

namespace {

double ref(const std::string& fn, double x) {
  const __float128 q = x;
  if (fn == "exp") return (double)expq(q);
  if (fn == "expm1") return (double)expm1q(q);
  return (double)log1pq(q);
}

double crm(const std::string& fn, double x) {
  if (fn == "exp") return cg::crm::exp(x);
  if (fn == "expm1") return cg::crm::expm1(x);
  return cg::crm::log1p(x);
}

bool same(double a, double b) {
  if (a != a && b != b) return true;
  return cg::crm::bits(a) == cg::crm::bits(b);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) return 2;
  const std::string mode = argv[1];
  if (mode == "eval") {
    const std::string fn = argv[2];
    char line[64];
    while (std::fgets(line, sizeof line, stdin)) {
      const int64_t b = (int64_t)std::strtoull(line, nullptr, 16);
      std::printf("%016" PRIx64 "\n", (uint64_t)cg::crm::bits(crm(fn, cg::crm::from_bits(b))));
    }
    return 0;
  }
  const std::string fn = mode;
  const long count = std::atol(argv[2]);
  const unsigned seed = argc > 3 ? (unsigned)std::atol(argv[3]) : 1u;
  double lo = fn == "log1p" ? -0.999 : -745.2, hi = fn == "log1p" ? 1e6 : 709.9;
  if (argc > 5) {
    lo = std::atof(argv[4]);
    hi = std::atof(argv[5]);
  }
  std::vector<double> xs = {0.0, -0.0, 1e-300, -1e-300, 0x1p-54, -0x1p-54, 0x1p-53, 1e-17, -1e-17, 1e-13,
                            -1e-13, 0.0054, -0.0054, 0.005415, 1.0, -1.0, 0.5, 2.0, 10.0, -10.0, 40.0, -40.0,
                            709.78, 709.79, -708.39, -708.4, -745.13, -745.14, -744.5, 1e300, 5e-324};
  // structured arguments (powers of two and their neighbours), where the
  // result can lie very close to a rounding midpoint
  for (int e = 1; e <= 80; ++e)
    for (double m : {1.0, 1.5, 1.25, 1.0 + 0x1p-52, 1.0 - 0x1p-53, 3.0, 5.0})
      for (double sg : {1.0, -1.0}) xs.push_back(sg * std::ldexp(m, -e));
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> uni(lo, hi);
  std::uniform_real_distribution<double> expo(-60.0, 0.0);
  for (long n = 0; n < count; ++n) {
    double x;
    switch (n % 4) {
      case 0: x = uni(rng); break;
      case 1: x = std::ldexp(1.0, (int)expo(rng)) * (uni(rng) / (hi - lo + 1e-300)); break;  // small magnitudes
      case 2: x = (uni(rng) - 0.5 * (lo + hi)) * 1e-4; break;
      default: x = std::ldexp(uni(rng) / (hi - lo + 1e-300), -(int)(rng() % 50)); break;
    }
    if (fn == "log1p" && x <= -1.0) x = -0.5;
    xs.push_back(x);
  }
  long mism = 0;
  double first = 0.0;
  if (fn == "exp") {
    // the batched form (exp_n) must return the same bits as exp()
    for (size_t q = 0; q + 4 <= xs.size(); q += 4) {
      const double in[4] = {xs[q], xs[q + 1], xs[q + 2], xs[q + 3]};
      double out[4];
      cg::crm::exp_n<4>(in, out);
      for (int n = 0; n < 4; ++n)
        if (!same(out[n], cg::crm::exp(in[n]))) {
          if (mism == 0) first = in[n];
          ++mism;
        }
    }
  }
  for (double x : xs) {
    if (fn == "log1p" && x < -1.0) continue;
    const double a = crm(fn, x), b = ref(fn, x);
    if (!same(a, b)) {
      if (mism == 0) first = x;
      ++mism;
    }
  }
  std::printf("%s checked=%zu mismatches=%ld first=%a\n", fn.c_str(), xs.size(), mism, first);
  return mism == 0 ? 0 : 1;
}
