// cg_crmath.h -- correctly rounded exp, expm1 and log1p in binary64
// (round to nearest, ties to even), for the FP64 parity build.
//
// Why: the reference evaluates e^x, expm1 and log1p through the host C
// library.  Libraries differ in the last bit of these functions (CUDA's are
// within 1-2 ulp, current glibc's exp within about 0.51 ulp), and a long BSSN
// run amplifies last-bit differences.  A correctly rounded result is the one
// value every exact implementation must return, so the parity build uses it,
// and the reference can be run against a correctly rounded C library to
// compare bit for bit.
//
// Method (written for this file; the standard published techniques):
//   * argument reduction x = k ln2/64 + r, |r| <= ln2/128, with ln2/64 split
//     into three parts (the first with 36 significant bits, so that k times
//     it is exact for |k| < 2^17) -- Cody-Waite reduction;
//   * e^x = 2^(k>>6) * 2^((k&63)/64) * e^r with a 64-entry table of
//     2^(j/64) held as double-double (Tang's table-driven method);
//   * e^r - 1 by its Taylor series, evaluated in double-double arithmetic
//     (Dekker's two-product through fma, Knuth's two-sum);
//   * Ziv's rounding test: a fast evaluation with a proven error bound
//     (below 2^-64 relative) is returned when every value inside the bound
//     rounds the same way; otherwise a double-double evaluation (error about
//     2^-100) decides;
//   * log1p by one Newton step on the double-double exponential from a 1-ulp
//     start value.
// The table and constants are values of 2^(j/64), ln2/64, 64/ln2 and 1/n!
// computed to 100 decimal digits and rounded to double / double-double.
//
// The same code compiles for the host (tests compare it against 113-bit
// quad-precision evaluations) and for the device; every operation is an
// explicit round-to-nearest add, multiply or fma, so no compiler contraction
// or reassociation changes a result.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define CRM_FN __host__ __device__ __forceinline__
#else
#define CRM_FN static inline
#endif

namespace cg {
namespace crm {

#if defined(__CUDA_ARCH__)
CRM_FN double add(double a, double b) { return __dadd_rn(a, b); }
CRM_FN double sub(double a, double b) { return __dsub_rn(a, b); }
CRM_FN double mul(double a, double b) { return __dmul_rn(a, b); }
CRM_FN double fma_(double a, double b, double c) { return __fma_rn(a, b, c); }
CRM_FN double rint_(double a) { return rint(a); }
CRM_FN int64_t bits(double a) { return __double_as_longlong(a); }
CRM_FN double from_bits(int64_t b) { return __longlong_as_double(b); }
#else
// host: the including translation unit is compiled without FP contraction
CRM_FN double add(double a, double b) { return a + b; }
CRM_FN double sub(double a, double b) { return a - b; }
CRM_FN double mul(double a, double b) { return a * b; }
CRM_FN double fma_(double a, double b, double c) { return std::fma(a, b, c); }
CRM_FN double rint_(double a) { return std::nearbyint(a); }
CRM_FN int64_t bits(double a) {
  int64_t b;
  std::memcpy(&b, &a, sizeof b);
  return b;
}
CRM_FN double from_bits(int64_t b) {
  double a;
  std::memcpy(&a, &b, sizeof a);
  return a;
}
#endif

struct DD {
  double hi, lo;
};

// a + b = s + e exactly (Knuth)
CRM_FN DD two_sum(double a, double b) {
  const double s = add(a, b);
  const double bb = sub(s, a);
  const double e = add(sub(a, sub(s, bb)), sub(b, bb));
  return {s, e};
}
// a * b = p + e exactly (fma)
CRM_FN DD two_prod(double a, double b) {
  const double p = mul(a, b);
  return {p, fma_(a, b, -p)};
}
// double-double arithmetic, relative error about 2^-104 per operation
CRM_FN DD dd_add(DD a, DD b) {
  DD s = two_sum(a.hi, b.hi);
  DD t = two_sum(a.lo, b.lo);
  s.lo = add(s.lo, t.hi);
  s = two_sum(s.hi, s.lo);
  s.lo = add(s.lo, t.lo);
  return two_sum(s.hi, s.lo);
}
CRM_FN DD dd_mul(DD a, DD b) {
  DD p = two_prod(a.hi, b.hi);
  p.lo = add(p.lo, add(mul(a.hi, b.lo), mul(a.lo, b.hi)));
  return two_sum(p.hi, p.lo);
}
CRM_FN DD dd_mul_d(DD a, double b) {
  DD p = two_prod(a.hi, b);
  p.lo = fma_(a.lo, b, p.lo);
  return two_sum(p.hi, p.lo);
}

// 2^(j/64), j = 0..63: hi = the nearest double, lo = the nearest double to
// the remainder
#define CG_CRM_EXP2_TABLE \
  0x1.0000000000000p+0, 0x0.0p+0, \
  0x1.02c9a3e778061p+0, -0x1.19083535b085dp-56, \
  0x1.059b0d3158574p+0, 0x1.d73e2a475b465p-55, \
  0x1.0874518759bc8p+0, 0x1.186be4bb284ffp-57, \
  0x1.0b5586cf9890fp+0, 0x1.8a62e4adc610bp-54, \
  0x1.0e3ec32d3d1a2p+0, 0x1.03a1727c57b53p-59, \
  0x1.11301d0125b51p+0, -0x1.6c51039449b3ap-54, \
  0x1.1429aaea92de0p+0, -0x1.32fbf9af1369ep-54, \
  0x1.172b83c7d517bp+0, -0x1.19041b9d78a76p-55, \
  0x1.1a35beb6fcb75p+0, 0x1.e5b4c7b4968e4p-55, \
  0x1.1d4873168b9aap+0, 0x1.e016e00a2643cp-54, \
  0x1.2063b88628cd6p+0, 0x1.dc775814a8495p-55, \
  0x1.2387a6e756238p+0, 0x1.9b07eb6c70573p-54, \
  0x1.26b4565e27cddp+0, 0x1.2bd339940e9d9p-55, \
  0x1.29e9df51fdee1p+0, 0x1.612e8afad1255p-55, \
  0x1.2d285a6e4030bp+0, 0x1.0024754db41d5p-54, \
  0x1.306fe0a31b715p+0, 0x1.6f46ad23182e4p-55, \
  0x1.33c08b26416ffp+0, 0x1.32721843659a6p-54, \
  0x1.371a7373aa9cbp+0, -0x1.63aeabf42eae2p-54, \
  0x1.3a7db34e59ff7p+0, -0x1.5e436d661f5e3p-56, \
  0x1.3dea64c123422p+0, 0x1.ada0911f09ebcp-55, \
  0x1.4160a21f72e2ap+0, -0x1.ef3691c309278p-58, \
  0x1.44e086061892dp+0, 0x1.89b7a04ef80d0p-59, \
  0x1.486a2b5c13cd0p+0, 0x1.3c1a3b69062f0p-56, \
  0x1.4bfdad5362a27p+0, 0x1.d4397afec42e2p-56, \
  0x1.4f9b2769d2ca7p+0, -0x1.4b309d25957e3p-54, \
  0x1.5342b569d4f82p+0, -0x1.07abe1db13cadp-55, \
  0x1.56f4736b527dap+0, 0x1.9bb2c011d93adp-54, \
  0x1.5ab07dd485429p+0, 0x1.6324c054647adp-54, \
  0x1.5e76f15ad2148p+0, 0x1.ba6f93080e65ep-54, \
  0x1.6247eb03a5585p+0, -0x1.383c17e40b497p-54, \
  0x1.6623882552225p+0, -0x1.bb60987591c34p-54, \
  0x1.6a09e667f3bcdp+0, -0x1.bdd3413b26456p-54, \
  0x1.6dfb23c651a2fp+0, -0x1.bbe3a683c88abp-57, \
  0x1.71f75e8ec5f74p+0, -0x1.16e4786887a99p-55, \
  0x1.75feb564267c9p+0, -0x1.0245957316dd3p-54, \
  0x1.7a11473eb0187p+0, -0x1.41577ee04992fp-55, \
  0x1.7e2f336cf4e62p+0, 0x1.05d02ba15797ep-56, \
  0x1.82589994cce13p+0, -0x1.d4c1dd41532d8p-54, \
  0x1.868d99b4492edp+0, -0x1.fc6f89bd4f6bap-54, \
  0x1.8ace5422aa0dbp+0, 0x1.6e9f156864b27p-54, \
  0x1.8f1ae99157736p+0, 0x1.5cc13a2e3976cp-55, \
  0x1.93737b0cdc5e5p+0, -0x1.75fc781b57ebcp-57, \
  0x1.97d829fde4e50p+0, -0x1.d185b7c1b85d1p-54, \
  0x1.9c49182a3f090p+0, 0x1.c7c46b071f2bep-56, \
  0x1.a0c667b5de565p+0, -0x1.359495d1cd533p-54, \
  0x1.a5503b23e255dp+0, -0x1.d2f6edb8d41e1p-54, \
  0x1.a9e6b5579fdbfp+0, 0x1.0fac90ef7fd31p-54, \
  0x1.ae89f995ad3adp+0, 0x1.7a1cd345dcc81p-54, \
  0x1.b33a2b84f15fbp+0, -0x1.2805e3084d708p-57, \
  0x1.b7f76f2fb5e47p+0, -0x1.5584f7e54ac3bp-56, \
  0x1.bcc1e904bc1d2p+0, 0x1.23dd07a2d9e84p-55, \
  0x1.c199bdd85529cp+0, 0x1.11065895048ddp-55, \
  0x1.c67f12e57d14bp+0, 0x1.2884dff483cadp-54, \
  0x1.cb720dcef9069p+0, 0x1.503cbd1e949dbp-56, \
  0x1.d072d4a07897cp+0, -0x1.cbc3743797a9cp-54, \
  0x1.d5818dcfba487p+0, 0x1.2ed02d75b3707p-55, \
  0x1.da9e603db3285p+0, 0x1.c2300696db532p-54, \
  0x1.dfc97337b9b5fp+0, -0x1.1a5cd4f184b5cp-54, \
  0x1.e502ee78b3ff6p+0, 0x1.39e8980a9cc8fp-55, \
  0x1.ea4afa2a490dap+0, -0x1.e9c23179c2893p-54, \
  0x1.efa1bee615a27p+0, 0x1.dc7f486a4b6b0p-54, \
  0x1.f50765b6e4540p+0, 0x1.9d3e12dd8a18bp-54, \
  0x1.fa7c1819e90d8p+0, 0x1.74853f3a5931ep-55, \

#if defined(__CUDACC__)
static __device__ const double kExp2TableDev[128] = {CG_CRM_EXP2_TABLE};
#endif
static const double kExp2TableHost[128] = {CG_CRM_EXP2_TABLE};
#undef CG_CRM_EXP2_TABLE

CRM_FN const double* exp2_table() {
#if defined(__CUDA_ARCH__)
  return kExp2TableDev;
#else
  return kExp2TableHost;
#endif
}

constexpr double kInvL = 0x1.71547652b82fep+6;   // 64 / ln 2
constexpr double kL1 = 0x1.62e42fefa0000p-7;     // ln2/64, first 36 bits
constexpr double kL2 = 0x1.cf79abc9e3b3ap-46;    // next 53 bits
constexpr double kL3 = -0x1.ff0342542fc33p-100;  // next 53 bits
constexpr double kExpMax = 710.0;                // e^x overflows beyond (the exact bound is 709.78...)
constexpr double kExpMin = -745.14;              // e^x rounds to +0 below (exact bound -745.1332...)
constexpr double kExpSub = -708.39;              // e^x is subnormal below (exact bound -708.3964...)

// x = k ln2/64 + (rh + rl); returns k.  |rh| <= ln2/128 + tiny, and
// rh + rl is within 2^-130 of x - k ln2/64 for |x| <= 746.
CRM_FN int reduce(double x, double& rh, double& rl) {
  const double kd = rint_(mul(x, kInvL));
  const double t = sub(x, mul(kd, kL1));  // exact: kd*kL1 has <= 53 bits, Sterbenz
  const DD u = two_prod(kd, kL2);
  const DD r = two_sum(t, -u.hi);
  rh = r.hi;
  rl = sub(sub(r.lo, u.lo), mul(kd, kL3));
  const DD n = two_sum(rh, rl);
  rh = n.hi;
  rl = n.lo;
  return (int)kd;
}

// 1/(n+1)!, n = 0..11: hi parts, and the lo parts of n <= 5 (the terms
// evaluated in double-double)
#define CG_CRM_COEF_HI 1.0, 0.5, 0x1.5555555555555p-3, 0x1.5555555555555p-5, 0x1.1111111111111p-7, \
    0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13, 0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19,      \
    0x1.27e4fb7789f5cp-22, 0x1.ae64567f544e4p-26, 0x1.1eed8eff8d898p-29
#define CG_CRM_COEF_LO 0.0, 0.0, 0x1.5555555555555p-57, 0x1.5555555555555p-59, 0x1.1111111111111p-63, \
    -0x1.f49f49f49f49fp-65
#if defined(__CUDACC__)
static __constant__ const double kCoefHiDev[12] = {CG_CRM_COEF_HI};
static __constant__ const double kCoefLoDev[6] = {CG_CRM_COEF_LO};
#endif
static const double kCoefHiHost[12] = {CG_CRM_COEF_HI};
static const double kCoefLoHost[6] = {CG_CRM_COEF_LO};
#undef CG_CRM_COEF_HI
#undef CG_CRM_COEF_LO
CRM_FN double coef_hi(int n) {
#if defined(__CUDA_ARCH__)
  return kCoefHiDev[n];
#else
  return kCoefHiHost[n];
#endif
}
CRM_FN double coef_lo(int n) {
#if defined(__CUDA_ARCH__)
  return kCoefLoDev[n];
#else
  return kCoefLoHost[n];
#endif
}

// e^r - 1 = r * P(r), P(r) = sum r^n/(n+1)!, r = rh + rl, in double-double
// (error below 2^-103 relative for |r| <= 0.0055).  Rolled loops: this is
// the accurate phase, which runs rarely, and a small body keeps the code of
// every call site small.
CRM_FN DD expm1_small_dd(double rh, double rl) {
  // tail n = 11..6 in double: |r^6/7!| < 2^-61, so its rounding stays below 2^-110
  double t = coef_hi(11);
#pragma unroll 1
  for (int n = 10; n >= 6; --n) t = fma_(t, rh, coef_hi(n));
  // n = 5..0 in double-double: P = P * r + 1/(n+1)!
  const DD r{rh, rl};
  DD P{t, 0.0};
#pragma unroll 1
  for (int n = 5; n >= 0; --n) P = dd_add(dd_mul(P, r), DD{coef_hi(n), coef_lo(n)});
  return dd_mul(P, r);
}

// 2^(j/64) (1 + s) in double-double, j = k & 63
CRM_FN DD table_times(int j, DD s) {
  const double* T = exp2_table();
  const DD Tj{T[2 * j], T[2 * j + 1]};
  return dd_add(Tj, dd_mul(Tj, s));
}

// x * 2^m for a finite double x and m in [-1100, 1100], with one rounding
// (the product is exact unless it under- or overflows)
CRM_FN double scale2(double x, int m) {
  // split m so that every factor 2^e is a normal double
  while (m > 1000) {
    x = mul(x, 0x1p+1000);
    m -= 1000;
  }
  while (m < -1000) {
    x = mul(x, 0x1p-1000);
    m += 1000;
  }
  return mul(x, from_bits((int64_t)(m + 1023) << 52));
}

// Round hi + lo (|lo| small) times 2^m onto the subnormal grid (multiples of
// 2^-1074) with one rounding; hi * 2^(m + 1074) must be below 2^52.
CRM_FN double round_subnormal(double hi, double lo, int m) {
  const int e = m + 1074;
  const double a = scale2(hi, e), b = scale2(lo, e);  // exact: both stay normal or zero
  double n = rint_(a);
  const double f = add(sub(a, n), b);                  // the remainder, |f| < 0.5 + tiny
  if (f > 0.5) n = add(n, 1.0);
  if (f < -0.5) n = sub(n, 1.0);
  return mul(n, 0x1p-1074);                            // exact
}

// The double nearest to h + a.hi + a.lo + b, where fl(h + a.hi) is within an
// ulp of the sum (|a.lo| and |b| far below its ulp).  The residual left by
// the candidate fl(h + a.hi) is carried exactly as a double-double and
// compared with the half-gaps to the neighbouring doubles, so that values
// within a few ulps of 2^-106 of a midpoint still round the right way.
CRM_FN double round_sum(double h, DD a, double b) {
  const DD z = two_sum(h, a.hi);  // z.hi: candidate; z.lo: exact residual
  DD w = two_sum(z.lo, a.lo);
  w.lo = add(w.lo, b);
  w = two_sum(w.hi, w.lo);
  const double c = z.hi;
  if (c == 0.0) return add(w.hi, w.lo);
  const int64_t bc = bits(c);
  // neighbours towards +inf and -inf
  const double up = from_bits(c > 0.0 ? bc + 1 : bc - 1), dn = from_bits(c > 0.0 ? bc - 1 : bc + 1);
  const double gup = mul(sub(up, c), 0.5), gdn = mul(sub(c, dn), 0.5);  // exact
  if (w.hi > gup || (w.hi == gup && w.lo > 0.0)) return up;
  if (w.hi < -gdn || (w.hi == -gdn && w.lo < 0.0)) return dn;
  if (w.lo == 0.0 && (w.hi == gup || w.hi == -gdn)) {  // an exact tie: the even neighbour
    if (bc & 1) return w.hi > 0.0 ? up : dn;
  }
  return c;
}

// x^2/2 exactly, x^3/6 to double-double, for the series of tiny arguments
CRM_FN DD half_square(double x) {
  const DD q = two_prod(x, x);
  return {mul(q.hi, 0.5), mul(q.lo, 0.5)};
}
CRM_FN DD cube_over(double x, DD third) {
  const DD q = two_prod(x, x);
  DD c = two_prod(x, q.hi);
  c.lo = fma_(x, q.lo, c.lo);
  c = two_sum(c.hi, c.lo);
  return dd_mul(c, third);
}
constexpr double kTiny = 0x1p-30;  // below: the explicit series

// e^x in double-double from the reduction (error about 2^-100 relative)
CRM_FN DD exp_dd_reduced(int k, double rh, double rl) {
  return table_times(k & 63, expm1_small_dd(rh, rl));
}

// e^x when the fast evaluation cannot decide the rounding, and for
// subnormal results.  Inline (a call in a kernel's straight-line code costs
// more than this rarely taken code).
CRM_FN double exp_accurate(double x, int k, double rh, double rl) {
  const int j = k & 63, m = k >> 6;
  const double ax = x < 0.0 ? -x : x;
  if (ax < kTiny) {  // 1 + x + x^2/2 + x^3/6 + x^4/24
    const DD h2 = half_square(x);
    const DD h3 = cube_over(x, DD{0x1.5555555555555p-3, 0x1.5555555555555p-57});
    const DD z = two_sum(1.0, x);
    return round_sum(z.hi, DD{z.lo, h2.hi},
                     add(h2.lo, add(h3.hi, add(h3.lo, mul(mul(h2.hi, h2.hi), 0x1.5555555555555p-3)))));
  }
  // 2^(j/64) (1 + s) with s = e^r - 1 in double-double
  const double* T = exp2_table();
  const double Th = T[2 * j], Tl = T[2 * j + 1];
  const DD sd = expm1_small_dd(rh, rl);
  const DD pp = two_prod(Th, sd.hi);
  const double rest = add(mul(Th, sd.lo), fma_(Tl, sd.hi, Tl));
  if (x < kExpSub) {
    const DD z = two_sum(Th, pp.hi);
    return round_subnormal(z.hi, add(z.lo, add(pp.lo, rest)), m);
  }
  return scale2(round_sum(Th, pp, rest), m);
}

// Accept y.hi + y.lo (|y.lo| <= ulp/2, within e of the exact value) when
// every value within e of it rounds to y.hi.
CRM_FN bool decided(DD y, double e) {
  const int64_t b = bits(y.hi);
  const double up = from_bits(b + 1), dn = from_bits(b - 1);
  const double gap_up = mul(sub(up, y.hi), 0.5), gap_dn = mul(sub(y.hi, dn), 0.5);  // exact
  return add(y.lo, e) < gap_up && sub(y.lo, e) > -gap_dn;
}

// The fast evaluation of e^x.  Returns false when it cannot decide the
// rounding (then exp_full decides); special values are decided here.
CRM_FN bool exp_fast(double x, double& y) {
  if (!(x == x)) { y = add(x, x); return true; }  // NaN
  if (x > kExpMax) { y = from_bits(0x7ff0000000000000LL); return true; }
  if (x < kExpMin) { y = 0.0; return true; }
  const double ax = x < 0.0 ? -x : x;
  if (ax <= 0.0054) {
    // |x| <= ln2/128 (k = 0): e^x = 1 + x + c with |error of c| < 2^-67
    double p = 0x1.a01a01a01a01ap-13;
    p = fma_(p, x, 0x1.6c16c16c16c17p-10);
    p = fma_(p, x, 0x1.1111111111111p-7);
    p = fma_(p, x, 0x1.5555555555555p-5);
    p = fma_(p, x, 0x1.5555555555555p-3);
    p = fma_(p, x, 0.5);
    const double c = mul(mul(x, x), p);
    const DD s = two_sum(x, c);
    DD z = two_sum(1.0, s.hi);
    z.lo = add(z.lo, s.lo);
    z = two_sum(z.hi, z.lo);
    y = z.hi;
    return decided(z, 0x1p-63);
  }
  if (x < kExpSub) return false;
  double rh, rl;
  const int k = reduce(x, rh, rl);
  const int j = k & 63, m = k >> 6;  // arithmetic shift: floor(k / 64)
  // e^r - 1 = rh + c, |error of c| < 2^-67 (|rh| <= 0.0055)
  double p = 0x1.a01a01a01a01ap-13;            // 1/7!
  p = fma_(p, rh, 0x1.6c16c16c16c17p-10);      // 1/6!
  p = fma_(p, rh, 0x1.1111111111111p-7);       // 1/5!
  p = fma_(p, rh, 0x1.5555555555555p-5);       // 1/4!
  p = fma_(p, rh, 0x1.5555555555555p-3);       // 1/3!
  p = fma_(p, rh, 0.5);
  const double c = add(mul(mul(rh, rh), p), fma_(rl, rh, rl));
  const DD s = two_sum(rh, c);
  const double* T = exp2_table();
  const double Th = T[2 * j], Tl = T[2 * j + 1];
  const DD ps = two_prod(Th, s.hi);
  DD z = two_sum(Th, ps.hi);
  z.lo = add(z.lo, add(ps.lo, add(mul(Th, s.lo), fma_(Tl, s.hi, Tl))));
  z = two_sum(z.hi, z.lo);
  // z is within 2^-64 (absolute; z < 2.02) of 2^(j/64) e^r
  y = scale2(z.hi, m);
  return decided(z, 0x1p-63);
}

// The accurate phase of e^x for any finite x in [kExpMin, kExpMax].
CRM_FN double exp_full(double x) {
  const double ax = x < 0.0 ? -x : x;
  if (ax <= 0.0054) return exp_accurate(x, 0, x, 0.0);
  double rh, rl;
  const int k = reduce(x, rh, rl);
  return exp_accurate(x, k, rh, rl);
}

// Correctly rounded e^x.
CRM_FN double exp(double x) {
  double y;
  if (exp_fast(x, y)) return y;
  return exp_full(x);
}

// Correctly rounded e^x of N arguments: the fast evaluation of each inline,
// the accurate phase (needed for about 0.15 % of arguments) in one rolled
// loop for all N, so that a kernel carries one copy of its code per batch.
template <int N>
CRM_FN void exp_n(const double (&x)[N], double (&y)[N]) {
  unsigned bad = 0;
#pragma unroll
  for (int n = 0; n < N; ++n)
    if (!exp_fast(x[n], y[n])) bad |= 1u << n;
  // one argument at a time, picked and stored by compare-and-select, so that
  // neither a call nor an indexed (local-memory) array enters the kernel
#pragma unroll 1
  while (bad) {
#if defined(__CUDA_ARCH__)
    const int q = __ffs(bad) - 1;
#else
    const int q = __builtin_ctz(bad);
#endif
    bad &= bad - 1u;
    double v = x[0];
#pragma unroll
    for (int n = 1; n < N; ++n) v = q == n ? x[n] : v;
    v = exp_full(v);
#pragma unroll
    for (int n = 0; n < N; ++n) y[n] = q == n ? v : y[n];
  }
}

// e^x - 1 in double-double with the same reduction (error about 2^-100
// relative to the result; 2^-92 for |x| > ln2/128, where the result exceeds
// 0.0054 in magnitude)
CRM_FN DD expm1_dd(double x) {
  double rh, rl;
  const int k = reduce(x, rh, rl);
  if (k == 0) return expm1_small_dd(rh, rl);
  DD y = exp_dd_reduced(k, rh, rl);
  const int m = k >> 6;
  y.hi = scale2(y.hi, m);
  y.lo = scale2(y.lo, m);
  return dd_add(y, DD{-1.0, 0.0});
}

// Correctly rounded e^x - 1.
CRM_FN double expm1(double x) {
  if (!(x == x)) return add(x, x);
  if (x > 709.78) return exp(x);  // e^x - 1 and e^x round alike (they differ by 2^-1022 relative)
  if (x < -40.0) return -1.0;     // e^x < 2^-57: -1 + e^x rounds to -1
  const double ax = x < 0.0 ? -x : x;
  if (ax < 0x1p-54) return x;  // x + x^2/2 rounds to x
  if (ax < kTiny) {            // x + x^2/2 + x^3/6 + x^4/24
    const DD h2 = half_square(x);
    const DD h3 = cube_over(x, DD{0x1.5555555555555p-3, 0x1.5555555555555p-57});
    return round_sum(x, h2, add(h3.hi, add(h3.lo, mul(mul(h2.hi, h2.hi), 0x1.5555555555555p-3))));
  }
  const DD z = expm1_dd(x);
  return round_sum(z.hi, DD{z.lo, 0.0}, 0.0);
}

// Correctly rounded log(1 + y): one Newton step z = z0 + log1p(t) from a
// start value z0 within a few ulp, with t = (1 + y) e^{-z0} - 1 formed in
// double-double (as y + q + y q, q = expm1(-z0), where the result is small,
// so that the error stays relative to the result).
CRM_FN double log1p(double y) {
  if (!(y == y)) return add(y, y);
  if (y < -1.0) return from_bits(0x7ff8000000000000LL);
  if (y == -1.0) return from_bits((int64_t)0xfff0000000000000ULL);
  if (y == from_bits(0x7ff0000000000000LL)) return y;
  const double ay = y < 0.0 ? -y : y;
  if (ay < 0x1p-54) return y;  // y - y^2/2 rounds to y
  if (ay < kTiny) {            // y - y^2/2 + y^3/3 - y^4/4
    const DD h2 = half_square(y);
    const DD h3 = cube_over(y, DD{0x1.5555555555555p-2, 0x1.5555555555555p-56});
    return round_sum(y, DD{-h2.hi, -h2.lo}, sub(add(h3.hi, h3.lo), mul(h2.hi, h2.hi)));
  }
  const double z0 = ::log1p(y);
  DD t;
  const double az = z0 < 0.0 ? -z0 : z0;
  if (az <= 0.0054) {
    const DD q = expm1_dd(-z0);
    t = dd_add(dd_add(DD{y, 0.0}, q), dd_mul_d(q, y));
  } else {
    // e^{-z0} = 2^m w with w in [0.99, 2.02]: scale 1 + y by 2^m instead of
    // w, so that nothing leaves the normal range
    double rh, rl;
    const int k = reduce(-z0, rh, rl);
    const DD w = exp_dd_reduced(k, rh, rl);
    const int m = k >> 6;
    DD u = two_sum(1.0, y);
    u.hi = scale2(u.hi, m);
    u.lo = scale2(u.lo, m);
    t = dd_add(dd_mul(u, w), DD{-1.0, 0.0});
  }
  // log1p(t) = t - t^2/2 + ..., |t| ~ ulp(z0): t^2 is far below the result's ulp
  return round_sum(z0, t, -mul(mul(t.hi, t.hi), 0.5));
}

}  // namespace crm
}  // namespace cg
