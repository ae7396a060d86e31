// cg_ics.cu -- BSSN + dust initial data on the GPU: the synchronous-gauge
// construction of the reference's dust_ic_set_random
// (components/dust_fluid/dust_ic.cc:23-140) from a Gaussian random density
// field, with spectral inverse Laplacians (utils/Fourier.h:251-298) on cuFFT
// and the reference's finite-difference stencils (utils/math.h:74-1085).
//
// Same steps, in the same order, as cosmograph_b200/ics.py (grf_dust), which
// is the host version:
//   delta      seeded Gaussian random field, P(k) ~ k^ns exp(-(k/kc)^2),
//              zero mean, rms normalised (or a caller-supplied field)
//   Phi_N      = invlap(3/2 delta)                     (lap Phi_N = 4 pi rho delta)
//   DIFFphi    = log1p(-10/3 Phi_N) / 4                (dust_ic.cc:70)
//   DIFFK      = -3 (1 + 2 Phi_N) + 2/3 lap Phi_N      (dust_ic.cc:71)
//   W_a        = -d_a Phi_N / 3 + invlap(e^{6 phi} d_a DIFFK) / 2   (:76-95)
//   A_ij       = e^{-6 phi} (d_i W_j + d_j W_i + 2/3 d_i d_j Phi_N
//                - delta_ij (2/3 d_k W_k + 2/9 lap Phi_N))          (:98-114)
//   rho_ADM    = (K^2/12 - A_ij A^ij / 8 - e^{-5 phi} lap e^phi) / (2 pi)
//   D          = e^{6 phi} (rho_ADM - rho_Lambda)                  (:135)
// The random field of this file uses its own counter-based generator; given
// the same delta the result matches the host construction to rounding.
//
// Scalar-field initial data (grf_scalar, the host version ics.grf_scalar):
//   dphi       seeded Gaussian random field, P(k) ~ k^-3 for k <= kc, else 0,
//              zero mean, rms normalised (or a caller-supplied field)
//   phi        = phi0 + dphi, Pi = 0, psi_a = d_a phi (the relation of the
//              reference's wave data, components/scalar/scalar_ic.cc:43-48)
//   DIFFK      = -sqrt(24 pi rho), rho = m^2 phi^2 / 2 + |d phi|^2 / 2
#include <cufft.h>

#include <cmath>
#include <string>

#include "cg_internal.h"
#include "cosmograph_b200.h"

namespace cg {
namespace ics {

namespace {

constexpr int kT = 256;
constexpr double kPiD = 3.141592653589793238462643383279502884;

__host__ __device__ inline int freq(int i, int n) { return i < (n + 1) / 2 ? i : i - n; }  // numpy fftfreq * n

// splitmix64 finaliser: a 64-bit hash of (seed, counter)
__device__ inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
__device__ inline double u01(uint64_t x) { return ((double)(x >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

// complex Gaussian noise times sqrt(P(k)) on the half spectrum (nx, ny, nz/2+1);
// P(k) = k^ns exp(-(k/kc)^2) (sharp = 0) or k^ns for k <= kc, else 0 (sharp = 1)
__global__ void noise_kernel(cufftDoubleComplex* out, int nx, int ny, int nz, uint64_t seed, double ns, double kc,
                             int sharp) {
  const int nzh = nz / 2 + 1;
  const long long total = (long long)nx * ny * nzh;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q % nzh), j = (int)((q / nzh) % ny), i = (int)(q / ((long long)nzh * ny));
    const double px = freq(i, nx), py = freq(j, ny), pz = k;
    const double kk = sqrt(px * px + py * py + pz * pz);
    const double pk = sharp ? (kk <= kc ? pow(kk, ns) : 0.0) : pow(kk, ns) * exp(-(kk / kc) * (kk / kc));
    const double amp = kk > 0.0 ? sqrt(pk) : 0.0;
    const uint64_t base = mix64(seed ^ 0x9e3779b97f4a7c15ULL);
    const double u1 = u01(mix64(base + 2 * (uint64_t)q)), u2 = u01(mix64(base + 2 * (uint64_t)q + 1));
    const double r = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    out[q].x = amp * r * c;
    out[q].y = amp * r * s;
  }
}

// spectral inverse Laplacian: multiply by -1/p^2 (zero mode removed) and by
// 1/N (cuFFT's inverse is unnormalised)
__global__ void invlap_kernel(cufftDoubleComplex* f, int nx, int ny, int nz, double two_pi_over_L) {
  const int nzh = nz / 2 + 1;
  const long long total = (long long)nx * ny * nzh;
  const double inv_n = 1.0 / ((double)nx * ny * nz);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total; q += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(q % nzh), j = (int)((q / nzh) % ny), i = (int)(q / ((long long)nzh * ny));
    const double px = freq(i, nx), py = freq(j, ny), pz = k;
    const double p2 = (px * px + py * py + pz * pz) * (two_pi_over_L * two_pi_over_L);
    if (q == 0) {
      f[q].x = 0.0;
      f[q].y = 0.0;
    } else {
      f[q].x = f[q].x / (-p2) * inv_n;
      f[q].y = f[q].y / (-p2) * inv_n;
    }
  }
}

// block partial sums of f (pass 0) or of (f - mean)^2 (pass 1), fixed order
__global__ void moment_kernel(const double* f, long long n, const double* mean, double* part) {
  __shared__ double s[kT];
  double a = 0.0;
  const double m = mean ? *mean : 0.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const double v = mean ? (f[q] - m) * (f[q] - m) : f[q];
    a += v;
  }
  s[threadIdx.x] = a;
  __syncthreads();
  for (int o = kT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}
__global__ void sum_parts_kernel(const double* part, int nblk, long long n, double* out) {
  __shared__ double s[kT];
  double a = 0.0;
  for (int b = threadIdx.x; b < nblk; b += kT) a += part[b];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int o = kT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0] / (double)n;
}
// delta = (f - mean) * rms / std
__global__ void normalise_kernel(double* f, long long n, const double* mean, const double* var, double rms) {
  const double m = *mean, sd = sqrt(*var);
  const double sc = sd > 0.0 ? rms / sd : 1.0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    f[q] = (f[q] - m) * sc;
}

struct Grid {
  int nx, ny, nz, order;
  double idx;  // 1 / dx
};

__device__ inline double at(const double* f, const Grid& g, int i, int j, int k) {
  i = i < 0 ? i + g.nx : (i >= g.nx ? i - g.nx : i);
  j = j < 0 ? j + g.ny : (j >= g.ny ? j - g.ny : j);
  k = k < 0 ? k + g.nz : (k >= g.nz ? k - g.nz : k);
  return f[((long long)i * g.ny + j) * g.nz + k];
}

// first derivative along a (the expressions of cosmograph_b200/ics.py)
__device__ double d1(const double* f, const Grid& g, int i, int j, int k, int a) {
  auto V = [&](int n) { return at(f, g, i + (a == 0) * n, j + (a == 1) * n, k + (a == 2) * n); };
  double s;
  switch (g.order) {
    case 2: s = (-1.0 / 2.0 * V(-1) + 1.0 / 2.0 * V(1)); break;
    case 4: s = (+1.0 / 12.0 * V(-2) - 2.0 / 3.0 * V(-1) + 2.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2)); break;
    case 6:
      s = (-1.0 / 60.0 * V(-3) + 3.0 / 20.0 * V(-2) - 3.0 / 4.0 * V(-1) + 3.0 / 4.0 * V(1) - 3.0 / 20.0 * V(2) +
           1.0 / 60.0 * V(3));
      break;
    default:
      s = ((1.0 / 280.0 * V(-4) - 1.0 / 280.0 * V(4)) - (4.0 / 105.0 * V(-3) - 4.0 / 105.0 * V(3)) +
           (1.0 / 5.0 * V(-2) - 1.0 / 5.0 * V(2)) - (4.0 / 5.0 * V(-1) - 4.0 / 5.0 * V(1)));
  }
  return s * g.idx;
}

// second derivative along a, b (diagonal-point stencils for a != b)
__device__ double d2(const double* f, const Grid& g, int i, int j, int k, int a, int b) {
  if (a == b) {
    auto V = [&](int n) { return at(f, g, i + (a == 0) * n, j + (a == 1) * n, k + (a == 2) * n); };
    double s;
    switch (g.order) {
      case 2: s = (V(-1) - 2.0 * V(0) + V(1)); break;
      case 4: s = (-1.0 / 12.0 * V(-2) + 4.0 / 3.0 * V(-1) - 5.0 / 2.0 * V(0) + 4.0 / 3.0 * V(1) - 1.0 / 12.0 * V(2)); break;
      case 6:
        s = (1.0 / 90.0 * V(-3) - 3.0 / 20.0 * V(-2) + 3.0 / 2.0 * V(-1) - 49.0 / 18.0 * V(0) + 3.0 / 2.0 * V(1) -
             3.0 / 20.0 * V(2) + 1.0 / 90.0 * V(3));
        break;
      default:
        s = (-1.0 / 560.0 * V(-4) + 8.0 / 315.0 * V(-3) - 1.0 / 5.0 * V(-2) + 8.0 / 5.0 * V(-1) - 205.0 / 72.0 * V(0) +
             8.0 / 5.0 * V(1) - 1.0 / 5.0 * V(2) + 8.0 / 315.0 * V(3) - 1.0 / 560.0 * V(4));
    }
    return s * g.idx * g.idx;
  }
  auto S = [&](int p, int q) {
    return at(f, g, i + (a == 0) * p + (b == 0) * q, j + (a == 1) * p + (b == 1) * q, k + (a == 2) * p + (b == 2) * q);
  };
  auto P = [&](int n) { return -S(n, -n) + S(n, n) + S(-n, -n) - S(-n, n); };
  double s;
  switch (g.order) {
    case 2: s = P(1) / 4.0; break;
    case 4: s = (P(1) - 1.0 / 16.0 * P(2)) / 3.0; break;
    case 6: s = (135.0 * P(1) - 27.0 / 2.0 * P(2) + P(3)) / 360.0; break;
    default: s = (2.0 / 5.0 * P(1) - 1.0 / 20.0 * P(2) + 2.0 / 315.0 * P(3) - 1.0 / 2240.0 * P(4));
  }
  return s * g.idx * g.idx;
}

__device__ inline double lap(const double* f, const Grid& g, int i, int j, int k) {
  return d2(f, g, i, j, k, 0, 0) + d2(f, g, i, j, k, 1, 1) + d2(f, g, i, j, k, 2, 2);
}

#define CG_IC_LOOP(g)                                                                                 \
  const long long n_ = (long long)(g).nx * (g).ny * (g).nz;                                           \
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n_;                        \
       q += (long long)gridDim.x * blockDim.x)

// Phi_N input: 3/2 delta
__global__ void scale_kernel(double* out, const double* in, long long n, double s) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    out[q] = s * in[q];
}

// lap Phi_N, DIFFphi, DIFFK
__global__ void phi_k_kernel(Grid g, const double* phiN, double* lapPhi, double* dphi, double* dK) {
  CG_IC_LOOP(g) {
    const int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.nz * g.ny));
    const double L = lap(phiN, g, i, j, k);
    lapPhi[q] = L;
    dphi[q] = log1p(-10.0 / 3.0 * phiN[q]) / 4.0;
    dK[q] = -3.0 * (1.0 + 2.0 * phiN[q]) + 2.0 / 3.0 * L;
  }
}

// e^{6 phi} d_a DIFFK
__global__ void src_w_kernel(Grid g, const double* dphi, const double* dK, int a, double* out) {
  CG_IC_LOOP(g) {
    const int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.nz * g.ny));
    out[q] = exp(6.0 * dphi[q]) * d1(dK, g, i, j, k, a);
  }
}

// W_a = -d_a Phi_N / 3 + inv / 2 (inv = invlap(e^{6 phi} d_a DIFFK))
__global__ void w_kernel(Grid g, const double* phiN, const double* inv, int a, double* W) {
  CG_IC_LOOP(g) {
    const int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.nz * g.ny));
    W[q] = -d1(phiN, g, i, j, k, a) / 3.0 + inv[q] / 2.0;
  }
}

// A_ij, rho_ADM and D; every other field zero.  fields: the _p block.
__global__ void assemble_kernel(Grid g, const double* phiN, const double* lapPhi, const double* dphi,
                                const double* dK, const double* W0, const double* W1, const double* W2,
                                double rho_L, double* P, unsigned* negative) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  CG_IC_LOOP(g) {
    const int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.nz * g.ny));
    const double* W[3] = {W0, W1, W2};
    const double c = exp(-6.0 * dphi[q]);
    const double DkWk = d1(W0, g, i, j, k, 0) + d1(W1, g, i, j, k, 1) + d1(W2, g, i, j, k, 2);
    double A[6];
    for (int I = 0; I < 3; ++I)
      for (int J = I; J < 3; ++J) {
        double v = d1(W[J], g, i, j, k, I) + d1(W[I], g, i, j, k, J) + 2.0 / 3.0 * d2(phiN, g, i, j, k, I, J);
        if (I == J) v = v - 2.0 / 3.0 * DkWk - 2.0 / 9.0 * lapPhi[q];
        A[sym(I, J)] = c * v;
      }
    const double AA = A[0] * A[0] + A[3] * A[3] + A[5] * A[5] + 2.0 * (A[1] * A[1] + A[2] * A[2] + A[4] * A[4]);
    const double gp0 = d1(dphi, g, i, j, k, 0), gp1 = d1(dphi, g, i, j, k, 1), gp2 = d1(dphi, g, i, j, k, 2);
    const double lap_e_p = exp(dphi[q]) * (lap(dphi, g, i, j, k) + (gp0 * gp0 + gp1 * gp1 + gp2 * gp2));
    const double rho_adm =
        1.0 / 2.0 / kPiD * (dK[q] * dK[q] / 12.0 - AA / 8.0 - exp(-5.0 * dphi[q]) * lap_e_p);
    const double rho0 = rho_adm - rho_L;
    if (!(rho0 >= 0.0)) atomicOr(negative, 1u);  // negative or NaN (log1p of a large potential)
    for (int f = 0; f < 22; ++f) {
      double v = 0.0;
      if (f == F_PHI) v = dphi[q];
      else if (f == F_K) v = dK[q];
      else if (f >= F_A11 && f < F_A11 + 6) v = A[f - F_A11];
      else if (f == F_D) v = exp(6.0 * dphi[q]) * rho0;
      P[(long long)f * N + q] = v;
    }
  }
}

// phi0 + dphi
__global__ void offset_kernel(double* out, const double* in, long long n, double phi0) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    out[q] = phi0 + in[q];
}

// scalar fields, psi_a, DIFFK; every other field zero (23 fields)
__global__ void assemble_scalar_kernel(Grid g, const double* phi, double mass, double* P) {
  const long long N = (long long)g.nx * g.ny * g.nz;
  CG_IC_LOOP(g) {
    const int k = (int)(q % g.nz), j = (int)((q / g.nz) % g.ny), i = (int)(q / ((long long)g.nz * g.ny));
    double d[3], grad2 = 0.0;
    for (int a = 0; a < 3; ++a) {
      d[a] = d1(phi, g, i, j, k, a);
      grad2 = grad2 + d[a] * d[a];
    }
    const double rho = 0.5 * mass * mass * phi[q] * phi[q] + 0.5 * grad2;
    for (int f = 0; f < 23; ++f) {
      double v = 0.0;
      if (f == F_K) v = -sqrt(24.0 * kPiD * rho);
      else if (f == F_SPHI) v = phi[q];
      else if (f >= F_SPSI1 && f < F_SPSI1 + 3) v = d[f - F_SPSI1];
      P[(long long)f * N + q] = v;
    }
  }
}

int blocks_for(long long n) {
  const long long b = (n + kT - 1) / kT;
  return (int)(b < 4096 ? b : 4096);
}

}  // namespace

size_t grf_scratch_doubles(const GridSpec& s) {
  const size_t N = (size_t)s.nx * s.ny * s.nz;
  return 9 * N + 2 * (size_t)s.nx * s.ny * (s.nz / 2 + 1) + 4098 + 1;
}

// Host driver; scratch (grf_scratch_doubles(s) doubles) is caller-owned
// device memory.  delta_host: optional host copy of the density contrast.
int grf_dust(const GridSpec& s, double* P, double* scratch, const double* delta_host, uint64_t seed, double rms,
             double ns, double kc, double rho_L, cudaStream_t st, std::string& err) {
  const long long N = (long long)s.nx * s.ny * s.nz;
  double* delta = scratch;
  double* phiN = scratch + N;
  double* lapPhi = scratch + 2 * N;
  double* dphi = scratch + 3 * N;
  double* dK = scratch + 4 * N;
  double* W0 = scratch + 5 * N;
  double* W1 = scratch + 6 * N;
  double* W2 = scratch + 7 * N;
  double* tmp = scratch + 8 * N;
  auto* spec = reinterpret_cast<cufftDoubleComplex*>(scratch + 9 * N);  // nx*ny*(nz/2+1) complex
  double* red = scratch + 9 * N + 2 * (long long)s.nx * s.ny * (s.nz / 2 + 1);  // 4096 partials + 2 results
  unsigned* flag = reinterpret_cast<unsigned*>(red + 4098);
  const Grid g{s.nx, s.ny, s.nz, s.order, 1.0 / s.dx};
  const double two_pi_over_L = 2.0 * kPiD / (s.dx * s.nx);
  const int nb = blocks_for(N);
  cufftHandle fwd = 0, inv = 0;
  auto cu = [&](cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
  };
  auto ff = [&](cufftResult r, const char* what) {
    if (r == CUFFT_SUCCESS) return true;
    err = std::string(what) + ": cuFFT error " + std::to_string((int)r);
    return false;
  };
  bool ok = ff(cufftPlan3d(&fwd, s.nx, s.ny, s.nz, CUFFT_D2Z), "cufftPlan3d D2Z") &&
            ff(cufftPlan3d(&inv, s.nx, s.ny, s.nz, CUFFT_Z2D), "cufftPlan3d Z2D") &&
            ff(cufftSetStream(fwd, st), "cufftSetStream") && ff(cufftSetStream(inv, st), "cufftSetStream");
  auto invlap = [&](const double* in, double* out) {
    return ff(cufftExecD2Z(fwd, const_cast<double*>(in), spec), "cufftExecD2Z") &&
           cu((invlap_kernel<<<nb, kT, 0, st>>>(spec, s.nx, s.ny, s.nz, two_pi_over_L), cudaGetLastError()),
              "invlap_kernel") &&
           ff(cufftExecZ2D(inv, spec, out), "cufftExecZ2D");
  };
  if (ok) {
    if (delta_host) {
      ok = cu(cudaMemcpyAsync(delta, delta_host, sizeof(double) * N, cudaMemcpyHostToDevice, st), "upload delta");
    } else {
      noise_kernel<<<nb, kT, 0, st>>>(spec, s.nx, s.ny, s.nz, seed, ns, kc, 0);
      ok = cu(cudaGetLastError(), "noise_kernel") && ff(cufftExecZ2D(inv, spec, delta), "cufftExecZ2D");
      if (ok) {
        // zero mean, rms normalised (population standard deviation)
        moment_kernel<<<nb, kT, 0, st>>>(delta, N, nullptr, red);
        sum_parts_kernel<<<1, kT, 0, st>>>(red, nb, N, red + 4096);
        moment_kernel<<<nb, kT, 0, st>>>(delta, N, red + 4096, red);
        sum_parts_kernel<<<1, kT, 0, st>>>(red, nb, N, red + 4097);
        normalise_kernel<<<nb, kT, 0, st>>>(delta, N, red + 4096, red + 4097, rms);
        ok = cu(cudaGetLastError(), "normalise");
      }
    }
  }
  if (ok) {
    scale_kernel<<<nb, kT, 0, st>>>(tmp, delta, N, 1.5);
    ok = cu(cudaGetLastError(), "scale_kernel") && invlap(tmp, phiN);
  }
  if (ok) {
    phi_k_kernel<<<nb, kT, 0, st>>>(g, phiN, lapPhi, dphi, dK);
    ok = cu(cudaGetLastError(), "phi_k_kernel");
  }
  double* W[3] = {W0, W1, W2};
  for (int a = 0; a < 3 && ok; ++a) {
    src_w_kernel<<<nb, kT, 0, st>>>(g, dphi, dK, a, tmp);
    ok = cu(cudaGetLastError(), "src_w_kernel") && invlap(tmp, tmp);
    if (ok) {
      w_kernel<<<nb, kT, 0, st>>>(g, phiN, tmp, a, W[a]);
      ok = cu(cudaGetLastError(), "w_kernel");
    }
  }
  if (ok) {
    ok = cu(cudaMemsetAsync(flag, 0, sizeof(unsigned), st), "cudaMemsetAsync");
    if (ok) {
      assemble_kernel<<<nb, kT, 0, st>>>(g, phiN, lapPhi, dphi, dK, W0, W1, W2, rho_L, P, flag);
      ok = cu(cudaGetLastError(), "assemble_kernel");
    }
  }
  unsigned neg = 0;
  if (ok) ok = cu(cudaMemcpyAsync(&neg, flag, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "flag") &&
               cu(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  if (fwd) cufftDestroy(fwd);
  if (inv) cufftDestroy(inv);
  if (!ok) return CG_ERR_CUDA;
  if (neg) {
    err = "negative density in some regions (lower rms_delta)";
    return CG_ERR_INVALID;
  }
  return CG_OK;
}

// Scalar-field initial data; scratch as for grf_dust.  dphi_host: optional
// host copy of the fluctuation.
int grf_scalar(const GridSpec& s, double* P, double* scratch, const double* dphi_host, uint64_t seed, double rms,
               double phi0, double mass, double kc, cudaStream_t st, std::string& err) {
  const long long N = (long long)s.nx * s.ny * s.nz;
  double* dphi = scratch;
  double* phi = scratch + N;
  auto* spec = reinterpret_cast<cufftDoubleComplex*>(scratch + 9 * N);
  double* red = scratch + 9 * N + 2 * (long long)s.nx * s.ny * (s.nz / 2 + 1);
  const Grid g{s.nx, s.ny, s.nz, s.order, 1.0 / s.dx};
  const int nb = blocks_for(N);
  cufftHandle inv = 0;
  auto cu = [&](cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
  };
  bool ok = true;
  if (dphi_host) {
    ok = cu(cudaMemcpyAsync(dphi, dphi_host, sizeof(double) * N, cudaMemcpyHostToDevice, st), "upload dphi");
  } else {
    cufftResult r = cufftPlan3d(&inv, s.nx, s.ny, s.nz, CUFFT_Z2D);
    if (r == CUFFT_SUCCESS) r = cufftSetStream(inv, st);
    if (r == CUFFT_SUCCESS) {
      noise_kernel<<<nb, kT, 0, st>>>(spec, s.nx, s.ny, s.nz, seed, -3.0, kc, 1);
      ok = cu(cudaGetLastError(), "noise_kernel");
      if (ok) r = cufftExecZ2D(inv, spec, dphi);
    }
    if (r != CUFFT_SUCCESS) {
      err = "cuFFT error " + std::to_string((int)r);
      ok = false;
    }
    if (ok) {
      // zero mean, rms normalised (population standard deviation)
      moment_kernel<<<nb, kT, 0, st>>>(dphi, N, nullptr, red);
      sum_parts_kernel<<<1, kT, 0, st>>>(red, nb, N, red + 4096);
      moment_kernel<<<nb, kT, 0, st>>>(dphi, N, red + 4096, red);
      sum_parts_kernel<<<1, kT, 0, st>>>(red, nb, N, red + 4097);
      normalise_kernel<<<nb, kT, 0, st>>>(dphi, N, red + 4096, red + 4097, rms);
      ok = cu(cudaGetLastError(), "normalise");
    }
  }
  if (ok) {
    offset_kernel<<<nb, kT, 0, st>>>(phi, dphi, N, phi0);
    assemble_scalar_kernel<<<nb, kT, 0, st>>>(g, phi, mass, P);
    ok = cu(cudaGetLastError(), "assemble_scalar_kernel") && cu(cudaStreamSynchronize(st), "cudaStreamSynchronize");
  }
  if (inv) cufftDestroy(inv);
  return ok ? CG_OK : CG_ERR_CUDA;
}

}  // namespace ics
}  // namespace cg
