// cg_abi.cu -- the C ABI (include/cosmograph_b200.h): contexts, device
// storage, the host-side FRW background and the substep sequencing.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

#include "cosmograph_b200.h"
#include "cg_internal.h"
#include "cg_mixed.cuh"

namespace {

using cg::BoxDev;
using cg::StageBg;

thread_local std::string g_create_error;

// FRW reference integrator (utils/FRW.h:94-254), FP64 on the host.  The
// substep kernels only need its getter values, which are grid-independent.
struct FrwHost {
  double phi = 0.0, K = 0.0;
  int n = 0;
  double rho[4] = {0, 0, 0, 0}, w[4] = {0, 0, 0, 0};
  double phi_K[4] = {0, 0, 0, 0}, K_K[4] = {0, 0, 0, 0}, fl_K[4][4] = {};
  double get_phi = 0.0, get_K = 0.0, get_rho = 0.0, get_S = 0.0;

  void set_gets(double p, double k, const double* r) {
    get_phi = p;
    get_K = k;
    get_rho = 0.0;
    get_S = 0.0;
    for (int m = 0; m < n; ++m) {
      get_rho += r[m];
      get_S += 3.0 * r[m] * w[m];
    }
  }
  // stage n = 1,2,3 : P{n}_step ; n = 4 : RK_total_step
  void stage(int s, double h) {
    static const long double kPiL = 3.141592653589793238462643383279502884L;
    double K_in = K, rho_in[4];
    if (s == 1) {
      for (int m = 0; m < n; ++m) rho_in[m] = rho[m];
    } else {
      const double c = s == 4 ? h : h / 2.0;
      K_in = K + c * K_K[s - 2];
      for (int m = 0; m < n; ++m) rho_in[m] = rho[m] + c * fl_K[s - 2][m];
    }
    phi_K[s - 1] = -1.0 * K_in / 6.0;
    double K_source = 0.0;
    for (int m = 0; m < n; ++m) K_source += 4.0 * kPiL * rho_in[m] * (1.0 + 3.0 * w[m]);
    K_K[s - 1] = 1.0 / 3.0 * K_in * K_in + K_source;
    for (int m = 0; m < n; ++m) fl_K[s - 1][m] = K_in * rho_in[m] * (1.0 + w[m]);
    if (s < 4) {
      const double c = s == 3 ? h : h / 2.0;
      double r[4];
      for (int m = 0; m < n; ++m) r[m] = rho[m] + c * fl_K[s - 1][m];
      set_gets(phi + c * phi_K[s - 1], K + c * K_K[s - 1], r);
    } else {
      phi += h / 6.0 * (phi_K[0] + 2.0 * phi_K[1] + 2.0 * phi_K[2] + phi_K[3]);
      K += h / 6.0 * (K_K[0] + 2.0 * K_K[1] + 2.0 * K_K[2] + K_K[3]);
      for (int m = 0; m < n; ++m) rho[m] += h / 6.0 * (fl_K[0][m] + 2.0 * fl_K[1][m] + 2.0 * fl_K[2][m] + fl_K[3][m]);
      set_gets(phi, K, rho);
    }
  }
};

struct Box {
  cg_box_desc desc{};
  BoxDev dev{};
  FrwHost frw;
  int variant = cg::kExact;
  int stage_next = 0;   // 0: inputs not built; 1..4: next substep
  double phi_prev = 0.0;
  int64_t steps = 0;
  bool needs_kavg = false;
  double* kavg_partial = nullptr;  // per-block partial sums for K_avg
  double* kavg = nullptr;          // device K_avg
  double* kavg_sums = nullptr;     // device sums of exp(6 phi) K and exp(6 phi) (x-slabs: cg_kavg_sums)
  bool kavg_set = false;           // x-slab: the caller set K_avg for the next substep (cg_set_kavg)
  int kavg_blocks = 0;
  double* cscratch = nullptr;      // constraint statistics scratch (allocated on first use)
  // FP32-mixed boxes
  bool mixed = false;
  cg::MixedBox mdev{};
  double bp[23] = {}, bf[23] = {}, ba[23] = {}, bprev[23] = {};  // uniform background registers
  // staged state copies (cg_prefetch_state_async): device copies of the
  // next input and of the last result, the prefetched host buffer, and the
  // events that order the staging buffers' producers and consumers
  double* stage_in = nullptr;
  double* stage_out = nullptr;
  const double* pre_host = nullptr;
  size_t pre_count = 0;
  cudaEvent_t in_ready = nullptr, in_free = nullptr, out_ready = nullptr, out_free = nullptr;
  // FP32-mixed background means set by the caller (cg_set_background) for
  // the next initialisation instead of this box's own means (x-slabs of one box)
  bool bg_set = false;
  double bg_means[5] = {};
};

}  // namespace

namespace {
// Boxes of the same arithmetic, order and matter model advanced by one launch
// per substep (see stage_group_kernel / mixed_group_kernel).
struct Group {
  std::vector<int> members;  // box indices in launch order
  bool mixed = false;
  int variant = 0, order = 0, matter = 0;
  void* table = nullptr;     // device GroupBox table in launch order
  int total = 0;             // bricks of all members
  int grid = 0;              // CTAs of a launch (0: one per brick)
  int lpt = 0;               // launch order: 0 box index, 1 largest box first
  bool tuned = false;
};
}  // namespace

struct cg_ctx {
  std::vector<Box> boxes;
  std::vector<Group> groups;
  std::vector<int> singles;  // boxes launched on their own
  bool grouped = false;      // groups and singles are current
  int opt_batch = 1, opt_graph = 0, opt_autotune = 1, opt_group_grid = 0, opt_tma = 1;
  cudaGraphExec_t gexec = nullptr;
  int gexec_steps = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  // cg_exchange_state_async: the device-to-host stream and one event per field;
  // cg_prefetch_state_async: the host-to-device stream
  cudaStream_t copy_stream = nullptr;
  cudaStream_t up_stream = nullptr;
  cudaEvent_t copy_start = nullptr;
  std::vector<cudaEvent_t> copy_done;
  unsigned* status = nullptr;
  double* red = nullptr;   // reduction scratch for cg_conformal_average
  int red_blocks = 0;
  std::string err;
};

namespace {

int fail(cg_ctx* ctx, int code, const std::string& msg) {
  if (ctx)
    ctx->err = msg;
  else
    g_create_error = msg;
  return code;
}

int cuda_fail(cg_ctx* ctx, cudaError_t e, const char* what) {
  return fail(ctx, CG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CG_CUDA(ctx, call)                          \
  do {                                              \
    cudaError_t e_ = (call);                        \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

// cycles a CTA waits for a TMA tile copy before it flags CG_STATUS_TILE_TIMEOUT
// (about a second; CG_OPT_TMA_WAIT changes it)
constexpr long long kTmaWaitDefault = 2000000000LL;

bool lapse_needs_kavg(int lapse) {
  return lapse == CG_LAPSE_CONFORMAL_FLRW || lapse == CG_LAPSE_ANHARMONIC || lapse == CG_LAPSE_ONE_PLUS_LOG;
}

// Conformal (volume-weighted) average of DIFFK, math.h:1403-1415 as used by
// BSSN::setExtraFieldData (bssn.cc:168): per-block partial sums in a fixed
// order, then one block combines them in a fixed order.
__global__ void kavg_partial_kernel(const double* __restrict__ K, const double* __restrict__ phi, int pts,
                                    double phi_FRW, double* partial) {
  __shared__ double sK[256], sV[256];
  double aK = 0.0, aV = 0.0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < pts; q += (long long)gridDim.x * blockDim.x) {
    const double e = exp(6.0 * (phi[q] + phi_FRW));
    aK += e * K[q];
    aV += e;
  }
  sK[threadIdx.x] = aK;
  sV[threadIdx.x] = aV;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sK[threadIdx.x] += sK[threadIdx.x + o];
      sV[threadIdx.x] += sV[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sK[0];
    partial[2 * blockIdx.x + 1] = sV[0];
  }
}

__global__ void kavg_final_kernel(const double* partial, int nblk, int pts, double* out) {
  __shared__ double sK[256], sV[256];
  double aK = 0.0, aV = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    aK += partial[2 * b];
    aV += partial[2 * b + 1];
  }
  sK[threadIdx.x] = aK;
  sV[threadIdx.x] = aV;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sK[threadIdx.x] += sK[threadIdx.x + o];
      sV[threadIdx.x] += sV[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double vol = sV[0] / pts;
    out[0] = sK[0] / pts / vol;
  }
}

// Fixed-order reduction of per-CTA partial results: out[m] = sum (m < nsum)
// or max (m >= nsum) of part[b*Q + m] over b < nblk.  One CTA of 256 threads.
__global__ void part_final_kernel(const double* part, int nblk, int Q, int nsum, double* out) {
  __shared__ double s[256];
  for (int m = 0; m < Q; ++m) {
    const bool sum = m < nsum;
    double a = sum ? 0.0 : -1.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
      const double x = part[(size_t)b * Q + m];
      a = sum ? a + x : fmax(a, x);
    }
    s[threadIdx.x] = a;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) s[threadIdx.x] = sum ? s[threadIdx.x] + s[threadIdx.x + o] : fmax(s[threadIdx.x], s[threadIdx.x + o]);
      __syncthreads();
    }
    if (threadIdx.x == 0) out[m] = s[0];
    __syncthreads();
  }
}

// Sums of five fields (for the mixed form's uniform background): per CTA,
// fixed order.  f3, f4 may be null (sum 0).
__global__ void field_sums_kernel(const double* f0, const double* f1, const double* f2, const double* f3,
                                  const double* f4, int n, double* part) {
  __shared__ double s[5][256];
  double a[5] = {0, 0, 0, 0, 0};
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    a[0] += f0[q];
    a[1] += f1[q];
    a[2] += f2[q];
    a[3] += f3 ? f3[q] : 0.0;
    a[4] += f4 ? f4[q] : 0.0;
  }
  for (int m = 0; m < 5; ++m) s[m][threadIdx.x] = a[m];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int m = 0; m < 5; ++m) s[m][threadIdx.x] += s[m][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int m = 0; m < 5; ++m) part[(size_t)blockIdx.x * 5 + m] = s[m][0];
}

// Second pass of BSSN::setConstraintCalcs (bssn.cc:1026-1054): squared
// deviations from the means of pass 1 (r1: sums of value in [0,5), of scaled
// value in [10,15)), per CTA, 10 partial sums, over the n points from index
// off of arrays `stride` apart.
__global__ void constraint_stdev_kernel(const double* cvals, size_t stride, int off, int n, const double* r1,
                                        double* part) {
  __shared__ double s[10][256];
  double acc[10];
  double mean[10];
  for (int m = 0; m < 5; ++m) {
    mean[2 * m] = r1[m] / n;
    mean[2 * m + 1] = r1[10 + m] / n;
  }
  for (int m = 0; m < 10; ++m) acc[m] = 0.0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    for (int m = 0; m < 10; ++m) {
      const double d = cvals[(size_t)m * stride + off + q] - mean[m];
      acc[m] += d * d;
    }
  for (int m = 0; m < 10; ++m) s[m][threadIdx.x] = acc[m];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int m = 0; m < 10; ++m) s[m][threadIdx.x] += s[m][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int m = 0; m < 10; ++m) part[(size_t)blockIdx.x * 10 + m] = s[m][0];
}

// Volume-weighted statistics of io_bssn_dump_statistics (IO/io.cc:8-14):
// pass 1, per CTA, sum_q w f_m (m < 4) and sum_q w, w = exp(6 (phi + phi_FRW))
// (conformal_average / volume_average, utils/math.h:1382-1415).
__global__ void wstats_sum_kernel(const double* f0, const double* f1, const double* f2, const double* f3,
                                  const double* __restrict__ phi, int n, double phi_frw, double* part) {
  __shared__ double s[5][256];
  double a[5] = {0, 0, 0, 0, 0};
  const double* f[4] = {f0, f1, f2, f3};
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const double w = exp(6.0 * (phi[q] + phi_frw));
    for (int m = 0; m < 4; ++m) a[m] += w * f[m][q];
    a[4] += w;
  }
  for (int m = 0; m < 5; ++m) s[m][threadIdx.x] = a[m];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int m = 0; m < 5; ++m) s[m][threadIdx.x] += s[m][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int m = 0; m < 5; ++m) part[(size_t)blockIdx.x * 5 + m] = s[m][0];
}

// pass 2: sum_q w (avg_m - f_m)^2 with avg_m = sum w f_m / sum w from pass 1
// (conformal_standard_deviation, utils/math.h:1455-1470)
__global__ void wstats_var_kernel(const double* f0, const double* f1, const double* f2, const double* f3,
                                  const double* __restrict__ phi, int n, double phi_frw, const double* r1,
                                  double* part) {
  __shared__ double s[4][256];
  double a[4] = {0, 0, 0, 0}, avg[4];
  const double* f[4] = {f0, f1, f2, f3};
  const double vol = r1[4] / n;
  for (int m = 0; m < 4; ++m) avg[m] = r1[m] / n / vol;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
    const double w = exp(6.0 * (phi[q] + phi_frw));
    for (int m = 0; m < 4; ++m) {
      const double d = avg[m] - f[m][q];
      a[m] += w * (d * d);
    }
  }
  for (int m = 0; m < 4; ++m) s[m][threadIdx.x] = a[m];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int m = 0; m < 4; ++m) s[m][threadIdx.x] += s[m][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int m = 0; m < 4; ++m) part[(size_t)blockIdx.x * 4 + m] = s[m][0];
}

}  // namespace

namespace cg {
void set_global_error(const char* msg) { g_create_error = msg; }

// Conformal average of `field` weighted by exp(6 (phi + phi_FRW)) into
// out[0] on the device, using `partial` (2*nblk doubles) as scratch.
// The status is that of these two launches alone (cudaLaunchKernel returns
// the launch's own error), so an error left pending by an earlier, unrelated
// launch on the calling thread is neither reported nor cleared here.
cudaError_t launch_conformal_average(const double* field, const double* phi, int n, double phi_frw,
                                     double* partial, int nblk, double* out, cudaStream_t st) {
  void* a1[] = {(void*)&field, (void*)&phi, (void*)&n, (void*)&phi_frw, (void*)&partial};
  cudaError_t e = cudaLaunchKernel((const void*)kavg_partial_kernel, dim3(nblk), dim3(256), a1, 0, st);
  if (e != cudaSuccess) return e;
  const double* cpartial = partial;
  void* a2[] = {(void*)&cpartial, (void*)&nblk, (void*)&n, (void*)&out};
  return cudaLaunchKernel((const void*)kavg_final_kernel, dim3(1), dim3(256), a2, 0, st);
}
}  // namespace cg

namespace {

// the register block holding the current substep input
double* current_a(Box& b) {
  switch (b.stage_next) {
    case 2: case 4: return b.dev.Y;
    default: return b.dev.X;
  }
}

StageBg bg_for(const Box& b, int stage, double phi_next) {
  StageBg bg{};
  bg.phi_FRW = b.frw.get_phi;
  bg.K_FRW = b.frw.get_K;
  bg.rho_FRW = b.frw.get_rho;
  bg.S_FRW = b.frw.get_S;
  bg.K_avg = 0.0;
  bg.phi_FRW_prev = stage == 1 ? b.frw.get_phi : b.phi_prev;
  bg.phi_FRW_next = phi_next;
  return bg;
}

// K_avg from two device sums: sum exp(6 (phi + phi_FRW)) K over sum exp(6 (phi + phi_FRW))
__global__ void kavg_from_sums_kernel(const double* sums, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) out[0] = sums[0] / sums[1];
}

int launch_kavg(cg_ctx* ctx, Box& b, const double* in) {
  if (!b.needs_kavg) return CG_OK;
  if (b.desc.x_ghost != 0) {
    // an x-slab's K_avg is the whole box's: the caller set it (cg_set_kavg)
    if (!b.kavg_set)
      return fail(ctx, CG_ERR_STATE, "an x-slab with this lapse needs cg_kavg_sums / cg_set_kavg before each substep");
    b.kavg_set = false;
    return CG_OK;
  }
  const double* K = in + (size_t)cg::F_K * b.dev.pts;
  const double* phi = in + (size_t)cg::F_PHI * b.dev.pts;
  kavg_partial_kernel<<<b.kavg_blocks, 256, 0, ctx->stream>>>(K, phi, b.dev.pts, b.frw.get_phi, b.kavg_partial);
  kavg_final_kernel<<<1, 256, 0, ctx->stream>>>(b.kavg_partial, b.kavg_blocks, b.dev.pts, b.kavg);
  CG_CUDA(ctx, cudaGetLastError());
  return CG_OK;
}

// dalpha/dt of the uniform background: the lapse gauges of
// BSSNGaugeHandler.cc:16-275 with K_avg = K (a uniform state) and K_FRW = 0
// (trivial FRW reference).
double mixed_bg_lapse(const cg_box_desc& d, double al, double Kd, double phi) {
  switch (d.lapse) {
    case CG_LAPSE_HARMONIC: return -1.0 * al * Kd;
    case CG_LAPSE_CONFORMAL_FLRW: return -1.0 / 3.0 * al * Kd;
    case CG_LAPSE_AWA_GAUGE_WAVE: return -1.0 * (al * al) * Kd;
    case CG_LAPSE_AWA_SHIFTED_WAVE: return -1.0 * Kd;
    case CG_LAPSE_DAMPED_WAVE: return (al * al) * (d.dw_mu_l * (12.0 * phi * d.dw_p - std::log(al)) - Kd);
    default: return 0.0;  // Static, ConformalSync (K_FRW = 0), Anharmonic and 1+log (K - K_avg = 0)
  }
}

// Hamiltonian constraint of the uniform background, bssn.cc:1073-1084 with
// every gradient, A_ij and theta zero: Hc = 2/3 K^2 - 16 pi rho, H = -e^{5 phi}/8 Hc
void mixed_bg_hamiltonian(const Box& b, const double* a, double phi_lag, double* Hc, double* H) {
  const double Kd = a[cg::F_K];
  double rho = 0.0;
  if (b.desc.matter == CG_MATTER_DUST) {
    rho = a[cg::F_D] * std::exp(-6.0 * phi_lag) + b.desc.lambda;  // W = 1
  } else if (b.desc.matter == CG_MATTER_SCALAR) {
    const double sphi = a[cg::F_SPHI], Pi = a[cg::F_SPI];
    const double m2 = b.desc.pot_mass * b.desc.pot_mass;
    rho = 0.5 * Pi * Pi + (b.desc.potential == CG_POT_QUADRATIC ? 0.5 * m2 * sphi * sphi : b.desc.pot_const);
  }
  *Hc = 2.0 / 3.0 * Kd * Kd - 16.0 * cg::kPi * rho;
  *H = -std::exp(5.0 * a[cg::F_PHI]) / 8.0 * *Hc;
}

// Right-hand side of the uniform background (the reference's equations for a
// spatially constant state, trivial FRW): dK/dt, dphi/dt, dalpha/dt and, for
// a scalar field, dphi_s/dt = -alpha Pi, dPi/dt = alpha (K Pi + V'(phi_s))
// (scalar.cc:142-163 with every gradient zero).
void mixed_bg_rhs(const Box& b, const double* a, double phi_lag, double* rhs) {
  for (int f = 0; f < 23; ++f) rhs[f] = 0.0;
  const double Kd = a[cg::F_K], ad = a[cg::F_ALPHA], al = ad + 1.0;
  double rS = 0.0;  // DIFFr + DIFFS of the uniform state
  if (b.desc.matter == CG_MATTER_DUST) {
    rS = (a[cg::F_D] * std::exp(-6.0 * phi_lag) + b.desc.lambda) + (-3.0 * b.desc.lambda);  // W = 1
  } else if (b.desc.matter == CG_MATTER_SCALAR) {
    const double sphi = a[cg::F_SPHI], Pi = a[cg::F_SPI];
    const bool quad = b.desc.potential == CG_POT_QUADRATIC;
    const double m2 = b.desc.pot_mass * b.desc.pot_mass;
    const double V = quad ? 0.5 * m2 * sphi * sphi : b.desc.pot_const;
    const double dV = quad ? m2 * sphi : 0.0;
    rS = 2.0 * Pi * Pi - 2.0 * V;  // rho + S with n^mu d_mu phi_s = -Pi
    rhs[cg::F_SPHI] = -al * Pi;
    rhs[cg::F_SPI] = al * (Kd * Pi + dV);
  }
  rhs[cg::F_K] = al * (1.0 / 3.0 * Kd * Kd) + 4.0 * cg::kPi * al * rS;
  rhs[cg::F_PHI] = -1.0 / 6.0 * (al * Kd);
  rhs[cg::F_ALPHA] = mixed_bg_lapse(b.desc, al, Kd, a[cg::F_PHI]);
  if (b.desc.a_adj_amp != 0.0 || b.desc.k_damping_amp != 0.0) {
    // constraint damping of phi and K (bssn.cc:766-820): 0.1 a_adj_amp dt H,
    // -k_damping_amp H e^{-5 phi}
    double Hc, H;
    mixed_bg_hamiltonian(b, a, phi_lag, &Hc, &H);
    rhs[cg::F_PHI] += 0.1 * b.desc.a_adj_amp * b.desc.dt * H;
    rhs[cg::F_K] += -1.0 * b.desc.k_damping_amp * H * std::exp(-5.0 * a[cg::F_PHI]);
  }
}

void pack_bg(const double* full, double* compact) {
  for (int f : {(int)cg::F_K, (int)cg::F_PHI, (int)cg::F_ALPHA, 18, 19}) compact[cg::mixed::bgi(f)] = full[f];
}

// Constraint / statistics scratch of a box: per-point values (12 arrays),
// per-CTA partials of the two constraint passes, their results, and the
// field-statistics partials (5 + 4 per block) and results (9).
size_t cscratch_doubles(const Box& b) {
  const size_t n = (size_t)b.dev.pts;
  const size_t nblk1 = (size_t)cg::exact::constraint_blocks(b.dev);
  const size_t nblk2 = std::min<size_t>(1024, (n + 255) / 256);
  return 12 * n + 27 * nblk1 + 10 * nblk2 + 37 + 9 * nblk2 + 9;
}

// Sums over the updated points of _p of the fields with a uniform
// background in the FP32-mixed form: K, phi, alpha, field 18 (D or the scalar
// field) and field 19 (Pi); into h[5].  Synchronous.
int background_sums(cg_ctx* ctx, Box& b, double h[5]) {
  const int N = b.dev.pts;
  const int off = b.dev.xg * b.dev.ny * b.dev.nz, n = (b.dev.nx - 2 * b.dev.xg) * b.dev.ny * b.dev.nz;
  const int nblk = std::min(1024, (n + 255) / 256);
  if (!b.cscratch) CG_CUDA(ctx, cudaMalloc(&b.cscratch, sizeof(double) * cscratch_doubles(b)));
  double* part = b.cscratch;
  double* res = part + 5 * (size_t)nblk;
  const double* P = b.dev.P + off;
  const bool dust = b.desc.matter == CG_MATTER_DUST, scalar = b.desc.matter == CG_MATTER_SCALAR;
  // D (dust) or the scalar phi and Pi (fields 18, 19) have a background
  field_sums_kernel<<<nblk, 256, 0, ctx->stream>>>(P + (size_t)cg::F_K * N, P + (size_t)cg::F_PHI * N,
                                                   P + (size_t)cg::F_ALPHA * N,
                                                   dust || scalar ? P + (size_t)18 * N : nullptr,
                                                   scalar ? P + (size_t)19 * N : nullptr, n, part);
  part_final_kernel<<<1, 256, 0, ctx->stream>>>(part, nblk, 5, 5, res);
  CG_CUDA(ctx, cudaGetLastError());
  CG_CUDA(ctx, cudaMemcpyAsync(h, res, sizeof(double) * 5, cudaMemcpyDeviceToHost, ctx->stream));
  CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CG_OK;
}

int mixed_init(cg_ctx* ctx, Box& b) {
  // background registers from the means of _p (K, phi, alpha, D), or the
  // means the caller set for the whole decomposed box
  const int n = (b.dev.nx - 2 * b.dev.xg) * b.dev.ny * b.dev.nz;
  const bool dust = b.desc.matter == CG_MATTER_DUST, scalar = b.desc.matter == CG_MATTER_SCALAR;
  double mean[5];
  if (b.bg_set) {
    for (int q = 0; q < 5; ++q) mean[q] = b.bg_means[q];
  } else {
    double h[5];
    int rc = background_sums(ctx, b, h);
    if (rc) return rc;
    for (int q = 0; q < 5; ++q) mean[q] = h[q] / n;
  }
  for (int f = 0; f < 23; ++f) b.bp[f] = b.ba[f] = b.bprev[f] = b.bf[f] = 0.0;
  b.bp[cg::F_K] = mean[0];
  b.bp[cg::F_PHI] = mean[1];
  b.bp[cg::F_ALPHA] = mean[2];
  if (dust || scalar) b.bp[18] = mean[3];
  if (scalar) b.bp[19] = mean[4];
  for (int f = 0; f < 23; ++f) b.ba[f] = b.bprev[f] = b.bp[f];
  cg::mixed::Bg bg{};
  pack_bg(b.ba, bg.in);
  CG_CUDA(ctx, cg::mixed::launch_init(b.mdev, bg, ctx->stream));
  b.stage_next = 1;
  return CG_OK;
}

// K_avg - Kbar of an FP32-mixed substep input: the conformal average of the
// perturbation, sum exp(6 dphi) dK / sum exp(6 dphi) (the factor exp(6 phibar)
// of the reference's weights cancels), per-block partials in a fixed order
// combined by kavg_final_kernel.
__global__ void mixed_kavg_partial_kernel(const float* __restrict__ dK, const float* __restrict__ dphi, int pts,
                                          double* partial) {
  __shared__ double sK[256], sV[256];
  double aK = 0.0, aV = 0.0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < pts; q += (long long)gridDim.x * blockDim.x) {
    const double e = exp(6.0 * (double)dphi[q]);
    aK += e * (double)dK[q];
    aV += e;
  }
  sK[threadIdx.x] = aK;
  sV[threadIdx.x] = aV;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      sK[threadIdx.x] += sK[threadIdx.x + o];
      sV[threadIdx.x] += sV[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = sK[0];
    partial[2 * blockIdx.x + 1] = sV[0];
  }
}

// Background of substep n of a mixed box: RK4 stage of the uniform state on
// the host (FP64), then the bookkeeping of K{n}Finalize.  The K_avg
// reduction the lapse may need is queued on the context's stream.
int mixed_prepare(cg_ctx* ctx, Box& b, int n, cg::mixed::Bg* out) {
  if (b.needs_kavg) {
    const float* in = (n == 1 || n == 3) ? b.mdev.X : b.mdev.Y;  // the substep's input
    const size_t N = (size_t)b.dev.pts;
    mixed_kavg_partial_kernel<<<b.kavg_blocks, 256, 0, ctx->stream>>>(in + (size_t)cg::F_K * N,
                                                                     in + (size_t)cg::F_PHI * N, b.dev.pts,
                                                                     b.kavg_partial);
    kavg_final_kernel<<<1, 256, 0, ctx->stream>>>(b.kavg_partial, b.kavg_blocks, b.dev.pts, b.kavg);
    CG_CUDA(ctx, cudaGetLastError());
  }
  cg::mixed::Bg& bg = *out;
  bg = cg::mixed::Bg{};
  const double phi_lag = n == 1 ? b.ba[cg::F_PHI] : b.bprev[cg::F_PHI];
  double rhs[23];
  mixed_bg_rhs(b, b.ba, phi_lag, rhs);
  const double dt = b.desc.dt;
  double o[23];
  for (int f = 0; f < 23; ++f) {
    const double cv = rhs[f], pv = b.bp[f];
    if (n == 1) {
      b.bf[f] = dt * cv / 6.0;
      o[f] = pv + dt * cv / 2.0;
    } else if (n == 2) {
      b.bf[f] = b.bf[f] + dt * cv / 3.0;
      o[f] = pv + dt * cv / 2.0;
    } else if (n == 3) {
      b.bf[f] = b.bf[f] + dt * cv / 3.0;
      o[f] = pv + dt * cv;
    } else {
      o[f] = b.bf[f] + (dt * cv / 6.0 + pv);
    }
  }
  pack_bg(b.ba, bg.in);
  pack_bg(b.bprev, bg.prev);
  pack_bg(o, bg.out);
  pack_bg(rhs, bg.rhs);
  bg.e6l = std::exp(-6.0 * phi_lag);
  bg.lambda = b.desc.lambda;
  bg.potential = b.desc.potential;
  bg.pot_const = b.desc.pot_const;
  bg.pot_mass = b.desc.pot_mass;
  bg.gd_c = b.desc.gd_c;
  bg.dw_mu_l = b.desc.dw_mu_l;
  bg.dw_p = b.desc.dw_p;
  {
    const double al = 1.0 + b.ba[cg::F_ALPHA];
    bg.dw_u = b.desc.dw_mu_l * (12.0 * b.ba[cg::F_PHI] * b.desc.dw_p - std::log(al)) - b.ba[cg::F_K];
  }
  bg.tma_wait = b.dev.ph.tma_wait;
  bg.damping = b.desc.a_adj_amp != 0.0 || b.desc.k_damping_amp != 0.0;
  if (bg.damping) {
    mixed_bg_hamiltonian(b, b.ba, phi_lag, &bg.Hcbar, &bg.Hbar);
    bg.e5phib = std::exp(5.0 * b.ba[cg::F_PHI]);
    bg.a_adj_dt = b.desc.a_adj_amp * b.desc.dt;
    bg.k_damp8 = b.desc.k_damping_amp / 8.0;
  }
  bg.ko_scale = b.desc.stencil_order == 2 ? b.desc.ko_coeff / (64.0 * b.desc.dx)
                                          : -b.desc.ko_coeff / (1024.0 * b.desc.dx);
  for (int f = 0; f < 23; ++f) {
    b.bprev[f] = b.ba[f];
    b.ba[f] = o[f];
    if (n == 4) b.bp[f] = o[f];
  }
  b.stage_next = n == 4 ? 1 : n + 1;
  if (n == 4) ++b.steps;
  return CG_OK;
}

int mixed_stage(cg_ctx* ctx, Box& b, int n) {
  cg::mixed::Bg bg;
  int rc = mixed_prepare(ctx, b, n, &bg);
  if (rc) return rc;
  CG_CUDA(ctx, cg::mixed::launch_stage(b.mdev, bg, n, ctx->stream));
  return CG_OK;
}

int do_init(cg_ctx* ctx, Box& b) {
  if (b.mixed) return mixed_init(ctx, b);
  StageBg bg = bg_for(b, 1, b.frw.get_phi);
  CG_CUDA(ctx, cg::launch_init(b.variant, b.dev, bg, ctx->stream));
  b.stage_next = 1;
  return CG_OK;
}

// Substep n of an FP64 box: the K_avg reduction its lapse may need (queued),
// the FRW values of the launch, then the bookkeeping of K{n}Finalize, which
// advances the FRW integrator (bssn.cc:267-305).
int fp64_prepare(cg_ctx* ctx, Box& b, int n, StageBg* bg) {
  FrwHost nxt = b.frw;  // FRW getters of the next substep (flux primitives of the output)
  nxt.stage(n, b.desc.dt);
  *bg = bg_for(b, n, nxt.get_phi);
  int rc = launch_kavg(ctx, b, current_a(b));
  if (rc) return rc;
  b.phi_prev = b.frw.get_phi;
  b.frw = nxt;
  b.stage_next = n == 4 ? 1 : n + 1;
  if (n == 4) ++b.steps;
  return CG_OK;
}

int do_stage(cg_ctx* ctx, Box& b, int n) {
  if (b.mixed) return mixed_stage(ctx, b, n);
  StageBg bg;
  int rc = fp64_prepare(ctx, b, n, &bg);
  if (rc) return rc;
  CG_CUDA(ctx, cg::launch_stage(b.variant, b.dev, bg, n, ctx->stream));
  return CG_OK;
}

int check_box(cg_ctx* ctx, int box) {
  if (!ctx) return CG_ERR_INVALID;
  if (box < 0 || box >= (int)ctx->boxes.size()) return fail(ctx, CG_ERR_INVALID, "box index out of range");
  return CG_OK;
}

int validate(const cg_box_desc& d, std::string& why) {
  const int r = d.stencil_order / 2;
  if (d.stencil_order != 2 && d.stencil_order != 4 && d.stencil_order != 6 && d.stencil_order != 8) {
    why = "stencil_order must be 2, 4, 6 or 8";
    return CG_ERR_INVALID;
  }
  if (d.nx < r + 1 || d.ny < r + 1 || d.nz < r + 1) {
    why = "every axis needs at least stencil_order/2 + 1 points";
    return CG_ERR_INVALID;
  }
  if ((long long)d.nx * d.ny * d.nz > 2000000000LL) {
    why = "box too large for 32-bit point indices";
    return CG_ERR_INVALID;
  }
  if (d.matter < 0 || d.matter > 3) { why = "unknown matter model"; return CG_ERR_INVALID; }
  if (d.matter == CG_MATTER_STATIC && d.lapse != CG_LAPSE_STATIC && d.lapse != CG_LAPSE_CONFORMAL_FLRW) {
    // StaticSim::StaticSim (sims/static.cc:11-17)
    why = "not using a constant lapse gauge: static matter needs the Static or ConformalFLRW lapse";
    return CG_ERR_INVALID;
  }
  if (d.lapse < 0 || d.lapse > 8) { why = "unknown lapse gauge"; return CG_ERR_INVALID; }
  if (d.precision != CG_PREC_FP64 && d.precision != CG_PREC_FP64_FMA && d.precision != CG_PREC_MIXED) {
    why = "unknown precision";
    return CG_ERR_INVALID;
  }
  if (d.z4c != 0 && d.z4c != 1) { why = "z4c must be 0 or 1"; return CG_ERR_INVALID; }
  if (d.shift < CG_SHIFT_NONE || d.shift > CG_SHIFT_AIJ_DRIVER) { why = "unknown shift gauge"; return CG_ERR_INVALID; }
  if (d.shift != CG_SHIFT_NONE) {
    // the reference's shift (USE_BSSN_SHIFT with USE_GAMMA_DRIVER) in the parity build
    if (d.precision != CG_PREC_FP64) { why = "the shift is available with CG_PREC_FP64 only"; return CG_ERR_INVALID; }
    if (d.matter == CG_MATTER_STATIC) { why = "static matter has no shift"; return CG_ERR_INVALID; }
    if (d.z4c) { why = "the shift and Z4c damping do not combine here"; return CG_ERR_INVALID; }
    if (d.x_ghost != 0) { why = "an x-slab has no shift"; return CG_ERR_INVALID; }
    if (d.nx < 4 || d.ny < 4 || d.nz < 4) {
      why = "the shift's upwinded stencils need at least 4 points per axis";
      return CG_ERR_INVALID;
    }
    if (d.gauge_wave_dir < 1 || d.gauge_wave_dir > 3) { why = "gauge_wave_dir must be 1, 2 or 3"; return CG_ERR_INVALID; }
  }
  if (d.precision == CG_PREC_MIXED) {
    if (d.z4c) {
      why = "Z4c damping is available in the FP64 precisions only";
      return CG_ERR_INVALID;
    }
    if (d.matter == CG_MATTER_STATIC) {
      why = "the FP32-mixed form evolves vacuum, dust or scalar boxes";
      return CG_ERR_INVALID;
    }
    if (d.frw_phi != 0.0 || d.frw_K != 0.0 || d.nfluids != 0) {
      why = "the FP32-mixed form evolves about its own uniform background (trivial FRW reference)";
      return CG_ERR_INVALID;
    }
  }
  if (d.ko_coeff != 0.0) {
    const int rko = d.stencil_order == 8 ? 5 : 2;  // orders 4 and 6: no dissipation (utils/math.h:36-72)
    if ((d.stencil_order == 2 || d.stencil_order == 8) && (d.nx < rko + 1 || d.ny < rko + 1 || d.nz < rko + 1)) {
      why = "Kreiss-Oliger dissipation needs stencil_order/2 + 2 points per axis (order 2) or 6 (order 8)";
      return CG_ERR_INVALID;
    }
  }
  if (d.nfluids < 0 || d.nfluids > 4) { why = "at most 4 FRW fluids"; return CG_ERR_INVALID; }
  if (!(d.dx > 0.0) || !std::isfinite(d.dt)) { why = "dx must be positive and dt finite"; return CG_ERR_INVALID; }
  if (d.x_ghost != 0) {
    // an x-slab: interior bricks only, ghost planes refreshed by the caller
    const int g = d.x_ghost;
    const int reach = d.ko_coeff != 0.0 && (d.stencil_order == 2 || d.stencil_order == 8)
                          ? (d.stencil_order == 8 ? 5 : 2)
                          : d.stencil_order / 2;
    if (g < 0 || g % 4 != 0 || g < reach) {
      why = "x_ghost must be a multiple of 4 and at least the stencil (and Kreiss-Oliger) radius";
      return CG_ERR_INVALID;
    }
    if (d.nx - 2 * g < 4 || (d.nx - 2 * g) % 4 != 0) {
      why = "an x-slab needs nx - 2 x_ghost interior planes, a positive multiple of 4";
      return CG_ERR_INVALID;
    }
    if (lapse_needs_kavg(d.lapse) && d.precision == CG_PREC_MIXED) {
      why = "an x-slab in the FP32-mixed form needs a lapse without K_avg";
      return CG_ERR_INVALID;
    }
  }
  return CG_OK;
}

bool is_pow2(double x) {
  int e;
  const double m = std::frexp(x, &e);
  return m == 0.5;
}

void free_box(Box& b) {
  cudaFree(b.cscratch);
  b.cscratch = nullptr;
  if (b.mixed) {
    cudaFree(b.mdev.X);
    cudaFree(b.mdev.Y);
    cudaFree(b.mdev.FP0);
    cudaFree(b.mdev.FP1);
    b.mdev.X = b.mdev.Y = nullptr;
    b.mdev.FP0 = b.mdev.FP1 = nullptr;
  }
  cudaFree(b.dev.P);
  cudaFree(b.dev.F);
  cudaFree(b.dev.X);
  cudaFree(b.dev.Y);
  cudaFree(b.dev.FP0);
  cudaFree(b.dev.FP1);
  cudaFree(b.kavg_partial);
  b.dev.P = b.dev.F = b.dev.X = b.dev.Y = b.dev.FP0 = b.dev.FP1 = nullptr;
  b.kavg_partial = nullptr;
  cudaFree(b.stage_in);
  cudaFree(b.stage_out);
  b.stage_in = b.stage_out = nullptr;
  for (cudaEvent_t* ev : {&b.in_ready, &b.in_free, &b.out_ready, &b.out_free}) {
    if (*ev) cudaEventDestroy(*ev);
    *ev = nullptr;
  }
}

}  // namespace

extern "C" {

int cg_version(void) { return CG_ABI_VERSION; }

int cg_num_fields(int matter) {
  return matter == CG_MATTER_DUST ? 22 : matter == CG_MATTER_SCALAR ? 23 : matter == CG_MATTER_STATIC ? 19 : 18;
}

const char* cg_field_name(int matter, int field) {
  static const char* bssn[18] = {"DIFFgamma11", "DIFFgamma12", "DIFFgamma13", "DIFFgamma22", "DIFFgamma23",
                                 "DIFFgamma33", "DIFFphi", "A11", "A12", "A13", "A22", "A23", "A33",
                                 "DIFFK", "Gamma1", "Gamma2", "Gamma3", "DIFFalpha"};
  static const char* dust[4] = {"D", "S1", "S2", "S3"};
  static const char* scal[5] = {"phi", "Pi", "psi1", "psi2", "psi3"};
  if (field < 0 || field >= cg_num_fields(matter)) return nullptr;
  if (field < 18) return bssn[field];
  if (matter == CG_MATTER_STATIC) return "DIFFD";
  return matter == CG_MATTER_DUST ? dust[field - 18] : scal[field - 18];
}

void cg_box_desc_default(cg_box_desc* d, int n) {
  if (!d) return;
  std::memset(d, 0, sizeof(*d));
  d->nx = d->ny = d->nz = n;
  d->stencil_order = 8;
  d->matter = CG_MATTER_DUST;
  d->lapse = CG_LAPSE_HARMONIC;
  d->precision = CG_PREC_FP64;
  d->normalize_metric = 1;
  d->potential = CG_POT_CONST;
  d->dx = 1.0 / n;
  d->dt = (double)(0.1L * (long double)d->dx);
  d->gd_c = 1.0;
  d->pot_const = 3.0e-4;
  d->pot_mass = 1.0;
  d->shift = CG_SHIFT_NONE;
  d->gauge_wave_dir = 1;      // BSSNGaugeHandler.h:139-147 defaults
  d->k_driver_coeff = 0.04;
}

int cg_create(const cg_box_desc* boxes, int nboxes, cg_ctx** out) {
  if (!out) return fail(nullptr, CG_ERR_INVALID, "out is null");
  *out = nullptr;
  if (!boxes || nboxes <= 0) return fail(nullptr, CG_ERR_INVALID, "need at least one box");
  for (int b = 0; b < nboxes; ++b) {
    std::string why;
    if (validate(boxes[b], why) != CG_OK)
      return fail(nullptr, CG_ERR_INVALID, "box " + std::to_string(b) + ": " + why);
  }
  cg_ctx* ctx = new (std::nothrow) cg_ctx();
  if (!ctx) return fail(nullptr, CG_ERR_MEMORY, "host allocation failed");
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete ctx;
    return fail(nullptr, CG_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  ctx->stream = ctx->own_stream;
  e = cudaMalloc(&ctx->status, sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMemset(ctx->status, 0, sizeof(unsigned));
  ctx->boxes.resize(nboxes);
  for (int bi = 0; bi < nboxes && e == cudaSuccess; ++bi) {
    Box& b = ctx->boxes[bi];
    b.desc = boxes[bi];
    const cg_box_desc& d = b.desc;
    b.variant = d.precision == CG_PREC_FP64_FMA ? cg::kFast : cg::kExact;
    b.dev.nx = d.nx;
    b.dev.xg = d.x_ghost;
    b.dev.ny = d.ny;
    b.dev.nz = d.nz;
    b.dev.pts = d.nx * d.ny * d.nz;
    b.dev.nfields = cg_num_fields(d.matter) + (d.z4c ? 1 : 0) + (d.shift != CG_SHIFT_NONE ? 7 : 0);
    b.dev.z4c = d.z4c ? 1 : 0;
    b.dev.shift = d.shift != CG_SHIFT_NONE ? 1 : 0;
    b.dev.order = d.stencil_order;
    b.dev.matter = d.matter;
    cg::Physics& ph = b.dev.ph;
    ph.matter = d.matter;
    ph.lapse = d.lapse;
    ph.potential = d.potential;
    ph.normalize = d.normalize_metric;
    ph.dx = d.dx;
    ph.inv_dx = 1.0 / d.dx;
    ph.dx_pow2 = is_pow2(d.dx) ? 1 : 0;
    ph.dt = d.dt;
    ph.lambda = d.lambda;
    ph.a_adj_amp = d.a_adj_amp;
    ph.ko_coeff = d.ko_coeff;
    ph.ko_pden = std::pow(d.dx, d.stencil_order == 8 ? 10.0 : 4.0);
    ph.ko_pnum = std::pow(d.dx, d.stencil_order == 8 ? 9.0 : 3.0);
    ph.k_damping_amp = d.k_damping_amp;
    ph.gd_c = d.gd_c;
    ph.dw_mu_l = d.dw_mu_l;
    ph.dw_p = d.dw_p;
    ph.pot_const = d.pot_const;
    ph.pot_mass = d.pot_mass;
    ph.shift = d.shift;
    ph.gauge_wave_dir = d.gauge_wave_dir;
    ph.gd_eta = d.gd_eta;
    ph.dw_mu_s = d.dw_mu_s;
    ph.k_driver_coeff = d.k_driver_coeff;
    ph.tma_wait = kTmaWaitDefault;
    b.frw.phi = d.frw_phi;
    b.frw.K = d.frw_K;
    b.frw.n = d.nfluids;
    for (int m = 0; m < d.nfluids; ++m) {
      b.frw.rho[m] = d.fluid_rho[m];
      b.frw.w[m] = d.fluid_w[m];
    }
    b.frw.set_gets(b.frw.phi, b.frw.K, b.frw.rho);
    const size_t reg = sizeof(double) * (size_t)b.dev.nfields * b.dev.pts;
    b.mixed = d.precision == CG_PREC_MIXED;
    e = cudaMalloc(&b.dev.P, reg);
    if (e == cudaSuccess) e = cudaMalloc(&b.dev.F, reg);
    if (!b.mixed) {
      if (e == cudaSuccess) e = cudaMalloc(&b.dev.X, reg);
      if (e == cudaSuccess) e = cudaMalloc(&b.dev.Y, reg);
      if (e == cudaSuccess && d.matter == CG_MATTER_DUST) {
        const size_t fp = sizeof(double) * (size_t)cg::P_N * b.dev.pts;
        e = cudaMalloc(&b.dev.FP0, fp);
        if (e == cudaSuccess) e = cudaMalloc(&b.dev.FP1, fp);
      }
      for (double* p : {b.dev.P, b.dev.F, b.dev.X, b.dev.Y})
        if (e == cudaSuccess) e = cudaMemset(p, 0, reg);
      if (e == cudaSuccess) {  // TMA tile copies where the layout allows
        if (b.variant == cg::kFast) cg::fast::make_tile_maps(b.dev);
        else cg::exact::make_tile_maps(b.dev);
        b.dev.tma = b.dev.tma && ctx->opt_tma;
      }
    } else {
      cg::MixedBox& m = b.mdev;
      m.nx = d.nx; m.ny = d.ny; m.nz = d.nz; m.pts = b.dev.pts; m.nfields = b.dev.nfields;
      m.order = d.stencil_order; m.matter = d.matter; m.lapse = d.lapse; m.normalize = d.normalize_metric;
      m.xg = d.x_ghost;
      m.dx = d.dx; m.dt = d.dt;
      m.ko = d.ko_coeff;
      m.kavg = nullptr;  // set below when the lapse uses K_avg
      m.P = b.dev.P;
      m.F = b.dev.F;
      m.status = ctx->status;
      const size_t reg32 = sizeof(float) * (size_t)b.dev.nfields * b.dev.pts;
      if (e == cudaSuccess) e = cudaMalloc(&m.X, reg32);
      if (e == cudaSuccess) e = cudaMalloc(&m.Y, reg32);
      if (e == cudaSuccess) {
        cg::mixed::make_tile_maps(m);  // TMA tile copies where the layout allows
        m.tma = m.tma && ctx->opt_tma;
      }
      if (e == cudaSuccess && d.matter == CG_MATTER_DUST) {
        const size_t fp = sizeof(float) * (size_t)cg::P_N * b.dev.pts;
        e = cudaMalloc(&m.FP0, fp);
        if (e == cudaSuccess) e = cudaMalloc(&m.FP1, fp);
      }
      for (double* p : {b.dev.P, b.dev.F})
        if (e == cudaSuccess) e = cudaMemset(p, 0, reg);
    }
    b.dev.status = ctx->status;
    b.needs_kavg = lapse_needs_kavg(d.lapse);
    if (e == cudaSuccess && b.needs_kavg) {
      b.kavg_blocks = std::min(1024, (b.dev.pts + 255) / 256);
      e = cudaMalloc(&b.kavg_partial, sizeof(double) * (2 * b.kavg_blocks + 3));
      b.kavg = b.kavg_partial + 2 * b.kavg_blocks;
      b.kavg_sums = b.kavg + 1;
      b.dev.kavg = b.kavg;
      if (b.mixed) b.mdev.kavg = b.kavg;
    }
  }
  if (e != cudaSuccess) {
    const std::string msg = std::string("device allocation: ") + cudaGetErrorString(e);
    for (Box& b : ctx->boxes) free_box(b);
    cudaFree(ctx->status);
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return fail(nullptr, e == cudaErrorMemoryAllocation ? CG_ERR_MEMORY : CG_ERR_CUDA, msg);
  }
  *out = ctx;
  return CG_OK;
}

int cg_destroy(cg_ctx* ctx) {
  if (!ctx) return CG_ERR_INVALID;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  for (Group& g : ctx->groups) cudaFree(g.table);
  for (Box& b : ctx->boxes) free_box(b);
  cudaFree(ctx->red);
  cudaFree(ctx->status);
  for (cudaStream_t* cs : {&ctx->copy_stream, &ctx->up_stream})
    if (*cs) {
      cudaStreamSynchronize(*cs);
      cudaStreamDestroy(*cs);
    }
  if (ctx->copy_start) cudaEventDestroy(ctx->copy_start);
  for (cudaEvent_t ev : ctx->copy_done) cudaEventDestroy(ev);
  if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
  delete ctx;
  return CG_OK;
}

int cg_set_stream(cg_ctx* ctx, void* stream) {
  if (!ctx) return CG_ERR_INVALID;
  ctx->stream = stream ? (cudaStream_t)stream : ctx->own_stream;
  return CG_OK;
}

int cg_get_stream(cg_ctx* ctx, void** stream) {
  if (!ctx || !stream) return CG_ERR_INVALID;
  *stream = (void*)ctx->stream;
  return CG_OK;
}

static int state_copy(cg_ctx* ctx, int box, double* host, size_t count, bool upload, bool async) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  Box& b = ctx->boxes[box];
  const size_t n = (size_t)b.dev.nfields * b.dev.pts;
  if (!host || count != n)
    return fail(ctx, CG_ERR_INVALID, "count must be nfields*nx*ny*nz = " + std::to_string(n));
  const size_t bytes = n * sizeof(double);
  if (upload) {
    CG_CUDA(ctx, cudaMemcpyAsync(b.dev.P, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    b.stage_next = 0;
    b.steps = 0;
  } else {
    // after the staged download of an earlier exchange (it may write the same host buffer)
    if (b.out_free) CG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, b.out_free, 0));
    CG_CUDA(ctx, cudaMemcpyAsync(host, b.dev.P, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  }
  if (!async) CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CG_OK;
}

int cg_upload_state(cg_ctx* ctx, int box, const double* host, size_t count) {
  return state_copy(ctx, box, const_cast<double*>(host), count, true, false);
}
int cg_download_state(cg_ctx* ctx, int box, double* host, size_t count) {
  return state_copy(ctx, box, host, count, false, false);
}
int cg_upload_state_async(cg_ctx* ctx, int box, const double* host, size_t count) {
  return state_copy(ctx, box, const_cast<double*>(host), count, true, true);
}
int cg_download_state_async(cg_ctx* ctx, int box, double* host, size_t count) {
  return state_copy(ctx, box, host, count, false, true);
}

// The download runs on a second stream, field by field, after the work queued
// so far on the context's stream; the context's stream uploads field f once
// field f has been downloaded.  Opposite copy directions overlap, so the pair
// takes about as long as the longer of the two.
static int ensure_event(cg_ctx* ctx, cudaEvent_t* ev) {
  if (!*ev) CG_CUDA(ctx, cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
  return CG_OK;
}

// The input is copied into the box's staging buffer on its own stream, at
// once; the exchange that names the same host buffer moves it into the
// registers by a device copy.
int cg_prefetch_state_async(cg_ctx* ctx, int box, const double* host_in, size_t count) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  Box& b = ctx->boxes[box];
  const size_t n = (size_t)b.dev.nfields * b.dev.pts;
  if (!host_in || count != n)
    return fail(ctx, CG_ERR_INVALID, "count must be nfields*nx*ny*nz = " + std::to_string(n));
  if (!ctx->up_stream) CG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->up_stream, cudaStreamNonBlocking));
  for (cudaEvent_t* ev : {&b.in_ready, &b.in_free})
    if ((rc = ensure_event(ctx, ev))) return rc;
  if (!b.stage_in) {
    const cudaError_t e = cudaMalloc(&b.stage_in, n * sizeof(double));
    if (e != cudaSuccess) {
      b.stage_in = nullptr;
      return fail(ctx, e == cudaErrorMemoryAllocation ? CG_ERR_MEMORY : CG_ERR_CUDA,
                  std::string("staging buffer: ") + cudaGetErrorString(e));
    }
  }
  // the previous staged input has been moved into the registers
  CG_CUDA(ctx, cudaStreamWaitEvent(ctx->up_stream, b.in_free, 0));
  CG_CUDA(ctx, cudaMemcpyAsync(b.stage_in, host_in, n * sizeof(double), cudaMemcpyHostToDevice, ctx->up_stream));
  CG_CUDA(ctx, cudaEventRecord(b.in_ready, ctx->up_stream));
  b.pre_host = host_in;
  b.pre_count = count;
  return CG_OK;
}

// staged exchange: the result leaves through stage_out (its download overlaps
// later work on the context's stream), the input comes from stage_in
static int exchange_staged(cg_ctx* ctx, Box& b, double* host_out, size_t n) {
  int rc = CG_OK;
  for (cudaEvent_t* ev : {&b.out_ready, &b.out_free})
    if ((rc = ensure_event(ctx, ev))) return rc;
  if (!b.stage_out) {
    const cudaError_t e = cudaMalloc(&b.stage_out, n * sizeof(double));
    if (e != cudaSuccess) {
      b.stage_out = nullptr;
      return fail(ctx, e == cudaErrorMemoryAllocation ? CG_ERR_MEMORY : CG_ERR_CUDA,
                  std::string("staging buffer: ") + cudaGetErrorString(e));
    }
  }
  const size_t bytes = n * sizeof(double);
  CG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, b.out_free, 0));  // the previous staged download is done
  CG_CUDA(ctx, cudaMemcpyAsync(b.stage_out, b.dev.P, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  CG_CUDA(ctx, cudaEventRecord(b.out_ready, ctx->stream));
  CG_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, b.out_ready, 0));
  CG_CUDA(ctx, cudaMemcpyAsync(host_out, b.stage_out, bytes, cudaMemcpyDeviceToHost, ctx->copy_stream));
  CG_CUDA(ctx, cudaEventRecord(b.out_free, ctx->copy_stream));
  CG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, b.in_ready, 0));  // the prefetched input has arrived
  CG_CUDA(ctx, cudaMemcpyAsync(b.dev.P, b.stage_in, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
  CG_CUDA(ctx, cudaEventRecord(b.in_free, ctx->stream));
  b.pre_host = nullptr;
  b.pre_count = 0;
  b.stage_next = 0;
  b.steps = 0;
  return CG_OK;
}

int cg_exchange_state_async(cg_ctx* ctx, int box, double* host_out, const double* host_in, size_t count) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  Box& b = ctx->boxes[box];
  const size_t n = (size_t)b.dev.nfields * b.dev.pts;
  if (!host_out || !host_in || count != n)
    return fail(ctx, CG_ERR_INVALID, "count must be nfields*nx*ny*nz = " + std::to_string(n));
  if (!ctx->copy_stream) CG_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
  if (b.pre_host == host_in && b.pre_count == count && b.stage_in) return exchange_staged(ctx, b, host_out, n);
  // after the staged download of an earlier exchange (it may write the same host buffer)
  if (b.out_free) CG_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, b.out_free, 0));
  if (!ctx->copy_start) CG_CUDA(ctx, cudaEventCreateWithFlags(&ctx->copy_start, cudaEventDisableTiming));
  while ((int)ctx->copy_done.size() < b.dev.nfields) {
    cudaEvent_t ev = nullptr;
    CG_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    ctx->copy_done.push_back(ev);
  }
  const size_t pts = (size_t)b.dev.pts, fbytes = pts * sizeof(double);
  CG_CUDA(ctx, cudaEventRecord(ctx->copy_start, ctx->stream));
  CG_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->copy_start, 0));
  for (int f = 0; f < b.dev.nfields; ++f) {
    CG_CUDA(ctx, cudaMemcpyAsync(host_out + f * pts, b.dev.P + f * pts, fbytes, cudaMemcpyDeviceToHost,
                                 ctx->copy_stream));
    CG_CUDA(ctx, cudaEventRecord(ctx->copy_done[f], ctx->copy_stream));
  }
  for (int f = 0; f < b.dev.nfields; ++f) {
    CG_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->copy_done[f], 0));
    CG_CUDA(ctx, cudaMemcpyAsync(b.dev.P + f * pts, host_in + f * pts, fbytes, cudaMemcpyHostToDevice, ctx->stream));
  }
  b.stage_next = 0;
  b.steps = 0;
  return CG_OK;
}

static int field_copy(cg_ctx* ctx, int box, int field, char reg, double* host, size_t n, bool upload) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  Box& b = ctx->boxes[box];
  if (field < 0 || field >= b.dev.nfields) return fail(ctx, CG_ERR_INVALID, "field index out of range");
  if (!host || n != (size_t)b.dev.pts) return fail(ctx, CG_ERR_INVALID, "n must be nx*ny*nz");
  double* base = nullptr;
  if (reg == 'p')
    base = b.dev.P;
  else if (reg == 'f')
    base = b.dev.F;
  else if (reg == 'a') {
    if (b.stage_next == 0) return fail(ctx, CG_ERR_STATE, "the 'a' register exists after cg_step_init");
    if (b.mixed) {
      // FP32 perturbation about the uniform background: a = abar + delta
      if (upload) return fail(ctx, CG_ERR_INVALID, "the 'a' register of a mixed box is read-only");
      const float* src = (b.stage_next == 2 || b.stage_next == 4 ? b.mdev.Y : b.mdev.X) + (size_t)field * b.dev.pts;
      std::vector<float> tmp(n);
      CG_CUDA(ctx, cudaMemcpyAsync(tmp.data(), src, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
      CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      const double abar = b.ba[field];
      for (size_t q = 0; q < n; ++q) host[q] = abar + (double)tmp[q];
      return CG_OK;
    }
    base = current_a(b);
  } else
    return fail(ctx, CG_ERR_INVALID, "reg must be 'p', 'a' or 'f'");
  double* d = base + (size_t)field * b.dev.pts;
  const size_t bytes = n * sizeof(double);
  if (upload) {
    CG_CUDA(ctx, cudaMemcpyAsync(d, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    if (reg == 'p') {
      b.stage_next = 0;
    }
  } else {
    CG_CUDA(ctx, cudaMemcpyAsync(host, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  }
  CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CG_OK;
}

int cg_upload_field(cg_ctx* ctx, int box, int field, char reg, const double* host, size_t n) {
  return field_copy(ctx, box, field, reg, const_cast<double*>(host), n, true);
}
int cg_download_field(cg_ctx* ctx, int box, int field, char reg, double* host, size_t n) {
  return field_copy(ctx, box, field, reg, host, n, false);
}

int cg_substep_input(cg_ctx* ctx, int box, void** input, void** flux) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  if (!input) return fail(ctx, CG_ERR_INVALID, "input is null");
  Box& b = ctx->boxes[box];
  if (b.stage_next == 0) return fail(ctx, CG_ERR_STATE, "the substep input exists after cg_step_init");
  const bool even = b.stage_next == 2 || b.stage_next == 4, dust = b.desc.matter == CG_MATTER_DUST;
  if (b.mixed) {
    *input = even ? b.mdev.Y : b.mdev.X;
    if (flux) *flux = dust ? (even ? b.mdev.FP1 : b.mdev.FP0) : nullptr;
  } else {
    *input = even ? b.dev.Y : b.dev.X;
    if (flux) *flux = dust ? (even ? b.dev.FP1 : b.dev.FP0) : nullptr;
  }
  return CG_OK;
}

int cg_kavg_sums(cg_ctx* ctx, int box, double** dsums) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  if (!dsums) return fail(ctx, CG_ERR_INVALID, "dsums is null");
  Box& b = ctx->boxes[box];
  if (!b.needs_kavg || b.mixed) return fail(ctx, CG_ERR_INVALID, "the box's lapse does not use K_avg");
  if (b.stage_next == 0) return fail(ctx, CG_ERR_STATE, "K_avg sums exist after cg_step_init");
  // over the updated points of the next substep's input
  const int N = b.dev.pts, off = b.dev.xg * b.dev.ny * b.dev.nz;
  const int n = (b.dev.nx - 2 * b.dev.xg) * b.dev.ny * b.dev.nz;
  const double* in = current_a(b);
  kavg_partial_kernel<<<b.kavg_blocks, 256, 0, ctx->stream>>>(in + (size_t)cg::F_K * N + off,
                                                               in + (size_t)cg::F_PHI * N + off, n, b.frw.get_phi,
                                                               b.kavg_partial);
  part_final_kernel<<<1, 256, 0, ctx->stream>>>(b.kavg_partial, b.kavg_blocks, 2, 2, b.kavg_sums);
  CG_CUDA(ctx, cudaGetLastError());
  *dsums = b.kavg_sums;
  return CG_OK;
}

int cg_set_kavg(cg_ctx* ctx, int box, const double* dsums) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  if (!dsums) return fail(ctx, CG_ERR_INVALID, "dsums is null");
  Box& b = ctx->boxes[box];
  if (!b.needs_kavg || b.mixed) return fail(ctx, CG_ERR_INVALID, "the box's lapse does not use K_avg");
  kavg_from_sums_kernel<<<1, 32, 0, ctx->stream>>>(dsums, b.kavg);
  CG_CUDA(ctx, cudaGetLastError());
  b.kavg_set = true;
  return CG_OK;
}

int cg_background_sums(cg_ctx* ctx, int box, double* out, int n) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  if (!out || n < 6) return fail(ctx, CG_ERR_INVALID, "out needs 6 entries");
  Box& b = ctx->boxes[box];
  rc = background_sums(ctx, b, out);
  if (rc) return rc;
  out[5] = (double)(b.dev.nx - 2 * b.dev.xg) * b.dev.ny * b.dev.nz;
  return CG_OK;
}

int cg_set_background(cg_ctx* ctx, int box, const double* means, int n) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  Box& b = ctx->boxes[box];
  if (!b.mixed) return fail(ctx, CG_ERR_INVALID, "the background belongs to FP32-mixed boxes");
  if (b.stage_next > 1) return fail(ctx, CG_ERR_STATE, "set the background between steps");
  if (!means) {
    b.bg_set = false;  // back to the box's own means
  } else {
    if (n < 5) return fail(ctx, CG_ERR_INVALID, "means needs 5 entries");
    for (int q = 0; q < 5; ++q) b.bg_means[q] = means[q];
    b.bg_set = true;
  }
  b.stage_next = 0;  // the next step starts from the initialisation
  return CG_OK;
}

int cg_device_register(cg_ctx* ctx, int box, char reg, double** dptr) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  if (!dptr) return fail(ctx, CG_ERR_INVALID, "dptr is null");
  Box& b = ctx->boxes[box];
  if (reg == 'p')
    *dptr = b.dev.P;
  else if (reg == 'f')
    *dptr = b.dev.F;
  else
    return fail(ctx, CG_ERR_INVALID, "reg must be 'p' or 'f'");
  // the caller may write _p through this pointer: rebuild the inputs
  b.stage_next = 0;
  return CG_OK;
}

}  // extern "C" (reopened below)
namespace {
// ---- launch groups --------------------------------------------------------------
// Boxes with the same arithmetic, stencil order and matter model (up to
// kMaxGroupBoxes per group) are advanced by one launch per substep when
// CG_OPT_BATCH is on; a box without a partner keeps its own launch.

template <class B>
int bricks_along(int n, int b) { return (n + b - 1) / b; }

// Device table of a group in its launch order (lpt: largest box first).
int write_table(cg_ctx* ctx, Group& g) {
  std::vector<int> order = g.members;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return g.lpt ? ctx->boxes[a].dev.pts > ctx->boxes[b].dev.pts : a < b;
  });
  g.members = order;
  const size_t m = order.size();
  int first = 0;
  if (g.mixed) {
    using Br = cg::tile::Brick32;
    std::vector<cg::mixed::GroupBox> t(m);
    for (size_t q = 0; q < m; ++q) {
      const Box& b = ctx->boxes[order[q]];
      cg::mixed::GroupBox& e = t[q];
      e.nx = b.mdev.nx; e.ny = b.mdev.ny; e.nz = b.mdev.nz; e.pts = b.mdev.pts;
      e.lapse = b.mdev.lapse; e.normalize = b.mdev.normalize;
      e.idx = (float)(1.0 / b.mdev.dx);
      e.dt = b.mdev.dt;
      e.P = b.mdev.P; e.F = b.mdev.F; e.X = b.mdev.X; e.Y = b.mdev.Y; e.FP0 = b.mdev.FP0; e.FP1 = b.mdev.FP1;
      e.status = b.mdev.status;
      e.kavg = b.mdev.kavg;
      e.mapX = b.mdev.mapX;
      e.mapY = b.mdev.mapY;
      e.tma = b.mdev.tma;
      e.nbx = bricks_along<Br>(e.nx, Br::BX); e.nby = bricks_along<Br>(e.ny, Br::BY); e.nbz = bricks_along<Br>(e.nz, Br::BZ);
      e.first = first;
      first += e.nbx * e.nby * e.nbz;
    }
    if (!g.table) CG_CUDA(ctx, cudaMalloc(&g.table, sizeof(cg::mixed::GroupBox) * m));
    CG_CUDA(ctx, cudaMemcpyAsync(g.table, t.data(), sizeof(cg::mixed::GroupBox) * m, cudaMemcpyHostToDevice, ctx->stream));
    CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  } else {
    using Br = cg::tile::Brick64;
    std::vector<cg::GroupBox> t(m);
    for (size_t q = 0; q < m; ++q) {
      const Box& b = ctx->boxes[order[q]];
      cg::GroupBox& e = t[q];
      e.nx = b.dev.nx; e.ny = b.dev.ny; e.nz = b.dev.nz; e.pts = b.dev.pts;
      e.ph = b.dev.ph;
      e.kavg = b.dev.kavg;
      e.P = b.dev.P; e.F = b.dev.F; e.X = b.dev.X; e.Y = b.dev.Y; e.FP0 = b.dev.FP0; e.FP1 = b.dev.FP1;
      e.status = b.dev.status;
      e.mapX = b.dev.mapX;
      e.mapY = b.dev.mapY;
      e.tma = b.dev.tma;
      e.nbx = bricks_along<Br>(e.nx, Br::BX); e.nby = bricks_along<Br>(e.ny, Br::BY); e.nbz = bricks_along<Br>(e.nz, Br::BZ);
      e.first = first;
      first += e.nbx * e.nby * e.nbz;
    }
    // the members' flux-primitive maps follow the GroupBox entries
    std::vector<cg::GroupFluxMaps> fm(m);
    for (size_t q = 0; q < m; ++q) {
      const Box& b = ctx->boxes[order[q]];
      for (int a = 0; a < 3; ++a) {
        fm[q].fp0[a] = b.dev.fmap0[a];
        fm[q].fp1[a] = b.dev.fmap1[a];
      }
      fm[q].valid = b.dev.fmaps && b.dev.tma;
    }
    const size_t tb = sizeof(cg::GroupBox) * m;
    if (!g.table) CG_CUDA(ctx, cudaMalloc(&g.table, tb + sizeof(cg::GroupFluxMaps) * m));
    CG_CUDA(ctx, cudaMemcpyAsync(g.table, t.data(), tb, cudaMemcpyHostToDevice, ctx->stream));
    CG_CUDA(ctx, cudaMemcpyAsync(static_cast<char*>(g.table) + tb, fm.data(), sizeof(cg::GroupFluxMaps) * m,
                                 cudaMemcpyHostToDevice, ctx->stream));
    CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  g.total = first;
  return CG_OK;
}

int ensure_groups(cg_ctx* ctx) {
  if (ctx->grouped) return CG_OK;
  for (Group& g : ctx->groups) cudaFree(g.table);
  ctx->groups.clear();
  ctx->singles.clear();
  if (ctx->gexec) {
    cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
  }
  std::vector<bool> used(ctx->boxes.size(), false);
  for (size_t a = 0; a < ctx->boxes.size(); ++a) {
    if (used[a]) continue;
    const Box& ba = ctx->boxes[a];
    Group g;
    g.mixed = ba.mixed;
    g.variant = ba.variant;
    g.order = ba.desc.stencil_order;
    g.matter = ba.desc.matter;
    g.members.push_back((int)a);
    used[a] = true;
    // boxes with Kreiss-Oliger dissipation, Z4c damping or a shift and x-slabs keep their own launches
    for (size_t b = a + 1; ba.desc.ko_coeff == 0.0 && ba.desc.z4c == 0 && ba.desc.shift == CG_SHIFT_NONE &&
                           ba.desc.x_ghost == 0 && b < ctx->boxes.size() &&
                           g.members.size() < (size_t)cg::kMaxGroupBoxes;
         ++b) {
      const Box& bb = ctx->boxes[b];
      if (used[b] || bb.mixed != g.mixed || bb.variant != g.variant || bb.desc.stencil_order != g.order ||
          bb.desc.matter != g.matter || bb.desc.ko_coeff != 0.0 || bb.desc.z4c != 0 ||
          bb.desc.shift != CG_SHIFT_NONE || bb.desc.x_ghost != 0)
        continue;
      g.members.push_back((int)b);
      used[b] = true;
    }
    if (!ctx->opt_batch || g.members.size() < 2) {
      for (int q : g.members) ctx->singles.push_back(q);
      continue;
    }
    g.grid = ctx->opt_group_grid;
    int rc = write_table(ctx, g);
    if (rc) {
      cudaFree(g.table);
      return rc;
    }
    ctx->groups.push_back(g);
  }
  std::sort(ctx->singles.begin(), ctx->singles.end());
  // every box is launched exactly once per substep
  size_t scheduled = ctx->singles.size();
  for (const Group& g : ctx->groups) scheduled += g.members.size();
  if (scheduled != ctx->boxes.size()) return fail(ctx, CG_ERR_STATE, "launch groups do not cover every box");
  ctx->grouped = true;
  return CG_OK;
}

// Substep n of every member: backgrounds prepared (and the host state
// advanced) box by box, one launch for the group.  `boxes` may be a scratch
// copy of the context's boxes (the autotuner's trial launches).
int group_launch(cg_ctx* ctx, Group& g, std::vector<Box>& boxes, int n) {
  if (g.grid < 0) {
    // the autotuner found the members' own launches faster
    for (int q : g.members) {
      int rc = do_stage(ctx, boxes[q], n);
      if (rc) return rc;
    }
    return CG_OK;
  }
  if (g.mixed) {
    cg::mixed::GroupBg gb{};
    gb.nboxes = (int)g.members.size();
    gb.total = g.total;
    for (size_t q = 0; q < g.members.size(); ++q) {
      int rc = mixed_prepare(ctx, boxes[g.members[q]], n, &gb.bg[q]);
      if (rc) return rc;
    }
    CG_CUDA(ctx, cg::mixed::launch_group(static_cast<const cg::mixed::GroupBox*>(g.table), gb, g.order, g.matter, n,
                                         g.grid, ctx->stream));
  } else {
    cg::GroupBg gb{};
    gb.nboxes = (int)g.members.size();
    gb.total = g.total;
    for (size_t q = 0; q < g.members.size(); ++q) {
      int rc = fp64_prepare(ctx, boxes[g.members[q]], n, &gb.bg[q]);
      if (rc) return rc;
    }
    CG_CUDA(ctx, cg::launch_group(g.variant, static_cast<const cg::GroupBox*>(g.table), gb, g.order, g.matter, n,
                                  g.grid, ctx->stream));
  }
  return CG_OK;
}

int all_stage(cg_ctx* ctx, int n) {
  for (Group& g : ctx->groups) {
    int rc = group_launch(ctx, g, ctx->boxes, n);
    if (rc) return rc;
  }
  for (int q : ctx->singles) {
    int rc = do_stage(ctx, ctx->boxes[q], n);
    if (rc) return rc;
  }
  return CG_OK;
}

// Autotuner: for each untuned group, time the substep-1 launch (it rewrites
// only _f, the substep-2 input and its flux primitives, so repeating it
// changes nothing) for both launch orders and for one CTA per brick or a
// persistent grid of 1, 2 or 4 waves of resident CTAs, and the members' own
// launches one after another; keep the fastest.
int tune_groups(cg_ctx* ctx) {
  if (!ctx->opt_autotune) return CG_OK;
  int dev = 0, sms = 0;
  CG_CUDA(ctx, cudaGetDevice(&dev));
  CG_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  cudaEvent_t e0, e1;
  CG_CUDA(ctx, cudaEventCreate(&e0));
  cudaError_t ce = cudaEventCreate(&e1);
  if (ce != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_fail(ctx, ce, "cudaEventCreate");
  }
  int rc = CG_OK;
  for (Group& g : ctx->groups) {
    if (g.tuned) continue;
    bool ready = true;
    for (int q : g.members) ready = ready && ctx->boxes[q].stage_next == 1;
    if (!ready) continue;
    const int per_sm = g.mixed ? cg::mixed::group_ctas_per_sm(g.order, g.matter)
                               : cg::group_ctas_per_sm(g.variant, g.order, g.matter);
    float best = 1e30f;
    int best_lpt = 0, best_grid = 0;
    for (int lpt = 0; lpt < 2 && rc == CG_OK; ++lpt) {
      g.lpt = lpt;
      rc = write_table(ctx, g);
      for (int waves : {-1, 0, 1, 2, 4}) {
        if (rc) break;
        if (waves < 0 && lpt) continue;  // own launches: the order does not matter
        const int grid = waves < 0 ? -1 : waves * sms * per_sm;
        if (waves > 0 && grid >= g.total) continue;
        g.grid = grid;
        float ms = 0.0f;
        for (int rep = 0; rep < 4 && rc == CG_OK; ++rep) {
          std::vector<Box> trial = ctx->boxes;  // the trial's host bookkeeping is discarded
          if (rep == 1) cudaEventRecord(e0, ctx->stream);
          rc = group_launch(ctx, g, trial, 1);
        }
        if (rc) break;
        cudaEventRecord(e1, ctx->stream);
        ce = cudaEventSynchronize(e1);
        if (ce != cudaSuccess) {
          rc = cuda_fail(ctx, ce, "autotune");
          break;
        }
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
          best = ms;
          best_lpt = lpt;
          best_grid = grid;
        }
      }
    }
    if (rc) break;
    g.lpt = best_lpt;
    g.grid = best_grid;
    rc = write_table(ctx, g);
    if (rc) break;
    g.tuned = true;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

// nsteps whole steps recorded as one CUDA graph and replayed; the executable
// graph is kept and updated in place while the launch sequence keeps its shape.
int graph_steps(cg_ctx* ctx, int nsteps) {
  cudaError_t e = cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    // e.g. the legacy default stream: run the launches directly
    cudaGetLastError();
    for (int s = 0; s < nsteps; ++s)
      for (int n = 1; n <= 4; ++n) {
        int rc = all_stage(ctx, n);
        if (rc) return rc;
      }
    return CG_OK;
  }
  int rc = CG_OK;
  for (int s = 0; s < nsteps && rc == CG_OK; ++s)
    for (int n = 1; n <= 4 && rc == CG_OK; ++n) rc = all_stage(ctx, n);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(ctx->stream, &graph);
  if (rc) {
    if (graph) cudaGraphDestroy(graph);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
  bool updated = false;
  if (ctx->gexec && ctx->gexec_steps == nsteps) {
    cudaGraphExecUpdateResultInfo info{};
    updated = cudaGraphExecUpdate(ctx->gexec, graph, &info) == cudaSuccess;
    if (!updated) cudaGetLastError();
  }
  if (!updated) {
    if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
    ctx->gexec = nullptr;
    e = cudaGraphInstantiate(&ctx->gexec, graph, 0);
    if (e != cudaSuccess) {
      ctx->gexec = nullptr;
      cudaGraphDestroy(graph);
      return cuda_fail(ctx, e, "cudaGraphInstantiate");
    }
    ctx->gexec_steps = nsteps;
  }
  cudaGraphDestroy(graph);
  CG_CUDA(ctx, cudaGraphLaunch(ctx->gexec, ctx->stream));
  return CG_OK;
}

}  // namespace
extern "C" {
int cg_step_init(cg_ctx* ctx) {
  if (!ctx) return CG_ERR_INVALID;
  for (Box& b : ctx->boxes) {
    int rc = do_init(ctx, b);
    if (rc) return rc;
  }
  return CG_OK;
}

int cg_rk_stage(cg_ctx* ctx, int n) {
  if (!ctx) return CG_ERR_INVALID;
  if (n < 1 || n > 4) return fail(ctx, CG_ERR_INVALID, "substep must be 1..4");
  for (Box& b : ctx->boxes)
    if (b.stage_next != n)
      return fail(ctx, CG_ERR_STATE, "substep " + std::to_string(n) + " called out of order (expected " +
                                          std::to_string(b.stage_next) + ")");
  int rc = ensure_groups(ctx);
  if (rc) return rc;
  if (n == 1) {
    rc = tune_groups(ctx);
    if (rc) return rc;
  }
  return all_stage(ctx, n);
}

int cg_step(cg_ctx* ctx, int nsteps) {
  if (!ctx) return CG_ERR_INVALID;
  if (nsteps < 0) return fail(ctx, CG_ERR_INVALID, "nsteps must be >= 0");
  for (Box& b : ctx->boxes) {
    if (b.stage_next > 1) return fail(ctx, CG_ERR_STATE, "a step is in progress; finish it with cg_rk_stage");
    if (b.desc.x_ghost != 0)
      return fail(ctx, CG_ERR_STATE,
                  "x-slab boxes step through cg_step_init / cg_rk_stage with a halo exchange before every substep");
  }
  if (nsteps == 0) return CG_OK;
  for (Box& b : ctx->boxes)
    if (b.stage_next == 0) {
      int rc = do_init(ctx, b);
      if (rc) return rc;
    }
  int rc = ensure_groups(ctx);
  if (rc) return rc;
  rc = tune_groups(ctx);
  if (rc) return rc;
  if (ctx->opt_graph) return graph_steps(ctx, nsteps);
  for (int s = 0; s < nsteps; ++s)
    for (int n = 1; n <= 4; ++n) {
      rc = all_stage(ctx, n);
      if (rc) return rc;
    }
  return CG_OK;
}

int cg_ic_grf_dust(cg_ctx* ctx, int box, const double* delta, uint64_t seed, double rms_delta, double ns,
                   double cutoff) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  Box& b = ctx->boxes[box];
  if (b.desc.matter != CG_MATTER_DUST) return fail(ctx, CG_ERR_INVALID, "GRF dust initial data need a dust box");
  if (!(rms_delta >= 0.0) || !std::isfinite(ns)) return fail(ctx, CG_ERR_INVALID, "rms_delta >= 0 and finite ns");
  for (Box& o : ctx->boxes)
    if (o.stage_next > 1) return fail(ctx, CG_ERR_STATE, "initial data are set between steps");
  const cg::GridSpec gs{b.desc.nx, b.desc.ny, b.desc.nz, b.desc.stencil_order, b.desc.dx};
  const double kc = cutoff > 0.0 ? cutoff : std::min({gs.nx, gs.ny, gs.nz}) / 4.0;
  double* scratch = nullptr;
  CG_CUDA(ctx, cudaMalloc(&scratch, sizeof(double) * cg::ics::grf_scratch_doubles(gs)));
  std::string err;
  rc = cg::ics::grf_dust(gs, b.dev.P, scratch, delta, seed, rms_delta, ns, kc, b.desc.lambda, ctx->stream, err);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(scratch);
  if (rc) return fail(ctx, rc, "GRF initial data: " + err);
  b.stage_next = 0;
  b.steps = 0;
  return CG_OK;
}

int cg_ic_grf_scalar(cg_ctx* ctx, int box, const double* dphi, uint64_t seed, double phi0, double rms,
                     double mass, double cutoff) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  Box& b = ctx->boxes[box];
  if (b.desc.matter != CG_MATTER_SCALAR) return fail(ctx, CG_ERR_INVALID, "GRF scalar initial data need a scalar box");
  if (!(rms >= 0.0) || !std::isfinite(phi0) || !std::isfinite(mass))
    return fail(ctx, CG_ERR_INVALID, "rms >= 0, finite phi0 and mass");
  for (Box& o : ctx->boxes)
    if (o.stage_next > 1) return fail(ctx, CG_ERR_STATE, "initial data are set between steps");
  const cg::GridSpec gs{b.desc.nx, b.desc.ny, b.desc.nz, b.desc.stencil_order, b.desc.dx};
  const double kc = cutoff > 0.0 ? cutoff : std::min({gs.nx, gs.ny, gs.nz}) / 4.0;
  if (b.dev.nfields > cg_num_fields(CG_MATTER_SCALAR))  // Z4c's theta and the shift fields start at zero
    CG_CUDA(ctx, cudaMemsetAsync(b.dev.P, 0, sizeof(double) * (size_t)b.dev.nfields * b.dev.pts, ctx->stream));
  double* scratch = nullptr;
  CG_CUDA(ctx, cudaMalloc(&scratch, sizeof(double) * cg::ics::grf_scratch_doubles(gs)));
  std::string err;
  rc = cg::ics::grf_scalar(gs, b.dev.P, scratch, dphi, seed, rms, phi0, mass, kc, ctx->stream, err);
  cudaStreamSynchronize(ctx->stream);
  cudaFree(scratch);
  if (rc) return fail(ctx, rc, "GRF scalar initial data: " + err);
  b.stage_next = 0;
  b.steps = 0;
  return CG_OK;
}

int cg_set_option(cg_ctx* ctx, int option, int value) {
  if (!ctx) return CG_ERR_INVALID;
  switch (option) {
    case CG_OPT_BATCH:
      if (ctx->opt_batch != (value != 0)) {
        for (Box& b : ctx->boxes)
          if (b.stage_next > 1) return fail(ctx, CG_ERR_STATE, "change CG_OPT_BATCH between steps");
        ctx->opt_batch = value != 0;
        ctx->grouped = false;
      }
      return CG_OK;
    case CG_OPT_TMA_WAIT:
      for (Box& b : ctx->boxes)
        if (b.stage_next > 1) return fail(ctx, CG_ERR_STATE, "change CG_OPT_TMA_WAIT between steps");
      if (value < 0) return fail(ctx, CG_ERR_INVALID, "CG_OPT_TMA_WAIT takes a cycle count >= 0");
      for (Box& b : ctx->boxes) b.dev.ph.tma_wait = value > 0 ? (long long)value : kTmaWaitDefault;
      ctx->grouped = false;  // the group tables carry the boxes' parameters
      return CG_OK;
    case CG_OPT_TMA:
      for (Box& b : ctx->boxes)
        if (b.stage_next > 1) return fail(ctx, CG_ERR_STATE, "change CG_OPT_TMA between steps");
      ctx->opt_tma = value != 0;
      for (Box& b : ctx->boxes) {
        if (b.mixed) b.mdev.tma = b.mdev.maps && ctx->opt_tma;
        else b.dev.tma = b.dev.maps && ctx->opt_tma;
      }
      ctx->grouped = false;  // the group tables carry the flag
      return CG_OK;
    case CG_OPT_GRAPH: ctx->opt_graph = value != 0; return CG_OK;
    case CG_OPT_AUTOTUNE: ctx->opt_autotune = value != 0; return CG_OK;
    case CG_OPT_GROUP_GRID:
      if (value < -1) return fail(ctx, CG_ERR_INVALID, "CG_OPT_GROUP_GRID must be >= -1");
      ctx->opt_group_grid = value;
      for (Group& g : ctx->groups)
        if (!g.tuned) g.grid = value;
      return CG_OK;
    default: return fail(ctx, CG_ERR_INVALID, "unknown option");
  }
}

int cg_num_groups(cg_ctx* ctx, int* n) {
  if (!ctx || !n) return CG_ERR_INVALID;
  int rc = ensure_groups(ctx);
  if (rc) return rc;
  *n = (int)ctx->groups.size();
  return CG_OK;
}

int cg_group_info(cg_ctx* ctx, int group, int* info, int n) {
  if (!ctx) return CG_ERR_INVALID;
  if (!info || n < 6) return fail(ctx, CG_ERR_INVALID, "info needs 6 entries");
  int rc = ensure_groups(ctx);
  if (rc) return rc;
  if (group < 0 || group >= (int)ctx->groups.size()) return fail(ctx, CG_ERR_INVALID, "group index out of range");
  const Group& g = ctx->groups[group];
  info[0] = (int)g.members.size();
  info[1] = g.total;
  info[2] = g.grid;
  info[3] = g.lpt;
  info[4] = g.tuned ? 1 : 0;
  info[5] = g.members.empty() ? -1 : g.members[0];
  return CG_OK;
}

int cg_status(cg_ctx* ctx, uint32_t* flags) {
  if (!ctx || !flags) return CG_ERR_INVALID;
  unsigned h = 0;
  CG_CUDA(ctx, cudaMemcpyAsync(&h, ctx->status, sizeof(unsigned), cudaMemcpyDeviceToHost, ctx->stream));
  CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  *flags = h;
  return CG_OK;
}

int cg_synchronize(cg_ctx* ctx) {
  uint32_t f = 0;
  int rc = cg_status(ctx, &f);
  if (!rc && ctx->copy_stream) CG_CUDA(ctx, cudaStreamSynchronize(ctx->copy_stream));  // staged downloads
  if (rc) return rc;
  if (f & CG_STATUS_TILE_TIMEOUT) return fail(ctx, CG_ERR_CUDA, "a TMA tile copy timed out");
  if (f & CG_STATUS_NAN) return fail(ctx, CG_ERR_NAN, "NaN detected in DIFFphi");
  return CG_OK;
}

int cg_frw_state(cg_ctx* ctx, int box, double* out, int n) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  const Box& b = ctx->boxes[box];
  if (!out || n < 2 + b.frw.n) return fail(ctx, CG_ERR_INVALID, "out needs 2 + nfluids entries");
  out[0] = b.frw.phi;
  out[1] = b.frw.K;
  for (int m = 0; m < b.frw.n; ++m) out[2 + m] = b.frw.rho[m];
  return CG_OK;
}

int cg_step_count(cg_ctx* ctx, int box, int64_t* steps) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  if (!steps) return fail(ctx, CG_ERR_INVALID, "steps is null");
  *steps = ctx->boxes[box].steps;
  return CG_OK;
}

// Scratch layout of the constraint pass (cscratch_doubles): cvals (12 n) |
// part1 (27 nblk1) | part2 (10 nblk2) | r1 (27) | r2 (10) | wpart (9 nblk2) | wres (9)
struct CScratch {
  double *cvals, *part1, *part2, *r1, *r2, *wpart, *wres;
  int n, nblk1, nblk2;
  int off, nin;  // the points the kernels update: from index off, nin of them (x-slabs skip ghost planes)
};

static CScratch cscratch_layout(const Box& b) {
  CScratch c{};
  c.n = b.dev.pts;
  c.nblk1 = cg::exact::constraint_blocks(b.dev);
  c.nblk2 = std::min(1024, (c.n + 255) / 256);
  c.cvals = b.cscratch;
  c.part1 = c.cvals + (size_t)12 * c.n;
  c.part2 = c.part1 + (size_t)27 * c.nblk1;
  c.r1 = c.part2 + (size_t)10 * c.nblk2;
  c.r2 = c.r1 + 27;
  c.wpart = c.r2 + 10;
  c.wres = c.wpart + (size_t)9 * c.nblk2;
  c.off = b.dev.xg * b.dev.ny * b.dev.nz;
  c.nin = (b.dev.nx - 2 * b.dev.xg) * b.dev.ny * b.dev.nz;
  return c;
}

// The constraint pass (BSSN::setConstraintCalcs, bssn.cc:965-1071) on the
// box's state between steps: per-point values and both reduction passes, on
// the context's stream.  dev gets the FP64 first-substep input; for a mixed
// box it is built in *xtmp, which the caller frees after the last use.
static int constraint_pass(cg_ctx* ctx, Box& b, cg::BoxDev& dev, double** xtmp) {
  *xtmp = nullptr;
  if (b.mixed && b.desc.x_ghost != 0)
    return fail(ctx, CG_ERR_INVALID, "constraints of an FP32-mixed x-slab would read stale ghost planes of _p");
  if (b.stage_next > 1) return fail(ctx, CG_ERR_STATE, "constraints are taken between steps");
  if (b.stage_next == 0) {
    const int rc = do_init(ctx, b);
    if (rc) return rc;
  }
  const int n = b.dev.pts;
  if (!b.cscratch) CG_CUDA(ctx, cudaMalloc(&b.cscratch, sizeof(double) * cscratch_doubles(b)));
  dev = b.dev;
  if (b.mixed) {
    // FP64 first-substep input of the current _p for the FP64 constraint pass
    const size_t nx64 = (size_t)b.dev.nfields * n + (size_t)cg::P_N * n;
    CG_CUDA(ctx, cudaMalloc(xtmp, sizeof(double) * nx64));
    dev.X = *xtmp;
    dev.FP0 = *xtmp + (size_t)b.dev.nfields * n;
    StageBg bg0 = bg_for(b, 1, b.frw.get_phi);
    cudaError_t ei = cg::launch_init(cg::kExact, dev, bg0, ctx->stream);
    if (ei != cudaSuccess) return cuda_fail(ctx, ei, "init");
  }
  const CScratch c = cscratch_layout(b);
  StageBg bg = bg_for(b, 1, b.frw.get_phi);
  cudaError_t ec = cg::exact::launch_constraints(dev, bg, c.cvals, c.part1, ctx->stream);
  if (ec != cudaSuccess) return cuda_fail(ctx, ec, "constraints");
  part_final_kernel<<<1, 256, 0, ctx->stream>>>(c.part1, c.nblk1, 27, 17, c.r1);
  constraint_stdev_kernel<<<c.nblk2, 256, 0, ctx->stream>>>(c.cvals, (size_t)n, c.off, c.nin, c.r1, c.part2);
  part_final_kernel<<<1, 256, 0, ctx->stream>>>(c.part2, c.nblk2, 10, 10, c.r2);
  CG_CUDA(ctx, cudaGetLastError());
  return CG_OK;
}

int cg_constraints(cg_ctx* ctx, int box, double* H, double* M, double* G, double* A, double* S) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  if (!H || !M || !G || !A || !S) return fail(ctx, CG_ERR_INVALID, "null output array");
  Box& b = ctx->boxes[box];
  cg::BoxDev dev{};
  double* xtmp = nullptr;
  rc = constraint_pass(ctx, b, dev, &xtmp);
  if (rc) {
    cudaFree(xtmp);
    return rc;
  }
  const CScratch c = cscratch_layout(b);
  const int n = c.nin;  // statistics over the updated points
  double h1[27], h2[10];
  CG_CUDA(ctx, cudaMemcpyAsync(h1, c.r1, sizeof(h1), cudaMemcpyDeviceToHost, ctx->stream));
  CG_CUDA(ctx, cudaMemcpyAsync(h2, c.r2, sizeof(h2), cudaMemcpyDeviceToHost, ctx->stream));
  CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(xtmp);
  // BSSN_NORMALIZE_MEAN / _STDEV and BSSN_STORE_CONSTRAINT_STAT_VARS (bssn_macros.h:539-560)
  double* outs[5] = {H, M, G, A, S};
  for (int k = 0; k < 5; ++k) {
    double* o = outs[k];
    o[0] = h1[k] / n;
    o[1] = std::sqrt(h2[2 * k] / (n - 1.0));
    o[2] = h1[17 + k];
    o[3] = h1[5 + k];
    o[4] = h1[10 + k] / n;
    o[5] = std::sqrt(h2[2 * k + 1] / (n - 1.0));
    o[6] = h1[22 + k];
  }
  H[7] = std::sqrt(h1[15]);
  M[7] = std::sqrt(h1[16]);
  return CG_OK;
}

int cg_field_statistics(cg_ctx* ctx, int box, double* out, int n_out) {
  int rc = check_box(ctx, box);
  if (rc) return rc;
  if (!out || n_out < 9) return fail(ctx, CG_ERR_INVALID, "out needs 9 entries");
  Box& b = ctx->boxes[box];
  cg::BoxDev dev{};
  double* xtmp = nullptr;
  rc = constraint_pass(ctx, b, dev, &xtmp);  // ricci_a and DIFFr_a per point
  if (rc) {
    cudaFree(xtmp);
    return rc;
  }
  const CScratch c = cscratch_layout(b);
  const int N = c.n, n = c.nin;  // statistics over the updated points
  const double* phi = dev.X + (size_t)cg::F_PHI * N + c.off;
  const double* K = dev.X + (size_t)cg::F_K * N + c.off;
  const double* ricci = c.cvals + (size_t)10 * N + c.off;
  const double* rho = c.cvals + (size_t)11 * N + c.off;
  const double phi_frw = b.frw.get_phi;
  wstats_sum_kernel<<<c.nblk2, 256, 0, ctx->stream>>>(phi, K, rho, ricci, phi, n, phi_frw, c.wpart);
  part_final_kernel<<<1, 256, 0, ctx->stream>>>(c.wpart, c.nblk2, 5, 5, c.wres);
  wstats_var_kernel<<<c.nblk2, 256, 0, ctx->stream>>>(phi, K, rho, ricci, phi, n, phi_frw, c.wres,
                                                      c.wpart + (size_t)5 * c.nblk2);
  part_final_kernel<<<1, 256, 0, ctx->stream>>>(c.wpart + (size_t)5 * c.nblk2, c.nblk2, 4, 4, c.wres + 5);
  cudaError_t e = cudaGetLastError();
  double h[9];
  if (e == cudaSuccess) e = cudaMemcpyAsync(h, c.wres, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  cudaFree(xtmp);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "field statistics");
  // DETAILS(field) for DIFFphi, DIFFK, DIFFr, ricci, then the volume average
  const double vol = h[4] / n;
  for (int m = 0; m < 4; ++m) {
    out[2 * m] = h[m] / n / vol;
    out[2 * m + 1] = std::sqrt(h[5 + m] / (n - 1.0) / vol);
  }
  out[8] = vol;
  return CG_OK;
}

int cg_conformal_average(cg_ctx* ctx, const double* d_field, const double* d_phi, size_t n, double phi_frw,
                         double* out) {
  if (!ctx) return CG_ERR_INVALID;
  if (!d_field || !d_phi || !out) return fail(ctx, CG_ERR_INVALID, "null pointer");
  if (n == 0 || n > (size_t)INT32_MAX) return fail(ctx, CG_ERR_INVALID, "n must be in 1..2^31-1");
  const int nblk = (int)std::min<size_t>(1024, (n + 255) / 256);
  if (ctx->red_blocks < nblk) {
    cudaFree(ctx->red);
    ctx->red = nullptr;
    ctx->red_blocks = 0;
    CG_CUDA(ctx, cudaMalloc(&ctx->red, sizeof(double) * (2 * 1024 + 1)));
    ctx->red_blocks = 1024;
  }
  double* res = ctx->red + 2 * 1024;
  CG_CUDA(ctx, cg::launch_conformal_average(d_field, d_phi, (int)n, phi_frw, ctx->red, nblk, res, ctx->stream));
  CG_CUDA(ctx, cudaMemcpyAsync(out, res, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  CG_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return CG_OK;
}

const char* cg_last_error(cg_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

}  // extern "C"
