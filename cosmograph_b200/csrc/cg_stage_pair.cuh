// cg_stage_pair.cuh -- the fused FP64 substep with two threads per grid point.
//
// The same substep as stage_body (cg_stage.cuh): every value is computed by
// the same expression in the same operand order, so results are identical
// bit for bit.  What changes is who computes it: a CTA of 256 threads owns
// the 4x2x16 brick, and each point has two threads in different warps --
// half A (threads 0-127) and half B (threads 128-255), thread t and t + 128
// on the same point, sharing that point's column of the shared-memory slot
// array.  The register and slot needs of one point are the same as before,
// so twice the warps fit on an SM (16 instead of 8) in the same shared
// memory; each thread carries about half the work.
//
// Work split (all CTA-wide barriers, reached by every thread):
//   phase 1, per stencil field: A the first and the diagonal second
//     derivatives, B the mixed second derivatives (for the metric, B parks
//     them in exchange slots and A contracts them with g^kl one field later);
//     first-derivative-only fields: A the x and y derivatives, B z;
//     dust flux divergences: A alpha*D and alpha*S_1, B alpha*S_2, alpha*S_3.
//   2.1  A: matter sources (and the matter right-hand sides); B: Gamma^I_jk.
//   2.2  A: lowered Gamma_{I,jk}; B: D_iD_j phi, (D_iD_j alpha)^TF and its trace.
//   2.3  Ricci R_ij: A the components 11, 12, 13, B 22, 23, 33.
//   2.4  A: gamma_ij, phi, K, alpha, matter fields; B: A_ij, Gamma^i
//        (right-hand side, Kreiss-Oliger term, register update); both form
//        the scalars they share (Gamma^I contraction, A^ij, R, H).
//   2.5  last substep: B hands its A_ij to A, which normalises gamma and A
//        (the next step's input) and forms the dust flux primitives.
// Included by cg_stage.cuh inside namespace cg::CG_VARIANT_NS.
#pragma once

constexpr int kPairThreads = 2 * kThreads;
// thread/row mapping of the tile copies when all 256 threads copy
struct PairCopy {
  static constexpr int THREADS = kPairThreads, WARPS = kPairThreads / 32;
};
// phase 1: B's mixed second derivatives of metric field q, for A's
// contraction one field later, in two sets of three (q even, q odd); they
// lie in the first tile buffer's region, past the tile and its row offsets
constexpr int kXch = S_MAT - 6;
// phase 2: one more slot after the matter slots, (D_i D_j alpha) trace from B to A
template <int MATTER>
struct PairSlots {
  static constexpr int xdda = Slots<MATTER>::value;
  static constexpr int value = xdda + 1;
};
template <int O, int MATTER>
constexpr size_t pair_smem() {
  return sizeof(double) * kThreads * PairSlots<MATTER>::value +
         (TileBuffers<O, MATTER, kEvolve>::kTwo ? TileBuffers<O, MATTER, kEvolve>::kBytes : 0);
}
static_assert(2 * (pair_smem<8, kDust>() + 2048) <= 228 * 1024, "two dust CTAs of the pair kernel fit on an SM");

// the half that finalises field f: B the A_ij and Gamma^i, A the rest
__host__ __device__ constexpr int pair_owner(int f) {
  return (f >= F_A11 && f <= F_A33) || (f >= F_GAM1 && f <= F_GAM3) ? 1 : 0;
}

// the derivatives of phase-1 field `it` that half h computes (see above);
// hd: A's diagonal second derivatives of the current metric field, kept for
// its contraction at the next field
template <int O, int MATTER>
__device__ __forceinline__ void pair_field_derivatives(int it, const tile::Taps<TileG<O>, double>& t, const Physics& ph,
                                                       double* sl, int h, double (&hd)[3]) {
  auto X = [&](int s) -> double& { return sl[s * kThreads]; };
  if (it < 8) {
    // calculate_dgamma / calculate_ddgamma / calculate_dalpha_dphi (bssn.cc:480-521)
    const int q = it;
    if (h == 0) {
      const double g1 = d1<O>(t, 0, ph), g2 = d1<O>(t, 1, ph), g3 = d1<O>(t, 2, ph);
      const double h11 = d2<O>(t, 0, ph), h22 = d2<O>(t, 1, ph), h33 = d2<O>(t, 2, ph);
      if (q < 6) {
        X(S_DG + 0 * 6 + q) = g1;
        X(S_DG + 1 * 6 + q) = g2;
        X(S_DG + 2 * 6 + q) = g3;
        hd[0] = h11;
        hd[1] = h22;
        hd[2] = h33;
      } else {
        const int b1 = q == 6 ? S_DPHI : S_DA, b2 = q == 6 ? S_DDPHI : S_DDA;
        X(b1 + 0) = g1;
        X(b1 + 1) = g2;
        X(b1 + 2) = g3;
        X(b2 + 0) = h11;
        X(b2 + 3) = h22;
        X(b2 + 5) = h33;
      }
    } else {
      const double h12 = dm<O>(t, 0, 1, ph), h13 = dm<O>(t, 0, 2, ph), h23 = dm<O>(t, 1, 2, ph);
      if (q < 6) {
        X(kXch + 3 * (q & 1) + 0) = h12;
        X(kXch + 3 * (q & 1) + 1) = h13;
        X(kXch + 3 * (q & 1) + 2) = h23;
      } else {
        const int b2 = q == 6 ? S_DDPHI : S_DDA;
        X(b2 + 1) = h12;
        X(b2 + 2) = h13;
        X(b2 + 4) = h23;
      }
    }
  } else {
    // K, Gamma^K (calculate_dK, bssn.cc:529-535; d_J Gamma^K of
    // BSSN_CALCULATE_RICCI_UNITARY_TERM2) and the scalar fields
    // (scalar.cc:109-127): first derivatives
    const int q = it - 8;
    const int b = q < 4 ? (q == 0 ? S_DK : S_DGAM + 3 * (q - 1)) : S_MAT + 3 * (q - 4);
    if (h == 0) {
      X(b + 0) = d1<O>(t, 0, ph);
      X(b + 1) = d1<O>(t, 1, ph);
    } else {
      X(b + 2) = d1<O>(t, 2, ph);
    }
  }
}

// Phase 1 of the pair kernel: the copies of `derivatives` (cg_stage.cuh) by
// all 256 threads, the derivatives split between the halves.
template <int O, int MATTER>
__device__ __forceinline__ bool pair_derivatives(const double* __restrict__ a, int N, const Physics& ph,
                                                 const double gi[6], double* sl, double* tl, double* tl2,
                                                 const int* rowoff, int tid, int h, int x0, int y0, int z0, int nz,
                                                 int cc, const CUtensorMap* tmap, uint64_t* bar, unsigned& phase) {
  using PF = Phase1<MATTER, kEvolve>;
  using G = TileG<O>;
  constexpr bool TWO = TileBuffers<O, MATTER, kEvolve>::kTwo;
  constexpr unsigned kBytes = (unsigned)(G::SIZE * sizeof(double));
  static_assert(G::SIZE * sizeof(double) + G::ROWS * sizeof(int) <= (size_t)(kXch - kTileSlot) * kThreads * sizeof(double),
                "the exchange slots lie past the tile and its row offsets");
  auto issue = [&](int it) {
    const int b = TWO ? (it & 1) : 0;
    tma::arrive_expect_tx(bar + b, kBytes);
    tma::load_4d(b ? tl2 : tl, tmap, z0 - G::ZO, y0 - G::R, x0 - G::R, PF::field(it), bar + b);
    if (it + 1 < PF::N) tma::prefetch_4d(tmap, z0 - G::ZO, y0 - G::R, x0 - G::R, PF::field(it + 1));
  };
  auto X = [&](int s) -> double& { return sl[s * kThreads]; };
  const bool by_tma = tmap != nullptr;
  bool ok = true;
  tile::Loader<G, PairCopy, double> ld;
  tile::AsyncLoader<G, PairCopy> ald;
  if (by_tma) {
    if (TWO) {
      tma::fence_proxy_async();
      __syncthreads();
      if (tid == 0) issue(0);
    }
  } else if (TWO) {
    ald.init(tid, z0, nz);
    ald.issue(tl, a + (size_t)PF::field(0) * N, rowoff);
  } else {
    ld.init(tid, z0, nz);
    ld.fetch(a + (size_t)PF::field(0) * N, rowoff);
  }
  double hd[3] = {0.0, 0.0, 0.0};
#pragma unroll 1
  for (int it = 0; it < PF::N; ++it) {
    int b = 0;
    if (by_tma) {
      tma::fence_proxy_async();
      __syncthreads();  // the buffer the next copy writes has been read
      if (tid == 0) {
        if (!TWO) issue(it);
        else if (it + 1 < PF::N) issue(it + 1);
      }
      b = TWO ? (it & 1) : 0;
      if (ok && !tma::wait(bar + b, (phase >> b) & 1u, kTmaWaitCycles64)) ok = false;
      phase ^= 1u << b;
    } else if (TWO) {
      __syncthreads();
      if (it + 1 < PF::N) {
        ald.issue((it + 1) & 1 ? tl2 : tl, a + (size_t)PF::field(it + 1) * N, rowoff);
        tile::cp_async_wait<1>();
      } else {
        tile::cp_async_wait<0>();
      }
      __syncthreads();
      b = it & 1;
    } else {
      __syncthreads();
      ld.store(tl);
      __syncthreads();
      if (it + 1 < PF::N) ld.fetch(a + (size_t)PF::field(it + 1) * N, rowoff);
    }
    if (h == 0 && it >= 1 && it <= 6) {
      // g^{kl} d_k d_l of metric field it - 1, with B's mixed derivatives
      // (BSSN_CALCULATE_RICCI_UNITARY_TERM1, bssn_macros.h:248-249, summed
      // over (k,l) in the reference's order)
      const int q = it - 1;
      const double h12 = X(kXch + 3 * (q & 1) + 0), h13 = X(kXch + 3 * (q & 1) + 1), h23 = X(kXch + 3 * (q & 1) + 2);
      double s = gi[0] * hd[0];
      s = s + gi[1] * h12;
      s = s + gi[2] * h13;
      s = s + gi[1] * h12;
      s = s + gi[3] * hd[1];
      s = s + gi[4] * h23;
      s = s + gi[2] * h13;
      s = s + gi[4] * h23;
      s = s + gi[5] * hd[2];
      X(S_T1 + q) = s;
    }
    pair_field_derivatives<O, MATTER>(it, tile::Taps<G, double>{b ? tl2 : tl, cc}, ph, sl, h, hd);
  }
  if (by_tma) ok = __syncthreads_and(ok);
  return ok;
}

// One brick, two threads per point.  Arguments as stage_body's.
template <int O, int MATTER, bool KO>
__device__ __forceinline__ void pair_stage_body(const BoxGeom& geo, const Physics& ph, StageBg bg, const StagePtrs& P,
                                                int stage, int cx, int cy, int cz, const CUtensorMap* tmap,
                                                uint64_t* bar, unsigned& phase, bool& tma_ok,
                                                const FluxMaps* fmaps) {
  constexpr int NFLD = NF<MATTER>::value;
  constexpr int NSLOT = PairSlots<MATTER>::value;
  constexpr int XDDA = PairSlots<MATTER>::xdda;
  constexpr int R = O / 2;
  extern __shared__ __align__(128) double smem[];
  const int tid = threadIdx.x;
  const int h = tid >> 7;             // 0: half A, 1: half B (uniform in a warp)
  const int pt = tid & (kThreads - 1);
  const int tz = pt % kBZ, ty = (pt / kBZ) % kBY, tx = pt / (kBZ * kBY);
  double* sl = smem + pt;  // this point's slot column
  auto S = [&](int s) -> double& { return sl[s * kThreads]; };

  const int k0 = cz * kBZ + tz, j0 = cy * kBY + ty, i0 = cx * kBX + tx;
  const bool live = i0 < geo.nx && j0 < geo.ny && k0 < geo.nz;
  // threads past the box edge compute a valid point, write nothing, and
  // take part in every barrier
  const int k = min(k0, geo.nz - 1), j = min(j0, geo.ny - 1), i = min(i0, geo.nx - 1);
  if (P.kavg) bg.K_avg = *P.kavg;
  const int N = geo.pts;
  const int c = (i * geo.ny + j) * geo.nz + k;
  const double* __restrict__ a = P.in;
  auto C = [&](int f) { return a[(size_t)f * N + c]; };
#pragma unroll 1
  for (int f = 0; f < NFLD; ++f) {
    if (pair_owner(f) != h) continue;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(P.p + (size_t)f * N + c));
    if (stage > 1) asm volatile("prefetch.global.L2 [%0];" ::"l"(P.f + (size_t)f * N + c));
  }

  // ---- centre values (set_local_vals, bssn.cc:430-435) ----------------------
  double g[6], gi[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) g[q] = C(F_G11 + q);
  inv_metric(g, gi);

  // ---- phase 1 ------------------------------------------------------------------
  const int x0 = cx * kBX, y0 = cy * kBY, z0 = cz * kBZ;
  bool flux_tiles = false;
  {
    using G = TileG<O>;
    double* tl = smem + kTileSlot * kThreads;
    int* rowoff = reinterpret_cast<int*>(tl + G::SIZE);
    const bool by_tma = tmap && tma_ok && x0 >= G::R && x0 + kBX + G::R <= geo.nx && y0 >= G::R &&
                        y0 + kBY + G::R <= geo.ny && z0 >= G::ZO && z0 + kBZ + G::R <= geo.nz;
    if (!by_tma) {
      tile::row_offsets<G, PairCopy>(x0, y0, geo.nx, geo.ny, geo.nz, tid, rowoff);
      __syncthreads();
    }
    double* tl2 = TileBuffers<O, MATTER, kEvolve>::kTwo ? smem + NSLOT * kThreads : nullptr;
    const bool ok = pair_derivatives<O, MATTER>(a, N, ph, gi, sl, tl, tl2, rowoff, tid, h, x0, y0, z0, geo.nz,
                                                tile::centre<G>(tx, ty, tz), by_tma ? tmap : nullptr, bar, phase);
    if (by_tma && !ok && tid == 0) atomicOr(P.status, kStatusTileTimeout64);
    tma_ok = ok && tma_ok;
    if constexpr (MATTER == kDust && TileBuffers<O, MATTER, kEvolve>::kTwo) {
      flux_tiles = fmaps && by_tma && tma_ok;
      if (flux_tiles) {
        tma_ok = flux_from_tiles<O>(fmaps, tl, tl2, tid, x0, y0, z0, ph, sl, bar, phase, tx, ty, tz, 2 * h, 2 * h + 2);
        if (!tma_ok && tid == 0) atomicOr(P.status, kStatusTileTimeout64);
      }
    }
    __syncthreads();  // the tile region becomes slots again
  }
  if (MATTER == kDust && !flux_tiles) {
    const bool interior =
        x0 >= R && x0 + kBX + R <= geo.nx && y0 >= R && y0 + kBY + R <= geo.ny && z0 >= R && z0 + kBZ + R <= geo.nz;
    if (interior)
      flux_divergences<O>(Taps<false>{i, j, k, geo.nx, geo.ny, geo.nz, geo.ny * geo.nz, geo.nz, c}, P.fp_in, N, ph,
                          sl, 2 * h, 2 * h + 2);
    else
      flux_divergences<O>(Taps<true>{i, j, k, geo.nx, geo.ny, geo.nz, geo.ny * geo.nz, geo.nz, c}, P.fp_in, N, ph,
                          sl, 2 * h, 2 * h + 2);
  }
  __syncthreads();  // every derivative of the point is in its slots

  // ---- phase 2: the algebra of set_bd_values (bssn.cc:361-421) ----------------
  const double phi = C(F_PHI) + bg.phi_FRW;
  const double Kd = C(F_K);
  const double K = Kd + bg.K_FRW;
  const double alphad = C(F_ALPHA);
  const double alpha = alphad + 1.0;
  double gm[6];
  gm[0] = g[0] + 1.0; gm[1] = g[1]; gm[2] = g[2];
  gm[3] = g[3] + 1.0; gm[4] = g[4]; gm[5] = g[5] + 1.0;
  // every e^x this point's substep takes, in one batch: of phi and, for dust
  // after the first substep, of the previous substep's phi (the lagged sources)
  double phip = phi;
  if (MATTER == kDust && stage > 1) phip = __ldcs(&P.prev[(size_t)F_PHI * N + c]) + bg.phi_FRW_prev;
  double ex[8];
  {
    const double xa[8] = {-4.0 * phi, 4.0 * phi, 6.0 * phi, 5.0 * phi, -5.0 * phi, -4.0 * phip, 4.0 * phip, 6.0 * phip};
    xexp_n<8>(xa, ex);
  }
  const double em4phi = ex[0], e4phi = ex[1], e6phi = ex[2], e5phi = ex[3], em5phi = ex[4];
  const double em4phip = ex[5], e4phip = ex[6], e6phip = ex[7];
  auto G = [&](int I, int qq) { return S(S_G + 6 * I + qq); };
  auto GL = [&](int I, int qq) { return S(S_DG + 6 * I + qq); };
  double dphi[3], da[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { dphi[d] = S(S_DPHI + d); da[d] = S(S_DA + d); }

  // -- 2.1: A the sources, B the Christoffel symbols --
  double rhs_m[5] = {0, 0, 0, 0, 0};
  if (h == 0) {
    if (MATTER == kDust) {
      const double D = C(F_D);
      const double Sv[3] = {C(F_S1), C(F_S2), C(F_S3)};
      double Wl, detgl, gph[6];
      if (stage == 1) {
        const DustPrim dp = dust_prim(gi, em4phi, e6phi, D, Sv);
        Wl = dp.W;
        const double e4 = e4phi;
        detgl = e6phi;
#pragma unroll
        for (int m = 0; m < 6; ++m) gph[m] = e4 * gm[m];
      } else {
        const double* pv = P.prev;
        double gp[6], gip[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) gp[m] = __ldcs(&pv[(size_t)(F_G11 + m) * N + c]);
        const double Dp = __ldcs(&pv[(size_t)F_D * N + c]);
        const double Sp[3] = {__ldcs(&pv[(size_t)F_S1 * N + c]), __ldcs(&pv[(size_t)F_S2 * N + c]),
                              __ldcs(&pv[(size_t)F_S3 * N + c])};
        inv_metric(gp, gip);
        const DustPrim dp = dust_prim(gip, em4phip, e6phip, Dp, Sp);
        Wl = dp.W;
        const double e4 = e4phip;
        detgl = e6phip;
        gph[0] = e4 * (gp[0] + 1.0); gph[1] = e4 * gp[1]; gph[2] = e4 * gp[2];
        gph[3] = e4 * (gp[3] + 1.0); gph[4] = e4 * gp[4]; gph[5] = e4 * (gp[5] + 1.0);
      }
      double q[Q_N];
      dust_sources(Wl, detgl, gph, D, Sv, ph.lambda, q);
#pragma unroll
      for (int m = 0; m < Q_N; ++m) S(S_SRC + m) = q[m];
      // momentum source S_m^src (dust.cc:135-146) with the current W, v
      const DustPrim cur = dust_prim(gi, em4phi, e6phi, D, Sv);
      const double e4 = e4phi;
      rhs_m[0] = S(S_MAT + 0);
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const double dp = S(S_DPHI + d);
        auto DG = [&](int qq) { return S(S_DG + 6 * d + qq); };
        const double src =
            1.0 / 2.0 * alpha * cur.W * D * e4 *
                (cur.v[0] * cur.v[0] * (4.0 * gm[0] * dp + DG(0)) + cur.v[1] * cur.v[1] * (4.0 * gm[3] * dp + DG(3)) +
                 cur.v[2] * cur.v[2] * (4.0 * gm[5] * dp + DG(5)) +
                 2.0 * (cur.v[0] * cur.v[1] * (4.0 * gm[1] * dp + DG(1)) + cur.v[0] * cur.v[2] * (4.0 * gm[2] * dp + DG(2)) +
                        cur.v[1] * cur.v[2] * (4.0 * gm[4] * dp + DG(4)))) -
            cur.W * D * S(S_DA + d);
        rhs_m[1 + d] = S(S_MAT + 1 + d) + src;
      }
    } else if (MATTER == kScalar) {
      // Scalar::addBSSNSource (scalar.cc:201-260) and RKEvolvePt (:85-199)
      const double sphi = C(F_SPHI), sPi = C(F_SPI);
      const double psi[3] = {C(F_SPSI1), C(F_SPSI1 + 1), C(F_SPSI1 + 2)};
      auto SD = [&](int m, int d) { return S(S_MAT + 3 * m + d); };
      const double nmu = ((-alpha * sPi)) / alpha;
      const double dd = (gi[0] * SD(0, 0) * SD(0, 0) + gi[3] * SD(0, 1) * SD(0, 1) + gi[5] * SD(0, 2) * SD(0, 2) +
                         2.0 * (gi[1] * SD(0, 0) * SD(0, 1) + gi[2] * SD(0, 0) * SD(0, 2) + gi[4] * SD(0, 1) * SD(0, 2)));
      const double V = pot_V(ph, sphi);
      S(S_SRC + Q_R) = 0.5 * nmu * nmu + 0.5 * em4phi * dd + V;
      S(S_SRC + Q_S) = 3.0 / 2.0 * nmu * nmu - 0.5 * em4phi * dd - 3.0 * V;
#pragma unroll
      for (int m = 0; m < 3; ++m) S(S_SRC + Q_S1 + m) = -nmu * SD(0, m);
#pragma unroll
      for (int I = 0; I < 3; ++I)
#pragma unroll
        for (int J = I; J < 3; ++J) S(S_SRC + Q_STF11 + sym(I, J)) = SD(0, I) * SD(0, J) - gm[sym(I, J)] / 3.0 * dd;
      double inner = 0.0;
#pragma unroll
      for (int X = 0; X < 3; ++X)
#pragma unroll
        for (int Y = 0; Y < 3; ++Y) {
          const double u = gi[sym(X, Y)] * (alpha * SD(2 + Y, X) + psi[X] * S(S_DA + Y));
          inner = (X == 0 && Y == 0) ? u : inner + u;
        }
      double gt[3];
#pragma unroll
      for (int I = 0; I < 3; ++I)
        gt[I] = (C(F_GAM1 + I) - 2.0 * (gi[sym(I, 0)] * S(S_DPHI + 0) + gi[sym(I, 1)] * S(S_DPHI + 1) +
                                        gi[sym(I, 2)] * S(S_DPHI + 2)));
      rhs_m[0] = (-alpha * sPi);
      rhs_m[1] = (-em4phi * (inner) +
                  alpha * ((gt[0]) * psi[0] * em4phi + (gt[1]) * psi[1] * em4phi + (gt[2]) * psi[2] * em4phi + K * sPi +
                           pot_dV(ph, sphi)));
#pragma unroll
      for (int m = 0; m < 3; ++m) rhs_m[2 + m] = (-alpha * SD(1, m) - sPi * S(S_DA + m));
    } else {
#pragma unroll
      for (int m = 0; m < Q_N; ++m) S(S_SRC + m) = 0.0;
    }
  } else {
    // Christoffels Gamma^I_q (bssn.cc:577-590, bssn_macros.h:221-229)
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = 0; J < 3; ++J)
#pragma unroll
        for (int Kx = J; Kx < 3; ++Kx) {
          auto dg = [&](int d, int qq) { return S(S_DG + 6 * d + qq); };
          double u = gi[sym(I, 0)] * (dg(J, sym(Kx, 0)) + dg(Kx, sym(J, 0)) - dg(0, sym(J, Kx)));
          u = u + gi[sym(I, 1)] * (dg(J, sym(Kx, 1)) + dg(Kx, sym(J, 1)) - dg(1, sym(J, Kx)));
          u = u + gi[sym(I, 2)] * (dg(J, sym(Kx, 2)) + dg(Kx, sym(J, 2)) - dg(2, sym(J, Kx)));
          S(S_G + 6 * I + sym(J, Kx)) = 0.5 * (u);
        }
  }
  __syncthreads();

  // -- 2.2: A the lowered symbols, B D_iD_j phi and (D_iD_j alpha)^TF --
  if (h == 0) {
    double GLv[3][6];
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = 0; J < 3; ++J)
#pragma unroll
        for (int Kx = J; Kx < 3; ++Kx) {
          auto dg = [&](int d, int qq) { return S(S_DG + 6 * d + qq); };
          GLv[I][sym(J, Kx)] = 0.5 * (dg(J, sym(Kx, I)) + dg(Kx, sym(J, I)) - dg(I, sym(J, Kx)));
        }
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int qq = 0; qq < 6; ++qq) S(S_DG + 6 * I + qq) = GLv[I][qq];
  } else {
    // D_i D_j phi (bssn.cc:592-602) and (D_i D_j alpha)^TF (:604-626)
    double DDa[6];
    double gld[3];
#pragma unroll
    for (int I = 0; I < 3; ++I) gld[I] = gi[sym(I, 0)] * dphi[0] + gi[sym(I, 1)] * dphi[1] + gi[sym(I, 2)] * dphi[2];
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = I; J < 3; ++J) {
        const int qq = sym(I, J);
        S(S_DDPHI + qq) = S(S_DDPHI + qq) - (G(0, qq) * dphi[0] + G(1, qq) * dphi[1] + G(2, qq) * dphi[2]);
        double t = 0.0;
#pragma unroll
        for (int L = 0; L < 3; ++L) {
          const double u = G(L, qq) + 2.0 * ((L == I ? 1.0 : 0.0) * dphi[J] + (L == J ? 1.0 : 0.0) * dphi[I] - gm[qq] * gld[L]);
          t = L == 0 ? u * da[L] : t + u * da[L];
        }
        DDa[qq] = S(S_DDA + qq) - (t);
      }
    double DDaTR = gi[0] * DDa[0] + gi[3] * DDa[3] + gi[5] * DDa[5] + 2.0 * (gi[1] * DDa[1] + gi[2] * DDa[2] + gi[4] * DDa[4]);
#pragma unroll
    for (int m = 0; m < 6; ++m) S(S_DDA + m) = DDa[m] - (1.0 / 3.0) * gm[m] * DDaTR;
    DDaTR *= em4phi;
    S(XDDA) = DDaTR;
  }
  // Gamma^I = g^jk Gamma^I_jk, and A^ij (calculate_Acont, bssn.cc:463-472): both halves
  double Gd[3];
#pragma unroll
  for (int I = 0; I < 3; ++I)
    Gd[I] = G(I, 0) * gi[0] + G(I, 3) * gi[3] + G(I, 5) * gi[5] + 2.0 * (G(I, 1) * gi[1] + G(I, 2) * gi[2] + G(I, 4) * gi[4]);
  double A[6], Ac[6];
#pragma unroll
  for (int q = 0; q < 6; ++q) A[q] = C(F_A11 + q);
#pragma unroll
  for (int I = 0; I < 3; ++I)
#pragma unroll
    for (int J = I; J < 3; ++J) {
      double t = gi[sym(I, 0)] * gi[sym(J, 0)] * A[sym(0, 0)];
      t = t + gi[sym(I, 1)] * gi[sym(J, 0)] * A[sym(1, 0)];
      t = t + gi[sym(I, 2)] * gi[sym(J, 0)] * A[sym(2, 0)];
      t = t + gi[sym(I, 0)] * gi[sym(J, 1)] * A[sym(0, 1)];
      t = t + gi[sym(I, 1)] * gi[sym(J, 1)] * A[sym(1, 1)];
      t = t + gi[sym(I, 2)] * gi[sym(J, 1)] * A[sym(2, 1)];
      t = t + gi[sym(I, 0)] * gi[sym(J, 2)] * A[sym(0, 2)];
      t = t + gi[sym(I, 1)] * gi[sym(J, 2)] * A[sym(1, 2)];
      t = t + gi[sym(I, 2)] * gi[sym(J, 2)] * A[sym(2, 2)];
      Ac[sym(I, J)] = t;
    }
  __syncthreads();

  // -- 2.3: Ricci (bssn.cc:629-674, bssn_macros.h:248-277), three components per half --
  auto DDphi = [&](int qq) { return S(S_DDPHI + qq); };
  const double expression =
      (gi[0] * (DDphi(0) + 2.0 * dphi[0] * dphi[0]) + gi[3] * (DDphi(3) + 2.0 * dphi[1] * dphi[1]) +
       gi[5] * (DDphi(5) + 2.0 * dphi[2] * dphi[2]) +
       2.0 * (gi[1] * (DDphi(1) + 2.0 * dphi[0] * dphi[1]) + gi[2] * (DDphi(2) + 2.0 * dphi[0] * dphi[2]) +
              gi[4] * (DDphi(4) + 2.0 * dphi[1] * dphi[2])));
  // Ricci term 4 (BSSN_CALCULATE_RICCI_UNITARY_TERM4): the parity build sums
  // the reference's 27 terms in its order; the FMA build contracts through
  // the raised symbols H^K_{MX} = sum_L g^{LM} G^K_{LX} (see stage_body)
  auto term4 = [&](int I, int J) {
    double acc = 0.0;
    if constexpr (kReferenceOrder) {
#pragma unroll
      for (int Kx = 0; Kx < 3; ++Kx)
#pragma unroll
        for (int L = 0; L < 3; ++L)
#pragma unroll
          for (int M = 0; M < 3; ++M) {
            const double u =
                gi[sym(L, M)] * (G(Kx, sym(L, I)) * GL(J, sym(Kx, M)) + G(Kx, sym(L, J)) * GL(I, sym(Kx, M)) +
                                 0.5 * (G(Kx, sym(I, M)) * GL(Kx, sym(L, J)) + G(Kx, sym(J, M)) * GL(Kx, sym(L, I))));
            acc = (Kx == 0 && L == 0 && M == 0) ? u : acc + u;
          }
    } else {
#pragma unroll
      for (int Kx = 0; Kx < 3; ++Kx) {
        double u = 0.0, w = 0.0;
#pragma unroll
        for (int M = 0; M < 3; ++M) {
          const double hI = gi[sym(0, M)] * G(Kx, sym(0, I)) + gi[sym(1, M)] * G(Kx, sym(1, I)) + gi[sym(2, M)] * G(Kx, sym(2, I));
          const double hJ = gi[sym(0, M)] * G(Kx, sym(0, J)) + gi[sym(1, M)] * G(Kx, sym(1, J)) + gi[sym(2, M)] * G(Kx, sym(2, J));
          u = u + (hI * GL(J, sym(Kx, M)) + hJ * GL(I, sym(Kx, M)));
          w = w + (hI * GL(Kx, sym(M, J)) + hJ * GL(Kx, sym(M, I)));
        }
        acc = acc + (u + 0.5 * w);
      }
    }
    return acc;
  };
  // the reference order for three components at once: each component's
  // sum runs over (K, L, M) as before, and the symbols of one K are loaded
  // once for all three
  auto term4_three = [&](const int (&I)[3], const int (&J)[3], double (&t)[3]) {
#pragma unroll
    for (int Kx = 0; Kx < 3; ++Kx)
#pragma unroll
      for (int L = 0; L < 3; ++L)
#pragma unroll
        for (int M = 0; M < 3; ++M)
#pragma unroll
          for (int n = 0; n < 3; ++n) {
            const double u = gi[sym(L, M)] *
                             (G(Kx, sym(L, I[n])) * GL(J[n], sym(Kx, M)) + G(Kx, sym(L, J[n])) * GL(I[n], sym(Kx, M)) +
                              0.5 * (G(Kx, sym(I[n], M)) * GL(Kx, sym(L, J[n])) + G(Kx, sym(J[n], M)) * GL(Kx, sym(L, I[n]))));
            t[n] = (Kx == 0 && L == 0 && M == 0) ? u : t[n] + u;
          }
  };
  auto ricci_component = [&](int I, int J, double t4) {
    const int ij = sym(I, J);
    auto dGam = [&](int Jx, int Kx) { return S(S_DGAM + 3 * Kx + Jx); };
    const double t2a = gm[sym(0, I)] * dGam(J, 0) + gm[sym(1, I)] * dGam(J, 1) + gm[sym(2, I)] * dGam(J, 2);
    const double t2b = gm[sym(0, J)] * dGam(I, 0) + gm[sym(1, J)] * dGam(I, 1) + gm[sym(2, J)] * dGam(I, 2);
    const double t3a = Gd[0] * GL(I, sym(J, 0)) + Gd[1] * GL(I, sym(J, 1)) + Gd[2] * GL(I, sym(J, 2));
    const double t3b = Gd[0] * GL(J, sym(I, 0)) + Gd[1] * GL(J, sym(I, 1)) + Gd[2] * GL(J, sym(I, 2));
    const double U = (-0.5 * (S(S_T1 + ij)) + 0.5 * (t2a + t2b) + 0.5 * (t3a + t3b) + t4);
    S(S_T1 + ij) = U - 2.0 * (DDphi(ij) - 2.0 * dphi[I] * dphi[J] + gm[ij] * (expression));
  };
  {
    // A: 11, 12, 13; B: 22, 23, 33
    double t4[3] = {0.0, 0.0, 0.0};
    if constexpr (kReferenceOrder) {
      if (h == 0) term4_three({0, 0, 0}, {0, 1, 2}, t4);
      else term4_three({1, 1, 2}, {1, 2, 2}, t4);
    } else {
#pragma unroll
      for (int n = 0; n < 3; ++n) t4[n] = h == 0 ? term4(0, n) : term4(n == 2 ? 2 : 1, n == 0 ? 1 : 2);
    }
    if (h == 0) {
      ricci_component(0, 0, t4[0]);
      ricci_component(0, 1, t4[1]);
      ricci_component(0, 2, t4[2]);
    } else {
      ricci_component(1, 1, t4[0]);
      ricci_component(1, 2, t4[1]);
      ricci_component(2, 2, t4[2]);
    }
  }
  __syncthreads();

  // -- 2.4: the scalars both halves use, then each half's fields --
  auto Ric = [&](int qq) { return S(S_T1 + qq); };  // full Ricci R_ij (bssn.cc:650-655)
  const double ricci = em4phi * (Ric(0) * gi[0] + Ric(3) * gi[3] + Ric(5) * gi[5] +
                                 2.0 * (Ric(1) * gi[1] + Ric(2) * gi[2] + Ric(4) * gi[4]));
  const double AijAij = Ac[0] * A[0] + Ac[3] * A[3] + Ac[5] * A[5] + 2.0 * (Ac[1] * A[1] + Ac[2] * A[2] + Ac[4] * A[4]);
  const double r = S(S_SRC + Q_R) + bg.rho_FRW;
  // Hamiltonian constraint, bssn.cc:1073-1084 (theta = 0)
  const double H = -e5phi / 8.0 * (ricci + 2.0 / 3.0 * ((K + 2.0 * 0.0) * (K + 2.0 * 0.0)) - AijAij - 16.0 * kPi * r);

  const double dt = ph.dt;
  double outv[NFLD];
  const bool renorm = ph.normalize != 0;
  constexpr int RKO = O == 8 ? 5 : 2;
  const bool ko_on = KO && (O == 2 || O == 8) && ph.ko_coeff != 0.0;
  const bool ko_inside = x0 >= RKO && x0 + kBX + RKO <= geo.nx && y0 >= RKO && y0 + kBY + RKO <= geo.ny &&
                         z0 >= RKO && z0 + kBZ + RKO <= geo.nz;
  // Kreiss-Oliger term of field fld (subtracted from its RHS, bssn.cc:748-831)
  auto ko = [&](int fld) -> double {
    if constexpr (KO) {
      if (ko_on)
        return ko_dissipation<O>(a + (size_t)fld * N, i, j, k, geo.nx, geo.ny, geo.nz, ko_inside, ph.ko_coeff, ph.dx);
    }
    return 0.0;
  };
  auto finalize = [&](int fld, double cv) {
    const double pv = __ldcs(&P.p[(size_t)fld * N + c]);
    double o, fo = 0.0;
    if (stage == 1) {
      fo = dt * cv / 6.0;
      o = pv + dt * cv / 2.0;
    } else if (stage == 2) {
      const double fv = __ldcs(&P.f[(size_t)fld * N + c]);
      fo = fv + dt * cv / 3.0;
      o = pv + dt * cv / 2.0;
    } else if (stage == 3) {
      const double fv = __ldcs(&P.f[(size_t)fld * N + c]);
      fo = fv + dt * cv / 3.0;
      o = pv + dt * cv;
    } else {
      const double fv = __ldcs(&P.f[(size_t)fld * N + c]);
      o = fv + (dt * cv / 6.0 + pv);
    }
    if (live) {
      if (stage < 4) __stcs(&P.f[(size_t)fld * N + c], fo);
      __stcs(&P.out[(size_t)fld * N + c], o);
      if (stage == 4 && !(renorm && fld < F_K && fld != F_PHI)) __stcs(&P.norm[(size_t)fld * N + c], o);
    }
    outv[fld] = o;
  };

  if (h == 0) {
    // ev_DIFFgammaIJ (bssn.cc:748-753)
#pragma unroll
    for (int m = 0; m < 6; ++m)
      finalize(F_G11 + m, (-2.0 * alpha * A[m]) + 0.5 * ph.a_adj_amp * dt * H * g[m] - ko(F_G11 + m));
    // ev_DIFFK (bssn.cc:766-795)
    {
      const double DDaTR = S(XDDA);
      double v = (-DDaTR + alpha * (1.0 / 3.0 * (Kd + 2.0 * 0.0) * (Kd + 2.0 * 0.0 + 2.0 * bg.K_FRW) + AijAij) +
                  4.0 * kPi * alpha * (S(S_SRC + Q_R) + S(S_SRC + Q_S)) + 4.0 * kPi * alphad * (bg.rho_FRW + bg.S_FRW));
      if (ph.k_damping_amp != 0.0) v = v - 1.0 * ph.k_damping_amp * H * em5phi;
      finalize(F_K, v - ko(F_K));
    }
    // ev_DIFFphi (bssn.cc:797-820)
    finalize(F_PHI, (0.1 * ph.a_adj_amp * dt * H - 1.0 / 6.0 * (alpha * (Kd + 2.0 * 0.0) + alphad * bg.K_FRW - (0.0 + 0.0 + 0.0))) -
                        ko(F_PHI));
    // ev_DIFFalpha (bssn.cc:822-831)
    finalize(F_ALPHA, ev_lapse(ph, bg, alpha, K, Kd, phi) - ko(F_ALPHA));
    if (MATTER == kDust) {
#pragma unroll
      for (int m = 0; m < 4; ++m) finalize(F_D + m, rhs_m[m]);
    } else if (MATTER == kScalar) {
#pragma unroll
      for (int m = 0; m < 5; ++m) finalize(F_SPHI + m, rhs_m[m]);
    }
  } else {
    // ev_AIJ (bssn.cc:755-760, BSSN_DT_AIJ bssn_macros.h:334-337)
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
      for (int J = I; J < 3; ++J) {
        const int qq = sym(I, J);
        double aa = 0.0;
#pragma unroll
        for (int X = 0; X < 3; ++X)
#pragma unroll
          for (int Y = 0; Y < 3; ++Y) {
            const double u = gi[sym(X, Y)] * A[sym(X, I)] * A[sym(Y, J)];
            aa = (X == 0 && Y == 0) ? u : aa + u;
          }
        const double RTF = Ric(qq) - (1.0 / 3.0) * e4phi * gm[qq] * ricci;
        const double dtA = (em4phi * (alpha * (RTF - 8.0 * kPi * S(S_SRC + Q_STF11 + qq)) - S(S_DDA + qq)) +
                            alpha * (((K + 2.0 * 0.0) * A[qq]) - 2.0 * (aa)));
        finalize(F_A11 + qq, dtA - 1.0 * ph.a_adj_amp * dt * A[qq] * H - ko(F_A11 + qq));
      }
    // ev_GammaI (bssn.cc:762-764, BSSN_DT_GAMMAI_NOSHIFT bssn_macros.h:342-361)
    const double sq[3] = {S(S_SRC + Q_S1), S(S_SRC + Q_S2), S(S_SRC + Q_S3)};
#pragma unroll
    for (int I = 0; I < 3; ++I) {
      auto Gs = [&](int qq) { return S(S_G + 6 * I + qq); };
      const double so = (Gs(0) * Ac[0] + Gs(3) * Ac[3] + Gs(5) * Ac[5] + 2.0 * (Gs(1) * Ac[1] + Gs(2) * Ac[2] + Gs(4) * Ac[4]) +
                         6.0 * (Ac[sym(I, 0)] * dphi[0] + Ac[sym(I, 1)] * dphi[1] + Ac[sym(I, 2)] * dphi[2]));
      const double ns =
          (-2.0 * (Ac[sym(I, 0)] * da[0] + Ac[sym(I, 1)] * da[1] + Ac[sym(I, 2)] * da[2]) +
           2.0 * alpha *
               (+so -
                (1.0 / 3.0) * (2.0 * (gi[sym(I, 0)] * S(S_DK + 0) + gi[sym(I, 1)] * S(S_DK + 1) + gi[sym(I, 2)] * S(S_DK + 2)) +
                               gi[sym(I, 0)] * 0.0 + gi[sym(I, 1)] * 0.0 + gi[sym(I, 2)] * 0.0) -
                2.0 * alpha * 0.0 * (C(F_GAM1 + I) - Gd[I]) -
                8.0 * kPi * (gi[sym(I, 0)] * sq[0] + gi[sym(I, 1)] * sq[1] + gi[sym(I, 2)] * sq[2])));
      finalize(F_GAM1 + I, ns + 0.0 - ko(F_GAM1 + I));
    }
  }

  // ---- the next substep's inputs -----------------------------------------------
  if (stage == 4) {
    // failure detection (sims/sim.cc:179-183 counts NaNs of DIFFphi): each
    // half checks the fields it wrote
    bool bad_any = false;
#pragma unroll
    for (int f = 0; f < NFLD; ++f)
      if (pair_owner(f) == h) bad_any |= !isfinite(outv[f]);
    if (live && bad_any) {
      if (h == 0 && isnan(outv[F_PHI])) atomicOr(P.status, kStatusNaN);
      atomicOr(P.status, kStatusNonFinite);
    }
    if (renorm) {
      // next step's first-substep input: normalised gamma/A (bssn.cc:224-225);
      // B's A_ij go to A through the Christoffel slots, which B has finished reading
      if (h == 1) {
#pragma unroll
        for (int m = 0; m < 6; ++m) S(S_G + m) = outv[F_A11 + m];
      }
      __syncthreads();
      if (h == 0) {
        double gn[6], An[6];
#pragma unroll
        for (int m = 0; m < 6; ++m) { gn[m] = outv[F_G11 + m]; An[m] = S(S_G + m); }
        normalize_point(gn, An);
#pragma unroll
        for (int m = 0; m < 6; ++m) {
          outv[F_G11 + m] = gn[m];
          if (live) {
            __stcs(&P.norm[(size_t)(F_G11 + m) * N + c], gn[m]);
            __stcs(&P.norm[(size_t)(F_A11 + m) * N + c], An[m]);
          }
        }
      }
    }
  }
  if (MATTER == kDust && h == 0) {
    // flux primitives of the output state for the next substep's divergence
    double go[6], gio[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) go[m] = outv[F_G11 + m];
    inv_metric(go, gio);
    const double So[3] = {outv[F_S1], outv[F_S2], outv[F_S3]};
    const double phio = outv[F_PHI] + bg.phi_FRW_next;
    double eo[2];
    {
      const double xo[2] = {-4.0 * phio, 6.0 * phio};
      xexp_n<2>(xo, eo);
    }
    const DustPrim dp = dust_prim(gio, eo[0], eo[1], outv[F_D], So);
    const double alo = outv[F_ALPHA] + 1.0;
    double* fo = P.fp_out;
    if (live) {
      __stcs(&fo[(size_t)P_AD * N + c], alo * outv[F_D]);
#pragma unroll
      for (int m = 0; m < 3; ++m) __stcs(&fo[(size_t)(P_AS1 + m) * N + c], alo * So[m]);
#pragma unroll
      for (int m = 0; m < 3; ++m) __stcs(&fo[(size_t)(P_V1 + m) * N + c], dp.v[m]);
    }
  }
}

// One box: one CTA of 256 threads per brick.
template <int O, int MATTER, bool KO = false>
__global__ void __launch_bounds__(kPairThreads, 2)
stage_pair_kernel(BoxGeom geo, Physics ph, StageBg bg, StagePtrs P, int stage, const __grid_constant__ CUtensorMap tmap,
                  int use_tma, const __grid_constant__ FluxMaps fmaps, int use_fmaps) {
  __shared__ __align__(8) uint64_t bar[2];
  init_tile_barriers(bar, use_tma != 0);
  unsigned phase = 0;
  bool tma_ok = true;
  pair_stage_body<O, MATTER, KO>(geo, ph, bg, P, stage, blockIdx.z + geo.bx0, blockIdx.y, blockIdx.x,
                                 use_tma ? &tmap : nullptr, bar, phase, tma_ok, use_tma && use_fmaps ? &fmaps : nullptr);
}

// The group kernel (stage_group_kernel) with the pair body.
template <int O, int MATTER>
__global__ void __launch_bounds__(kPairThreads, 2)
stage_pair_group_kernel(const GroupBox* __restrict__ boxes, GroupBg gb, int stage) {
  __shared__ GroupBox sb;
  __shared__ StagePtrs sp;
  __shared__ StageBg sbg;
  __shared__ const CUtensorMap* stm;
  __shared__ const FluxMaps* sfm;
  __shared__ __align__(8) uint64_t bar[2];
  const bool lead = threadIdx.x == 0;
  init_tile_barriers(bar, true);
  unsigned phase = 0;
  bool tma_ok = true;
  for (int w = blockIdx.x; w < gb.total; w += gridDim.x) {
    __syncthreads();  // the previous brick is finished with the slots, the tile and sb
    if (lead) {
      int lo = 0, hi = gb.nboxes - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (boxes[mid].first <= w) lo = mid; else hi = mid - 1;
      }
      sb = boxes[lo];
      sp = group_ptrs(sb, stage);
      sbg = gb.bg[lo];
      stm = boxes[lo].tma ? (stage == 1 || stage == 3 ? &boxes[lo].mapX : &boxes[lo].mapY) : nullptr;
      if (stm) tma::acquire_map(stm);
      sfm = nullptr;
      if (MATTER == kDust && stm) {
        const GroupFluxMaps& fx = reinterpret_cast<const GroupFluxMaps*>(boxes + gb.nboxes)[lo];
        if (fx.valid) {
          sfm = reinterpret_cast<const FluxMaps*>(stage == 1 || stage == 3 ? fx.fp0 : fx.fp1);
          for (int a = 0; a < 3; ++a) tma::acquire_map(&sfm->m[a]);
        }
      }
    }
    __syncthreads();
    const int l = w - sb.first;
    const int cz = l % sb.nbz, cy = (l / sb.nbz) % sb.nby, cx = l / (sb.nbz * sb.nby);
    const BoxGeom geo{sb.nx, sb.ny, sb.nz, sb.pts, 0};
    pair_stage_body<O, MATTER, false>(geo, sb.ph, sbg, sp, stage, cx, cy, cz, stm, bar, phase, tma_ok, sfm);
  }
}
