// Fused Maxwell stage kernel: residual (maxwell.py:603-729) + Runge-Kutta stage.
//
// Conserved B (3) and D (3); face fluxes are the antisymmetric curl tensors of
// H = B/mu and E = D/eps (maxwell.py:145-181) evaluated on reconstructed face
// states, combined by Rusanov or HLL with wave speeds -+c (c = 1/sqrt(mu eps),
// :256-260).  Sources: geometric (:365-374), Ohmic J = -sigma E (:414-420) and
// divergence cleaning -chi grad r with r = div B or div D - rho_c computed on
// interior cells and edge-padded at the domain boundary (:490-528).
// z-march with HH = 2: at step K the TMA ring receives plane K+2, the
// cleaning residuals of plane K+1 are computed on the tile plus one cell,
// x3 slopes at K+1 and the x3 face flux at K+1/2 go to registers, and the
// x1/x2 fluxes of plane K go through shared memory.
#pragma once
#include "stage_ns.cuh"

namespace fvm {

template <typename Real>
struct MaxwellParams {
  Layout lay;
  Metric<Real> met;
  const Real* u0;
  Real* out;
  Real* acc;
  const double* dt;
  const int* active;
  StageCoef coef;
  double mu, ep, sigma, rho_c, chi_b, chi_d, c;
  unsigned* status;
  int zchunk, ntx, nty, nzc;
  unsigned long long wait_ns;  // limit of each wait for a TMA plane (ns)
  unsigned long long drain_ns;  // limit of the wait for copies in flight after a timeout (ns)
  unsigned extra_tx;  // test of the timeout path: bytes a ring copy never delivers (0 normally)
};

template <typename Real, int TY>
struct MaxwellCfg {
  static constexpr int TX = 32;
  static constexpr int NT = TX * (TY + 2);
  static constexpr int NV = 6;
  static constexpr int HH = 2;
  static constexpr int W = 40;
  static constexpr int ROWS = TY + 2 * HH;
  static constexpr int PL = ROWS * W;
  static constexpr int NSLOT = HH + 2;
  static constexpr int SLOT = round_up(NV * PL * (int)sizeof(Real), 128) / (int)sizeof(Real);
  static constexpr int XB = cmax(TY * (TX + 2), (TY + 2) * TX);
  static constexpr int FB = cmax(TY * (TX + 1), (TY + 1) * TX);
  static constexpr int OFF_U = 0;
  static constexpr int OFF_R = OFF_U + NSLOT * SLOT;
  static constexpr int OFF_FL = OFF_R + 3 * 2 * PL;
  static constexpr int OFF_FR = OFF_FL + NV * XB;
  static constexpr int OFF_FB = OFF_FR + NV * XB;
  // U0 and acc of the plane's output cells copied in by cp.async at the start
  // of each step ([U0 | acc][variable][output thread]).  Off: with the extra
  // 9 KB per block the three float32 blocks per SM leave too little L1 for
  // the metric tables, and the step was slower (2.48 -> 2.53 ms on C2a).
  static constexpr bool STAGED = false;
  static constexpr int OFF_G = OFF_FB + NV * FB;
  static constexpr int END = OFF_G + (STAGED ? 2 * NV * TX * TY : 0);
  static constexpr int BYTES = round_up(END * (int)sizeof(Real), 16) + NSLOT * 8;
  static constexpr unsigned TX_BYTES = NV * PL * sizeof(Real);
};

// Normal curl flux along axis D of face state q = (B1,B2,B3,D1,D2,D3):
// F_B[c] = FB[c][D], F_D[c] = FD[c][D] with FB12 = E3, FB13 = -E2, FB23 = E1,
// FD12 = -H3, FD13 = H2, FD23 = -H1 and antisymmetry (maxwell.py:145-165).
template <typename R, int D>
__device__ __forceinline__ void maxwell_face(const R* q, R mu, R ep, R F[6]) {
  R H0, H1, H2, E0, E1, E2;
  if constexpr (sizeof(R) == 4) {
    const R imu = rcp_approx(mu), iep = rcp_approx(ep);
    H0 = q[0] * imu; H1 = q[1] * imu; H2 = q[2] * imu;
    E0 = q[3] * iep; E1 = q[4] * iep; E2 = q[5] * iep;
  } else {
    H0 = q[0] / mu; H1 = q[1] / mu; H2 = q[2] / mu;
    E0 = q[3] / ep; E1 = q[4] / ep; E2 = q[5] / ep;
  }
  if constexpr (D == 0) {
    F[0] = R(0); F[1] = -E2; F[2] = E1;
    F[3] = R(0); F[4] = H2; F[5] = -H1;
  } else if constexpr (D == 1) {
    F[0] = E2; F[1] = R(0); F[2] = -E0;
    F[3] = -H2; F[4] = R(0); F[5] = H0;
  } else {
    F[0] = -E1; F[1] = E0; F[2] = R(0);
    F[3] = H1; F[4] = -H0; F[5] = R(0);
  }
}

template <typename R, int D, int RIEM>
__device__ __forceinline__ void maxwell_flux(const R* qL, const R* qR, R mu, R ep, R c, R F[6]) {
  R FL[6], FR[6];
  maxwell_face<R, D>(qL, mu, ep, FL);
  maxwell_face<R, D>(qR, mu, ep, FR);
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    if constexpr (RIEM == RIEM_HLL) {
      const R smin = -c, smax = c;
      const R num = ((smax * FL[v]) - (smin * FR[v])) + ((smin * smax) * (qR[v] - qL[v]));
      if constexpr (sizeof(R) == 4) F[v] = num * (0.5f * rcp_approx(c));
      else F[v] = num / (smax - smin);
    } else {
      F[v] = ((FL[v] + FR[v]) / R(2)) - ((c * (qR[v] - qL[v])) / R(2));
    }
    F[v] = F[v] + R(0);
  }
}

template <typename Real, int LIM, int RIEM, int COORD, int TY, int MINB>
__global__ void __launch_bounds__(MaxwellCfg<Real, TY>::NT, MINB)
    maxwell_stage_kernel(const __grid_constant__ CUtensorMap tmap, const MaxwellParams<Real> p) {
  using C = MaxwellCfg<Real, TY>;
  using G = Geo<Real, COORD>;
  constexpr int TX = C::TX, NT = C::NT, W = C::W, PL = C::PL, HH = C::HH, NV = C::NV;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Real* sm = reinterpret_cast<Real*>(smem_raw);
  Real* uring = sm + C::OFF_U;
  Real* rring = sm + C::OFF_R;
  Real* fL = sm + C::OFF_FL;
  Real* fR = sm + C::OFF_FR;
  Real* fb = sm + C::OFF_FB;
  Real* gst = sm + C::OFF_G;
  constexpr bool STAGED = C::STAGED;
  constexpr int NO = TX * TY;  // output threads
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + (C::BYTES - C::NSLOT * 8));
  if (p.active && !*p.active) return;
  if (smem_u32(smem_raw) & 127u) {
    if (threadIdx.x == 0) atomicOr(p.status, ST_TMA_TIMEOUT);
    return;
  }
  const int tid = threadIdx.x;
  const Layout& L = p.lay;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const Real mu = Real(p.mu), ep = Real(p.ep), cl = Real(p.c);
  const Real dt = Real(*p.dt);
  if (tid == 0) {
    tma_prefetch_desc(&tmap);
    for (int s = 0; s < C::NSLOT; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  unsigned phase_bits = 0, pending = 0;
  // ring access through per-step plane bases (no modulo per access)
  auto UA = [&](const Real* b, int q, int r, int c) -> Real { return b[q * PL + r * W + c]; };

  const bool is_out = tid < TX * TY;
  const int otx = tid % TX, oty = tid / TX;
  const int ntiles = p.ntx * p.nty * p.nzc;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int x0 = (tile % p.ntx) * TX, y0 = ((tile / p.ntx) % p.nty) * TY;
    const int Z0 = 1 + (tile / (p.ntx * p.nty)) * p.zchunk;
    const int Zl = min(Z0 + p.zchunk - 1, nz);
    const int Pfirst = Z0 - HH, Plast = Zl + HH, Kfirst = Z0 - 2 * HH;
    const int oi = x0 + otx, oj = y0 + oty;
    const bool out_valid = is_out && oi < nx && oj < ny;
    Real zs[NV], Fzp[NV], Fzn[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) { zs[v] = Real(0); Fzp[v] = Real(0); Fzn[v] = Real(0); }
    const Real S3c = out_valid ? G::S3(p.met, oi, oj) : Real(0);
    auto issue = [&](int pl) {
      const int s = pmod(pl, C::NSLOT);
      pending |= 1u << s;
      fence_proxy_async();
      mbar_arrive_expect_tx(&bars[s], C::TX_BYTES + p.extra_tx);
      tma_load_4d(&uring[s * C::SLOT], &tmap, &bars[s], x0 - 3 + L.padx, y0 + 1 - HH, pl, 0);
    };
    if (tid == 0) issue(Pfirst);
    for (int K = Kfirst; K <= Zl; ++K) {
      {
        const int s = pmod(K + HH, C::NSLOT);
        const bool got = mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.wait_ns);
        if (!__syncthreads_and(got)) {
          if (tid == 0) atomicOr(p.status, ST_TMA_TIMEOUT);
          ok = false;
          break;
        }
        phase_bits ^= 1u << s;
        pending &= ~(1u << s);
      }
      // Prefetch plane K+HH+1 into the slot of plane K-1.  Issued after the
      // barrier above, which every thread reaches only after its last read of
      // the previous step, so the steps need no barrier at their end.
      if (tid == 0 && K + HH + 1 <= Plast) issue(K + HH + 1);
      // U0 and acc of this plane's output cells, fetched now so that the
      // step hides their latency: copied into this thread's shared-memory
      // slots (STAGED), or lane 0 of each row asks L2 for them
      if (K >= Z0 && out_valid) {
        const long long g0 = L.idx(0, K, oj + 1, oi + 1);
        if constexpr (STAGED) {
#pragma unroll
          for (int v = 0; v < NV; ++v) {
            if (needs_u0<Real>(p.coef) && !p.coef.u0_is_input) cp_async4(&gst[v * NO + tid], p.u0 + g0 + v * L.var_stride);
            if (needs_acc(p.coef)) cp_async4(&gst[(NV + v) * NO + tid], p.acc + g0 + v * L.var_stride);
          }
        } else if (otx == 0) {
          for (int v = 0; v < NV; ++v) {
            if (needs_u0<Real>(p.coef) && !p.coef.u0_is_input) prefetch_l2(p.u0 + g0 + v * L.var_stride);
            if (needs_acc(p.coef)) prefetch_l2(p.acc + g0 + v * L.var_stride);
          }
        }
      }
      const Real* uK = uring + pmod(K, C::NSLOT) * C::SLOT;
      const Real* uK1 = uring + pmod(K + 1, C::NSLOT) * C::SLOT;
      const Real* uK2 = uring + pmod(K + 2, C::NSLOT) * C::SLOT;
      const Real* rKm = rring + pmod(K - 1, 3) * 2 * PL;
      const Real* rK = rring + pmod(K, 3) * 2 * PL;
      Real* rK1 = rring + pmod(K + 1, 3) * 2 * PL;
      // cleaning residuals of plane K+1 on interior cells of the tile + 1
      {
        const int pl = K + 1, k = pl - 1;
        if (K >= Z0 - 2 && k >= 0 && k < nz) {
          for (int it = tid; it < (TY + 2) * (TX + 2); it += NT) {
            const int r = HH - 1 + it / (TX + 2), c = 3 + it % (TX + 2);
            const int i = x0 + c - 4, j = y0 + r - HH;
            if (i < 0 || i >= nx || j < 0 || j >= ny) continue;
            Real div[2];
            Lame<Real> lm;
            if constexpr (COORD != COORD_CART) lame_at<Real, COORD>(p.met, i, j, lm);
#pragma unroll
            for (int f = 0; f < 2; ++f) {
              const int q0 = 3 * f;
              Real d1, d2, d3;
              if constexpr (sizeof(Real) == 4) {
                d1 = (UA(uK1, q0, r, c + 1) - UA(uK1, q0, r, c - 1)) * (0.5f * inv_len<Real, COORD, 0>(p.met, i, j, k));
                d2 = (UA(uK1, q0 + 1, r + 1, c) - UA(uK1, q0 + 1, r - 1, c)) * (0.5f * inv_len<Real, COORD, 1>(p.met, i, j, k));
                d3 = (UA(uK2, q0 + 2, r, c) - UA(uK, q0 + 2, r, c)) * (0.5f * inv_len<Real, COORD, 2>(p.met, i, j, k));
              } else {
                const Real l1 = G::L1(p.met, i, j, k), l2 = G::L2(p.met, i, j, k), l3 = G::L3(p.met, i, j, k);
                d1 = (UA(uK1, q0, r, c + 1) - UA(uK1, q0, r, c - 1)) / (Real(2) * l1);
                d2 = (UA(uK1, q0 + 1, r + 1, c) - UA(uK1, q0 + 1, r - 1, c)) / (Real(2) * l2);
                d3 = (UA(uK2, q0 + 2, r, c) - UA(uK, q0 + 2, r, c)) / (Real(2) * l3);
              }
              Real dv = (d1 + d2) + d3;
              if constexpr (COORD != COORD_CART) {
                if constexpr (sizeof(Real) == 4) {
                  dv = ((dv + (UA(uK1, q0, r, c) * (lm.dl[0][1] + lm.dl[0][2])) * recip(lm.h[0])) +
                        (UA(uK1, q0 + 1, r, c) * (lm.dl[1][0] + lm.dl[1][2])) * recip(lm.h[1])) +
                       (UA(uK1, q0 + 2, r, c) * (lm.dl[2][0] + lm.dl[2][1])) * recip(lm.h[2]);
                } else {
                  dv = ((dv + ((UA(uK1, q0, r, c) * (lm.dl[0][1] + lm.dl[0][2])) / lm.h[0])) +
                        ((UA(uK1, q0 + 1, r, c) * (lm.dl[1][0] + lm.dl[1][2])) / lm.h[1])) +
                       ((UA(uK1, q0 + 2, r, c) * (lm.dl[2][0] + lm.dl[2][1])) / lm.h[2]);
                }
              }
              div[f] = dv;
            }
            rK1[r * W + c] = div[0];
            rK1[PL + r * W + c] = div[1] - Real(p.rho_c);
          }
        }
      }
      // x3 slopes at K+1 and the x3 face flux at K+1/2
      if (K >= Z0 - 2 && is_out) {
        const int r = oty + HH, c = otx + 4;
        Real qm[NV], q0[NV], qp[NV], zn[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) { qm[v] = UA(uK, v, r, c); q0[v] = UA(uK1, v, r, c); qp[v] = UA(uK2, v, r, c); }
        const bool ghost = (K + 1 <= 0 || K + 1 >= nz + 1);
        if (ghost || !out_valid) {
#pragma unroll
          for (int v = 0; v < NV; ++v) zn[v] = Real(0);
        } else {
          const Real l3 = G::L3(p.met, oi, oj, K);
#pragma unroll
          for (int v = 0; v < NV; ++v) zn[v] = muscl_slope<LIM>(qm[v], q0[v], qp[v], l3);
        }
        if (K >= Z0 - 1) {
          Real qL[NV], qR[NV], F[NV];
#pragma unroll
          for (int v = 0; v < NV; ++v) { qL[v] = qm[v] + zs[v] / Real(2); qR[v] = q0[v] - zn[v] / Real(2); }
          maxwell_flux<Real, 2, RIEM>(qL, qR, mu, ep, cl, F);
#pragma unroll
          for (int v = 0; v < NV; ++v) { Fzp[v] = Fzn[v]; Fzn[v] = F[v] * S3c; }
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) zs[v] = zn[v];
      }
      __syncthreads();
      if (K < Z0) continue;
      const int kK = K - 1;
      // x1 faces
      for (int it = tid; it < TY * (TX + 2); it += NT) {
        const int ty = it / (TX + 2), tx = it % (TX + 2) - 1;
        const int r = ty + HH, c = tx + 4, i = x0 + tx, j = y0 + ty;
        const bool interior = i >= 0 && i < nx && j < ny;
        const Real l1 = interior ? G::L1(p.met, i, j, kK) : Real(1);
        const int o = ty * (TX + 2) + tx + 1;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const Real f0 = UA(uK, v, r, c);
          const Real s = interior ? muscl_slope<LIM>(UA(uK, v, r, c - 1), f0, UA(uK, v, r, c + 1), l1) : Real(0);
          fL[v * C::XB + o] = f0 + s / Real(2);
          fR[v * C::XB + o] = f0 - s / Real(2);
        }
      }
      __syncthreads();
      for (int it = tid; it < TY * (TX + 1); it += NT) {
        const int ty = it / (TX + 1), fx = it % (TX + 1), fi = x0 + fx, j = y0 + ty;
        Real F[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) F[v] = Real(0);
        if (fi <= nx && j < ny) {
          Real qL[NV], qR[NV];
          const int o = ty * (TX + 2) + fx;
#pragma unroll
          for (int v = 0; v < NV; ++v) { qL[v] = fL[v * C::XB + o]; qR[v] = fR[v * C::XB + o + 1]; }
          maxwell_flux<Real, 0, RIEM>(qL, qR, mu, ep, cl, F);
          const Real s1 = G::S1(p.met, fi, j, kK);
#pragma unroll
          for (int v = 0; v < NV; ++v) F[v] = F[v] * s1;
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) fb[v * C::FB + ty * (TX + 1) + fx] = F[v];
      }
      __syncthreads();
      Real Fxm[NV], Fxp[NV];
      if (is_out) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          Fxm[v] = fb[v * C::FB + oty * (TX + 1) + otx];
          Fxp[v] = fb[v * C::FB + oty * (TX + 1) + otx + 1];
        }
      }
      // x2 faces
      for (int it = tid; it < (TY + 2) * TX; it += NT) {
        const int ty = it / TX - 1, tx = it % TX;
        const int r = ty + HH, c = tx + 4, i = x0 + tx, j = y0 + ty;
        const bool interior = i < nx && j >= 0 && j < ny;
        const Real l2 = interior ? G::L2(p.met, i, j, kK) : Real(1);
        const int o = (ty + 1) * TX + tx;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const Real f0 = UA(uK, v, r, c);
          const Real s = interior ? muscl_slope<LIM>(UA(uK, v, r - 1, c), f0, UA(uK, v, r + 1, c), l2) : Real(0);
          fL[v * C::XB + o] = f0 + s / Real(2);
          fR[v * C::XB + o] = f0 - s / Real(2);
        }
      }
      __syncthreads();
      for (int it = tid; it < (TY + 1) * TX; it += NT) {
        const int fy = it / TX, tx = it % TX, fj = y0 + fy, i = x0 + tx;
        Real F[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) F[v] = Real(0);
        if (fj <= ny && i < nx) {
          Real qL[NV], qR[NV];
          const int o = fy * TX + tx;
#pragma unroll
          for (int v = 0; v < NV; ++v) { qL[v] = fL[v * C::XB + o]; qR[v] = fR[v * C::XB + o + TX]; }
          maxwell_flux<Real, 1, RIEM>(qL, qR, mu, ep, cl, F);
          const Real s2 = G::S2(p.met, i, fj, kK);
#pragma unroll
          for (int v = 0; v < NV; ++v) F[v] = F[v] * s2;
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) fb[v * C::FB + fy * TX + tx] = F[v];
      }
      __syncthreads();
      if (out_valid) {
        const int r = oty + HH, c = otx + 4;
        Real q[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) q[v] = UA(uK, v, r, c);
        // geometric source from the cell curl tensors (zero in cartesian)
        Real sg[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) sg[v] = Real(0);
        if constexpr (COORD != COORD_CART) {
          Lame<Real> lm;
          lame_at<Real, COORD>(p.met, oi, oj, lm);
          const Real H0 = q[0] / mu, H1 = q[1] / mu, H2 = q[2] / mu;
          const Real E0 = q[3] / ep, E1 = q[4] / ep, E2 = q[5] / ep;
          Real FB[3][3], FD[3][3];
          FB[0][1] = E2; FB[0][2] = -E1; FB[1][2] = E0;
          FD[0][1] = -H2; FD[0][2] = H1; FD[1][2] = -H0;
          FB[1][0] = -FB[0][1]; FB[2][0] = -FB[0][2]; FB[2][1] = -FB[1][2];
          FD[1][0] = -FD[0][1]; FD[2][0] = -FD[0][2]; FD[2][1] = -FD[1][2];
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) {
            const int o0 = cc == 0 ? 1 : 0, o1 = cc == 2 ? 1 : 2;
            sg[cc] = ((FB[cc][o0] * lm.dl[o0][cc]) / lm.h[o0]) + ((FB[cc][o1] * lm.dl[o1][cc]) / lm.h[o1]);
            sg[3 + cc] = ((FD[cc][o0] * lm.dl[o0][cc]) / lm.h[o0]) + ((FD[cc][o1] * lm.dl[o1][cc]) / lm.h[o1]);
          }
        }
        // cleaning: gradient of the edge-padded residuals (clamp to interior)
        const int im = max(oi - 1, 0) - oi, ip = min(oi + 1, nx - 1) - oi;
        const int jm = max(oj - 1, 0) - oj, jp = min(oj + 1, ny - 1) - oj;
        const int km = (K - 1 >= 1) ? -1 : 0, kp = (K + 1 <= nz) ? 1 : 0;
        Real h1, h2, h3;  // 1/(2L) (float32) or 2L (float64)
        if constexpr (sizeof(Real) == 4) {
          h1 = 0.5f * inv_len<Real, COORD, 0>(p.met, oi, oj, kK);
          h2 = 0.5f * inv_len<Real, COORD, 1>(p.met, oi, oj, kK);
          h3 = 0.5f * inv_len<Real, COORD, 2>(p.met, oi, oj, kK);
        } else {
          h1 = Real(2) * G::L1(p.met, oi, oj, kK);
          h2 = Real(2) * G::L2(p.met, oi, oj, kK);
          h3 = Real(2) * G::L3(p.met, oi, oj, kK);
        }
        auto grad = [&](Real d, Real h) -> Real {
          if constexpr (sizeof(Real) == 4) return d * h;
          else return d / h;
        };
        Real sc[NV];
#pragma unroll
        for (int f = 0; f < 2; ++f) {
          const Real chi = f == 0 ? Real(p.chi_b) : Real(p.chi_d);
          const Real* rb = rK + f * PL + r * W + c;
          const Real* rbp = (kp ? rK1 : rK) + f * PL + r * W + c;
          const Real* rbm = (km ? rKm : rK) + f * PL + r * W + c;
          const Real g1 = grad(rb[ip] - rb[im], h1);
          const Real g2 = grad(rb[jp * W] - rb[jm * W], h2);
          const Real g3 = grad(rbp[0] - rbm[0], h3);
          sc[3 * f + 0] = (-chi) * g1;
          sc[3 * f + 1] = (-chi) * g2;
          sc[3 * f + 2] = (-chi) * g3;
        }
        const Real Vc = G::V(p.met, oi, oj, kK);
        const long long gidx = L.idx(0, K, oj + 1, oi + 1);
        // residual of each variable first (the flux registers die), then
        // every global load of the cell before its first store: the stores
        // may alias later loads as far as the compiler knows, which would
        // otherwise cost one memory round trip per variable
        Real kv[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const Real Fym = fb[v * C::FB + oty * TX + otx], Fyp = fb[v * C::FB + (oty + 1) * TX + otx];
          const Real sum = ((((Fxp[v] - Fxm[v]) + Fyp) - Fym) + Fzn[v]) - Fzp[v];
          const Real sp = v < 3 ? Real(0) : (-Real(p.sigma)) * (q[v] / ep);
          if constexpr (sizeof(Real) == 4) kv[v] = (-sum) * rcp_approx(Vc) + ((sg[v] + sp) + sc[v]);
          else kv[v] = (-sum) / Vc + ((sg[v] + sp) + sc[v]);
        }
        Real u0v[NV], accv[NV];
        if constexpr (STAGED) cp_async_wait_all();
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const long long gi = gidx + (long long)v * L.var_stride;
          if constexpr (STAGED) {
            u0v[v] = needs_u0<Real>(p.coef) ? (p.coef.u0_is_input ? q[v] : gst[v * NO + tid]) : Real(0);
            accv[v] = needs_acc(p.coef) ? gst[(NV + v) * NO + tid] : Real(0);
          } else {
            u0v[v] = needs_u0<Real>(p.coef) ? (p.coef.u0_is_input ? q[v] : p.u0[gi]) : Real(0);
            accv[v] = needs_acc(p.coef) ? p.acc[gi] : Real(0);
          }
        }
        unsigned bad = 0;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          const long long gi = gidx + (long long)v * L.var_stride;
          const Real o = stage_combine(p.coef, dt, kv[v], q[v], u0v[v], accv[v]);
          p.out[gi] = o;
          if (p.coef.accmode != ACC_NONE) p.acc[gi] = acc_update(p.coef, dt, kv[v], u0v[v], accv[v]);
          if (!isfinite(o)) bad |= ST_NONFINITE;
        }
        if (bad) atomicOr(p.status, bad);
      }
    }
    __syncthreads();  // the next tile's first loads reuse every ring slot
  }
  if constexpr (STAGED) cp_async_wait_all();  // none left in flight at exit
  if (!ok && tid == 0)
    for (int s = 0; s < C::NSLOT; ++s)
      if ((pending >> s) & 1u) mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.drain_ns);
}

}  // namespace fvm
