// Fused heat stage kernel: residual (heat.py:354-473) + Runge-Kutta stage.
//
// rhs = -sum_faces (phi_a,L + phi_a,R)/2 * S / V + q with phi = -k grad T,
// T = rho_cp_T / (rho cp), phi zero-padded in the ghosts (heat.py:40-102) and
// phi_a reconstructed along axis a (piecewise constant or MUSCL).
// Same z-march skeleton as the Navier-Stokes kernel: at step K the TMA ring
// receives plane K+HH; T of that plane, phi of plane K+HH-1, x3 slopes of
// phi_3 at K+1 and the x3 face flux at K+1/2 follow; then the x1/x2 fluxes
// of plane K go through shared memory.  HH = 3 for MUSCL (phi at K+2 needs T
// at K+3), 2 for piecewise constant.
#pragma once
#include "stage_ns.cuh"

namespace fvm {

template <typename Real>
struct HeatParams {
  Layout lay;
  Metric<Real> met;
  const Real* u0;
  Real* out;
  Real* acc;
  const double* dt;
  const int* active;
  StageCoef coef;
  double rho_cp, k, q, inv_rho_cp;
  unsigned* status;
  int zchunk, ntx, nty, nzc;
  unsigned long long wait_ns;  // limit of each wait for a TMA plane (ns)
  unsigned long long drain_ns;  // limit of the wait for copies in flight after a timeout (ns)
  unsigned extra_tx;  // test of the timeout path: bytes a ring copy never delivers (0 normally)
};

template <typename Real, int LIM, int TY>
struct HeatCfg {
  static constexpr int TX = 32;
  // enough threads for one phi task each over the tile + 1 halo, and for the
  // (TY+2) x TX x2-face tasks
  static constexpr int NT = round_up((TX + 2) * (TY + 2), 32);
  static constexpr int HH = LIM == LIM_PC ? 2 : 3;
  static constexpr int W = 40;
  static constexpr int ROWS = TY + 2 * HH;
  static constexpr int PL = ROWS * W;
  static constexpr int NSLOT = HH + 2;
  static constexpr int SLOT = round_up(PL * (int)sizeof(Real), 128) / (int)sizeof(Real);
  static constexpr int XB = cmax(TY * (TX + 2), (TY + 2) * TX);
  static constexpr int FB = cmax(TY * (TX + 1), (TY + 1) * TX);
  static constexpr int OFF_U = 0;
  static constexpr int OFF_T = OFF_U + NSLOT * SLOT;
  static constexpr int OFF_PHI = OFF_T + 3 * PL;
  static constexpr int OFF_FL = OFF_PHI + 3 * 3 * PL;
  static constexpr int OFF_FR = OFF_FL + XB;
  static constexpr int OFF_FB = OFF_FR + XB;
  static constexpr int END = OFF_FB + FB;
  static constexpr int BYTES = round_up(END * (int)sizeof(Real), 16) + NSLOT * 8;
  static constexpr unsigned TX_BYTES = PL * sizeof(Real);
};

template <typename Real, int LIM, int COORD, int TY, class Src>
__global__ void __launch_bounds__(HeatCfg<Real, LIM, TY>::NT, 1)
    heat_stage_kernel(const __grid_constant__ Src src) {
  using C = HeatCfg<Real, LIM, TY>;
  using G = Geo<Real, COORD>;
  constexpr int TX = C::TX, NT = C::NT, W = C::W, PL = C::PL, HH = C::HH;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Real* sm = reinterpret_cast<Real*>(smem_raw);
  Real* uring = sm + C::OFF_U;
  Real* tring = sm + C::OFF_T;
  Real* phring = sm + C::OFF_PHI;
  Real* fL = sm + C::OFF_FL;
  Real* fR = sm + C::OFF_FR;
  Real* fb = sm + C::OFF_FB;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + (C::BYTES - C::NSLOT * 8));
  if (smem_u32(smem_raw) & 127u) {
    if (threadIdx.x == 0) atomicOr(src.params(0).status, ST_TMA_TIMEOUT);
    return;
  }
  const int tid = threadIdx.x;
  constexpr bool F32 = sizeof(Real) == 4;
  if (tid == 0) {
    for (int s = 0; s < C::NSLOT; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  unsigned phase_bits = 0, pending = 0;
  auto U = [&](int pl, int r, int c) -> Real& { return uring[pmod(pl, C::NSLOT) * C::SLOT + r * W + c]; };
  auto T = [&](int pl, int r, int c) -> Real& { return tring[pmod(pl, 3) * PL + r * W + c]; };
  auto Ph = [&](int pl, int a, int r, int c) -> Real& { return phring[(pmod(pl, 3) * 3 + a) * PL + r * W + c]; };

  const bool is_out = tid < TX * TY;
  const int otx = tid % TX, oty = tid / TX;
  const int ntiles = src.total();
  bool ok = true;
  for (int gtile = blockIdx.x; gtile < ntiles && ok; gtile += gridDim.x) {
    const int inst = src.instance(gtile);
    const HeatParams<Real>& p = src.params(inst);
    if (p.active && !*p.active) continue;  // this grid's clock passed t_end
    const CUtensorMap* tmap = src.map(inst);
    const int tile = src.local(gtile, inst);
    const Layout& L = p.lay;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const Real rcp = Real(p.rho_cp), kk = Real(p.k), qsrc = Real(p.q), ircp = Real(p.inv_rho_cp);
    const Real dt = Real(*p.dt);
    if (tid == 0) tma_prefetch_desc(tmap);
    const int x0 = (tile % p.ntx) * TX, y0 = ((tile / p.ntx) % p.nty) * TY;
    const int Z0 = 1 + (tile / (p.ntx * p.nty)) * p.zchunk;
    const int Zl = min(Z0 + p.zchunk - 1, nz);
    const int Pfirst = Z0 - HH, Plast = Zl + HH, Kfirst = Z0 - 2 * HH;
    const int oi = x0 + otx, oj = y0 + oty;
    const bool out_valid = is_out && oi < nx && oj < ny;
    Real zs = Real(0), Fzp = Real(0), Fzn = Real(0);
    const Real S3c = out_valid ? G::S3(p.met, oi, oj) : Real(0);
    auto issue = [&](int pl) {
      const int s = pmod(pl, C::NSLOT);
      pending |= 1u << s;
      fence_proxy_async();
      mbar_arrive_expect_tx(&bars[s], C::TX_BYTES + p.extra_tx);
      tma_load_4d(&uring[s * C::SLOT], tmap, &bars[s], x0 - 3 + L.padx, y0 + 1 - HH, pl, 0);
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
      // U0 and acc of this plane's output cell, loaded now so that the rest
      // of the step hides their latency
      Real eu0 = Real(0), eacc = Real(0);
      if (K >= Z0 && out_valid) {
        const long long g0 = L.idx(0, K, oj + 1, oi + 1);
        if (needs_u0<Real>(p.coef) && !p.coef.u0_is_input) eu0 = p.u0[g0];
        if (needs_acc(p.coef)) eacc = p.acc[g0];
      }
      // T on the newest plane (heat.py:74).  T = U / (rho cp) is linear in U,
      // so the float32 path differences the U ring directly and folds
      // 1/(rho cp) into the gradient factor (no T ring, no barrier); float64
      // keeps the reference's T = U / (rho cp) first.
      if constexpr (!F32) {
        const int pl = K + HH;
        const Real* ub = uring + pmod(pl, C::NSLOT) * C::SLOT;
        Real* tb = tring + pmod(pl, 3) * PL;
        for (int it = tid; it < C::ROWS * (TX + 6); it += NT) {
          const int o = (it / (TX + 6)) * W + 1 + it % (TX + 6);
          tb[o] = ub[o] / rcp;
        }
        __syncthreads();
      }
      // phi = -k grad T on plane K+HH-1 (heat.py:85-95), zero on ghosts, over
      // the tile plus PH = HH-1 cells (what the x1/x2 face states read)
      if (K >= Z0 - 2 * HH + 2) {
        constexpr int PH = HH - 1;
        const int pl = K + HH - 1, k = pl - 1;
        const bool zg = k < 0 || k >= nz;
        const Real* tm = F32 ? uring + pmod(pl - 1, C::NSLOT) * C::SLOT : tring + pmod(pl - 1, 3) * PL;
        const Real* t0 = F32 ? uring + pmod(pl, C::NSLOT) * C::SLOT : tring + pmod(pl, 3) * PL;
        const Real* tp = F32 ? uring + pmod(pl + 1, C::NSLOT) * C::SLOT : tring + pmod(pl + 1, 3) * PL;
        Real* pw = phring + pmod(pl, 3) * 3 * PL;
        for (int it = tid; it < (TY + 2 * PH) * (TX + 2 * PH); it += NT) {
          const int r = HH - PH + it / (TX + 2 * PH), c = 4 - PH + it % (TX + 2 * PH);
          const int i = x0 + c - 4, j = y0 + r - HH;
          Real f0 = Real(0), f1 = Real(0), f2 = Real(0);
          if (!(zg || i < 0 || i >= nx || j < 0 || j >= ny)) {
            const int o = r * W + c;
            if constexpr (F32) {
              const Real h = -0.5f * kk * ircp;  // the ring holds U = rho cp T
              f0 = (t0[o + 1] - t0[o - 1]) * (h * inv_len<Real, COORD, 0>(p.met, i, j, k));
              f1 = (t0[o + W] - t0[o - W]) * (h * inv_len<Real, COORD, 1>(p.met, i, j, k));
              f2 = (tp[o] - tm[o]) * (h * inv_len<Real, COORD, 2>(p.met, i, j, k));
            } else {
              const Real l1 = G::L1(p.met, i, j, k), l2 = G::L2(p.met, i, j, k), l3 = G::L3(p.met, i, j, k);
              f0 = (-kk) * ((t0[o + 1] - t0[o - 1]) / (Real(2) * l1));
              f1 = (-kk) * ((t0[o + W] - t0[o - W]) / (Real(2) * l2));
              f2 = (-kk) * ((tp[o] - tm[o]) / (Real(2) * l3));
            }
          }
          const int o = r * W + c;
          pw[o] = f0;
          pw[PL + o] = f1;
          pw[2 * PL + o] = f2;
        }
      }
      __syncthreads();
      // x3: slope of phi_3 at K+1 (MUSCL) and the face flux at K+1/2
      if (K >= Z0 - 2 && is_out) {
        const int r = oty + HH, c = otx + 4;
        Real zn = Real(0);
        if constexpr (LIM != LIM_PC) {
          const bool ghost = (K + 1 <= 0 || K + 1 >= nz + 1);
          if (!ghost && out_valid)
            zn = muscl_slope<LIM>(Ph(K, 2, r, c), Ph(K + 1, 2, r, c), Ph(K + 2, 2, r, c), G::L3(p.met, oi, oj, K));
        }
        if (K >= Z0 - 1) {
          const Real fl = Ph(K, 2, r, c) + zs / Real(2);
          const Real fr = Ph(K + 1, 2, r, c) - zn / Real(2);
          Fzp = Fzn;
          Fzn = (Real(0) + (fl + fr) / Real(2)) * S3c;
        }
        zs = zn;
      }
      if (K < Z0) { __syncthreads(); continue; }
      const int kK = K - 1;
      if constexpr (LIM == LIM_PC) {
        // Piecewise-constant faces: phi_L, phi_R are the cell values, so each
        // output cell forms its four in-plane face fluxes straight from the
        // phi ring (no exchange phases).
        if (out_valid) {
          const Real* p0 = phring + pmod(K, 3) * 3 * PL + (oty + HH) * W + otx + 4;  // phi_1 at the cell
          const Real* p1 = p0 + PL;                                                   // phi_2
          const Real Fxm = (Real(0) + (p0[-1] + p0[0]) / Real(2)) * G::S1(p.met, oi, oj, kK);
          const Real Fxp = (Real(0) + (p0[0] + p0[1]) / Real(2)) * G::S1(p.met, oi + 1, oj, kK);
          const Real Fym = (Real(0) + (p1[-W] + p1[0]) / Real(2)) * G::S2(p.met, oi, oj, kK);
          const Real Fyp = (Real(0) + (p1[0] + p1[W]) / Real(2)) * G::S2(p.met, oi, oj + 1, kK);
          const Real sum = ((((Fxp - Fxm) + Fyp) - Fym) + Fzn) - Fzp;
          Real k;
          if constexpr (F32) k = (-sum) * rcp_approx(G::V(p.met, oi, oj, kK)) + qsrc;
          else k = (-sum) / G::V(p.met, oi, oj, kK) + qsrc;
          const long long gi = L.idx(0, K, oj + 1, oi + 1);
          const Real ucur = U(K, oty + HH, otx + 4);
          const Real u0v = (needs_u0<Real>(p.coef) && p.coef.u0_is_input) ? ucur : eu0, accv = eacc;
          const Real o = stage_combine(p.coef, dt, k, ucur, u0v, accv);
          p.out[gi] = o;
          if (p.coef.accmode != ACC_NONE) p.acc[gi] = acc_update(p.coef, dt, k, u0v, accv);
          if (!isfinite(o)) atomicOr(p.status, ST_NONFINITE);
        }
        continue;
      }
      // x1 faces of plane K
      for (int it = tid; it < TY * (TX + 2); it += NT) {
        const int ty = it / (TX + 2), tx = it % (TX + 2) - 1;
        const int r = ty + HH, c = tx + 4, i = x0 + tx, j = y0 + ty;
        const Real f0 = Ph(K, 0, r, c);
        Real s = Real(0);
        if constexpr (LIM != LIM_PC) {
          if (i >= 0 && i < nx && j < ny) s = muscl_slope<LIM>(Ph(K, 0, r, c - 1), f0, Ph(K, 0, r, c + 1), G::L1(p.met, i, j, kK));
        }
        const int o = ty * (TX + 2) + tx + 1;
        fL[o] = f0 + s / Real(2);
        fR[o] = f0 - s / Real(2);
      }
      __syncthreads();
      for (int it = tid; it < TY * (TX + 1); it += NT) {
        const int ty = it / (TX + 1), fx = it % (TX + 1), fi = x0 + fx, j = y0 + ty;
        Real F = Real(0);
        if (fi <= nx && j < ny) {
          const int o = ty * (TX + 2) + fx;
          F = (Real(0) + (fL[o] + fR[o + 1]) / Real(2)) * G::S1(p.met, fi, j, kK);
        }
        fb[ty * (TX + 1) + fx] = F;
      }
      __syncthreads();
      Real Fxm = Real(0), Fxp = Real(0);
      if (is_out) { Fxm = fb[oty * (TX + 1) + otx]; Fxp = fb[oty * (TX + 1) + otx + 1]; }
      // x2 faces
      for (int it = tid; it < (TY + 2) * TX; it += NT) {
        const int ty = it / TX - 1, tx = it % TX;
        const int r = ty + HH, c = tx + 4, i = x0 + tx, j = y0 + ty;
        const Real f0 = Ph(K, 1, r, c);
        Real s = Real(0);
        if constexpr (LIM != LIM_PC) {
          if (i < nx && j >= 0 && j < ny) s = muscl_slope<LIM>(Ph(K, 1, r - 1, c), f0, Ph(K, 1, r + 1, c), G::L2(p.met, i, j, kK));
        }
        const int o = (ty + 1) * TX + tx;
        fL[o] = f0 + s / Real(2);
        fR[o] = f0 - s / Real(2);
      }
      __syncthreads();
      for (int it = tid; it < (TY + 1) * TX; it += NT) {
        const int fy = it / TX, tx = it % TX, fj = y0 + fy, i = x0 + tx;
        Real F = Real(0);
        if (fj <= ny && i < nx) {
          const int o = fy * TX + tx;
          F = (Real(0) + (fL[o] + fR[o + TX]) / Real(2)) * G::S2(p.met, i, fj, kK);
        }
        fb[fy * TX + tx] = F;
      }
      __syncthreads();
      if (out_valid) {
        const Real Fym = fb[oty * TX + otx], Fyp = fb[(oty + 1) * TX + otx];
        const Real sum = ((((Fxp - Fxm) + Fyp) - Fym) + Fzn) - Fzp;
        Real k;
        if constexpr (F32) k = (-sum) * rcp_approx(G::V(p.met, oi, oj, kK)) + qsrc;
        else k = (-sum) / G::V(p.met, oi, oj, kK) + qsrc;
        const long long gi = L.idx(0, K, oj + 1, oi + 1);
        const Real ucur = U(K, oty + HH, otx + 4);
        const Real u0v = (needs_u0<Real>(p.coef) && p.coef.u0_is_input) ? ucur : eu0, accv = eacc;
        const Real o = stage_combine(p.coef, dt, k, ucur, u0v, accv);
        p.out[gi] = o;
        if (p.coef.accmode != ACC_NONE) p.acc[gi] = acc_update(p.coef, dt, k, u0v, accv);
        if (!isfinite(o)) atomicOr(p.status, ST_NONFINITE);
      }
    }
    __syncthreads();  // the next tile's first loads reuse every ring slot
  }
  if (!ok && tid == 0)
    for (int s = 0; s < C::NSLOT; ++s)
      if ((pending >> s) & 1u) mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, src.params(0).drain_ns);
}

}  // namespace fvm
