// Float32 cartesian viscous Navier-Stokes stage kernel with register-blocked
// columns: the layout of stage_ns_strip.cuh plus the Stokes stress
// (navier_stokes.py:102-142, zero in ghost cells) reconstructed with U and P
// (9 fields per face direction) and the centred diffusive flux
// (diffusive_solvers.py:11-30, navier_stokes.py:217-277).
//
// Tile: 32 columns x TY = NW*R rows; output warp w owns rows w*R .. w*R+R-1,
// the halo warp forms the x1 data outside the warps and the border cells of
// the P / stress planes.  Halo HH = 3 (the stress at K+2 needs v at K+3).
//
// Per step K (ghosted output plane K; ring planes K..K+2 resident, K+3
// arriving):
//   1. thread 0 issues plane K+3 into the slot of plane K-1 and the staged
//      U0 / accumulator tile of plane K;
//   2. x2/x1 sweep of plane K in registers (U, P and the stress row of each
//      face axis); the halo warp forms the x1 halo data of plane K+1;
//   3. wait for plane K+3; v = m / rho of plane K+3 over the tile + 3;
//      block barrier;
//   4. P and the stress of plane K+2 over the tile + 2 (own cells by their
//      owners, kept in registers for x3; border cells by the halo warp);
//   5. x3 slope of plane K+1 and the flux at K+1/2 (left state and the flux
//      at K-1/2 carried in registers);
//   6. divergence, gravity, stage combination, stores; block barrier.
// The first step of a tile (K = Z0 - 3) only fills v, P and the stress of
// planes Z0-2 and Z0-1.
#pragma once
#include "stage_ns_strip.cuh"

namespace fvm {

template <int R, int NW>
struct NsStripViscCfg {
  static constexpr int TX = 32, TY = R * NW;
  static constexpr int NO = 32 * NW;
  static constexpr int NT = NO + 32;
  static constexpr int NV = 5, NF = 9, HH = 3;
  static constexpr int W = 40;  // U / v ring column c <-> tile x offset c - 4
  static constexpr int ROWS = TY + 2 * HH;
  static constexpr int PL = ROWS * W;
  static constexpr int NSLOT = 4;  // planes K, K+1, K+2 resident, K+3 arriving
  static constexpr int SLOT = round_up(NV * PL, 32);
  static constexpr int W2 = TX + 4, R2 = TY + 4, PL2 = W2 * R2;  // P / stress planes: tile + 2
  static constexpr int NBORDER = 4 * W2 + 4 * TY;
  static constexpr int VW = TX + 6, VR = TY + 6, NVC = VW * VR;  // v region: tile + 3
  static constexpr int STG = NV * TY * TX;
  static constexpr int OFF_U = 0;
  static constexpr int OFF_V = OFF_U + NSLOT * SLOT;  // [slot][component][PL]
  static constexpr int OFF_P = OFF_V + 3 * 3 * PL;
  static constexpr int OFF_T = OFF_P + 3 * PL2;       // [slot][component][PL2]
  static constexpr int OFF_HL = OFF_T + 3 * 6 * PL2;
  static constexpr int OFF_FR = OFF_HL + 2 * NF * TY;
  static constexpr int END = OFF_FR + 2 * NV * TY;
  static constexpr int NBAR = NSLOT + 1;
  static constexpr int BAR_BYTES = round_up(END * 4, 8);
  static constexpr int STG_OFF_BYTES = round_up(BAR_BYTES + NBAR * 8, 128);
  static constexpr unsigned TX_BYTES = NV * PL * 4;
  static constexpr unsigned STG_BYTES = STG * 4;
  static constexpr int bytes(int nbuf) { return STG_OFF_BYTES + nbuf * (int)STG_BYTES; }
  static_assert(2 * TY <= 32, "one halo lane per tile row and task");
  static_assert((SLOT * 4) % 128 == 0 && (STG_BYTES % 128) == 0, "TMA destinations need 128-byte alignment");
};

// Stress components stored as [t11, t22, t33, t12, t13, t23]; the row of the
// face axis D (tau_D1, tau_D2, tau_D3) is components TI<D>.
template <int D>
__device__ __forceinline__ constexpr int tau_row(int c) {
  return D == 0 ? (c == 0 ? 0 : (c == 1 ? 3 : 4)) : (D == 1 ? (c == 0 ? 3 : (c == 1 ? 1 : 5)) : (c == 0 ? 4 : (c == 1 ? 5 : 2)));
}

// Riemann flux + centred diffusive flux along axis D from face states
// q = {rho, m1, m2, m3, E, P, tau_D1, tau_D2, tau_D3}.
template <int D, int RIEM>
__device__ __forceinline__ void strip_flux_visc(const float* qL, const float* qR, float gam, float* F) {
  const float irL = rcp_approx(qL[0]), irR = rcp_approx(qR[0]);
  float vL[3], vR[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    vL[c] = qL[1 + c] * irL;
    vR[c] = qR[1 + c] * irR;
  }
  const float cL = sqrt_approx((gam * qL[5]) * irL), cR = sqrt_approx((gam * qR[5]) * irR);
  float FL[5], FR[5];
  FL[0] = qL[1 + D];
  FR[0] = qR[1 + D];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    FL[1 + c] = qL[1 + c] * vL[D];
    FR[1 + c] = qR[1 + c] * vR[D];
  }
  FL[1 + D] += qL[5];
  FR[1 + D] += qR[5];
  FL[4] = (qL[4] + qL[5]) * vL[D];
  FR[4] = (qR[4] + qR[5]) * vR[D];
  if constexpr (RIEM == RIEM_HLL) {
    const float sl = fminf(fminf(vL[D] - cL, vR[D] - cR), 0.f);
    const float sr = fmaxf(fmaxf(vL[D] + cL, vR[D] + cR), 0.f);
    const float rd = rcp_approx(fmaxf(sr - sl, 1e-30f));
    const float a = sr * rd, b = -sl * rd, c = (sl * sr) * rd;
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = fmaf(a, FL[v], fmaf(b, FR[v], c * (qR[v] - qL[v])));
  } else {
    const float h = 0.5f * fmaxf(fabsf(vL[D]) + cL, fabsf(vR[D]) + cR);
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = fmaf(0.5f, FL[v] + FR[v], -h * (qR[v] - qL[v]));
  }
  // diffusive flux -tau_D. and -(tau_D . v), averaged over the two states
#pragma unroll
  for (int c = 0; c < 3; ++c) F[1 + c] -= 0.5f * (qL[6 + c] + qR[6 + c]);
  const float eL = fmaf(qL[6], vL[0], fmaf(qL[7], vL[1], qL[8] * vL[2]));
  const float eR = fmaf(qR[6], vR[0], fmaf(qR[7], vR[1], qR[8] * vR[2]));
  F[4] -= 0.5f * (eL + eR);
}

template <int LIM, int RIEM, int R, int NW, int MINB>
__global__ void __launch_bounds__(NsStripViscCfg<R, NW>::NT, MINB)
    ns_strip_visc_kernel(const __grid_constant__ NsStripSource src) {
  using C = NsStripViscCfg<R, NW>;
  constexpr int TX = C::TX, TY = C::TY, W = C::W, PL = C::PL, HH = C::HH, NF = C::NF, W2 = C::W2;
  constexpr int PL2 = C::PL2, NT = C::NT;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* sm = reinterpret_cast<float*>(smem_raw);
  float* uring = sm + C::OFF_U;
  float* vring = sm + C::OFF_V;
  float* pring = sm + C::OFF_P;
  float* tring = sm + C::OFF_T;
  float* hl = sm + C::OFF_HL;
  float* fr = sm + C::OFF_FR;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + C::BAR_BYTES);
  uint64_t* gbar = bars + C::NSLOT;
  float* gst = reinterpret_cast<float*>(smem_raw + C::STG_OFF_BYTES);
  const NsParams<float>& p = src.p;

  if (smem_u32(smem_raw) & 127u) {
    if (threadIdx.x == 0) atomicOr(p.status, ST_TMA_TIMEOUT);
    return;
  }
  if (p.active && !*p.active) return;
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < C::NBAR; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  unsigned phase_bits = 0, pending = 0;
  const Layout& L = p.lay;
  const Metric<float>& m = p.met;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const float gam = float(p.gamma), gm1 = float(p.gamma) - 1.f, mu = float(p.mu);
  const float dt = float(*p.dt);
  const float gx = float(p.g1), gy = float(p.g2), gz = float(p.g3);
  const bool need_u0 = needs_u0<float>(p.coef) && !p.coef.u0_is_input;
  const bool need_acc = needs_acc(p.coef);
  const unsigned stg_bytes = (need_u0 ? C::STG_BYTES : 0u) + (need_acc ? C::STG_BYTES : 0u);
  const float* gu0 = gst;
  const float* gacc = gst + (need_u0 ? C::STG : 0);
  const int w = tid >> 5, lane = tid & 31;
  const bool is_out = w < NW;
  if (tid == 0) {
    tma_prefetch_desc(&src.tmap);
    if (need_u0) tma_prefetch_desc(&src.u0map);
    if (need_acc) tma_prefetch_desc(&src.accmap);
  }
  const int ntiles = p.ntx * p.nty * p.nzc;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int x0 = (tile % p.ntx) * TX, y0 = ((tile / p.ntx) % p.nty) * TY;
    const int Z0 = 1 + (tile / (p.ntx * p.nty)) * p.zchunk;
    const int Zl = min(Z0 + p.zchunk - 1, nz);
    const int Kfirst = Z0 - 3, Plast = Zl + HH;
    const int i = x0 + lane;
    const float idx = (is_out && i < nx) ? __ldg(m.inv_dx1 + i) : 0.f;

    auto issue = [&](int pl) {
      const int s = pmod(pl, C::NSLOT);
      pending |= 1u << s;
      fence_proxy_async();
      mbar_arrive_expect_tx(&bars[s], C::TX_BYTES + p.extra_tx);
      tma_load_4d(&uring[s * C::SLOT], &src.tmap, &bars[s], x0 - 3 + L.padx, y0 + 1 - HH, pl, 0);
    };
    if (tid == 0)
      for (int pl = Kfirst; pl <= Kfirst + 3; ++pl) issue(pl);

    // v = m / rho of one ring plane over the tile + 3 (all threads)
    auto velocity = [&](int pl) {
      const float* ub = uring + pmod(pl, C::NSLOT) * C::SLOT;
      float* vb = vring + pmod(pl, 3) * 3 * PL;
      for (int it = tid; it < C::NVC; it += NT) {
        const int o = (it / C::VW) * W + 1 + it % C::VW;  // rows -3..TY+2, columns -3..TX+2
        const float ir = rcp_approx(ub[o]);
        vb[o] = ub[PL + o] * ir;
        vb[PL + o] = ub[2 * PL + o] * ir;
        vb[2 * PL + o] = ub[3 * PL + o] * ir;
      }
    };
    // P and the six stress components of plane pl at tile offset (x, y),
    // written to the rings; returns {P, t13, t23, t33} for the x3 phase
    auto closure_at = [&](int pl, int x, int y, float* out4) {
      const int o = (y + HH) * W + x + 4, op = (y + 2) * W2 + x + 2;
      const float* ub = uring + pmod(pl, C::NSLOT) * C::SLOT;
      const float Pv = strip_pressure(ub + o, PL, gm1);
      pring[pmod(pl, 3) * PL2 + op] = Pv;
      const int ii = x0 + x, jj = y0 + y, kk = pl - 1;
      float t[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (!(kk < 0 || kk >= nz || ii < 0 || ii >= nx || jj < 0 || jj >= ny)) {
        const float* vm = vring + pmod(pl - 1, 3) * 3 * PL;
        const float* v0 = vring + pmod(pl, 3) * 3 * PL;
        const float* vp = vring + pmod(pl + 1, 3) * 3 * PL;
        const float h1 = 0.5f * __ldg(m.inv_dx1 + ii), h2 = 0.5f * __ldg(m.inv_dx2 + jj);
        const float h3 = 0.5f * __ldg(m.inv_dx3 + kk);
        float g[3][3];  // g[c][a] = d v_c / d x_a
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const int oc = c * PL + o;
          g[c][0] = (v0[oc + 1] - v0[oc - 1]) * h1;
          g[c][1] = (v0[oc + W] - v0[oc - W]) * h2;
          g[c][2] = (vp[oc] - vm[oc]) * h3;
        }
        const float tt = 2.f / 3.f;
        const float divv = (g[0][0] + g[1][1]) + g[2][2];
        t[0] = mu * (2.f * g[0][0] - tt * divv);
        t[1] = mu * (2.f * g[1][1] - tt * divv);
        t[2] = mu * (2.f * g[2][2] - tt * divv);
        t[3] = mu * (g[0][1] + g[1][0]);
        t[4] = mu * (g[0][2] + g[2][0]);
        t[5] = mu * (g[1][2] + g[2][1]);
      }
      float* tb = tring + pmod(pl, 3) * 6 * PL2 + op;
#pragma unroll
      for (int c = 0; c < 6; ++c) tb[c * PL2] = t[c];
      out4[0] = Pv;
      out4[1] = t[4];
      out4[2] = t[5];
      out4[3] = t[2];
    };
    // P and stress of plane pl over the tile + 2: own cells by the output
    // threads (results kept in `own`), border cells by the halo warp
    auto closure_plane = [&](int pl, float (*own)[4]) {
      if (is_out) {
#pragma unroll
        for (int r = 0; r < R; ++r) closure_at(pl, lane, w * R + r, own[r]);
      } else {
        for (int b = lane; b < C::NBORDER; b += 32) {
          int x, y;
          if (b < 2 * W2) {
            y = b / W2 - 2;
            x = b % W2 - 2;
          } else if (b < 4 * W2) {
            y = TY + (b - 2 * W2) / W2;
            x = (b - 2 * W2) % W2 - 2;
          } else {
            const int c = b - 4 * W2;
            y = c >> 2;
            x = (c & 3) < 2 ? (c & 3) - 2 : (c & 3) + 30;
          }
          float dummy[4];
          closure_at(pl, x, y, dummy);
        }
      }
    };

    float qlz[R][NF], fzp[R][5];
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int f = 0; f < NF; ++f) qlz[r][f] = 0.f;
#pragma unroll
      for (int v = 0; v < 5; ++v) fzp[r][v] = 0.f;
    }

    for (int K = Kfirst; K <= Zl; ++K) {
      const bool outstep = K >= Z0;
      const float* uK = uring + pmod(K, C::NSLOT) * C::SLOT;
      const float* uK1 = uring + pmod(K + 1, C::NSLOT) * C::SLOT;
      const float* uK2 = uring + pmod(K + 2, C::NSLOT) * C::SLOT;
      const float* pK = pring + pmod(K, 3) * PL2;
      const float* pK1 = pring + pmod(K + 1, 3) * PL2;
      const float* tK = tring + pmod(K, 3) * 6 * PL2;
      const float* tK1 = tring + pmod(K + 1, 3) * 6 * PL2;
      // ------------------------------------------------------------ 1 ----
      if (tid == 0) {
        if (K > Kfirst && K + 3 <= Plast) issue(K + 3);
        if (outstep && stg_bytes) {
          pending |= 1u << C::NSLOT;
          fence_proxy_async();
          mbar_arrive_expect_tx(gbar, stg_bytes);
          const int gxc = x0 + 1 + L.padx;
          if (need_u0) tma_load_4d(gst, &src.u0map, gbar, gxc, y0 + 1, K, 0);
          if (need_acc) tma_load_4d(gst + (need_u0 ? C::STG : 0), &src.accmap, gbar, gxc, y0 + 1, K, 0);
        }
      }
      float kv[R][5];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int v = 0; v < 5; ++v) kv[r][v] = 0.f;
      // ------------------------------------------------------------ 2 ----
      if (is_out) {
        if (outstep) {
          const int par = K & 1;
          const int jb = y0 + w * R;
          // U, P and the stress row of axis D at tile offset (tx, ty) of plane K
          auto ldf1 = [&](float* f, int ty, int tx) {
            const int o = (ty + HH) * W + tx + 4, op = (ty + 2) * W2 + tx + 2;
#pragma unroll
            for (int v = 0; v < 5; ++v) f[v] = uK[v * PL + o];
            f[5] = pK[op];
#pragma unroll
            for (int c = 0; c < 3; ++c) f[6 + c] = tK[tau_row<1>(c) * PL2 + op];
          };
          float fa[NF], fb[NF], fc[NF], ql[NF];
          ldf1(fa, w * R - 2, lane);
          ldf1(fb, w * R - 1, lane);
#pragma unroll
          for (int t = 0; t <= R + 1; ++t) {
            const int ty = w * R - 1 + t;
            const int j = jb - 1 + t;
            ldf1(fc, ty + 1, lane);
            const bool yghost = j < 0 || j >= ny;
            float s[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) s[f] = yghost ? 0.f : strip_slope<LIM>(fb[f] - fa[f], fc[f] - fb[f]);
            if (t >= 1) {
              float qr[NF], F[5];
#pragma unroll
              for (int f = 0; f < NF; ++f) qr[f] = fmaf(-0.5f, s[f], fb[f]);
              strip_flux_visc<1, RIEM>(ql, qr, gam, F);
              if (t >= 2) {
                const float idym = __ldg(m.inv_dx2 + min(max(j - 1, 0), ny - 1));
#pragma unroll
                for (int v = 0; v < 5; ++v) kv[t - 2][v] = fmaf(F[v], idym, kv[t - 2][v]);
              }
              if (t <= R) {
                const float idy = __ldg(m.inv_dx2 + min(j, ny - 1));
#pragma unroll
                for (int v = 0; v < 5; ++v) kv[t - 1][v] = fmaf(-F[v], idy, kv[t - 1][v]);
              }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) ql[f] = fmaf(0.5f, s[f], fb[f]);
            if (t >= 1 && t <= R) {
              // x1 for own row r = t - 1: fields with the stress row of axis 1
              const int r = t - 1;
              auto ldf0 = [&](float* f, int tx) {
                const int o = (ty + HH) * W + tx + 4, op = (ty + 2) * W2 + tx + 2;
#pragma unroll
                for (int v = 0; v < 5; ++v) f[v] = uK[v * PL + o];
                f[5] = pK[op];
#pragma unroll
                for (int c = 0; c < 3; ++c) f[6 + c] = tK[tau_row<0>(c) * PL2 + op];
              };
              float fm[NF], f0[NF], fp[NF], qlx[NF], qrx[NF], F[5];
              ldf0(fm, lane - 1);
              ldf0(f0, lane);
              ldf0(fp, lane + 1);
              const bool xghost = i >= nx;
#pragma unroll
              for (int f = 0; f < NF; ++f) {
                const float s1 = xghost ? 0.f : strip_slope<LIM>(f0[f] - fm[f], fp[f] - f0[f]);
                const float su = __shfl_up_sync(0xffffffffu, s1, 1);
                const float sl = lane == 0 ? hl[(par * NF + f) * TY + ty] : su;
                qlx[f] = fmaf(0.5f, sl, fm[f]);
                qrx[f] = fmaf(-0.5f, s1, f0[f]);
              }
              strip_flux_visc<0, RIEM>(qlx, qrx, gam, F);
#pragma unroll
              for (int v = 0; v < 5; ++v) {
                const float fd = __shfl_down_sync(0xffffffffu, F[v], 1);
                const float fe = lane == 31 ? fr[(par * 5 + v) * TY + ty] : fd;
                kv[r][v] = fmaf(fe - F[v], idx, kv[r][v]);
              }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) { fa[f] = fb[f]; fb[f] = fc[f]; }
          }
        }
      } else {
        // --------------------------------------------------- halo warp ----
        const int Kh = K + 1;
        const int row = lane < TY ? lane : lane - TY;
        const int j = y0 + row;
        if (Kh >= Z0 && Kh <= Zl && lane < 2 * TY && j < ny) {
          const int hpar = Kh & 1;
          auto ldh = [&](float* f, int tx) {
            const int o = (row + HH) * W + tx + 4, op = (row + 2) * W2 + tx + 2;
#pragma unroll
            for (int v = 0; v < 5; ++v) f[v] = uK1[v * PL + o];
            f[5] = pK1[op];
#pragma unroll
            for (int c = 0; c < 3; ++c) f[6 + c] = tK1[tau_row<0>(c) * PL2 + op];
          };
          if (lane < TY) {
            float a[NF], b[NF], c[NF];
            ldh(a, -2);
            ldh(b, -1);
            ldh(c, 0);
#pragma unroll
            for (int f = 0; f < NF; ++f)
              hl[(hpar * NF + f) * TY + row] = x0 == 0 ? 0.f : strip_slope<LIM>(b[f] - a[f], c[f] - b[f]);
          } else {
            float F[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
            if (x0 + TX <= nx) {
              float a[NF], b[NF], c[NF], d[NF], qlh[NF], qrh[NF];
              ldh(a, TX - 2);
              ldh(b, TX - 1);
              ldh(c, TX);
              ldh(d, TX + 1);
              const bool g32 = x0 + TX >= nx;
#pragma unroll
              for (int f = 0; f < NF; ++f) {
                const float sm1 = strip_slope<LIM>(b[f] - a[f], c[f] - b[f]);
                const float s0 = g32 ? 0.f : strip_slope<LIM>(c[f] - b[f], d[f] - c[f]);
                qlh[f] = fmaf(0.5f, sm1, b[f]);
                qrh[f] = fmaf(-0.5f, s0, c[f]);
              }
              strip_flux_visc<0, RIEM>(qlh, qrh, gam, F);
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) fr[(hpar * 5 + v) * TY + row] = F[v];
          }
        }
      }
      // ------------------------------------------------------------ 3 ----
      // each thread waits for the plane itself; the barrier after v of the
      // new plane also takes the block out if any wait ran out
      {
        bool got = true;
        for (int pl = (K == Kfirst ? Kfirst : K + 3); pl <= K + 3; ++pl) {
          const int s = pmod(pl, C::NSLOT);
          const bool g = got && mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.wait_ns);
          if (g) {
            phase_bits ^= 1u << s;
            if (tid == 0) pending &= ~(1u << s);
          }
          got = g;
        }
        if (K != Kfirst && got) velocity(K + 3);
        if (!__syncthreads_and(got)) {
          if (tid == 0) atomicOr(p.status, ST_TMA_TIMEOUT);
          ok = false;
          break;
        }
      }
      float own[R][4];  // P, t13, t23, t33 of plane K+2 at the own cells
      if (K == Kfirst) {
        // v of planes K..K+2, then P / stress of plane K+1; v of plane K+3
        // (into plane K's slot), then P / stress of plane K+2
        velocity(K);
        velocity(K + 1);
        velocity(K + 2);
        __syncthreads();
        float skip[R][4];
        closure_plane(K + 1, skip);
        __syncthreads();
        velocity(K + 3);
        __syncthreads();
      }
      // ------------------------------------------------------------ 4 ----
      closure_plane(K + 2, own);
      bool step_ok = true;
      if (is_out) {
        // ------------------------------------------------------------ 5 ----
        const bool zghost = K + 1 <= 0 || K + 1 >= nz + 1;
        const bool zslope = K >= Z0 - 2, zface = K >= Z0 - 1;
        const float idz = outstep ? __ldg(m.inv_dx3 + (K - 1)) : 0.f;
        if (zslope) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int ty = w * R + r;
            const int o = (ty + HH) * W + lane + 4, op = (ty + 2) * W2 + lane + 2;
            float qr[NF], qn[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
              float a0, a1, a2;
              if (f < 5) {
                a0 = uK[f * PL + o];
                a1 = uK1[f * PL + o];
                a2 = uK2[f * PL + o];
              } else if (f == 5) {
                a0 = pK[op];
                a1 = pK1[op];
                a2 = own[r][0];
              } else {
                const int c = tau_row<2>(f - 6);
                a0 = tK[c * PL2 + op];
                a1 = tK1[c * PL2 + op];
                a2 = own[r][f - 5];
              }
              const float s = zghost ? 0.f : strip_slope<LIM>(a1 - a0, a2 - a1);
              qr[f] = fmaf(-0.5f, s, a1);
              qn[f] = fmaf(0.5f, s, a1);
            }
            if (zface) {
              float F[5];
              strip_flux_visc<2, RIEM>(qlz[r], qr, gam, F);
#pragma unroll
              for (int v = 0; v < 5; ++v) {
                kv[r][v] = fmaf(F[v] - fzp[r][v], idz, kv[r][v]);
                fzp[r][v] = F[v];
              }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) qlz[r][f] = qn[f];
          }
        }
        // ------------------------------------------------------------ 6 ----
        if (outstep) {
          bool staged_ok = true;
          if (stg_bytes) {
            staged_ok = mbar_wait_bounded(gbar, (phase_bits >> C::NSLOT) & 1u, p.wait_ns);
            if (staged_ok) {
              phase_bits ^= 1u << C::NSLOT;
              if (tid == 0) pending &= ~(1u << C::NSLOT);
            }
          }
          step_ok = staged_ok;
          unsigned bad = staged_ok ? 0u : ST_TMA_TIMEOUT;
          const int jb = y0 + w * R;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int ty = w * R + r, j = jb + r;
            if (i < nx && j < ny && staged_ok) {
              const int o = (ty + HH) * W + lane + 4;
              float q[5];
#pragma unroll
              for (int v = 0; v < 5; ++v) q[v] = uK[v * PL + o];
              const float sg[5] = {0.f, q[0] * gx, q[0] * gy, q[0] * gz, fmaf(gx, q[1], fmaf(gy, q[2], gz * q[3]))};
              const long long g = L.idx(0, K, j + 1, i + 1);
              const int so = ty * TX + lane;
#pragma unroll
              for (int v = 0; v < 5; ++v) {
                const float k = sg[v] - kv[r][v];
                const float u0v = need_u0 ? gu0[v * TY * TX + so] : q[v];
                const float accv = need_acc ? gacc[v * TY * TX + so] : 0.f;
                const long long gi = g + (long long)v * L.var_stride;
                const float o2 = stage_combine(p.coef, dt, k, q[v], u0v, accv);
                p.out[gi] = o2;
                if (p.coef.accmode != ACC_NONE) p.acc[gi] = acc_update(p.coef, dt, k, u0v, accv);
                if (!isfinite(o2)) bad |= ST_NONFINITE;
                if (v == 0 && p.coef.mode != MODE_RHS && !(o2 > 0.f)) bad |= ST_DENSITY;
              }
            }
          }
          if (bad) atomicOr(p.status, bad);
        }
      }
      if (!__syncthreads_and(step_ok)) {
        ok = false;
        break;
      }
    }
  }
  if (!ok && tid == 0) {
    for (int s = 0; s < C::NBAR; ++s)
      if ((pending >> s) & 1u) mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.drain_ns);
  }
}

}  // namespace fvm
