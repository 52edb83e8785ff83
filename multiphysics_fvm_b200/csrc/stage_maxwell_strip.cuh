// Float32 Maxwell stage kernel with register-blocked columns: residual
// (maxwell.py:603-729) + Runge-Kutta stage in one pass, for every coordinate
// system.
//
// Same layout as stage_ns_strip.cuh: a 32 x TY tile, output warp w owns rows
// w*R .. w*R+R-1 of its lane's column, one halo warp.  Per step K (ghosted
// output plane K; ring planes K, K+1 resident, K+2 arriving):
//   1. thread 0 issues plane K+2 and the staged U0 / accumulator tiles;
//   2. x2/x1 sweep of plane K in registers; the halo warp forms the x1 halo
//      data of plane K+1 (slopes left of the tile, fluxes through its right
//      edge);
//   3. wait for plane K+2;
//   4. cleaning residuals r = (div B, div D - rho_c) of plane K+1 on the
//      interior cells of the tile + 1 (maxwell.py:490-512; own cells by their
//      owners, kept in registers, border cells by the halo warp);
//   5. x3 slope of plane K+1 and the flux at K+1/2 (carried state);
//   6. divergence with per-column face-area / volume factors, geometric
//      source (:365-374), Ohmic J = -sigma E (:414-420), cleaning
//      -chi grad r of the edge-padded residuals (:514-528), stage
//      combination, stores; one block barrier.
// The face flux F = (F_L + F_R)/2 - c (q_R - q_L)/2 is Rusanov; HLL with wave
// speeds -c, +c is the same function for Maxwell (riemann_solvers.py:13-89).
// The float32 MC limiter is written as copysign(k m, a + b) with
// m = min(|a + b|/2, 2|a|, 2|b|), k = 1 when a b > 0 and 1/3 otherwise, which
// is the reference's three-sign form (slope_limiters.py:42-73) for every sign
// pattern.
#pragma once
#include "stage_ns_strip.cuh"
#include "stage_maxwell.cuh"

namespace fvm {

template <int R, int NW>
struct MxStripCfg {
  static constexpr int TX = 32, TY = R * NW;
  static constexpr int NO = 32 * NW;
  static constexpr int NT = NO + 32;
  static constexpr int NV = 6, HH = 2;
  static constexpr int W = 40;
  static constexpr int ROWS = TY + 2 * HH, PL = ROWS * W;
  static constexpr int NSLOT = 3;
  static constexpr int SLOT = round_up(NV * PL, 32);
  static constexpr int WR = TX + 2, RR = TY + 2, PLR = WR * RR;  // residual planes: tile + 1
  static constexpr int NBORDER = 2 * WR + 2 * TY;
  static constexpr int STG = NV * TY * TX;
  static constexpr int OFF_U = 0;
  static constexpr int OFF_R = OFF_U + NSLOT * SLOT;   // [slot][field][PLR]
  static constexpr int OFF_HL = OFF_R + 3 * 2 * PLR;   // [parity][var][row]
  static constexpr int OFF_FR = OFF_HL + 2 * NV * TY;  // [parity][var][row]
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

struct MxStripSource {
  CUtensorMap tmap, u0map, accmap;
  MaxwellParams<float> p;
};

template <int LIM>
__device__ __forceinline__ float mx_slope(float a, float b) {
  if constexpr (LIM == LIM_MC) {
    const float s = a + b;
    const float mm = fminf(0.5f * fabsf(s), 2.f * fminf(fabsf(a), fabsf(b)));
    return copysignf(a * b > 0.f ? mm : mm * (1.f / 3.f), s);
  } else {
    return strip_slope<LIM>(a, b);
  }
}

// Face flux along axis D of states q = (B1, B2, B3, D1, D2, D3):
// (F(q_L) + F(q_R))/2 - hc (q_R - q_L) with the curl tensors of H = B/mu and
// E = D/eps (maxwell.py:145-165); ihm = 0.5/mu, ihe = 0.5/eps, hc = c/2.
template <int D>
__device__ __forceinline__ void mx_flux(const float* qL, const float* qR, float ihm, float ihe, float hc, float* F) {
  float s[6], d[6];
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    s[v] = qL[v] + qR[v];
    d[v] = qR[v] - qL[v];
  }
  const float H0 = s[0] * ihm, H1 = s[1] * ihm, H2 = s[2] * ihm;
  const float E0 = s[3] * ihe, E1 = s[4] * ihe, E2 = s[5] * ihe;
  float C[6];
  if constexpr (D == 0) {
    C[0] = 0.f; C[1] = -E2; C[2] = E1; C[3] = 0.f; C[4] = H2; C[5] = -H1;
  } else if constexpr (D == 1) {
    C[0] = E2; C[1] = 0.f; C[2] = -E0; C[3] = -H2; C[4] = 0.f; C[5] = H0;
  } else {
    C[0] = -E1; C[1] = E0; C[2] = 0.f; C[3] = H1; C[4] = -H0; C[5] = 0.f;
  }
#pragma unroll
  for (int v = 0; v < 6; ++v) F[v] = fmaf(-hc, d[v], C[v]);
}

template <int LIM, int COORD, int R, int NW, int MINB>
__global__ void __launch_bounds__(MxStripCfg<R, NW>::NT, MINB)
    mx_strip_kernel(const __grid_constant__ MxStripSource src) {
  using C = MxStripCfg<R, NW>;
  using G = Geo<float, COORD>;
  constexpr int TX = C::TX, TY = C::TY, W = C::W, PL = C::PL, HH = C::HH, NV = C::NV;
  constexpr int WR = C::WR, PLR = C::PLR;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float* sm = reinterpret_cast<float*>(smem_raw);
  float* uring = sm + C::OFF_U;
  float* rring = sm + C::OFF_R;
  float* hl = sm + C::OFF_HL;
  float* fr = sm + C::OFF_FR;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + C::BAR_BYTES);
  uint64_t* gbar = bars + C::NSLOT;
  float* gst = reinterpret_cast<float*>(smem_raw + C::STG_OFF_BYTES);
  const MaxwellParams<float>& p = src.p;
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
  const float mu = float(p.mu), ep = float(p.ep);
  const float ihm = 0.5f / mu, ihe = 0.5f / ep, hc = 0.5f * float(p.c);
  const float imu = 1.f / mu, iep = 1.f / ep;
  const float sigma = float(p.sigma), rho_c = float(p.rho_c), chib = float(p.chi_b), chid = float(p.chi_d);
  const float dt = float(*p.dt);
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
  // divergence of B (f = 0) or D - rho_c (f = 1) at tile offset (x, y) of
  // ring plane K+1 (uK, uK1, uK2 = planes K, K+1, K+2); interior cells only
  auto residual = [&](const float* uK, const float* uK1, const float* uK2, int x, int y, int i, int j, int k,
                      float* rv) {
    const int o = (y + HH) * W + x + 4;
    const float h1 = 0.5f * inv_len<float, COORD, 0>(m, i, j, k);
    const float h2 = 0.5f * inv_len<float, COORD, 1>(m, i, j, k);
    const float h3 = 0.5f * inv_len<float, COORD, 2>(m, i, j, k);
    Lame<float> lm;
    if constexpr (COORD != COORD_CART) lame_at<float, COORD>(m, i, j, lm);
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      const int q0 = 3 * f;
      float dv = ((uK1[q0 * PL + o + 1] - uK1[q0 * PL + o - 1]) * h1 +
                  (uK1[(q0 + 1) * PL + o + W] - uK1[(q0 + 1) * PL + o - W]) * h2) +
                 (uK2[(q0 + 2) * PL + o] - uK[(q0 + 2) * PL + o]) * h3;
      if constexpr (COORD != COORD_CART) {
        dv = ((dv + (uK1[q0 * PL + o] * (lm.dl[0][1] + lm.dl[0][2])) * rcp_approx(lm.h[0])) +
              (uK1[(q0 + 1) * PL + o] * (lm.dl[1][0] + lm.dl[1][2])) * rcp_approx(lm.h[1])) +
             (uK1[(q0 + 2) * PL + o] * (lm.dl[2][0] + lm.dl[2][1])) * rcp_approx(lm.h[2]);
      }
      rv[f] = f == 0 ? dv : dv - rho_c;
    }
  };

  const int ntiles = p.ntx * p.nty * p.nzc;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int x0 = (tile % p.ntx) * TX, y0 = ((tile / p.ntx) % p.nty) * TY;
    const int Z0 = 1 + (tile / (p.ntx * p.nty)) * p.zchunk;
    const int Zl = min(Z0 + p.zchunk - 1, nz);
    const int Kfirst = Z0 - 2, Plast = Zl + HH;
    const int i = x0 + lane, jb = y0 + w * R;
    const int ic = min(i, nx - 1);

    auto issue = [&](int pl) {
      const int s = pmod(pl, C::NSLOT);
      pending |= 1u << s;
      fence_proxy_async();
      mbar_arrive_expect_tx(&bars[s], C::TX_BYTES + p.extra_tx);
      tma_load_4d(&uring[s * C::SLOT], &src.tmap, &bars[s], x0 - 3 + L.padx, y0 + 1 - HH, pl, 0);
    };
    if (tid == 0)
      for (int pl = Kfirst; pl <= Kfirst + 2; ++pl) issue(pl);

    // per-column metric factors of the own cells (k = 0; the x3 length only
    // scales the x3 terms)
    float a1p = 0.f, a1m = 0.f, la = 0.f, lb = 0.f, g1 = 0.f;
    float a2p[R], a2m[R], a3[R], lc[R], g2[R], g3[R];
    if (is_out) {
      const float iv0 = 1.f / G::V(m, ic, 0, 0);
      a1p = G::S1(m, ic + 1, 0, 0) * iv0;
      a1m = G::S1(m, ic, 0, 0) * iv0;
      g1 = 0.5f * __ldg(m.inv_dx1 + ic);
      Lame<float> l0;
      lame_at<float, COORD>(m, ic, 0, l0);
      la = l0.dl[0][1] / l0.h[0];
      lb = l0.dl[0][2] / l0.h[0];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int jc = min(jb + r, ny - 1);
        const float iv = 1.f / G::V(m, ic, jc, 0);
        a2p[r] = G::S2(m, ic, jc + 1, 0) * iv;
        a2m[r] = G::S2(m, ic, jc, 0) * iv;
        a3[r] = G::S3(m, ic, jc) * iv * __ldg(m.dx3);
        Lame<float> lj;
        lame_at<float, COORD>(m, ic, jc, lj);
        lc[r] = lj.dl[1][2] / lj.h[1];
        g2[r] = 0.5f * inv_len<float, COORD, 1>(m, ic, jc, 0);
        g3[r] = 0.5f * inv_len<float, COORD, 2>(m, ic, jc, 0) * __ldg(m.dx3);
      }
    }

    float qlz[R][NV], fzp[R][NV];
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int v = 0; v < NV; ++v) { qlz[r][v] = 0.f; fzp[r][v] = 0.f; }

    for (int K = Kfirst; K <= Zl; ++K) {
      const bool outstep = K >= Z0;
      const float* uK = uring + pmod(K, C::NSLOT) * C::SLOT;
      const float* uK1 = uring + pmod(K + 1, C::NSLOT) * C::SLOT;
      const float* uK2 = uring + pmod(K + 2, C::NSLOT) * C::SLOT;
      const float* rKm = rring + pmod(K - 1, 3) * 2 * PLR;
      const float* rK = rring + pmod(K, 3) * 2 * PLR;
      float* rK1 = rring + pmod(K + 1, 3) * 2 * PLR;
      // ------------------------------------------------------------ 1 ----
      if (tid == 0) {
        if (K > Kfirst && K + 2 <= Plast) issue(K + 2);
        if (outstep && stg_bytes) {
          pending |= 1u << C::NSLOT;
          fence_proxy_async();
          mbar_arrive_expect_tx(gbar, stg_bytes);
          const int gxc = x0 + 1 + L.padx;
          if (need_u0) tma_load_4d(gst, &src.u0map, gbar, gxc, y0 + 1, K, 0);
          if (need_acc) tma_load_4d(gst + (need_u0 ? C::STG : 0), &src.accmap, gbar, gxc, y0 + 1, K, 0);
        }
      }
      float kv[R][NV];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int v = 0; v < NV; ++v) kv[r][v] = 0.f;
      // ------------------------------------------------------------ 2 ----
      if (is_out) {
        if (outstep) {
          const int par = K & 1;
          auto ldf = [&](float* f, int ty, int tx) {
            const int o = (ty + HH) * W + tx + 4;
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = uK[v * PL + o];
          };
          float fa[NV], fb[NV], fc[NV], ql[NV];
          ldf(fa, w * R - 2, lane);
          ldf(fb, w * R - 1, lane);
#pragma unroll
          for (int t = 0; t <= R + 1; ++t) {
            const int ty = w * R - 1 + t;
            const int j = jb - 1 + t;
            ldf(fc, ty + 1, lane);
            const bool yghost = j < 0 || j >= ny;
            float s[NV];
#pragma unroll
            for (int f = 0; f < NV; ++f) s[f] = yghost ? 0.f : mx_slope<LIM>(fb[f] - fa[f], fc[f] - fb[f]);
            if (t >= 1) {
              float qr[NV], F[NV];
#pragma unroll
              for (int f = 0; f < NV; ++f) qr[f] = fmaf(-0.5f, s[f], fb[f]);
              mx_flux<1>(ql, qr, ihm, ihe, hc, F);
              if (t >= 2) {
#pragma unroll
                for (int v = 0; v < NV; ++v) kv[t - 2][v] = fmaf(F[v], a2p[t - 2], kv[t - 2][v]);
              }
              if (t <= R) {
#pragma unroll
                for (int v = 0; v < NV; ++v) kv[t - 1][v] = fmaf(-F[v], a2m[t - 1], kv[t - 1][v]);
              }
            }
#pragma unroll
            for (int f = 0; f < NV; ++f) ql[f] = fmaf(0.5f, s[f], fb[f]);
            if (t >= 1 && t <= R) {
              const int r = t - 1;
              float fm[NV], fp[NV], qlx[NV], qrx[NV], F[NV];
              ldf(fm, ty, lane - 1);
              ldf(fp, ty, lane + 1);
              const bool xghost = i >= nx;
#pragma unroll
              for (int f = 0; f < NV; ++f) {
                const float s1 = xghost ? 0.f : mx_slope<LIM>(fb[f] - fm[f], fp[f] - fb[f]);
                const float su = __shfl_up_sync(0xffffffffu, s1, 1);
                const float sl = lane == 0 ? hl[(par * NV + f) * TY + ty] : su;
                qlx[f] = fmaf(0.5f, sl, fm[f]);
                qrx[f] = fmaf(-0.5f, s1, fb[f]);
              }
              mx_flux<0>(qlx, qrx, ihm, ihe, hc, F);
#pragma unroll
              for (int v = 0; v < NV; ++v) {
                const float fd = __shfl_down_sync(0xffffffffu, F[v], 1);
                const float fe = lane == 31 ? fr[(par * NV + v) * TY + ty] : fd;
                kv[r][v] = fmaf(fe, a1p, fmaf(-F[v], a1m, kv[r][v]));
              }
            }
#pragma unroll
            for (int f = 0; f < NV; ++f) { fa[f] = fb[f]; fb[f] = fc[f]; }
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
            const int o = (row + HH) * W + tx + 4;
#pragma unroll
            for (int v = 0; v < NV; ++v) f[v] = uK1[v * PL + o];
          };
          if (lane < TY) {
            float a[NV], b[NV], c[NV];
            ldh(a, -2);
            ldh(b, -1);
            ldh(c, 0);
#pragma unroll
            for (int f = 0; f < NV; ++f)
              hl[(hpar * NV + f) * TY + row] = x0 == 0 ? 0.f : mx_slope<LIM>(b[f] - a[f], c[f] - b[f]);
          } else {
            float F[NV] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
            if (x0 + TX <= nx) {
              float a[NV], b[NV], c[NV], d[NV], qlh[NV], qrh[NV];
              ldh(a, TX - 2);
              ldh(b, TX - 1);
              ldh(c, TX);
              ldh(d, TX + 1);
              const bool g32 = x0 + TX >= nx;
#pragma unroll
              for (int f = 0; f < NV; ++f) {
                const float sm1 = mx_slope<LIM>(b[f] - a[f], c[f] - b[f]);
                const float s0 = g32 ? 0.f : mx_slope<LIM>(c[f] - b[f], d[f] - c[f]);
                qlh[f] = fmaf(0.5f, sm1, b[f]);
                qrh[f] = fmaf(-0.5f, s0, c[f]);
              }
              mx_flux<0>(qlh, qrh, ihm, ihe, hc, F);
            }
#pragma unroll
            for (int v = 0; v < NV; ++v) fr[(hpar * NV + v) * TY + row] = F[v];
          }
        }
      }
      // ------------------------------------------------------------ 3 ----
      {
        bool got = true;
        for (int pl = (K == Kfirst ? Kfirst : K + 2); pl <= K + 2; ++pl) {
          const int s = pmod(pl, C::NSLOT);
          const bool g = got && mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.wait_ns);
          if (g) {
            phase_bits ^= 1u << s;
            if (tid == 0) pending &= ~(1u << s);
          }
          got = g;
        }
        if (!__syncthreads_and(got)) {
          if (tid == 0) atomicOr(p.status, ST_TMA_TIMEOUT);
          ok = false;
          break;
        }
      }
      // ------------------------------------------------------------ 4 ----
      // cleaning residuals of plane K+1 (interior cells of the tile + 1)
      const int kr = K;  // interior index of plane K+1
      const bool rplane = kr >= 0 && kr < nz;
      float rown[R][2];
      bool step_ok = true;
      if (is_out) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int ty = w * R + r, j = jb + r;
          rown[r][0] = rown[r][1] = 0.f;
          if (rplane && i < nx && j < ny) {
            residual(uK, uK1, uK2, lane, ty, i, j, kr, rown[r]);
            rK1[(ty + 1) * WR + lane + 1] = rown[r][0];
            rK1[PLR + (ty + 1) * WR + lane + 1] = rown[r][1];
          }
        }
        // ------------------------------------------------------------ 5 ----
        const bool zghost = K + 1 <= 0 || K + 1 >= nz + 1;
        const bool zface = K >= Z0 - 1;
        const float idz = outstep ? __ldg(m.inv_dx3 + (K - 1)) : 0.f;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int ty = w * R + r;
          const int o = (ty + HH) * W + lane + 4;
          float qr[NV], qn[NV];
#pragma unroll
          for (int f = 0; f < NV; ++f) {
            const float b0 = uK[f * PL + o], b1 = uK1[f * PL + o], b2 = uK2[f * PL + o];
            const float s = zghost ? 0.f : mx_slope<LIM>(b1 - b0, b2 - b1);
            qr[f] = fmaf(-0.5f, s, b1);
            qn[f] = fmaf(0.5f, s, b1);
          }
          if (zface) {
            float F[NV];
            mx_flux<2>(qlz[r], qr, ihm, ihe, hc, F);
            const float a3k = a3[r] * idz;
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              kv[r][v] = fmaf(F[v] - fzp[r][v], a3k, kv[r][v]);
              fzp[r][v] = F[v];
            }
          }
#pragma unroll
          for (int f = 0; f < NV; ++f) qlz[r][f] = qn[f];
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
          const float h3k = idz;  // 0.5/L3 = g3 * idz
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int ty = w * R + r, j = jb + r;
            if (i < nx && j < ny && staged_ok) {
              const int o = (ty + HH) * W + lane + 4;
              float q[NV];
#pragma unroll
              for (int v = 0; v < NV; ++v) q[v] = uK[v * PL + o];
              const float H0 = q[0] * imu, H1 = q[1] * imu, H2 = q[2] * imu;
              const float E0 = q[3] * iep, E1 = q[4] * iep, E2 = q[5] * iep;
              // geometric source (zero in cartesian): the only non-zero
              // d_a ln h_b / h_a here are dl01/h0, dl02/h0 and dl12/h1
              float src_[NV];
              src_[0] = 0.f;
              src_[1] = -E2 * la;
              src_[2] = fmaf(E1, lb, -E0 * lc[r]);
              src_[3] = -sigma * E0;
              src_[4] = fmaf(H2, la, -sigma * E1);
              src_[5] = fmaf(-H1, lb, fmaf(H0, lc[r], -sigma * E2));
              // cleaning: centred gradient of the edge-padded residuals
              const int ro = (ty + 1) * WR + lane + 1;
              const int dxm = i > 0 ? -1 : 0, dxp = i + 1 < nx ? 1 : 0;
              const int dym = j > 0 ? -WR : 0, dyp = j + 1 < ny ? WR : 0;
#pragma unroll
              for (int f = 0; f < 2; ++f) {
                const float* rb = rK + f * PLR + ro;
                const float rzp = K + 1 <= nz ? rown[r][f] : rb[0];
                const float rzm = K - 1 >= 1 ? rKm[f * PLR + ro] : rb[0];
                const float chi = f == 0 ? chib : chid;
                src_[3 * f + 0] = fmaf(-chi * g1, rb[dxp] - rb[dxm], src_[3 * f + 0]);
                src_[3 * f + 1] = fmaf(-chi * g2[r], rb[dyp] - rb[dym], src_[3 * f + 1]);
                src_[3 * f + 2] = fmaf(-chi * (g3[r] * h3k), rzp - rzm, src_[3 * f + 2]);
              }
              const long long g = L.idx(0, K, j + 1, i + 1);
              const int so = ty * TX + lane;
#pragma unroll
              for (int v = 0; v < NV; ++v) {
                const float k = src_[v] - kv[r][v];
                const float u0v = need_u0 ? gu0[v * TY * TX + so] : q[v];
                const float accv = need_acc ? gacc[v * TY * TX + so] : 0.f;
                const long long gi = g + (long long)v * L.var_stride;
                const float o2 = stage_combine(p.coef, dt, k, q[v], u0v, accv);
                p.out[gi] = o2;
                if (p.coef.accmode != ACC_NONE) p.acc[gi] = acc_update(p.coef, dt, k, u0v, accv);
                if (!isfinite(o2)) bad |= ST_NONFINITE;
              }
            }
          }
          if (bad) atomicOr(p.status, bad);
        }
      } else if (rplane) {
        // residuals of the border cells of the tile + 1
        for (int b = lane; b < C::NBORDER; b += 32) {
          int x, y;
          if (b < 2 * WR) {
            y = b < WR ? -1 : TY;
            x = (b < WR ? b : b - WR) - 1;
          } else {
            const int c = b - 2 * WR;
            y = c >> 1;
            x = (c & 1) ? TX : -1;
          }
          const int ii = x0 + x, jj = y0 + y;
          if (ii < 0 || ii >= nx || jj < 0 || jj >= ny) continue;
          float rv[2];
          residual(uK, uK1, uK2, x, y, ii, jj, kr, rv);
          rK1[(y + 1) * WR + x + 1] = rv[0];
          rK1[PLR + (y + 1) * WR + x + 1] = rv[1];
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
