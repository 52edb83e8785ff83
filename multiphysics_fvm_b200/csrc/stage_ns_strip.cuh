// Float32 cartesian Navier-Stokes stage kernel with register-blocked columns:
// residual (navier_stokes.py:588-711) + Runge-Kutta stage combination in one
// pass, built to issue few instructions per cell.
//
// Tile: 32 columns (x1) x TY = NW*R rows (x2), marching a chunk of planes
// along x3.  Output warp w (< NW) owns the strip of R rows w*R .. w*R+R-1;
// lane l owns column l.  One more warp (the halo warp) forms, for every tile
// row, the x1 data that lies outside the warp: the slopes of the cell left of
// the tile and the flux through the tile's right edge, and the pressure of
// the tile's halo cells.
//
// Per step K (ghosted output plane K; the TMA ring holds planes K, K+1 and,
// once it has arrived, K+2):
//   1. thread 0 issues the TMA of plane K+2 into the slot that plane K-1 left,
//      and of this plane's U0 / k-accumulator tile when the stage combination
//      reads them;
//   2. x2 and x1 for plane K in one sweep up the strip: x2 slopes and face
//      fluxes in registers (the strip computes its R+1 faces itself), x1 slopes
//      per row with the left slope and the right-face flux from neighbouring
//      lanes by shuffle (lane 0 / lane 31 from the halo warp's data).  The halo
//      warp meanwhile forms that data for plane K+1;
//   3. every thread waits (bounded) for plane K+2;
//   4. P of plane K+2: own cells by their owners (kept in registers), halo
//      cells by the halo warp (navier_stokes.py:94-100);
//   5. x3: slope of plane K+1 at the thread's cells and the face flux at
//      K+1/2; the left state and the flux at K-1/2 are carried in registers;
//   6. divergence with the inverse cell lengths, gravity, stage combination
//      with U0 / acc from shared memory, coalesced stores;
//   7. one block barrier per step (after it, plane K's slot is free).
// Face values are the reference's: MUSCL slopes limiter(f_i - f_i-1,
// f_i+1 - f_i) (zero in ghost cells, reconstructors.py:120-132), states
// f +- s/2, Euler flux from the face U and the reconstructed face P, HLL or
// Rusanov (riemann_solvers.py:13-89).  float32 arithmetic with the
// approximate reciprocal and square root; HLL's three-way choice is written
// with clamped wave speeds (s- = min(s_min, 0), s+ = max(s_max, 0)), which is
// the same function.
#pragma once
#include "stage_ns.cuh"

namespace fvm {

template <int R, int NW>
struct NsStripCfg {
  static constexpr int TX = 32, TY = R * NW;
  static constexpr int NO = 32 * NW;  // output threads
  static constexpr int NT = NO + 32;  // + the halo warp
  static constexpr int NV = 5, NF = 6, HH = 2;
  static constexpr int W = 40;  // ring column c <-> tile x offset c - 4
  static constexpr int ROWS = TY + 2 * HH;
  static constexpr int PL = ROWS * W;
  static constexpr int NSLOT = 3;  // planes K, K+1 and K+2 (arriving)
  static constexpr int SLOT = round_up(NV * PL, 32);
  static constexpr int W2 = TX + 4, R2 = TY + 4, PL2 = W2 * R2;  // P plane: tile + 2
  static constexpr int NBORDER = 4 * W2 + 4 * TY;                 // P halo cells per plane
  static constexpr int STG = NV * TY * TX;                        // one staged U0 / acc tile
  static constexpr int OFF_U = 0;
  static constexpr int OFF_P = OFF_U + NSLOT * SLOT;
  static constexpr int OFF_HL = OFF_P + 3 * PL2;       // [parity][field][row]: slopes left of the tile
  static constexpr int OFF_FR = OFF_HL + 2 * NF * TY;  // [parity][var][row]: right-edge fluxes
  static constexpr int END = OFF_FR + 2 * NV * TY;
  static constexpr int NBAR = NSLOT + 1;               // ring slots + the staged tiles
  static constexpr int BAR_BYTES = round_up(END * 4, 8);
  static constexpr int STG_OFF_BYTES = round_up(BAR_BYTES + NBAR * 8, 128);
  static constexpr unsigned TX_BYTES = NV * PL * 4;
  static constexpr unsigned STG_BYTES = STG * 4;
  // dynamic shared memory with `nbuf` staged tiles (0: none, 1: U0 or acc, 2: both)
  static constexpr int bytes(int nbuf) { return STG_OFF_BYTES + nbuf * (int)STG_BYTES; }
  static_assert(2 * TY <= 32, "one halo lane per tile row and task");
  static_assert((SLOT * 4) % 128 == 0 && (STG_BYTES % 128) == 0, "TMA destinations need 128-byte alignment");
};

// Tensor maps and parameters of one launch: the ring map of the stage input
// and the maps of the U0 / accumulator buffers (box 32 x TY x 1 x 5).
struct NsStripSource {
  CUtensorMap tmap, u0map, accmap;
  NsParams<float> p;
};

// Limited slope from the backward and forward differences (float32; zero
// for piecewise constant).  minmod is the median of (a, b, 0), which equals
// (sign a + sign b)/2 * min(|a|, |b|) (slope_limiters.py:13-39).
template <int LIM>
__device__ __forceinline__ float strip_slope(float a, float b) {
  if constexpr (LIM == LIM_PC) return 0.f;
  else if constexpr (LIM == LIM_MINMOD) return fmaxf(fminf(a, b), fminf(fmaxf(a, b), 0.f));
  else if constexpr (LIM == LIM_MC) return flim_mc(a, b);
  else return flim_vanleer(a, b);
}

// Inviscid Riemann flux along axis D from face states q = {rho, m1, m2, m3, E, P}
// (navier_stokes.py:159-214 fluxes, :280-355 wave speeds).
template <int D, int RIEM>
__device__ __forceinline__ void strip_flux(const float* qL, const float* qR, float gam, float* F) {
  const float irL = rcp_approx(qL[0]), irR = rcp_approx(qR[0]);
  const float vL = qL[1 + D] * irL, vR = qR[1 + D] * irR;
  const float cL = sqrt_approx((gam * qL[5]) * irL), cR = sqrt_approx((gam * qR[5]) * irR);
  float FL[5], FR[5];
  FL[0] = qL[1 + D];
  FR[0] = qR[1 + D];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    FL[1 + c] = qL[1 + c] * vL;
    FR[1 + c] = qR[1 + c] * vR;
  }
  FL[1 + D] += qL[5];
  FR[1 + D] += qR[5];
  FL[4] = (qL[4] + qL[5]) * vL;
  FR[4] = (qR[4] + qR[5]) * vR;
  if constexpr (RIEM == RIEM_HLL) {
    const float sl = fminf(fminf(vL - cL, vR - cR), 0.f);
    const float sr = fmaxf(fmaxf(vL + cL, vR + cR), 0.f);
    const float rd = rcp_approx(fmaxf(sr - sl, 1e-30f));
    const float a = sr * rd, b = -sl * rd, c = (sl * sr) * rd;
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = fmaf(a, FL[v], fmaf(b, FR[v], c * (qR[v] - qL[v])));
  } else {
    const float h = 0.5f * fmaxf(fabsf(vL) + cL, fabsf(vR) + cR);
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = fmaf(0.5f, FL[v] + FR[v], -h * (qR[v] - qL[v]));
  }
}

// P = (gamma - 1)(E - |m|^2 / (2 rho)) of one ring cell (navier_stokes.py:94-100).
__device__ __forceinline__ float strip_pressure(const float* u, int PL, float gm1) {
  const float rho = u[0], m1 = u[PL], m2 = u[2 * PL], m3 = u[3 * PL], E = u[4 * PL];
  const float ke = fmaf(m1, m1, fmaf(m2, m2, m3 * m3)) * (0.5f * rcp_approx(rho));
  return gm1 * (E - ke);
}

// One tile of the stage (all planes of its z-chunk).  `bars` holds the ring
// barriers (indices 0..2, phase bits 0..2), `gbar` the staged-tile barrier with
// phase bit `gbit`; `phase_bits` and `pending` carry over from tile to tile.
// Returns false when a wait ran out: the block must stop and drain.
template <int LIM, int RIEM, int R, int NW>
__device__ __forceinline__ bool ns_strip_tile(const NsParams<float>& p, const CUtensorMap* tmap,
                                              const CUtensorMap* u0map, const CUtensorMap* accmap, int tile,
                                              unsigned char* smem_raw, uint64_t* bars, uint64_t* gbar, int gbit,
                                              unsigned& phase_bits, unsigned& pending) {
  using C = NsStripCfg<R, NW>;
  constexpr int TX = C::TX, TY = C::TY, W = C::W, PL = C::PL, HH = C::HH, NF = C::NF, W2 = C::W2;
  constexpr int PL2 = C::PL2;
  float* sm = reinterpret_cast<float*>(smem_raw);
  float* uring = sm + C::OFF_U;
  float* pring = sm + C::OFF_P;
  float* hl = sm + C::OFF_HL;
  float* fr = sm + C::OFF_FR;
  float* gst = reinterpret_cast<float*>(smem_raw + C::STG_OFF_BYTES);
  const int tid = threadIdx.x;
  const Layout& L = p.lay;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const float gam = float(p.gamma), gm1 = float(p.gamma) - 1.f;
  const float dt = float(*p.dt);
  const float gx = float(p.g1), gy = float(p.g2), gz = float(p.g3);
  const bool need_u0 = needs_u0<float>(p.coef) && !p.coef.u0_is_input;
  const bool need_acc = needs_acc(p.coef);
  const unsigned stg_bytes = (need_u0 ? C::STG_BYTES : 0u) + (need_acc ? C::STG_BYTES : 0u);
  const float* gu0 = gst;                            // staged U0 tile [var][row][column]
  const float* gacc = gst + (need_u0 ? C::STG : 0);  // staged acc tile
  const int w = tid >> 5, lane = tid & 31;
  const bool is_out = w < NW;
  {
    const int tx_i = tile % p.ntx;
    const int ty_i = (tile / p.ntx) % p.nty;
    const int zc_i = tile / (p.ntx * p.nty);
    const int Z0 = 1 + zc_i * p.zchunk;         // first ghosted output plane
    const int Zl = min(Z0 + p.zchunk - 1, nz);  // last ghosted output plane
    // A one-plane grid whose x3 ghosts copy the plane ("flat") has x3 fluxes
    // that cancel exactly: plane 1 alone, no x3 pipeline.  Its tile marches
    // instead over p.ysub row tiles along x2 (the steps of the march), each
    // step's plane copy issued one step ahead into the next ring slot.
    const bool flat = p.flat != 0;
    const int ysub = flat ? p.ysub : 1;
    const int x0 = tx_i * TX, ybase = ty_i * ysub * TY;
    int y0 = ybase;  // the current step's first row
    const int nsteps = flat ? min(ysub, (ny + TY - 1) / TY - ty_i * ysub) : 0;
    const int Kfirst = flat ? Z0 : Z0 - 2, Plast = flat ? Zl : Zl + HH;
    const int i = x0 + lane;
    const float idx = (is_out && i < nx) ? __ldg(p.met.inv_dx1 + i) : 0.f;

    // plane pl of the rows from yrow - HH into ring slot s
    auto issue_at = [&](int pl, int s, int yrow) {
      pending |= 1u << s;
      fence_proxy_async();
      mbar_arrive_expect_tx(&bars[s], C::TX_BYTES + p.extra_tx);
      tma_load_4d(&uring[s * C::SLOT], tmap, &bars[s], x0 - 3 + L.padx, yrow + 1 - HH, pl, 0);
    };
    auto issue = [&](int pl) { issue_at(pl, pmod(pl, C::NSLOT), y0); };
    // planes Kfirst .. Kfirst + 2 (the first step's; a flat grid's first row tile)
    if (tid == 0) {
      if (flat) issue_at(Kfirst, 0, ybase);
      else
        for (int pl = Kfirst; pl <= Kfirst + 2; ++pl) issue(pl);
    }

    // Halo warp: x1 data of plane Kh (ring plane uH, P plane pH) outside the
    // warps: lanes 0..TY-1 the slopes of the cell left of the tile, lanes
    // TY..2TY-1 the flux through the tile's right edge
    auto halo_x1 = [&](int Kh, const float* uH, const float* pH) {
      const int row = lane < TY ? lane : lane - TY;
      const int j = y0 + row;
      if (Kh >= Z0 && Kh <= Zl && lane < 2 * TY && j < ny) {
        const int hpar = Kh & 1;
        auto ldh = [&](float* f, int tx) {
          const int o = (row + HH) * W + tx + 4;
#pragma unroll
          for (int v = 0; v < 5; ++v) f[v] = uH[v * PL + o];
          f[5] = pH[(row + 2) * W2 + tx + 2];
        };
        if (lane < TY) {
          float a[NF], b[NF], c[NF];
          ldh(a, -2);
          ldh(b, -1);
          ldh(c, 0);
#pragma unroll
          for (int f = 0; f < NF; ++f)  // zero on the left ghost column
            hl[(hpar * NF + f) * TY + row] = x0 == 0 ? 0.f : strip_slope<LIM>(b[f] - a[f], c[f] - b[f]);
        } else {
          float F[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
          if (x0 + TX <= nx) {  // the face between x0 + 31 and x0 + 32 is needed
            float a[NF], b[NF], c[NF], d[NF], ql[NF], qr[NF];
            ldh(a, TX - 2);
            ldh(b, TX - 1);
            ldh(c, TX);
            ldh(d, TX + 1);
            const bool g32 = x0 + TX >= nx;  // x0 + 32 is the right ghost column
#pragma unroll
            for (int f = 0; f < NF; ++f) {
              const float sm1 = strip_slope<LIM>(b[f] - a[f], c[f] - b[f]);
              const float s0 = g32 ? 0.f : strip_slope<LIM>(c[f] - b[f], d[f] - c[f]);
              ql[f] = fmaf(0.5f, sm1, b[f]);
              qr[f] = fmaf(-0.5f, s0, c[f]);
            }
            strip_flux<0, RIEM>(ql, qr, gam, F);
          }
#pragma unroll
          for (int v = 0; v < 5; ++v) fr[(hpar * 5 + v) * TY + row] = F[v];
        }
      }
    };
    // Halo warp: P of ring plane usrc on the cells of the P plane no output
    // thread owns
    auto border_p = [&](float* pdst, const float* usrc) {
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
        pdst[(y + 2) * W2 + x + 2] = strip_pressure(usrc + (y + HH) * W + x + 4, PL, gm1);
      }
    };

    // x3 state carried from step to step, per own cell: the left state of the
    // face above the last slope plane and the flux of the face below the
    // output plane
    float qlz[R][NF], fzp[R][5];
#pragma unroll
    for (int r = 0; r < R; ++r) {
#pragma unroll
      for (int f = 0; f < NF; ++f) qlz[r][f] = 0.f;
#pragma unroll
      for (int v = 0; v < 5; ++v) fzp[r][v] = 0.f;
    }

    const int nstep = flat ? nsteps : Zl - Kfirst + 1;
    for (int st = 0; st < nstep; ++st) {
      const int K = flat ? Kfirst : Kfirst + st;
      if (flat) y0 = ybase + st * TY;
      const int sK = flat ? st % C::NSLOT : pmod(K, C::NSLOT), pK0 = flat ? 0 : pmod(K, 3);
      const bool outstep = K >= Z0;
      const int sK1 = sK == C::NSLOT - 1 ? 0 : sK + 1, sK2 = sK1 == C::NSLOT - 1 ? 0 : sK1 + 1;
      const int pK1i = pK0 == 2 ? 0 : pK0 + 1, pK2i = pK1i == 2 ? 0 : pK1i + 1;
      const float* uK = uring + sK * C::SLOT;
      const float* uK1 = uring + sK1 * C::SLOT;
      const float* uK2 = uring + sK2 * C::SLOT;
      float* pK = pring + pK0 * PL2;
      float* pK1 = pring + pK1i * PL2;
      float* pK2 = pring + pK2i * PL2;
      // ------------------------------------------------------------ 1 ----
      if (tid == 0) {
        if (flat) {
          // the next row tile's plane, into the slot two steps back left
          if (st + 1 < nstep) issue_at(Kfirst, (st + 1) % C::NSLOT, y0 + TY);
        } else if (K > Kfirst && K + 2 <= Plast) {
          issue(K + 2);
        }
        if (outstep && stg_bytes) {
          pending |= 1u << gbit;
          fence_proxy_async();
          mbar_arrive_expect_tx(gbar, stg_bytes);
          const int gxc = x0 + 1 + L.padx;
          if (need_u0) tma_load_4d(gst, u0map, gbar, gxc, y0 + 1, K, 0);
          if (need_acc) tma_load_4d(gst + (need_u0 ? C::STG : 0), accmap, gbar, gxc, y0 + 1, K, 0);
        }
      }
      float kv[R][5];
#pragma unroll
      for (int r = 0; r < R; ++r)
#pragma unroll
        for (int v = 0; v < 5; ++v) kv[r][v] = 0.f;
      if (flat) {
        // the plane itself, its P over the tile + 2 and the halo warp's x1
        // data, before the sweep
        const bool g = mbar_wait_bounded(&bars[sK], (phase_bits >> sK) & 1u, p.wait_ns);
        if (g) {
          phase_bits ^= 1u << sK;
          if (tid == 0) pending &= ~(1u << sK);
          if (is_out) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
              const int ty = w * R + r;
              pK[(ty + 2) * W2 + lane + 2] = strip_pressure(uK + (ty + HH) * W + lane + 4, PL, gm1);
            }
          } else {
            border_p(pK, uK);
          }
        } else {
          atomicOr(p.status, ST_TMA_TIMEOUT);
        }
        if (!__syncthreads_and(g)) return false;
        if (!is_out) halo_x1(K, uK, pK);
        __syncthreads();
      }
      // ------------------------------------------------------------ 2 ----
      if (is_out) {
        if (outstep) {
          const int par = K & 1;
          const int jb = y0 + w * R;  // first row of the strip
          auto ldf = [&](float* f, int ty, int tx) {
            const int o = (ty + HH) * W + tx + 4;
#pragma unroll
            for (int v = 0; v < 5; ++v) f[v] = uK[v * PL + o];
            f[5] = pK[(ty + 2) * W2 + tx + 2];
          };
          float fa[NF], fb[NF], fc[NF], ql[NF];
          ldf(fa, w * R - 2, lane);
          ldf(fb, w * R - 1, lane);
#pragma unroll
          for (int t = 0; t <= R + 1; ++t) {
            // row ty = w*R - 1 + t: its x2 slope; for t >= 1 the x2 face
            // below it (the upper face of own row t - 2, the lower face of
            // own row t - 1); for 1 <= t <= R (own rows) its x1 work
            const int ty = w * R - 1 + t;
            const int j = jb - 1 + t;
            ldf(fc, ty + 1, lane);
            const bool yghost = j < 0 || j >= ny;
            float s[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) s[f] = yghost ? 0.f : strip_slope<LIM>(fb[f] - fa[f], fc[f] - fb[f]);
            if (t >= 1) {
              float qr[NF], F[5];
#pragma unroll
              for (int f = 0; f < NF; ++f) qr[f] = fmaf(-0.5f, s[f], fb[f]);
              strip_flux<1, RIEM>(ql, qr, gam, F);
              if (t >= 2) {
                const float idym = __ldg(p.met.inv_dx2 + min(max(j - 1, 0), ny - 1));
#pragma unroll
                for (int v = 0; v < 5; ++v) kv[t - 2][v] = fmaf(F[v], idym, kv[t - 2][v]);
              }
              if (t <= R) {
                const float idy = __ldg(p.met.inv_dx2 + min(j, ny - 1));
#pragma unroll
                for (int v = 0; v < 5; ++v) kv[t - 1][v] = fmaf(-F[v], idy, kv[t - 1][v]);
              }
            }
#pragma unroll
            for (int f = 0; f < NF; ++f) ql[f] = fmaf(0.5f, s[f], fb[f]);
            if (t >= 1 && t <= R) {
              // x1 for own row r = t - 1 (cell i, row j): the flux through
              // the cell's left face, the right face's from the next lane
              const int r = t - 1;
              float fm[NF], fp[NF], qlx[NF], qrx[NF], F[5];
              ldf(fm, ty, lane - 1);
              ldf(fp, ty, lane + 1);
              const bool xghost = i >= nx;  // i == nx: the right ghost column
#pragma unroll
              for (int f = 0; f < NF; ++f) {
                const float s1 = xghost ? 0.f : strip_slope<LIM>(fb[f] - fm[f], fp[f] - fb[f]);
                const float su = __shfl_up_sync(0xffffffffu, s1, 1);
                const float sl = lane == 0 ? hl[(par * NF + f) * TY + ty] : su;
                qlx[f] = fmaf(0.5f, sl, fm[f]);
                qrx[f] = fmaf(-0.5f, s1, fb[f]);
              }
              strip_flux<0, RIEM>(qlx, qrx, gam, F);
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
        // x1 data of plane K+1, the next output plane (a flat grid's was
        // formed before the sweep)
        if (!flat) halo_x1(K + 1, uK1, pK1);
      }
      // ------------------------------------------------------------ 3 ----
      // Every thread waits for the plane itself; nothing read after the wait
      // was written by another thread in this step, so the block needs no
      // barrier here.  A thread whose wait ran out skips the rest of the step
      // and the barrier at its end takes the block out.
      bool got = true;
      for (int pl = (K == Kfirst ? Kfirst : K + 2); !flat && pl <= K + 2; ++pl) {
        const int s = pmod(pl, C::NSLOT);
        const bool g = got && mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.wait_ns);
        if (g) {
          phase_bits ^= 1u << s;
          if (tid == 0) pending &= ~(1u << s);
        }
        got = g;
      }
      if (!got) atomicOr(p.status, ST_TMA_TIMEOUT);
      bool step_ok = got;
      if (!got) {
        // skip to the barrier
      } else if (is_out) {
        if (!flat) {  // x3 (a flat grid has none)
          // ------------------------------------------------------------ 4 ----
          float pnew[R];
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int ty = w * R + r;
            const int o = (ty + HH) * W + lane + 4, op = (ty + 2) * W2 + lane + 2;
            pnew[r] = strip_pressure(uK2 + o, PL, gm1);
            pK2[op] = pnew[r];
            if (K == Kfirst) {
              pK[op] = strip_pressure(uK + o, PL, gm1);
              pK1[op] = strip_pressure(uK1 + o, PL, gm1);
            }
          }
          // ------------------------------------------------------------ 5 ----
          // slope of plane K+1 (zero on a ghost plane) and the flux at K+1/2
          const bool zghost = K + 1 <= 0 || K + 1 >= nz + 1;
          const bool zface = K >= Z0 - 1;
          const float idz = outstep ? __ldg(p.met.inv_dx3 + (K - 1)) : 0.f;
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int ty = w * R + r;
            const int o = (ty + HH) * W + lane + 4, op = (ty + 2) * W2 + lane + 2;
            float qr[NF], qn[NF];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
              const float a0 = f < 5 ? uK[f * PL + o] : pK[op];
              const float a1 = f < 5 ? uK1[f * PL + o] : pK1[op];
              const float a2 = f < 5 ? uK2[f * PL + o] : pnew[r];
              const float s = zghost ? 0.f : strip_slope<LIM>(a1 - a0, a2 - a1);
              qr[f] = fmaf(-0.5f, s, a1);
              qn[f] = fmaf(0.5f, s, a1);
            }
            if (zface) {
              float F[5];
              strip_flux<2, RIEM>(qlz[r], qr, gam, F);
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
            staged_ok = mbar_wait_bounded(gbar, (phase_bits >> gbit) & 1u, p.wait_ns);
            if (staged_ok) {
              phase_bits ^= 1u << gbit;
              if (tid == 0) pending &= ~(1u << gbit);
            }
          }
          step_ok = step_ok && staged_ok;
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
              // gravity (navier_stokes.py:499-504): rho g and rho g.v = g.m
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
      } else {
        // P of plane K+2 (and on the first step of K, K+1) on the cells of
        // the P plane no output thread owns
        if (!flat) {
          border_p(pK2, uK2);
          if (K == Kfirst) {
            border_p(pK, uK);
            border_p(pK1, uK1);
          }
        }
      }
      // ------------------------------------------------------------ 7 ----
      if (!__syncthreads_and(step_ok)) return false;
    }
  }
  return true;
}

template <int LIM, int RIEM, int R, int NW, int MINB>
__global__ void __launch_bounds__(NsStripCfg<R, NW>::NT, MINB)
    ns_strip_kernel(const __grid_constant__ NsStripSource src) {
  using C = NsStripCfg<R, NW>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + C::BAR_BYTES);
  const NsParams<float>& p = src.p;
  if (smem_u32(smem_raw) & 127u) {  // TMA destinations need 128-byte alignment
    if (threadIdx.x == 0) atomicOr(p.status, ST_TMA_TIMEOUT);
    return;
  }
  if (p.active && !*p.active) return;  // the clock passed t_end: the stage is a no-op
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < C::NBAR; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    tma_prefetch_desc(&src.tmap);
    if (needs_u0<float>(p.coef) && !p.coef.u0_is_input) tma_prefetch_desc(&src.u0map);
    if (needs_acc(p.coef)) tma_prefetch_desc(&src.accmap);
  }
  __syncthreads();
  unsigned phase_bits = 0;  // expected parity per barrier (identical in the threads that wait)
  unsigned pending = 0;     // barriers with a copy in flight (thread 0)
  const int ntiles = p.ntx * p.nty * p.nzc;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    if (!ns_strip_tile<LIM, RIEM, R, NW>(p, &src.tmap, &src.u0map, &src.accmap, tile, smem_raw, bars,
                                         bars + C::NSLOT, C::NSLOT, phase_bits, pending)) {
      ok = false;
      break;
    }
  // On a timeout, wait (bounded) for every copy this block may still have in flight.
  if (!ok && tid == 0) {
    for (int s = 0; s < C::NBAR; ++s)
      if ((pending >> s) & 1u) mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.drain_ns);
  }
}

}  // namespace fvm
