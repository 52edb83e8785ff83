// Float32 heat stage kernel for piecewise-constant face states (the centred
// diffusion scheme): residual (heat.py:354-473) + Runge-Kutta stage in one
// pass with few instructions per cell.
//
// With piecewise-constant faces the face flux is the mean of the two cell
// fluxes phi_a = -k dT/dx_a (centred, zero in ghost cells, heat.py:85-95), so
//   rhs = q - [ A1+ (phi1_i + phi1_i+1) - A1- (phi1_i-1 + phi1_i)
//             + A2+ (phi2_j + phi2_j+1) - A2- (phi2_j-1 + phi2_j)
//             + A3  (phi3_k+1 - phi3_k-1) ]
// with A_a+- = S_a(face +-1/2) / (2 V) and phi_a = g_a (U_+1 - U_-1),
// g_a = -k / (2 rho cp L_a) (T = U / (rho cp), heat.py:74).  Every grid metric
// is a product of per-axis factors (geometry.py:37-171), so the A and g of a
// cell column are formed once per tile in registers; only 1/dx3 of the plane
// varies along the z-march.
//
// Tile: 32 columns x TY = NW*R rows; warp w owns rows w*R .. w*R+R-1, lane l
// column l.  Each step reads the TMA ring (tile + 2 halo, planes K..K+2) and
// keeps phi3 of planes K-1 and K in registers; one block barrier per step.
#pragma once
#include "stage_heat.cuh"

namespace fvm {

template <int R, int NW>
struct HeatPcCfg {
  static constexpr int TX = 32, TY = R * NW, NT = 32 * NW, HH = 2;
  static constexpr int W = 40;  // ring column c <-> tile x offset c - 4
  static constexpr int ROWS = TY + 2 * HH, PL = ROWS * W;
  static constexpr int NSLOT = 6;  // planes K..K+2 in use, K+3..K+5 in flight
  static constexpr int SLOT = round_up(PL, 32);
  static constexpr int BYTES = NSLOT * SLOT * 4 + NSLOT * 8;
  static constexpr unsigned TX_BYTES = PL * 4;
  static_assert((SLOT * 4) % 128 == 0, "TMA destinations need 128-byte alignment");
};

// One tile of the stage (all planes of its z-chunk) with the ring barriers
// `bars` (phase bits 0..5); `phase_bits` and `pending` carry over from tile to
// tile.  Returns false when a wait ran out: the block must stop and drain.
// MERGED: the two warm-up steps of the z-march (phi3 of planes Z0-1 and Z0)
// are one prologue step.  It pays where z-chunks are short and many (the
// batched launch); a single-grid launch of one wave of long chunks ran 2 %
// slower with it.
template <int COORD, int R, int NW, bool MERGED = false>
__device__ __forceinline__ bool heat_pc_tile(const HeatParams<float>& p, const CUtensorMap* tmap, int tile,
                                             unsigned char* smem_raw, uint64_t* bars, unsigned& phase_bits,
                                             unsigned& pending) {
  using C = HeatPcCfg<R, NW>;
  using G = Geo<float, COORD>;
  constexpr int TX = C::TX, TY = C::TY, W = C::W, HH = C::HH;
  float* uring = reinterpret_cast<float*>(smem_raw);
  const int tid = threadIdx.x;
  const Layout& L = p.lay;
  const Metric<float>& m = p.met;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const float qsrc = float(p.q), dt = float(*p.dt);
  const float kap = float(p.k * p.inv_rho_cp);  // k / (rho cp)
  const bool need_u0 = needs_u0<float>(p.coef) && !p.coef.u0_is_input;
  const bool need_acc = needs_acc(p.coef);
  const int w = tid >> 5, lane = tid & 31;
  {
    const int x0 = (tile % p.ntx) * TX, y0 = ((tile / p.ntx) % p.nty) * TY;
    const int Z0 = 1 + (tile / (p.ntx * p.nty)) * p.zchunk;
    const int Zl = min(Z0 + p.zchunk - 1, nz);
    const int Kfirst = Z0 - 2, Plast = Zl + 2;
    const int i = x0 + lane, jb = y0 + w * R;
    const bool icol = i < nx;
    const int ic = min(i, nx - 1);  // metric index of this column (garbage lanes clamp)

    auto issue = [&](int pl) {
      const int s = pmod(pl, C::NSLOT);
      pending |= 1u << s;
      fence_proxy_async();
      mbar_arrive_expect_tx(&bars[s], C::TX_BYTES + p.extra_tx);
      tma_load_4d(&uring[s * C::SLOT], tmap, &bars[s], x0 - 3 + L.padx, y0 + 1 - HH, pl, 0);
    };
    if (tid == 0)
      for (int pl = Kfirst; pl <= Kfirst + C::NSLOT - 1 && pl <= Plast; ++pl) issue(pl);

    // per-column and per-row metric factors (zero g in ghost cells: phi is
    // zero-padded there)
    const float g1m = (i - 1 >= 0 && i - 1 < nx) ? -0.5f * kap * __ldg(m.inv_dx1 + i - 1) : 0.f;
    const float g10 = icol ? -0.5f * kap * __ldg(m.inv_dx1 + i) : 0.f;
    const float g1p = (i + 1 < nx) ? -0.5f * kap * __ldg(m.inv_dx1 + i + 1) : 0.f;
    float g2[R + 2];  // rows jb-1 .. jb+R
#pragma unroll
    for (int t = 0; t < R + 2; ++t) {
      const int j = jb - 1 + t;
      g2[t] = (icol && j >= 0 && j < ny) ? -0.5f * kap * inv_len<float, COORD, 1>(m, i, j, 0) : 0.f;
    }
    float a1p[R], a1m[R], a2p[R], a2m[R], a3[R], g3[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int jc = min(jb + r, ny - 1);
      // V and the face areas at plane 0; their x3 factor dx3 cancels in S1/V
      // and S2/V, and S3/V scales with 1/dx3 of the plane
      const float iv = 0.5f / G::V(m, ic, jc, 0);
      a1p[r] = G::S1(m, ic + 1, jc, 0) * iv;
      a1m[r] = G::S1(m, ic, jc, 0) * iv;
      a2p[r] = G::S2(m, ic, jc + 1, 0) * iv;
      a2m[r] = G::S2(m, ic, jc, 0) * iv;
      a3[r] = G::S3(m, ic, jc) * iv * __ldg(m.dx3);
      g3[r] = -0.5f * kap;
      if constexpr (COORD == COORD_SPH) g3[r] *= __ldg(m.inv_r + ic) * __ldg(m.inv_sin_c2 + jc);
    }
    // phi3 of plane P at the own cells from the ring planes P-1 (um) and P+1
    // (up); zero on a ghost plane
    auto phi3 = [&](int P, const float* um, const float* up, float* out) {
      const bool zg = P <= 0 || P >= nz + 1;
      const float idz1 = zg ? 0.f : __ldg(m.inv_dx3 + min(max(P - 1, 0), nz - 1));
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int o = (w * R + r + HH) * W + lane + 4;
        out[r] = (g3[r] * idz1) * (up[o] - um[o]);
      }
    };
    float phz0[R], phz1[R];  // phi3 of planes K-1 and K at the own cells
#pragma unroll
    for (int r = 0; r < R; ++r) { phz0[r] = 0.f; phz1[r] = 0.f; }
    if constexpr (MERGED) {
      // prologue: planes Z0-2 .. Z0+1 give phi3 of planes Z0-1 and Z0 in one
      // step (one set of waits and one barrier pair for both)
      bool got = true;
      for (int pl = Kfirst; pl <= Kfirst + 3; ++pl) {
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
        return false;
      }
      phi3(Z0 - 1, uring + pmod(Kfirst, C::NSLOT) * C::SLOT, uring + pmod(Kfirst + 2, C::NSLOT) * C::SLOT, phz0);
      phi3(Z0, uring + pmod(Kfirst + 1, C::NSLOT) * C::SLOT, uring + pmod(Kfirst + 3, C::NSLOT) * C::SLOT, phz1);
      __syncthreads();  // planes Z0-2 and Z0-1 are refilled at the first step
    }

    const int K0 = MERGED ? Z0 : Kfirst;
    int next_pl = Kfirst + C::NSLOT;  // MERGED: the next plane to issue (thread 0)
    for (int K = K0, sK = pmod(K0, C::NSLOT); K <= Zl; ++K, sK = (sK == C::NSLOT - 1 ? 0 : sK + 1)) {
      if constexpr (MERGED) {
        // the prologue freed two slots: the first step refills both
        if (tid == 0)
          for (; next_pl <= K + C::NSLOT - 1 && next_pl <= Plast; ++next_pl) issue(next_pl);
      } else {
        if (tid == 0 && K > Kfirst && K + C::NSLOT - 1 <= Plast) issue(K + C::NSLOT - 1);
      }
      const bool outstep = MERGED || K >= Z0;  // the merged loop starts at Z0
      // U0 / acc of the plane's own cells, loaded before anything is stored
      // in this step so that the step hides their latency
      float eu0[R], eacc[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        eu0[r] = 0.f;
        eacc[r] = 0.f;
        if (outstep && icol && jb + r < ny) {
          const long long g = L.idx(0, K, jb + r + 1, i + 1);
          if (need_u0) eu0[r] = p.u0[g];
          if (need_acc) eacc[r] = p.acc[g];
        }
      }
      {
        bool got = true;
        for (int pl = (!MERGED && K == Kfirst ? Kfirst : K + 2); pl <= K + 2; ++pl) {
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
          return false;
        }
      }
      const int s2 = sK + 2 >= C::NSLOT ? sK + 2 - C::NSLOT : sK + 2;
      const float* uK = uring + sK * C::SLOT;
      const float* uK2 = uring + s2 * C::SLOT;
      float phz2[R];  // phi3 of plane K+1 at the own cells (zero on a ghost plane)
      if constexpr (MERGED) {
        phi3(K + 1, uK, uK2, phz2);
      } else {
        // 1/dx3 of interior plane K (ghosted K+1)
        const bool zg = K + 1 <= 0 || K + 1 >= nz + 1;
        const float idz1 = zg ? 0.f : __ldg(m.inv_dx3 + min(max(K, 0), nz - 1));
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int o = (w * R + r + HH) * W + lane + 4;
          phz2[r] = (g3[r] * idz1) * (uK2[o] - uK[o]);
        }
      }
      if (outstep) {
        const float idz = __ldg(m.inv_dx3 + (K - 1));
        // x2: phi2 along the strip (rows jb-1 .. jb+R) from the ring
        float ph2[R + 2];
#pragma unroll
        for (int t = 0; t < R + 2; ++t) {
          const int o = (w * R - 1 + t + HH) * W + lane + 4;
          ph2[t] = g2[t] * (uK[o + W] - uK[o - W]);
        }
        unsigned bad = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int o = (w * R + r + HH) * W + lane + 4;
          const float um2 = uK[o - 2], um1 = uK[o - 1], u0c = uK[o], up1 = uK[o + 1], up2 = uK[o + 2];
          const float p1m = g1m * (u0c - um2), p10 = g10 * (up1 - um1), p1p = g1p * (up2 - u0c);
          float div = a1p[r] * (p10 + p1p) - a1m[r] * (p1m + p10);
          div = fmaf(a2p[r], ph2[r + 1] + ph2[r + 2], div);
          div = fmaf(-a2m[r], ph2[r] + ph2[r + 1], div);
          div = fmaf(a3[r] * idz, phz2[r] - phz0[r], div);
          const int j = jb + r;
          if (icol && j < ny) {
            const float k = qsrc - div;
            const long long gi = L.idx(0, K, j + 1, i + 1);
            const float u0v = need_u0 ? eu0[r] : u0c;
            const float o2 = stage_combine(p.coef, dt, k, u0c, u0v, eacc[r]);
            p.out[gi] = o2;
            if (p.coef.accmode != ACC_NONE) p.acc[gi] = acc_update(p.coef, dt, k, u0v, eacc[r]);
            if (!isfinite(o2)) bad |= ST_NONFINITE;
          }
        }
        if (bad) atomicOr(p.status, bad);
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        phz0[r] = phz1[r];
        phz1[r] = phz2[r];
      }
      __syncthreads();  // plane K's slot is refilled at the next step
    }
  }
  return true;
}

template <int COORD, int R, int NW>
__global__ void __launch_bounds__(HeatPcCfg<R, NW>::NT)
    heat_pc_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ HeatParams<float> p) {
  using C = HeatPcCfg<R, NW>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + C::NSLOT * C::SLOT * 4);
  if (smem_u32(smem_raw) & 127u) {
    if (threadIdx.x == 0) atomicOr(p.status, ST_TMA_TIMEOUT);
    return;
  }
  if (p.active && !*p.active) return;  // the clock passed t_end
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < C::NSLOT; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
    tma_prefetch_desc(&tmap);
  }
  __syncthreads();
  unsigned phase_bits = 0, pending = 0;
  const int ntiles = p.ntx * p.nty * p.nzc;
  bool ok = true;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    if (!heat_pc_tile<COORD, R, NW>(p, &tmap, tile, smem_raw, bars, phase_bits, pending)) {
      ok = false;
      break;
    }
  if (!ok && tid == 0)
    for (int s = 0; s < C::NSLOT; ++s)
      if ((pending >> s) & 1u) mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.drain_ns);
}

}  // namespace fvm
