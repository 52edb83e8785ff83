// Fused Navier-Stokes stage kernel: residual (navier_stokes.py:588-711) and
// the Runge-Kutta stage combination (time_integrators.py) in one pass.
//
// Tiling: a block owns a 32 x TY column tile of interior cells and marches a
// chunk of ZC planes along x3.  Each step K (ghosted plane index):
//   A  TMA brings plane K+HH of all 5 conserved variables (tile + HH halo)
//      into a shared-memory ring (one mbarrier per slot, bounded waits);
//   B  v = m/rho on plane K+3                         (viscous only)
//   C  P on plane K+2                     (navier_stokes.py:94-100)
//   D  Stokes stress on plane K+2, zero on ghosts     (viscous only, :102-142)
//   E  x3 MUSCL slopes of cell K+1 for the block's columns (registers)
//   F  x3 face flux at K+1/2 (registers; K-1/2 kept from the previous step)
//   G  x1 slopes, face states and fluxes in registers (one warp per tile
//      row, neighbours by shuffle); x2 slopes -> face states -> fluxes
//      through shared memory; divergence, sources, stage combination,
//      coalesced store of plane K.
// HH = 3 with viscosity (tau at K+2 needs v at K+3), 2 without.
#pragma once
#include "fvm_common.cuh"

namespace fvm {

template <typename Real>
struct NsParams {
  Layout lay;
  Metric<Real> met;
  const Real* u0;     // step base state (ghosted layout), read at the cell
  Real* out;          // stage output (interior written)
  Real* acc;          // k accumulator (interior), may be null
  const double* dt;   // device time step
  const int* active;  // device flag: 0 once t > t_end (the step is a no-op)
  StageCoef coef;
  double gamma, mu, g1, g2, g3;
  unsigned* status;
  int zchunk, ntx, nty, nzc;
  int flat;  // nx3 == 1 with x3 ghosts equal to the plane: x3 fluxes cancel, no z-march
  int ysub;  // register-blocked kernel, flat grids: row tiles a tile marches over along x2
  unsigned long long wait_ns;  // limit of each wait for a TMA plane (ns)
  unsigned long long drain_ns;  // limit of the wait for copies in flight after a timeout (ns)
  unsigned extra_tx;  // test of the timeout path: bytes a ring copy never delivers (0 normally)
};

// Tile sources: one grid (params + tensor map in kernel parameter space) or a
// batch of independent grids (per-instance params and maps in global memory,
// one flat tile list, instance found by binary search over tile offsets).
template <class P>
struct SingleSource {
  CUtensorMap tmap;
  P p;
  __device__ __forceinline__ int total() const { return p.ntx * p.nty * p.nzc; }
  __device__ __forceinline__ int instance(int) const { return 0; }
  __device__ __forceinline__ const P& params(int) const { return p; }
  __device__ __forceinline__ const CUtensorMap* map(int) const { return &tmap; }
  __device__ __forceinline__ int local(int g, int) const { return g; }
};
template <class P>
struct BatchSource {
  const P* prm;             // per instance (this stage)
  const CUtensorMap* maps;  // per instance: map of this stage's input buffer
  const int* tile_start;    // ninst+1 prefix sums of tiles
  int ninst;
  __device__ __forceinline__ int total() const { return __ldg(tile_start + ninst); }
  __device__ __forceinline__ int instance(int g) const {
    int lo = 0, hi = ninst - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(tile_start + mid) <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
  }
  __device__ __forceinline__ const P& params(int i) const { return prm[i]; }
  __device__ __forceinline__ const CUtensorMap* map(int i) const { return maps + i; }
  __device__ __forceinline__ int local(int g, int i) const { return g - __ldg(tile_start + i); }
};

constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int round_up(int a, int b) { return (a + b - 1) / b * b; }
__device__ __forceinline__ int pmod(int a, int m) { int r = a % m; return r < 0 ? r + m : r; }

template <typename Real, bool VISC, int TY>
struct NsCfg {
  static constexpr int TX = 32;
  static constexpr int NT = TX * (TY + 2);
  static constexpr int NV = 5;
  static constexpr int HH = VISC ? 3 : 2;
  static constexpr int W = 40;  // U/v ring column c <-> tile x offset c-4
  static constexpr int ROWS = TY + 2 * HH;
  static constexpr int PL = ROWS * W;  // one U/v field plane
  static constexpr int NSLOT = HH + 2;
  static constexpr int SLOT = round_up(NV * PL * (int)sizeof(Real), 128) / (int)sizeof(Real);
  // P and tau planes cover the tile plus 2 cells: column c2 <-> x offset c2-2,
  // row r2 <-> y offset r2-2
  static constexpr int W2 = TX + 4;
  static constexpr int R2 = TY + 4;
  static constexpr int PL2 = W2 * R2;
  static constexpr int NREC = VISC ? 9 : 6;
  static constexpr int XB = cmax(TY * (TX + 2), (TY + 2) * TX);  // slopes of one field
  static constexpr int FB = cmax(TY * (TX + 1), (TY + 1) * TX);  // fluxes of one variable
  static constexpr int OFF_U = 0;
  static constexpr int OFF_V = OFF_U + NSLOT * SLOT;
  static constexpr int OFF_P = OFF_V + (VISC ? 3 * 3 * PL : 0);
  static constexpr int OFF_T = OFF_P + 3 * PL2;
  static constexpr int OFF_S = OFF_T + (VISC ? 3 * 6 * PL2 : 0);
  static constexpr int OFF_FB = OFF_S + NREC * XB;
  // x1 halo data per plane parity: slopes of the cell left of the tile (per
  // field and row) and fluxes through the tile's right edge (per row)
  static constexpr int OFF_HL = OFF_FB + 5 * FB;
  static constexpr int OFF_FR = OFF_HL + 2 * NREC * TY;
  // float32 inviscid: U0 and acc of the plane's output cells, copied in by
  // cp.async at the start of each step ([U0 | acc][variable][output thread])
  static constexpr bool STAGED = sizeof(Real) == 4 && !VISC;
  static constexpr int OFF_G = OFF_FR + 2 * 5 * TY;
  static constexpr int END = OFF_G + (STAGED ? 2 * 5 * TX * TY : 0);
  static constexpr int BYTES = round_up(END * (int)sizeof(Real), 16) + NSLOT * 8;
  static constexpr unsigned TX_BYTES = NV * PL * sizeof(Real);
};

// Normal fluxes and wave data of one face state along axis D
// (navier_stokes.py:159-316).  q = [rho, m1, m2, m3, e, P, tau_D1, tau_D2, tau_D3].
template <typename R, int D, bool VISC>
__device__ __forceinline__ void ns_face(const R* q, R gam, R Fc[5], R Fd[5], R& vn, R& cs) {
  const R rho = q[0];
  R v0, v1, v2, E, ir = R(0);
  if constexpr (sizeof(R) == 4) {
    ir = rcp_approx(rho);
    v0 = q[1] * ir; v1 = q[2] * ir; v2 = q[3] * ir; E = q[4] * ir;
  } else {
    v0 = q[1] / rho; v1 = q[2] / rho; v2 = q[3] / rho; E = q[4] / rho;
  }
  const R P = q[5];
  const R va = D == 0 ? v0 : (D == 1 ? v1 : v2);
  Fc[0] = rho * va;
  Fc[1] = (rho * v0) * va;
  Fc[2] = (rho * v1) * va;
  Fc[3] = (rho * v2) * va;
  Fc[1 + D] = Fc[1 + D] + P;
  Fc[4] = ((rho * E) + P) * va;
  if constexpr (VISC) {
    Fd[0] = R(0);
    Fd[1] = -q[6];
    Fd[2] = -q[7];
    Fd[3] = -q[8];
    Fd[4] = (((-q[6]) * v0) - (q[7] * v1)) - (q[8] * v2);
  }
  if constexpr (sizeof(R) == 4) cs = sqrt_approx((gam * P) * ir);
  else cs = sqrt((gam * P) / rho);
  vn = va;
}

// Riemann flux + centred diffusive flux (riemann_solvers.py, diffusive_solvers.py).
template <typename R, int D, int RIEM, bool VISC>
__device__ __forceinline__ void ns_flux(const R* qL, const R* qR, R gam, R F[5]) {
  R FcL[5], FcR[5], FdL[5], FdR[5], vnL, vnR, csL, csR;
  ns_face<R, D, VISC>(qL, gam, FcL, FdL, vnL, csL);
  ns_face<R, D, VISC>(qR, gam, FcR, FdR, vnR, csR);
  if constexpr (RIEM == RIEM_HLL) {
    const R smin = fmin(vnL - csL, vnR - csR);
    const R smax = fmax(vnL + csL, vnR + csR);
    const R den = smax - smin;
    const R rden = recip(den);
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const R num = ((smax * FcL[v]) - (smin * FcR[v])) + ((smin * smax) * (qR[v] - qL[v]));
      R mid;
      if constexpr (sizeof(R) == 4) mid = num * rden;
      else mid = num / den;
      F[v] = smin >= R(0) ? FcL[v] : (smax <= R(0) ? FcR[v] : mid);
    }
  } else {
    const R vs = fmax(fabs(vnL) + csL, fabs(vnR) + csR);
#pragma unroll
    for (int v = 0; v < 5; ++v) F[v] = ((FcL[v] + FcR[v]) / R(2)) - ((vs * (qR[v] - qL[v])) / R(2));
  }
  if constexpr (VISC) {
#pragma unroll
    for (int v = 1; v < 5; ++v) F[v] = F[v] + ((FdL[v] + FdR[v]) / R(2));
  }
}

template <typename Real, int LIM, int RIEM, int COORD, bool VISC, int TY, int MINB, class Src>
__global__ void __launch_bounds__(NsCfg<Real, VISC, TY>::NT, MINB)
    ns_stage_kernel(const __grid_constant__ Src src) {
  using C = NsCfg<Real, VISC, TY>;
  using G = Geo<Real, COORD>;
  constexpr int TX = C::TX, NT = C::NT, W = C::W, PL = C::PL, HH = C::HH, NREC = C::NREC;
  constexpr int W2 = C::W2, PL2 = C::PL2;
  constexpr bool F32 = sizeof(Real) == 4;
  // U0/acc of each step's output cells: loaded into registers at the start of
  // the step where registers permit (EARLY); the float32 inviscid kernels (64
  // registers) copy them into shared memory instead (C::STAGED)
  constexpr bool EARLY = VISC;
  constexpr bool STAGED = C::STAGED;
  constexpr int NO = TX * TY;  // output threads
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Real* sm = reinterpret_cast<Real*>(smem_raw);
  Real* uring = sm + C::OFF_U;
  Real* vring = sm + C::OFF_V;
  Real* pring = sm + C::OFF_P;
  Real* tring = sm + C::OFF_T;
  Real* sl = sm + C::OFF_S;
  Real* fb = sm + C::OFF_FB;
  Real* hl = sm + C::OFF_HL;
  Real* fr = sm + C::OFF_FR;
  Real* gst = sm + C::OFF_G;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + (C::BYTES - C::NSLOT * 8));

  if (smem_u32(smem_raw) & 127u) {  // TMA destinations need 128-byte alignment
    if (threadIdx.x == 0) atomicOr(src.params(0).status, ST_TMA_TIMEOUT);
    return;
  }
  const int tid = threadIdx.x;
  if (tid == 0) {
    for (int s = 0; s < C::NSLOT; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  unsigned phase_bits = 0;  // expected parity per slot (identical in all threads)
  unsigned pending = 0;     // slots with a load in flight (meaningful in thread 0)

  // Value of recon field f (U 0..4, P 5, tau row-d component 6..8) at tile
  // offset (tx, ty) of one plane, given that plane's ring bases (computed once
  // per step); ti = tau indices of the row of the face axis.
  auto field = [&](const Real* ub, const Real* pb, const Real* tb, const int* ti, int f, int tx, int ty) -> Real {
    if (f < 5) return ub[f * PL + (ty + HH) * W + tx + 4];
    if (f == 5) return pb[(ty + 2) * W2 + tx + 2];
    return tb[ti[f - 6] * PL2 + (ty + 2) * W2 + tx + 2];
  };

  const bool is_out = tid < TX * TY;
  const int otx = tid % TX, oty = tid / TX;

  const int ntiles = src.total();
  bool ok = true;
  for (int gtile = blockIdx.x; gtile < ntiles && ok; gtile += gridDim.x) {
    const int inst = src.instance(gtile);
    const NsParams<Real>& p = src.params(inst);
    if (p.active && !*p.active) continue;  // this grid's clock passed t_end
    const CUtensorMap* tmap = src.map(inst);
    const int tile = src.local(gtile, inst);
    const Layout& L = p.lay;
    const int nx = L.nx, ny = L.ny, nz = L.nz;
    const Real gam = Real(p.gamma), mu = Real(p.mu);
    const Real dt = Real(*p.dt);
    const bool flat = p.flat != 0;
    if (tid == 0) tma_prefetch_desc(tmap);
    const int tx_i = tile % p.ntx;
    const int ty_i = (tile / p.ntx) % p.nty;
    const int zc_i = tile / (p.ntx * p.nty);
    const int x0 = tx_i * TX, y0 = ty_i * TY;
    const int Z0 = 1 + zc_i * p.zchunk;         // first ghosted output plane
    const int Zl = min(Z0 + p.zchunk - 1, nz);  // last ghosted output plane
    // flat grids: only plane 1, no x3 pipeline
    const int Pfirst = flat ? Z0 : Z0 - HH, Plast = flat ? Zl : Zl + HH;
    const int Kfirst = flat ? Z0 : Z0 - 4;  // first step: P (and tau) of plane Z0-2

    const int oi = x0 + otx, oj = y0 + oty;  // output cell (interior 0-based)
    const bool out_valid = is_out && oi < nx && oj < ny;
    Real zs[NREC];
    Real Fzp[5], Fzn[5];
#pragma unroll
    for (int f = 0; f < NREC; ++f) zs[f] = Real(0);
#pragma unroll
    for (int v = 0; v < 5; ++v) { Fzp[v] = Real(0); Fzn[v] = Real(0); }
    const Real S3c = out_valid ? G::S3(p.met, oi, oj) : Real(0);

    auto issue = [&](int pl) {
      const int s = pmod(pl, C::NSLOT);
      pending |= 1u << s;
      fence_proxy_async();
      mbar_arrive_expect_tx(&bars[s], C::TX_BYTES + p.extra_tx);
      tma_load_4d(&uring[s * C::SLOT], tmap, &bars[s], x0 - 3 + L.padx, y0 + 1 - HH, pl, 0);
    };
    // planes needed by the first step plus one of prefetch
    if (tid == 0)
      for (int pl = Pfirst; pl <= Kfirst + HH + 1 && pl <= Plast; ++pl) issue(pl);

    // Ring slots of plane K+d, d >= 0 small: bu = K mod NSLOT and b3 = K mod 3
    // are carried from step to step, so each slot is a compare and subtract.
    for (int K = Kfirst, bu = pmod(Kfirst, C::NSLOT), b3 = pmod(Kfirst, 3); K <= Zl;
         ++K, bu = (bu + 1 == C::NSLOT ? 0 : bu + 1), b3 = (b3 == 2 ? 0 : b3 + 1)) {
      auto su = [&](int d) { const int t = bu + d; return t >= C::NSLOT ? t - C::NSLOT : t; };  // d < NSLOT
      auto s3 = [&](int d) { const int t = b3 + d; return t >= 3 ? t - 3 : t; };                // d <= 3
      // ---------------------------------------------------------- A ----
      {
        bool got = true;
        const int wlast = flat ? K : K + HH;
        for (int pl = (K == Kfirst ? Pfirst : K + HH); pl <= wlast; ++pl) {
          // the phase bit flips (and thread 0 drops the slot from `pending`)
          // only after a completed wait, so a drain after a timeout waits for
          // the phase still outstanding
          const int s = su(pl - K);
          const bool g = got && mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, p.wait_ns);
          if (g) {
            phase_bits ^= (1u << s);
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
      // Prefetch plane K+HH+1 into the slot of plane K-1.  Issued after the
      // barrier above, which every thread reaches only after its last read of
      // plane K-1 (the previous step's output phase), so the steps need no
      // barrier at their end.
      if (tid == 0 && K > Kfirst && K + HH + 1 <= Plast) issue(K + HH + 1);
      const int sK = su(0), sK1 = su(1), sK2 = su(2);
      // ring bases of planes K, K+1, K+2 (uniform, once per step)
      const Real* uK = uring + sK * C::SLOT;
      const Real* uK1 = uring + sK1 * C::SLOT;
      const Real* uK2 = uring + sK2 * C::SLOT;
      const Real* pK = pring + s3(0) * PL2;
      const Real* pK1 = pring + s3(1) * PL2;
      const Real* pK2 = pring + s3(2) * PL2;
      const Real* tK = tring + s3(0) * 6 * PL2;
      const Real* tK1 = tring + s3(1) * 6 * PL2;
      const Real* tK2 = tring + s3(2) * 6 * PL2;
      // U0 and acc of this plane's output cells, fetched here so that the
      // whole step hides their latency: into registers (EARLY), into this
      // thread's shared-memory slots (STAGED), or else lane 0 of each output
      // row asks L2 for the rows and the output phase loads them.
      Real eu0[5], eacc[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) { eu0[v] = Real(0); eacc[v] = Real(0); }
      if (K >= Z0 && out_valid) {
        const long long g0 = L.idx(0, K, oj + 1, oi + 1);
        if constexpr (EARLY) {
#pragma unroll
          for (int v = 0; v < 5; ++v) {
            if (needs_u0<Real>(p.coef) && !p.coef.u0_is_input) eu0[v] = p.u0[g0 + v * L.var_stride];
            if (needs_acc(p.coef)) eacc[v] = p.acc[g0 + v * L.var_stride];
          }
        } else if constexpr (STAGED) {
#pragma unroll
          for (int v = 0; v < 5; ++v) {
            if (needs_u0<Real>(p.coef) && !p.coef.u0_is_input) cp_async4(&gst[v * NO + tid], p.u0 + g0 + v * L.var_stride);
            if (needs_acc(p.coef)) cp_async4(&gst[(5 + v) * NO + tid], p.acc + g0 + v * L.var_stride);
          }
        } else if (otx == 0) {
          for (int v = 0; v < 5; ++v) {
            if (needs_u0<Real>(p.coef) && !p.coef.u0_is_input) prefetch_l2(p.u0 + g0 + v * L.var_stride);
            if (needs_acc(p.coef)) prefetch_l2(p.acc + g0 + v * L.var_stride);
          }
        }
      }
      // ---------------------------------------------------------- B ----
      // v on the newest plane(s), tile + 3 (viscous only)
      if constexpr (VISC) {
        for (int pl = (K == Kfirst ? Pfirst : K + 3); pl <= K + 3; ++pl) {
          const Real* ub = uring + su(pl - K) * C::SLOT;  // pl - K in 1..3
          Real* vb = vring + s3(pl - K) * 3 * PL;
          for (int it = tid; it < C::ROWS * (TX + 6); it += NT) {
            const int r = it / (TX + 6), c = 1 + it % (TX + 6);
            const int o = r * W + c;
            const Real rho = ub[o];
            if constexpr (F32) {
              const Real ir = rcp_approx(rho);
              vb[o] = ub[PL + o] * ir;
              vb[PL + o] = ub[2 * PL + o] * ir;
              vb[2 * PL + o] = ub[3 * PL + o] * ir;
            } else {
              vb[o] = ub[PL + o] / rho;
              vb[PL + o] = ub[2 * PL + o] / rho;
              vb[2 * PL + o] = ub[3 * PL + o] / rho;
            }
          }
        }
      }
      // ---------------------------------------------------------- C ----
      // P on plane K+2, tile + 2 (navier_stokes.py:94-100); with viscosity it
      // is formed inside the stress loop below (same cells)
      Real* const pw = pring + s3(flat ? 0 : 2) * PL2;
      const Real* const usrc = flat ? uK : uK2;
      auto pressure_at = [&](int it) {
        const int r2 = it / W2, c2 = it % W2;
        const Real* u = usrc + (r2 + HH - 2) * W + c2 + 2;
        const Real rho = u[0];
        Real v0, v1, v2, E;
        if constexpr (F32) {
          const Real ir = rcp_approx(rho);
          v0 = u[PL] * ir; v1 = u[2 * PL] * ir; v2 = u[3 * PL] * ir;
          E = u[4 * PL] * ir;
        } else {
          v0 = u[PL] / rho; v1 = u[2 * PL] / rho; v2 = u[3 * PL] / rho;
          E = u[4 * PL] / rho;
        }
        pw[it] = ((gam - Real(1)) * rho) * (E - (((v0 * v0) + (v1 * v1)) + (v2 * v2)) / Real(2));
      };
      if constexpr (!VISC) {
        for (int it = tid; it < C::PL2; it += NT) pressure_at(it);
      } else {
        __syncthreads();  // v of plane K+3 (phase B) before the stress loop
      }
      // ---------------------------------------------------------- D ----
      // Stokes stress on plane K+2, tile + 2, zero on ghosts (:102-142)
      if constexpr (VISC) {
        const int pl = K + 2;
        const int k = pl - 1;  // interior plane index
        const bool zghost = (k < 0 || k >= nz);
        const Real* vm = vring + s3(1) * 3 * PL;  // v of planes K+1, K+2, K+3
        const Real* v0p = vring + s3(2) * 3 * PL;
        const Real* vp = vring + s3(3) * 3 * PL;
        Real* tw = tring + s3(2) * 6 * PL2;
        for (int it = tid; it < C::PL2; it += NT) {
          pressure_at(it);
          const int r2 = it / W2, c2 = it % W2;
          const int r = r2 + 1, c = c2 + 2;
          const int i = x0 + c2 - 2, j = y0 + r2 - 2;
          Real t[6];
          if (zghost || i < 0 || i >= nx || j < 0 || j >= ny) {
#pragma unroll
            for (int m = 0; m < 6; ++m) t[m] = Real(0);
          } else {
            Real g[3][3];  // g[cc][a] = d v_cc / d x_a
            if constexpr (F32) {
              const Real h1 = 0.5f * inv_len<Real, COORD, 0>(p.met, i, j, k);
              const Real h2 = 0.5f * inv_len<Real, COORD, 1>(p.met, i, j, k);
              const Real h3 = 0.5f * inv_len<Real, COORD, 2>(p.met, i, j, k);
#pragma unroll
              for (int cc = 0; cc < 3; ++cc) {
                const int o = cc * PL + r * W + c;
                g[cc][0] = (v0p[o + 1] - v0p[o - 1]) * h1;
                g[cc][1] = (v0p[o + W] - v0p[o - W]) * h2;
                g[cc][2] = (vp[o] - vm[o]) * h3;
              }
            } else {
              const Real l1 = G::L1(p.met, i, j, k), l2 = G::L2(p.met, i, j, k), l3 = G::L3(p.met, i, j, k);
#pragma unroll
              for (int cc = 0; cc < 3; ++cc) {
                const int o = cc * PL + r * W + c;
                g[cc][0] = (v0p[o + 1] - v0p[o - 1]) / (Real(2) * l1);
                g[cc][1] = (v0p[o + W] - v0p[o - W]) / (Real(2) * l2);
                g[cc][2] = (vp[o] - vm[o]) / (Real(2) * l3);
              }
            }
            const Real tt = Real(2.0 / 3.0);
            if constexpr (COORD == COORD_CART) {
              const Real divv = (g[0][0] + g[1][1]) + g[2][2];
              t[0] = mu * ((Real(2) * g[0][0]) - (tt * divv));
              t[1] = mu * ((Real(2) * g[1][1]) - (tt * divv));
              t[2] = mu * ((Real(2) * g[2][2]) - (tt * divv));
              t[3] = mu * (g[0][1] + g[1][0]);
              t[4] = mu * (g[0][2] + g[2][0]);
              t[5] = mu * (g[1][2] + g[2][1]);
            } else {
              Lame<Real> lm;
              lame_at<Real, COORD>(p.met, i, j, lm);
              const Real v0 = v0p[r * W + c], v1 = v0p[PL + r * W + c], v2 = v0p[2 * PL + r * W + c];
              const Real divv = (((((g[0][0] + g[1][1]) + g[2][2]) + ((v0 * (lm.dl[0][1] + lm.dl[0][2])) / lm.h[0])) +
                                  ((v1 * (lm.dl[1][0] + lm.dl[1][2])) / lm.h[1])) +
                                 ((v2 * (lm.dl[2][0] + lm.dl[2][1])) / lm.h[2]));
              t[0] = mu * ((Real(2) * g[0][0]) - (tt * divv));
              t[1] = mu * ((Real(2) * (g[1][1] + ((v0 * lm.dl[0][1]) / lm.h[0]))) - (tt * divv));
              t[2] = mu * ((Real(2) * ((g[2][2] + ((v0 * lm.dl[0][2]) / lm.h[0])) + ((v1 * lm.dl[1][2]) / lm.h[1]))) -
                           (tt * divv));
              t[3] = mu * (((g[0][1] + g[1][0]) - ((v1 * lm.dl[0][1]) / lm.h[0])) + ((v0 * lm.dl[1][0]) / lm.h[1]));
              t[4] = mu * (((g[0][2] + g[2][0]) - ((v2 * lm.dl[0][2]) / lm.h[0])) + ((v0 * lm.dl[2][0]) / lm.h[2]));
              t[5] = mu * (((g[1][2] + g[2][1]) - ((v2 * lm.dl[1][2]) / lm.h[1])) + ((v1 * lm.dl[2][1]) / lm.h[2]));
            }
          }
#pragma unroll
          for (int m = 0; m < 6; ++m) tw[m * PL2 + it] = t[m];
        }
      }
      __syncthreads();
      // -------------------------------------------------------- E, F ----
      // x3 slopes of cell K+1 and the x3 face flux at K+1/2 (registers);
      // tau row 3 = (t13, t23, t33)
      if (!flat && K >= Z0 - 2 && is_out) {
        constexpr int ti[3] = {4, 5, 2};
        const int kk = K;  // interior index of plane K+1
        const bool ghost = (K + 1 <= 0 || K + 1 >= nz + 1);
        Real zn[NREC];
        Real qm[NREC], q0[NREC], qp[NREC];
#pragma unroll
        for (int f = 0; f < NREC; ++f) {
          qm[f] = field(uK, pK, tK, ti, f, otx, oty);
          q0[f] = field(uK1, pK1, tK1, ti, f, otx, oty);
          qp[f] = field(uK2, pK2, tK2, ti, f, otx, oty);
        }
        if (ghost || !out_valid) {
#pragma unroll
          for (int f = 0; f < NREC; ++f) zn[f] = Real(0);
        } else {
          const Real l3 = F32 ? Real(1) : G::L3(p.met, oi, oj, kk);
#pragma unroll
          for (int f = 0; f < NREC; ++f) zn[f] = muscl_slope<LIM>(qm[f], q0[f], qp[f], l3);
        }
        if (K >= Z0 - 1) {
          Real qL[NREC], qR[NREC], F[5];
#pragma unroll
          for (int f = 0; f < NREC; ++f) {
            qL[f] = qm[f] + zs[f] / Real(2);
            qR[f] = q0[f] - zn[f] / Real(2);
          }
          ns_flux<Real, 2, RIEM, VISC>(qL, qR, gam, F);
#pragma unroll
          for (int v = 0; v < 5; ++v) { Fzp[v] = Fzn[v]; Fzn[v] = F[v] * S3c; }
        }
#pragma unroll
        for (int f = 0; f < NREC; ++f) zs[f] = zn[f];
      }
      // ------------------------------------------------------ x1 halo ----
      // While the output warps run E and F, the spare warps form the x1 halo
      // data of plane Kh (the next output plane; on a flat grid this one):
      // the first spare warp the slopes of the cell left of the tile, the
      // second the flux through the tile's right edge, one lane per row.
      {
        const int Kh = flat ? K : K + 1;
        const int hh = tid - TX * TY, row = hh & 31;
        if (!is_out && row < TY && Kh >= Z0 && Kh <= Zl) {
          constexpr int ti[3] = {0, 3, 4};  // tau row 1 = (t11, t12, t13)
          const Real* uh = uring + su(Kh - K) * C::SLOT;
          const Real* ph = pring + s3(Kh - K) * PL2;
          const Real* th = tring + s3(Kh - K) * 6 * PL2;
          const int kh = Kh - 1, j = y0 + row, par = Kh & 1;
          if (hh < 32) {
            const int i = x0 - 1;
            const bool in = i >= 0 && j < ny;  // i < nx as x0 < nx
            const Real l1 = (F32 || !in) ? Real(1) : G::L1(p.met, i, j, kh);
#pragma unroll
            for (int f = 0; f < NREC; ++f)
              hl[(par * NREC + f) * TY + row] =
                  in ? muscl_slope<LIM>(field(uh, ph, th, ti, f, -2, row), field(uh, ph, th, ti, f, -1, row),
                                        field(uh, ph, th, ti, f, 0, row), l1)
                     : Real(0);
          } else {
            const int i = x0 + TX;  // face between cells i-1 and i
            Real F[5] = {Real(0), Real(0), Real(0), Real(0), Real(0)};
            if (i <= nx && j < ny) {
              const bool in0 = i < nx;  // cell i-1 is interior here
              const Real l1m = F32 ? Real(1) : G::L1(p.met, i - 1, j, kh);
              const Real l1 = (F32 || !in0) ? Real(1) : G::L1(p.met, i, j, kh);
              Real qL[NREC], qR[NREC];
#pragma unroll
              for (int f = 0; f < NREC; ++f) {
                const Real fa = field(uh, ph, th, ti, f, TX - 2, row), fb1 = field(uh, ph, th, ti, f, TX - 1, row);
                const Real fc = field(uh, ph, th, ti, f, TX, row), fd = field(uh, ph, th, ti, f, TX + 1, row);
                const Real sm1 = muscl_slope<LIM>(fa, fb1, fc, l1m);
                const Real s0 = in0 ? muscl_slope<LIM>(fb1, fc, fd, l1) : Real(0);
                qL[f] = fb1 + sm1 / Real(2);
                qR[f] = fc - s0 / Real(2);
              }
              ns_flux<Real, 0, RIEM, VISC>(qL, qR, gam, F);
              const Real s1 = G::S1(p.met, i, j, kh);
#pragma unroll
              for (int v = 0; v < 5; ++v) F[v] = F[v] * s1;
            }
#pragma unroll
            for (int v = 0; v < 5; ++v) fr[(par * 5 + v) * TY + row] = F[v];
          }
        }
      }
      if (K < Z0) { __syncthreads(); continue; }
      if (flat) __syncthreads();  // a flat grid's halo data is this step's
      const int kK = K - 1;  // interior index of the output plane
      // ------------------------------------------------------ G: x1 ----
      // Warp w < TY owns tile row w.  Each lane forms the x1 slopes of its
      // cell and the flux through the cell's left face in registers; the left
      // cell's slope comes from the previous lane (shuffle) and, for lane 0,
      // from the halo data.  The right-face flux is the next lane's left-face
      // flux and, for lane 31, the halo flux through the tile's right edge.
      // Each face's arithmetic is that of a slopes-then-faces pass, so the
      // results are the same.
      Real Fxm[5], Fxp[5];
      if (is_out) {
        constexpr int ti[3] = {0, 3, 4};  // tau row 1 = (t11, t12, t13)
        const int tx = otx, ty = oty, par = K & 1;
        const int i = x0 + tx, j = y0 + ty;
        const bool in0 = i < nx && j < ny;  // this cell (i >= 0)
        const Real l1 = (F32 || !in0) ? Real(1) : G::L1(p.met, i, j, kK);
        Real qL[NREC], qR[NREC];
#pragma unroll
        for (int f = 0; f < NREC; ++f) {
          const Real fm = field(uK, pK, tK, ti, f, tx - 1, ty);
          const Real f0 = field(uK, pK, tK, ti, f, tx, ty);
          const Real s0 = in0 ? muscl_slope<LIM>(fm, f0, field(uK, pK, tK, ti, f, tx + 1, ty), l1) : Real(0);
          const Real su = __shfl_up_sync(0xffffffffu, s0, 1);
          const Real sh = hl[(par * NREC + f) * TY + ty];
          qL[f] = fm + (tx == 0 ? sh : su) / Real(2);
          qR[f] = f0 - s0 / Real(2);
        }
        Real F[5] = {Real(0), Real(0), Real(0), Real(0), Real(0)};
        if (i <= nx && j < ny) {  // face i, between cells i-1 and i
          ns_flux<Real, 0, RIEM, VISC>(qL, qR, gam, F);
          const Real s1 = G::S1(p.met, i, j, kK);
#pragma unroll
          for (int v = 0; v < 5; ++v) F[v] = F[v] * s1;
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          Fxm[v] = F[v];
          const Real fd = __shfl_down_sync(0xffffffffu, F[v], 1);
          const Real fe = fr[(par * 5 + v) * TY + ty];
          Fxp[v] = tx == TX - 1 ? fe : fd;
        }
      }
      // ------------------------------------------------ G: x2 slopes ----
      {
        constexpr int ti[3] = {3, 1, 5};  // tau row 2 = (t12, t22, t23)
        static_assert((TY + 2) * TX == NT, "one x2-slope task per thread");
        {
          const int it = tid;
          const int ty = it / TX - 1, tx = it % TX;
          const int i = x0 + tx, j = y0 + ty;
          const bool interior = i < nx && j >= 0 && j < ny;
          const Real l2 = (F32 || !interior) ? Real(1) : G::L2(p.met, i, j, kK);
#pragma unroll
          for (int f = 0; f < NREC; ++f) {
            const Real s = interior ? muscl_slope<LIM>(field(uK, pK, tK, ti, f, tx, ty - 1), field(uK, pK, tK, ti, f, tx, ty),
                                                       field(uK, pK, tK, ti, f, tx, ty + 1), l2)
                                    : Real(0);
            sl[f * C::XB + it] = s;
          }
        }
      }
      __syncthreads();
      {
        constexpr int ti[3] = {3, 1, 5};
        if (tid < (TY + 1) * TX) {
          const int it = tid;
          const int fy = it / TX, tx = it % TX;
          const int fj = y0 + fy, i = x0 + tx;
          Real F[5] = {Real(0), Real(0), Real(0), Real(0), Real(0)};
          if (fj <= ny && i < nx) {
            Real qL[NREC], qR[NREC];
            const int oL = fy * TX + tx;  // slope slot of the lower cell (ty = fy-1)
#pragma unroll
            for (int f = 0; f < NREC; ++f) {
              qL[f] = field(uK, pK, tK, ti, f, tx, fy - 1) + sl[f * C::XB + oL] / Real(2);
              qR[f] = field(uK, pK, tK, ti, f, tx, fy) - sl[f * C::XB + oL + TX] / Real(2);
            }
            ns_flux<Real, 1, RIEM, VISC>(qL, qR, gam, F);
            const Real s2 = G::S2(p.met, i, fj, kK);
#pragma unroll
            for (int v = 0; v < 5; ++v) F[v] = F[v] * s2;
          }
#pragma unroll
          for (int v = 0; v < 5; ++v) fb[v * C::FB + it] = F[v];
        }
      }
      __syncthreads();
      // ------------------------------------------------- G: output ----
      if (out_valid) {
        const int r = oty + HH, c = otx + 4;
        Real q[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) q[v] = uK[v * PL + r * W + c];
        const Real rho = q[0];
        Real v0, v1, v2;
        if constexpr (F32) {
          const Real ir = rcp_approx(rho);
          v0 = q[1] * ir; v1 = q[2] * ir; v2 = q[3] * ir;
        } else {
          v0 = q[1] / rho; v1 = q[2] / rho; v2 = q[3] / rho;
        }
        // sources: geometric (navier_stokes.py:437-452) + gravity (:499-504)
        Real src[5];
        const Real gx = Real(p.g1), gy = Real(p.g2), gz = Real(p.g3);
        src[0] = Real(0);
        src[1] = rho * gx;
        src[2] = rho * gy;
        src[3] = rho * gz;
        src[4] = rho * (((gx * v0) + (gy * v1)) + (gz * v2));
        if constexpr (COORD != COORD_CART) {
          Lame<Real> lm;
          lame_at<Real, COORD>(p.met, oi, oj, lm);
          const Real P = pK[(oty + 2) * W2 + otx + 2];
          const Real vv[3] = {v0, v1, v2};
          Real tc[3][3];
          if constexpr (VISC) {
            const int r2 = oty + 2, c2 = otx + 2;
            const Real* tc0 = tK + r2 * W2 + c2;
            tc[0][0] = tc0[0]; tc[1][1] = tc0[PL2]; tc[2][2] = tc0[2 * PL2];
            tc[0][1] = tc[1][0] = tc0[3 * PL2];
            tc[0][2] = tc[2][0] = tc0[4 * PL2];
            tc[1][2] = tc[2][1] = tc0[5 * PL2];
          } else {
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
              for (int b = 0; b < 3; ++b) tc[a][b] = Real(0);
          }
#pragma unroll
          for (int cc = 0; cc < 3; ++cc) {
            const int o0 = cc == 0 ? 1 : 0, o1 = cc == 2 ? 1 : 2;
            const Real sgc = (((((P * lm.d123[cc]) / lm.h[cc]) + ((((rho * vv[o0]) * vv[o0]) * lm.dl[cc][o0]) / lm.h[cc])) +
                               ((((rho * vv[o1]) * vv[o1]) * lm.dl[cc][o1]) / lm.h[cc])) -
                              ((((rho * vv[cc]) * vv[o0]) * lm.dl[o0][cc]) / lm.h[o0])) -
                             ((((rho * vv[cc]) * vv[o1]) * lm.dl[o1][cc]) / lm.h[o1]);
            const Real sgd = ((((tc[cc][o0] * lm.dl[o0][cc]) / lm.h[o0]) + ((tc[cc][o1] * lm.dl[o1][cc]) / lm.h[o1])) -
                              ((tc[o0][o0] * lm.dl[cc][o0]) / lm.h[cc])) -
                             ((tc[o1][o1] * lm.dl[cc][o1]) / lm.h[cc]);
            src[1 + cc] = (sgc + sgd) + src[1 + cc];
          }
        }
        const Real Vc = G::V(p.met, oi, oj, kK);
        const Real iV = recip(Vc);
        const long long gidx = L.idx(0, K, oj + 1, oi + 1);
        // residual of each variable first (the flux registers die), then
        // every global load of the cell before its first store: the stores
        // may alias later loads as far as the compiler knows, which would
        // otherwise cost one memory round trip per variable
        Real kv[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const Real Fym = fb[v * C::FB + oty * TX + otx];
          const Real Fyp = fb[v * C::FB + (oty + 1) * TX + otx];
          const Real sum = ((((Fxp[v] - Fxm[v]) + Fyp) - Fym) + Fzn[v]) - Fzp[v];
          if constexpr (F32) kv[v] = (-sum) * iV + src[v];
          else kv[v] = (-sum) / Vc + src[v];
        }
        Real u0v[5], accv[5];
        if constexpr (STAGED) cp_async_wait_all();
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const long long gi = gidx + (long long)v * L.var_stride;
          if constexpr (STAGED) {
            u0v[v] = needs_u0<Real>(p.coef) ? (p.coef.u0_is_input ? q[v] : gst[v * NO + tid]) : Real(0);
            accv[v] = needs_acc(p.coef) ? gst[(5 + v) * NO + tid] : Real(0);
          } else if constexpr (EARLY) {
            u0v[v] = (needs_u0<Real>(p.coef) && p.coef.u0_is_input) ? q[v] : eu0[v];
            accv[v] = eacc[v];
          } else {
            u0v[v] = needs_u0<Real>(p.coef) ? (p.coef.u0_is_input ? q[v] : p.u0[gi]) : Real(0);
            accv[v] = needs_acc(p.coef) ? p.acc[gi] : Real(0);
          }
        }
        unsigned bad = 0;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const long long gi = gidx + (long long)v * L.var_stride;
          const Real o = stage_combine(p.coef, dt, kv[v], q[v], u0v[v], accv[v]);
          p.out[gi] = o;
          if (p.coef.accmode != ACC_NONE) p.acc[gi] = acc_update(p.coef, dt, kv[v], u0v[v], accv[v]);
          if (!isfinite(o)) bad |= ST_NONFINITE;
          if (v == 0 && p.coef.mode != MODE_RHS && !(o > Real(0))) bad |= ST_DENSITY;
        }
        if (bad) atomicOr(p.status, bad);
      }
    }
    __syncthreads();  // the next tile's first loads reuse every ring slot
  }
  if constexpr (STAGED) cp_async_wait_all();  // none left in flight at exit
  // On a timeout, wait (bounded) for every load this block may still have in flight.
  if (!ok && tid == 0) {
    for (int s = 0; s < C::NSLOT; ++s)
      if ((pending >> s) & 1u) mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, src.params(0).drain_ns);
  }
}

}  // namespace fvm
