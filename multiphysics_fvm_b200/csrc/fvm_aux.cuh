// Auxiliary kernels: ghost fill, layout transposes, CFL reduction, totals.
#pragma once
#include "fvm_common.cuh"

namespace fvm {

struct BcSpec {
  signed char kind[6][6];  // [var][side]: 0 periodic, 1 neumann, 2 reflecting, 3 dirichlet
  double value[6][6];
};

// Reference layout (C order, last axis fastest) <-> device layout (x1 fastest).
// src/dst reference arrays have dims (nv, m1, m2, m3) and map to ghosted device
// indices g = m + off.  32x32 shared-memory tiles over (x1, x3) per (var, x2).
// Ghost edges and corners of a reference-layout float64 state (NV, n1+2,
// n2+2, n3+2) on the device, as src/solver.py:39-61: an edge is the mean of
// the two adjacent ghost faces, a corner the mean of the three adjacent ghost
// edges.  Edges read only face cells, so they are independent; corners run
// after them.  blockIdx.y = variable * 12 + edge.
__global__ void edges_kernel(double* f, int n1, int n2, int n3) {
  const int N[3] = {n1 + 2, n2 + 2, n3 + 2};
  const int q = blockIdx.y / 12, e = blockIdx.y % 12;
  const int pair = e >> 2, ea = (e >> 1) & 1, eb = e & 1;
  const int a = pair == 2 ? 1 : 0, b = pair == 0 ? 1 : 2, c = 3 - a - b;
  double* g = f + (long long)q * N[0] * N[1] * N[2];
  for (int t = 1 + blockIdx.x * blockDim.x + threadIdx.x; t <= N[c] - 2; t += gridDim.x * blockDim.x) {
    int idx[3], pi[3], qi[3];
    idx[a] = ea ? N[a] - 1 : 0;
    idx[b] = eb ? N[b] - 1 : 0;
    idx[c] = t;
    for (int z = 0; z < 3; ++z) { pi[z] = idx[z]; qi[z] = idx[z]; }
    pi[a] = ea ? N[a] - 2 : 1;
    qi[b] = eb ? N[b] - 2 : 1;
    auto at = [&](const int* x) -> double& { return g[((long long)x[0] * N[1] + x[1]) * N[2] + x[2]]; };
    at(idx) = 0.5 * (at(pi) + at(qi));
  }
}
__global__ void corners_kernel(double* f, int n1, int n2, int n3, int nv) {
  const int N[3] = {n1 + 2, n2 + 2, n3 + 2};
  const int id = threadIdx.x;
  if (id >= 8 * nv) return;
  const int q = id >> 3, ci = (id >> 2) & 1, cj = (id >> 1) & 1, ck = id & 1;
  double* g = f + (long long)q * N[0] * N[1] * N[2];
  auto at = [&](int i, int j, int k) -> double& { return g[((long long)i * N[1] + j) * N[2] + k]; };
  const int i = ci ? N[0] - 1 : 0, j = cj ? N[1] - 1 : 0, k = ck ? N[2] - 1 : 0;
  const int ii = ci ? N[0] - 2 : 1, jj = cj ? N[1] - 2 : 1, kk = ck ? N[2] - 2 : 1;
  at(i, j, k) = (at(ii, j, k) + at(i, jj, k) + at(i, j, kk)) / 3.0;
}

template <typename Real, bool TO_DEVICE>
__global__ void transpose_kernel(const double* __restrict__ hsrc, double* __restrict__ hdst,
                                 const Real* __restrict__ dsrc, Real* __restrict__ ddst, Layout L, int m1,
                                 int m2, int m3, int off) {
  __shared__ double tile[32][33];
  const int q = blockIdx.z / m2, j = blockIdx.z % m2;
  const int k0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  if (TO_DEVICE) {
    for (int m = ty; m < 32; m += 8) {
      const int i = i0 + m, k = k0 + tx;
      if (i < m1 && k < m3) tile[m][tx] = hsrc[(((long long)q * m1 + i) * m2 + j) * m3 + k];
    }
    __syncthreads();
    for (int m = ty; m < 32; m += 8) {
      const int k = k0 + m, i = i0 + tx;
      if (i < m1 && k < m3) ddst[L.idx(q, k + off, j + off, i + off)] = Real(tile[tx][m]);
    }
  } else {
    for (int m = ty; m < 32; m += 8) {
      const int k = k0 + m, i = i0 + tx;
      if (i < m1 && k < m3) tile[tx][m] = double(dsrc[L.idx(q, k + off, j + off, i + off)]);
    }
    __syncthreads();
    for (int m = ty; m < 32; m += 8) {
      const int i = i0 + m, k = k0 + tx;
      if (i < m1 && k < m3) hdst[(((long long)q * m1 + i) * m2 + j) * m3 + k] = tile[m][tx];
    }
  }
}


// ------------------------------------------------------------- batches ----
// Per-instance data of the batched auxiliary kernels.
struct BatchAux {
  Layout lay;
  void* U[3];
  Clock* clk;
  unsigned* status;
  BcSpec bc;
  int nv, cmode;  // clock mode (0 NS rates, 1 fixed, 2 constant)
  int no_x3;      // one-plane grid whose kernels never read the x3 ghost slabs
  double max_inv_l2, const_rate;
};

__device__ __forceinline__ void atomic_max_pos(unsigned long long* a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// CFL rates of the Navier-Stokes state (navier_stokes.py:512-585) in float64:
// red[0] = max_cells max_d max_w |v_d + kappa_w| / L_d, red[1] = max mu/rho.
// Block bx of the nbx blocks that share the grid.
template <typename Real, int COORD>
__device__ __forceinline__ void ns_dt_reduce_body(const Real* __restrict__ u, const Layout& L, const Metric<double>& m,
                                                  double gam, double mu, Clock* clk, unsigned* status, int bx,
                                                  int nbx);

template <typename Real, int COORD>
__global__ void __launch_bounds__(256, 3)
    ns_dt_reduce_kernel(const Real* __restrict__ u, Layout L, Metric<double> m, double gam, double mu, Clock* clk,
                        unsigned* status) {
  ns_dt_reduce_body<Real, COORD>(u, L, m, gam, mu, clk, status, blockIdx.x, gridDim.x);
}

// Per-instance CFL rates of a batch of Navier-Stokes grids: a static list of
// blocks, each grid's count proportional to its cells (DT_CELLS per block, at
// least one), so a large grid does not leave one block per SM working while
// the small grids' blocks have finished.  The maximum does not depend on the
// split: the dt is bitwise that of the single-grid reduction.
constexpr int DT_CELLS = 2048;
struct DtBlock {
  int grid, bx, nbx;
};
struct BatchDt {
  const void* u;
  Layout lay;
  Metric<double> md;
  double gam, mu;
  Clock* clk;
  unsigned* status;
};
template <typename Real, int COORD>
__global__ void __launch_bounds__(256, 3) batch_ns_dt_kernel(const BatchDt* __restrict__ b,
                                                             const DtBlock* __restrict__ blk) {
  const DtBlock k = blk[blockIdx.x];
  const BatchDt& x = b[k.grid];
  ns_dt_reduce_body<Real, COORD>(static_cast<const Real*>(x.u), x.lay, x.md, x.gam, x.mu, x.clk, x.status, k.bx,
                                 k.nbx);
}

template <typename Real, int COORD>
__device__ __forceinline__ void ns_dt_reduce_body(const Real* __restrict__ u, const Layout& L, const Metric<double>& m,
                                                  double gam, double mu, Clock* clk, unsigned* status, int bx,
                                                  int nbx) {
  if (!clk->active) return;
  __shared__ double s_rc[32], s_nu[32];
  double rc = 0.0, nu = 0.0;
  unsigned bad = 0;
  // Work items are 32-cell pieces of x1 rows, one per warp at a time, so narrow
  // grids keep every lane busy.  A warp's items are nwarp apart in the order
  // (piece, j, k); its cursor (c, j, k) advances by that stride with carries,
  // without divisions.  A warp loads IB items ahead of the float64 arithmetic,
  // whose division and square-root chains would otherwise leave the loads
  // exposed.
  constexpr int IB = 2;
  const int nch = (L.nx + 31) >> 5;
  const int lane = threadIdx.x & 31;
  const int nwarp = nbx * (blockDim.x >> 5);
  const int w0 = bx * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int dq = nwarp / nch, dr = nwarp % nch, rj = dq % L.ny, rk = dq / L.ny;
  int cc = w0 % nch, cj = (w0 / nch) % L.ny, ck = (w0 / nch) / L.ny;  // load cursor
  auto advance = [&]() {
    cc += dr;
    cj += rj;
    ck += rk;
    if (cc >= nch) { cc -= nch; cj += 1; }
    if (cj >= L.ny) { cj -= L.ny; ck += 1; }
  };
  auto load = [&](Real* q, int* ijk) {
    const int i = cc * 32 + lane;
    const bool in = ck < L.nz && i < L.nx;
    ijk[0] = in ? i : -1;
    ijk[1] = cj;
    ijk[2] = ck;
    const long long g = in ? L.idx(0, ck + 1, cj + 1, i + 1) : 0;
#pragma unroll
    for (int v = 0; v < 5; ++v) q[v] = in ? u[g + v * L.var_stride] : Real(1);
    advance();
  };
  Real q[IB][5];
  int at[IB][3];
#pragma unroll
  for (int b = 0; b < IB; ++b) load(q[b], at[b]);
  for (;;) {
    bool any = false;
#pragma unroll
    for (int b = 0; b < IB; ++b) any |= at[b][2] < L.nz;
    if (!any) break;  // warp-uniform: every lane's cursor has left the grid
    Real qn[IB][5];
    int an[IB][3];
#pragma unroll
    for (int b = 0; b < IB; ++b) load(qn[b], an[b]);
#pragma unroll
    for (int b = 0; b < IB; ++b) {
      if (at[b][0] >= 0) {
        const int i = at[b][0], j = at[b][1], k = at[b][2];
        // float64 throughout; one reciprocal of rho and the inverse-length
        // tables replace the eight divisions (dt moves by ulps, inside 1e-12)
        const double rho = double(q[b][0]);
        const double ir = 1.0 / rho;
        const double v0 = double(q[b][1]) * ir, v1 = double(q[b][2]) * ir, v2 = double(q[b][3]) * ir;
        const double E = double(q[b][4]) * ir;
        const double P = ((gam - 1.0) * rho) * (E - (((v0 * v0) + (v1 * v1)) + (v2 * v2)) / 2.0);
        const double cs = sqrt((gam * P) * ir);
        if (!(rho > 0.0)) bad |= ST_DENSITY;
        if (!(P > 0.0)) bad |= ST_PRESSURE;
        // max(|v|, |v - c|, |v + c|) of the reference's three waves is
        // fl(|v| + c) for c >= 0: |v - c| and |v + c| are |v| -+ c up to sign,
        // and rounding is monotone
        const double ml[3] = {fabs(v0) + cs, fabs(v1) + cs, fabs(v2) + cs};
        const double r = fmax(fmax(ml[0] * inv_len<double, COORD, 0>(m, i, j, k), ml[1] * inv_len<double, COORD, 1>(m, i, j, k)),
                              ml[2] * inv_len<double, COORD, 2>(m, i, j, k));
        const double nl = mu * ir;
        if (!(r >= 0.0) || !(nl >= 0.0)) bad |= ST_NONFINITE;
        rc = fmax(rc, r);
        nu = fmax(nu, nl);
      }
    }
#pragma unroll
    for (int b = 0; b < IB; ++b) {
#pragma unroll
      for (int c = 0; c < 3; ++c) at[b][c] = an[b][c];
#pragma unroll
      for (int v = 0; v < 5; ++v) q[b][v] = qn[b][v];
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    rc = fmax(rc, __shfl_xor_sync(0xffffffffu, rc, o));
    nu = fmax(nu, __shfl_xor_sync(0xffffffffu, nu, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { s_rc[w] = rc; s_nu[w] = nu; }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    rc = l < nw ? s_rc[l] : 0.0;
    nu = l < nw ? s_nu[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      rc = fmax(rc, __shfl_xor_sync(0xffffffffu, rc, o));
      nu = fmax(nu, __shfl_xor_sync(0xffffffffu, nu, o));
    }
    if (l == 0) {
      atomic_max_pos(&clk->red[0], rc);
      atomic_max_pos(&clk->red[1], nu);
    }
  }
  if (bad) atomicOr(status, bad);
}

// One thread: close the step's clock.  mode 0: dt from the reduced NS rates,
// mode 1: fixed dt, mode 2: dt = cfl / const_rate (state-independent heat and
// Maxwell steps).  `max_inv_l2` = max over cells of sum_d 1/L_d^2.
__device__ __forceinline__ void clock_one(Clock* clk, int mode, double max_inv_l2, double const_rate,
                                          unsigned* status) {
  clk->active = clk->t <= clk->t_end ? 1 : 0;
  double dt;
  if (mode == 0) {
    const double rc = __longlong_as_double((long long)clk->red[0]);
    const double nu = __longlong_as_double((long long)clk->red[1]);
    clk->red[0] = 0ull;
    clk->red[1] = 0ull;
    const double rd = (2 * nu) * max_inv_l2;
    dt = clk->cfl / (rc + rd);
  } else if (mode == 1) {
    dt = clk->dt_fixed;
  } else {
    dt = clk->cfl / const_rate;
  }
  if (!clk->active) return;
  if (!(dt > 0.0) || !isfinite(dt)) atomicOr(status, ST_DT);
  clk->dt = dt;
  clk->t = clk->t + dt;
  clk->steps = clk->steps + 1;
}

// The step's clock update (clock_one), when a ghost fill carries it.
struct ClockArgs {
  Clock* clk;  // null: the fill has no clock work
  int mode;
  double max_inv_l2, const_rate;
  unsigned* status;
};

// One grid's ghost faces: blockIdx.y = variable * 6 + side; the face's cells
// (a along the face row, b over rows) are dealt to the blocks of that grid row,
// BCF per thread with every load issued before the stores: an x1 face is
// strided (one sector per cell), so the fill is latency-bound and wants many
// loads in flight.  The first fill of a step also closes the step's clock in
// block (0, 0) (ck.clk set).  The fill does not read the clock: filling the
// ghosts of a state whose step turns out to be a no-op changes nothing a
// later read sees (the ghost faces are a function of the interior, and
// downloads fill them again).  `skip_sides` (bit s) leaves out side s: the
// x3 slabs of a one-plane grid, whose stage kernels never read them.
constexpr int BCF = 4;
template <typename Real>
__global__ void __launch_bounds__(256) bc_fill_kernel(Real* __restrict__ u, Layout L, int nv, BcSpec bc, ClockArgs ck,
                                                      int skip_sides) {
  if (ck.clk && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
    clock_one(ck.clk, ck.mode, ck.max_inv_l2, ck.const_rate, ck.status);
  const int q = blockIdx.y / 6, side = blockIdx.y % 6;
  if (q >= nv || ((skip_sides >> side) & 1)) return;
  const int axis = side >> 1, high = side & 1;
  const int A = axis == 0 ? L.ny : L.nx;  // along a row
  const int B = axis == 2 ? L.ny : L.nz;  // rows
  const int kind = bc.kind[q][side];
  const int n = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  const int g = high ? n + 1 : 0;                       // ghost index along axis
  const int inner = high ? n : 1;                       // adjacent interior
  const int src = kind == 0 ? (high ? 1 : n) : inner;  // periodic: opposite layer
  const Real two_w = Real(2) * Real(bc.value[q][side]);
  const int total = A * B, stride = gridDim.x * blockDim.x;
  for (int t0 = blockIdx.x * blockDim.x + threadIdx.x; t0 < total; t0 += BCF * stride) {
    Real v[BCF];
    long long gi[BCF];
#pragma unroll
    for (int m = 0; m < BCF; ++m) {
      const int t = t0 + m * stride;
      const int a = t % A, b = t / A;
      long long si;
      if (axis == 0) { gi[m] = L.idx(q, b + 1, a + 1, g); si = L.idx(q, b + 1, a + 1, src); }
      else if (axis == 1) { gi[m] = L.idx(q, b + 1, g, a + 1); si = L.idx(q, b + 1, src, a + 1); }
      else { gi[m] = L.idx(q, g, b + 1, a + 1); si = L.idx(q, src, b + 1, a + 1); }
      v[m] = t < total ? u[si] : Real(0);
    }
#pragma unroll
    for (int m = 0; m < BCF; ++m)
      if (t0 + m * stride < total) u[gi[m]] = kind == 2 ? -v[m] : (kind == 3 ? two_w - v[m] : v[m]);
  }
}

// A batch's ghost faces as a static list of chunks: up to BC_CHUNK
// consecutive cells of one face slab (grid, variable, side), one block each,
// so a block needs no search for its grid and no per-cell decode of the slab.
constexpr int BC_CHUNK = 256 * BCF;
struct BcChunk {
  int grid, q, side, start, count;
};

// The ghost faces (bc_fill_kernel's arithmetic) of the chunks' state buffer
// `buf`; grids whose clock passed t_end are skipped.
template <typename Real>
__global__ void __launch_bounds__(256) batch_bc_chunk_kernel(const BatchAux* __restrict__ a,
                                                             const BcChunk* __restrict__ ch, int buf) {
  const BcChunk c = ch[blockIdx.x];
  const BatchAux& x = a[c.grid];
  if (!x.clk->active) return;
  Real* __restrict__ u = static_cast<Real*>(x.U[buf]);
  const Layout& L = x.lay;
  const int q = c.q, side = c.side, axis = side >> 1, high = side & 1;
  const int A = axis == 0 ? L.ny : L.nx;  // along a row
  const int kind = x.bc.kind[q][side];
  const int n = axis == 0 ? L.nx : (axis == 1 ? L.ny : L.nz);
  const int g = high ? n + 1 : 0;                       // ghost index along axis
  const int inner = high ? n : 1;                       // adjacent interior
  const int src = kind == 0 ? (high ? 1 : n) : inner;  // periodic: opposite layer
  const Real two_w = Real(2) * Real(x.bc.value[q][side]);
  Real v[BCF];
  long long gi[BCF];
#pragma unroll
  for (int m = 0; m < BCF; ++m) {
    const int k = threadIdx.x + m * 256;
    const int t = c.start + k;
    const int a0 = t % A, b0 = t / A;
    long long si;
    if (axis == 0) { gi[m] = L.idx(q, b0 + 1, a0 + 1, g); si = L.idx(q, b0 + 1, a0 + 1, src); }
    else if (axis == 1) { gi[m] = L.idx(q, b0 + 1, g, a0 + 1); si = L.idx(q, b0 + 1, src, a0 + 1); }
    else { gi[m] = L.idx(q, g, b0 + 1, a0 + 1); si = L.idx(q, src, b0 + 1, a0 + 1); }
    v[m] = k < c.count ? u[si] : Real(0);
  }
#pragma unroll
  for (int m = 0; m < BCF; ++m)
    if (threadIdx.x + m * 256 < c.count) u[gi[m]] = kind == 2 ? -v[m] : (kind == 3 ? two_w - v[m] : v[m]);
}

__global__ void batch_clock_kernel(const BatchAux* __restrict__ a, int n, int fixed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) clock_one(a[i].clk, fixed ? 1 : a[i].cmode, a[i].max_inv_l2, a[i].const_rate, a[i].status);
}

// Conserved totals with Neumaier compensation: per-thread, then per-block
// (fixed order), then a single-thread pass over the block partials.
__device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
  const double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x;
  else c += (x - t) + s;
  s = t;
}

template <typename Real, int COORD>
__global__ void totals_kernel(const Real* __restrict__ u, Layout L, Metric<double> m, int nv, int nt,
                              double em_mu, double em_ep, double* __restrict__ partials) {
  // nt totals: the nv conserved sums, plus (Maxwell) EM energy when nt == nv + 1
  __shared__ double ss[256][8];
  double s[8], c[8];
  for (int q = 0; q < 8; ++q) { s[q] = 0.0; c[q] = 0.0; }
  const long long n = (long long)L.nx * L.ny * L.nz;
  for (long long cell = blockIdx.x * (long long)blockDim.x + threadIdx.x; cell < n;
       cell += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(cell % L.nx), j = (int)((cell / L.nx) % L.ny), k = (int)(cell / ((long long)L.nx * L.ny));
    const double V = Geo<double, COORD>::V(m, i, j, k);
    const long long g = L.idx(0, k + 1, j + 1, i + 1);
    double em = 0.0;
    for (int q = 0; q < nv; ++q) {
      const double x = double(u[g + q * L.var_stride]);
      neumaier_add(s[q], c[q], x * V);
      if (nt > nv) em += q < 3 ? (x * x) / em_mu : (x * x) / em_ep;
    }
    if (nt > nv) neumaier_add(s[nv], c[nv], 0.5 * em * V);
  }
  for (int q = 0; q < nt; ++q) ss[threadIdx.x][q] = s[q] + c[q];
  __syncthreads();
  if (threadIdx.x < nt) {
    double bs = 0.0, bc = 0.0;
    for (int t = 0; t < (int)blockDim.x; ++t) neumaier_add(bs, bc, ss[t][threadIdx.x]);
    partials[blockIdx.x * 8 + threadIdx.x] = bs + bc;
  }
}

__global__ void totals_final_kernel(const double* __restrict__ partials, int nblocks, int nt, double* out) {
  if (threadIdx.x >= nt) return;
  double s = 0.0, c = 0.0;
  for (int b = 0; b < nblocks; ++b) neumaier_add(s, c, partials[b * 8 + threadIdx.x]);
  out[threadIdx.x] = s + c;
}

// ------------------------------------------------------ device initial state ----
// Uniform value in [-1, 1) from a splitmix64 hash of (seed, stream, index).
__device__ __forceinline__ double hash_unit(unsigned long long seed, unsigned long long stream, long long i) {
  unsigned long long z = seed * 0x9E3779B97F4A7C15ull + (stream + 1) * 0xD1B54A32D192ED03ull + (unsigned long long)i;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

struct KhInit {
  double rho_in, rho_out, shear, pres, amp, wavenumber, noise, phase, gamma;
  double x1_min, dx1, x2_min, dx2;
  int noise_all;
  unsigned long long seed;
};

// Sharp Kelvin-Helmholtz state (float64 arithmetic, stored in Real) on the
// interior of buffer u.
template <typename Real>
__global__ void kh_init_kernel(Real* u, Layout L, KhInit k) {
  const long long n = (long long)L.nx * L.ny * L.nz;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % L.nx), j = (int)((p / L.nx) % L.ny), kk = (int)(p / ((long long)L.nx * L.ny));
    const double x = k.x1_min + (i + 0.5) * k.dx1, y = k.x2_min + (j + 0.5) * k.dx2;
    const bool inner = fabs(y - 0.5) < 0.25;
    const double rho = inner ? k.rho_in : k.rho_out;
    double v1 = inner ? k.shear : -k.shear;
    double v2 = k.amp * sin(2.0 * 3.141592653589793 * k.wavenumber * x + k.phase) + k.noise * hash_unit(k.seed, 1, p);
    double v3 = 0.0;
    if (k.noise_all) {
      v1 += k.noise * hash_unit(k.seed, 0, p);
      v3 += k.noise * hash_unit(k.seed, 2, p);
    }
    const double e = k.pres / (k.gamma - 1.0) + 0.5 * rho * (v1 * v1 + v2 * v2 + v3 * v3);
    u[L.idx(0, kk + 1, j + 1, i + 1)] = (Real)rho;
    u[L.idx(1, kk + 1, j + 1, i + 1)] = (Real)(rho * v1);
    u[L.idx(2, kk + 1, j + 1, i + 1)] = (Real)(rho * v2);
    u[L.idx(3, kk + 1, j + 1, i + 1)] = (Real)(rho * v3);
    u[L.idx(4, kk + 1, j + 1, i + 1)] = (Real)e;
  }
}

}  // namespace fvm
