// Shared device code for the fused finite-volume stage kernels (sm_100a).
//
// Device layout of a state buffer (one allocation per state, structure of
// arrays): element (var q, ghosted plane gz, ghosted row gy, ghosted column gx)
// lives at  q*var_stride + gz*plane + gy*pitch + (gx + padx).  One ghost layer
// per side, as in the reference (navier_stokes.py:33-39).  `padx` is chosen so
// that the first interior column (gx = 1) starts on a 16-byte boundary, which
// lets a TMA box start at an aligned x coordinate and lets warps store whole
// aligned 128-byte rows.
#pragma once
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace fvm {

// ---------------------------------------------------------------- enums ----
enum Coord : int { COORD_CART = 0, COORD_CYL = 1, COORD_SPH = 2 };
enum Limiter : int { LIM_PC = 0, LIM_MINMOD = 1, LIM_MC = 2, LIM_VANLEER = 3 };
enum Riemann : int { RIEM_RUSANOV = 0, RIEM_HLL = 1 };
// Stage epilogue modes (time_integrators.py:42-221 stage combinations).
enum StageMode : int {
  MODE_RHS = 0,    // out = k (single residual, for parity checks)
  MODE_EULER = 1,  // out = Ucur + dt*k
  MODE_AXPY = 2,   // out = U0 + (ca*dt)*k
  MODE_SSP = 3,    // out = ca*U0 + cb*(Ucur + dt*k)
  MODE_FINAL = 4   // out = U0 + (dt/6)*(acc + k)
};
enum AccMode : int { ACC_NONE = 0, ACC_SET = 1, ACC_ADD = 2 };  // acc = k | acc = acc + w*k

// Status bits written by kernels (never a trap).
enum Status : unsigned {
  ST_NONFINITE = 1u, ST_DENSITY = 2u, ST_PRESSURE = 4u, ST_DT = 8u, ST_TMA_TIMEOUT = 16u
};

// ------------------------------------------------------- grid metadata ----
// Per-axis 1D metric tables, built on the host with the reference's own
// expressions (geometry.py:37-171) in float64 and cast once to Real.
template <typename Real>
struct Metric {
  const Real* dx1;    // nx1: face differences along x1
  const Real* dx2;    // nx2
  const Real* dx3;    // nx3
  const Real* r_c;    // nx1: x1 cell centres
  const Real* r_f;    // nx1+1: x1 faces
  const Real* r_f2;   // nx1+1: x1 faces squared
  const Real* a1;     // nx1: (rf+^2 - rf-^2)/2
  const Real* b1;     // nx1: (rf+^3 - rf-^3)/3
  const Real* inv_r;  // nx1: 1/x1
  const Real* two_inv_r;  // nx1: 2/x1
  const Real* c2;     // nx2: cos(th-) - cos(th+)
  const Real* sin_f2; // nx2+1: sin(theta faces)
  const Real* sin_c2; // nx2: sin(theta centres)
  const Real* cot_c2; // nx2: 1/tan(theta centres)
  const Real* inv_dx1;   // nx1: 1/dx1  (float32 fast path)
  const Real* inv_dx2;   // nx2
  const Real* inv_dx3;   // nx3
  const Real* inv_sin_c2;  // nx2: 1/sin(theta centres)
};

struct Layout {
  int nx, ny, nz;         // interior cells
  long long pitch;        // elements per x row (>= nx+2+padx)
  long long plane;        // pitch*(ny+2)
  long long var_stride;   // >= plane*(nz+2)
  int padx;               // front pad so that gx=1 is 16-byte aligned
  __host__ __device__ long long idx(int q, int gz, int gy, int gx) const {
    return (long long)q * var_stride + (long long)gz * plane + (long long)gy * pitch + gx + padx;
  }
};

// Cell metrics (interior cell i,j,k, 0-based).  Products keep the reference's
// left-to-right order so that the float64 build reproduces NumPy bitwise.
template <typename Real, int COORD>
struct Geo {
  static __device__ __forceinline__ Real L1(const Metric<Real>& m, int i, int, int) { return __ldg(m.dx1 + i); }
  static __device__ __forceinline__ Real L2(const Metric<Real>& m, int i, int j, int) {
    if constexpr (COORD == COORD_CART) return __ldg(m.dx2 + j);
    else return __ldg(m.r_c + i) * __ldg(m.dx2 + j);
  }
  static __device__ __forceinline__ Real L3(const Metric<Real>& m, int i, int j, int k) {
    if constexpr (COORD == COORD_SPH) return (__ldg(m.r_c + i) * __ldg(m.sin_c2 + j)) * __ldg(m.dx3 + k);
    else return __ldg(m.dx3 + k);
  }
  template <int D>
  static __device__ __forceinline__ Real L(const Metric<Real>& m, int i, int j, int k) {
    if constexpr (D == 0) return L1(m, i, j, k);
    else if constexpr (D == 1) return L2(m, i, j, k);
    else return L3(m, i, j, k);
  }
  static __device__ __forceinline__ Real V(const Metric<Real>& m, int i, int j, int k) {
    if constexpr (COORD == COORD_CART) return (__ldg(m.dx1 + i) * __ldg(m.dx2 + j)) * __ldg(m.dx3 + k);
    else if constexpr (COORD == COORD_CYL) return (__ldg(m.a1 + i) * __ldg(m.dx2 + j)) * __ldg(m.dx3 + k);
    else return (__ldg(m.b1 + i) * __ldg(m.c2 + j)) * __ldg(m.dx3 + k);
  }
  // Face areas: S1 at x1-face index fi (0..nx1), S2 at x2-face fj, S3 any k.
  static __device__ __forceinline__ Real S1(const Metric<Real>& m, int fi, int j, int k) {
    if constexpr (COORD == COORD_CART) return __ldg(m.dx2 + j) * __ldg(m.dx3 + k);
    else if constexpr (COORD == COORD_CYL) return (__ldg(m.r_f + fi) * __ldg(m.dx2 + j)) * __ldg(m.dx3 + k);
    else return (__ldg(m.r_f2 + fi) * __ldg(m.c2 + j)) * __ldg(m.dx3 + k);
  }
  static __device__ __forceinline__ Real S2(const Metric<Real>& m, int i, int fj, int k) {
    if constexpr (COORD == COORD_SPH) return (__ldg(m.a1 + i) * __ldg(m.sin_f2 + fj)) * __ldg(m.dx3 + k);
    else return __ldg(m.dx1 + i) * __ldg(m.dx3 + k);
  }
  static __device__ __forceinline__ Real S3(const Metric<Real>& m, int i, int j) {
    if constexpr (COORD == COORD_CART) return __ldg(m.dx1 + i) * __ldg(m.dx2 + j);
    else return __ldg(m.a1 + i) * __ldg(m.dx2 + j);
  }
};

// 1/L_D at a cell, from the inverse tables (float32 fast path only).
template <typename Real, int COORD, int D>
__device__ __forceinline__ Real inv_len(const Metric<Real>& m, int i, int j, int k) {
  if constexpr (D == 0) return __ldg(m.inv_dx1 + i);
  else if constexpr (D == 1) {
    if constexpr (COORD == COORD_CART) return __ldg(m.inv_dx2 + j);
    else return __ldg(m.inv_r + i) * __ldg(m.inv_dx2 + j);
  } else {
    if constexpr (COORD == COORD_SPH) return (__ldg(m.inv_r + i) * __ldg(m.inv_sin_c2 + j)) * __ldg(m.inv_dx3 + k);
    else return __ldg(m.inv_dx3 + k);
  }
}

// Lame data at a cell: h[3], dl[a][b] = d_a ln h_b, d123[a] = d_a ln(h1h2h3).
template <typename Real>
struct Lame {
  Real h[3];
  Real dl[3][3];
  Real d123[3];
};
template <typename Real, int COORD>
__device__ __forceinline__ void lame_at(const Metric<Real>& m, int i, int j, Lame<Real>& L) {
  for (int a = 0; a < 3; ++a) {
    L.h[a] = Real(1);
    L.d123[a] = Real(0);
    for (int b = 0; b < 3; ++b) L.dl[a][b] = Real(0);
  }
  if constexpr (COORD == COORD_CYL) {
    Real r = __ldg(m.r_c + i), ir = __ldg(m.inv_r + i);
    L.h[1] = r;
    L.dl[0][1] = ir;
    L.d123[0] = ir;
  } else if constexpr (COORD == COORD_SPH) {
    Real r = __ldg(m.r_c + i), ir = __ldg(m.inv_r + i), cot = __ldg(m.cot_c2 + j);
    L.h[1] = r;
    L.h[2] = r * __ldg(m.sin_c2 + j);
    L.dl[0][1] = ir;
    L.dl[0][2] = ir;
    L.dl[1][2] = cot;
    L.d123[0] = __ldg(m.two_inv_r + i);
    L.d123[1] = cot;
  }
}

// ------------------------------------------------------------ limiters ----
template <typename R>
__device__ __forceinline__ R sgn(R x) { return x > R(0) ? R(1) : (x < R(0) ? R(-1) : R(0)); }

// slope_limiters.py:13-39
template <typename R>
__device__ __forceinline__ R lim_minmod(R a, R b) {
  R ss = (sgn(a) + sgn(b)) / R(2);
  return ss * fmin(fabs(a), fabs(b));
}
// slope_limiters.py:42-73 (three-sign test divided by 3, nonzero for opposite signs)
template <typename R>
__device__ __forceinline__ R lim_mc(R a, R b) {
  R c = R(0.5) * (a + b);
  R a2 = R(2) * a, b2 = R(2) * b;
  R ss = ((sgn(c) + sgn(a2)) + sgn(b2)) / R(3);
  return ss * fmin(fabs(c), fmin(fabs(a2), fabs(b2)));
}
// slope_limiters.py:76-105
template <typename R>
__device__ __forceinline__ R lim_vanleer(R a, R b) {
  R ss = (sgn(a) + sgn(b)) / R(2);
  R den = fabs(a) + fabs(b);
  R hm = den > R(0) ? ((R(2) * a) * b) / den : R(0);
  return ss * hm;
}
template <int LIM, typename R>
__device__ __forceinline__ R limiter(R a, R b) {
  if constexpr (LIM == LIM_MINMOD) return lim_minmod(a, b);
  else if constexpr (LIM == LIM_MC) return lim_mc(a, b);
  else return lim_vanleer(a, b);
}
// ------------------------------------------- float32 fast arithmetic ----
// The float32 build trades IEEE division/sqrt for the approximate SFU
// instructions (<= 2 ulp); the float64 build keeps the reference's exact
// operation sequence.
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
template <typename R>
__device__ __forceinline__ R recip(R x) {
  if constexpr (sizeof(R) == 4) return rcp_approx(x);
  else return R(1) / x;
}
// Limiters are positively homogeneous of degree one, so limiter(a/L, b/L)*L
// equals limiter(a, b); the float32 path evaluates that form directly.
__device__ __forceinline__ float flim_minmod(float a, float b) {
  return a * b > 0.f ? copysignf(fminf(fabsf(a), fabsf(b)), a) : 0.f;
}
__device__ __forceinline__ float flim_vanleer(float a, float b) {
  const float ab = a * b;
  return ab > 0.f ? 2.f * ab * rcp_approx(a + b) : 0.f;
}
__device__ __forceinline__ float flim_mc(float a, float b) {
  const float c = 0.5f * (a + b);
  const float ss = (sgn(c) + sgn(a) + sgn(b)) * (1.f / 3.f);
  return ss * fminf(fabsf(c), 2.f * fminf(fabsf(a), fabsf(b)));
}

// MUSCL slope of a cell (reconstructors.py:120-132): limiter(bwd/L, fwd/L)*L.
template <int LIM, typename R>
__device__ __forceinline__ R muscl_slope(R fm, R f0, R fp, R L) {
  if constexpr (LIM == LIM_PC) return R(0);
  else if constexpr (sizeof(R) == 4) {
    const float a = f0 - fm, b = fp - f0;
    if constexpr (LIM == LIM_MINMOD) return flim_minmod(a, b);
    else if constexpr (LIM == LIM_MC) return flim_mc(a, b);
    else return flim_vanleer(a, b);
  } else {
    return limiter<LIM>((f0 - fm) / L, (fp - f0) / L) * L;
  }
}

// Device-resident time-loop scalars.
struct Clock {
  double t, t_end, dt, cfl, dt_fixed;
  long long steps;
  int active;
  unsigned long long red[2];  // running maxima (bit patterns of non-negative doubles)
};

// --------------------------------------------------------- PTX helpers ----
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on an mbarrier phase: gives up after `limit_ns` and reports it.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_ns() - t0 > limit_ns) return false;
  }
  return true;
}
// TMA: 4D tiled load (x, y, z, var) into shared memory, completion on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1,
                                            int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// ------------------------------------------------------- stage epilogue ----
struct StageCoef {
  int mode, accmode;
  double ca, cb, wacc;  // mode constants (see StageMode), acc weight
  int u0_is_input;      // the stage input buffer is the step base U0 (first stage)
};

// Ask L2 for the 128-byte line holding p (the epilogue's U0/acc rows), so the
// dependent loads at the end of a z-march step hit L2 instead of DRAM.
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
// One 4-byte asynchronous copy global -> shared (completion: cp_async_wait_all
// by the issuing thread, after which the thread may read the destination).
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Combine one variable.  `k` is the residual, `ucur` the stage input, `u0`
// the step's base state, `acc` the running k-sum.  Op order follows
// time_integrators.py:47,91-103,147-159,203-221.
template <typename R>
__device__ __forceinline__ R stage_combine(const StageCoef& c, R dt, R k, R ucur, R u0, R acc) {
  switch (c.mode) {
    case MODE_RHS: return k;
    case MODE_EULER: return ucur + dt * k;
    case MODE_AXPY: return u0 + (R(c.ca) * dt) * k;
    case MODE_SSP:
      // float32: U0 + cb((Ucur - U0) + dt k), equal to ca U0 + cb (Ucur + dt k)
      // because ca + cb = 1, and exact when nothing changes (the float32
      // coefficients 1/3, 2/3 do not sum to one and would bias the totals)
      if constexpr (sizeof(R) == 4) return u0 + R(c.cb) * ((ucur - u0) + dt * k);
      else return R(c.ca) * u0 + R(c.cb) * (ucur + dt * k);
    default:
      // float32 keeps acc = U0 + (dt/6) sum_s w_s k_s (low storage: the last
      // stage reads only its input and acc); float64 keeps the k-sum and the
      // reference's summation order U0 + (dt/6)(k1 + w k2 + ... + k_last)
      if constexpr (sizeof(R) == 4) return acc + (dt / R(6)) * k;
      else return u0 + (dt / R(6)) * (acc + k);
  }
}

// The stage epilogue needs U0 from memory (not from the input ring)?
template <typename R>
__device__ __forceinline__ bool needs_u0(const StageCoef& c) {
  if (c.mode < MODE_AXPY) return false;
  if constexpr (sizeof(R) == 4) {
    if (c.mode == MODE_FINAL) return false;
  }
  return true;
}
__device__ __forceinline__ bool needs_acc(const StageCoef& c) {
  return c.mode == MODE_FINAL || c.accmode == ACC_ADD;
}
// New accumulator value after this stage (see stage_combine).
template <typename R>
__device__ __forceinline__ R acc_update(const StageCoef& c, R dt, R k, R u0, R acc) {
  if constexpr (sizeof(R) == 4) {
    if (c.accmode == ACC_SET) return u0 + (dt / R(6)) * k;
    return acc + ((R(c.wacc) * dt) / R(6)) * k;
  } else {
    if (c.accmode == ACC_SET) return k;
    return acc + R(c.wacc) * k;
  }
}

}  // namespace fvm
