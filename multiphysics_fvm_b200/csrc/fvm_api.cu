// C ABI of libfvm_b200 (declared in include/fvm.h): handle life cycle, layout
// transforms, the device-resident time loop (CUDA graphs), CFL reduction and
// conserved totals.  The stencil work is in the fused stage kernels.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <algorithm>
#include <vector>

#include "../../include/fvm.h"
#include "../../include/fvm_closure.h"
#include "closure_host.h"
#include "fvm_aux.cuh"
#include "launch.cuh"

using namespace fvm;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

#define FVM_CK(x)                                                                                \
  do {                                                                                           \
    cudaError_t e_ = (x);                                                                        \
    if (e_ != cudaSuccess) return fail(FVM_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace

int fvm::set_error(int code, const std::string& msg) { return fail(code, msg); }

namespace {

// Host copy of the per-axis metric tables (float64), built with the
// reference's expressions (src/grid/geometry.py:37-171).
struct HostMetric {
  std::vector<double> dx1, dx2, dx3, r_c, r_f, r_f2, a1, b1, inv_r, two_inv_r, c2, sin_f2, sin_c2, cot_c2;
  std::vector<double> inv_dx1, inv_dx2, inv_dx3, inv_sin_c2;
};

HostMetric build_metric(const fvm_desc& d) {
  HostMetric m;
  const int n[3] = {d.nx1, d.nx2, d.nx3};
  const double lo[3] = {d.x1_min, d.x2_min, d.x3_min}, hi[3] = {d.x1_max, d.x2_max, d.x3_max};
  std::vector<double> xc[3], xf[3], dl[3];
  for (int a = 0; a < 3; ++a) {
    const double dd = (hi[a] - lo[a]) / n[a];
    for (int i = 0; i < n[a]; ++i) xc[a].push_back(lo[a] + ((double)i + 0.5) * dd);
    for (int i = 0; i <= n[a]; ++i) xf[a].push_back(lo[a] + (double)i * dd);
    for (int i = 0; i < n[a]; ++i) dl[a].push_back(xf[a][i + 1] - xf[a][i]);
  }
  m.dx1 = dl[0]; m.dx2 = dl[1]; m.dx3 = dl[2];
  m.r_c = xc[0]; m.r_f = xf[0];
  for (int i = 0; i <= n[0]; ++i) m.r_f2.push_back(xf[0][i] * xf[0][i]);
  for (int i = 0; i < n[0]; ++i) {
    const double p = xf[0][i + 1], q = xf[0][i];
    m.a1.push_back((p * p - q * q) / 2.0);
    m.b1.push_back((std::pow(p, 3.0) - std::pow(q, 3.0)) / 3.0);
    m.inv_r.push_back(1.0 / xc[0][i]);
    m.two_inv_r.push_back(2.0 / xc[0][i]);
  }
  for (int j = 0; j < n[1]; ++j) {
    m.c2.push_back(std::cos(xf[1][j]) - std::cos(xf[1][j + 1]));
    m.sin_c2.push_back(std::sin(xc[1][j]));
    m.cot_c2.push_back(1.0 / std::tan(xc[1][j]));
  }
  for (int j = 0; j <= n[1]; ++j) m.sin_f2.push_back(std::sin(xf[1][j]));
  for (double v : m.dx1) m.inv_dx1.push_back(1.0 / v);
  for (double v : m.dx2) m.inv_dx2.push_back(1.0 / v);
  for (double v : m.dx3) m.inv_dx3.push_back(1.0 / v);
  for (double v : m.sin_c2) m.inv_sin_c2.push_back(1.0 / v);
  return m;
}

// Cell lengths on the host, same products as Geo<> (geometry.py:80-171).
void host_lengths(const HostMetric& m, int coords, int i, int j, int k, double L[3]) {
  L[0] = m.dx1[i];
  L[1] = coords == FVM_CARTESIAN ? m.dx2[j] : m.r_c[i] * m.dx2[j];
  L[2] = coords == FVM_SPHERICAL ? (m.r_c[i] * m.sin_c2[j]) * m.dx3[k] : m.dx3[k];
}

}  // namespace

struct fvm_handle {
  fvm_desc d{};
  int nv = 0;
  bool f64 = false;
  size_t esz = 4;
  Layout lay{};
  int nsm = 148;
  cudaStream_t stream = nullptr;
  void* U[3] = {nullptr, nullptr, nullptr};  // base, stage a, stage b
  void* acc = nullptr;
  void* met_real = nullptr;     // metric tables in the state precision
  double* met_f64 = nullptr;    // metric tables in float64 (reductions)
  Metric<float> mf{};
  Metric<double> md{};
  Clock* clk = nullptr;
  unsigned* status = nullptr;
  double* partials = nullptr;
  double* totals_dev = nullptr;
  double* stage_dev = nullptr;   // reference-layout float64 staging on the device
  double* stage_host = nullptr;  // pinned staging
  size_t stage_elems = 0;
  // pipelined host transfers (fvm_upload_async / fvm_download_async): a second
  // device staging buffer for downloads, one stream per copy direction and the
  // events that order them against the handle's stream
  double* stage_out = nullptr;
  cudaStream_t s_in = nullptr, s_out = nullptr;
  cudaEvent_t ev_in_ready = nullptr, ev_in_free = nullptr, ev_out_ready = nullptr, ev_out_free = nullptr;
  CUtensorMap tmap[3];
  CUtensorMap smap{}, amap{};  // staged U0 / accumulator tiles of the float32 cartesian NS kernel
  bool legacy = false;         // batch member: runs the batched (tile-list) kernels
  unsigned long long wait_ns = 2000000000ull;  // limit of each wait for a TMA plane
  unsigned long long drain_ns = 1000000000ull; // limit of the wait for copies in flight after a timeout
  unsigned extra_tx = 0;                       // test of the timeout path (fvm_set_wait_limit)
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  double max_inv_l2 = 0.0, const_rate = 0.0;
  int zchunk = 64;
  int tile_ty = 0;  // tile rows of the stage kernel (its tensor maps are built for it)
  long long device_bytes = 0;
  fvm_closure* closure = nullptr;  // learned flux correction run inside every step
  double closure_beta = 0.5;
  unsigned long long* closure_nswitch = nullptr;
};

namespace {

int default_tile_ty(const fvm_desc& d);
int alt_tile_ty(const fvm_desc& d);
int tile_halo(const fvm_desc& d);

// float32 cartesian Navier-Stokes grids run the register-blocked stage
// kernels (stage_ns_strip.cuh, stage_ns_strip_visc.cuh) and float32
// piecewise-constant heat grids stage_heat_pc.cuh; batch members keep the
// tile-list kernels.
bool strip_desc(const fvm_desc& d) {
  return d.precision == FVM_FP32 && d.physics == FVM_NAVIER_STOKES && d.coords == FVM_CARTESIAN;
}
// viscous grids run it when the handle's block shape is the strip kernel's
// (their default); the autotuner's second viscous shape is the general kernel's
bool strip_kernel(const fvm_handle* h) {
  return !h->legacy && strip_desc(h->d) && (h->d.params[1] == 0.0 || h->tile_ty == NS_STRIP_VISC_TY);
}
bool heat_pc_desc(const fvm_desc& d) {
  return d.precision == FVM_FP32 && d.physics == FVM_HEAT && d.reconstructor == FVM_PIECEWISE_CONSTANT;
}
bool heat_pc_kernel(const fvm_handle* h) { return !h->legacy && heat_pc_desc(h->d); }
bool mx_strip_desc(const fvm_desc& d) { return d.precision == FVM_FP32 && d.physics == FVM_MAXWELL; }
// kernels whose stage combination reads TMA-staged U0 / accumulator tiles
bool staged_kernel(const fvm_handle* h) { return strip_kernel(h) || mx_strip_desc(h->d); }

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 4D map (x, y, z, var) over one ghosted state buffer.  Box: 40 columns
// starting 3 cells left of the tile (x coordinate aligned), `rows` rows, one
// plane, all variables.
int make_tmap(fvm_handle* h, int b, int rows) {
  auto enc = get_encode();
  if (!enc) return fail(FVM_E_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const Layout& L = h->lay;
  cuuint64_t dims[4] = {(cuuint64_t)(L.nx + 2 + L.padx), (cuuint64_t)(L.ny + 2), (cuuint64_t)(L.nz + 2),
                        (cuuint64_t)h->nv};
  cuuint64_t strides[3] = {(cuuint64_t)(L.pitch * h->esz), (cuuint64_t)(L.plane * h->esz),
                           (cuuint64_t)(L.var_stride * h->esz)};
  cuuint32_t box[4] = {40, (cuuint32_t)rows, 1, (cuuint32_t)h->nv};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(&h->tmap[b], h->f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                   h->U[b], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(FVM_E_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return FVM_OK;
}

// 4D map of a staged tile (U0 or the k accumulator): 32 columns starting at
// the tile's first interior column (16-byte aligned), `rows` rows, one plane,
// all variables.
int make_stage_tmap(fvm_handle* h, CUtensorMap* m, void* base, int rows) {
  auto enc = get_encode();
  if (!enc) return fail(FVM_E_CUDA, "cuTensorMapEncodeTiled is unavailable");
  const Layout& L = h->lay;
  cuuint64_t dims[4] = {(cuuint64_t)(L.nx + 2 + L.padx), (cuuint64_t)(L.ny + 2), (cuuint64_t)(L.nz + 2),
                        (cuuint64_t)h->nv};
  cuuint64_t strides[3] = {(cuuint64_t)(L.pitch * h->esz), (cuuint64_t)(L.plane * h->esz),
                           (cuuint64_t)(L.var_stride * h->esz)};
  cuuint32_t box[4] = {32, (cuuint32_t)rows, 1, (cuuint32_t)h->nv};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(FVM_E_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return FVM_OK;
}

// Tensor maps of the three state buffers for the handle's tile rows (and the
// staged-tile maps of the float32 cartesian NS kernel).
int make_tmaps(fvm_handle* h) {
  const int rows = h->tile_ty + 2 * tile_halo(h->d);
  for (int b = 0; b < 3; ++b)
    if (int rc = make_tmap(h, b, rows)) return rc;
  if (staged_kernel(h)) {
    if (int rc = make_stage_tmap(h, &h->smap, h->U[0], h->tile_ty)) return rc;
    if (h->acc)
      if (int rc = make_stage_tmap(h, &h->amap, h->acc, h->tile_ty)) return rc;
  }
  return FVM_OK;
}

int validate(const fvm_desc* d) {
  if (!d) return fail(FVM_E_INVALID, "null desc");
  if (d->physics < FVM_NAVIER_STOKES || d->physics > FVM_MAXWELL)
    return fail(FVM_E_INVALID, "Unknown physics " + std::to_string(d->physics));
  if (d->precision != FVM_FP32 && d->precision != FVM_FP64) return fail(FVM_E_INVALID, "unknown precision");
  if (d->coords < 0 || d->coords > 2)
    return fail(FVM_E_INVALID, "Unknown coordinate system. Expected one of: cartesian, cylindrical, spherical.");
  if (d->nx1 < 1 || d->nx2 < 1 || d->nx3 < 1) return fail(FVM_E_INVALID, "grid sizes must be >= 1");
  if ((long long)d->nx1 * d->nx2 * d->nx3 > (1ll << 31)) return fail(FVM_E_INVALID, "grid too large");
  if (d->reconstructor < 0 || d->reconstructor > 1) return fail(FVM_E_INVALID, "unknown reconstructor");
  if (d->limiter < 0 || d->limiter > 2) return fail(FVM_E_INVALID, "unknown slope limiter");
  if (d->riemann < 0 || d->riemann > 1) return fail(FVM_E_INVALID, "unknown riemann solver");
  if (d->integrator < 0 || d->integrator > 3) return fail(FVM_E_INVALID, "unknown time integrator");
  if (d->tile_ty != 0 && d->tile_ty != default_tile_ty(*d) && d->tile_ty != alt_tile_ty(*d))
    return fail(FVM_E_INVALID, "tile_ty must be 0 (default), " + std::to_string(default_tile_ty(*d)) + " or " +
                                   std::to_string(alt_tile_ty(*d)) + " for this physics and precision");
  const int nv = d->physics == FVM_NAVIER_STOKES ? 5 : (d->physics == FVM_HEAT ? 1 : 6);
  for (int q = 0; q < nv; ++q)
    for (int s = 0; s < 6; ++s) {
      if (d->bc_kind[q][s] < 0 || d->bc_kind[q][s] > 3) return fail(FVM_E_INVALID, "Unknown boundary condition");
      const bool p0 = d->bc_kind[q][s & ~1] == FVM_BC_PERIODIC, p1 = d->bc_kind[q][s | 1] == FVM_BC_PERIODIC;
      if (p0 != p1) return fail(FVM_E_INVALID, "periodic boundaries must be set on both sides of an axis");
    }
  return FVM_OK;
}

int kernel_limiter(const fvm_desc& d) {
  if (d.reconstructor == FVM_PIECEWISE_CONSTANT) return LIM_PC;
  return d.limiter == FVM_MINMOD ? LIM_MINMOD : (d.limiter == FVM_MONOTONIZED_CENTRAL ? LIM_MC : LIM_VANLEER);
}

// Tile rows: the default block shape of the physics/precision, and the second
// one the float32 NS and heat kernels are also built with (equal if none).
int default_tile_ty(const fvm_desc& d) {
  const bool f64 = d.precision == FVM_FP64, visc = d.physics == FVM_NAVIER_STOKES && d.params[1] != 0.0;
  if (strip_desc(d)) return visc ? NS_STRIP_VISC_TY : NS_STRIP_TY;
  if (heat_pc_desc(d)) return HEAT_PC_TY;
  if (d.physics == FVM_HEAT) return HEAT_TY;
  if (d.physics == FVM_MAXWELL) return f64 ? maxwell_tile_ty<double>() : MX_STRIP_TY;
  if (f64) return visc ? ns_tile_ty<double, true>() : ns_tile_ty<double, false>();
  return visc ? ns_tile_ty<float, true>() : ns_tile_ty<float, false>();
}
int alt_tile_ty(const fvm_desc& d) {
  if (mx_strip_desc(d)) return MX_STRIP_TY_ALT;
  if (d.precision == FVM_FP64 || d.physics == FVM_MAXWELL) return default_tile_ty(d);
  if (heat_pc_desc(d)) return HEAT_PC_TY_ALT;
  if (d.physics == FVM_HEAT) return HEAT_TY_ALT;
  if (strip_desc(d)) return d.params[1] != 0.0 ? ns_tile_ty<float, true>() : NS_STRIP_TY_ALT;
  return d.params[1] != 0.0 ? ns_tile_ty_alt<float, true>() : ns_tile_ty_alt<float, false>();
}
// Halo rows staged on each side of a tile (TMA box height = rows + 2*halo).
int tile_halo(const fvm_desc& d) {
  if (d.physics == FVM_HEAT) return d.reconstructor == FVM_PIECEWISE_CONSTANT ? 2 : 3;
  if (d.physics == FVM_MAXWELL) return 2;
  return d.params[1] != 0.0 ? 3 : 2;
}

BcSpec make_bc(const fvm_desc& d, int nv) {
  BcSpec b{};
  for (int q = 0; q < 6; ++q)
    for (int s = 0; s < 6; ++s) {
      b.kind[q][s] = (signed char)(q < nv ? d.bc_kind[q][s] : 0);
      b.value[q][s] = d.bc_value[q][s];
    }
  return b;
}

// Stage table of each integrator (time_integrators.py:10-221): input buffer,
// output buffer, epilogue mode, constants and accumulator update.
struct StageDef {
  int in, out, mode, accmode;
  double ca, cb, w;
};
std::vector<StageDef> stage_table(int integrator) {
  switch (integrator) {
    case FVM_EULER_EXPLICIT: return {{0, 1, MODE_EULER, ACC_NONE, 0, 0, 0}};
    case FVM_RK3:
      return {{0, 1, MODE_AXPY, ACC_SET, 0.5, 0, 0},
              {1, 2, MODE_AXPY, ACC_ADD, 1.0, 0, 4.0},
              {2, 0, MODE_FINAL, ACC_NONE, 0, 0, 0}};
    case FVM_RK3_SSP:
      return {{0, 1, MODE_AXPY, ACC_NONE, 1.0, 0, 0},
              {1, 2, MODE_SSP, ACC_NONE, 0.75, 0.25, 0},
              {2, 0, MODE_SSP, ACC_NONE, 1.0 / 3.0, 2.0 / 3.0, 0}};
    default:
      return {{0, 1, MODE_AXPY, ACC_SET, 0.5, 0, 0},
              {1, 2, MODE_AXPY, ACC_ADD, 0.5, 0, 2.0},
              {2, 1, MODE_AXPY, ACC_ADD, 1.0, 0, 2.0},
              {1, 0, MODE_FINAL, ACC_NONE, 0, 0, 0}};
  }
}

template <typename Real>
Metric<Real> metric_ptrs(const Real* base, const fvm_desc& d) {
  Metric<Real> m;
  const Real* p = base;
  auto take = [&](int n) { const Real* r = p; p += n; return r; };
  m.dx1 = take(d.nx1); m.dx2 = take(d.nx2); m.dx3 = take(d.nx3);
  m.r_c = take(d.nx1); m.r_f = take(d.nx1 + 1); m.r_f2 = take(d.nx1 + 1);
  m.a1 = take(d.nx1); m.b1 = take(d.nx1); m.inv_r = take(d.nx1); m.two_inv_r = take(d.nx1);
  m.c2 = take(d.nx2); m.sin_f2 = take(d.nx2 + 1); m.sin_c2 = take(d.nx2); m.cot_c2 = take(d.nx2);
  m.inv_dx1 = take(d.nx1); m.inv_dx2 = take(d.nx2); m.inv_dx3 = take(d.nx3); m.inv_sin_c2 = take(d.nx2);
  return m;
}

std::vector<double> pack_metric(const HostMetric& m) {
  std::vector<double> v;
  for (auto* t : {&m.dx1, &m.dx2, &m.dx3, &m.r_c, &m.r_f, &m.r_f2, &m.a1, &m.b1, &m.inv_r, &m.two_inv_r, &m.c2,
                  &m.sin_f2, &m.sin_c2, &m.cot_c2, &m.inv_dx1, &m.inv_dx2, &m.inv_dx3, &m.inv_sin_c2})
    v.insert(v.end(), t->begin(), t->end());
  return v;
}

template <typename Real, typename P>
void fill_common(fvm_handle* h, const StageDef& sd, bool rhs_only, P& p) {
  p.lay = h->lay;
  p.met = metric_ptrs<Real>(static_cast<const Real*>(h->met_real), h->d);
  p.u0 = static_cast<const Real*>(h->U[0]);
  p.out = static_cast<Real*>(h->U[sd.out]);
  p.acc = static_cast<Real*>(h->acc);
  p.dt = &h->clk->dt;
  p.active = rhs_only ? nullptr : &h->clk->active;
  p.coef.mode = sd.mode;
  p.coef.accmode = sd.accmode;
  p.coef.ca = sd.ca;
  p.coef.cb = sd.cb;
  p.coef.wacc = sd.w;
  p.coef.u0_is_input = sd.in == 0 ? 1 : 0;
  p.status = h->status;
  p.zchunk = h->zchunk;
  p.wait_ns = h->wait_ns;
  p.drain_ns = h->drain_ns;
  p.extra_tx = h->extra_tx;
}

// x3 fluxes cancel exactly on a one-plane grid whose x3 ghosts copy the plane
// (periodic or Neumann for every variable): the float32 inviscid path then
// skips the x3 pipeline ("flat").
bool flat_grid(const fvm_handle* h) {
  const fvm_desc& d = h->d;
  if (h->f64 || d.nx3 != 1 || d.physics != FVM_NAVIER_STOKES || d.params[1] != 0.0) return false;
  for (int q = 0; q < h->nv; ++q)
    for (int s = 4; s < 6; ++s)
      if (d.bc_kind[q][s] != FVM_BC_PERIODIC && d.bc_kind[q][s] != FVM_BC_NEUMANN) return false;
  return true;
}

template <typename Real>
NsParams<Real> make_ns_params(fvm_handle* h, const StageDef& sd, bool rhs_only) {
  const fvm_desc& d = h->d;
  NsParams<Real> p{};
  fill_common<Real>(h, sd, rhs_only, p);
  p.gamma = d.params[0];
  p.mu = d.params[1];
  p.g1 = d.params[2];
  p.g2 = d.params[3];
  p.g3 = d.params[4];
  p.flat = (!rhs_only && flat_grid(h)) ? 1 : 0;
  p.ysub = 1;
  return p;
}

template <typename Real>
HeatParams<Real> make_heat_params(fvm_handle* h, const StageDef& sd, bool rhs_only) {
  const fvm_desc& d = h->d;
  HeatParams<Real> p{};
  fill_common<Real>(h, sd, rhs_only, p);
  p.rho_cp = d.params[0] * d.params[1];
  p.inv_rho_cp = 1.0 / (d.params[0] * d.params[1]);
  p.k = d.params[2];
  p.q = d.params[3];
  return p;
}

// The float32 stage combination reads U0 from memory (fvm_common.cuh needs_u0).
bool needs_u0_host(const StageDef& sd) {
  return sd.mode >= MODE_AXPY && sd.mode != MODE_FINAL && sd.in != 0;
}

template <typename Real>
cudaError_t launch_stage(fvm_handle* h, const StageDef& sd, bool rhs_only, bool prepare_only = false) {
  const fvm_desc& d = h->d;
  const int nsm = prepare_only ? -1 : h->nsm;
  if (d.physics == FVM_HEAT) {
    if constexpr (std::is_same<Real, float>::value) {
      if (heat_pc_kernel(h))
        return launch_heat_pc(d.coords, h->tmap[sd.in], make_heat_params<float>(h, sd, rhs_only), h->stream, nsm,
                              h->tile_ty);
    }
    return launch_heat<Real>(kernel_limiter(d), d.coords, h->tmap[sd.in], make_heat_params<Real>(h, sd, rhs_only),
                             h->stream, nsm, h->tile_ty);
  }
  if (d.physics == FVM_MAXWELL) {
    MaxwellParams<Real> p{};
    fill_common<Real>(h, sd, rhs_only, p);
    p.mu = d.params[0];
    p.ep = d.params[1];
    p.sigma = d.params[2];
    p.rho_c = d.params[3];
    p.chi_b = d.params[4];
    p.chi_d = d.params[5];
    p.c = 1 / std::sqrt(d.params[0] * d.params[1]);
    if constexpr (std::is_same<Real, float>::value) {
      MxStripSource src;
      src.tmap = h->tmap[sd.in];
      src.u0map = h->smap;
      src.accmap = h->amap;
      src.p = p;
      const int nbuf = (needs_u0_host(sd) ? 1 : 0) + (sd.mode == MODE_FINAL || sd.accmode == ACC_ADD ? 1 : 0);
      return launch_mx_strip(kernel_limiter(d), d.coords, src, h->tile_ty, nbuf, h->stream, nsm);
    }
    return launch_maxwell<Real>(kernel_limiter(d), d.riemann, d.coords, h->tmap[sd.in], p, h->stream, nsm);
  }
  const bool visc = d.params[1] != 0.0;
  if constexpr (std::is_same<Real, float>::value) {
    if (strip_kernel(h)) {
      NsStripSource src;
      src.tmap = h->tmap[sd.in];
      src.u0map = h->smap;
      src.accmap = h->amap;
      src.p = make_ns_params<float>(h, sd, rhs_only);
      const int nbuf = (needs_u0_host(sd) ? 1 : 0) + (sd.mode == MODE_FINAL || sd.accmode == ACC_ADD ? 1 : 0);
      return visc ? launch_ns_strip_visc(kernel_limiter(d), d.riemann, src, h->tile_ty, nbuf, h->stream, nsm)
                  : launch_ns_strip(kernel_limiter(d), d.riemann, src, h->tile_ty, nbuf, h->stream, nsm);
    }
  }
  return launch_ns<Real>(kernel_limiter(d), d.riemann, d.coords, visc, h->tmap[sd.in],
                         make_ns_params<Real>(h, sd, rhs_only), h->stream, nsm, h->tile_ty);
}

// Ghost fill of state buffer b; `ck` (optional) also closes the step's clock.
// `in_step`: a fill inside a step, which leaves out the x3 slabs of a
// one-plane grid (its stage kernels never read them; downloads fill them).
cudaError_t launch_bc(fvm_handle* h, int b, const ClockArgs* ck = nullptr, bool in_step = false) {
  const Layout& L = h->lay;
  const long long face = std::max({(long long)L.ny * L.nz, (long long)L.nx * L.nz, (long long)L.nx * L.ny});
  // about one resident wave: blocks per face row up to 8 blocks/SM over all rows
  const long long per_row = std::max(1LL, std::min((face + 256LL * BCF - 1) / (256LL * BCF),
                                                   (8LL * h->nsm + 6 * h->nv - 1) / (6 * h->nv)));
  const dim3 grid((unsigned)per_row, (unsigned)(6 * h->nv));
  const BcSpec bc = make_bc(h->d, h->nv);
  const ClockArgs c = ck ? *ck : ClockArgs{nullptr, 0, 0.0, 0.0, nullptr};
  const int skip = in_step && flat_grid(h) ? (1 << 4) | (1 << 5) : 0;
  if (h->f64) bc_fill_kernel<double><<<grid, 256, 0, h->stream>>>(static_cast<double*>(h->U[b]), L, h->nv, bc, c, skip);
  else bc_fill_kernel<float><<<grid, 256, 0, h->stream>>>(static_cast<float*>(h->U[b]), L, h->nv, bc, c, skip);
  return cudaGetLastError();
}

template <typename Real>
cudaError_t launch_dt_reduce(fvm_handle* h) {
  const int blocks = h->nsm * 3;  // the kernel's resident blocks per SM (__launch_bounds__)
  const Real* u = static_cast<const Real*>(h->U[0]);
  const double g = h->d.params[0], mu = h->d.params[1];
  switch (h->d.coords) {
    case FVM_CARTESIAN: ns_dt_reduce_kernel<Real, COORD_CART><<<blocks, 256, 0, h->stream>>>(u, h->lay, h->md, g, mu, h->clk, h->status); break;
    case FVM_CYLINDRICAL: ns_dt_reduce_kernel<Real, COORD_CYL><<<blocks, 256, 0, h->stream>>>(u, h->lay, h->md, g, mu, h->clk, h->status); break;
    default: ns_dt_reduce_kernel<Real, COORD_SPH><<<blocks, 256, 0, h->stream>>>(u, h->lay, h->md, g, mu, h->clk, h->status); break;
  }
  return cudaGetLastError();
}

// Per-kernel device times of un-captured steps (CUDA events on the handle's
// stream around each launch).
struct Prof {
  cudaEvent_t a = nullptr, b = nullptr;
  double stage_ms = 0.0, other_ms = 0.0;
  int stage_launches = 0;
  ~Prof() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Two CUDA events, destroyed on every return path.
struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Enqueue one time step on the handle's stream: [dt reduction], clock, then
// per stage {ghost fill, fused stage kernel}.
int enqueue_step(fvm_handle* h, int dt_mode, Prof* pf) {
  auto mark = [&](cudaEvent_t e) -> int {
    if (pf) FVM_CK(cudaEventRecord(e, h->stream));
    return FVM_OK;
  };
  auto close = [&](bool stage) -> int {
    if (!pf) return FVM_OK;
    FVM_CK(cudaEventRecord(pf->b, h->stream));
    FVM_CK(cudaEventSynchronize(pf->b));
    float ms = 0.f;
    FVM_CK(cudaEventElapsedTime(&ms, pf->a, pf->b));
    if (stage) { pf->stage_ms += ms; pf->stage_launches += 1; }
    else pf->other_ms += ms;
    return FVM_OK;
  };
  int rc;
  const bool state_dt = h->d.physics == FVM_NAVIER_STOKES;
  if ((rc = mark(pf ? pf->a : nullptr))) return rc;
  if (dt_mode == 0 && state_dt) {
    cudaError_t e = h->f64 ? launch_dt_reduce<double>(h) : launch_dt_reduce<float>(h);
    if (e != cudaSuccess) return fail(FVM_E_CUDA, std::string("dt reduction: ") + cudaGetErrorString(e));
  }
  // the first stage's ghost fill also closes the clock (dt, t, step count, active)
  const int cmode = dt_mode == 1 ? 1 : (state_dt ? 0 : 2);
  const ClockArgs ck{h->clk, cmode, h->max_inv_l2, h->const_rate, h->status};
  const std::vector<StageDef> stages = stage_table(h->d.integrator);
  {
    cudaError_t e = launch_bc(h, stages.front().in, &ck, true);
    if (e != cudaSuccess) return fail(FVM_E_CUDA, std::string("ghost fill: ") + cudaGetErrorString(e));
  }
  if (h->closure) {
    // face corrections from the step's base state (periodic: no ghosts read)
    cudaError_t e = closure::enqueue_infer(h->closure, static_cast<const float*>(h->U[0]), h->lay,
                                           (float)h->d.params[0], h->stream);
    if (e != cudaSuccess) return fail(FVM_E_CUDA, std::string("closure: ") + cudaGetErrorString(e));
  }
  bool first = true;
  for (const StageDef& sd : stages) {
    cudaError_t e = first ? cudaSuccess : launch_bc(h, sd.in, nullptr, true);
    first = false;
    if (e != cudaSuccess) return fail(FVM_E_CUDA, std::string("ghost fill: ") + cudaGetErrorString(e));
    if ((rc = close(false))) return rc;
    if ((rc = mark(pf ? pf->a : nullptr))) return rc;
    e = h->f64 ? launch_stage<double>(h, sd, false) : launch_stage<float>(h, sd, false);
    if (e != cudaSuccess) return fail(FVM_E_CUDA, std::string("stage kernel: ") + cudaGetErrorString(e));
    if (h->closure) {
      // d(out)/d(dt k) of the stage combination
      const double coef = sd.mode == MODE_EULER ? 1.0 : (sd.mode == MODE_AXPY ? sd.ca : sd.cb);
      const double hh[3] = {(h->d.x1_max - h->d.x1_min) / h->d.nx1, (h->d.x2_max - h->d.x2_min) / h->d.nx2,
                            (h->d.x3_max - h->d.x3_min) / h->d.nx3};
      e = closure::enqueue_fix(h->closure, static_cast<const float*>(h->U[sd.in]), static_cast<float*>(h->U[sd.out]),
                               h->lay, (float)h->d.params[0], (float)coef, (float)h->closure_beta, hh, h->clk,
                               h->closure_nswitch, h->stream);
      if (e != cudaSuccess) return fail(FVM_E_CUDA, std::string("closure correction: ") + cudaGetErrorString(e));
    }
    if ((rc = close(true))) return rc;
    if ((rc = mark(pf ? pf->a : nullptr))) return rc;
  }
  if (h->d.integrator == FVM_EULER_EXPLICIT) {
    // Euler writes stage buffer 1; the state lives in buffer 0.
    FVM_CK(cudaMemcpyAsync(h->U[0], h->U[1], h->lay.var_stride * h->nv * h->esz, cudaMemcpyDeviceToDevice,
                           h->stream));
  }
  return close(false);
}

int ensure_graph(fvm_handle* h, int dt_mode) {
  cudaGraphExec_t& ge = h->graph[dt_mode];
  if (ge) return FVM_OK;
  cudaGraph_t g;
  {
    StageDef sd{0, 1, MODE_RHS, ACC_NONE, 0, 0, 0};
    FVM_CK(h->f64 ? launch_stage<double>(h, sd, true, true) : launch_stage<float>(h, sd, true, true));
  }
  FVM_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(h, dt_mode, nullptr);
  cudaError_t ce = cudaStreamEndCapture(h->stream, &g);
  if (rc) return rc;
  FVM_CK(ce);
  ce = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  FVM_CK(ce);
  return FVM_OK;
}

}  // namespace

extern "C" {

int fvm_last_error(char* buf, int len) {
  if (!buf || len <= 0) return FVM_E_INVALID;
  std::snprintf(buf, (size_t)len, "%s", g_err.c_str());
  return FVM_OK;
}

int fvm_create(const fvm_desc* desc, fvm_handle** out) {
  if (!out) return fail(FVM_E_INVALID, "null output pointer");
  *out = nullptr;
  int rc = validate(desc);
  if (rc) return rc;
  fvm_handle* h = new fvm_handle();
  h->d = *desc;
  const fvm_desc& d = h->d;
  h->nv = d.physics == FVM_NAVIER_STOKES ? 5 : (d.physics == FVM_HEAT ? 1 : 6);
  h->f64 = d.precision == FVM_FP64;
  h->esz = h->f64 ? 8 : 4;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, dev);
  Layout& L = h->lay;
  L.nx = d.nx1; L.ny = d.nx2; L.nz = d.nx3;
  L.padx = h->f64 ? 1 : 3;
  const long long row = (long long)L.nx + 2 + L.padx;
  L.pitch = (row + 31) / 32 * 32;
  L.plane = L.pitch * (L.ny + 2);
  L.var_stride = (L.plane * (L.nz + 2) + 63) / 64 * 64;
  h->zchunk = d.zchunk > 0 ? d.zchunk : 64;
  auto cleanup = [&](int code) { fvm_destroy(h); return code; };
#define FVM_CKC(x)                                                                                         \
  do {                                                                                                     \
    cudaError_t e_ = (x);                                                                                  \
    if (e_ != cudaSuccess) return cleanup(fail(e_ == cudaErrorMemoryAllocation ? FVM_E_NOMEM : FVM_E_CUDA, \
                                               std::string(#x) + ": " + cudaGetErrorString(e_)));          \
  } while (0)
  FVM_CKC(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  const size_t state_bytes = (size_t)L.var_stride * h->nv * h->esz;
  for (int b = 0; b < 3; ++b) {
    FVM_CKC(cudaMalloc(&h->U[b], state_bytes));
    FVM_CKC(cudaMemsetAsync(h->U[b], 0, state_bytes, h->stream));
  }
  h->device_bytes = 3 * (long long)state_bytes;
  if (d.integrator == FVM_RK3 || d.integrator == FVM_RK4) {
    FVM_CKC(cudaMalloc(&h->acc, state_bytes));
    FVM_CKC(cudaMemsetAsync(h->acc, 0, state_bytes, h->stream));
    h->device_bytes += state_bytes;
  }
  // metric tables
  const HostMetric hm = build_metric(d);
  const std::vector<double> packed = pack_metric(hm);
  FVM_CKC(cudaMalloc(&h->met_f64, packed.size() * sizeof(double)));
  FVM_CKC(cudaMemcpy(h->met_f64, packed.data(), packed.size() * sizeof(double), cudaMemcpyHostToDevice));
  h->md = metric_ptrs<double>(h->met_f64, d);
  if (h->f64) {
    h->met_real = h->met_f64;
  } else {
    std::vector<float> pf(packed.begin(), packed.end());
    FVM_CKC(cudaMalloc(&h->met_real, pf.size() * sizeof(float)));
    FVM_CKC(cudaMemcpy(h->met_real, pf.data(), pf.size() * sizeof(float), cudaMemcpyHostToDevice));
    h->mf = metric_ptrs<float>(static_cast<float*>(h->met_real), d);
  }
  // constant parts of the CFL step (navier_stokes.py:575, heat.py:331-338, maxwell.py:586-598)
  double mx = 0.0, rmax = 0.0;
  for (int k = 0; k < d.nx3; ++k)
    for (int j = 0; j < d.nx2; ++j)
      for (int i = 0; i < d.nx1; ++i) {
        double Ls[3];
        host_lengths(hm, d.coords, i, j, k, Ls);
        const double s = (1.0 / (Ls[0] * Ls[0]) + 1.0 / (Ls[1] * Ls[1])) + 1.0 / (Ls[2] * Ls[2]);
        mx = std::max(mx, s);
        if (d.physics == FVM_MAXWELL) {
          const double c = 1 / std::sqrt(d.params[0] * d.params[1]);
          const double ml = std::max(std::fabs(-c), std::fabs(c));
          rmax = std::max(rmax, std::max(std::max(ml / Ls[0], ml / Ls[1]), ml / Ls[2]));
        }
      }
  h->max_inv_l2 = mx;
  if (d.physics == FVM_HEAT) {
    const double nu = d.params[2] / (d.params[0] * d.params[1]);
    h->const_rate = 0.0 + (2 * nu) * mx;
  } else if (d.physics == FVM_MAXWELL) {
    const double chi = std::max(d.params[4], d.params[5]);
    h->const_rate = rmax + (2.0 * chi) * mx;
  }
  FVM_CKC(cudaMalloc(&h->clk, sizeof(Clock)));
  Clock c0{};
  c0.t = 0.0;
  c0.t_end = std::numeric_limits<double>::infinity();
  c0.cfl = 0.4;
  c0.active = 1;
  FVM_CKC(cudaMemcpy(h->clk, &c0, sizeof(Clock), cudaMemcpyHostToDevice));
  FVM_CKC(cudaMalloc(&h->status, sizeof(unsigned)));
  FVM_CKC(cudaMemset(h->status, 0, sizeof(unsigned)));
  FVM_CKC(cudaMalloc(&h->partials, sizeof(double) * 8 * 1024));
  FVM_CKC(cudaMalloc(&h->totals_dev, sizeof(double) * 8));
  h->stage_elems = (size_t)h->nv * (d.nx1 + 2) * (d.nx2 + 2) * (d.nx3 + 2);
  FVM_CKC(cudaMalloc(&h->stage_dev, h->stage_elems * sizeof(double)));
  FVM_CKC(cudaMallocHost(&h->stage_host, h->stage_elems * sizeof(double)));
  h->device_bytes += h->stage_elems * sizeof(double);
#undef FVM_CKC
  h->tile_ty = d.tile_ty > 0 ? d.tile_ty : default_tile_ty(d);
  rc = make_tmaps(h);
  if (rc) {
    fvm_destroy(h);
    return rc;
  }
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
    fvm_destroy(h);
    return fail(FVM_E_CUDA, "initialisation failed");
  }
  *out = h;
  return FVM_OK;
}

int fvm_destroy(fvm_handle* h) {
  if (!h) return FVM_OK;
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto& g : h->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& b : h->U)
    if (b) cudaFree(b);
  if (h->acc) cudaFree(h->acc);
  if (h->met_real && h->met_real != h->met_f64) cudaFree(h->met_real);
  if (h->met_f64) cudaFree(h->met_f64);
  if (h->clk) cudaFree(h->clk);
  if (h->status) cudaFree(h->status);
  if (h->partials) cudaFree(h->partials);
  if (h->totals_dev) cudaFree(h->totals_dev);
  if (h->stage_dev) cudaFree(h->stage_dev);
  if (h->stage_host) cudaFreeHost(h->stage_host);
  if (h->s_in) cudaStreamSynchronize(h->s_in);
  if (h->s_out) cudaStreamSynchronize(h->s_out);
  if (h->stage_out) cudaFree(h->stage_out);
  for (cudaEvent_t e : {h->ev_in_ready, h->ev_in_free, h->ev_out_ready, h->ev_out_free})
    if (e) cudaEventDestroy(e);
  if (h->s_in) cudaStreamDestroy(h->s_in);
  if (h->s_out) cudaStreamDestroy(h->s_out);
  if (h->closure_nswitch) cudaFree(h->closure_nswitch);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return FVM_OK;
}

int fvm_info(const fvm_handle* h, int* nvars, long long* device_bytes) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (nvars) *nvars = h->nv;
  if (device_bytes) *device_bytes = h->device_bytes;
  return FVM_OK;
}

static int transpose(fvm_handle* h, bool to_device, int buf, bool interior, double* stage = nullptr) {
  const fvm_desc& d = h->d;
  if (!stage) stage = h->stage_dev;
  const int m1 = interior ? d.nx1 : d.nx1 + 2, m2 = interior ? d.nx2 : d.nx2 + 2, m3 = interior ? d.nx3 : d.nx3 + 2;
  const int off = interior ? 1 : 0;
  dim3 grid((m3 + 31) / 32, (m1 + 31) / 32, m2 * h->nv), block(32, 8);
  if (h->f64) {
    if (to_device)
      transpose_kernel<double, true><<<grid, block, 0, h->stream>>>(stage, nullptr, nullptr,
                                                                     static_cast<double*>(h->U[buf]), h->lay, m1, m2, m3, off);
    else
      transpose_kernel<double, false><<<grid, block, 0, h->stream>>>(nullptr, stage,
                                                                      static_cast<const double*>(h->U[buf]), nullptr,
                                                                      h->lay, m1, m2, m3, off);
  } else {
    if (to_device)
      transpose_kernel<float, true><<<grid, block, 0, h->stream>>>(stage, nullptr, nullptr,
                                                                    static_cast<float*>(h->U[buf]), h->lay, m1, m2, m3, off);
    else
      transpose_kernel<float, false><<<grid, block, 0, h->stream>>>(nullptr, stage,
                                                                     static_cast<const float*>(h->U[buf]), nullptr,
                                                                     h->lay, m1, m2, m3, off);
  }
  FVM_CK(cudaGetLastError());
  return FVM_OK;
}

int fvm_upload(fvm_handle* h, const double* host_state) {
  if (!h || !host_state) return fail(FVM_E_INVALID, "null argument");
  const size_t bytes = h->stage_elems * sizeof(double);
  FVM_CK(cudaMemcpyAsync(h->stage_dev, host_state, bytes, cudaMemcpyHostToDevice, h->stream));
  int rc = transpose(h, true, 0, false);
  if (rc) return rc;
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

static void fill_edges_corners(double* f, int n1, int n2, int n3) {
  // ghost edges/corners as averages of adjacent ghost faces (src/solver.py:39-61)
  const int N[3] = {n1 + 2, n2 + 2, n3 + 2};
  auto at = [&](int i, int j, int k) -> double& { return f[((long long)i * N[1] + j) * N[2] + k]; };
  for (int a = 0; a < 3; ++a)
    for (int b = a + 1; b < 3; ++b) {
      const int c = 3 - a - b;
      for (int ea = 0; ea < 2; ++ea)
        for (int eb = 0; eb < 2; ++eb)
          for (int t = 1; t <= N[c] - 2; ++t) {
            int idx[3], p[3], q[3];
            idx[a] = ea ? N[a] - 1 : 0;
            idx[b] = eb ? N[b] - 1 : 0;
            idx[c] = t;
            for (int z = 0; z < 3; ++z) { p[z] = idx[z]; q[z] = idx[z]; }
            p[a] = ea ? N[a] - 2 : 1;
            q[b] = eb ? N[b] - 2 : 1;
            at(idx[0], idx[1], idx[2]) = 0.5 * (at(p[0], p[1], p[2]) + at(q[0], q[1], q[2]));
          }
    }
  for (int ci = 0; ci < 2; ++ci)
    for (int cj = 0; cj < 2; ++cj)
      for (int ck = 0; ck < 2; ++ck) {
        const int i = ci ? N[0] - 1 : 0, j = cj ? N[1] - 1 : 0, k = ck ? N[2] - 1 : 0;
        const int ii = ci ? N[0] - 2 : 1, jj = cj ? N[1] - 2 : 1, kk = ck ? N[2] - 2 : 1;
        at(i, j, k) = (at(ii, j, k) + at(i, jj, k) + at(i, j, kk)) / 3.0;
      }
}

int fvm_download(fvm_handle* h, double* host_state) {
  if (!h || !host_state) return fail(FVM_E_INVALID, "null argument");
  FVM_CK(launch_bc(h, 0));
  int rc = transpose(h, false, 0, false);
  if (rc) return rc;
  FVM_CK(cudaMemcpyAsync(host_state, h->stage_dev, h->stage_elems * sizeof(double), cudaMemcpyDeviceToHost,
                         h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  const size_t per = h->stage_elems / h->nv;
  for (int q = 0; q < h->nv; ++q) fill_edges_corners(host_state + q * per, h->d.nx1, h->d.nx2, h->d.nx3);
  return FVM_OK;
}

namespace {
// Streams, events and the second staging buffer of the pipelined transfers,
// made on first use.
int ensure_async(fvm_handle* h) {
  if (h->s_in) return FVM_OK;
  FVM_CK(cudaStreamCreateWithFlags(&h->s_in, cudaStreamNonBlocking));
  FVM_CK(cudaStreamCreateWithFlags(&h->s_out, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&h->ev_in_ready, &h->ev_in_free, &h->ev_out_ready, &h->ev_out_free})
    FVM_CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  const cudaError_t e = cudaMalloc(&h->stage_out, h->stage_elems * sizeof(double));
  if (e != cudaSuccess) return fail(FVM_E_NOMEM, std::string("download staging: ") + cudaGetErrorString(e));
  h->device_bytes += h->stage_elems * sizeof(double);
  // nothing is in flight yet: both staging buffers start free
  FVM_CK(cudaEventRecord(h->ev_in_free, h->stream));
  FVM_CK(cudaEventRecord(h->ev_out_free, h->s_out));
  return FVM_OK;
}
}  // namespace

int fvm_upload_async(fvm_handle* h, const double* host_state) {
  if (!h || !host_state) return fail(FVM_E_INVALID, "null argument");
  int rc = ensure_async(h);
  if (rc) return rc;
  // copy stream: wait until the previous upload's transpose has read the
  // staging buffer, then copy; the handle's stream transposes once it lands
  FVM_CK(cudaStreamWaitEvent(h->s_in, h->ev_in_free, 0));
  FVM_CK(cudaMemcpyAsync(h->stage_dev, host_state, h->stage_elems * sizeof(double), cudaMemcpyHostToDevice, h->s_in));
  FVM_CK(cudaEventRecord(h->ev_in_ready, h->s_in));
  FVM_CK(cudaStreamWaitEvent(h->stream, h->ev_in_ready, 0));
  if ((rc = transpose(h, true, 0, false))) return rc;
  FVM_CK(cudaEventRecord(h->ev_in_free, h->stream));
  return FVM_OK;
}

int fvm_download_async(fvm_handle* h, double* host_state) {
  if (!h || !host_state) return fail(FVM_E_INVALID, "null argument");
  int rc = ensure_async(h);
  if (rc) return rc;
  FVM_CK(launch_bc(h, 0));
  // the previous download's copy must have drained the staging buffer
  FVM_CK(cudaStreamWaitEvent(h->stream, h->ev_out_free, 0));
  if ((rc = transpose(h, false, 0, false, h->stage_out))) return rc;
  const fvm_desc& d = h->d;
  const int longest = std::max(d.nx1, std::max(d.nx2, d.nx3));
  edges_kernel<<<dim3((longest + 255) / 256, 12 * h->nv), 256, 0, h->stream>>>(h->stage_out, d.nx1, d.nx2, d.nx3);
  FVM_CK(cudaGetLastError());
  corners_kernel<<<1, 64, 0, h->stream>>>(h->stage_out, d.nx1, d.nx2, d.nx3, h->nv);
  FVM_CK(cudaGetLastError());
  FVM_CK(cudaEventRecord(h->ev_out_ready, h->stream));
  FVM_CK(cudaStreamWaitEvent(h->s_out, h->ev_out_ready, 0));
  FVM_CK(cudaMemcpyAsync(host_state, h->stage_out, h->stage_elems * sizeof(double), cudaMemcpyDeviceToHost,
                         h->s_out));
  FVM_CK(cudaEventRecord(h->ev_out_free, h->s_out));
  return FVM_OK;
}

int fvm_step_async(fvm_handle* h, int n_steps, int dt_mode) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (dt_mode != 0 && dt_mode != 1) return fail(FVM_E_INVALID, "dt_mode must be 0 (CFL) or 1 (fixed)");
  if (n_steps <= 0) return FVM_OK;
  int rc = ensure_graph(h, dt_mode);
  if (rc) return rc;
  for (int s = 0; s < n_steps; ++s) FVM_CK(cudaGraphLaunch(h->graph[dt_mode], h->stream));
  return FVM_OK;
}

int fvm_synchronize(fvm_handle* h) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  FVM_CK(cudaStreamSynchronize(h->stream));
  if (h->s_in) FVM_CK(cudaStreamSynchronize(h->s_in));
  if (h->s_out) FVM_CK(cudaStreamSynchronize(h->s_out));
  return FVM_OK;
}

int fvm_residual(fvm_handle* h, double* host_rhs) {
  if (!h || !host_rhs) return fail(FVM_E_INVALID, "null argument");
  StageDef sd{0, 1, MODE_RHS, ACC_NONE, 0, 0, 0};
  cudaError_t e = h->f64 ? launch_stage<double>(h, sd, true) : launch_stage<float>(h, sd, true);
  if (e != cudaSuccess) return fail(FVM_E_CUDA, std::string("stage kernel: ") + cudaGetErrorString(e));
  int rc = transpose(h, false, 1, true);
  if (rc) return rc;
  const size_t n = (size_t)h->nv * h->d.nx1 * h->d.nx2 * h->d.nx3;
  FVM_CK(cudaMemcpyAsync(host_rhs, h->stage_dev, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

int fvm_set_time(fvm_handle* h, double t, double t_end, double cfl) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (!(cfl > 0.0)) return fail(FVM_E_INVALID, "CFL must be positive");
  Clock c;
  FVM_CK(cudaMemcpyAsync(&c, h->clk, sizeof(Clock), cudaMemcpyDeviceToHost, h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  c.t = t;
  c.t_end = t_end;
  c.cfl = cfl;
  c.active = 1;
  FVM_CK(cudaMemcpyAsync(h->clk, &c, sizeof(Clock), cudaMemcpyHostToDevice, h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

int fvm_set_dt(fvm_handle* h, double dt) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (!(dt > 0.0)) return fail(FVM_E_INVALID, "dt must be positive");
  FVM_CK(cudaMemcpyAsync(&h->clk->dt_fixed, &dt, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

int fvm_get_time(fvm_handle* h, double* t, long long* steps, double* last_dt) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  Clock c;
  FVM_CK(cudaMemcpyAsync(&c, h->clk, sizeof(Clock), cudaMemcpyDeviceToHost, h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  if (t) *t = c.t;
  if (steps) *steps = c.steps;
  if (last_dt) *last_dt = c.dt;
  return FVM_OK;
}

int fvm_compute_dt(fvm_handle* h, double cfl, double* dt_out) {
  if (!h || !dt_out) return fail(FVM_E_INVALID, "null argument");
  if (!(cfl > 0.0)) return fail(FVM_E_INVALID, "CFL must be positive");
  if (h->d.physics != FVM_NAVIER_STOKES) {
    *dt_out = cfl / h->const_rate;
    return FVM_OK;
  }
  cudaError_t e = h->f64 ? launch_dt_reduce<double>(h) : launch_dt_reduce<float>(h);
  FVM_CK(e);
  unsigned long long red[2];
  FVM_CK(cudaMemcpyAsync(red, h->clk->red, sizeof(red), cudaMemcpyDeviceToHost, h->stream));
  FVM_CK(cudaMemsetAsync(h->clk->red, 0, sizeof(red), h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  double rc, nu;
  std::memcpy(&rc, &red[0], 8);
  std::memcpy(&nu, &red[1], 8);
  *dt_out = cfl / (rc + (2 * nu) * h->max_inv_l2);
  return FVM_OK;
}

int fvm_step(fvm_handle* h, int n_steps, int dt_mode) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (dt_mode != 0 && dt_mode != 1) return fail(FVM_E_INVALID, "dt_mode must be 0 (CFL) or 1 (fixed)");
  if (n_steps <= 0) return FVM_OK;
  int rc = ensure_graph(h, dt_mode);
  if (rc) return rc;
  for (int s = 0; s < n_steps; ++s) FVM_CK(cudaGraphLaunch(h->graph[dt_mode], h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

int fvm_time_steps(fvm_handle* h, int n_steps, int dt_mode, double* ms) {
  if (!h || !ms) return fail(FVM_E_INVALID, "null argument");
  if (dt_mode != 0 && dt_mode != 1) return fail(FVM_E_INVALID, "dt_mode must be 0 (CFL) or 1 (fixed)");
  int rc = ensure_graph(h, dt_mode);
  if (rc) return rc;
  EventPair ev;
  FVM_CK(cudaEventCreate(&ev.a));
  FVM_CK(cudaEventCreate(&ev.b));
  FVM_CK(cudaStreamSynchronize(h->stream));
  FVM_CK(cudaEventRecord(ev.a, h->stream));
  for (int s = 0; s < n_steps; ++s) FVM_CK(cudaGraphLaunch(h->graph[dt_mode], h->stream));
  FVM_CK(cudaEventRecord(ev.b, h->stream));
  FVM_CK(cudaEventSynchronize(ev.b));
  float t = 0.f;
  FVM_CK(cudaEventElapsedTime(&t, ev.a, ev.b));
  *ms = t;
  return FVM_OK;
}

int fvm_totals(fvm_handle* h, double* totals) {
  if (!h || !totals) return fail(FVM_E_INVALID, "null argument");
  const int nt = h->d.physics == FVM_MAXWELL ? h->nv + 1 : h->nv;
  const int blocks = std::min(1024, h->nsm * 4);
  const double emu = h->d.params[0], eep = h->d.params[1];
#define FVM_TOT(R, C)                                                                                          \
  totals_kernel<R, C><<<blocks, 256, 0, h->stream>>>(static_cast<const R*>(h->U[0]), h->lay, h->md, h->nv, nt, \
                                                     emu, eep, h->partials)
  if (h->f64) {
    if (h->d.coords == FVM_CARTESIAN) FVM_TOT(double, COORD_CART);
    else if (h->d.coords == FVM_CYLINDRICAL) FVM_TOT(double, COORD_CYL);
    else FVM_TOT(double, COORD_SPH);
  } else {
    if (h->d.coords == FVM_CARTESIAN) FVM_TOT(float, COORD_CART);
    else if (h->d.coords == FVM_CYLINDRICAL) FVM_TOT(float, COORD_CYL);
    else FVM_TOT(float, COORD_SPH);
  }
#undef FVM_TOT
  FVM_CK(cudaGetLastError());
  totals_final_kernel<<<1, 32, 0, h->stream>>>(h->partials, blocks, nt, h->totals_dev);
  FVM_CK(cudaGetLastError());
  FVM_CK(cudaMemcpyAsync(totals, h->totals_dev, nt * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

int fvm_status(fvm_handle* h, unsigned* status) {
  if (!h || !status) return fail(FVM_E_INVALID, "null argument");
  FVM_CK(cudaMemcpyAsync(status, h->status, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

int fvm_clear_status(fvm_handle* h) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  FVM_CK(cudaMemsetAsync(h->status, 0, sizeof(unsigned), h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

int fvm_set_wait_limit(fvm_handle* h, unsigned long long data_wait_ns, int never_complete) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (data_wait_ns == 0) return fail(FVM_E_INVALID, "fvm_set_wait_limit: the limit must be > 0 ns");
  FVM_CK(cudaStreamSynchronize(h->stream));
  h->wait_ns = data_wait_ns;
  // test switch: every ring copy expects 16 bytes more than it delivers, so
  // no ring wait completes; the copies themselves land within microseconds,
  // so the wait for them after a timeout needs only a short limit
  h->extra_tx = never_complete ? 16u : 0u;
  h->drain_ns = never_complete ? 100000000ull : 1000000000ull;
  for (auto& g : h->graph)  // the captured steps hold the old limit
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  return FVM_OK;
}

int fvm_step_launches(fvm_handle* h, int dt_mode, int* launches) {
  if (!h || !launches) return fail(FVM_E_INVALID, "null handle or output");
  // the launch sequence of enqueue_step, without the closure's kernels
  const int stages = (int)stage_table(h->d.integrator).size();
  *launches = (dt_mode == 0 && h->d.physics == FVM_NAVIER_STOKES ? 1 : 0) + 2 * stages;
  return FVM_OK;
}

int fvm_profile_steps(fvm_handle* h, int n_steps, int dt_mode, double* stage_kernel_ms, double* other_kernel_ms,
                      int* stage_launches) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (dt_mode != 0 && dt_mode != 1) return fail(FVM_E_INVALID, "dt_mode must be 0 (CFL) or 1 (fixed)");
  Prof pf;
  FVM_CK(cudaEventCreate(&pf.a));
  FVM_CK(cudaEventCreate(&pf.b));
  int rc = FVM_OK;
  for (int s = 0; s < n_steps && !rc; ++s) rc = enqueue_step(h, dt_mode, &pf);
  if (rc) return rc;
  FVM_CK(cudaStreamSynchronize(h->stream));
  if (stage_kernel_ms) *stage_kernel_ms = pf.stage_ms;
  if (other_kernel_ms) *other_kernel_ms = pf.other_ms;
  if (stage_launches) *stage_launches = pf.stage_launches;
  return FVM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Conserved totals without any device allocation (fvm_totals_noalloc).
//
// Callers that cannot allocate device memory themselves -- code running inside
// a host that owns and pre-plans every allocation (a memory-pool-managed
// framework, a captured or replayed command stream, an embedded runtime that
// forbids cudaMalloc after start-up) -- still need the float64 compensated
// totals.  This variant keeps the per-block partial sums in a fixed
// file-scope device array instead of the handle's `partials` buffer, so it
// needs neither a handle nor a cudaMalloc: the caller passes only its input
// cells, its cell volumes and the output array.
namespace {

constexpr int NOALLOC_BLOCKS = 1024;  // partial-sum rows held by the scratch array
constexpr int NOALLOC_MAX_VARS = 8;   // sums per row
constexpr int NOALLOC_MAX_DEVICES = 64;

// 64 KiB, resident on every GPU that loads the library until the process exits.
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_BLOCKS * NOALLOC_MAX_VARS];

std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

__global__ void totals_dense_kernel(const float* __restrict__ cells, const double* __restrict__ volumes, int nv,
                                    long long n, double* __restrict__ partials) {
  __shared__ double ss[256][NOALLOC_MAX_VARS];
  double s[NOALLOC_MAX_VARS], c[NOALLOC_MAX_VARS];
  for (int q = 0; q < NOALLOC_MAX_VARS; ++q) { s[q] = 0.0; c[q] = 0.0; }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double V = volumes[i];
    for (int q = 0; q < nv; ++q) neumaier_add(s[q], c[q], double(cells[(long long)q * n + i]) * V);
  }
  for (int q = 0; q < nv; ++q) ss[threadIdx.x][q] = s[q] + c[q];
  __syncthreads();
  if (threadIdx.x < nv) {
    double bs = 0.0, bc = 0.0;
    for (int t = 0; t < (int)blockDim.x; ++t) neumaier_add(bs, bc, ss[t][threadIdx.x]);
    partials[blockIdx.x * NOALLOC_MAX_VARS + threadIdx.x] = bs + bc;
  }
}

}  // namespace

extern "C" int fvm_totals_noalloc(const float* cells, const double* volumes, int nvars, long long ncells,
                                  double* totals, void* stream) {
  if (!cells || !volumes || !totals) return fail(FVM_E_INVALID, "fvm_totals_noalloc: null pointer");
  if (nvars < 1 || nvars > NOALLOC_MAX_VARS)
    return fail(FVM_E_INVALID, "fvm_totals_noalloc: nvars must be in [1, " + std::to_string(NOALLOC_MAX_VARS) +
                                   "], got " + std::to_string(nvars));
  if (ncells < 1) return fail(FVM_E_INVALID, "fvm_totals_noalloc: ncells must be >= 1");
  int dev = 0;
  FVM_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return fail(FVM_E_INVALID, "fvm_totals_noalloc: device ordinal above " + std::to_string(NOALLOC_MAX_DEVICES - 1));
  double* partials = nullptr;
  {
    // First call on this device (with it current): resolve the device address
    // of the scratch array.  Host code must not pass the symbol itself.
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
      if (e != cudaSuccess)
        return fail(FVM_E_CUDA, std::string("fvm_totals_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    partials = g_noalloc_ptr[dev];
  }
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long want = (ncells + 255) / 256;
  const int blocks = (int)(want < NOALLOC_BLOCKS ? want : NOALLOC_BLOCKS);
  // Every used row of the scratch array is overwritten before it is read, so
  // nothing has to be cleared between calls.
  totals_dense_kernel<<<blocks, 256, 0, s>>>(cells, volumes, nvars, ncells, partials);
  FVM_CK(cudaGetLastError());
  totals_final_kernel<<<1, 32, 0, s>>>(partials, blocks, nvars, totals);
  FVM_CK(cudaGetLastError());
  return FVM_OK;
}

// ---------------------------------------------------------------------------
// Batches of independent grids advanced together (one persistent launch per
// kernel specialisation and stage, a flat tile list over all grids, each grid
// with its own CFL time step).
struct fvm_batch {
  std::vector<fvm_handle*> h;
  int integrator = 0, nsm = 148;
  bool f64 = false;
  cudaStream_t stream = nullptr;
  struct Group {
    int physics = 0, lim = 0, riem = 0, coords = 0;
    bool visc = false;
    bool mixed = false;  // navier_stokes (lim, riem) and heat (coords) grids in one launch
    int heat_ty = MIX_HEAT_TY;        // mixed: the heat members' tile rows
    std::vector<int> nbuf;            // mixed: staged tiles of each stage
    std::vector<int> members;
    std::vector<void*> prm;           // device params array per stage
    std::vector<CUtensorMap*> maps;   // device tensor-map array per stage
    int* tile_start = nullptr;
    long long ntiles = 0;
  };
  std::vector<Group> groups;
  BatchAux* aux = nullptr;
  BcChunk* bc_chunks = nullptr;  // the ghost faces of all grids, BC_CHUNK cells per block
  int n_chunks = 0;
  struct DtGroup {
    int coords = 0;
    BatchDt* d = nullptr;
    int n = 0;
    DtBlock* blk = nullptr;  // the reduction's blocks (DT_CELLS cells each)
    int nblk = 0;
  };
  std::vector<DtGroup> dtg;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
};

namespace {

// Per-stage instance tables of the mixed group (float32 only).
int build_mixed_arrays(fvm_batch* b, fvm_batch::Group& g) {
  const std::vector<StageDef> st = stage_table(b->integrator);
  for (void* x : g.prm) cudaFree(x);
  if (g.tile_start) cudaFree(g.tile_start);
  g.prm.clear();
  g.nbuf.clear();
  g.tile_start = nullptr;
  std::vector<int> starts(1, 0);
  for (size_t si = 0; si < st.size(); ++si) {
    std::vector<MixedInst> mi(g.members.size());
    for (size_t k = 0; k < g.members.size(); ++k) {
      fvm_handle* h = b->h[g.members[k]];
      MixedInst& m = mi[k];
      m.tmap = h->tmap[st[si].in];
      int tiles = 0;
      if (h->d.physics == FVM_NAVIER_STOKES) {
        m.kind = 0;
        m.u0map = h->smap;
        m.accmap = h->amap;
        m.ns = make_ns_params<float>(h, st[si], false);
        ns_strip_tiles(m.ns, MIX_NS_TY);
        tiles = m.ns.ntx * m.ns.nty * m.ns.nzc;
      } else {
        m.kind = 1;
        m.heat = make_heat_params<float>(h, st[si], false);
        m.heat.ntx = (h->lay.nx + 31) / 32;
        m.heat.nty = (h->lay.ny + g.heat_ty - 1) / g.heat_ty;
        m.heat.nzc = (h->lay.nz + m.heat.zchunk - 1) / m.heat.zchunk;
        tiles = m.heat.ntx * m.heat.nty * m.heat.nzc;
      }
      if (si == 0) starts.push_back(starts.back() + tiles);
    }
    void* dev = nullptr;
    FVM_CK(cudaMalloc(&dev, mi.size() * sizeof(MixedInst)));
    FVM_CK(cudaMemcpy(dev, mi.data(), mi.size() * sizeof(MixedInst), cudaMemcpyHostToDevice));
    g.prm.push_back(dev);
    g.nbuf.push_back((needs_u0_host(st[si]) ? 1 : 0) + (st[si].mode == MODE_FINAL || st[si].accmode == ACC_ADD ? 1 : 0));
  }
  g.ntiles = starts.back();
  FVM_CK(cudaMalloc(&g.tile_start, starts.size() * sizeof(int)));
  FVM_CK(cudaMemcpy(g.tile_start, starts.data(), starts.size() * sizeof(int), cudaMemcpyHostToDevice));
  return FVM_OK;
}

template <typename Real>
int build_group_arrays(fvm_batch* b, fvm_batch::Group& g) {
  if (g.mixed) return build_mixed_arrays(b, g);
  const std::vector<StageDef> st = stage_table(b->integrator);
  for (void* x : g.prm) cudaFree(x);
  for (CUtensorMap* x : g.maps) cudaFree(x);
  if (g.tile_start) cudaFree(g.tile_start);
  g.prm.clear();
  g.maps.clear();
  g.tile_start = nullptr;
  std::vector<int> starts(1, 0);
  for (size_t si = 0; si < st.size(); ++si) {
    std::vector<CUtensorMap> maps;
    void* dev = nullptr;
    if (g.physics == FVM_NAVIER_STOKES) {
      std::vector<NsParams<Real>> ps;
      for (int i : g.members) {
        NsParams<Real> p = make_ns_params<Real>(b->h[i], st[si], false);
        if (g.visc) ns_tile_counts<Real, true>(p);
        else ns_tile_counts<Real, false>(p);
        ps.push_back(p);
        maps.push_back(b->h[i]->tmap[st[si].in]);
        if (si == 0) starts.push_back(starts.back() + p.ntx * p.nty * p.nzc);
      }
      FVM_CK(cudaMalloc(&dev, ps.size() * sizeof(ps[0])));
      FVM_CK(cudaMemcpy(dev, ps.data(), ps.size() * sizeof(ps[0]), cudaMemcpyHostToDevice));
    } else {
      std::vector<HeatParams<Real>> ps;
      for (int i : g.members) {
        HeatParams<Real> p = make_heat_params<Real>(b->h[i], st[si], false);
        heat_tile_counts(p);
        ps.push_back(p);
        maps.push_back(b->h[i]->tmap[st[si].in]);
        if (si == 0) starts.push_back(starts.back() + p.ntx * p.nty * p.nzc);
      }
      FVM_CK(cudaMalloc(&dev, ps.size() * sizeof(ps[0])));
      FVM_CK(cudaMemcpy(dev, ps.data(), ps.size() * sizeof(ps[0]), cudaMemcpyHostToDevice));
    }
    g.prm.push_back(dev);
    CUtensorMap* dm = nullptr;
    FVM_CK(cudaMalloc(&dm, maps.size() * sizeof(CUtensorMap)));
    FVM_CK(cudaMemcpy(dm, maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
    g.maps.push_back(dm);
  }
  g.ntiles = starts.back();
  FVM_CK(cudaMalloc(&g.tile_start, starts.size() * sizeof(int)));
  FVM_CK(cudaMemcpy(g.tile_start, starts.data(), starts.size() * sizeof(int), cudaMemcpyHostToDevice));
  return FVM_OK;
}

template <typename Real>
cudaError_t launch_group_stage(fvm_batch* b, fvm_batch::Group& g, int si, int nsm) {
  if (g.mixed) {
    const int nbuf = g.nbuf[si];
    const MixedSource src{static_cast<const MixedInst*>(g.prm[si]), g.tile_start, (int)g.members.size(),
                          mixed_bar_offset(nbuf)};
    return launch_mixed(g.lim, g.riem, g.coords, g.heat_ty, src, g.ntiles, nbuf, b->stream, nsm);
  }
  if (g.physics == FVM_NAVIER_STOKES) {
    BatchSource<NsParams<Real>> src{static_cast<const NsParams<Real>*>(g.prm[si]), g.maps[si], g.tile_start,
                                    (int)g.members.size()};
    return launch_ns_batch<Real>(g.lim, g.riem, g.coords, g.visc, src, g.ntiles, b->stream, nsm);
  }
  BatchSource<HeatParams<Real>> src{static_cast<const HeatParams<Real>*>(g.prm[si]), g.maps[si], g.tile_start,
                                    (int)g.members.size()};
  return launch_heat_batch<Real>(g.lim, g.coords, src, g.ntiles, b->stream, nsm);
}

int enqueue_batch_step(fvm_batch* b, int dt_mode) {
  const int n = (int)b->h.size();
  if (dt_mode == 0) {
    for (auto& dg : b->dtg) {
#define FVM_BDT(R, C) batch_ns_dt_kernel<R, C><<<dg.nblk, 256, 0, b->stream>>>(dg.d, dg.blk)
      if (b->f64) {
        if (dg.coords == FVM_CARTESIAN) FVM_BDT(double, COORD_CART);
        else if (dg.coords == FVM_CYLINDRICAL) FVM_BDT(double, COORD_CYL);
        else FVM_BDT(double, COORD_SPH);
      } else {
        if (dg.coords == FVM_CARTESIAN) FVM_BDT(float, COORD_CART);
        else if (dg.coords == FVM_CYLINDRICAL) FVM_BDT(float, COORD_CYL);
        else FVM_BDT(float, COORD_SPH);
      }
#undef FVM_BDT
      FVM_CK(cudaGetLastError());
    }
  }
  batch_clock_kernel<<<(n + 127) / 128, 128, 0, b->stream>>>(b->aux, n, dt_mode == 1 ? 1 : 0);
  FVM_CK(cudaGetLastError());
  const std::vector<StageDef> st = stage_table(b->integrator);
  for (size_t si = 0; si < st.size(); ++si) {
    if (b->f64) batch_bc_chunk_kernel<double><<<b->n_chunks, 256, 0, b->stream>>>(b->aux, b->bc_chunks, st[si].in);
    else batch_bc_chunk_kernel<float><<<b->n_chunks, 256, 0, b->stream>>>(b->aux, b->bc_chunks, st[si].in);
    FVM_CK(cudaGetLastError());
    for (auto& g : b->groups) {
      cudaError_t e = b->f64 ? launch_group_stage<double>(b, g, (int)si, b->nsm)
                             : launch_group_stage<float>(b, g, (int)si, b->nsm);
      if (e != cudaSuccess) return fail(FVM_E_CUDA, std::string("batched stage kernel: ") + cudaGetErrorString(e));
    }
  }
  if (b->integrator == FVM_EULER_EXPLICIT)
    for (fvm_handle* h : b->h)
      FVM_CK(cudaMemcpyAsync(h->U[0], h->U[1], h->lay.var_stride * h->nv * h->esz, cudaMemcpyDeviceToDevice,
                             b->stream));
  return FVM_OK;
}

int batch_prepare(fvm_batch* b) {
  for (auto& g : b->groups) {
    cudaError_t e = b->f64 ? launch_group_stage<double>(b, g, 0, -1) : launch_group_stage<float>(b, g, 0, -1);
    FVM_CK(e);
  }
  return FVM_OK;
}

int batch_graph(fvm_batch* b, int dt_mode) {
  cudaGraphExec_t& ge = b->graph[dt_mode];
  if (ge) return FVM_OK;
  int rc = batch_prepare(b);
  if (rc) return rc;
  for (fvm_handle* h : b->h) FVM_CK(cudaStreamSynchronize(h->stream));
  cudaGraph_t g;
  FVM_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  rc = enqueue_batch_step(b, dt_mode);
  cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
  if (rc) return rc;
  FVM_CK(ce);
  ce = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  FVM_CK(ce);
  return FVM_OK;
}

void batch_drop_graphs(fvm_batch* b) {
  for (auto& g : b->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
}

}  // namespace

extern "C" {

int fvm_batch_destroy(fvm_batch* b) {
  if (!b) return FVM_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  batch_drop_graphs(b);
  for (auto& g : b->groups) {
    for (void* x : g.prm) cudaFree(x);
    for (CUtensorMap* x : g.maps) cudaFree(x);
    if (g.tile_start) cudaFree(g.tile_start);
  }
  for (auto& dg : b->dtg) {
    if (dg.d) cudaFree(dg.d);
    if (dg.blk) cudaFree(dg.blk);
  }
  if (b->aux) cudaFree(b->aux);
  if (b->bc_chunks) cudaFree(b->bc_chunks);
  for (fvm_handle* h : b->h) fvm_destroy(h);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return FVM_OK;
}

int fvm_batch_create(const fvm_desc* descs, int n, fvm_batch** out) {
  if (!descs || !out || n < 1) return fail(FVM_E_INVALID, "fvm_batch_create: need n >= 1 descriptors");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (descs[i].integrator != descs[0].integrator)
      return fail(FVM_E_INVALID, "fvm_batch_create: all grids of a batch must use the same time integrator");
    if (descs[i].precision != descs[0].precision)
      return fail(FVM_E_INVALID, "fvm_batch_create: all grids of a batch must use the same precision");
    if (descs[i].physics == FVM_MAXWELL)
      return fail(FVM_E_INVALID, "fvm_batch_create: batches hold navier_stokes and heat grids");
  }
  fvm_batch* b = new fvm_batch();
  b->integrator = descs[0].integrator;
  b->f64 = descs[0].precision == FVM_FP64;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev);
  auto bail = [&](int rc) { fvm_batch_destroy(b); return rc; };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(FVM_E_CUDA, "stream creation failed"));
  // One launch per stage for the whole batch when every grid is float32
  // inviscid cartesian navier_stokes (one limiter / Riemann solver pair) or
  // float32 piecewise-constant heat (one coordinate system).
  bool mixed = true;
  int mlim = -1, mriem = -1, mcoords = -1;
  // heat tile rows of a mixed launch: MIX_HEAT_TY, or MIX_HEAT_TY_ALT when the
  // heat descriptors ask for it (tile_ty; the same in all of them)
  int mheat_ty = 0;
  for (int i = 0; i < n && mixed; ++i) {
    const fvm_desc& d = descs[i];
    if (strip_desc(d) && d.params[1] == 0.0) {
      if (mlim < 0) { mlim = kernel_limiter(d); mriem = d.riemann; }
      mixed = kernel_limiter(d) == mlim && d.riemann == mriem;
    } else if (heat_pc_desc(d)) {
      if (mcoords < 0) mcoords = d.coords;
      mixed = d.coords == mcoords;
      const int want = d.tile_ty == MIX_HEAT_TY_ALT ? MIX_HEAT_TY_ALT : MIX_HEAT_TY;
      if (mheat_ty && want != mheat_ty) return bail(fail(FVM_E_INVALID, "batch: heat grids ask for different tile rows"));
      mheat_ty = want;
    } else {
      mixed = false;
    }
  }
  for (int i = 0; i < n; ++i) {
    fvm_handle* h = nullptr;
    fvm_desc di = descs[i];
    di.tile_ty = 0;  // the batched kernels use each physics' default block shape
    int rc = fvm_create(&di, &h);
    if (rc) return bail(rc);
    b->h.push_back(h);
    if (mixed) {  // the block shapes of the mixed launch's two bodies
      h->tile_ty = heat_pc_desc(di) ? mheat_ty : MIX_NS_TY;
      if ((rc = make_tmaps(h))) return bail(rc);
    } else if (strip_desc(di) || heat_pc_desc(di)) {  // the tile-list kernels' shape, not the single-grid kernel's
      h->legacy = true;
      h->tile_ty = strip_desc(di) ? (di.params[1] != 0.0 ? ns_tile_ty<float, true>() : ns_tile_ty<float, false>())
                                  : HEAT_TY;
      if ((rc = make_tmaps(h))) return bail(rc);
    }
  }
  // group by kernel specialisation (one mixed group holds every grid)
  if (mixed) {
    b->groups.emplace_back();
    fvm_batch::Group& g = b->groups.back();
    g.mixed = true;
    g.heat_ty = mheat_ty ? mheat_ty : MIX_HEAT_TY;
    g.lim = std::max(mlim, 0);
    g.riem = std::max(mriem, 0);
    g.coords = std::max(mcoords, 0);
    for (int i = 0; i < n; ++i) g.members.push_back(i);
  }
  for (int i = 0; i < n && !mixed; ++i) {
    const fvm_desc& d = descs[i];
    const int lim = kernel_limiter(d);
    const bool visc = d.physics == FVM_NAVIER_STOKES && d.params[1] != 0.0;
    fvm_batch::Group* g = nullptr;
    for (auto& x : b->groups)
      if (x.physics == d.physics && x.lim == lim && x.riem == d.riemann && x.coords == d.coords && x.visc == visc) g = &x;
    if (!g) {
      b->groups.emplace_back();
      g = &b->groups.back();
      g->physics = d.physics; g->lim = lim; g->riem = d.riemann; g->coords = d.coords; g->visc = visc;
    }
    g->members.push_back(i);
  }
  for (auto& g : b->groups) {
    const int rc = b->f64 ? build_group_arrays<double>(b, g) : build_group_arrays<float>(b, g);
    if (rc) return bail(rc);
  }
  // auxiliary per-instance table and NS dt groups
  std::vector<BatchAux> aux(n);
  std::vector<BcChunk> chunks;
  for (int i = 0; i < n; ++i) {
    fvm_handle* h = b->h[i];
    BatchAux& a = aux[i];
    a.lay = h->lay;
    for (int k = 0; k < 3; ++k) a.U[k] = h->U[k];
    a.clk = h->clk;
    a.status = h->status;
    a.bc = make_bc(h->d, h->nv);
    a.nv = h->nv;
    a.cmode = h->d.physics == FVM_NAVIER_STOKES ? 0 : 2;
    a.max_inv_l2 = h->max_inv_l2;
    a.const_rate = h->const_rate;
    a.no_x3 = flat_grid(h) ? 1 : 0;
    // the six face slabs of every variable (the two x3 slabs of a one-plane
    // grid are never read by its stage kernels), in chunks of BC_CHUNK cells
    const Layout& L = h->lay;
    for (int q = 0; q < h->nv; ++q)
      for (int side = 0; side < (a.no_x3 ? 4 : 6); ++side) {
        const int axis = side >> 1;
        const long long cells = axis == 0 ? (long long)L.ny * L.nz
                                          : (axis == 1 ? (long long)L.nx * L.nz : (long long)L.nx * L.ny);
        if (cells >= (1ll << 31)) return bail(fail(FVM_E_INVALID, "batch member: a ghost face exceeds 2^31 cells"));
        for (long long s0 = 0; s0 < cells; s0 += BC_CHUNK)
          chunks.push_back(BcChunk{i, q, side, (int)s0, (int)std::min<long long>(BC_CHUNK, cells - s0)});
      }
  }
  b->n_chunks = (int)chunks.size();
  if (cudaMalloc(&b->aux, n * sizeof(BatchAux)) != cudaSuccess ||
      cudaMemcpy(b->aux, aux.data(), n * sizeof(BatchAux), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMalloc(&b->bc_chunks, chunks.size() * sizeof(BcChunk)) != cudaSuccess ||
      cudaMemcpy(b->bc_chunks, chunks.data(), chunks.size() * sizeof(BcChunk), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(FVM_E_CUDA, "batch table upload failed"));
  for (int c = 0; c < 3; ++c) {
    std::vector<BatchDt> v;
    std::vector<DtBlock> blk;
    for (int i = 0; i < n; ++i) {
      fvm_handle* h = b->h[i];
      if (h->d.physics != FVM_NAVIER_STOKES || h->d.coords != c) continue;
      const long long cells = (long long)h->lay.nx * h->lay.ny * h->lay.nz;
      const int nbx = (int)std::max(1LL, std::min((cells + DT_CELLS - 1) / DT_CELLS, 3LL * b->nsm));
      for (int k = 0; k < nbx; ++k) blk.push_back(DtBlock{(int)v.size(), k, nbx});
      v.push_back(BatchDt{h->U[0], h->lay, h->md, h->d.params[0], h->d.params[1], h->clk, h->status});
    }
    if (v.empty()) continue;
    fvm_batch::DtGroup dg;
    dg.coords = c;
    dg.n = (int)v.size();
    dg.nblk = (int)blk.size();
    // owned by the batch from here on (freed by fvm_batch_destroy on every path)
    b->dtg.push_back(dg);
    fvm_batch::DtGroup& g = b->dtg.back();
    if (cudaMalloc(&g.d, v.size() * sizeof(BatchDt)) != cudaSuccess ||
        cudaMemcpy(g.d, v.data(), v.size() * sizeof(BatchDt), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMalloc(&g.blk, blk.size() * sizeof(DtBlock)) != cudaSuccess ||
        cudaMemcpy(g.blk, blk.data(), blk.size() * sizeof(DtBlock), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(FVM_E_CUDA, "batch dt table upload failed"));
  }
  *out = b;
  return FVM_OK;
}

int fvm_batch_launches(const fvm_batch* b, int* per_stage) {
  if (!b || !per_stage) return fail(FVM_E_INVALID, "null batch or output");
  int k = 0;
  for (auto& g : b->groups) k += g.ntiles > 0 ? 1 : 0;
  *per_stage = k;
  return FVM_OK;
}

int fvm_batch_size(const fvm_batch* b, int* n, long long* tiles) {
  if (!b) return fail(FVM_E_INVALID, "null batch");
  if (n) *n = (int)b->h.size();
  if (tiles) {
    long long t = 0;
    for (auto& g : b->groups) t += g.ntiles;
    *tiles = t;
  }
  return FVM_OK;
}

int fvm_batch_handle(fvm_batch* b, int i, fvm_handle** h) {
  if (!b || !h || i < 0 || i >= (int)b->h.size()) return fail(FVM_E_INVALID, "fvm_batch_handle: bad index");
  *h = b->h[i];
  return FVM_OK;
}

int fvm_batch_step(fvm_batch* b, int n_steps, int dt_mode) {
  if (!b) return fail(FVM_E_INVALID, "null batch");
  if (dt_mode != 0 && dt_mode != 1) return fail(FVM_E_INVALID, "dt_mode must be 0 (CFL) or 1 (fixed)");
  int rc = batch_graph(b, dt_mode);
  if (rc) return rc;
  for (int s = 0; s < n_steps; ++s) FVM_CK(cudaGraphLaunch(b->graph[dt_mode], b->stream));
  FVM_CK(cudaStreamSynchronize(b->stream));
  return FVM_OK;
}

int fvm_batch_time_steps(fvm_batch* b, int n_steps, int dt_mode, double* ms) {
  if (!b || !ms) return fail(FVM_E_INVALID, "null argument");
  if (dt_mode != 0 && dt_mode != 1) return fail(FVM_E_INVALID, "dt_mode must be 0 (CFL) or 1 (fixed)");
  int rc = batch_graph(b, dt_mode);
  if (rc) return rc;
  EventPair ev;
  FVM_CK(cudaEventCreate(&ev.a));
  FVM_CK(cudaEventCreate(&ev.b));
  FVM_CK(cudaEventRecord(ev.a, b->stream));
  for (int s = 0; s < n_steps; ++s) FVM_CK(cudaGraphLaunch(b->graph[dt_mode], b->stream));
  FVM_CK(cudaEventRecord(ev.b, b->stream));
  FVM_CK(cudaEventSynchronize(ev.b));
  float t = 0.f;
  FVM_CK(cudaEventElapsedTime(&t, ev.a, ev.b));
  *ms = t;
  return FVM_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner: z-march depth (planes per tile) chosen by timing candidate
// values on the actual grid(s); the state is saved and restored around the
// trials.  Tile rows, the 32-column warp-wide tile and the 4-byte lane width
// of the coalesced 128-byte rows are fixed per kernel specialisation.
namespace {

// Depths: a fixed ladder plus ceil(nz / c) for every chunk count c (equal
// chunks).  The persistent grid deals tiles round-robin, so a launch takes
// ceil(tiles / resident blocks) tile times; some chunk count puts the tile
// count just under a whole number of waves, and timing finds it.
std::vector<int> zchunk_candidates(int nz) {
  std::vector<int> c;
  for (int z : {8, 16, 32, 48, 64, 96, 128, 192, 256})
    if (z < nz) c.push_back(z);
  c.push_back(nz);
  for (int k = 2; k <= nz / 8; ++k) c.push_back((nz + k - 1) / k);
  std::sort(c.begin(), c.end());
  c.erase(std::unique(c.begin(), c.end()), c.end());
  return c;
}

struct Saved {
  std::vector<void*> buf;
  std::vector<Clock> clk;
};

int save_states(const std::vector<fvm_handle*>& hs, Saved& s) {
  for (fvm_handle* h : hs) {
    void* p = nullptr;
    const size_t bytes = (size_t)h->lay.var_stride * h->nv * h->esz;
    FVM_CK(cudaMalloc(&p, bytes));
    FVM_CK(cudaMemcpy(p, h->U[0], bytes, cudaMemcpyDeviceToDevice));
    s.buf.push_back(p);
    Clock c;
    FVM_CK(cudaMemcpy(&c, h->clk, sizeof(Clock), cudaMemcpyDeviceToHost));
    s.clk.push_back(c);
  }
  return FVM_OK;
}

int restore_states(const std::vector<fvm_handle*>& hs, Saved& s, bool release) {
  for (size_t i = 0; i < hs.size(); ++i) {
    fvm_handle* h = hs[i];
    FVM_CK(cudaMemcpy(h->U[0], s.buf[i], (size_t)h->lay.var_stride * h->nv * h->esz, cudaMemcpyDeviceToDevice));
    FVM_CK(cudaMemcpy(h->clk, &s.clk[i], sizeof(Clock), cudaMemcpyHostToDevice));
    if (release) cudaFree(s.buf[i]);
  }
  return FVM_OK;
}

}  // namespace

extern "C" {

int fvm_autotune(fvm_handle* h, int* best_zchunk, double* best_ms) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  FVM_CK(cudaStreamSynchronize(h->stream));
  Saved sv;
  int rc = save_states({h}, sv);
  if (rc) return rc;
  int best = h->zchunk, best_ty = h->tile_ty;
  double bt = 1e30;
  std::vector<int> tys{default_tile_ty(h->d)};
  if (alt_tile_ty(h->d) != tys[0]) tys.push_back(alt_tile_ty(h->d));
  for (int ty : tys) {
    h->tile_ty = ty;
    if ((rc = make_tmaps(h))) break;
    for (int z : zchunk_candidates(h->d.nx3)) {
      h->zchunk = z;
      for (auto& g : h->graph)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
      double ms = 0.0;
      if ((rc = fvm_time_steps(h, 1, 0, &ms))) break;  // warm-up (builds the graph)
      if ((rc = fvm_time_steps(h, 3, 0, &ms))) break;
      if (ms < bt) { bt = ms; best = z; best_ty = ty; }
      if ((rc = restore_states({h}, sv, false))) break;
    }
    if (rc) break;
  }
  const int rr = restore_states({h}, sv, true);
  h->zchunk = best;
  h->tile_ty = best_ty;
  const int rt = make_tmaps(h);
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  if (rc) return rc;
  if (rr) return rr;
  if (rt) return rt;
  if (best_zchunk) *best_zchunk = best;
  if (best_ms) *best_ms = bt / 3.0;
  return FVM_OK;
}

int fvm_tiling(fvm_handle* h, int* tile_ty, int* zchunk) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (tile_ty) *tile_ty = h->tile_ty;
  if (zchunk) *zchunk = h->zchunk;
  return FVM_OK;
}

int fvm_batch_autotune(fvm_batch* b, int* best_zchunk, double* best_ms) {
  if (!b) return fail(FVM_E_INVALID, "null batch");
  for (fvm_handle* h : b->h) FVM_CK(cudaStreamSynchronize(h->stream));
  int nzmax = 1;
  for (fvm_handle* h : b->h) nzmax = std::max(nzmax, h->d.nx3);
  Saved sv;
  int rc = save_states(b->h, sv);
  if (rc) return rc;
  int best = b->h[0]->zchunk;
  double bt = 1e30;
  // heat tile rows of the mixed group (the other bodies have one shape)
  fvm_batch::Group* mg = nullptr;
  for (auto& g : b->groups)
    if (g.mixed) mg = &g;
  bool any_heat = false;
  if (mg)
    for (int i : mg->members) any_heat = any_heat || b->h[i]->d.physics == FVM_HEAT;
  std::vector<int> heat_tys{mg ? mg->heat_ty : 0};
  if (any_heat) heat_tys = {MIX_HEAT_TY, MIX_HEAT_TY_ALT};
  int best_hty = heat_tys[0];
  auto apply = [&](int z, int hty) -> int {
    for (fvm_handle* h : b->h) h->zchunk = z;
    if (mg && mg->heat_ty != hty) {
      mg->heat_ty = hty;
      for (int i : mg->members) {
        fvm_handle* h = b->h[i];
        if (h->d.physics != FVM_HEAT) continue;
        h->tile_ty = hty;
        if (int r = make_tmaps(h)) return r;
      }
    }
    batch_drop_graphs(b);
    for (auto& g : b->groups) {
      const int r = b->f64 ? build_group_arrays<double>(b, g) : build_group_arrays<float>(b, g);
      if (r) return r;
    }
    return FVM_OK;
  };
  for (int hty : heat_tys) {
    for (int z : zchunk_candidates(nzmax)) {
      if ((rc = apply(z, hty))) break;
      double ms = 0.0;
      if ((rc = fvm_batch_time_steps(b, 1, 0, &ms))) break;
      if ((rc = fvm_batch_time_steps(b, 3, 0, &ms))) break;
      if (ms < bt) { bt = ms; best = z; best_hty = hty; }
      if ((rc = restore_states(b->h, sv, false))) break;
    }
    if (rc) break;
  }
  const int rr = restore_states(b->h, sv, true);
  const int ra = apply(best, best_hty);
  if (rc) return rc;
  if (rr) return rr;
  if (ra) return ra;
  if (best_zchunk) *best_zchunk = best;
  if (best_ms) *best_ms = bt / 3.0;
  return FVM_OK;
}

}  // extern "C"

// ------------------------------------------------------------ closure hook ----
extern "C" {

int fvm_closure_attach(fvm_handle* h, fvm_closure* c, double beta) {
  if (!h) return fail(FVM_E_INVALID, "null handle");
  if (c) {
    const fvm_desc& d = h->d;
    if (d.physics != FVM_NAVIER_STOKES || h->f64 || d.coords != FVM_CARTESIAN)
      return fail(FVM_E_INVALID, "closure: needs a float32 cartesian navier_stokes handle");
    if (d.integrator != FVM_RK3_SSP && d.integrator != FVM_EULER_EXPLICIT)
      return fail(FVM_E_INVALID, "closure: integrator must be rk3_ssp or euler_explicit");
    for (int q = 0; q < h->nv; ++q)
      for (int s = 0; s < 6; ++s)
        if (d.bc_kind[q][s] != FVM_BC_PERIODIC) return fail(FVM_E_INVALID, "closure: every face must be periodic");
    if (!closure::grid_matches(c, d.nx1, d.nx2, d.nx3)) return fail(FVM_E_INVALID, "closure: grid size differs");
    if (!(beta >= 0.0)) return fail(FVM_E_INVALID, "closure: beta must be >= 0");
    if (!h->closure_nswitch) {
      FVM_CK(cudaMalloc(&h->closure_nswitch, sizeof(unsigned long long)));
    }
    FVM_CK(cudaMemset(h->closure_nswitch, 0, sizeof(unsigned long long)));
  }
  FVM_CK(cudaStreamSynchronize(h->stream));
  for (auto& g : h->graph)
    if (g) { cudaGraphExecDestroy(g); g = nullptr; }
  h->closure = c;
  h->closure_beta = beta;
  return FVM_OK;
}

int fvm_closure_switch_count(fvm_handle* h, unsigned long long* out) {
  if (!h || !out) return fail(FVM_E_INVALID, "null argument");
  *out = 0;
  if (!h->closure_nswitch) return FVM_OK;
  FVM_CK(cudaStreamSynchronize(h->stream));
  FVM_CK(cudaMemcpy(out, h->closure_nswitch, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return FVM_OK;
}

int fvm_filter_state(fvm_handle* h, int factor, float* coarse_dense_dev) {
  if (!h || !coarse_dense_dev) return fail(FVM_E_INVALID, "null argument");
  if (h->f64) return fail(FVM_E_INVALID, "filter: float32 handles only");
  const Layout& L = h->lay;
  if (factor < 1 || L.nx % factor || L.ny % factor || L.nz % factor)
    return fail(FVM_E_INVALID, "filter: factor must divide every grid dimension");
  FVM_CK(closure::launch_box_filter(static_cast<const float*>(h->U[0]), L, h->nv, factor, coarse_dense_dev, h->nsm,
                                    h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

static int dense_copy(fvm_handle* h, float* dense, int to_state) {
  if (!h || !dense) return fail(FVM_E_INVALID, "null argument");
  if (h->f64) return fail(FVM_E_INVALID, "dense copy: float32 handles only");
  FVM_CK(cudaStreamSynchronize(h->stream));
  FVM_CK(closure::launch_dense_copy(static_cast<float*>(h->U[0]), h->lay, h->nv, dense, to_state, h->nsm, h->stream));
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}

int fvm_upload_dense(fvm_handle* h, const float* dense_dev) { return dense_copy(h, const_cast<float*>(dense_dev), 1); }
int fvm_download_dense(fvm_handle* h, float* dense_dev) { return dense_copy(h, dense_dev, 0); }

}  // extern "C"

// ------------------------------------------------------ device initial state ----
extern "C" int fvm_init_kelvin_helmholtz(fvm_handle* h, const double params[9], unsigned long long seed) {
  if (!h || !params) return fail(FVM_E_INVALID, "null argument");
  if (h->d.physics != FVM_NAVIER_STOKES) return fail(FVM_E_INVALID, "Kelvin-Helmholtz state: navier_stokes only");
  KhInit k{};
  k.rho_in = params[0];
  k.rho_out = params[1];
  k.shear = params[2];
  k.pres = params[3];
  k.amp = params[4];
  k.wavenumber = params[5];
  k.noise = params[6];
  k.phase = params[7];
  k.noise_all = params[8] != 0.0;
  k.gamma = h->d.params[0];
  k.x1_min = h->d.x1_min;
  k.dx1 = (h->d.x1_max - h->d.x1_min) / h->d.nx1;
  k.x2_min = h->d.x2_min;
  k.dx2 = (h->d.x2_max - h->d.x2_min) / h->d.nx2;
  k.seed = seed;
  FVM_CK(cudaStreamSynchronize(h->stream));
  if (h->f64) kh_init_kernel<double><<<4 * h->nsm, 256, 0, h->stream>>>(static_cast<double*>(h->U[0]), h->lay, k);
  else kh_init_kernel<float><<<4 * h->nsm, 256, 0, h->stream>>>(static_cast<float*>(h->U[0]), h->lay, k);
  FVM_CK(cudaGetLastError());
  FVM_CK(cudaStreamSynchronize(h->stream));
  return FVM_OK;
}
