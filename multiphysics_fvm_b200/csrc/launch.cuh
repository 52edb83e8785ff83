// Launch helpers for the fused stage kernels: persistent grids sized from the
// occupancy of each instantiation, runtime dispatch over the scheme enums.
#pragma once
#include <type_traits>
#include "stage_ns.cuh"
#include "stage_ns_strip.cuh"
#include "stage_ns_strip_visc.cuh"
#include "stage_heat.cuh"
#include "stage_heat_pc.cuh"
#include "stage_batch_mixed.cuh"
#include "stage_maxwell.cuh"
#include "stage_maxwell_strip.cuh"

namespace fvm {

// Tile rows of the Navier-Stokes kernel and the blocks per SM it is built
// for: float32 viscous 6 rows (2 blocks of 256 threads, ~109 KB each),
// float32 inviscid 8 rows (2 blocks), float64 viscous 4 rows, inviscid 8.
template <typename Real, bool VISC>
constexpr int ns_tile_ty() { return std::is_same<Real, double>::value ? (VISC ? 4 : 8) : (VISC ? 6 : 8); }
// The float32 kernels also come with 4-row tiles (a second block shape for
// the autotuner: fewer threads and less shared memory per block, more halo
// per cell); float64 has the default shape only.
template <typename Real, bool VISC>
constexpr int ns_tile_ty_alt() { return std::is_same<Real, double>::value ? ns_tile_ty<Real, VISC>() : 4; }
template <typename Real, bool VISC, int TY = ns_tile_ty<Real, VISC>()>
constexpr int ns_min_blocks() {
  return std::is_same<Real, double>::value ? 1 : (VISC ? 2 : (TY == 8 ? 3 : 4));
}
constexpr int HEAT_TY = 8, HEAT_TY_ALT = 4;

template <typename K>
static cudaError_t prepare_kernel(K kern, int threads, int bytes, int* blocks_per_sm) {
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e != cudaSuccess) return e;
  // all of the unified L1/shared array as shared memory: the ring planes are
  // the blocks' working set, so more resident blocks beat a larger L1
  e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, threads, bytes);
  if (e != cudaSuccess) return e;
  if (*blocks_per_sm < 1) return cudaErrorInvalidConfiguration;
  return cudaSuccess;
}

// nsm < 0: only set the kernel's shared-memory attribute and query its
// occupancy (done once, outside any stream capture).
template <typename Real, int LIM, int RIEM, int COORD, bool VISC, class Src, int TY = ns_tile_ty<Real, VISC>()>
cudaError_t launch_ns_src(const Src& src, long long ntiles, cudaStream_t s, int nsm) {
  using C = NsCfg<Real, VISC, TY>;
  auto kern = ns_stage_kernel<Real, LIM, RIEM, COORD, VISC, TY, ns_min_blocks<Real, VISC, TY>(), Src>;
  static int bps = 0;
  if (bps == 0 || nsm < 0) {
    cudaError_t e = prepare_kernel(kern, C::NT, C::BYTES, &bps);
    if (e != cudaSuccess) return e;
  }
  if (nsm < 0) return cudaSuccess;
  if (ntiles <= 0) return cudaSuccess;
  const int grid = (int)(ntiles < (long long)bps * nsm ? ntiles : (long long)bps * nsm);
  kern<<<grid, C::NT, C::BYTES, s>>>(src);
  return cudaGetLastError();
}

template <typename Real, bool VISC>
void ns_tile_counts(NsParams<Real>& p, int ty = ns_tile_ty<Real, VISC>()) {
  p.ntx = (p.lay.nx + 31) / 32;
  p.nty = (p.lay.ny + ty - 1) / ty;
  p.nzc = p.flat ? 1 : (p.lay.nz + p.zchunk - 1) / p.zchunk;
}

// ty: tile rows of the handle (its tensor maps were built for it).
template <typename Real, int LIM, int RIEM, int COORD, bool VISC>
cudaError_t launch_ns_one(const CUtensorMap& map, NsParams<Real> p, cudaStream_t s, int nsm, int ty) {
  constexpr int TD = ns_tile_ty<Real, VISC>(), TA = ns_tile_ty_alt<Real, VISC>();
  SingleSource<NsParams<Real>> src;
  src.tmap = map;
  if constexpr (TA != TD) {
    if (ty == TA) {
      ns_tile_counts<Real, VISC>(p, TA);
      src.p = p;
      return launch_ns_src<Real, LIM, RIEM, COORD, VISC, SingleSource<NsParams<Real>>, TA>(
          src, (long long)p.ntx * p.nty * p.nzc, s, nsm);
    }
  }
  ns_tile_counts<Real, VISC>(p, TD);
  src.p = p;
  return launch_ns_src<Real, LIM, RIEM, COORD, VISC>(src, (long long)p.ntx * p.nty * p.nzc, s, nsm);
}

template <typename Real, int COORD>
cudaError_t launch_ns_coord(int lim, int riem, bool visc, const CUtensorMap& map, const NsParams<Real>& p,
                            cudaStream_t s, int nsm, int ty) {
#define FVM_NS_CASE(L, R)                                                          \
  if (lim == L && riem == R)                                                       \
    return visc ? launch_ns_one<Real, L, R, COORD, true>(map, p, s, nsm, ty)       \
                : launch_ns_one<Real, L, R, COORD, false>(map, p, s, nsm, ty);
  FVM_NS_CASE(LIM_PC, RIEM_RUSANOV)
  FVM_NS_CASE(LIM_PC, RIEM_HLL)
  FVM_NS_CASE(LIM_MINMOD, RIEM_RUSANOV)
  FVM_NS_CASE(LIM_MINMOD, RIEM_HLL)
  FVM_NS_CASE(LIM_MC, RIEM_RUSANOV)
  FVM_NS_CASE(LIM_MC, RIEM_HLL)
  FVM_NS_CASE(LIM_VANLEER, RIEM_RUSANOV)
  FVM_NS_CASE(LIM_VANLEER, RIEM_HLL)
#undef FVM_NS_CASE
  return cudaErrorInvalidValue;
}

// Batched launch: every instance shares the kernel specialisation; the tile
// counts of each instance's params must already be filled in.
template <typename Real, int COORD>
cudaError_t launch_ns_batch_coord(int lim, int riem, bool visc, const BatchSource<NsParams<Real>>& src,
                                  long long ntiles, cudaStream_t s, int nsm) {
#define FVM_NS_CASE(L, R)                                                                                \
  if (lim == L && riem == R)                                                                             \
    return visc ? launch_ns_src<Real, L, R, COORD, true>(src, ntiles, s, nsm)                            \
                : launch_ns_src<Real, L, R, COORD, false>(src, ntiles, s, nsm);
  FVM_NS_CASE(LIM_PC, RIEM_RUSANOV)
  FVM_NS_CASE(LIM_PC, RIEM_HLL)
  FVM_NS_CASE(LIM_MINMOD, RIEM_RUSANOV)
  FVM_NS_CASE(LIM_MINMOD, RIEM_HLL)
  FVM_NS_CASE(LIM_MC, RIEM_RUSANOV)
  FVM_NS_CASE(LIM_MC, RIEM_HLL)
  FVM_NS_CASE(LIM_VANLEER, RIEM_RUSANOV)
  FVM_NS_CASE(LIM_VANLEER, RIEM_HLL)
#undef FVM_NS_CASE
  return cudaErrorInvalidValue;
}

// Declarations of the per-(precision, coordinate) instantiations.
#define FVM_DECLARE_NS(REAL, COORD)                                                                      \
  extern template cudaError_t launch_ns_coord<REAL, COORD>(int, int, bool, const CUtensorMap&,          \
                                                          const NsParams<REAL>&, cudaStream_t, int, int); \
  extern template cudaError_t launch_ns_batch_coord<REAL, COORD>(                                        \
      int, int, bool, const BatchSource<NsParams<REAL>>&, long long, cudaStream_t, int);
FVM_DECLARE_NS(float, COORD_CART)
FVM_DECLARE_NS(float, COORD_CYL)
FVM_DECLARE_NS(float, COORD_SPH)
FVM_DECLARE_NS(double, COORD_CART)
FVM_DECLARE_NS(double, COORD_CYL)
FVM_DECLARE_NS(double, COORD_SPH)

template <typename Real>
cudaError_t launch_ns_batch(int lim, int riem, int coord, bool visc, const BatchSource<NsParams<Real>>& src,
                            long long ntiles, cudaStream_t s, int nsm) {
  if (coord == COORD_CART) return launch_ns_batch_coord<Real, COORD_CART>(lim, riem, visc, src, ntiles, s, nsm);
  if (coord == COORD_CYL) return launch_ns_batch_coord<Real, COORD_CYL>(lim, riem, visc, src, ntiles, s, nsm);
  return launch_ns_batch_coord<Real, COORD_SPH>(lim, riem, visc, src, ntiles, s, nsm);
}

template <typename Real>
cudaError_t launch_ns(int lim, int riem, int coord, bool visc, const CUtensorMap& map, const NsParams<Real>& p,
                      cudaStream_t s, int nsm, int ty) {
  if (coord == COORD_CART) return launch_ns_coord<Real, COORD_CART>(lim, riem, visc, map, p, s, nsm, ty);
  if (coord == COORD_CYL) return launch_ns_coord<Real, COORD_CYL>(lim, riem, visc, map, p, s, nsm, ty);
  return launch_ns_coord<Real, COORD_SPH>(lim, riem, visc, map, p, s, nsm, ty);
}

// ------------------------------------------------ float32 cartesian NS ----
// Register-blocked stage kernel (stage_ns_strip.cuh) for float32 inviscid
// cartesian grids, 2 rows per thread: TY = 8 (4 output warps, 3 blocks/SM at
// 128 registers) or 16 (8 output warps, 2 blocks/SM).
constexpr int NS_STRIP_TY = 8, NS_STRIP_TY_ALT = 16;

template <int LIM, int RIEM, int TY>
cudaError_t launch_ns_strip_ty(const NsStripSource& src, int nbuf, cudaStream_t s, int nsm) {
  constexpr int R = 2, NW = TY / R;
  using C = NsStripCfg<R, NW>;
  auto kern = ns_strip_kernel<LIM, RIEM, R, NW, TY == 8 ? 3 : 2>;
  static int bps[3] = {0, 0, 0};
  if (bps[0] == 0 || nsm < 0) {
    // occupancy with 0, 1 and 2 staged tiles; the attribute ends at the largest
    for (int nb = 0; nb < 3; ++nb) {
      cudaError_t e = prepare_kernel(kern, C::NT, C::bytes(nb), &bps[nb]);
      if (e != cudaSuccess) return e;
    }
  }
  if (nsm < 0) return cudaSuccess;
  const long long ntiles = (long long)src.p.ntx * src.p.nty * src.p.nzc;
  if (ntiles <= 0) return cudaSuccess;
  const int grid = (int)(ntiles < (long long)bps[nbuf] * nsm ? ntiles : (long long)bps[nbuf] * nsm);
  kern<<<grid, C::NT, C::bytes(nbuf), s>>>(src);
  return cudaGetLastError();
}

// Row tiles a flat tile marches over along x2 (stage_ns_strip.cuh).
constexpr int NS_FLAT_YSUB = 4;
// Tile counts of the register-blocked kernel for block rows ty.
inline void ns_strip_tiles(NsParams<float>& p, int ty) {
  p.ntx = (p.lay.nx + 31) / 32;
  p.ysub = p.flat ? NS_FLAT_YSUB : 1;
  p.nty = ((p.lay.ny + ty - 1) / ty + p.ysub - 1) / p.ysub;
  p.nzc = (p.lay.nz + p.zchunk - 1) / p.zchunk;
}

template <int LIM, int RIEM>
cudaError_t launch_ns_strip_lr(NsStripSource& src, int ty, int nbuf, cudaStream_t s, int nsm) {
  NsParams<float>& p = src.p;
  ns_strip_tiles(p, ty);
  if (ty == NS_STRIP_TY_ALT) return launch_ns_strip_ty<LIM, RIEM, NS_STRIP_TY_ALT>(src, nbuf, s, nsm);
  return launch_ns_strip_ty<LIM, RIEM, NS_STRIP_TY>(src, nbuf, s, nsm);
}

cudaError_t launch_ns_strip(int lim, int riem, NsStripSource& src, int ty, int nbuf, cudaStream_t s, int nsm);

// Viscous float32 cartesian grids (stage_ns_strip_visc.cuh): 1 row per
// thread, TY = 7 (7 output warps + the halo warp, 2 blocks/SM: 16 warps per SM,
// 4 per scheduler, fit 128 registers without spills; 8 output warps left 96
// registers and spilled, 2-row strips held 168 and ran 8 warps per SM).  It is
// these grids' default block shape; the second one runs the general kernel
// (stage_ns.cuh).
constexpr int NS_STRIP_VISC_TY = 7;

template <int LIM, int RIEM, int TY>
cudaError_t launch_ns_strip_visc_ty(const NsStripSource& src, int nbuf, cudaStream_t s, int nsm) {
  constexpr int R = 1, NW = TY / R;
  using C = NsStripViscCfg<R, NW>;
  auto kern = ns_strip_visc_kernel<LIM, RIEM, R, NW, 2>;
  static int bps[3] = {0, 0, 0};
  if (bps[0] == 0 || nsm < 0) {
    for (int nb = 0; nb < 3; ++nb) {
      cudaError_t e = prepare_kernel(kern, C::NT, C::bytes(nb), &bps[nb]);
      if (e != cudaSuccess) return e;
    }
  }
  if (nsm < 0) return cudaSuccess;
  const long long ntiles = (long long)src.p.ntx * src.p.nty * src.p.nzc;
  if (ntiles <= 0) return cudaSuccess;
  const int grid = (int)(ntiles < (long long)bps[nbuf] * nsm ? ntiles : (long long)bps[nbuf] * nsm);
  kern<<<grid, C::NT, C::bytes(nbuf), s>>>(src);
  return cudaGetLastError();
}

template <int LIM, int RIEM>
cudaError_t launch_ns_strip_visc_lr(NsStripSource& src, int ty, int nbuf, cudaStream_t s, int nsm) {
  NsParams<float>& p = src.p;
  p.ntx = (p.lay.nx + 31) / 32;
  p.nty = (p.lay.ny + ty - 1) / ty;
  p.nzc = (p.lay.nz + p.zchunk - 1) / p.zchunk;
  (void)ty;
  return launch_ns_strip_visc_ty<LIM, RIEM, NS_STRIP_VISC_TY>(src, nbuf, s, nsm);
}

cudaError_t launch_ns_strip_visc(int lim, int riem, NsStripSource& src, int ty, int nbuf, cudaStream_t s, int nsm);

// ---------------------------------------------------------------- heat ----
template <typename Real, int LIM, int COORD, class Src, int TY = HEAT_TY>
cudaError_t launch_heat_src(const Src& src, long long ntiles, cudaStream_t s, int nsm) {
  using C = HeatCfg<Real, LIM, TY>;
  auto kern = heat_stage_kernel<Real, LIM, COORD, TY, Src>;
  static int bps = 0;
  if (bps == 0 || nsm < 0) {
    cudaError_t e = prepare_kernel(kern, C::NT, C::BYTES, &bps);
    if (e != cudaSuccess) return e;
  }
  if (nsm < 0 || ntiles <= 0) return cudaSuccess;
  const int grid = (int)(ntiles < (long long)bps * nsm ? ntiles : (long long)bps * nsm);
  kern<<<grid, C::NT, C::BYTES, s>>>(src);
  return cudaGetLastError();
}

template <typename Real>
void heat_tile_counts(HeatParams<Real>& p, int ty = HEAT_TY) {
  p.ntx = (p.lay.nx + 31) / 32;
  p.nty = (p.lay.ny + ty - 1) / ty;
  p.nzc = (p.lay.nz + p.zchunk - 1) / p.zchunk;
}

template <typename Real, class Src, int TY = HEAT_TY>
cudaError_t launch_heat_any(int lim, int coord, const Src& src, long long ntiles, cudaStream_t s, int nsm) {
#define FVM_HEAT_CASE(L)                                                                               \
  if (lim == L) {                                                                                      \
    if (coord == COORD_CART) return launch_heat_src<Real, L, COORD_CART, Src, TY>(src, ntiles, s, nsm); \
    if (coord == COORD_CYL) return launch_heat_src<Real, L, COORD_CYL, Src, TY>(src, ntiles, s, nsm);   \
    return launch_heat_src<Real, L, COORD_SPH, Src, TY>(src, ntiles, s, nsm);                           \
  }
  FVM_HEAT_CASE(LIM_PC)
  FVM_HEAT_CASE(LIM_MINMOD)
  FVM_HEAT_CASE(LIM_MC)
  FVM_HEAT_CASE(LIM_VANLEER)
#undef FVM_HEAT_CASE
  return cudaErrorInvalidValue;
}

// Float32 piecewise-constant heat (stage_heat_pc.cuh): 4 rows per thread,
// TY = 16 (4 warps) or 8 (2 warps); mixed-batch members also run 20 (4 x 5
// warps) and 10 (2-row strips, 5 warps).
constexpr int HEAT_PC_TY = 16, HEAT_PC_TY_ALT = 8;

template <int COORD, int TY>
cudaError_t launch_heat_pc_ty(const CUtensorMap& map, const HeatParams<float>& p, cudaStream_t s, int nsm) {
  constexpr int R = TY % 4 == 0 ? 4 : 2, NW = TY / R;
  using C = HeatPcCfg<R, NW>;
  auto kern = heat_pc_kernel<COORD, R, NW>;
  static int bps = 0;
  if (bps == 0 || nsm < 0) {
    cudaError_t e = prepare_kernel(kern, C::NT, C::BYTES, &bps);
    if (e != cudaSuccess) return e;
  }
  if (nsm < 0) return cudaSuccess;
  const long long ntiles = (long long)p.ntx * p.nty * p.nzc;
  if (ntiles <= 0) return cudaSuccess;
  const int grid = (int)(ntiles < (long long)bps * nsm ? ntiles : (long long)bps * nsm);
  kern<<<grid, C::NT, C::BYTES, s>>>(map, p);
  return cudaGetLastError();
}

cudaError_t launch_heat_pc(int coord, const CUtensorMap& map, HeatParams<float> p, cudaStream_t s, int nsm, int ty);

// Mixed batch (stage_batch_mixed.cuh): navier_stokes (limiter, Riemann
// solver) and heat (coordinate system) tiles in one launch.
template <int LIM, int RIEM, int HCOORD, int HR>
cudaError_t launch_mixed_lrc(const MixedSource& src, long long ntiles, int nbuf, cudaStream_t s, int nsm) {
  auto kern = batch_mixed_kernel<LIM, RIEM, HCOORD, HR>;
  static int bps[3] = {0, 0, 0};
  if (bps[0] == 0 || nsm < 0) {
    for (int nb = 0; nb < 3; ++nb) {
      cudaError_t e = prepare_kernel(kern, MIX_NT, mixed_bytes(nb), &bps[nb]);
      if (e != cudaSuccess) return e;
    }
  }
  if (nsm < 0 || ntiles <= 0) return cudaSuccess;
  const int grid = (int)(ntiles < (long long)bps[nbuf] * nsm ? ntiles : (long long)bps[nbuf] * nsm);
  kern<<<grid, MIX_NT, mixed_bytes(nbuf), s>>>(src);
  return cudaGetLastError();
}
// heat_ty: the heat members' tile rows (MIX_HEAT_TY or MIX_HEAT_TY_ALT)
cudaError_t launch_mixed_h4(int lim, int riem, int hcoord, const MixedSource& src, long long ntiles, int nbuf,
                            cudaStream_t s, int nsm);
cudaError_t launch_mixed_h2(int lim, int riem, int hcoord, const MixedSource& src, long long ntiles, int nbuf,
                            cudaStream_t s, int nsm);
inline cudaError_t launch_mixed(int lim, int riem, int hcoord, int heat_ty, const MixedSource& src, long long ntiles,
                                int nbuf, cudaStream_t s, int nsm) {
  return heat_ty == MIX_HEAT_TY_ALT ? launch_mixed_h2(lim, riem, hcoord, src, ntiles, nbuf, s, nsm)
                                    : launch_mixed_h4(lim, riem, hcoord, src, ntiles, nbuf, s, nsm);
}

template <typename Real>
cudaError_t launch_heat(int lim, int coord, const CUtensorMap& map, const HeatParams<Real>& p0, cudaStream_t s,
                        int nsm, int ty) {
  HeatParams<Real> p = p0;
  SingleSource<HeatParams<Real>> src;
  src.tmap = map;
  if constexpr (std::is_same<Real, float>::value) {
    if (ty == HEAT_TY_ALT) {
      heat_tile_counts(p, HEAT_TY_ALT);
      src.p = p;
      return launch_heat_any<Real, SingleSource<HeatParams<Real>>, HEAT_TY_ALT>(
          lim, coord, src, (long long)p.ntx * p.nty * p.nzc, s, nsm);
    }
  }
  heat_tile_counts(p);
  src.p = p;
  return launch_heat_any<Real>(lim, coord, src, (long long)p.ntx * p.nty * p.nzc, s, nsm);
}
template <typename Real>
cudaError_t launch_heat_batch(int lim, int coord, const BatchSource<HeatParams<Real>>& src, long long ntiles,
                              cudaStream_t s, int nsm) {
  return launch_heat_any<Real>(lim, coord, src, ntiles, s, nsm);
}
extern template cudaError_t launch_heat<float>(int, int, const CUtensorMap&, const HeatParams<float>&, cudaStream_t, int,
                                              int);
extern template cudaError_t launch_heat<double>(int, int, const CUtensorMap&, const HeatParams<double>&, cudaStream_t,
                                               int, int);
extern template cudaError_t launch_heat_batch<float>(int, int, const BatchSource<HeatParams<float>>&, long long,
                                                     cudaStream_t, int);
extern template cudaError_t launch_heat_batch<double>(int, int, const BatchSource<HeatParams<double>>&, long long,
                                                      cudaStream_t, int);

// ------------------------------------------------------------- maxwell ----
// Maxwell: 6 rows x 32 columns, 2 blocks of 256 threads per SM (float32).
template <typename Real>
constexpr int maxwell_tile_ty() { return std::is_same<Real, double>::value ? 8 : 6; }

template <typename Real, int LIM, int RIEM, int COORD>
cudaError_t launch_maxwell_one(const CUtensorMap& map, MaxwellParams<Real> p, cudaStream_t s, int nsm) {
  constexpr int TY = maxwell_tile_ty<Real>();
  using C = MaxwellCfg<Real, TY>;
  auto kern = maxwell_stage_kernel<Real, LIM, RIEM, COORD, TY, std::is_same<Real, double>::value ? 1 : 3>;
  static int bps = 0;
  if (bps == 0 || nsm < 0) {
    cudaError_t e = prepare_kernel(kern, C::NT, C::BYTES, &bps);
    if (e != cudaSuccess) return e;
  }
  if (nsm < 0) return cudaSuccess;
  p.ntx = (p.lay.nx + C::TX - 1) / C::TX;
  p.nty = (p.lay.ny + TY - 1) / TY;
  p.nzc = (p.lay.nz + p.zchunk - 1) / p.zchunk;
  const long long ntiles = (long long)p.ntx * p.nty * p.nzc;
  const int grid = (int)(ntiles < (long long)bps * nsm ? ntiles : (long long)bps * nsm);
  kern<<<grid, C::NT, C::BYTES, s>>>(map, p);
  return cudaGetLastError();
}

template <typename Real, int COORD>
cudaError_t launch_maxwell_coord(int lim, int riem, const CUtensorMap& map, const MaxwellParams<Real>& p,
                                 cudaStream_t s, int nsm) {
#define FVM_MX_CASE(L)                                                                           \
  if (lim == L) return riem == RIEM_HLL ? launch_maxwell_one<Real, L, RIEM_HLL, COORD>(map, p, s, nsm) \
                                        : launch_maxwell_one<Real, L, RIEM_RUSANOV, COORD>(map, p, s, nsm);
  FVM_MX_CASE(LIM_PC)
  FVM_MX_CASE(LIM_MINMOD)
  FVM_MX_CASE(LIM_MC)
  FVM_MX_CASE(LIM_VANLEER)
#undef FVM_MX_CASE
  return cudaErrorInvalidValue;
}
#define FVM_DECLARE_MX(REAL, COORD)                                                                      \
  extern template cudaError_t launch_maxwell_coord<REAL, COORD>(int, int, const CUtensorMap&,           \
                                                               const MaxwellParams<REAL>&, cudaStream_t, int);
FVM_DECLARE_MX(float, COORD_CART)
FVM_DECLARE_MX(float, COORD_CYL)
FVM_DECLARE_MX(float, COORD_SPH)
FVM_DECLARE_MX(double, COORD_CART)
FVM_DECLARE_MX(double, COORD_CYL)
FVM_DECLARE_MX(double, COORD_SPH)

template <typename Real>
cudaError_t launch_maxwell(int lim, int riem, int coord, const CUtensorMap& map, const MaxwellParams<Real>& p,
                           cudaStream_t s, int nsm) {
  if (coord == COORD_CART) return launch_maxwell_coord<Real, COORD_CART>(lim, riem, map, p, s, nsm);
  if (coord == COORD_CYL) return launch_maxwell_coord<Real, COORD_CYL>(lim, riem, map, p, s, nsm);
  return launch_maxwell_coord<Real, COORD_SPH>(lim, riem, map, p, s, nsm);
}

// Float32 Maxwell (stage_maxwell_strip.cuh): TY = 8 (2 rows per thread, 4
// output warps) or 16 (4 rows per thread, 4 output warps).
constexpr int MX_STRIP_TY = 8, MX_STRIP_TY_ALT = 16;

template <int LIM, int COORD, int TY>
cudaError_t launch_mx_strip_ty(const MxStripSource& src, int nbuf, cudaStream_t s, int nsm) {
  constexpr int R = TY == 8 ? 2 : 4, NW = TY / R;
  using C = MxStripCfg<R, NW>;
  auto kern = mx_strip_kernel<LIM, COORD, R, NW, TY == 8 ? 3 : 2>;
  static int bps[3] = {0, 0, 0};
  if (bps[0] == 0 || nsm < 0) {
    for (int nb = 0; nb < 3; ++nb) {
      cudaError_t e = prepare_kernel(kern, C::NT, C::bytes(nb), &bps[nb]);
      if (e != cudaSuccess) return e;
    }
  }
  if (nsm < 0) return cudaSuccess;
  const long long ntiles = (long long)src.p.ntx * src.p.nty * src.p.nzc;
  if (ntiles <= 0) return cudaSuccess;
  const int grid = (int)(ntiles < (long long)bps[nbuf] * nsm ? ntiles : (long long)bps[nbuf] * nsm);
  kern<<<grid, C::NT, C::bytes(nbuf), s>>>(src);
  return cudaGetLastError();
}

cudaError_t launch_mx_strip(int lim, int coord, MxStripSource& src, int ty, int nbuf, cudaStream_t s, int nsm);

}  // namespace fvm

