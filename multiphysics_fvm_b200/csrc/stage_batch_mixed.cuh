// One persistent launch per stage for a batch of float32 grids of two kinds:
// inviscid cartesian Navier-Stokes (the register-blocked body of
// stage_ns_strip.cuh, 8-row tiles) and piecewise-constant heat (the body of
// stage_heat_pc.cuh, 20-row tiles).  A flat work-list of tiles over all grids
// drives the launch; a block finds its grid by binary search over the tile
// offsets and runs that grid's body on the tile, with the grid's own
// parameters (stage coefficients, time step, clock) and tensor maps.  Both
// bodies use 160 threads and share the block's mbarriers: ring barriers 0..5
// (Navier-Stokes uses 0..2) and the Navier-Stokes staged-tile barrier 6, so
// each barrier's phase is tracked by the same threads across tiles of either
// kind.
#pragma once
#include "stage_ns_strip.cuh"
#include "stage_heat_pc.cuh"

namespace fvm {

constexpr int MIX_NS_R = 2, MIX_NS_NW = 4;  // Navier-Stokes: 2-row strips, 8-row tiles
constexpr int MIX_HEAT_NW = 5;              // heat: 4-row strips (20-row tiles) or 2-row (10-row tiles)
constexpr int MIX_NT = 160;
constexpr int MIX_NBAR = 7;
constexpr int MIX_NS_TY = MIX_NS_R * MIX_NS_NW, MIX_HEAT_TY = 4 * MIX_HEAT_NW, MIX_HEAT_TY_ALT = 2 * MIX_HEAT_NW;
static_assert(NsStripCfg<MIX_NS_R, MIX_NS_NW>::NT == MIX_NT && HeatPcCfg<4, MIX_HEAT_NW>::NT == MIX_NT,
              "both bodies run on the same block");

// Shared memory of a launch with `nbuf` staged Navier-Stokes tiles: the larger
// body, then the barriers.
__host__ __device__ constexpr int mixed_bar_offset(int nbuf) {
  return round_up(cmax(NsStripCfg<MIX_NS_R, MIX_NS_NW>::bytes(nbuf),
                       HeatPcCfg<4, MIX_HEAT_NW>::NSLOT * HeatPcCfg<4, MIX_HEAT_NW>::SLOT * 4),
                  8);
}
__host__ __device__ constexpr int mixed_bytes(int nbuf) { return mixed_bar_offset(nbuf) + MIX_NBAR * 8; }

// Per grid and stage: what a tile of that grid needs.
struct alignas(64) MixedInst {
  CUtensorMap tmap;    // ring map of the stage input
  CUtensorMap u0map;   // staged U0 tile (Navier-Stokes)
  CUtensorMap accmap;  // staged accumulator tile (Navier-Stokes)
  NsParams<float> ns;
  HeatParams<float> heat;
  int kind;  // 0 Navier-Stokes, 1 heat
};

struct MixedSource {
  const MixedInst* inst;  // per grid, this stage
  const int* tile_start;  // ninst + 1 prefix sums of tiles
  int ninst;
  int bar_off;            // byte offset of the barriers in shared memory
};

// HR: heat rows per strip (4: 20-row heat tiles, 2: 10-row).
template <int LIM, int RIEM, int HCOORD, int HR>
__global__ void __launch_bounds__(MIX_NT, 3) batch_mixed_kernel(const __grid_constant__ MixedSource src) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + src.bar_off);
  const int tid = threadIdx.x;
  if (smem_u32(smem_raw) & 127u) {  // TMA destinations need 128-byte alignment
    if (tid == 0) {
      const MixedInst& in = src.inst[0];
      atomicOr(in.kind == 0 ? in.ns.status : in.heat.status, ST_TMA_TIMEOUT);
    }
    return;
  }
  if (tid == 0) {
    for (int s = 0; s < MIX_NBAR; ++s) mbar_init(&bars[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  unsigned phase_bits = 0, pending = 0;
  const int ntiles = __ldg(src.tile_start + src.ninst);
  bool ok = true;
  for (int gtile = blockIdx.x; gtile < ntiles; gtile += gridDim.x) {
    int lo = 0, hi = src.ninst - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(src.tile_start + mid) <= gtile) lo = mid;
      else hi = mid - 1;
    }
    const MixedInst& in = src.inst[lo];
    const int tile = gtile - __ldg(src.tile_start + lo);
    if (in.kind == 0) {
      if (in.ns.active && !*in.ns.active) continue;  // this grid's clock passed t_end
      if (!ns_strip_tile<LIM, RIEM, MIX_NS_R, MIX_NS_NW>(in.ns, &in.tmap, &in.u0map, &in.accmap, tile, smem_raw,
                                                         bars, bars + 6, 6, phase_bits, pending)) {
        ok = false;
        break;
      }
    } else {
      if (in.heat.active && !*in.heat.active) continue;
      if (!heat_pc_tile<HCOORD, HR, MIX_HEAT_NW, true>(in.heat, &in.tmap, tile, smem_raw, bars, phase_bits, pending)) {
        ok = false;
        break;
      }
    }
  }
  // On a timeout, wait (bounded) for every copy this block may still have in flight.
  if (!ok && tid == 0) {
    const MixedInst& in = src.inst[0];
    const unsigned long long lim = in.kind == 0 ? in.ns.drain_ns : in.heat.drain_ns;
    for (int s = 0; s < MIX_NBAR; ++s)
      if ((pending >> s) & 1u) mbar_wait_bounded(&bars[s], (phase_bits >> s) & 1u, lim);
  }
}

}  // namespace fvm
