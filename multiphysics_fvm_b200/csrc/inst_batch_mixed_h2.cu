// Explicit instantiation: mixed navier_stokes + heat batch kernels (float32),
// 2-row heat strips (10-row heat tiles).
#include "launch.cuh"
namespace fvm {
cudaError_t launch_mixed_h2(int lim, int riem, int hcoord, const MixedSource& src, long long ntiles, int nbuf,
                            cudaStream_t s, int nsm) {
#define FVM_MIX_CASE(L, R, CO) \
  if (lim == L && riem == R && hcoord == CO) return launch_mixed_lrc<L, R, CO, 2>(src, ntiles, nbuf, s, nsm);
#define FVM_MIX_COORDS(L, R) FVM_MIX_CASE(L, R, COORD_CART) FVM_MIX_CASE(L, R, COORD_CYL) FVM_MIX_CASE(L, R, COORD_SPH)
  FVM_MIX_COORDS(LIM_PC, RIEM_RUSANOV)
  FVM_MIX_COORDS(LIM_PC, RIEM_HLL)
  FVM_MIX_COORDS(LIM_MINMOD, RIEM_RUSANOV)
  FVM_MIX_COORDS(LIM_MINMOD, RIEM_HLL)
  FVM_MIX_COORDS(LIM_MC, RIEM_RUSANOV)
  FVM_MIX_COORDS(LIM_MC, RIEM_HLL)
  FVM_MIX_COORDS(LIM_VANLEER, RIEM_RUSANOV)
  FVM_MIX_COORDS(LIM_VANLEER, RIEM_HLL)
#undef FVM_MIX_COORDS
#undef FVM_MIX_CASE
  return cudaErrorInvalidValue;
}
}  // namespace fvm
