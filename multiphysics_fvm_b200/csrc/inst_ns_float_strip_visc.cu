// Explicit instantiation: register-blocked float32 cartesian viscous Navier-Stokes stage kernels.
#include "launch.cuh"
namespace fvm {
cudaError_t launch_ns_strip_visc(int lim, int riem, NsStripSource& src, int ty, int nbuf, cudaStream_t s, int nsm) {
#define FVM_STRIP_CASE(L, R) \
  if (lim == L && riem == R) return launch_ns_strip_visc_lr<L, R>(src, ty, nbuf, s, nsm);
  FVM_STRIP_CASE(LIM_PC, RIEM_RUSANOV)
  FVM_STRIP_CASE(LIM_PC, RIEM_HLL)
  FVM_STRIP_CASE(LIM_MINMOD, RIEM_RUSANOV)
  FVM_STRIP_CASE(LIM_MINMOD, RIEM_HLL)
  FVM_STRIP_CASE(LIM_MC, RIEM_RUSANOV)
  FVM_STRIP_CASE(LIM_MC, RIEM_HLL)
  FVM_STRIP_CASE(LIM_VANLEER, RIEM_RUSANOV)
  FVM_STRIP_CASE(LIM_VANLEER, RIEM_HLL)
#undef FVM_STRIP_CASE
  return cudaErrorInvalidValue;
}
}  // namespace fvm
