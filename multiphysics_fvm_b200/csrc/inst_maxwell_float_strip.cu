// Explicit instantiation: register-blocked float32 Maxwell stage kernels.
#include "launch.cuh"
namespace fvm {
cudaError_t launch_mx_strip(int lim, int coord, MxStripSource& src, int ty, int nbuf, cudaStream_t s, int nsm) {
  MaxwellParams<float>& p = src.p;
  p.ntx = (p.lay.nx + 31) / 32;
  p.nty = (p.lay.ny + ty - 1) / ty;
  p.nzc = (p.lay.nz + p.zchunk - 1) / p.zchunk;
#define FVM_MX_CASE(L, CO)                                                                          \
  if (lim == L && coord == CO)                                                                      \
    return ty == MX_STRIP_TY_ALT ? launch_mx_strip_ty<L, CO, MX_STRIP_TY_ALT>(src, nbuf, s, nsm)   \
                                 : launch_mx_strip_ty<L, CO, MX_STRIP_TY>(src, nbuf, s, nsm);
#define FVM_MX_COORDS(L) FVM_MX_CASE(L, COORD_CART) FVM_MX_CASE(L, COORD_CYL) FVM_MX_CASE(L, COORD_SPH)
  FVM_MX_COORDS(LIM_PC)
  FVM_MX_COORDS(LIM_MINMOD)
  FVM_MX_COORDS(LIM_MC)
  FVM_MX_COORDS(LIM_VANLEER)
#undef FVM_MX_COORDS
#undef FVM_MX_CASE
  return cudaErrorInvalidValue;
}
}  // namespace fvm
