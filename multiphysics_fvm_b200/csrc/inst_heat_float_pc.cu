// Explicit instantiation: float32 piecewise-constant heat stage kernels.
#include "launch.cuh"
namespace fvm {
cudaError_t launch_heat_pc(int coord, const CUtensorMap& map, HeatParams<float> p, cudaStream_t s, int nsm, int ty) {
  p.ntx = (p.lay.nx + 31) / 32;
  p.nty = (p.lay.ny + ty - 1) / ty;
  p.nzc = (p.lay.nz + p.zchunk - 1) / p.zchunk;
#define FVM_HEAT_PC_CASE(CO)                                                                     \
  if (coord == CO)                                                                               \
    return ty == HEAT_PC_TY_ALT    ? launch_heat_pc_ty<CO, HEAT_PC_TY_ALT>(map, p, s, nsm)     \
           : ty == MIX_HEAT_TY     ? launch_heat_pc_ty<CO, MIX_HEAT_TY>(map, p, s, nsm)        \
           : ty == MIX_HEAT_TY_ALT ? launch_heat_pc_ty<CO, MIX_HEAT_TY_ALT>(map, p, s, nsm)    \
                                   : launch_heat_pc_ty<CO, HEAT_PC_TY>(map, p, s, nsm);
  FVM_HEAT_PC_CASE(COORD_CART)
  FVM_HEAT_PC_CASE(COORD_CYL)
  FVM_HEAT_PC_CASE(COORD_SPH)
#undef FVM_HEAT_PC_CASE
  return cudaErrorInvalidValue;
}
}  // namespace fvm
