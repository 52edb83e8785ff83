// Explicit instantiation: Maxwell stage kernels, float, COORD_CYL.
#include "launch.cuh"
namespace fvm {
template cudaError_t launch_maxwell_coord<float, COORD_CYL>(int, int, const CUtensorMap&, const MaxwellParams<float>&,
                                                          cudaStream_t, int);
}
