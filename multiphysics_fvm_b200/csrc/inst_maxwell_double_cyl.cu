// Explicit instantiation: Maxwell stage kernels, double, COORD_CYL.
#include "launch.cuh"
namespace fvm {
template cudaError_t launch_maxwell_coord<double, COORD_CYL>(int, int, const CUtensorMap&, const MaxwellParams<double>&,
                                                          cudaStream_t, int);
}
