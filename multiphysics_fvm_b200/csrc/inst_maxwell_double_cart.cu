// Explicit instantiation: Maxwell stage kernels, double, COORD_CART.
#include "launch.cuh"
namespace fvm {
template cudaError_t launch_maxwell_coord<double, COORD_CART>(int, int, const CUtensorMap&, const MaxwellParams<double>&,
                                                          cudaStream_t, int);
}
