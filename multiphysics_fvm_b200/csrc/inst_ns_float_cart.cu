// Explicit instantiation: Navier-Stokes stage kernels, float, COORD_CART.
#include "launch.cuh"
namespace fvm {
template cudaError_t launch_ns_coord<float, COORD_CART>(int, int, bool, const CUtensorMap&, const NsParams<float>&,
                                                     cudaStream_t, int, int);
template cudaError_t launch_ns_batch_coord<float, COORD_CART>(int, int, bool, const BatchSource<NsParams<float>>&, long long,
                                                           cudaStream_t, int);
}
