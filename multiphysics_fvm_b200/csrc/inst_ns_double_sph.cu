// Explicit instantiation: Navier-Stokes stage kernels, double, COORD_SPH.
#include "launch.cuh"
namespace fvm {
template cudaError_t launch_ns_coord<double, COORD_SPH>(int, int, bool, const CUtensorMap&, const NsParams<double>&,
                                                     cudaStream_t, int, int);
template cudaError_t launch_ns_batch_coord<double, COORD_SPH>(int, int, bool, const BatchSource<NsParams<double>>&, long long,
                                                           cudaStream_t, int);
}
