// Explicit instantiation: heat stage kernels, double, all limiters and coordinates.
#include "launch.cuh"
namespace fvm {
template cudaError_t launch_heat<double>(int, int, const CUtensorMap&, const HeatParams<double>&, cudaStream_t, int, int);
template cudaError_t launch_heat_batch<double>(int, int, const BatchSource<HeatParams<double>>&, long long, cudaStream_t,
                                                int);
}
