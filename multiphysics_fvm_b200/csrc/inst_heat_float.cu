// Explicit instantiation: heat stage kernels, float, all limiters and coordinates.
#include "launch.cuh"
namespace fvm {
template cudaError_t launch_heat<float>(int, int, const CUtensorMap&, const HeatParams<float>&, cudaStream_t, int, int);
template cudaError_t launch_heat_batch<float>(int, int, const BatchSource<HeatParams<float>>&, long long, cudaStream_t,
                                                int);
}
