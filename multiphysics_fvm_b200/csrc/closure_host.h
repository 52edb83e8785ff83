// Internal interface between the solver handle code and the closure code.
#pragma once
#include <string>
#include "fvm_common.cuh"

struct fvm_closure;

namespace fvm {
// Records `msg` as the calling thread's last error and returns `code`.
int set_error(int code, const std::string& msg);

namespace closure {
bool grid_matches(const fvm_closure* c, int nx, int ny, int nz);
// Features of the state `u` (solver layout) and the forward pass into Z3.
cudaError_t enqueue_infer(fvm_closure* c, const float* u, const Layout& lay, float gamma, cudaStream_t s);
// f^3 box filter of a float32 state into a dense coarse array.
cudaError_t launch_box_filter(const float* u, const Layout& lay, int nv, int f, float* out, int nsm, cudaStream_t s);
cudaError_t launch_dense_copy(float* u, const Layout& lay, int nv, float* dense, int to_state, int nsm,
                              cudaStream_t s);
// Correction of one stage (see closure_fix_kernel).
cudaError_t enqueue_fix(fvm_closure* c, const float* uin, float* uout, const Layout& lay, float gamma, float coef,
                        float beta, const double h[3], const Clock* clk, unsigned long long* nswitch,
                        cudaStream_t s);
}  // namespace closure
}  // namespace fvm
