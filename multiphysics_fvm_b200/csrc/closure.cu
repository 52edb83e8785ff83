// Learned flux-correction closure: host side of the C ABI (include/fvm_closure.h)
// and the launch sequences for inference, training and the solver hook.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fvm_closure.h"
#include "closure.cuh"
#include "closure_host.h"

using namespace fvm;
using namespace fvm::closure;

namespace {

constexpr int NLAYER = 3;
constexpr int LCOUT[NLAYER] = {C_HID, C_HID, C_OUT};
constexpr int LCIN[NLAYER] = {C_IN0, C_HID, C_HID};

#define CL_CK(x)                                                                                     \
  do {                                                                                               \
    cudaError_t e_ = (x);                                                                            \
    if (e_ != cudaSuccess) return set_error(FVM_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define CL_RET(x)                           \
  do {                                      \
    cudaError_t e_ = (x);                   \
    if (e_ != cudaSuccess) return e_;       \
  } while (0)

int largest_zc(int n3, long long ctas_xy, long long target) {
  // Smallest z-chunk (a divisor of n3) that keeps the grid at or below
  // `target` CTAs; at least one plane.
  for (int zc = 1; zc <= n3; ++zc)
    if (n3 % zc == 0 && ctas_xy * (n3 / zc) <= target) return zc;
  return n3;
}

}  // namespace

struct fvm_closure {
  int n1 = 0, n2 = 0, n3 = 0;
  long long npos = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  // workspace
  __nv_bfloat16 *x0 = nullptr, *a1 = nullptr, *a2 = nullptr, *g3 = nullptr, *g2 = nullptr, *g1 = nullptr;
  float *z3 = nullptr, *e = nullptr;
  // parameters per layer: master weights, bias, Adam moments, gradients, packs
  float *w[NLAYER] = {}, *b[NLAYER] = {}, *mw[NLAYER] = {}, *vw[NLAYER] = {}, *mb[NLAYER] = {}, *vb[NLAYER] = {};
  float *gw[NLAYER] = {}, *gb[NLAYER] = {};
  __nv_bfloat16 *pf[NLAYER] = {}, *pb[NLAYER] = {};
  float* partial = nullptr;  // wgrad / bias partial sums
  size_t partial_elems = 0;
  double* loss_part = nullptr;
  double* loss_dev = nullptr;
  int loss_blocks = 0;
  long long adam_step = 0;
  // normalisation
  float gamma = 1.4f;
  float in_mean[5] = {0, 0, 0, 0, 0}, in_inv_scale[5] = {1, 1, 1, 1, 1};
  float out_scale[5] = {1, 1, 1, 1, 1}, loss_w[5] = {1, 1, 1, 1, 1};
  int zc_conv = 1, zc_wg = 1;
  unsigned* status = nullptr;  // ST_TMA_TIMEOUT when a tensor-core wait gave up
  int fct = 0;                 // 1: flux-corrected transport bound on the corrections
  float* ratio = nullptr;      // FCT fractions [10][cells]
};

namespace {

size_t wcount(int l) { return (size_t)27 * LCOUT[l] * LCIN[l]; }

template <int CIN, int COUT>
constexpr int wgrad_smem() {
  // One CTA per SM: the accumulator block takes up to all of an SM's tensor
  // memory, so the launch asks for more than half of its shared memory.
  return WgCfg<CIN, COUT>::BYTES > 120 * 1024 ? WgCfg<CIN, COUT>::BYTES : 120 * 1024;
}

// Opt every tensor-core kernel into its dynamic shared memory once per
// process (before any graph capture).
cudaError_t set_attributes() {
  static bool done = false;
  if (done) return cudaSuccess;
  const auto A = cudaFuncAttributeMaxDynamicSharedMemorySize;
  CL_RET(cudaFuncSetAttribute(conv3_kernel<C_IN0, C_HID, EPI_RELU_BF16>, A, ConvCfg<C_IN0, C_HID>::BYTES));
  CL_RET(cudaFuncSetAttribute(conv3_kernel<C_HID, C_HID, EPI_RELU_BF16>, A, ConvCfg<C_HID, C_HID>::BYTES));
  CL_RET(cudaFuncSetAttribute(conv3_kernel<C_HID, C_OUT, EPI_LIN_F32>, A, ConvCfg<C_HID, C_OUT>::BYTES));
  CL_RET(cudaFuncSetAttribute(conv3_kernel<C_OUT, C_HID, EPI_MASK_BF16>, A, ConvCfg<C_OUT, C_HID>::BYTES));
  CL_RET(cudaFuncSetAttribute(conv3_kernel<C_HID, C_HID, EPI_MASK_BF16>, A, ConvCfg<C_HID, C_HID>::BYTES));
  CL_RET(cudaFuncSetAttribute(wgrad_kernel<C_HID, C_OUT>, A, wgrad_smem<C_HID, C_OUT>()));
  CL_RET(cudaFuncSetAttribute(wgrad_kernel<C_HID, C_HID>, A, wgrad_smem<C_HID, C_HID>()));
  CL_RET(cudaFuncSetAttribute(wgrad_kernel<C_IN0, C_HID>, A, wgrad_smem<C_IN0, C_HID>()));
  done = true;
  return cudaSuccess;
}

template <int CIN, int COUT, int EPI>
cudaError_t conv(fvm_closure* c, const __nv_bfloat16* x, const __nv_bfloat16* wpack, const float* bias, void* y,
                 const __nv_bfloat16* mask, cudaStream_t s) {
  using C = ConvCfg<CIN, COUT>;
  const ConvArgs a{x, wpack, bias, y, mask, c->n1, c->n2, c->n3, c->zc_conv, c->status};
  const dim3 grid(c->n1 / 8, c->n2 / 16, c->n3 / c->zc_conv);
  conv3_kernel<CIN, COUT, EPI><<<grid, 128, C::BYTES, s>>>(a);
  return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t wgrad(fvm_closure* c, const __nv_bfloat16* x, const __nv_bfloat16* g, float* dw, float* db,
                  cudaStream_t s) {
  using C = WgCfg<CIN, COUT>;
  const dim3 grid(c->n1 / C::TX, c->n2 / C::TY, c->n3 / c->zc_wg);
  const int nblk = grid.x * grid.y * grid.z;
  const WgradArgs a{x, g, c->partial, c->n1, c->n2, c->n3, c->zc_wg, c->status};
  wgrad_kernel<CIN, COUT><<<grid, 128, wgrad_smem<CIN, COUT>(), s>>>(a);
  CL_RET(cudaGetLastError());
  const int n = 27 * COUT * CIN;
  reduce_partials_kernel<<<(n + 255) / 256, 256, 0, s>>>(c->partial, nblk, n, dw);
  CL_RET(cudaGetLastError());
  // bias gradient
  const int cblk = 2 * c->nsm;
  float* cpart = c->partial + (size_t)nblk * n;
  channel_sum_kernel<COUT><<<cblk, 256, 0, s>>>(g, c->npos, cpart);
  CL_RET(cudaGetLastError());
  reduce_partials_kernel<<<1, 64, 0, s>>>(cpart, cblk, COUT, db);
  return cudaGetLastError();
}

cudaError_t forward(fvm_closure* c, cudaStream_t s) {
  CL_RET((conv<C_IN0, C_HID, EPI_RELU_BF16>(c, c->x0, c->pf[0], c->b[0], c->a1, nullptr, s)));
  CL_RET((conv<C_HID, C_HID, EPI_RELU_BF16>(c, c->a1, c->pf[1], c->b[1], c->a2, nullptr, s)));
  return conv<C_HID, C_OUT, EPI_LIN_F32>(c, c->a2, c->pf[2], c->b[2], c->z3, nullptr, s);
}

LossArgs loss_args(fvm_closure* c, const float* d, double dt, const double h[3]) {
  LossArgs a{};
  a.z3 = c->z3;
  a.d = d;
  a.e = c->e;
  a.g3 = c->g3;
  for (int q = 0; q < 5; ++q) {
    a.s[q] = c->out_scale[q];
    a.w[q] = c->loss_w[q];
  }
  for (int ax = 0; ax < 3; ++ax) a.coef[ax] = (float)(dt / h[ax]);
  a.inv_n = (float)(1.0 / (double)c->npos);
  a.partial = c->loss_part;
  a.n1 = c->n1;
  a.n2 = c->n2;
  a.n3 = c->n3;
  return a;
}

cudaError_t backward(fvm_closure* c, const float* d, double dt, const double h[3], cudaStream_t s) {
  const LossArgs la = loss_args(c, d, dt, h);
  loss_residual_kernel<<<c->loss_blocks, 256, 0, s>>>(la);
  CL_RET(cudaGetLastError());
  sum_partials_kernel<<<1, 256, 0, s>>>(c->loss_part, c->loss_blocks, c->loss_dev);
  CL_RET(cudaGetLastError());
  loss_grad_kernel<<<4 * c->nsm, 256, 0, s>>>(la);
  CL_RET(cudaGetLastError());
  // layer 3: X = A2 (32), G = G3 (16)
  CL_RET((wgrad<C_HID, C_OUT>(c, c->a2, c->g3, c->gw[2], c->gb[2], s)));
  CL_RET((conv<C_OUT, C_HID, EPI_MASK_BF16>(c, c->g3, c->pb[2], nullptr, c->g2, c->a2, s)));
  // layer 2
  CL_RET((wgrad<C_HID, C_HID>(c, c->a1, c->g2, c->gw[1], c->gb[1], s)));
  CL_RET((conv<C_HID, C_HID, EPI_MASK_BF16>(c, c->g2, c->pb[1], nullptr, c->g1, c->a1, s)));
  // layer 1
  return wgrad<C_IN0, C_HID>(c, c->x0, c->g1, c->gw[0], c->gb[0], s);
}

cudaError_t adam_all(fvm_closure* c, bool update, float lr, float b1, float b2, float eps, cudaStream_t s) {
  float c1 = 1.f, c2 = 1.f;
  if (update) {
    c->adam_step += 1;
    c1 = (float)(1.0 / (1.0 - std::pow((double)b1, (double)c->adam_step)));
    c2 = (float)(1.0 / (1.0 - std::pow((double)b2, (double)c->adam_step)));
  }
  for (int l = 0; l < NLAYER; ++l) {
    AdamLayer L{c->w[l], c->mw[l], c->vw[l], c->b[l], c->mb[l], c->vb[l], c->gw[l], c->gb[l],
                c->pf[l], l > 0 ? c->pb[l] : nullptr, LCOUT[l], LCIN[l]};
    const int n = (int)wcount(l) + LCOUT[l];
    adam_pack_kernel<<<(n + 255) / 256, 256, 0, s>>>(L, update ? 1 : 0, lr, b1, b2, eps, c1, c2);
    CL_RET(cudaGetLastError());
  }
  return cudaSuccess;
}

Layout dense_layout(int n1, int n2, int n3) {
  Layout L{};
  L.nx = n1;
  L.ny = n2;
  L.nz = n3;
  L.pitch = n1;
  L.plane = (long long)n1 * n2;
  L.var_stride = L.plane * n3;
  // idx(q, k+1, j+1, i+1) = q*var_stride + k*plane + j*pitch + i
  L.padx = -(int)(L.plane + L.pitch + 1);
  return L;
}

cudaError_t features(fvm_closure* c, const float* u, const Layout& lay, float gamma, cudaStream_t s) {
  FeatArgs a{};
  a.u = u;
  a.lay = lay;
  a.gamma = gamma;
  for (int q = 0; q < 5; ++q) {
    a.mean[q] = c->in_mean[q];
    a.inv_scale[q] = c->in_inv_scale[q];
  }
  a.x = c->x0;
  features_kernel<<<4 * c->nsm, 256, 0, s>>>(a);
  return cudaGetLastError();
}

FixArgs fix_args(fvm_closure* c, const float* uin, float* uout, const Layout& lay, float gamma, float coef,
                 float beta, const double h[3], const Clock* clk, float dt, unsigned long long* nswitch) {
  FixArgs a{};
  a.uin = uin;
  a.uout = uout;
  a.lay = lay;
  a.z3 = c->z3;
  for (int q = 0; q < 5; ++q) a.s[q] = c->out_scale[q];
  a.beta = beta;
  a.gamma = gamma;
  a.coef = coef;
  for (int ax = 0; ax < 3; ++ax) a.inv_h[ax] = (float)(1.0 / h[ax]);
  a.clk = clk;
  a.dt_host = dt;
  a.nswitch = nswitch;
  a.ratio = c->ratio;
  return a;
}

// The correction of one stage: clip-only, or the two FCT passes.
cudaError_t launch_fix(fvm_closure* c, const FixArgs& a, cudaStream_t s) {
  // one block of 128 threads per x1 row (for_each_cell)
  const int rows = a.lay.ny * a.lay.nz;
  if (c->fct) {
    fct_ratio_kernel<<<rows, 128, 0, s>>>(a);
    CL_RET(cudaGetLastError());
    fct_apply_kernel<<<rows, 128, 0, s>>>(a);
  } else {
    closure_fix_kernel<<<rows, 128, 0, s>>>(a);
  }
  return cudaGetLastError();
}

template <typename T>
int dalloc(T** p, size_t n) {
  if (cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return set_error(FVM_E_NOMEM, "closure: device allocation failed");
  }
  return FVM_OK;
}

void he_init(std::vector<float>& w, int cin, double scale, unsigned long long& state) {
  // splitmix64 + Box-Muller: deterministic across platforms
  auto next = [&]() {
    unsigned long long z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  const double sd = scale * std::sqrt(2.0 / (27.0 * cin));
  for (size_t i = 0; i < w.size(); i += 2) {
    const double u1 = ((next() >> 11) + 1.0) * (1.0 / 9007199254740993.0);
    const double u2 = (next() >> 11) * (1.0 / 9007199254740992.0);
    const double r = std::sqrt(-2.0 * std::log(u1));
    w[i] = (float)(sd * r * std::cos(6.283185307179586 * u2));
    if (i + 1 < w.size()) w[i + 1] = (float)(sd * r * std::sin(6.283185307179586 * u2));
  }
}

int check(const fvm_closure* c) { return c ? FVM_OK : set_error(FVM_E_INVALID, "null closure"); }

// Wait for the closure's stream and report a tensor-core wait that gave up.
int sync_status(fvm_closure* c) {
  CL_CK(cudaStreamSynchronize(c->stream));
  unsigned st = 0;
  CL_CK(cudaMemcpy(&st, c->status, sizeof(st), cudaMemcpyDeviceToHost));
  if (st) return set_error(FVM_E_STATE, "closure: a tensor-core wait timed out (status " + std::to_string(st) + ")");
  return FVM_OK;
}

// Device time (CUDA events on the closure's stream) of `iters` back-to-back
// launches of work, after one untimed warm-up.
template <class F>
int time_on_stream(fvm_closure* c, int iters, double* ms, F work) {
  if (!ms || iters < 1) return set_error(FVM_E_INVALID, "closure timing: iters >= 1 and a result pointer");
  cudaEvent_t a = nullptr, b = nullptr;
  CL_CK(cudaEventCreate(&a));
  CL_CK(cudaEventCreate(&b));
  cudaError_t e = work();
  if (e == cudaSuccess) e = cudaEventRecord(a, c->stream);
  for (int i = 0; i < iters && e == cudaSuccess; ++i) e = work();
  if (e == cudaSuccess) e = cudaEventRecord(b, c->stream);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) return set_error(FVM_E_CUDA, std::string("closure timing: ") + cudaGetErrorString(e));
  *ms = t / iters;
  return sync_status(c);
}

}  // namespace

namespace fvm {
namespace closure {
bool grid_matches(const fvm_closure* c, int nx, int ny, int nz) {
  return c && c->n1 == nx && c->n2 == ny && c->n3 == nz;
}
cudaError_t enqueue_infer(fvm_closure* c, const float* u, const Layout& lay, float gamma, cudaStream_t s) {
  CL_RET(features(c, u, lay, gamma, s));
  return forward(c, s);
}
cudaError_t launch_box_filter(const float* u, const Layout& lay, int nv, int f, float* out, int nsm, cudaStream_t s) {
  box_filter_kernel<<<4 * nsm, 256, 0, s>>>(u, lay, nv, f, out);
  return cudaGetLastError();
}
cudaError_t launch_dense_copy(float* u, const Layout& lay, int nv, float* dense, int to_state, int nsm,
                              cudaStream_t s) {
  dense_copy_kernel<float><<<4 * nsm, 256, 0, s>>>(u, lay, nv, dense, to_state);
  return cudaGetLastError();
}
cudaError_t enqueue_fix(fvm_closure* c, const float* uin, float* uout, const Layout& lay, float gamma, float coef,
                        float beta, const double h[3], const Clock* clk, unsigned long long* nswitch,
                        cudaStream_t s) {
  const FixArgs a = fix_args(c, uin, uout, lay, gamma, coef, beta, h, clk, 0.f, nswitch);
  return launch_fix(c, a, s);
}
}  // namespace closure
}  // namespace fvm

extern "C" {

int fvm_closure_create(int n1, int n2, int n3, unsigned long long seed, fvm_closure** out) {
  if (!out) return set_error(FVM_E_INVALID, "null output pointer");
  *out = nullptr;
  if (n1 < 16 || n2 < 16 || n3 < 1 || n1 % 16 || n2 % 16)
    return set_error(FVM_E_INVALID, "closure grid: n1 and n2 must be multiples of 16, n3 >= 1");
  int dev = 0, major = 0;
  CL_CK(cudaGetDevice(&dev));
  CL_CK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) return set_error(FVM_E_INVALID, "closure kernels need an sm_100 device");
  auto* c = new fvm_closure();
  c->n1 = n1;
  c->n2 = n2;
  c->n3 = n3;
  c->npos = (long long)n1 * n2 * n3;
  cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, dev);
  // conv CTAs are serial load -> MMA -> epilogue chains: aim for about four
  // resident per SM (shared memory allows 3-4) so their waits overlap
  c->zc_conv = largest_zc(n3, (long long)(n1 / 8) * (n2 / 16), 4ll * c->nsm);
  c->zc_wg = largest_zc(n3, (long long)(n1 / 16) * (n2 / 8), 2ll * c->nsm);
  const long long wg_blocks = (long long)(n1 / 16) * (n2 / 8) * (n3 / c->zc_wg);
  c->partial_elems = (size_t)wg_blocks * 27 * C_HID * C_HID + (size_t)2 * c->nsm * C_HID;
  c->loss_blocks = 4 * c->nsm;
  int rc = FVM_OK;
  const size_t np = (size_t)c->npos;
  if (!rc) rc = dalloc(&c->x0, np * C_IN0);
  if (!rc) rc = dalloc(&c->a1, np * C_HID);
  if (!rc) rc = dalloc(&c->a2, np * C_HID);
  if (!rc) rc = dalloc(&c->z3, np * C_OUT);
  if (!rc) rc = dalloc(&c->g3, np * C_OUT);
  if (!rc) rc = dalloc(&c->g2, np * C_HID);
  if (!rc) rc = dalloc(&c->g1, np * C_HID);
  if (!rc) rc = dalloc(&c->e, np * 5);
  if (!rc) rc = dalloc(&c->ratio, np * 10);
  if (!rc) rc = dalloc(&c->partial, c->partial_elems);
  if (!rc) rc = dalloc(&c->loss_part, (size_t)c->loss_blocks);
  if (!rc) rc = dalloc(&c->loss_dev, 1);
  if (!rc) rc = dalloc(&c->status, 1);
  if (!rc && set_attributes() != cudaSuccess) rc = set_error(FVM_E_CUDA, "closure: kernel attributes");
  for (int l = 0; l < NLAYER && !rc; ++l) {
    const size_t nw = wcount(l);
    rc = dalloc(&c->w[l], nw);
    if (!rc) rc = dalloc(&c->mw[l], nw);
    if (!rc) rc = dalloc(&c->vw[l], nw);
    if (!rc) rc = dalloc(&c->gw[l], nw);
    if (!rc) rc = dalloc(&c->b[l], (size_t)LCOUT[l]);
    if (!rc) rc = dalloc(&c->mb[l], (size_t)LCOUT[l]);
    if (!rc) rc = dalloc(&c->vb[l], (size_t)LCOUT[l]);
    if (!rc) rc = dalloc(&c->gb[l], (size_t)LCOUT[l]);
    if (!rc) rc = dalloc(&c->pf[l], nw);
    if (!rc) rc = dalloc(&c->pb[l], nw);
  }
  if (!rc && cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    rc = set_error(FVM_E_CUDA, "closure: stream creation failed");
  if (rc) {
    fvm_closure_destroy(c);
    return rc;
  }
  // zero workspace (ReLU masks of unused channels, padding channels)
  cudaMemset(c->x0, 0, np * C_IN0 * 2);
  cudaMemset(c->g3, 0, np * C_OUT * 2);
  cudaMemset(c->z3, 0, np * C_OUT * 4);
  cudaMemset(c->status, 0, sizeof(unsigned));
  unsigned long long st = seed;
  for (int l = 0; l < NLAYER; ++l) {
    std::vector<float> w(wcount(l)), b(LCOUT[l], 0.f);
    he_init(w, LCIN[l], l == NLAYER - 1 ? 0.1 : 1.0, st);
    rc = fvm_closure_set_weights(c, l + 1, w.data(), b.data());
    if (rc) {
      fvm_closure_destroy(c);
      return rc;
    }
  }
  *out = c;
  return FVM_OK;
}

int fvm_closure_destroy(fvm_closure* c) {
  if (!c) return FVM_OK;
  if (c->stream) cudaStreamSynchronize(c->stream);
  void* ptrs[] = {c->x0,      c->a1,        c->a2,       c->z3,      c->g3,    c->g2,
                  c->g1,      c->e,         c->partial,  c->loss_part, c->loss_dev, c->status, c->ratio};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (int l = 0; l < NLAYER; ++l) {
    void* lp[] = {c->w[l], c->b[l], c->mw[l], c->vw[l], c->mb[l], c->vb[l], c->gw[l], c->gb[l], c->pf[l], c->pb[l]};
    for (void* p : lp)
      if (p) cudaFree(p);
  }
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return FVM_OK;
}

int fvm_closure_set_norm(fvm_closure* c, double gamma, const double in_mean[5], const double in_scale[5],
                         const double out_scale[5], const double loss_weight[5]) {
  if (int rc = check(c)) return rc;
  if (!in_mean || !in_scale || !out_scale || !loss_weight || !(gamma > 1.0))
    return set_error(FVM_E_INVALID, "closure norm: null array or gamma <= 1");
  for (int q = 0; q < 5; ++q)
    if (!(in_scale[q] > 0) || !(out_scale[q] > 0) || !(loss_weight[q] >= 0))
      return set_error(FVM_E_INVALID, "closure norm: scales must be positive");
  c->gamma = (float)gamma;
  for (int q = 0; q < 5; ++q) {
    c->in_mean[q] = (float)in_mean[q];
    c->in_inv_scale[q] = (float)(1.0 / in_scale[q]);
    c->out_scale[q] = (float)out_scale[q];
    c->loss_w[q] = (float)loss_weight[q];
  }
  return FVM_OK;
}

int fvm_closure_set_limiter(fvm_closure* c, int fct) {
  if (int rc = check(c)) return rc;
  if (fct != 0 && fct != 1) return set_error(FVM_E_INVALID, "closure limiter: 0 (face clip) or 1 (face clip + FCT)");
  CL_CK(cudaStreamSynchronize(c->stream));
  c->fct = fct;
  return FVM_OK;
}

int fvm_closure_set_weights(fvm_closure* c, int layer, const float* w_host, const float* b_host) {
  if (int rc = check(c)) return rc;
  if (layer < 1 || layer > NLAYER || !w_host || !b_host) return set_error(FVM_E_INVALID, "closure layer 1..3");
  const int l = layer - 1;
  const size_t nw = wcount(l);
  CL_CK(cudaStreamSynchronize(c->stream));
  CL_CK(cudaMemcpy(c->w[l], w_host, nw * 4, cudaMemcpyHostToDevice));
  CL_CK(cudaMemcpy(c->b[l], b_host, LCOUT[l] * 4, cudaMemcpyHostToDevice));
  CL_CK(cudaMemset(c->mw[l], 0, nw * 4));
  CL_CK(cudaMemset(c->vw[l], 0, nw * 4));
  CL_CK(cudaMemset(c->mb[l], 0, LCOUT[l] * 4));
  CL_CK(cudaMemset(c->vb[l], 0, LCOUT[l] * 4));
  CL_CK(cudaMemset(c->gw[l], 0, nw * 4));
  CL_CK(cudaMemset(c->gb[l], 0, LCOUT[l] * 4));
  c->adam_step = 0;  // fresh moments: bias correction restarts
  CL_CK(adam_all(c, false, 0.f, 0.f, 0.f, 0.f, c->stream));
  CL_CK(cudaStreamSynchronize(c->stream));
  return FVM_OK;
}

int fvm_closure_get_weights(fvm_closure* c, int layer, float* w_host, float* b_host) {
  if (int rc = check(c)) return rc;
  if (layer < 1 || layer > NLAYER || !w_host || !b_host) return set_error(FVM_E_INVALID, "closure layer 1..3");
  const int l = layer - 1;
  CL_CK(cudaStreamSynchronize(c->stream));
  CL_CK(cudaMemcpy(w_host, c->w[l], wcount(l) * 4, cudaMemcpyDeviceToHost));
  CL_CK(cudaMemcpy(b_host, c->b[l], LCOUT[l] * 4, cudaMemcpyDeviceToHost));
  return FVM_OK;
}

int fvm_closure_get_grads(fvm_closure* c, int layer, float* dw_host, float* db_host) {
  if (int rc = check(c)) return rc;
  if (layer < 1 || layer > NLAYER || !dw_host || !db_host) return set_error(FVM_E_INVALID, "closure layer 1..3");
  const int l = layer - 1;
  CL_CK(cudaStreamSynchronize(c->stream));
  CL_CK(cudaMemcpy(dw_host, c->gw[l], wcount(l) * 4, cudaMemcpyDeviceToHost));
  CL_CK(cudaMemcpy(db_host, c->gb[l], LCOUT[l] * 4, cudaMemcpyDeviceToHost));
  return FVM_OK;
}

int fvm_closure_buffer(fvm_closure* c, int which, void* host, long long bytes, int to_device) {
  if (int rc = check(c)) return rc;
  void* p = nullptr;
  long long size = 0;
  const long long np = c->npos;
  switch (which) {
    case FVM_CB_X0: p = c->x0; size = np * C_IN0 * 2; break;
    case FVM_CB_A1: p = c->a1; size = np * C_HID * 2; break;
    case FVM_CB_A2: p = c->a2; size = np * C_HID * 2; break;
    case FVM_CB_Z3: p = c->z3; size = np * C_OUT * 4; break;
    case FVM_CB_G3: p = c->g3; size = np * C_OUT * 2; break;
    case FVM_CB_G2: p = c->g2; size = np * C_HID * 2; break;
    case FVM_CB_G1: p = c->g1; size = np * C_HID * 2; break;
    case FVM_CB_E: p = c->e; size = np * 5 * 4; break;
    default: return set_error(FVM_E_INVALID, "unknown closure buffer");
  }
  if (!host || bytes != size) return set_error(FVM_E_INVALID, "closure buffer: size mismatch");
  CL_CK(cudaStreamSynchronize(c->stream));
  CL_CK(cudaMemcpy(to_device ? p : host, to_device ? host : p, (size_t)size,
                   to_device ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost));
  return FVM_OK;
}

int fvm_closure_features(fvm_closure* c, const float* u_dense_dev) {
  if (int rc = check(c)) return rc;
  if (!u_dense_dev) return set_error(FVM_E_INVALID, "null state");
  CL_CK(features(c, u_dense_dev, dense_layout(c->n1, c->n2, c->n3), c->gamma, c->stream));
  return sync_status(c);
}

int fvm_closure_forward(fvm_closure* c) {
  if (int rc = check(c)) return rc;
  CL_CK(forward(c, c->stream));
  return sync_status(c);
}

int fvm_closure_backward(fvm_closure* c, const float* defect_dense_dev, double dt, const double h[3]) {
  if (int rc = check(c)) return rc;
  if (!defect_dense_dev || !h || !(h[0] > 0 && h[1] > 0 && h[2] > 0))
    return set_error(FVM_E_INVALID, "closure backward: bad defect or spacing");
  CL_CK(backward(c, defect_dense_dev, dt, h, c->stream));
  return sync_status(c);
}

int fvm_closure_adam(fvm_closure* c, double lr, double beta1, double beta2, double eps) {
  if (int rc = check(c)) return rc;
  CL_CK(adam_all(c, true, (float)lr, (float)beta1, (float)beta2, (float)eps, c->stream));
  return sync_status(c);
}

int fvm_closure_train_step(fvm_closure* c, const float* u_dense_dev, const float* defect_dense_dev, double dt,
                           const double h[3], double lr) {
  if (int rc = check(c)) return rc;
  if (!u_dense_dev || !defect_dense_dev || !h || !(h[0] > 0 && h[1] > 0 && h[2] > 0))
    return set_error(FVM_E_INVALID, "closure train step: bad arguments");
  CL_CK(features(c, u_dense_dev, dense_layout(c->n1, c->n2, c->n3), c->gamma, c->stream));
  CL_CK(forward(c, c->stream));
  CL_CK(backward(c, defect_dense_dev, dt, h, c->stream));
  CL_CK(adam_all(c, true, (float)lr, 0.9f, 0.999f, 1e-8f, c->stream));
  // inputs belong to the caller: finish with them before returning
  return sync_status(c);
}

int fvm_closure_time_forward(fvm_closure* c, int iters, double* ms) {
  if (int rc = check(c)) return rc;
  return time_on_stream(c, iters, ms, [&]() { return forward(c, c->stream); });
}

int fvm_closure_time_train(fvm_closure* c, const float* u_dense_dev, const float* defect_dense_dev, double dt,
                           const double h[3], double lr, int iters, double* ms) {
  if (int rc = check(c)) return rc;
  if (!u_dense_dev || !defect_dense_dev || !h || !(h[0] > 0 && h[1] > 0 && h[2] > 0))
    return set_error(FVM_E_INVALID, "closure timing: bad arguments");
  const Layout L = dense_layout(c->n1, c->n2, c->n3);
  return time_on_stream(c, iters, ms, [&]() {
    cudaError_t e = features(c, u_dense_dev, L, c->gamma, c->stream);
    if (e == cudaSuccess) e = forward(c, c->stream);
    if (e == cudaSuccess) e = backward(c, defect_dense_dev, dt, h, c->stream);
    if (e == cudaSuccess) e = adam_all(c, true, (float)lr, 0.9f, 0.999f, 1e-8f, c->stream);
    return e;
  });
}

int fvm_closure_loss(fvm_closure* c, double* out) {
  if (int rc = check(c)) return rc;
  if (!out) return set_error(FVM_E_INVALID, "null output");
  CL_CK(cudaStreamSynchronize(c->stream));
  CL_CK(cudaMemcpy(out, c->loss_dev, sizeof(double), cudaMemcpyDeviceToHost));
  return FVM_OK;
}

int fvm_closure_correct_dense(fvm_closure* c, const float* uin_dense_dev, float* uout_dense_dev, double coef,
                              double dt, double beta, const double h[3], unsigned long long* n_switched) {
  if (int rc = check(c)) return rc;
  if (!uin_dense_dev || !uout_dense_dev || !h || uin_dense_dev == uout_dense_dev)
    return set_error(FVM_E_INVALID, "closure correct: bad arguments");
  unsigned long long* cnt = nullptr;
  CL_CK(cudaMalloc(&cnt, sizeof(unsigned long long)));
  cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), c->stream);
  const FixArgs a = fix_args(c, uin_dense_dev, uout_dense_dev, dense_layout(c->n1, c->n2, c->n3), c->gamma,
                             (float)coef, (float)beta, h, nullptr, (float)dt, cnt);
  cudaError_t e = launch_fix(c, a, c->stream);
  unsigned long long v = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&v, cnt, sizeof(v), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(cnt);
  if (e != cudaSuccess) return set_error(FVM_E_CUDA, std::string("closure correct: ") + cudaGetErrorString(e));
  if (n_switched) *n_switched = v;
  return FVM_OK;
}

}  // extern "C"
