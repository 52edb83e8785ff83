// Learned flux-correction closure: device code (sm_100a).
//
// A 3-layer periodic 3x3x3 CNN (16 -> 32 -> 32 -> 16 channels, ReLU between)
// maps normalised primitive variables of a coarse navier_stokes state to face
// flux corrections dF (channel a*5+q: variable q on the +x_a face of the
// cell).  The reference has no learned part; this file holds
//
//   * conv3_kernel: forward conv and data-gradient conv as one BF16 implicit
//     GEMM on the 5th-generation tensor cores (tcgen05.mma, FP32 accumulators
//     in tensor memory), M = 128 positions (an 8 x 16 x-y tile), N = output
//     channels, K = 27 taps x input channels, marching along z;
//   * wgrad_kernel: weight gradient as tcgen05 GEMMs contracting over
//     positions (MN-major operands; three y-taps share one M = 128 MMA);
//   * Adam with bias correction that also writes the packed BF16 operands;
//   * features, the a-priori loss and its gradient, the box filter, and the
//     per-stage correction (clipped, positivity-gated) used by the solver.
//
// Activations are channels-last ([z][y][x][c], x fastest among positions),
// periodic in all three directions.  Tap t = (dz+1)*9 + (dy+1)*3 + (dx+1),
// weights W[t][co][ci].
#pragma once
#include <cuda_bf16.h>
#include "fvm_common.cuh"

namespace fvm {
namespace closure {

constexpr int C_IN0 = 16;   // input features (5 used, zero padded)
constexpr int C_HID = 32;   // hidden channels
constexpr int C_OUT = 16;   // face corrections (15 used)
constexpr int N_VAR = 5;
constexpr uint64_t WAIT_NS = 2000000000ull;  // 2 s bound on every wait

// ------------------------------------------------------ tcgen05 helpers ----
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// D[tmem] (+)= A[smem] * B[smem]^T, BF16 inputs, FP32 accumulate.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  const uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(z)
      : "memory");
}
// Arrive on `bar` once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 32 lanes x N columns of 32-bit accumulators, one row per thread.
template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t* v);
template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
template <>
__device__ __forceinline__ void tmem_ld<32>(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]),
        "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
        "=r"(v[30]), "=r"(v[31])
      : "r"(taddr));
}

// Shared-memory matrix descriptor, no swizzle (canonical "interleave"
// layout of 8 rows x 16 bytes core matrices).  K-major: LBO = stride between
// the two 8-element K halves, SBO = stride between 8-row groups.  MN-major:
// LBO = stride between 8-row K groups, SBO = stride between 8-element MN
// chunks.  Bits 46-47 hold the descriptor version (1).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor: BF16 x BF16 -> FP32, dense, M x N, operand majors
// (0 = K-major, 1 = MN-major).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// One contiguous global -> shared bulk copy completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ uint4 ldg16(const void* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }
__device__ __forceinline__ void sts16(uint8_t* p, uint4 v) { *reinterpret_cast<uint4*>(p) = v; }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }

// Packed B operand (K-major, N x K per MMA of K = 16): element (tap t, row n,
// reduction index k) of a layer with K-extent kin and N-extent nout.
__host__ __device__ inline long long pack_index(int t, int n, int k, int kin, int nout) {
  const int ks = kin / 16;
  return ((((long long)t * ks + k / 16) * 2 + (k % 16) / 8) * nout + n) * 8 + (k % 8);
}

// ------------------------------------------------------ forward / dgrad ----
enum Epi : int {
  EPI_RELU_BF16 = 0,  // y = max(acc + b, 0), BF16
  EPI_LIN_F32 = 1,    // y = acc + b, FP32
  EPI_MASK_BF16 = 2   // y = acc where mask > 0 else 0, BF16 (ReLU backward)
};

struct ConvArgs {
  const __nv_bfloat16* x;     // input [pos][CIN]
  const void* wpack;          // packed weights (pack_index layout), 27*CIN*COUT bf16
  const float* bias;          // COUT (EPI_RELU_BF16 / EPI_LIN_F32)
  void* y;                    // output [pos][COUT]
  const __nv_bfloat16* mask;  // EPI_MASK_BF16: [pos][COUT]
  int n1, n2, n3, zc;
  unsigned* status;
};

template <int CIN, int COUT>
struct ConvCfg {
  static constexpr int NCH = CIN / 8;      // 16-byte channel chunks
  static constexpr int KS = CIN / 16;      // K = 16 steps per tap
  static constexpr int XE = 10, YE = 18;   // staged x, y extent (tile + halo)
  static constexpr int CHB = XE * 16;      // chunk stride inside a row
  static constexpr int ROWB = NCH * CHB;   // row stride (= SBO of A)
  static constexpr int PLANEB = YE * ROWB;
  static constexpr int NSLOT = 4;
  static constexpr int WB = 27 * CIN * COUT * 2;
  static constexpr int OFF_W = 0;
  static constexpr int OFF_RING = WB;
  static constexpr int OFF_BIAS = OFF_RING + NSLOT * PLANEB;
  static constexpr int OFF_BAR = OFF_BIAS + COUT * 4;
  static constexpr int BYTES = OFF_BAR + 64;
  static constexpr int ELEMS = YE * XE * NCH;
  static constexpr int PER = (ELEMS + 127) / 128;
  static constexpr int TCOLS = 2 * COUT < 32 ? 32 : 2 * COUT;
  // CTAs per SM that shared memory allows (227 KB usable, 1 KB reserved each),
  // at most four: the register budget the compiler may use follows from it
  static constexpr int MINB = (227 * 1024) / (BYTES + 1024) > 4 ? 4 : (227 * 1024) / (BYTES + 1024);
  static_assert(WB % 128 == 0 && PLANEB % 16 == 0, "alignment");
};

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(128, ConvCfg<CIN, COUT>::MINB) conv3_kernel(const ConvArgs a) {
  using C = ConvCfg<CIN, COUT>;
  extern __shared__ __align__(128) uint8_t smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + C::OFF_BAR);  // [0] weights, [1],[2] accumulators
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + C::OFF_BAR + 32);
  int* abort_flag = reinterpret_cast<int*>(smem + C::OFF_BAR + 40);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
  const int x0 = blockIdx.x * 8, y0 = blockIdx.y * 16, z0 = blockIdx.z * a.zc;
  const uint32_t sbase = smem_u32(smem);

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    tmem_alloc(tslot, C::TCOLS);
    tmem_relinquish();
  }
  if constexpr (EPI != EPI_MASK_BF16) {
    if (tid < COUT) reinterpret_cast<float*>(smem + C::OFF_BIAS)[tid] = __ldg(a.bias + tid);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar[0], C::WB);
    bulk_g2s(smem + C::OFF_W, a.wpack, C::WB, &bar[0]);
  }

  // The (periodic) x-y offsets of this thread's plane elements do not depend
  // on z: decompose them once.
  uint4 reg[C::PER];
  int goff[C::PER], soff[C::PER];
#pragma unroll
  for (int u = 0; u < C::PER; ++u) {
    const int e = tid + u * 128;
    const int r = e / (C::XE * C::NCH), rem = e - r * (C::XE * C::NCH);
    const int xe = rem / C::NCH, c = rem - xe * C::NCH;
    int y = y0 - 1 + r, x = x0 - 1 + xe;
    y = y < 0 ? y + n2 : (y >= n2 ? y - n2 : y);
    x = x < 0 ? x + n1 : (x >= n1 ? x - n1 : x);
    goff[u] = (y * n1 + x) * CIN + c * 8;
    soff[u] = ((r * C::NCH + c) * C::XE + xe) * 16;
  }
  const size_t zstride = (size_t)n2 * n1 * CIN;
  auto load_plane = [&](int z) {
    z = z < 0 ? z + n3 : (z >= n3 ? z - n3 : z);
    const __nv_bfloat16* zb = a.x + (size_t)z * zstride;
#pragma unroll
    for (int u = 0; u < C::PER; ++u)
      if (tid + u * 128 < C::ELEMS) reg[u] = ldg16(zb + goff[u]);
  };
  auto store_plane = [&](int slot) {
    uint8_t* base = smem + C::OFF_RING + slot * C::PLANEB;
#pragma unroll
    for (int u = 0; u < C::PER; ++u)
      if (tid + u * 128 < C::ELEMS) sts16(base + soff[u], reg[u]);
  };
  for (int j = 0; j < 3; ++j) {
    load_plane(z0 - 1 + j);
    store_plane(j);
  }
  fence_proxy_async();
  if (tid == 0 && !mbar_wait_bounded(&bar[0], 0, WAIT_NS)) {
    *abort_flag = 1;
    atomicOr(a.status, ST_TMA_TIMEOUT);
  }
  tc_fence_before();
  __syncthreads();

  constexpr uint32_t IDESC = idesc_bf16(128, COUT, 0, 0);
  int pending[2] = {-1, -1};  // committed, not yet waited step per accumulator buffer
  const int m = warp * 32 + lane, xl = m & 7, yl = m >> 3;
  const float* bias = reinterpret_cast<const float*>(smem + C::OFF_BIAS);

  auto epilogue = [&](int s) {
    const int b = s & 1;
    bool ok = mbar_wait_bounded(&bar[1 + b], (s >> 1) & 1, WAIT_NS);
    pending[b] = -1;
    if (!ok) {
      *abort_flag = 1;
      atomicOr(a.status, ST_TMA_TIMEOUT);
    }
    tc_fence_after();
    uint32_t v[COUT];
    tmem_ld<COUT>(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * COUT), v);
    tmem_wait_ld();
    const size_t pos = ((size_t)(z0 + s) * n2 + (y0 + yl)) * n1 + (x0 + xl);
    if constexpr (EPI == EPI_LIN_F32) {
      float4* out = reinterpret_cast<float4*>(static_cast<float*>(a.y) + pos * COUT);
#pragma unroll
      for (int q = 0; q < COUT / 4; ++q)
        out[q] = make_float4(__uint_as_float(v[4 * q]) + bias[4 * q], __uint_as_float(v[4 * q + 1]) + bias[4 * q + 1],
                             __uint_as_float(v[4 * q + 2]) + bias[4 * q + 2],
                             __uint_as_float(v[4 * q + 3]) + bias[4 * q + 3]);
    } else {
      uint4* out = reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(a.y) + pos * COUT);
      // every mask load before the first store (the stores may alias the mask
      // as far as the compiler knows: one memory round trip per chunk otherwise)
      uint4 mks[EPI == EPI_MASK_BF16 ? COUT / 8 : 1];
      if constexpr (EPI == EPI_MASK_BF16) {
#pragma unroll
        for (int q = 0; q < COUT / 8; ++q) mks[q] = ldg16(a.mask + pos * COUT + 8 * q);
      }
#pragma unroll
      for (int q = 0; q < COUT / 8; ++q) {
        float f[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) f[e] = __uint_as_float(v[8 * q + e]);
        if constexpr (EPI == EPI_RELU_BF16) {
#pragma unroll
          for (int e = 0; e < 8; ++e) f[e] = fmaxf(f[e] + bias[8 * q + e], 0.f);
        } else {
          const uint4 mk = mks[q];
          const uint32_t mw[4] = {mk.x, mk.y, mk.z, mk.w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            if (!(bf16_lo(mw[e]) > 0.f)) f[2 * e] = 0.f;
            if (!(bf16_hi(mw[e]) > 0.f)) f[2 * e + 1] = 0.f;
          }
        }
        out[q] = make_uint4(pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]), pack_bf16x2(f[4], f[5]),
                            pack_bf16x2(f[6], f[7]));
      }
    }
  };

  for (int i = 0; i < a.zc; ++i) {
    const bool aborted = *abort_flag != 0;  // uniform: read after a barrier
    if (!aborted) {
      if (tid == 0) {
        tc_fence_after();
        const uint32_t dcol = tbase + (uint32_t)((i & 1) * COUT);
        // A tap shift only moves the 14-bit start-address field, so every
        // descriptor is a per-step base plus a compile-time constant (the
        // addresses stay below 256 KB: no carry out of the field).
        uint64_t abase[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) abase[d] = sdesc(sbase + C::OFF_RING + ((i + d) & 3) * C::PLANEB, C::CHB, C::ROWB);
        const uint64_t bbase = sdesc(sbase + C::OFF_W, COUT * 16, 128);
#pragma unroll
        for (int t = 0; t < 27; ++t) {
#pragma unroll
          for (int s = 0; s < C::KS; ++s) {
            const uint64_t ad = abase[t / 9] + (uint64_t)(((t / 3) % 3 * C::ROWB + 2 * s * C::CHB + (t % 3) * 16) >> 4);
            const uint64_t bd = bbase + (uint64_t)(((t * C::KS + s) * 2 * COUT * 16) >> 4);
            umma_bf16(dcol, ad, bd, IDESC, (t | s) != 0 ? 1u : 0u);
          }
        }
        umma_commit(&bar[1 + (i & 1)]);
      }
      pending[i & 1] = i;
    }
    const bool more = i + 1 < a.zc;
    if (more) load_plane(z0 + i + 2);
    if (i >= 1 && !aborted) epilogue(i - 1);
    if (more) store_plane((i + 3) & 3);
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
  }
  if (*abort_flag == 0) epilogue(a.zc - 1);
  // Drain any MMA still in flight (only after a timeout) before freeing TMEM.
  if (tid == 0) {
    for (int b = 0; b < 2; ++b)
      if (pending[b] >= 0) mbar_wait_bounded(&bar[1 + b], (pending[b] >> 1) & 1, WAIT_NS);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, C::TCOLS);
  }
}

// ------------------------------------------------------------- wgrad ----
// dW[t][co][ci] = sum_p G[p][co] X[p + off_t][ci].  Per (dz, dx) pair one
// accumulator D[(j, ci)][co] (j = dy + 1 in rows j*CIN + ci; rows of j >= 3
// are unused), A = X shifted (MN-major, M = NSH*CIN = 128), B = G (MN-major,
// N = COUT), K = 16 consecutive x positions of one row.
struct WgradArgs {
  const __nv_bfloat16* x;  // [pos][CIN]
  const __nv_bfloat16* g;  // [pos][COUT]
  float* partial;          // [block][27][COUT][CIN]
  int n1, n2, n3, zc;
  unsigned* status;
};

template <int CIN, int COUT>
struct WgCfg {
  static constexpr int NCH = CIN / 8, NCHG = COUT / 8;
  static constexpr int NSH = 128 / CIN;
  static constexpr int TY = 8, TX = 16;
  static constexpr int XE = TX + 2, YE = TY + 2;
  static constexpr int CHB = XE * 16;
  static constexpr int ROWB = NCH * CHB;
  static constexpr int PLANEB = YE * ROWB;
  static constexpr int PADB = (NSH - 3) * ROWB;  // rows read by the unused shifts past the last slot
  static constexpr int GCHB = TX * 16;
  static constexpr int GROWB = NCHG * GCHB;
  static constexpr int GPLANEB = TY * GROWB;
  static constexpr int OFF_X = 0;
  static constexpr int OFF_G = 4 * PLANEB + PADB;
  static constexpr int OFF_BAR = OFF_G + 2 * GPLANEB;
  static constexpr int BYTES = OFF_BAR + 64;
  static constexpr int XELEMS = YE * XE * NCH, XPER = (XELEMS + 127) / 128;
  static constexpr int GELEMS = TY * TX * NCHG, GPER = (GELEMS + 127) / 128;
  static constexpr int TCOLS = 9 * COUT <= 256 ? 256 : 512;
  static_assert(NSH >= 3, "three y taps per MMA");
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(128, 1) wgrad_kernel(const WgradArgs a) {
  using C = WgCfg<CIN, COUT>;
  extern __shared__ __align__(128) uint8_t smem[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem + C::OFF_BAR);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + C::OFF_BAR + 32);
  int* abort_flag = reinterpret_cast<int*>(smem + C::OFF_BAR + 40);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n1 = a.n1, n2 = a.n2, n3 = a.n3;
  const int x0 = blockIdx.x * C::TX, y0 = blockIdx.y * C::TY, z0 = blockIdx.z * a.zc;
  const uint32_t sbase = smem_u32(smem);

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    *abort_flag = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    tmem_alloc(tslot, C::TCOLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;

  // z-independent element offsets, decomposed once (periodic wrap in x, y)
  uint4 xr[C::XPER], gr[C::GPER];
  int xg[C::XPER], xs[C::XPER], gg[C::GPER], gs[C::GPER];
#pragma unroll
  for (int u = 0; u < C::XPER; ++u) {
    const int e = tid + u * 128;
    const int r = e / (C::XE * C::NCH), rem = e - r * (C::XE * C::NCH);
    const int xe = rem / C::NCH, c = rem - xe * C::NCH;
    int y = y0 - 1 + r, x = x0 - 1 + xe;
    y = y < 0 ? y + n2 : (y >= n2 ? y - n2 : y);
    x = x < 0 ? x + n1 : (x >= n1 ? x - n1 : x);
    xg[u] = (y * n1 + x) * CIN + c * 8;
    xs[u] = ((r * C::NCH + c) * C::XE + xe) * 16;
  }
#pragma unroll
  for (int u = 0; u < C::GPER; ++u) {
    const int e = tid + u * 128;
    const int r = e / (C::TX * C::NCHG), rem = e - r * (C::TX * C::NCHG);
    const int xe = rem / C::NCHG, c = rem - xe * C::NCHG;
    gg[u] = ((y0 + r) * n1 + (x0 + xe)) * COUT + c * 8;
    gs[u] = ((r * C::NCHG + c) * C::TX + xe) * 16;
  }
  auto load_x = [&](int z) {
    z = z < 0 ? z + n3 : (z >= n3 ? z - n3 : z);
    const __nv_bfloat16* zb = a.x + (size_t)z * n2 * n1 * CIN;
#pragma unroll
    for (int u = 0; u < C::XPER; ++u)
      if (tid + u * 128 < C::XELEMS) xr[u] = ldg16(zb + xg[u]);
  };
  auto store_x = [&](int slot) {
    uint8_t* base = smem + C::OFF_X + slot * C::PLANEB;
#pragma unroll
    for (int u = 0; u < C::XPER; ++u)
      if (tid + u * 128 < C::XELEMS) sts16(base + xs[u], xr[u]);
  };
  auto load_g = [&](int z) {
    const __nv_bfloat16* zb = a.g + (size_t)z * n2 * n1 * COUT;
#pragma unroll
    for (int u = 0; u < C::GPER; ++u)
      if (tid + u * 128 < C::GELEMS) gr[u] = ldg16(zb + gg[u]);
  };
  auto store_g = [&](int slot) {
    uint8_t* base = smem + C::OFF_G + slot * C::GPLANEB;
#pragma unroll
    for (int u = 0; u < C::GPER; ++u)
      if (tid + u * 128 < C::GELEMS) sts16(base + gs[u], gr[u]);
  };
  for (int j = 0; j < 3; ++j) {
    load_x(z0 - 1 + j);
    store_x(j);
  }
  load_g(z0);
  store_g(0);
  fence_proxy_async();
  tc_fence_before();
  __syncthreads();

  constexpr uint32_t IDESC = idesc_bf16(128, COUT, 1, 1);
  int pending[2] = {-1, -1};
  auto wait_step = [&](int s) {
    const int b = s & 1;
    if (!mbar_wait_bounded(&bar[b], (s >> 1) & 1, WAIT_NS)) {
      *abort_flag = 1;
      atomicOr(a.status, ST_TMA_TIMEOUT);
    }
    pending[b] = -1;
  };

  for (int i = 0; i < a.zc; ++i) {
    const bool aborted = *abort_flag != 0;
    if (!aborted) {
      if (tid == 0) {
        tc_fence_after();
        // descriptors = per-step bases + compile-time offsets (see conv3_kernel)
        const uint64_t bbase = sdesc(sbase + C::OFF_G + (i & 1) * C::GPLANEB, 128, C::GCHB);
        uint64_t abase[3];
#pragma unroll
        for (int dz = 0; dz < 3; ++dz) abase[dz] = sdesc(sbase + C::OFF_X + ((i + dz) & 3) * C::PLANEB, 128, C::CHB);
        const uint32_t acc0 = i != 0 ? 1u : 0u;
#pragma unroll
        for (int yl = 0; yl < C::TY; ++yl) {
          const uint64_t bd = bbase + (uint64_t)((yl * C::GROWB) >> 4);
#pragma unroll
          for (int dz = 0; dz < 3; ++dz) {
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
              const uint64_t ad = abase[dz] + (uint64_t)((yl * C::ROWB + dx * 16) >> 4);
              umma_bf16(tbase + (uint32_t)((dz * 3 + dx) * COUT), ad, bd, IDESC, yl != 0 ? 1u : acc0);
            }
          }
        }
        umma_commit(&bar[i & 1]);
      }
      pending[i & 1] = i;
    }
    const bool more = i + 1 < a.zc;
    if (more) {
      load_x(z0 + i + 2);
      load_g(z0 + i + 1);
    }
    if (i >= 1 && !aborted) wait_step(i - 1);
    if (more) {
      store_x((i + 3) & 3);
      store_g((i + 1) & 1);
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
  }
  if (*abort_flag == 0) wait_step(a.zc - 1);
  if (tid == 0) {
    for (int b = 0; b < 2; ++b)
      if (pending[b] >= 0) mbar_wait_bounded(&bar[b], (pending[b] >> 1) & 1, WAIT_NS);
  }
  tc_fence_after();

  // Epilogue: row m = j*CIN + ci of accumulator (dz, dx) -> tap (dz, j-1, dx).
  const int m = warp * 32 + lane, j = m / CIN, ci = m % CIN;
  const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  float* part = a.partial + blk * 27 * COUT * CIN;
  const bool live = *abort_flag == 0;
#pragma unroll 1
  for (int cidx = 0; cidx < 9; ++cidx) {
    uint32_t v[COUT];
    tmem_ld<COUT>(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cidx * COUT), v);
    tmem_wait_ld();
    if (j < 3) {
      const int t = (cidx / 3) * 9 + j * 3 + (cidx % 3);
#pragma unroll
      for (int co = 0; co < COUT; ++co)
        part[((size_t)t * COUT + co) * CIN + ci] = live ? __uint_as_float(v[co]) : 0.f;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, C::TCOLS);
  }
}

// ------------------------------------------------------- small kernels ----
// Per-block channel sums of a [pos][C] BF16 field (bias gradients).
template <int C>
__global__ void __launch_bounds__(256) channel_sum_kernel(const __nv_bfloat16* g, long long npos,
                                                          float* partial) {
  constexpr int NCHK = C / 8;
  __shared__ float red[256][9];
  const int tid = threadIdx.x, c = tid % NCHK;
  float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const long long stride = (long long)gridDim.x * (256 / NCHK);
  for (long long p = (long long)blockIdx.x * (256 / NCHK) + tid / NCHK; p < npos; p += stride) {
    const uint4 v = ldg16(g + p * C + c * 8);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      acc[2 * e] += bf16_lo(w[e]);
      acc[2 * e + 1] += bf16_hi(w[e]);
    }
  }
#pragma unroll
  for (int e = 0; e < 8; ++e) red[tid][e] = acc[e];
  __syncthreads();
  if (tid < C) {
    const int cc = tid / 8, e = tid % 8;
    float s = 0.f;
    for (int r = cc; r < 256; r += NCHK) s += red[r][e];
    partial[(size_t)blockIdx.x * C + tid] = s;
  }
}

// out[e] = sum_b partial[b*n + e] (float64 accumulation, fixed order).
__global__ void reduce_partials_kernel(const float* partial, int nblk, int n, float* out) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += partial[(size_t)b * n + e];
    out[e] = (float)s;
  }
}

// Adam (Kingma & Ba 2015, bias-corrected) on one layer's FP32 master weights
// and bias, then the packed BF16 operands: forward (N = cout, K = cin) and,
// when `pack_bwd` is set, data gradient (tap flipped, N = cin, K = cout).
struct AdamLayer {
  float *w, *m, *v, *b, *mb, *vb;
  const float *gw, *gb;
  __nv_bfloat16 *pack_fwd, *pack_bwd;
  int cout, cin;
};
__global__ void adam_pack_kernel(AdamLayer L, int update, float lr, float b1, float b2, float eps, float c1,
                                 float c2) {
  const int nw = 27 * L.cout * L.cin;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nw + L.cout; e += gridDim.x * blockDim.x) {
    const bool isw = e < nw;
    float* p = isw ? L.w + e : L.b + (e - nw);
    if (update) {
      float* mm = isw ? L.m + e : L.mb + (e - nw);
      float* vv = isw ? L.v + e : L.vb + (e - nw);
      const float g = isw ? L.gw[e] : L.gb[e - nw];
      const float mn = b1 * *mm + (1.f - b1) * g;
      const float vn = b2 * *vv + (1.f - b2) * g * g;
      *mm = mn;
      *vv = vn;
      *p = *p - lr * (mn * c1) / (sqrtf(vn * c2) + eps);
    }
    if (isw) {
      const int t = e / (L.cout * L.cin), co = (e / L.cin) % L.cout, ci = e % L.cin;
      const __nv_bfloat16 h = __float2bfloat16_rn(*p);
      L.pack_fwd[pack_index(t, co, ci, L.cin, L.cout)] = h;
      if (L.pack_bwd) L.pack_bwd[pack_index(26 - t, ci, co, L.cout, L.cin)] = h;
    }
  }
}

// Normalised primitive features (rho, v1, v2, v3, p) of a float32 state in
// the solver layout (interior only) -> [pos][16] BF16, channels 5..15 zero.
struct FeatArgs {
  const float* u;
  Layout lay;
  float gamma;
  float mean[5], inv_scale[5];
  __nv_bfloat16* x;
};
__global__ void features_kernel(const FeatArgs a) {
  const Layout& L = a.lay;
  const long long n = (long long)L.nx * L.ny * L.nz;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % L.nx), j = (int)((p / L.nx) % L.ny), k = (int)(p / ((long long)L.nx * L.ny));
    float u[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) u[q] = __ldg(a.u + L.idx(q, k + 1, j + 1, i + 1));
    const float rinv = 1.f / u[0];
    const float v1 = u[1] * rinv, v2 = u[2] * rinv, v3 = u[3] * rinv;
    const float pr = (a.gamma - 1.f) * (u[4] - 0.5f * u[0] * (v1 * v1 + v2 * v2 + v3 * v3));
    const float f[5] = {u[0], v1, v2, v3, pr};
    uint32_t w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float h[6];
#pragma unroll
    for (int q = 0; q < 5; ++q) h[q] = (f[q] - a.mean[q]) * a.inv_scale[q];
    h[5] = 0.f;
    w[0] = pack_bf16x2(h[0], h[1]);
    w[1] = pack_bf16x2(h[2], h[3]);
    w[2] = pack_bf16x2(h[4], 0.f);
    uint4* out = reinterpret_cast<uint4*>(a.x + p * C_IN0);
    out[0] = make_uint4(w[0], w[1], w[2], w[3]);
    out[1] = make_uint4(w[4], w[5], w[6], w[7]);
  }
}

// A-priori loss: E = dt * (-sum_a (s F[p] - s F[p - e_a]) / h_a) - D,
// loss = sum_p sum_q w_q E^2 / N (float64 block partials).
struct LossArgs {
  const float* z3;  // [pos][16] network output
  const float* d;   // target defect, dense [q][pos]
  float* e;         // residual E, dense [q][pos]
  __nv_bfloat16* g3;
  float s[5], w[5];
  float coef[3];    // dt / h_a
  float inv_n;
  double* partial;
  int n1, n2, n3;
};
__global__ void __launch_bounds__(256) loss_residual_kernel(const LossArgs a) {
  __shared__ double red[256];
  const long long n = (long long)a.n1 * a.n2 * a.n3;
  double acc = 0.0;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % a.n1), j = (int)((p / a.n1) % a.n2), k = (int)(p / ((long long)a.n1 * a.n2));
    const long long pm[3] = {p - i + (i + a.n1 - 1) % a.n1,
                             p + (long long)(((j + a.n2 - 1) % a.n2) - j) * a.n1,
                             p + (long long)(((k + a.n3 - 1) % a.n3) - k) * a.n1 * a.n2};
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      float r = 0.f;
#pragma unroll
      for (int ax = 0; ax < 3; ++ax)
        r -= a.coef[ax] * (a.s[q] * __ldg(a.z3 + p * 16 + ax * 5 + q) - a.s[q] * __ldg(a.z3 + pm[ax] * 16 + ax * 5 + q));
      const float ev = r - __ldg(a.d + q * n + p);
      a.e[q * n + p] = ev;
      acc += (double)a.w[q] * (double)ev * (double)ev;
    }
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.partial[blockIdx.x] = red[0] * (double)a.inv_n;
}
// dL/dZ3[p][a*5+q] = s_q (dt/h_a) (2 w_q / N) (E[q][p + e_a] - E[q][p]), BF16.
__global__ void loss_grad_kernel(const LossArgs a) {
  const long long n = (long long)a.n1 * a.n2 * a.n3;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(p % a.n1), j = (int)((p / a.n1) % a.n2), k = (int)(p / ((long long)a.n1 * a.n2));
    const long long pp[3] = {p - i + (i + 1) % a.n1, p + (long long)(((j + 1) % a.n2) - j) * a.n1,
                             p + (long long)(((k + 1) % a.n3) - k) * a.n1 * a.n2};
    float g[16];
#pragma unroll
    for (int ax = 0; ax < 3; ++ax)
#pragma unroll
      for (int q = 0; q < 5; ++q)
        g[ax * 5 + q] = a.s[q] * a.coef[ax] * (2.f * a.w[q] * a.inv_n) *
                        (__ldg(a.e + q * n + pp[ax]) - __ldg(a.e + q * n + p));
    g[15] = 0.f;
    uint4* out = reinterpret_cast<uint4*>(a.g3 + p * 16);
    out[0] = make_uint4(pack_bf16x2(g[0], g[1]), pack_bf16x2(g[2], g[3]), pack_bf16x2(g[4], g[5]),
                        pack_bf16x2(g[6], g[7]));
    out[1] = make_uint4(pack_bf16x2(g[8], g[9]), pack_bf16x2(g[10], g[11]), pack_bf16x2(g[12], g[13]),
                        pack_bf16x2(g[14], g[15]));
  }
}
__global__ void sum_partials_kernel(const double* partial, int n, double* out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int b = threadIdx.x; b < n; b += 256) s += partial[b];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = 128; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

// Conservative f^3 box filter of a float32 state (solver layout) -> dense
// coarse [q][k][j][i] (float64 sums).
__global__ void box_filter_kernel(const float* u, Layout lay, int nv, int f, float* out) {
  const int c1 = lay.nx / f, c2 = lay.ny / f, c3 = lay.nz / f;
  const long long nc = (long long)c1 * c2 * c3;
  const double inv = 1.0 / ((double)f * f * f);
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nc * nv;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(e / nc);
    const long long p = e % nc;
    const int i = (int)(p % c1), j = (int)((p / c1) % c2), k = (int)(p / ((long long)c1 * c2));
    double s = 0.0;
    for (int dk = 0; dk < f; ++dk)
      for (int dj = 0; dj < f; ++dj)
        for (int di = 0; di < f; ++di)
          s += (double)__ldg(u + lay.idx(q, k * f + dk + 1, j * f + dj + 1, i * f + di + 1));
    out[e] = (float)(s * inv);
  }
}

// Interior copy between a solver-layout state and a dense [q][k][j][i] array.
template <typename Real>
__global__ void dense_copy_kernel(Real* u, Layout lay, int nv, Real* dense, int to_state) {
  const long long n = (long long)lay.nx * lay.ny * lay.nz;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n * nv;
       e += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(e / n);
    const long long p = e % n;
    const int i = (int)(p % lay.nx), j = (int)((p / lay.nx) % lay.ny), k = (int)(p / ((long long)lay.nx * lay.ny));
    const long long s = lay.idx(q, k + 1, j + 1, i + 1);
    if (to_state) u[s] = dense[e];
    else dense[e] = u[s];
  }
}

// Per-stage correction.  For the stage input Uin (the state the stage's
// residual was taken of) and face x_a + 1/2 of cell p:
//   F = clip(s_q Z3[p][a*5+q], +-beta * smax * |Uq(p + e_a) - Uq(p)|),
//   smax = max(|v_a| + c) over the two cells (the first-order upwind
//   dissipation of the face bounds the anti-dissipative correction),
// R_q = -sum_a (F(p) - F(p - e_a)) / h_a and Uout += coef * dt * R unless the
// result has rho <= 0 or p <= 0, in which case the cell keeps the plain
// update (counted in `nswitch`).  Grids are periodic in all three directions.
struct FixArgs {
  const float* uin;
  float* uout;
  Layout lay;
  const float* z3;
  float s[5];
  float beta, gamma, coef;
  float inv_h[3];
  const Clock* clk;   // dt and the active flag of the solver clock, or null
  float dt_host;      // dt when clk is null
  unsigned long long* nswitch;
  float* ratio;       // flux-corrected transport fractions [10][cells] (fct mode)
};
__device__ __forceinline__ void load_cell(const FixArgs& a, int i, int j, int k, float* u) {
#pragma unroll
  for (int q = 0; q < 5; ++q) u[q] = __ldg(a.uin + a.lay.idx(q, k + 1, j + 1, i + 1));
}
__device__ __forceinline__ float wave_speed(const float* u, int ax, float gamma) {
  const float rinv = 1.f / u[0];
  const float v1 = u[1] * rinv, v2 = u[2] * rinv, v3 = u[3] * rinv;
  const float pr = (gamma - 1.f) * (u[4] - 0.5f * u[0] * (v1 * v1 + v2 * v2 + v3 * v3));
  const float c = (pr > 0.f && u[0] > 0.f) ? sqrtf(gamma * pr * rinv) : 0.f;
  const float va = ax == 0 ? v1 : (ax == 1 ? v2 : v3);
  return fabsf(va) + c;
}
// Clipped face corrections of cell c: Fp[ax][q] on its +x_ax face, Fm[ax][q]
// on its -x_ax face (the +face of the neighbour below), and the dense
// indices of the six neighbours (nb[ax][0] = -e_ax, nb[ax][1] = +e_ax).
__device__ __forceinline__ void face_corrections(const FixArgs& a, const int c[3], long long p, float Fp[3][5],
                                                 float Fm[3][5], long long nb[3][2], int nc[3][2][3] = nullptr) {
  const Layout& L = a.lay;
  const int dims[3] = {L.nx, L.ny, L.nz};
  float u0[5];
  load_cell(a, c[0], c[1], c[2], u0);
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) {
    int cp[3] = {c[0], c[1], c[2]}, cm[3] = {c[0], c[1], c[2]};
    cp[ax] = c[ax] + 1 == dims[ax] ? 0 : c[ax] + 1;  // periodic neighbours
    cm[ax] = c[ax] == 0 ? dims[ax] - 1 : c[ax] - 1;
    if (nc) {
#pragma unroll
      for (int d = 0; d < 3; ++d) { nc[ax][0][d] = cm[d]; nc[ax][1][d] = cp[d]; }
    }
    float up[5], um[5];
    load_cell(a, cp[0], cp[1], cp[2], up);
    load_cell(a, cm[0], cm[1], cm[2], um);
    const float s0 = wave_speed(u0, ax, a.gamma);
    const float sp = fmaxf(s0, wave_speed(up, ax, a.gamma));
    const float sm = fmaxf(s0, wave_speed(um, ax, a.gamma));
    nb[ax][0] = ((long long)cm[2] * L.ny + cm[1]) * L.nx + cm[0];
    nb[ax][1] = ((long long)cp[2] * L.ny + cp[1]) * L.nx + cp[0];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const float bp = a.beta * sp * fabsf(up[q] - u0[q]);
      const float bm = a.beta * sm * fabsf(u0[q] - um[q]);
      Fp[ax][q] = fminf(fmaxf(a.s[q] * __ldg(a.z3 + p * 16 + ax * 5 + q), -bp), bp);
      Fm[ax][q] = fminf(fmaxf(a.s[q] * __ldg(a.z3 + nb[ax][0] * 16 + ax * 5 + q), -bm), bm);
    }
  }
}

// Write un to the cell unless it breaks positivity (then count the switch-off).
__device__ __forceinline__ void gated_store(const FixArgs& a, const int c[3], const float un[5]) {
  const Layout& L = a.lay;
  const float ke = 0.5f * (un[1] * un[1] + un[2] * un[2] + un[3] * un[3]) / un[0];
  const float pr = (a.gamma - 1.f) * (un[4] - ke);
  if (un[0] > 0.f && pr > 0.f && isfinite(pr)) {
#pragma unroll
    for (int q = 0; q < 5; ++q) a.uout[L.idx(q, c[2] + 1, c[1] + 1, c[0] + 1)] = un[q];
  } else if (a.nswitch) {
    atomicAdd(a.nswitch, 1ull);
  }
}

// Interior cells of the correction kernels: one x1 row per block iteration,
// threads along the row, so (i, j, k) and the dense index p = row * nx + i
// need no 64-bit division.
template <class Body>
__device__ __forceinline__ void for_each_cell(const Layout& L, Body body) {
  const int rows = L.ny * L.nz;
  for (int row = blockIdx.x; row < rows; row += gridDim.x) {
    const int j = row % L.ny, k = row / L.ny;
    const long long p0 = (long long)row * L.nx;
    for (int i = threadIdx.x; i < L.nx; i += blockDim.x) {
      const int c[3] = {i, j, k};
      body(c, p0 + i);
    }
  }
}

__global__ void __launch_bounds__(128) closure_fix_kernel(const FixArgs a) {
  if (a.clk && !a.clk->active) return;
  const float cdt = a.coef * (a.clk ? (float)a.clk->dt : a.dt_host);
  const Layout& L = a.lay;
  for_each_cell(L, [&](const int c[3], long long p) {
    float Fp[3][5], Fm[3][5];
    long long nb[3][2];
    face_corrections(a, c, p, Fp, Fm, nb);
    float un[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      float r = 0.f;
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) r -= (Fp[ax][q] - Fm[ax][q]) * a.inv_h[ax];
      un[q] = a.uout[L.idx(q, c[2] + 1, c[1] + 1, c[0] + 1)] + cdt * r;
    }
    gated_store(a, c, un);
  });
}

// Flux-corrected transport (Zalesak 1979) bound on the corrections: the
// corrected stage result stays inside [min, max] of the plain stage result
// (uout before correction) over the cell and its six face neighbours, so the
// corrections create no new extrema.  Pass 1: per cell and variable the
// fractions R+ (of the summed inflows) and R- (of the summed outflows) that
// fit inside those bounds, ratio[q][p] and ratio[5+q][p].
__global__ void __launch_bounds__(128) fct_ratio_kernel(const FixArgs a) {
  if (a.clk && !a.clk->active) return;
  const float cdt = a.coef * (a.clk ? (float)a.clk->dt : a.dt_host);
  const Layout& L = a.lay;
  const long long n = (long long)L.nx * L.ny * L.nz;
  for_each_cell(L, [&](const int c[3], long long p) {
    float Fp[3][5], Fm[3][5];
    long long nb[3][2];
    int nc[3][2][3];
    face_corrections(a, c, p, Fp, Fm, nb, nc);
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const float ul = a.uout[L.idx(q, c[2] + 1, c[1] + 1, c[0] + 1)];
      float hi = ul, lo = ul, pin = 0.f, pout = 0.f;
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        // inflow through the +face is -cdt*Fp/h, through the -face +cdt*Fm/h
        const float tp = -cdt * Fp[ax][q] * a.inv_h[ax], tm = cdt * Fm[ax][q] * a.inv_h[ax];
        pin += fmaxf(tp, 0.f) + fmaxf(tm, 0.f);
        pout += fmaxf(-tp, 0.f) + fmaxf(-tm, 0.f);
#pragma unroll
        for (int sd = 0; sd < 2; ++sd) {
          const int* m = nc[ax][sd];
          const float un = a.uout[L.idx(q, m[2] + 1, m[1] + 1, m[0] + 1)];
          hi = fmaxf(hi, un);
          lo = fminf(lo, un);
        }
      }
      a.ratio[(long long)q * n + p] = pin > 0.f ? fminf(1.f, (hi - ul) / pin) : 1.f;
      a.ratio[(long long)(5 + q) * n + p] = pout > 0.f ? fminf(1.f, (ul - lo) / pout) : 1.f;
    }
  });
}

// Pass 2: each face transfer T (from the lower to the upper cell) is scaled
// by C = min(R+ of the receiving cell, R- of the giving cell), the same factor
// seen from both cells, so the limited correction stays conservative.
__global__ void __launch_bounds__(128) fct_apply_kernel(const FixArgs a) {
  if (a.clk && !a.clk->active) return;
  const float cdt = a.coef * (a.clk ? (float)a.clk->dt : a.dt_host);
  const Layout& L = a.lay;
  const long long n = (long long)L.nx * L.ny * L.nz;
  for_each_cell(L, [&](const int c[3], long long p) {
    float Fp[3][5], Fm[3][5];
    long long nb[3][2];
    face_corrections(a, c, p, Fp, Fm, nb);
    float un[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
      const float* Rp = a.ratio + (long long)q * n;        // R+
      const float* Rm = a.ratio + (long long)(5 + q) * n;  // R-
      const float rp0 = Rp[p], rm0 = Rm[p];
      float d = 0.f;
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        // +face: transfer T from this cell to the one above
        const float T = cdt * Fp[ax][q] * a.inv_h[ax];
        const long long up = nb[ax][1], dn = nb[ax][0];
        const float Cp = T >= 0.f ? fminf(Rp[up], rm0) : fminf(rp0, Rm[up]);
        // -face: transfer T' from the cell below to this one
        const float Tm = cdt * Fm[ax][q] * a.inv_h[ax];
        const float Cm = Tm >= 0.f ? fminf(rp0, Rm[dn]) : fminf(Rp[dn], rm0);
        d += Cm * Tm - Cp * T;
      }
      un[q] = a.uout[L.idx(q, c[2] + 1, c[1] + 1, c[0] + 1)] + d;
    }
    gated_store(a, c, un);
  });
}

}  // namespace closure
}  // namespace fvm
