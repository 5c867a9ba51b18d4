// mlp.cu -- the learned proposal filter's network: a 32 -> 256 -> 256 -> 1
// ReLU MLP on BF16 tensor cores with FP32 accumulation, with hand-written
// forward, backward and Adam kernels.  The annealing engine ranks thousands
// of candidate swaps with it every step and trains it online on the exact
// changes of ASPL the evaluator measures for the candidates it evaluates.
// No counterpart in the reference, whose annealing draws one random swap at a
// time (general/sa.c:217-369).
//
// Numerics (the CPU oracle restates them): inputs and weights are rounded to
// BF16; every product is accumulated in FP32; the first hidden layer is
// stored as BF16 after bias and ReLU; the second stays FP32 and feeds the FP32
// output dot product.  Backward: dy = 2 (y - t) / B; the gradients that enter
// a tensor-core product (dZ2, dZ1) are rounded to BF16; weight and bias
// gradients are FP32.
//
// The inference forward that ranks the proposals (4096 rows a step) is one
// kernel on the fifth-generation tensor cores, forward_tc_kernel: per 128
// rows, tcgen05.mma with both layers' FP32 accumulators in tensor memory,
// operands staged in shared memory by bulk copies, bias, ReLU and the output
// head applied between tcgen05.ld and the next product, no round trip through
// global memory.  It replaced an mma.sync kernel of the same fusion (ldmatrix
// fragments, 32 rows a CTA): 8.2 us against 10.3 us for 4096 rows.  The
// training products (at most 256 rows, with the pre-activations the backward
// needs) are one warp per 16 x 8 output tile issuing mma.sync.m16n8k16 (BF16
// in, FP32 accumulate) on operands read straight from L2.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/graphgolf_b200.h"
#include "core_internal.h"
#include "mlp_internal.h"

using ggb::core_fail;

#define MCUDA(call)                                                                                  \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return core_fail(GGB_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                       __LINE__);                                                                    \
  } while (0)

namespace ggb {
namespace mlp {

using bf16 = __nv_bfloat16;

__device__ __forceinline__ uint32_t ld_pair(const bf16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// D = A (16x16, row) * B (16x8, col) + D, BF16 inputs, FP32 accumulators.
__device__ __forceinline__ void mma_16816(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                          uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

enum Epi : int {
  kEpiBiasReluBf16 = 0,   // out_b[m][n] = bf16(relu(c + bias[n]))
  kEpiBiasReluF32 = 1,    // out_f[m][n] = relu(c + bias[n]); out_z[m][n] = c + bias[n] (if out_z)
  kEpiF32 = 2,            // out_f[m][n] = c
  kEpiMask = 3,           // v = c * (mask[m][n] > 0): out_b = bf16(v), out_f = v
};

struct EpiArgs {
  const float* bias;
  const bf16* mask;       // [M][N]
  bf16* out_b;
  float* out_f;
  float* out_z;
};

// C[M][N] = A[M][K] * Bt[N][K]^T with the epilogue EPI; M % 16 == 0,
// N % 8 == 0, K % 16 == 0, lda/ldb even.  One warp per 16 x 8 tile.
template <int EPI>
__global__ void __launch_bounds__(128) gemm_tn_kernel(int M, int N, int K, const bf16* __restrict__ A, int lda,
                                                      const bf16* __restrict__ Bt, int ldb, EpiArgs e) {
  const int lane = threadIdx.x & 31;
  const long long tile = (long long)blockIdx.x * 4 + (threadIdx.x >> 5);
  const int tiles_n = N / 8;
  if (tile >= (long long)(M / 16) * tiles_n) return;
  const int m0 = (int)(tile / tiles_n) * 16, n0 = (int)(tile % tiles_n) * 8;
  const int g = lane >> 2, t = lane & 3;
  float c[4] = {0.f, 0.f, 0.f, 0.f};
  const bf16* a_r0 = A + (long long)(m0 + g) * lda + 2 * t;
  const bf16* a_r1 = a_r0 + 8LL * lda;
  const bf16* b_n = Bt + (long long)(n0 + g) * ldb + 2 * t;
  for (int k0 = 0; k0 < K; k0 += 16) {
    const uint32_t a0 = ld_pair(a_r0 + k0), a1 = ld_pair(a_r1 + k0);
    const uint32_t a2 = ld_pair(a_r0 + k0 + 8), a3 = ld_pair(a_r1 + k0 + 8);
    const uint32_t b0 = ld_pair(b_n + k0), b1 = ld_pair(b_n + k0 + 8);
    mma_16816(c, a0, a1, a2, a3, b0, b1);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int m = m0 + g + (i >= 2 ? 8 : 0);
    const int n = n0 + 2 * t + (i & 1);
    const long long o = (long long)m * N + n;
    float v = c[i];
    if (EPI == kEpiBiasReluBf16) {
      v += e.bias[n];
      e.out_b[o] = __float2bfloat16_rn(v > 0.f ? v : 0.f);
    } else if (EPI == kEpiBiasReluF32) {
      v += e.bias[n];
      if (e.out_z) e.out_z[o] = v;
      e.out_f[o] = v > 0.f ? v : 0.f;
    } else if (EPI == kEpiF32) {
      e.out_f[o] = v;
    } else {
      v = __bfloat162float(e.mask[o]) > 0.f ? v : 0.f;
      e.out_b[o] = __float2bfloat16_rn(v);
      e.out_f[o] = v;
    }
  }
}

// Bulk copies global -> shared (cp.async.bulk, completion on an mbarrier).
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait_parity(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---- the tcgen05 inference forward ---------------------------------------------------
// The same y = w3 . relu(W2 relu(W1 x + b1) + b2) + b3, on the fifth-generation
// tensor cores: one CTA per 128 rows (M of one tcgen05.mma), both layers'
// accumulators in tensor memory (TMEM), operands in shared memory.
//   * Staging: W1 and W2 sit in global memory already in the operand layout
//     (written by the cast and Adam kernels), so bulk copies bring them in:
//     W1 (16 KB) on one mbarrier, W2 (8 x 16 KB) on another, so that layer 1
//     and its epilogue run while W2 is still arriving; the CTA's rows of x are
//     stored into the same layout by plain 16-byte stores.
//   * Layer 1: two tcgen05.mma (M 128, N 256, K 16) into TMEM columns 0-255.
//   * Epilogue 1: warp w reads TMEM lanes 32 (w % 4) .. +32 (its rows) and
//     columns 128 (w / 4) .. +128 with tcgen05.ld, adds b1, applies ReLU,
//     rounds to BF16 and stores H1 in the operand layout.
//   * Layer 2: sixteen tcgen05.mma (K 16 each) into columns 256-511.
//   * Epilogue 2: bias, ReLU and the w3 dot product per thread (a thread owns
//     a row), the two column halves added in shared memory.
// One thread issues the MMAs; tcgen05.commit arrives on an mbarrier that the
// CTA waits on (bounded by %globaltimer, 2 s; a wait that runs out leaves
// NaN for the CTA's rows).  Numerics as the other forwards: BF16 operands,
// FP32 accumulation, H1 rounded to BF16.
namespace tc {
constexpr int kRows = 128;
constexpr int kThreads = 256;
constexpr uint32_t kW2Bytes = kHidden * kHidden * 2;      // 131072
constexpr uint32_t kW1Bytes = kHidden * kFeatures * 2;    // 16384
constexpr uint32_t kXBytes = kRows * kFeatures * 2;       // 8192
constexpr uint32_t kH1Bytes = kRows * kHidden * 2;        // 65536
constexpr uint32_t kSOffW1 = kW2Bytes;
constexpr uint32_t kSOffX = kSOffW1 + kW1Bytes;
constexpr uint32_t kSOffH1 = kSOffX + kXBytes;
constexpr uint32_t kSOffVec = kSOffH1 + kH1Bytes;          // b1, b2, w3 (FP32)
constexpr uint32_t kSOffPart = kSOffVec + 3 * kHidden * 4; // [kRows][2] FP32
constexpr size_t kSmem = kSOffPart + kRows * 2 * 4;
constexpr uint32_t kTmemCols = 512;                       // layer 1: 0-255, layer 2: 256-511
// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A and
// B BF16 (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0), N >> 3
// in bits 17-22, M >> 4 in bits 24-28.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kHidden >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);
static_assert(kSmem + 1024 <= 227 * 1024, "the operands and the static barriers must fit one CTA's shared memory");
}  // namespace tc

// Element offset of (row r, column k) of a [rows][K] BF16 operand in the
// K-major, no-swizzle layout: 8 x 8 core matrices of 128 contiguous bytes,
// core (r / 8, k / 8) at byte (r / 8) * 16 K + (k / 8) * 128.  Descriptor:
// leading-dimension offset 128 bytes (next 8 columns), stride offset 16 K
// bytes (next 8 rows).
__host__ __device__ constexpr int umma_k_off(int r, int k, int K) {
  return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

// Shared-memory matrix descriptor: start, leading and stride byte offsets in
// 16-byte units, descriptor version 1 (bits 46-47), no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void umma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
        "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
        "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity) {
  if (mbar_try_wait_parity(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  while (!mbar_try_wait_parity(bar, parity))
    if (global_ns() - t0 > 2000000000ULL) return false;
  return true;
}

__global__ void __launch_bounds__(tc::kThreads, 1) forward_tc_kernel(const bf16* __restrict__ X, int rows,
                                                                   const bf16* __restrict__ W1u,
                                                                   const bf16* __restrict__ W2u,
                                                                   const float* __restrict__ params,
                                                                   float* __restrict__ y) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char s_tc[];
  __shared__ alignas(8) unsigned long long s_bars[3];   // [0] W1 staged, [1] MMA completion, [2] W2 staged
  __shared__ uint32_t s_tmem;
  __shared__ int s_ok;
  bf16* const W2s = reinterpret_cast<bf16*>(s_tc);
  bf16* const W1s = reinterpret_cast<bf16*>(s_tc + kSOffW1);
  bf16* const Xs = reinterpret_cast<bf16*>(s_tc + kSOffX);
  bf16* const H1s = reinterpret_cast<bf16*>(s_tc + kSOffH1);
  float* const b1s = reinterpret_cast<float*>(s_tc + kSOffVec);
  float* const b2s = b1s + kHidden;
  float* const w3s = b2s + kHidden;
  float* const part = reinterpret_cast<float*>(s_tc + kSOffPart);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.x * kRows;
  const int valid = min(kRows, rows - r0);
  const unsigned bar_st = smem_u32(&s_bars[0]), bar_mma = smem_u32(&s_bars[1]), bar_w2 = smem_u32(&s_bars[2]);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_st) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_mma) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar_w2) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    // W1 first, on its own barrier: layer 1 and its epilogue run while W2 arrives
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_st), "r"(kW1Bytes) : "memory");
    bulk_copy(W1s, W1u, kW1Bytes, bar_st);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar_w2), "r"(kW2Bytes) : "memory");
    for (uint32_t c = 0; c < kW2Bytes; c += 16384u)
      bulk_copy(s_tc + c, reinterpret_cast<const unsigned char*>(W2u) + c, 16384u, bar_w2);
  }
  // this CTA's rows of x (zeros past the last row) into the operand layout
  for (int i = tid; i < kRows * (kFeatures / 8); i += kThreads) {
    const int r = i / (kFeatures / 8), c = (i % (kFeatures / 8)) * 8;
    uint4 v = make_uint4(0u, 0u, 0u, 0u);
    if (r < valid) v = *reinterpret_cast<const uint4*>(X + (long long)(r0 + r) * kFeatures + c);
    *reinterpret_cast<uint4*>(Xs + umma_k_off(r, c, kFeatures)) = v;
  }
  for (int i = tid; i < kHidden; i += kThreads) {
    b1s[i] = params[kOffB1 + i];
    b2s[i] = params[kOffB2 + i];
    w3s[i] = params[kOffW3 + i];
  }
  // the generic-proxy stores of x must be visible to the tensor cores' reads
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = s_tmem;
  if (tid == 0) {
    const bool staged = mbar_wait_bounded(bar_st, 0u);
    if (staged) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < kFeatures / 16; ++ks)
        umma_bf16(tmem, umma_desc(smem_u32(Xs) + 256u * ks, 128u, 16u * kFeatures),
                  umma_desc(smem_u32(W1s) + 256u * ks, 128u, 16u * kFeatures), kIdesc, ks > 0);
      umma_commit(bar_mma);
    }
    s_ok = staged;
  }
  __syncthreads();
  const bool ok1 = s_ok && mbar_wait_bounded(bar_mma, 0u);
  const int q = warp & 3, h = warp >> 2;
  const int row = 32 * q + lane;
  const uint32_t lane_base = tmem + ((uint32_t)(32 * q) << 16);
  bool failed = __syncthreads_or(!ok1);
  if (!failed) {
    tc_fence_after();
    // epilogue 1: H1 = bf16(relu(acc + b1)) into the operand layout
#pragma unroll 1
    for (int j = 0; j < 4; ++j) {
      const int col0 = 128 * h + 32 * j;
      uint32_t v[32];
      tmem_ld32(lane_base + (uint32_t)col0, v);
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        uint32_t pk[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int c = col0 + 8 * m + 2 * e;
          const float f0 = fmaxf(__uint_as_float(v[8 * m + 2 * e]) + b1s[c], 0.f);
          const float f1 = fmaxf(__uint_as_float(v[8 * m + 2 * e + 1]) + b1s[c + 1], 0.f);
          const __nv_bfloat162 b2v = __floats2bfloat162_rn(f0, f1);
          pk[e] = *reinterpret_cast<const uint32_t*>(&b2v);
        }
        *reinterpret_cast<uint4*>(H1s + umma_k_off(row, col0 + 8 * m, kHidden)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
      }
    }
    bool w2_ok = true;
    if (tid == 0) w2_ok = mbar_wait_bounded(bar_w2, 0u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    failed = __syncthreads_or(!w2_ok);
  }
  if (!failed) {
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int ks = 0; ks < kHidden / 16; ++ks)
        umma_bf16(tmem + (uint32_t)kHidden, umma_desc(smem_u32(H1s) + 256u * ks, 128u, 16u * kHidden),
                  umma_desc(smem_u32(W2s) + 256u * ks, 128u, 16u * kHidden), kIdesc, ks > 0);
      umma_commit(bar_mma);
    }
    const bool ok2 = mbar_wait_bounded(bar_mma, 1u);
    failed = __syncthreads_or(!ok2);
    if (!failed) {
      tc_fence_after();
      // epilogue 2: this thread's row, columns 128 h .. +128
      float s = 0.f;
#pragma unroll 1
      for (int j = 0; j < 4; ++j) {
        const int col0 = 128 * h + 32 * j;
        uint32_t v[32];
        tmem_ld32(lane_base + (uint32_t)(kHidden + col0), v);
#pragma unroll
        for (int e = 0; e < 32; ++e) s = fmaf(fmaxf(__uint_as_float(v[e]) + b2s[col0 + e], 0.f), w3s[col0 + e], s);
      }
      part[row * 2 + h] = s;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid < valid) y[r0 + tid] = failed ? __int_as_float(0x7fc00000) : (part[2 * tid] + part[2 * tid + 1]) + params[kOffB3];
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
  }
}

// y[r] = H2[r][:] . w3 + b3 (one warp per row, fixed summation order).
__global__ void head_kernel(const float* __restrict__ H2, const float* __restrict__ w3, const float* __restrict__ b3,
                            float* __restrict__ y, int rows) {
  const int lane = threadIdx.x & 31;
  const long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= rows) return;
  float s = 0.f;
  for (int n = lane; n < kHidden; n += 32) s = fmaf(H2[r * kHidden + n], w3[n], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[r] = s + b3[0];
}

// Backward through the output layer for B rows: dy, dZ2 (BF16, both
// layouts), the gradients of w3, b3 and b2, and the loss.  One block of 256
// threads: thread n owns hidden unit n.
__global__ void __launch_bounds__(kHidden) out_backward_kernel(const float* __restrict__ y,
                                                               const float* __restrict__ t,
                                                               const float* __restrict__ Z2,
                                                               const float* __restrict__ H2,
                                                               const float* __restrict__ w3, int B,
                                                               bf16* __restrict__ dZ2, bf16* __restrict__ dZ2t,
                                                               float* __restrict__ grad, float* __restrict__ loss) {
  __shared__ float s_dy[kMaxTrainRows];
  const int n = threadIdx.x;
  for (int r = n; r < B; r += kHidden) s_dy[r] = 2.f * (y[r] - t[r]) / (float)B;
  __syncthreads();
  const float wn = w3[n];
  float gw3 = 0.f, gb2 = 0.f;
  for (int r = 0; r < B; ++r) {
    const float dy = s_dy[r];
    gw3 = fmaf(dy, H2[(long long)r * kHidden + n], gw3);
    const float dz = Z2[(long long)r * kHidden + n] > 0.f ? dy * wn : 0.f;
    const bf16 db = __float2bfloat16_rn(dz);
    dZ2[(long long)r * kHidden + n] = db;
    dZ2t[(long long)n * B + r] = db;
    gb2 += dz;
  }
  grad[kOffW3 + n] = gw3;
  grad[kOffB2 + n] = gb2;
  if (n == 0) {
    float gb3 = 0.f, l = 0.f;
    for (int r = 0; r < B; ++r) {
      gb3 += s_dy[r];
      const float d = y[r] - t[r];
      l = fmaf(d, d, l);
    }
    grad[kOffB3] = gb3;
    if (loss) *loss = l / (float)B;
  }
}

// out[c][r] = in[r][c] for a rows x cols BF16 matrix.
__global__ void transpose_bf16_kernel(const bf16* __restrict__ in, bf16* __restrict__ out, int rows, int cols) {
  const long long n = (long long)rows * cols;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / cols), c = (int)(i % cols);
    out[(long long)c * rows + r] = in[i];
  }
}

// grad[off + c] = sum_r in[r][c] (fixed order).
__global__ void col_sum_kernel(const float* __restrict__ in, int rows, int cols, float* __restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += in[(long long)r * cols + c];
  out[c] = s;
}

// The BF16 copies of parameter i (value v) that the products read: W1 and
// W2 row-major, W2 transposed, and W1 / W2 in the tcgen05 operand layout.
__device__ __forceinline__ void store_bf16_copies(int i, float v, bf16* __restrict__ w1b, bf16* __restrict__ w2b,
                                                  bf16* __restrict__ w2tb, bf16* __restrict__ w1u,
                                                  bf16* __restrict__ w2u) {
  const bf16 b = __float2bfloat16_rn(v);
  if (i < kOffB1) {
    w1b[i] = b;
    w1u[umma_k_off(i / kFeatures, i % kFeatures, kFeatures)] = b;
  } else if (i >= kOffW2 && i < kOffB2) {
    const int q = i - kOffW2, n = q / kHidden, k = q % kHidden;
    w2b[q] = b;
    w2tb[k * kHidden + n] = b;
    w2u[umma_k_off(n, k, kHidden)] = b;
  }
}

// Adam on the FP32 master parameters, then the BF16 copies the products
// read (W1, W2 and W2 transposed).  The step counter lives on the device so
// that a replayed graph keeps counting; adam_step_kernel advances it after
// every block of this kernel has used it.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, const int* __restrict__ step, AdamHyper h, bf16* __restrict__ w1b,
                            bf16* __restrict__ w2b, bf16* __restrict__ w2tb, bf16* __restrict__ w1u,
                            bf16* __restrict__ w2u) {
  const int t = *step + 1;
  const float c1 = 1.f / (1.f - powf(h.beta1, (float)t));
  const float c2 = 1.f / (1.f - powf(h.beta2, (float)t));
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float a = h.beta1 * m1[i] + (1.f - h.beta1) * gi;
    const float b = h.beta2 * m2[i] + (1.f - h.beta2) * gi * gi;
    m1[i] = a;
    m2[i] = b;
    const float pi = p[i] - h.lr * (a * c1) / (sqrtf(b * c2) + h.eps);
    p[i] = pi;
    store_bf16_copies(i, pi, w1b, w2b, w2tb, w1u, w2u);
  }
}

__global__ void adam_step_kernel(int* step) { *step += 1; }

// BF16 copies of freshly written FP32 parameters.
__global__ void cast_params_kernel(const float* __restrict__ p, bf16* __restrict__ w1b, bf16* __restrict__ w2b,
                                   bf16* __restrict__ w2tb, bf16* __restrict__ w1u, bf16* __restrict__ w2u) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x)
    store_bf16_copies(i, p[i], w1b, w2b, w2tb, w1u, w2u);
}

// Rows idx[0..B) of X (rows 0..B when idx is null) into Xs.
__global__ void gather_rows_kernel(const bf16* __restrict__ X, const int* __restrict__ idx, int B,
                                   bf16* __restrict__ Xs) {
  const int n = B * kFeatures;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = i / kFeatures, c = i % kFeatures;
    const int src = idx ? idx[r] : r;
    Xs[i] = X[(long long)src * kFeatures + c];
  }
}

int blocks_for(long long tiles) { return (int)((tiles + 3) / 4); }

}  // namespace mlp

using namespace mlp;

// ---- enqueue helpers the annealing engine uses ---------------------------------

int mlp_forward(ggb_mlp* m, const bf16* X, int rows, float* y, cudaStream_t st, bool keep_z) {
  if (rows % 16 || rows > m->max_rows) return core_fail(GGB_EINVAL, "mlp rows %d (max %d, multiple of 16)", rows, m->max_rows);
  if (!keep_z) {
    // inference: one fused launch on the tcgen05 tensor cores, the activations never leave the SM
    forward_tc_kernel<<<(rows + tc::kRows - 1) / tc::kRows, tc::kThreads, tc::kSmem, st>>>(X, rows, m->W1u, m->W2u,
                                                                                         m->p, y);
    core_add_launches(1);
    MCUDA(cudaGetLastError());
    return GGB_OK;
  }
  EpiArgs e1 = {m->p + kOffB1, nullptr, m->H1, nullptr, nullptr};
  gemm_tn_kernel<kEpiBiasReluBf16><<<blocks_for((long long)(rows / 16) * (kHidden / 8)), 128, 0, st>>>(
      rows, kHidden, kFeatures, X, kFeatures, m->W1b, kFeatures, e1);
  EpiArgs e2 = {m->p + kOffB2, nullptr, nullptr, m->H2, keep_z ? m->Z2 : nullptr};
  gemm_tn_kernel<kEpiBiasReluF32><<<blocks_for((long long)(rows / 16) * (kHidden / 8)), 128, 0, st>>>(
      rows, kHidden, kHidden, m->H1, kHidden, m->W2b, kHidden, e2);
  head_kernel<<<(rows + 7) / 8, 256, 0, st>>>(m->H2, m->p + kOffW3, m->p + kOffB3, y, rows);
  core_add_launches(3);
  MCUDA(cudaGetLastError());
  return GGB_OK;
}

int mlp_backward(ggb_mlp* m, const bf16* Xs, const float* t, int B, cudaStream_t st) {
  if (B % 16 || B > kMaxTrainRows || B > m->max_rows) return core_fail(GGB_EINVAL, "mlp training rows %d", B);
  int rc = mlp_forward(m, Xs, B, m->y_train, st, true);
  if (rc) return rc;
  out_backward_kernel<<<1, kHidden, 0, st>>>(m->y_train, t, m->Z2, m->H2, m->p + kOffW3, B, m->dZ2, m->dZ2t, m->g,
                                             m->loss);
  transpose_bf16_kernel<<<64, 256, 0, st>>>(m->H1, m->H1t, B, kHidden);
  // gW2[n][k] = sum_r dZ2[r][n] H1[r][k]:  A = dZ2t [256][B], Bt = H1t [256][B]
  EpiArgs e2 = {nullptr, nullptr, nullptr, m->g + kOffW2, nullptr};
  gemm_tn_kernel<kEpiF32><<<blocks_for((kHidden / 16) * (kHidden / 8)), 128, 0, st>>>(kHidden, kHidden, B, m->dZ2t, B,
                                                                                   m->H1t, B, e2);
  // dZ1[r][k] = (sum_n dZ2[r][n] W2[n][k]) * (H1[r][k] > 0):  A = dZ2 [B][256], Bt = W2t [256][256]
  EpiArgs e3 = {nullptr, m->H1, m->dZ1, m->dZ1f, nullptr};
  gemm_tn_kernel<kEpiMask><<<blocks_for((long long)(B / 16) * (kHidden / 8)), 128, 0, st>>>(B, kHidden, kHidden, m->dZ2,
                                                                                        kHidden, m->W2tb, kHidden, e3);
  col_sum_kernel<<<1, kHidden, 0, st>>>(m->dZ1f, B, kHidden, m->g + kOffB1);
  transpose_bf16_kernel<<<64, 256, 0, st>>>(m->dZ1, m->dZ1t, B, kHidden);
  transpose_bf16_kernel<<<16, 256, 0, st>>>(Xs, m->Xt, B, kFeatures);
  // gW1[k][j] = sum_r dZ1[r][k] X[r][j]:  A = dZ1t [256][B], Bt = Xt [32][B]
  EpiArgs e4 = {nullptr, nullptr, nullptr, m->g + kOffW1, nullptr};
  gemm_tn_kernel<kEpiF32><<<blocks_for((kHidden / 16) * (kFeatures / 8)), 128, 0, st>>>(kHidden, kFeatures, B, m->dZ1t,
                                                                                     B, m->Xt, B, e4);
  core_add_launches(7);
  MCUDA(cudaGetLastError());
  return GGB_OK;
}

int mlp_adam(ggb_mlp* m, cudaStream_t st) {
  adam_kernel<<<(kParams + 255) / 256, 256, 0, st>>>(m->p, m->g, m->m1, m->m2, m->step, m->hyper, m->W1b, m->W2b,
                                                     m->W2tb, m->W1u, m->W2u);
  adam_step_kernel<<<1, 1, 0, st>>>(m->step);
  core_add_launches(2);
  MCUDA(cudaGetLastError());
  return GGB_OK;
}

int mlp_train_rows(ggb_mlp* m, const bf16* X, const int* idx, const float* t, int B, cudaStream_t st) {
  gather_rows_kernel<<<8, 256, 0, st>>>(X, idx, B, m->Xs);
  core_add_launches(1);
  int rc = mlp_backward(m, m->Xs, t, B, st);
  if (rc) return rc;
  return mlp_adam(m, st);
}

size_t mlp_state_bytes() { return 3 * (size_t)kParams * sizeof(float) + sizeof(int); }

int mlp_save_state(ggb_mlp* m, void* host) {
  unsigned char* h = static_cast<unsigned char*>(host);
  const size_t pb = (size_t)kParams * sizeof(float);
  MCUDA(cudaDeviceSynchronize());
  MCUDA(cudaMemcpy(h, m->p, pb, cudaMemcpyDeviceToHost));
  MCUDA(cudaMemcpy(h + pb, m->m1, pb, cudaMemcpyDeviceToHost));
  MCUDA(cudaMemcpy(h + 2 * pb, m->m2, pb, cudaMemcpyDeviceToHost));
  MCUDA(cudaMemcpy(h + 3 * pb, m->step, sizeof(int), cudaMemcpyDeviceToHost));
  return GGB_OK;
}

int mlp_load_state(ggb_mlp* m, const void* host) {
  const unsigned char* h = static_cast<const unsigned char*>(host);
  const size_t pb = (size_t)kParams * sizeof(float);
  MCUDA(cudaDeviceSynchronize());
  MCUDA(cudaMemcpy(m->p, h, pb, cudaMemcpyHostToDevice));
  MCUDA(cudaMemcpy(m->m1, h + pb, pb, cudaMemcpyHostToDevice));
  MCUDA(cudaMemcpy(m->m2, h + 2 * pb, pb, cudaMemcpyHostToDevice));
  MCUDA(cudaMemcpy(m->step, h + 3 * pb, sizeof(int), cudaMemcpyHostToDevice));
  cast_params_kernel<<<64, 256>>>(m->p, m->W1b, m->W2b, m->W2tb, m->W1u, m->W2u);
  MCUDA(cudaGetLastError());
  MCUDA(cudaDeviceSynchronize());
  return GGB_OK;
}

}  // namespace ggb

namespace {

using ggb::mlp::bf16;

template <typename T>
int mdev(T** p, size_t n) {
  if (cudaMalloc(p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return core_fail(GGB_ENOMEM, "cudaMalloc of %zu bytes failed", n * sizeof(T));
  }
  return GGB_OK;
}

// He-uniform initial weights, zero biases, from a splitmix64 stream.
void init_params(std::vector<float>& p, unsigned long long seed) {
  unsigned long long s = seed ^ 0x6a09e667f3bcc909ULL;
  auto next = [&]() {
    s += 0x9e3779b97f4a7c15ULL;
    unsigned long long z = s;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  p.assign(ggb::mlp::kParams, 0.f);
  const double a1 = std::sqrt(6.0 / ggb::mlp::kFeatures), a2 = std::sqrt(6.0 / ggb::mlp::kHidden);
  for (int i = 0; i < ggb::mlp::kOffB1; ++i) p[i] = (float)((2.0 * next() - 1.0) * a1);
  for (int i = ggb::mlp::kOffW2; i < ggb::mlp::kOffB2; ++i) p[i] = (float)((2.0 * next() - 1.0) * a2);
  for (int i = ggb::mlp::kOffW3; i < ggb::mlp::kOffB3; ++i) p[i] = (float)((2.0 * next() - 1.0) * a2 * 0.1);
}

int create(ggb_mlp* m, int max_rows, unsigned long long seed) {
  using namespace ggb::mlp;
  m->max_rows = max_rows;
  int rc;
  MCUDA(cudaFuncSetAttribute((const void*)forward_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)tc::kSmem));
  const size_t R = (size_t)max_rows;
  if ((rc = mdev(&m->p, kParams)) || (rc = mdev(&m->g, kParams)) || (rc = mdev(&m->m1, kParams)) ||
      (rc = mdev(&m->m2, kParams)) || (rc = mdev(&m->step, 1)) || (rc = mdev(&m->W1b, (size_t)kOffB1)) ||
      (rc = mdev(&m->W2b, (size_t)kHidden * kHidden)) || (rc = mdev(&m->W2tb, (size_t)kHidden * kHidden)) ||
      (rc = mdev(&m->W1u, (size_t)kOffB1)) || (rc = mdev(&m->W2u, (size_t)kHidden * kHidden)) ||
      (rc = mdev(&m->H1, R * kHidden)) || (rc = mdev(&m->H2, R * kHidden)) || (rc = mdev(&m->Z2, R * kHidden)) ||
      (rc = mdev(&m->y_train, (size_t)kMaxTrainRows)) || (rc = mdev(&m->dZ2, (size_t)kMaxTrainRows * kHidden)) ||
      (rc = mdev(&m->dZ2t, (size_t)kMaxTrainRows * kHidden)) || (rc = mdev(&m->H1t, (size_t)kMaxTrainRows * kHidden)) ||
      (rc = mdev(&m->dZ1, (size_t)kMaxTrainRows * kHidden)) || (rc = mdev(&m->dZ1f, (size_t)kMaxTrainRows * kHidden)) ||
      (rc = mdev(&m->dZ1t, (size_t)kMaxTrainRows * kHidden)) || (rc = mdev(&m->Xt, (size_t)kMaxTrainRows * kFeatures)) ||
      (rc = mdev(&m->Xs, (size_t)kMaxTrainRows * kFeatures)) || (rc = mdev(&m->loss, 1)) ||
      (rc = mdev(&m->X, R * kFeatures)) || (rc = mdev(&m->y, R)) || (rc = mdev(&m->t, (size_t)kMaxTrainRows)))
    return rc;
  std::vector<float> p;
  init_params(p, seed);
  return ggb_mlp_set_params(m, p.data());
}

void destroy(ggb_mlp* m) {
  if (!m) return;
  for (void* q : {(void*)m->p, (void*)m->g, (void*)m->m1, (void*)m->m2, (void*)m->step, (void*)m->W1b, (void*)m->W2b,
                  (void*)m->W2tb, (void*)m->W1u, (void*)m->W2u, (void*)m->H1, (void*)m->H2, (void*)m->Z2, (void*)m->y_train, (void*)m->dZ2,
                  (void*)m->dZ2t, (void*)m->H1t, (void*)m->dZ1, (void*)m->dZ1f, (void*)m->dZ1t, (void*)m->Xt,
                  (void*)m->Xs, (void*)m->loss, (void*)m->X, (void*)m->y, (void*)m->t})
    cudaFree(q);
  cudaGetLastError();
  delete m;
}

// Host FP32 features -> device BF16 rows of m->X.
int upload_x(ggb_mlp* m, const float* x, int rows) {
  std::vector<bf16> xb((size_t)rows * ggb::mlp::kFeatures);
  for (size_t i = 0; i < xb.size(); ++i) xb[i] = __float2bfloat16_rn(x[i]);
  MCUDA(cudaMemcpy(m->X, xb.data(), xb.size() * sizeof(bf16), cudaMemcpyHostToDevice));
  return GGB_OK;
}

}  // namespace

extern "C" {

int ggb_mlp_create(int max_rows, unsigned long long seed, ggb_mlp** out) {
  if (!out || max_rows <= 0 || max_rows % 16) return core_fail(GGB_EINVAL, "max_rows must be a positive multiple of 16");
  *out = nullptr;
  ggb_mlp* m = new ggb_mlp();
  m->hyper = {1e-3f, 0.9f, 0.999f, 1e-8f};
  int rc = create(m, max_rows, seed);
  if (rc) {
    destroy(m);
    return rc;
  }
  *out = m;
  return GGB_OK;
}

void ggb_mlp_destroy(ggb_mlp* m) { destroy(m); }

int ggb_mlp_param_count(void) { return ggb::mlp::kParams; }

int ggb_mlp_set_params(ggb_mlp* m, const float* params) {
  using namespace ggb::mlp;
  if (!m || !params) return core_fail(GGB_EINVAL, "null pointer");
  MCUDA(cudaMemcpy(m->p, params, kParams * sizeof(float), cudaMemcpyHostToDevice));
  MCUDA(cudaMemset(m->m1, 0, kParams * sizeof(float)));
  MCUDA(cudaMemset(m->m2, 0, kParams * sizeof(float)));
  MCUDA(cudaMemset(m->step, 0, sizeof(int)));
  cast_params_kernel<<<64, 256>>>(m->p, m->W1b, m->W2b, m->W2tb, m->W1u, m->W2u);
  MCUDA(cudaGetLastError());
  MCUDA(cudaDeviceSynchronize());
  return GGB_OK;
}

int ggb_mlp_get_params(ggb_mlp* m, float* params) {
  if (!m || !params) return core_fail(GGB_EINVAL, "null pointer");
  MCUDA(cudaDeviceSynchronize());
  MCUDA(cudaMemcpy(params, m->p, ggb::mlp::kParams * sizeof(float), cudaMemcpyDeviceToHost));
  return GGB_OK;
}

int ggb_mlp_set_adam(ggb_mlp* m, float lr, float beta1, float beta2, float eps) {
  if (!m || !(lr > 0.f) || !(beta1 >= 0.f && beta1 < 1.f) || !(beta2 >= 0.f && beta2 < 1.f) || !(eps > 0.f))
    return core_fail(GGB_EINVAL, "bad Adam hyper-parameters");
  m->hyper = {lr, beta1, beta2, eps};
  return GGB_OK;
}

int ggb_mlp_forward_host(ggb_mlp* m, const float* x, int rows, float* y) {
  if (!m || !x || !y) return core_fail(GGB_EINVAL, "null pointer");
  if (rows <= 0 || rows % 16 || rows > m->max_rows) return core_fail(GGB_EINVAL, "rows must be a multiple of 16 up to max_rows");
  int rc = upload_x(m, x, rows);
  if (rc) return rc;
  rc = ggb::mlp_forward(m, m->X, rows, m->y, nullptr, false);
  if (rc) return rc;
  MCUDA(cudaMemcpy(y, m->y, (size_t)rows * sizeof(float), cudaMemcpyDeviceToHost));
  return GGB_OK;
}

int ggb_mlp_time_forward(ggb_mlp* m, const float* x, int rows, int reps, double* ms) {
  if (!m || !x || !ms) return core_fail(GGB_EINVAL, "null pointer");
  if (rows <= 0 || rows % 16 || rows > m->max_rows || reps <= 0)
    return core_fail(GGB_EINVAL, "rows must be a multiple of 16 up to max_rows, reps positive");
  int rc = upload_x(m, x, rows);
  if (rc) return rc;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float t = 0.f;
  if (e == cudaSuccess) {
    rc = ggb::mlp_forward(m, m->X, rows, m->y, st, false);   // warm-up
    if (rc == GGB_OK) e = cudaEventRecord(e0, st);
    for (int i = 0; i < reps && rc == GGB_OK && e == cudaSuccess; ++i)
      rc = ggb::mlp_forward(m, m->X, rows, m->y, st, false);
    if (rc == GGB_OK && e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (rc == GGB_OK && e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (rc == GGB_OK && e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  }
  if (e1) cudaEventDestroy(e1);
  if (e0) cudaEventDestroy(e0);
  if (st) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  if (rc) return rc;
  if (e != cudaSuccess) return core_fail(GGB_ECUDA, "forward timing: %s", cudaGetErrorString(e));
  *ms = (double)t / reps;
  return GGB_OK;
}

int ggb_mlp_grads_host(ggb_mlp* m, const float* x, const float* t, int rows, float* loss, float* grads) {
  if (!m || !x || !t || !grads) return core_fail(GGB_EINVAL, "null pointer");
  if (rows <= 0 || rows % 16 || rows > ggb::mlp::kMaxTrainRows || rows > m->max_rows)
    return core_fail(GGB_EINVAL, "training rows must be a multiple of 16 up to %d", ggb::mlp::kMaxTrainRows);
  int rc = upload_x(m, x, rows);
  if (rc) return rc;
  MCUDA(cudaMemcpy(m->t, t, (size_t)rows * sizeof(float), cudaMemcpyHostToDevice));
  rc = ggb::mlp_backward(m, m->X, m->t, rows, nullptr);
  if (rc) return rc;
  MCUDA(cudaDeviceSynchronize());
  MCUDA(cudaMemcpy(grads, m->g, ggb::mlp::kParams * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss) MCUDA(cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return GGB_OK;
}

int ggb_mlp_train_host(ggb_mlp* m, const float* x, const float* t, int rows, int steps, float* last_loss) {
  if (!m || !x || !t) return core_fail(GGB_EINVAL, "null pointer");
  if (rows <= 0 || rows % 16 || rows > ggb::mlp::kMaxTrainRows || rows > m->max_rows || steps <= 0)
    return core_fail(GGB_EINVAL, "training rows must be a multiple of 16 up to %d", ggb::mlp::kMaxTrainRows);
  int rc = upload_x(m, x, rows);
  if (rc) return rc;
  MCUDA(cudaMemcpy(m->t, t, (size_t)rows * sizeof(float), cudaMemcpyHostToDevice));
  for (int s = 0; s < steps; ++s) {
    rc = ggb::mlp_backward(m, m->X, m->t, rows, nullptr);
    if (rc) return rc;
    rc = ggb::mlp_adam(m, nullptr);
    if (rc) return rc;
  }
  MCUDA(cudaDeviceSynchronize());
  if (last_loss) MCUDA(cudaMemcpy(last_loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return GGB_OK;
}

}  // extern "C"
