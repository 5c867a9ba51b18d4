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
// fused kernel, forward_fused_kernel: weights staged in shared memory,
// ldmatrix-fed mma.sync.m16n8k16, both layers and the output head without a
// round trip through memory.  The training products (at most 256 rows) are
// one warp per 16 x 8 output tile issuing mma.sync.m16n8k16 (BF16 in, FP32
// accumulate) on operands read straight from L2.  At these sizes (0.5 GFLOP
// a forward pass, tiles of 32 rows) the tcgen05/TMEM pipeline's set-up --
// TMEM allocation, descriptors, an mbarrier round trip per tile -- would not
// pay.
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

// ---- the fused inference forward ---------------------------------------------------
// y = w3 . relu(W2 relu(W1 x + b1) + b2) + b3 for kFuseRows rows a CTA, in one
// launch.  The CTA stages both weight matrices (BF16) and its rows of x in
// shared memory with one cp.async.bulk copy per row, all completing on one
// mbarrier, each row padded by 16 bytes so that the eight 16-byte rows an
// ldmatrix reads fall in eight different bank groups;
// ldmatrix.x4 feeds mma.sync.m16n8k16 (BF16 in, FP32 accumulate); the first
// hidden layer goes back to shared memory as BF16 after bias and ReLU, the
// second is never stored: each lane applies bias, ReLU and w3 to its
// accumulators and the row sums meet in shared memory.  Numerics as the
// unfused path (BF16 operands, FP32 accumulation, H1 rounded to BF16); only
// the summation order of the output dot product differs.  8 warps: warp w
// owns rows 16 (w % 2) .. +16 and output columns 64 (w / 2) .. +64.  With
// 64 rows and 16 warps a CTA, tensor-pipe activity rose from 16 % to 26 % of
// active cycles, but the 4096-row pass took 12.3 us against 10.5 us: half as
// many CTAs stage the weights.
constexpr int kFuseRows = 32;
constexpr int kFuseThreads = 32 * (kFuseRows / 16) * 4;   // a warp per (16-row tile, 64 columns)
constexpr int kLdW2 = kHidden + 8;      // padded row of W2 / H1 (bf16 elements)
constexpr int kLdW1 = kFeatures + 8;    // padded row of W1 / x
constexpr size_t kFuseSmem = ((size_t)kHidden * kLdW2 + (size_t)kHidden * kLdW1 + (size_t)kFuseRows * kLdW1 +
                              (size_t)kFuseRows * kLdW2) * sizeof(bf16) +
                             (3 * (size_t)kHidden + (size_t)kFuseRows * 4) * sizeof(float);

__device__ __forceinline__ void ldmatrix_x4(uint32_t (&r)[4], const bf16* p) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
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

// acc[nt][4] += A (16 rows at a, row stride lda) * B^T (8 * NT rows at b, row
// stride ldb) over K columns; A and B^T are [.][K] BF16 in shared memory.
template <int NT, int K>
__device__ __forceinline__ void warp_mma_tile(float (&acc)[NT][4], const bf16* a, int lda, const bf16* b, int ldb) {
  const int lane = threadIdx.x & 31;
  const int ar = lane & 15, ak = (lane >> 4) * 8;                 // A: rows 0-15, k halves
  const int bn = (lane >> 4) * 8 + (lane & 7), bk = ((lane >> 3) & 1) * 8;   // B: two n-tiles, k halves
  // unrolled: the next k-step's fragments load while this step's products issue
#pragma unroll
  for (int k0 = 0; k0 < K; k0 += 16) {
    uint32_t af[4];
    ldmatrix_x4(af, a + ar * lda + k0 + ak);
#pragma unroll
    for (int p = 0; p < NT / 2; ++p) {
      uint32_t bf[4];
      ldmatrix_x4(bf, b + (p * 16 + bn) * ldb + k0 + bk);
      mma_16816(acc[2 * p], af[0], af[1], af[2], af[3], bf[0], bf[1]);
      mma_16816(acc[2 * p + 1], af[0], af[1], af[2], af[3], bf[2], bf[3]);
    }
  }
}

__global__ void __launch_bounds__(kFuseThreads) forward_fused_kernel(const bf16* __restrict__ X, int rows,
                                                                      const bf16* __restrict__ W1b,
                                                                      const bf16* __restrict__ W2b,
                                                                      const float* __restrict__ params,
                                                                      float* __restrict__ y) {
  extern __shared__ uint4 s_fuse[];
  bf16* const W2s = reinterpret_cast<bf16*>(s_fuse);
  bf16* const W1s = W2s + kHidden * kLdW2;
  bf16* const Xs = W1s + kHidden * kLdW1;
  bf16* const H1s = Xs + kFuseRows * kLdW1;
  float* const b1s = reinterpret_cast<float*>(H1s + kFuseRows * kLdW2);
  float* const b2s = b1s + kHidden;
  float* const w3s = b2s + kHidden;
  float* const part = w3s + kHidden;   // [kFuseRows][4] partial output sums
  __shared__ alignas(8) unsigned long long s_bar;
  const int r0 = blockIdx.x * kFuseRows;
  const int valid = min(kFuseRows, rows - r0);
  // Staging: one bulk copy per matrix row (W2: 512 bytes, W1 and x: 64 bytes)
  // into the padded rows, all in flight at once, completing on one mbarrier.
  const unsigned bar = smem_u32(&s_bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned bytes = (unsigned)(kHidden * (kHidden + kFeatures) + valid * kFeatures) * (unsigned)sizeof(bf16);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
  }
  __syncthreads();
  asm volatile("fence.proxy.async.global;" ::: "memory");
  for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
    bulk_copy(W2s + i * kLdW2, W2b + (long long)i * kHidden, kHidden * sizeof(bf16), bar);
    bulk_copy(W1s + i * kLdW1, W1b + (long long)i * kFeatures, kFeatures * sizeof(bf16), bar);
  }
  for (int i = threadIdx.x; i < kFuseRows; i += blockDim.x) {
    if (i < valid) {
      bulk_copy(Xs + i * kLdW1, X + (long long)(r0 + i) * kFeatures, kFeatures * sizeof(bf16), bar);
    } else {
      for (int c = 0; c < kFeatures; c += 8) *reinterpret_cast<uint4*>(Xs + i * kLdW1 + c) = make_uint4(0u, 0u, 0u, 0u);
    }
  }
  for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
    b1s[i] = params[kOffB1 + i];
    b2s[i] = params[kOffB2 + i];
    w3s[i] = params[kOffW3 + i];
  }
  // bounded wait (2 s); a wait that runs out leaves NaN for this CTA's rows
  bool staged = mbar_try_wait_parity(bar, 0u);
  if (!staged) {
    const unsigned long long t0 = global_ns();
    while (!(staged = mbar_try_wait_parity(bar, 0u)))
      if (global_ns() - t0 > 2000000000ULL) break;
  }
  __syncthreads();
  if (__syncthreads_or(!staged)) {
    if (threadIdx.x < valid) y[r0 + threadIdx.x] = __int_as_float(0x7fc00000);
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kRowTiles = kFuseRows / 16;
  const int mrow = (warp % kRowTiles) * 16, ncol = (warp / kRowTiles) * 64;
  const int g = lane >> 2, t = lane & 3;
  // layer 1: H1 = relu(x W1^T + b1), K = 32
  {
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
    warp_mma_tile<8, kFeatures>(acc, Xs + mrow * kLdW1, kLdW1, W1s + ncol * kLdW1, kLdW1);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int n = ncol + i * 8 + 2 * t;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = mrow + g + (q >= 2 ? 8 : 0), nn = n + (q & 1);
        const float v = acc[i][q] + b1s[nn];
        H1s[m * kLdW2 + nn] = __float2bfloat16_rn(v > 0.f ? v : 0.f);
      }
    }
  }
  __syncthreads();
  // layer 2 and the head: y = w3 . relu(H1 W2^T + b2) + b3, K = 256
  float acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.f;
  warp_mma_tile<8, kHidden>(acc, H1s + mrow * kLdW2, kLdW2, W2s + ncol * kLdW2, kLdW2);
  float s_lo = 0.f, s_hi = 0.f;   // rows mrow + g and mrow + g + 8
#pragma unroll
  for (int i = 0; i < 8; ++i) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int nn = ncol + i * 8 + 2 * t + (q & 1);
      float v = acc[i][q] + b2s[nn];
      v = (v > 0.f ? v : 0.f) * w3s[nn];
      if (q < 2) s_lo += v; else s_hi += v;
    }
  }
#pragma unroll
  for (int o = 1; o < 4; o <<= 1) {
    s_lo += __shfl_xor_sync(0xffffffffu, s_lo, o);
    s_hi += __shfl_xor_sync(0xffffffffu, s_hi, o);
  }
  if (t == 0) {
    part[(mrow + g) * 4 + ncol / 64] = s_lo;
    part[(mrow + g + 8) * 4 + ncol / 64] = s_hi;
  }
  __syncthreads();
  if (threadIdx.x < valid) {
    const float* pr = part + threadIdx.x * 4;
    y[r0 + threadIdx.x] = ((pr[0] + pr[1]) + (pr[2] + pr[3])) + params[kOffB3];
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

// Adam on the FP32 master parameters, then the BF16 copies the products
// read (W1, W2 and W2 transposed).  The step counter lives on the device so
// that a replayed graph keeps counting; adam_step_kernel advances it after
// every block of this kernel has used it.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, const int* __restrict__ step, AdamHyper h, bf16* __restrict__ w1b,
                            bf16* __restrict__ w2b, bf16* __restrict__ w2tb) {
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
    if (i < kOffB1) {
      w1b[i] = __float2bfloat16_rn(pi);
    } else if (i >= kOffW2 && i < kOffB2) {
      const int q = i - kOffW2, n = q / kHidden, k = q % kHidden;
      const bf16 v = __float2bfloat16_rn(pi);
      w2b[q] = v;
      w2tb[k * kHidden + n] = v;
    }
  }
}

__global__ void adam_step_kernel(int* step) { *step += 1; }

// BF16 copies of freshly written FP32 parameters.
__global__ void cast_params_kernel(const float* __restrict__ p, bf16* __restrict__ w1b, bf16* __restrict__ w2b,
                                   bf16* __restrict__ w2tb) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kParams; i += gridDim.x * blockDim.x) {
    if (i < kOffB1) {
      w1b[i] = __float2bfloat16_rn(p[i]);
    } else if (i >= kOffW2 && i < kOffB2) {
      const int q = i - kOffW2, n = q / kHidden, k = q % kHidden;
      const bf16 v = __float2bfloat16_rn(p[i]);
      w2b[q] = v;
      w2tb[k * kHidden + n] = v;
    }
  }
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
    // inference: one fused launch, the activations never leave the SM
    forward_fused_kernel<<<(rows + kFuseRows - 1) / kFuseRows, kFuseThreads, kFuseSmem, st>>>(X, rows, m->W1b, m->W2b,
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
                                                     m->W2tb);
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
  MCUDA(cudaFuncSetAttribute((const void*)forward_fused_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)kFuseSmem));
  const size_t R = (size_t)max_rows;
  if ((rc = mdev(&m->p, kParams)) || (rc = mdev(&m->g, kParams)) || (rc = mdev(&m->m1, kParams)) ||
      (rc = mdev(&m->m2, kParams)) || (rc = mdev(&m->step, 1)) || (rc = mdev(&m->W1b, (size_t)kOffB1)) ||
      (rc = mdev(&m->W2b, (size_t)kHidden * kHidden)) || (rc = mdev(&m->W2tb, (size_t)kHidden * kHidden)) ||
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
                  (void*)m->W2tb, (void*)m->H1, (void*)m->H2, (void*)m->Z2, (void*)m->y_train, (void*)m->dZ2,
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
  cast_params_kernel<<<64, 256>>>(m->p, m->W1b, m->W2b, m->W2tb);
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
