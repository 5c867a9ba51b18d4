// apsp_probe.cu -- measures the ceiling the dense sweeps run against.
//
// The sweeps' working set (two bitset matrices of a source window) is
// L2-resident by design, so the roof that bounds them is not the HBM copy
// bandwidth but the rate at which L2 delivers bytes to the SMs.
// ggb_probe_l2_stream measures that ceiling: bulk copies of an L2-resident
// buffer into shared memory, which keep far more bytes in flight than
// registers can; bench.py reports it as the roofline's peak.
// ggb_probe_l2_gather times the sweeps' own access pattern -- every vertex
// ORs its own row and the rows of its d random neighbours out of a matrix of
// the same shape, with the same 32-byte accesses, one launch per sweep, at
// two CTAs per SM -- on buffers it allocates itself, and reports the sweep's
// algorithmic bytes per second, beside the peak.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/graphgolf_b200.h"
#include "apsp_kernel.cuh"

namespace {

// One sweep: every vertex ORs its own row and its d neighbours' rows and
// writes the result, with the accesses the evaluator's dense sweeps issue:
// 16-byte ld.global.cg for rows of one uint4 (windows of 64 or 128 sources),
// otherwise 32-byte ld.global.cg.v8 accesses, LP lanes a row (a half-warp for
// 512-byte rows, as in the 4096-source sweeps), U neighbour rows in flight.
template <int R>
__global__ void __launch_bounds__(512, 2) probe_gather_kernel(const uint4* __restrict__ src, uint4* __restrict__ dst,
                                                             const int* __restrict__ adj, int N, int d,
                                                             unsigned long long* sink) {
  constexpr int PARTS = R >= 2 ? R / 2 : 1;          // accesses per row (32 bytes each, 16 for R = 1)
  constexpr int LP = PARTS >= 32 ? 32 : PARTS;        // lanes per row
  constexpr int PPL = PARTS / LP;                     // accesses per lane and row
  constexpr int RPW = 32 / LP;                        // rows per warp step
  constexpr int U = R >= 2 ? 4 : 8;                   // neighbour rows in flight
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane / LP, li = lane % LP;
  const long long slot = ((long long)blockIdx.x * 16 + warp) * RPW + sub;
  const long long n_slots = (long long)gridDim.x * 16 * RPW;
  unsigned c = 0;
  for (long long v = slot; v < N; v += n_slots) {
    uint4 acc[PPL][2];
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      if constexpr (R >= 2) {
        ggb::ld_cg2(src + v * R + 2 * (li + p * LP), acc[p]);
      } else {
        acc[p][0] = __ldcg(src + v);
        acc[p][1] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    for (int j = 0; j < d; j += U) {
      uint4 x[U][PPL][2];
#pragma unroll
      for (int q = 0; q < U; ++q) {
        const int u = j + q < d ? __ldg(adj + v * d + j + q) : (int)v;
#pragma unroll
        for (int p = 0; p < PPL; ++p) {
          if constexpr (R >= 2) {
            ggb::ld_cg2(src + (long long)u * R + 2 * (li + p * LP), x[q][p]);
          } else {
            x[q][p][0] = __ldcg(src + u);
            x[q][p][1] = make_uint4(0u, 0u, 0u, 0u);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < U; ++q)
#pragma unroll
        for (int p = 0; p < PPL; ++p) {
          ggb::or_into(acc[p][0], x[q][p][0]);
          ggb::or_into(acc[p][1], x[q][p][1]);
        }
    }
#pragma unroll
    for (int p = 0; p < PPL; ++p) {
      if constexpr (R >= 2) {
        ggb::st_cg2(dst + v * R + 2 * (li + p * LP), acc[p]);
      } else {
        __stcg(dst + v, acc[p][0]);
      }
      c += ggb::popc4(acc[p][0]) + ggb::popc4(acc[p][1]);
    }
  }
  if (c == 0xffffffffu) atomicAdd(sink, 1ULL);   // keeps the loads alive
}

template <int R>
float time_sweeps(uint4* a, uint4* b, const int* adj, int N, int d, int iters, unsigned long long* sink, int sms) {
  constexpr int PARTS = R >= 2 ? R / 2 : 1;
  constexpr int RPW = 32 / (PARTS >= 32 ? 32 : PARTS);
  const long long want = ((long long)N + RPW * 16 - 1) / (RPW * 16);
  const int grid = (int)std::min<long long>(want, 2LL * sms);
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return -1.f;
  for (int w = 0; w < 3; ++w) probe_gather_kernel<R><<<grid, 512>>>(a, b, adj, N, d, sink);
  cudaEventRecord(e0);
  for (int it = 0; it < iters; ++it) {
    if (it & 1)
      probe_gather_kernel<R><<<grid, 512>>>(b, a, adj, N, d, sink);
    else
      probe_gather_kernel<R><<<grid, 512>>>(a, b, adj, N, d, sink);
  }
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / iters;
}

// ---- the L2 streaming roof ----------------------------------------------------
// One CTA per SM, one thread driving a ring of kStreamStages shared-memory
// stages: each stage receives a kStreamChunk-byte cp.async.bulk copy of the
// L2-resident buffer and is refilled as soon as its mbarrier completes, so
// about 192 KB per SM are in flight without any register holding them.  The
// data are not read by the threads: the probe measures how fast L2 delivers
// bytes to the SMs, the ceiling every L2-resident kernel runs under.  Every
// wait is bounded (2 s by %globaltimer); one that runs out sets *err and the
// remaining stages are drained with the same bound.
constexpr int kStreamStages = 6;
constexpr unsigned kStreamChunk = 32768;

__device__ __forceinline__ bool stream_wait(unsigned bar, unsigned parity) {
  unsigned long long t0 = 0;
  for (;;) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
    const unsigned long long t = ggb::globaltimer_ns();
    if (t0 == 0) t0 = t;
    else if (t - t0 > 2000000000ULL) return false;
  }
}

__global__ void __launch_bounds__(32, 1) probe_stream_kernel(const unsigned char* __restrict__ src, long long chunks,
                                                            int passes, int* err) {
  extern __shared__ __align__(128) unsigned char ring[];
  __shared__ alignas(8) unsigned long long bars[kStreamStages];
  if (threadIdx.x != 0) return;
  for (int s = 0; s < kStreamStages; ++s) {
    const unsigned b = (unsigned)__cvta_generic_to_shared(&bars[s]);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
  }
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  const long long per = chunks > blockIdx.x ? (chunks - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  const long long total = per * passes;
  bool ok = true;
  long long i = 0;
  for (; i < total; ++i) {
    const int s = (int)(i % kStreamStages);
    const unsigned b = (unsigned)__cvta_generic_to_shared(&bars[s]);
    const long long use = i / kStreamStages;
    if (use > 0 && !(ok = stream_wait(b, (unsigned)((use - 1) & 1)))) break;
    const long long c = blockIdx.x + (i % per) * (long long)gridDim.x;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kStreamChunk) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     (unsigned)__cvta_generic_to_shared(ring + (size_t)s * kStreamChunk)),
                 "l"(src + c * (long long)kStreamChunk), "r"(kStreamChunk), "r"(b)
                 : "memory");
  }
  // drain: the last use of every stage that was issued
  for (int s = 0; s < kStreamStages; ++s) {
    const long long uses = i > s ? (i - s + kStreamStages - 1) / kStreamStages : 0;
    if (uses == 0) continue;
    const unsigned b = (unsigned)__cvta_generic_to_shared(&bars[s]);
    if (!stream_wait(b, (unsigned)((uses - 1) & 1))) ok = false;
  }
  if (!ok) atomicExch(err, 1);
}

}  // namespace

// GB/s at which L2 delivers an L2-resident buffer of `mib` MiB (at most 96)
// to the SMs: bulk copies into shared memory, one CTA per SM, averaged over
// `iters` launches of 16 passes each after one warm-up launch.  No
// counterpart in the reference; the streaming ceiling beside the gather roof.
extern "C" int ggb_probe_l2_stream(int mib, int iters, double* gbs) {
  if (mib <= 0 || mib > 96 || iters <= 0 || !gbs) return GGB_EINVAL;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return GGB_ECUDA;
  }
  const size_t smem = (size_t)kStreamStages * kStreamChunk;
  if (cudaFuncSetAttribute((const void*)probe_stream_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess) {
    cudaGetLastError();
    return GGB_ECUDA;
  }
  const long long chunks = (long long)mib * (1 << 20) / kStreamChunk;
  unsigned char* buf = nullptr;
  int* err = nullptr;
  if (cudaMalloc(&buf, (size_t)chunks * kStreamChunk) != cudaSuccess || cudaMalloc(&err, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(buf);
    cudaFree(err);
    return GGB_ENOMEM;
  }
  cudaMemset(buf, 0x5a, (size_t)chunks * kStreamChunk);
  cudaMemset(err, 0, sizeof(int));
  constexpr int kPasses = 16;   // 1 GiB a launch at 64 MiB, so the launch gaps stay small
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  float ms = 0.f;
  int h_err = 0;
  if (e == cudaSuccess) {
    probe_stream_kernel<<<sms, 32, smem>>>(buf, chunks, kPasses, err);   // warm-up: the buffer into L2
    e = cudaEventRecord(e0);
    for (int it = 0; it < iters && e == cudaSuccess; ++it) probe_stream_kernel<<<sms, 32, smem>>>(buf, chunks, kPasses, err);
    if (e == cudaSuccess) e = cudaEventRecord(e1);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess) e = cudaMemcpy(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost);
  }
  if (e1) cudaEventDestroy(e1);
  if (e0) cudaEventDestroy(e0);
  cudaFree(buf);
  cudaFree(err);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return GGB_ECUDA;
  }
  if (h_err) return GGB_ETIMEOUT;
  if (ms <= 0.f) return GGB_ECUDA;
  *gbs = (double)chunks * kStreamChunk * kPasses * iters / (ms * 1e-3) / 1e9;
  return GGB_OK;
}

// GB/s of random-row OR sweeps over an N x (window_bits/8)-byte matrix with d
// random neighbours per row (a fixed-seed LCG graph), averaged over `iters`
// sweeps after warm-up, on the current device.  The bytes are counted as the
// evaluator's algorithmic bytes of one dense sweep are: N*d*4 adjacency +
// N*d*W/8 gathered rows + 2*N*W/8 own row read and new row written.
extern "C" int ggb_probe_l2_gather(int N, int d, int window_bits, int iters, double* gbs) {
  // 64-source windows use rows of one uint4, as the evaluator does
  const int R = window_bits == 64 ? 1 : window_bits / 128;
  if (N <= 0 || d <= 0 || iters <= 0 || !gbs || window_bits <= 0 ||
      (window_bits != 64 && (window_bits % 128 || (R & (R - 1)) || R > 64)))
    return GGB_EINVAL;
  std::vector<int> adj((size_t)N * d);
  unsigned long long x = 0x9e3779b97f4a7c15ULL;
  for (auto& v : adj) {
    x = x * 6364136223846793005ULL + 1442695040888963407ULL;
    v = (int)((x >> 33) % (unsigned long long)N);
  }
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return GGB_ECUDA;
  }
  int* dadj = nullptr;
  uint4* buf = nullptr;
  unsigned long long* sink = nullptr;
  const size_t cells = (size_t)N * R;
  if (cudaMalloc(&dadj, adj.size() * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&buf, 2 * cells * sizeof(uint4)) != cudaSuccess ||
      cudaMalloc(&sink, sizeof(unsigned long long)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(dadj);
    cudaFree(buf);
    cudaFree(sink);
    return GGB_ENOMEM;
  }
  cudaMemcpy(dadj, adj.data(), adj.size() * sizeof(int), cudaMemcpyHostToDevice);
  cudaMemset(buf, 0x5a, 2 * cells * sizeof(uint4));
  float ms = 0.f;
  switch (R) {
    case 1: ms = time_sweeps<1>(buf, buf + cells, dadj, N, d, iters, sink, sms); break;
    case 2: ms = time_sweeps<2>(buf, buf + cells, dadj, N, d, iters, sink, sms); break;
    case 4: ms = time_sweeps<4>(buf, buf + cells, dadj, N, d, iters, sink, sms); break;
    case 8: ms = time_sweeps<8>(buf, buf + cells, dadj, N, d, iters, sink, sms); break;
    case 16: ms = time_sweeps<16>(buf, buf + cells, dadj, N, d, iters, sink, sms); break;
    case 32: ms = time_sweeps<32>(buf, buf + cells, dadj, N, d, iters, sink, sms); break;
    default: ms = time_sweeps<64>(buf, buf + cells, dadj, N, d, iters, sink, sms); break;
  }
  cudaError_t e = cudaGetLastError();
  cudaFree(dadj);
  cudaFree(buf);
  cudaFree(sink);
  if (e != cudaSuccess || ms <= 0.f) return GGB_ECUDA;
  const double row = window_bits / 8.0;
  *gbs = ((double)N * d * 4.0 + (double)N * d * row + 2.0 * N * row) / (ms * 1e-3) / 1e9;
  return GGB_OK;
}
