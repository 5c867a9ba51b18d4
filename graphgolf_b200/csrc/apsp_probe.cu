// apsp_probe.cu -- measures the ceiling the dense sweeps run against.
//
// The sweeps' working set (two bitset matrices of a source window) is
// L2-resident by design, so the roof that bounds them is not the HBM copy
// bandwidth but the rate at which the SMs can gather random rows of that size
// from L2.  ggb_probe_l2_gather times exactly that access pattern -- every
// vertex ORs its own row and the rows of its d random neighbours out of a
// matrix of the same shape, one launch per sweep -- on buffers it allocates
// itself, and reports gathered bytes per second.  bench.py uses it for the
// roofline report.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../include/graphgolf_b200.h"

namespace {

template <int R>
__global__ void __launch_bounds__(512, 2) probe_gather_kernel(const uint4* __restrict__ src, uint4* __restrict__ dst,
                                                             const int* __restrict__ adj, int N, int d,
                                                             unsigned long long* sink) {
  constexpr int LPR = R >= 32 ? 32 : R;
  constexpr int VPW = 32 / LPR;
  constexpr int UPL = R / LPR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane / LPR, li = lane % LPR;
  const long long slot = ((long long)blockIdx.x * 16 + warp) * VPW + sub;
  const long long n_slots = (long long)gridDim.x * 16 * VPW;
  unsigned c = 0;
  for (long long v = slot; v < N; v += n_slots) {
    uint4 acc[UPL];
#pragma unroll
    for (int k = 0; k < UPL; ++k) acc[k] = __ldcg(src + v * R + li + k * LPR);
    for (int j = 0; j < d; j += 8) {
      uint4 x[8][UPL];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int u = j + q < d ? __ldg(adj + v * d + j + q) : (int)v;
#pragma unroll
        for (int k = 0; k < UPL; ++k) x[q][k] = __ldcg(src + (long long)u * R + li + k * LPR);
      }
#pragma unroll
      for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int k = 0; k < UPL; ++k) {
          acc[k].x |= x[q][k].x;
          acc[k].y |= x[q][k].y;
          acc[k].z |= x[q][k].z;
          acc[k].w |= x[q][k].w;
        }
    }
#pragma unroll
    for (int k = 0; k < UPL; ++k) {
      __stcg(dst + v * R + li + k * LPR, acc[k]);
      c += __popc(acc[k].x) + __popc(acc[k].y) + __popc(acc[k].z) + __popc(acc[k].w);
    }
  }
  if (c == 0xffffffffu) atomicAdd(sink, 1ULL);   // keeps the loads alive
}

template <int R>
float time_sweeps(uint4* a, uint4* b, const int* adj, int N, int d, int iters, unsigned long long* sink, int sms) {
  constexpr int VPW = 32 / (R >= 32 ? 32 : R);
  const long long want = ((long long)N + VPW * 16 - 1) / (VPW * 16);
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

}  // namespace

// Gathered GB/s of random-row OR sweeps over an N x (window_bits/8)-byte
// matrix with d random neighbours per row (a fixed-seed LCG graph), averaged
// over `iters` sweeps after warm-up, on the current device.
extern "C" int ggb_probe_l2_gather(int N, int d, int window_bits, int iters, double* gbs) {
  const int R = window_bits / 128;
  if (N <= 0 || d <= 0 || iters <= 0 || !gbs || window_bits <= 0 || window_bits % 128 || (R & (R - 1)) || R > 64)
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
  *gbs = (double)N * d * 16.0 * R / (ms * 1e-3) / 1e9;
  return GGB_OK;
}
