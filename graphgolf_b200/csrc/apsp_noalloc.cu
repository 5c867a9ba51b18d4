// apsp_noalloc.cu -- the general evaluator without any device allocation.
//
// Some callers cannot let a library call cudaMalloc: a host program whose
// device memory is owned by another allocator (a framework's caching pool or
// a fixed budget carved out at start-up), or a simulated-annealing loop that
// must not allocate while it runs.  ggb_eval_general_noalloc serves them.  It
// runs the same persistent kernel as ggb_eval_general_device, with the
// kernel's scratch -- the control block and the two bitset matrices of a
// source window -- placed in one file-scope __device__ array of
// kNoAllocScratchBytes (16 MiB) instead of in cudaMalloc'd buffers.  Every GPU
// that loads this library holds that array until the process exits.
//
// The array's host-side name is only a stand-in for the symbol: host code
// must never hand it to a kernel.  The first call on a device, with that
// device current, asks the runtime for the array's device address
// (cudaGetSymbolAddress) and keeps it for later calls on that device; make
// that first call before any stream capture.  Every call waits for its own
// result: it copies the result block to the host and synchronises `stream`.
// All calls share the one array
// and it keeps the previous call's contents: the control block is cleared at
// the start of every call (the bitset rows are always fully written before
// they are read).  Calls that overlap on the GPU -- from two host threads, or
// on two streams -- race on the array and give wrong results; serialise them.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <mutex>

#include "../../include/graphgolf_b200.h"
#include "apsp_kernel.cuh"

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;   // 16 MiB
constexpr size_t kCtrlBytes = 256;                          // control block, padded
constexpr int kMaxDevices = 64;
static_assert(sizeof(ggb::ApspCtrl) <= kCtrlBytes, "the control block must fit its padded slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct DeviceSlot {
  unsigned char* scratch = nullptr;   // device address of g_noalloc_scratch on this device
  int sms = 0;
  int occ[7] = {0, 0, 0, 0, 0, 0, 0};  // co-resident CTAs per SM, per R = 1..64
};
DeviceSlot g_slots[kMaxDevices];
std::mutex g_mu;
char g_err[256] = "";
// Bound on every grid-barrier wait, as for the other entry points:
// GGB_BARRIER_TIMEOUT_NS when set, else 2 s.  Read at the first call.
long long g_timeout_ns = 0;

int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

const void* kernel_for(int R) {
  switch (R) {
    case 1: return (const void*)ggb::apsp_persistent_kernel<1>;
    case 2: return (const void*)ggb::apsp_persistent_kernel<2>;
    case 4: return (const void*)ggb::apsp_persistent_kernel<4>;
    case 8: return (const void*)ggb::apsp_persistent_kernel<8>;
    case 16: return (const void*)ggb::apsp_persistent_kernel<16>;
    case 32: return (const void*)ggb::apsp_persistent_kernel<32>;
    case 64: return (const void*)ggb::apsp_persistent_kernel<64>;
    default: return nullptr;
  }
}

size_t smem_for(int R) {
  switch (R) {
    case 1: return ggb::apsp_smem_bytes<1>();
    case 2: return ggb::apsp_smem_bytes<2>();
    case 4: return ggb::apsp_smem_bytes<4>();
    case 8: return ggb::apsp_smem_bytes<8>();
    case 16: return ggb::apsp_smem_bytes<16>();
    case 32: return ggb::apsp_smem_bytes<32>();
    case 64: return ggb::apsp_smem_bytes<64>();
    default: return 0;
  }
}

int log2i(int R) {
  int k = 0;
  while ((1 << k) < R) ++k;
  return k;
}

// Once per device, with that device current: resolve the scratch array's
// device address and the kernels' occupancy.  Allocates nothing.
int setup_device(int dev, DeviceSlot** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(GGB_EINVAL, "device index %d out of range", dev);
  if (g_timeout_ns <= 0) {
    const char* env = getenv("GGB_BARRIER_TIMEOUT_NS");
    const long long t = env ? atoll(env) : 0;
    g_timeout_ns = t > 0 ? t : 2000000000LL;
  }
  DeviceSlot& s = g_slots[dev];
  if (!s.scratch) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      cudaGetLastError();
      return fail(GGB_ECUDA, "cudaGetSymbolAddress of the no-alloc scratch array failed");
    }
    if (cudaDeviceGetAttribute(&s.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return fail(GGB_ECUDA, "cudaDeviceGetAttribute failed");
    for (int R = 1; R <= 64; R *= 2) {
      int nb = 0;
      if (cudaFuncSetAttribute(kernel_for(R), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_for(R)) !=
              cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel_for(R), ggb::kThreads, smem_for(R)) !=
              cudaSuccess || nb < 1) {
        cudaGetLastError();
        return fail(GGB_ECUDA, "the persistent kernel cannot be made resident");
      }
      s.occ[log2i(R)] = nb;
    }
    s.scratch = static_cast<unsigned char*>(p);
  }
  *out = &s;
  return GGB_OK;
}

}  // namespace

extern "C" const char* ggb_noalloc_last_error(void) { return g_err; }

extern "C" long long ggb_noalloc_scratch_bytes(void) { return (long long)kNoAllocScratchBytes; }

extern "C" int ggb_eval_general_noalloc(int nodes, int based_nodes, int groups, int degree, const int* adj_dev,
                                        int added_centers, void* stream, ggb_result* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!out || (!adj_dev && (long long)nodes * degree > 0)) return fail(GGB_EINVAL, "null pointer");
  if (nodes <= 0 || based_nodes <= 0 || groups <= 0 || degree < 0 || added_centers < 0 ||
      (long long)based_nodes * groups + added_centers != nodes)
    return fail(GGB_EINVAL, "nodes must equal based_nodes*groups + added_centers, all sizes positive");
  // The kernels index the adjacency with int offsets, as the reference's int
  // adjacency does.
  if ((long long)nodes * degree > INT_MAX)
    return fail(GGB_EINVAL, "nodes*degree exceeds the int32 adjacency of the reference");
  // The two bitset matrices of a window need 2 * nodes * 16 bytes per 128
  // sources; the narrowest window (128 sources) must fit.
  const size_t avail = kNoAllocScratchBytes - kCtrlBytes;
  const size_t per_r = 2 * (size_t)nodes * sizeof(uint4);
  if (per_r > avail)
    return fail(GGB_EINVAL, "graph too large for the no-alloc scratch (nodes must be at most 524280)");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(GGB_ECUDA, "cudaGetDevice failed");
  }
  DeviceSlot* slot = nullptr;
  int rc = setup_device(dev, &slot);
  if (rc) return rc;

  // Window: as many sources as are needed, up to 8192 and what the scratch holds.
  const int nsrc = std::max(based_nodes, added_centers);
  int R = 1;
  while (R < 64 && 128 * R < nsrc && per_r * (size_t)(2 * R) <= avail) R *= 2;
  const size_t cells = (size_t)nodes * R;

  ggb::ApspCtrl* ctrl = reinterpret_cast<ggb::ApspCtrl*>(slot->scratch);
  uint4* bufs = reinterpret_cast<uint4*>(slot->scratch + kCtrlBytes);
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  ggb::ApspArgs a;
  a.adj = adj_dev;
  a.adj2 = nullptr;
  a.buf0 = bufs;
  a.buf1 = bufs + cells;
  a.ctrl = ctrl;
  a.timeout_ns = g_timeout_ns;
  a.N = nodes;
  a.d = degree;
  a.n_src1 = based_nodes;
  a.split = based_nodes * groups;
  a.ac = added_centers;
  a.groups = groups;
  a.win_first = 0;
  a.win_stride = 1;
  a.vec4 = (degree % 4 == 0 && ((uintptr_t)adj_dev % 16) == 0) ? 1 : 0;
  a.ball = nullptr;
  a.ball_cnt = nullptr;
  a.trace = nullptr;
  a.trace_cap = 0;
  a.phantom = 0;
  a.stats = nullptr;
  a.levels = nullptr;
  a.level_counts = nullptr;
  a.win_levels = nullptr;
  a.level_cap = 0;

  const int lpr = R >= 32 ? 32 : R;
  const int vpw = 32 / lpr;
  const long long want = ((long long)nodes + (long long)vpw * ggb::kWarps - 1) / ((long long)vpw * ggb::kWarps);
  const int ctas = (int)std::min<long long>(std::max<long long>(want, 1), (long long)slot->occ[log2i(R)] * slot->sms);

  if (cudaMemsetAsync(ctrl, 0, sizeof(ggb::ApspCtrl), st) != cudaSuccess) {
    cudaGetLastError();
    return fail(GGB_ECUDA, "cudaMemsetAsync of the control block failed");
  }
  void* params[] = {(void*)&a};
  if (cudaLaunchCooperativeKernel(kernel_for(R), dim3(ctas), dim3(ggb::kThreads), params, smem_for(R), st) !=
      cudaSuccess) {
    cudaGetLastError();
    return fail(GGB_ECUDA, "cooperative launch of the persistent kernel failed");
  }
  ggb::ApspCtrl c;
  if (cudaMemcpyAsync(&c, ctrl, sizeof(c), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return fail(GGB_ECUDA, "reading the result block failed");
  }
  if (c.error == ggb::kErrAdj)
    return fail(GGB_EADJ, "adjacency entry outside [0, nodes) (reported by CTA/vertex %d)", c.error_info);
  if (c.error == ggb::kErrTimeout) return fail(GGB_ETIMEOUT, "a grid-barrier wait ran out (CTA %d)", c.error_info);
  if (c.error == ggb::kErrDegree)
    return fail(GGB_EINVAL, "degree of vertex %d outside [0, max_degree]", c.error_info);
  if (c.error != 0) return fail(GGB_ECUDA, "device error code %d (at %d)", c.error, c.error_info);
  if (!c.done) return fail(GGB_ECUDA, "the persistent kernel did not complete");
  ggb_partial p;
  p.diam = c.diam;
  p.disconnected = c.disconnected;
  p.sum = c.sum;
  p.levels = c.levels;
  p.windows = c.windows;
  p.window_bits = 128 * R;
  p.dense_levels = c.dense_levels;
  return ggb_finish_general(nodes, &p, out);
}
