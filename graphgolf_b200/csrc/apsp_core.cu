// apsp_core.cu -- host side of the core library libgraphgolf_b200.so.
//
// Owns the device state the reference keeps in module globals
// (A_dev/B_dev/result/adjacency_dev, general/evaluation.cu:2-4): one stream,
// grow-only device buffers, pinned staging for the adjacency and the result.
// Every entry point is extern "C" with plain pointers (include/graphgolf_b200.h).
//
// Per evaluation the device does all the work of the reference's host loop
// (general/evaluation.cu:85-112): there is no per-level launch and no
// per-level device-to-host copy; the persistent kernel decides termination
// itself and the host reads one 64-byte control block at the end.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <mutex>

#include "../../include/graphgolf_b200.h"
#include "apsp_kernel.cuh"
#include "core_internal.h"

namespace ggb {

// Grid relabel (grid/evaluation.c:148-151): row rotate_hash[i] of the
// relabelled adjacency holds rotate_hash[adj[i][j]].  inv[] must be -1 on
// entry; it receives the inverse permutation so a second kernel can verify
// that rotate_hash is a bijection.
// With deg (non-regular grids, degree[i] entries of row i are edges), the
// slots j >= deg[i] are filled with the row's own relabelled id: OR-ing a
// row's own set into itself changes nothing, so the sweep needs no per-row
// degree.
__global__ void relabel_adjacency_kernel(const int* __restrict__ adj, const int* __restrict__ rh,
                                         int* __restrict__ out, int* __restrict__ inv, int N, int d,
                                         ApspCtrl* ctrl, const int* __restrict__ deg) {
  const long long n = (long long)N * d;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / d), j = (int)(e % d);
    const int r = rh[i];
    if (deg && ((unsigned)deg[i] > (unsigned)d)) { set_error(ctrl, kErrDegree, i); continue; }
    const int nb = (deg && j >= deg[i]) ? i : adj[e];
    if ((unsigned)r >= (unsigned)N) { set_error(ctrl, kErrPerm, i); continue; }
    if ((unsigned)nb >= (unsigned)N) { set_error(ctrl, kErrAdj, i); continue; }
    const int rn = rh[nb];
    if ((unsigned)rn >= (unsigned)N) { set_error(ctrl, kErrPerm, nb); continue; }
    out[(long long)r * d + j] = rn;
    if (j == 0) inv[r] = i;
  }
  if (d == 0) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
      const int r = rh[i];
      if ((unsigned)r >= (unsigned)N) { set_error(ctrl, kErrPerm, (int)i); continue; }
      inv[r] = (int)i;
    }
  }
}

// Non-regular general graphs: out[i][j] = adj[i][j] for j < deg[i], else i
// (a self entry, which the recurrence ignores).
__global__ void pad_adjacency_kernel(const int* __restrict__ adj, const int* __restrict__ deg,
                                     int* __restrict__ out, int N, int d, ApspCtrl* ctrl) {
  const long long n = (long long)N * d;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / d), j = (int)(e % d);
    const int di = deg[i];
    if ((unsigned)di > (unsigned)d) { set_error(ctrl, kErrDegree, i); continue; }
    out[e] = j < di ? adj[e] : i;
  }
}

__global__ void check_permutation_kernel(const int* __restrict__ inv, int N, ApspCtrl* ctrl) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x)
    if (inv[i] < 0) set_error(ctrl, kErrPerm, (int)i);
}

}  // namespace ggb

namespace {

using ggb::ApspArgs;
using ggb::ApspCtrl;

struct State {
  bool ready = false;
  int device = -1;
  int sms = 0;
  size_t l2_bytes = 0;
  cudaStream_t stream = nullptr;
  // device buffers (grow-only)
  int* d_adj = nullptr;       size_t cap_adj = 0;     // ints
  uint16_t* d_adj16 = nullptr; size_t cap_adj16 = 0; // 16-bit ids on their way to d_adj
  int* d_adj2 = nullptr;      size_t cap_adj2 = 0;    // ints (grid relabel)
  int* d_rh = nullptr;        size_t cap_rh = 0;      // ints
  int* d_inv = nullptr;       size_t cap_inv = 0;     // ints
  int* d_deg = nullptr;       size_t cap_deg = 0;     // ints (non-regular degrees)
  int* h_deg = nullptr;       size_t cap_hdeg = 0;
  uint4* d_bufs = nullptr;    size_t cap_buf = 0;     // uint4, both bitset matrices
  ApspCtrl* d_ctrl = nullptr;
  // pinned host staging
  int* h_adj = nullptr;       size_t cap_hadj = 0;
  int* h_rh = nullptr;        size_t cap_hrh = 0;
  ApspCtrl* h_ctrl = nullptr;
  // tuning
  int force_R = 0;
  int force_W = 0;            // forced sources per window below 128 (64), else 0
  int force_ctas = 0;
  long long timeout_ns = 2000000000LL;
  int phantom = 0;
  uint4* d_ball = nullptr;    size_t cap_ball = 0;    // uint4, ball pre-pass matrix
  unsigned* d_stamps = nullptr; size_t cap_stamps = 0; // full-row stamps, one per vertex
  unsigned long long* d_ball_cnt = nullptr; size_t cap_ball_cnt = 0;
  int ball_mode = -1;         // -1 automatic, 0 never, 1 whenever feasible
  int ball_occ = 0;           // co-resident ball CTAs per SM at the last size
  // optional per-kernel timing (ggb_set_timing): events around the two kernels
  bool timing = false;
  cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};   // before ball, between, after persistent
  bool ev_ball = false;                              // the last launch ran the ball pre-pass
  long long* d_trace = nullptr;   // optional barrier trace (ggb_trace_enable)
  int trace_cap = 0;
  int trace_len = 0;
  int occ[8] = {0, 0, 0, 0, 0, 0, 0, 0};   // co-resident CTAs per SM, per R index
  int tocc[4] = {0, 0, 0, 0};             // the same for the window-team kernel, R = 1, 2, 4, 8
  int smem_optin = 0;
  // window teams (narrow windows of one graph, several at a time): the batch
  // kernel's per-team entries, results and control blocks, and pinned staging
  ggb::BatchGraph* d_tgraphs = nullptr;
  ggb::BatchOut* d_tout = nullptr;
  ggb::ApspCtrl* d_tctrl = nullptr;
  int* d_tint = nullptr;          // team_start [kMaxTeams + 1], team_list [kMaxTeams]
  long long* d_tll = nullptr;     // team_off [kMaxTeams], team_cells [kMaxTeams]
  unsigned char* h_team = nullptr;   // pinned: the above for upload, then results for read-back
  int last_teams = 0;
  // last launch bookkeeping (for ggb_collect)
  int last_N = 0, last_R = 0, last_W = 0;
  bool pending = false;
  bool last_grid = false;
};

State g;
std::mutex g_mu;
char g_err[512] = "";
long long g_launches = 0;
std::atomic<long long> g_h2d{0};   // adjacency bytes sent host to device (staging threads add to it)

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(call)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess)                                                                    \
      return fail(GGB_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                  __LINE__);                                                                  \
  } while (0)

int r_index(int R) {
  switch (R) {
    case 1: return 0; case 2: return 1; case 4: return 2; case 8: return 3;
    case 16: return 4; case 32: return 5; case 64: return 6; default: return -1;
  }
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

constexpr int kMaxTeams = 256;

const void* team_kernel_for(int R) {
  switch (R) {
    case 1: return (const void*)ggb::apsp_batch_kernel<1>;
    case 2: return (const void*)ggb::apsp_batch_kernel<2>;
    case 4: return (const void*)ggb::apsp_batch_kernel<4>;
    case 8: return (const void*)ggb::apsp_batch_kernel<8>;
    default: return nullptr;
  }
}

int ensure_ready(int device) {
  if (g.ready) return GGB_OK;
  if (device < 0) {
    int cur = 0;
    CUDA_TRY(cudaGetDevice(&cur));
    device = cur;
  }
  CUDA_TRY(cudaSetDevice(device));
  g.device = device;
  CUDA_TRY(cudaDeviceGetAttribute(&g.sms, cudaDevAttrMultiProcessorCount, device));
  int l2 = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device));
  g.l2_bytes = (size_t)l2;
  int coop = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device));
  if (!coop) return fail(GGB_ECUDA, "device %d does not support cooperative launch", device);
  CUDA_TRY(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
  CUDA_TRY(cudaMalloc(&g.d_ctrl, sizeof(ApspCtrl)));
  CUDA_TRY(cudaHostAlloc(&g.h_ctrl, sizeof(ApspCtrl), cudaHostAllocDefault));
  for (int R = 1; R <= 64; R *= 2) {
    int nb = 0;
    CUDA_TRY(cudaFuncSetAttribute(kernel_for(R), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_for(R)));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel_for(R), ggb::kThreads, smem_for(R)));
    if (nb < 1) return fail(GGB_ECUDA, "persistent kernel R=%d cannot be resident", R);
    g.occ[r_index(R)] = nb;
  }
  for (int R = 1; R <= 8; R *= 2) {
    int nb = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, team_kernel_for(R), ggb::kThreads, smem_for(R)));
    g.tocc[r_index(R)] = nb;
  }
  int smem_optin = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  g.smem_optin = smem_optin;
  CUDA_TRY(cudaFuncSetAttribute((const void*)ggb::ball_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem_optin - 4096));
  CUDA_TRY(cudaFuncSetAttribute((const void*)ggb::ball_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                smem_optin - 4096));
  if (const char* s = getenv("GGB_BARRIER_TIMEOUT_NS")) g.timeout_ns = atoll(s);
  g.ready = true;
  return GGB_OK;
}

template <typename T>
int grow_device(T** p, size_t* cap, size_t n) {
  if (n <= *cap && *p) return GGB_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  size_t want = std::max<size_t>(n, 1);
  if (cudaMalloc(p, want * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    return fail(GGB_ENOMEM, "cudaMalloc of %zu bytes failed", want * sizeof(T));
  }
  *cap = want;
  return GGB_OK;
}

template <typename T>
int grow_pinned(T** p, size_t* cap, size_t n) {
  if (n <= *cap && *p) return GGB_OK;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *cap = 0;
  size_t want = std::max<size_t>(n, 1);
  if (cudaHostAlloc(p, want * sizeof(T), cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    return fail(GGB_ENOMEM, "cudaHostAlloc of %zu bytes failed", want * sizeof(T));
  }
  *cap = want;
  return GGB_OK;
}

int max_ctas(int R) { return g.occ[r_index(R)] * g.sms; }

// Window width: the number of uint4 per bitset row.  Both matrices of a
// window must stay in L2 next to the adjacency, so 2*N*16*R is capped at 55%
// of the L2.  Among the widths that fit, the one with the least modelled time
// wins: per window, the two-hop seeding (d + d^2 adjacency reads and two row
// writes per vertex) plus about four dense sweeps of d gathered rows of 16R
// bytes, at the L2 gather rate, plus a fixed cost per sweep for the grid
// barrier.  Results never depend on the choice.
int choose_R(int N, int d, int nsrc_max) {
  if (g.force_R) return g.force_R;
  const double budget = std::max<double>(8.0 * 1024 * 1024, (double)g.l2_bytes * 0.55);
  double best = 1e300;
  int bestR = 1;
  const double dd = std::max(d, 1);
  for (int R = 1; R <= 64; R *= 2) {
    const double bytes_per_buf = (double)N * 16.0 * R;
    if (R > 1 && 2.0 * bytes_per_buf > budget) break;
    const int W = 128 * R;
    const long long nwin = (nsrc_max + W - 1) / W;
    const double seed_bytes = (double)N * (dd + dd * dd) * 4.0 + 2.0 * bytes_per_buf;
    const double level_bytes = (double)N * dd * (16.0 * R + 4.0) + 2.0 * bytes_per_buf;
    const double t = nwin * ((seed_bytes + 4.0 * level_bytes) / 14.0e12 + 5.0 * 2.5e-6);
    if (t < best * 0.999) { best = t; bestR = R; }
    if (nwin == 1) break;   // wider windows only add zero bits
  }
  return bestR;
}

size_t team_pinned_bytes() {
  return kMaxTeams * (sizeof(ggb::BatchGraph) + sizeof(ggb::BatchOut) + sizeof(ggb::ApspCtrl)) +
         (2 * kMaxTeams + 2) * sizeof(int) + 2 * kMaxTeams * sizeof(long long) + 256;
}

// Narrow windows of one graph on teams of CTAs: team j of T runs this rank's
// windows rank + procs*j, rank + procs*(j + T), ... with its own grid barrier
// and its own two window matrices, so the per-window latency (seeding, a
// barrier per level) of T windows overlaps.  The batch kernel does the work;
// its answer per team is a partial like a rank's.
int launch_teams(const int* d_adj, int N, int d, int n_src1, int groups, int rank, int procs, int R, int W, int T,
                 int team_ctas, bool vec4, cudaStream_t st) {
  const size_t cells = (size_t)N * R;
  int rc = grow_device(&g.d_bufs, &g.cap_buf, 2 * cells * T);
  if (rc) return rc;
  if (!g.d_tgraphs) {
    CUDA_TRY(cudaMalloc(&g.d_tgraphs, kMaxTeams * sizeof(ggb::BatchGraph)));
    CUDA_TRY(cudaMalloc(&g.d_tout, kMaxTeams * sizeof(ggb::BatchOut)));
    CUDA_TRY(cudaMalloc(&g.d_tctrl, kMaxTeams * sizeof(ggb::ApspCtrl)));
    CUDA_TRY(cudaMalloc(&g.d_tint, (2 * kMaxTeams + 1) * sizeof(int)));
    CUDA_TRY(cudaMalloc(&g.d_tll, 2 * kMaxTeams * sizeof(long long)));
    CUDA_TRY(cudaHostAlloc(&g.h_team, team_pinned_bytes(), cudaHostAllocDefault));
  }
  // the previous launch's read-back is complete: every host entry point waits
  ggb::BatchGraph* hg = reinterpret_cast<ggb::BatchGraph*>(g.h_team);
  int* hi = reinterpret_cast<int*>(hg + kMaxTeams);
  long long* hl = reinterpret_cast<long long*>(hi + 2 * kMaxTeams + 2);
  for (int j = 0; j < T; ++j) {
    hg[j].adj = d_adj;
    hg[j].N = N;
    hg[j].d = d;
    hg[j].n_src = n_src1;
    hg[j].groups = groups;
    hg[j].vec4 = vec4 ? 1 : 0;
    hg[j].win_first = rank + procs * j;
    hg[j].win_stride = procs * T;
    hg[j].win_bits = W < 128 * R ? W : 0;
    hi[j] = j;                      // team_start
    hi[kMaxTeams + 1 + j] = j;      // team_list
    hl[j] = (long long)(2 * cells) * j;   // team_off
    hl[kMaxTeams + j] = (long long)cells; // team_cells
  }
  hi[T] = T;
  CUDA_TRY(cudaMemcpyAsync(g.d_tgraphs, hg, T * sizeof(ggb::BatchGraph), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(g.d_tint, hi, (2 * kMaxTeams + 1) * sizeof(int), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemcpyAsync(g.d_tll, hl, 2 * kMaxTeams * sizeof(long long), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemsetAsync(g.d_tctrl, 0, T * sizeof(ggb::ApspCtrl), st));
  CUDA_TRY(cudaMemsetAsync(g.d_tout, 0, T * sizeof(ggb::BatchOut), st));
  ggb::BatchArgs b;
  b.graphs = g.d_tgraphs;
  b.out = g.d_tout;
  b.team_ctrl = g.d_tctrl;
  b.team_start = g.d_tint;
  b.team_list = g.d_tint + kMaxTeams + 1;
  b.scratch = g.d_bufs;
  b.team_off = g.d_tll;
  b.team_cells = g.d_tll + kMaxTeams;
  b.timeout_ns = g.timeout_ns;
  b.stop = nullptr;
  b.sticky = nullptr;
  b.n_teams = T;
  b.team_ctas = team_ctas;
  if (g.timing) {
    CUDA_TRY(cudaEventRecord(g.ev[0], st));
    CUDA_TRY(cudaEventRecord(g.ev[1], st));
  }
  void* params[] = {(void*)&b};
  CUDA_TRY(cudaLaunchCooperativeKernel(team_kernel_for(R), dim3(T * team_ctas), dim3(ggb::kThreads), params,
                                       smem_for(R), st));
  ++g_launches;
  if (g.timing) CUDA_TRY(cudaEventRecord(g.ev[2], st));
  g.ev_ball = false;
  g.last_N = N;
  g.last_R = R;
  g.last_W = W;
  g.last_teams = T;
  g.pending = true;
  return GGB_OK;
}

int launch_apsp(const int* d_adj, int N, int d, int n_src1, int split, int ac, int groups,
                int rank, int procs, cudaStream_t st, const int* d_adj2 = nullptr) {
  const int R = choose_R(N, d, std::max(n_src1, ac));
  const int ri = r_index(R);
  if (ri < 0) return fail(GGB_EINVAL, "window of %d uint4 per row is not supported", R);
  g.last_teams = 0;
  {
    // narrow windows (rows of at most 128 bytes), no added centres: teams of
    // windows when at least two fit in the L2 budget and there are windows
    // enough for them
    const int Wt = (R == 1 && g.force_W > 0) ? g.force_W : 128 * R;
    const int nwin1t = n_src1 > 0 ? (n_src1 + Wt - 1) / Wt : 0;
    const int n_loc = nwin1t > rank ? (nwin1t - rank + procs - 1) / procs : 0;
    const double budget = std::max<double>(8.0 * 1024 * 1024, (double)g.l2_bytes * 0.55);
    const long long fit = (long long)(budget / (2.0 * N * 16.0 * R));
    const int total = R <= 8 ? std::min(max_ctas(R), g.tocc[r_index(R)] * g.sms) : 0;
    int T = (int)std::min<long long>(std::min<long long>(fit, n_loc), std::min(total / 2, kMaxTeams));
    if (R <= 8 && ac == 0 && !d_adj2 && g.force_ctas == 0 && T >= 2 && n_loc >= 4) {
      const int team_ctas = total / T;
      T = total / team_ctas;   // every CTA in a team
      T = std::min<long long>(std::min<long long>(T, fit), std::min(n_loc, kMaxTeams));
      const bool vec4t = (d % 4 == 0 && ((uintptr_t)d_adj % 16) == 0);
      return launch_teams(d_adj, N, d, n_src1, groups, rank, procs, R, Wt, T, team_ctas, vec4t, st);
    }
  }
  const size_t cells = (size_t)N * R;
  // Both matrices live in one allocation: buf0 = [0, cells), buf1 = [cells, 2*cells).
  int rc = grow_device(&g.d_bufs, &g.cap_buf, 2 * cells);
  if (rc) return rc;
  const int lpr = R >= 32 ? 32 : R;
  const int vpw = 32 / lpr;
  long long want = ((long long)N + (long long)vpw * ggb::kWarps - 1) / ((long long)vpw * ggb::kWarps);
  int ctas = (int)std::min<long long>(std::max<long long>(want, 1), max_ctas(R));
  if (g.force_ctas > 0) ctas = std::min(g.force_ctas, max_ctas(R));

  // Ball pre-pass: worth it when its one-off cost (d + d^2 + d^3 adjacency
  // reads per vertex, one HBM write of every window's S_3 rows) is below what
  // it saves (per window: the two-hop seeding and one dense sweep).
  const bool vec4 = (d % 4 == 0 && ((uintptr_t)d_adj % 16) == 0);
  const int W = (R == 1 && g.force_W > 0) ? g.force_W : 128 * R;
  const int nwin1 = n_src1 > 0 ? (n_src1 + W - 1) / W : 0;
  const int n_local = nwin1 > rank ? (nwin1 - rank + procs - 1) / procs : 0;
  const size_t ball_cells = (size_t)n_local * N * R;
  const size_t ball_smem = ggb::ball_smem_bytes(n_src1, d, std::max(n_local, 1));
  bool use_ball = g.ball_mode != 0 && ac == 0 && W == 128 * R && n_local >= 1 && n_local <= ggb::kBallMaxWindows && d >= 1 &&
                  d <= ggb::kBallMaxDegree && ball_smem <= (size_t)(g.smem_optin - 4096) &&
                  ball_cells * 16 <= ((size_t)8 << 30);
  if (use_ball && g.ball_mode < 0) {
    const double dd = d;
    const double t_ball = (double)N * (dd + dd * dd + dd * dd * dd) * 4.0 / 12.0e12 +
                          (double)ball_cells * 16.0 / 6.0e12 + 10.0e-6;
    const double level = (double)N * dd * (16.0 * R + 4.0) / 14.0e12 + 2.5e-6;
    const double seed = (double)N * (dd + dd * dd) * 4.0 / 12.0e12 + (double)N * 16.0 * R / 8.0e12 + 2.5e-6;
    use_ball = t_ball < 0.8 * n_local * (level + seed);
  }
  if (use_ball) {
    rc = grow_device(&g.d_ball, &g.cap_ball, ball_cells);
    if (rc) return rc;
    rc = grow_device(&g.d_ball_cnt, &g.cap_ball_cnt, (size_t)n_local * 6);
    if (rc) return rc;
    CUDA_TRY(cudaMemsetAsync(g.d_ball_cnt, 0, (size_t)n_local * 6 * sizeof(unsigned long long), st));
  }

  ApspArgs a;
  a.adj = d_adj;
  a.adj2 = d_adj2;
  a.buf0 = g.d_bufs;
  a.buf1 = g.d_bufs + cells;
  a.ctrl = g.d_ctrl;
  a.timeout_ns = g.timeout_ns;
  a.N = N;
  a.d = d;
  a.n_src1 = n_src1;
  a.split = split;
  a.ac = ac;
  a.groups = groups;
  a.win_first = rank;
  a.win_stride = procs;
  a.phantom = g.phantom;
  a.stats = nullptr;
  a.levels = nullptr;
  a.level_counts = nullptr;
  a.win_levels = nullptr;
  a.level_cap = 0;
  a.trace = g.d_trace;
  a.trace_cap = g.trace_cap;
  a.vec4 = vec4 ? 1 : 0;
  a.ball = use_ball ? g.d_ball : nullptr;
  a.ball_cnt = use_ball ? g.d_ball_cnt : nullptr;
  a.win_bits = W < 128 * R ? W : 0;
  // full-row stamps: the skipping sweep of 4096-bit rows, degree <= 16
  if (R == 32 && d <= 16 && W == 128 * R) {
    rc = grow_device(&g.d_stamps, &g.cap_stamps, (size_t)N);
    if (rc) return rc;
    CUDA_TRY(cudaMemsetAsync(g.d_stamps, 0, (size_t)N * sizeof(unsigned), st));
    a.stamps = g.d_stamps;
  }
  CUDA_TRY(cudaMemsetAsync(g.d_ctrl, 0, sizeof(ApspCtrl), st));
  if (g.timing) CUDA_TRY(cudaEventRecord(g.ev[0], st));
  if (use_ball) {
    ggb::BallArgs b;
    b.adj = d_adj;
    b.ball = g.d_ball;
    b.cnt = g.d_ball_cnt;
    b.ctrl = g.d_ctrl;
    b.N = N;
    b.d = d;
    b.n_src = n_src1;
    b.split = split;
    b.R = R;
    b.win_first = rank;
    b.win_stride = procs;
    b.n_local = n_local;
    const void* bk = vec4 ? (const void*)ggb::ball_kernel<4> : (const void*)ggb::ball_kernel<1>;
    int nb = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, bk, ggb::kBallThreads, ball_smem));
    if (nb < 1) return fail(GGB_ECUDA, "ball pre-pass cannot be resident with %zu bytes of shared memory", ball_smem);
    g.ball_occ = nb;
    const long long need = ((long long)N + ggb::kBallThreads / 32 - 1) / (ggb::kBallThreads / 32);
    const int bgrid = (int)std::min<long long>(need, (long long)nb * g.sms);
    if (vec4)
      ggb::ball_kernel<4><<<bgrid, ggb::kBallThreads, ball_smem, st>>>(b);
    else
      ggb::ball_kernel<1><<<bgrid, ggb::kBallThreads, ball_smem, st>>>(b);
    CUDA_TRY(cudaGetLastError());
    ++g_launches;
  }
  if (g.timing) CUDA_TRY(cudaEventRecord(g.ev[1], st));
  void* params[] = {(void*)&a};
  CUDA_TRY(cudaLaunchCooperativeKernel(kernel_for(R), dim3(ctas), dim3(ggb::kThreads), params, smem_for(R), st));
  ++g_launches;
  if (g.timing) CUDA_TRY(cudaEventRecord(g.ev[2], st));
  g.ev_ball = use_ball;
  g.last_N = N;
  g.last_R = R;
  g.last_W = W;
  g.pending = true;
  return GGB_OK;
}

// The teams' results joined into one partial (MAX diameter, SUM of the
// sums), after their errors.
int read_teams(cudaStream_t st, ggb_partial* p) {
  const int T = g.last_teams;
  ggb::BatchGraph* hg = reinterpret_cast<ggb::BatchGraph*>(g.h_team);
  long long* hl = reinterpret_cast<long long*>(reinterpret_cast<int*>(hg + kMaxTeams) + 2 * kMaxTeams + 2);
  ggb::BatchOut* ho = reinterpret_cast<ggb::BatchOut*>(hl + 2 * kMaxTeams);
  ApspCtrl* hc = reinterpret_cast<ApspCtrl*>(ho + kMaxTeams);
  CUDA_TRY(cudaMemcpyAsync(ho, g.d_tout, T * sizeof(ggb::BatchOut), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaMemcpyAsync(hc, g.d_tctrl, T * sizeof(ApspCtrl), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  g.pending = false;
  g.trace_len = 0;
  for (int j = 0; j < T; ++j) {
    const ApspCtrl& c = hc[j];
    if (c.error == ggb::kErrAdj)
      return fail(GGB_EADJ, "adjacency entry outside [0, nodes) (reported by CTA/vertex %d)", c.error_info);
    if (c.error == ggb::kErrTimeout) return fail(GGB_ETIMEOUT, "a team barrier wait ran out (CTA %d)", c.error_info);
    if (c.error != 0) return fail(GGB_ECUDA, "device error code %d", c.error);
    if (!ho[j].done) return fail(GGB_ECUDA, "window team %d did not complete", j);
  }
  p->diam = 1;
  p->disconnected = 0;
  p->sum = 0;
  p->levels = 0;
  p->dense_levels = 0;
  p->windows = 0;
  for (int j = 0; j < T; ++j) {
    p->diam = std::max(p->diam, ho[j].diam);
    p->disconnected |= ho[j].disconnected;
    p->sum += ho[j].sum;
    p->levels += ho[j].levels;
    p->dense_levels += ho[j].dense_levels;
    p->windows += ho[j].windows;
  }
  p->window_bits = g.last_W;
  return GGB_OK;
}

int read_ctrl(cudaStream_t st, ggb_partial* p) {
  if (g.last_teams > 0) return read_teams(st, p);
  CUDA_TRY(cudaMemcpyAsync(g.h_ctrl, g.d_ctrl, sizeof(ApspCtrl), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  g.pending = false;
  const ApspCtrl& c = *g.h_ctrl;
  if (c.error == ggb::kErrAdj)
    return fail(GGB_EADJ, "adjacency entry outside [0, nodes) (reported by CTA/vertex %d)", c.error_info);
  if (c.error == ggb::kErrPerm)
    return fail(GGB_EPERM, "rotate_hash is not a permutation of [0, nodes) (at %d)", c.error_info);
  if (c.error == ggb::kErrTimeout)
    return fail(GGB_ETIMEOUT, "a grid-barrier wait ran out (CTA %d)", c.error_info);
  if (c.error == ggb::kErrDegree)
    return fail(GGB_EINVAL, "degree of vertex %d outside [0, max_degree]", c.error_info);
  if (c.error != 0) return fail(GGB_ECUDA, "device error code %d", c.error);
  if (!c.done) return fail(GGB_ECUDA, "the persistent kernel did not complete");
  p->diam = c.diam;
  p->disconnected = c.disconnected;
  p->sum = c.sum;
  p->levels = c.levels;
  p->dense_levels = c.dense_levels;
  p->windows = c.windows;
  p->window_bits = g.last_W;
  g.trace_len = c.trace_len;
  return GGB_OK;
}

cudaStream_t pick_stream(void* s) { return s ? (cudaStream_t)s : g.stream; }

}  // namespace

namespace ggb {

int core_fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

void core_add_launches(long long n) { g_launches += n; }

void core_add_h2d(long long bytes) { g_h2d.fetch_add(bytes, std::memory_order_relaxed); }

}  // namespace ggb

namespace {

int check_general(int nodes, int based_nodes, int groups, int degree, int added_centers) {
  if (nodes <= 0 || based_nodes <= 0 || groups <= 0 || degree < 0 || added_centers < 0)
    return fail(GGB_EINVAL, "nodes, based_nodes, groups must be > 0 and degree, added_centers >= 0");
  if ((long long)based_nodes * groups + added_centers != nodes)
    return fail(GGB_EINVAL, "nodes (%d) != based_nodes*groups + added_centers (%d*%d+%d)", nodes,
                based_nodes, groups, added_centers);
  if ((long long)nodes * degree > INT_MAX)
    return fail(GGB_EINVAL, "nodes*degree exceeds the int32 adjacency of the reference");
  return GGB_OK;
}

int stage_adj(const int* adj, size_t n, int nodes, cudaStream_t st) {
  int rc = grow_device(&g.d_adj, &g.cap_adj, n);
  if (rc) return rc;
  rc = grow_pinned(&g.h_adj, &g.cap_hadj, n);
  if (rc) return rc;
  // Valid ids of a graph with at most 65536 vertices fit 16 bits: send them
  // narrowed (half the PCIe bytes) and widen them on the device (stage.cu).
  uint16_t* d16 = nullptr;
  if (nodes <= 65536) {
    if ((rc = grow_device(&g.d_adj16, &g.cap_adj16, n))) return rc;
    d16 = g.d_adj16;
  }
  // The pinned copy must not be overwritten while a previous copy from it is
  // in flight: the stream is idle here (every host entry point waits).
  const ggb::StageSeg seg = {adj, 0, n};
  CUDA_TRY(ggb::stage_upload_ids(g.device, g.h_adj, d16, g.d_adj, &seg, 1, n, st));
  return GGB_OK;
}

int stage_deg(const int* deg, size_t n, cudaStream_t st) {
  int rc = grow_device(&g.d_deg, &g.cap_deg, n);
  if (rc) return rc;
  rc = grow_pinned(&g.h_deg, &g.cap_hdeg, n);
  if (rc) return rc;
  std::memcpy(g.h_deg, deg, n * sizeof(int));
  CUDA_TRY(cudaMemcpyAsync(g.d_deg, g.h_deg, n * sizeof(int), cudaMemcpyHostToDevice, st));
  return GGB_OK;
}

}  // namespace

extern "C" {

const char* ggb_version(void) { return "graphgolf_b200 0.1 (sm_100a)"; }
const char* ggb_last_error(void) { return g_err; }
long long ggb_kernel_launches(void) { return g_launches; }

long long ggb_h2d_bytes(void) { return g_h2d.load(std::memory_order_relaxed); }

int ggb_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int ggb_init(int device, int nodes, int degree) {
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = ensure_ready(device);
  if (rc) return rc;
  if (nodes > 0 && degree >= 0) {
    rc = grow_device(&g.d_adj, &g.cap_adj, (size_t)nodes * degree);
    if (rc) return rc;
    rc = grow_pinned(&g.h_adj, &g.cap_hadj, (size_t)nodes * degree);
    if (rc) return rc;
  }
  return GGB_OK;
}

void ggb_finalize(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g.ready) return;
  cudaSetDevice(g.device);
  if (g.stream) cudaStreamSynchronize(g.stream);
  cudaFree(g.d_adj);
  cudaFree(g.d_adj16);
  cudaFree(g.d_adj2);
  cudaFree(g.d_rh);
  cudaFree(g.d_inv);
  cudaFree(g.d_deg);
  cudaFreeHost(g.h_deg);
  cudaFree(g.d_bufs);
  cudaFree(g.d_ctrl);
  cudaFree(g.d_trace);
  for (cudaEvent_t& e : g.ev)
    if (e) cudaEventDestroy(e);
  cudaFree(g.d_ball);
  cudaFree(g.d_ball_cnt);
  cudaFree(g.d_tgraphs);
  cudaFree(g.d_tout);
  cudaFree(g.d_tctrl);
  cudaFree(g.d_tint);
  cudaFree(g.d_tll);
  cudaFreeHost(g.h_team);
  cudaFree(g.d_stamps);
  cudaFreeHost(g.h_adj);
  cudaFreeHost(g.h_rh);
  cudaFreeHost(g.h_ctrl);
  if (g.stream) cudaStreamDestroy(g.stream);
  const int fr = g.force_R, fw = g.force_W, fc = g.force_ctas, bm = g.ball_mode;
  g = State();
  g.force_R = fr;
  g.force_W = fw;
  g.force_ctas = fc;
  g.ball_mode = bm;
}

int ggb_set_tuning(int window_bits, int ctas) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (window_bits < 0 || ctas < 0) return fail(GGB_EINVAL, "negative tuning value");
  if (window_bits && window_bits != 64) {
    if (window_bits % 128 || r_index(window_bits / 128) < 0)
      return fail(GGB_EINVAL, "window_bits must be 64 or 128 * (1,2,4,...,64)");
  }
  // 64-source windows run on one-uint4 rows (R = 1) with the upper half unused
  g.force_R = window_bits == 64 ? 1 : window_bits / 128;
  g.force_W = window_bits == 64 ? 64 : 0;
  g.force_ctas = ctas;
  return GGB_OK;
}

// Ball pre-pass policy: -1 automatic (cost model), 0 never, 1 whenever the
// sizes allow it.  Results never depend on the choice.
int ggb_set_ball(int mode) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (mode < -1 || mode > 1) return fail(GGB_EINVAL, "ball mode must be -1, 0 or 1");
  g.ball_mode = mode;
  return GGB_OK;
}

// Test hook for the bounded waits: timeout (ns) of every grid-barrier wait
// and a number of arrivals that never come.  phantom > 0 makes every wait run
// out, which must surface as GGB_ETIMEOUT with the context still usable.
int ggb_set_barrier_test(long long timeout_ns, int phantom) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (timeout_ns <= 0 || phantom < 0) return fail(GGB_EINVAL, "timeout must be > 0, phantom >= 0");
  g.timeout_ns = timeout_ns;
  g.phantom = phantom;
  return GGB_OK;
}

// Per-kernel timing with CUDA events recorded on the launching stream around
// the ball pre-pass and the persistent kernel of every following launch.
int ggb_set_timing(int enable) {
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = ensure_ready(-1);
  if (rc) return rc;
  if (enable && !g.ev[0])
    for (cudaEvent_t& e : g.ev) CUDA_TRY(cudaEventCreate(&e));
  g.timing = enable != 0;
  return GGB_OK;
}

// Milliseconds of the last launch's ball pre-pass (0 if it had none) and of
// its persistent kernel.  Waits for the launch to finish.
int ggb_kernel_times(double* ms_ball, double* ms_persistent) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g.timing || !g.ev[0]) return fail(GGB_EINVAL, "timing is not enabled");
  CUDA_TRY(cudaEventSynchronize(g.ev[2]));
  float a = 0.f, b = 0.f;
  CUDA_TRY(cudaEventElapsedTime(&a, g.ev[0], g.ev[1]));
  CUDA_TRY(cudaEventElapsedTime(&b, g.ev[1], g.ev[2]));
  if (ms_ball) *ms_ball = g.ev_ball ? a : 0.0;
  if (ms_persistent) *ms_persistent = b;
  return GGB_OK;
}

// Barrier trace: with capacity > 0, CTA 0 records (globaltimer ns, tag) after
// every grid barrier of the following evaluations; 0 turns it off.
int ggb_trace_enable(int capacity) {
  std::lock_guard<std::mutex> lk(g_mu);
  int rc = ensure_ready(-1);
  if (rc) return rc;
  if (g.d_trace) cudaFree(g.d_trace);
  g.d_trace = nullptr;
  g.trace_cap = 0;
  g.trace_len = 0;
  if (capacity > 0) {
    CUDA_TRY(cudaMalloc(&g.d_trace, (size_t)capacity * 2 * sizeof(long long)));
    g.trace_cap = capacity;
  }
  return GGB_OK;
}

// Copies the trace of the last evaluation (pairs of long long) to `out`;
// returns the number of pairs, or a negative error.
int ggb_trace_read(long long* out, int max_pairs) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g.d_trace) return 0;
  const int n = std::min(g.trace_len, max_pairs);
  if (n > 0) CUDA_TRY(cudaMemcpy(out, g.d_trace, (size_t)n * 2 * sizeof(long long), cudaMemcpyDeviceToHost));
  return n;
}

int ggb_eval_general_partial(int nodes, int based_nodes, int groups, int degree, const int* adj,
                             int added_centers, int rank, int procs, ggb_partial* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!out || (!adj && nodes * degree)) return fail(GGB_EINVAL, "null pointer");
  if (procs <= 0 || rank < 0 || rank >= procs) return fail(GGB_EINVAL, "rank %d of %d", rank, procs);
  int rc = check_general(nodes, based_nodes, groups, degree, added_centers);
  if (rc) return rc;
  rc = ensure_ready(-1);
  if (rc) return rc;
  rc = stage_adj(adj, (size_t)nodes * degree, nodes, g.stream);
  if (rc) return rc;
  rc = launch_apsp(g.d_adj, nodes, degree, based_nodes, based_nodes * groups, added_centers, groups,
                   rank, procs, g.stream);
  if (rc) return rc;
  return read_ctrl(g.stream, out);
}

int ggb_finish_general(int nodes, const ggb_partial* p, ggb_result* out) {
  if (!p || !out) return fail(GGB_EINVAL, "null pointer");
  out->levels = p->levels;
  out->dense_levels = p->dense_levels;
  out->windows = p->windows;
  out->window_bits = p->window_bits;
  // general/evaluation.c:249-262: connected iff diam < nodes.
  if (!p->disconnected && p->diam < nodes) {
    out->connected = 1;
    out->diameter = p->diam;
    out->total = p->sum + (long long)nodes * (nodes - 1);
    out->aspl = (double)out->total / (((double)nodes - 1) * nodes);
  } else {
    out->connected = 0;
    out->diameter = INT_MAX;
    out->aspl = DBL_MAX;
    out->total = 0;
  }
  return GGB_OK;
}

int ggb_finish_grid(int nodes, const ggb_partial* p, ggb_result* out) {
  if (!p || !out) return fail(GGB_EINVAL, "null pointer");
  out->levels = p->levels;
  out->dense_levels = p->dense_levels;
  out->windows = p->windows;
  out->window_bits = p->window_bits;
  // grid/evaluation.c:178-189: disconnected iff diameter > nodes; the
  // diameter is written either way, ASPL only when connected.
  const int diam = p->disconnected ? nodes + 1 : p->diam;
  out->diameter = diam;
  if (diam > nodes) {
    out->connected = 0;
    out->aspl = NAN;
    out->total = 0;
  } else {
    out->connected = 1;
    out->total = p->sum + (long long)nodes * (nodes - 1);
    out->aspl = (double)out->total / (((double)nodes - 1) * nodes);
  }
  return GGB_OK;
}

int ggb_eval_general(int nodes, int based_nodes, int groups, int degree, const int* adj,
                     int added_centers, ggb_result* out) {
  ggb_partial p;
  int rc = ggb_eval_general_partial(nodes, based_nodes, groups, degree, adj, added_centers, 0, 1, &p);
  if (rc) return rc;
  return ggb_finish_general(nodes, &p, out);
}

int ggb_launch_general_device(int nodes, int based_nodes, int groups, int degree, const int* adj_dev,
                              int added_centers, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!adj_dev && nodes * degree) return fail(GGB_EINVAL, "null adjacency");
  int rc = check_general(nodes, based_nodes, groups, degree, added_centers);
  if (rc) return rc;
  rc = ensure_ready(-1);
  if (rc) return rc;
  g.last_grid = false;
  return launch_apsp(adj_dev, nodes, degree, based_nodes, based_nodes * groups, added_centers, groups, 0,
                     1, pick_stream(stream));
}

int ggb_launch_general_partial_device(int nodes, int based_nodes, int groups, int degree, const int* adj_dev,
                                      int added_centers, int rank, int procs, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!adj_dev && nodes * degree) return fail(GGB_EINVAL, "null adjacency");
  if (procs <= 0 || rank < 0 || rank >= procs) return fail(GGB_EINVAL, "rank %d of %d", rank, procs);
  int rc = check_general(nodes, based_nodes, groups, degree, added_centers);
  if (rc) return rc;
  rc = ensure_ready(-1);
  if (rc) return rc;
  g.last_grid = false;
  return launch_apsp(adj_dev, nodes, degree, based_nodes, based_nodes * groups, added_centers, groups, rank,
                     procs, pick_stream(stream));
}

int ggb_collect_partial(void* stream, ggb_partial* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!out) return fail(GGB_EINVAL, "null pointer");
  if (!g.ready) return fail(GGB_EINVAL, "nothing launched");
  return read_ctrl(pick_stream(stream), out);
}

int ggb_collect(void* stream, ggb_result* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!out) return fail(GGB_EINVAL, "null pointer");
  if (!g.ready) return fail(GGB_EINVAL, "nothing launched");
  ggb_partial p;
  int rc = read_ctrl(pick_stream(stream), &p);
  if (rc) return rc;
  return g.last_grid ? ggb_finish_grid(g.last_N, &p, out) : ggb_finish_general(g.last_N, &p, out);
}

int ggb_eval_general_device(int nodes, int based_nodes, int groups, int degree, const int* adj_dev,
                            int added_centers, void* stream, ggb_result* out) {
  int rc = ggb_launch_general_device(nodes, based_nodes, groups, degree, adj_dev, added_centers, stream);
  if (rc) return rc;
  return ggb_collect(stream, out);
}

}  // extern "C"

namespace {

// Grid evaluation, regular (deg == nullptr) or not: relabel by rotate_hash
// on the device (padding the rows of a non-regular grid with their own id),
// check the relabel is a bijection, then run the persistent kernel.
int eval_grid_impl(int nodes, int degree, const int* deg, int groups, const int* adj, int based_nodes,
                   const int* rotate_hash, ggb_result* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!out || !rotate_hash || (!adj && nodes * degree)) return fail(GGB_EINVAL, "null pointer");
  if (nodes <= 0 || based_nodes <= 0 || groups <= 0 || degree < 0 || based_nodes > nodes)
    return fail(GGB_EINVAL, "nodes, based_nodes, groups must be > 0, degree >= 0, based_nodes <= nodes");
  if ((long long)nodes * degree > INT_MAX) return fail(GGB_EINVAL, "nodes*degree too large");
  int rc = ensure_ready(-1);
  if (rc) return rc;
  const size_t n = (size_t)nodes * degree;
  cudaStream_t st = g.stream;
  rc = stage_adj(adj, n, nodes, st);
  if (rc) return rc;
  if ((rc = grow_device(&g.d_adj2, &g.cap_adj2, n))) return rc;
  if ((rc = grow_device(&g.d_rh, &g.cap_rh, (size_t)nodes))) return rc;
  if ((rc = grow_device(&g.d_inv, &g.cap_inv, (size_t)nodes))) return rc;
  if ((rc = grow_pinned(&g.h_rh, &g.cap_hrh, (size_t)nodes))) return rc;
  if (deg && (rc = stage_deg(deg, (size_t)nodes, st))) return rc;
  std::memcpy(g.h_rh, rotate_hash, (size_t)nodes * sizeof(int));
  CUDA_TRY(cudaMemcpyAsync(g.d_rh, g.h_rh, (size_t)nodes * sizeof(int), cudaMemcpyHostToDevice, st));
  CUDA_TRY(cudaMemsetAsync(g.d_ctrl, 0, sizeof(ApspCtrl), st));
  CUDA_TRY(cudaMemsetAsync(g.d_inv, 0xff, (size_t)nodes * sizeof(int), st));
  const int threads = 256;
  const long long work = std::max<long long>((long long)n, nodes);
  const int blocks = (int)std::min<long long>((work + threads - 1) / threads, (long long)g.sms * 8);
  ggb::relabel_adjacency_kernel<<<blocks, threads, 0, st>>>(g.d_adj, g.d_rh, g.d_adj2, g.d_inv, nodes, degree,
                                                            g.d_ctrl, deg ? g.d_deg : nullptr);
  CUDA_TRY(cudaGetLastError());
  ggb::check_permutation_kernel<<<std::min(blocks, g.sms * 4), threads, 0, st>>>(g.d_inv, nodes, g.d_ctrl);
  CUDA_TRY(cudaGetLastError());
  g_launches += 2;
  CUDA_TRY(cudaMemcpyAsync(g.h_ctrl, g.d_ctrl, sizeof(ApspCtrl), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (g.h_ctrl->error == ggb::kErrAdj)
    return fail(GGB_EADJ, "adjacency entry outside [0, nodes) (row %d)", g.h_ctrl->error_info);
  if (g.h_ctrl->error == ggb::kErrDegree)
    return fail(GGB_EINVAL, "degree[%d] outside [0, max_degree]", g.h_ctrl->error_info);
  if (g.h_ctrl->error != 0)
    return fail(GGB_EPERM, "rotate_hash is not a permutation of [0, nodes) (at %d)", g.h_ctrl->error_info);
  g.last_grid = true;
  rc = launch_apsp(g.d_adj2, nodes, degree, based_nodes, nodes, 0, groups, 0, 1, st);
  if (rc) return rc;
  ggb_partial p;
  rc = read_ctrl(st, &p);
  if (rc) return rc;
  return ggb_finish_grid(nodes, &p, out);
}

}  // namespace

extern "C" {

int ggb_eval_grid(int nodes, int degree, int groups, const int* adj, int based_nodes,
                  const int* rotate_hash, ggb_result* out) {
  return eval_grid_impl(nodes, degree, nullptr, groups, adj, based_nodes, rotate_hash, out);
}

int ggb_eval_grid_nonregular(int nodes, int max_degree, const int* degree, int groups, const int* adj,
                             int based_nodes, const int* rotate_hash, ggb_result* out) {
  if (!degree) return fail(GGB_EINVAL, "null degree array");
  return eval_grid_impl(nodes, max_degree, degree, groups, adj, based_nodes, rotate_hash, out);
}

int ggb_eval_general_nonregular(int nodes, int based_nodes, int groups, int max_degree, const int* num_degrees,
                                const int* adj, int added_centers, ggb_result* out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!out || !num_degrees || (!adj && nodes * max_degree)) return fail(GGB_EINVAL, "null pointer");
  int rc = check_general(nodes, based_nodes, groups, max_degree, added_centers);
  if (rc) return rc;
  rc = ensure_ready(-1);
  if (rc) return rc;
  const size_t n = (size_t)nodes * max_degree;
  cudaStream_t st = g.stream;
  rc = stage_adj(adj, n, nodes, st);
  if (rc) return rc;
  if ((rc = grow_device(&g.d_adj2, &g.cap_adj2, n))) return rc;
  if ((rc = stage_deg(num_degrees, (size_t)nodes, st))) return rc;
  CUDA_TRY(cudaMemsetAsync(g.d_ctrl, 0, sizeof(ApspCtrl), st));
  const int threads = 256;
  const int blocks = (int)std::min<long long>(((long long)n + threads - 1) / threads + 1, (long long)g.sms * 8);
  ggb::pad_adjacency_kernel<<<blocks, threads, 0, st>>>(g.d_adj, g.d_deg, g.d_adj2, nodes, max_degree, g.d_ctrl);
  CUDA_TRY(cudaGetLastError());
  ++g_launches;
  CUDA_TRY(cudaMemcpyAsync(g.h_ctrl, g.d_ctrl, sizeof(ApspCtrl), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (g.h_ctrl->error != 0)
    return fail(GGB_EINVAL, "num_degrees[%d] outside [0, max_degree]", g.h_ctrl->error_info);
  g.last_grid = false;
  // phase 1 gathers the padded rows; the added-centre phase gathers whole rows
  // (variants/not_regular_general_graph/evaluation.c:180 vs :226)
  rc = launch_apsp(g.d_adj2, nodes, max_degree, based_nodes, based_nodes * groups, added_centers, groups, 0, 1, st,
                   added_centers ? g.d_adj : nullptr);
  if (rc) return rc;
  ggb_partial p;
  rc = read_ctrl(st, &p);
  if (rc) return rc;
  return ggb_finish_general(nodes, &p, out);
}

}  // extern "C"
