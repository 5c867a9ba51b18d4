// apsp_batch.cu -- exact APSP of many graphs, of uneven sizes, in one launch.
//
// A batch is a fixed list of graphs (nodes, based_nodes, groups, degree each)
// whose adjacency arrays sit packed in one device buffer.  One cooperative
// launch of apsp_batch_kernel evaluates all of them: the launch's CTAs form
// teams of `team_ctas` CTAs, the graphs are dealt to the teams longest-first
// (each to the team with the least modelled work so far), and every team
// runs its graphs' source windows exactly as the single-graph kernel runs one
// graph's, with a barrier of its own.  Per graph the answer is the one
// ggb_eval_general gives (general/evaluation.c:153-263 per graph); the plan
// -- window width and team size -- changes only the time.
//
// The launch (two memsets of the control blocks and the kernel) is captured
// once per plan in a CUDA graph and replayed, so a step of a batched
// annealing loop costs one graph launch.  ggb_batch_autotune times every
// feasible (window width, team size) pair on the batch's current adjacency
// and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <queue>
#include <vector>

#include "../../include/graphgolf_b200.h"
#include "apsp_kernel.cuh"
#include "batch_internal.h"
#include "core_internal.h"

using ggb::core_fail;

#define BCUDA(call)                                                                                  \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return core_fail(GGB_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                       __LINE__);                                                                    \
  } while (0)

namespace {

constexpr int kMaxR = 32;   // widest window of the batch kernel: 4096 sources

const void* batch_kernel_for(int R) {
  switch (R) {
    case 1: return (const void*)ggb::apsp_batch_kernel<1>;
    case 2: return (const void*)ggb::apsp_batch_kernel<2>;
    case 4: return (const void*)ggb::apsp_batch_kernel<4>;
    case 8: return (const void*)ggb::apsp_batch_kernel<8>;
    case 16: return (const void*)ggb::apsp_batch_kernel<16>;
    case 32: return (const void*)ggb::apsp_batch_kernel<32>;
    default: return nullptr;
  }
}

size_t batch_smem_for(int R) {
  switch (R) {
    case 1: return ggb::apsp_smem_bytes<1>();
    case 2: return ggb::apsp_smem_bytes<2>();
    case 4: return ggb::apsp_smem_bytes<4>();
    case 8: return ggb::apsp_smem_bytes<8>();
    case 16: return ggb::apsp_smem_bytes<16>();
    case 32: return ggb::apsp_smem_bytes<32>();
    default: return 0;
  }
}

int log2i(int x) {
  int r = 0;
  while ((1 << r) < x) ++r;
  return r;
}

template <typename T>
int dev_alloc(T** p, size_t n) {
  if (cudaMalloc(p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return core_fail(GGB_ENOMEM, "cudaMalloc of %zu bytes failed", n * sizeof(T));
  }
  return GGB_OK;
}

}  // namespace

namespace {

// Modelled seconds of one graph on a team of T CTAs with windows of 128*R
// sources: per window the two-hop seeding plus about five dense sweeps of
// d gathered 16R-byte rows per vertex, each sweep at least one memory round
// trip and one team barrier.  A CTA gathers about 1e11 bytes/s from L2.
double graph_cost(int N, int d, int nsrc, int R, int T) {
  const double W = 128.0 * R;
  const double nwin = std::ceil(nsrc / W);
  const double dd = std::max(d, 1);
  const double rate = 1.0e11 * T;
  const double bar = 1.5e-6 + 0.01e-6 * T;
  const double seed = (double)N * (dd + dd * dd) * 4.0 / rate + bar + 1.5e-6;
  const double level = std::max((double)N * (dd * (16.0 * R + 4.0) + 32.0 * R) / rate, 1.5e-6) + bar;
  return nwin * (seed + 5.0 * level);
}

// Deals the graphs to the teams (longest first, each to the least loaded
// team) and returns the modelled makespan; fills the plan arrays when
// `keep`.
double make_plan(ggb_batch* b, int R, int T, bool keep) {
  const int ctas_max = b->occ[log2i(R)] * b->sms;
  T = std::max(1, std::min(T, ctas_max));
  int n_teams = std::max(1, std::min(ctas_max / T, b->n));
  std::vector<double> cost(b->n);
  for (int i = 0; i < b->n; ++i) cost[i] = graph_cost(b->N[i], b->d[i], b->bn[i], R, T);
  std::vector<int> order(b->n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  using Load = std::pair<double, int>;
  std::priority_queue<Load, std::vector<Load>, std::greater<Load>> pq;
  for (int t = 0; t < n_teams; ++t) pq.push({0.0, t});
  std::vector<std::vector<int>> lists(n_teams);
  double makespan = 0.0;
  for (int i : order) {
    Load l = pq.top();
    pq.pop();
    l.first += cost[i];
    lists[l.second].push_back(i);
    makespan = std::max(makespan, l.first);
    pq.push(l);
  }
  // Working set of the teams running at once: each team's adjacency and two
  // matrices.  Past about 60% of L2 the gathers spill to HBM.
  double ws = 0.0;
  for (int t = 0; t < n_teams; ++t) {
    long long mx = 0;
    for (int i : lists[t]) mx = std::max<long long>(mx, (long long)b->N[i] * (b->d[i] * 4 + 32 * R));
    ws += (double)mx;
  }
  if (ws > 0.6 * (double)b->l2) makespan *= 1.0 + 1.5 * std::min(1.0, (ws - 0.6 * b->l2) / (0.6 * b->l2));
  if (!keep) return makespan;
  b->R = R;
  b->T = T;
  b->n_teams = n_teams;
  b->ctas = n_teams * T;
  b->team_start.assign(n_teams + 1, 0);
  b->team_list.clear();
  b->team_off.assign(n_teams, 0);
  b->team_cells.assign(n_teams, 0);
  long long off = 0;
  for (int t = 0; t < n_teams; ++t) {
    b->team_start[t] = (int)b->team_list.size();
    long long cells = 1;
    for (int i : lists[t]) {
      b->team_list.push_back(i);
      cells = std::max<long long>(cells, (long long)b->N[i] * R);
    }
    b->team_off[t] = off;
    b->team_cells[t] = cells;
    off += 2 * cells;
  }
  b->team_start[n_teams] = (int)b->team_list.size();
  // Stamps pay where the stamping sweeps run: 4096-source windows, degree <= 16.
  b->team_soff.assign(n_teams, 0);
  b->stamp_ints = 0;
  bool stamping = false;
  for (int i = 0; i < b->n; ++i) stamping = stamping || (R == 32 && b->d[i] <= 16);
  if (stamping) {
    for (int t = 0; t < n_teams; ++t) {
      int mx = 0;
      for (int k = b->team_start[t]; k < b->team_start[t + 1]; ++k) mx = std::max(mx, b->N[b->team_list[k]]);
      b->team_soff[t] = b->stamp_ints;
      b->stamp_ints += (mx + 31) / 32 * 32;   // each slice on a 128-byte boundary
    }
  }
  return makespan;
}

int drop_graph(ggb_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
  return GGB_OK;
}

// Uploads the plan made by make_plan(keep = true).
int upload_plan(ggb_batch* b) {
  drop_graph(b);
  const long long cells = b->team_off.back() + 2 * b->team_cells.back();
  if ((size_t)cells > b->cap_scratch) {
    if (b->d_scratch) cudaFree(b->d_scratch);
    b->d_scratch = nullptr;
    b->cap_scratch = 0;
    int rc = dev_alloc(&b->d_scratch, (size_t)cells);
    if (rc) return rc;
    b->cap_scratch = (size_t)cells;
  }
  BCUDA(cudaMemcpyAsync(b->d_tstart, b->team_start.data(), b->team_start.size() * sizeof(int),
                        cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaMemcpyAsync(b->d_tlist, b->team_list.data(), b->team_list.size() * sizeof(int),
                        cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaMemcpyAsync(b->d_toff, b->team_off.data(), b->team_off.size() * sizeof(long long),
                        cudaMemcpyHostToDevice, b->stream));
  BCUDA(cudaMemcpyAsync(b->d_tcells, b->team_cells.data(), b->team_cells.size() * sizeof(long long),
                        cudaMemcpyHostToDevice, b->stream));
  if (b->stamp_ints > 0) {
    if ((size_t)b->stamp_ints > b->cap_stamps) {
      if (b->d_stamps) cudaFree(b->d_stamps);
      b->d_stamps = nullptr;
      b->cap_stamps = 0;
      int rc = dev_alloc(&b->d_stamps, (size_t)b->stamp_ints);
      if (rc) return rc;
      b->cap_stamps = (size_t)b->stamp_ints;
    }
    BCUDA(cudaMemcpyAsync(b->d_tsoff, b->team_soff.data(), b->team_soff.size() * sizeof(long long),
                          cudaMemcpyHostToDevice, b->stream));
  }
  BCUDA(cudaStreamSynchronize(b->stream));
  return GGB_OK;
}

ggb::BatchArgs batch_args(const ggb_batch* b) {
  ggb::BatchArgs a;
  a.graphs = b->d_graphs;
  a.out = b->d_out;
  a.team_ctrl = b->d_ctrl;
  a.team_start = b->d_tstart;
  a.team_list = b->d_tlist;
  a.scratch = b->d_scratch;
  a.team_off = b->d_toff;
  a.team_cells = b->d_tcells;
  a.timeout_ns = b->timeout_ns;
  a.stop = b->stop;
  a.sticky = b->sticky;
  a.n_teams = b->n_teams;
  a.team_ctas = b->T;
  a.stamps = b->stamp_ints > 0 ? b->d_stamps : nullptr;
  a.team_soff = b->stamp_ints > 0 ? b->d_tsoff : nullptr;
  return a;
}

}  // namespace

// The launch itself: zero the control blocks and results, then the kernel.
int ggb::batch_enqueue(ggb_batch* b, cudaStream_t st) {
  BCUDA(cudaMemsetAsync(b->d_ctrl, 0, (size_t)b->n_teams * sizeof(ggb::ApspCtrl), st));
  BCUDA(cudaMemsetAsync(b->d_out, 0, (size_t)b->n * sizeof(ggb::BatchOut), st));
  if (b->stamp_ints > 0) BCUDA(cudaMemsetAsync(b->d_stamps, 0, (size_t)b->stamp_ints * sizeof(unsigned), st));
  ggb::BatchArgs args = batch_args(b);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(b->ctas);
  cfg.blockDim = dim3(ggb::kThreads);
  cfg.dynamicSmemBytes = batch_smem_for(b->R);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* params[] = {(void*)&args};
  BCUDA(cudaLaunchKernelExC(&cfg, batch_kernel_for(b->R), params));
  return GGB_OK;
}

namespace {

int capture(ggb_batch* b) {
  if (b->exec) return GGB_OK;
  BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = ggb::batch_enqueue(b, b->stream);
  cudaGraph_t gph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(b->stream, &gph);
  if (rc) {
    if (gph) cudaGraphDestroy(gph);
    return rc;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return core_fail(GGB_ECUDA, "capturing the batch launch failed: %s", cudaGetErrorString(e));
  }
  b->graph = gph;
  BCUDA(cudaGraphInstantiate(&b->exec, gph, 0));
  return GGB_OK;
}

int launch(ggb_batch* b, cudaStream_t st, bool use_graph) {
  BCUDA(cudaSetDevice(b->device));
  BCUDA(cudaEventRecord(b->ev[0], st));
  if (use_graph) {
    int rc = capture(b);
    if (rc) return rc;
    BCUDA(cudaGraphLaunch(b->exec, st));
  } else {
    int rc = ggb::batch_enqueue(b, st);
    if (rc) return rc;
  }
  BCUDA(cudaEventRecord(b->ev[1], st));
  ggb::core_add_launches(1);
  b->pending = true;
  return GGB_OK;
}

int collect(ggb_batch* b, cudaStream_t st, ggb_result* res) {
  BCUDA(cudaMemcpyAsync(b->h_out, b->d_out, (size_t)b->n * sizeof(ggb::BatchOut), cudaMemcpyDeviceToHost, st));
  BCUDA(cudaMemcpyAsync(b->h_ctrl, b->d_ctrl, (size_t)b->n_teams * sizeof(ggb::ApspCtrl), cudaMemcpyDeviceToHost,
                        st));
  BCUDA(cudaStreamSynchronize(st));
  b->pending = false;
  for (int t = 0; t < b->n_teams; ++t) {
    const ggb::ApspCtrl& c = b->h_ctrl[t];
    if (c.error == 0) continue;
    int gi = -1;
    for (int k = b->team_start[t]; k < b->team_start[t + 1]; ++k)
      if (!b->h_out[b->team_list[k]].done) { gi = b->team_list[k]; break; }
    if (c.error == ggb::kErrAdj)
      return core_fail(GGB_EADJ, "batch graph %d: adjacency entry outside [0, nodes)", gi);
    if (c.error == ggb::kErrTimeout)
      return core_fail(GGB_ETIMEOUT, "batch graph %d: a team-barrier wait ran out (CTA %d)", gi, c.error_info);
    return core_fail(GGB_ECUDA, "batch graph %d: device error code %d", gi, c.error);
  }
  for (int i = 0; i < b->n; ++i) {
    const ggb::BatchOut& o = b->h_out[i];
    if (!o.done) return core_fail(GGB_ECUDA, "batch graph %d was not evaluated", i);
    if (!res) continue;
    ggb_partial p;
    p.diam = o.diam;
    p.disconnected = o.disconnected;
    p.sum = o.sum;
    p.levels = o.levels;
    p.windows = o.windows;
    p.window_bits = 128 * b->R;
    p.dense_levels = o.dense_levels;
    int rc = ggb_finish_general(b->N[i], &p, res + i);
    if (rc) return rc;
  }
  return GGB_OK;
}

void destroy(ggb_batch* b) {
  if (!b) return;
  if (b->device >= 0) cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  cudaFree(b->d_adj);
  cudaFree(b->d_adj16);
  cudaFreeHost(b->h_adj);
  cudaFree(b->d_graphs);
  cudaFree(b->d_out);
  cudaFreeHost(b->h_out);
  cudaFree(b->d_ctrl);
  cudaFreeHost(b->h_ctrl);
  cudaFree(b->d_tstart);
  cudaFree(b->d_tlist);
  cudaFree(b->d_toff);
  cudaFree(b->d_tcells);
  cudaFree(b->d_tsoff);
  cudaFree(b->d_stamps);
  cudaFree(b->d_scratch);
  for (auto& e : b->ev)
    if (e) cudaEventDestroy(e);
  if (b->stream) cudaStreamDestroy(b->stream);
  cudaGetLastError();
  delete b;
}

int create(int n_graphs, const int* nodes, const int* based_nodes, const int* groups, const int* degree,
           ggb_batch* b) {
  b->n = n_graphs;
  b->N.assign(nodes, nodes + n_graphs);
  b->bn.assign(based_nodes, based_nodes + n_graphs);
  b->grp.assign(groups, groups + n_graphs);
  b->d.assign(degree, degree + n_graphs);
  b->off.resize(n_graphs);
  long long off = 0;
  for (int i = 0; i < n_graphs; ++i) {
    const int Ni = nodes[i], bi = based_nodes[i], gi = groups[i], di = degree[i];
    if (Ni <= 0 || bi <= 0 || gi <= 0 || di < 0)
      return core_fail(GGB_EINVAL, "batch graph %d: nodes, based_nodes, groups must be > 0, degree >= 0", i);
    if ((long long)bi * gi != Ni)
      return core_fail(GGB_EINVAL, "batch graph %d: nodes (%d) != based_nodes*groups (%d*%d)", i, Ni, bi, gi);
    if ((long long)Ni * di > INT_MAX) return core_fail(GGB_EINVAL, "batch graph %d: nodes*degree too large", i);
    b->off[i] = off;
    off += ((long long)Ni * di + 3) / 4 * 4;
  }
  b->adj_ints = off;
  int dev = 0;
  BCUDA(cudaGetDevice(&dev));
  b->device = dev;
  BCUDA(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev));
  int l2 = 0;
  BCUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
  b->l2 = (size_t)l2;
  for (int R = 1; R <= kMaxR; R *= 2) {
    int nb = 0;
    BCUDA(cudaFuncSetAttribute(batch_kernel_for(R), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)batch_smem_for(R)));
    BCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, batch_kernel_for(R), ggb::kThreads,
                                                        batch_smem_for(R)));
    if (nb < 1) return core_fail(GGB_ECUDA, "batch kernel R=%d cannot be resident", R);
    b->occ[log2i(R)] = nb;
    b->max_teams = std::max(b->max_teams, nb * b->sms);
  }
  if (const char* s = getenv("GGB_BARRIER_TIMEOUT_NS")) b->timeout_ns = atoll(s);
  BCUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  BCUDA(cudaEventCreate(&b->ev[0]));
  BCUDA(cudaEventCreate(&b->ev[1]));
  int rc = dev_alloc(&b->d_adj, (size_t)b->adj_ints);
  if (rc) return rc;
  if (cudaHostAlloc(&b->h_adj, std::max<size_t>((size_t)b->adj_ints, 1) * sizeof(int), cudaHostAllocDefault) !=
      cudaSuccess) {
    cudaGetLastError();
    b->h_adj = nullptr;
    return core_fail(GGB_ENOMEM, "pinned staging of %lld ints failed", b->adj_ints);
  }
  // Graphs of at most 65536 vertices have 16-bit ids: uploads send them narrowed.
  if (*std::max_element(b->N.begin(), b->N.end()) <= 65536 &&
      (rc = dev_alloc(&b->d_adj16, (size_t)b->adj_ints)))
    return rc;
  if ((rc = dev_alloc(&b->d_graphs, (size_t)n_graphs))) return rc;
  if ((rc = dev_alloc(&b->d_out, (size_t)n_graphs))) return rc;
  const size_t mt = (size_t)b->max_teams;
  if ((rc = dev_alloc(&b->d_ctrl, mt))) return rc;
  if ((rc = dev_alloc(&b->d_tstart, mt + 1))) return rc;
  if ((rc = dev_alloc(&b->d_tlist, (size_t)n_graphs))) return rc;
  if ((rc = dev_alloc(&b->d_toff, mt))) return rc;
  if ((rc = dev_alloc(&b->d_tcells, mt))) return rc;
  if ((rc = dev_alloc(&b->d_tsoff, mt))) return rc;
  BCUDA(cudaHostAlloc(&b->h_out, (size_t)n_graphs * sizeof(ggb::BatchOut), cudaHostAllocDefault));
  BCUDA(cudaHostAlloc(&b->h_ctrl, mt * sizeof(ggb::ApspCtrl), cudaHostAllocDefault));
  std::vector<ggb::BatchGraph> gs(n_graphs);
  for (int i = 0; i < n_graphs; ++i) {
    gs[i].adj = b->d_adj + b->off[i];
    gs[i].N = b->N[i];
    gs[i].d = b->d[i];
    gs[i].n_src = b->bn[i];
    gs[i].groups = b->grp[i];
    gs[i].vec4 = (b->d[i] % 4 == 0) ? 1 : 0;   // every graph starts on a 16-byte boundary
    gs[i].win_first = 0;
    gs[i].win_stride = 1;
    gs[i].win_bits = 0;
  }
  BCUDA(cudaMemcpy(b->d_graphs, gs.data(), gs.size() * sizeof(ggb::BatchGraph), cudaMemcpyHostToDevice));
  BCUDA(cudaMemset(b->d_adj, 0, std::max<size_t>((size_t)b->adj_ints, 1) * sizeof(int)));
  return ggb_batch_set_plan(b, 0, 0);
}

// The plan the model prefers: the (R, T) pair with the least modelled makespan.
void model_choice(ggb_batch* b, int* R, int* T) {
  double best = 1e300;
  int nsrc_max = *std::max_element(b->bn.begin(), b->bn.end());
  for (int r = 1; r <= kMaxR; r *= 2) {
    for (int t = 1; t <= b->occ[log2i(r)] * b->sms; t *= 2) {
      const double m = make_plan(b, r, t, false);
      if (m < best * 0.999) { best = m; *R = r; *T = t; }
    }
    if (128 * r >= nsrc_max) break;
  }
}

}  // namespace

extern "C" {

int ggb_batch_create(int n_graphs, const int* nodes, const int* based_nodes, const int* groups, const int* degree,
                     ggb_batch** out) {
  if (!out || !nodes || !based_nodes || !groups || !degree || n_graphs <= 0)
    return core_fail(GGB_EINVAL, "ggb_batch_create: null pointer or n_graphs <= 0");
  *out = nullptr;
  ggb_batch* b = new ggb_batch();
  int rc = create(n_graphs, nodes, based_nodes, groups, degree, b);
  if (rc) {
    destroy(b);
    return rc;
  }
  *out = b;
  return GGB_OK;
}

void ggb_batch_destroy(ggb_batch* b) { destroy(b); }

int ggb_batch_set_plan(ggb_batch* b, int window_bits, int team_ctas) {
  if (!b) return core_fail(GGB_EINVAL, "null batch");
  if (window_bits < 0 || team_ctas < 0) return core_fail(GGB_EINVAL, "negative plan value");
  int R = window_bits / 128, T = team_ctas;
  if (window_bits && (window_bits % 128 || (R & (R - 1)) || R > kMaxR))
    return core_fail(GGB_EINVAL, "window_bits must be 128 * 2^k, at most %d", 128 * kMaxR);
  BCUDA(cudaSetDevice(b->device));
  if (!R || !T) {
    int mr = 1, mt = 1;
    model_choice(b, &mr, &mt);
    if (!R) R = mr;
    if (!T) T = mt;
  }
  make_plan(b, R, T, true);
  return upload_plan(b);
}

int ggb_batch_get_plan(const ggb_batch* b, int* window_bits, int* team_ctas, int* teams) {
  if (!b) return core_fail(GGB_EINVAL, "null batch");
  if (window_bits) *window_bits = 128 * b->R;
  if (team_ctas) *team_ctas = b->T;
  if (teams) *teams = b->n_teams;
  return GGB_OK;
}

int ggb_batch_adj_device(ggb_batch* b, int graph, int** adj_dev) {
  if (!b || !adj_dev || graph < 0 || graph >= b->n) return core_fail(GGB_EINVAL, "bad batch graph index");
  *adj_dev = b->d_adj + b->off[graph];
  return GGB_OK;
}

int ggb_batch_upload(ggb_batch* b, const int* const* adj, void* stream) {
  if (!b || !adj) return core_fail(GGB_EINVAL, "null pointer");
  BCUDA(cudaSetDevice(b->device));
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  // The staging buffer may still feed an earlier copy on this stream.
  BCUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < b->n; ++i)
    if ((size_t)b->N[i] * b->d[i] && !adj[i]) return core_fail(GGB_EINVAL, "batch graph %d: null adjacency", i);
  // The copy into the pinned buffer is spread over the staging threads; each
  // unit of 128 Ki ids or more is sent as soon as it is copied, as 16-bit ids
  // when they fit (stage.cu).
  std::vector<ggb::StageSeg> segs(b->n);
  for (int i = 0; i < b->n; ++i) segs[i] = {adj[i], (size_t)b->off[i], (size_t)b->N[i] * b->d[i]};
  BCUDA(ggb::stage_upload_ids(b->device, b->h_adj, b->d_adj16, b->d_adj, segs.data(), b->n, (size_t)b->adj_ints,
                              st));
  return GGB_OK;
}

int ggb_batch_launch(ggb_batch* b, void* stream) {
  if (!b) return core_fail(GGB_EINVAL, "null batch");
  return launch(b, stream ? (cudaStream_t)stream : b->stream, true);
}

int ggb_batch_collect(ggb_batch* b, void* stream, ggb_result* results) {
  if (!b) return core_fail(GGB_EINVAL, "null batch");
  BCUDA(cudaSetDevice(b->device));
  return collect(b, stream ? (cudaStream_t)stream : b->stream, results);
}

int ggb_batch_eval(ggb_batch* b, const int* const* adj, ggb_result* results) {
  int rc = ggb_batch_upload(b, adj, nullptr);
  if (rc) return rc;
  rc = launch(b, b->stream, true);
  if (rc) return rc;
  return collect(b, b->stream, results);
}

int ggb_batch_kernel_ms(const ggb_batch* b, double* ms) {
  if (!b || !ms) return core_fail(GGB_EINVAL, "null pointer");
  if (b->pending) return core_fail(GGB_EPERM, "the last launch has not been collected");
  float f = 0.f;
  BCUDA(cudaEventElapsedTime(&f, b->ev[0], b->ev[1]));
  *ms = f;
  return GGB_OK;
}

int ggb_batch_autotune(ggb_batch* b, int iters, int* window_bits, int* team_ctas, double* best_ms) {
  if (!b) return core_fail(GGB_EINVAL, "null batch");
  if (iters <= 0) iters = 2;
  BCUDA(cudaSetDevice(b->device));
  const int nsrc_max = *std::max_element(b->bn.begin(), b->bn.end());
  double best = 1e300;
  int bR = b->R, bT = b->T;
  for (int r = 1; r <= kMaxR; r *= 2) {
    const int ctas_max = b->occ[log2i(r)] * b->sms;
    std::vector<int> ts;
    for (int t = 1; t <= ctas_max; t *= 2) ts.push_back(t);
    for (int t : {b->sms / 4, b->sms / 2, b->sms})
      if (t >= 1 && t <= ctas_max && std::find(ts.begin(), ts.end(), t) == ts.end()) ts.push_back(t);
    for (int t : ts) {
      make_plan(b, r, t, true);
      int rc = upload_plan(b);
      if (rc) return rc;
      double ms_min = 1e300;
      for (int it = 0; it <= iters; ++it) {
        rc = launch(b, b->stream, false);
        if (rc) return rc;
        rc = collect(b, b->stream, nullptr);
        if (rc) return rc;
        float f = 0.f;
        BCUDA(cudaEventElapsedTime(&f, b->ev[0], b->ev[1]));
        if (it > 0) ms_min = std::min(ms_min, (double)f);   // the first launch warms up
      }
      if (ms_min < best) { best = ms_min; bR = r; bT = t; }
    }
    if (128 * r >= nsrc_max) break;   // wider windows only add zero bits
  }
  make_plan(b, bR, bT, true);
  int rc = upload_plan(b);
  if (rc) return rc;
  if (window_bits) *window_bits = 128 * bR;
  if (team_ctas) *team_ctas = bT;
  if (best_ms) *best_ms = best;
  return GGB_OK;
}

}  // extern "C"
