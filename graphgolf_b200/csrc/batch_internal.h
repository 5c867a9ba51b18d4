// batch_internal.h -- the batch object shared by the translation units that
// enqueue batch evaluations (the batch API and the device annealing engine).
// Not part of the public C ABI.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <vector>

#include "apsp_kernel.cuh"

struct ggb_batch {
  int device = -1;
  int sms = 0;
  size_t l2 = 0;
  int n = 0;
  std::vector<int> N, bn, grp, d;
  std::vector<long long> off;        // ints; every graph starts on a 16-byte boundary
  long long adj_ints = 0;
  int* d_adj = nullptr;
  int* h_adj = nullptr;              // pinned staging for ggb_batch_eval
  uint16_t* d_adj16 = nullptr;       // 16-bit ids on their way to d_adj (every N <= 65536)
  ggb::BatchGraph* d_graphs = nullptr;
  ggb::BatchOut* d_out = nullptr;
  ggb::BatchOut* h_out = nullptr;
  // the plan
  int R = 0, T = 0, n_teams = 0, ctas = 0;
  std::vector<int> team_start, team_list;
  std::vector<long long> team_off, team_cells;
  ggb::ApspCtrl* d_ctrl = nullptr;   // [max_teams]
  ggb::ApspCtrl* h_ctrl = nullptr;
  int* d_tstart = nullptr;           // [max_teams + 1]
  int* d_tlist = nullptr;            // [n]
  long long* d_toff = nullptr;       // [max_teams]
  long long* d_tcells = nullptr;     // [max_teams]
  uint4* d_scratch = nullptr;
  size_t cap_scratch = 0;            // uint4
  // full-row stamps of the plan (4096-source windows, some degree <= 16):
  // team t's slice starts at team_soff[t]; stamp_ints == 0 when unused
  std::vector<long long> team_soff;
  long long stamp_ints = 0;
  long long* d_tsoff = nullptr;      // [max_teams]
  unsigned* d_stamps = nullptr;
  size_t cap_stamps = 0;             // unsigned
  int occ[6] = {0, 0, 0, 0, 0, 0};   // co-resident batch CTAs per SM, per log2(R)
  int max_teams = 0;                 // largest CTA count of any plan
  long long timeout_ns = 2000000000LL;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  bool pending = false;
  const int* stop = nullptr;         // device flag: the launch does nothing while it is non-zero
  int* sticky = nullptr;             // device flag: first error code of any launch (set, never cleared)
};

namespace ggb {

// Enqueues one evaluation of the batch's device adjacency on `st` (zeroing
// of the control blocks and results, then the cooperative kernel); usable
// inside a stream capture.
int batch_enqueue(ggb_batch* b, cudaStream_t st);

}  // namespace ggb
