// apsp_delta.cuh -- exact evaluation of 2-opt candidates relative to a base.
//
// A 2-opt swap changes four adjacency entries, and only a few thousand of
// the N^2 distances.  The base build (apsp_base_kernel) evaluates the
// current graph once with windows of 1024 sources and keeps every level's
// bitset rows S_k; base_counts_kernel and sub_levels_kernel derive each
// level's popcount and the completion level of every 128-source sub-window.
// A candidate is then evaluated sub-window by sub-window from the base alone:
//
//   S'_0 = S_0 (the identity), and for k >= 0
//   S'_{k+1}[v] = S'_k[v] | OR_{u in N'(v)} S'_k[u]          (the recurrence of
//                                                             apsp_kernel.cuh)
//
// S'_{k+1}[v] can differ from S_{k+1}[v] only if v's neighbour list changed
// (the four endpoints P) or v or one of its neighbours differed at level k.
// So level k+1 is re-derived only on P, the dirty set D_k = {v : S'_k[v] !=
// S_k[v]} and the neighbours of D_k; rows that come out equal to the base are
// dropped, the others form D_{k+1}, and the level's popcount changes by
// delta_{k+1} = sum over D_{k+1} of popc(S'_{k+1}[v]) - popc(S_{k+1}[v]).
// With C_k the base counts (N*l from the base's completion level on), the
// candidate's window is complete at the first k with C_k + delta_k == N*l,
// and its distance sum is the base's minus sum_k delta_k -- the same
// integers the full evaluation produces (general/evaluation.c:183-200 per
// level).  A stall (a level that adds nothing before completion) is a
// disconnected candidate.  A window whose dirty set outgrows the task's
// shared memory (typically one holding a swap endpoint, whose own distances
// change for many vertices) continues as a dense sweep of that window alone,
// in a slot of a scratch pool; only when the pool is exhausted does it
// report "not evaluated" instead of guessing.
#pragma once
#include <cuda_runtime.h>

#include "apsp_kernel.cuh"

namespace ggb {

// One 2-opt swap in canonical form: lines line[0] = {x0,x1} and
// line[1] = {x2,x3} become {x0,x2} and {x1,x3}.  pos[k] is the slot of row
// x_k whose entry changes: row x0: x1 -> x2, row x1: x0 -> x3,
// row x2: x3 -> x0, row x3: x2 -> x1.  A valid swap has 4 distinct endpoints.
// On a graph with symmetry groups (the annealer's orbit moves) the swap is
// applied to every copy of the two lines (kind 0), or it re-pairs the edge
// orbit of line[0] = {x0,x1} with shift x2 (kind 1, x3 unused); pos is then
// unused and each copy's slot is found by value.
struct Swap {
  int line[2];
  int x[4];
  int pos[4];
  int valid;
  int kind;
};

// ---- the base build: one graph, windows split over CTA teams, levels kept ------
// The base is evaluated with windows of 1024 sources (rows of kBaseR = 8
// uint4) and keeps every level in the evaluator's own layout
// [window][level][vertex][8]; its readers serve 128-source sub-windows: sub-
// window s is chunk s % 8 of window s / 8.
constexpr int kBaseR = 8;

__device__ __forceinline__ const uint4* sub_row(const uint4* levels, int cap, int N, int s, int k, int v) {
  return levels + ((((size_t)(s >> 3) * (cap + 1) + k) * N + v) << 3) + (s & 7);
}

struct BaseResult {
  long long sum;          // the graph's distance sum before + N(N-1)
  int diam;
  int disconnected;
  int bad;                // windows whose levels did not fit (or that stalled)
  int pad_;
};

struct BaseArgs {
  ApspCtrl* grid_ctrl;    // one barrier over the whole launch, zeroed before it
  ApspCtrl* team_ctrl;    // [n_teams], zeroed before the launch
  uint4* scratch;         // team t: 2*N*R cells at scratch + t*2*N*R
  BaseResult* result;     // written by the launch
  const int* gate;        // the launch does nothing while *gate == 0 (null: always runs)
  int* sticky;            // first error code (never cleared here)
  long long* sub_counts;  // per 128-source sub-window and level, zeroed here for base_counts_kernel
  long long sub_count_len;
  int n_teams, team_ctas;
};

// Team t evaluates windows t, t + n_teams, ... of the graph in `a` (phase 1
// only), writing their levels, counts and completion levels into a's level
// arrays and, when a.stats is set, the per-vertex statistics.
template <int R>
__global__ void __launch_bounds__(kThreads, 1) apsp_base_kernel(ApspArgs a, const BaseArgs b) {
  __shared__ ApspSmem sm;
  extern __shared__ unsigned s_dyn[];
  if (b.gate && ld_volatile_i32(b.gate) == 0) return;   // written before the launch: the same in every CTA
  const long long n_tid = (long long)gridDim.x * blockDim.x;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (a.stats)
    for (long long i = tid; i < (long long)a.N * kStatLevels; i += n_tid) a.stats[i] = 0u;
  for (long long i = tid; i < b.sub_count_len; i += n_tid) b.sub_counts[i] = 0;
  if (tid == 0) {
    b.result->sum = 0;
    b.result->diam = 1;
    b.result->disconnected = 0;
    b.result->bad = 0;
  }
  if (threadIdx.x < 8) sm.seen[threadIdx.x >> 1][threadIdx.x & 1] = 0ULL;
  unsigned long long gt = gridDim.x;
  if (!grid_barrier(b.grid_ctrl, gt, a.timeout_ns, &sm.flag)) {
    if (b.sticky && threadIdx.x == 0) atomicCAS(b.sticky, 0, kErrTimeout);
    return;
  }
  const int team = (int)blockIdx.x / b.team_ctas, cta = (int)blockIdx.x % b.team_ctas;
  if (team >= b.n_teams) return;
  a.ctrl = b.team_ctrl + team;
  a.win_first = team;
  a.win_stride = b.n_teams;
  a.buf0 = b.scratch + (size_t)team * 2 * a.N * R;
  a.buf1 = a.buf0 + (size_t)a.N * R;
  unsigned long long bar_target = 0;
  unsigned gl = 0;
  int ntrace = 0;
  EvalOut o;
  const bool ok = a.stats ? eval_windows<R, true>(a, cta, b.team_ctas, sm, s_dyn, bar_target, gl, ntrace, o)
                          : eval_windows<R, false>(a, cta, b.team_ctas, sm, s_dyn, bar_target, gl, ntrace, o);
  if (!ok) {
    if (b.sticky && threadIdx.x == 0) atomicCAS(b.sticky, 0, max(1, ld_volatile_i32(&a.ctrl->error)));
    return;
  }
  if (cta == 0 && threadIdx.x == 0 && o.windows > 0) {
    atomicAdd(reinterpret_cast<unsigned long long*>(&b.result->sum), (unsigned long long)o.sum);
    atomicMax(&b.result->diam, o.diam);
    atomicOr(&b.result->disconnected, o.disconnected);
  }
}

// ---- per-vertex statistics and sub-window counts from the kept levels -------------
// One pass over the base's rows: stats[v][k] = sum over sub-windows of
// (l - popc(S_k[v])) for k < kStatLevels (the sources not within distance k
// of v -- the statistics the profile kernel accumulates during its sweeps),
// and sub_counts[s][k] = popcount of sub-window s at level k (what the delta
// evaluation compares against).  A block takes 32 vertices, whose rows of one
// (window, level) are 4 KB of contiguous memory, and its 8 warps split the
// windows.  A warp reads them in eight 512-byte loads, lane = (row r of four,
// chunk c): a row's total is reduced over its 8 lanes into shared memory, a
// chunk's over the lanes holding it and added atomically (lanes 0..7).
// Levels past a window's completion are full and add nothing.  Runs only
// while *gate != 0.
constexpr int kStatsWarps = 8;
__global__ void __launch_bounds__(kStatsWarps * 32) base_counts_kernel(const uint4* __restrict__ levels,
                                                                       const int* __restrict__ win_levels, int cap,
                                                                       int N, int nbw, int n_src,
                                                                       unsigned* __restrict__ stats,
                                                                       long long* __restrict__ sub_counts,
                                                                       const int* gate) {
  static_assert(kBaseR == 8, "a lane reads one 16-byte chunk of a 128-byte row");
  __shared__ unsigned s_part[kStatsWarps][kStatLevels][32];
  if (gate && ld_volatile_i32(gate) == 0) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = lane & 7, rl = lane >> 3;
  const int v0 = blockIdx.x * 32;
  for (int i = lane; i < kStatLevels * 32; i += 32) (&s_part[warp][0][0])[i] = 0u;
  __syncwarp();
  for (int t = warp; t < nbw; t += kStatsWarps) {        // warp-uniform
    const int lsub = max(0, min(128, n_src - (t * kBaseR + c) * 128));   // sources of chunk c
    const unsigned lw = (unsigned)max(0, min(128 * kBaseR, n_src - t * 128 * kBaseR));
    const int L = win_levels[t];
    const int top = min(L > 0 ? L : cap, cap);
    if (v0 + lane < N) s_part[warp][0][lane] += lw - ((unsigned)(v0 + lane - t * 128 * kBaseR) < lw ? 1u : 0u);
    for (int k = 1; k <= top; ++k) {                     // counts of every kept level
      const bool stat = k < kStatLevels;                   // statistics of the first 32
      const uint4* rows = levels + (((size_t)t * (cap + 1) + k) * N + v0) * kBaseR;
      uint4 x[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int r = 4 * i + rl;
        x[i] = v0 + r < N ? __ldg(rows + r * kBaseR + c) : make_uint4(0u, 0u, 0u, 0u);
      }
      unsigned csum = 0;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int r = 4 * i + rl;
        const unsigned pc = popc4(x[i]);
        csum += pc;
        unsigned rs = pc;
        rs += __shfl_xor_sync(0xffffffffu, rs, 1);
        rs += __shfl_xor_sync(0xffffffffu, rs, 2);
        rs += __shfl_xor_sync(0xffffffffu, rs, 4);
        if (stat && c == 0 && v0 + r < N) s_part[warp][k][r] += lw - rs;
      }
      csum += __shfl_xor_sync(0xffffffffu, csum, 8);
      csum += __shfl_xor_sync(0xffffffffu, csum, 16);
      if (lane < 8 && lsub > 0)
        atomicAdd(reinterpret_cast<unsigned long long*>(sub_counts) + (size_t)(t * kBaseR + c) * (cap + 1) + k,
                  (unsigned long long)csum);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 32 * kStatLevels; i += blockDim.x) {
    const int vl = i / kStatLevels, k = i % kStatLevels;
    const int vv = v0 + vl;
    if (vv >= N) continue;
    unsigned t = 0u;
#pragma unroll
    for (int q = 0; q < kStatsWarps; ++q) t += s_part[q][k][vl];
    stats[(size_t)vv * kStatLevels + k] = t;
  }
}

// Completion level of every 128-source sub-window: the first level whose
// count is N * l (the window holding it completed by its own level, so the
// sub-window did too); level 0's count is l.  -1 or -2 carried over from a
// window that stalled or ran past the kept levels.  Runs only while *gate != 0.
__global__ void sub_levels_kernel(long long* __restrict__ sub_counts, const int* __restrict__ win_levels, int cap,
                                  int N, int nwin, int n_src, int* __restrict__ sub_levels, const int* gate) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nwin) return;
  if (gate && ld_volatile_i32(gate) == 0) return;
  const long long l = max(0, min(128, n_src - s * 128));
  long long* lc = sub_counts + (size_t)s * (cap + 1);
  lc[0] = l;
  const int Lp = win_levels[s / kBaseR];
  int L = Lp;
  if (Lp >= 0) {
    L = -1;
    for (int k = 0; k <= Lp && k <= cap; ++k)
      if (lc[k] == (long long)N * l) { L = k; break; }
  }
  sub_levels[s] = L;
}

// ---- the delta evaluation: one CTA per (candidate, window), window-major ------------
constexpr int kDeltaThreads = 256;
constexpr int kDeltaRows = 512;        // dirty rows a task can hold per level
constexpr int kDeltaHash = 1024;       // hash slots for the dirty rows (power of two)
constexpr int kDeltaLevels = 48;       // levels a task may run past level 0
constexpr int kGrp = 6;                // neighbour rows loaded together

struct DeltaArgs {
  const uint4* levels;                 // base rows: [window of 1024][level_cap + 1][N][8] (sub_row)
  const long long* level_counts;       // [nwin][level_cap + 1] per 128-source sub-window
  const int* win_levels;               // [nwin] per 128-source sub-window
  const int* adj;                      // base adjacency [N][d]
  const Swap* sw;
  const int* sel;                      // candidate c is sw[sel[c]] (sw[c] when null)
  const int* stop;                     // nothing runs while *stop != 0 (may be null)
  long long* dsum;                     // [K][nwin] sum_k delta_k
  int* dlev;                           // [K][nwin] completion level; -1 stalled; -2 not evaluated
  const unsigned* stats;               // base per-vertex statistics [N][kStatLevels]
  long long* ep_sum;                   // [K][4] transmission of endpoint q in the candidate graph
  int* ep_ecc;                         // [K][4] its eccentricity; -1 if some vertex is unreachable
  uint4* dense_pool;                   // dense_slots slots of 2*N rows for tasks whose dirty set overflows
  int* dense_used;                     // slots taken (zeroed before the launch)
  int dense_slots;
  int N, d, nwin, n_src, level_cap, K;
};

// a[i] of four values held in registers (a local array indexed at run time
// would live in local memory)
__device__ __forceinline__ int pick4(int i, int a0, int a1, int a2, int a3) {
  return i == 0 ? a0 : i == 1 ? a1 : i == 2 ? a2 : a3;
}

__device__ __forceinline__ uint4 identity_row(int v, int base, int l) {
  const unsigned b = (unsigned)(v - base);
  uint4 r = make_uint4(0u, 0u, 0u, 0u);
  if (b < (unsigned)l) {
    const unsigned m = 1u << (b & 31);
    const int wd = (int)(b >> 5);
    r.x = wd == 0 ? m : 0u;
    r.y = wd == 1 ? m : 0u;
    r.z = wd == 2 ? m : 0u;
    r.w = wd == 3 ? m : 0u;
  }
  return r;
}

__global__ void __launch_bounds__(kDeltaThreads, 4) delta_kernel(const DeltaArgs a) {
  extern __shared__ unsigned s_claim[];                 // [ceil(N/32)]: rows claimed this level, then
                                                        // [ceil(N/32)]: rows in D_k (s_dbits)
  __shared__ int s_ids[2][kDeltaRows];
  __shared__ uint4 s_val[2][kDeltaRows];
  __shared__ int s_key[kDeltaHash];
  __shared__ int s_slot[kDeltaHash];
  __shared__ int s_n[2];
  __shared__ int s_over;
  __shared__ int s_near;                                // levels 1..s_near are the base's
  __shared__ unsigned long long s_red[kDeltaThreads / 32];
  if (a.stop && ld_volatile_i32(a.stop) != 0) return;
  // window-major: the CTAs resident together share one window's base rows in L2
  const int c = blockIdx.x % a.K, w = blockIdx.x / a.K;
  const Swap sw = a.sw[a.sel ? a.sel[c] : c];
  const int N = a.N, d = a.d;
  const int base = w * 128;
  const int l = min(128, a.n_src - base);
  const int L = a.win_levels[w];
  long long* const out_sum = a.dsum + (size_t)c * a.nwin + w;
  int* const out_lev = a.dlev + (size_t)c * a.nwin + w;
  if (!sw.valid || L < 0) {            // no change, or a base window that cannot serve
    if (threadIdx.x == 0) {
      *out_sum = 0;
      *out_lev = sw.valid ? -2 : L;
    }
    return;
  }
  // A swap endpoint's own distances change for many vertices; its source bit
  // is masked out here and its distances come from endpoint_sweep_kernel.
  // The masked window counts only the other sources: its base counts lose
  // the endpoint's reached vertices, N - stats[x][k] at level k.
  const int X0 = sw.x[0], X1 = sw.x[1], X2 = sw.x[2], X3 = sw.x[3];
  const int P0 = sw.pos[0], P1 = sw.pos[1], P2 = sw.pos[2], P3 = sw.pos[3];
  uint4 fullm = chunk_full_mask(0, l);
  unsigned mq = 0u;                    // endpoints whose source bit lies in the window
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const unsigned b = (unsigned)(sw.x[q] - base);
    if (b < (unsigned)l) {
      const unsigned m = ~(1u << (b & 31));
      if ((b >> 5) == 0) fullm.x &= m; else if ((b >> 5) == 1) fullm.y &= m; else if ((b >> 5) == 2) fullm.z &= m; else fullm.w &= m;
      mq |= 1u << q;
    }
  }
  const int lm = l - __popc(mq);
  const long long full_count = (long long)N * lm;
  auto masked_base_count = [&](int k, long long ck) -> long long {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if ((mq >> q) & 1u)
        ck -= N - (long long)(k < kStatLevels ? __ldg(a.stats + (size_t)sw.x[q] * kStatLevels + k) : 0u);
    return ck;
  };
  if (lm == 0) {                       // every source of the window is an endpoint
    if (threadIdx.x == 0) {
      *out_sum = 0;
      *out_lev = 0;
    }
    return;
  }
  const int cap = a.level_cap;

  const long long* const lc = a.level_counts + (size_t)w * (cap + 1);
  const int nclaim = (N + 31) / 32;
  unsigned* const s_dbits = s_claim + nclaim;
  for (int i = threadIdx.x; i < 2 * nclaim; i += blockDim.x) s_claim[i] = 0u;
  for (int i = threadIdx.x; i < kDeltaHash; i += blockDim.x) s_key[i] = -1;
  if (threadIdx.x == 0) {
    s_n[0] = 0;
    s_n[1] = 0;
    s_over = 0;
    s_near = 0x7fffffff;
  }
  __syncthreads();
  // candidate neighbour j of row x
  auto nb = [&](int x, int j) -> int {
    const int q = x == X0 ? 0 : x == X1 ? 1 : x == X2 ? 2 : x == X3 ? 3 : -1;
    if (q >= 0 && j == pick4(q, P0, P1, P2, P3)) return pick4(q, X2, X3, X0, X1);
    return __ldg(a.adj + (long long)x * d + j);
  };
  auto base_row = [&](int k, int v) -> uint4 {
    if (k > L) return fullm;
    uint4 r = k == 0 ? identity_row(v, base, l) : __ldg(sub_row(a.levels, cap, N, w, k, v));
    r.x &= fullm.x; r.y &= fullm.y; r.z &= fullm.z; r.w &= fullm.w;
    return r;
  };
  // S'_k of row y: its dirty value when y is in D_k (table s_key), else the base
  // slot of row y in D_k's table, or -1 (the bitmap answers most lookups)
  auto dirty_slot = [&](int nd, int y) -> int {
    if (nd > 0 && ((s_dbits[y >> 5] >> (y & 31)) & 1u)) {
      unsigned h = ((unsigned)y * 2654435761u) & (kDeltaHash - 1);
      for (int p = 0; p < kDeltaHash; ++p) {
        const int key = s_key[h];
        if (key == y) return s_slot[h];
        if (key < 0) break;
        h = (h + 1) & (kDeltaHash - 1);
      }
    }
    return -1;
  };
  // this sub-window's rows: level k of vertex v at lev_w + (k * N + v) * 8
  const uint4* const lev_w = sub_row(a.levels, cap, N, w, 0, 0);
  // S'_{k+1}[x] = S'_k[x] | OR_j S'_k[N'(x)_j]: neighbour ids, then their
  // dirty slots (shared memory), then all row loads of a group at once.  The
  // base rows are ORed unmasked and the mask applied once at the end (the
  // dirty rows are masked already).
  auto derive = [&](int k, int nd, int cur, int x) -> uint4 {
    const int qx = x == X0 ? 0 : x == X1 ? 1 : x == X2 ? 2 : x == X3 ? 3 : -1;
    const int px = qx >= 0 ? pick4(qx, P0, P1, P2, P3) : -1;
    const int vx = pick4(qx, X2, X3, X0, X1);
    const int* row = a.adj + (long long)x * d;
    const uint4* const lk = lev_w + (size_t)k * N * 8;
    auto raw_row = [&](int v) -> uint4 {
      return k > L ? fullm : (k == 0 ? identity_row(v, base, l) : __ldg(lk + (size_t)v * 8));
    };
    const int dx = dirty_slot(nd, x);
    uint4 acc = dx >= 0 ? s_val[cur][dx] : raw_row(x);
    for (int j0 = 0; j0 < d; j0 += kGrp) {
      int u[kGrp], ds[kGrp];
      if ((d & 1) == 0) {                // pairs of ids in one 8-byte load (x * d + j is even)
#pragma unroll
        for (int q = 0; q < kGrp; q += 2) {
          const int j = j0 + q;
          if (j < d) {
            const int2 t = __ldg(reinterpret_cast<const int2*>(row + j));
            u[q] = j == px ? vx : t.x;
            u[q + 1] = j + 1 == px ? vx : t.y;
          } else {
            u[q] = -1;
            u[q + 1] = -1;
          }
        }
      } else {
#pragma unroll
        for (int q = 0; q < kGrp; ++q) {
          const int j = j0 + q;
          u[q] = j < d ? (j == px ? vx : __ldg(row + j)) : -1;
        }
      }
#pragma unroll
      for (int q = 0; q < kGrp; ++q) ds[q] = u[q] >= 0 ? dirty_slot(nd, u[q]) : -1;
      uint4 r[kGrp];
#pragma unroll
      for (int q = 0; q < kGrp; ++q)
        r[q] = u[q] < 0 ? make_uint4(0u, 0u, 0u, 0u) : (ds[q] >= 0 ? s_val[cur][ds[q]] : raw_row(u[q]));
#pragma unroll
      for (int q = 0; q < kGrp; ++q) or_into(acc, r[q]);
    }
    acc.x &= fullm.x; acc.y &= fullm.y; acc.z &= fullm.z; acc.w &= fullm.w;
    return acc;
  };
  auto row_k = [&](int k, int nd, int cur, int y) -> uint4 {
    if (nd > 0 && ((s_dbits[y >> 5] >> (y & 31)) & 1u)) {
      unsigned h = ((unsigned)y * 2654435761u) & (kDeltaHash - 1);
      for (int p = 0; p < kDeltaHash; ++p) {
        const int key = s_key[h];
        if (key == y) return s_val[cur][s_slot[h]];
        if (key < 0) break;
        h = (h + 1) & (kDeltaHash - 1);
      }
    }
    return base_row(k, y);
  };
  // Levels the candidate shares with the base.  A path of length <= k from
  // source s that uses a swapped edge reaches an endpoint within k - 1 steps,
  // so S'_k = S_k for every k <= m = min over the window's (unmasked) sources
  // of the distance to the nearest endpoint -- the same in both graphs, and
  // the first level at which some endpoint's base row meets the window.
  for (int i = threadIdx.x; i < 4 * L; i += blockDim.x) {
    const uint4 r = base_row(1 + (i >> 2), pick4(i & 3, X0, X1, X2, X3));
    if (r.x | r.y | r.z | r.w) atomicMin(&s_near, 1 + (i >> 2));
  }
  __syncthreads();
  const int m = s_near <= L ? s_near : 0;
  int cur = 0;
  long long total_delta = 0, prev_count = lm;
  int Lc = -1;
  int status = -2;   // becomes the completion level, or -1 when the candidate stalls
  int k = 0;
  bool dense = false;
  // The levels past k carry the base's counts (delta 0): the decisions of the
  // level loop below on those counts.  Returns true once decided.
  auto base_levels = [&](int k_end) -> bool {
    for (; k < k_end; ++k) {
      const long long count = (k + 1 <= L) ? masked_base_count(k + 1, lc[k + 1]) : full_count;
      if (Lc < 0 && count == full_count) Lc = k + 1;
      if (Lc >= 0 && k + 1 >= L) { status = Lc; return true; }
      if (Lc < 0 && count == prev_count) { status = -1; return true; }
      prev_count = count;
    }
    return false;
  };
  if (base_levels(m)) k = kDeltaLevels;   // decided within the shared levels
  for (; k < kDeltaLevels; ++k) {
    const int nd = s_n[cur];
    if (nd == 0) {
      // S'_k = S_k.  With every endpoint's row full as well, every later
      // level is the base's too: non-endpoints keep their neighbours, and an
      // endpoint's row stays full in both graphs.
      bool all_full = true;
#pragma unroll
      for (int q = 0; q < 4; ++q) all_full = all_full && equal4(base_row(k, sw.x[q]), fullm);
      if (all_full) {
        base_levels(kDeltaLevels);
        break;
      }
    }
    const int nxt = cur ^ 1;
    const int items = 4 + nd * (d + 1);
    unsigned long long pos_cnt = 0, neg_cnt = 0;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
      int x;
      if (it < 4) {
        x = pick4(it, X0, X1, X2, X3);
      } else {
        const int q = (it - 4) / (d + 1), j = (it - 4) % (d + 1);
        const int v = s_ids[cur][q];
        x = j == d ? v : nb(v, j);
      }
      const unsigned bit = 1u << (x & 31);
      if (atomicOr(&s_claim[x >> 5], bit) & bit) continue;
      const uint4 acc = derive(k, nd, cur, x);
      const uint4 bn = base_row(k + 1, x);
      if (!equal4(acc, bn)) {
        const int idx = atomicAdd(&s_n[nxt], 1);
        if (idx < kDeltaRows) {
          s_ids[nxt][idx] = x;
          s_val[nxt][idx] = acc;
        } else {
          s_over = 1;
        }
        const unsigned pa = popc4(acc), pb = popc4(bn);
        if (pa > pb) pos_cnt += pa - pb; else neg_cnt += pb - pa;
      }
    }
    // delta_{k+1} = pos - neg, reduced over the block
    long long dl = (long long)pos_cnt - (long long)neg_cnt;
    for (int o = 16; o > 0; o >>= 1) dl += __shfl_xor_sync(0xffffffffu, dl, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = (unsigned long long)dl;
    __syncthreads();
    // Three barriers a level.  Between the first two, D_k's table is retired
    // and the claims are cleared; between the second and third, D_{k+1} is
    // entered.  The next level's items start after the third.
    if (s_over) { dense = true; break; }   // D_k and its table are still intact
    long long delta = 0;
    for (int i = 0; i < kDeltaThreads / 32; ++i) delta += (long long)s_red[i];
    // clear the claims: the whole bitmap when it is small against the items,
    // else the words the items touched (every claimed row lies in one)
    if (nclaim <= 2 * items) {
      for (int i = threadIdx.x; i < nclaim; i += blockDim.x) s_claim[i] = 0u;
    } else {
      for (int it = threadIdx.x; it < items; it += blockDim.x) {
        int x;
        if (it < 4) {
          x = pick4(it, X0, X1, X2, X3);
        } else {
          const int q = (it - 4) / (d + 1), j = (it - 4) % (d + 1);
          const int v = s_ids[cur][q];
          x = j == d ? v : nb(v, j);
        }
        s_claim[x >> 5] = 0u;
      }
    }
    // the next level's lookup table and bitmap (every set bit is a D_k row,
    // so clearing the words of D_k's rows clears the bitmap)
    for (int i = threadIdx.x; i < kDeltaHash; i += blockDim.x) s_key[i] = -1;
    for (int i = threadIdx.x; i < nd; i += blockDim.x) s_dbits[s_ids[cur][i] >> 5] = 0u;
    __syncthreads();
    const int nn = s_n[nxt];
    for (int i = threadIdx.x; i < nn; i += blockDim.x) {
      const int y = s_ids[nxt][i];
      unsigned h = ((unsigned)y * 2654435761u) & (kDeltaHash - 1);
      while (atomicCAS(&s_key[h], -1, y) != -1) h = (h + 1) & (kDeltaHash - 1);
      s_slot[h] = i;
      atomicOr(&s_dbits[y >> 5], 1u << (y & 31));
    }
    if (threadIdx.x == 0) s_n[cur] = 0;    // D_k's count: read before the first barrier only
    total_delta += delta;
    const long long ck = (k + 1 <= L) ? masked_base_count(k + 1, lc[k + 1]) : full_count;
    const long long count = ck + delta;
    if (Lc < 0 && count == full_count) Lc = k + 1;
    __syncthreads();
    if (Lc >= 0 && k + 1 >= L) { status = Lc; break; }
    if (Lc < 0 && count == prev_count) { status = -1; break; }
    prev_count = count;
    cur = nxt;
  }
  if (dense) {
    // The dirty set outgrew shared memory while deriving level k+1: from
    // S'_k (the base with D_k's rows) the window is swept in full, level by
    // level, in a slot of the pool; counts are exact popcounts.
    __shared__ int s_pool;
    if (threadIdx.x == 0) s_pool = atomicAdd(a.dense_used, 1);
    __syncthreads();
    const int slot = s_pool;
    if (slot < a.dense_slots) {
      uint4* A = a.dense_pool + (size_t)slot * 2 * N;
      uint4* B = A + N;
      const int nd = s_n[cur];
      for (int v = threadIdx.x; v < N; v += blockDim.x) __stcg(A + v, row_k(k, nd, cur, v));
      __syncthreads();
      for (; k < kDeltaLevels; ++k) {
        unsigned long long cnt = 0;
        for (int v = threadIdx.x; v < N; v += blockDim.x) {
          uint4 acc = __ldcg(A + v);
          const int qv = v == X0 ? 0 : v == X1 ? 1 : v == X2 ? 2 : v == X3 ? 3 : -1;
          const int pv = qv >= 0 ? pick4(qv, P0, P1, P2, P3) : -1;
          const int nvv = pick4(qv, X2, X3, X0, X1);
          const int* row = a.adj + (long long)v * d;
          for (int j0 = 0; j0 < d; j0 += kGrp) {
            int u[kGrp];
#pragma unroll
            for (int q = 0; q < kGrp; ++q) {
              const int j = j0 + q;
              u[q] = j < d ? (j == pv ? nvv : __ldg(row + j)) : -1;
            }
            uint4 r[kGrp];
#pragma unroll
            for (int q = 0; q < kGrp; ++q) r[q] = u[q] >= 0 ? __ldcg(A + u[q]) : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
            for (int q = 0; q < kGrp; ++q) or_into(acc, r[q]);
          }
          __stcg(B + v, acc);
          cnt += popc4(acc);
        }
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        __syncthreads();
        if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = cnt;
        __syncthreads();
        long long count = 0;
        for (int i = 0; i < kDeltaThreads / 32; ++i) count += (long long)s_red[i];
        const long long ck = (k + 1 <= L) ? masked_base_count(k + 1, lc[k + 1]) : full_count;
        total_delta += count - ck;
        if (Lc < 0 && count == full_count) Lc = k + 1;
        if (Lc >= 0 && k + 1 >= L) { status = Lc; break; }
        if (Lc < 0 && count == prev_count) { status = -1; break; }
        prev_count = count;
        uint4* t = A;
        A = B;
        B = t;
        __syncthreads();
      }
    }
  }
  if (threadIdx.x == 0) {
    *out_sum = total_delta;
    *out_lev = status;
  }
}

// ---- the endpoints' own distances: one bit-parallel search ------------------------
// The distances from every endpoint x_q of every candidate c, each in its
// own candidate graph, as one bit-parallel breadth-first search: source bit
// i = 4c + q (one 32-bit word per lane, nw <= 32 words per vertex row), the
// recurrence S_{k+1}[v] = S_k[v] | OR_{u in N(v)} S_k[u] of the evaluator
// over the base adjacency, and then, for every row x_q(c) a candidate
// patched, candidate c's four bits re-derived with its swapped neighbour
// list (only those rows differ in c's graph).  Per source bit the sum of the
// levels at which vertices are first reached is its transmission, the last
// level that reaches a vertex its eccentricity.  Cooperative launch, one
// 512-thread CTA per SM, levels separated by the bounded grid barrier.
struct EndpointArgs {
  const int* adj;                      // base adjacency [N][d], d <= 32
  const Swap* sw;
  const int* sel;
  const int* stop;
  ApspCtrl* ctrl;                      // grid barrier, zeroed before the launch
  unsigned* rows;                      // 2 * N * nw words
  int* head;                           // [N] first fix-up of a row (-1: none)
  int* next;                           // [4K] next fix-up of the same row
  unsigned* changed;                   // [kDeltaLevels]: any bit set at that level
  unsigned* newbits;                   // [kDeltaLevels][nw]: sources that reached a vertex at that level
  unsigned* tsum;                      // [nw * 32] per source: sum of distances
  unsigned* unreach;                   // [nw] sources with an unreachable vertex
  long long* ep_sum;                   // [K][4] outputs
  int* ep_ecc;                         // [K][4]: -1 unreachable vertex, -2 did not converge
  long long timeout_ns;
  int N, d, K, nw;
};

__global__ void __launch_bounds__(kThreads, 1) endpoint_sweep_kernel(const EndpointArgs e) {
  __shared__ int s_flag;
  __shared__ unsigned s_t[32 * 32];
  if (e.stop && ld_volatile_i32(e.stop) != 0) return;   // written before the launch: the same in every CTA
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  const int gw = blockIdx.x * kWarps + warp, nwarps = gridDim.x * kWarps;
  const int N = e.N, d = e.d, nw = e.nw, nsrc = 4 * e.K;
  unsigned* A = e.rows;
  unsigned* B = e.rows + (size_t)N * nw;
  // phase 0: clear
  for (long long i = tid; i < (long long)N * nw; i += nthreads) A[i] = 0u;
  for (long long i = tid; i < N; i += nthreads) e.head[i] = -1;
  for (long long i = tid; i < (long long)kDeltaLevels * nw; i += nthreads) e.newbits[i] = 0u;
  for (long long i = tid; i < kDeltaLevels; i += nthreads) e.changed[i] = 0u;
  for (long long i = tid; i < 32 * nw; i += nthreads) e.tsum[i] = 0u;
  for (long long i = tid; i < nw; i += nthreads) e.unreach[i] = 0u;
  for (int i = threadIdx.x; i < 32 * 32; i += blockDim.x) s_t[i] = 0u;
  unsigned long long bar = gridDim.x;
  if (!grid_barrier(e.ctrl, bar, e.timeout_ns, &s_flag)) return;
  // phase 1: identity bits and the fix-up lists of the patched rows
  for (long long i = tid; i < nsrc; i += nthreads) {
    const int c = (int)i >> 2, q = (int)i & 3;
    const Swap w = e.sw[e.sel ? e.sel[c] : c];
    if (!w.valid) continue;
    const int v = w.x[q];
    atomicOr(A + (size_t)v * nw + (i >> 5), 1u << (i & 31));
    e.next[i] = atomicExch(e.head + v, (int)i);
  }
  bar += gridDim.x;
  if (!grid_barrier(e.ctrl, bar, e.timeout_ns, &s_flag)) return;
  unsigned T[32];
#pragma unroll
  for (int b = 0; b < 32; ++b) T[b] = 0u;
  int L = 0;
  bool converged = false;
  for (; L < kDeltaLevels; ++L) {
    unsigned ornew = 0u;
    for (int v = gw; v < N; v += nwarps) {
      const int nb = lane < d ? __ldg(e.adj + (long long)v * d + lane) : 0;
      const unsigned own = lane < nw ? __ldcg(A + (size_t)v * nw + lane) : 0u;
      unsigned acc = own;
      for (int j0 = 0; j0 < d; j0 += 8) {   // eight neighbour words in flight a lane
        unsigned x[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int j = j0 + q;
          const int u = __shfl_sync(0xffffffffu, nb, j & 31);
          x[q] = (j < d && lane < nw) ? __ldcg(A + (size_t)u * nw + lane) : 0u;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) acc |= x[q];
      }
      for (int f = __ldcg(e.head + v); f >= 0; f = __ldcg(e.next + f)) {   // the same list in every lane
        const int c = f >> 2, q = f & 3;
        const Swap w = e.sw[e.sel ? e.sel[c] : c];
        const int wc = (4 * c) >> 5;
        const unsigned m = 0xFu << ((4 * c) & 31);
        const int nv = q == 0 ? w.x[2] : q == 1 ? w.x[3] : q == 2 ? w.x[0] : w.x[1];
        unsigned accc = own;
        for (int j = 0; j < d; ++j) {
          int u = __shfl_sync(0xffffffffu, nb, j);
          if (j == w.pos[q]) u = nv;
          if (lane == wc) accc |= __ldcg(A + (size_t)u * nw + wc);
        }
        if (lane == wc) acc = (acc & ~m) | (accc & m);
      }
      if (lane < nw) {
        const unsigned nb_new = acc & ~own;
        __stcg(B + (size_t)v * nw + lane, acc);
        ornew |= nb_new;
#pragma unroll
        for (int b = 0; b < 32; ++b) T[b] += ((nb_new >> b) & 1u) ? (unsigned)(L + 1) : 0u;
      }
    }
    if (lane < nw && ornew) {
      atomicOr(e.newbits + (size_t)L * nw + lane, ornew);
      atomicOr(e.changed + L, 1u);
    }
    bar += gridDim.x;
    if (!grid_barrier(e.ctrl, bar, e.timeout_ns, &s_flag)) return;
    if (ld_volatile_i32(reinterpret_cast<const int*>(e.changed + L)) == 0) { converged = true; break; }
    unsigned* t = A;
    A = B;
    B = t;
  }
  // A holds the final rows: sources with a vertex never reached, and the sums
  if (lane < nw) {
    unsigned un = 0u;
    for (int v = gw; v < N; v += nwarps) un |= ~__ldcg(A + (size_t)v * nw + lane);
    if (un) atomicOr(e.unreach + lane, un);
#pragma unroll
    for (int b = 0; b < 32; ++b)
      if (T[b]) atomicAdd(s_t + lane * 32 + b, T[b]);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 32 * nw; i += blockDim.x)
    if (s_t[i]) atomicAdd(e.tsum + i, s_t[i]);
  bar += gridDim.x;
  if (!grid_barrier(e.ctrl, bar, e.timeout_ns, &s_flag)) return;
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < nsrc; i += blockDim.x) {
      int ecc = 0;
      for (int k = 0; k < L; ++k)
        if ((__ldcg(e.newbits + (size_t)k * nw + (i >> 5)) >> (i & 31)) & 1u) ecc = k + 1;
      const bool un = (__ldcg(e.unreach + (i >> 5)) >> (i & 31)) & 1u;
      e.ep_sum[i] = (long long)__ldcg(e.tsum + i);
      e.ep_ecc[i] = !converged ? -2 : (un ? -1 : ecc);
    }
  }
}

// Per candidate: the base's result changed by its windows' deltas and its
// endpoints' searches, as the record a batch evaluation writes (done = 0
// when a window was not evaluated).  With T the base transmission of an
// endpoint (the sum of its statistics) and T' the searched one:
//   sum' = sum - sum_{w,k} delta_{w,k} + sum_q (T'_q - T_q),
//   diameter' = max(completion levels, endpoint eccentricities).
// One warp per candidate.
__global__ void delta_reduce_kernel(const DeltaArgs a, const BaseResult* __restrict__ base, BatchOut* __restrict__ out) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= a.K) return;
  if (a.stop && ld_volatile_i32(a.stop) != 0) return;
  long long s = 0;
  int mx = 0, stalled = 0, missing = 0;
  const Swap sw = a.sw[a.sel ? a.sel[c] : c];
  if (sw.valid && lane < 4) {
    const unsigned* st = a.stats + (size_t)sw.x[lane] * kStatLevels;
    long long t = 0;
    for (int k = 0; k < kStatLevels; ++k) t += st[k];
    const int e = a.ep_ecc[c * 4 + lane];
    s += t - a.ep_sum[c * 4 + lane];   // r.sum = base sum - s: adds T'_q - T_q
    if (e == -1) stalled = 1;
    else if (e < 0) missing = 1;
    else mx = max(mx, e);
    // The statistics keep kStatLevels levels: an endpoint that reaches past
    // them in the base has neither its transmission nor (in the windows that
    // mask it) its reached counts there.  Such a candidate is not served.
    if (st[kStatLevels - 1] != 0u) missing = 1;
  }
  for (int w = lane; w < a.nwin; w += 32) {
    s += a.dsum[(size_t)c * a.nwin + w];
    const int lv = a.dlev[(size_t)c * a.nwin + w];
    if (lv == -1) stalled = 1;
    else if (lv < 0) missing = 1;
    else mx = max(mx, lv);
  }
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    stalled |= __shfl_xor_sync(0xffffffffu, stalled, o);
    missing |= __shfl_xor_sync(0xffffffffu, missing, o);
  }
  if (lane == 0) {
    BatchOut r;
    r.sum = base->sum - s;
    r.levels = 0;
    r.dense_levels = 0;
    r.diam = stalled ? a.N + 1 : mx;
    r.disconnected = stalled;
    r.windows = a.nwin;
    r.done = (missing || base->disconnected) ? 0 : 1;
    out[c] = r;
  }
}

}  // namespace ggb
