// sa_device.cu -- simulated annealing with the whole step on the device.
//
// The reference's annealing (general/sa.c:413-520) is a host loop: draw one
// 2-opt swap (exchange_edge_2opt, :217-369), evaluate the graph, accept or
// reject (accept, :371-411), cool.  Here a step is one replay of a CUDA graph
// and never returns to the host:
//
//   gen        K (or G) candidate swaps of the current graph, each checked in
//              O(degree) against the current adjacency (no self-loop, no
//              repeated edge -- the reference's simple-graph rule);
//   [learned]  features of every candidate from the last exact profile of the
//              current graph, the MLP's predicted change of the distance
//              total, and the K best predictions (plus a few random ones) kept;
//   materialize  the K candidate adjacencies (the current one with 4 entries
//              changed) into the slots of a batch;
//   evaluate   all K exactly in one batch launch;
//   compose    the strictly improving candidates with disjoint endpoints,
//              best first, applied together to one more graph, which is
//              evaluated exactly too;
//   decide     the better of the best single candidate and the composite,
//              accepted by the reference's rule (smaller diameter; equal
//              diameter and ASPL not worse; else exp(diff/temp) > uniform);
//              the swaps are applied to the current graph in place;
//   [learned]  the K exact changes train the MLP (one Adam step), and an
//              accepted move re-profiles the current graph for the features.
//
// Plain annealing is K = 1 without composition: the reference's step, on the
// device.  Every acceptance is decided on exact values.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/graphgolf_b200.h"
#include "apsp_delta.cuh"
#include "batch_internal.h"
#include "core_internal.h"
#include "mlp_internal.h"

using ggb::core_fail;

#define SCUDA(call)                                                                                  \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return core_fail(GGB_ECUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                       __LINE__);                                                                    \
  } while (0)

namespace ggb {
namespace sa {

using bf16 = __nv_bfloat16;

using ggb::Swap;

struct State {
  int N, d, lines, K;
  int* edges;            // [lines][2], current graph
  int* adj;              // [N][d], current graph
  int* best_edges;       // [lines][2]
  long long cur_total, best_total, prev_total;
  int cur_diam, best_diam;
  double temp, cooling;
  int hill;              // 1: accept only when not worse (the reference's -H)
  int done;              // target reached: every kernel of a step returns at once
  int accepted;          // the last step moved the current graph
  int n_comp;            // swaps in this step's composite
  int best_k;            // rank-0 candidate of this step
  int pad_;
  long long step, accepts, multi_accepts, moved_swaps, evals, best_step, pred_accepts, unevaluated;
  int n_pred;            // swaps in this step's predicted list (learned mode)
  int pad2_;
  long long target_total;
  int target_diam;
  int stop_on_target;
  unsigned long long seed;
  float label_scale, label_clip;
  // Symmetry groups: the graph is invariant under v -> v + B (mod N), B = N / groups,
  // and line k*BL + i is line i shifted by k*B (BL = lines / groups), the
  // reference's symmetric line order (general/main.c:175-183).  groups = 1: none.
  int groups, B, BL;
  // Grid graphs: vertex v = x*grid_height + y on the lattice; every new edge
  // must stay within Manhattan length grid_length (0: no length limit).
  int grid_height, grid_length;
  int move_error;        // a move's old neighbour was not found where the state says (never expected)
};

constexpr unsigned long long kGolden = 0x9e3779b97f4a7c15ULL;

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

// A counter-based stream: one 64-bit draw per (seed, a, b, c).
__device__ __forceinline__ unsigned long long draw(unsigned long long seed, unsigned long long a, unsigned long long b,
                                                   unsigned long long c) {
  return mix64(seed + kGolden * (mix64(a + kGolden) ^ mix64(b * 0xd1b54a32d192ed03ULL + c + 1)));
}

__device__ __forceinline__ int below(unsigned long long h, int n) {
  return (int)(((h >> 32) * (unsigned long long)(unsigned)n) >> 32);
}

__device__ __forceinline__ int find_in_row(const int* row, int d, int x) {
  for (int j = 0; j < d; ++j)
    if (row[j] == x) return j;
  return -1;
}

// ---- gen: candidate swaps ------------------------------------------------------
__device__ __forceinline__ int manhattan(int v, int w, int H) {
  const int dx = v / H - w / H, dy = v % H - w % H;
  return (dx < 0 ? -dx : dx) + (dy < 0 ? -dy : dy);
}

// v shifted by k copies: v + k*B (mod N), 0 <= v < N, -groups < k < 2*groups.
__device__ __forceinline__ int shift_copy(const State* s, int v, int k) {
  long long y = (long long)v + (long long)k * s->B;
  y %= s->N;
  if (y < 0) y += s->N;
  return (int)y;
}

// An orbit move of a graph with symmetry groups (general/sa.c:217-369 and
// general/common.c:162-276, restated for the device): two random lines; when
// they lie in the same orbit (their indices agree modulo BL) the orbit's edges
// {x0 + kB, x1 + kB} are re-paired as {x0 + kB, x1 + (k + p)B} for a random
// shift p in [1, groups) (1g-opt), otherwise the two lines and all their copies
// are swapped alike (2g-opt).  The endpoints' classes (v mod B) must be
// pairwise distinct, so that every changed row changes once and no orbit
// repeats or loses an edge; a new edge must not exist yet.  Both keep the
// graph simple, regular and symmetric.
__device__ bool gen_orbit_move(const State* s, unsigned long long h, Swap& w) {
  const int lines = s->lines, d = s->d, B = s->B;
  const int* __restrict__ E = s->edges;
  const int* __restrict__ A = s->adj;
  const int i = below(h, lines), j = below(h << 32, lines);
  if (i == j) return false;
  const int a = E[2 * i], b = E[2 * i + 1];
  if (a % B == b % B) return false;
  if ((i - j) % s->BL == 0) {
    const int p = 1 + below(mix64(h ^ 0x6a09e667f3bcc909ULL), s->groups - 1);
    const int bp = shift_copy(s, b, p);
    if (find_in_row(A + (long long)a * d, d, bp) >= 0) return false;
    w.kind = 1;
    w.line[0] = i; w.line[1] = i;
    w.x[0] = a; w.x[1] = b; w.x[2] = p; w.x[3] = -1;
    return true;
  }
  const int r = (int)(mix64(h) & 1);
  const int c = E[2 * j], e = E[2 * j + 1];
  const int x0 = a, x1 = b, x2 = r ? e : c, x3 = r ? c : e;
  const int c0 = x0 % B, c1 = x1 % B, c2 = x2 % B, c3 = x3 % B;
  if (c0 == c2 || c0 == c3 || c1 == c2 || c1 == c3 || c2 == c3) return false;
  if (find_in_row(A + (long long)x0 * d, d, x2) >= 0 || find_in_row(A + (long long)x1 * d, d, x3) >= 0)
    return false;
  w.kind = 0;
  w.line[0] = i; w.line[1] = j;
  w.x[0] = x0; w.x[1] = x1; w.x[2] = x2; w.x[3] = x3;
  return true;
}

__global__ void gen_kernel(const State* __restrict__ s, Swap* __restrict__ out, int G) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G) return;
  Swap w;
  w.valid = 0;
  w.kind = 0;
  if (!s->done) {
    const int lines = s->lines, d = s->d;
    const int* __restrict__ E = s->edges;
    const int* __restrict__ A = s->adj;
    const unsigned long long seed = s->seed, step = (unsigned long long)s->step;
    // a length limit rejects most random pairs of lines (both new edges must be
    // short): draw more of them; the length test comes before any row scan
    const int attempts = s->grid_length > 0 ? 1024 : 64;
    for (int attempt = 0; attempt < attempts && !w.valid; ++attempt) {
      const unsigned long long h = draw(seed, step, (unsigned long long)k, (unsigned long long)attempt);
      if (s->groups > 1) {
        if (gen_orbit_move(s, h, w)) w.valid = 1;
        continue;
      }
      const int i = below(h, lines), j = below(h << 32, lines);
      if (i == j) continue;
      const int r = (int)(mix64(h) & 1);
      const int a = E[2 * i], b = E[2 * i + 1], c = E[2 * j], e = E[2 * j + 1];
      const int x0 = a, x1 = b, x2 = r ? e : c, x3 = r ? c : e;
      if (x0 == x2 || x1 == x3) continue;
      // grid graphs: both new edges within the length limit (grid/sa.c:196-201)
      if (s->grid_length > 0 && (manhattan(x0, x2, s->grid_height) > s->grid_length ||
                                 manhattan(x1, x3, s->grid_height) > s->grid_length))
        continue;
      const int* r0 = A + (long long)x0 * d;
      const int* r1 = A + (long long)x1 * d;
      if (find_in_row(r0, d, x2) >= 0 || find_in_row(r1, d, x3) >= 0) continue;
      const int p0 = find_in_row(r0, d, x1), p1 = find_in_row(r1, d, x0);
      const int p2 = find_in_row(A + (long long)x2 * d, d, x3), p3 = find_in_row(A + (long long)x3 * d, d, x2);
      if (p0 < 0 || p1 < 0 || p2 < 0 || p3 < 0) continue;
      w.line[0] = i;
      w.line[1] = j;
      w.x[0] = x0; w.x[1] = x1; w.x[2] = x2; w.x[3] = x3;
      w.pos[0] = p0; w.pos[1] = p1; w.pos[2] = p2; w.pos[3] = p3;
      w.valid = 1;
    }
  }
  out[k] = w;
}

// ---- materialize: candidate adjacencies into the batch slots ---------------------
// Slot k (blockIdx.y) = the current adjacency with candidate sel[k]'s four
// entries changed (the current adjacency itself for an invalid candidate).
__global__ void materialize_kernel(const State* __restrict__ s, const Swap* __restrict__ sw,
                                   const int* __restrict__ sel, int* __restrict__ slots, long long slot_stride) {
  if (s->done) return;
  const int k = blockIdx.y;
  const Swap w = sw[sel ? sel[k] : k];
  const int d = s->d;
  const long long n = (long long)s->N * d;
  long long off[4] = {-1, -1, -1, -1};
  int val[4] = {0, 0, 0, 0};
  if (w.valid && s->groups == 1) {   // orbit moves are patched by patch_orbit_kernel
    const int nv[4] = {w.x[2], w.x[3], w.x[0], w.x[1]};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      off[q] = (long long)w.x[q] * d + w.pos[q];
      val[q] = nv[q];
    }
  }
  const int* __restrict__ src = s->adj;
  int* __restrict__ dst = slots + (long long)k * slot_stride;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int v = src[i];
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if (i == off[q]) v = val[q];
    dst[i] = v;
  }
}

__device__ __forceinline__ void apply_swap(int* adj, int d, const Swap& w) {
  adj[(long long)w.x[0] * d + w.pos[0]] = w.x[2];
  adj[(long long)w.x[1] * d + w.pos[1]] = w.x[3];
  adj[(long long)w.x[2] * d + w.pos[2]] = w.x[0];
  adj[(long long)w.x[3] * d + w.pos[3]] = w.x[1];
}

// In row v, the entry equal to `from` becomes `to`; false if there is none.
__device__ __forceinline__ bool replace_in_row(int* adj, int d, int v, int from, int to) {
  int* row = adj + (long long)v * d;
  const int j = find_in_row(row, d, from);
  if (j < 0) return false;
  row[j] = to;
  return true;
}

// Applies one move to `adj` and, when given, to the edge list in the
// symmetric line order.  Copy k of an orbit move changes the rows of the
// endpoints shifted by k*B; their classes are distinct (gen_orbit_move), so
// every changed row changes once and the copies can be found by value.
// Returns false if an old neighbour was missing (a state inconsistency).
__device__ bool apply_move(const State* s, int* adj, int* edges, const Swap& w) {
  const int d = s->d;
  if (s->groups == 1) {
    apply_swap(adj, d, w);
    if (edges) {
      edges[2 * w.line[0]] = w.x[0];
      edges[2 * w.line[0] + 1] = w.x[2];
      edges[2 * w.line[1]] = w.x[1];
      edges[2 * w.line[1] + 1] = w.x[3];
    }
    return true;
  }
  bool ok = true;
  for (int k = 0; k < s->groups; ++k) {
    if (w.kind == 1) {
      const int p = w.x[2];
      const int va = shift_copy(s, w.x[0], k), vb = shift_copy(s, w.x[1], k);
      const int nb = shift_copy(s, w.x[1], k + p), na = shift_copy(s, w.x[0], k - p);
      ok &= replace_in_row(adj, d, va, vb, nb);
      ok &= replace_in_row(adj, d, vb, va, na);
      if (edges) {
        const int l = (int)(((long long)w.line[0] + (long long)k * s->BL) % s->lines);
        edges[2 * l] = va;
        edges[2 * l + 1] = nb;
      }
    } else {
      const int v0 = shift_copy(s, w.x[0], k), v1 = shift_copy(s, w.x[1], k);
      const int v2 = shift_copy(s, w.x[2], k), v3 = shift_copy(s, w.x[3], k);
      ok &= replace_in_row(adj, d, v0, v1, v2);
      ok &= replace_in_row(adj, d, v1, v0, v3);
      ok &= replace_in_row(adj, d, v2, v3, v0);
      ok &= replace_in_row(adj, d, v3, v2, v1);
      if (edges) {
        const int l0 = (int)(((long long)w.line[0] + (long long)k * s->BL) % s->lines);
        const int l1 = (int)(((long long)w.line[1] + (long long)k * s->BL) % s->lines);
        edges[2 * l0] = v0;
        edges[2 * l0 + 1] = v2;
        edges[2 * l1] = v1;
        edges[2 * l1 + 1] = v3;
      }
    }
  }
  return ok;
}

// The vertex classes (v mod B; the vertices themselves without symmetry) a
// move touches: moves with disjoint classes change disjoint rows and can be
// applied together.  Returns how many of out[0..4) it wrote.
__device__ __forceinline__ int move_classes(const State* s, const Swap& w, int* out) {
  if (s->groups > 1 && w.kind == 1) {
    out[0] = w.x[0] % s->B;
    out[1] = w.x[1] % s->B;
    return 2;
  }
  for (int q = 0; q < 4; ++q) out[q] = s->groups > 1 ? w.x[q] % s->B : w.x[q];
  return 4;
}

__device__ __forceinline__ bool classes_free(const unsigned* vmark, const int* c, int n) {
  bool f = true;
  for (int q = 0; q < n; ++q) f &= !((vmark[c[q] >> 5] >> (c[q] & 31)) & 1u);
  return f;
}

__device__ __forceinline__ void classes_set(unsigned* vmark, const int* c, int n, bool on) {
  for (int q = 0; q < n; ++q) {
    if (on) vmark[c[q] >> 5] |= 1u << (c[q] & 31);
    else vmark[c[q] >> 5] = 0u;
  }
}

// Orbit moves of the candidates: slot k (block k) = the current adjacency,
// copied by materialize_kernel, with candidate sel[k]'s move applied.
__global__ void patch_orbit_kernel(State* __restrict__ s, const Swap* __restrict__ sw, const int* __restrict__ sel,
                                   int* __restrict__ slots, long long slot_stride) {
  if (s->done || s->groups == 1 || threadIdx.x != 0) return;
  const int k = blockIdx.x;
  const Swap w = sw[sel ? sel[k] : k];
  if (w.valid && !apply_move(s, slots + (long long)k * slot_stride, nullptr, w)) atomicExch(&s->move_error, 1);
}

struct Key {
  int diam;           // INT_MAX when disconnected or not evaluated
  long long total;
};

__device__ __forceinline__ Key key_of(const BatchOut& o, int N) {
  Key k;
  if (o.done && !o.disconnected && o.diam < N) {
    k.diam = o.diam;
    k.total = o.sum + (long long)N * (N - 1);
  } else {
    k.diam = INT_MAX;
    k.total = LLONG_MAX;
  }
  return k;
}

// Key of candidate k: a candidate whose draw found no valid move (its slot
// holds the unchanged graph) never competes.
__device__ __forceinline__ Key cand_key(const Swap* sw, const int* sel, const BatchOut* out, int k, int N) {
  if (!sw[sel ? sel[k] : k].valid) {
    Key no;
    no.diam = INT_MAX;
    no.total = LLONG_MAX;
    return no;
  }
  return key_of(out[k], N);
}

__device__ __forceinline__ bool key_less(const Key& a, const Key& b) {
  return a.diam < b.diam || (a.diam == b.diam && a.total < b.total);
}

// ---- compose: rank the candidates, build the composite -----------------------------
// One block of kComposeThreads threads, K <= kComposeThreads.
constexpr int kComposeThreads = 256;
__global__ void __launch_bounds__(kComposeThreads) compose_kernel(State* __restrict__ s, const Swap* __restrict__ sw,
                                                                  const int* __restrict__ sel,
                                                                  const BatchOut* __restrict__ out, int K,
                                                                  Swap* __restrict__ comp, int compose_max,
                                                                  unsigned* __restrict__ vmark) {
  __shared__ int s_order[kComposeThreads];
  __shared__ Key s_keys[kComposeThreads];
  if (s->done) return;
  const int N = s->N;
  const int k = threadIdx.x;
  if (k < K) s_keys[k] = cand_key(sw, sel, out, k, N);
  __syncthreads();
  if (k < K) {
    const Key me = s_keys[k];
    int rank = 0;
    for (int j = 0; j < K; ++j) {
      const Key o = s_keys[j];
      rank += key_less(o, me) || (!key_less(me, o) && j < k);
    }
    s_order[rank] = k;
  }
  __syncthreads();
  if (k != 0) return;
  s->prev_total = s->cur_total;
  s->best_k = s_order[0];
  const Key cur = {s->cur_diam, s->cur_total};
  int m = 0;
  for (int r = 0; r < K && m < compose_max; ++r) {
    const int c = s_order[r];
    const Key kc = s_keys[c];
    if (!key_less(kc, cur)) break;   // sorted: nothing further improves
    const Swap w = sw[sel ? sel[c] : c];
    if (!w.valid) continue;
    int cl[4];
    const int nc = move_classes(s, w, cl);
    if (!classes_free(vmark, cl, nc)) continue;
    classes_set(vmark, cl, nc, true);
    comp[m++] = w;
  }
  for (int i = 0; i < m; ++i) {
    int cl[4];
    const int nc = move_classes(s, comp[i], cl);
    classes_set(vmark, cl, nc, false);
  }
  s->n_comp = m;
}

// Size of predicted composite c: the first n_pred >> c swaps of the list.
__device__ __forceinline__ int pred_size(int n_pred, int c) { return n_pred >> c; }



// ---- decide ---------------------------------------------------------------------------
// general/sa.c:371-411 on exact totals: the reference's
// diff = (current_ASPL - new_ASPL) * N(N-1) / groups is the change of the
// (group-weighted) distance total divided by groups.  Threads k < K also
// write the training labels of this step.
// comp_out (when there is a composite batch): [0] the exact composite,
// [1 + c] predicted composite c.
__global__ void decide_kernel(State* __restrict__ s, const Swap* __restrict__ sw, const int* __restrict__ sel,
                              const BatchOut* __restrict__ out, int K, const Swap* __restrict__ comp,
                              const BatchOut* __restrict__ comp_out, float* __restrict__ labels,
                              const Swap* __restrict__ pred, int C) {
  if (s->done) return;
  const int N = s->N;
  const int k = threadIdx.x;
  if (k < K && !out[k].done) atomicAdd(reinterpret_cast<unsigned long long*>(&s->unevaluated), 1ULL);
  if (labels && k < K) {
    const Key kk = key_of(out[k], N);
    float lab = out[k].done ? s->label_clip : 0.f;   // a candidate the delta path could not serve teaches nothing
    if (kk.diam != INT_MAX) {
      lab = (float)((double)(kk.total - s->prev_total) * (double)s->label_scale);
      lab = fminf(fmaxf(lab, -s->label_clip), s->label_clip);
    }
    labels[k] = lab;
  }
  if (k != 0) return;
  const Key cur = {s->cur_diam, s->cur_total};
  const int bk = s->best_k;
  Key cand = cand_key(sw, sel, out, bk, N);
  bool use_comp = false;
  int use_pred = 0;   // swaps of the chosen predicted composite (0: none)
  if (comp_out && s->n_comp >= 2) {
    const Key kc = key_of(comp_out[0], N);
    if (key_less(kc, cand)) {
      cand = kc;
      use_comp = true;
    }
  }
  for (int c = 0; c < C && comp_out; ++c) {
    const int m = pred_size(s->n_pred, c);
    if (m < 1) break;
    const Key kp = key_of(comp_out[1 + c], N);
    if (key_less(kp, cand)) {
      cand = kp;
      use_comp = false;
      use_pred = m;
    }
  }
  bool acc = false;
  if (cand.diam != INT_MAX) {
    if (cand.diam < cur.diam) {
      acc = true;
    } else if (cand.diam == cur.diam) {
      if (cand.total <= cur.total) {
        acc = true;
      } else if (!s->hill) {
        const double diff = (double)(cur.total - cand.total) / (double)s->groups;
        const unsigned long long h = draw(s->seed ^ 0x5bd1e995ULL, (unsigned long long)s->step, 0x0dec1deULL, 7);
        const double u = ((double)(h >> 11) + 1.0) / (9007199254740992.0 + 2.0);
        acc = exp(diff / s->temp) > u;
      }
    }
  }
  s->evals += K + C + (comp_out ? 1 : 0);
  if (acc) {
    bool ok = true;
    if (use_pred) {
      for (int i = 0; i < use_pred; ++i) ok &= apply_move(s, s->adj, s->edges, pred[i]);
      s->multi_accepts += 1;
      s->pred_accepts += 1;
      s->moved_swaps += use_pred;
    } else if (use_comp) {
      for (int i = 0; i < s->n_comp; ++i) ok &= apply_move(s, s->adj, s->edges, comp[i]);
      s->multi_accepts += 1;
      s->moved_swaps += s->n_comp;
    } else {
      ok &= apply_move(s, s->adj, s->edges, sw[sel ? sel[bk] : bk]);
      s->moved_swaps += 1;
    }
    if (!ok) s->move_error = 1;
    s->accepts += 1;
    s->cur_diam = cand.diam;
    s->cur_total = cand.total;
    if (cand.diam < s->best_diam || (cand.diam == s->best_diam && cand.total < s->best_total)) {
      s->best_diam = cand.diam;
      s->best_total = cand.total;
      s->best_step = s->step;
    }
  }
  s->accepted = acc ? 1 : 0;
  if (s->stop_on_target && s->cur_diam <= s->target_diam && s->cur_total <= s->target_total) s->done = 1;
  s->temp *= s->cooling;
  s->step += 1;
}

// Copies the current edges to the best edges when this step set a new best.
__global__ void best_copy_kernel(const State* __restrict__ s) {
  if (s->best_step != s->step - 1) return;
  const long long n = 2LL * s->lines;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    s->best_edges[i] = s->edges[i];
}

// ---- learned mode: features and selection ---------------------------------------------
constexpr int kMaxFeatDegree = 32;

// Exact distance d(x, y) read from the base: the first level k whose row x
// (in the window holding source y) has y's bit, i.e. y in S_k[x].  Window
// completion bounds the search; a stalled window gives level_cap + 1.
__device__ int base_distance(const uint4* __restrict__ levels, const int* __restrict__ win_levels, int cap, int N,
                             int x, int y) {
  if (x == y) return 0;
  const int w = y >> 7, b = y & 127;
  const int L = win_levels[w];
  const int top = L > 0 ? L : cap;
  for (int k = 1; k <= top; ++k) {
    const uint4 r = __ldg(ggb::sub_row(levels, cap, N, w, k, x));
    const unsigned wd = b < 64 ? (b < 32 ? r.x : r.y) : (b < 96 ? r.z : r.w);
    if ((wd >> (b & 31)) & 1u) return k;
  }
  return cap + 1;
}

__device__ int common_neighbours(const int* __restrict__ A, int d, int x, int y) {
  const int* rx = A + (long long)x * d;
  const int* ry = A + (long long)y * d;
  int c = 0;
  for (int i = 0; i < d; ++i) {
    const int u = rx[i];
    for (int j = 0; j < d; ++j) c += (ry[j] == u);
  }
  return c;
}

// 32 features per candidate, from the current graph's profile (stats) and
// adjacency: per endpoint (6 each) eccentricity / 8, mean distance / 8 and
// log-scaled counts of vertices at distance 2..5; the exact distances (read
// from the base's level rows) of the pairs the swap joins and of the two
// cross pairs, / 8;
// the common-neighbour counts of the pairs it separates; and the
// transmission gaps of the joined pairs.
__global__ void features_kernel(const State* __restrict__ s, const Swap* __restrict__ sw, int G,
                                const unsigned* __restrict__ stats, const uint4* __restrict__ levels,
                                const int* __restrict__ win_levels, int cap, bf16* __restrict__ X) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= G) return;
  float f[mlp::kFeatures];
#pragma unroll
  for (int i = 0; i < mlp::kFeatures; ++i) f[i] = 0.f;
  const Swap w = sw[k];
  if (!s->done && w.valid) {
    const int N = s->N, d = s->d;
    const float inv_logn = 1.f / logf(1.f + (float)N);
    float T[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const unsigned* st = stats + (long long)w.x[e] * kStatLevels;
      int ecc = kStatLevels - 1;
      double tr = 0.0;
      for (int q = 0; q < kStatLevels; ++q) {
        tr += st[q];
        if (st[q] == 0u && q < ecc) ecc = q;
      }
      T[e] = (float)tr;
      f[6 * e + 0] = (float)ecc * 0.125f;
      f[6 * e + 1] = (float)(tr / (double)(N - 1)) * 0.125f;
#pragma unroll
      for (int q = 2; q <= 5; ++q) {
        const float nq = (float)(st[q - 1] - st[q]);
        f[6 * e + q] = logf(1.f + nq) * inv_logn;
      }
    }
    const int* A = s->adj;
    f[24] = base_distance(levels, win_levels, cap, N, w.x[0], w.x[2]) * 0.125f;
    f[25] = base_distance(levels, win_levels, cap, N, w.x[1], w.x[3]) * 0.125f;
    f[26] = base_distance(levels, win_levels, cap, N, w.x[0], w.x[3]) * 0.125f;
    f[27] = base_distance(levels, win_levels, cap, N, w.x[1], w.x[2]) * 0.125f;
    f[28] = (float)common_neighbours(A, d, w.x[0], w.x[1]) / (float)d;
    f[29] = (float)common_neighbours(A, d, w.x[2], w.x[3]) / (float)d;
    f[30] = fabsf(T[0] - T[2]) / (float)(N - 1);
    f[31] = fabsf(T[1] - T[3]) / (float)(N - 1);
  }
  bf16* row = X + (long long)k * mlp::kFeatures;
#pragma unroll
  for (int i = 0; i < mlp::kFeatures; ++i) row[i] = __float2bfloat16_rn(f[i]);
}

// Keeps the K - n_rand candidates with the smallest predicted change
// (invalid ones last) and n_rand more drawn from the rest, and writes the
// whole ranking (rank, rank_key) for the predicted composites.  One block of
// 1024 threads, bitonic sort of G <= kMaxProposals (key, index) pairs.
constexpr int kMaxProposals = 4096;
__global__ void __launch_bounds__(1024) select_kernel(const State* __restrict__ s, const Swap* __restrict__ sw,
                                                      const float* __restrict__ y, int G, int K, int n_rand,
                                                      int* __restrict__ sel, int* __restrict__ rank,
                                                      float* __restrict__ rank_key) {
  __shared__ float s_key[kMaxProposals];
  __shared__ int s_idx[kMaxProposals];
  if (s->done) return;
  int P = 1;
  while (P < G) P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    const bool ok = i < G && sw[i].valid;
    s_key[i] = ok ? y[i] : FLT_MAX;
    s_idx[i] = i < G ? i : 0;
  }
  __syncthreads();
  for (int size = 2; size <= P; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        const int j = i ^ stride;
        if (j > i) {
          const bool up = (i & size) == 0;
          const float ki = s_key[i], kj = s_key[j];
          const int ii = s_idx[i], ij = s_idx[j];
          const bool gt = ki > kj || (ki == kj && ii > ij);
          if (gt == up) {
            s_key[i] = kj; s_key[j] = ki;
            s_idx[i] = ij; s_idx[j] = ii;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int q = threadIdx.x; q < G; q += blockDim.x) {
    rank[q] = s_idx[q];
    rank_key[q] = s_key[q];
  }
  const int top = K - n_rand;
  for (int q = threadIdx.x; q < K; q += blockDim.x) {
    if (q < top) {
      sel[q] = s_idx[q];
    } else {
      const unsigned long long h = draw(s->seed ^ 0x243f6a8885a308d3ULL, (unsigned long long)s->step, 0x5e1ecULL, q);
      sel[q] = s_idx[top + below(h, G - top)];
    }
  }
}

// The predicted list: walking the ranking best first, every valid proposal
// predicted to lower the distance total (key < 0) whose endpoints are not
// yet used, up to pred_max swaps.  One thread.
__global__ void pred_list_kernel(State* __restrict__ s, const Swap* __restrict__ sw, const int* __restrict__ rank,
                                 const float* __restrict__ rank_key, int G, int pred_max, Swap* __restrict__ pred,
                                 unsigned* __restrict__ vmark) {
  if (s->done || threadIdx.x != 0) return;
  int m = 0;
  for (int r = 0; r < G && m < pred_max; ++r) {
    if (!(rank_key[r] < 0.f)) break;   // sorted: no further predicted gain
    const Swap w = sw[rank[r]];
    if (!w.valid) continue;
    int cl[4];
    const int nc = move_classes(s, w, cl);
    if (!classes_free(vmark, cl, nc)) continue;
    classes_set(vmark, cl, nc, true);
    pred[m++] = w;
  }
  for (int i = 0; i < m; ++i) {
    int cl[4];
    const int nc = move_classes(s, pred[i], cl);
    classes_set(vmark, cl, nc, false);
  }
  s->n_pred = m;
}

// The composite batch: slot 0 the exact composite, slot 1 + c predicted
// composite c.  Every slot first gets the current adjacency (blockIdx.y =
// slot), then patch_composites_kernel applies each slot's swaps.
__global__ void copy_composites_kernel(const State* __restrict__ s, int* __restrict__ slots, long long slot_stride) {
  if (s->done) return;
  const long long n = (long long)s->N * s->d;
  int* dst = slots + (long long)blockIdx.y * slot_stride;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] = s->adj[i];
}

__global__ void patch_composites_kernel(State* __restrict__ s, const Swap* __restrict__ comp,
                                        const Swap* __restrict__ pred, int* __restrict__ slots,
                                        long long slot_stride) {
  if (s->done) return;
  const int slot = blockIdx.x;
  int* dst = slots + (long long)slot * slot_stride;
  const Swap* list = slot == 0 ? comp : pred;
  const int m = slot == 0 ? s->n_comp : pred_size(s->n_pred, slot - 1);
  // the moves of a list touch disjoint vertex classes: they change disjoint rows
  for (int i = threadIdx.x; i < m; i += blockDim.x)
    if (!apply_move(s, dst, nullptr, list[i])) atomicExch(&s->move_error, 1);
}

}  // namespace sa
}  // namespace ggb

using ggb::sa::State;
using ggb::sa::Swap;

struct ggb_sa {
  int device = -1;
  int sms = 0;
  int N = 0, d = 0, lines = 0;
  int groups = 1;                 // symmetry groups: orbit moves, full evaluation of N/groups sources
  int K = 0, G = 0, n_rand = 0, compose_max = 0;
  int C = 0, pred_max = 0;        // predicted composites (learned mode) and their largest size
  bool learned = false;
  bool delta = false;             // candidates evaluated against the base, not in full
  bool has_base = false;          // the base is kept (delta evaluation, the filter's features)
  bool broken = false;            // a restore failed while re-sizing the base: only destroy is allowed
  State h{};                      // host mirror of the device state
  State* d_state = nullptr;
  int* d_edges = nullptr;
  int* d_adj = nullptr;
  int* d_best_edges = nullptr;
  Swap* d_swaps = nullptr;        // [max(G, K)]
  int* d_sel = nullptr;           // [K]
  Swap* d_comp = nullptr;         // [compose_max]
  Swap* d_pred = nullptr;         // [pred_max]
  unsigned* d_vmark = nullptr;    // [N/32 + 1]
  float* d_labels = nullptr;      // [K]
  float* d_scores = nullptr;      // [max(G, K)]
  int* d_rank = nullptr;          // [G] ranking of the proposals
  float* d_rank_key = nullptr;    // [G]
  __nv_bfloat16* d_X = nullptr;   // [max(G, K)][32]
  unsigned* d_stats = nullptr;    // [N][kStatLevels]
  int* d_sticky = nullptr;        // first device error of any evaluation in a step
  ggb_batch* cand = nullptr;      // full mode: the K candidates
  ggb_batch* comp = nullptr;      // slot 0: exact composite; slot 1 + c: predicted composite c
  ggb_mlp* mlp = nullptr;
  // profile launch (learned mode without delta)
  int pR = 0;
  ggb::ApspCtrl* d_pctrl = nullptr;
  uint4* d_pbuf = nullptr;
  // the base (delta mode): the current graph's levels, all kept, built with
  // 1024-source windows and read as 128-source sub-windows (nwin of them)
  int nwin = 0, level_cap = 0, base_T = 0, base_teams = 0;
  uint4* d_levels = nullptr;
  int nbw = 0;                        // base windows of 1024 sources
  long long* d_lcounts = nullptr;     // per 128-source sub-window and level
  int* d_winlev = nullptr;            // per sub-window completion level
  long long* d_pcounts = nullptr;     // per base window and level (the build's own bookkeeping)
  int* d_pwinlev = nullptr;           // per base window completion level
  ggb::ApspCtrl* d_bctrl = nullptr;   // [0]: the grid barrier, [1 + t]: team t
  uint4* d_bscratch = nullptr;
  ggb::BaseResult* d_bres = nullptr;
  long long* d_dsum = nullptr;        // [K][nwin]
  int* d_dlev = nullptr;              // [K][nwin]
  ggb::BatchOut* d_dout = nullptr;    // [K]
  long long* d_epsum = nullptr;       // [K][4] endpoint transmissions in the candidates
  int* d_epecc = nullptr;             // [K][4]
  // the endpoints' bit-parallel search
  int ep_nw = 0;                      // words per row: ceil(4K / 32)
  unsigned* d_eprows = nullptr;       // [2][N][ep_nw]
  int* d_ephead = nullptr;            // [N]
  int* d_epnext = nullptr;            // [4K]
  unsigned* d_epmisc = nullptr;       // changed [kDeltaLevels], newbits [kDeltaLevels][32], tsum [1024], unreach [32]
  ggb::ApspCtrl* d_epctrl = nullptr;
  uint4* d_dpool = nullptr;           // dense fallback slots of the delta evaluation
  int* d_dused = nullptr;
  int dense_slots = 0;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

template <typename T>
int sdev(T** p, size_t n) {
  if (cudaMalloc(p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return core_fail(GGB_ENOMEM, "cudaMalloc of %zu bytes failed", n * sizeof(T));
  }
  return GGB_OK;
}

const void* profile_kernel_for(int R) {
  switch (R) {
    case 16: return (const void*)ggb::apsp_profile_kernel<16>;
    case 32: return (const void*)ggb::apsp_profile_kernel<32>;
    case 64: return (const void*)ggb::apsp_profile_kernel<64>;
    default: return nullptr;
  }
}

size_t profile_smem_for(int R) {
  switch (R) {
    case 16: return ggb::apsp_smem_bytes<16>();
    case 32: return ggb::apsp_smem_bytes<32>();
    case 64: return ggb::apsp_smem_bytes<64>();
    default: return 0;
  }
}

ggb::ApspArgs graph_args(ggb_sa* a) {
  ggb::ApspArgs p;
  std::memset(&p, 0, sizeof p);
  p.adj = a->d_adj;
  p.timeout_ns = 2000000000LL;
  p.N = a->N;
  p.d = a->d;
  p.n_src1 = a->N / a->groups;
  p.split = a->N;
  p.groups = a->groups;
  p.win_first = 0;
  p.win_stride = 1;
  p.vec4 = (a->d % 4 == 0) ? 1 : 0;
  return p;
}

int coop_launch(const void* fn, int grid, size_t smem, void** params, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(ggb::kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  SCUDA(cudaLaunchKernelExC(&cfg, fn, params));
  ggb::core_add_launches(1);
  return GGB_OK;
}

// Profile of the current graph (per-vertex statistics), gated on *gate.
int enqueue_profile(ggb_sa* a, const int* gate, cudaStream_t st) {
  SCUDA(cudaMemsetAsync(a->d_pctrl, 0, sizeof(ggb::ApspCtrl), st));
  ggb::ApspArgs p = graph_args(a);
  p.buf0 = a->d_pbuf;
  p.buf1 = a->d_pbuf + (size_t)a->N * a->pR;
  p.ctrl = a->d_pctrl;
  p.stats = a->d_stats;
  int* sticky = a->d_sticky;
  void* params[] = {(void*)&p, (void*)&gate, (void*)&sticky};
  return coop_launch(profile_kernel_for(a->pR), a->sms, profile_smem_for(a->pR), params, st);
}

// The base of the delta evaluation and the per-vertex statistics read back
// from its levels (the delta path and the filter's features use them),
// gated on *gate.
int enqueue_base(ggb_sa* a, const int* gate, cudaStream_t st) {
  SCUDA(cudaMemsetAsync(a->d_bctrl, 0, (size_t)(1 + a->base_teams) * sizeof(ggb::ApspCtrl), st));
  ggb::ApspArgs p = graph_args(a);
  p.stats = nullptr;   // the filter's statistics are read back from the levels (base_counts_kernel)
  p.levels = a->d_levels;
  p.level_counts = a->d_pcounts;
  p.win_levels = a->d_pwinlev;
  p.level_cap = a->level_cap;
  ggb::BaseArgs b;
  b.sub_counts = a->d_lcounts;
  b.sub_count_len = (long long)a->nwin * (a->level_cap + 1);
  b.grid_ctrl = a->d_bctrl;
  b.team_ctrl = a->d_bctrl + 1;
  b.scratch = a->d_bscratch;
  b.result = a->d_bres;
  b.gate = gate;
  b.sticky = a->d_sticky;
  b.n_teams = a->base_teams;
  b.team_ctas = a->base_T;
  void* params[] = {(void*)&p, (void*)&b};
  int rc = coop_launch((const void*)ggb::apsp_base_kernel<ggb::kBaseR>, a->base_teams * a->base_T,
                       ggb::apsp_smem_bytes<ggb::kBaseR>(), params, st);
  if (rc) return rc;
  ggb::base_counts_kernel<<<(a->N + 31) / 32, ggb::kStatsWarps * 32, 0, st>>>(
      a->d_levels, a->d_pwinlev, a->level_cap, a->N, a->nbw, a->N, a->d_stats, a->d_lcounts, gate);
  ggb::sub_levels_kernel<<<(a->nwin + 127) / 128, 128, 0, st>>>(a->d_lcounts, a->d_pwinlev, a->level_cap, a->N,
                                                               a->nwin, a->N, a->d_winlev, gate);
  ggb::core_add_launches(2);
  SCUDA(cudaGetLastError());
  return GGB_OK;
}

ggb::DeltaArgs delta_args(ggb_sa* a, const int* sel) {
  ggb::DeltaArgs g;
  g.levels = a->d_levels;
  g.level_counts = a->d_lcounts;
  g.win_levels = a->d_winlev;
  g.adj = a->d_adj;
  g.sw = a->d_swaps;
  g.sel = sel;
  g.stop = &a->d_state->done;
  g.dsum = a->d_dsum;
  g.dlev = a->d_dlev;
  g.stats = a->d_stats;
  g.ep_sum = a->d_epsum;
  g.ep_ecc = a->d_epecc;
  g.dense_pool = a->d_dpool;
  g.dense_used = a->d_dused;
  g.dense_slots = a->dense_slots;
  g.N = a->N;
  g.d = a->d;
  g.nwin = a->nwin;
  g.n_src = a->N;
  g.level_cap = a->level_cap;
  g.K = a->K;
  return g;
}

int enqueue_delta(ggb_sa* a, const int* sel, cudaStream_t st) {
  const ggb::DeltaArgs g = delta_args(a, sel);
  const size_t smem = 2 * (size_t)((a->N + 31) / 32) * sizeof(unsigned);   // claims, dirty bitmap
  SCUDA(cudaMemsetAsync(a->d_dused, 0, sizeof(int), st));
  {
    ggb::EndpointArgs e;
    e.adj = a->d_adj;
    e.sw = a->d_swaps;
    e.sel = sel;
    e.stop = &a->d_state->done;
    e.ctrl = a->d_epctrl;
    e.rows = a->d_eprows;
    e.head = a->d_ephead;
    e.next = a->d_epnext;
    e.changed = a->d_epmisc;
    e.newbits = a->d_epmisc + ggb::kDeltaLevels;
    e.tsum = e.newbits + ggb::kDeltaLevels * 32;
    e.unreach = e.tsum + 1024;
    e.ep_sum = a->d_epsum;
    e.ep_ecc = a->d_epecc;
    e.timeout_ns = 2000000000LL;
    e.N = a->N;
    e.d = a->d;
    e.K = a->K;
    e.nw = a->ep_nw;
    SCUDA(cudaMemsetAsync(a->d_epctrl, 0, sizeof(ggb::ApspCtrl), st));
    void* params[] = {(void*)&e};
    int rc = coop_launch((const void*)ggb::endpoint_sweep_kernel, a->sms, 0, params, st);
    if (rc) return rc;
  }
  ggb::delta_kernel<<<a->K * a->nwin, ggb::kDeltaThreads, smem, st>>>(g);
  ggb::delta_reduce_kernel<<<(a->K + 7) / 8, 256, 0, st>>>(g, a->d_bres, a->d_dout);
  ggb::core_add_launches(3);
  SCUDA(cudaGetLastError());
  return GGB_OK;
}

// Every kernel of one step, in order, on `st` (captured once).
int enqueue_step(ggb_sa* a, cudaStream_t st) {
  using namespace ggb::sa;
  State* s = a->d_state;
  const int G = a->learned ? a->G : a->K;
  gen_kernel<<<(G + 127) / 128, 128, 0, st>>>(s, a->d_swaps, G);
  int launches = 1;
  const int* sel = nullptr;
  if (a->learned) {
    features_kernel<<<(G + 127) / 128, 128, 0, st>>>(s, a->d_swaps, G, a->d_stats, a->d_levels, a->d_winlev,
                                                     a->level_cap, a->d_X);
    int rc = ggb::mlp_forward(a->mlp, a->d_X, G, a->d_scores, st, false);
    if (rc) return rc;
    select_kernel<<<1, 1024, 0, st>>>(s, a->d_swaps, a->d_scores, G, a->K, a->n_rand, a->d_sel, a->d_rank,
                                      a->d_rank_key);
    sel = a->d_sel;
    launches += 2;
  }
  int rc;
  const ggb::BatchOut* singles;
  if (a->delta) {
    rc = enqueue_delta(a, sel, st);
    if (rc) return rc;
    singles = a->d_dout;
  } else {
    const long long stride = a->cand->off.size() > 1 ? a->cand->off[1] - a->cand->off[0] : 0;
    const int bx = std::max(1, std::min(a->sms * 4 / std::max(a->K, 1), (int)(((long long)a->N * a->d + 255) / 256)));
    materialize_kernel<<<dim3(bx, a->K), 256, 0, st>>>(s, a->d_swaps, sel, a->cand->d_adj, stride);
    if (a->groups > 1) {
      patch_orbit_kernel<<<a->K, 32, 0, st>>>(s, a->d_swaps, sel, a->cand->d_adj, stride);
      launches += 1;
    }
    rc = ggb::batch_enqueue(a->cand, st);
    if (rc) return rc;
    singles = a->cand->d_out;
    launches += 1;
  }
  compose_kernel<<<1, kComposeThreads, 0, st>>>(s, a->d_swaps, sel, singles, a->K, a->d_comp, a->compose_max,
                                                a->d_vmark);
  launches += 1;
  const ggb::BatchOut* comp_out = nullptr;
  if (a->comp) {
    if (a->C > 0) {
      pred_list_kernel<<<1, 32, 0, st>>>(s, a->d_swaps, a->d_rank, a->d_rank_key, G, a->pred_max, a->d_pred,
                                         a->d_vmark);
      launches += 1;
    }
    const long long stride = a->comp->off.size() > 1 ? a->comp->off[1] - a->comp->off[0] : 0;
    const int slots = 1 + a->C;
    const int bx = std::max(1, std::min(a->sms * 4 / slots, (int)(((long long)a->N * a->d + 255) / 256)));
    copy_composites_kernel<<<dim3(bx, slots), 256, 0, st>>>(s, a->comp->d_adj, stride);
    patch_composites_kernel<<<slots, 128, 0, st>>>(s, a->d_comp, a->d_pred, a->comp->d_adj, stride);
    rc = ggb::batch_enqueue(a->comp, st);
    if (rc) return rc;
    comp_out = a->comp->d_out;
    launches += 2;
  }
  decide_kernel<<<1, std::max(32, (a->K + 31) / 32 * 32), 0, st>>>(s, a->d_swaps, sel, singles, a->K, a->d_comp,
                                                                   comp_out, a->learned ? a->d_labels : nullptr,
                                                                   a->d_pred, a->comp ? a->C : 0);
  launches += 1;
  if (a->learned) {
    rc = ggb::mlp_train_rows(a->mlp, a->d_X, a->d_sel, a->d_labels, a->K, st);
    if (rc) return rc;
  }
  if (a->has_base) {
    rc = enqueue_base(a, &s->accepted, st);
    if (rc) return rc;
  } else if (a->learned) {
    rc = enqueue_profile(a, &s->accepted, st);
    if (rc) return rc;
  }
  best_copy_kernel<<<a->sms, 256, 0, st>>>(s);
  launches += 1;
  ggb::core_add_launches(launches);
  SCUDA(cudaGetLastError());
  return GGB_OK;
}

int capture_step(ggb_sa* a) {
  if (a->exec) return GGB_OK;
  SCUDA(cudaStreamBeginCapture(a->st, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(a, a->st);
  cudaGraph_t gph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(a->st, &gph);
  if (rc) {
    if (gph) cudaGraphDestroy(gph);
    return rc;
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return core_fail(GGB_ECUDA, "capturing the annealing step failed: %s", cudaGetErrorString(e));
  }
  a->graph = gph;
  SCUDA(cudaGraphInstantiate(&a->exec, gph, 0));
  return GGB_OK;
}

void drop_graph(ggb_sa* a) {
  if (a->exec) cudaGraphExecDestroy(a->exec);
  if (a->graph) cudaGraphDestroy(a->graph);
  a->exec = nullptr;
  a->graph = nullptr;
}

int pull_state(ggb_sa* a) {
  SCUDA(cudaMemcpyAsync(&a->h, a->d_state, sizeof(State), cudaMemcpyDeviceToHost, a->st));
  SCUDA(cudaStreamSynchronize(a->st));
  return GGB_OK;
}

int push_state(ggb_sa* a) {
  SCUDA(cudaMemcpyAsync(a->d_state, &a->h, sizeof(State), cudaMemcpyHostToDevice, a->st));
  SCUDA(cudaStreamSynchronize(a->st));
  return GGB_OK;
}

void destroy(ggb_sa* a) {
  if (!a) return;
  if (a->device >= 0) cudaSetDevice(a->device);
  if (a->st) cudaStreamSynchronize(a->st);
  drop_graph(a);
  for (void* q : {(void*)a->d_state, (void*)a->d_edges, (void*)a->d_adj, (void*)a->d_best_edges, (void*)a->d_swaps,
                  (void*)a->d_sel, (void*)a->d_comp, (void*)a->d_pred, (void*)a->d_vmark, (void*)a->d_labels,
                  (void*)a->d_scores, (void*)a->d_rank, (void*)a->d_rank_key, (void*)a->d_X, (void*)a->d_stats,
                  (void*)a->d_sticky, (void*)a->d_pctrl, (void*)a->d_pbuf, (void*)a->d_levels, (void*)a->d_lcounts,
                  (void*)a->d_winlev, (void*)a->d_pcounts, (void*)a->d_pwinlev, (void*)a->d_bctrl, (void*)a->d_bscratch, (void*)a->d_bres, (void*)a->d_dsum,
                  (void*)a->d_dlev, (void*)a->d_dout, (void*)a->d_dpool, (void*)a->d_dused,
                  (void*)a->d_epsum, (void*)a->d_epecc, (void*)a->d_eprows, (void*)a->d_ephead,
                  (void*)a->d_epnext, (void*)a->d_epmisc, (void*)a->d_epctrl})
    cudaFree(q);
  if (a->cand) ggb_batch_destroy(a->cand);
  if (a->comp) ggb_batch_destroy(a->comp);
  if (a->mlp) ggb_mlp_destroy(a->mlp);
  if (a->st) cudaStreamDestroy(a->st);
  cudaGetLastError();
  delete a;
}

int check_sticky(ggb_sa* a) {
  int sticky = 0;
  SCUDA(cudaMemcpy(&sticky, a->d_sticky, sizeof sticky, cudaMemcpyDeviceToHost));
  if (sticky == ggb::kErrTimeout) return core_fail(GGB_ETIMEOUT, "a barrier wait of an annealing step ran out");
  if (sticky == ggb::kErrAdj) return core_fail(GGB_EADJ, "an annealing candidate had an entry outside [0, nodes)");
  if (sticky) return core_fail(GGB_ECUDA, "an annealing evaluation failed (device error %d)", sticky);
  return GGB_OK;
}

// Evaluates the current graph exactly (ungated base build or profile) and
// sets the current and best values from it.
int evaluate_current(ggb_sa* a) {
  long long sum = 0;
  int diam = 0, disc = 0;
  if (a->has_base) {
    int rc = enqueue_base(a, nullptr, a->st);
    if (rc) return rc;
    ggb::BaseResult r;
    SCUDA(cudaMemcpyAsync(&r, a->d_bres, sizeof r, cudaMemcpyDeviceToHost, a->st));
    SCUDA(cudaStreamSynchronize(a->st));
    rc = check_sticky(a);
    if (rc) return rc;
    sum = r.sum;
    diam = r.diam;
    disc = r.disconnected;
  } else {
    int rc = enqueue_profile(a, nullptr, a->st);
    if (rc) return rc;
    ggb::ApspCtrl c;
    SCUDA(cudaMemcpyAsync(&c, a->d_pctrl, sizeof c, cudaMemcpyDeviceToHost, a->st));
    SCUDA(cudaStreamSynchronize(a->st));
    rc = check_sticky(a);
    if (rc) return rc;
    if (!c.done) return core_fail(GGB_ECUDA, "profile evaluation did not complete");
    sum = c.sum;
    diam = c.diam;
    disc = c.disconnected;
  }
  if (disc || diam >= a->N) return core_fail(GGB_EINVAL, "the initial graph is not connected");
  a->h.cur_diam = a->h.best_diam = diam;
  a->h.cur_total = a->h.best_total = a->h.prev_total = sum + (long long)a->N * (a->N - 1);
  return GGB_OK;
}

void set_base_team(ggb_sa* a, int T) {
  a->base_T = T;
  a->base_teams = std::max(1, std::min(a->sms / T, a->nbw));
}

// Times the base build of the current graph with teams of 1, 2, 4, 8 and 16
// CTAs and the size that gives every 1024-source window its own team on the
// whole GPU (two launches each after one warm-up) and keeps the fastest.  The
// result never depends on the choice.
int tune_base(ggb_sa* a) {
  // Each team size is timed in three rounds of one warm-up and two timed
  // builds, the rounds interleaved so that a clock ramp or a noisy moment
  // does not decide the choice; the least time of a size's rounds counts.
  cudaEvent_t e0, e1;
  SCUDA(cudaEventCreate(&e0));
  SCUDA(cudaEventCreate(&e1));
  const int sizes[] = {1, 2, 4, 8, 16, std::max(1, a->sms / a->nbw)};
  float best_ms[6];
  for (float& b : best_ms) b = 1e30f;
  for (int round = 0; round < 3; ++round) {
    for (int i = 0; i < 6; ++i) {
      const int T = sizes[i];
      if (T > a->sms) continue;
      set_base_team(a, T);
      int rc = enqueue_base(a, nullptr, a->st);
      if (rc) return rc;
      SCUDA(cudaEventRecord(e0, a->st));
      for (int k = 0; k < 2 && !rc; ++k) rc = enqueue_base(a, nullptr, a->st);
      if (rc) return rc;
      SCUDA(cudaEventRecord(e1, a->st));
      SCUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      SCUDA(cudaEventElapsedTime(&ms, e0, e1));
      best_ms[i] = std::min(best_ms[i], ms);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int bestT = 4;
  float best = 1e30f;
  for (int i = 0; i < 6; ++i)
    if (sizes[i] <= a->sms && best_ms[i] < best) { best = best_ms[i]; bestT = sizes[i]; }
  set_base_team(a, bestT);
  return check_sticky(a);
}

int alloc_base(ggb_sa* a) {
  a->nwin = (a->N + 127) / 128;
  a->nbw = (a->N + 1023) / 1024;
  // a->level_cap is set by create() from the initial graph's diameter
  set_base_team(a, 1);   // sizes the team arrays for the most teams any plan uses
  int nb = 0;
  const void* bk = (const void*)ggb::apsp_base_kernel<ggb::kBaseR>;
  const size_t bsm = ggb::apsp_smem_bytes<ggb::kBaseR>();
  SCUDA(cudaFuncSetAttribute(bk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bsm));
  SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, bk, ggb::kThreads, bsm));
  if (nb < 1) return core_fail(GGB_ECUDA, "base kernel cannot be resident");
  const size_t cells = (size_t)a->nbw * (a->level_cap + 1) * a->N * ggb::kBaseR;
  int rc;
  if ((rc = sdev(&a->d_levels, cells)) || (rc = sdev(&a->d_lcounts, (size_t)a->nwin * (a->level_cap + 1))) ||
      (rc = sdev(&a->d_winlev, (size_t)a->nwin)) || (rc = sdev(&a->d_pcounts, (size_t)a->nbw * (a->level_cap + 1))) ||
      (rc = sdev(&a->d_pwinlev, (size_t)a->nbw)) || (rc = sdev(&a->d_bctrl, (size_t)1 + a->base_teams)) ||
      (rc = sdev(&a->d_bscratch, (size_t)a->base_teams * 2 * a->N * ggb::kBaseR)) || (rc = sdev(&a->d_bres, 1)) ||
      (rc = sdev(&a->d_dsum, (size_t)a->K * a->nwin)) || (rc = sdev(&a->d_dlev, (size_t)a->K * a->nwin)) ||
      (rc = sdev(&a->d_dout, (size_t)a->K)))
    return rc;
  // dense fallback: up to 8 windows per candidate, at most 1 GiB
  a->dense_slots = (int)std::max<long long>(1, std::min<long long>(8LL * a->K, (1LL << 30) / (32LL * a->N)));
  if ((rc = sdev(&a->d_dpool, (size_t)a->dense_slots * 2 * a->N)) || (rc = sdev(&a->d_dused, 1)) ||
      (rc = sdev(&a->d_epsum, (size_t)4 * a->K)) || (rc = sdev(&a->d_epecc, (size_t)4 * a->K)) ||
      (rc = sdev(&a->d_eprows, (size_t)2 * a->N * ((4 * a->K + 31) / 32))) || (rc = sdev(&a->d_ephead, (size_t)a->N)) ||
      (rc = sdev(&a->d_epnext, (size_t)4 * a->K)) ||
      (rc = sdev(&a->d_epmisc, (size_t)ggb::kDeltaLevels * 33 + 1024 + 32)) || (rc = sdev(&a->d_epctrl, 1)))
    return rc;
  a->ep_nw = (4 * a->K + 31) / 32;
  return GGB_OK;
}

int create(ggb_sa* a, int nodes, int degree, int groups, const int* edges, int K, int G, int compose_max,
           unsigned long long seed) {
  using namespace ggb::sa;
  a->N = nodes;
  a->d = degree;
  a->groups = groups;
  a->lines = (int)((long long)nodes * degree / 2);
  a->K = K;
  a->G = G;
  a->learned = G > K;
  // the endpoint search hands neighbour ids over by warp shuffle; orbit moves
  // change 4*groups rows, which the delta path does not serve
  a->delta = K > 1 && degree <= 32 && groups == 1;
  a->compose_max = compose_max;
  a->n_rand = a->learned ? std::max(1, K / 4) : 0;
  a->C = a->learned ? 4 : 0;
  a->pred_max = a->learned ? 64 : 0;
  int dev = 0;
  SCUDA(cudaGetDevice(&dev));
  a->device = dev;
  SCUDA(cudaDeviceGetAttribute(&a->sms, cudaDevAttrMultiProcessorCount, dev));
  int l2 = 0;
  SCUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
  SCUDA(cudaStreamCreateWithFlags(&a->st, cudaStreamNonBlocking));
  // edges -> adjacency (general/sa.c:61-74 order), with the checks of a simple regular graph
  std::vector<int> adj((size_t)nodes * degree), fill(nodes, 0);
  for (int i = 0; i < a->lines; ++i) {
    const int u = edges[2 * i], v = edges[2 * i + 1];
    if (u < 0 || u >= nodes || v < 0 || v >= nodes || u == v)
      return core_fail(GGB_EINVAL, "line %d: bad endpoint or self-loop", i);
    if (fill[u] >= degree || fill[v] >= degree) return core_fail(GGB_EINVAL, "the graph is not %d-regular", degree);
    for (int j = 0; j < fill[u]; ++j)
      if (adj[(size_t)u * degree + j] == v) return core_fail(GGB_EINVAL, "line %d repeats an edge", i);
    adj[(size_t)u * degree + fill[u]++] = v;
    adj[(size_t)v * degree + fill[v]++] = u;
  }
  if (groups > 1) {
    // the reference's symmetric line order: line k*BL + i is line i shifted by k*B
    const int B = nodes / groups, BL = a->lines / groups;
    for (int l = BL; l < a->lines; ++l) {
      const int i = l % BL, k = l / BL;
      if (edges[2 * l] != (edges[2 * i] + k * B) % nodes || edges[2 * l + 1] != (edges[2 * i + 1] + k * B) % nodes)
        return core_fail(GGB_EINVAL, "line %d is not line %d shifted by %d*%d: not in the symmetric line order", l,
                         i, k, B);
    }
  }
  int rc;
  const size_t L2 = (size_t)2 * a->lines;
  const size_t GK = (size_t)std::max(G, K);
  if ((rc = sdev(&a->d_state, 1)) || (rc = sdev(&a->d_edges, L2)) || (rc = sdev(&a->d_adj, adj.size())) ||
      (rc = sdev(&a->d_best_edges, L2)) || (rc = sdev(&a->d_swaps, GK)) || (rc = sdev(&a->d_sel, (size_t)K)) ||
      (rc = sdev(&a->d_comp, (size_t)std::max(compose_max, 1))) ||
      (rc = sdev(&a->d_pred, (size_t)std::max(a->pred_max, 1))) ||
      (rc = sdev(&a->d_vmark, (size_t)nodes / 32 + 1)) || (rc = sdev(&a->d_labels, (size_t)K)) ||
      (rc = sdev(&a->d_scores, GK)) || (rc = sdev(&a->d_rank, GK)) || (rc = sdev(&a->d_rank_key, GK)) ||
      (rc = sdev(&a->d_X, GK * ggb::mlp::kFeatures)) || (rc = sdev(&a->d_stats, (size_t)nodes * ggb::kStatLevels)) ||
      (rc = sdev(&a->d_pctrl, 1)) || (rc = sdev(&a->d_sticky, 1)))
    return rc;
  SCUDA(cudaMemset(a->d_sticky, 0, sizeof(int)));
  SCUDA(cudaMemcpy(a->d_edges, edges, L2 * sizeof(int), cudaMemcpyHostToDevice));
  SCUDA(cudaMemcpy(a->d_best_edges, edges, L2 * sizeof(int), cudaMemcpyHostToDevice));
  SCUDA(cudaMemcpy(a->d_adj, adj.data(), adj.size() * sizeof(int), cudaMemcpyHostToDevice));
  SCUDA(cudaMemset(a->d_vmark, 0, ((size_t)nodes / 32 + 1) * sizeof(unsigned)));
  SCUDA(cudaMemset(a->d_swaps, 0, GK * sizeof(Swap)));
  SCUDA(cudaMemset(a->d_X, 0, GK * ggb::mlp::kFeatures * sizeof(__nv_bfloat16)));
  // profile window: the widest of 2048 / 4096 / 8192 sources whose two matrices fit in about half the L2
  a->pR = 16;
  for (int R = 64; R >= 16; R /= 2)
    if ((double)2 * nodes * 16.0 * R <= 0.55 * l2) { a->pR = R; break; }
  for (int R = 16; R <= 64; R *= 2) {
    int nb = 0;
    SCUDA(cudaFuncSetAttribute(profile_kernel_for(R), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)profile_smem_for(R)));
    SCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, profile_kernel_for(R), ggb::kThreads,
                                                        profile_smem_for(R)));
    if (nb < 1) return core_fail(GGB_ECUDA, "profile kernel R=%d cannot be resident", R);
  }
  if ((rc = sdev(&a->d_pbuf, (size_t)2 * nodes * a->pR))) return rc;
  if (a->delta) {
    // The base keeps levels 0..diameter of every 128-source window: no
    // window of a later current graph needs more, because no accepted move
    // ever lengthens the diameter (general/sa.c:371-384).  When that does not
    // fit in a quarter of the free device memory (or the initial graph is not
    // connected, which create() reports below), candidates are evaluated in
    // full instead.
    rc = enqueue_profile(a, nullptr, a->st);
    if (rc) return rc;
    ggb::ApspCtrl c;
    SCUDA(cudaMemcpyAsync(&c, a->d_pctrl, sizeof c, cudaMemcpyDeviceToHost, a->st));
    SCUDA(cudaStreamSynchronize(a->st));
    if ((rc = check_sticky(a))) return rc;
    size_t free_b = 0, total_b = 0;
    SCUDA(cudaMemGetInfo(&free_b, &total_b));
    // the kept levels plus the build's two row buffers per team (at most one team per SM or per window)
    const int nbw = (nodes + 1023) / 1024;
    const double base_bytes = (double)nbw * ggb::kBaseR * (c.diam + 1) * nodes * 16.0 +
                              (double)std::min(a->sms, nbw) * 2 * nodes * ggb::kBaseR * 16.0;
    if (c.done && !c.disconnected && c.diam < nodes && base_bytes <= 0.25 * (double)free_b) {
      a->level_cap = std::max(2, c.diam);
      if ((rc = alloc_base(a))) return rc;
      a->has_base = true;
    } else {
      a->delta = false;
      if (a->learned)
        return core_fail(GGB_EINVAL, "the proposal filter reads its features from the base, which does not fit "
                                     "(%.1f GB for this graph)", base_bytes / 1e9);
    }
  }
  // the candidate batch (full mode) and the composite batch
  const int nc = 1 + a->C;
  const int nmax = std::max(K, nc);
  std::vector<int> nn(nmax, nodes), bn(nmax, nodes / groups), gg(nmax, groups), dd(nmax, degree);
  if (!a->delta) {
    if ((rc = ggb_batch_create(K, nn.data(), bn.data(), gg.data(), dd.data(), &a->cand))) return rc;
    a->cand->stop = &a->d_state->done;
    a->cand->sticky = a->d_sticky;
  }
  if (compose_max >= 2 || a->C > 0) {
    if ((rc = ggb_batch_create(nc, nn.data(), bn.data(), gg.data(), dd.data(), &a->comp))) return rc;
    a->comp->stop = &a->d_state->done;
    a->comp->sticky = a->d_sticky;
  }
  if (a->learned) {
    if ((rc = ggb_mlp_create((int)GK, seed ^ 0x4d4c50ULL, &a->mlp))) return rc;
  }
  // initial state
  std::memset(&a->h, 0, sizeof a->h);
  a->h.N = nodes;
  a->h.d = degree;
  a->h.lines = a->lines;
  a->h.K = K;
  a->h.edges = a->d_edges;
  a->h.adj = a->d_adj;
  a->h.best_edges = a->d_best_edges;
  a->h.temp = 0.0;
  a->h.cooling = 1.0;
  a->h.hill = 1;
  a->h.seed = seed;
  a->h.best_step = -1;
  a->h.target_diam = INT_MAX;
  a->h.target_total = LLONG_MIN;
  a->h.label_scale = 16.0f / (float)nodes;
  a->h.label_clip = 16.0f;
  a->h.groups = groups;
  a->h.B = nodes / groups;
  a->h.BL = a->lines / groups;
  a->h.grid_height = 0;
  a->h.grid_length = 0;
  a->h.move_error = 0;
  if ((rc = push_state(a))) return rc;
  if (a->has_base && (rc = tune_base(a))) return rc;
  if ((rc = evaluate_current(a))) return rc;
  if ((rc = push_state(a))) return rc;
  if (a->delta) {
    // One trial step of the delta path: when more than a quarter of the
    // candidates cannot be served (graphs whose swaps change most distances,
    // e.g. sparse graphs of large diameter), candidates are evaluated in full.
    gen_kernel<<<(K + 127) / 128, 128, 0, a->st>>>(a->d_state, a->d_swaps, K);
    if ((rc = enqueue_delta(a, nullptr, a->st))) return rc;
    std::vector<ggb::BatchOut> t(K);
    SCUDA(cudaMemcpyAsync(t.data(), a->d_dout, K * sizeof(ggb::BatchOut), cudaMemcpyDeviceToHost, a->st));
    SCUDA(cudaStreamSynchronize(a->st));
    if ((rc = check_sticky(a))) return rc;
    int unserved = 0;
    for (const auto& o : t) unserved += o.done ? 0 : 1;
    if (4 * unserved > K) {
      a->delta = false;
      if ((rc = ggb_batch_create(K, nn.data(), bn.data(), gg.data(), dd.data(), &a->cand))) return rc;
      a->cand->stop = &a->d_state->done;
      a->cand->sticky = a->d_sticky;
      for (int k = 0; k < K; ++k) {
        int* slot = nullptr;
        ggb_batch_adj_device(a->cand, k, &slot);
        SCUDA(cudaMemcpy(slot, a->d_adj, adj.size() * sizeof(int), cudaMemcpyDeviceToDevice));
      }
    }
  }
  // batch slots hold the current graph until the first step
  for (ggb_batch* b : {a->cand, a->comp}) {
    if (!b) continue;
    for (int k = 0; k < b->n; ++k) {
      int* slot = nullptr;
      ggb_batch_adj_device(b, k, &slot);
      SCUDA(cudaMemcpy(slot, a->d_adj, adj.size() * sizeof(int), cudaMemcpyDeviceToDevice));
    }
  }
  return GGB_OK;
}

// ---- checkpoints -------------------------------------------------------------
// Layout: header, the device State (pointer fields replaced on restore), the
// current and the best edge lists, and with a filter the network's training
// state.  Only the library that wrote a checkpoint reads it (state_bytes and
// the version are checked).
constexpr unsigned kCkptMagic = 0x31434747u;   // "GGC1"
constexpr unsigned kCkptVersion = 1u;
struct CkptHeader {
  unsigned magic, version, state_bytes, mlp_bytes;
  int N, d, groups, lines, K, G, compose_max, C, pred_max, learned;
  int level_cap;   // the base's kept levels (from the first graph's diameter)
  int delta;       // candidates evaluated against the base (1) or in full (0)
};

bool same_config(const CkptHeader& x, const CkptHeader& y) {
  return x.mlp_bytes == y.mlp_bytes && x.N == y.N && x.d == y.d && x.groups == y.groups && x.lines == y.lines &&
         x.K == y.K && x.G == y.G && x.compose_max == y.compose_max && x.C == y.C && x.pred_max == y.pred_max &&
         x.learned == y.learned;
}

// Re-sizes the base to keep levels 0..cap and rebuilds it from the current
// graph.  A resumed run keeps the level cap of the run it continues: the cap
// decides which candidates the delta path serves, hence the counters and,
// with a filter, the training labels.
int reset_level_cap(ggb_sa* a, int cap) {
  SCUDA(cudaStreamSynchronize(a->st));
  drop_graph(a);
  const int T = a->base_T;
  for (void** q : {(void**)&a->d_levels, (void**)&a->d_lcounts, (void**)&a->d_winlev, (void**)&a->d_pcounts,
                   (void**)&a->d_pwinlev, (void**)&a->d_bctrl, (void**)&a->d_bscratch, (void**)&a->d_bres,
                   (void**)&a->d_dsum, (void**)&a->d_dlev, (void**)&a->d_dout, (void**)&a->d_dpool,
                   (void**)&a->d_dused, (void**)&a->d_epsum, (void**)&a->d_epecc, (void**)&a->d_eprows,
                   (void**)&a->d_ephead, (void**)&a->d_epnext, (void**)&a->d_epmisc, (void**)&a->d_epctrl}) {
    cudaFree(*q);
    *q = nullptr;
  }
  a->level_cap = cap;
  a->broken = true;   // until the base is whole again
  int rc = alloc_base(a);
  if (rc) return rc;
  set_base_team(a, T);
  rc = evaluate_current(a);
  if (rc == GGB_OK) a->broken = false;
  return rc;
}

int refuse_broken(const ggb_sa* a) {
  return core_fail(GGB_EPERM, "a restore of this annealer failed while re-sizing its base; destroy it");
}

size_t ckpt_bytes(const ggb_sa* a) {
  return sizeof(CkptHeader) + sizeof(State) + (size_t)4 * a->lines * sizeof(int) +
         (a->learned ? ggb::mlp_state_bytes() : 0);
}

CkptHeader ckpt_header(const ggb_sa* a) {
  CkptHeader h{};
  h.magic = kCkptMagic;
  h.version = kCkptVersion;
  h.state_bytes = (unsigned)sizeof(State);
  h.mlp_bytes = a->learned ? (unsigned)ggb::mlp_state_bytes() : 0u;
  h.N = a->N;
  h.d = a->d;
  h.groups = a->groups;
  h.lines = a->lines;
  h.K = a->K;
  h.G = a->G;
  h.compose_max = a->compose_max;
  h.C = a->C;
  h.pred_max = a->pred_max;
  h.learned = a->learned ? 1 : 0;
  h.level_cap = a->has_base ? a->level_cap : 0;
  h.delta = a->delta ? 1 : 0;
  return h;
}

}  // namespace

extern "C" {

int ggb_sa_create(int nodes, int degree, const int* edges, int candidates, int proposals, int compose_max,
                  unsigned long long seed, ggb_sa** out) {
  if (!out || !edges) return core_fail(GGB_EINVAL, "null pointer");
  *out = nullptr;
  if (nodes < 4 || degree < 1 || ((long long)nodes * degree) % 2 || (long long)nodes * degree > INT_MAX)
    return core_fail(GGB_EINVAL, "nodes >= 4, degree >= 1 and nodes*degree even are required");
  if (candidates < 1 || candidates > ggb::sa::kComposeThreads)
    return core_fail(GGB_EINVAL, "candidates must be in [1, %d]", ggb::sa::kComposeThreads);
  if (proposals < candidates) proposals = candidates;
  if (proposals > candidates) {
    if (proposals > ggb::sa::kMaxProposals || proposals % 16)
      return core_fail(GGB_EINVAL, "proposals must be a multiple of 16 up to %d", ggb::sa::kMaxProposals);
    if (candidates % 16 || candidates > ggb::mlp::kMaxTrainRows)
      return core_fail(GGB_EINVAL, "with a proposal filter, candidates must be a multiple of 16 up to %d",
                       ggb::mlp::kMaxTrainRows);
    if (degree > ggb::sa::kMaxFeatDegree)
      return core_fail(GGB_EINVAL, "the proposal filter's features support degree <= %d", ggb::sa::kMaxFeatDegree);
  }
  if (compose_max < 0 || compose_max > 4096) return core_fail(GGB_EINVAL, "compose_max must be in [0, 4096]");
  ggb_sa* a = new ggb_sa();
  int rc = create(a, nodes, degree, 1, edges, candidates, proposals, compose_max, seed);
  if (rc) {
    destroy(a);
    return rc;
  }
  *out = a;
  return GGB_OK;
}

int ggb_sa_create_symmetric(int nodes, int degree, int groups, const int* edges, int candidates, int compose_max,
                            unsigned long long seed, ggb_sa** out) {
  if (groups == 1) return ggb_sa_create(nodes, degree, edges, candidates, candidates, compose_max, seed, out);
  if (!out || !edges) return core_fail(GGB_EINVAL, "null pointer");
  *out = nullptr;
  if (groups < 2 || nodes % groups || nodes / groups < 3)
    return core_fail(GGB_EINVAL, "groups must divide nodes, with at least 3 vertices per group");
  if (nodes < 4 || degree < 1 || ((long long)nodes * degree) % (2LL * groups) || (long long)nodes * degree > INT_MAX)
    return core_fail(GGB_EINVAL, "nodes*degree must be a multiple of 2*groups");
  if (candidates < 1 || candidates > ggb::sa::kComposeThreads)
    return core_fail(GGB_EINVAL, "candidates must be in [1, %d]", ggb::sa::kComposeThreads);
  if (compose_max < 0 || compose_max > 4096) return core_fail(GGB_EINVAL, "compose_max must be in [0, 4096]");
  ggb_sa* a = new ggb_sa();
  int rc = create(a, nodes, degree, groups, edges, candidates, candidates, compose_max, seed);
  if (rc) {
    destroy(a);
    return rc;
  }
  *out = a;
  return GGB_OK;
}

int ggb_sa_set_grid(ggb_sa* a, int height, int max_length) {
  if (!a) return core_fail(GGB_EINVAL, "null annealer");
  if (a->groups != 1) return core_fail(GGB_EPERM, "grid length limits are served for graphs without symmetry");
  if (height < 1 || a->N % height || max_length < 1)
    return core_fail(GGB_EINVAL, "height must divide nodes and max_length must be >= 1");
  SCUDA(cudaSetDevice(a->device));
  SCUDA(cudaStreamSynchronize(a->st));
  std::vector<int> e((size_t)2 * a->lines);
  SCUDA(cudaMemcpy(e.data(), a->d_edges, e.size() * sizeof(int), cudaMemcpyDeviceToHost));
  for (int l = 0; l < a->lines; ++l) {
    const int u = e[2 * l], v = e[2 * l + 1];
    const int len = std::abs(u / height - v / height) + std::abs(u % height - v % height);
    if (len > max_length)
      return core_fail(GGB_EINVAL, "line %d (%d, %d) is longer than %d on the lattice", l, u, v, max_length);
  }
  int rc = pull_state(a);
  if (rc) return rc;
  a->h.grid_height = height;
  a->h.grid_length = max_length;
  return push_state(a);
}

void ggb_sa_destroy(ggb_sa* a) { destroy(a); }

int ggb_sa_set_schedule(ggb_sa* a, double temp, double cooling_rate, int hill_climbing) {
  if (!a) return core_fail(GGB_EINVAL, "null annealer");
  if (a->broken) return refuse_broken(a);
  if (!(temp >= 0.0) || !(cooling_rate > 0.0)) return core_fail(GGB_EINVAL, "temp >= 0 and cooling_rate > 0");
  if (!hill_climbing && !(temp > 0.0)) return core_fail(GGB_EINVAL, "annealing needs temp > 0");
  SCUDA(cudaSetDevice(a->device));
  int rc = pull_state(a);
  if (rc) return rc;
  a->h.temp = temp;
  a->h.cooling = cooling_rate;
  a->h.hill = hill_climbing ? 1 : 0;
  return push_state(a);
}

int ggb_sa_set_predicted(ggb_sa* a, int composites, int max_swaps) {
  if (!a) return core_fail(GGB_EINVAL, "null annealer");
  if (composites < 0 || composites > 8 || max_swaps < 1 || max_swaps > 4096)
    return core_fail(GGB_EINVAL, "composites in [0, 8] and max_swaps in [1, 4096]");
  if (composites > 0 && !a->learned) return core_fail(GGB_EPERM, "predicted composites need a proposal filter");
  SCUDA(cudaSetDevice(a->device));
  SCUDA(cudaStreamSynchronize(a->st));
  drop_graph(a);
  if (a->comp) ggb_batch_destroy(a->comp);
  a->comp = nullptr;
  cudaFree(a->d_pred);
  a->d_pred = nullptr;
  a->C = composites;
  a->pred_max = max_swaps;
  int rc = sdev(&a->d_pred, (size_t)max_swaps);
  if (rc) return rc;
  if (a->compose_max >= 2 || a->C > 0) {
    const int nc = 1 + a->C;
    std::vector<int> nn(nc, a->N), bn(nc, a->N / a->groups), gg(nc, a->groups), dd(nc, a->d);
    if ((rc = ggb_batch_create(nc, nn.data(), bn.data(), gg.data(), dd.data(), &a->comp))) return rc;
    a->comp->stop = &a->d_state->done;
    a->comp->sticky = a->d_sticky;
    for (int k = 0; k < nc; ++k) {
      int* slot = nullptr;
      ggb_batch_adj_device(a->comp, k, &slot);
      SCUDA(cudaMemcpy(slot, a->d_adj, (size_t)a->N * a->d * sizeof(int), cudaMemcpyDeviceToDevice));
    }
  }
  return GGB_OK;
}

int ggb_sa_set_target(ggb_sa* a, int diameter, long long total) {
  if (!a) return core_fail(GGB_EINVAL, "null annealer");
  SCUDA(cudaSetDevice(a->device));
  int rc = pull_state(a);
  if (rc) return rc;
  a->h.stop_on_target = 1;
  a->h.target_diam = diameter;
  a->h.target_total = total;
  a->h.done = (a->h.cur_diam <= diameter && a->h.cur_total <= total) ? 1 : 0;
  return push_state(a);
}

int ggb_sa_autotune(ggb_sa* a, int iters, int* window_bits, int* team_ctas, double* best_ms) {
  if (!a) return core_fail(GGB_EINVAL, "null annealer");
  if (a->broken) return refuse_broken(a);
  SCUDA(cudaSetDevice(a->device));
  drop_graph(a);
  ggb_batch* b = a->cand ? a->cand : a->comp;
  if (!b) {
    if (window_bits) *window_bits = 0;
    if (team_ctas) *team_ctas = 0;
    if (best_ms) *best_ms = 0.0;
    return GGB_OK;
  }
  return ggb_batch_autotune(b, iters, window_bits, team_ctas, best_ms);
}

int ggb_sa_run(ggb_sa* a, long long steps, ggb_sa_stats* stats) {
  if (!a || steps < 0) return core_fail(GGB_EINVAL, "null annealer or negative steps");
  if (a->broken) return refuse_broken(a);
  SCUDA(cudaSetDevice(a->device));
  int rc = capture_step(a);
  if (rc) return rc;
  for (long long i = 0; i < steps; ++i) SCUDA(cudaGraphLaunch(a->exec, a->st));
  SCUDA(cudaStreamSynchronize(a->st));
  rc = check_sticky(a);
  if (rc) return rc;
  rc = pull_state(a);
  if (rc) return rc;
  if (a->h.move_error) return core_fail(GGB_ECUDA, "an accepted move did not match the current graph");
  if (stats) {
    const double pairs = (double)a->N * (a->N - 1);
    stats->step = a->h.step;
    stats->accepts = a->h.accepts;
    stats->multi_accepts = a->h.multi_accepts;
    stats->moved_swaps = a->h.moved_swaps;
    stats->pred_accepts = a->h.pred_accepts;
    stats->unevaluated = a->h.unevaluated;
    stats->delta = a->delta ? 1 : 0;
    stats->evals = a->h.evals;
    stats->cur_diam = a->h.cur_diam;
    stats->best_diam = a->h.best_diam;
    stats->cur_total = a->h.cur_total;
    stats->best_total = a->h.best_total;
    stats->cur_aspl = (double)a->h.cur_total / pairs;
    stats->best_aspl = (double)a->h.best_total / pairs;
    stats->temp = a->h.temp;
    stats->done = a->h.done;
  }
  return GGB_OK;
}

int ggb_sa_edges(ggb_sa* a, int best, int* edges) {
  if (!a || !edges) return core_fail(GGB_EINVAL, "null pointer");
  SCUDA(cudaSetDevice(a->device));
  SCUDA(cudaStreamSynchronize(a->st));
  SCUDA(cudaMemcpy(edges, best ? a->d_best_edges : a->d_edges, (size_t)2 * a->lines * sizeof(int),
                   cudaMemcpyDeviceToHost));
  return GGB_OK;
}

int ggb_sa_last_step(ggb_sa* a, float* predicted, float* label) {
  if (!a || !predicted || !label) return core_fail(GGB_EINVAL, "null pointer");
  if (!a->learned) return core_fail(GGB_EPERM, "the annealer has no proposal filter");
  SCUDA(cudaSetDevice(a->device));
  SCUDA(cudaStreamSynchronize(a->st));
  std::vector<int> sel(a->K);
  std::vector<float> sc(a->G);
  SCUDA(cudaMemcpy(sel.data(), a->d_sel, a->K * sizeof(int), cudaMemcpyDeviceToHost));
  SCUDA(cudaMemcpy(sc.data(), a->d_scores, a->G * sizeof(float), cudaMemcpyDeviceToHost));
  SCUDA(cudaMemcpy(label, a->d_labels, a->K * sizeof(float), cudaMemcpyDeviceToHost));
  for (int k = 0; k < a->K; ++k) predicted[k] = sc[sel[k]];
  return GGB_OK;
}

int ggb_sa_check_delta(ggb_sa* a, int* compared, int* mismatches, int* unevaluated, int* dense_windows) {
  using namespace ggb::sa;
  if (!a || !compared || !mismatches || !unevaluated) return core_fail(GGB_EINVAL, "null pointer");
  if (a->broken) return refuse_broken(a);
  if (!a->has_base) return core_fail(GGB_EPERM, "the annealer keeps no base for the delta evaluation");
  SCUDA(cudaSetDevice(a->device));
  int rc = pull_state(a);
  if (rc) return rc;
  if (a->h.done) return core_fail(GGB_EPERM, "the annealer has reached its target");
  // fresh candidates of the current graph, evaluated both ways
  gen_kernel<<<(a->K + 127) / 128, 128, 0, a->st>>>(a->d_state, a->d_swaps, a->K);
  rc = enqueue_delta(a, nullptr, a->st);
  if (rc) return rc;
  std::vector<int> nn(a->K, a->N), gg1(a->K, 1), dd(a->K, a->d);
  ggb_batch* full = nullptr;
  rc = ggb_batch_create(a->K, nn.data(), nn.data(), gg1.data(), dd.data(), &full);
  if (rc) return rc;
  const long long stride = full->off.size() > 1 ? full->off[1] - full->off[0] : 0;
  materialize_kernel<<<dim3(64, a->K), 256, 0, a->st>>>(a->d_state, a->d_swaps, nullptr, full->d_adj, stride);
  rc = ggb::batch_enqueue(full, a->st);
  if (!rc) rc = ggb_batch_collect(full, a->st, nullptr);
  std::vector<ggb::BatchOut> d(a->K);
  if (!rc && cudaMemcpy(d.data(), a->d_dout, a->K * sizeof(ggb::BatchOut), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = core_fail(GGB_ECUDA, "copying the delta results failed");
  int cmp = 0, bad = 0, unev = 0;
  if (!rc) {
    for (int k = 0; k < a->K; ++k) {
      const ggb::BatchOut& f = full->h_out[k];
      if (!d[k].done) { ++unev; continue; }
      ++cmp;
      const bool fc = !f.disconnected && f.diam < a->N, dc = !d[k].disconnected;
      if (fc != dc || (fc && (f.diam != d[k].diam || f.sum != d[k].sum))) ++bad;
    }
  }
  ggb_batch_destroy(full);
  if (rc) return rc;
  *compared = cmp;
  *mismatches = bad;
  *unevaluated = unev;
  if (dense_windows) SCUDA(cudaMemcpy(dense_windows, a->d_dused, sizeof(int), cudaMemcpyDeviceToHost));
  return check_sticky(a);
}

int ggb_sa_profile(ggb_sa* a, unsigned* stats) {
  if (!a || !stats) return core_fail(GGB_EINVAL, "null pointer");
  if (a->broken) return refuse_broken(a);
  SCUDA(cudaSetDevice(a->device));
  // the statistics the features read: from the base build when it makes them
  int rc = a->has_base ? enqueue_base(a, nullptr, a->st) : enqueue_profile(a, nullptr, a->st);
  if (rc) return rc;
  SCUDA(cudaStreamSynchronize(a->st));
  rc = check_sticky(a);
  if (rc) return rc;
  SCUDA(cudaMemcpy(stats, a->d_stats, (size_t)a->N * ggb::kStatLevels * sizeof(unsigned), cudaMemcpyDeviceToHost));
  return GGB_OK;
}

int ggb_sa_base_plan(const ggb_sa* a, int* team_ctas, int* teams) {
  if (!a || !team_ctas || !teams) return core_fail(GGB_EINVAL, "null pointer");
  *team_ctas = a->has_base ? a->base_T : 0;
  *teams = a->has_base ? a->base_teams : 0;
  return GGB_OK;
}

long long ggb_sa_checkpoint_bytes(const ggb_sa* a) { return a ? (long long)ckpt_bytes(a) : -1; }

int ggb_sa_checkpoint_info(const void* buf, long long bytes, int* nodes, int* degree, int* groups, int* lines) {
  if (!buf || !nodes || !degree || !groups || !lines) return core_fail(GGB_EINVAL, "null pointer");
  CkptHeader h;
  if (bytes < (long long)sizeof h) return core_fail(GGB_EINVAL, "checkpoint too short");
  std::memcpy(&h, buf, sizeof h);
  if (h.magic != kCkptMagic || h.version != kCkptVersion || h.state_bytes != (unsigned)sizeof(State))
    return core_fail(GGB_EINVAL, "not a checkpoint of this library version");
  *nodes = h.N;
  *degree = h.d;
  *groups = h.groups;
  *lines = h.lines;
  return GGB_OK;
}

int ggb_sa_checkpoint_edges(const void* buf, long long bytes, int best, int* edges) {
  int n = 0, d = 0, g = 0, lines = 0;
  int rc = ggb_sa_checkpoint_info(buf, bytes, &n, &d, &g, &lines);
  if (rc) return rc;
  if (!edges) return core_fail(GGB_EINVAL, "null pointer");
  const size_t eb = (size_t)2 * lines * sizeof(int);
  const size_t off = sizeof(CkptHeader) + sizeof(State) + (best ? eb : 0);
  if (bytes < (long long)(off + eb)) return core_fail(GGB_EINVAL, "checkpoint too short");
  std::memcpy(edges, static_cast<const unsigned char*>(buf) + off, eb);
  return GGB_OK;
}

int ggb_sa_save(ggb_sa* a, void* buf, long long bytes) {
  if (!a || !buf) return core_fail(GGB_EINVAL, "null pointer");
  if (a->broken) return refuse_broken(a);
  if (bytes < (long long)ckpt_bytes(a)) return core_fail(GGB_EINVAL, "checkpoint buffer of %lld bytes, %zu needed", bytes, ckpt_bytes(a));
  SCUDA(cudaSetDevice(a->device));
  int rc = pull_state(a);
  if (rc) return rc;
  unsigned char* p = static_cast<unsigned char*>(buf);
  const CkptHeader h = ckpt_header(a);
  std::memcpy(p, &h, sizeof h);
  p += sizeof h;
  std::memcpy(p, &a->h, sizeof(State));
  p += sizeof(State);
  const size_t eb = (size_t)2 * a->lines * sizeof(int);
  SCUDA(cudaMemcpy(p, a->d_edges, eb, cudaMemcpyDeviceToHost));
  p += eb;
  SCUDA(cudaMemcpy(p, a->d_best_edges, eb, cudaMemcpyDeviceToHost));
  p += eb;
  if (a->learned) return ggb::mlp_save_state(a->mlp, p);
  return GGB_OK;
}

int ggb_sa_restore(ggb_sa* a, const void* buf, long long bytes) {
  if (!a || !buf) return core_fail(GGB_EINVAL, "null pointer");
  if (a->broken) return refuse_broken(a);
  if (bytes < (long long)sizeof(CkptHeader)) return core_fail(GGB_EINVAL, "checkpoint too short");
  const unsigned char* p = static_cast<const unsigned char*>(buf);
  CkptHeader h;
  std::memcpy(&h, p, sizeof h);
  const CkptHeader want = ckpt_header(a);
  if (h.magic != kCkptMagic || h.version != kCkptVersion || h.state_bytes != want.state_bytes)
    return core_fail(GGB_EINVAL, "not a checkpoint of this library version");
  if (!same_config(h, want) || (h.level_cap > 0) != (want.level_cap > 0))
    return core_fail(GGB_EINVAL, "the checkpoint was written by an annealer of another configuration "
                                 "(nodes, degree, groups, candidates, proposals, composites)");
  if (h.delta != want.delta)
    return core_fail(GGB_EINVAL, "the resumed annealer evaluates candidates %s, the saved run did %s",
                     want.delta ? "against the base" : "in full", h.delta ? "against the base" : "in full");
  if (bytes < (long long)ckpt_bytes(a)) return core_fail(GGB_EINVAL, "checkpoint too short");
  p += sizeof h;
  State s;
  std::memcpy(&s, p, sizeof s);
  p += sizeof s;
  const size_t eb = (size_t)2 * a->lines * sizeof(int);
  SCUDA(cudaSetDevice(a->device));
  SCUDA(cudaStreamSynchronize(a->st));
  // the annealer must hold the checkpoint's current graph, line for line: its
  // adjacency and, with a base, its kept levels were built from it
  std::vector<int> cur((size_t)2 * a->lines);
  SCUDA(cudaMemcpy(cur.data(), a->d_edges, eb, cudaMemcpyDeviceToHost));
  if (std::memcmp(cur.data(), p, eb) != 0)
    return core_fail(GGB_EINVAL, "create the annealer from the checkpoint's current edges before restoring");
  p += eb;
  int rc;
  if (a->has_base && h.level_cap != a->level_cap && (rc = reset_level_cap(a, h.level_cap))) return rc;
  rc = pull_state(a);
  if (rc) return rc;
  if (s.cur_diam != a->h.cur_diam || s.cur_total != a->h.cur_total)
    return core_fail(GGB_EINVAL, "the checkpoint's current values differ from the evaluation of its edges");
  s.edges = a->h.edges;
  s.adj = a->h.adj;
  s.best_edges = a->h.best_edges;
  a->h = s;
  rc = push_state(a);
  if (rc) return rc;
  SCUDA(cudaMemcpy(a->d_best_edges, p, eb, cudaMemcpyHostToDevice));
  p += eb;
  if (a->learned) return ggb::mlp_load_state(a->mlp, p);
  return GGB_OK;
}

}  // extern "C"
