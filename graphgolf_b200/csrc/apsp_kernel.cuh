// apsp_kernel.cuh -- the persistent bit-parallel BFS kernel (sm_100a).
//
// One launch evaluates one graph.  The sources are cut into windows of
// W = 128*R bits; a window keeps two bitset matrices S_cur and S_prev of
// nodes x W bits, small enough to stay resident in the 126 MB L2 while the
// window runs.  Every level is one sweep of all CTAs over all vertices:
//
//     S_next[v] = S_prev[v] | OR_{j<d} S_cur[adj[v][j]]          (*)
//
// which is the reference's recurrence B |= A[adj]; swap(A,B)
// (general/evaluation.c:175-181,194-197, grid/evaluation.c:143-151).  The
// popcount of S_next is reduced in the same sweep (warp shuffles, one 64-bit
// atomic per CTA), and after a bounded-spin grid barrier every CTA reads the
// level's count and takes the same decision the reference takes on the host:
// stop when all (vertex, source) pairs are reached (:192), else add the
// unreached pairs times the group weight to the sum (:199-200).
//
// A window also stops when a level adds no bit at all.  (*) makes every
// per-source set monotone, and a level that adds nothing is a fixed point, so
// the reference would run on to kk == nodes and report a disconnected graph;
// stopping there gives the identical answer without the N-level walk.
//
// Bitset rows are read with ld.global.cg (L2, no L1 allocation): rows written
// by other SMs in the previous level must never be served from a stale L1
// line, and random gathers get no L1 reuse anyway.  The adjacency is
// read-only for the whole launch and goes through the read-only path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ggb {

constexpr int kThreads = 512;         // threads per CTA
constexpr int kWarps = kThreads / 32;

// Error codes written to ApspCtrl::error (host maps them to GGB_E*).
enum : int { kErrNone = 0, kErrAdj = 1, kErrTimeout = 2, kErrPerm = 3 };

// Device-side control block.  Zeroed by the host before every launch.
struct ApspCtrl {
  unsigned long long bar;         // grid-barrier arrivals (monotone)
  unsigned long long cnt[2][2];   // [level parity][lo rows, hi rows] cumulative popcounts
  int error;                      // first error code
  int error_info;                 // e.g. the offending vertex
  // outputs (written by CTA 0, thread 0, at the end)
  int diam;                       // max over windows of kk+1; nodes+1 if disconnected
  int disconnected;
  long long sum;                  // Σ weighted unreached pairs (before + N(N-1))
  long long levels;               // levels executed over all windows
  int windows;
  int done;                       // 1 once the outputs are written
};

struct ApspArgs {
  const int* adj;        // [N][d], device, rows already relabelled (grid)
  uint4* buf0;           // [N][R]
  uint4* buf1;           // [N][R]
  ApspCtrl* ctrl;
  long long timeout_ns;  // bound on every grid-barrier wait
  int N, d;
  int n_src1;            // phase-1 sources: rows 0 .. n_src1-1 (based_nodes)
  int split;             // rows < split are "lo" (based_nodes*groups)
  int ac;                // added centres: phase-2 sources are rows N-ac .. N-1
  int groups;
  int win_first, win_stride;   // this rank's windows: t = win_first + k*win_stride
  int phantom;           // extra arrivals every barrier waits for: 0 in normal use; the
                         // fault-path test sets 1 so that every bounded wait runs out
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_volatile_i32(const int* p) {
  return *reinterpret_cast<const volatile int*>(p);
}

__device__ __forceinline__ void set_error(ApspCtrl* c, int code, int info) {
  if (atomicCAS(&c->error, 0, code) == 0) atomicExch(&c->error_info, info);
}

// Grid barrier with a time bound.  Every CTA calls it the same number of
// times (all control flow below is decided from values every CTA reads after
// the previous barrier).  Returns false if the wait ran out or another CTA
// reported an error; the caller then leaves the kernel.
__device__ __forceinline__ bool grid_barrier(ApspCtrl* c, unsigned long long target, long long timeout_ns,
                                             int* s_flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&c->bar, 1ULL);
    int ok = 1;
    if (ld_acquire_u64(&c->bar) < target) {
      const unsigned long long t0 = globaltimer_ns();
      while (ld_acquire_u64(&c->bar) < target) {
        if (ld_volatile_i32(&c->error) != 0) { ok = 0; break; }
        if ((long long)(globaltimer_ns() - t0) > timeout_ns) {
          set_error(c, kErrTimeout, (int)blockIdx.x);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    *s_flag = ok;
  }
  __syncthreads();
  return *s_flag != 0;
}

__device__ __forceinline__ uint4 ld_cg(const uint4* p) { return __ldcg(p); }
__device__ __forceinline__ void st_cg(uint4* p, const uint4& v) { __stcg(p, v); }

__device__ __forceinline__ void or_into(uint4& a, const uint4& b) {
  a.x |= b.x; a.y |= b.y; a.z |= b.z; a.w |= b.w;
}
__device__ __forceinline__ unsigned popc4(const uint4& a) {
  return __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w);
}

// R = uint4 words per row (W = 128*R source bits).  LPR lanes share a row,
// each lane owning UPL uint4 of it; a warp covers VPW vertices per step.
template <int R>
__global__ void __launch_bounds__(kThreads, 2) apsp_persistent_kernel(const ApspArgs a) {
  constexpr int LPR = R >= 32 ? 32 : R;
  constexpr int VPW = 32 / LPR;
  constexpr int UPL = R / LPR;
  constexpr int W = 128 * R;
  constexpr int U = UPL >= 2 ? 2 : 8;  // neighbour rows in flight per thread

  __shared__ unsigned long long s_red[kWarps][2];
  __shared__ unsigned long long s_cnt[2];
  __shared__ int s_flag;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sub = lane / LPR;          // which vertex of the warp's VPW
  const int li = lane % LPR;           // lane within the row
  const long long slot = ((long long)blockIdx.x * kWarps + warp) * VPW + sub;
  const long long n_slots = (long long)gridDim.x * kWarps * VPW;
  const int N = a.N, d = a.d;
  const unsigned grid = gridDim.x;

  unsigned long long bar_target = 0;
  unsigned long long seen[2][2] = {{0ULL, 0ULL}, {0ULL, 0ULL}};
  unsigned gl = 0;                     // global level counter (parity selects cnt slot)
  long long sum = 0, levels = 0;
  int diam = 1, disconnected = 0, windows = 0;
  bool adj_ok = true;

  for (int phase = 1; phase <= 2 && !disconnected; ++phase) {
    const int nsrc = phase == 1 ? a.n_src1 : a.ac;
    if (nsrc <= 0) continue;
    const int row0 = phase == 1 ? 0 : N - a.ac;
    const int nwin = (nsrc + W - 1) / W;
    for (int t = a.win_first; t < nwin && !disconnected; t += a.win_stride) {
      const int first = t * W;
      const int l = min(W, nsrc - first);
      const long long lo_rows = a.split, hi_rows = (long long)N - a.split;
      ++windows;

      // Window start: both matrices hold the identity (reference :168-172):
      // bit i of row row0+first+i for i < l, every other bit zero.
      for (long long v = slot; v < N; v += n_slots) {
        const long long bit = v - row0 - first;
#pragma unroll
        for (int k = 0; k < UPL; ++k) {
          const int col = li + k * LPR;      // uint4 index within the row
          uint4 x = make_uint4(0u, 0u, 0u, 0u);
          if (bit >= 0 && bit < l && (int)(bit >> 7) == col) {
            const unsigned b = (unsigned)(bit & 127);
            const unsigned m = 1u << (b & 31);
            if ((b >> 5) == 0) x.x = m; else if ((b >> 5) == 1) x.y = m;
            else if ((b >> 5) == 2) x.z = m; else x.w = m;
          }
          st_cg(a.buf0 + v * R + col, x);
          st_cg(a.buf1 + v * R + col, x);
        }
      }
      bar_target += grid;
      if (!grid_barrier(a.ctrl, bar_target + a.phantom, a.timeout_ns, &s_flag)) return;

      long long prev_total = l;   // popcount of the identity
      long long kk;
      for (kk = 0; kk < N; ++kk) {
        const uint4* __restrict__ src = (kk & 1) ? a.buf1 : a.buf0;
        uint4* __restrict__ dst = (kk & 1) ? a.buf0 : a.buf1;
        unsigned c_lo = 0, c_hi = 0;
        for (long long v = slot; v < N; v += n_slots) {
          const int* arow = a.adj + v * d;
          uint4 acc[UPL];
#pragma unroll
          for (int k = 0; k < UPL; ++k) acc[k] = ld_cg(dst + v * R + li + k * LPR);
          int j = 0;
          for (; j + U <= d; j += U) {
            int u[U];
#pragma unroll
            for (int q = 0; q < U; ++q) u[q] = __ldg(arow + j + q);
#pragma unroll
            for (int q = 0; q < U; ++q) {
              if ((unsigned)u[q] >= (unsigned)N) { adj_ok = false; u[q] = 0; }
            }
            uint4 x[U][UPL];
#pragma unroll
            for (int q = 0; q < U; ++q)
#pragma unroll
              for (int k = 0; k < UPL; ++k) x[q][k] = ld_cg(src + (long long)u[q] * R + li + k * LPR);
#pragma unroll
            for (int q = 0; q < U; ++q)
#pragma unroll
              for (int k = 0; k < UPL; ++k) or_into(acc[k], x[q][k]);
          }
          for (; j < d; ++j) {
            int u = __ldg(arow + j);
            if ((unsigned)u >= (unsigned)N) { adj_ok = false; u = 0; }
#pragma unroll
            for (int k = 0; k < UPL; ++k) or_into(acc[k], ld_cg(src + (long long)u * R + li + k * LPR));
          }
          unsigned c = 0;
#pragma unroll
          for (int k = 0; k < UPL; ++k) {
            st_cg(dst + v * R + li + k * LPR, acc[k]);
            c += popc4(acc[k]);
          }
          if (v < a.split) c_lo += c; else c_hi += c;
        }
        if (!adj_ok) set_error(a.ctrl, kErrAdj, (int)blockIdx.x);

        // CTA reduction of the level's popcounts, one atomic per CTA.
        unsigned long long r_lo = c_lo, r_hi = c_hi;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          r_lo += __shfl_xor_sync(0xffffffffu, r_lo, o);
          r_hi += __shfl_xor_sync(0xffffffffu, r_hi, o);
        }
        if (lane == 0) { s_red[warp][0] = r_lo; s_red[warp][1] = r_hi; }
        __syncthreads();
        if (threadIdx.x == 0) {
          unsigned long long b_lo = 0, b_hi = 0;
#pragma unroll
          for (int w = 0; w < kWarps; ++w) { b_lo += s_red[w][0]; b_hi += s_red[w][1]; }
          if (b_lo) atomicAdd(&a.ctrl->cnt[gl & 1][0], b_lo);
          if (b_hi) atomicAdd(&a.ctrl->cnt[gl & 1][1], b_hi);
        }
        bar_target += grid;
        if (!grid_barrier(a.ctrl, bar_target + a.phantom, a.timeout_ns, &s_flag)) return;
        if (threadIdx.x == 0) {
          s_cnt[0] = ld_acquire_u64(&a.ctrl->cnt[gl & 1][0]);
          s_cnt[1] = ld_acquire_u64(&a.ctrl->cnt[gl & 1][1]);
        }
        __syncthreads();
        const unsigned long long now_lo = s_cnt[0], now_hi = s_cnt[1];
        __syncthreads();   // s_cnt is rewritten after the next barrier only
        const long long lvl_lo = (long long)(now_lo - seen[gl & 1][0]);
        const long long lvl_hi = (long long)(now_hi - seen[gl & 1][1]);
        seen[gl & 1][0] = now_lo;
        seen[gl & 1][1] = now_hi;
        ++gl;
        ++levels;
        if (ld_volatile_i32(&a.ctrl->error) != 0) return;   // same answer in every CTA after the barrier

        const long long total = lvl_lo + lvl_hi;
        const bool full = phase == 1 ? (total == (long long)N * l) : (lvl_hi == hi_rows * l);
        if (full) break;
        if (total == prev_total) { disconnected = 1; break; }
        if (phase == 1) {
          sum += (lo_rows * l - lvl_lo) * a.groups;
          sum += (hi_rows * l - lvl_hi) * 2LL * a.groups;
        } else {
          sum += hi_rows * l - lvl_hi;
        }
        prev_total = total;
      }
      if (disconnected) diam = N + 1;
      else if (kk + 1 > diam) diam = (int)(kk + 1);
    }
  }

  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ApspCtrl* c = a.ctrl;
    c->diam = diam;
    c->disconnected = disconnected;
    c->sum = sum;
    c->levels = levels;
    c->windows = windows;
    __threadfence();
    c->done = 1;
  }
}

// Grid relabel (grid/evaluation.c:148-151): row rotate_hash[i] of the
// relabelled adjacency holds rotate_hash[adj[i][j]].  inv[] must be -1 on
// entry; it receives the inverse permutation so a second kernel can verify
// that rotate_hash is a bijection.
__global__ void relabel_adjacency_kernel(const int* __restrict__ adj, const int* __restrict__ rh,
                                         int* __restrict__ out, int* __restrict__ inv, int N, int d,
                                         ApspCtrl* ctrl) {
  const long long n = (long long)N * d;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / d), j = (int)(e % d);
    const int r = rh[i];
    const int nb = adj[e];
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

__global__ void check_permutation_kernel(const int* __restrict__ inv, int N, ApspCtrl* ctrl) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
       i += (long long)gridDim.x * blockDim.x)
    if (inv[i] < 0) set_error(ctrl, kErrPerm, (int)i);
}

}  // namespace ggb
