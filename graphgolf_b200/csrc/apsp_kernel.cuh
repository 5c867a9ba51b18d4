// apsp_kernel.cuh -- the bit-parallel BFS kernels (sm_100a).
//
// One evaluation = (optionally) one ball pre-pass kernel + one persistent
// cooperative kernel.  The sources are cut into windows of W = 128*R bits; a
// window keeps two bitset matrices of nodes x W bits, small enough to stay
// resident in the 126 MB L2 while the window runs.  Every dense level is one
// sweep of all CTAs over all vertices:
//
//     S_{k+1}[v] = S_k[v] | OR_{j<d} S_k[adj[v][j]]                      (*)
//
// The reference's recurrence is S_{k+1}[v] = S_{k-1}[v] | OR_j S_k[adj[v][j]]
// (B |= A[adj]; swap(A,B), general/evaluation.c:175-181,194-197,
// grid/evaluation.c:143-151).  Both give the same sets for ANY adjacency:
// the reference's sets are monotone (S_{k-1} <= S_k, by induction from
// S_{-1} = S_0 = identity), so S_{k-1}[v] <= S_k[v], and
// S_k[v] = S_{k-2}[v] | OR_j S_{k-1}[u_j] <= S_{k-1}[v] | OR_j S_k[u_j].
// Using S_k[v] makes the destination matrix write-only.
//
// The popcount of S_{k+1} is reduced in the same sweep (warp shuffles, one
// 64-bit atomic per CTA), and after a bounded-spin grid barrier every CTA
// reads the level's count and takes the decision the reference takes on the
// host: stop when all (vertex, source) pairs are reached (:192), else add the
// unreached pairs times the group weight to the sum (:199-200).  A window also
// stops when a level adds no bit at all: the sets are monotone, a level that
// adds nothing is a fixed point, and the reference would run on to
// kk == nodes and report a disconnected graph -- the identical answer.
//
// The first levels of a window are not swept.  Either
//  - the ball pre-pass (ball_kernel) has written S_3 of every window into a
//    window-major matrix in HBM together with the exact counts of S_1..S_3,
//    and dense sweeps start at S_4; or
//  - the window's first step builds S_2 directly from the two-hop adjacency
//    (seed_window) and dense sweeps start at S_3.
//
// Bitset rows are read with ld.global.cg (L2, no L1 allocation): rows written
// by other SMs in the previous level must never be served from a stale L1
// line, and random gathers get no L1 reuse anyway.  The adjacency is
// read-only for the whole launch and goes through the read-only path.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ggb {

constexpr int kThreads = 512;         // threads per CTA (one CTA per SM, up to 128 registers per thread)
constexpr int kWarps = kThreads / 32;
constexpr int kBallThreads = 256;     // threads per CTA of the ball pre-pass
constexpr int kBallMaxWindows = 32;   // windows of one rank in the ball pre-pass (one per lane)
constexpr int kBallMaxDegree = 32;
constexpr int kStatLevels = 32;       // levels the per-vertex statistics keep (profile kernel)

// Error codes written to ApspCtrl::error (host maps them to GGB_E*).
enum : int { kErrNone = 0, kErrAdj = 1, kErrTimeout = 2, kErrPerm = 3, kErrDegree = 4 };

// Device-side control block.  Zeroed by the host before every launch.
struct ApspCtrl {
  unsigned long long bar;         // grid-barrier arrivals (monotone)
  unsigned long long cnt[4][2];   // [level mod 4][lo rows, hi rows] cumulative popcounts
  int error;                      // first error code
  int error_info;                 // e.g. the offending vertex
  // outputs (written by CTA 0, thread 0, at the end)
  int diam;                       // max over windows of kk+1; nodes+1 if disconnected
  int disconnected;
  long long sum;                  // Σ weighted unreached pairs (before + N(N-1))
  long long levels;               // levels executed over all windows
  long long dense_levels;         // of which dense OR-gather sweeps
  int windows;
  int trace_len;                  // trace pairs written
  int done;                       // 1 once the outputs are written
};

struct ApspArgs {
  const int* adj;        // [N][d], device, rows already relabelled (grid)
  const int* adj2;       // rows the added-centre phase gathers, or null for adj; the non-regular
                         // evaluators gather padded rows in phase 1 but whole rows here
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
  int vec4;              // 1: degree % 4 == 0 and adj 16-byte aligned (vector adjacency loads)
  const uint4* ball;     // phase-1 S_3 rows, [local window][N][R], or null (two-hop seeding)
  const unsigned long long* ball_cnt;  // [local window][3][lo, hi]: counts of S_1 and S_2 (slot 2 unused)
  long long* trace;      // optional: (globaltimer ns, tag) pairs written by CTA 0 after every barrier
  int trace_cap;         // pairs available in trace
  int phantom;           // extra arrivals every barrier waits for: 0 in normal use; the
                         // fault-path test sets 1 so that every bounded wait runs out
  unsigned* stats;       // profile kernel only: [N][kStatLevels] unreached sources per level
  // base builds only (null otherwise): every level's rows of window t at
  // levels + (t * (level_cap + 1) + k) * N * R for k <= level_cap, the
  // level's popcount at level_counts[t * (level_cap + 1) + k], and the
  // window's completion level (first k with S_k full; -1 if it stalls) at
  // win_levels[t]
  uint4* levels;
  long long* level_counts;
  int* win_levels;
  int level_cap;
  // Sources per window when narrower than the rows: 64 runs 64-source windows
  // (the reference's one-word chunk, general/evaluation.cu:27-44) on rows of
  // one uint4 whose upper 64 bits stay zero.  0: W = 128 * R.
  int win_bits = 0;
  // The skipping sweep runs once the gathered level is at least this full
  // (per mille of N * sources).
  int skip_permille = 900;
  // Optional full-row stamps, one per vertex, zeroed before the launch:
  // stamp = (window id << 8) | L records that the vertex's row of that window
  // is full from level L on.  The window id is stamp_base + t + 1 for window
  // t, unique among the windows that share the stamps in one launch (the
  // batch kernel advances stamp_base from one graph of a team to the next).
  // The sweeps that set and read them are described at sweep_stamped.
  unsigned* stamps = nullptr;
  unsigned stamp_base = 0;
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
// 32 bytes (two adjacent uint4, 32-byte aligned) in one L2-cached access
__device__ __forceinline__ void ld_cg2(const uint4* p, uint4 (&v)[2]) {
  asm volatile("ld.global.cg.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0].x), "=r"(v[0].y), "=r"(v[0].z), "=r"(v[0].w), "=r"(v[1].x), "=r"(v[1].y), "=r"(v[1].z),
                 "=r"(v[1].w)
               : "l"(p));
}
__device__ __forceinline__ void st_cg2(uint4* p, const uint4 (&v)[2]) {
  asm volatile("st.global.cg.v8.u32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(v[0].x), "r"(v[0].y),
               "r"(v[0].z), "r"(v[0].w), "r"(v[1].x), "r"(v[1].y), "r"(v[1].z), "r"(v[1].w)
               : "memory");
}

__device__ __forceinline__ void or_into(uint4& a, const uint4& b) {
  a.x |= b.x; a.y |= b.y; a.z |= b.z; a.w |= b.w;
}
__device__ __forceinline__ unsigned popc4(const uint4& a) {
  return __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w);
}

// Popcount bookkeeping of one BFS level, identical in every CTA: returns 1
// when the window is complete (reference :192), 2 when the level added no bit
// (a fixed point: the reference would report a disconnected graph), else adds
// the unreached pairs to the sum (:199-200) and returns 0.
__device__ __forceinline__ int level_decision(int phase, long long lvl_lo, long long lvl_hi, long long l,
                                              long long N, long long lo_rows, long long hi_rows, long long groups,
                                              long long& prev_total, long long& sum) {
  const long long total = lvl_lo + lvl_hi;
  const bool full = phase == 1 ? (total == N * l) : (lvl_hi == hi_rows * l);
  if (full) return 1;
  if (total == prev_total) return 2;
  if (phase == 1) {
    sum += (lo_rows * l - lvl_lo) * groups;
    sum += (hi_rows * l - lvl_hi) * 2 * groups;
  } else {
    sum += hi_rows * l - lvl_hi;
  }
  prev_total = total;
  return 0;
}

// Trace record after a barrier (CTA 0, thread 0 only; no-op without a buffer).
// tag: 1 = seeding of a window done, 2 = dense sweep done; the level kk is
// stored above the tag byte.
__device__ __forceinline__ void trace_mark(const ApspArgs& a, int& n, int tag, long long kk) {
  if (a.trace && blockIdx.x == 0 && threadIdx.x == 0 && n < a.trace_cap) {
    a.trace[2 * n] = (long long)globaltimer_ns();
    a.trace[2 * n + 1] = (kk << 8) | tag;
    ++n;
  }
}

// Sums NV per-thread counters over the CTA; thread 0 adds value i to
// ctrl->cnt[(g0 + i/2) & 3][i & 1] (lo/hi counts of one or two levels).
template <int NV>
__device__ __forceinline__ void cta_add_counts(const unsigned* c, ApspCtrl* ctrl, unsigned g0,
                                               unsigned long long (*s_red)[4]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long r[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i) r[i] = c[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int i = 0; i < NV; ++i) r[i] += __shfl_xor_sync(0xffffffffu, r[i], o);
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) s_red[warp][i] = r[i];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      unsigned long long b = 0;
      for (int w = 0; w < kWarps; ++w) b += s_red[w][i];
      if (b) atomicAdd(&ctrl->cnt[(g0 + i / 2) & 3][i & 1], b);
    }
  }
}

// After the barrier that ends `nl` levels (1 or 2), thread 0 reads their
// cumulative counts, turns them into per-level counts with the values it saw
// last time, and publishes them in s_lvl[0..2*nl).  Every CTA reads the same
// counter values (no CTA can add to these slots again before all CTAs have
// passed the next barrier), so all take identical decisions.
__device__ __forceinline__ void read_level_counts(ApspCtrl* ctrl, unsigned g0, int nl,
                                                  unsigned long long (*s_seen)[2], long long* s_lvl) {
  if (threadIdx.x == 0) {
    for (int i = 0; i < nl; ++i) {
      const unsigned slot = (g0 + i) & 3;
      const unsigned long long lo = ld_acquire_u64(&ctrl->cnt[slot][0]);
      const unsigned long long hi = ld_acquire_u64(&ctrl->cnt[slot][1]);
      s_lvl[2 * i] = (long long)(lo - s_seen[slot][0]);
      s_lvl[2 * i + 1] = (long long)(hi - s_seen[slot][1]);
      s_seen[slot][0] = lo;
      s_seen[slot][1] = hi;
    }
  }
  __syncthreads();
}

// ---- adjacency loads ---------------------------------------------------------
template <int VEC> struct AdjVec;
template <> struct AdjVec<1> {
  int v;
  __device__ __forceinline__ void load(const int* p) { v = __ldg(p); }
  __device__ __forceinline__ void fill(int x) { v = x; }
  __device__ __forceinline__ int at(int) const { return v; }
};
template <> struct AdjVec<4> {
  int4 v;
  __device__ __forceinline__ void load(const int* p) { v = __ldg(reinterpret_cast<const int4*>(p)); }
  __device__ __forceinline__ void fill(int x) { v = make_int4(x, x, x, x); }
  __device__ __forceinline__ int at(int i) const { return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w; }
};

// OR `v` into a 32-bit word of shared memory with a shared-space reduction
// (the pointer is turned into a shared-window address, so the compiler can
// never fall back to a generic atomic).
__device__ __forceinline__ void smem_or(unsigned* p, unsigned v) {
  const unsigned addr = (unsigned)__cvta_generic_to_shared(p);
  asm volatile("red.shared.or.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

// OR `v` into a shared word and return the previous value.
__device__ __forceinline__ unsigned smem_or_old(unsigned* p, unsigned v) {
  const unsigned addr = (unsigned)__cvta_generic_to_shared(p);
  unsigned old;
  asm volatile("atom.shared.or.b32 %0, [%1], %2;" : "=r"(old) : "r"(addr), "r"(v) : "memory");
  return old;
}

__device__ __forceinline__ void set_bit_in(unsigned* row, int x, int base, int nbits) {
  const unsigned b = (unsigned)(x - base);
  if (b < (unsigned)nbits) smem_or(row + (b >> 5), 1u << (b & 31));
}

// Sets, in `row`, bit (x - base) of every entry x of the `nrows` adjacency
// rows whose ids are ids[0..nrows) when 0 <= x - base < nbits (row ids are
// checked against N; an entry outside [0, N) clears adj_ok).  The G lanes of
// a group split each row into its d/VEC vectors: when a row has at most G
// vectors, lane r always loads vector r % per of rows r / per, r / per + G/per,
// ... so a lane's loads follow a fixed pattern with no division in the loop;
// longer rows are taken one at a time.  Up to 8 loads are in flight per lane
// and the bit sets are predicated, not branched.  With out_ids, entry e of
// row j is also stored at out_ids[j*d + e] (-1 for an invalid row id).
// The warp's count of newly set bits by window, in shared memory (one
// counter per window, shared atomics: only the d + d^2 bits of the first two
// steps are counted, and a per-lane array would cost the occupancy of a CTA
// per SM).  Bit b lies in global window b >> log2w; only this rank's windows
// (first, first + stride, ...) are counted.
struct NewBitCount {
  unsigned* col;
  int log2w, first, stride, nwin;
  __device__ __forceinline__ void add(unsigned b) const {
    int k = (int)(b >> log2w) - first;
    if (k < 0) return;
    if (stride != 1) {
      if (k % stride) return;
      k /= stride;
    }
    if (k < nwin) atomicAdd(col + k, 1u);
  }
};

__device__ __forceinline__ void set_bit_counted(unsigned* row, unsigned b, const NewBitCount* nbc) {
  const unsigned m = 1u << (b & 31);
  if (nbc) {
    if (!(smem_or_old(row + (b >> 5), m) & m)) nbc->add(b);
  } else {
    smem_or(row + (b >> 5), m);
  }
}

template <int VEC, int G>
__device__ __forceinline__ void set_rows_bits(const int* __restrict__ adj, int N, int d, const int* ids, int nrows,
                                              unsigned* row, int base, int nbits, int r, bool& adj_ok,
                                              int* out_ids, const NewBitCount* nbc = nullptr) {
  const int per = d / VEC;
  bool bad = false;
  if (per <= G) {
    const int rpi = G / per;                 // rows per group step
    const bool active = r < rpi * per;
    const int roff = r / per, part = r - roff * per;
    for (int r0 = 0; r0 < nrows; r0 += rpi * 8) {
      AdjVec<VEC> val[8];
      bool ok[8];
      int pos[8];
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const int j = r0 + t * rpi + roff;
        const bool in = active && j < nrows;
        const int u = in ? ids[j] : -1;
        ok[t] = in && (unsigned)u < (unsigned)N;
        pos[t] = in ? j * d + part * VEC : -1;
        if (ok[t]) val[t].load(adj + (long long)u * d + part * VEC);
      }
#pragma unroll
      for (int t = 0; t < 8; ++t) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
          const int x = ok[t] ? val[t].at(e) : -1;
          if (out_ids && pos[t] >= 0) out_ids[pos[t] + e] = x;
          bad |= ok[t] && (unsigned)x >= (unsigned)N;
          const unsigned b = (unsigned)(x - base);
          if (ok[t] && b < (unsigned)nbits) set_bit_counted(row, b, nbc);
        }
      }
    }
  } else {
    for (int j = 0; j < nrows; ++j) {
      const int u = ids[j];
      const bool okr = (unsigned)u < (unsigned)N;
      for (int p0 = 0; p0 < per; p0 += G * 8) {
        AdjVec<VEC> val[8];
        bool ok[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const int part = p0 + t * G + r;
          ok[t] = okr && part < per;
          if (ok[t]) val[t].load(adj + (long long)u * d + part * VEC);
          if (out_ids && !okr && part < per)
#pragma unroll
            for (int e = 0; e < VEC; ++e) out_ids[j * d + part * VEC + e] = -1;
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) {
          const int part = p0 + t * G + r;
#pragma unroll
          for (int e = 0; e < VEC; ++e) {
            const int x = ok[t] ? val[t].at(e) : -1;
            if (out_ids && ok[t]) out_ids[j * d + part * VEC + e] = x;
            bad |= ok[t] && (unsigned)x >= (unsigned)N;
            const unsigned b = (unsigned)(x - base);
            if (ok[t] && b < (unsigned)nbits) set_bit_counted(row, b, nbc);
          }
        }
      }
    }
  }
  if (bad) adj_ok = false;
}

// ---- per-window seeding: S_2 from the two-hop adjacency ----------------------
constexpr int kSeedGroup = 8;                    // lanes per vertex
constexpr int kSeedVerts = 32 / kSeedGroup;      // vertices per warp and step
constexpr int kSeedNb = 64;                      // neighbour ids staged per vertex and pass

// Builds S_1 (counted only) and S_2 (-> s2_out) rows of every vertex for the
// window whose bit 0 is vertex `base`, counting their bits into c[4] (S_1
// lo/hi, S_2 lo/hi):  S_1[v] = {v} u adj[v][*] and
// S_2[v] = S_1[v] u U_j adj[u_j][*] restricted to the window, which is (*)
// applied twice to the identity.  A warp takes 4 vertices per step, 8 lanes
// each: the lanes stage the vertex's neighbour ids in shared memory, set the
// bits of v and its neighbours, then load the neighbours' adjacency rows and
// set the bits of every two-hop vertex; the warp then writes the 4 S_2 rows
// out coalesced.  Replaces the reference's clear + identity set-up (:168-172)
// and its first two OR-gather sweeps.
template <int R, int VEC, bool STATS = false>
__device__ __forceinline__ void seed_window(const ApspArgs& a, const int* __restrict__ adj, int base, int l,
                                            uint4* s2_out, int* s_nb,
                                            unsigned* s_rw, unsigned (&c)[4], bool& adj_ok, long long warp_id,
                                            long long n_warps, uint4* s1_out = nullptr) {
  constexpr int SROW = 4 * R;
  const int N = a.N, d = a.d;
  const int lane = threadIdx.x & 31, g = lane / kSeedGroup, r = lane % kSeedGroup;
  uint4* const rows4 = reinterpret_cast<uint4*>(s_rw);
  int* const nb = s_nb + g * kSeedNb;
  unsigned* const s1 = s_rw + (2 * g) * SROW;
  unsigned* const s2 = s1 + SROW;
  for (long long v0 = warp_id * kSeedVerts; v0 < N; v0 += n_warps * kSeedVerts) {
    for (int i = lane; i < 2 * kSeedVerts * R; i += 32) rows4[i] = make_uint4(0u, 0u, 0u, 0u);
    const long long v = v0 + g;
    const bool live = v < N;
    __syncwarp();   // rows zeroed before any bit is set
    if (live && r == 0) set_bit_in(s1, (int)v, base, l);
    for (int jb = 0; jb < d; jb += kSeedNb) {
      const int dc = min(kSeedNb, d - jb);
      __syncwarp();
      if (live)
        for (int j = r; j < dc; j += kSeedGroup) nb[j] = __ldg(adj + v * d + jb + j);
      __syncwarp();
      if (!live) continue;
      for (int j = r; j < dc; j += kSeedGroup) {
        const int x = nb[j];
        if ((unsigned)x >= (unsigned)N) { adj_ok = false; continue; }
        set_bit_in(s1, x, base, l);
      }
      set_rows_bits<VEC, kSeedGroup>(adj, N, d, nb, dc, s2, base, l, r, adj_ok, nullptr);
    }
    __syncwarp();
#pragma unroll
    for (int i = 0; i < kSeedVerts; ++i) {
      const long long vi = v0 + i;
      if (vi >= N) break;
      unsigned c1 = 0, c2 = 0;
      for (int col = lane; col < R; col += 32) {
        const uint4 x1 = rows4[(2 * i) * R + col];
        uint4 x2 = rows4[(2 * i + 1) * R + col];
        or_into(x2, x1);   // S_2 includes S_1
        st_cg(s2_out + vi * R + col, x2);
        if (s1_out) st_cg(s1_out + vi * R + col, x1);
        c1 += popc4(x1);
        c2 += popc4(x2);
      }
      if (vi < a.split) { c[0] += c1; c[2] += c2; } else { c[1] += c1; c[3] += c2; }
      if constexpr (STATS) {
        const unsigned t1 = __reduce_add_sync(0xffffffffu, c1), t2 = __reduce_add_sync(0xffffffffu, c2);
        if (lane == 0) {
          unsigned* st = a.stats + vi * kStatLevels;
          atomicAdd(st + 0, (unsigned)l - ((unsigned)(vi - base) < (unsigned)l ? 1u : 0u));
          atomicAdd(st + 1, (unsigned)l - t1);
          atomicAdd(st + 2, (unsigned)l - t2);
        }
      }
    }
    __syncwarp();
  }
}

// The ball's last step: OR into `row` the bit of every entry below nbits of
// the rows ids[0..nrows), d / VEC <= 32 lanes a row, 8 loads in flight per
// lane.  A row id outside [0, N) is skipped and so is an entry outside
// [0, nbits); neither is reported here, because the ball's first step reads
// every row of the adjacency and reports any entry outside [0, N).  One
// compare, two shifts, an add and the shared reduction per entry.
template <int VEC>
__device__ __forceinline__ void scatter_plain(const int* __restrict__ adj, int N, int d, const int* ids, int nrows,
                                              unsigned* row, int nbits, int lane) {
  const unsigned rs = (unsigned)__cvta_generic_to_shared(row);
  const int per = d / VEC;
  const int rpi = 32 / per;
  const int roff = lane / per, part = lane - roff * per;
  const bool active = roff < rpi;
  for (int r0 = 0; r0 < nrows; r0 += rpi * 8) {
    AdjVec<VEC> val[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      const int j = r0 + t * rpi + roff;
      const int u = (active && j < nrows) ? ids[j] : -1;
      if ((unsigned)u < (unsigned)N) val[t].load(adj + (long long)u * d + part * VEC);
      else val[t].fill(-1);
    }
#pragma unroll
    for (int t = 0; t < 8; ++t)
#pragma unroll
      for (int e = 0; e < VEC; ++e) {
        const unsigned x = (unsigned)val[t].at(e);
        if (x < (unsigned)nbits)
          asm volatile("red.shared.or.b32 [%0], %1;" ::"r"(rs + ((x >> 5) << 2)), "r"(1u << (x & 31)) : "memory");
      }
  }
}

// ---- the ball pre-pass: S_3 of every window at once --------------------------
//
// One warp per vertex v builds, in shared memory, the row of all phase-1
// sources within three applications of (*) from v:
//     S_1[v] = {v} u N(v),  S_2[v] = S_1[v] u N(N(v)),  S_3[v] = S_2[v] u N(N(N(v)))
// (N(x) = adj[x][*]; exact for any adjacency), counting after each step the
// bits that fall into every window of this rank, and finally writes the S_3
// segment of every window to ball[local window][v].  That is 1 + d + d^2 + d^3
// adjacency entries per vertex read once per evaluation, instead of the two
// seeding steps and the first dense sweep of every window.
struct BallArgs {
  const int* adj;
  uint4* ball;                    // [local windows][N][R]
  unsigned long long* cnt;        // [local windows][3][2], zeroed by the host
  ApspCtrl* ctrl;                 // error reporting
  int N, d, n_src, split;
  int R;                          // uint4 per window row
  int win_first, win_stride, n_local;
};

// uint4 of one full ball row (all phase-1 sources), padded to a multiple of 4.
__host__ __device__ __forceinline__ int ball_row_u4(int n_src) { return ((n_src + 127) / 128 + 3) / 4 * 4; }

// Shared memory of one warp of ball_kernel, in uint4: the full row, the one-
// and two-hop neighbour ids (d + d^2 ints, padded) and the warp's new-bit
// counters of S_1 and S_2 for nwin windows.
__host__ __device__ __forceinline__ int ball_warp_u4(int n_src, int d, int nwin) {
  return ball_row_u4(n_src) + (d + d * d + 3) / 4 + (2 * nwin + 3) / 4;
}

// The ball pre-pass runs only without added centres (every row is a "lo"
// row) and with at most 32 windows per rank.  It writes the counts of S_1
// and S_2 per window (counted exactly, as new bits, while they are set); the
// count of S_3 is taken by the window's first dense sweep, which reads every
// S_3 row anyway.
template <int VEC>
__global__ void __launch_bounds__(kBallThreads, 3) ball_kernel(const BallArgs b) {
  extern __shared__ uint4 s_ball[];
  constexpr int kWarpsB = kBallThreads / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int N = b.N, d = b.d, R = b.R;
  const int nwin = b.n_local;
  const int row_u4 = ball_row_u4(b.n_src);
  uint4* const row4 = s_ball + (size_t)warp * ball_warp_u4(b.n_src, d, nwin);
  unsigned* const row = reinterpret_cast<unsigned*>(row4);
  int* const nb1 = reinterpret_cast<int*>(row4 + row_u4);
  int* const nb2 = nb1 + d;
  unsigned* const lc = reinterpret_cast<unsigned*>(row4 + row_u4 + (d + d * d + 3) / 4);  // [2][nwin]
  for (int i = lane; i < 2 * nwin; i += 32) lc[i] = 0u;
  int log2w = 0;
  while ((128 * R) >> log2w > 1) ++log2w;
  const NewBitCount c1{lc, log2w, b.win_first, b.win_stride, nwin};
  const NewBitCount c2{lc + nwin, log2w, b.win_first, b.win_stride, nwin};
  bool adj_ok = true;
  const long long warp_id = (long long)blockIdx.x * kWarpsB + warp;
  const long long n_warps = (long long)gridDim.x * kWarpsB;
  for (long long v = warp_id; v < N; v += n_warps) {
    for (int i = lane; i < row_u4; i += 32) row4[i] = make_uint4(0u, 0u, 0u, 0u);
    for (int j = lane; j < d; j += 32) nb1[j] = __ldg(b.adj + v * d + j);
    __syncwarp();
    // S_1 = {v} u N(v)
    if (lane == 0 && v < b.n_src) set_bit_counted(row, (unsigned)v, &c1);
    for (int j = lane; j < d; j += 32) {
      const int x = nb1[j];
      if ((unsigned)x >= (unsigned)N) { adj_ok = false; continue; }
      if (x < b.n_src) set_bit_counted(row, (unsigned)x, &c1);
    }
    __syncwarp();
    // S_2 = S_1 u N(N(v))
    set_rows_bits<VEC, 32>(b.adj, N, d, nb1, d, row, 0, b.n_src, lane, adj_ok, nb2, &c2);
    __syncwarp();
    // S_3 = S_2 u N(N(N(v)))
    if (d / VEC <= 32)
      scatter_plain<VEC>(b.adj, N, d, nb2, d * d, row, b.n_src, lane);
    else
      set_rows_bits<VEC, 32>(b.adj, N, d, nb2, d * d, row, 0, b.n_src, lane, adj_ok, nullptr, nullptr);
    __syncwarp();
    for (int k = 0; k < nwin; ++k) {
      const int t = b.win_first + k * b.win_stride;
      uint4* dst = b.ball + ((size_t)k * N + v) * R;
      for (int col = lane; col < R; col += 32) {
        const int idx = t * R + col;
        st_cg(dst + col, idx < row_u4 ? row4[idx] : make_uint4(0u, 0u, 0u, 0u));
      }
    }
    __syncwarp();
  }
  if (!adj_ok) set_error(b.ctrl, kErrAdj, (int)blockIdx.x);
  // lane k adds window k's counts: S_1 = new bits of step 1, S_2 = S_1 + new bits of step 2
  __syncwarp();
  if (lane < nwin) {
    const unsigned long long s1 = lc[lane], s2 = lc[nwin + lane];
    if (s1) atomicAdd(b.cnt + (size_t)lane * 6 + 0, s1);
    if (s1 + s2) atomicAdd(b.cnt + (size_t)lane * 6 + 2, s1 + s2);
  }
}

// Shared memory of ball_kernel, in bytes.
inline size_t ball_smem_bytes(int n_src, int d, int nwin) {
  return (size_t)(kBallThreads / 32) * (size_t)ball_warp_u4(n_src, d, nwin) * sizeof(uint4);
}

// ---- one dense sweep, wide rows ------------------------------------------------
// Valid-bit mask of the 128-bit chunk `col` of a row of a window with l sources.
__device__ __forceinline__ uint4 chunk_full_mask(int col, int l) {
  const int nvalid = max(0, min(128, l - 128 * col));
  unsigned m[4];
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const int vw = max(0, min(32, nvalid - 32 * w));
    m[w] = vw == 32 ? 0xffffffffu : ((1u << vw) - 1u);
  }
  return make_uint4(m[0], m[1], m[2], m[3]);
}

__device__ __forceinline__ bool equal4(const uint4& a, const uint4& b) {
  return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w;
}

// One sweep of (*) for rows of R >= 32 uint4 (one warp per row, lane L owns
// uint4 L, L+32, ...) and degree d <= 32.  Lane j holds the neighbour id u_j
// of the current vertex and hands it to the warp by shuffle; the next
// vertex's ids and own row are loaded while the current gathers are in
// flight.  A lane whose chunk of the vertex's own row is already full (every
// valid bit set) loads nothing: the OR cannot change it.  Near the last
// level, when most rows are almost full, this drops most of the gathered
// sectors.  The fullness is checked again after every group of U = 8
// neighbour rows, which drops more of them at the cost of a memory round
// trip a group (on a 16-regular graph of 65536 vertices this took the
// evaluation from 2.20 to 2.14 ms; used on levels only half full, or
// pipelined over two vertices, it was slower: 2.41 and 2.46 ms).
template <int R, bool STATS = false>
__device__ __forceinline__ void sweep_wide(const uint4* __restrict__ src, uint4* __restrict__ dst,
                                           const int* __restrict__ adj, int N, int d, int split, long long v0,
                                           long long stride, int l, bool own_count, unsigned (&cl)[4],
                                           bool& adj_ok, unsigned* stats = nullptr, int lvl = 0) {
  constexpr int UPL = R / 32;
  constexpr int U = 8;                 // neighbour rows a group loads; lanes re-check fullness between groups
  const int lane = threadIdx.x & 31;
  uint4 fm[UPL];
#pragma unroll
  for (int k = 0; k < UPL; ++k) fm[k] = chunk_full_mask(lane + 32 * k, l);
  int u_nx = 0;
  uint4 own_nx[UPL];
#pragma unroll
  for (int k = 0; k < UPL; ++k) own_nx[k] = make_uint4(0u, 0u, 0u, 0u);
  if (v0 < N) {
    u_nx = lane < d ? __ldg(adj + v0 * d + lane) : 0;
#pragma unroll
    for (int k = 0; k < UPL; ++k) own_nx[k] = ld_cg(src + v0 * R + lane + 32 * k);
  }
  for (long long v = v0; v < N; v += stride) {
    int u_me = u_nx;
    uint4 acc[UPL];
#pragma unroll
    for (int k = 0; k < UPL; ++k) acc[k] = own_nx[k];
    const long long vn = v + stride;
    if (vn < N) {
      u_nx = lane < d ? __ldg(adj + vn * d + lane) : 0;
#pragma unroll
      for (int k = 0; k < UPL; ++k) own_nx[k] = ld_cg(src + vn * R + lane + 32 * k);
    }
    if (lane < d && (unsigned)u_me >= (unsigned)N) { adj_ok = false; u_me = 0; }
    if (own_count) {
      unsigned co = 0;
#pragma unroll
      for (int k = 0; k < UPL; ++k) co += popc4(acc[k]);
      if (v < split) cl[2] += co; else cl[3] += co;
    }
    bool need[UPL];
#pragma unroll
    for (int k = 0; k < UPL; ++k) need[k] = !equal4(acc[k], fm[k]);
    for (int j0 = 0; j0 < d; j0 += U) {
      uint4 x[U][UPL];
#pragma unroll
      for (int q = 0; q < U; ++q) {
        const int j = j0 + q;
        const int u = __shfl_sync(0xffffffffu, u_me, j & 31);
#pragma unroll
        for (int k = 0; k < UPL; ++k)
          x[q][k] = (j < d && need[k]) ? ld_cg(src + (long long)u * R + lane + 32 * k) : make_uint4(0u, 0u, 0u, 0u);
      }
#pragma unroll
      for (int q = 0; q < U; ++q)
#pragma unroll
        for (int k = 0; k < UPL; ++k) or_into(acc[k], x[q][k]);
#pragma unroll
      for (int k = 0; k < UPL; ++k) need[k] = !equal4(acc[k], fm[k]);
    }
    unsigned cc = 0;
#pragma unroll
    for (int k = 0; k < UPL; ++k) {
      st_cg(dst + v * R + lane + 32 * k, acc[k]);
      cc += popc4(acc[k]);
    }
    if (v < split) cl[0] += cc; else cl[1] += cc;
    if constexpr (STATS) {
      const unsigned tot = __reduce_add_sync(0xffffffffu, cc);
      if (lane == 0 && lvl < kStatLevels) atomicAdd(stats + v * kStatLevels + lvl, (unsigned)l - tot);
    }
  }
}

// The same sweep for rows of 32 uint4 and degree d <= 16 with 32-byte
// accesses: a half-warp per row (lane hl owns uint4 2hl and 2hl + 1), two
// rows per warp step (vertex v and the one `stride` further).  Lane hl < d
// of a half holds neighbour hl of its vertex; the next step's ids and own
// rows are loaded while the current gathers are in flight; a lane whose 32
// bytes are full loads nothing, checked again after every group of 8
// neighbour rows.
template <int R, bool STATS = false>
__device__ __forceinline__ void sweep_wide_half(const uint4* __restrict__ src, uint4* __restrict__ dst,
                                                const int* __restrict__ adj, int N, int d, int split, long long v0,
                                                long long stride, int l, unsigned (&cl)[4], bool& adj_ok,
                                                unsigned* stats = nullptr, int lvl = 0) {
  static_assert(R == 32, "two uint4 of the row a lane");
  constexpr int U = 4;
  const int lane = threadIdx.x & 31, h = lane >> 4, hl = lane & 15;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  const uint4 fm[2] = {chunk_full_mask(2 * hl, l), chunk_full_mask(2 * hl + 1, l)};
  auto full = [&](const uint4 (&r)[2]) { return equal4(r[0], fm[0]) && equal4(r[1], fm[1]); };
  // ids and own row of this half's vertex of the step at vb (past N: a full
  // row, so nothing is gathered for it)
  auto fetch = [&](long long vb, int& ids, uint4 (&own)[2]) {
    const long long v = vb + h * stride;
    if (v < N) {
      ids = hl < d ? __ldg(adj + v * d + hl) : 0;
      ld_cg2(src + v * R + 2 * hl, own);
    } else {
      ids = 0;
      own[0] = fm[0];
      own[1] = fm[1];
    }
  };
  int u_nx;
  uint4 own_nx[2];
  fetch(v0, u_nx, own_nx);
  for (long long vb = v0; vb < N; vb += 2 * stride) {
    const long long v = vb + h * stride;
    const bool live = v < N;
    int u_me = u_nx;
    uint4 acc[2] = {own_nx[0], own_nx[1]};
    fetch(vb + 2 * stride, u_nx, own_nx);
    if (hl < d && (unsigned)u_me >= (unsigned)N) { adj_ok = false; u_me = 0; }
    bool need = live && !full(acc);
    for (int j0 = 0; j0 < d; j0 += U) {
      uint4 x[U][2];
#pragma unroll
      for (int q = 0; q < U; ++q) {
        const int j = j0 + q;
        const int u = __shfl_sync(0xffffffffu, u_me, (h << 4) | (j & 15));
        if (j < d && need) {
          ld_cg2(src + (long long)u * R + 2 * hl, x[q]);
        } else {
          x[q][0] = zero;
          x[q][1] = zero;
        }
      }
#pragma unroll
      for (int q = 0; q < U; ++q) {
        or_into(acc[0], x[q][0]);
        or_into(acc[1], x[q][1]);
      }
      need = live && !full(acc);
    }
    const unsigned cc = live ? popc4(acc[0]) + popc4(acc[1]) : 0u;
    if (live) {
      st_cg2(dst + v * R + 2 * hl, acc);
      if (v < split) cl[0] += cc; else cl[1] += cc;
    }
    if constexpr (STATS) {
      unsigned tot = cc;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
      if (live && hl == 0 && lvl < kStatLevels) atomicAdd(stats + v * kStatLevels + lvl, (unsigned)l - tot);
    }
  }
}

// Full-row stamps.  A row that is full at level L stays full (the sets are
// monotone), so its later rows need neither a read nor a write: the plain
// sweep stamps every row it finds full, and the stamped sweep below -- the
// skipping sweep of 4096-bit rows, degree <= 16 -- counts a stamped row as
// full without touching it, treats a row with a stamped neighbour as full
// (S_{k+1}[v] contains S_k[u]), and stamps instead of writing every row that
// turns full.  Its readers are therefore all stamp-aware: a row is read only
// when its stamp says it is not full, and such a row was written by the sweep
// that produced it.  The skipping sweeps are the last sweeps of a window (its
// levels only fill up), so no plain sweep ever reads a row left unwritten.
__device__ __forceinline__ bool stamped_full(unsigned st, unsigned id, int k) {
  return (st >> 8) == id && (int)(st & 0xffu) <= k;
}

template <int R>
__device__ __forceinline__ void sweep_stamped(const uint4* __restrict__ src, uint4* __restrict__ dst,
                                              const int* __restrict__ adj, int N, int d, int split, long long warp_id,
                                              long long n_warps, int l, unsigned (&cl)[4], bool& adj_ok,
                                              unsigned* __restrict__ stamps, unsigned id, int k) {
  static_assert(R == 32, "two uint4 of the row a lane");
  constexpr int U = 4;
  const int lane = threadIdx.x & 31, h = lane >> 4, hl = lane & 15;
  const uint4 zero = make_uint4(0u, 0u, 0u, 0u);
  const uint4 fm[2] = {chunk_full_mask(2 * hl, l), chunk_full_mask(2 * hl + 1, l)};
  auto full = [&](const uint4 (&r)[2]) { return equal4(r[0], fm[0]) && equal4(r[1], fm[1]); };
  const unsigned new_stamp = (id << 8) | (unsigned)(k + 1);
  const bool can_stamp = k + 1 < 255;
  // a contiguous block of vertices per warp: one coalesced stamp load per 32
  const long long per = ((long long)N + n_warps - 1) / n_warps;
  const long long v_lo = warp_id * per, v_hi = min((long long)N, v_lo + per);
  for (long long b = v_lo; b < v_hi; b += 32) {
    const long long v = b + lane;
    const bool in = v < v_hi;
    const bool fl = in && stamped_full(__ldcg(stamps + v), id, k);
    const unsigned fullm = __ballot_sync(0xffffffffu, fl);
    unsigned todo = __ballot_sync(0xffffffffu, in) & ~fullm;
    if (lane == 0 && fullm) {
      // full rows count l each, lo rows (v < split) and hi rows apart
      const long long lo_n = split - b;
      const unsigned lo_m = lo_n >= 32 ? 0xffffffffu : (lo_n <= 0 ? 0u : ((1u << lo_n) - 1u));
      cl[0] += (unsigned)__popc(fullm & lo_m) * (unsigned)l;
      cl[1] += (unsigned)__popc(fullm & ~lo_m) * (unsigned)l;
    }
    while (todo) {   // warp-uniform: two vertices per step, one per half-warp
      const int i0 = __ffs(todo) - 1;
      todo &= todo - 1;
      int i1 = -1;
      if (todo) {
        i1 = __ffs(todo) - 1;
        todo &= todo - 1;
      }
      const int my = h == 0 ? i0 : i1;
      const bool live = my >= 0;
      const long long vv = b + (live ? my : 0);
      int u = 0;
      bool nfull = false;
      if (live && hl < d) {
        u = __ldg(adj + vv * d + hl);
        if ((unsigned)u >= (unsigned)N) { adj_ok = false; u = 0; }
        nfull = stamped_full(__ldcg(stamps + u), id, k);
      }
      const unsigned nb = __ballot_sync(0xffffffffu, nfull);
      const bool any_nfull = ((nb >> (h << 4)) & 0xffffu) != 0u;
      uint4 acc[2] = {fm[0], fm[1]};
      if (live && !any_nfull) ld_cg2(src + vv * R + 2 * hl, acc);
      bool need = live && !any_nfull && !full(acc);
      for (int j0 = 0; j0 < d; j0 += U) {
        uint4 x[U][2];
#pragma unroll
        for (int q = 0; q < U; ++q) {
          const int j = j0 + q;
          const int uj = __shfl_sync(0xffffffffu, u, (h << 4) | (j & 15));
          if (j < d && need) {
            ld_cg2(src + (long long)uj * R + 2 * hl, x[q]);
          } else {
            x[q][0] = zero;
            x[q][1] = zero;
          }
        }
#pragma unroll
        for (int q = 0; q < U; ++q) {
          or_into(acc[0], x[q][0]);
          or_into(acc[1], x[q][1]);
        }
        need = need && !full(acc);
      }
      const unsigned fb = __ballot_sync(0xffffffffu, full(acc));
      const bool row_full = ((fb >> (h << 4)) & 0xffffu) == 0xffffu;
      if (live) {
        if (row_full && can_stamp) {
          if (hl == 0) {
            stamps[vv] = new_stamp;
            if (vv < split) cl[0] += (unsigned)l; else cl[1] += (unsigned)l;
          }
        } else {
          st_cg2(dst + vv * R + 2 * hl, acc);
          const unsigned cc = popc4(acc[0]) + popc4(acc[1]);
          if (vv < split) cl[0] += cc; else cl[1] += cc;
        }
      }
    }
  }
}

// Drops every full 128-byte line of [p, p + cells * 16) from L2 without a
// write-back (discard.global.L2), the lines split over the threads of CTAs
// cta .. ncta - 1.  Lines that straddle the range's ends are left alone.
__device__ __forceinline__ void discard_l2(const void* p, size_t cells, int cta, int ncta) {
  const unsigned long long b = (unsigned long long)p, e = b + (unsigned long long)cells * 16ull;
  const unsigned long long first = (b + 127ull) & ~127ull, last = e & ~127ull;
  if (last <= first) return;
  const unsigned long long lines = (last - first) >> 7;
  for (unsigned long long i = (unsigned long long)cta * kThreads + threadIdx.x; i < lines;
       i += (unsigned long long)ncta * kThreads)
    asm volatile("discard.global.L2 [%0], 128;" ::"l"(first + (i << 7)) : "memory");
}

// ---- one graph on a team of CTAs ------------------------------------------------
// R = uint4 words per row (W = 128*R source bits).  LPR lanes share a row,
// each lane owning UPL uint4 of it; a warp covers VPW vertices per step.
//
// eval_windows runs every window of this rank of one graph on the `ncta`
// CTAs of a team (this CTA is number `cta`), which synchronise through the
// team's control block a.ctrl.  The single-graph kernel is one team of all
// CTAs; the batch kernel runs many teams, each over its own list of graphs.
// bar_target and gl carry over from one graph to the next of a team: the
// barrier counter and the level-count slots of a.ctrl only grow.  Returns
// false when a wait ran out or a CTA of the team reported an error (the
// caller then leaves the kernel).
struct ApspSmem {
  unsigned long long red[kWarps][4];
  unsigned long long seen[4][2];   // must be zero before a team's first graph
  long long lvl[4];
  int flag;
};

struct EvalOut {
  long long sum, levels, dense_levels;
  int diam, disconnected, windows;
};

template <int R, bool STATS = false>
__device__ __forceinline__ bool eval_windows(const ApspArgs& a, int cta, int ncta, ApspSmem& sm, unsigned* s_dyn,
                                             unsigned long long& bar_target, unsigned& gl, int& ntrace,
                                             EvalOut& out) {
  constexpr int LPR = R >= 32 ? 32 : R;
  constexpr int VPW = 32 / LPR;
  constexpr int UPL = R / LPR;
  const int W = (a.win_bits > 0 && a.win_bits < 128 * R) ? a.win_bits : 128 * R;
  constexpr int U = UPL >= 2 ? 8 : 16;  // neighbour rows in flight per thread
  constexpr int SROW = 4 * R;          // 32-bit words per row in shared memory
  unsigned long long (*const s_red)[4] = sm.red;
  unsigned long long (*const s_seen)[2] = sm.seen;
  long long* const s_lvl = sm.lvl;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int sub = lane / LPR;          // which vertex of the warp's VPW
  const int li = lane % LPR;           // lane within the row
  const long long slot = ((long long)cta * kWarps + warp) * VPW + sub;
  const long long n_slots = (long long)ncta * kWarps * VPW;
  const int N = a.N, d = a.d;
  const unsigned grid = (unsigned)ncta;
  int* const my_nb = reinterpret_cast<int*>(s_dyn) + (size_t)warp * (kSeedVerts * kSeedNb + 2 * kSeedVerts * SROW);
  unsigned* const my_rows = reinterpret_cast<unsigned*>(my_nb + kSeedVerts * kSeedNb);
  const long long warp_id = (long long)cta * kWarps + warp;
  const long long n_warps = (long long)ncta * kWarps;

  // Level counts live in cnt[gl & 3]: between two barriers a CTA adds to the
  // slots of at most two levels while slower CTAs may still read the (at most
  // two) slots of the levels that ended at the previous barrier; four slots
  // keep those sets disjoint.  The counters only grow; s_seen holds the value
  // this CTA read last time, so a level's count is the difference.
  long long sum = 0, levels = 0, dense_levels = 0;
  int diam = 1, disconnected = 0, windows = 0;
  bool adj_ok = true;

  for (int phase = 1; phase <= 2 && !disconnected; ++phase) {
    const int nsrc = phase == 1 ? a.n_src1 : a.ac;
    if (nsrc <= 0) continue;
    const int row0 = phase == 1 ? 0 : N - a.ac;
    const int nwin = (nsrc + W - 1) / W;
    const bool use_ball = phase == 1 && a.ball != nullptr;
    const int* __restrict__ adjp = (phase == 2 && a.adj2) ? a.adj2 : a.adj;
    int local = 0;
    // The added-centre windows of rank r start at (r - based_nodes % procs)
    // mod procs, as the reference's do (general/evaluation.c:209-212).
    const int t_first = phase == 1 ? a.win_first
                                   : ((a.win_first - a.n_src1 % a.win_stride) % a.win_stride + a.win_stride) %
                                         a.win_stride;
    for (int t = t_first; t < nwin && !disconnected; t += a.win_stride, ++local) {
      const int first = t * W;
      const int l = min(W, nsrc - first);
      const long long lo_rows = a.split, hi_rows = (long long)N - a.split;
      const int base = row0 + first;   // vertex id of the window's bit 0
      ++windows;

      long long prev_total = l;   // popcount of the identity S_0
      long long kk = 0;
      int act = 0;
      const uint4* cur;           // S_kk rows the next sweep gathers from
      uint4* nxt;                 // rows it writes
      bool own_count = false;     // the first sweep of a ball window also reports S_3
      // full-row stamps: phase-1 windows without level recording; ids keep to 24 bits
      const unsigned stamp_id = a.stamp_base + (unsigned)t + 1u;
      unsigned* const stamps =
          (phase == 1 && a.levels == nullptr && !STATS && stamp_id < (1u << 24)) ? a.stamps : nullptr;
      // base builds: this window's level rows and counts (never with the ball pre-pass)
      uint4* const lev0 = a.levels ? a.levels + (size_t)t * (a.level_cap + 1) * N * R : nullptr;
      long long* const lcnt = a.levels ? a.level_counts + (size_t)t * (a.level_cap + 1) : nullptr;
      const bool rec = lev0 && cta == 0 && threadIdx.x == 0;
      bool lev_over = false;
      if (use_ball) {
        // ---- levels 0 and 1 from the ball pre-pass; S_3 rows are in HBM --------
        const unsigned long long* bc = a.ball_cnt + (size_t)local * 6;
        for (kk = 0; kk < 2; ++kk) {
          ++levels;
          act = level_decision(phase, (long long)__ldcg(bc + 2 * kk), (long long)__ldcg(bc + 2 * kk + 1), l, N,
                               lo_rows, hi_rows, a.groups, prev_total, sum);
          if (act) break;
        }
        if (!act) kk = 3;
        own_count = true;
        cur = a.ball + (size_t)local * N * R;
        nxt = a.buf0;
        // buf1 holds the previous window's rows, all dead: this window's first
        // sweep writes buf0 only, and every later reader of buf1 reads rows
        // written in this window.  Dropping those dirty lines from L2 saves
        // their write-back to DRAM; the grid barrier that ends the first sweep
        // orders the drops before the second sweep writes buf1.
        if (!lev0 && local > 0 && !act) discard_l2(a.buf1, (size_t)N * R, cta, ncta);
      } else {
        // ---- levels 0 and 1 by two-hop seeding into buf0 -----------------------
        unsigned c[4] = {0u, 0u, 0u, 0u};  // S_1 lo, S_1 hi, S_2 lo, S_2 hi
        uint4* const s2_out = lev0 ? lev0 + (size_t)2 * N * R : a.buf0;
        uint4* const s1_out = lev0 ? lev0 + (size_t)N * R : nullptr;
        if (a.vec4)
          seed_window<R, 4, STATS>(a, adjp, base, l, s2_out, my_nb, my_rows, c, adj_ok, warp_id, n_warps, s1_out);
        else
          seed_window<R, 1, STATS>(a, adjp, base, l, s2_out, my_nb, my_rows, c, adj_ok, warp_id, n_warps, s1_out);
        if (!adj_ok) set_error(a.ctrl, kErrAdj, (int)blockIdx.x);
        cta_add_counts<4>(c, a.ctrl, gl, s_red);
        bar_target += grid;
        if (!grid_barrier(a.ctrl, bar_target + a.phantom, a.timeout_ns, &sm.flag)) return false;
        trace_mark(a, ntrace, 1, 1);
        read_level_counts(a.ctrl, gl, 2, s_seen, s_lvl);
        const long long seed_lvl[4] = {s_lvl[0], s_lvl[1], s_lvl[2], s_lvl[3]};
        __syncthreads();
        if (ld_volatile_i32(&a.ctrl->error) != 0) return false;
        gl += 2;
        ++levels;
        act = level_decision(phase, seed_lvl[0], seed_lvl[1], l, N, lo_rows, hi_rows, a.groups, prev_total, sum);
        if (!act) {
          kk = 1;
          ++levels;
          act = level_decision(phase, seed_lvl[2], seed_lvl[3], l, N, lo_rows, hi_rows, a.groups, prev_total,
                               sum);
        }
        if (!act) kk = 2;
        if (rec) {
          lcnt[0] = l;
          lcnt[1] = seed_lvl[0] + seed_lvl[1];
          lcnt[2] = seed_lvl[2] + seed_lvl[3];
        }
        cur = s2_out;
        nxt = lev0 ? a.buf0 : a.buf1;
      }
      if (!act) {
        // ---- dense OR-gather sweeps ------------------------------------------------
        for (; kk < N; ++kk) {
          const uint4* __restrict__ src = cur;
          const bool to_level = lev0 && kk + 1 <= a.level_cap;
          if (lev0 && !to_level) lev_over = true;
          uint4* __restrict__ dst = to_level ? lev0 + (size_t)(kk + 1) * N * R : nxt;
          unsigned cl[4] = {0u, 0u, 0u, 0u};   // new rows lo/hi, then (own_count) own rows lo/hi
          // The skipping sweep pays once the gathered level is nearly full
          // (its count, prev_total, is known); on denser-to-come levels the
          // plain sweep is faster.
          bool wide = false;
          if constexpr (LPR == 32) {
            if (d <= 32 && !own_count && prev_total * 1000 >= (long long)N * l * a.skip_permille) {
              wide = true;
              bool half = false;
              if constexpr (R == 32) {
                if (d <= 16) {
                  half = true;
                  if (!STATS && stamps)
                    sweep_stamped<R>(src, dst, adjp, N, d, a.split, warp_id, n_warps, l, cl, adj_ok, stamps,
                                     stamp_id, (int)kk);
                  else
                    sweep_wide_half<R, STATS>(src, dst, adjp, N, d, a.split, slot, n_slots, l, cl, adj_ok,
                                              a.stats, (int)kk + 1);
                }
              }
              if (!half)
                sweep_wide<R, STATS>(src, dst, adjp, N, d, a.split, slot, n_slots, l, own_count, cl, adj_ok,
                                     a.stats, (int)kk + 1);
            }
          }
          if constexpr (R >= 8) {
            // 32-byte accesses: each group of LPR lanes serves two rows, LP
            // lanes a row, PPL 32-byte parts a lane (vertex v of the step and
            // the one n_slots further); half the load instructions of
            // 16-byte accesses
            constexpr int LP = LPR / 2;
            constexpr int PPL = R / (2 * LP);
            constexpr int U2 = 8 / PPL;
            const int h = li / LP, hl = li % LP;
            for (long long vb = wide ? N : slot; vb < N; vb += 2 * n_slots) {
              const long long v = vb + h * n_slots;
              const bool live = v < N;
              const long long vv = live ? v : vb;   // a dead half reads a live row and drops the result
              const int* arow = adjp + vv * d;
              uint4 acc[PPL][2];
#pragma unroll
              for (int p = 0; p < PPL; ++p) ld_cg2(src + vv * R + 2 * (hl + p * LP), acc[p]);
              if (own_count && live) {
                unsigned co = 0;
#pragma unroll
                for (int p = 0; p < PPL; ++p) co += popc4(acc[p][0]) + popc4(acc[p][1]);
                if (v < a.split) cl[2] += co; else cl[3] += co;
              }
              int j = 0;
              // After a group of neighbour rows, a part of the row whose 256
              // bits are all set needs no further gathers (full-width windows
              // only: every bit of the part is a source).
              bool need[PPL];
#pragma unroll
              for (int p = 0; p < PPL; ++p) need[p] = true;
              for (; j + U2 <= d; j += U2) {
                int u[U2];
#pragma unroll
                for (int q = 0; q < U2; ++q) u[q] = __ldg(arow + j + q);
#pragma unroll
                for (int q = 0; q < U2; ++q) {
                  if ((unsigned)u[q] >= (unsigned)N) { adj_ok = false; u[q] = 0; }
                }
                if (j > 0 && l == W) {
#pragma unroll
                  for (int p = 0; p < PPL; ++p)
                    need[p] = (acc[p][0].x & acc[p][0].y & acc[p][0].z & acc[p][0].w & acc[p][1].x & acc[p][1].y &
                               acc[p][1].z & acc[p][1].w) != 0xffffffffu;
                }
                uint4 x[U2][PPL][2];
#pragma unroll
                for (int q = 0; q < U2; ++q)
#pragma unroll
                  for (int p = 0; p < PPL; ++p) {
                    if (need[p]) {
                      ld_cg2(src + (long long)u[q] * R + 2 * (hl + p * LP), x[q][p]);
                    } else {
                      x[q][p][0] = make_uint4(0u, 0u, 0u, 0u);
                      x[q][p][1] = make_uint4(0u, 0u, 0u, 0u);
                    }
                  }
#pragma unroll
                for (int q = 0; q < U2; ++q)
#pragma unroll
                  for (int p = 0; p < PPL; ++p) {
                    or_into(acc[p][0], x[q][p][0]);
                    or_into(acc[p][1], x[q][p][1]);
                  }
              }
              for (; j < d; ++j) {
                int u = __ldg(arow + j);
                if ((unsigned)u >= (unsigned)N) { adj_ok = false; u = 0; }
#pragma unroll
                for (int p = 0; p < PPL; ++p) {
                  uint4 x[2];
                  ld_cg2(src + (long long)u * R + 2 * (hl + p * LP), x);
                  or_into(acc[p][0], x[0]);
                  or_into(acc[p][1], x[1]);
                }
              }
              unsigned cc = 0;
              if (live) {
#pragma unroll
                for (int p = 0; p < PPL; ++p) {
                  st_cg2(dst + v * R + 2 * (hl + p * LP), acc[p]);
                  cc += popc4(acc[p][0]) + popc4(acc[p][1]);
                }
                if (v < a.split) cl[0] += cc; else cl[1] += cc;
              }
              if constexpr (R == 32) {
                // (one row pair per warp step at R = 32, so the loop is warp-uniform); rows
                // turn full only once the gathered level is well filled: below 30 % of
                // N * sources nothing is stamped
                if (stamps && d <= 16 && prev_total * 10 >= (long long)N * l * 3) {
                  // the LP lanes of this row hold its popcount in parts
                  unsigned tot = cc;
#pragma unroll
                  for (int o = LP / 2; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
                  if (live && hl == 0 && tot == (unsigned)l && kk + 1 < 255)
                    stamps[v] = (stamp_id << 8) | (unsigned)(kk + 1);
                }
              }
              if constexpr (STATS) {
                // the LP lanes of this row hold its popcount in parts; with several rows a
                // warp step (R < 32) the groups may leave the loop apart, so only the lanes
                // still in it take part
                unsigned tot = cc;
                const unsigned am = __activemask();
#pragma unroll
                for (int o = LP / 2; o > 0; o >>= 1) tot += __shfl_xor_sync(am, tot, o);
                if (live && hl == 0 && kk + 1 < kStatLevels)
                  atomicAdd(a.stats + v * kStatLevels + kk + 1, (unsigned)l - tot);
              }
            }
          } else
          for (long long v = wide ? N : slot; v < N; v += n_slots) {
            const int* arow = adjp + v * d;
            uint4 acc[UPL];
#pragma unroll
            for (int k = 0; k < UPL; ++k) acc[k] = ld_cg(src + v * R + li + k * LPR);
            if (own_count) {
              unsigned co = 0;
#pragma unroll
              for (int k = 0; k < UPL; ++k) co += popc4(acc[k]);
              if (v < a.split) cl[2] += co; else cl[3] += co;
            }
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
            unsigned cc = 0;
#pragma unroll
            for (int k = 0; k < UPL; ++k) {
              st_cg(dst + v * R + li + k * LPR, acc[k]);
              cc += popc4(acc[k]);
            }
            if (v < a.split) cl[0] += cc; else cl[1] += cc;
            if constexpr (STATS) {
              // the LPR lanes of this row hold its popcount in parts
              const unsigned gmask = LPR == 32 ? 0xffffffffu : (((1u << LPR) - 1u) << (sub * LPR));
              unsigned tot = cc;
#pragma unroll
              for (int o = LPR / 2; o > 0; o >>= 1) tot += __shfl_xor_sync(gmask, tot, o);
              if (li == 0 && kk + 1 < kStatLevels) atomicAdd(a.stats + v * kStatLevels + kk + 1, (unsigned)l - tot);
            }
          }
          if (!adj_ok) set_error(a.ctrl, kErrAdj, (int)blockIdx.x);
          if (own_count) {
            // slot gl: S_kk (own rows, level kk-1); slot gl+1: S_kk+1 (level kk)
            const unsigned c4[4] = {cl[2], cl[3], cl[0], cl[1]};
            cta_add_counts<4>(c4, a.ctrl, gl, s_red);
          } else {
            cta_add_counts<2>(cl, a.ctrl, gl, s_red);
          }
          bar_target += grid;
          if (!grid_barrier(a.ctrl, bar_target + a.phantom, a.timeout_ns, &sm.flag)) return false;
          trace_mark(a, ntrace, 2, kk);
          read_level_counts(a.ctrl, gl, own_count ? 2 : 1, s_seen, s_lvl);
          const long long l0 = s_lvl[0], l1 = s_lvl[1], l2 = s_lvl[2], l3 = s_lvl[3];
          __syncthreads();   // s_lvl is rewritten after the next barrier only
          if (ld_volatile_i32(&a.ctrl->error) != 0) return false;   // same answer in every CTA after the barrier
          ++dense_levels;
          if (own_count) {
            ++gl;
            ++levels;
            act = level_decision(phase, l0, l1, l, N, lo_rows, hi_rows, a.groups, prev_total, sum);
            if (act) { --kk; ++gl; break; }   // complete (or stalled) at S_kk: this sweep was not needed
            own_count = false;
            ++gl;
            ++levels;
            act = level_decision(phase, l2, l3, l, N, lo_rows, hi_rows, a.groups, prev_total, sum);
          } else {
            ++gl;
            ++levels;
            act = level_decision(phase, l0, l1, l, N, lo_rows, hi_rows, a.groups, prev_total, sum);
            if (rec && kk + 1 <= a.level_cap) lcnt[kk + 1] = l0 + l1;
          }
          if (act) break;
          cur = dst;
          nxt = (dst == a.buf0) ? a.buf1 : a.buf0;
        }
      }
      if (act == 2) { disconnected = 1; diam = N + 1; }
      else if (kk + 1 > diam) diam = (int)(kk + 1);
      if (rec) a.win_levels[t] = act == 2 ? -1 : (lev_over ? -2 : (int)(kk + 1));
    }
  }

  out.sum = sum;
  out.levels = levels;
  out.dense_levels = dense_levels;
  out.diam = diam;
  out.disconnected = disconnected;
  out.windows = windows;
  return true;
}

// ---- the single-graph persistent kernel ---------------------------------------
template <int R>
__global__ void __launch_bounds__(kThreads, 1) apsp_persistent_kernel(const ApspArgs a) {
  __shared__ ApspSmem sm;
  extern __shared__ unsigned s_dyn[];   // per warp: neighbour ids [4][64], then rows [4][2][SROW]
  if (threadIdx.x < 8) sm.seen[threadIdx.x >> 1][threadIdx.x & 1] = 0ULL;
  __syncthreads();
  unsigned long long bar_target = 0;
  unsigned gl = 0;                     // global level counter
  int ntrace = 0;
  trace_mark(a, ntrace, 0, 0);
  EvalOut o;
  if (!eval_windows<R>(a, (int)blockIdx.x, (int)gridDim.x, sm, s_dyn, bar_target, gl, ntrace, o)) return;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ApspCtrl* c = a.ctrl;
    c->diam = o.diam;
    c->disconnected = o.disconnected;
    c->sum = o.sum;
    c->levels = o.levels;
    c->dense_levels = o.dense_levels;
    c->windows = o.windows;
    c->trace_len = ntrace;
    __threadfence();
    c->done = 1;
  }
}

// ---- the batch kernel: many graphs, one launch -----------------------------------
// The CTAs of the launch form n_teams teams of team_ctas CTAs (CTAs past the
// last full team return at once).  Team t evaluates the graphs
// team_list[team_start[t] .. team_start[t+1]) one after the other, every
// window of each on all of its CTAs, synchronising through its own control
// block team_ctrl[t] and keeping its two bitset matrices in its own slice of
// the scratch.  A graph's answer depends only on its adjacency: the team size
// and the window width change the schedule, never a count.
struct BatchGraph {
  const int* adj;        // [N][d], device
  int N, d;
  int n_src;             // phase-1 sources (based_nodes); N = n_src * groups
  int groups;
  int vec4;              // d % 4 == 0 and adj 16-byte aligned
  int win_first;         // the graph's source windows this entry runs: win_first, win_first + win_stride,
  int win_stride;        // ... (0, 1: all of them; one graph's windows spread over teams otherwise)
  int win_bits;          // sources per window below 128 * R (64), or 0
};

struct BatchOut {        // per graph, written by the team's first CTA
  long long sum, levels, dense_levels;
  int diam, disconnected, windows, done;
};

struct BatchArgs {
  const BatchGraph* graphs;
  BatchOut* out;
  ApspCtrl* team_ctrl;            // [n_teams], zeroed before the launch
  const int* team_start;          // [n_teams + 1]
  const int* team_list;           // graph ids, in run order per team
  uint4* scratch;
  const long long* team_off;      // team t: buf0 = scratch + team_off[t], buf1 = buf0 + team_cells[t]
  const long long* team_cells;
  long long timeout_ns;
  const int* stop;                // when non-null and *stop != 0 the launch does nothing
  int* sticky;                    // when non-null: receives the first team's error code (never cleared here)
  int n_teams, team_ctas;
  // Optional full-row stamps, zeroed before the launch: team t uses
  // stamps + team_soff[t], one per vertex of its largest graph.
  unsigned* stamps = nullptr;
  const long long* team_soff = nullptr;
};

template <int R>
__global__ void __launch_bounds__(kThreads, 1) apsp_batch_kernel(const BatchArgs b) {
  __shared__ ApspSmem sm;
  extern __shared__ unsigned s_dyn[];
  const int team = (int)blockIdx.x / b.team_ctas;
  const int cta = (int)blockIdx.x % b.team_ctas;
  if (team >= b.n_teams) return;
  if (b.stop && ld_volatile_i32(b.stop) != 0) return;   // written before the launch: the same in every CTA
  if (threadIdx.x < 8) sm.seen[threadIdx.x >> 1][threadIdx.x & 1] = 0ULL;
  __syncthreads();
  ApspArgs a;
  a.adj2 = nullptr;
  a.buf0 = b.scratch + b.team_off[team];
  a.buf1 = a.buf0 + b.team_cells[team];
  a.ctrl = b.team_ctrl + team;
  a.timeout_ns = b.timeout_ns;
  a.ac = 0;
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
  a.stamps = b.stamps ? b.stamps + b.team_soff[team] : nullptr;
  a.stamp_base = 0;
  unsigned long long bar_target = 0;
  unsigned gl = 0;
  int ntrace = 0;
  const int k1 = b.team_start[team + 1];
  for (int k = b.team_start[team]; k < k1; ++k) {
    const int gi = b.team_list[k];
    const BatchGraph gr = b.graphs[gi];
    a.adj = gr.adj;
    a.N = gr.N;
    a.d = gr.d;
    a.n_src1 = gr.n_src;
    a.split = gr.N;
    a.groups = gr.groups;
    a.vec4 = gr.vec4;
    a.win_first = gr.win_first;
    a.win_stride = gr.win_stride;
    a.win_bits = gr.win_bits;
    EvalOut o;
    if (!eval_windows<R>(a, cta, b.team_ctas, sm, s_dyn, bar_target, gl, ntrace, o)) {
      if (b.sticky && threadIdx.x == 0) atomicCAS(b.sticky, 0, max(1, ld_volatile_i32(&a.ctrl->error)));
      return;
    }
    if (cta == 0 && threadIdx.x == 0) {
      BatchOut* w = b.out + gi;
      w->sum = o.sum;
      w->levels = o.levels;
      w->dense_levels = o.dense_levels;
      w->diam = o.diam;
      w->disconnected = o.disconnected;
      w->windows = o.windows;
      w->done = 1;
    }
    // the next graph's windows take the stamp ids after this graph's
    const int W = (gr.win_bits > 0 && gr.win_bits < 128 * R) ? gr.win_bits : 128 * R;
    a.stamp_base += (unsigned)((gr.n_src + W - 1) / W);
  }
}

// ---- the profile kernel: one graph plus per-vertex level statistics -------------
// stats[v][k] = number of sources not yet reached from v after k levels,
// summed over all windows (kStatLevels levels kept; the window's rows are
// complete once a window stops, so later levels add nothing).  From it:
// eccentricity(v) = first k with stats[v][k] == 0, transmission(v) =
// sum_k stats[v][k], and the level histogram stats[v][k-1] - stats[v][k].
// Runs only when *gate != 0 (the annealing engine re-profiles its current
// graph after an accepted move); the statistics are zeroed here, then the
// graph is evaluated exactly as the persistent kernel does it, without the
// ball pre-pass.  A failure also sets *sticky (when given).
template <int R>
__global__ void __launch_bounds__(kThreads, 1) apsp_profile_kernel(const ApspArgs a, const int* gate, int* sticky) {
  __shared__ ApspSmem sm;
  extern __shared__ unsigned s_dyn[];
  if (gate && ld_volatile_i32(gate) == 0) return;   // written before the launch: every CTA sees the same value
  const long long n = (long long)a.N * kStatLevels;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a.stats[i] = 0u;
  if (threadIdx.x < 8) sm.seen[threadIdx.x >> 1][threadIdx.x & 1] = 0ULL;
  unsigned long long bar_target = gridDim.x;
  unsigned gl = 0;
  int ntrace = 0;
  EvalOut o;
  if (!grid_barrier(a.ctrl, bar_target, a.timeout_ns, &sm.flag) ||
      !eval_windows<R, true>(a, (int)blockIdx.x, (int)gridDim.x, sm, s_dyn, bar_target, gl, ntrace, o)) {
    if (sticky && threadIdx.x == 0) atomicCAS(sticky, 0, max(1, ld_volatile_i32(&a.ctrl->error)));
    return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    ApspCtrl* c = a.ctrl;
    c->diam = o.diam;
    c->disconnected = o.disconnected;
    c->sum = o.sum;
    c->levels = o.levels;
    c->dense_levels = o.dense_levels;
    c->windows = o.windows;
    __threadfence();
    c->done = 1;
  }
}

// Shared memory the persistent kernel needs for its seeding rows, in bytes.
template <int R>
constexpr size_t apsp_smem_bytes() {
  return (size_t)kWarps * (kSeedVerts * kSeedNb + 2 * kSeedVerts * 4 * R) * sizeof(unsigned);
}

}  // namespace ggb
