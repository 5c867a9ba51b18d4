// stage.cu -- host staging of adjacency from pageable memory onto the device.
//
// The reference's programs hand evaluation() a plain malloc'd adjacency
// (general/main.c, grid/main.c), so every host entry point must first copy it
// into pinned memory before the DMA engine can read it.  One core streams
// about 15-20 GB/s of non-temporal stores, which at N=65536, d=16 (4 MiB) is
// as long as a sixth of the evaluation itself.  This file spreads that copy
// over a small pool of host threads: the range is cut into units of at least
// 512 KiB, threads claim units from one packed atomic word, copy them with
// non-temporal stores and enqueue each unit's host-to-device copy themselves,
// so the CPU copy of one unit overlaps the DMA of the units before it.
//
// The calling thread works too and waits only for units some thread has
// claimed: a helper that wakes late finds nothing left and costs nothing.
// Helpers spin briefly after each job, then sleep on a condition variable.
// GGB_STAGE_THREADS (1..16) sets the number of copying threads, the caller
// included; the default is min(4, hardware threads / 4), at least 1.
//
// Past the CPU copy the bound is the PCIe DMA (about 40-50 GB/s measured for
// pinned host-to-device copies on the B200 hosts), so stage_upload_ids()
// sends vertex ids as 16-bit values when every one fits: the threads narrow
// them with saturating AVX2 packs while they copy, the DMA moves half the
// bytes, and widen_ids_kernel restores the int32 adjacency on the device.
// If some int lies outside [0, 65535] nothing narrowed is used: the call
// waits for the stream and sends the ints as they are, so the evaluator sees
// exactly the caller's values either way.  GGB_STAGE_NARROW=0 turns the
// 16-bit path off.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include <immintrin.h>
#include <unistd.h>

#include "core_internal.h"
#include "stage_plan.h"

namespace {

// Copies n ints with 32-byte non-temporal stores: the pinned staging buffer
// is never read by the CPU, so its lines need not be read for ownership or
// kept in the caches.  dst needs 4-byte alignment only.
__attribute__((target("avx2"))) void copy_stream(int* dst, const int* src, size_t n) {
  size_t i = 0;
  for (; i < n && ((uintptr_t)(dst + i) & 31u); ++i) dst[i] = src[i];
  for (; i + 32 <= n; i += 32) {
    const __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + i));
    const __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + i + 8));
    const __m256i c = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + i + 16));
    const __m256i d = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + i + 24));
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + i), a);
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + i + 8), b);
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + i + 16), c);
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + i + 24), d);
  }
  for (; i < n; ++i) dst[i] = src[i];
  _mm_sfence();
}

// Narrows n ints to 16 bits with non-temporal stores; returns false if some
// value lies outside [0, 65535] (dst is then unspecified).  packus saturates
// each 32-bit lane to 16 bits and interleaves the 128-bit halves of its two
// sources; the 64-bit permute (0, 2, 1, 3) puts the ids back in order.
__attribute__((target("avx2"))) bool narrow_stream(uint16_t* dst, const int* src, size_t n) {
  uint32_t bad = 0;
  size_t i = 0;
  for (; i < n && ((uintptr_t)(dst + i) & 31u); ++i) {
    bad |= (uint32_t)src[i];
    dst[i] = (uint16_t)src[i];
  }
  __m256i acc = _mm256_setzero_si256();
  for (; i + 32 <= n; i += 32) {
    const __m256i a = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + i));
    const __m256i b = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + i + 8));
    const __m256i c = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + i + 16));
    const __m256i d = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(src + i + 24));
    acc = _mm256_or_si256(acc, _mm256_or_si256(_mm256_or_si256(a, b), _mm256_or_si256(c, d)));
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + i),
                        _mm256_permute4x64_epi64(_mm256_packus_epi32(a, b), 0xD8));
    _mm256_stream_si256(reinterpret_cast<__m256i*>(dst + i + 16),
                        _mm256_permute4x64_epi64(_mm256_packus_epi32(c, d), 0xD8));
  }
  for (; i < n; ++i) {
    bad |= (uint32_t)src[i];
    dst[i] = (uint16_t)src[i];
  }
  _mm_sfence();
  return (bad & 0xFFFF0000u) == 0 && _mm256_testz_si256(acc, _mm256_set1_epi32((int)0xFFFF0000u));
}

bool narrow_plain(uint16_t* dst, const int* src, size_t n) {
  uint32_t bad = 0;
  for (size_t i = 0; i < n; ++i) {
    bad |= (uint32_t)src[i];
    dst[i] = (uint16_t)src[i];
  }
  return (bad & 0xFFFF0000u) == 0;
}

bool narrow_copy(uint16_t* dst, const int* src, size_t n) {
  static const bool avx2 = __builtin_cpu_supports("avx2");
  return avx2 ? narrow_stream(dst, src, n) : narrow_plain(dst, src, n);
}

// Widens n 16-bit ids into ints: 8 ids per thread and step, one 16-byte load
// and two 16-byte stores (both buffers start 256-byte aligned).
__global__ void widen_ids_kernel(const uint16_t* __restrict__ src, int* __restrict__ dst, long long n) {
  const long long n8 = n / 8;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n8; i += stride) {
    const uint4 v = __ldcs(reinterpret_cast<const uint4*>(src) + i);
    int4 lo, hi;
    lo.x = (int)(v.x & 0xFFFFu), lo.y = (int)(v.x >> 16), lo.z = (int)(v.y & 0xFFFFu), lo.w = (int)(v.y >> 16);
    hi.x = (int)(v.z & 0xFFFFu), hi.y = (int)(v.z >> 16), hi.z = (int)(v.w & 0xFFFFu), hi.w = (int)(v.w >> 16);
    reinterpret_cast<int4*>(dst)[2 * i] = lo;
    reinterpret_cast<int4*>(dst)[2 * i + 1] = hi;
  }
  for (long long i = n8 * 8 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += stride)
    dst[i] = (int)src[i];
}

using ggb::StagePiece;
using ggb::StageUnit;

// The claim word: generation (24 bits) | unit count (20 bits) | next unit (20 bits).
constexpr int kUnitBits = 20;
constexpr uint64_t kUnitMask = (1ull << kUnitBits) - 1;
constexpr int kMaxUnits = (1 << kUnitBits) - 1;

inline uint64_t pack(uint64_t gen, uint64_t n, uint64_t next) {
  return (gen << (2 * kUnitBits)) | (n << kUnitBits) | next;
}

class Pool {
 public:
  static Pool& get() {
    // Never destroyed: helper threads may still sleep on cv_ at exit.
    static Pool* p = new Pool();
    if (p->pid_ != getpid()) p = new Pool();   // a forked child has no helpers
    return *p;
  }

  int threads() const { return helpers_ + 1; }

  // Runs one job; the calling thread works on it too.  With narrow set the
  // units are sent as 16-bit ids; *in_range then tells whether every id fit
  // (if not, some units may have been sent and the rest were not).
  cudaError_t run(int device, void* pinned, void* dev, bool narrow, cudaStream_t st,
                  const std::vector<StagePiece>& pieces, const std::vector<StageUnit>& units, bool* in_range) {
    std::lock_guard<std::mutex> job_lock(job_mu_);
    device_ = device;
    pinned_ = pinned;
    dev_ = dev;
    narrow_ = narrow;
    stream_ = st;
    pieces_ = &pieces;
    units_ = &units;
    done_.store(0, std::memory_order_relaxed);
    err_.store(0, std::memory_order_relaxed);
    range_bad_.store(0, std::memory_order_relaxed);
    const uint64_t gen = (++gen_) & ((1ull << (64 - 2 * kUnitBits)) - 1);
    const int n = (int)units.size();
    claim_.store(pack(gen, n, 0), std::memory_order_release);
    if (helpers_ > 0 && n > 1) {
      {
        std::lock_guard<std::mutex> lk(mu_);
        wake_ = gen;
      }
      cv_.notify_all();
    }
    work(gen, /*set_device=*/false);
    // Every unit has been claimed; wait for those other threads still hold.
    for (int spin = 0; done_.load(std::memory_order_acquire) != n; ++spin) {
      if (spin < 4096)
        _mm_pause();
      else
        std::this_thread::yield();
    }
    if (in_range) *in_range = range_bad_.load(std::memory_order_relaxed) == 0;
    return (cudaError_t)err_.load(std::memory_order_relaxed);
  }

 private:
  Pool() : pid_(getpid()) {
    int t = 0;
    if (const char* e = std::getenv("GGB_STAGE_THREADS")) t = std::atoi(e);
    if (t <= 0) t = std::max(1, std::min(4, (int)std::thread::hardware_concurrency() / 4));
    t = std::min(t, 16);
    for (int i = 0; i < t - 1; ++i) {
      try {
        std::thread(&Pool::helper, this).detach();
        ++helpers_;
      } catch (...) {
        break;
      }
    }
  }

  // Claims and runs units of job `gen` until none is left.
  void work(uint64_t gen, bool set_device) {
    bool device_set = !set_device;
    for (;;) {
      uint64_t c = claim_.load(std::memory_order_acquire);
      int u;
      for (;;) {
        if ((c >> (2 * kUnitBits)) != gen) return;
        const uint64_t n = (c >> kUnitBits) & kUnitMask, next = c & kUnitMask;
        if (next >= n) return;
        if (claim_.compare_exchange_weak(c, c + 1, std::memory_order_acq_rel, std::memory_order_acquire)) {
          u = (int)next;
          break;
        }
      }
      // A claimed unit keeps the job alive: run() returns only after done_
      // counts it, so the job's fields are stable here.
      if (!device_set) {
        if (cudaSetDevice(device_) != cudaSuccess) fail(cudaGetLastError());
        device_set = true;
      }
      const StageUnit& un = (*units_)[u];
      if (narrow_) {
        uint16_t* h = static_cast<uint16_t*>(pinned_);
        bool ok = true;
        for (int p = un.p0; p < un.p1 && ok; ++p) {
          const StagePiece& pc = (*pieces_)[p];
          ok = narrow_copy(h + pc.off, pc.src, pc.n);
        }
        if (!ok) range_bad_.store(1, std::memory_order_relaxed);
        if (un.hi > un.lo && !range_bad_.load(std::memory_order_relaxed)) {
          const cudaError_t e = cudaMemcpyAsync(static_cast<uint16_t*>(dev_) + un.lo, h + un.lo,
                                                (un.hi - un.lo) * sizeof(uint16_t), cudaMemcpyHostToDevice, stream_);
          if (e != cudaSuccess) fail(e);
          ggb::core_add_h2d((long long)((un.hi - un.lo) * sizeof(uint16_t)));
        }
      } else {
        int* h = static_cast<int*>(pinned_);
        for (int p = un.p0; p < un.p1; ++p) {
          const StagePiece& pc = (*pieces_)[p];
          ggb::stage_copy(h + pc.off, pc.src, pc.n);
        }
        if (un.hi > un.lo) {
          const cudaError_t e = cudaMemcpyAsync(static_cast<int*>(dev_) + un.lo, h + un.lo,
                                                (un.hi - un.lo) * sizeof(int), cudaMemcpyHostToDevice, stream_);
          if (e != cudaSuccess) fail(e);
          ggb::core_add_h2d((long long)((un.hi - un.lo) * sizeof(int)));
        }
      }
      done_.fetch_add(1, std::memory_order_acq_rel);
    }
  }

  void fail(cudaError_t e) {
    int expect = 0;
    err_.compare_exchange_strong(expect, (int)e);
  }

  void helper() {
    uint64_t seen = 0;
    for (;;) {
      uint64_t gen = 0;
      // Spin about 50 microseconds for the next job, then sleep.
      for (int spin = 0; spin < 20000; ++spin) {
        const uint64_t c = claim_.load(std::memory_order_acquire);
        gen = c >> (2 * kUnitBits);
        if (gen != seen) break;
        _mm_pause();
      }
      if (gen == seen) {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return wake_ != seen; });
        gen = wake_;
      }
      seen = gen;
      work(gen, /*set_device=*/true);
    }
  }

  const pid_t pid_;
  int helpers_ = 0;
  std::mutex job_mu_;   // one job at a time
  std::mutex mu_;
  std::condition_variable cv_;
  uint64_t wake_ = 0;   // guarded by mu_
  uint64_t gen_ = 0;    // guarded by job_mu_
  std::atomic<uint64_t> claim_{0};
  std::atomic<int> done_{0};
  std::atomic<int> err_{0};
  std::atomic<int> range_bad_{0};
  int device_ = 0;
  void* pinned_ = nullptr;
  void* dev_ = nullptr;
  bool narrow_ = false;
  cudaStream_t stream_ = nullptr;
  const std::vector<StagePiece>* pieces_ = nullptr;
  const std::vector<StageUnit>* units_ = nullptr;
};

}  // namespace

namespace ggb {

void stage_copy(int* dst, const int* src, size_t n) {
  static const bool avx2 = __builtin_cpu_supports("avx2");
  if (avx2)
    copy_stream(dst, src, n);
  else
    std::memcpy(dst, src, n * sizeof(int));
}

int stage_threads() { return Pool::get().threads(); }

namespace {

// Cuts the upload into units: at least 128 Ki ids each, and about 8 per
// thread for large totals so the last DMA is short (at most 1 Mi ids).
cudaError_t plan(const StageSeg* segs, int nsegs, size_t total, int threads, std::vector<StagePiece>& pieces,
                 std::vector<StageUnit>& units) {
  const size_t chunk =
      std::min<size_t>(std::max<size_t>(128 * 1024, total / (8 * (size_t)threads)), 1024 * 1024);
  stage_plan(segs, nsegs, total, chunk, pieces, units);
  return (int)units.size() > kMaxUnits ? cudaErrorInvalidValue : cudaSuccess;
}

}  // namespace

cudaError_t stage_upload(int device, int* pinned, int* dev, const StageSeg* segs, int nsegs, size_t total,
                         cudaStream_t st) {
  if (total == 0) return cudaSuccess;
  Pool& pool = Pool::get();
  std::vector<StagePiece> pieces;
  std::vector<StageUnit> units;
  cudaError_t e = plan(segs, nsegs, total, pool.threads(), pieces, units);
  if (e != cudaSuccess) return e;
  return pool.run(device, pinned, dev, false, st, pieces, units, nullptr);
}

cudaError_t stage_upload_ids(int device, int* pinned, uint16_t* dev16, int* dev, const StageSeg* segs, int nsegs,
                             size_t total, cudaStream_t st) {
  static const bool narrow_on = [] {
    const char* e = std::getenv("GGB_STAGE_NARROW");
    return !(e && e[0] == '0');
  }();
  if (total == 0) return cudaSuccess;
  if (!dev16 || !narrow_on) return stage_upload(device, pinned, dev, segs, nsegs, total, st);
  Pool& pool = Pool::get();
  std::vector<StagePiece> pieces;
  std::vector<StageUnit> units;
  cudaError_t e = plan(segs, nsegs, total, pool.threads(), pieces, units);
  if (e != cudaSuccess) return e;
  bool in_range = false;
  e = pool.run(device, pinned, dev16, true, st, pieces, units, &in_range);
  if (e != cudaSuccess) return e;
  if (!in_range) {
    // Some DMAs from the pinned buffer may still run: wait, then send ints.
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    return stage_upload(device, pinned, dev, segs, nsegs, total, st);
  }
  const int threads = 256;
  const long long blocks = std::min<long long>(((long long)total / 8 + threads - 1) / threads + 1, 148 * 8);
  widen_ids_kernel<<<(unsigned)blocks, threads, 0, st>>>(dev16, dev, (long long)total);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  core_add_launches(1);
  return cudaSuccess;
}

}  // namespace ggb
