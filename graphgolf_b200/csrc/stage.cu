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

  // Runs one job; the calling thread works on it too.
  cudaError_t run(int device, int* pinned, int* dev, cudaStream_t st, const std::vector<StagePiece>& pieces,
                  const std::vector<StageUnit>& units) {
    std::lock_guard<std::mutex> job_lock(job_mu_);
    device_ = device;
    pinned_ = pinned;
    dev_ = dev;
    stream_ = st;
    pieces_ = &pieces;
    units_ = &units;
    done_.store(0, std::memory_order_relaxed);
    err_.store(0, std::memory_order_relaxed);
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
      for (int p = un.p0; p < un.p1; ++p) {
        const StagePiece& pc = (*pieces_)[p];
        ggb::stage_copy(pinned_ + pc.off, pc.src, pc.n);
      }
      if (un.hi > un.lo) {
        const cudaError_t e = cudaMemcpyAsync(dev_ + un.lo, pinned_ + un.lo, (un.hi - un.lo) * sizeof(int),
                                              cudaMemcpyHostToDevice, stream_);
        if (e != cudaSuccess) fail(e);
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
  int device_ = 0;
  int* pinned_ = nullptr;
  int* dev_ = nullptr;
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

cudaError_t stage_upload(int device, int* pinned, int* dev, const StageSeg* segs, int nsegs, size_t total,
                         cudaStream_t st) {
  if (total == 0) return cudaSuccess;
  Pool& pool = Pool::get();
  // Units of at least 512 KiB, and about 8 per thread for large totals so the
  // last DMA is short (at most 4 MiB).
  const size_t chunk = std::min<size_t>(std::max<size_t>(128 * 1024, total / (8 * (size_t)pool.threads())),
                                        1024 * 1024);
  std::vector<StagePiece> pieces;
  std::vector<StageUnit> units;
  stage_plan(segs, nsegs, total, chunk, pieces, units);
  if ((int)units.size() > kMaxUnits) return cudaErrorInvalidValue;
  return pool.run(device, pinned, dev, st, pieces, units);
}

}  // namespace ggb
