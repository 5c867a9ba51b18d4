// core_internal.h -- helpers the translation units of libgraphgolf_b200.so
// share: the ggb_last_error() message, the count of kernel launches that
// ggb_kernel_launches() reports, and the host copy into pinned staging.
// Not part of the public C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace ggb {

// Formats the message ggb_last_error() returns and gives back `code`.
int core_fail(int code, const char* fmt, ...);

// Adds n to the launch counter.
void core_add_launches(long long n);

// Adds to the count of adjacency bytes sent host to device (thread-safe).
void core_add_h2d(long long bytes);

// Copies n ints from pageable memory into pinned staging (non-temporal
// stores where the CPU has AVX2, memcpy otherwise).
void stage_copy(int* dst, const int* src, size_t n);

// One source array of an upload: it fills ints [off, off + n) of the pinned
// and device buffers.
struct StageSeg {
  const int* src;
  size_t off;
  size_t n;
};

// Copies the segments into the pinned buffer and enqueues the host-to-device
// copy of ints [0, total) of it into `dev` on stream st of `device`, spread
// over the staging threads (stage.cu).  total must cover every segment; ints
// between segments are sent as they lie in the pinned buffer.  The pinned
// buffer must not feed a copy still in flight.  Returns the first CUDA error.
cudaError_t stage_upload(int device, int* pinned, int* dev, const StageSeg* segs, int nsegs, size_t total,
                         cudaStream_t st);

// Like stage_upload(), but when dev16 is given and every int lies in
// [0, 65535], sends the ids as 16-bit values into dev16 and widens them into
// dev on the device (one kernel launch on st).  Otherwise sends the ints as
// they are.  Either way dev ends up holding exactly the caller's ints.
cudaError_t stage_upload_ids(int device, int* pinned, uint16_t* dev16, int* dev, const StageSeg* segs, int nsegs,
                             size_t total, cudaStream_t st);

// Number of threads stage_upload() copies with, the caller included.
int stage_threads();

}  // namespace ggb
