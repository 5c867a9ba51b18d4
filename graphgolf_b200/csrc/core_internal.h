// core_internal.h -- helpers the translation units of libgraphgolf_b200.so
// share: the ggb_last_error() message, the count of kernel launches that
// ggb_kernel_launches() reports, and the host copy into pinned staging.
// Not part of the public C ABI.
#pragma once
#include <cstddef>

namespace ggb {

// Formats the message ggb_last_error() returns and gives back `code`.
int core_fail(int code, const char* fmt, ...);

// Adds n to the launch counter.
void core_add_launches(long long n);

// Copies n ints from pageable memory into pinned staging (non-temporal
// stores where the CPU has AVX2, memcpy otherwise).
void stage_copy(int* dst, const int* src, size_t n);

}  // namespace ggb
