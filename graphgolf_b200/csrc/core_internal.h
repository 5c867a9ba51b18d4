// core_internal.h -- helpers the translation units of libgraphgolf_b200.so
// share: the ggb_last_error() message and the count of kernel launches that
// ggb_kernel_launches() reports.  Not part of the public C ABI.
#pragma once

namespace ggb {

// Formats the message ggb_last_error() returns and gives back `code`.
int core_fail(int code, const char* fmt, ...);

// Adds n to the launch counter.
void core_add_launches(long long n);

}  // namespace ggb
