// Helpers shared by the library's translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace ss_internal {
// Records the message that ss_last_error() returns on this thread and returns `code`.
int fail(int code, const std::string& msg);
// Clears that message (every entry point starts with it).
void clear_error();
}  // namespace ss_internal

#define SS_TRY_CUDA(call)                                                                            \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return ss_internal::fail(SS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)
