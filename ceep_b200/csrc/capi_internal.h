// Error helpers shared by the translation units behind include/ceep_b200.h.
#pragma once
#include <cuda_runtime.h>

namespace ceep {
// Record a printf-style message for ceep_last_error() and return `code`.
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
}  // namespace ceep
