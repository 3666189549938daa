// Shared helpers for the pytme_b200 CUDA library: status codes, the per-thread
// last-error message and launch checking. Every exported entry point returns an
// int status (TM_OK on success) and records a message that tm_last_error reads.
#pragma once

#include <cuda_runtime.h>
#include <cstdarg>
#include <cstdio>
#include <cstdint>
#include <cstring>

#include "pytme_b200.h"

namespace tmb {

void set_error(const char* fmt, ...);
void set_device_memory_limit(int64_t bytes);
int64_t device_memory_limit();

inline int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return TM_OK;
  set_error("%s: %s", what, cudaGetErrorString(e));
  return e == cudaErrorMemoryAllocation ? TM_E_OOM : TM_E_CUDA;
}

inline int check_launch(const char* what) {
  return cuda_status(cudaGetLastError(), what);
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace tmb

#define TM_TRY(expr)               \
  do {                             \
    int _st = (expr);              \
    if (_st != TM_OK) return _st;  \
  } while (0)

#define TM_REQUIRE(cond, ...)                 \
  do {                                        \
    if (!(cond)) {                            \
      ::tmb::set_error(__VA_ARGS__);           \
      return TM_E_INVALID;                    \
    }                                         \
  } while (0)
