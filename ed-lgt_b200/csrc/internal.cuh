// Shared internals of libedgpu: status codes, error recording, launch helpers.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstdarg>

#include "edgpu.h"

namespace edg {

// Per-thread message of the most recent failure (read by edg_get_last_error).
void set_error(const char* fmt, ...);

// Maps a CUDA runtime error to EDG_ERR_CUDA after recording it.
int cuda_status(cudaError_t e, const char* where);

constexpr int kSmCount = 148;  // B200: 2 dies x 74 SMs

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Grid size for a grid-stride loop over n items: a multiple of the SM count,
// capped so that every SM holds a few resident CTAs.
inline unsigned grid_for(int64_t n, int threads, int ctas_per_sm = 8) {
  int64_t need = ceil_div(n, threads);
  int64_t cap = (int64_t)kSmCount * ctas_per_sm;
  if (need < 1) need = 1;
  return (unsigned)(need < cap ? need : cap);
}

}  // namespace edg

#define EDG_CHECK_LAUNCH(where)                                         \
  do {                                                                  \
    cudaError_t _e = cudaGetLastError();                                \
    if (_e != cudaSuccess) return edg::cuda_status(_e, where);          \
  } while (0)

#define EDG_REQUIRE(cond, ...)                                          \
  do {                                                                  \
    if (!(cond)) {                                                      \
      edg::set_error(__VA_ARGS__);                                      \
      return EDG_ERR_ARG;                                               \
    }                                                                   \
  } while (0)
