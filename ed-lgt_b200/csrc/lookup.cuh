// Device-side config->index search over a sorted sector key array.
#pragma once
#include "internal.cuh"

namespace edg {

// Lower-bound search restricted to the bucket of the query's top bits;
// returns the row index of q or -1 when q is not a sector state.
__device__ __forceinline__ int64_t find_key(const edg_lookup_table& t, uint64_t q) {
  uint64_t b = q >> t.shift;
  if (b >= (uint64_t)t.n_buckets) return -1;
  int64_t lo = __ldg(t.bucket_start + b);
  int64_t hi = __ldg(t.bucket_start + b + 1);
  const int64_t end = hi;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    uint64_t k = __ldg(t.keys + mid);
    if (k < q)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < end && __ldg(t.keys + lo) == q) ? lo : -1;
}

}  // namespace edg
