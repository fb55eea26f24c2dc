// Device-side config->index search over a sorted sector key array.
#pragma once
#include "internal.cuh"
#include "keys.cuh"

namespace edg {

// Lower-bound search restricted to the bucket of the query's top bits;
// returns the row index of q or -1 when q is not a sector state.  K is the
// key type of the table (uint64_t for one-word keys, u128 for two).
template <typename K>
__device__ __forceinline__ int64_t find_key_t(const edg_lookup_table& t, K q) {
  const u128 dq = key_dense(q, t.lo_space);
  const u128 b = dq >> t.shift;
  if (b >= (u128)(uint64_t)t.n_buckets) return -1;
  int64_t lo = __ldg(t.bucket_start + (int64_t)b);
  int64_t hi = __ldg(t.bucket_start + (int64_t)b + 1);
  const int64_t end = hi;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    K k = ld_key<K>(t.keys, mid);
    if (k < q)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < end && ld_key<K>(t.keys, lo) == q) ? lo : -1;
}

// One-word tables (every caller that does not handle two-word keys).
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
