// config -> index lookup: bucket table build and batched queries.
#include "lookup.cuh"

namespace {

__global__ void build_buckets(const uint64_t* __restrict__ keys, int64_t n, int shift, int64_t n_buckets,
                              int64_t* __restrict__ bucket_start) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b <= n_buckets;
       b += (int64_t)gridDim.x * blockDim.x) {
    if (b == n_buckets) {
      bucket_start[b] = n;
      continue;
    }
    uint64_t q = (uint64_t)b << shift;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < q)
        lo = mid + 1;
      else
        hi = mid;
    }
    bucket_start[b] = lo;
  }
}

// Any key width: bucket b starts at the first key whose dense position
// (keys.cuh) is >= b << shift; the dense position is monotone in the key.
template <typename K>
__global__ void build_buckets_dense(const uint64_t* __restrict__ keys, int64_t n, uint64_t lo_space, int shift,
                                    int64_t n_buckets, int64_t* __restrict__ bucket_start) {
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b <= n_buckets;
       b += (int64_t)gridDim.x * blockDim.x) {
    if (b == n_buckets) {
      bucket_start[b] = n;
      continue;
    }
    const edg::u128 q = (edg::u128)(uint64_t)b << shift;
    int64_t lo = 0, hi = n;
    while (lo < hi) {
      int64_t mid = (lo + hi) >> 1;
      if (edg::key_dense(edg::ld_key<K>(keys, mid), lo_space) < q)
        lo = mid + 1;
      else
        hi = mid;
    }
    bucket_start[b] = lo;
  }
}

__global__ void lookup_k(edg_lookup_table t, const uint64_t* __restrict__ queries, int64_t m, int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = edg::find_key(t, queries[i]);
}

__global__ void lookup_wide_k(edg_lookup_table t, const uint64_t* __restrict__ queries, int64_t m,
                              int64_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = edg::find_key_t(t, edg::ld_key<edg::u128>(queries, i));
}

}  // namespace

extern "C" int edg_lookup_build(const uint64_t* keys, int64_t n, int32_t shift, int64_t n_buckets,
                                int64_t* bucket_start, cudaStream_t stream) {
  EDG_REQUIRE(n >= 0 && n_buckets > 0 && shift >= 0 && shift < 64, "edg_lookup_build: bad sizes");
  EDG_REQUIRE(bucket_start != nullptr && (n == 0 || keys != nullptr), "edg_lookup_build: null pointer");
  build_buckets<<<edg::grid_for(n_buckets + 1, 256), 256, 0, stream>>>(keys, n, shift, n_buckets, bucket_start);
  EDG_CHECK_LAUNCH("edg_lookup_build");
  return EDG_OK;
}

extern "C" int edg_lookup_build_wide(const uint64_t* keys, int64_t n, int32_t key_words, uint64_t lo_space,
                                     int32_t shift, int64_t n_buckets, int64_t* bucket_start, cudaStream_t stream) {
  EDG_REQUIRE(key_words == 1 || key_words == 2, "edg_lookup_build_wide: key_words must be 1 or 2");
  EDG_REQUIRE(n >= 0 && n_buckets > 0 && shift >= 0 && shift < (key_words == 2 ? 127 : 64),
              "edg_lookup_build_wide: bad sizes");
  EDG_REQUIRE(key_words == 1 || lo_space > 0, "edg_lookup_build_wide: lo_space must be positive");
  EDG_REQUIRE(bucket_start != nullptr && (n == 0 || keys != nullptr), "edg_lookup_build_wide: null pointer");
  EDG_REQUIRE(key_words == 1 || (reinterpret_cast<uintptr_t>(keys) & 15) == 0,
              "edg_lookup_build_wide: two-word keys must be 16-byte aligned");
  const unsigned g = edg::grid_for(n_buckets + 1, 256);
  if (key_words == 2)
    build_buckets_dense<edg::u128><<<g, 256, 0, stream>>>(keys, n, lo_space, shift, n_buckets, bucket_start);
  else
    build_buckets_dense<uint64_t><<<g, 256, 0, stream>>>(keys, n, lo_space, shift, n_buckets, bucket_start);
  EDG_CHECK_LAUNCH("edg_lookup_build_wide");
  return EDG_OK;
}

extern "C" int edg_lookup(const edg_lookup_table* table, const uint64_t* queries, int64_t m, int64_t* index_out,
                          cudaStream_t stream) {
  EDG_REQUIRE(table != nullptr && m >= 0, "edg_lookup: bad arguments");
  EDG_REQUIRE(table->key_words >= 0 && table->key_words <= 2, "edg_lookup: key_words must be 1 or 2");
  if (m == 0) return EDG_OK;
  if (table->key_words == 2) {
    EDG_REQUIRE((reinterpret_cast<uintptr_t>(queries) & 15) == 0 && (reinterpret_cast<uintptr_t>(table->keys) & 15) == 0,
                "edg_lookup: two-word keys must be 16-byte aligned");
    lookup_wide_k<<<edg::grid_for(m, 256), 256, 0, stream>>>(*table, queries, m, index_out);
    EDG_CHECK_LAUNCH("edg_lookup");
    return EDG_OK;
  }
  lookup_k<<<edg::grid_for(m, 256), 256, 0, stream>>>(*table, queries, m, index_out);
  EDG_CHECK_LAUNCH("edg_lookup");
  return EDG_OK;
}
