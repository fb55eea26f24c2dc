// Symmetry-sector enumeration on packed keys of one or two 64-bit words.
//
// One level = one site.  Candidate i of level `depth` is (parent p = i / d,
// state c = i % d) with d = loc_dims[depth]; it survives when
//   * the state is allowed on that site (string constraints),
//   * every global U(1) sum can still reach its target (branch and bound with
//     the remaining min/max) or, at the last site, equals it; Z2 parities are
//     checked at the last site,
//   * every link pair and n-body constraint whose last site is `depth` holds.
// Survivors are written in candidate order, which keeps parents in order and
// states ascending: the final level is sorted by key, i.e. lexicographically
// (the order produced by edlgt/symmetries/symmetry_sector.py:785-967).
// Digits of earlier sites are decoded from the parent key.  Kernels are
// templated on the key type (keys.cuh): uint64_t, or a 128-bit pair of words
// when the key space exceeds 63 bits.
#include "internal.cuh"
#include "keys.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;
constexpr int kMaxGlob = 4;

template <typename K>
__device__ __forceinline__ int digit_of(const edg_sector_tables& t, K key, int site) {
  return edg::key_digit(key, site, t.n_hi, t.strides[site], (uint64_t)t.loc_dims[site]);
}

// Evaluates candidate (parent_key, parent sums, state c) at `depth`.
template <typename K>
__device__ __forceinline__ bool candidate_ok(const edg_sector_tables& t, int depth, K pkey,
                                             const int32_t* __restrict__ psums, int c, int32_t* nsums) {
  const int n = t.n_sites, dm = t.dmax;
  if (!t.site_allowed[depth * dm + c]) return false;
  const bool last = depth == n - 1;
  for (int g = 0; g < t.n_glob; ++g) {
    int32_t v = t.glob_val[((int64_t)g * n + depth) * dm + c];
    int32_t prev = psums ? psums[g] : 0;
    if (t.glob_type == 0) {
      int32_t s = prev + v;
      nsums[g] = s;
      int32_t target = t.glob_target[g];
      if (last) {
        if (s != target) return false;
      } else {
        if (target < s + t.glob_rem_min[g * (n + 1) + depth + 1]) return false;
        if (target > s + t.glob_rem_max[g * (n + 1) + depth + 1]) return false;
      }
    } else {
      int32_t s = prev ^ v;
      nsums[g] = s;
      if (last && s != t.glob_target[g]) return false;
    }
  }
  for (int p = t.pair_start[depth]; p < t.pair_start[depth + 1]; ++p) {
    int s0 = t.pair_s0[p], s1 = t.pair_s1[p], dir = t.pair_dir[p];
    int c0 = s0 == depth ? c : digit_of(t, pkey, s0);
    int c1 = s1 == depth ? c : digit_of(t, pkey, s1);
    int32_t v = t.link_val[(((int64_t)dir * 2 + 0) * n + s0) * dm + c0] +
                t.link_val[(((int64_t)dir * 2 + 1) * n + s1) * dm + c1];
    if (v != t.link_target[dir]) return false;
  }
  if (t.nb_start != nullptr) {
    for (int a = t.nb_start[depth]; a < t.nb_start[depth + 1]; ++a) {
      int id = t.nb_id[a];
      int32_t acc = 0;
      for (int q = t.nb_site_start[id]; q < t.nb_site_start[id + 1]; ++q) {
        int s = t.nb_sites[q];
        int cs = s == depth ? c : digit_of(t, pkey, s);
        int32_t v = t.nb_val[((int64_t)id * n + s) * dm + cs];
        acc = t.nbody_type == 0 ? acc + v : (acc ^ v);
      }
      if (acc != t.nb_target[id]) return false;
    }
  }
  return true;
}

struct Level {
  int depth;
  int d;
  int n_glob;
  const uint64_t* prev_keys;
  const int32_t* prev_sums;
  int64_t n_cand;
};

template <typename K>
__device__ __forceinline__ bool eval_candidate(const edg_sector_tables& t, const Level& L, int64_t i, K* key_out,
                                               int32_t* sums_out) {
  if (i >= L.n_cand) return false;
  int64_t p = i / L.d;
  int c = (int)(i - p * L.d);
  K pkey = L.depth == 0 ? K(0) : edg::ld_key<K>(L.prev_keys, p);
  const int32_t* ps = (L.depth == 0 || L.n_glob == 0) ? nullptr : L.prev_sums + p * L.n_glob;
  bool ok = candidate_ok(t, L.depth, pkey, ps, c, sums_out);
  *key_out = pkey + edg::key_step<K>((int64_t)c * (int64_t)t.strides[L.depth], L.depth, t.n_hi);
  return ok;
}

template <typename K>
__global__ void __launch_bounds__(kThreads) level_count(edg_sector_tables t, Level L, int64_t* __restrict__ block_counts) {
  int64_t base = (int64_t)blockIdx.x * kTile;
  int local = 0;
  K key;
  int32_t sums[kMaxGlob];
#pragma unroll 1
  for (int it = 0; it < kItems; ++it) {
    int64_t i = base + (int64_t)it * kThreads + threadIdx.x;
    local += eval_candidate(t, L, i, &key, sums) ? 1 : 0;
  }
  // block reduction of per-thread counts
  __shared__ int warp_tot[kThreads / 32];
  int v = local;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) warp_tot[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < kThreads / 32; ++w) s += warp_tot[w];
    block_counts[blockIdx.x] = s;
  }
}

template <typename K>
__global__ void __launch_bounds__(kThreads) level_fill(edg_sector_tables t, Level L, const int64_t* __restrict__ block_offsets,
                                                       uint64_t* __restrict__ next_keys, int32_t* __restrict__ next_sums) {
  __shared__ int warp_cnt[kThreads / 32];
  __shared__ int64_t running;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) running = block_offsets[blockIdx.x];
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * kTile;
#pragma unroll 1
  for (int it = 0; it < kItems; ++it) {
    int64_t i = base + (int64_t)it * kThreads + threadIdx.x;
    K key = 0;
    int32_t sums[kMaxGlob];
    bool ok = eval_candidate(t, L, i, &key, sums);
    unsigned ballot = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) warp_cnt[warp] = __popc(ballot);
    __syncthreads();
    int64_t pos = running;
    for (int w = 0; w < warp; ++w) pos += warp_cnt[w];
    pos += __popc(ballot & ((1u << lane) - 1u));
    if (ok) {
      edg::st_key(next_keys, pos, key);
      for (int g = 0; g < L.n_glob; ++g) next_sums[pos * L.n_glob + g] = sums[g];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int w = 0; w < kThreads / 32; ++w) s += warp_cnt[w];
      running += s;
    }
    __syncthreads();
  }
}

int check_tables(const edg_sector_tables* t, int32_t depth, int64_t n_prev, const char* who) {
  EDG_REQUIRE(t != nullptr, "%s: null tables", who);
  EDG_REQUIRE(t->n_sites > 0 && t->n_sites <= EDG_MAX_SITES, "%s: n_sites out of range", who);
  EDG_REQUIRE(depth >= 0 && depth < t->n_sites, "%s: depth %d out of range", who, depth);
  EDG_REQUIRE(t->n_glob >= 0 && t->n_glob <= kMaxGlob, "%s: at most %d global symmetries", who, kMaxGlob);
  EDG_REQUIRE(n_prev >= 0, "%s: negative parent count", who);
  EDG_REQUIRE(depth == 0 ? n_prev == 1 : true, "%s: level 0 expands one empty parent", who);
  EDG_REQUIRE(t->key_words == 0 || t->key_words == 1 || t->key_words == 2, "%s: key_words must be 1 or 2", who);
  EDG_REQUIRE(t->key_words != 2 || (t->n_hi > 0 && t->n_hi < t->n_sites), "%s: n_hi out of range", who);
  return EDG_OK;
}

}  // namespace

extern "C" int64_t edg_sector_level_blocks(int64_t n_candidates) {
  return edg::ceil_div(n_candidates > 0 ? n_candidates : 1, kTile);
}

extern "C" int edg_sector_level_count(const edg_sector_tables* t, int32_t depth, const uint64_t* prev_keys,
                                      const int32_t* prev_sums, int64_t n_prev, int64_t* block_offsets,
                                      int64_t* scratch, cudaStream_t stream) {
  int st = check_tables(t, depth, n_prev, "edg_sector_level_count");
  if (st) return st;
  int d = t->loc_dims[depth];
  EDG_REQUIRE(d > 0 && d <= t->dmax, "edg_sector_level_count: bad local dimension");
  EDG_REQUIRE(t->key_words != 2 || depth == 0 || (reinterpret_cast<uintptr_t>(prev_keys) & 15) == 0,
              "edg_sector_level_count: two-word keys must be 16-byte aligned");
  Level L{depth, d, t->n_glob, prev_keys, prev_sums, n_prev * (int64_t)d};
  int64_t nb = edg_sector_level_blocks(L.n_cand);
  if (t->key_words == 2)
    level_count<edg::u128><<<(unsigned)nb, kThreads, 0, stream>>>(*t, L, block_offsets);
  else
    level_count<uint64_t><<<(unsigned)nb, kThreads, 0, stream>>>(*t, L, block_offsets);
  EDG_CHECK_LAUNCH("edg_sector_level_count");
  return edg_scan_i64(block_offsets, block_offsets, nb, scratch, stream);
}

extern "C" int edg_sector_level_fill(const edg_sector_tables* t, int32_t depth, const uint64_t* prev_keys,
                                     const int32_t* prev_sums, int64_t n_prev, const int64_t* block_offsets,
                                     uint64_t* next_keys, int32_t* next_sums, cudaStream_t stream) {
  int st = check_tables(t, depth, n_prev, "edg_sector_level_fill");
  if (st) return st;
  int d = t->loc_dims[depth];
  EDG_REQUIRE(d > 0 && d <= t->dmax, "edg_sector_level_fill: bad local dimension");
  EDG_REQUIRE(t->key_words != 2 || ((depth == 0 || (reinterpret_cast<uintptr_t>(prev_keys) & 15) == 0) &&
                                     (reinterpret_cast<uintptr_t>(next_keys) & 15) == 0),
              "edg_sector_level_fill: two-word keys must be 16-byte aligned");
  Level L{depth, d, t->n_glob, prev_keys, prev_sums, n_prev * (int64_t)d};
  int64_t nb = edg_sector_level_blocks(L.n_cand);
  if (t->key_words == 2)
    level_fill<edg::u128><<<(unsigned)nb, kThreads, 0, stream>>>(*t, L, block_offsets, next_keys, next_sums);
  else
    level_fill<uint64_t><<<(unsigned)nb, kThreads, 0, stream>>>(*t, L, block_offsets, next_keys, next_sums);
  EDG_CHECK_LAUNCH("edg_sector_level_fill");
  return EDG_OK;
}

// ---------------------------------------------------------------------------
// key <-> configuration conversion
// ---------------------------------------------------------------------------
namespace {

__global__ void keys_to_configs_k(const uint64_t* __restrict__ keys, int64_t n, int n_sites,
                                  const int32_t* __restrict__ loc_dims, uint16_t* __restrict__ configs) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = keys[i];
    for (int s = n_sites - 1; s >= 0; --s) {
      uint64_t d = (uint64_t)loc_dims[s];
      configs[i * n_sites + s] = (uint16_t)(k % d);
      k /= d;
    }
  }
}

__global__ void configs_to_keys_k(const uint16_t* __restrict__ configs, int64_t n, int n_sites,
                                  const uint64_t* __restrict__ strides, uint64_t* __restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = 0;
    for (int s = 0; s < n_sites; ++s) k += (uint64_t)configs[i * n_sites + s] * strides[s];
    keys[i] = k;
  }
}

// Two-word keys: digits of sites [n_hi, n) from the low word, of [0, n_hi)
// from the high word.
__global__ void keys_to_configs_wide_k(const uint64_t* __restrict__ keys, int64_t n, int n_sites, int n_hi,
                                       const int32_t* __restrict__ loc_dims, uint16_t* __restrict__ configs) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t lo = keys[2 * i], hi = keys[2 * i + 1];
    for (int s = n_sites - 1; s >= n_hi; --s) {
      uint64_t d = (uint64_t)loc_dims[s];
      configs[i * n_sites + s] = (uint16_t)(lo % d);
      lo /= d;
    }
    for (int s = n_hi - 1; s >= 0; --s) {
      uint64_t d = (uint64_t)loc_dims[s];
      configs[i * n_sites + s] = (uint16_t)(hi % d);
      hi /= d;
    }
  }
}

__global__ void configs_to_keys_wide_k(const uint16_t* __restrict__ configs, int64_t n, int n_sites, int n_hi,
                                       const uint64_t* __restrict__ strides, uint64_t* __restrict__ keys) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t hi = 0, lo = 0;
    for (int s = 0; s < n_hi; ++s) hi += (uint64_t)configs[i * n_sites + s] * strides[s];
    for (int s = n_hi; s < n_sites; ++s) lo += (uint64_t)configs[i * n_sites + s] * strides[s];
    keys[2 * i] = lo;
    keys[2 * i + 1] = hi;
  }
}

}  // namespace

extern "C" int edg_keys_to_configs_wide(const uint64_t* keys, int64_t n, int32_t n_sites, int32_t n_hi,
                                        const int32_t* loc_dims, uint16_t* configs, cudaStream_t stream) {
  EDG_REQUIRE(n >= 0 && n_sites > 1 && n_sites <= EDG_MAX_SITES && n_hi > 0 && n_hi < n_sites,
              "edg_keys_to_configs_wide: bad sizes");
  if (n == 0) return EDG_OK;
  keys_to_configs_wide_k<<<edg::grid_for(n, 256), 256, 0, stream>>>(keys, n, n_sites, n_hi, loc_dims, configs);
  EDG_CHECK_LAUNCH("edg_keys_to_configs_wide");
  return EDG_OK;
}

extern "C" int edg_configs_to_keys_wide(const uint16_t* configs, int64_t n, int32_t n_sites, int32_t n_hi,
                                        const uint64_t* strides, uint64_t* keys, cudaStream_t stream) {
  EDG_REQUIRE(n >= 0 && n_sites > 1 && n_sites <= EDG_MAX_SITES && n_hi > 0 && n_hi < n_sites,
              "edg_configs_to_keys_wide: bad sizes");
  if (n == 0) return EDG_OK;
  configs_to_keys_wide_k<<<edg::grid_for(n, 256), 256, 0, stream>>>(configs, n, n_sites, n_hi, strides, keys);
  EDG_CHECK_LAUNCH("edg_configs_to_keys_wide");
  return EDG_OK;
}

extern "C" int edg_keys_to_configs(const uint64_t* keys, int64_t n, int32_t n_sites, const int32_t* loc_dims,
                                   uint16_t* configs, cudaStream_t stream) {
  EDG_REQUIRE(n >= 0 && n_sites > 0 && n_sites <= EDG_MAX_SITES, "edg_keys_to_configs: bad sizes");
  if (n == 0) return EDG_OK;
  keys_to_configs_k<<<edg::grid_for(n, 256), 256, 0, stream>>>(keys, n, n_sites, loc_dims, configs);
  EDG_CHECK_LAUNCH("edg_keys_to_configs");
  return EDG_OK;
}

extern "C" int edg_configs_to_keys(const uint16_t* configs, int64_t n, int32_t n_sites, const uint64_t* strides,
                                   uint64_t* keys, cudaStream_t stream) {
  EDG_REQUIRE(n >= 0 && n_sites > 0 && n_sites <= EDG_MAX_SITES, "edg_configs_to_keys: bad sizes");
  if (n == 0) return EDG_OK;
  configs_to_keys_k<<<edg::grid_for(n, 256), 256, 0, stream>>>(configs, n, n_sites, strides, keys);
  EDG_CHECK_LAUNCH("edg_configs_to_keys");
  return EDG_OK;
}
