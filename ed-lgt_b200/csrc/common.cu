// Library-wide utilities: error recording, version, int64 exclusive scan.
#include "internal.cuh"

#include <cstring>

namespace edg {

static thread_local char g_last_error[512] = {0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* where) {
  set_error("%s: %s", where, cudaGetErrorString(e));
  return EDG_ERR_CUDA;
}

}  // namespace edg

extern "C" int edg_get_last_error(char* buf, int len) {
  if (buf == nullptr || len <= 0) return EDG_ERR_ARG;
  strncpy(buf, edg::g_last_error, (size_t)len - 1);
  buf[len - 1] = '\0';
  return EDG_OK;
}

extern "C" int edg_version(void) { return 100; }

// ---------------------------------------------------------------------------
// Three-phase exclusive scan: per-tile sums, scan of the tile sums (one CTA),
// per-tile scan with the tile offset.  Tiles are 1024 threads x 4 items.
// ---------------------------------------------------------------------------
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int64_t warp_inclusive(int64_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int64_t o = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += o;
  }
  return v;
}

// Exclusive block scan of one value per thread; returns the block total.
__device__ __forceinline__ int64_t block_exclusive(int64_t v, int64_t* total) {
  __shared__ int64_t warp_sums[32];
  __shared__ int64_t block_total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t inc = warp_inclusive(v);
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int nw = (blockDim.x + 31) >> 5;
    int64_t s = lane < nw ? warp_sums[lane] : 0;
    int64_t si = warp_inclusive(s);
    if (lane < nw) warp_sums[lane] = si - s;
    if (lane == nw - 1) block_total = si;  // nw <= 32
  }
  __syncthreads();
  int64_t out = warp_sums[warp] + inc - v;
  *total = block_total;
  __syncthreads();
  return out;
}

__global__ void tile_sums(const int64_t* __restrict__ in, int64_t n, int64_t* __restrict__ sums) {
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  int64_t acc = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = base + (int64_t)i * kScanThreads + threadIdx.x;
    if (idx < n) acc += in[idx];
  }
  int64_t total;
  block_exclusive(acc, &total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

// Single CTA: exclusive scan of the tile sums in place, total at sums[n_tiles].
__global__ void scan_tile_sums(int64_t* sums, int64_t n_tiles) {
  int64_t carry = 0;
  for (int64_t base = 0; base < n_tiles; base += kScanThreads) {
    int64_t idx = base + threadIdx.x;
    int64_t v = idx < n_tiles ? sums[idx] : 0;
    int64_t total;
    int64_t ex = block_exclusive(v, &total);
    if (idx < n_tiles) sums[idx] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) sums[n_tiles] = carry;
}

__global__ void tile_scan(const int64_t* in, int64_t n, const int64_t* __restrict__ tile_off, int64_t* out) {
  int64_t base = (int64_t)blockIdx.x * kScanTile;
  // each thread owns kScanItems consecutive items
  int64_t first = base + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t acc = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = first + i;
    v[i] = idx < n ? in[idx] : 0;
    acc += v[i];
  }
  int64_t total;
  int64_t ex = block_exclusive(acc, &total) + tile_off[blockIdx.x];
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    int64_t idx = first + i;
    if (idx < n) out[idx] = ex;
    ex += v[i];
  }
}

__global__ void write_total(const int64_t* tile_off, int64_t n_tiles, int64_t* out, int64_t n) {
  out[n] = tile_off[n_tiles];
}

}  // namespace

extern "C" int64_t edg_scan_scratch_elems(int64_t n) { return edg::ceil_div(n > 0 ? n : 1, kScanTile) + 1; }

extern "C" int edg_scan_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* scratch, cudaStream_t stream) {
  EDG_REQUIRE(n >= 0, "edg_scan_i64: negative length");
  EDG_REQUIRE(out != nullptr && scratch != nullptr && (n == 0 || in != nullptr), "edg_scan_i64: null pointer");
  int64_t n_tiles = edg::ceil_div(n > 0 ? n : 1, kScanTile);
  if (n > 0) {
    tile_sums<<<(unsigned)n_tiles, kScanThreads, 0, stream>>>(in, n, scratch);
  } else {
    cudaMemsetAsync(scratch, 0, sizeof(int64_t), stream);
  }
  scan_tile_sums<<<1, kScanThreads, 0, stream>>>(scratch, n_tiles);
  // tile_scan reads `in` tile by tile before writing the same tile of `out`,
  // so in-place use (in == out) is safe: tiles are disjoint.
  if (n > 0) tile_scan<<<(unsigned)n_tiles, kScanThreads, 0, stream>>>(in, n, scratch, out);
  write_total<<<1, 1, 0, stream>>>(scratch, n_tiles, out, n);
  EDG_CHECK_LAUNCH("edg_scan_i64");
  return EDG_OK;
}
