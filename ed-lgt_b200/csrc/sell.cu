// Sliced ELL matvec (SELL-32-sigma) with packed entries.
//
// The off-diagonal CSR matrix is re-laid out once: rows are sorted by length
// (descending, stable) inside windows of kSellWindow rows, cut into slices of
// 32 consecutive sorted rows, and each slice stores its entries column-major:
// entry k of the slice's 32 rows is 32 consecutive 8-byte (column, value)
// pairs.  In the matvec one lane owns one row of a slice, so every load of the
// entry stream is one 256-byte contiguous warp access (the CSR kernel's loads
// of columns and values touch one segment per row of the warp), and only the
// x gathers stay scattered.  Rows shorter than their slice's width are padded
// with (column -1, value 0) entries, which the matvec loads but does not
// gather.  The sort window sigma trades padding (a long window) against the
// locality of the x gathers (neighbouring rows of the basis order touch
// neighbouring columns, which the L1 cache serves): sigma = 32 keeps the basis
// order.  perm[sorted position] gives the original row (-1 for the slice
// padding of the last window); y and the diagonal are addressed through it.
#include "spmv.cuh"

namespace {

constexpr int kSellWindowMax = 4096;  // longest sorting window (128 slices)
constexpr int kLenBuckets = 256;   // lengths >= 255 share the last bucket

// One CTA per window: stable counting sort of its rows by length, descending.
// The bucket of every row is staged in shared memory and the histogram is
// parallel; thread 0 then places the rows in row order (deterministic).
__global__ void __launch_bounds__(256) sell_sort_k(const int64_t* __restrict__ rowptr, int64_t n, int window,
                                                   int32_t* __restrict__ perm, int32_t* __restrict__ width,
                                                   int64_t* __restrict__ counts) {
  __shared__ int hist[kLenBuckets];
  __shared__ unsigned char bucket[kSellWindowMax];
  const int64_t w0 = (int64_t)blockIdx.x * window;
  const int64_t w1 = w0 + window < n ? w0 + window : n;
  for (int b = threadIdx.x; b < kLenBuckets; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  for (int64_t r = w0 + threadIdx.x; r < w1; r += blockDim.x) {
    const int64_t len = rowptr[r + 1] - rowptr[r];
    const int b = len < kLenBuckets - 1 ? (int)len : kLenBuckets - 1;
    bucket[r - w0] = (unsigned char)b;
    atomicAdd(&hist[b], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int b = kLenBuckets - 1; b >= 0; --b) {  // descending lengths; hist becomes the start
      const int h = hist[b];
      hist[b] = acc;
      acc += h;
    }
    for (int64_t r = w0; r < w1; ++r) perm[w0 + hist[bucket[r - w0]]++] = (int32_t)r;
  }
  __syncthreads();
  // slice padding of the last window, then every slice's width (its first
  // row is its longest)
  const int64_t w_end = w0 + window;
  for (int64_t q = w1 + threadIdx.x; q < w_end && q < (n + 31) / 32 * 32; q += blockDim.x) perm[q] = -1;
  __syncthreads();
  for (int64_t sl = w0 / 32 + threadIdx.x; sl * 32 < w1; sl += blockDim.x) {
    const int32_t r = perm[sl * 32];
    width[sl] = (int32_t)(rowptr[r + 1] - rowptr[r]);
    counts[sl] = 32 * (rowptr[r + 1] - rowptr[r]);
  }
}

// entries of slice sl: (column, value bits) for k < width, lane-major inside
// each k; off[sl] = first entry (in pairs) of the slice
template <typename V>
__global__ void sell_fill_k(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                            const V* __restrict__ vals, int64_t n_slices, const int32_t* __restrict__ perm,
                            const int32_t* __restrict__ width, const int64_t* __restrict__ off,
                            uint2* __restrict__ entries) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_slices * 32;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t sl = t >> 5;
    const int lane = (int)(t & 31);
    const int32_t r = perm[t];
    const int w = width[sl];
    const int64_t beg = r >= 0 ? rowptr[r] : 0, len = r >= 0 ? rowptr[r + 1] - beg : 0;
    uint2* e = entries + off[sl];
    for (int k = 0; k < w; ++k) {
      uint2 p = make_uint2(0xFFFFFFFFu, 0u);  // padding: no gather
      if (k < len) {
        p.x = (unsigned)cols[beg + k];
        p.y = __float_as_uint((float)vals[beg + k]);
      }
      e[(int64_t)k * 32 + lane] = p;
    }
  }
}

// y (planar, y[v * y_plane + row]) = (A + diag) x for NV problems with
// interleaved x rows at stride XS; one lane per row, four entries of the
// stream in flight per lane, f64 accumulation.
template <typename SX, int NV, int XS>
__global__ void __launch_bounds__(256) sell_spmv_k(int64_t n_slices, const int32_t* __restrict__ perm,
                                                   const int32_t* __restrict__ width, const int64_t* __restrict__ off,
                                                   const uint2* __restrict__ entries, const float* __restrict__ diag,
                                                   const SX* __restrict__ x, double* __restrict__ y, int64_t y_plane,
                                                   const int* __restrict__ skip) {
  if (skip != nullptr && *skip) return;
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t sl = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; sl < n_slices; sl += warps) {
    const int32_t r = __ldg(perm + sl * 32 + lane);
    const int w = __ldg(width + sl);
    const uint2* e = entries + __ldg(off + sl) + lane;
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
    constexpr int U = 4;
    for (int k0 = 0; k0 < w; k0 += U) {
      uint2 p[U];
#pragma unroll
      for (int u = 0; u < U; ++u) p[u] = k0 + u < w ? __ldg(e + (int64_t)(k0 + u) * 32) : make_uint2(0xFFFFFFFFu, 0u);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (p[u].x != 0xFFFFFFFFu) {
          double xr[NV];
          edg::RowX<SX, NV, XS>::ld(x, (int64_t)p[u].x, xr);
          const double a = (double)__uint_as_float(p[u].y);
#pragma unroll
          for (int v = 0; v < NV; ++v) acc[v] = fma(a, xr[v], acc[v]);
        }
      }
    }
    if (r >= 0) {
      double xr[NV];
      edg::RowX<SX, NV, XS>::ld(x, (int64_t)r, xr);
#pragma unroll
      for (int v = 0; v < NV; ++v) y[v * y_plane + r] = fma((double)__ldg(diag + (int64_t)r * NV + v), xr[v], acc[v]);
    }
  }
}

}  // namespace

namespace edg {

int launch_sell_spmv(int nvec, int x_stride, int64_t n_slices, const int32_t* perm, const int32_t* width,
                     const int64_t* off, const uint2* entries, const float* diag, const float* x, double* y,
                     int64_t y_plane, const int* skip, cudaStream_t s) {
  const unsigned grid = edg::grid_for(n_slices * 32, 256, 8);
#define EDG_SELL(NV, XS) sell_spmv_k<float, NV, XS><<<grid, 256, 0, s>>>(n_slices, perm, width, off, entries, diag, \
                                                                          x, y, y_plane, skip)
  switch (nvec) {
    case 1: EDG_SELL(1, 1); break;
    case 2: EDG_SELL(2, 2); break;
    case 3:
      if (x_stride == 4)
        EDG_SELL(3, 4);
      else
        EDG_SELL(3, 3);
      break;
    case 4: EDG_SELL(4, 4); break;
    default: set_error("sell spmv: nvec must be 1..4, got %d", nvec); return EDG_ERR_ARG;
  }
#undef EDG_SELL
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "sell spmv");
  return EDG_OK;
}

}  // namespace edg

extern "C" int64_t edg_sell_slices(int64_t n_rows) { return n_rows < 0 ? -1 : (n_rows + 31) / 32; }

extern "C" int edg_sell_order(const int64_t* rowptr, int64_t n_rows, int32_t window, int32_t* perm,
                              int32_t* width, int64_t* counts, cudaStream_t stream) {
  EDG_REQUIRE(n_rows >= 0 && n_rows < INT32_MAX, "edg_sell_order: n_rows out of range");
  EDG_REQUIRE(window >= 32 && window <= kSellWindowMax && window % 32 == 0,
              "edg_sell_order: window must be a multiple of 32 in [32, %d], got %d", kSellWindowMax, window);
  EDG_REQUIRE(rowptr && perm && width && counts, "edg_sell_order: null pointer");
  if (n_rows == 0) return EDG_OK;
  const unsigned windows = (unsigned)((n_rows + window - 1) / window);
  sell_sort_k<<<windows, 256, 0, stream>>>(rowptr, n_rows, window, perm, width, counts);
  EDG_CHECK_LAUNCH("edg_sell_order");
  return EDG_OK;
}

extern "C" int edg_sell_fill(int32_t dtype, const int64_t* rowptr, const int32_t* cols, const void* vals,
                             int64_t n_rows, const int32_t* perm, const int32_t* width, const int64_t* off,
                             void* entries, cudaStream_t stream) {
  EDG_REQUIRE(dtype == 0 || dtype == 1, "edg_sell_fill: dtype must be 0 (f64 values) or 1 (f32 values)");
  EDG_REQUIRE(rowptr && perm && width && off && entries, "edg_sell_fill: null pointer");
  const int64_t n_slices = (n_rows + 31) / 32;
  if (n_slices == 0) return EDG_OK;
  const unsigned grid = edg::grid_for(n_slices * 32, 256);
  if (dtype == 0)
    sell_fill_k<double><<<grid, 256, 0, stream>>>(rowptr, cols, (const double*)vals, n_slices, perm, width, off,
                                                  (uint2*)entries);
  else
    sell_fill_k<float><<<grid, 256, 0, stream>>>(rowptr, cols, (const float*)vals, n_slices, perm, width, off,
                                                 (uint2*)entries);
  EDG_CHECK_LAUNCH("edg_sell_fill");
  return EDG_OK;
}

extern "C" int edg_spmv_sell(int64_t n_rows, int32_t nvec, const int32_t* perm, const int32_t* width,
                             const int64_t* off, const void* entries, const float* diag, const float* x,
                             int32_t x_stride, double* y, int64_t y_plane, cudaStream_t stream) {
  EDG_REQUIRE(n_rows >= 0 && nvec >= 1 && nvec <= 4, "edg_spmv_sell: bad size");
  EDG_REQUIRE(x_stride == nvec || (nvec == 3 && x_stride == 4), "edg_spmv_sell: x_stride must be nvec "
                                                                "(or 4 for nvec = 3)");
  EDG_REQUIRE(perm && width && off && entries && diag && x && y, "edg_spmv_sell: null pointer");
  if (n_rows == 0) return EDG_OK;
  return edg::launch_sell_spmv(nvec, x_stride, (n_rows + 31) / 32, perm, width, off, (const uint2*)entries, diag, x,
                               y, y_plane > 0 ? y_plane : n_rows, nullptr, stream);
}

// CSR matvec in the f32 Krylov path's configuration (f32 values, diagonal
// and x with rows at stride x_stride, f64 planar output), for the autotuner's
// comparison with the SELL layout.
extern "C" int edg_spmv_f32_planar(int64_t n_rows, int64_t nnz, const int64_t* rowptr, const int32_t* cols,
                                   const float* vals, const float* diag, int32_t nvec, const float* x,
                                   int32_t x_stride, double* y, int64_t y_plane, int32_t group, cudaStream_t stream) {
  EDG_REQUIRE(n_rows >= 0 && nnz >= 0 && nvec >= 1 && nvec <= 4, "edg_spmv_f32_planar: bad size");
  EDG_REQUIRE(x_stride == nvec || (nvec == 3 && x_stride == 4), "edg_spmv_f32_planar: x_stride must be nvec "
                                                               "(or 4 for nvec = 3)");
  EDG_REQUIRE(rowptr && diag && x && y && (nnz == 0 || (cols && vals)), "edg_spmv_f32_planar: null pointer");
  if (n_rows == 0) return EDG_OK;
  return edg::launch_spmv<float, float, double>(nvec, n_rows, nnz, rowptr, cols, vals, diag, x, y, stream,
                                                y_plane > 0 ? y_plane : n_rows, group, nullptr, x_stride);
}
