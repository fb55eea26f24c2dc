// CSR + diagonal matvec kernels: y = (A_offdiag + diag) x for nvec right-hand
// sides stored interleaved ([row][vec]), with a shared off-diagonal matrix.
// G threads cooperate on one row (G = 4..32, chosen from the mean row
// length); products are accumulated in double precision.
#pragma once
#include "internal.cuh"

namespace edg {

struct cd {  // double complex accumulator
  double re, im;
};

// Scalar storage traits: real (double/float) or complex (double2/float2).
template <typename S>
struct Store;
template <>
struct Store<double> {
  using acc = double;
  using acc_t = double;
  static constexpr bool cplx = false;
  __device__ static double zero() { return 0.0; }
  __device__ static double ld(const double* p, int64_t i) { return __ldg(p + i); }
  __device__ static void st(double* p, int64_t i, double v) { p[i] = v; }
};
template <>
struct Store<float> {
  using acc = double;
  using acc_t = double;
  static constexpr bool cplx = false;
  __device__ static double zero() { return 0.0; }
  __device__ static double ld(const float* p, int64_t i) { return (double)__ldg(p + i); }
  __device__ static void st(float* p, int64_t i, double v) { p[i] = (float)v; }
};
template <>
struct Store<double2> {
  using acc = cd;
  using acc_t = cd;
  static constexpr bool cplx = true;
  __device__ static cd zero() { return {0.0, 0.0}; }
  __device__ static cd ld(const double2* p, int64_t i) {
    double2 v = __ldg(p + i);
    return {v.x, v.y};
  }
  __device__ static void st(double2* p, int64_t i, cd v) { p[i] = make_double2(v.re, v.im); }
};
template <>
struct Store<float2> {
  using acc = cd;
  using acc_t = cd;
  static constexpr bool cplx = true;
  __device__ static cd zero() { return {0.0, 0.0}; }
  __device__ static cd ld(const float2* p, int64_t i) {
    float2 v = __ldg(p + i);
    return {(double)v.x, (double)v.y};
  }
  __device__ static void st(float2* p, int64_t i, cd v) { p[i] = make_float2((float)v.re, (float)v.im); }
};

__device__ __forceinline__ void fma_acc(double& a, double v, double x) { a = fma(v, x, a); }
// real matrix entry times complex vector entry
__device__ __forceinline__ void fma_acc(cd& a, double v, cd x) {
  a.re = fma(v, x.re, a.re);
  a.im = fma(v, x.im, a.im);
}
__device__ __forceinline__ void fma_acc(cd& a, cd v, cd x) {
  a.re = fma(v.re, x.re, fma(-v.im, x.im, a.re));
  a.im = fma(v.re, x.im, fma(v.im, x.re, a.im));
}
__device__ __forceinline__ void zero_acc(double& a) { a = 0.0; }
__device__ __forceinline__ void zero_acc(cd& a) { a.re = a.im = 0.0; }
template <int G>
__device__ __forceinline__ void group_reduce(double& a) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o, G);
}
template <int G>
__device__ __forceinline__ void group_reduce(cd& a) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    a.re += __shfl_xor_sync(0xffffffffu, a.re, o, G);
    a.im += __shfl_xor_sync(0xffffffffu, a.im, o, G);
  }
}

// One row of x (NV entries at stride XS): a single 16-byte (f32) or two
// 16-byte (f64) loads when the rows are padded to four entries, else one
// load per entry.
template <typename SX, int NV, int XS>
struct RowX {
  __device__ static void ld(const SX* x, int64_t c, typename Store<SX>::acc (&out)[NV]) {
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = Store<SX>::ld(x, c * XS + v);
  }
};
template <int NV>
struct RowX<float, NV, 4> {
  __device__ static void ld(const float* x, int64_t c, double (&out)[NV]) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(x) + c);
    const float f[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = (double)f[v];
  }
};
template <int NV>
struct RowX<double, NV, 4> {
  __device__ static void ld(const double* x, int64_t c, double (&out)[NV]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(x) + 2 * c);
    const double2 b = __ldg(reinterpret_cast<const double2*>(x) + 2 * c + 1);
    const double f[4] = {a.x, a.y, b.x, b.y};
#pragma unroll
    for (int v = 0; v < NV; ++v) out[v] = f[v];
  }
};

// SV: matrix value/diag storage, SX: x storage, SY: y storage.  The
// accumulator is complex when either the matrix or the vector is.
template <typename SV, typename SX>
struct AccOf {
  using type = typename Store<SX>::acc;
};
template <>
struct AccOf<double2, double> {
  using type = cd;
};
template <>
struct AccOf<float2, float> {
  using type = cd;
};

template <typename SV, typename SX, typename SY, int NV, int G, int XS>
__global__ void __launch_bounds__(256) spmv_k(int64_t n, const int64_t* __restrict__ rowptr,
                                              const int32_t* __restrict__ cols, const SV* __restrict__ vals,
                                              const SV* __restrict__ diag, const SX* __restrict__ x,
                                              SY* __restrict__ y, int64_t y_plane, const int* __restrict__ skip) {
  using A = typename AccOf<SV, SX>::type;
  if (skip != nullptr && *skip) return;  // a device-driven solver has finished
  const int lane = threadIdx.x & (G - 1);
  const int64_t group = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / G;
  const int64_t n_groups = ((int64_t)gridDim.x * blockDim.x) / G;
  // every lane of a warp iterates the same number of times (shuffles need it)
  const int64_t n_iter = (n + n_groups - 1) / n_groups;
  for (int64_t it = 0; it < n_iter; ++it) {
    const int64_t r = group + it * n_groups;
    A acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) zero_acc(acc[v]);
    if (r < n) {
      const int64_t beg = __ldg(rowptr + r), end = __ldg(rowptr + r + 1);
      // four entries of the lane at a time: their columns and values are
      // loaded first, then all gathers of x are in flight together (the
      // accumulation order is the entry order, as in a one-at-a-time loop)
      constexpr int U = 4;
      for (int64_t p0 = beg + lane; p0 < end; p0 += U * G) {
        int64_t c[U];
        typename Store<SV>::acc_t a[U];
#pragma unroll
        for (int k = 0; k < U; ++k) {
          const int64_t p = p0 + (int64_t)k * G;
          c[k] = p < end ? (int64_t)__ldg(cols + p) : r;
          a[k] = p < end ? Store<SV>::ld(vals, p) : Store<SV>::zero();
        }
#pragma unroll
        for (int k = 0; k < U; ++k)
          if (p0 + (int64_t)k * G < end) {
            typename Store<SX>::acc xr[NV];
            RowX<SX, NV, XS>::ld(x, c[k], xr);
#pragma unroll
            for (int v = 0; v < NV; ++v) fma_acc(acc[v], a[k], xr[v]);
          }
      }
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) group_reduce<G>(acc[v]);
    if (r < n && lane == 0) {
      typename Store<SX>::acc xr[NV];
      RowX<SX, NV, XS>::ld(x, r, xr);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        fma_acc(acc[v], Store<SV>::ld(diag, r * NV + v), xr[v]);
        Store<SY>::st(y, y_plane > 0 ? v * y_plane + r : r * NV + v, acc[v]);
      }
    }
  }
}

// Threads per row from the mean row length (used when no tuned choice is given).
inline int spmv_group(int64_t n, int64_t nnz) {
  double avg = n > 0 ? (double)nnz / (double)n : 0.0;
  if (avg < 3) return 2;
  if (avg < 6) return 4;
  if (avg < 20) return 8;
  if (avg < 48) return 16;
  return 32;
}

// y_plane > 0 writes y planar (y[v * y_plane + r]) instead of interleaved;
// group = threads per row (2, 4, 8, 16, 32) or 0 for the heuristic.
template <typename SV, typename SX, typename SY, int NV, int XS>
int launch_spmv_xs(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* cols, const SV* vals,
                   const SV* diag, const SX* x, SY* y, cudaStream_t s, int64_t y_plane, int group, const int* skip) {
  const int threads = 256;
  int g = group > 0 ? group : spmv_group(n, nnz);
  // one row per thread group: enough resident groups to hide the gather latency
  int64_t blocks = ceil_div(n * g, threads);
  unsigned grid = (unsigned)(blocks < (int64_t)kSmCount * 256 ? blocks : (int64_t)kSmCount * 256);
  switch (g) {
    case 2: spmv_k<SV, SX, SY, NV, 2, XS><<<grid, threads, 0, s>>>(n, rowptr, cols, vals, diag, x, y, y_plane, skip); break;
    case 4: spmv_k<SV, SX, SY, NV, 4, XS><<<grid, threads, 0, s>>>(n, rowptr, cols, vals, diag, x, y, y_plane, skip); break;
    case 8: spmv_k<SV, SX, SY, NV, 8, XS><<<grid, threads, 0, s>>>(n, rowptr, cols, vals, diag, x, y, y_plane, skip); break;
    case 16: spmv_k<SV, SX, SY, NV, 16, XS><<<grid, threads, 0, s>>>(n, rowptr, cols, vals, diag, x, y, y_plane, skip); break;
    default: spmv_k<SV, SX, SY, NV, 32, XS><<<grid, threads, 0, s>>>(n, rowptr, cols, vals, diag, x, y, y_plane, skip); break;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "spmv");
  return EDG_OK;
}

template <typename SV, typename SX, typename SY, int NV>
int launch_spmv_nv(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* cols, const SV* vals,
                   const SV* diag, const SX* x, SY* y, cudaStream_t s, int64_t y_plane = 0, int group = 0,
                   const int* skip = nullptr, int x_stride = NV) {
  if constexpr (NV == 3 && !Store<SX>::cplx) {
    // rows of x padded to four entries: one aligned vector load per gather
    if (x_stride == 4)
      return launch_spmv_xs<SV, SX, SY, NV, 4>(n, nnz, rowptr, cols, vals, diag, x, y, s, y_plane, group, skip);
  }
  return launch_spmv_xs<SV, SX, SY, NV, NV>(n, nnz, rowptr, cols, vals, diag, x, y, s, y_plane, group, skip);
}

template <typename SV, typename SX, typename SY>
int launch_spmv(int nvec, int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* cols, const SV* vals,
                const SV* diag, const SX* x, SY* y, cudaStream_t s, int64_t y_plane = 0, int group = 0,
                const int* skip = nullptr, int x_stride = 0) {
  if (group != 0 && group != 2 && group != 4 && group != 8 && group != 16 && group != 32) {
    set_error("spmv: group must be 0, 2, 4, 8, 16 or 32, got %d", group);
    return EDG_ERR_ARG;
  }
  switch (nvec) {
    case 1: return launch_spmv_nv<SV, SX, SY, 1>(n, nnz, rowptr, cols, vals, diag, x, y, s, y_plane, group, skip,
                                                       x_stride ? x_stride : 1);
    case 2: return launch_spmv_nv<SV, SX, SY, 2>(n, nnz, rowptr, cols, vals, diag, x, y, s, y_plane, group, skip,
                                                       x_stride ? x_stride : 2);
    case 3: return launch_spmv_nv<SV, SX, SY, 3>(n, nnz, rowptr, cols, vals, diag, x, y, s, y_plane, group, skip,
                                                       x_stride ? x_stride : 3);
    case 4: return launch_spmv_nv<SV, SX, SY, 4>(n, nnz, rowptr, cols, vals, diag, x, y, s, y_plane, group, skip,
                                                       x_stride ? x_stride : 4);
    default: set_error("spmv: nvec must be 1..4, got %d", nvec); return EDG_ERR_ARG;
  }
}

// Sliced ELL (SELL-32-sigma) matvec of the f32 Krylov path (sell.cu):
// y[v * y_plane + row] = (A + diag) x, x rows at stride x_stride.
int launch_sell_spmv(int nvec, int x_stride, int64_t n_slices, const int32_t* perm, const int32_t* width,
                     const int64_t* off, const uint2* entries, const float* diag, const float* x, double* y,
                     int64_t y_plane, const int* skip, cudaStream_t s);

// Dictionary-packed tiled matvec (packed.cu): y[v * y_plane + row] (f64;
// interleaved y[row * nvec + v] when y_plane is 0) = (A + diag) x, entries
// col | (value index << colbits), T = f32 or f64; diag_shared: one diagonal
// value per row for all nvec (a complex vector of a real matrix); a stage
// wait that runs out writes EDG_ERR_TIMEOUT to *err (if not null).
template <typename T>
int launch_packed_spmv(int nvec, int x_stride, int64_t n, const int32_t* tile_off, const uint32_t* words,
                       const T* table, int count, int colbits, const T* diag, const T* x, double* y, int64_t y_plane,
                       const int* skip, int* err, cudaStream_t s, int diag_shared = 0);

}  // namespace edg
