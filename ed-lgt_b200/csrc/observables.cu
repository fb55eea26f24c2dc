// Diagonal (local) observables: out[s] += sum_r |psi_r|^2 * diag[s][c_s(r)] for
// every site s at once.  This is LocalTerm.get_expval in a symmetry sector
// (edlgt/modeling/local_term.py:119-237 with exp_val_data,
// edlgt/modeling/qmb_state.py:631-654): local terms only keep the operator
// diagonal, so an expectation value is a weighted reduction over the basis.
#include "internal.cuh"

namespace {

constexpr int kThreads = 256;

template <int PT>
__device__ __forceinline__ double prob(const void* psi, int64_t r, int64_t stride) {
  if (PT == 0) {
    double a = ((const double*)psi)[r * stride];
    return a * a;
  } else if (PT == 1) {
    double a = ((const float*)psi)[r * stride];
    return a * a;
  } else if (PT == 2) {
    double2 a = ((const double2*)psi)[r * stride];
    return a.x * a.x + a.y * a.y;
  } else {
    float2 a = ((const float2*)psi)[r * stride];
    return (double)a.x * a.x + (double)a.y * a.y;
  }
}

// W = 1: one-word keys; W = 2: two-word keys (low word first) whose high
// word holds sites [0, n_hi).
template <int PT, int W>
__global__ void __launch_bounds__(kThreads) local_expval_k(const uint64_t* __restrict__ keys, int64_t n, int n_hi, int n_sites,
                                                           edg_site_dims dims, const void* __restrict__ psi,
                                                           int64_t psi_stride, const double* __restrict__ diag,
                                                           int dmax, double* __restrict__ out) {
  __shared__ double acc[EDG_MAX_SITES];
  for (int s = threadIdx.x; s < n_sites; s += kThreads) acc[s] = 0.0;
  __syncthreads();
  double loc[EDG_MAX_SITES];
  for (int s = 0; s < n_sites; ++s) loc[s] = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    const double p2 = prob<PT>(psi, r, psi_stride);
    uint64_t k = keys[W * r];
    const int split = W == 2 ? n_hi : 0;
    for (int s = n_sites - 1; s >= split; --s) {
      uint64_t d = (uint64_t)dims.d[s];
      int c = (int)(k % d);
      k /= d;
      loc[s] = fma(p2, diag[s * dmax + c], loc[s]);
    }
    if (W == 2) {
      k = keys[2 * r + 1];
      for (int s = split - 1; s >= 0; --s) {
        uint64_t d = (uint64_t)dims.d[s];
        int c = (int)(k % d);
        k /= d;
        loc[s] = fma(p2, diag[s * dmax + c], loc[s]);
      }
    }
  }
  for (int s = 0; s < n_sites; ++s) {
    double v = loc[s];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&acc[s], v);
  }
  __syncthreads();
  for (int s = threadIdx.x; s < n_sites; s += kThreads) atomicAdd(out + s, acc[s]);
}

template <int W>
int local_expval(const uint64_t* keys, int64_t n, int32_t n_hi, const edg_site_dims* dims, int32_t n_sites,
                 const void* psi, int32_t psi_dtype, int64_t psi_stride, const double* diag, int32_t dmax, double* out,
                 cudaStream_t stream) {
  EDG_REQUIRE(dims != nullptr && n >= 0 && n_sites > 0 && n_sites <= EDG_MAX_SITES && dmax > 0 && psi_stride >= 1,
              "edg_local_expval: bad arguments");
  EDG_REQUIRE(W == 1 || (n_hi > 0 && n_hi < n_sites), "edg_local_expval_wide: n_hi out of range");
  EDG_REQUIRE(psi_dtype >= 0 && psi_dtype <= 3, "edg_local_expval: psi_dtype must be 0..3");
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * n_sites, stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_local_expval: reset");
  if (n == 0) return EDG_OK;
  const unsigned g = edg::grid_for(n, kThreads, 4);
  switch (psi_dtype) {
    case 0: local_expval_k<0, W><<<g, kThreads, 0, stream>>>(keys, n, n_hi, n_sites, *dims, psi, psi_stride, diag, dmax, out); break;
    case 1: local_expval_k<1, W><<<g, kThreads, 0, stream>>>(keys, n, n_hi, n_sites, *dims, psi, psi_stride, diag, dmax, out); break;
    case 2: local_expval_k<2, W><<<g, kThreads, 0, stream>>>(keys, n, n_hi, n_sites, *dims, psi, psi_stride, diag, dmax, out); break;
    default: local_expval_k<3, W><<<g, kThreads, 0, stream>>>(keys, n, n_hi, n_sites, *dims, psi, psi_stride, diag, dmax, out); break;
  }
  EDG_CHECK_LAUNCH("edg_local_expval");
  return EDG_OK;
}

}  // namespace

extern "C" int edg_local_expval(const uint64_t* keys, int64_t n, const edg_site_dims* dims, int32_t n_sites,
                                const void* psi, int32_t psi_dtype, int64_t psi_stride, const double* diag,
                                int32_t dmax, double* out, cudaStream_t stream) {
  return local_expval<1>(keys, n, 0, dims, n_sites, psi, psi_dtype, psi_stride, diag, dmax, out, stream);
}

extern "C" int edg_local_expval_wide(const uint64_t* keys, int64_t n, int32_t n_hi, const edg_site_dims* dims,
                                     int32_t n_sites, const void* psi, int32_t psi_dtype, int64_t psi_stride,
                                     const double* diag, int32_t dmax, double* out, cudaStream_t stream) {
  return local_expval<2>(keys, n, n_hi, dims, n_sites, psi, psi_dtype, psi_stride, diag, dmax, out, stream);
}
