// Dense form of the canonical sector matrix, for full diagonalisation.
//
// QMB_hamiltonian.convert_hamiltonian("dense") followed by array_eigh
// (edlgt/modeling/qmb_hamiltonian.py:227-258, 300-302) turns the sparse
// Hamiltonian into a dense array before eigh.  Here each thread writes one
// row of the off-diagonal CSR plus its diagonal entry into a zeroed
// row-major (n, n) array; the eigendecomposition itself is a library call.
#include "internal.cuh"

namespace {

constexpr int kThreads = 256;

template <typename T>
__device__ __forceinline__ void add_to(T& a, T b);
template <>
__device__ __forceinline__ void add_to<double>(double& a, double b) { a += b; }
template <>
__device__ __forceinline__ void add_to<double2>(double2& a, double2 b) {
  a.x += b.x;
  a.y += b.y;
}

template <typename T>
__global__ void to_dense_k(int64_t n, const int64_t* __restrict__ rowptr, const int32_t* __restrict__ cols,
                           const T* __restrict__ vals, const T* __restrict__ diag, T* __restrict__ out,
                           int32_t* __restrict__ err) {
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    T* row = out + r * n;
    for (int64_t p = rowptr[r]; p < rowptr[r + 1]; ++p) {
      const int64_t c = cols[p];
      if (c < 0 || c >= n) {
        atomicExch(err, 1);
        continue;
      }
      add_to(row[c], vals[p]);
    }
    add_to(row[r], diag[r]);
  }
}

}  // namespace

extern "C" int edg_csr_to_dense(int32_t dtype, int64_t n, const int64_t* rowptr, const int32_t* cols,
                                const void* vals, const void* diag, void* out, int32_t* err_flag,
                                cudaStream_t stream) {
  EDG_REQUIRE(dtype == 0 || dtype == 2, "edg_csr_to_dense: dtype 0 (f64) or 2 (complex128)");
  EDG_REQUIRE(n >= 0 && n <= (1LL << 31) && rowptr && diag && out && err_flag, "edg_csr_to_dense: bad argument");
  const size_t esz = dtype == 2 ? 16 : 8;
  cudaError_t e = cudaMemsetAsync(out, 0, esz * (size_t)n * (size_t)n, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(err_flag, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_csr_to_dense: clear");
  if (n == 0) return EDG_OK;
  const unsigned grid = edg::grid_for(n, kThreads);
  if (dtype == 0)
    to_dense_k<double><<<grid, kThreads, 0, stream>>>(n, rowptr, cols, (const double*)vals, (const double*)diag,
                                                      (double*)out, err_flag);
  else
    to_dense_k<double2><<<grid, kThreads, 0, stream>>>(n, rowptr, cols, (const double2*)vals, (const double2*)diag,
                                                       (double2*)out, err_flag);
  EDG_CHECK_LAUNCH("edg_csr_to_dense");
  int32_t h = 0;
  e = cudaMemcpyAsync(&h, err_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_csr_to_dense: flag read");
  if (h) {
    edg::set_error("edg_csr_to_dense: a column index is out of range");
    return EDG_ERR_ARG;
  }
  return EDG_OK;
}
