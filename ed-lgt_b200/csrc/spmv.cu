// Public matvec and dtype-conversion entry points.
#include "spmv.cuh"

namespace {

template <typename A, typename B>
__global__ void convert_k(const A* __restrict__ in, B* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (B)in[i];
}

}  // namespace

extern "C" int edg_spmv(int32_t dtype, int64_t n_rows, int64_t nnz, const int64_t* rowptr, const int32_t* cols,
                        const void* vals, const void* diag, int32_t nvec, const void* x, void* y,
                        cudaStream_t stream) {
  return edg_spmv_group(dtype, n_rows, nnz, rowptr, cols, vals, diag, nvec, x, y, 0, stream);
}

extern "C" int edg_spmv_group(int32_t dtype, int64_t n_rows, int64_t nnz, const int64_t* rowptr,
                              const int32_t* cols, const void* vals, const void* diag, int32_t nvec, const void* x,
                              void* y, int32_t group, cudaStream_t stream) {
  EDG_REQUIRE(n_rows >= 0 && nnz >= 0, "edg_spmv: negative size");
  EDG_REQUIRE(rowptr && diag && x && y && (nnz == 0 || (cols && vals)), "edg_spmv: null pointer");
  if (n_rows == 0) return EDG_OK;
  switch (dtype) {
    case 0:
      return edg::launch_spmv<double, double, double>(nvec, n_rows, nnz, rowptr, cols, (const double*)vals,
                                                      (const double*)diag, (const double*)x, (double*)y, stream, 0, group);
    case 1:
      return edg::launch_spmv<float, float, float>(nvec, n_rows, nnz, rowptr, cols, (const float*)vals,
                                                   (const float*)diag, (const float*)x, (float*)y, stream, 0, group);
    case 2:
      return edg::launch_spmv<double2, double2, double2>(nvec, n_rows, nnz, rowptr, cols, (const double2*)vals,
                                                         (const double2*)diag, (const double2*)x, (double2*)y,
                                                         stream, 0, group);
    case 3:
      return edg::launch_spmv<float2, float2, float2>(nvec, n_rows, nnz, rowptr, cols, (const float2*)vals,
                                                      (const float2*)diag, (const float2*)x, (float2*)y, stream, 0, group);
    default:
      edg::set_error("edg_spmv: unknown dtype %d", dtype);
      return EDG_ERR_ARG;
  }
}

extern "C" int edg_convert(int32_t dtype_in, const void* in, int32_t dtype_out, void* out, int64_t n_scalars,
                           cudaStream_t stream) {
  EDG_REQUIRE(n_scalars >= 0, "edg_convert: negative size");
  if (n_scalars == 0) return EDG_OK;
  // complex arrays are converted as 2*n real scalars by the caller's count
  bool in64 = dtype_in == 0 || dtype_in == 2, out64 = dtype_out == 0 || dtype_out == 2;
  EDG_REQUIRE((dtype_in == 0 || dtype_in == 1) == (dtype_out == 0 || dtype_out == 1), "edg_convert: real/complex mismatch");
  unsigned grid = edg::grid_for(n_scalars, 256);
  if (in64 && !out64)
    convert_k<double, float><<<grid, 256, 0, stream>>>((const double*)in, (float*)out, n_scalars);
  else if (!in64 && out64)
    convert_k<float, double><<<grid, 256, 0, stream>>>((const float*)in, (double*)out, n_scalars);
  else if (in64)
    convert_k<double, double><<<grid, 256, 0, stream>>>((const double*)in, (double*)out, n_scalars);
  else
    convert_k<float, float><<<grid, 256, 0, stream>>>((const float*)in, (float*)out, n_scalars);
  EDG_CHECK_LAUNCH("edg_convert");
  return EDG_OK;
}
