// Bipartitions of a symmetry sector and the state matrix of a bipartition.
//
// QuantumModel._get_partition (edlgt/models/quantum_model.py:715-791) splits
// each sector configuration into its subsystem and environment columns and
// finds the distinct rows of each with _unique_configs_with_inverse
// (quantum_model.py:73-117: np.unique on packed keys, which sorts them).
// Here a part's key is read straight off the sector key, digit by digit, and
// the distinct keys are found without a sort: one bit per possible part key
// in a bitmap, a popcount scan over its words, and each row's index is the
// number of set bits below its key, which is its position in ascending key
// order, the same as np.unique's.  build_psi_matrix
// (edlgt/modeling/qmb_state.py:596-627) becomes one scatter.
#include "internal.cuh"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ uint64_t part_key(uint64_t key, const edg_part_spec& p) {
  uint64_t pk = 0;
  for (int k = 0; k < p.n_part; ++k) pk += ((key / p.src_stride[k]) % p.dim[k]) * p.part_stride[k];
  return pk;
}

__global__ void part_mark_k(const uint64_t* __restrict__ keys, int64_t n, const edg_part_spec p,
                            unsigned long long* __restrict__ bitmap, int64_t* __restrict__ index) {
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    const uint64_t pk = part_key(__ldg(keys + r), p);
    index[r] = (int64_t)pk;
    atomicOr(bitmap + (pk >> 6), 1ull << (pk & 63));
  }
}

__global__ void popc_k(const unsigned long long* __restrict__ bitmap, int64_t words, int64_t* __restrict__ counts) {
  for (int64_t w = (int64_t)blockIdx.x * kThreads + threadIdx.x; w < words; w += (int64_t)gridDim.x * kThreads)
    counts[w] = __popcll(bitmap[w]);
}

// index[r] (the part key) -> rank of that key among the set bits
__global__ void part_rank_k(int64_t n, const unsigned long long* __restrict__ bitmap,
                            const int64_t* __restrict__ offsets, int64_t* __restrict__ index) {
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    const uint64_t pk = (uint64_t)index[r];
    const unsigned long long below = bitmap[pk >> 6] & ((1ull << (pk & 63)) - 1);
    index[r] = offsets[pk >> 6] + __popcll(below);
  }
}

__global__ void part_list_k(const unsigned long long* __restrict__ bitmap, int64_t words,
                            const int64_t* __restrict__ offsets, uint64_t* __restrict__ unique_keys) {
  for (int64_t w = (int64_t)blockIdx.x * kThreads + threadIdx.x; w < words; w += (int64_t)gridDim.x * kThreads) {
    unsigned long long b = bitmap[w];
    int64_t o = offsets[w];
    while (b) {
      const int bit = __ffsll((long long)b) - 1;
      unique_keys[o++] = ((uint64_t)w << 6) | (uint64_t)bit;
      b &= b - 1;
    }
  }
}

template <typename TI, typename TO>
__global__ void psi_matrix_k(const TI* __restrict__ psi, int64_t n, const int64_t* __restrict__ sub,
                             const int64_t* __restrict__ env, int64_t sub_dim, int64_t env_dim, TO* __restrict__ out,
                             int32_t* __restrict__ err) {
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    const int64_t a = sub[r], b = env[r];
    if (a < 0 || a >= sub_dim || b < 0 || b >= env_dim) {
      atomicExch(err, 1);
      continue;
    }
    out[a * env_dim + b] = TO(psi[r]);
  }
}

struct C128 {
  double x, y;
  __device__ C128() {}
  __device__ C128(double r) : x(r), y(0.0) {}
  __device__ C128(float r) : x(r), y(0.0) {}
  __device__ C128(double2 v) : x(v.x), y(v.y) {}
  __device__ C128(float2 v) : x(v.x), y(v.y) {}
};

int64_t words_of(uint64_t key_space) { return (int64_t)((key_space + 63) / 64); }

}  // namespace

extern "C" int64_t edg_part_scratch_elems(uint64_t key_space) {
  if (key_space < 1 || key_space > EDG_PART_MAX_KEY_SPACE) return -1;
  const int64_t w = words_of(key_space);
  return w + (w + 1) + edg_scan_scratch_elems(w);
}

extern "C" int edg_part_map(const uint64_t* keys, int64_t n, const edg_part_spec* spec, int64_t* index,
                            uint64_t* unique_keys, int64_t unique_cap, int64_t* n_unique, uint64_t* scratch,
                            int64_t scratch_elems, cudaStream_t stream) {
  EDG_REQUIRE(spec != nullptr && n_unique != nullptr && scratch != nullptr && n >= 0 &&
                  (n == 0 || (keys != nullptr && index != nullptr)),
              "edg_part_map: null argument");
  EDG_REQUIRE(spec->n_part >= 0 && spec->n_part <= EDG_MAX_SITES, "edg_part_map: n_part out of range");
  uint64_t space = 1;
  for (int k = 0; k < spec->n_part; ++k) {
    EDG_REQUIRE(spec->dim[k] >= 1 && spec->src_stride[k] >= 1, "edg_part_map: bad site %d", k);
    EDG_REQUIRE(spec->part_stride[k] == (k + 1 < spec->n_part ? spec->part_stride[k + 1] * spec->dim[k + 1] : 1),
                "edg_part_map: part strides must be mixed radix, last part site fastest");
    EDG_REQUIRE(space <= EDG_PART_MAX_KEY_SPACE / spec->dim[k], "edg_part_map: part key space above 2^34");
    space *= spec->dim[k];
  }
  EDG_REQUIRE(space == spec->key_space, "edg_part_map: key_space is not the product of the part dims");
  EDG_REQUIRE(scratch_elems >= edg_part_scratch_elems(space), "edg_part_map: scratch too small");
  *n_unique = 0;
  if (n == 0) return EDG_OK;
  const int64_t words = words_of(space);
  unsigned long long* bitmap = reinterpret_cast<unsigned long long*>(scratch);
  int64_t* offsets = reinterpret_cast<int64_t*>(scratch + words);
  int64_t* scan_scratch = offsets + words + 1;
  cudaError_t e = cudaMemsetAsync(bitmap, 0, sizeof(uint64_t) * (size_t)words, stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_part_map: clear");
  part_mark_k<<<edg::grid_for(n, kThreads), kThreads, 0, stream>>>(keys, n, *spec, bitmap, index);
  EDG_CHECK_LAUNCH("edg_part_map: mark");
  popc_k<<<edg::grid_for(words, kThreads), kThreads, 0, stream>>>(bitmap, words, offsets);
  EDG_CHECK_LAUNCH("edg_part_map: popcount");
  int st = edg_scan_i64(offsets, offsets, words, scan_scratch, stream);
  if (st != EDG_OK) return st;
  part_rank_k<<<edg::grid_for(n, kThreads), kThreads, 0, stream>>>(n, bitmap, offsets, index);
  EDG_CHECK_LAUNCH("edg_part_map: rank");
  int64_t total = 0;
  e = cudaMemcpyAsync(&total, offsets + words, sizeof(int64_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_part_map: count read");
  *n_unique = total;
  if (unique_keys != nullptr) {
    EDG_REQUIRE(unique_cap >= total, "edg_part_map: unique_keys holds %lld, %lld needed", (long long)unique_cap,
                (long long)total);
    part_list_k<<<edg::grid_for(words, kThreads), kThreads, 0, stream>>>(bitmap, words, offsets, unique_keys);
    EDG_CHECK_LAUNCH("edg_part_map: list");
  }
  return EDG_OK;
}

extern "C" int edg_psi_matrix(const void* psi, int32_t psi_dtype, int64_t n, const int64_t* sub_index,
                              const int64_t* env_index, int64_t sub_dim, int64_t env_dim, void* out,
                              int32_t out_dtype, int32_t* err_flag, cudaStream_t stream) {
  EDG_REQUIRE(out != nullptr && err_flag != nullptr && n >= 0 &&
                  (n == 0 || (psi != nullptr && sub_index != nullptr && env_index != nullptr)),
              "edg_psi_matrix: null argument");
  EDG_REQUIRE(psi_dtype >= 0 && psi_dtype <= 3 && (out_dtype == 0 || out_dtype == 2),
              "edg_psi_matrix: psi_dtype 0..3, out_dtype 0 (f64) or 2 (complex128)");
  EDG_REQUIRE(out_dtype == 2 || psi_dtype <= 1, "edg_psi_matrix: a complex state needs a complex matrix");
  EDG_REQUIRE(sub_dim >= 1 && env_dim >= 1 && sub_dim <= INT64_MAX / env_dim, "edg_psi_matrix: bad dims");
  const size_t esz = out_dtype == 2 ? 16 : 8;
  cudaError_t e = cudaMemsetAsync(out, 0, esz * (size_t)(sub_dim * env_dim), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(err_flag, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_psi_matrix: clear");
  if (n == 0) return EDG_OK;
  const unsigned grid = edg::grid_for(n, kThreads);
  if (out_dtype == 0) {
    if (psi_dtype == 0)
      psi_matrix_k<double, double><<<grid, kThreads, 0, stream>>>((const double*)psi, n, sub_index, env_index,
                                                                   sub_dim, env_dim, (double*)out, err_flag);
    else
      psi_matrix_k<float, double><<<grid, kThreads, 0, stream>>>((const float*)psi, n, sub_index, env_index,
                                                                  sub_dim, env_dim, (double*)out, err_flag);
  } else {
    C128* o = (C128*)out;
    switch (psi_dtype) {
      case 0: psi_matrix_k<double, C128><<<grid, kThreads, 0, stream>>>((const double*)psi, n, sub_index, env_index, sub_dim, env_dim, o, err_flag); break;
      case 1: psi_matrix_k<float, C128><<<grid, kThreads, 0, stream>>>((const float*)psi, n, sub_index, env_index, sub_dim, env_dim, o, err_flag); break;
      case 2: psi_matrix_k<double2, C128><<<grid, kThreads, 0, stream>>>((const double2*)psi, n, sub_index, env_index, sub_dim, env_dim, o, err_flag); break;
      default: psi_matrix_k<float2, C128><<<grid, kThreads, 0, stream>>>((const float2*)psi, n, sub_index, env_index, sub_dim, env_dim, o, err_flag); break;
    }
  }
  EDG_CHECK_LAUNCH("edg_psi_matrix");
  int32_t h = 0;
  e = cudaMemcpyAsync(&h, err_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_psi_matrix: flag read");
  if (h) {
    edg::set_error("edg_psi_matrix: a row index is outside [0, sub_dim) x [0, env_dim)");
    return EDG_ERR_ARG;
  }
  return EDG_OK;
}
