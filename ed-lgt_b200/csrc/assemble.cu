// Sector Hamiltonian assembly, one thread per matrix row (bra state).
//
// For every off-diagonal term instance (a product of up to EDG_MAX_OPS site
// operators) the row enumerates the product of the local transitions of its
// bra states, forms the ket key as bra_key + sum_j (ket_j - bra_j) * stride_j,
// finds the ket row by binary search and emits (col, coef * prod amp).  This
// is the n-body triplet builder of edlgt/symmetries/sym_qmb_operations.py:
// 297-562 with the configuration copy replaced by key arithmetic.  Diagonal
// terms use only the operator diagonal and drop |op_cc| < 1e-10 exactly like
// localbody_data_par (sym_qmb_operations.py:565-602).  Each row's entries are
// then sorted by column and duplicates are summed, which yields the canonical
// (summed) matrix of edlgt/modeling/qmb_hamiltonian.py:196-199.  Kernels are
// templated on the key type (one word, or two words past 63 bits of key
// space: keys.cuh).
#include "lookup.cuh"

namespace {

constexpr double kOpTol = 1e-10;  // OP_TOL of the reference
constexpr int kThreads = 128;

struct Real {
  double v;
  __device__ static Real zero() { return {0.0}; }
  __device__ static Real load(const double* p, int64_t i) { return {p[i]}; }
  __device__ void store(double* p, int64_t i) const { p[i] = v; }
  __device__ Real operator*(const Real& o) const { return {v * o.v}; }
  __device__ Real& operator+=(const Real& o) { v += o.v; return *this; }
  __device__ double abs() const { return fabs(v); }
};

struct Cplx {
  double re, im;
  __device__ static Cplx zero() { return {0.0, 0.0}; }
  __device__ static Cplx load(const double* p, int64_t i) { return {p[2 * i], p[2 * i + 1]}; }
  __device__ void store(double* p, int64_t i) const { p[2 * i] = re; p[2 * i + 1] = im; }
  __device__ Cplx operator*(const Cplx& o) const { return {re * o.re - im * o.im, re * o.im + im * o.re}; }
  __device__ Cplx& operator+=(const Cplx& o) { re += o.re; im += o.im; return *this; }
  __device__ double abs() const { return hypot(re, im); }
};

__device__ __forceinline__ void decode_digits(const edg_assembly& a, uint64_t key, uint8_t* dig) {
  for (int s = a.n_sites - 1; s >= 0; --s) {
    uint64_t d = (uint64_t)a.loc_dims[s];
    dig[s] = (uint8_t)(key % d);
    key /= d;
  }
}
__device__ __forceinline__ void decode_digits(const edg_assembly& a, edg::u128 key, uint8_t* dig) {
  const int n_hi = a.sector.n_hi;
  uint64_t w = (uint64_t)key;
  for (int s = a.n_sites - 1; s >= n_hi; --s) {
    uint64_t d = (uint64_t)a.loc_dims[s];
    dig[s] = (uint8_t)(w % d);
    w /= d;
  }
  w = (uint64_t)(key >> 64);
  for (int s = n_hi - 1; s >= 0; --s) {
    uint64_t d = (uint64_t)a.loc_dims[s];
    dig[s] = (uint8_t)(w % d);
    w /= d;
  }
}

template <typename K>
__device__ __forceinline__ int64_t find_row(const edg_lookup_table& t, K q) {
  if constexpr (sizeof(K) == 8)
    return edg::find_key(t, q);
  else
    return edg::find_key_t(t, q);
}

template <typename K>
__global__ void __launch_bounds__(kThreads) count_k(edg_assembly a, int64_t* __restrict__ row_bound) {
  uint8_t dig[EDG_MAX_SITES];
  const int dm = a.dmax;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.sector.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    decode_digits(a, edg::ld_key<K>(a.sector.keys, r), dig);
    int64_t total = 0;
    for (int k = 0; k < a.n_terms; ++k) {
      int nops = a.term_nops[k];
      int64_t prod = 1;
      for (int j = 0; j < nops; ++j) {
        int site = a.term_site[k * EDG_MAX_OPS + j];
        int tab = a.term_table[k * EDG_MAX_OPS + j];
        prod *= a.t_count[tab * dm + dig[site]];
      }
      total += prod;
    }
    row_bound[r] = total;
  }
}

template <typename V, typename K>
__global__ void __launch_bounds__(kThreads) fill_k(edg_assembly a, const int64_t* __restrict__ offsets,
                                                   int32_t* __restrict__ tcols, double* __restrict__ tvals,
                                                   int64_t* __restrict__ row_nnz, double* __restrict__ diag,
                                                   uint8_t* __restrict__ diag_present, int32_t* __restrict__ err) {
  uint8_t dig[EDG_MAX_SITES];
  const int dm = a.dmax;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < a.sector.n;
       r += (int64_t)gridDim.x * blockDim.x) {
    const K key = edg::ld_key<K>(a.sector.keys, r);
    decode_digits(a, key, dig);
    // ---- diagonal terms ----
    V d = V::zero();
    bool present = false;
    for (int k = 0; k < a.n_dterms; ++k) {
      int site = a.dterm_site[k];
      V v = V::load(a.dterm_diag, (int64_t)k * dm + dig[site]);
      if (v.abs() >= kOpTol) {
        present = true;
        d += V::load(a.dterm_coef, k) * v;
      }
    }
    // ---- off-diagonal terms ----
    const int64_t off = offsets[r];
    int64_t n = 0;
    for (int k = 0; k < a.n_terms; ++k) {
      const int nops = a.term_nops[k];
      int site[EDG_MAX_OPS], tab[EDG_MAX_OPS], bra[EDG_MAX_OPS], cnt[EDG_MAX_OPS], idx[EDG_MAX_OPS];
      bool empty = false;
      for (int j = 0; j < nops; ++j) {
        site[j] = a.term_site[k * EDG_MAX_OPS + j];
        tab[j] = a.term_table[k * EDG_MAX_OPS + j];
        bra[j] = dig[site[j]];
        cnt[j] = a.t_count[tab[j] * dm + bra[j]];
        idx[j] = 0;
        empty |= cnt[j] == 0;
      }
      if (empty) continue;
      const V coef = V::load(a.term_coef, k);
      while (true) {
        K kk = key;
        V amp = coef;
        for (int j = 0; j < nops; ++j) {
          int64_t e = ((int64_t)tab[j] * dm + bra[j]) * dm + idx[j];
          int ket = a.t_ket[e];
          amp = amp * V::load(a.t_amp, e);
          kk += edg::key_step<K>((int64_t)(ket - bra[j]) * (int64_t)a.strides[site[j]], site[j], a.sector.n_hi);
        }
        int64_t col = find_row(a.sector, kk);
        if (col < 0) {
          atomicExch(err, EDG_ERR_MISSING_KET);
        } else if (col == r) {
          d += amp;
          present = true;
        } else {
          tcols[off + n] = (int32_t)col;
          amp.store(tvals, off + n);
          ++n;
        }
        // mixed-radix increment, last factor fastest
        int j = nops - 1;
        for (; j >= 0; --j) {
          if (++idx[j] < cnt[j]) break;
          idx[j] = 0;
        }
        if (j < 0) break;
      }
    }
    // ---- sort the row window by column and merge duplicates ----
    for (int64_t i = 1; i < n; ++i) {
      int32_t c = tcols[off + i];
      V v = V::load(tvals, off + i);
      int64_t j = i - 1;
      while (j >= 0 && tcols[off + j] > c) {
        tcols[off + j + 1] = tcols[off + j];
        V::load(tvals, off + j).store(tvals, off + j + 1);
        --j;
      }
      tcols[off + j + 1] = c;
      v.store(tvals, off + j + 1);
    }
    int64_t m = 0;
    for (int64_t i = 0; i < n; ++i) {
      if (m > 0 && tcols[off + m - 1] == tcols[off + i]) {
        V acc = V::load(tvals, off + m - 1);
        acc += V::load(tvals, off + i);
        acc.store(tvals, off + m - 1);
      } else {
        tcols[off + m] = tcols[off + i];
        V::load(tvals, off + i).store(tvals, off + m);
        ++m;
      }
    }
    row_nnz[r] = m;
    d.store(diag, r);
    diag_present[r] = present ? 1 : 0;
  }
}

template <int W>
__global__ void __launch_bounds__(kThreads) compact_k(int64_t n_rows, const int64_t* __restrict__ offsets,
                                                      const int32_t* __restrict__ tcols, const double* __restrict__ tvals,
                                                      const int64_t* __restrict__ rowptr, int32_t* __restrict__ cols,
                                                      double* __restrict__ vals) {
  // one warp per row: coalesced copy of the merged window
  const int lane = threadIdx.x & 31;
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < n_rows; r += nwarps) {
    int64_t src = offsets[r], dst = rowptr[r], m = rowptr[r + 1] - dst;
    for (int64_t i = lane; i < m; i += 32) {
      cols[dst + i] = tcols[src + i];
#pragma unroll
      for (int w = 0; w < W; ++w) vals[(dst + i) * W + w] = tvals[(src + i) * W + w];
    }
  }
}

int check_assembly(const edg_assembly* a, const char* who) {
  EDG_REQUIRE(a != nullptr, "%s: null description", who);
  EDG_REQUIRE(a->n_sites > 0 && a->n_sites <= EDG_MAX_SITES, "%s: n_sites out of range", who);
  EDG_REQUIRE(a->dmax > 0 && a->dmax <= 255, "%s: dmax out of range", who);
  EDG_REQUIRE(a->sector.n >= 0 && a->sector.n < (int64_t(1) << 31), "%s: sector too large for int32 columns", who);
  EDG_REQUIRE(a->n_terms >= 0 && a->n_dterms >= 0, "%s: negative term count", who);
  EDG_REQUIRE(a->sector.key_words >= 0 && a->sector.key_words <= 2, "%s: key_words must be 1 or 2", who);
  EDG_REQUIRE(a->sector.key_words != 2 ||
                  (a->sector.n_hi > 0 && a->sector.n_hi < a->n_sites &&
                   (reinterpret_cast<uintptr_t>(a->sector.keys) & 15) == 0),
              "%s: two-word keys need 0 < n_hi < n_sites and 16-byte aligned keys", who);
  return EDG_OK;
}

}  // namespace

extern "C" int edg_assemble_count(const edg_assembly* a, int64_t* row_bound, cudaStream_t stream) {
  int st = check_assembly(a, "edg_assemble_count");
  if (st) return st;
  if (a->sector.n == 0) return EDG_OK;
  const unsigned grid = edg::grid_for(a->sector.n, kThreads);
  if (a->sector.key_words == 2)
    count_k<edg::u128><<<grid, kThreads, 0, stream>>>(*a, row_bound);
  else
    count_k<uint64_t><<<grid, kThreads, 0, stream>>>(*a, row_bound);
  EDG_CHECK_LAUNCH("edg_assemble_count");
  return EDG_OK;
}

extern "C" int edg_assemble_fill(const edg_assembly* a, const int64_t* offsets, int32_t* tmp_cols, double* tmp_vals,
                                 int64_t* row_nnz, double* diag, uint8_t* diag_present, int32_t* error_flag,
                                 cudaStream_t stream) {
  int st = check_assembly(a, "edg_assemble_fill");
  if (st) return st;
  if (a->sector.n == 0) return EDG_OK;
  unsigned grid = edg::grid_for(a->sector.n, kThreads);
  const bool wide = a->sector.key_words == 2;
  if (a->complex_values && wide)
    fill_k<Cplx, edg::u128><<<grid, kThreads, 0, stream>>>(*a, offsets, tmp_cols, tmp_vals, row_nnz, diag, diag_present,
                                                            error_flag);
  else if (a->complex_values)
    fill_k<Cplx, uint64_t><<<grid, kThreads, 0, stream>>>(*a, offsets, tmp_cols, tmp_vals, row_nnz, diag, diag_present,
                                                          error_flag);
  else if (wide)
    fill_k<Real, edg::u128><<<grid, kThreads, 0, stream>>>(*a, offsets, tmp_cols, tmp_vals, row_nnz, diag, diag_present,
                                                            error_flag);
  else
    fill_k<Real, uint64_t><<<grid, kThreads, 0, stream>>>(*a, offsets, tmp_cols, tmp_vals, row_nnz, diag, diag_present,
                                                          error_flag);
  EDG_CHECK_LAUNCH("edg_assemble_fill");
  return EDG_OK;
}

extern "C" int edg_assemble_compact(int64_t n_rows, int32_t complex_values, const int64_t* offsets,
                                    const int32_t* tmp_cols, const double* tmp_vals, const int64_t* rowptr,
                                    int32_t* cols, double* vals, cudaStream_t stream) {
  EDG_REQUIRE(n_rows >= 0, "edg_assemble_compact: negative size");
  if (n_rows == 0) return EDG_OK;
  unsigned grid = edg::grid_for(n_rows * 32, kThreads);
  if (complex_values)
    compact_k<2><<<grid, kThreads, 0, stream>>>(n_rows, offsets, tmp_cols, tmp_vals, rowptr, cols, vals);
  else
    compact_k<1><<<grid, kThreads, 0, stream>>>(n_rows, offsets, tmp_cols, tmp_vals, rowptr, cols, vals);
  EDG_CHECK_LAUNCH("edg_assemble_compact");
  return EDG_OK;
}
