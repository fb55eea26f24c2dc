// Momentum (translation) basis of a symmetry sector and the projected matvec.
//
// Follows edlgt/symmetries/translational_sym.py: build_all_translations
// (:567-617) records, for every sector row and every block translation, the
// row of the translated configuration; select_references (:620-694) keeps one
// reference per orbit (the first row of the orbit in sector order, i.e. the
// smallest row index), its period along each axis and whether the momentum is
// compatible with it; momentum_basis_zero_k / _finite_k (:697-949) sum the
// Bloch phases of the period box per orbit row, drop cancelled entries,
// normalise and store the projector B column by column with rows ascending.
//
// Here the translations are key arithmetic plus the bucketed key search, the
// references come from a per-row minimum over the orbit and a scan, and each
// column is one thread's work over at most n_shifts images.  B has at most
// one entry per row (orbits are disjoint), so B x is a gather and B^dagger w a
// per-column sum in a fixed order: H_k = B^dagger H B is applied without
// being formed, around the sector matvec.
#include "internal.cuh"
#include "lookup.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxShifts = EDG_MAX_SITES;

__global__ void translations_k(const edg_lookup_table sec, const uint64_t* __restrict__ strides,
                               const int32_t* __restrict__ loc_dims, int n_sites,
                               const int32_t* __restrict__ source_sites, int n_shifts,
                               const int32_t* __restrict__ local_map, int map_dim,
                               const double* __restrict__ label_sign, double* __restrict__ row_sign,
                               int32_t* __restrict__ trans, int32_t* __restrict__ err) {
  uint8_t dig[EDG_MAX_SITES];
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < sec.n; r += (int64_t)gridDim.x * kThreads) {
    uint64_t x = __ldg(sec.keys + r);
    for (int s = n_sites - 1; s >= 0; --s) {
      const uint64_t d = (uint64_t)__ldg(loc_dims + s);
      const uint64_t q = x / d;
      dig[s] = (uint8_t)(x - q * d);
      x = q;
    }
    if (row_sign != nullptr) {  // product of the local labels' signs
      double sg = 1.0;
      for (int s = 0; s < n_sites; ++s) sg *= dig[s] < map_dim ? __ldg(label_sign + dig[s]) : 1.0;
      row_sign[r] = sg;
    }
    for (int t = 0; t < n_shifts; ++t) {
      uint64_t key = 0;
      const int32_t* src = source_sites + (int64_t)t * n_sites;
      bool ok = true;
      for (int s = 0; s < n_sites; ++s) {
        const int from = __ldg(src + s);
        uint32_t c = dig[from];
        if (local_map != nullptr) {  // the local map applied once per unit shift
          for (int k = 0; k < t; ++k) c = c < (uint32_t)map_dim ? (uint32_t)__ldg(local_map + c) : 0xFFFFu;
        }
        ok = ok && c < (uint32_t)__ldg(loc_dims + s);  // a local state the destination site cannot hold
        key += (uint64_t)c * __ldg(strides + s);
      }
      const int64_t col = ok ? edg::find_key(sec, key) : -1;
      if (col < 0) atomicExch(err, 1);
      trans[r * n_shifts + t] = (int32_t)col;
    }
  }
}

// flag[r] = 1 when r is its orbit's smallest row and the momentum is
// compatible with its axis periods; pvec[r][d] = those periods.
__global__ void references_k(const int32_t* __restrict__ trans, int64_t n, int n_shifts, const edg_momentum_group g,
                             int64_t* __restrict__ flag, int32_t* __restrict__ pvec) {
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    const int32_t* row = trans + r * n_shifts;
    bool is_ref = true;
    for (int t = 0; t < n_shifts; ++t) is_ref = is_ref && row[t] >= r;
    bool keep = is_ref;
    for (int d = 0; d < g.lattice_dim; ++d) {
      const int R = g.shifts_per_dir[d];
      int p = R;
      for (int q = 1; q <= R; ++q) {
        if (row[(q % R) * g.shift_strides[d]] == (int32_t)r) {
          p = q;
          break;
        }
      }
      pvec[r * g.lattice_dim + d] = p;
      keep = keep && ((int64_t)g.k_vals[d] * p) % R == 0;
    }
    flag[r] = keep ? 1 : 0;
  }
}

__global__ void list_refs_k(const int64_t* __restrict__ offsets, int64_t n, int64_t* __restrict__ refs) {
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads)
    if (offsets[r + 1] > offsets[r]) refs[offsets[r]] = r;
}

// One column: the period box of its reference, images deduplicated with
// their summed phases, cancelled entries dropped (finite k), rows ascending.
// Returns the entry count; vals are not yet normalised.
__device__ int column_entries(const int32_t* __restrict__ row, const int32_t* __restrict__ p,
                              const edg_momentum_group& g, const double2* __restrict__ phase_table, int max_r,
                              int zero_k, double odd_sign, int32_t* rows, double2* vals) {
  int t_local[4] = {0, 0, 0, 0};
  int full = 0, len = 0;
  for (;;) {
    double2 ph = make_double2(1.0, 0.0);
    if (!zero_k) {
      for (int d = 0; d < g.lattice_dim; ++d) {
        const double2 f = phase_table[d * max_r + t_local[d]];
        ph = make_double2(ph.x * f.x - ph.y * f.y, ph.x * f.y + ph.y * f.x);
      }
    }
    if (full & 1) ph = make_double2(ph.x * odd_sign, ph.y * odd_sign);
    const int32_t rr = row[full];
    int u = 0;
    while (u < len && rows[u] != rr) ++u;
    if (u == len) {
      rows[len] = rr;
      vals[len] = ph;
      ++len;
    } else {
      vals[u].x += ph.x;
      vals[u].y += ph.y;
    }
    // advance the period-box counter, last axis fastest
    int d = g.lattice_dim - 1;
    for (; d >= 0; --d) {
      ++t_local[d];
      full += g.shift_strides[d];
      if (t_local[d] < p[d]) break;
      full -= t_local[d] * g.shift_strides[d];
      t_local[d] = 0;
    }
    if (d < 0) break;
  }
  if (!zero_k) {
    int kept = 0;
    for (int u = 0; u < len; ++u) {
      if (sqrt(vals[u].x * vals[u].x + vals[u].y * vals[u].y) > 1e-14) {
        rows[kept] = rows[u];
        vals[kept] = vals[u];
        ++kept;
      }
    }
    len = kept;
  }
  for (int i = 1; i < len; ++i) {  // insertion sort by row
    const int32_t rk = rows[i];
    const double2 vk = vals[i];
    int j = i - 1;
    while (j >= 0 && rows[j] > rk) {
      rows[j + 1] = rows[j];
      vals[j + 1] = vals[j];
      --j;
    }
    rows[j + 1] = rk;
    vals[j + 1] = vk;
  }
  return len;
}

__global__ void columns_k(const int32_t* __restrict__ trans, int n_shifts, const int64_t* __restrict__ refs,
                          int64_t n_cols, const int32_t* __restrict__ pvec, const edg_momentum_group g,
                          const double2* __restrict__ phase_table, int max_r, int zero_k,
                          const double* __restrict__ row_sign, int64_t* __restrict__ counts,
                          const int64_t* __restrict__ col_ptr, int32_t* __restrict__ row_idx,
                          double2* __restrict__ data) {
  int32_t rows[kMaxShifts];
  double2 vals[kMaxShifts];
  for (int64_t c = (int64_t)blockIdx.x * kThreads + threadIdx.x; c < n_cols; c += (int64_t)gridDim.x * kThreads) {
    const int64_t ref = refs[c];
    const double odd_sign = row_sign != nullptr ? row_sign[ref] : 1.0;
    const int len = column_entries(trans + ref * n_shifts, pvec + ref * g.lattice_dim, g, phase_table, max_r, zero_k,
                                   odd_sign, rows, vals);
    double norm2 = 0.0;
    for (int u = 0; u < len; ++u) norm2 += vals[u].x * vals[u].x + vals[u].y * vals[u].y;
    // zero k keeps every image (a sign-twisted orbit may still cancel: its
    // column is then written as zeros); finite k drops cancelled images
    const bool empty = zero_k ? norm2 <= 1e-8 : (norm2 <= 1e-30 || len == 0);
    if (counts != nullptr) {
      counts[c] = len;  // the count pass keeps what survived the pruning
      continue;
    }
    if (empty && !zero_k) continue;
    const double inv = empty ? 0.0 : 1.0 / sqrt(norm2);
    int64_t w = col_ptr[c];
    for (int u = 0; u < len; ++u, ++w) {
      row_idx[w] = rows[u];
      data[w] = make_double2(vals[u].x * inv, vals[u].y * inv);
    }
  }
}

__global__ void rowmap_k(const int64_t* __restrict__ col_ptr, const int32_t* __restrict__ row_idx,
                         const double2* __restrict__ data, int64_t n_cols, int64_t n_rows,
                         int64_t* __restrict__ row_col, double2* __restrict__ row_val, int32_t* __restrict__ err) {
  for (int64_t c = (int64_t)blockIdx.x * kThreads + threadIdx.x; c < n_cols; c += (int64_t)gridDim.x * kThreads) {
    for (int64_t p = col_ptr[c]; p < col_ptr[c + 1]; ++p) {
      const int64_t r = row_idx[p];
      if (r < 0 || r >= n_rows) {
        atomicExch(err, 2);
        continue;
      }
      const unsigned long long prev =
          atomicCAS(reinterpret_cast<unsigned long long*>(row_col + r), (unsigned long long)-1LL, (unsigned long long)c);
      if (prev != (unsigned long long)-1LL) {
        atomicExch(err, 1);
        continue;
      }
      row_val[r] = data[p];
    }
  }
}

__global__ void expand_k(int64_t n_rows, const int64_t* __restrict__ row_col, const double2* __restrict__ row_val,
                         const double2* __restrict__ x, double2* __restrict__ v) {
  for (int64_t r = (int64_t)blockIdx.x * kThreads + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * kThreads) {
    const int64_t c = row_col[r];
    double2 o = make_double2(0.0, 0.0);
    if (c >= 0) {
      const double2 b = row_val[r], xc = x[c];
      o = make_double2(b.x * xc.x - b.y * xc.y, b.x * xc.y + b.y * xc.x);
    }
    v[r] = o;
  }
}

__global__ void reduce_k(int64_t n_cols, const int64_t* __restrict__ col_ptr, const int32_t* __restrict__ row_idx,
                         const double2* __restrict__ data, const double2* __restrict__ w, double2* __restrict__ y) {
  for (int64_t c = (int64_t)blockIdx.x * kThreads + threadIdx.x; c < n_cols; c += (int64_t)gridDim.x * kThreads) {
    double re = 0.0, im = 0.0;
    for (int64_t p = col_ptr[c]; p < col_ptr[c + 1]; ++p) {
      const double2 b = data[p], wv = w[row_idx[p]];
      re = fma(b.x, wv.x, fma(b.y, wv.y, re));  // conj(b) * w
      im = fma(b.x, wv.y, fma(-b.y, wv.x, im));
    }
    y[c] = make_double2(re, im);
  }
}

int check_group(const edg_momentum_group* g) {
  EDG_REQUIRE(g != nullptr && g->lattice_dim >= 1 && g->lattice_dim <= 3, "momentum: lattice_dim must be 1..3");
  int total = 1;
  for (int d = 0; d < g->lattice_dim; ++d) {
    EDG_REQUIRE(g->shifts_per_dir[d] >= 1, "momentum: shifts_per_dir must be positive");
    total *= g->shifts_per_dir[d];
  }
  EDG_REQUIRE(total == g->n_shifts && total <= kMaxShifts, "momentum: n_shifts must be prod(shifts_per_dir) <= %d",
              kMaxShifts);
  int stride = 1;
  for (int d = g->lattice_dim - 1; d >= 0; --d) {
    EDG_REQUIRE(g->shift_strides[d] == stride, "momentum: shift strides must be row-major");
    stride *= g->shifts_per_dir[d];
  }
  return EDG_OK;
}

}  // namespace

extern "C" int edg_momentum_translations(const edg_lookup_table* sector, const uint64_t* strides,
                                         const int32_t* loc_dims, int32_t n_sites, const int32_t* source_sites,
                                         int32_t n_shifts, const int32_t* local_map, int32_t map_dim,
                                         const double* label_sign, double* row_sign, int32_t* trans,
                                         int32_t* err_flag, cudaStream_t stream) {
  EDG_REQUIRE(sector != nullptr && strides != nullptr && loc_dims != nullptr && source_sites != nullptr &&
                  trans != nullptr && err_flag != nullptr,
              "edg_momentum_translations: null argument");
  EDG_REQUIRE(n_sites >= 1 && n_sites <= EDG_MAX_SITES && n_shifts >= 1 && n_shifts <= kMaxShifts,
              "edg_momentum_translations: bad sizes");
  EDG_REQUIRE(sector->n < (int64_t)INT32_MAX, "edg_momentum_translations: sector above 2^31 rows");
  EDG_REQUIRE(sector->key_words <= 1, "edg_momentum_translations: one-word keys only (key space below 2^63)");
  EDG_REQUIRE((local_map == nullptr && row_sign == nullptr) || (map_dim >= 1 && map_dim <= 256),
              "edg_momentum_translations: map_dim must be 1..256");
  EDG_REQUIRE((row_sign == nullptr) == (label_sign == nullptr), "edg_momentum_translations: label_sign and row_sign go together");
  cudaError_t e = cudaMemsetAsync(err_flag, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_momentum_translations: flag");
  if (sector->n == 0) return EDG_OK;
  translations_k<<<edg::grid_for(sector->n, kThreads), kThreads, 0, stream>>>(*sector, strides, loc_dims, n_sites,
                                                                             source_sites, n_shifts, local_map, map_dim,
                                                                             label_sign, row_sign, trans, err_flag);
  EDG_CHECK_LAUNCH("edg_momentum_translations");
  int32_t h = 0;
  e = cudaMemcpyAsync(&h, err_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_momentum_translations: flag read");
  if (h) {
    edg::set_error("edg_momentum_translations: a translated configuration is outside the sector "
                   "(the sector is not translation invariant for this unit cell)");
    return EDG_ERR_MISSING_KET;
  }
  return EDG_OK;
}

extern "C" int64_t edg_momentum_scratch_elems(int64_t n_rows) {
  return n_rows < 0 ? -1 : (n_rows + 1) + edg_scan_scratch_elems(n_rows);
}

extern "C" int edg_momentum_references(const int32_t* trans, int64_t n_rows, const edg_momentum_group* g,
                                       int32_t* pvec, int64_t* refs, int64_t* n_cols, int64_t* scratch,
                                       int64_t scratch_elems, cudaStream_t stream) {
  if (check_group(g) != EDG_OK) return EDG_ERR_ARG;
  EDG_REQUIRE(n_cols != nullptr && scratch != nullptr && n_rows >= 0 &&
                  (n_rows == 0 || (trans != nullptr && pvec != nullptr && refs != nullptr)),
              "edg_momentum_references: null argument");
  EDG_REQUIRE(scratch_elems >= edg_momentum_scratch_elems(n_rows), "edg_momentum_references: scratch too small");
  *n_cols = 0;
  if (n_rows == 0) return EDG_OK;
  int64_t* offsets = scratch;
  references_k<<<edg::grid_for(n_rows, kThreads), kThreads, 0, stream>>>(trans, n_rows, g->n_shifts, *g, offsets,
                                                                         pvec);
  EDG_CHECK_LAUNCH("edg_momentum_references");
  int st = edg_scan_i64(offsets, offsets, n_rows, scratch + n_rows + 1, stream);
  if (st != EDG_OK) return st;
  list_refs_k<<<edg::grid_for(n_rows, kThreads), kThreads, 0, stream>>>(offsets, n_rows, refs);
  EDG_CHECK_LAUNCH("edg_momentum_references: list");
  cudaError_t e = cudaMemcpyAsync(n_cols, offsets + n_rows, sizeof(int64_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_momentum_references: count read");
  return EDG_OK;
}

extern "C" int edg_momentum_columns(const int32_t* trans, const int64_t* refs, int64_t n_cols, const int32_t* pvec,
                                    const edg_momentum_group* g, const double* phase_table, int32_t max_r,
                                    int32_t zero_k, const double* row_sign, int64_t* col_ptr, int64_t* nnz,
                                    int32_t* row_idx, double* data, int64_t* scratch, int64_t scratch_elems,
                                    cudaStream_t stream) {
  if (check_group(g) != EDG_OK) return EDG_ERR_ARG;
  EDG_REQUIRE(col_ptr != nullptr && nnz != nullptr && scratch != nullptr && phase_table != nullptr && n_cols >= 0 &&
                  (n_cols == 0 || (trans != nullptr && refs != nullptr && pvec != nullptr)),
              "edg_momentum_columns: null argument");
  EDG_REQUIRE(((uintptr_t)phase_table & 15) == 0 && (data == nullptr || ((uintptr_t)data & 15) == 0),
              "edg_momentum_columns: phase_table and data must be 16-byte aligned");
  EDG_REQUIRE(scratch_elems >= edg_scan_scratch_elems(n_cols), "edg_momentum_columns: scratch too small");
  for (int d = 0; d < g->lattice_dim; ++d)
    EDG_REQUIRE(g->shifts_per_dir[d] <= max_r, "edg_momentum_columns: phase table narrower than shifts_per_dir");
  const auto* ph = reinterpret_cast<const double2*>(phase_table);
  if (row_idx == nullptr) {  // count pass: col_ptr = exclusive scan of the column counts, *nnz = total
    *nnz = 0;
    if (n_cols == 0) {
      cudaError_t e = cudaMemsetAsync(col_ptr, 0, sizeof(int64_t), stream);
      return e == cudaSuccess ? EDG_OK : edg::cuda_status(e, "edg_momentum_columns");
    }
    columns_k<<<edg::grid_for(n_cols, kThreads), kThreads, 0, stream>>>(trans, g->n_shifts, refs, n_cols, pvec, *g, ph,
                                                                        max_r, zero_k, row_sign, col_ptr, nullptr,
                                                                        nullptr, nullptr);
    EDG_CHECK_LAUNCH("edg_momentum_columns: count");
    int st = edg_scan_i64(col_ptr, col_ptr, n_cols, scratch, stream);
    if (st != EDG_OK) return st;
    cudaError_t e = cudaMemcpyAsync(nnz, col_ptr + n_cols, sizeof(int64_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e == cudaSuccess ? EDG_OK : edg::cuda_status(e, "edg_momentum_columns: count read");
  }
  EDG_REQUIRE(data != nullptr, "edg_momentum_columns: data is null");
  if (n_cols == 0) return EDG_OK;
  columns_k<<<edg::grid_for(n_cols, kThreads), kThreads, 0, stream>>>(trans, g->n_shifts, refs, n_cols, pvec, *g, ph,
                                                                      max_r, zero_k, row_sign, nullptr, col_ptr,
                                                                      row_idx, reinterpret_cast<double2*>(data));
  EDG_CHECK_LAUNCH("edg_momentum_columns: fill");
  return EDG_OK;
}

extern "C" int edg_momentum_rowmap(const int64_t* col_ptr, const int32_t* row_idx, const double* data, int64_t n_cols,
                                   int64_t n_rows, int64_t* row_col, double* row_val, int32_t* err_flag,
                                   cudaStream_t stream) {
  EDG_REQUIRE(col_ptr != nullptr && row_col != nullptr && row_val != nullptr && err_flag != nullptr && n_cols >= 0 &&
                  n_rows >= 0,
              "edg_momentum_rowmap: null argument");
  cudaError_t e = cudaMemsetAsync(row_col, 0xff, sizeof(int64_t) * (size_t)n_rows, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(row_val, 0, 16 * (size_t)n_rows, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(err_flag, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_momentum_rowmap: clear");
  if (n_cols > 0) {
    rowmap_k<<<edg::grid_for(n_cols, kThreads), kThreads, 0, stream>>>(col_ptr, row_idx, (const double2*)data, n_cols,
                                                                       n_rows, row_col, (double2*)row_val, err_flag);
    EDG_CHECK_LAUNCH("edg_momentum_rowmap");
  }
  int32_t h = 0;
  e = cudaMemcpyAsync(&h, err_flag, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_momentum_rowmap: flag read");
  if (h) {
    edg::set_error(h == 2 ? "edg_momentum_rowmap: a row index is out of range"
                          : "edg_momentum_rowmap: a row belongs to two columns");
    return EDG_ERR_ARG;
  }
  return EDG_OK;
}

extern "C" int edg_momentum_expand(int64_t n_rows, const int64_t* row_col, const double* row_val, const double* x,
                                   double* v, cudaStream_t stream) {
  EDG_REQUIRE(n_rows >= 0 && (n_rows == 0 || (row_col && row_val && x && v)), "edg_momentum_expand: null argument");
  if (n_rows == 0) return EDG_OK;
  expand_k<<<edg::grid_for(n_rows, kThreads), kThreads, 0, stream>>>(n_rows, row_col, (const double2*)row_val,
                                                                     (const double2*)x, (double2*)v);
  EDG_CHECK_LAUNCH("edg_momentum_expand");
  return EDG_OK;
}

extern "C" int edg_momentum_reduce(int64_t n_cols, const int64_t* col_ptr, const int32_t* row_idx, const double* data,
                                   const double* w, double* y, cudaStream_t stream) {
  EDG_REQUIRE(n_cols >= 0 && (n_cols == 0 || (col_ptr && y && w)), "edg_momentum_reduce: null argument");
  if (n_cols == 0) return EDG_OK;
  reduce_k<<<edg::grid_for(n_cols, kThreads), kThreads, 0, stream>>>(n_cols, col_ptr, row_idx, (const double2*)data,
                                                                     (const double2*)w, (double2*)y);
  EDG_CHECK_LAUNCH("edg_momentum_reduce");
  return EDG_OK;
}
