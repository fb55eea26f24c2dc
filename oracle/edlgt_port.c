/*
 * CPU port of ed-lgt's hot loops -- TEST AND CPU-BASELINE INFRASTRUCTURE ONLY.
 *
 * Multithreaded (OpenMP) C restatement of:
 *   - nbody_data / nbody_data_2sites / nbody_data_4sites
 *     (edlgt/symmetries/sym_qmb_operations.py:297-562): per bra row the
 *     product of local transitions, ket located by binary search in the
 *     sorted sector, triplets written at offsets from a count pass and an
 *     exclusive scan (:95-164);
 *   - localbody_data_par (:565-602): diagonal entries with |op_cc| >= 1e-10;
 *   - csr_spmv (edlgt/modeling/qmb_hamiltonian.py:705-730): row-parallel
 *     complex128 matvec.
 * Keys replace the uint16 configuration rows (same order, same search).
 * Used by bench.py's CPU baseline and by tests; the engine never calls it.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <complex.h>

#define OP_TOL 1e-10

static int64_t find_key(const uint64_t* keys, int64_t n, uint64_t q) {
  int64_t lo = 0, hi = n - 1;
  while (lo <= hi) {
    int64_t mid = (lo + hi) / 2;
    uint64_t k = keys[mid];
    if (k == q) return mid;
    if (k < q) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

static int digit(uint64_t key, const uint64_t* strides, const int32_t* loc_dims, int s) {
  return (int)((key / strides[s]) % (uint64_t)loc_dims[s]);
}

/* Count pass of one term instance: nnz per row = prod of transition counts. */
int64_t port_nbody_count(const uint64_t* keys, int64_t n, const uint64_t* strides, const int32_t* loc_dims,
                         int nops, const int32_t* sites, const int32_t* counts /* [nops][dmax] */, int dmax,
                         int64_t* row_nnz) {
  int64_t total = 0;
#pragma omp parallel for reduction(+ : total) schedule(static)
  for (int64_t r = 0; r < n; ++r) {
    int64_t c = 1;
    for (int j = 0; j < nops; ++j) c *= counts[j * dmax + digit(keys[r], strides, loc_dims, sites[j])];
    row_nnz[r] = c;
    total += c;
  }
  return total;
}

/* Fill pass: rows/cols/vals at offsets[r] (exclusive scan of row_nnz). */
void port_nbody_fill(const uint64_t* keys, int64_t n, const uint64_t* strides, const int32_t* loc_dims, int nops,
                     const int32_t* sites, const int32_t* counts, const int32_t* kets /* [nops][dmax][dmax] */,
                     const double complex* amps, int dmax, const int64_t* offsets, int32_t* rows, int32_t* cols,
                     double complex* vals) {
#pragma omp parallel for schedule(dynamic, 1024)
  for (int64_t r = 0; r < n; ++r) {
    int bra[8], cnt[8], idx[8];
    int64_t p = offsets[r];
    int empty = 0;
    for (int j = 0; j < nops; ++j) {
      bra[j] = digit(keys[r], strides, loc_dims, sites[j]);
      cnt[j] = counts[j * dmax + bra[j]];
      idx[j] = 0;
      if (cnt[j] == 0) empty = 1;
    }
    if (empty) continue;
    for (;;) {
      uint64_t kk = keys[r];
      double complex a = 1.0;
      for (int j = 0; j < nops; ++j) {
        int64_t e = ((int64_t)j * dmax + bra[j]) * dmax + idx[j];
        kk += (uint64_t)((int64_t)(kets[e] - bra[j]) * (int64_t)strides[sites[j]]);
        a *= amps[e];
      }
      rows[p] = (int32_t)r;
      cols[p] = (int32_t)find_key(keys, n, kk);
      vals[p] = a;
      ++p;
      int j = nops - 1;
      for (; j >= 0; --j) {
        if (++idx[j] < cnt[j]) break;
        idx[j] = 0;
      }
      if (j < 0) break;
    }
  }
}

/* Diagonal term: value op_cc of the row's state at `site` when |op_cc| >= OP_TOL. */
int64_t port_local_diag(const uint64_t* keys, int64_t n, const uint64_t* strides, const int32_t* loc_dims, int site,
                        const double complex* diag, int32_t* rows, double complex* vals) {
  int64_t m = 0;
  for (int64_t r = 0; r < n; ++r) {
    double complex v = diag[digit(keys[r], strides, loc_dims, site)];
    if (cabs(v) >= OP_TOL) {
      rows[m] = (int32_t)r;
      vals[m] = v;
      ++m;
    }
  }
  return m;
}

/* y = A x for CSR A (complex128), rows in parallel. */
void port_csr_spmv(int64_t n, const int64_t* indptr, const int32_t* indices, const double complex* data,
                   const double complex* x, double complex* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double complex acc = 0.0;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) acc += data[p] * x[indices[p]];
    y[i] = acc;
  }
}

/* y = A x for CSR A with real (double) values. */
void port_csr_spmv_real(int64_t n, const int64_t* indptr, const int32_t* indices, const double* data,
                        const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double acc = 0.0;
    for (int64_t p = indptr[i]; p < indptr[i + 1]; ++p) acc += data[p] * x[indices[p]];
    y[i] = acc;
  }
}
