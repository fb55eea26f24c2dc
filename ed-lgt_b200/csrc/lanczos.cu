// Lanczos ground states with full reorthogonalisation, for nvec independent
// real-symmetric problems sharing the off-diagonal matrix (batched in one
// matvec).  Krylov vectors are stored in T (double or float), interleaved
// [row][vec]; the working vector w, every inner product, the recurrence
// coefficients and the tridiagonal eigen-solve are double precision.
//
// Step j (v_j in V[j]):
//   w = H v_j                                  (spmv, double output)
//   two classical Gram-Schmidt passes:         h = V[0..j]^T w ; w -= V h
//   alpha_j = h1_j + h2_j ; beta_{j+1} = |w| ; V[j+1] = w / beta_{j+1}
// Every check_every steps the k lowest Ritz pairs of the tridiagonal matrix are
// computed on the device (multisection + inverse iteration) and the residual
// bound |beta_{j+1} s_{j}| is compared with tol * max(1, |theta|).
#include "spmv.cuh"

#include <cmath>
#include <mutex>
#include <vector>

namespace {

constexpr int kThreads = 256;
constexpr int kItile = 8;  // Krylov vectors per reduction tile
constexpr int kMaxK = 16;

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

template <typename T>
__device__ __forceinline__ double ldv(const T* p, int64_t i) { return (double)p[i]; }

// w = uniform(-1, 1) or w = v0
template <typename T>
__global__ void start_k(int64_t len, uint64_t seed, const T* __restrict__ v0, double* __restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < len; i += (int64_t)gridDim.x * blockDim.x) {
    if (v0) {
      w[i] = (double)v0[i];
    } else {
      uint64_t r = splitmix64(seed ^ splitmix64((uint64_t)i));
      w[i] = ((double)(r >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
    }
  }
}

// Block-reduces NV doubles per thread; thread 0 gets the totals in out[].
template <int NV>
__device__ __forceinline__ void block_sum(double* vals, double* smem /*[kThreads/32][NV]*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double a = vals[v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) smem[warp * NV + v] = a;
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double a = 0.0;
    for (int wi = 0; wi < kThreads / 32; ++wi) a += smem[wi * NV + threadIdx.x];
    vals[threadIdx.x] = a;  // only meaningful in threads < NV
  }
  __syncthreads();
}

// partial[b][i][v] = sum over the rows of block b of V[i][r][v] * w[r][v], i <= j.
template <typename T, int NV>
__global__ void __launch_bounds__(kThreads) dots_k(const T* __restrict__ V, int64_t n, int j,
                                                   const double* __restrict__ w, double* __restrict__ partial,
                                                   int ld_i, int64_t stride_i /* entries per Krylov vector */) {
  __shared__ double red[(kThreads / 32) * kItile * NV];
  __shared__ double out[kItile * NV];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * chunk;
  const int64_t r1 = min(n, r0 + chunk);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i0 = 0; i0 <= j; i0 += kItile) {
    double acc[kItile][NV];
#pragma unroll
    for (int t = 0; t < kItile; ++t)
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[t][v] = 0.0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) {
      double wr[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) wr[v] = w[r * NV + v];
#pragma unroll
      for (int t = 0; t < kItile; ++t) {
        if (i0 + t <= j) {
          const T* Vi = V + (int64_t)(i0 + t) * stride_i + r * NV;
#pragma unroll
          for (int v = 0; v < NV; ++v) acc[t][v] = fma(ldv(Vi, v), wr[v], acc[t][v]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < kItile; ++t)
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double a = acc[t][v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) red[(warp * kItile + t) * NV + v] = a;
      }
    __syncthreads();
    if (threadIdx.x < kItile * NV) {
      double a = 0.0;
      for (int wi = 0; wi < kThreads / 32; ++wi) a += red[wi * kItile * NV + threadIdx.x];
      out[threadIdx.x] = a;
    }
    __syncthreads();
    if (threadIdx.x < kItile * NV) {
      int t = threadIdx.x / NV, v = threadIdx.x % NV;
      if (i0 + t <= j) partial[((int64_t)blockIdx.x * ld_i + (i0 + t)) * NV + v] = out[threadIdx.x];
    }
    __syncthreads();
  }
}

// h[i][v] = sum_b partial[b][i][v] (one CTA per Krylov index i, fixed summation
// order); alpha accumulates h[j].
template <int NV>
__global__ void __launch_bounds__(kThreads) reduce_h_k(const double* __restrict__ partial, int nblocks, int ld_i,
                                                       int j, double* __restrict__ h, double* __restrict__ alpha_j) {
  __shared__ double red[(kThreads / 32) * NV];
  const int i = blockIdx.x;
  double a[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) a[v] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kThreads)
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] += partial[((int64_t)b * ld_i + i) * NV + v];
  block_sum<NV>(a, red);
  if (threadIdx.x < NV) {
    h[i * NV + threadIdx.x] = a[threadIdx.x];
    if (alpha_j && i == j) alpha_j[threadIdx.x] += a[threadIdx.x];
  }
}

// Pass 1 update fused with pass 2 inner products:
//   w[r] -= sum_i V[i][r] h[i] ;  partial[b][i] = sum_{r in block b} V[i][r] w[r]
// Each CTA owns a contiguous row chunk; the Krylov entries of a row tile are
// read once for the update and then again (from L1) for the new dots.
template <typename T, int NV>
__global__ void __launch_bounds__(kThreads) update_dots_k(const T* __restrict__ V, int64_t n, int j,
                                                          const double* __restrict__ h, double* __restrict__ w,
                                                          double* __restrict__ partial, int ld_i, int64_t stride_i) {
  extern __shared__ double hs[];  // [(j+1)][NV]
  __shared__ double red[(kThreads / 32) * kItile * NV];
  __shared__ double out[kItile * NV];
  for (int t = threadIdx.x; t < (j + 1) * NV; t += kThreads) hs[t] = h[t];
  __syncthreads();
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * chunk;
  const int64_t r1 = min(n, r0 + chunk);
  // update all rows of the chunk first (each thread its own rows)
  for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) {
    double s[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = 0.0;
    for (int i = 0; i <= j; ++i) {
      const T* Vi = V + (int64_t)i * stride_i + r * NV;
#pragma unroll
      for (int v = 0; v < NV; ++v) s[v] = fma(ldv(Vi, v), hs[i * NV + v], s[v]);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) w[r * NV + v] -= s[v];
  }
  // the same thread re-reads the rows it updated: no barrier needed for w
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i0 = 0; i0 <= j; i0 += kItile) {
    double acc[kItile][NV];
#pragma unroll
    for (int t = 0; t < kItile; ++t)
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[t][v] = 0.0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) {
      double wr[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) wr[v] = w[r * NV + v];
#pragma unroll
      for (int t = 0; t < kItile; ++t) {
        if (i0 + t <= j) {
          const T* Vi = V + (int64_t)(i0 + t) * stride_i + r * NV;
#pragma unroll
          for (int v = 0; v < NV; ++v) acc[t][v] = fma(ldv(Vi, v), wr[v], acc[t][v]);
        }
      }
    }
#pragma unroll
    for (int t = 0; t < kItile; ++t)
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double a = acc[t][v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
        if (lane == 0) red[(warp * kItile + t) * NV + v] = a;
      }
    __syncthreads();
    if (threadIdx.x < kItile * NV) {
      double a = 0.0;
      for (int wi = 0; wi < kThreads / 32; ++wi) a += red[wi * kItile * NV + threadIdx.x];
      out[threadIdx.x] = a;
    }
    __syncthreads();
    if (threadIdx.x < kItile * NV) {
      int t = threadIdx.x / NV, v = threadIdx.x % NV;
      if (i0 + t <= j) partial[((int64_t)blockIdx.x * ld_i + (i0 + t)) * NV + v] = out[threadIdx.x];
    }
    __syncthreads();
  }
}

// w[r][v] -= sum_i V[i][r][v] h[i][v]; block partial of |w|^2 per vector.
template <typename T, int NV>
__global__ void __launch_bounds__(kThreads) update_k(const T* __restrict__ V, int64_t n, int j, const double* __restrict__ h,
                                                     double* __restrict__ w, double* __restrict__ norm_partial,
                                                     int64_t stride_i) {
  extern __shared__ double hs[];  // [(j+1)][NV]
  __shared__ double red[(kThreads / 32) * NV];
  for (int t = threadIdx.x; t < (j + 1) * NV; t += kThreads) hs[t] = h[t];
  __syncthreads();
  double nrm[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) nrm[v] = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    double s[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) s[v] = 0.0;
    for (int i = 0; i <= j; ++i) {
      const T* Vi = V + (int64_t)i * stride_i + r * NV;
#pragma unroll
      for (int v = 0; v < NV; ++v) s[v] = fma(ldv(Vi, v), hs[i * NV + v], s[v]);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      double x = w[r * NV + v] - s[v];
      w[r * NV + v] = x;
      nrm[v] = fma(x, x, nrm[v]);
    }
  }
  block_sum<NV>(nrm, red);
  if (threadIdx.x < NV) norm_partial[blockIdx.x * NV + threadIdx.x] = nrm[threadIdx.x];
}

// |w|^2 block partials (start vector)
template <int NV>
__global__ void __launch_bounds__(kThreads) norm_k(const double* __restrict__ w, int64_t n, double* __restrict__ norm_partial) {
  __shared__ double red[(kThreads / 32) * NV];
  double nrm[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) nrm[v] = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads)
#pragma unroll
    for (int v = 0; v < NV; ++v) nrm[v] = fma(w[r * NV + v], w[r * NV + v], nrm[v]);
  block_sum<NV>(nrm, red);
  if (threadIdx.x < NV) norm_partial[blockIdx.x * NV + threadIdx.x] = nrm[threadIdx.x];
}

// beta[v] = sqrt(sum_b norm_partial[b][v]) (one CTA, fixed order)
template <int NV>
__global__ void __launch_bounds__(kThreads) beta_k(const double* __restrict__ norm_partial, int nblocks,
                                                   double* __restrict__ beta) {
  __shared__ double red[(kThreads / 32) * NV];
  double a[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) a[v] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kThreads)
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] += norm_partial[b * NV + v];
  block_sum<NV>(a, red);
  if (threadIdx.x < NV) beta[threadIdx.x] = sqrt(a[threadIdx.x]);
}

// V[j+1] = w / beta (beta = 0 leaves a zero vector: invariant subspace)
template <typename T, int NV>
__global__ void scale_store_k(const double* __restrict__ w, int64_t n, const double* __restrict__ beta,
                              T* __restrict__ out) {
  double inv[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) inv[v] = beta[v] > 0.0 ? 1.0 / beta[v] : 0.0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
#pragma unroll
    for (int v = 0; v < NV; ++v) out[r * NV + v] = (T)(w[r * NV + v] * inv[v]);
}

// ---------------------------------------------------------------------------
// Tridiagonal eigen-solve (one CTA per problem)
// ---------------------------------------------------------------------------
__device__ int sturm_count(const double* a, const double* b2, int m, double x, double pivmin) {
  int cnt = 0;
  double q = a[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += q < 0.0;
  for (int i = 1; i < m; ++i) {
    q = a[i] - x - b2[i] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// alpha: [m] ; beta: [m] with beta[i] coupling i-1 and i (beta[0] unused);
// stride between problems given by lda (alpha) / ldb (beta) in doubles.
__global__ void __launch_bounds__(kThreads) tridiag_k(const double* __restrict__ alpha, int lda,
                                                      const double* __restrict__ beta, int ldb, int m, int k,
                                                      double* __restrict__ evals, double* __restrict__ evecs,
                                                      int ldv, double* __restrict__ work, int ldw) {
  const int prob = blockIdx.x;
  const double* a = alpha + (int64_t)prob * lda;
  const double* bb = beta + (int64_t)prob * ldb;
  double* wk = work + (int64_t)prob * ldw;  // [m] b^2, then scratch for inverse iteration
  double* b2 = wk;
  __shared__ double lo_s, hi_s, xs[kThreads + 1];
  __shared__ int cnt_s[kThreads + 1];
  __shared__ double gl_s, gu_s, pivmin_s;
  for (int i = threadIdx.x; i < m; i += kThreads) b2[i] = i == 0 ? 0.0 : bb[i] * bb[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    double gl = 1e300, gu = -1e300, bmax = 0.0;
    for (int i = 0; i < m; ++i) {
      double off = (i > 0 ? fabs(bb[i]) : 0.0) + (i + 1 < m ? fabs(bb[i + 1]) : 0.0);
      gl = fmin(gl, a[i] - off);
      gu = fmax(gu, a[i] + off);
      if (i > 0) bmax = fmax(bmax, b2[i]);
    }
    double span = fmax(fabs(gl), fabs(gu));
    gl_s = gl - 2.0 * span * 1e-15 - 1e-300;
    gu_s = gu + 2.0 * span * 1e-15 + 1e-300;
    pivmin_s = fmax(1e-290, 2.2e-308 * fmax(1.0, bmax));
  }
  __syncthreads();
  for (int e = 0; e < k && e < m; ++e) {
    if (threadIdx.x == 0) {
      lo_s = gl_s;
      hi_s = gu_s;
    }
    __syncthreads();
    for (int round = 0; round < 12; ++round) {
      double lo = lo_s, hi = hi_s;
      if (!(hi - lo > 2.2e-16 * fmax(fabs(lo), fabs(hi)) + 1e-300)) break;
      // kThreads interior points; count(x) = #eigenvalues < x
      double x = lo + (hi - lo) * (double)(threadIdx.x + 1) / (double)(kThreads + 1);
      xs[threadIdx.x] = x;
      cnt_s[threadIdx.x] = sturm_count(a, b2, m, x, pivmin_s);
      __syncthreads();
      if (threadIdx.x == 0) {
        // first point with count >= e+1 bounds eigenvalue e from above
        double nlo = lo, nhi = hi;
        for (int t = 0; t < kThreads; ++t) {
          if (cnt_s[t] >= e + 1) {
            nhi = xs[t];
            break;
          }
          nlo = xs[t];
        }
        lo_s = nlo;
        hi_s = nhi;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) evals[(int64_t)prob * k + e] = 0.5 * (lo_s + hi_s);
    __syncthreads();
  }
  // inverse iteration for eigenvectors (thread 0; m is small)
  if (threadIdx.x == 0 && evecs != nullptr) {
    double* dl = wk + m;      // LU factors of tridiagonal T - theta
    double* dd = wk + 2 * m;
    double* du = wk + 3 * m;
    double* du2 = wk + 4 * m;
    int* piv = (int*)(wk + 5 * m);
    for (int e = 0; e < k && e < m; ++e) {
      double theta = evals[(int64_t)prob * k + e];
      double* s = evecs + ((int64_t)prob * k + e) * ldv;
      double scale = 0.0;
      for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(a[i]) + (i > 0 ? fabs(bb[i]) : 0.0));
      double eps_shift = 2.2e-16 * fmax(scale, 1e-300);
      // factor (T - theta I) with partial pivoting (dgttrf)
      for (int i = 0; i < m; ++i) {
        dd[i] = a[i] - theta;
        if (i + 1 < m) {
          dl[i] = bb[i + 1];
          du[i] = bb[i + 1];
        }
        du2[i] = 0.0;
      }
      for (int i = 0; i < m - 1; ++i) {
        if (fabs(dd[i]) >= fabs(dl[i])) {
          piv[i] = i;
          if (dd[i] == 0.0) dd[i] = eps_shift;
          double f = dl[i] / dd[i];
          dl[i] = f;
          dd[i + 1] -= f * du[i];
          if (i + 1 < m - 1) du2[i] = 0.0;
        } else {
          piv[i] = i + 1;
          double f = dd[i] / dl[i];
          dd[i] = dl[i];
          dl[i] = f;
          double tmp = du[i];
          du[i] = dd[i + 1];
          dd[i + 1] = tmp - f * dd[i + 1];
          if (i + 1 < m - 1) {
            du2[i] = du[i + 1];
            du[i + 1] = -f * du[i + 1];
          }
        }
      }
      if (dd[m - 1] == 0.0) dd[m - 1] = eps_shift;
      for (int i = 0; i < m; ++i) s[i] = 1.0 / sqrt((double)m) * (1.0 + 0.01 * (double)((i * 7 + e * 3) % 5));
      for (int it = 0; it < 3; ++it) {
        // solve L U x = P s
        for (int i = 0; i < m - 1; ++i) {
          if (piv[i] == i) {
            s[i + 1] -= dl[i] * s[i];
          } else {
            double t = s[i];
            s[i] = s[i + 1];
            s[i + 1] = t - dl[i] * s[i];
          }
        }
        s[m - 1] /= dd[m - 1];
        if (m > 1) s[m - 2] = (s[m - 2] - du[m - 2] * s[m - 1]) / dd[m - 2];
        for (int i = m - 3; i >= 0; --i) s[i] = (s[i] - du[i] * s[i + 1] - du2[i] * s[i + 2]) / dd[i];
        // orthogonalise against earlier eigenvectors (near-degenerate pairs)
        for (int f = 0; f < e; ++f) {
          const double* sf = evecs + ((int64_t)prob * k + f) * ldv;
          double p = 0.0;
          for (int i = 0; i < m; ++i) p += sf[i] * s[i];
          for (int i = 0; i < m; ++i) s[i] -= p * sf[i];
        }
        double nn = 0.0;
        for (int i = 0; i < m; ++i) nn += s[i] * s[i];
        nn = 1.0 / sqrt(nn);
        for (int i = 0; i < m; ++i) s[i] *= nn;
      }
      // sign convention: largest component positive
      int imax = 0;
      for (int i = 1; i < m; ++i)
        if (fabs(s[i]) > fabs(s[imax])) imax = i;
      if (s[imax] < 0.0)
        for (int i = 0; i < m; ++i) s[i] = -s[i];
    }
  }
}

// x[r][v] (for eigenpair e) = sum_i V[i][r][v] S[v][e][i]
template <typename T, int NV>
__global__ void ritz_k(const T* __restrict__ V, int64_t n, int m, const double* __restrict__ S, int k, int e,
                       int lds, int64_t stride_i, double* __restrict__ x) {
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    double acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = 0.0;
    for (int i = 0; i < m; ++i) {
      const T* Vi = V + (int64_t)i * stride_i + r * NV;
#pragma unroll
      for (int v = 0; v < NV; ++v) acc[v] = fma(ldv(Vi, v), S[((int64_t)v * k + e) * lds + i], acc[v]);
    }
#pragma unroll
    for (int v = 0; v < NV; ++v) x[r * NV + v] = acc[v];
  }
}

// ---------------------------------------------------------------------------
// Workspace layout
// ---------------------------------------------------------------------------
struct Layout {
  int64_t V, w, h, partial, normp, alpha, beta, tri_eval, tri_vec, tri_work, total;
  int nblk_dot, nblk_upd, m_max, ld_h;
};

inline int64_t align256(int64_t x) { return (x + 255) & ~int64_t(255); }

Layout make_layout(const edg_lanczos_problem* p) {
  Layout L{};
  const int64_t n = p->n_rows, nv = p->nvec;
  const int esz = p->dtype == 0 ? 8 : 4;
  L.m_max = p->max_iter;
  L.ld_h = L.m_max + 1;
  L.nblk_dot = edg::kSmCount * 4;
  L.nblk_upd = edg::kSmCount * 8;
  int64_t off = 0;
  L.V = off; off = align256(off + (int64_t)(L.m_max + 1) * n * nv * esz);
  L.w = off; off = align256(off + n * nv * 8);
  L.h = off; off = align256(off + (int64_t)(L.m_max + 1) * nv * 8);
  L.partial = off; off = align256(off + (int64_t)L.nblk_dot * (L.m_max + 1) * nv * 8);
  L.normp = off; off = align256(off + (int64_t)L.nblk_upd * nv * 8);
  L.alpha = off; off = align256(off + (int64_t)nv * (L.m_max + 1) * 8);   // [nv][m_max+1]
  L.beta = off; off = align256(off + (int64_t)nv * (L.m_max + 2) * 8);    // [nv][m_max+2]
  L.tri_eval = off; off = align256(off + (int64_t)nv * kMaxK * 8);
  L.tri_vec = off; off = align256(off + (int64_t)nv * kMaxK * (L.m_max + 1) * 8);
  L.tri_work = off; off = align256(off + (int64_t)nv * 6 * (L.m_max + 1) * 8);
  L.total = off;
  return L;
}

// column-major per-problem recurrence storage: alpha[v][i], beta[v][i]
template <int NV>
__global__ void scatter_coef_k(const double* __restrict__ src, double* __restrict__ dst, int ld, int i) {
  int v = threadIdx.x;
  if (v < NV) dst[(int64_t)v * ld + i] = src[v];
}

template <int NV>
__global__ void zero_k(double* p, int n) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = 0.0;
}

template <typename T, int NV>
int run_lanczos(const edg_lanczos_problem* p, char* ws, double* evals, void* evecs, int32_t* iters_out,
                double* resid_out, cudaStream_t s) {
  const Layout L = make_layout(p);
  const int64_t n = p->n_rows;
  const int k = p->k;
  T* V = (T*)(ws + L.V);
  double* w = (double*)(ws + L.w);
  double* h = (double*)(ws + L.h);
  double* partial = (double*)(ws + L.partial);
  double* normp = (double*)(ws + L.normp);
  double* alpha = (double*)(ws + L.alpha);  // [NV][m_max+1]
  double* beta = (double*)(ws + L.beta);    // [NV][m_max+2], beta[v][i] couples i-1 and i
  double* tri_eval = (double*)(ws + L.tri_eval);
  double* tri_vec = (double*)(ws + L.tri_vec);  // [NV][kMaxK][m_max+1]
  double* tri_work = (double*)(ws + L.tri_work);
  const int ld_a = L.m_max + 1, ld_b = L.m_max + 2, ld_s = L.m_max + 1;
  const int64_t stride_i = n * NV;
  double* alpha_cur = h + (int64_t)L.m_max * NV;  // last NV slots of h (h[i] only used for i < m_max)
  const unsigned g_vec = edg::grid_for(n * NV, 256);
  cudaError_t e;
  start_k<T><<<g_vec, 256, 0, s>>>(n * NV, p->seed, (const T*)p->v0, w);
  norm_k<NV><<<L.nblk_upd, kThreads, 0, s>>>(w, n, normp);
  beta_k<NV><<<1, kThreads, 0, s>>>(normp, L.nblk_upd, h);
  scale_store_k<T, NV><<<g_vec, 256, 0, s>>>(w, n, h, V);
  zero_k<NV><<<(NV * ld_b + 255) / 256, 256, 0, s>>>(beta, NV * ld_b);
  zero_k<NV><<<(NV * ld_a + 255) / 256, 256, 0, s>>>(alpha, NV * ld_a);
  if ((e = cudaGetLastError()) != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: start");
  const size_t upd_smem = (size_t)(L.m_max + 1) * NV * sizeof(double);
  if (upd_smem > 40 * 1024) {
    e = cudaFuncSetAttribute(update_k<T, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(update_dots_k<T, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem + 8192);
    if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: smem attribute");
  }
  std::vector<double> hb((size_t)NV * ld_b), ha((size_t)NV * ld_a), hev((size_t)NV * kMaxK),
      hs((size_t)NV * kMaxK * ld_s), res((size_t)NV * k, 0.0);
  std::vector<int> m_conv(NV, 0), m_use(NV, 0);
  auto tridiag_all = [&](const std::vector<int>& mv) -> int {
    cudaError_t err = cudaMemsetAsync(tri_vec, 0, sizeof(double) * NV * kMaxK * ld_s, s);
    if (err != cudaSuccess) return edg::cuda_status(err, "edg_lanczos: tridiag reset");
    for (int v = 0; v < NV; ++v) {
      int kk = k < mv[v] ? k : mv[v];
      tridiag_k<<<1, kThreads, 0, s>>>(alpha + (int64_t)v * ld_a, ld_a, beta + (int64_t)v * ld_b, ld_b, mv[v], kk,
                                       tri_eval + v * kMaxK, tri_vec + (int64_t)v * kMaxK * ld_s, ld_s,
                                       tri_work + (int64_t)v * 6 * ld_s, 6 * ld_s);
    }
    err = cudaGetLastError();
    if (err != cudaSuccess) return edg::cuda_status(err, "edg_lanczos: tridiag");
    return EDG_OK;
  };
  int status = EDG_OK;
  int j = 0;
  // optional phase timing with CUDA events on the launch stream
  const bool timing = p->stats != nullptr;
  std::vector<cudaEvent_t> ev;
  int ev_done = 0;  // steps whose events were already accumulated
  double t_spmv = 0.0, t_reorth = 0.0, t_check = 0.0;
  int64_t launches = 7;  // start-vector kernels
  auto event_at = [&](int idx) -> cudaEvent_t {
    while ((int)ev.size() <= idx) {
      cudaEvent_t e2;
      cudaEventCreate(&e2);
      ev.push_back(e2);
    }
    return ev[idx];
  };
  auto accumulate = [&](int upto) {
    for (; ev_done < upto; ++ev_done) {
      float a = 0.f, b = 0.f;
      cudaEventElapsedTime(&a, ev[3 * ev_done], ev[3 * ev_done + 1]);
      cudaEventElapsedTime(&b, ev[3 * ev_done + 1], ev[3 * ev_done + 2]);
      t_spmv += a;
      t_reorth += b;
    }
  };
  for (; j < L.m_max; ++j) {
    const T* vj = V + (int64_t)j * stride_i;
    if (timing) cudaEventRecord(event_at(3 * j), s);
    int st = edg::launch_spmv<T, T, double>(NV, n, p->nnz, p->rowptr, p->cols, (const T*)p->vals, (const T*)p->diag,
                                            vj, w, s);
    if (st) return st;
    if (timing) cudaEventRecord(event_at(3 * j + 1), s);
    launches += 10;
    zero_k<NV><<<1, 32, 0, s>>>(alpha_cur, NV);
    // classical Gram-Schmidt twice: dots | update+dots | update (3 reads of V)
    dots_k<T, NV><<<L.nblk_dot, kThreads, 0, s>>>(V, n, j, w, partial, ld_a, stride_i);
    reduce_h_k<NV><<<j + 1, kThreads, 0, s>>>(partial, L.nblk_dot, ld_a, j, h, alpha_cur);
    update_dots_k<T, NV><<<L.nblk_dot, kThreads, upd_smem, s>>>(V, n, j, h, w, partial, ld_a, stride_i);
    reduce_h_k<NV><<<j + 1, kThreads, 0, s>>>(partial, L.nblk_dot, ld_a, j, h, alpha_cur);
    update_k<T, NV><<<L.nblk_upd, kThreads, upd_smem, s>>>(V, n, j, h, w, normp, stride_i);
    scatter_coef_k<NV><<<1, 32, 0, s>>>(alpha_cur, alpha, ld_a, j);
    beta_k<NV><<<1, kThreads, 0, s>>>(normp, L.nblk_upd, h);  // h[0..NV) = beta_{j+1}
    scatter_coef_k<NV><<<1, 32, 0, s>>>(h, beta, ld_b, j + 1);
    scale_store_k<T, NV><<<g_vec, 256, 0, s>>>(w, n, h, V + (int64_t)(j + 1) * stride_i);
    if (timing) cudaEventRecord(event_at(3 * j + 2), s);
    if ((e = cudaGetLastError()) != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: step");
    const int m = j + 1;
    const bool check = (m % p->check_every == 0) || m == L.m_max || (int64_t)m == n;
    if (!check) continue;
    // recurrence coefficients to the host (a few KB) to detect invariant subspaces
    e = cudaMemcpyAsync(hb.data(), beta, sizeof(double) * NV * ld_b, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ha.data(), alpha, sizeof(double) * NV * ld_a, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: coefficients");
    if (timing) accumulate(m);
    cudaEvent_t c0 = nullptr, c1 = nullptr;
    if (timing) {
      c0 = event_at(3 * L.m_max + 0);
      c1 = event_at(3 * L.m_max + 1);
      cudaEventRecord(c0, s);
    }
    launches += 1 + NV;
    std::vector<bool> exact(NV, false);
    for (int v = 0; v < NV; ++v) {
      if (m_conv[v]) { m_use[v] = m_conv[v]; continue; }
      double scale = 0.0;
      for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(ha[v * ld_a + i]) + fabs(hb[v * ld_b + i]));
      int mv = m;
      for (int i = 1; i <= m; ++i)
        if (fabs(hb[v * ld_b + i]) <= 1e-12 * fmax(scale, 1e-300)) { mv = i; break; }
      exact[v] = mv < m || (mv == m && fabs(hb[v * ld_b + m]) <= 1e-12 * fmax(scale, 1e-300)) || (int64_t)m == n;
      m_use[v] = mv;
    }
    if ((st = tridiag_all(m_use))) return st;
    e = cudaMemcpyAsync(hev.data(), tri_eval, sizeof(double) * NV * kMaxK, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(hs.data(), tri_vec, sizeof(double) * NV * kMaxK * ld_s, cudaMemcpyDeviceToHost, s);
    if (timing && e == cudaSuccess) e = cudaEventRecord(c1, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: ritz values");
    if (timing) {
      float a = 0.f;
      cudaEventElapsedTime(&a, c0, c1);
      t_check += a;
    }
    bool all = true;
    for (int v = 0; v < NV; ++v) {
      if (m_conv[v]) continue;
      const int mv = m_use[v], kk = k < mv ? k : mv;
      bool ok = kk == k || exact[v];
      for (int q = 0; q < kk; ++q) {
        double theta = hev[v * kMaxK + q];
        double last = hs[((size_t)v * kMaxK + q) * ld_s + (mv - 1)];
        double r = exact[v] ? 0.0 : fabs(hb[v * ld_b + mv] * last);
        res[v * k + q] = r;
        if (r > p->tol * fmax(1.0, fabs(theta))) ok = false;
      }
      if (ok) m_conv[v] = mv;
      else all = false;
    }
    if (all) { ++j; break; }
    if (m == L.m_max) { status = EDG_ERR_NOT_CONVERGED; ++j; break; }
  }
  for (int v = 0; v < NV; ++v) m_use[v] = m_conv[v] ? m_conv[v] : (j < 1 ? 1 : j);
  int st = tridiag_all(m_use);
  if (st) return st;
  e = cudaMemcpyAsync(hev.data(), tri_eval, sizeof(double) * NV * kMaxK, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: final ritz values");
  int m_all = 1;
  for (int v = 0; v < NV; ++v) {
    const int kk = k < m_use[v] ? k : m_use[v];
    for (int q = 0; q < k; ++q) {
      evals[v * k + q] = q < kk ? hev[v * kMaxK + q] : NAN;
      if (resid_out) resid_out[v * k + q] = q < kk ? res[v * k + q] : NAN;
    }
    if (iters_out) iters_out[v] = m_use[v];
    m_all = m_use[v] > m_all ? m_use[v] : m_all;
  }
  if (evecs) {
    // S rows beyond each problem's m are zero, so one pass over m_all vectors serves all problems
    for (int q = 0; q < k; ++q) {
      ritz_k<T, NV><<<g_vec, 256, 0, s>>>(V, n, m_all, tri_vec, kMaxK, q, ld_s, stride_i, w);
      norm_k<NV><<<L.nblk_upd, kThreads, 0, s>>>(w, n, normp);
      beta_k<NV><<<1, kThreads, 0, s>>>(normp, L.nblk_upd, h);
      scale_store_k<T, NV><<<g_vec, 256, 0, s>>>(w, n, h, (T*)evecs + (int64_t)q * stride_i);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: ritz vectors");
  }
  e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: finish");
  if (timing) {
    accumulate(j);
    launches += 1 + NV + (evecs ? 4 * k : 0);
    p->stats[0] = t_spmv;
    p->stats[1] = (double)ev_done;
    p->stats[2] = t_reorth;
    p->stats[3] = (double)launches;
    p->stats[4] = (double)j;
    p->stats[5] = t_check;
    for (auto& x : ev) cudaEventDestroy(x);
  }
  if (status == EDG_ERR_NOT_CONVERGED) edg::set_error("edg_lanczos: not converged in %d steps", L.m_max);
  return status;
}

template <typename T>
int dispatch_nv(const edg_lanczos_problem* p, char* ws, double* ev, void* evec, int32_t* it, double* res,
                cudaStream_t s) {
  switch (p->nvec) {
    case 1: return run_lanczos<T, 1>(p, ws, ev, evec, it, res, s);
    case 2: return run_lanczos<T, 2>(p, ws, ev, evec, it, res, s);
    case 3: return run_lanczos<T, 3>(p, ws, ev, evec, it, res, s);
    case 4: return run_lanczos<T, 4>(p, ws, ev, evec, it, res, s);
    default: edg::set_error("edg_lanczos: nvec must be 1..4"); return EDG_ERR_ARG;
  }
}

int check_problem(const edg_lanczos_problem* p) {
  EDG_REQUIRE(p != nullptr, "edg_lanczos: null problem");
  EDG_REQUIRE(p->dtype == 0 || p->dtype == 1, "edg_lanczos: dtype must be 0 (f64) or 1 (f32)");
  EDG_REQUIRE(p->n_rows > 0, "edg_lanczos: empty matrix");
  EDG_REQUIRE(p->nvec >= 1 && p->nvec <= 4, "edg_lanczos: nvec must be 1..4");
  EDG_REQUIRE(p->k >= 1 && p->k <= kMaxK, "edg_lanczos: k must be 1..%d", kMaxK);
  EDG_REQUIRE(p->max_iter >= 1 && p->max_iter <= 2000, "edg_lanczos: max_iter must be 1..2000");
  EDG_REQUIRE(p->check_every >= 1, "edg_lanczos: check_every must be >= 1");
  EDG_REQUIRE(p->rowptr && p->diag, "edg_lanczos: null matrix pointer");
  return EDG_OK;
}

}  // namespace

extern "C" int64_t edg_lanczos_workspace_bytes(const edg_lanczos_problem* p) {
  if (check_problem(p)) return -1;
  edg_lanczos_problem q = *p;
  if (q.max_iter > q.n_rows) q.max_iter = (int32_t)q.n_rows;
  return make_layout(&q).total;
}

extern "C" int edg_lanczos(const edg_lanczos_problem* p, void* workspace, int64_t workspace_bytes, double* evals,
                           void* evecs, int32_t* iters_out, double* resid_out, cudaStream_t stream) {
  int st = check_problem(p);
  if (st) return st;
  edg_lanczos_problem q = *p;
  if (q.max_iter > q.n_rows) q.max_iter = (int32_t)q.n_rows;
  EDG_REQUIRE(workspace != nullptr && workspace_bytes >= make_layout(&q).total, "edg_lanczos: workspace too small");
  EDG_REQUIRE(evals != nullptr, "edg_lanczos: null evals");
  if (q.dtype == 0) return dispatch_nv<double>(&q, (char*)workspace, evals, evecs, iters_out, resid_out, stream);
  return dispatch_nv<float>(&q, (char*)workspace, evals, evecs, iters_out, resid_out, stream);
}

extern "C" int edg_tridiag_lowest(const double* alpha, const double* beta, int32_t m, int32_t k, double* evals,
                                  double* evecs, double* work, cudaStream_t stream) {
  EDG_REQUIRE(m >= 1 && k >= 1 && k <= m && k <= kMaxK, "edg_tridiag_lowest: need 1 <= k <= min(m, %d)", kMaxK);
  EDG_REQUIRE(alpha && beta && evals && work, "edg_tridiag_lowest: null pointer");
  tridiag_k<<<1, kThreads, 0, stream>>>(alpha, m, beta, m, m, k, evals, evecs, m, work, 6 * m);
  EDG_CHECK_LAUNCH("edg_tridiag_lowest");
  return EDG_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of edg_tridiag_lowest.
//
// For callers that cannot call cudaMalloc (for example code running inside a
// host callback, a memory-capped plugin host, or a language runtime without a
// device allocator): the 6*m doubles of scratch live in a file-scope device
// array of fixed size, so the call allocates nothing.  Every GPU that loads
// the library holds this array (6 * 4096 doubles = 192 KiB) until exit.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxM = 4096;
static __device__ __align__(256) double g_tridiag_scratch[6 * kNoAllocMaxM];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_tridiag_scratch on the current device.  The host-side
// symbol is only a stand-in for the device array: it must not be passed to a
// kernel, so the address is looked up once per device with that device current.
int scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_tridiag_lowest_noalloc: current device");
  EDG_REQUIRE(dev >= 0 && dev < kMaxDevices, "edg_tridiag_lowest_noalloc: device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_tridiag_scratch);
    if (e != cudaSuccess) return edg::cuda_status(e, "edg_tridiag_lowest_noalloc: cudaGetSymbolAddress");
    g_scratch_ptr[dev] = (double*)p;
  }
  *out = g_scratch_ptr[dev];
  return EDG_OK;
}

}  // namespace

extern "C" int edg_tridiag_lowest_noalloc(const double* alpha, const double* beta, int32_t m, int32_t k,
                                          double* evals, double* evecs, cudaStream_t stream) {
  EDG_REQUIRE(m >= 1 && k >= 1 && k <= m && k <= kMaxK, "edg_tridiag_lowest_noalloc: need 1 <= k <= min(m, %d)",
              kMaxK);
  EDG_REQUIRE(m <= kNoAllocMaxM, "edg_tridiag_lowest_noalloc: m = %d exceeds the static scratch limit of %d", m,
              kNoAllocMaxM);
  EDG_REQUIRE(alpha && beta && evals, "edg_tridiag_lowest_noalloc: null pointer");
  double* work = nullptr;
  int st = scratch_address(&work);
  if (st) return st;
  // tridiag_k writes every scratch element before reading it, so the array
  // needs no clearing between calls.
  tridiag_k<<<1, kThreads, 0, stream>>>(alpha, m, beta, m, m, k, evals, evecs, m, work, 6 * m);
  EDG_CHECK_LAUNCH("edg_tridiag_lowest_noalloc");
  return EDG_OK;
}
