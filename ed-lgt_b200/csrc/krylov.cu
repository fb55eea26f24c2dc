// Krylov time evolution psi <- exp(-i H dt) psi for a Hermitian sector
// Hamiltonian (real form or complex), with complex Krylov vectors stored in
// complex64 or complex128 and every inner product, the Lanczos recurrence and
// the small exponential in double precision.
//
// One step: v_0 = psi/|psi|; m Lanczos steps w = H v_j, orthogonalised against
// the basis (one classical Gram-Schmidt pass over all previous vectors, or
// two), alpha_j = Re<v_j, w>, beta_{j+1} = |w|; then c = |psi| exp(-i T dt) e_1
// for the m x m tridiagonal T (scaling and squaring of a Taylor series on the
// device, exact to double precision) and psi = V c.  A breakdown (beta = 0)
// leaves zero vectors whose block of T decouples from e_1, so the step needs
// no host synchronisation.  Replaces scipy's expm_multiply as called by
// QMB_hamiltonian.time_evolution (edlgt/modeling/qmb_hamiltonian.py:334-426).
#include "spmv.cuh"

#include <type_traits>

#include <cmath>

namespace {

constexpr int kThreads = 256;
constexpr int kItile = 8;
constexpr int kMaxM = 64;

template <typename T>
__device__ __forceinline__ edg::cd ldc(const T* p, int64_t i);
template <>
__device__ __forceinline__ edg::cd ldc<float2>(const float2* p, int64_t i) {
  float2 v = p[i];
  return {(double)v.x, (double)v.y};
}
template <>
__device__ __forceinline__ edg::cd ldc<double2>(const double2* p, int64_t i) {
  double2 v = p[i];
  return {v.x, v.y};
}
template <typename T>
__device__ __forceinline__ void stc(T* p, int64_t i, double re, double im);
template <>
__device__ __forceinline__ void stc<float2>(float2* p, int64_t i, double re, double im) {
  p[i] = make_float2((float)re, (float)im);
}
template <>
__device__ __forceinline__ void stc<double2>(double2* p, int64_t i, double re, double im) {
  p[i] = make_double2(re, im);
}

__device__ __forceinline__ double block_sum1(double a, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
  if (lane == 0) red[warp] = a;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kThreads / 32; ++w) t += red[w];
  __syncthreads();
  return t;  // valid in thread 0
}

// |x|^2 block partials of a complex vector (T storage or double2 working)
template <typename T>
__global__ void __launch_bounds__(kThreads) norm_k(const T* __restrict__ x, int64_t n, double* __restrict__ part) {
  __shared__ double red[kThreads / 32];
  double a = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    edg::cd v = ldc<T>(x, r);
    a = fma(v.re, v.re, fma(v.im, v.im, a));
  }
  double t = block_sum1(a, red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// out[0] = sqrt(sum partials)
__global__ void __launch_bounds__(kThreads) sqrt_sum_k(const double* __restrict__ part, int nb, double* __restrict__ out) {
  __shared__ double red[kThreads / 32];
  double a = 0.0;
  for (int b = threadIdx.x; b < nb; b += kThreads) a += part[b];
  double t = block_sum1(a, red);
  if (threadIdx.x == 0) out[0] = sqrt(t);
}

// dst = src / s[0] (s = 0 gives zeros)
template <typename TS, typename TD>
__global__ void scale_k(const TS* __restrict__ src, int64_t n, const double* __restrict__ s, TD* __restrict__ dst) {
  const double inv = s[0] > 0.0 ? 1.0 / s[0] : 0.0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    edg::cd v = ldc<TS>(src, r);
    stc<TD>(dst, r, v.re * inv, v.im * inv);
  }
}

// partial[b][i] = sum_{r in block b} conj(V[i][r]) w[r] for i <= j (complex double)
template <typename T>
__global__ void __launch_bounds__(kThreads) dots_k(const T* __restrict__ V, int64_t n, int ilo, int j,
                                                   const double2* __restrict__ w, double2* __restrict__ partial,
                                                   int ld_i) {
  __shared__ double red[(kThreads / 32) * kItile * 2];
  __shared__ double out[kItile * 2];
  const int64_t chunk = (n + gridDim.x - 1) / gridDim.x;
  const int64_t r0 = blockIdx.x * chunk, r1 = min(n, r0 + chunk);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i0 = ilo; i0 <= j; i0 += kItile) {
    double re[kItile], im[kItile];
#pragma unroll
    for (int t = 0; t < kItile; ++t) re[t] = im[t] = 0.0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) {
      double2 wr = w[r];
#pragma unroll
      for (int t = 0; t < kItile; ++t)
        if (i0 + t <= j) {
          edg::cd v = ldc<T>(V, (int64_t)(i0 + t) * n + r);
          re[t] = fma(v.re, wr.x, fma(v.im, wr.y, re[t]));
          im[t] = fma(v.re, wr.y, fma(-v.im, wr.x, im[t]));
        }
    }
#pragma unroll
    for (int t = 0; t < kItile; ++t) {
      double a = re[t], b = im[t];
      for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        b += __shfl_down_sync(0xffffffffu, b, o);
      }
      if (lane == 0) {
        red[(warp * kItile + t) * 2] = a;
        red[(warp * kItile + t) * 2 + 1] = b;
      }
    }
    __syncthreads();
    if (threadIdx.x < kItile * 2) {
      double a = 0.0;
      for (int wi = 0; wi < kThreads / 32; ++wi) a += red[wi * kItile * 2 + threadIdx.x];
      out[threadIdx.x] = a;
    }
    __syncthreads();
    if (threadIdx.x < kItile) {
      int t = threadIdx.x;
      if (i0 + t <= j) partial[(int64_t)blockIdx.x * ld_i + i0 + t] = make_double2(out[2 * t], out[2 * t + 1]);
    }
    __syncthreads();
  }
}

// h[i] = sum_b partial[b][i]; alpha[j] += Re h[j]
__global__ void __launch_bounds__(kThreads) reduce_h_k(const double2* __restrict__ partial, int nb, int ld_i, int ilo,
                                                       int j, double2* __restrict__ h, double* __restrict__ alpha_j) {
  __shared__ double red[kThreads / 32];
  const int i = ilo + blockIdx.x;
  double a = 0.0, b = 0.0;
  for (int q = threadIdx.x; q < nb; q += kThreads) {
    double2 p = partial[(int64_t)q * ld_i + i];
    a += p.x;
    b += p.y;
  }
  double ta = block_sum1(a, red);
  double tb = block_sum1(b, red);
  if (threadIdx.x == 0) {
    h[i] = make_double2(ta, tb);
    if (i == j) alpha_j[0] += ta;
  }
}

// w[r] -= sum_{i<=j} V[i][r] h[i]; |w|^2 block partials
template <typename T>
__global__ void __launch_bounds__(kThreads) update_k(const T* __restrict__ V, int64_t n, int ilo, int j,
                                                     const double2* __restrict__ h, double2* __restrict__ w,
                                                     double* __restrict__ part) {
  __shared__ double2 hs[kMaxM + 1];
  __shared__ double red[kThreads / 32];
  for (int t = ilo + threadIdx.x; t <= j; t += kThreads) hs[t] = h[t];
  __syncthreads();
  double a = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)kThreads + threadIdx.x; r < n; r += (int64_t)gridDim.x * kThreads) {
    double sr = 0.0, si = 0.0;
    for (int i = ilo; i <= j; ++i) {
      edg::cd v = ldc<T>(V, (int64_t)i * n + r);
      sr = fma(v.re, hs[i].x, fma(-v.im, hs[i].y, sr));
      si = fma(v.re, hs[i].y, fma(v.im, hs[i].x, si));
    }
    double2 x = w[r];
    x.x -= sr;
    x.y -= si;
    w[r] = x;
    a = fma(x.x, x.x, fma(x.y, x.y, a));
  }
  double t = block_sum1(a, red);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// c = beta0 * exp(-i T dt) e_1, T = tridiag(beta[1..m-1], alpha[0..m-1]); one thread.
// Scaling and squaring: exp(-iTdt) = (exp(-iTdt/2^s))^(2^s) applied to the
// vector, each factor a Taylor series truncated below 1e-18 relative.
__global__ void small_expm_k(const double* __restrict__ alpha, const double* __restrict__ beta, int m, double dt,
                             const double* __restrict__ beta0, double2* __restrict__ c, double* __restrict__ err) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double nrm = 0.0;  // infinity norm of T
  for (int i = 0; i < m; ++i) {
    double r = fabs(alpha[i]) + (i > 0 ? fabs(beta[i]) : 0.0) + (i + 1 < m ? fabs(beta[i + 1]) : 0.0);
    nrm = fmax(nrm, r);
  }
  int s = 0;
  double h = fabs(dt) * nrm;
  while (h > 0.5 && s < 60) {
    h *= 0.5;
    ++s;
  }
  const double tau = dt / ldexp(1.0, s);
  double vr[kMaxM], vi[kMaxM], tr[kMaxM], ti[kMaxM], ur[kMaxM], ui[kMaxM];
  for (int i = 0; i < m; ++i) vr[i] = vi[i] = 0.0;
  vr[0] = 1.0;
  const long reps = 1L << s;
  for (long rep = 0; rep < reps; ++rep) {
    // u = sum_k (-i tau T)^k v / k!
    for (int i = 0; i < m; ++i) {
      ur[i] = tr[i] = vr[i];
      ui[i] = ti[i] = vi[i];
    }
    for (int k = 1; k <= 40; ++k) {
      // t <- (-i tau T) t / k : (-i)(a + ib) = b - ia
      double nr[kMaxM], ni[kMaxM];
      double tmax = 0.0;
      for (int i = 0; i < m; ++i) {
        double xr = alpha[i] * tr[i], xi = alpha[i] * ti[i];
        if (i > 0) {
          xr += beta[i] * tr[i - 1];
          xi += beta[i] * ti[i - 1];
        }
        if (i + 1 < m) {
          xr += beta[i + 1] * tr[i + 1];
          xi += beta[i + 1] * ti[i + 1];
        }
        nr[i] = tau * xi / k;
        ni[i] = -tau * xr / k;
        tmax = fmax(tmax, fabs(nr[i]) + fabs(ni[i]));
      }
      double umax = 0.0;
      for (int i = 0; i < m; ++i) {
        tr[i] = nr[i];
        ti[i] = ni[i];
        ur[i] += tr[i];
        ui[i] += ti[i];
        umax = fmax(umax, fabs(ur[i]) + fabs(ui[i]));
      }
      if (tmax <= 1e-18 * umax) break;
    }
    for (int i = 0; i < m; ++i) {
      vr[i] = ur[i];
      vi[i] = ui[i];
    }
  }
  const double b0 = beta0[0];
  for (int i = 0; i < m; ++i) c[i] = make_double2(b0 * vr[i], b0 * vi[i]);
  // a posteriori estimate: beta_m |e_m^T exp(-iTdt) e_1| |psi|
  err[0] = fabs(beta[m]) * hypot(vr[m - 1], vi[m - 1]) * b0;
}

// psi[r] = sum_{i<m} V[i][r] c[i]
template <typename T>
__global__ void combine_k(const T* __restrict__ V, int64_t n, int m, const double2* __restrict__ c, T* __restrict__ psi) {
  __shared__ double2 cs[kMaxM];
  for (int t = threadIdx.x; t < m; t += blockDim.x) cs[t] = c[t];
  __syncthreads();
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
    double a = 0.0, b = 0.0;
    for (int i = 0; i < m; ++i) {
      edg::cd v = ldc<T>(V, (int64_t)i * n + r);
      a = fma(v.re, cs[i].x, fma(-v.im, cs[i].y, a));
      b = fma(v.re, cs[i].y, fma(v.im, cs[i].x, b));
    }
    stc<T>(psi, r, a, b);
  }
}

struct KLayout {
  int64_t V, w, h, partial, normp, alpha, beta, c, misc, total;
  int nblk;
};

inline int64_t al(int64_t x) { return (x + 255) & ~int64_t(255); }

KLayout klayout(const edg_krylov_problem* p) {
  KLayout L{};
  const int64_t n = p->n_rows;
  const int esz = p->vec_dtype == 2 ? 16 : 8;
  L.nblk = edg::kSmCount * 4;
  int64_t o = 0;
  L.V = o; o = al(o + (int64_t)(p->m + 1) * n * esz);
  L.w = o; o = al(o + n * 16);
  L.h = o; o = al(o + (int64_t)(kMaxM + 1) * 16);
  L.partial = o; o = al(o + (int64_t)L.nblk * (kMaxM + 1) * 16);
  L.normp = o; o = al(o + (int64_t)edg::kSmCount * 8 * 8);
  L.alpha = o; o = al(o + (kMaxM + 1) * 8);
  L.beta = o; o = al(o + (kMaxM + 2) * 8);
  L.c = o; o = al(o + (kMaxM + 1) * 16);
  L.misc = o; o = al(o + 8 * 8);  // [0] beta0, [1] err, [2] scratch
  L.total = o;
  return L;
}

template <typename T, typename SV>
int run_step(const edg_krylov_problem* p, T* psi, double dt, char* ws, double* err_out, cudaStream_t s) {
  const KLayout L = klayout(p);
  const int64_t n = p->n_rows;
  const int m = p->m;
  T* V = (T*)(ws + L.V);
  double2* w = (double2*)(ws + L.w);
  double2* h = (double2*)(ws + L.h);
  double2* partial = (double2*)(ws + L.partial);
  double* normp = (double*)(ws + L.normp);
  double* alpha = (double*)(ws + L.alpha);
  double* beta = (double*)(ws + L.beta);
  double2* c = (double2*)(ws + L.c);
  double* misc = (double*)(ws + L.misc);
  const int nb_norm = edg::kSmCount * 8;
  const unsigned gv = edg::grid_for(n, 256);
  cudaError_t e;
  if ((e = cudaMemsetAsync(alpha, 0, (kMaxM + 1) * 8, s)) != cudaSuccess) return edg::cuda_status(e, "krylov");
  if ((e = cudaMemsetAsync(beta, 0, (kMaxM + 2) * 8, s)) != cudaSuccess) return edg::cuda_status(e, "krylov");
  norm_k<T><<<nb_norm, kThreads, 0, s>>>(psi, n, normp);
  sqrt_sum_k<<<1, kThreads, 0, s>>>(normp, nb_norm, misc);  // beta0
  scale_k<T, T><<<gv, 256, 0, s>>>(psi, n, misc, V);
  for (int j = 0; j < m; ++j) {
    const T* vj = V + (int64_t)j * n;
    int st;
    if constexpr (std::is_same<SV, double>::value || std::is_same<SV, float>::value) {
      if (p->pk_words != nullptr)  // real packed matrix: (re, im) as two interleaved right-hand sides
        st = edg::launch_packed_spmv<SV>(2, 2, n, p->pk_tile_off, p->pk_words, (const SV*)p->pk_table, p->pk_count,
                                         p->pk_colbits, (const SV*)p->diag, (const SV*)vj, (double*)w, 0, nullptr,
                                         p->status, s, 1);
      else
        st = edg::launch_spmv<SV, T, double2>(1, n, p->nnz, p->rowptr, p->cols, (const SV*)p->vals,
                                              (const SV*)p->diag, vj, w, s, 0, p->spmv_group);
    } else {
      st = edg::launch_spmv<SV, T, double2>(1, n, p->nnz, p->rowptr, p->cols, (const SV*)p->vals, (const SV*)p->diag,
                                            vj, w, s, 0, p->spmv_group);
    }
    if (st) return st;
    // reorth_passes = 0: local recurrence (against v_{j-1}, v_j only);
    // 1 or 2: classical Gram-Schmidt over the whole basis, once or twice
    const int passes = p->reorth_passes == 0 ? 1 : p->reorth_passes;
    const int ilo = p->reorth_passes == 0 ? (j > 0 ? j - 1 : 0) : 0;
    for (int pass = 0; pass < passes; ++pass) {
      dots_k<T><<<L.nblk, kThreads, 0, s>>>(V, n, ilo, j, w, partial, kMaxM + 1);
      reduce_h_k<<<j + 1 - ilo, kThreads, 0, s>>>(partial, L.nblk, kMaxM + 1, ilo, j, h, alpha + j);
      update_k<T><<<nb_norm, kThreads, 0, s>>>(V, n, ilo, j, h, w, normp);
    }
    sqrt_sum_k<<<1, kThreads, 0, s>>>(normp, nb_norm, beta + j + 1);
    scale_k<double2, T><<<gv, 256, 0, s>>>(w, n, beta + j + 1, V + (int64_t)(j + 1) * n);
    if ((e = cudaGetLastError()) != cudaSuccess) return edg::cuda_status(e, "edg_krylov_step: lanczos");
  }
  small_expm_k<<<1, 1, 0, s>>>(alpha, beta, m, dt, misc, c, misc + 1);
  combine_k<T><<<gv, 256, 0, s>>>(V, n, m, c, psi);
  if ((e = cudaGetLastError()) != cudaSuccess) return edg::cuda_status(e, "edg_krylov_step: combine");
  if (err_out) {
    e = cudaMemcpyAsync(err_out, misc + 1, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return edg::cuda_status(e, "edg_krylov_step: error estimate");
  }
  return EDG_OK;
}

int check_k(const edg_krylov_problem* p) {
  EDG_REQUIRE(p != nullptr, "edg_krylov: null problem");
  EDG_REQUIRE(p->vec_dtype == 2 || p->vec_dtype == 3, "edg_krylov: vec_dtype must be 2 (c128) or 3 (c64)");
  EDG_REQUIRE(p->mat_dtype >= 0 && p->mat_dtype <= 3, "edg_krylov: bad mat_dtype");
  EDG_REQUIRE((p->mat_dtype == 0 || p->mat_dtype == 2) == (p->vec_dtype == 2),
              "edg_krylov: matrix and vectors must share the precision (f64/c128 or f32/c64)");
  EDG_REQUIRE(p->m >= 1 && p->m <= kMaxM, "edg_krylov: m must be 1..%d", kMaxM);
  EDG_REQUIRE(p->reorth_passes >= 0 && p->reorth_passes <= 2, "edg_krylov: reorth_passes must be 0..2");
  EDG_REQUIRE(p->n_rows > 0 && p->rowptr && p->diag, "edg_krylov: empty matrix");
  EDG_REQUIRE(p->pk_words == nullptr ||
                  ((p->mat_dtype == 0 || p->mat_dtype == 1) && p->pk_tile_off && p->pk_table && p->pk_count >= 1 &&
                   p->pk_count <= EDG_PACK_MAX_VALUES && p->pk_colbits >= 1 && p->pk_colbits <= 31 &&
                   p->n_rows < ((int64_t)1 << p->pk_colbits)),
              "edg_krylov: a packed layout needs a real matrix (mat_dtype 0 or 1) and a complete layout");
  return EDG_OK;
}

}  // namespace

extern "C" int64_t edg_krylov_workspace_bytes(const edg_krylov_problem* p) {
  if (check_k(p)) return -1;
  return klayout(p).total;
}

extern "C" int edg_krylov_step(const edg_krylov_problem* p, void* psi, double dt, void* workspace,
                               int64_t workspace_bytes, double* err_out, cudaStream_t stream) {
  int st = check_k(p);
  if (st) return st;
  EDG_REQUIRE(psi != nullptr && workspace != nullptr && workspace_bytes >= klayout(p).total,
              "edg_krylov_step: workspace too small");
  const bool c128 = p->vec_dtype == 2;
  (void)c128;
  switch (p->mat_dtype) {
    case 0: return run_step<double2, double>(p, (double2*)psi, dt, (char*)workspace, err_out, stream);
    case 2: return run_step<double2, double2>(p, (double2*)psi, dt, (char*)workspace, err_out, stream);
    case 1: return run_step<float2, float>(p, (float2*)psi, dt, (char*)workspace, err_out, stream);
    default: return run_step<float2, float2>(p, (float2*)psi, dt, (char*)workspace, err_out, stream);
  }
}
