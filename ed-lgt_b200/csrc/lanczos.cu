// Lanczos ground states with full or windowed reorthogonalisation, for nvec
// independent real-symmetric problems sharing the off-diagonal matrix
// (batched in one matvec).  Krylov vectors are stored in T (double or float),
// planar [vector][problem][row] with rows padded to four; the matvec input X
// is an interleaved [row][problem] copy of the candidate; the working vector
// w, every inner product, the recurrence coefficients and the tridiagonal
// eigen-solve are double precision.  The reorthogonalisation of a step reads
// V[lo..j] (lo = 0, or j - window): through the bulk-copy ring passes, or,
// when at most kSmallMax vectors are read, in one cooperative launch
// (reorth_small_k).
//
// Step j, delayed classical Gram-Schmidt with reorthogonalisation (DCGS2,
// Swirydowicz, Langou, Ananthan, Yang, Thomas, Numer. Linear Algebra Appl.
// 28 (2021) e2343): V[j] holds the candidate u_j, which has had one
// Gram-Schmidt pass; its second pass is done in this step.
//   w = H u_j                                   (spmv, double output)
//   one read of V[0..j]: s = V[0..j)^T u_j, alpha_u = u_j.u_j,
//                        z = V[0..j)^T w,   omega = u_j.w
//   r = sqrt(alpha_u - s.s), c = (omega - s.z) / r
//   alpha_j = (omega - 2 z.s + s.T s) / r^2, beta_j = (z_{j-1} - (T s)_{j-1}) / r
//   one read of V[0..j): V[j] = q_j = (u_j - V s) / r ; w -= V z + q_j c
//   V[j+1] = w / r (the next candidate, written by the update pass; the
//   step's formulas do not depend on a candidate's scale), beta_{j+1} = |w| / r
//   (refined at j+1)
// T is the j x j tridiagonal block of the previous steps.
// Every check_every steps the k lowest Ritz pairs of the tridiagonal matrix are
// computed on the device (multisection + inverse iteration) and the residual
// bound |beta_{j+1} s_{j}| is compared with tol * max(1, |theta|).
#include "reorth_bulk.cuh"
#include "spmv.cuh"
#include "tridiag.cuh"

#include <chrono>
#include <cmath>
#include <mutex>
#include <thread>
#include <vector>

namespace {

using edg::tridiag_body;
constexpr int kThreads = 256;
constexpr int kItile = 8;  // Krylov vectors per reduction tile
static_assert(kItile == edg::bulk::kVecs, "a ring stage of the dots pass is one reduction tile");
constexpr int kMaxK = 16;

// State of a device-driven solve (in the workspace).  The step kernels read
// j, the update pass advances it, the check kernel decides and schedules.
struct DevState {
  int j;           // Krylov vectors finished; the candidate is V[j]
  int done;        // every problem converged, or the Krylov limit reached
  int next_check;  // Krylov dimension of the next convergence check
  int checks;      // checks made
  int status;      // EDG_OK or EDG_ERR_NOT_CONVERGED
  int prev_m;      // dimension of the previous check
  int m_conv[4];   // per problem: dimension at convergence, 0 while running
  int m_use[4];    // per problem: dimension of its last tridiagonal solve
  int ticket;      // last-CTA counter of the check kernel
  int win;         // reorthogonalisation window (0: all of V[0..j))
  double prev_worst;
  double worst[4];       // worst relative residual of an unconverged problem
  double resid[4][kMaxK];
};

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

template <typename T>
__device__ __forceinline__ double ldv(const T* p, int64_t i) { return (double)p[i]; }

// Four consecutive Krylov entries (16-byte aligned: planes are padded to 4 rows).
__device__ __forceinline__ void ld4(const float* p, double* out) {
  float4 v = *reinterpret_cast<const float4*>(p);
  out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
}
__device__ __forceinline__ void ld4(const double* p, double* out) {
  double2 a = *reinterpret_cast<const double2*>(p);
  double2 b = *reinterpret_cast<const double2*>(p + 2);
  out[0] = a.x; out[1] = a.y; out[2] = b.x; out[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const double* v) {
  *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
__device__ __forceinline__ void st4(double* p, const double* v) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
}

// w (planar [NV][n_pad]) = uniform(-1, 1) or the interleaved start vectors v0
template <typename T, int NV>
__global__ void start_k(int64_t n, int64_t n_pad, uint64_t seed, const T* __restrict__ v0, double* __restrict__ w) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_pad * NV; i += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(i / n_pad);
    const int64_t r = i - v * n_pad;
    double x = 0.0;
    if (r < n) {
      if (v0) {
        x = (double)v0[r * NV + v];
      } else {
        uint64_t z = splitmix64(seed ^ splitmix64((uint64_t)(r * NV + v)));
        x = ((double)(z >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
      }
    }
    w[i] = x;
  }
}

// Block-reduces NV doubles per thread; threads < NV get the totals in vals[tid].
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
    vals[threadIdx.x] = a;
  }
  __syncthreads();
}

// |w_v|^2 block partials (planar w)
template <int NV>
__global__ void __launch_bounds__(kThreads) norm_k(const double* __restrict__ w, int64_t n_pad,
                                                   double* __restrict__ norm_partial) {
  __shared__ double red[(kThreads / 32) * NV];
  double nrm[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) nrm[v] = 0.0;
  for (int64_t r = blockIdx.x * (int64_t)kThreads + threadIdx.x; r < n_pad; r += (int64_t)gridDim.x * kThreads)
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double x = w[(int64_t)v * n_pad + r];
      nrm[v] = fma(x, x, nrm[v]);
    }
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

// v = w / beta (beta = 0 leaves a zero vector: invariant subspace), written to
// the planar Krylov slot (may be null) and to the interleaved matvec input X
// (may be null).
template <typename T, int NV>
__global__ void scale_store_k(const double* __restrict__ w, int64_t n, int64_t n_pad, const double* __restrict__ beta,
                              T* __restrict__ plane, T* __restrict__ X, int xs) {
  double inv[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) inv[v] = beta[v] > 0.0 ? 1.0 / beta[v] : 0.0;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n_pad; r += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const T x = (T)(w[(int64_t)v * n_pad + r] * inv[v]);
      if (plane) plane[(int64_t)v * n_pad + r] = x;
      if (X && r < n) X[r * xs + v] = x;
    }
  }
}

// First Krylov vector of the reorthogonalisation window at step j.
__device__ __forceinline__ int window_start(const DevState* st, int j) {
  const int w = st->win;
  return (w > 0 && j > w) ? j - w : 0;
}

// Sums of 16 per-lane values over a warp, scattered: afterwards lanes L and
// L^1 hold the total of value index ((L>>4)&1)*8 + ((L>>3)&1)*4 + ((L>>2)&1)*2
// + ((L>>1)&1).  Recursive halving: 8 + 4 + 2 + 1 + 1 shuffles instead of
// 16 x 5 for separate butterflies.
__device__ __forceinline__ double warp_reduce_scatter16(const double* v16) {
  const int lane = threadIdx.x & 31;
  double a[8];
  {
    const bool hi = lane & 16;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const double send = hi ? v16[k] : v16[k + 8];
      const double keep = hi ? v16[k + 8] : v16[k];
      a[k] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
  }
  {
    const bool hi = lane & 8;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const double send = hi ? a[k] : a[k + 4];
      const double keep = hi ? a[k + 4] : a[k];
      a[k] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
  }
  {
    const bool hi = lane & 4;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const double send = hi ? a[k] : a[k + 2];
      const double keep = hi ? a[k + 2] : a[k];
      a[k] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
  }
  {
    const bool hi = lane & 2;
    const double send = hi ? a[0] : a[1];
    const double keep = hi ? a[1] : a[0];
    a[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
  return a[0] + __shfl_xor_sync(0xffffffffu, a[0], 1);
}

// Coefficients of the delayed step from the totals hu, hw of V[lo..j] . u and
// V[lo..j] . w: one warp per problem computes r and c and the new
// tridiagonal entries alpha_j, beta_j from hu, hw and the previous alpha,
// beta (run by the last CTA of the pass that formed the totals).
template <int NV>
__device__ __forceinline__ void coef_epilogue(int lo, int j, const double* __restrict__ hu,
                                              const double* __restrict__ hw, double* __restrict__ alpha, int lda,
                                              double* __restrict__ beta, int ldb, double* __restrict__ rc) {
  const int lane = threadIdx.x & 31, v = threadIdx.x >> 5;
  if (v < NV) {
    const double* al = alpha + (int64_t)v * lda;
    double* be = beta + (int64_t)v * ldb;
    double ss = 0.0, sz = 0.0, sts = 0.0;
    for (int k = lo + lane; k < j; k += 32) {
      const double sk = __ldcg(hu + k * NV + v), zk = __ldcg(hw + k * NV + v);
      // (T s)_k over the leading j x j tridiagonal block (s = 0 below lo)
      double ts = al[k] * sk;
      if (k > lo) ts = fma(be[k], __ldcg(hu + (k - 1) * NV + v), ts);
      if (k + 1 < j) ts = fma(be[k + 1], __ldcg(hu + (k + 1) * NV + v), ts);
      ss = fma(sk, sk, ss);
      sz = fma(sk, zk, sz);
      sts = fma(sk, ts, sts);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ss += __shfl_xor_sync(0xffffffffu, ss, o);
      sz += __shfl_xor_sync(0xffffffffu, sz, o);
      sts += __shfl_xor_sync(0xffffffffu, sts, o);
    }
    if (lane == 0) {
      double ts_last = 0.0;
      if (j > lo) {
        ts_last = al[j - 1] * __ldcg(hu + (j - 1) * NV + v);
        if (j - 2 >= lo) ts_last = fma(be[j - 1], __ldcg(hu + (j - 2) * NV + v), ts_last);
      }
      const double r2 = __ldcg(hu + j * NV + v) - ss;
      const double rr = r2 > 0.0 ? sqrt(r2) : 0.0;
      const double ri = rr > 0.0 ? 1.0 / rr : 0.0;
      const double omega = __ldcg(hw + j * NV + v);
      rc[v] = ri;
      rc[NV + v] = (omega - sz) * ri;
      alpha[(int64_t)v * lda + j] = (omega - 2.0 * sz + sts) * ri * ri;
      if (j > lo) be[j] = (__ldcg(hw + (j - 1) * NV + v) - ts_last) * ri;
    }
  }
}

// hu[i][v] (r = 0), hw[i][v] (r = 1) = sum over the segment partials (fixed
// order), for i <= j strided over the CTA pairs of a fixed grid.  The last
// CTA to finish (ticket counter, reset by it) then computes, one warp per
// problem, r and c of the delayed step and the new tridiagonal entries
// alpha_j, beta_j from hu, hw and the previous alpha, beta.
template <int NV>
__global__ void __launch_bounds__(kThreads) reduce2_coef_k(const double* __restrict__ partial, int nblocks,
                                                           int64_t ld_p, const DevState* __restrict__ st,
                                                           double* __restrict__ hu, double* __restrict__ hw,
                                                           double* __restrict__ alpha, int lda,
                                                           double* __restrict__ beta, int ldb,
                                                           double* __restrict__ rc, int* __restrict__ counter) {
  __shared__ double red[(kThreads / 32) * NV];
  __shared__ int last;
  if (st->done) return;
  const int j = st->j;
  const int lo = window_start(st, j);
  const int r = blockIdx.x % 2;
  for (int i = lo + blockIdx.x / 2; i <= j; i += gridDim.x / 2) {
    double a[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += kThreads)
#pragma unroll
      for (int v = 0; v < NV; ++v) a[v] += partial[(((int64_t)i * 2 + r) * NV + v) * ld_p + b];
    block_sum<NV>(a, red);
    if (threadIdx.x < NV) (r == 0 ? hu : hw)[i * NV + threadIdx.x] = a[threadIdx.x];
  }
  if (threadIdx.x < NV) __threadfence();  // the writers publish before the ticket
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  coef_epilogue<NV>(lo, j, hu, hw, alpha, lda, beta, ldb, rc);
  if (threadIdx.x == 0) *counter = 0;
}

// ---------------------------------------------------------------------------
// Reorthogonalisation passes streamed through shared memory (reorth_bulk.cuh)
// ---------------------------------------------------------------------------

// Dots pass: partial[i][r][v][g] for the 1024-row segment g of problem v:
// V[i] . u (r = 0) and V[i] . w (r = 1) for i <= j, u = V[j].  Consumers
// reduce each tile of 8 vectors with a warp reduce-scatter and one sum over
// the 8 warps.
template <typename T, int NV>
__global__ void __launch_bounds__(edg::bulk::kThreadsAll) dots_bulk_k(const T* __restrict__ V, int64_t n_pad,
                                                                       const DevState* __restrict__ st,
                                                                       const double* __restrict__ w,
                                                                       double* __restrict__ partial, int64_t stride_i,
                                                                       int64_t n_seg, int* __restrict__ err_out) {
  using namespace edg::bulk;
  if (st->done) return;
  const int j = st->j;
  extern __shared__ __align__(128) unsigned char smraw[];
  Smem<T>& sm = *reinterpret_cast<Smem<T>*>(smraw);
  init_barriers(sm);
  const Run run = run_of((int64_t)NV * n_seg);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lo = window_start(st, j);
  const int n_vec = j + 1 - lo;
  if (warp == kConsumers / 32) {
    if (lane == 0) {
      produce(sm, V + (int64_t)lo * stride_i, n_pad, stride_i, n_seg, n_vec, run);
      if (sm.err) atomicExch(err_out, EDG_ERR_TIMEOUT);
    }
    return;
  }
  const int tid = threadIdx.x;
  const int64_t nq = n_pad / 4;
  const int idx = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
  int64_t k = 0;
  for (int64_t item = run.first; item < run.last; ++item) {
    const int64_t v = item / n_seg, g = item - v * n_seg;
    const int64_t q = g * kSegQuads + tid;
    const bool has = q < nq;
    double u4[4] = {0, 0, 0, 0}, w4[4] = {0, 0, 0, 0};
    if (has) {
      ld4(V + (int64_t)j * stride_i + v * n_pad + 4 * q, u4);
      ld4(w + v * n_pad + 4 * q, w4);
    }
    for (int i0 = 0; i0 < n_vec; i0 += kItile, ++k) {
      const int nt = min(kItile, n_vec - i0);
      double acc[2 * kItile];
#pragma unroll
      for (int t = 0; t < 2 * kItile; ++t) acc[t] = 0.0;
      const bool ok = acquire(sm, k);
      if (ok && has) {
        const T* st = &sm.ring[k % Smem<T>::S][0][4 * tid];
#pragma unroll
        for (int t = 0; t < kItile; ++t) {
          if (t < nt) {
            double x4[4];
            lds4(st + t * kSegRows, x4);
            acc[2 * t] = fma(x4[0], u4[0], fma(x4[1], u4[1], fma(x4[2], u4[2], fma(x4[3], u4[3], acc[2 * t]))));
            acc[2 * t + 1] =
                fma(x4[0], w4[0], fma(x4[1], w4[1], fma(x4[2], w4[2], fma(x4[3], w4[3], acc[2 * t + 1]))));
          }
        }
      }
      release(sm, k);
      const double tot = warp_reduce_scatter16(acc);
      if ((lane & 1) == 0) sm.red[warp][idx] = tot;
      edg::bulk::consumers_sync();
      if (tid < 2 * nt) {
        double a = 0.0;
        for (int wi = 0; wi < kConsumers / 32; ++wi) a += sm.red[wi][tid];
        const int t = tid >> 1, r = tid & 1;
        partial[(((int64_t)(lo + i0 + t) * 2 + r) * NV + v) * n_seg + g] = a;
      }
      edg::bulk::consumers_sync();
    }
  }
}

// Update pass: for every row of the CTA's segments, V[j] <- (u - sum_{i<j}
// V[i] s_i) / r, w <- w - sum_{i<j} V[i] z_i - V[j] c; the next candidate
// V[j+1] = w / r goes straight to the Krylov slot and the matvec input X (its
// norm, beta_{j+1}, is what the next step's dots see: every formula of the
// step is invariant under the candidate's scale); per-CTA partials of
// |w_v|^2, and the last CTA (ticket) forms |w_v| and beta_{j+1}.
template <typename T, int NV>
__global__ void __launch_bounds__(edg::bulk::kThreadsAll) update_bulk_k(
    T* __restrict__ V, int64_t n_pad, DevState* __restrict__ st, const double* __restrict__ hu,
    const double* __restrict__ hw, const double* __restrict__ rc, const double* __restrict__ w,
    double* __restrict__ norm_partial, int64_t stride_i, double* __restrict__ wnorm, double* __restrict__ beta,
    int ldb, int* __restrict__ counter, int64_t n_seg, int* __restrict__ err_out, T* __restrict__ X, int xs,
    int64_t n) {
  using namespace edg::bulk;
  if (st->done) return;
  const int j = st->j;
  extern __shared__ __align__(128) unsigned char smraw[];
  Smem<T>& sm = *reinterpret_cast<Smem<T>*>(smraw);
  init_barriers(sm);
  const Run run = run_of((int64_t)NV * n_seg);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int lo = window_start(st, j);
  if (warp == kConsumers / 32) {
    if (lane == 0) {
      produce(sm, (const T*)V + (int64_t)lo * stride_i, n_pad, stride_i, n_seg, j - lo, run);
      if (sm.err) atomicExch(err_out, EDG_ERR_TIMEOUT);
    }
    return;
  }
  const int tid = threadIdx.x;
  const int64_t nq = n_pad / 4;
  double nrm[NV];
#pragma unroll
  for (int vv = 0; vv < NV; ++vv) nrm[vv] = 0.0;
  int64_t k = 0;
  for (int64_t item = run.first; item < run.last; ++item) {
    const int v = (int)(item / n_seg);
    const int64_t g = item - (int64_t)v * n_seg;
    const int64_t q = g * kSegQuads + tid;
    const bool has = q < nq;
    T* U = V + (int64_t)j * stride_i + (int64_t)v * n_pad + 4 * q;
    const double* wp = w + (int64_t)v * n_pad + 4 * q;
    double u4[4] = {0, 0, 0, 0}, w4[4] = {0, 0, 0, 0};
    if (has) {
      ld4(U, u4);
      ld4(wp, w4);
    }
    for (int i0 = 0; i0 < j - lo; i0 += kVecs, ++k) {
      const int nt = min(kVecs, j - lo - i0);
      // the tile's coefficients (the same addresses in every lane: L1
      // broadcasts), loaded before the stage wait so they overlap it
      double si[kVecs], zi[kVecs];
#pragma unroll
      for (int t = 0; t < kVecs; ++t) {
        si[t] = t < nt ? __ldg(hu + (lo + i0 + t) * NV + v) : 0.0;
        zi[t] = t < nt ? __ldg(hw + (lo + i0 + t) * NV + v) : 0.0;
      }
      const bool ok = acquire(sm, k);
      if (ok && has) {
        const T* st = &sm.ring[k % Smem<T>::S][0][4 * tid];
#pragma unroll
        for (int t = 0; t < kVecs; ++t) {
          if (t < nt) {
            double x4[4];
            lds4(st + t * kSegRows, x4);
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              u4[e] = fma(-x4[e], si[t], u4[e]);
              w4[e] = fma(-x4[e], zi[t], w4[e]);
            }
          }
        }
      }
      release(sm, k);
    }
    if (has && !sm.err) {
      const double ri = rc[v], c = rc[NV + v];
      double q4[4], sq = 0.0;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        q4[e] = (double)(T)(u4[e] * ri);
        w4[e] = fma(-q4[e], c, w4[e]);
        sq = fma(w4[e], w4[e], sq);
        w4[e] *= ri;
      }
      st4(U, q4);
      st4(U + stride_i, w4);
#pragma unroll
      for (int e = 0; e < 4; ++e)
        if (4 * q + e < n) X[(4 * q + e) * xs + v] = (T)w4[e];
#pragma unroll
      for (int vv = 0; vv < NV; ++vv)
        if (vv == v) nrm[vv] += sq;
    }
  }
  // CTA partials of |w_v|^2 (consumer threads only: the producer warp has left)
#pragma unroll
  for (int vv = 0; vv < NV; ++vv) {
    double a = nrm[vv];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) sm.red[warp][vv] = a;
  }
  edg::bulk::consumers_sync();
  if (tid < NV) {
    double a = 0.0;
    for (int wi = 0; wi < kConsumers / 32; ++wi) a += sm.red[wi][tid];
    norm_partial[(int64_t)blockIdx.x * NV + tid] = a;
    __threadfence();
  }
  edg::bulk::consumers_sync();
  if (tid == 0) sm.last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
  edg::bulk::consumers_sync();
  if (!sm.last) return;
  __threadfence();
  if (warp < NV) {  // warp v: lanes stride over the CTAs, fixed-order butterfly
    double a = 0.0;
    for (int b = lane; b < (int)gridDim.x; b += 32) a += __ldcg(norm_partial + (int64_t)b * NV + warp);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) {
      const double nv = sqrt(a);
      wnorm[warp] = nv;
      beta[(int64_t)warp * ldb + j + 1] = nv * rc[warp];
    }
  }
  if (tid == 0) {
    *counter = 0;
    st->j = j + 1;  // every CTA read j before arriving at the ticket
  }
}

// ---------------------------------------------------------------------------
// Reorthogonalisation of one step for a short basis window (at most kSmallMax
// vectors V[lo..j]: the local window of the f32 phase, or the steps of a
// short refinement) as ONE cooperative launch: the dots phase, a grid-wide
// barrier, the step's coefficients formed by every CTA from the dots
// partials (the same sums in the same order everywhere), and the update
// phase over the rows in reverse order (the rows read last by the dots
// phase, still in L2, come first).  Every load of a row quad is in flight at
// once.  Same arithmetic as the ring passes row by row; only the order of
// the cross-CTA sums differs.
// ---------------------------------------------------------------------------
constexpr int kSmallMax = 8;        // vectors of V[lo..j] the small pass takes
constexpr int kSmallThreads = 256;  // threads of a small-pass CTA
constexpr int kSmallGridMax = edg::kSmCount * 4;  // CTAs of a small pass at most (the resident ones)

// four consecutive Krylov entries as loaded (converted to double when used)
template <typename T>
struct Raw4;
template <>
struct Raw4<float> {
  float4 a;
  __device__ void ld(const float* p) { a = *reinterpret_cast<const float4*>(p); }
  __device__ double operator[](int e) const { return (double)(e == 0 ? a.x : e == 1 ? a.y : e == 2 ? a.z : a.w); }
};
template <>
struct Raw4<double> {
  double2 a, b;
  __device__ void ld(const double* p) {
    a = *reinterpret_cast<const double2*>(p);
    b = *reinterpret_cast<const double2*>(p + 2);
  }
  __device__ double operator[](int e) const { return e == 0 ? a.x : e == 1 ? a.y : e == 2 ? b.x : b.y; }
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier of the small pass (every CTA is resident: cooperative
// launch).  bar[0] counts arrivals, bar[1] is the generation.  A wait longer
// than 1 s writes EDG_ERR_TIMEOUT to *err; once *err is set no CTA waits any
// more and every thread gets false.
__device__ bool small_barrier(unsigned* bar, int* err) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned g = ld_acquire_u32(bar + 1);
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const uint64_t t0 = edg::bulk::now_ns();
      for (unsigned spins = 1; ld_acquire_u32(bar + 1) == g; ++spins) {
        if ((spins & 255u) == 0) {
          if (*(volatile int*)err) break;
          if (edg::bulk::now_ns() - t0 > 1000000000ull) {
            atomicExch(err, EDG_ERR_TIMEOUT);
            break;
          }
        }
      }
    }
    __threadfence();
    ok_s = *(volatile int*)err == 0;
  }
  __syncthreads();
  return ok_s != 0;
}

// Coefficients of the delayed step for one problem (one warp) from its
// totals tot[2t] = V[lo+t] . u, tot[2t+1] = V[lo+t] . w (t <= j - lo) and the
// previous alpha, beta (entries below j only): 1/r, c, alpha_j, beta_j (the
// same formulas as coef_epilogue); lane 0 returns them.
__device__ __forceinline__ void coef_small(int lo, int j, const double* tot, const double* __restrict__ al,
                                           const double* __restrict__ be, double* out /*[4]*/) {
  const int lane = threadIdx.x & 31;
  double ss = 0.0, sz = 0.0, sts = 0.0;
  for (int k = lo + lane; k < j; k += 32) {
    const int t = k - lo;
    const double sk = tot[2 * t], zk = tot[2 * t + 1];
    double ts = al[k] * sk;
    if (k > lo) ts = fma(be[k], tot[2 * (t - 1)], ts);
    if (k + 1 < j) ts = fma(be[k + 1], tot[2 * (t + 1)], ts);
    ss = fma(sk, sk, ss);
    sz = fma(sk, zk, sz);
    sts = fma(sk, ts, sts);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ss += __shfl_xor_sync(0xffffffffu, ss, o);
    sz += __shfl_xor_sync(0xffffffffu, sz, o);
    sts += __shfl_xor_sync(0xffffffffu, sts, o);
  }
  if (lane == 0) {
    const int tj = j - lo;
    double ts_last = 0.0;
    if (j > lo) {
      ts_last = al[j - 1] * tot[2 * (tj - 1)];
      if (j - 2 >= lo) ts_last = fma(be[j - 1], tot[2 * (tj - 2)], ts_last);
    }
    const double r2 = tot[2 * tj] - ss;
    const double rr = r2 > 0.0 ? sqrt(r2) : 0.0;
    const double ri = rr > 0.0 ? 1.0 / rr : 0.0;
    const double omega = tot[2 * tj + 1];
    out[0] = ri;
    out[1] = (omega - sz) * ri;
    out[2] = (omega - 2.0 * sz + sts) * ri * ri;
    out[3] = j > lo ? (tot[2 * (tj - 1) + 1] - ts_last) * ri : 0.0;
  }
}

// The small pass.  Dots phase: CTA block b of problem v (gridDim.x = NV * G, v
// = blockIdx.x / G) sums V[lo+t] . u and V[lo+t] . w over its row quads into
// partial[cta][2t + r].  After the barrier every CTA forms the totals of all
// problems and their coefficients (CTA 0 writes them out: hu, hw, alpha_j,
// beta_j, rc).  Update phase: every thread takes row quads of all NV
// problems: V[j] <- (u - sum V[i] s_i) / r, w <- w - sum V[i] z_i - V[j] c,
// the next candidate V[j+1] = w / r to its Krylov slot and whole interleaved
// rows of the matvec input X; per-CTA partials of |w_v|^2, and the last CTA
// (ticket) forms |w_v| and beta_{j+1} and advances the step.  A barrier that
// runs out ends the solve (done flag; the error word says why).
template <typename T, int NV, int KV>
__global__ void __launch_bounds__(kSmallThreads) reorth_small_k(
    T* __restrict__ V, int64_t n_pad, DevState* __restrict__ st, const double* __restrict__ w,
    double* __restrict__ partial, int64_t stride_i, double* __restrict__ hu, double* __restrict__ hw,
    double* __restrict__ alpha, int lda, double* __restrict__ beta, int ldb, double* __restrict__ rc,
    double* __restrict__ norm_partial, double* __restrict__ wnorm, int* __restrict__ ticket,
    unsigned* __restrict__ bar, int* __restrict__ err, T* __restrict__ X, int xs, int64_t n) {
  __shared__ double red[kSmallThreads / 32][2 * kSmallMax];
  __shared__ double tot[NV][2 * kSmallMax];
  __shared__ double coef[NV][4];
  __shared__ double nred[kSmallThreads / 32][NV];
  __shared__ int last;
  if (st->done) return;
  const int j = st->j;
  const int lo = window_start(st, j);
  const int n_vec = j + 1 - lo;  // <= KV (the host picks this pass only then)
  const int n_w = n_vec - 1;     // window vectors besides the candidate
  const int G = (int)gridDim.x / NV;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t nq = n_pad / 4;
  // ---- dots phase --------------------------------------------------------
  {
    const int v = (int)blockIdx.x / G, b = (int)blockIdx.x - v * G;
    const T* Vv = V + (int64_t)lo * stride_i + (int64_t)v * n_pad;
    const T* U = V + (int64_t)j * stride_i + (int64_t)v * n_pad;
    const double* wv = w + (int64_t)v * n_pad;
    double acc[2 * kSmallMax];
#pragma unroll
    for (int t = 0; t < 2 * kSmallMax; ++t) acc[t] = 0.0;
    // two row quads per iteration (q and q + S) with all their loads in
    // flight (the update phase sets the kernel's registers; this phase fits
    // twice its loads in them); quads summed in the order q, q + S, ...
    const int64_t S = (int64_t)G * kSmallThreads;
    for (int64_t q = (int64_t)b * kSmallThreads + tid; q < nq; q += 2 * S) {
      Raw4<T> x[2][KV], u[2];
      Raw4<double> ww[2];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t qq = q + h * S;
        if (h == 0 || qq < nq) {
          u[h].ld(U + 4 * qq);
          ww[h].ld(wv + 4 * qq);
#pragma unroll
          for (int t = 0; t < KV; ++t)
            if (t < n_vec) x[h][t].ld(Vv + (int64_t)t * stride_i + 4 * qq);
        }
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (h == 1 && q + S >= nq) break;
#pragma unroll
        for (int t = 0; t < KV; ++t)
          if (t < n_vec) {
            const Raw4<T>& xt = x[h][t];
            acc[2 * t] =
                fma(xt[0], u[h][0], fma(xt[1], u[h][1], fma(xt[2], u[h][2], fma(xt[3], u[h][3], acc[2 * t]))));
            acc[2 * t + 1] = fma(xt[0], ww[h][0],
                                 fma(xt[1], ww[h][1], fma(xt[2], ww[h][2], fma(xt[3], ww[h][3], acc[2 * t + 1]))));
          }
      }
    }
    const int idx = ((lane >> 4) & 1) * 8 + ((lane >> 3) & 1) * 4 + ((lane >> 2) & 1) * 2 + ((lane >> 1) & 1);
    const double sum = warp_reduce_scatter16(acc);
    if ((lane & 1) == 0) red[warp][idx] = sum;
    __syncthreads();
    if (tid < 2 * n_vec) {
      double a = 0.0;
      for (int wi = 0; wi < kSmallThreads / 32; ++wi) a += red[wi][tid];
      partial[(int64_t)blockIdx.x * (2 * kSmallMax) + tid] = a;
    }
  }
  if (!small_barrier(bar, err)) {
    if (tid == 0) atomicExch(&st->done, 1);
    return;
  }
  // ---- totals and coefficients (every CTA, the same order everywhere) -----
  for (int e = warp; e < NV * 2 * n_vec; e += kSmallThreads / 32) {
    const int vv = e / (2 * n_vec), rem = e - vv * 2 * n_vec;
    double a = 0.0;
    for (int bb = lane; bb < G; bb += 32) a += __ldcg(partial + (int64_t)(vv * G + bb) * (2 * kSmallMax) + rem);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) tot[vv][rem] = a;
  }
  __syncthreads();
  if (warp < NV) {
    double out[4];
    coef_small(lo, j, tot[warp], alpha + (int64_t)warp * lda, beta + (int64_t)warp * ldb, out);
    if (lane == 0) {
#pragma unroll
      for (int q = 0; q < 4; ++q) coef[warp][q] = out[q];
      if (blockIdx.x == 0) {
        rc[warp] = out[0];
        rc[NV + warp] = out[1];
        alpha[(int64_t)warp * lda + j] = out[2];
        if (j > lo) beta[(int64_t)warp * ldb + j] = out[3];
        for (int t = 0; t < n_vec; ++t) {
          hu[(lo + t) * NV + warp] = tot[warp][2 * t];
          hw[(lo + t) * NV + warp] = tot[warp][2 * t + 1];
        }
      }
    }
  }
  __syncthreads();
  // ---- update phase: quads of all problems, the grid's quads in reverse ---
  double nrm[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) nrm[v] = 0.0;
  {
    const int64_t S = (int64_t)gridDim.x * kSmallThreads;
    const int64_t first = (int64_t)blockIdx.x * kSmallThreads + tid;
    const int64_t q_last = first < nq ? first + ((nq - 1 - first) / S) * S : -1;
    for (int64_t q = q_last; q >= 0; q -= S) {
      T xo[NV][4];  // the next candidate's rows of X, as stored
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        T* U = V + (int64_t)j * stride_i + (int64_t)v * n_pad + 4 * q;
        Raw4<T> x[KV - 1], u;
        Raw4<double> ww;
        u.ld(U);
        ww.ld(w + (int64_t)v * n_pad + 4 * q);
#pragma unroll
        for (int t = 0; t < KV - 1; ++t)
          if (t < n_w) x[t].ld(V + (int64_t)(lo + t) * stride_i + (int64_t)v * n_pad + 4 * q);
        double u4[4], w4[4], q4[4], sq = 0.0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          u4[e] = u[e];
          w4[e] = ww[e];
        }
#pragma unroll
        for (int t = 0; t < KV - 1; ++t)
          if (t < n_w) {
            const double s_t = tot[v][2 * t], z_t = tot[v][2 * t + 1];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
              u4[e] = fma(-x[t][e], s_t, u4[e]);
              w4[e] = fma(-x[t][e], z_t, w4[e]);
            }
          }
        const double ri = coef[v][0], c = coef[v][1];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          q4[e] = (double)(T)(u4[e] * ri);
          w4[e] = fma(-q4[e], c, w4[e]);
          sq = fma(w4[e], w4[e], sq);
          w4[e] *= ri;
          xo[v][e] = (T)w4[e];
        }
        st4(U, q4);
        st4(U + stride_i, w4);
        nrm[v] += sq;
      }
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int64_t r = 4 * q + e;
        if (r >= n) break;
        if (xs == 4) {
          double row[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
          for (int v = 0; v < NV && v < 4; ++v) row[v] = (double)xo[v][e];
          st4(X + r * 4, row);
        } else {
#pragma unroll
          for (int v = 0; v < NV; ++v) X[r * xs + v] = xo[v][e];
        }
      }
    }
  }
  // ---- |w_v|^2: CTA partials, the last CTA finishes the step ------------
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double a = nrm[v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) nred[warp][v] = a;
  }
  __syncthreads();
  if (tid < NV) {
    double a = 0.0;
    for (int wi = 0; wi < kSmallThreads / 32; ++wi) a += nred[wi][tid];
    norm_partial[(int64_t)blockIdx.x * NV + tid] = a;
    __threadfence();
  }
  __syncthreads();
  if (tid == 0) last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (warp < NV) {  // warp v: lanes stride over the CTAs, fixed-order butterfly
    double a = 0.0;
    for (int bb = lane; bb < (int)gridDim.x; bb += 32) a += __ldcg(norm_partial + (int64_t)bb * NV + warp);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) {
      const double nv = sqrt(a);
      wnorm[warp] = nv;
      beta[(int64_t)warp * ldb + j + 1] = nv * coef[warp][0];
    }
  }
  if (tid == 0) {
    *ticket = 0;
    st->j = j + 1;  // every CTA read j before arriving at the ticket
  }
}

// Convergence check after a step, launched after every step (one CTA per
// problem).  It works only when the state's schedule says a check is due:
// then each CTA of an unconverged problem finds the invariant-subspace
// dimension, solves its tridiagonal matrix and tests the residual bounds;
// the last CTA sets the done flag, schedules the next check from the
// contraction of the worst residual (never sooner than check_every steps,
// never later than 4 * check_every) and writes the progress words to the
// host.  Otherwise block 0 only publishes the step count.
template <int NV>
__global__ void __launch_bounds__(kThreads) check_k(DevState* __restrict__ st, const double* __restrict__ alpha,
                                                    int lda, const double* __restrict__ beta, int ldb, int m_max,
                                                    int64_t n, int k, double tol, int check_every,
                                                    double* __restrict__ tri_eval, double* __restrict__ tri_vec,
                                                    int ld_s, double* __restrict__ tri_work,
                                                    int32_t* __restrict__ host_progress) {
  __shared__ int mv_s, exact_s, last_s;
  volatile DevState* vst = st;
  if (vst->done) return;
  const int m = vst->j;
  const bool due = m >= vst->next_check || m >= m_max || (int64_t)m >= n;
  if (!due) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && host_progress) {
      volatile int32_t* hp = host_progress;
      hp[0] = m;
    }
    return;
  }
  const int v = blockIdx.x;
  if (vst->m_conv[v] == 0) {
    const double* al = alpha + (int64_t)v * lda;
    const double* be = beta + (int64_t)v * ldb;
    if (threadIdx.x == 0) {
      double scale = 0.0;
      for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(al[i]) + fabs(be[i]));
      const double thr = 1e-12 * fmax(scale, 1e-300);
      int mv = m;
      for (int i = 1; i <= m; ++i)
        if (fabs(be[i]) <= thr) {
          mv = i;
          break;
        }
      mv_s = mv;
      exact_s = mv < m || (mv == m && fabs(be[m]) <= thr) || (int64_t)m == n;
    }
    __syncthreads();
    const int mv = mv_s, kk = k < mv ? k : mv;
    double* S = tri_vec + (int64_t)v * kMaxK * ld_s;
    for (int e = threadIdx.x; e < kMaxK * ld_s; e += kThreads) S[e] = 0.0;
    __syncthreads();
    tridiag_body(al, be, mv, kk, tri_eval + (int64_t)v * kMaxK, S, ld_s, tri_work + (int64_t)v * 6 * ld_s);
    __syncthreads();
    if (threadIdx.x == 0) {
      const bool exact = exact_s != 0;
      bool ok = kk == k || exact;
      double worst = 0.0;
      for (int q = 0; q < kk; ++q) {
        const double theta = tri_eval[(int64_t)v * kMaxK + q];
        const double last = S[(int64_t)q * ld_s + (mv - 1)];
        const double r = exact ? 0.0 : fabs(be[mv] * last);
        vst->resid[v][q] = r;
        if (r > tol * fmax(1.0, fabs(theta))) ok = false;
        worst = fmax(worst, r / fmax(1.0, fabs(theta)));
      }
      vst->m_use[v] = mv;
      vst->worst[v] = ok ? 0.0 : worst;
      if (ok) vst->m_conv[v] = mv;
      __threadfence();
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) last_s = atomicAdd(&st->ticket, 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!last_s || threadIdx.x != 0) return;
  __threadfence();
  vst->ticket = 0;
  bool all = true;
  double worst = 0.0;
  for (int vv = 0; vv < NV; ++vv)
    if (vst->m_conv[vv] == 0) {
      all = false;
      worst = fmax(worst, vst->worst[vv]);
    }
  int done = all ? 1 : 0;
  if (!all && (m >= m_max || (int64_t)m >= n)) {
    done = 1;
    vst->status = EDG_ERR_NOT_CONVERGED;
  }
  if (!done) {
    int step = check_every;
    const double pw = vst->prev_worst;
    if (pw > 0.0 && worst > 0.0 && worst < pw && m > vst->prev_m) {
      const double rate = log(worst / pw) / (double)(m - vst->prev_m);  // < 0
      const double need = log(tol / worst) / rate;                       // steps to reach tol
      const int predicted = (int)floor(need * 0.8);
      if (predicted > step) step = predicted < 4 * check_every ? predicted : 4 * check_every;
    }
    vst->prev_worst = worst;
    vst->prev_m = m;
    vst->next_check = m + step;
  }
  vst->checks = vst->checks + 1;
  vst->done = done;
  __threadfence();
  if (host_progress) {
    volatile int32_t* hp = host_progress;
    hp[1] = done;
    __threadfence_system();
    hp[0] = m;
  }
}

__global__ void state_init_k(DevState* st, int first_check, int win) {
  if (threadIdx.x != 0) return;
  DevState s{};
  s.next_check = first_check;
  s.win = win;
  s.prev_worst = -1.0;
  *st = s;
}

// ---------------------------------------------------------------------------
// Tridiagonal eigen-solve (one CTA per problem)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) tridiag_k(const double* __restrict__ alpha, int lda,
                                                      const double* __restrict__ beta, int ldb, int m, int k,
                                                      double* __restrict__ evals, double* __restrict__ evecs,
                                                      int ldv, double* __restrict__ work, int ldw) {
  const int prob = blockIdx.x;
  tridiag_body(alpha + (int64_t)prob * lda, beta + (int64_t)prob * ldb, m, k, evals + (int64_t)prob * k,
               evecs ? evecs + (int64_t)prob * k * ldv : nullptr, ldv, work + (int64_t)prob * ldw);
}

// w (planar) = sum_{i<m} V[i][v][r] S[v][e][i]
template <typename T, int NV>
__global__ void ritz_k(const T* __restrict__ V, int64_t n_pad, int m, const double* __restrict__ S, int ldk, int e,
                       int lds, int64_t stride_i, double* __restrict__ w) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_pad * NV; g += (int64_t)gridDim.x * blockDim.x) {
    const int v = (int)(g / n_pad);
    const double* s = S + ((int64_t)v * ldk + e) * lds;
    double acc = 0.0;
    for (int i = 0; i < m; ++i) acc = fma(ldv(V, (int64_t)i * stride_i + g), s[i], acc);
    w[g] = acc;
  }
}

// ---------------------------------------------------------------------------
// Workspace layout
// ---------------------------------------------------------------------------
struct Layout {
  int64_t V, X, w, h, partial, small, normp, alpha, beta, tri_eval, tri_vec, tri_work, sync, state, total;
  int nblk_dot, nblk_upd, m_max, ld_h;
  int64_t n_pad;
};

inline int64_t align256(int64_t x) { return (x + 255) & ~int64_t(255); }

Layout make_layout(const edg_lanczos_problem* p) {
  Layout L{};
  const int64_t n = p->n_rows, nv = p->nvec;
  const int esz = p->dtype == 0 ? 8 : 4;
  L.n_pad = (n + 3) & ~int64_t(3);
  L.m_max = p->max_iter;
  L.ld_h = L.m_max + 1;
  // partial slots: one per warp row block of the dots kernel, one per CTA of
  // the update kernel; the norm kernels use at least kSmCount * 8 CTAs
  // dot partials: one slot per 1024-row segment of a problem; norm partials:
  // one per CTA of the update pass (at most kSmCount * 8)
  const int64_t n_seg = (L.n_pad / 4 + edg::bulk::kSegQuads - 1) / edg::bulk::kSegQuads;
  L.nblk_dot = (int)(n_seg > edg::kSmCount * 8 ? n_seg : edg::kSmCount * 8);
  L.nblk_upd = edg::kSmCount * 8;
  int64_t off = 0;
  L.V = off; off = align256(off + (int64_t)(L.m_max + 1) * L.n_pad * nv * esz);
  L.X = off; off = align256(off + n * (nv == 3 ? 4 : nv) * esz);  // matvec input, rows padded to 4 for nv = 3
  L.w = off; off = align256(off + L.n_pad * nv * 8);
  L.h = off; off = align256(off + (int64_t)(2 * (L.m_max + 1) + 3) * nv * 8);  // hu | hw | rc | |w|
  L.partial = off; off = align256(off + (int64_t)L.nblk_dot * (L.m_max + 1) * 2 * nv * 8);
  L.small = off; off = align256(off + (int64_t)kSmallGridMax * 2 * kSmallMax * 8);  // dots partials of the small passes
  L.normp = off; off = align256(off + (int64_t)L.nblk_upd * nv * 8);
  L.alpha = off; off = align256(off + (int64_t)nv * (L.m_max + 1) * 8);   // [nv][m_max+1]
  L.beta = off; off = align256(off + (int64_t)nv * (L.m_max + 2) * 8);    // [nv][m_max+2]
  L.tri_eval = off; off = align256(off + (int64_t)nv * kMaxK * 8);
  L.tri_vec = off; off = align256(off + (int64_t)nv * kMaxK * (L.m_max + 1) * 8);
  L.tri_work = off; off = align256(off + (int64_t)nv * 6 * (L.m_max + 1) * 8);
  L.sync = off; off = align256(off + 8 * (int64_t)sizeof(int));  // last-CTA tickets | error word | grid barrier
  L.state = off; off = align256(off + (int64_t)sizeof(DevState));
  L.total = off;
  return L;
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
  const int64_t n = p->n_rows, n_pad = L.n_pad;
  const int k = p->k;
  T* V = (T*)(ws + L.V);
  T* X = (T*)(ws + L.X);
  double* w = (double*)(ws + L.w);
  double* h = (double*)(ws + L.h);
  double* partial = (double*)(ws + L.partial);
  double* normp = (double*)(ws + L.normp);
  double* alpha = (double*)(ws + L.alpha);  // [NV][m_max+1]
  double* beta = (double*)(ws + L.beta);    // [NV][m_max+2], beta[v][i] couples i-1 and i
  double* tri_eval = (double*)(ws + L.tri_eval);
  double* tri_vec = (double*)(ws + L.tri_vec);  // [NV][kMaxK][m_max+1]
  double* tri_work = (double*)(ws + L.tri_work);
  DevState* st = (DevState*)(ws + L.state);
  const int ld_a = L.m_max + 1, ld_b = L.m_max + 2, ld_s = L.m_max + 1;
  const int64_t stride_i = n_pad * NV;  // entries per Krylov vector (all problems)
  double* hu = h;                                   // [m_max+1][NV] dots with the candidate
  double* hw = h + (int64_t)(L.m_max + 1) * NV;      // [m_max+1][NV] dots with w
  double* rc = hw + (int64_t)(L.m_max + 1) * NV;     // [2][NV]: 1/r, c of the current step
  double* wnorm = rc + 2 * NV;                        // [NV]: |w| of the next candidate
  int* tickets = (int*)(ws + L.sync);                  // [2] last-CTA counters (left at 0)
  int* err_word = tickets + 2;                          // EDG_ERR_TIMEOUT when a ring or barrier wait ran out
  unsigned* small_bar = (unsigned*)(tickets + 4);       // [2] grid barrier of the small pass (count, generation)
  const unsigned g_vec = edg::grid_for(n_pad, 256);
  const int first_check = p->check_every > 8 ? p->check_every : 8;
  constexpr int kXs = NV == 3 ? 4 : NV;  // row stride of the matvec input X
  cudaError_t e;
  // device address of the caller's pinned progress words (NULL: host syncs)
  int32_t* progress_dev = nullptr;
  volatile int32_t* progress = p->host_progress;
  if (progress) {
    if (cudaHostGetDevicePointer((void**)&progress_dev, (void*)p->host_progress, 0) != cudaSuccess) {
      cudaGetLastError();  // not pinned and mapped: fall back to synchronising
      progress = nullptr;
      progress_dev = nullptr;
    } else {
      progress[0] = 0;
      progress[1] = 0;
    }
  }
  // padding rows (r >= n) of w are zero from start_k on, so every Krylov plane
  // written from w has zero padding and no reset of V is needed
  start_k<T, NV><<<edg::grid_for(n_pad * NV, 256), 256, 0, s>>>(n, n_pad, p->seed, (const T*)p->v0, w);
  norm_k<NV><<<L.nblk_upd, kThreads, 0, s>>>(w, n_pad, normp);
  beta_k<NV><<<1, kThreads, 0, s>>>(normp, L.nblk_upd, h);
  scale_store_k<T, NV><<<g_vec, 256, 0, s>>>(w, n, n_pad, h, V, X, kXs);
  zero_k<NV><<<(NV * ld_b + 255) / 256, 256, 0, s>>>(beta, NV * ld_b);
  zero_k<NV><<<(NV * ld_a + 255) / 256, 256, 0, s>>>(alpha, NV * ld_a);
  state_init_k<<<1, 32, 0, s>>>(st, first_check, p->reorth_window);
  if ((e = cudaMemsetAsync(tickets, 0, 8 * sizeof(int), s)) != cudaSuccess)
    return edg::cuda_status(e, "edg_lanczos: tickets");
  if ((e = cudaGetLastError()) != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: start");
  // the reorthogonalisation passes: persistent grids of the bulk-copy kernels
  const size_t dot_smem = sizeof(edg::bulk::Smem<T>);
  const size_t upd_smem = sizeof(edg::bulk::Smem<T>);
  const int64_t n_seg = (n_pad / 4 + edg::bulk::kSegQuads - 1) / edg::bulk::kSegQuads;
  int occ_dot = 0, occ_upd = 0, n_sm = 0, dev = 0;
  e = cudaFuncSetAttribute(dots_bulk_k<T, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dot_smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(update_bulk_k<T, NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)upd_smem);
  if (e == cudaSuccess) e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_dot, dots_bulk_k<T, NV>, edg::bulk::kThreadsAll, dot_smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_upd, update_bulk_k<T, NV>, edg::bulk::kThreadsAll,
                                                      upd_smem);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: reorthogonalisation set-up");
  if (occ_dot < 1 || occ_upd < 1) {
    edg::set_error("edg_lanczos: the reorthogonalisation kernels do not fit on an SM");
    return EDG_ERR_ARG;
  }
  const int64_t items = n_seg * NV;
  auto grid_of = [&](int occ) {
    int64_t g = (int64_t)n_sm * (occ < 2 ? occ : 2);
    if (g > items) g = items;
    if (g > edg::kSmCount * 8) g = edg::kSmCount * 8;
    return (unsigned)(g < 1 ? 1 : g);
  };
  const unsigned g_dot = grid_of(occ_dot), g_upd = grid_of(occ_upd);
  const unsigned g_red = 2u * (unsigned)(L.m_max + 1 < 2 * edg::kSmCount ? L.m_max + 1 : 2 * edg::kSmCount);
  // one Lanczos step and its check; every kernel reads the step index and the
  // done flag from the device state
  // short windows (the local window of the f32 phase, or a refinement of at
  // most kSmallMax steps) take the streaming small passes
  const bool small_passes = (p->reorth_window > 0 && p->reorth_window < kSmallMax) || L.m_max <= kSmallMax;
  // most vectors of V[lo..j] a step reads: window + 1, or the Krylov limit
  const int small_kv = p->reorth_window > 0 && p->reorth_window < kSmallMax
                           ? (p->reorth_window + 1 < L.m_max ? p->reorth_window + 1 : L.m_max)
                           : L.m_max;
  double* small_partial = (double*)(ws + L.small);
  const int64_t nq = n_pad / 4;
  auto clamp_grid = [](int64_t want, int64_t cap) { return (unsigned)(want < 1 ? 1 : (want < cap ? want : cap)); };
  // the small pass: one cooperative launch whose grid is the CTAs resident at
  // once, split evenly over the problems
  const int small_kv_t = small_kv <= 5 ? 5 : kSmallMax;
  int occ_small = 0;
  if (small_passes) {
    int coop = 0;
    cudaError_t eo = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
    if (eo == cudaSuccess)
      eo = small_kv_t == 5 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_small, reorth_small_k<T, NV, 5>,
                                                                           kSmallThreads, 0)
                           : cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                                 &occ_small, reorth_small_k<T, NV, kSmallMax>, kSmallThreads, 0);
    if (eo != cudaSuccess) return edg::cuda_status(eo, "edg_lanczos: small-pass occupancy");
    if (!coop || occ_small < 1) {
      edg::set_error("edg_lanczos: the small reorthogonalisation pass needs a cooperative launch");
      return EDG_ERR_ARG;
    }
  }
  const int64_t small_resident = (int64_t)n_sm * (occ_small < 1 ? 1 : occ_small);
  const unsigned g_small =
      clamp_grid((nq + kSmallThreads - 1) / kSmallThreads,
                 (small_resident < kSmallGridMax ? small_resident : kSmallGridMax) / NV) * NV;
  const bool sell = p->sell_entries != nullptr && p->dtype == 1;
  auto matvec = [&](cudaStream_t cs) -> int {
    if (p->pk_words != nullptr)
      return edg::launch_packed_spmv<T>(NV, kXs, n, p->pk_tile_off, p->pk_words, (const T*)p->pk_table,
                                        p->pk_count, p->pk_colbits, (const T*)p->diag, X, w, n_pad, &st->done,
                                        err_word, cs);
    if (sell)
      return edg::launch_sell_spmv(NV, kXs, (n + 31) / 32, p->sell_perm, p->sell_width, p->sell_off,
                                   (const uint2*)p->sell_entries, (const float*)p->diag, (const float*)X, w, n_pad,
                                   &st->done, cs);
    return edg::launch_spmv<T, T, double>(NV, n, p->nnz, p->rowptr, p->cols, (const T*)p->vals, (const T*)p->diag, X,
                                          w, cs, n_pad, p->spmv_group, &st->done, kXs);
  };
  // the reorthogonalisation of one step: dots, coefficients, update
  auto enqueue_reorth = [&](cudaStream_t cs) -> cudaError_t {
    if (small_passes) {
      int* tk = tickets + 1;
      void* args[] = {&V, (void*)&n_pad, &st, &w, &small_partial, (void*)&stride_i, &hu, &hw, &alpha, (void*)&ld_a,
                      &beta, (void*)&ld_b, &rc, &normp, &wnorm, &tk, &small_bar, &err_word, &X, (void*)&kXs,
                      (void*)&n};
      const void* fn = small_kv_t == 5 ? (const void*)reorth_small_k<T, NV, 5>
                                       : (const void*)reorth_small_k<T, NV, kSmallMax>;
      return cudaLaunchCooperativeKernel(fn, dim3(g_small), dim3(kSmallThreads), args, 0, cs);
    }
    dots_bulk_k<T, NV><<<g_dot, edg::bulk::kThreadsAll, dot_smem, cs>>>(V, n_pad, st, w, partial, stride_i, n_seg,
                                                                          err_word);
    reduce2_coef_k<NV><<<g_red, kThreads, 0, cs>>>(partial, (int)n_seg, n_seg, st, hu, hw, alpha, ld_a, beta, ld_b, rc,
                                                   tickets);
    update_bulk_k<T, NV><<<g_upd, edg::bulk::kThreadsAll, upd_smem, cs>>>(V, n_pad, st, hu, hw, rc, w, normp, stride_i,
                                                                            wnorm, beta, ld_b, tickets + 1, n_seg,
                                                                            err_word, X, kXs, n);
    return cudaGetLastError();
  };
  const int launches_per_step = small_passes ? 3 : 5;  // matvec, reorthogonalisation, check
  auto enqueue_step = [&](cudaStream_t cs) -> int {
    int st_ = matvec(cs);
    if (st_) return st_;
    const cudaError_t er = enqueue_reorth(cs);
    return er == cudaSuccess ? EDG_OK : edg::cuda_status(er, "edg_lanczos: reorthogonalisation");
  };
  auto enqueue_check = [&](cudaStream_t cs) {
    check_k<NV><<<NV, kThreads, 0, cs>>>(st, alpha, ld_a, beta, ld_b, L.m_max, n, k, p->tol, p->check_every,
                                         tri_eval, tri_vec, ld_s, tri_work, progress_dev);
  };
  // wait until `target` steps are done or the solve has finished
  auto wait_progress = [&](int target) -> int {
    if (!progress) {
      cudaError_t err = cudaStreamSynchronize(s);
      return err == cudaSuccess ? EDG_OK : edg::cuda_status(err, "edg_lanczos: step");
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned it = 0; progress[0] < target && progress[1] == 0; ++it) {
      if ((it & 255u) == 255u) {
        cudaError_t q = cudaStreamQuery(s);
        if (q == cudaSuccess) break;  // nothing more will come
        if (q != cudaErrorNotReady) return edg::cuda_status(q, "edg_lanczos: step");
        if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(120)) {
          edg::set_error("edg_lanczos: no progress from the device for 120 s");
          return EDG_ERR_TIMEOUT;
        }
        std::this_thread::yield();
      }
    }
    return EDG_OK;
  };
  auto read_state = [&](DevState* hs) -> int {
    cudaError_t err = cudaMemcpyAsync(hs, st, sizeof(DevState), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    return err == cudaSuccess ? EDG_OK : edg::cuda_status(err, "edg_lanczos: state");
  };
  const bool timing = p->stats != nullptr;
  double t_spmv = 0.0, t_reorth = 0.0, t_check = 0.0;
  int64_t launches = 9;
  DevState hs{};
  int rc_ = EDG_OK;
  if (timing) {
    // instrumented: steps launched one by one with events around each phase
    cudaEvent_t ev[4];
    for (auto& x : ev) cudaEventCreate(&x);
    for (int j = 0; j < L.m_max; ++j) {
      cudaEventRecord(ev[0], s);
      int st_ = matvec(s);
      if (st_) return st_;
      cudaEventRecord(ev[1], s);
      if ((e = enqueue_reorth(s)) != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: reorthogonalisation");
      cudaEventRecord(ev[2], s);
      enqueue_check(s);
      cudaEventRecord(ev[3], s);
      if ((e = cudaGetLastError()) != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: step");
      if ((rc_ = read_state(&hs))) return rc_;
      float a = 0.f, b = 0.f, c = 0.f;
      cudaEventElapsedTime(&a, ev[0], ev[1]);
      cudaEventElapsedTime(&b, ev[1], ev[2]);
      cudaEventElapsedTime(&c, ev[2], ev[3]);
      t_spmv += a;
      t_reorth += b;
      t_check += c;
      launches += launches_per_step;
      if (hs.done) break;
    }
    for (auto& x : ev) cudaEventDestroy(x);
  } else {
    // graph of kStepsPerGraph steps (each with its check), replayed one
    // replay ahead of the host, which polls the device's progress words
    constexpr int kStepsPerGraph = 4;
    cudaStream_t cs = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: capture");
    for (int q = 0; q < kStepsPerGraph && rc_ == EDG_OK; ++q) {
      rc_ = enqueue_step(cs);
      if (rc_ == EDG_OK) enqueue_check(cs);
    }
    cudaError_t ec = cudaStreamEndCapture(cs, &graph);
    if (rc_ == EDG_OK && ec != cudaSuccess) rc_ = edg::cuda_status(ec, "edg_lanczos: capture");
    if (rc_ == EDG_OK && (ec = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess)
      rc_ = edg::cuda_status(ec, "edg_lanczos: graph instantiate");
    int enq = 0;
    const int limit = (int)(L.m_max < n ? L.m_max : n);
    if (rc_ == EDG_OK) {
      ec = cudaGraphLaunch(exec, s);
      if (ec != cudaSuccess) rc_ = edg::cuda_status(ec, "edg_lanczos: graph launch");
      enq += kStepsPerGraph;
    }
    while (rc_ == EDG_OK) {
      const bool more = enq < limit;
      if (more) {
        ec = cudaGraphLaunch(exec, s);
        if (ec != cudaSuccess) {
          rc_ = edg::cuda_status(ec, "edg_lanczos: graph launch");
          break;
        }
        enq += kStepsPerGraph;
      }
      const int target = more ? enq - kStepsPerGraph : limit;
      rc_ = wait_progress(target < limit ? target : limit);
      if (rc_) break;
      if (progress ? progress[1] != 0 : (read_state(&hs) == EDG_OK && hs.done)) break;
      if (!more) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(cs);
    if (rc_) return rc_;
    launches += (int64_t)enq * launches_per_step;
  }
  if ((rc_ = read_state(&hs))) return rc_;
  const int j_end = hs.j;
  std::vector<double> hev((size_t)NV * kMaxK);
  e = cudaMemcpyAsync(hev.data(), tri_eval, sizeof(double) * NV * kMaxK, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: ritz values");
  int m_all = 1;
  for (int v = 0; v < NV; ++v) {
    const int mv = hs.m_conv[v] ? hs.m_conv[v] : (hs.m_use[v] ? hs.m_use[v] : 1);
    const int kk = k < mv ? k : mv;
    for (int q = 0; q < k; ++q) {
      evals[v * k + q] = q < kk ? hev[v * kMaxK + q] : NAN;
      if (resid_out) resid_out[v * k + q] = q < kk ? hs.resid[v][q] : NAN;
    }
    if (iters_out) iters_out[v] = mv;
    m_all = mv > m_all ? mv : m_all;
  }
  if (evecs) {
    // S rows beyond each problem's m are zero, so one pass over m_all vectors serves all problems
    for (int q = 0; q < k; ++q) {
      ritz_k<T, NV><<<edg::grid_for(n_pad * NV, 256), 256, 0, s>>>(V, n_pad, m_all, tri_vec, kMaxK, q, ld_s,
                                                                   stride_i, w);
      norm_k<NV><<<L.nblk_upd, kThreads, 0, s>>>(w, n_pad, normp);
      beta_k<NV><<<1, kThreads, 0, s>>>(normp, L.nblk_upd, h);
      scale_store_k<T, NV><<<g_vec, 256, 0, s>>>(w, n, n_pad, h, (T*)nullptr, (T*)evecs + (int64_t)q * n * NV, NV);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: ritz vectors");
  }
  int h_err = 0;
  e = cudaMemcpyAsync(&h_err, err_word, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos: finish");
  if (h_err != 0) {
    edg::set_error("edg_lanczos: a shared-memory ring wait of the reorthogonalisation ran out");
    return EDG_ERR_TIMEOUT;
  }
  if (timing) {
    launches += 2 + (evecs ? 4 * k : 0);
    p->stats[0] = t_spmv;
    p->stats[1] = (double)j_end;
    p->stats[2] = t_reorth;
    p->stats[3] = (double)launches;
    p->stats[4] = (double)j_end;
    p->stats[5] = t_check;
  }
  if (hs.status == EDG_ERR_NOT_CONVERGED) {
    edg::set_error("edg_lanczos: not converged in %d steps", L.m_max);
    return EDG_ERR_NOT_CONVERGED;
  }
  return EDG_OK;
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
  EDG_REQUIRE(p->reorth_window >= 0, "edg_lanczos: reorth_window must be >= 0");
  EDG_REQUIRE(p->sell_entries == nullptr || (p->sell_perm && p->sell_width && p->sell_off),
              "edg_lanczos: incomplete SELL layout");
  EDG_REQUIRE(p->pk_words == nullptr ||
                  (p->pk_tile_off && p->pk_table && p->pk_count >= 1 && p->pk_count <= EDG_PACK_MAX_VALUES &&
                   p->pk_colbits >= 1 && p->pk_colbits <= 31 && p->n_rows < ((int64_t)1 << p->pk_colbits)),
              "edg_lanczos: incomplete or inconsistent packed layout");
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
