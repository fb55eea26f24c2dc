// Batched Lanczos for many small sector Hamiltonians (charge sectors, coupling
// sweeps) in one persistent launch.
//
// Each CTA pulls instance ids from a device work queue (one atomic counter)
// until the queue is empty, and solves its instance alone: Lanczos with full
// reorthogonalisation (classical Gram-Schmidt twice), all arithmetic in f64,
// the working vector in shared memory and the Krylov basis in a per-instance
// slice of global memory (L2-resident for these sizes).  Convergence is tested
// every check_every steps with the CTA-level tridiagonal eigen-solve; an
// instance ends early on convergence or on an invariant subspace.  Instances
// of different dimension share the launch, which is what the reference does
// as a sequential loop of eigsh calls (one per instance).
#include "internal.cuh"
#include "tridiag.cuh"

namespace {

constexpr int kThreads = edg::kTriThreads;  // 256
constexpr int kWarps = kThreads / 32;
constexpr int kMaxDimSmem = 4096;           // shared working vector limit

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// h[i] = <V_i, w> for i in [0, m): warp w handles i = w, w + kWarps, ...
__device__ void all_dots(const double* __restrict__ V, int n, int m, const double* __restrict__ w,
                         double* __restrict__ h) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = warp; i < m; i += kWarps) {
    const double* Vi = V + (int64_t)i * n;
    double a = 0.0;
    for (int r = lane; r < n; r += 32) a = fma(Vi[r], w[r], a);
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) h[i] = a;
  }
}

__device__ double cta_norm2(const double* __restrict__ w, int n, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double a = 0.0;
  for (int r = threadIdx.x; r < n; r += kThreads) a = fma(w[r], w[r], a);
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (lane == 0) red[warp] = a;
  __syncthreads();
  double t = 0.0;
  for (int k = 0; k < kWarps; ++k) t += red[k];
  __syncthreads();
  return t;
}

__global__ void __launch_bounds__(kThreads) batched_lanczos_k(edg_small_batch b, int* __restrict__ queue) {
  extern __shared__ double sm[];  // w [max_dim] | h [max_iter+1] | alpha | beta [max_iter+2]
  __shared__ double red[kWarps];
  __shared__ int inst_s;
  __shared__ int stop_s, m_s;
  double* w = sm;
  double* h = w + b.max_dim;
  double* alpha = h + (b.max_iter + 1);
  double* beta = alpha + (b.max_iter + 1);
  while (true) {
    if (threadIdx.x == 0) inst_s = atomicAdd(queue, 1);
    __syncthreads();
    const int inst = inst_s;
    __syncthreads();
    if (inst >= b.n_inst) break;
    const int n = (int)b.dims[inst];
    const int64_t* rp = b.rowptr + b.rowptr_off[inst];
    const int64_t r_off = b.row_off[inst];
    const double* diag = b.diag + r_off;
    double* V = b.work + b.work_off[inst];           // [max_iter+1][n]
    double* tw = V + (int64_t)(b.max_iter + 1) * n;  // tridiagonal scratch 6*(max_iter+1)
    double* S = tw + 6 * (int64_t)(b.max_iter + 1); // [k][max_iter+1] eigenvectors of T
    const int m_cap = n < b.max_iter ? n : b.max_iter;
    const int k = b.k < n ? b.k : n;
    // start vector: deterministic uniform(-1, 1), normalised
    for (int r = threadIdx.x; r < n; r += kThreads)
      w[r] = ((double)(mix64(b.seed ^ mix64(((uint64_t)inst << 32) | (uint64_t)r)) >> 11) *
              (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
    __syncthreads();
    double nrm = sqrt(cta_norm2(w, n, red));
    for (int r = threadIdx.x; r < n; r += kThreads) V[r] = w[r] / nrm;
    if (threadIdx.x == 0) {
      stop_s = 0;
      m_s = m_cap;
    }
    __syncthreads();
    double scale = 0.0;
    for (int j = 0; j < m_cap; ++j) {
      const double* vj = V + (int64_t)j * n;
      // w = H v_j
      for (int r = threadIdx.x; r < n; r += kThreads) {
        double a = diag[r] * vj[r];
        for (int64_t p = rp[r]; p < rp[r + 1]; ++p) a = fma(b.vals[p], vj[b.cols[p]], a);
        w[r] = a;
      }
      __syncthreads();
      double alpha_j = 0.0;
      for (int pass = 0; pass < 2; ++pass) {
        all_dots(V, n, j + 1, w, h);
        __syncthreads();
        alpha_j += h[j];
        for (int r = threadIdx.x; r < n; r += kThreads) {
          double s = 0.0;
          for (int i = 0; i <= j; ++i) s = fma(V[(int64_t)i * n + r], h[i], s);
          w[r] -= s;
        }
        __syncthreads();
      }
      const double bj = sqrt(cta_norm2(w, n, red));
      if (threadIdx.x == 0) {
        alpha[j] = alpha_j;
        beta[j + 1] = bj;
      }
      scale = fmax(scale, fabs(alpha_j) + bj);
      const bool breakdown = bj <= 1e-12 * fmax(scale, 1e-300);
      if (!breakdown && j + 1 < m_cap) {
        double* vn = V + (int64_t)(j + 1) * n;
        for (int r = threadIdx.x; r < n; r += kThreads) vn[r] = w[r] / bj;
      }
      __syncthreads();
      const int m = j + 1;
      const bool last = breakdown || m == m_cap;
      if (last || (m >= k && m % b.check_every == 0)) {
        // alpha/beta live in shared memory; the solver reads them directly
        edg::tridiag_body(alpha, beta, m, k, b.evals + (int64_t)inst * b.k, S, b.max_iter + 1, tw);
        __syncthreads();
        if (threadIdx.x == 0) {
          bool ok = true;
          for (int q = 0; q < k; ++q) {
            const double theta = b.evals[(int64_t)inst * b.k + q];
            const double res = breakdown ? 0.0 : fabs(bj * S[(int64_t)q * (b.max_iter + 1) + m - 1]);
            if (res > b.tol * fmax(1.0, fabs(theta))) ok = false;
          }
          if (ok || last) {
            stop_s = 1;
            m_s = m;
          }
          if (b.iters) b.iters[inst] = m;
        }
        __syncthreads();
        if (stop_s) break;
      }
    }
    // ground-state Ritz vector (eigenpair 0) if requested: x = V s, normalised
    if (b.evecs != nullptr) {
      const int m = m_s;
      double* x = b.evecs + r_off;
      for (int r = threadIdx.x; r < n; r += kThreads) {
        double a = 0.0;
        for (int i = 0; i < m; ++i) a = fma(V[(int64_t)i * n + r], S[i], a);
        w[r] = a;
      }
      __syncthreads();
      const double nx = sqrt(cta_norm2(w, n, red));
      for (int r = threadIdx.x; r < n; r += kThreads) x[r] = w[r] / nx;
      __syncthreads();
    }
  }
}

}  // namespace

extern "C" int64_t edg_small_batch_work_elems(int64_t dim, int32_t max_iter, int32_t k) {
  if (dim <= 0 || max_iter <= 0 || k <= 0) return -1;
  return (int64_t)(max_iter + 1) * dim + 6 * (int64_t)(max_iter + 1) + (int64_t)k * (max_iter + 1);
}

extern "C" int edg_lanczos_small_batched(const edg_small_batch* b, int32_t* queue, cudaStream_t stream) {
  EDG_REQUIRE(b != nullptr && queue != nullptr, "edg_lanczos_small_batched: null argument");
  EDG_REQUIRE(b->n_inst >= 0, "edg_lanczos_small_batched: negative instance count");
  EDG_REQUIRE(b->max_dim >= 1 && b->max_dim <= kMaxDimSmem,
              "edg_lanczos_small_batched: instance dimension must be 1..%d", kMaxDimSmem);
  EDG_REQUIRE(b->k >= 1 && b->k <= 16 && b->max_iter >= 1 && b->check_every >= 1,
              "edg_lanczos_small_batched: need 1 <= k <= 16, max_iter >= 1, check_every >= 1");
  if (b->n_inst == 0) return EDG_OK;
  const size_t smem = sizeof(double) * ((size_t)b->max_dim + 2 * (size_t)(b->max_iter + 1) + (size_t)b->max_iter + 2);
  EDG_REQUIRE(smem <= 200 * 1024, "edg_lanczos_small_batched: max_dim + max_iter too large for shared memory");
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(batched_lanczos_k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos_small_batched: smem attribute");
  }
  const int grid = b->n_inst < edg::kSmCount * 2 ? b->n_inst : edg::kSmCount * 2;
  // the queue counter must be zero when the kernel starts (stream-ordered reset)
  cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos_small_batched: queue reset");
  batched_lanczos_k<<<grid, kThreads, smem, stream>>>(*b, queue);
  EDG_CHECK_LAUNCH("edg_lanczos_small_batched");
  return EDG_OK;
}
