// Batched interleaved vectors: nvec instances stored [row][nvec], so one row
// of all instances is one contiguous 32-byte sector (8 f32) and the
// matrix-free matvec gathers every instance of a column with one load.
//
// Kernels for the Gram-Schmidt steps of a batched (thick-restart) Lanczos.
// The streaming updates own slots of 4 consecutive elements (one float4 / two
// double2), so the instance of slot element j is (4 * slot + j) % nvec; for
// nvec = 8 that is fixed by the slot parity, which the grid-stride loop keeps.
// Dots tile the basis (grid y) so that their f64 accumulators stay few.
// Dots accumulate in f64 and reduce deterministically (per-CTA partials, then
// one CTA per output in a fixed order).
#include "internal.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxM = 32;  // basis vectors per combine

template <typename T>
struct Slot;
template <>
struct Slot<float> {
  __device__ static __forceinline__ void load(const float* p, double (&v)[4]) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
  }
  __device__ static __forceinline__ void store(float* p, const double (&v)[4]) {
    *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
  }
};
template <>
struct Slot<double> {
  __device__ static __forceinline__ void load(const double* p, double (&v)[4]) {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
  }
  __device__ static __forceinline__ void store(double* p, const double (&v)[4]) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
  }
};

// Number of lane classes: slots with different instance maps (2 for nvec 8).
template <int NV>
constexpr int classes() { return NV > 4 ? NV / 4 : 1; }

// h[i * nvec + v] = sum over CTAs and over the slot entries of instance v.
template <int NV>
__global__ void __launch_bounds__(kThreads) dots_reduce_k(const double* __restrict__ partial, int nblk, int m,
                                                          double* __restrict__ h) {
  constexpr int P = classes<NV>();
  __shared__ double red[kWarps][P * 4];
  const int i = blockIdx.x;
  double a[P * 4];
#pragma unroll
  for (int q = 0; q < P * 4; ++q) a[q] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += kThreads)
#pragma unroll
    for (int q = 0; q < P * 4; ++q) a[q] += partial[((int64_t)b * m + i) * (P * 4) + q];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < P * 4; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a[q] += __shfl_xor_sync(0xffffffffu, a[q], o);
    if (lane == 0) red[warp][q] = a[q];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int v = threadIdx.x;
    double t = 0.0;
    // slot entry q = 4 c + j holds instance (4 c + j) % NV
    for (int q = 0; q < P * 4; ++q)
      if (q % NV == v)
        for (int k = 0; k < kWarps; ++k) t += red[k][q];
    h[(int64_t)i * NV + v] = t;
  }
}

// partial[block][i][class][4] over a tile of KT basis vectors [i0, i0 + KT):
// float4 / double2 slot loads (narrower loads do not keep HBM busy), f64
// accumulators; KT = 4 keeps them to 16 registers pairs, KT = 8 reads w once
// for m <= 8.
template <typename T, int NV, int KT>
__global__ void __launch_bounds__(kThreads) dots_k(const T* __restrict__ V, int64_t stride, int m,
                                                   const T* __restrict__ w, int64_t n_slots,
                                                   double* __restrict__ partial) {
  constexpr int P = classes<NV>();
  __shared__ double red[kWarps][KT][P][4];
  const int i0 = blockIdx.y * KT;
  const int ni = min(KT, m - i0);
  double acc[KT][4];
#pragma unroll
  for (int i = 0; i < KT; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x; s < n_slots; s += (int64_t)gridDim.x * kThreads) {
    double wv[4], vv[4];
    Slot<T>::load(w + 4 * s, wv);
#pragma unroll
    for (int i = 0; i < KT; ++i) {
      if (i < ni) {
        Slot<T>::load(V + (int64_t)(i0 + i) * stride + 4 * s, vv);
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(vv[j], wv[j], acc[i][j]);
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < KT; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      double a = acc[i][j];
#pragma unroll
      for (int o = 16; o >= P; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
      if (lane < P) red[warp][i][lane][j] = a;
    }
  __syncthreads();
  for (int t = threadIdx.x; t < KT * P * 4; t += kThreads) {
    const int i = t / (P * 4), c = (t / 4) % P, j = t % 4;
    double a = 0.0;
    for (int k = 0; k < kWarps; ++k) a += red[k][i][c][j];
    if (i < ni) partial[((int64_t)blockIdx.x * m + i0 + i) * (P * 4) + c * 4 + j] = a;
  }
}

template <typename T, int NV>
__global__ void __launch_bounds__(kThreads) update_k(const T* __restrict__ V, int64_t stride, int m,
                                                     const double* __restrict__ h, T* __restrict__ w,
                                                     int64_t n_slots) {
  __shared__ double hs[kMaxM * 8];
  for (int t = threadIdx.x; t < m * NV; t += kThreads) hs[t] = h[t];
  __syncthreads();
  for (int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x; s < n_slots; s += (int64_t)gridDim.x * kThreads) {
    double wv[4], vv[4];
    Slot<T>::load(w + 4 * s, wv);
    const int base = (int)((4 * s) % NV);
    for (int i = 0; i < m; ++i) {
      Slot<T>::load(V + (int64_t)i * stride + 4 * s, vv);
#pragma unroll
      for (int j = 0; j < 4; ++j) wv[j] = fma(-vv[j], hs[i * NV + (base + j) % NV], wv[j]);
    }
    Slot<T>::store(w + 4 * s, wv);
  }
}

template <typename T, int NV>
__global__ void __launch_bounds__(kThreads) scale_k(const T* __restrict__ w, const double* __restrict__ sq,
                                                    T* __restrict__ out, int64_t n_slots) {
  __shared__ double inv[8];
  if (threadIdx.x < NV) inv[threadIdx.x] = sq[threadIdx.x] > 0.0 ? 1.0 / sqrt(sq[threadIdx.x]) : 0.0;
  __syncthreads();
  for (int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x; s < n_slots; s += (int64_t)gridDim.x * kThreads) {
    double wv[4];
    Slot<T>::load(w + 4 * s, wv);
    const int base = (int)((4 * s) % NV);
#pragma unroll
    for (int j = 0; j < 4; ++j) wv[j] *= inv[(base + j) % NV];
    Slot<T>::store(out + 4 * s, wv);
  }
}

// In place per element: V_q <- sum_i V_i S[v][i][q], q < k.  Streams over
// the m inputs with the k outputs in f64 registers (KB >= k); every input of
// an element is read before any output of it is written.  The coefficient
// blocks of the instances are stored with an odd stride (m k + 1) so the
// eight instances of a warp read different shared-memory banks.
template <typename T, int NV, int KB>
__global__ void __launch_bounds__(kThreads) combine_k(T* __restrict__ V, int64_t stride, int m,
                                                      const double* __restrict__ S, int k, int64_t n_elems) {
  extern __shared__ double Ss[];  // [NV][m k + 1]
  const int sp = m * k + 1;
  for (int t = threadIdx.x; t < NV * m * k; t += kThreads) Ss[(t / (m * k)) * sp + t % (m * k)] = S[t];
  __syncthreads();
  for (int64_t e = (int64_t)blockIdx.x * kThreads + threadIdx.x; e < n_elems; e += (int64_t)gridDim.x * kThreads) {
    const double* Sv = Ss + (int)(e % NV) * sp;
    double acc[KB];
#pragma unroll
    for (int q = 0; q < KB; ++q) acc[q] = 0.0;
#pragma unroll 4
    for (int i = 0; i < m; ++i) {
      const double x = (double)V[(int64_t)i * stride + e];
#pragma unroll
      for (int q = 0; q < KB; ++q)
        if (q < k) acc[q] = fma(x, Sv[i * k + q], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < KB; ++q)
      if (q < k) V[(int64_t)q * stride + e] = (T)acc[q];
  }
}

// Dots of a tile of KT basis vectors against two vectors at once (the
// lagged candidate u and the new matvec result w of a delayed Gram-Schmidt
// step): partial[block][i][r][class][4], r = 0 for x1, 1 for x2.
template <typename T, int NV, int KT>
__global__ void __launch_bounds__(kThreads) dots2_k(const T* __restrict__ V, int64_t stride, int m,
                                                    const T* __restrict__ x1, const T* __restrict__ x2,
                                                    int64_t n_slots, double* __restrict__ partial) {
  constexpr int P = classes<NV>();
  __shared__ double red[kWarps][KT][2][P][4];
  const int i0 = blockIdx.y * KT;
  const int ni = min(KT, m - i0);
  double acc[KT][2][4];
#pragma unroll
  for (int i = 0; i < KT; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][0][j] = acc[i][1][j] = 0.0;
  for (int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x; s < n_slots; s += (int64_t)gridDim.x * kThreads) {
    double a[4], b[4], vv[4];
    Slot<T>::load(x1 + 4 * s, a);
    Slot<T>::load(x2 + 4 * s, b);
#pragma unroll
    for (int i = 0; i < KT; ++i) {
      if (i < ni) {
        Slot<T>::load(V + (int64_t)(i0 + i) * stride + 4 * s, vv);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][0][j] = fma(vv[j], a[j], acc[i][0][j]);
          acc[i][1][j] = fma(vv[j], b[j], acc[i][1][j]);
        }
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < KT; ++i)
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        double x = acc[i][r][j];
#pragma unroll
        for (int o = 16; o >= P; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane < P) red[warp][i][r][lane][j] = x;
      }
  __syncthreads();
  for (int t = threadIdx.x; t < KT * 2 * P * 4; t += kThreads) {
    const int i = t / (2 * P * 4), r = (t / (P * 4)) % 2, q = t % (P * 4);
    double x = 0.0;
    for (int k = 0; k < kWarps; ++k) x += red[k][i][r][q / 4][q % 4];
    if (i < ni) partial[(((int64_t)blockIdx.x * m + i0 + i) * 2 + r) * (P * 4) + q] = x;
  }
}

// h_r[i * NV + v] from the dots2_k partials; one CTA per (i, r).
template <int NV>
__global__ void __launch_bounds__(kThreads) dots2_reduce_k(const double* __restrict__ partial, int nblk, int m,
                                                           double* __restrict__ h1, double* __restrict__ h2) {
  constexpr int P = classes<NV>();
  __shared__ double red[kWarps][P * 4];
  const int i = blockIdx.x / 2, r = blockIdx.x % 2;
  double a[P * 4];
#pragma unroll
  for (int q = 0; q < P * 4; ++q) a[q] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += kThreads)
#pragma unroll
    for (int q = 0; q < P * 4; ++q) a[q] += partial[(((int64_t)b * m + i) * 2 + r) * (P * 4) + q];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < P * 4; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a[q] += __shfl_xor_sync(0xffffffffu, a[q], o);
    if (lane == 0) red[warp][q] = a[q];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int v = threadIdx.x;
    double t = 0.0;
    for (int q = 0; q < P * 4; ++q)
      if (q % NV == v)
        for (int k = 0; k < kWarps; ++k) t += red[k][q];
    (r == 0 ? h1 : h2)[(int64_t)i * NV + v] = t;
  }
}

// One delayed classical Gram-Schmidt step in one pass over V_0..V_{j-1}.
// With s = hu[0..j), alpha = hu[j] (= u.u), z = hw[0..j), omega = hw[j]
// (= u.w), u = V_j:  r = sqrt(alpha - s.s), q = (u - sum_i V_i s_i) / r is
// written to V_j (u's lagged second pass), c = (omega - s.z) / r, and
// w <- w - sum_i V_i z_i - q c (one pass of w against V_0..V_j), with the
// squared norm of the stored w per CTA and slot class (reduced by
// dots_reduce_k).
template <typename T, int NV>
__global__ void __launch_bounds__(kThreads) dcgs_update_k(T* __restrict__ V, int64_t stride, int j,
                                                          const double* __restrict__ hu,
                                                          const double* __restrict__ hw, T* __restrict__ w,
                                                          int64_t n_slots, double* __restrict__ partial) {
  constexpr int P = classes<NV>();
  __shared__ double ss[kMaxM * 8], zs[kMaxM * 8];
  __shared__ double rinv[8], cq[8];
  __shared__ double red[kWarps][P][4];
  for (int t = threadIdx.x; t < j * NV; t += kThreads) {
    ss[t] = hu[t];
    zs[t] = hw[t];
  }
  if (threadIdx.x < NV) {
    const int v = threadIdx.x;
    double s2 = 0.0, sz = 0.0;
    for (int i = 0; i < j; ++i) {
      s2 = fma(hu[i * NV + v], hu[i * NV + v], s2);
      sz = fma(hu[i * NV + v], hw[i * NV + v], sz);
    }
    const double r2 = hu[j * NV + v] - s2;
    const double ri = r2 > 0.0 ? 1.0 / sqrt(r2) : 0.0;
    rinv[v] = ri;
    cq[v] = (hw[j * NV + v] - sz) * ri;
  }
  __syncthreads();
  T* U = V + (int64_t)j * stride;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x; s < n_slots; s += (int64_t)gridDim.x * kThreads) {
    double uv[4], wv[4], vv[4];
    Slot<T>::load(U + 4 * s, uv);
    Slot<T>::load(w + 4 * s, wv);
    const int base = (int)((4 * s) % NV);
    for (int i = 0; i < j; ++i) {
      Slot<T>::load(V + (int64_t)i * stride + 4 * s, vv);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int v = (base + k) % NV;
        uv[k] = fma(-vv[k], ss[i * NV + v], uv[k]);
        wv[k] = fma(-vv[k], zs[i * NV + v], wv[k]);
      }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int v = (base + k) % NV;
      uv[k] = (double)(T)(uv[k] * rinv[v]);
      wv[k] = (double)(T)fma(-uv[k], cq[v], wv[k]);
      acc[k] = fma(wv[k], wv[k], acc[k]);
    }
    Slot<T>::store(U + 4 * s, uv);
    Slot<T>::store(w + 4 * s, wv);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double a = acc[k];
#pragma unroll
    for (int o = 16; o >= P; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane < P) red[warp][lane][k] = a;
  }
  __syncthreads();
  if (threadIdx.x < P * 4) {
    const int c = threadIdx.x / 4, k = threadIdx.x % 4;
    double a = 0.0;
    for (int q = 0; q < kWarps; ++q) a += red[q][c][k];
    partial[(int64_t)blockIdx.x * (P * 4) + threadIdx.x] = a;
  }
}

// Second Gram-Schmidt pass fused with the norm (update_k's slot layout):
// w <- w - sum_{i<m} V_i h[i][v], and per CTA the squared norms of the
// stored (rounded) w by slot class, partial[blk][class * 4 + j], reduced by
// dots_reduce_k like a one-vector dot.
template <typename T, int NV>
__global__ void __launch_bounds__(kThreads) update_norm_k(const T* __restrict__ V, int64_t stride, int m,
                                                          const double* __restrict__ h, T* __restrict__ w,
                                                          int64_t n_slots, double* __restrict__ partial) {
  constexpr int P = classes<NV>();
  __shared__ double hs[kMaxM * 8];
  __shared__ double red[kWarps][P][4];
  for (int t = threadIdx.x; t < m * NV; t += kThreads) hs[t] = h[t];
  __syncthreads();
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t s = (int64_t)blockIdx.x * kThreads + threadIdx.x; s < n_slots; s += (int64_t)gridDim.x * kThreads) {
    double wv[4], vv[4];
    Slot<T>::load(w + 4 * s, wv);
    const int base = (int)((4 * s) % NV);
    for (int i = 0; i < m; ++i) {
      Slot<T>::load(V + (int64_t)i * stride + 4 * s, vv);
#pragma unroll
      for (int j = 0; j < 4; ++j) wv[j] = fma(-vv[j], hs[i * NV + (base + j) % NV], wv[j]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      wv[j] = (double)(T)wv[j];
      acc[j] = fma(wv[j], wv[j], acc[j]);
    }
    Slot<T>::store(w + 4 * s, wv);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double a = acc[j];
#pragma unroll
    for (int o = 16; o >= P; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane < P) red[warp][lane][j] = a;
  }
  __syncthreads();
  if (threadIdx.x < P * 4) {
    const int c = threadIdx.x / 4, j = threadIdx.x % 4;
    double a = 0.0;
    for (int k = 0; k < kWarps; ++k) a += red[k][c][j];
    partial[(int64_t)blockIdx.x * (P * 4) + threadIdx.x] = a;
  }
}

// out[o * NV + v] = sum over blocks of partial[blk][o][v]; one CTA per o.
template <int NV>
__global__ void __launch_bounds__(kThreads) reduce_nv_k(const double* __restrict__ partial, int nblk, int n_out,
                                                        double* __restrict__ out) {
  __shared__ double red[kWarps][NV];
  const int o = blockIdx.x;
  double a[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) a[v] = 0.0;
  for (int b = threadIdx.x; b < nblk; b += kThreads)
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] += partial[((int64_t)b * n_out + o) * NV + v];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a[v] += __shfl_xor_sync(0xffffffffu, a[v], off);
    if (lane == 0) red[warp][v] = a[v];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double t = 0.0;
    for (int k = 0; k < kWarps; ++k) t += red[k][threadIdx.x];
    out[(int64_t)o * NV + threadIdx.x] = t;
  }
}

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

template <typename T>
__global__ void random_k(T* __restrict__ x, int64_t n_valid, int64_t n_elems, uint64_t seed) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_elems; e += (int64_t)gridDim.x * blockDim.x) {
    const double u = (double)(mix64(seed ^ mix64((uint64_t)e)) >> 11) * (1.0 / 9007199254740992.0);
    x[e] = e < n_valid ? (T)(2.0 * u - 1.0) : (T)0;
  }
}

int check_common(int dtype, int64_t n_elems, int nvec, const char* where) {
  EDG_REQUIRE(dtype == 0 || dtype == 1, "%s: dtype must be 0 (f64) or 1 (f32)", where);
  EDG_REQUIRE(nvec == 1 || nvec == 2 || nvec == 4 || nvec == 8, "%s: nvec must be 1, 2, 4 or 8", where);
  EDG_REQUIRE(n_elems >= 0 && n_elems % 4 == 0 && n_elems % nvec == 0,
              "%s: n_elems must be a multiple of 4 and of nvec", where);
  return EDG_OK;
}

template <typename T, int NV, int KT>
int run_dots_kt(int64_t n_elems, const void* V, int64_t stride, int m, const void* w, double* h, double* scratch,
                cudaStream_t stream) {
  const int64_t n_slots = n_elems / 4;
  const int tiles = (m + KT - 1) / KT;
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dots_k<T, NV, KT>, kThreads, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  int64_t nbx = edg::ceil_div(n_slots, kThreads);
  const int64_t cap = (int64_t)edg::kSmCount * (per_sm < 8 ? per_sm : 8);
  const int64_t cap_t = cap / tiles > edg::kSmCount ? cap / tiles : edg::kSmCount;
  if (nbx > cap_t) nbx = cap_t;
  if (nbx < 1) nbx = 1;
  dots_k<T, NV, KT><<<dim3((unsigned)nbx, tiles), kThreads, 0, stream>>>((const T*)V, stride, m, (const T*)w,
                                                                        n_slots, scratch);
  dots_reduce_k<NV><<<m, kThreads, 0, stream>>>(scratch, (int)nbx, m, h);
  return EDG_OK;
}

template <typename T, int NV>
int run_dots(int64_t n_elems, const void* V, int64_t stride, int m, const void* w, double* h, double* scratch,
             cudaStream_t stream) {
  if (m <= 8) return run_dots_kt<T, NV, 8>(n_elems, V, stride, m, w, h, scratch, stream);
  return run_dots_kt<T, NV, 4>(n_elems, V, stride, m, w, h, scratch, stream);
}

template <typename T, int NV, int KT>
int run_dots2(int64_t n_elems, const void* V, int64_t stride, int m, const void* x1, const void* x2, double* h1,
              double* h2, double* scratch, cudaStream_t stream) {
  const int64_t n_slots = n_elems / 4;
  const int tiles = (m + KT - 1) / KT;
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dots2_k<T, NV, KT>, kThreads, 0) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  int64_t nbx = edg::ceil_div(n_slots, kThreads);
  const int64_t cap = (int64_t)edg::kSmCount * (per_sm < 8 ? per_sm : 8);
  const int64_t cap_t = cap / tiles > edg::kSmCount ? cap / tiles : edg::kSmCount;
  if (nbx > cap_t) nbx = cap_t;
  if (nbx < 1) nbx = 1;
  dots2_k<T, NV, KT><<<dim3((unsigned)nbx, tiles), kThreads, 0, stream>>>((const T*)V, stride, m, (const T*)x1,
                                                                         (const T*)x2, n_slots, scratch);
  dots2_reduce_k<NV><<<2 * m, kThreads, 0, stream>>>(scratch, (int)nbx, m, h1, h2);
  return EDG_OK;
}

template <typename T, int NV>
int run_dcgs(int64_t n_elems, void* V, int64_t stride, int j, const double* hu, const double* hw, void* w,
             double* sq, double* scratch, cudaStream_t stream) {
  const int64_t n_slots = n_elems / 4;
  const unsigned nblk = edg::grid_for(n_slots, kThreads, 8);
  dcgs_update_k<T, NV><<<nblk, kThreads, 0, stream>>>((T*)V, stride, j, hu, hw, (T*)w, n_slots, scratch);
  dots_reduce_k<NV><<<1, kThreads, 0, stream>>>(scratch, (int)nblk, 1, sq);
  return EDG_OK;
}

template <typename T, int NV>
int run_norm(int64_t n_elems, const void* V, int64_t stride, int m, const double* h, void* w, double* out,
             double* scratch, cudaStream_t stream) {
  const int64_t n_slots = n_elems / 4;
  const unsigned nblk = edg::grid_for(n_slots, kThreads, 8);
  update_norm_k<T, NV><<<nblk, kThreads, 0, stream>>>((const T*)V, stride, m, h, (T*)w, n_slots, scratch);
  dots_reduce_k<NV><<<1, kThreads, 0, stream>>>(scratch, (int)nblk, 1, out);
  return EDG_OK;
}

template <typename T, int NV>
int run_combine(int64_t n_elems, void* V, int64_t stride, int m, const double* S, int k, size_t smem,
                cudaStream_t stream) {
  const unsigned grid = edg::grid_for(n_elems, kThreads, 8);
  if (k <= 4)
    combine_k<T, NV, 4><<<grid, kThreads, smem, stream>>>((T*)V, stride, m, S, k, n_elems);
  else if (k <= 8)
    combine_k<T, NV, 8><<<grid, kThreads, smem, stream>>>((T*)V, stride, m, S, k, n_elems);
  else if (k <= 16)
    combine_k<T, NV, 16><<<grid, kThreads, smem, stream>>>((T*)V, stride, m, S, k, n_elems);
  else
    combine_k<T, NV, 32><<<grid, kThreads, smem, stream>>>((T*)V, stride, m, S, k, n_elems);
  return EDG_OK;
}

}  // namespace

extern "C" int64_t edg_iv_scratch_elems(int64_t n_elems, int32_t m) {
  if (n_elems < 0 || m < 1) return -1;
  return (int64_t)edg::kSmCount * 8 * m * 2 * 8;  // blocks * m * 2 right-hand sides * (P * 4 <= 8)
}

#define EDG_IV_DISPATCH(CALL)                                \
  switch (nvec) {                                            \
    case 1: st = dtype ? CALL(float, 1) : CALL(double, 1); break; \
    case 2: st = dtype ? CALL(float, 2) : CALL(double, 2); break; \
    case 4: st = dtype ? CALL(float, 4) : CALL(double, 4); break; \
    default: st = dtype ? CALL(float, 8) : CALL(double, 8); break; \
  }

extern "C" int edg_iv_dots(int32_t dtype, int64_t n_elems, int32_t nvec, const void* V, int64_t stride, int32_t m,
                           const void* w, double* h, double* scratch, cudaStream_t stream) {
  int st = check_common(dtype, n_elems, nvec, "edg_iv_dots");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(m >= 1 && V != nullptr && w != nullptr && h != nullptr && scratch != nullptr,
              "edg_iv_dots: need m >= 1 and non-null buffers");
  EDG_REQUIRE(stride % 4 == 0, "edg_iv_dots: stride must be a multiple of 4");
  if (n_elems == 0) {
    cudaError_t e = cudaMemsetAsync(h, 0, sizeof(double) * (size_t)m * nvec, stream);
    return e == cudaSuccess ? EDG_OK : edg::cuda_status(e, "edg_iv_dots");
  }
#define CALL(T, NV) run_dots<T, NV>(n_elems, V, stride, m, w, h, scratch, stream)
  EDG_IV_DISPATCH(CALL)
#undef CALL
  if (st != EDG_OK) return st;
  EDG_CHECK_LAUNCH("edg_iv_dots");
  return EDG_OK;
}

extern "C" int edg_iv_update(int32_t dtype, int64_t n_elems, int32_t nvec, const void* V, int64_t stride, int32_t m,
                             const double* h, void* w, cudaStream_t stream) {
  int st = check_common(dtype, n_elems, nvec, "edg_iv_update");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(m >= 1 && m <= kMaxM && V != nullptr && w != nullptr && h != nullptr,
              "edg_iv_update: need 1 <= m <= %d and non-null buffers", kMaxM);
  EDG_REQUIRE(stride % 4 == 0, "edg_iv_update: stride must be a multiple of 4");
  if (n_elems == 0) return EDG_OK;
  const int64_t n_slots = n_elems / 4;
  const unsigned grid = edg::grid_for(n_slots, kThreads, 8);
#define CALL(T, NV) (update_k<T, NV><<<grid, kThreads, 0, stream>>>((const T*)V, stride, m, h, (T*)w, n_slots), EDG_OK)
  EDG_IV_DISPATCH(CALL)
#undef CALL
  EDG_CHECK_LAUNCH("edg_iv_update");
  return st;
}

extern "C" int edg_iv_scale(int32_t dtype, int64_t n_elems, int32_t nvec, const void* w, const double* sq, void* out,
                            cudaStream_t stream) {
  int st = check_common(dtype, n_elems, nvec, "edg_iv_scale");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(w != nullptr && sq != nullptr && out != nullptr, "edg_iv_scale: null argument");
  if (n_elems == 0) return EDG_OK;
  const int64_t n_slots = n_elems / 4;
  const unsigned grid = edg::grid_for(n_slots, kThreads, 8);
#define CALL(T, NV) (scale_k<T, NV><<<grid, kThreads, 0, stream>>>((const T*)w, sq, (T*)out, n_slots), EDG_OK)
  EDG_IV_DISPATCH(CALL)
#undef CALL
  EDG_CHECK_LAUNCH("edg_iv_scale");
  return st;
}

extern "C" int edg_iv_combine(int32_t dtype, int64_t n_elems, int32_t nvec, void* V, int64_t stride, int32_t m,
                              const double* S, int32_t k, cudaStream_t stream) {
  int st = check_common(dtype, n_elems, nvec, "edg_iv_combine");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(m >= 1 && m <= kMaxM && k >= 1 && k <= m, "edg_iv_combine: need 1 <= k <= m <= %d", kMaxM);
  EDG_REQUIRE(V != nullptr && S != nullptr, "edg_iv_combine: null argument");
  if (n_elems == 0) return EDG_OK;
  const size_t smem = sizeof(double) * ((size_t)nvec * (m * k + 1));
  EDG_REQUIRE(smem <= 48 * 1024, "edg_iv_combine: nvec * m * k too large for shared memory");
#define CALL(T, NV) run_combine<T, NV>(n_elems, V, stride, m, S, k, smem, stream)
  EDG_IV_DISPATCH(CALL)
#undef CALL
  EDG_CHECK_LAUNCH("edg_iv_combine");
  return st;
}

extern "C" int edg_iv_random(int32_t dtype, int64_t n_rows, int64_t n_elems, int32_t nvec, uint64_t seed, void* x,
                             cudaStream_t stream) {
  int st = check_common(dtype, n_elems, nvec, "edg_iv_random");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(x != nullptr && n_rows >= 0 && n_rows * nvec <= n_elems, "edg_iv_random: bad sizes");
  if (n_elems == 0) return EDG_OK;
  const unsigned grid = edg::grid_for(n_elems, kThreads, 8);
  if (dtype == 0)
    random_k<double><<<grid, kThreads, 0, stream>>>((double*)x, n_rows * nvec, n_elems, seed);
  else
    random_k<float><<<grid, kThreads, 0, stream>>>((float*)x, n_rows * nvec, n_elems, seed);
  EDG_CHECK_LAUNCH("edg_iv_random");
  return EDG_OK;
}

extern "C" int edg_iv_update_norm(int32_t dtype, int64_t n_elems, int32_t nvec, const void* V, int64_t stride,
                                  int32_t m, const double* h, void* w, double* sq, double* scratch,
                                  cudaStream_t stream) {
  int st = check_common(dtype, n_elems, nvec, "edg_iv_update_norm");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(m >= 1 && m <= kMaxM && V != nullptr && h != nullptr && w != nullptr && sq != nullptr &&
                  scratch != nullptr,
              "edg_iv_update_norm: need 1 <= m <= %d and non-null buffers", kMaxM);
  if (n_elems == 0) {
    cudaError_t e = cudaMemsetAsync(sq, 0, sizeof(double) * (size_t)nvec, stream);
    return e == cudaSuccess ? EDG_OK : edg::cuda_status(e, "edg_iv_update_norm");
  }
#define CALL(T, NV) run_norm<T, NV>(n_elems, V, stride, m, h, w, sq, scratch, stream)
  EDG_IV_DISPATCH(CALL)
#undef CALL
  if (st != EDG_OK) return st;
  EDG_CHECK_LAUNCH("edg_iv_update_norm");
  return EDG_OK;
}

extern "C" int edg_iv_dots2(int32_t dtype, int64_t n_elems, int32_t nvec, const void* V, int64_t stride, int32_t m,
                            const void* x1, const void* x2, double* h1, double* h2, double* scratch,
                            cudaStream_t stream) {
  int st = check_common(dtype, n_elems, nvec, "edg_iv_dots2");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(m >= 1 && V != nullptr && x1 != nullptr && x2 != nullptr && h1 != nullptr && h2 != nullptr &&
                  scratch != nullptr,
              "edg_iv_dots2: need m >= 1 and non-null buffers");
  EDG_REQUIRE(stride % 4 == 0, "edg_iv_dots2: stride must be a multiple of 4");
  if (n_elems == 0) {
    cudaError_t e = cudaMemsetAsync(h1, 0, sizeof(double) * (size_t)m * nvec, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(h2, 0, sizeof(double) * (size_t)m * nvec, stream);
    return e == cudaSuccess ? EDG_OK : edg::cuda_status(e, "edg_iv_dots2");
  }
#define CALL(T, NV) run_dots2<T, NV, 4>(n_elems, V, stride, m, x1, x2, h1, h2, scratch, stream)
  EDG_IV_DISPATCH(CALL)
#undef CALL
  if (st != EDG_OK) return st;
  EDG_CHECK_LAUNCH("edg_iv_dots2");
  return EDG_OK;
}

extern "C" int edg_iv_dcgs_update(int32_t dtype, int64_t n_elems, int32_t nvec, void* V, int64_t stride, int32_t j,
                                  const double* hu, const double* hw, void* w, double* sq, double* scratch,
                                  cudaStream_t stream) {
  int st = check_common(dtype, n_elems, nvec, "edg_iv_dcgs_update");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(j >= 0 && j < kMaxM && V != nullptr && hu != nullptr && hw != nullptr && w != nullptr &&
                  sq != nullptr && scratch != nullptr,
              "edg_iv_dcgs_update: need 0 <= j < %d and non-null buffers", kMaxM);
  EDG_REQUIRE(stride % 4 == 0, "edg_iv_dcgs_update: stride must be a multiple of 4");
  if (n_elems == 0) {
    cudaError_t e = cudaMemsetAsync(sq, 0, sizeof(double) * (size_t)nvec, stream);
    return e == cudaSuccess ? EDG_OK : edg::cuda_status(e, "edg_iv_dcgs_update");
  }
#define CALL(T, NV) run_dcgs<T, NV>(n_elems, V, stride, j, hu, hw, w, sq, scratch, stream)
  EDG_IV_DISPATCH(CALL)
#undef CALL
  if (st != EDG_OK) return st;
  EDG_CHECK_LAUNCH("edg_iv_dcgs_update");
  return EDG_OK;
}
