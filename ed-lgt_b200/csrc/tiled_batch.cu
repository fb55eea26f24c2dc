// Batched Lanczos over an (instance, row-tile) work queue, in one persistent
// cooperative launch per solve.
//
// Many sector Hamiltonians of uneven dimension (charge sectors, coupling
// sweeps, lattice sizes) are solved together: each instance is cut into
// tiles of tile_rows rows, and every phase of a Lanczos step walks the list of
// (instance, tile) items with a grid-stride loop, so an instance of any size
// is spread over many CTAs while small instances share the grid.  The
// replaced reference path is the sequential loop of eigsh calls
// (edlgt/modeling/qmb_hamiltonian.py:260-332), one per instance.
//
// Step j of every active instance (delayed classical Gram-Schmidt with
// reorthogonalisation, DCGS2, as in lanczos.cu; Swirydowicz et al., Numer.
// Linear Algebra Appl. 28 (2021) e2343), phases separated by grid barriers:
//   M  V[j] = T(w_prev / |w_prev|) on the item's rows; w = H V[j]
//      (the gathered x entries are rounded to T exactly as V[j] is stored)
//   D  per-tile partial dots of V[0..j] with u = V[j] and with w
//   R  per (instance, i): sum of the tile partials; the last CTA of the
//      instance (ticket counter) forms r, c, alpha_j, beta_j
//   U  V[j] <- (u - V s) / r ; w <- w - V z - V[j] c ; tile partials of |w|^2,
//      the last CTA forms |w| and beta_{j+1}
//   C  (steps marked in check_at) one CTA per instance: tridiagonal
//      eigen-solve, residual bounds, invariant-subspace test; converged
//      instances leave the queue
// The working vector is double-buffered (M of step j reads the buffer U of
// step j-1 finished while writing the other), so normalisation needs no phase
// of its own.  T = float keeps the Krylov basis and the matvec operands in
// f32 while w, every inner product, the recurrence and the eigen-solve stay
// f64; T = double is the plain f64 solver.
//
// Grid barriers wait with a time limit (2 s on the global timer); a wait that
// runs out writes EDG_ERR_TIMEOUT to the status word and every CTA returns.
// Data written by other CTAs during the launch is read with ld.global.cg
// (L2, coherent) and never through the read-only path.
#include "internal.cuh"
#include "tridiag.cuh"

#include <algorithm>
#include <vector>

namespace {

constexpr int kThreads = edg::kTriThreads;  // 256 (the tridiagonal solver's CTA size)
constexpr int kWarps = kThreads / 32;
constexpr int kChunk = 8;     // Krylov vectors per dot chunk
constexpr int kMaxK = 8;      // eigenpairs per instance
constexpr int kMaxIter = 2000;

// instance table fields (int64 each)
enum { F_DIM = 0, F_ROW_OFF, F_ROWPTR_OFF, F_V_OFF, F_F_OFF, F_TILES, F_ITEM0, F_MCAP, F_N };

// per-instance int32 state
enum { S_ACTIVE = 0, S_TICK_R, S_TICK_U, S_TICK_N, S_N };

// workspace header (int32 words)
enum { H_BAR_COUNT = 0, H_BAR_GEN, H_STATUS, H_ACTIVE, H_WORDS = 64 };

inline int64_t al256(int64_t x) { return (x + 255) & ~int64_t(255); }

// f64 block of an instance (offsets in doubles, relative to its F_F_OFF)
struct FLayout {
  int64_t w0, w1, part, hu, hw, alpha, beta, misc, tri, S, total;
};
__host__ __device__ inline FLayout f_layout(int64_t dim_pad, int64_t tiles, int64_t m_cap, int k) {
  FLayout f{};
  const int64_t ld = m_cap + 1;
  int64_t o = 0;
  f.w0 = o; o += dim_pad;
  f.w1 = o; o += dim_pad;
  f.part = o; o += tiles * ld * 2;
  f.hu = o; o += ld;
  f.hw = o; o += ld;
  f.alpha = o; o += ld;
  f.beta = o; o += ld + 1;
  f.misc = o; o += 8 + 2 * kMaxK;  // rc[2], inv, wnorm, ... | resid[kMaxK] | evals[kMaxK]
  f.tri = o; o += 6 * ld;
  f.S = o; o += (int64_t)k * ld;
  f.total = (o + 31) & ~int64_t(31);
  return f;
}
enum { M_RI = 0, M_C, M_INV, M_WNORM };

struct Params {
  int n_inst, n_items, tile_rows, k, max_iter;
  double tol;
  uint64_t seed;
  const int64_t* inst;
  const int32_t* item_inst;
  const uint8_t* check_at;
  const int64_t* rowptr;
  const int32_t* cols;
  const void* vals;
  const void* diag;
  const double* v0;
  char* ws;  // header | int state | f64 arena | V arena (offsets in the instance table)
  double* evals;
  double* resid;
  int32_t* iters;
  double* evecs;
  int32_t* status;
};

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid-wide barrier with a 2 s limit; returns false (all threads) when the
// launch must stop (a wait ran out here or in another CTA).
__device__ bool grid_barrier(int* hdr) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned* count = reinterpret_cast<unsigned*>(hdr + H_BAR_COUNT);
    unsigned* gen = reinterpret_cast<unsigned*>(hdr + H_BAR_GEN);
    const unsigned g = ld_acquire(gen);
    __threadfence();
    const unsigned arrived = atomicAdd(count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      const uint64_t t0 = global_ns();
      unsigned spins = 0;
      while (ld_acquire(gen) == g) {
        __nanosleep(64);
        if ((++spins & 1023u) == 0 && global_ns() - t0 > 2000000000ull) {
          atomicExch(hdr + H_STATUS, EDG_ERR_TIMEOUT);
          break;
        }
      }
    }
    __threadfence();
    ok_s = atomicAdd(hdr + H_STATUS, 0) == 0;
  }
  __syncthreads();
  return ok_s != 0;
}

template <int NV>
__device__ __forceinline__ void block_sum(double* v, double* red /*[kWarps][NV]*/) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double a = v[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if (lane == 0) red[warp * NV + q] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double a = 0.0;
      for (int w = 0; w < kWarps; ++w) a += red[w * NV + q];
      v[q] = a;
    }
  }
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ T round_to(double x) { return (T)x; }

template <typename T>
__device__ __forceinline__ double ldv(const T* p) { return (double)__ldcg(p); }

__device__ __forceinline__ void ld4(const float* p, double* o) {
  const float4 v = __ldcg(reinterpret_cast<const float4*>(p));
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void ld4(const double* p, double* o) {
  const double2 a = __ldcg(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcg(reinterpret_cast<const double2*>(p) + 1);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const double* v) {
  *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
__device__ __forceinline__ void st4(double* p, const double* v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
  reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
}

struct InstView {
  int64_t dim, dim_pad, row_off, rowptr_off, tiles, item0, m_cap;
  double* f;     // f64 block
  FLayout L;
  int* st;       // int32 state
};

template <typename T>
__device__ __forceinline__ InstView inst_view(const Params& p, int i, T** V) {
  InstView v;
  const int64_t* r = p.inst + (int64_t)i * F_N;
  v.dim = r[F_DIM];
  v.dim_pad = (v.dim + 3) & ~int64_t(3);
  v.row_off = r[F_ROW_OFF];
  v.rowptr_off = r[F_ROWPTR_OFF];
  v.tiles = r[F_TILES];
  v.item0 = r[F_ITEM0];
  v.m_cap = r[F_MCAP];
  v.f = reinterpret_cast<double*>(p.ws + r[F_F_OFF]);
  v.L = f_layout(v.dim_pad, v.tiles, v.m_cap, p.k);
  v.st = reinterpret_cast<int*>(p.ws) + H_WORDS + (int64_t)i * S_N;
  *V = reinterpret_cast<T*>(p.ws + r[F_V_OFF]);
  return v;
}

// Last-of-count ticket: true in the CTA whose arrival completes the count
// (the counter is reset by it).  Writers fence before arriving.
__device__ __forceinline__ bool last_arrival(int* tick, int count) {
  __shared__ int last_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last_s = atomicAdd(tick, 1) == count - 1;
    if (last_s) {
      atomicExch(tick, 0);
      __threadfence();
    }
  }
  __syncthreads();
  return last_s != 0;
}

template <typename T, int G>
__global__ void __launch_bounds__(kThreads) tiled_lanczos_k(Params p) {
  __shared__ double red[kWarps * kChunk * 2];
  __shared__ double sz[2 * (kMaxIter + 1)];
  int* hdr = reinterpret_cast<int*>(p.ws);
  const int TR = p.tile_rows;
  const T* vals = reinterpret_cast<const T*>(p.vals);
  const T* diag = reinterpret_cast<const T*>(p.diag);
  if (blockIdx.x == 0 && threadIdx.x == 0) hdr[H_ACTIVE] = p.n_inst;

  // ---------------- start: w_prev (buffer 1) = v0 or uniform(-1, 1) -------
  for (int item = blockIdx.x; item < p.n_items; item += gridDim.x) {
    const int ii = p.item_inst[item];
    T* V;
    InstView I = inst_view<T>(p, ii, &V);
    const int64_t t = item - I.item0;
    const int64_t r0 = t * TR, r1 = min(I.dim_pad, r0 + TR);
    double* w = I.f + I.L.w1;
    double nrm = 0.0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) {
      double x = 0.0;
      if (r < I.dim) {
        if (p.v0) {
          x = p.v0[I.row_off + r];
        } else {
          const uint64_t z = splitmix64(p.seed ^ splitmix64((uint64_t)r));
          x = ((double)(z >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
        }
      }
      w[r] = x;
      nrm = fma(x, x, nrm);
    }
    block_sum<1>(&nrm, red);
    if (threadIdx.x == 0) I.f[I.L.part + t * 2] = nrm;
    if (last_arrival(I.st + S_TICK_N, (int)I.tiles) && threadIdx.x == 0) {
      double s = 0.0;
      for (int64_t q = 0; q < I.tiles; ++q) s += __ldcg(I.f + I.L.part + q * 2);
      const double nv = sqrt(s);
      I.f[I.L.misc + M_WNORM] = nv;
      I.f[I.L.misc + M_INV] = nv > 0.0 ? 1.0 / nv : 0.0;
      I.st[S_ACTIVE] = 1;
      // outputs of an instance that never reaches a check stay NaN / 0
      p.iters[ii] = 0;
      for (int q = 0; q < p.k; ++q) {
        p.evals[(int64_t)ii * p.k + q] = NAN;
        p.resid[(int64_t)ii * p.k + q] = NAN;
      }
    }
  }
  if (!grid_barrier(hdr)) return;

  int j = 0;
  for (; j < p.max_iter; ++j) {
    // ---------------- M: V[j] from w_prev; w = H V[j] --------------------
    for (int item = blockIdx.x; item < p.n_items; item += gridDim.x) {
      const int ii = p.item_inst[item];
      T* V;
      InstView I = inst_view<T>(p, ii, &V);
      if (__ldcg(I.st + S_ACTIVE) == 0 || j >= I.m_cap) continue;
      const int64_t t = item - I.item0;
      const int64_t r0 = t * TR, r1 = min(I.dim, r0 + TR), r1p = min(I.dim_pad, r0 + TR);
      const double* wp = I.f + ((j & 1) ? I.L.w0 : I.L.w1);
      double* wc = I.f + ((j & 1) ? I.L.w1 : I.L.w0);
      const double inv = __ldcg(I.f + I.L.misc + M_INV);
      T* Vj = V + (int64_t)j * I.dim_pad;
      for (int64_t r = r0 + threadIdx.x; r < r1p; r += kThreads) Vj[r] = round_to<T>(__ldcg(wp + r) * inv);
      const int64_t* rp = p.rowptr + I.rowptr_off;
      const T* dg = diag + I.row_off;
      const int lane = threadIdx.x & (G - 1);
      const int64_t grp = threadIdx.x / G;
      constexpr int kRowsPass = kThreads / G;
      const int64_t n_pass = (r1 - r0 + kRowsPass - 1) / kRowsPass;
      for (int64_t it = 0; it < n_pass; ++it) {
        const int64_t r = r0 + it * kRowsPass + grp;
        double acc = 0.0;
        if (r < r1) {
          const int64_t beg = __ldg(rp + r), end = __ldg(rp + r + 1);
          for (int64_t q = beg + lane; q < end; q += G) {
            const int64_t c = __ldg(p.cols + q);
            const double xc = (double)round_to<T>(__ldcg(wp + c) * inv);
            acc = fma((double)__ldg(vals + q), xc, acc);
          }
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, G);
        if (r < r1 && lane == 0) {
          const double xr = (double)round_to<T>(__ldcg(wp + r) * inv);
          wc[r] = fma((double)__ldg(dg + r), xr, acc);
        }
      }
      for (int64_t r = r1 + threadIdx.x; r < r1p; r += kThreads) wc[r] = 0.0;
    }
    if (!grid_barrier(hdr)) return;

    // ---------------- D: tile partial dots of V[0..j] with u and w --------
    for (int item = blockIdx.x; item < p.n_items; item += gridDim.x) {
      const int ii = p.item_inst[item];
      T* V;
      InstView I = inst_view<T>(p, ii, &V);
      if (__ldcg(I.st + S_ACTIVE) == 0 || j >= I.m_cap) continue;
      const int64_t t = item - I.item0;
      const int64_t q0 = (t * TR) / 4, q1 = min(I.dim_pad, t * TR + TR) / 4;
      const double* wc = I.f + ((j & 1) ? I.L.w1 : I.L.w0);
      const T* U = V + (int64_t)j * I.dim_pad;
      const int64_t ld = I.m_cap + 1;
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      for (int i0 = 0; i0 <= j; i0 += kChunk) {
        const int nt = min(kChunk, j + 1 - i0);
        double au[kChunk], aw[kChunk];
#pragma unroll
        for (int c = 0; c < kChunk; ++c) au[c] = aw[c] = 0.0;
        for (int64_t q = q0 + threadIdx.x; q < q1; q += kThreads) {
          double u4[4], w4[4];
          ld4(U + 4 * q, u4);
          ld4(wc + 4 * q, w4);
#pragma unroll
          for (int c = 0; c < kChunk; ++c) {
            if (c < nt) {
              double x4[4];
              ld4(V + (int64_t)(i0 + c) * I.dim_pad + 4 * q, x4);
              au[c] = fma(x4[0], u4[0], fma(x4[1], u4[1], fma(x4[2], u4[2], fma(x4[3], u4[3], au[c]))));
              aw[c] = fma(x4[0], w4[0], fma(x4[1], w4[1], fma(x4[2], w4[2], fma(x4[3], w4[3], aw[c]))));
            }
          }
        }
#pragma unroll
        for (int c = 0; c < kChunk; ++c) {
          double a = au[c], b = aw[c];
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            b += __shfl_down_sync(0xffffffffu, b, o);
          }
          if (lane == 0) {
            red[(warp * kChunk + c) * 2 + 0] = a;
            red[(warp * kChunk + c) * 2 + 1] = b;
          }
        }
        __syncthreads();
        if (threadIdx.x < 2 * nt) {
          const int c = threadIdx.x / 2, s = threadIdx.x % 2;
          double a = 0.0;
          for (int w = 0; w < kWarps; ++w) a += red[(w * kChunk + c) * 2 + s];
          I.f[I.L.part + (t * ld + i0 + c) * 2 + s] = a;
        }
        __syncthreads();
      }
    }
    if (!grid_barrier(hdr)) return;

    // ---------------- R: h = sum of tile partials; coefficients -----------
    {
      const int64_t nv = (int64_t)p.n_inst * (j + 1);
      for (int64_t v = blockIdx.x; v < nv; v += gridDim.x) {
        const int ii = (int)(v / (j + 1)), i = (int)(v - (int64_t)ii * (j + 1));
        T* V;
        InstView I = inst_view<T>(p, ii, &V);
        if (__ldcg(I.st + S_ACTIVE) == 0 || j >= I.m_cap) continue;
        const int64_t ld = I.m_cap + 1;
        double a[2] = {0.0, 0.0};
        for (int64_t q = threadIdx.x; q < I.tiles; q += kThreads) {
          a[0] += __ldcg(I.f + I.L.part + (q * ld + i) * 2 + 0);
          a[1] += __ldcg(I.f + I.L.part + (q * ld + i) * 2 + 1);
        }
        block_sum<2>(a, red);
        if (threadIdx.x == 0) {
          I.f[I.L.hu + i] = a[0];
          I.f[I.L.hw + i] = a[1];
        }
        if (last_arrival(I.st + S_TICK_R, j + 1) && threadIdx.x < 32) {
          const int lane = threadIdx.x;
          const double* hu = I.f + I.L.hu;
          const double* hw = I.f + I.L.hw;
          double* al = I.f + I.L.alpha;
          double* be = I.f + I.L.beta;
          double ss = 0.0, szz = 0.0, sts = 0.0;
          for (int k2 = lane; k2 < j; k2 += 32) {
            const double sk = __ldcg(hu + k2), zk = __ldcg(hw + k2);
            double ts = __ldcg(al + k2) * sk;
            if (k2 > 0) ts = fma(__ldcg(be + k2), __ldcg(hu + k2 - 1), ts);
            if (k2 + 1 < j) ts = fma(__ldcg(be + k2 + 1), __ldcg(hu + k2 + 1), ts);
            ss = fma(sk, sk, ss);
            szz = fma(sk, zk, szz);
            sts = fma(sk, ts, sts);
          }
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            ss += __shfl_xor_sync(0xffffffffu, ss, o);
            szz += __shfl_xor_sync(0xffffffffu, szz, o);
            sts += __shfl_xor_sync(0xffffffffu, sts, o);
          }
          if (lane == 0) {
            double ts_last = 0.0;
            if (j > 0) {
              ts_last = __ldcg(al + j - 1) * __ldcg(hu + j - 1);
              if (j > 1) ts_last = fma(__ldcg(be + j - 1), __ldcg(hu + j - 2), ts_last);
            }
            const double r2 = __ldcg(hu + j) - ss;
            const double rr = r2 > 0.0 ? sqrt(r2) : 0.0;
            const double ri = rr > 0.0 ? 1.0 / rr : 0.0;
            const double omega = __ldcg(hw + j);
            I.f[I.L.misc + M_RI] = ri;
            I.f[I.L.misc + M_C] = (omega - szz) * ri;
            al[j] = (omega - 2.0 * szz + sts) * ri * ri;
            if (j > 0) be[j] = (__ldcg(hw + j - 1) - ts_last) * ri;
          }
        }
      }
    }
    if (!grid_barrier(hdr)) return;

    // ---------------- U: finish q_j, project w, |w|^2 partials ------------
    for (int item = blockIdx.x; item < p.n_items; item += gridDim.x) {
      const int ii = p.item_inst[item];
      T* V;
      InstView I = inst_view<T>(p, ii, &V);
      if (__ldcg(I.st + S_ACTIVE) == 0 || j >= I.m_cap) continue;
      const int64_t t = item - I.item0;
      const int64_t q0 = (t * TR) / 4, q1 = min(I.dim_pad, t * TR + TR) / 4;
      double* wc = I.f + ((j & 1) ? I.L.w1 : I.L.w0);
      T* U = V + (int64_t)j * I.dim_pad;
      __syncthreads();
      for (int c = threadIdx.x; c < j; c += kThreads) {
        sz[c] = __ldcg(I.f + I.L.hu + c);
        sz[j + c] = __ldcg(I.f + I.L.hw + c);
      }
      __syncthreads();
      const double ri = __ldcg(I.f + I.L.misc + M_RI), cc = __ldcg(I.f + I.L.misc + M_C);
      double nrm = 0.0;
      for (int64_t q = q0 + threadIdx.x; q < q1; q += kThreads) {
        double u4[4], w4[4];
        ld4(U + 4 * q, u4);
        ld4(wc + 4 * q, w4);
        for (int i = 0; i < j; ++i) {
          double a4[4];
          ld4(V + (int64_t)i * I.dim_pad + 4 * q, a4);
          const double si = sz[i], zi = sz[j + i];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            u4[e] = fma(-a4[e], si, u4[e]);
            w4[e] = fma(-a4[e], zi, w4[e]);
          }
        }
        double qv[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const T qe = round_to<T>(u4[e] * ri);
          qv[e] = (double)qe;
          w4[e] = fma(-qv[e], cc, w4[e]);
          nrm = fma(w4[e], w4[e], nrm);
        }
        st4(U + 4 * q, qv);
        st4(wc + 4 * q, w4);
      }
      block_sum<1>(&nrm, red);
      if (threadIdx.x == 0) I.f[I.L.part + t * 2] = nrm;
      if (last_arrival(I.st + S_TICK_U, (int)I.tiles) && threadIdx.x == 0) {
        double s = 0.0;
        for (int64_t q = 0; q < I.tiles; ++q) s += __ldcg(I.f + I.L.part + q * 2);
        const double nv = sqrt(s);
        I.f[I.L.misc + M_WNORM] = nv;
        I.f[I.L.misc + M_INV] = nv > 0.0 ? 1.0 / nv : 0.0;
        I.f[I.L.beta + j + 1] = nv * ri;
      }
    }
    if (!grid_barrier(hdr)) return;

    // ---------------- C: convergence check ---------------------------------
    if (p.check_at[j]) {
      const int m = j + 1;
      for (int ii = blockIdx.x; ii < p.n_inst; ii += gridDim.x) {
        T* V;
        InstView I = inst_view<T>(p, ii, &V);
        if (__ldcg(I.st + S_ACTIVE) == 0) continue;
        if (m > I.m_cap) continue;
        const double* al = I.f + I.L.alpha;
        const double* be = I.f + I.L.beta;
        __shared__ int mv_s, exact_s, done_s;
        if (threadIdx.x == 0) {
          double scale = 0.0;
          for (int i = 0; i < m; ++i) scale = fmax(scale, fabs(__ldcg(al + i)) + fabs(__ldcg(be + i)));
          const double thr = 1e-12 * fmax(scale, 1e-300);
          int mv = m;
          for (int i = 1; i <= m; ++i)
            if (fabs(__ldcg(be + i)) <= thr) { mv = i; break; }
          mv_s = mv;
          exact_s = mv < m || (mv == m && fabs(__ldcg(be + m)) <= thr) || (int64_t)m == I.dim;
        }
        __syncthreads();
        const int mv = mv_s, kk = p.k < mv ? p.k : mv;
        const int64_t ld = I.m_cap + 1;
        for (int64_t e = threadIdx.x; e < (int64_t)p.k * ld; e += kThreads) I.f[I.L.S + e] = 0.0;
        // the coefficients were written by other CTAs: stage them through L2
        double* a_s = sz;
        double* b_s = sz + (kMaxIter + 1);
        for (int i = threadIdx.x; i <= mv; i += kThreads) {
          if (i < mv) a_s[i] = __ldcg(al + i);
          b_s[i] = __ldcg(be + i);
        }
        __syncthreads();
        double* ev = I.f + I.L.misc + 8 + kMaxK;
        edg::tridiag_body(a_s, b_s, mv, kk, ev, I.f + I.L.S, (int)ld, I.f + I.L.tri);
        __syncthreads();
        if (threadIdx.x == 0) {
          const bool exact = exact_s != 0;
          bool ok = kk == p.k || exact;
          double* rs = I.f + I.L.misc + 8;
          for (int q = 0; q < kk; ++q) {
            const double theta = ev[q];
            const double last = I.f[I.L.S + (int64_t)q * ld + (mv - 1)];
            const double r = exact ? 0.0 : fabs(__ldcg(be + mv) * last);
            rs[q] = r;
            if (r > p.tol * fmax(1.0, fabs(theta))) ok = false;
          }
          done_s = ok || m >= I.m_cap || m >= p.max_iter;
          if (done_s) {
            for (int q = 0; q < p.k; ++q) {
              p.evals[(int64_t)ii * p.k + q] = q < kk ? ev[q] : NAN;
              p.resid[(int64_t)ii * p.k + q] = q < kk ? rs[q] : NAN;
            }
            p.iters[ii] = mv;
            I.st[S_ACTIVE] = 0;
            atomicSub(hdr + H_ACTIVE, 1);
          }
        }
        __syncthreads();
      }
      if (!grid_barrier(hdr)) return;
      if (atomicAdd(hdr + H_ACTIVE, 0) == 0) break;
    }
  }

  // ---------------- ground-state Ritz vectors (f64), normalised ----------
  if (!p.evecs) return;
  for (int item = blockIdx.x; item < p.n_items; item += gridDim.x) {
    const int ii = p.item_inst[item];
    T* V;
    InstView I = inst_view<T>(p, ii, &V);
    const int64_t t = item - I.item0;
    const int64_t r0 = t * TR, r1 = min(I.dim, r0 + TR);
    int m = __ldcg(p.iters + ii);
    m = m < 0 ? 0 : (m > I.m_cap ? (int)I.m_cap : m);
    const double* S0 = I.f + I.L.S;
    double* y = I.f + I.L.w0;
    double nrm = 0.0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) {
      double a = 0.0;
      for (int i = 0; i < m; ++i) a = fma(ldv(V + (int64_t)i * I.dim_pad + r), __ldcg(S0 + i), a);
      y[r] = a;
      nrm = fma(a, a, nrm);
    }
    block_sum<1>(&nrm, red);
    if (threadIdx.x == 0) I.f[I.L.part + t * 2] = nrm;
    if (last_arrival(I.st + S_TICK_N, (int)I.tiles) && threadIdx.x == 0) {
      double s = 0.0;
      for (int64_t q = 0; q < I.tiles; ++q) s += __ldcg(I.f + I.L.part + q * 2);
      I.f[I.L.misc + M_INV] = s > 0.0 ? 1.0 / sqrt(s) : 0.0;
    }
  }
  if (!grid_barrier(hdr)) return;
  for (int item = blockIdx.x; item < p.n_items; item += gridDim.x) {
    const int ii = p.item_inst[item];
    T* V;
    InstView I = inst_view<T>(p, ii, &V);
    const int64_t t = item - I.item0;
    const int64_t r0 = t * TR, r1 = min(I.dim, r0 + TR);
    const double inv = __ldcg(I.f + I.L.misc + M_INV);
    const double* y = I.f + I.L.w0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += kThreads) p.evecs[I.row_off + r] = __ldcg(y + r) * inv;
  }
}

template <typename T>
void* kernel_for(int lanes) {
  switch (lanes) {
    case 2: return (void*)tiled_lanczos_k<T, 2>;
    case 4: return (void*)tiled_lanczos_k<T, 4>;
    case 8: return (void*)tiled_lanczos_k<T, 8>;
    case 16: return (void*)tiled_lanczos_k<T, 16>;
    case 32: return (void*)tiled_lanczos_k<T, 32>;
    default: return nullptr;
  }
}

}  // namespace

extern "C" int edg_tiled_batch_plan(int32_t n_inst, const int64_t* dims, int32_t dtype, int32_t max_iter, int32_t k,
                                    int32_t tile_rows, int32_t check_every, int64_t* inst_out,
                                    int32_t* item_inst_out, uint8_t* check_at_out, int32_t* n_items_out,
                                    int64_t* workspace_bytes_out) {
  EDG_REQUIRE(n_inst >= 1 && dims != nullptr, "edg_tiled_batch_plan: need at least one instance");
  EDG_REQUIRE(dtype == 0 || dtype == 1, "edg_tiled_batch_plan: dtype must be 0 (f64) or 1 (f32)");
  EDG_REQUIRE(max_iter >= 1 && max_iter <= kMaxIter, "edg_tiled_batch_plan: max_iter must be 1..%d", kMaxIter);
  EDG_REQUIRE(k >= 1 && k <= kMaxK, "edg_tiled_batch_plan: k must be 1..%d", kMaxK);
  EDG_REQUIRE(tile_rows >= 4 && tile_rows % 4 == 0, "edg_tiled_batch_plan: tile_rows must be a positive multiple of 4");
  EDG_REQUIRE(check_every >= 1, "edg_tiled_batch_plan: check_every must be >= 1");
  const int esz = dtype == 0 ? 8 : 4;
  int64_t off = al256((int64_t)(H_WORDS + (int64_t)n_inst * S_N) * 4);
  int64_t items = 0;
  // f64 blocks first, then the Krylov bases
  std::vector<int64_t> rec((size_t)n_inst * F_N);
  int64_t row_off = 0, rp_off = 0;
  for (int i = 0; i < n_inst; ++i) {
    EDG_REQUIRE(dims[i] >= 1, "edg_tiled_batch_plan: instance %d has dimension %lld", i, (long long)dims[i]);
    const int64_t dim = dims[i], dim_pad = (dim + 3) & ~int64_t(3);
    const int64_t tiles = (dim_pad + tile_rows - 1) / tile_rows;
    const int64_t m_cap = dim < max_iter ? dim : max_iter;
    int64_t* r = rec.data() + (int64_t)i * F_N;
    r[F_DIM] = dim;
    r[F_ROW_OFF] = row_off;
    r[F_ROWPTR_OFF] = rp_off;
    r[F_TILES] = tiles;
    r[F_ITEM0] = items;
    r[F_MCAP] = m_cap;
    r[F_F_OFF] = off;
    off = al256(off + f_layout(dim_pad, tiles, m_cap, k).total * 8);
    row_off += dim;
    rp_off += dim + 1;
    items += tiles;
  }
  EDG_REQUIRE(items <= INT32_MAX, "edg_tiled_batch_plan: too many work items");
  for (int i = 0; i < n_inst; ++i) {
    int64_t* r = rec.data() + (int64_t)i * F_N;
    const int64_t dim_pad = (r[F_DIM] + 3) & ~int64_t(3);
    r[F_V_OFF] = off;
    off = al256(off + (r[F_MCAP] + 1) * dim_pad * esz);
  }
  if (inst_out) std::copy(rec.begin(), rec.end(), inst_out);
  if (item_inst_out)
    for (int i = 0; i < n_inst; ++i)
      for (int64_t t = 0; t < rec[(size_t)i * F_N + F_TILES]; ++t)
        item_inst_out[rec[(size_t)i * F_N + F_ITEM0] + t] = i;
  if (check_at_out) {
    // every check_every steps, at the last step, and where an instance
    // reaches its Krylov cap (so every instance is finalised)
    for (int j = 0; j < max_iter; ++j) check_at_out[j] = (uint8_t)((j + 1) % check_every == 0 || j + 1 == max_iter);
    for (int i = 0; i < n_inst; ++i) check_at_out[rec[(size_t)i * F_N + F_MCAP] - 1] = 1;
  }
  if (n_items_out) *n_items_out = (int32_t)items;
  if (workspace_bytes_out) *workspace_bytes_out = off;
  return EDG_OK;
}

extern "C" int edg_tiled_batch_header_bytes(int32_t n_inst) {
  return (int)((H_WORDS + (int64_t)n_inst * S_N) * 4);
}

extern "C" int edg_lanczos_tiled_batch(const edg_tiled_batch* b, cudaStream_t stream) {
  EDG_REQUIRE(b != nullptr, "edg_lanczos_tiled_batch: null batch");
  EDG_REQUIRE(b->dtype == 0 || b->dtype == 1, "edg_lanczos_tiled_batch: dtype must be 0 or 1");
  EDG_REQUIRE(b->n_inst >= 1 && b->n_items >= b->n_inst, "edg_lanczos_tiled_batch: bad instance or item count");
  EDG_REQUIRE(b->k >= 1 && b->k <= kMaxK, "edg_lanczos_tiled_batch: k must be 1..%d", kMaxK);
  EDG_REQUIRE(b->max_iter >= 1 && b->max_iter <= kMaxIter, "edg_lanczos_tiled_batch: max_iter must be 1..%d",
              kMaxIter);
  EDG_REQUIRE(b->tile_rows >= 4 && b->tile_rows % 4 == 0, "edg_lanczos_tiled_batch: tile_rows must be a multiple of 4");
  EDG_REQUIRE(b->inst && b->item_inst && b->check_at && b->rowptr && b->diag && b->workspace && b->evals &&
                  b->resid && b->iters && b->status,
              "edg_lanczos_tiled_batch: null pointer");
  EDG_REQUIRE(((uintptr_t)b->workspace & 255) == 0, "edg_lanczos_tiled_batch: workspace must be 256-byte aligned");
  void* fn = b->dtype == 0 ? kernel_for<double>(b->lanes) : kernel_for<float>(b->lanes);
  EDG_REQUIRE(fn != nullptr, "edg_lanczos_tiled_batch: lanes must be 2, 4, 8, 16 or 32, got %d", b->lanes);
  int dev = 0, n_sm = 0, per_sm = 0, coop = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos_tiled_batch: device query");
  EDG_REQUIRE(coop != 0 && per_sm >= 1, "edg_lanczos_tiled_batch: cooperative launch unavailable");
  int64_t want = b->n_items > b->n_inst ? b->n_items : b->n_inst;
  int64_t cap = (int64_t)n_sm * per_sm;
  const unsigned grid = (unsigned)(want < cap ? want : cap);
  // barrier words, status, active count and tickets start at zero
  e = cudaMemsetAsync(b->workspace, 0, (size_t)edg_tiled_batch_header_bytes(b->n_inst), stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->status, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos_tiled_batch: reset");
  Params p{};
  p.n_inst = b->n_inst;
  p.n_items = b->n_items;
  p.tile_rows = b->tile_rows;
  p.k = b->k;
  p.max_iter = b->max_iter;
  p.tol = b->tol;
  p.seed = b->seed;
  p.inst = b->inst;
  p.item_inst = b->item_inst;
  p.check_at = b->check_at;
  p.rowptr = b->rowptr;
  p.cols = b->cols;
  p.vals = b->vals;
  p.diag = b->diag;
  p.v0 = b->v0;
  p.ws = (char*)b->workspace;
  p.evals = b->evals;
  p.resid = b->resid;
  p.iters = b->iters;
  p.evecs = b->evecs;
  p.status = b->status;
  void* args[] = {&p};
  e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, 0, stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos_tiled_batch: launch");
  // the barrier status word of the workspace header is the launch's verdict
  e = cudaMemcpyAsync(b->status, (int*)b->workspace + H_STATUS, sizeof(int32_t), cudaMemcpyDeviceToDevice, stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_lanczos_tiled_batch: status");
  return EDG_OK;
}
