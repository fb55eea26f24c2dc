// Reorthogonalisation passes of the delayed Gram-Schmidt Lanczos step with the
// Krylov basis streamed through shared memory by bulk asynchronous copies.
//
// Both passes read V[0..j) (or V[0..j]) once, row segment by row segment.  A
// persistent grid of one CTA per SM owns an equal, contiguous run of (problem,
// segment) work items.  Warp 8 of the CTA is the producer: one lane issues
// cp.async.bulk copies (this GPU's memory only, no multicast) of one Krylov
// vector's segment per ring stage and signals the stage's "full" mbarrier
// through its transaction count.  Warps 0..7 consume: each thread owns one
// row quad of the segment, waits for the stage, computes from shared memory
// and releases the stage on its "empty" mbarrier.  The ring keeps
// kStages x 4 KB (f32) of copies in flight per SM whatever the register use
// of the consumers, which is what the bandwidth of a streaming pass needs.
//
// Every wait is bounded (1 s on the global timer).  A wait that runs out sets
// the error word; from then on no role waits any more and no data is used,
// so every thread still reaches every named barrier, and before leaving the
// producer waits (bounded) for the copies it issued.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace edg {
namespace bulk {

constexpr int kConsumers = 256;               // 8 consumer warps
constexpr int kThreadsAll = kConsumers + 32;  // + producer warp
constexpr int kSegQuads = kConsumers;         // one quad per consumer thread
constexpr int kSegRows = 4 * kSegQuads;       // 1024 rows per segment
constexpr int kVecs = 8;                    // Krylov vectors per ring stage (one tile)
// ring stages: 96 KB (f32, 3 stages) or 128 KB (f64, 2 stages) in flight
template <typename T>
struct Ring {
  static constexpr int kStages = sizeof(T) == 4 ? 3 : 2;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 1-D bulk copy global -> shared (16-byte aligned addresses, size a multiple
// of 16), completion counted on bar's transaction count.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void consumers_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// Bounded wait on (bar, parity).  Returns false without waiting once *err is
// set, and sets it when the wait runs out.
__device__ __forceinline__ bool wait_bounded(uint64_t* bar, unsigned parity, volatile int* err) {
  if (*err) return false;
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = now_ns();
  for (unsigned it = 1;; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 63u) == 0) {
      if (*err) return false;
      if (now_ns() - t0 > 1000000000ull) {
        *err = 1;
        return false;
      }
    }
  }
}

// The run of (problem, segment) items of CTA c: items are numbered
// v * n_seg + g and split evenly over the grid.
struct Run {
  int64_t first, last;  // [first, last)
};
__device__ __forceinline__ Run run_of(int64_t n_items) {
  const int64_t c = blockIdx.x, C = gridDim.x;
  return {n_items * c / C, n_items * (c + 1) / C};
}

// Shared-memory layout of a pass: ring of segments of one vector, full/empty
// barriers, the error word and the reduction scratch (dynamic shared memory;
// a pass may append its coefficients after it).
template <typename T>
struct Smem {
  static constexpr int S = Ring<T>::kStages;
  alignas(128) T ring[S][kVecs][kSegRows];
  alignas(8) uint64_t full[S];
  alignas(8) uint64_t empty[S];
  int err;
  int last;
  alignas(8) double red[kConsumers / 32][16];
};

// Producer lane: streams n_vec vectors (V + i * stride_i) of every item of the
// CTA's run, one tile of up to kVecs vectors per ring stage (one bulk copy per
// vector segment, all counted on the stage's full barrier).  Stops issuing when
// the error word is set; before returning it waits (1 s at most, error or
// not) until the copies it issued into every stage have landed, so none is in
// flight at exit.
template <typename T>
__device__ void produce(Smem<T>& sm, const T* V, int64_t n_pad, int64_t stride_i, int64_t n_seg, int n_vec,
                        Run run) {
  constexpr int S = Smem<T>::S;
  int64_t issued[S];
#pragma unroll
  for (int s = 0; s < S; ++s) issued[s] = 0;
  const int64_t nq = n_pad / 4;
  int64_t k = 0;
  bool stop = false;
  for (int64_t item = run.first; item < run.last && !stop; ++item) {
    const int64_t v = item / n_seg, g = item - v * n_seg;
    const int64_t q0 = g * kSegQuads;
    const int64_t nqs = nq - q0 < kSegQuads ? nq - q0 : kSegQuads;
    const unsigned bytes = (unsigned)(nqs * 4 * sizeof(T));
    const T* src = V + v * n_pad + 4 * q0;
    for (int i0 = 0; i0 < n_vec; i0 += kVecs, ++k) {
      const int nt = n_vec - i0 < kVecs ? n_vec - i0 : kVecs;
      const int s = (int)(k % S);
      const int64_t round = k / S;
      if (round > 0 && !wait_bounded(&sm.empty[s], (unsigned)((round - 1) & 1), &sm.err)) {
        stop = true;
        break;
      }
      mbar_expect_tx(&sm.full[s], bytes * (unsigned)nt);
      for (int t = 0; t < nt; ++t) bulk_g2s(sm.ring[s][t], src + (int64_t)(i0 + t) * stride_i, bytes, &sm.full[s]);
      issued[s] = round + 1;
    }
  }
#pragma unroll 1
  for (int s = 0; s < S; ++s) {
    if (issued[s] == 0) continue;
    const unsigned parity = (unsigned)((issued[s] - 1) & 1);
    const uint64_t t0 = now_ns();
    while (!mbar_try_wait(&sm.full[s], parity))
      if (now_ns() - t0 > 1000000000ull) break;
  }
}

// Consumer side of ring stage k (one tile of vectors): wait for it, return
// whether the data may be used; release() hands the stage back (one arrival
// per warp).
template <typename T>
__device__ __forceinline__ bool acquire(Smem<T>& sm, int64_t k) {
  constexpr int S = Smem<T>::S;
  return wait_bounded(&sm.full[k % S], (unsigned)((k / S) & 1), &sm.err);
}
template <typename T>
__device__ __forceinline__ void release(Smem<T>& sm, int64_t k) {
  __syncwarp();
  if ((threadIdx.x & 31) == 0) mbar_arrive(&sm.empty[k % Smem<T>::S]);
}

template <typename T>
__device__ __forceinline__ void init_barriers(Smem<T>& sm) {
  if (threadIdx.x == 0) {
    for (int s = 0; s < Smem<T>::S; ++s) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.empty[s], kConsumers / 32);
    }
    sm.err = 0;
    sm.last = 0;
    fence_mbar_init();
  }
  __syncthreads();
}

__device__ __forceinline__ void lds4(const float* p, double* o) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
}
__device__ __forceinline__ void lds4(const double* p, double* o) {
  const double2 a = reinterpret_cast<const double2*>(p)[0];
  const double2 b = reinterpret_cast<const double2*>(p)[1];
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}

}  // namespace bulk
}  // namespace edg
