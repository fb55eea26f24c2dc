// Dictionary-packed tiles: the off-diagonal matrix with one 32-bit word per
// entry slot.
//
// The sector Hamiltonians of the lattice gauge models have very few distinct
// off-diagonal values (products of a handful of local matrix elements: eight
// on the periodic SU(2) j = 1/2 chain in its real form), so each entry is
//     word = column | (value index << colbits),  colbits = bits of n_rows,
// with the distinct values in a small table.  Rows are grouped in tiles of
// 16, each tile as wide as its longest row and stored k-major (layout below);
// the stream is 4 bytes a slot instead of 8 (f32 value + int32 column) or 12
// (f64) an entry.  The product is the same as the CSR one (csr_spmv,
// edlgt/modeling/qmb_hamiltonian.py:705-730).
//
// Build (on the device, once per matrix):
//   edg_pack_collect      inserts the bit patterns of the values into a hash
//                         set; the host reads the set, sorts the distinct
//                         values and uploads them as the table;
//   edg_pack_tile_counts  the tiles' word counts (a scan gives their offsets);
//   edg_pack_encode       writes the tile offsets and the packed words (binary
//                         search of each value in the sorted table).
//
// Matvec (packed_spmv_k): one warp takes tiles of 16 consecutive rows.  A
// tile is a contiguous, 64-byte-aligned range of the stream, which lane 0
// copies into one of the warp's two shared-memory stages with a bulk
// asynchronous copy (completion on the stage's mbarrier) one tile ahead,
// while the tile offsets are loaded two tiles ahead; two lanes per row then
// walk their row from shared memory (lane j takes entries j, j + 2, j + 4,
// ...; the two lanes of all 16 rows read 32 consecutive words), gathering x
// rows.  The stream is read with whole-range copies that bypass the load
// pipeline (the CSR kernel's loads touch one segment per row of the warp on
// every load), which leaves the L1 data pipe to the gathers.  f32 matrices
// (the f32 Krylov phase) sum each lane's products in f32 and add the lane
// sums and the diagonal term in f64, so no conversion happens per entry; f64
// matrices sum in f64 in the CSR kernel's order (bit-identical to the CSR
// kernel with two threads a row).
#include <algorithm>

#include "reorth_bulk.cuh"
#include "spmv.cuh"

namespace {

constexpr int kTileRows = 16;   // rows of a warp tile (two lanes a row)
constexpr int kTileWords = 512;  // staged entries of a tile; longer tiles read the stream directly
constexpr int kStageWords = kTileWords + 4;
constexpr int kWarps = 8;  // warps of a CTA

template <typename T>
struct Pat;  // bit pattern of a value, and the empty-slot marker (a NaN pattern: NaN values are refused)
template <>
struct Pat<float> {
  using U = unsigned int;
  static constexpr U kEmpty = 0xFFFFFFFFu;
  __device__ static U of(float v) { return __float_as_uint(v); }
  __device__ static uint32_t hash(U b) { return b * 2654435761u; }
};
template <>
struct Pat<double> {
  using U = unsigned long long;
  static constexpr U kEmpty = 0xFFFFFFFFFFFFFFFFull;
  __device__ static U of(double v) { return (U)__double_as_longlong(v); }
  __device__ static uint32_t hash(U b) { return (uint32_t)((b * 0x9E3779B97F4A7C15ull) >> 32); }
};

// Distinct bit patterns of vals into an open-addressing set of 2^log2_slots
// slots (pre-filled with 0xFF bytes).  Each CTA first records the values in
// a small shared-memory set and only the first of its threads to meet a
// value probes the global set (a matrix has a handful of values, so without
// this millions of probes would hit the same few global words); a plain read
// comes before any atomic.  overflow[0] is set when a global probe sequence
// runs past max_probe slots or a value is a NaN.
template <typename T>
__global__ void pack_collect_k(const T* __restrict__ vals, int64_t nnz, typename Pat<T>::U* __restrict__ set,
                               int log2_slots, int max_probe, int* __restrict__ overflow) {
  using U = typename Pat<T>::U;
  constexpr int kLocalBits = 8;  // CTA-local set of 256 slots
  constexpr int kLocalProbe = 16;
  __shared__ U local[1 << kLocalBits];
  for (int i = threadIdx.x; i < (1 << kLocalBits); i += blockDim.x) local[i] = Pat<T>::kEmpty;
  __syncthreads();
  const uint32_t mask = (1u << log2_slots) - 1u;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
    const T v = __ldg(vals + i);
    const U b = Pat<T>::of(v);
    if (isnan(v)) {
      atomicExch(overflow, 1);
      continue;
    }
    // CTA-local set: a value found there has been (or is being) inserted
    // into the global set by the thread that recorded it
    bool seen = false;
    uint32_t ls = Pat<T>::hash(b) >> (32 - kLocalBits);
    for (int probe = 0; probe < kLocalProbe; ++probe, ls = (ls + 1) & ((1u << kLocalBits) - 1)) {
      U cur = *(volatile U*)(local + ls);
      if (cur == b) {
        seen = true;
        break;
      }
      if (cur == Pat<T>::kEmpty) {
        cur = atomicCAS(local + ls, Pat<T>::kEmpty, b);
        if (cur == b) seen = true;
        if (cur == Pat<T>::kEmpty || cur == b) break;
      }
    }
    if (seen) continue;
    uint32_t s = Pat<T>::hash(b) >> (32 - log2_slots);
    bool placed = false;
    for (int probe = 0; probe < max_probe; ++probe, s = (s + 1) & mask) {
      U cur = *(volatile U*)(set + s);
      if (cur == b) {
        placed = true;
        break;
      }
      if (cur == Pat<T>::kEmpty) {
        cur = atomicCAS(set + s, Pat<T>::kEmpty, b);
        if (cur == Pat<T>::kEmpty || cur == b) {
          placed = true;
          break;
        }
      }
    }
    if (!placed) atomicExch(overflow, 1);
  }
}

// Index of v in the ascending table (bit comparison: -0.0 and +0.0 are
// distinct entries), or -1.
template <typename T>
__device__ __forceinline__ int table_index(const T* tab, int count, T v) {
  int lo = 0, hi = count;  // first table entry >= v
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (tab[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  int idx = -1;
  for (int q = lo > 0 ? lo - 1 : 0; q < count && q <= lo + 1; ++q)
    if (Pat<T>::of(tab[q]) == Pat<T>::of(v)) idx = q;
  return idx;
}

// The tile layout.  Tiles are 16 consecutive rows; tile t is w_t = the
// length of its longest row wide, and its 16 w_t words [tile_off[t],
// tile_off[t+1]) hold entry k of the tile's row s at tile_off[t] + 16 k + s
// (k-major), rows shorter than w_t padded with the all-ones word, whose
// column (2^colbits - 1 >= n_rows) is never a real one.  Entry k of the
// tile's 16 rows is then one run of 16 words.

// counts[t] = 16 w_t
__global__ void pack_counts_k(int64_t n, const int64_t* __restrict__ rowptr, int64_t* __restrict__ counts) {
  const int64_t n_tiles = (n + kTileRows - 1) / kTileRows;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n_tiles; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r0 = t * kTileRows, r1 = r0 + kTileRows < n ? r0 + kTileRows : n;
    int64_t w = 0;
    for (int64_t r = r0; r < r1; ++r) w = max(w, rowptr[r + 1] - rowptr[r]);
    counts[t] = kTileRows * w;
  }
}

// One thread per (tile, row slot): the slot's words, the value of each entry
// replaced by its table index; padding slots all ones.  offsets [n_tiles+1]
// (int64, the scan of counts) becomes tile_off (int32).  missing[0] is set
// when a value is not in the table.
template <typename T>
__global__ void pack_encode_k(int64_t n, int64_t total, const int64_t* __restrict__ rowptr,
                              const int32_t* __restrict__ cols, const T* __restrict__ vals,
                              const T* __restrict__ table, int count, int colbits,
                              const int64_t* __restrict__ offsets, int32_t* __restrict__ tile_off,
                              uint32_t* __restrict__ words, int* __restrict__ missing) {
  extern __shared__ __align__(16) unsigned char enc_raw[];
  T* tab = reinterpret_cast<T*>(enc_raw);
  for (int i = threadIdx.x; i < count; i += blockDim.x) tab[i] = table[i];
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t n_tiles = (n + kTileRows - 1) / kTileRows;
  for (int64_t t = t0; t <= n_tiles; t += stride) tile_off[t] = (int32_t)offsets[t];
  for (int64_t q = t0; q < n_tiles * kTileRows; q += stride) {
    const int64_t t = q / kTileRows, r = q;
    const int s = (int)(q - t * kTileRows);
    const int64_t base = offsets[t], w = (offsets[t + 1] - base) / kTileRows;
    const int64_t beg = r < n ? rowptr[r] : 0, len = r < n ? rowptr[r + 1] - beg : 0;
    for (int64_t k = 0; k < w; ++k) {
      uint32_t word = 0xFFFFFFFFu;
      if (k < len) {
        const int idx = table_index(tab, count, __ldg(vals + beg + k));
        if (idx < 0) atomicExch(missing, 1);
        word = (uint32_t)__ldg(cols + beg + k) | ((uint32_t)(idx < 0 ? 0 : idx) << colbits);
      }
      words[base + kTileRows * k + s] = word;
    }
  }
  // four words after the stream (a whole-quad read past the end stays in
  // the allocation)
  if (t0 < 4) words[total + t0] = 0xFFFFFFFFu;
}

struct Tile {
  int64_t r0;
  int nr;  // rows of the tile (0: past the end)
};
__device__ __forceinline__ Tile tile_of(int64_t t, int64_t n) {
  const int64_t r0 = t * kTileRows;
  const int64_t left = n - r0;
  return {r0, left <= 0 ? 0 : (int)(left < kTileRows ? left : kTileRows)};
}

// Lanes 0 and 1 hold tile_off[t], tile_off[t + 1].
__device__ __forceinline__ int32_t load_head(const int32_t* __restrict__ tile_off, int64_t t, Tile tl, int lane) {
  return tl.nr > 0 && lane < 2 ? __ldg(tile_off + t + lane) : 0;
}

// A tile's words [e0, e0 + 16 width) (e0 a multiple of 16: 64-byte aligned);
// `fits` when they fit the stage.
struct Range {
  int32_t e0, width, quads;
  bool fits;
};
__device__ __forceinline__ Range range_of(Tile tl, int32_t head) {
  const int32_t e0 = __shfl_sync(0xffffffffu, head, 0);
  const int32_t e1 = __shfl_sync(0xffffffffu, head, 1);
  const int32_t width = tl.nr > 0 ? (e1 - e0) / kTileRows : 0;
  const int32_t quads = width * (kTileRows / 4);
  return {e0, width, quads, width * kTileRows <= kTileWords};
}

// Lane 0 copies the tile's range into a stage with one bulk asynchronous copy
// (this GPU's memory, no multicast) completing on the stage's mbarrier;
// returns whether a copy was issued (warp-uniform).
__device__ __forceinline__ bool stage_tile(const uint32_t* __restrict__ words, Range rg, uint32_t* stage,
                                           uint64_t* bar, int lane) {
  const bool issue = rg.fits && rg.quads > 0;
  if (issue && lane == 0) {
    // the stage was last read through the generic proxy (ordered by __syncwarp)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    edg::bulk::mbar_expect_tx(bar, (unsigned)rg.quads * 16u);
    edg::bulk::bulk_g2s(stage, words + rg.e0, (unsigned)rg.quads * 16u, bar);
  }
  return issue;
}

// x row (NV entries at stride XS) as stored
template <typename T, int NV, int XS>
struct XRow {
  __device__ static void ld(const T* x, int64_t c, T (&o)[NV]) {
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = __ldg(x + c * XS + v);
  }
};
template <int NV>
struct XRow<float, NV, 4> {
  __device__ static void ld(const float* x, int64_t c, float (&o)[NV]) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(x) + c);
    const float f[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = f[v];
  }
};
template <>
struct XRow<float, 2, 2> {  // a complex64 entry as two real parts
  __device__ static void ld(const float* x, int64_t c, float (&o)[2]) {
    const float2 q = __ldg(reinterpret_cast<const float2*>(x) + c);
    o[0] = q.x;
    o[1] = q.y;
  }
};
template <>
struct XRow<double, 2, 2> {  // a complex128 entry as two real parts
  __device__ static void ld(const double* x, int64_t c, double (&o)[2]) {
    const double2 q = __ldg(reinterpret_cast<const double2*>(x) + c);
    o[0] = q.x;
    o[1] = q.y;
  }
};
template <int NV>
struct XRow<double, NV, 4> {
  __device__ static void ld(const double* x, int64_t c, double (&o)[NV]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(x) + 2 * c);
    const double2 b = __ldg(reinterpret_cast<const double2*>(x) + 2 * c + 1);
    const double f[4] = {a.x, a.y, b.x, b.y};
#pragma unroll
    for (int v = 0; v < NV; ++v) o[v] = f[v];
  }
};

// The tile's rows, two lanes a row (lane j of row s takes entries k = j,
// j + 2, ... of it), from the stage (shared) or the stream: acc[v] +=
// table[idx] x[col][v] in the accumulator type A (f32 lane sums for an f32
// matrix, f64 for f64), four gathers in flight.  Entry k of the tile's rows
// is the run of words [16 k, 16 k + 16), so lanes j = 0, 1 read 32
// consecutive words (no bank conflicts); padding words are skipped.
template <typename T, typename A, int NV, int XS>
__device__ __forceinline__ void gather_tile(const uint32_t* src, int width, int s, int j, const T* tab, int colbits,
                                            uint32_t cmask, const T* __restrict__ x, A (&acc)[NV], bool shared) {
  for (int k0 = j; k0 < width; k0 += 8) {
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = k0 + 2 * q;
      const int off = kTileRows * k + s;
      w[q] = k < width ? (shared ? src[off] : __ldg(src + off)) : 0xFFFFFFFFu;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
      if ((w[q] & cmask) != cmask) {
        T xr[NV];
        XRow<T, NV, XS>::ld(x, (int64_t)(w[q] & cmask), xr);
        const A a = (A)tab[w[q] >> colbits];
#pragma unroll
        for (int v = 0; v < NV; ++v) acc[v] = fma(a, (A)xr[v], acc[v]);
      }
  }
}

// y[v * y_plane + r] (f64; y[r * NV + v] when y_plane is 0) = sum over the
// row's entries of table[idx] x[col][v] + diag[r][v] x[r][v] (diag[r] for
// every v when diag_shared: a complex vector as NV = 2 real parts of one
// real matrix); T = f32 or f64 table, diagonal and x.  With f32 (the
// f32 Krylov phase) every lane sums its products in f32 and the two lane sums
// and the diagonal term are added in f64 (a few f32 roundings per row, no
// conversion per entry); with f64 the products and sums are f64, in the CSR
// kernel's order.  A stage wait that runs out (1 s) sets *err (if given) and
// ends the warp's work.
template <typename T, int NV, int XS>
__global__ void __launch_bounds__(kWarps * 32, 4)
    packed_spmv_k(int64_t n, const int32_t* __restrict__ tile_off, const uint32_t* __restrict__ words,
                  const T* __restrict__ table, int count, int colbits, const T* __restrict__ diag,
                  const T* __restrict__ x, double* __restrict__ y, int64_t y_plane, int diag_shared,
                  const int* __restrict__ skip, int* __restrict__ err) {
  using A = T;  // lane accumulator: f32 lanes for the f32 phase, f64 otherwise
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ int s_err;
  if (skip != nullptr && *skip) return;
  uint32_t* stage_all = reinterpret_cast<uint32_t*>(smem_raw);  // [kWarps][2][kStageWords]
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem_raw + sizeof(uint32_t) * kWarps * 2 * kStageWords);
  T* tab = reinterpret_cast<T*>(smem_raw + sizeof(uint32_t) * kWarps * 2 * kStageWords + sizeof(uint64_t) * kWarps * 2);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t* const bar = bars + 2 * warp;
  if (threadIdx.x == 0) s_err = 0;
  if (lane == 0) {
    edg::bulk::mbar_init(&bar[0], 1);
    edg::bulk::mbar_init(&bar[1], 1);
    edg::bulk::fence_mbar_init();
  }
  for (int i = threadIdx.x; i < count; i += blockDim.x) tab[i] = table[i];
  __syncthreads();
  uint32_t* const stage0 = stage_all + warp * 2 * kStageWords;  // two stages of kStageWords
  const uint32_t cmask = (1u << colbits) - 1u;
  const int64_t n_tiles = (n + kTileRows - 1) / kTileRows;
  const int64_t step = (int64_t)gridDim.x * kWarps;
  const int s = lane >> 1, j = lane & 1;
  int64_t t = (int64_t)blockIdx.x * kWarps + warp;
  // pipeline: the words of tile t are staged one tile ahead, the tile
  // offsets loaded two tiles ahead
  Tile cur = tile_of(t, n), nxt = tile_of(t + step, n);
  int32_t h_cur = load_head(tile_off, t, cur, lane);
  int32_t h_nxt = load_head(tile_off, t + step, nxt, lane);
  Range rg_cur = range_of(cur, h_cur);
  // bit s of pend: a copy into stage s is in flight; bit s of phase: the
  // parity of that stage's mbarrier for its next completion
  unsigned pend = stage_tile(words, rg_cur, stage0, &bar[0], lane) ? 1u : 0u;
  unsigned phase = 0u;
  int b = 0;
  for (; t < n_tiles; t += step) {
    const Tile nn = tile_of(t + 2 * step, n);
    const Range rg_nxt = range_of(nxt, h_nxt);
    if (stage_tile(words, rg_nxt, stage0 + (b ^ 1) * kStageWords, &bar[b ^ 1], lane)) pend |= 2u >> b;
    const int32_t h_nn = load_head(tile_off, t + 2 * step, nn, lane);
    if (pend & (1u << b)) {
      const bool ok = edg::bulk::wait_bounded(&bar[b], (phase >> b) & 1u, &s_err);
      if (!__all_sync(0xffffffffu, ok)) break;  // warp-uniform
      pend &= ~(1u << b);
      phase ^= 1u << b;
    }
    A acc[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[v] = (A)0;
    if (rg_cur.fits)
      gather_tile<T, A, NV, XS>(stage0 + b * kStageWords, rg_cur.width, s, j, tab, colbits, cmask, x, acc, true);
    else
      gather_tile<T, A, NV, XS>(words + rg_cur.e0, rg_cur.width, s, j, tab, colbits, cmask, x, acc, false);
    double tot[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      tot[v] = (double)acc[v];
      tot[v] += __shfl_xor_sync(0xffffffffu, tot[v], 1, 2);
    }
    if (s < cur.nr && j == 0) {
      const int64_t r = cur.r0 + s;
      T xr[NV];
      XRow<T, NV, XS>::ld(x, r, xr);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double d = (double)__ldg(diag_shared ? diag + r : diag + r * NV + v);
        y[y_plane > 0 ? v * y_plane + r : r * NV + v] = fma(d, (double)xr[v], tot[v]);
      }
    }
    __syncwarp();  // this stage is refilled by the next iteration
    cur = nxt;
    nxt = nn;
    h_cur = h_nxt;
    h_nxt = h_nn;
    rg_cur = rg_nxt;
    b ^= 1;
  }
  if (pend != 0u) {  // only after a wait ran out
    if (lane == 0 && err != nullptr) atomicExch(err, EDG_ERR_TIMEOUT);
    // copies still in flight land before the CTA leaves (bounded again)
    for (int s2 = 0; s2 < 2; ++s2)
      if (pend & (1u << s2)) {
        const uint64_t t0 = edg::bulk::now_ns();
        while (!edg::bulk::mbar_try_wait(&bar[s2], (phase >> s2) & 1u))
          if (edg::bulk::now_ns() - t0 > 1000000000ull) break;
      }
  }
}

template <typename T>
size_t packed_smem(int count) {
  return sizeof(uint32_t) * kWarps * 2 * kStageWords + sizeof(uint64_t) * kWarps * 2 + sizeof(T) * (size_t)count;
}

template <typename T>
int pack_collect(const T* vals, int64_t nnz, void* set, int log2_slots, int* overflow, cudaStream_t s) {
  pack_collect_k<T><<<edg::grid_for(nnz, 256), 256, 0, s>>>(vals, nnz, (typename Pat<T>::U*)set, log2_slots, 64,
                                                             overflow);
  return EDG_OK;
}

template <typename T>
int pack_encode(int64_t n, int64_t total, const int64_t* rowptr, const int32_t* cols, const T* vals, const T* table,
                int count, int colbits, const int64_t* offsets, int32_t* tile_off, uint32_t* words, int* missing,
                cudaStream_t s) {
  const int64_t n_tiles = (n + kTileRows - 1) / kTileRows;
  const unsigned grid = edg::grid_for(n_tiles * kTileRows + 4, 256);
  const size_t smem = sizeof(T) * (size_t)count;
  cudaFuncSetAttribute(pack_encode_k<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  pack_encode_k<T><<<grid, 256, smem, s>>>(n, total, rowptr, cols, vals, table, count, colbits, offsets, tile_off,
                                           words, missing);
  return EDG_OK;
}

}  // namespace

namespace edg {

template <typename T>
int launch_packed_spmv(int nvec, int x_stride, int64_t n, const int32_t* tile_off, const uint32_t* words,
                       const T* table, int count, int colbits, const T* diag, const T* x, double* y, int64_t y_plane,
                       const int* skip, int* err, cudaStream_t s, int diag_shared) {
  const int64_t n_tiles = (n + kTileRows - 1) / kTileRows;
  const int64_t need = (n_tiles + kWarps - 1) / kWarps;
  const unsigned grid = (unsigned)(need < (int64_t)kSmCount * 4 ? need : (int64_t)kSmCount * 4);
  const size_t smem = packed_smem<T>(count);
  cudaError_t e = cudaSuccess;
#define EDG_PACKED(NV, XS)                                                                                          \
  do {                                                                                                              \
    e = cudaFuncSetAttribute(packed_spmv_k<T, NV, XS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);    \
    if (e == cudaSuccess)                                                                                           \
      packed_spmv_k<T, NV, XS><<<grid, kWarps * 32, smem, s>>>(n, tile_off, words, table, count, colbits, diag, x, \
                                                               y, y_plane, diag_shared, skip, err);                 \
  } while (0)
  switch (nvec) {
    case 1: EDG_PACKED(1, 1); break;
    case 2: EDG_PACKED(2, 2); break;
    case 3:
      if (x_stride == 4)
        EDG_PACKED(3, 4);
      else
        EDG_PACKED(3, 3);
      break;
    case 4: EDG_PACKED(4, 4); break;
    default: set_error("packed spmv: nvec must be 1..4, got %d", nvec); return EDG_ERR_ARG;
  }
#undef EDG_PACKED
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "packed spmv");
  return EDG_OK;
}

template int launch_packed_spmv<float>(int, int, int64_t, const int32_t*, const uint32_t*, const float*, int, int,
                                       const float*, const float*, double*, int64_t, const int*, int*, cudaStream_t,
                                       int);
template int launch_packed_spmv<double>(int, int, int64_t, const int32_t*, const uint32_t*, const double*, int, int,
                                        const double*, const double*, double*, int64_t, const int*, int*,
                                        cudaStream_t, int);

}  // namespace edg

extern "C" int64_t edg_pack_tiles(int64_t n_rows) { return n_rows < 0 ? -1 : (n_rows + kTileRows - 1) / kTileRows; }

extern "C" int edg_pack_tile_counts(int64_t n_rows, const int64_t* rowptr, int64_t* counts, cudaStream_t stream) {
  EDG_REQUIRE(n_rows >= 0, "edg_pack_tile_counts: negative n_rows");
  EDG_REQUIRE(rowptr && counts, "edg_pack_tile_counts: null pointer");
  const int64_t n_tiles = (n_rows + kTileRows - 1) / kTileRows;
  if (n_tiles == 0) return EDG_OK;
  pack_counts_k<<<edg::grid_for(n_tiles, 256), 256, 0, stream>>>(n_rows, rowptr, counts);
  EDG_CHECK_LAUNCH("edg_pack_tile_counts");
  return EDG_OK;
}

extern "C" int edg_pack_collect(int32_t dtype, const void* vals, int64_t nnz, void* set, int32_t log2_slots,
                                int32_t* overflow, cudaStream_t stream) {
  EDG_REQUIRE(dtype == 0 || dtype == 1, "edg_pack_collect: dtype must be 0 (f64) or 1 (f32)");
  EDG_REQUIRE(nnz >= 0, "edg_pack_collect: negative nnz");
  EDG_REQUIRE(log2_slots >= 4 && log2_slots <= 20, "edg_pack_collect: log2_slots must be in [4, 20], got %d",
              log2_slots);
  EDG_REQUIRE(set && overflow && (nnz == 0 || vals), "edg_pack_collect: null pointer");
  if (nnz == 0) return EDG_OK;
  if (dtype == 1)
    pack_collect<float>((const float*)vals, nnz, set, log2_slots, overflow, stream);
  else
    pack_collect<double>((const double*)vals, nnz, set, log2_slots, overflow, stream);
  EDG_CHECK_LAUNCH("edg_pack_collect");
  return EDG_OK;
}

extern "C" int edg_pack_encode(int32_t dtype, int64_t n_rows, int64_t total, const int64_t* rowptr,
                               const int32_t* cols, const void* vals, const void* table, int32_t count,
                               int32_t colbits, const int64_t* offsets, int32_t* tile_off, uint32_t* words,
                               int32_t* missing, cudaStream_t stream) {
  EDG_REQUIRE(dtype == 0 || dtype == 1, "edg_pack_encode: dtype must be 0 (f64) or 1 (f32)");
  EDG_REQUIRE(n_rows > 0 && total >= 0 && total < INT32_MAX - 4, "edg_pack_encode: sizes out of range");
  EDG_REQUIRE(colbits >= 1 && colbits <= 31 && n_rows < ((int64_t)1 << colbits),
              "edg_pack_encode: colbits %d cannot hold %lld rows and the padding column", colbits,
              (long long)n_rows);
  EDG_REQUIRE(count >= 1 && count <= EDG_PACK_MAX_VALUES && ((int64_t)(count - 1) >> (32 - colbits)) == 0,
              "edg_pack_encode: %d values do not fit %d index bits (at most %d values)", count, 32 - colbits,
              EDG_PACK_MAX_VALUES);
  EDG_REQUIRE(rowptr && table && offsets && tile_off && words && missing && (total == 0 || (cols && vals)),
              "edg_pack_encode: null pointer");
  if (dtype == 1)
    pack_encode<float>(n_rows, total, rowptr, cols, (const float*)vals, (const float*)table, count, colbits, offsets,
                       tile_off, words, missing, stream);
  else
    pack_encode<double>(n_rows, total, rowptr, cols, (const double*)vals, (const double*)table, count, colbits,
                        offsets, tile_off, words, missing, stream);
  EDG_CHECK_LAUNCH("edg_pack_encode");
  return EDG_OK;
}

extern "C" int edg_spmv_packed(int32_t dtype, int64_t n_rows, int32_t nvec, const int32_t* tile_off,
                               const uint32_t* words, const void* table, int32_t count, int32_t colbits,
                               const void* diag, const void* x, int32_t x_stride, double* y, int64_t y_plane,
                               int32_t* err, cudaStream_t stream) {
  EDG_REQUIRE(dtype == 0 || dtype == 1, "edg_spmv_packed: dtype must be 0 (f64) or 1 (f32)");
  EDG_REQUIRE(n_rows >= 0 && nvec >= 1 && nvec <= 4, "edg_spmv_packed: bad size");
  EDG_REQUIRE(x_stride == nvec || (nvec == 3 && x_stride == 4), "edg_spmv_packed: x_stride must be nvec "
                                                                "(or 4 for nvec = 3)");
  EDG_REQUIRE(colbits >= 1 && colbits <= 31 && n_rows < ((int64_t)1 << colbits), "edg_spmv_packed: bad colbits");
  EDG_REQUIRE(count >= 1 && count <= EDG_PACK_MAX_VALUES, "edg_spmv_packed: bad table size %d", count);
  EDG_REQUIRE(tile_off && words && table && diag && x && y, "edg_spmv_packed: null pointer");
  if (n_rows == 0) return EDG_OK;
  const int64_t yp = y_plane > 0 ? y_plane : n_rows;
  if (dtype == 1)
    return edg::launch_packed_spmv<float>(nvec, x_stride, n_rows, tile_off, words, (const float*)table, count,
                                          colbits, (const float*)diag, (const float*)x, y, yp, nullptr, err, stream);
  return edg::launch_packed_spmv<double>(nvec, x_stride, n_rows, tile_off, words, (const double*)table, count,
                                         colbits, (const double*)diag, (const double*)x, y, yp, nullptr, err, stream);
}
