// Matrix-free Z_n lattice gauge theory with staggered fermions: zero-momentum
// basis construction and the batched matvec.
//
// Basis.  The Gauss-law sector is indexed densely (gidx = colex rank of the
// occupied-site set * zn^n_cot + cotree fields as base-zn digits), so a
// configuration is decoded from its index by peeling the spanning tree from
// the leaves (every tree field follows from the Gauss law at its child site)
// and encoded with two small tables (cotree digits per key byte, colex rank
// per occupation pattern).  The representatives of the translation orbits
// are marked in a bitmap over gidx (one thread per 64-bit word, no atomics),
// counted, scanned and written out in gidx order; then every orbit member's
// gidx gets, in a 4-byte orbit table, the row of its representative, the
// stabiliser size and the fermionic sign of the translation that maps the
// representative onto it.  This replaces the reference's translation table
// found by binary search and its projector B
// (edlgt/symmetries/translational_sym.py:567-819).
//
// Matvec.  One thread per representative row (persistent grid, lookup
// tables in shared memory): the diagonal from the key, then each hopping and
// plaquette image is encoded, looked up in the orbit table (one 4-byte
// load) and its x row gathered (nvec interleaved instances, one 32-byte
// sector for 8 f32 instances).  Element: amplitude * sign *
// sqrt(|Stab r'| / |Stab r|), the zero-momentum projection of
// nbody_data_momentum (translational_sym.py:1394-1969) done on the fly.
#include "internal.cuh"

namespace {

template <int ZN>
struct Zn {
  static constexpr int kBits = ZN == 2 ? 1 : 2;
  static constexpr uint64_t kMask = (1ull << kBits) - 1;
  __device__ static __forceinline__ int field(uint64_t key, int l) { return (int)((key >> (kBits * l)) & kMask); }
  __device__ static __forceinline__ uint64_t set(uint64_t key, int l, int v) {
    const int sh = kBits * l;
    return (key & ~(kMask << sh)) | ((uint64_t)v << sh);
  }
  __device__ static __forceinline__ int inc(int v) { return v + 1 == ZN ? 0 : v + 1; }
  __device__ static __forceinline__ int dec(int v) { return v == 0 ? ZN - 1 : v - 1; }
  __device__ static __forceinline__ int mod(int v) {
    v %= ZN;
    return v < 0 ? v + ZN : v;
  }
};

// Key of T(config): the lane array (one lane per row of sites) rotated by
// whole rows, then every lane rotated by whole sites; the same on the
// occupation bits.
__device__ __forceinline__ uint64_t translate_key(const edg_zn_translation& T, uint64_t key, int F, int N, int lane_f,
                                                  int lx) {
  const uint64_t fmask = (F == 64) ? ~0ull : ((1ull << F) - 1);
  const uint32_t mmask = (uint32_t)((1u << N) - 1);
  uint64_t f = key & fmask;
  uint32_t m = (uint32_t)(key >> F) & mmask;
  if (T.sf) f = ((f << T.sf) | (f >> (F - T.sf))) & fmask;
  if (T.sx) f = ((f << T.sx) & T.hif) | ((f >> (lane_f - T.sx)) & T.lof);
  if (T.sm) m = ((m << T.sm) | (m >> (N - T.sm))) & mmask;
  if (T.smx) m = ((m << T.smx) & T.him) | ((m >> (lx - T.smx)) & T.lom);
  return f | ((uint64_t)m << F);
}

// Parity (1 = negative) of the reordering T makes among occupied sites: rows
// that wrap in y pass every fermion of the rows that do not; inside a row the
// wrapping sites pass the staying ones.
__device__ __forceinline__ int translate_sign(const edg_zn_translation& T, uint32_t occ, int lx, int ly) {
  int par = (__popc(occ & T.ylow) & __popc(occ & T.yhigh)) & 1;
  if (T.smx) {
    for (int y = 0; y < ly; ++y) {
      const uint32_t row = occ >> (lx * y);
      par ^= (__popc(row & T.xhead) & __popc(row & T.xtail)) & 1;
    }
  }
  return par;
}

// Configuration of Gauss index g.
template <int ZN>
__device__ uint64_t decode(const edg_zn_lattice& L, uint64_t g) {
  using Z = Zn<ZN>;
  const uint64_t r = g / (uint64_t)L.pow_cot;
  uint32_t d = (uint32_t)(g - r * (uint64_t)L.pow_cot);
  const uint32_t occ = L.rank_occ[r];
  uint64_t key = (uint64_t)occ << L.field_bits;
  for (int c = 0; c < L.n_cot; ++c) {
    const uint32_t e = d % ZN;
    d /= ZN;
    key |= (uint64_t)e << (Z::kBits * L.cot_link[c]);
  }
  for (int k = 0; k < L.n_sites - 1; ++k) {
    const int v = L.peel_site[k];
    int s = (int)((occ >> v) & 1u) - (int)((L.odd_mask >> v) & 1u);
#pragma unroll
    for (int o = 0; o < 3; ++o) s -= L.peel_osign[k][o] * Z::field(key, L.peel_other[k][o]);
    key |= (uint64_t)Z::mod(L.peel_sign[k] * s) << (Z::kBits * L.peel_link[k]);
  }
  return key;
}

__device__ __forceinline__ int lane_bits(const edg_zn_lattice& L) { return 2 * L.link_bits * L.lx; }

// True when key is the smallest key of its orbit and no stabiliser element
// maps it onto minus itself.
__device__ bool is_rep(const edg_zn_lattice& L, uint64_t key) {
  const uint32_t occ = (uint32_t)(key >> L.field_bits);
  const int lf = lane_bits(L);
  for (int g = 1; g < L.n_group; ++g) {
    const uint64_t k2 = translate_key(L.group[g], key, L.field_bits, L.n_sites, lf, L.lx);
    if (k2 < key) return false;
    if (k2 == key && translate_sign(L.group[g], occ, L.lx, L.ly)) return false;
  }
  return true;
}

template <int ZN>
__global__ void __launch_bounds__(256) zn_mark_k(const __grid_constant__ edg_zn_lattice L, uint64_t* __restrict__ bitmap,
                                                 int64_t* __restrict__ counts, int64_t n_words) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_words; w += (int64_t)gridDim.x * blockDim.x) {
    uint64_t bits = 0;
    const uint64_t g0 = (uint64_t)w * 64;
    for (int j = 0; j < 64; ++j) {
      const uint64_t g = g0 + j;
      if (g >= (uint64_t)L.n_gauss) break;
      if (is_rep(L, decode<ZN>(L, g))) bits |= 1ull << j;
    }
    bitmap[w] = bits;
    counts[w] = __popcll(bits);
  }
}

template <int ZN>
__global__ void __launch_bounds__(256) zn_fill_k(const __grid_constant__ edg_zn_lattice L, const uint64_t* __restrict__ bitmap,
                                                 const int64_t* __restrict__ offsets, uint64_t* __restrict__ keys,
                                                 int64_t n_words) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_words; w += (int64_t)gridDim.x * blockDim.x) {
    uint64_t bits = bitmap[w];
    int64_t o = offsets[w];
    while (bits) {
      const int j = __ffsll((long long)bits) - 1;
      bits &= bits - 1;
      keys[o++] = decode<ZN>(L, (uint64_t)w * 64 + j);
    }
  }
}

// Gauss index from the two lookup tables (held in shared memory by the callers).
__device__ __forceinline__ uint64_t gauss_index(const uint64_t* __restrict__ lut, const uint32_t* __restrict__ rank,
                                                uint64_t key, int F, int n_chunks, uint64_t pow_cot) {
  uint64_t g = (uint64_t)rank[(uint32_t)(key >> F)] * pow_cot;
  for (int k = 0; k < n_chunks; ++k) g += lut[k * 256 + (int)((key >> (8 * k)) & 255u)];
  return g;
}

__device__ void load_tables(const edg_zn_lattice& L, uint64_t* lut, uint32_t* rank) {
  const int n_chunks = (L.field_bits + 7) / 8;
  for (int i = threadIdx.x; i < n_chunks * 256; i += blockDim.x) lut[i] = L.chunk_lut[i];
  for (int i = threadIdx.x; i < (1 << L.n_sites); i += blockDim.x) rank[i] = L.occ_rank[i];
  __syncthreads();
}

__global__ void __launch_bounds__(256) zn_orbit_k(const __grid_constant__ edg_zn_lattice L, const uint64_t* __restrict__ keys, int64_t n_rows,
                                                  uint32_t* __restrict__ orbit) {
  extern __shared__ uint64_t zsm[];
  const int n_chunks = (L.field_bits + 7) / 8;
  uint64_t* lut = zsm;
  uint32_t* rank = (uint32_t*)(zsm + n_chunks * 256);
  load_tables(L, lut, rank);
  const int lf = lane_bits(L);
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t key = keys[r];
    const uint32_t occ = (uint32_t)(key >> L.field_bits);
    int stab = 0;
    for (int g = 0; g < L.n_group; ++g)
      stab += translate_key(L.group[g], key, L.field_bits, L.n_sites, lf, L.lx) == key;
    int dv = 0;
    while (dv < L.n_div - 1 && L.divisors[dv] != stab) ++dv;
    const uint32_t base = (uint32_t)r | ((uint32_t)dv << 28);
    for (int g = 0; g < L.n_group; ++g) {
      const uint64_t k2 = translate_key(L.group[g], key, L.field_bits, L.n_sites, lf, L.lx);
      const uint32_t sg = (uint32_t)translate_sign(L.group[g], occ, L.lx, L.ly);
      orbit[gauss_index(lut, rank, k2, L.field_bits, n_chunks, (uint64_t)L.pow_cot)] = base | (sg << 31);
    }
  }
}

// ---------------------------------------------------------------- matvec
// One x row (the nvec interleaved instances of a column) in 16-byte loads.
template <typename T, int NV>
__device__ __forceinline__ void load_row(const T* __restrict__ p, T (&v)[NV]) {
  if constexpr (NV * sizeof(T) >= 16) {
    constexpr int kVec = 16 / sizeof(T);
#pragma unroll
    for (int i = 0; i < NV / kVec; ++i) {
      if constexpr (sizeof(T) == 4) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p) + i);
        v[4 * i] = a.x; v[4 * i + 1] = a.y; v[4 * i + 2] = a.z; v[4 * i + 3] = a.w;
      } else {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p) + i);
        v[2 * i] = a.x; v[2 * i + 1] = a.y;
      }
    }
  } else {
#pragma unroll
    for (int i = 0; i < NV; ++i) v[i] = __ldg(p + i);
  }
}

constexpr int kMvThreads = 256;

// Images whose loads are in flight together: four for f32 rows, two for f64
// rows (register budget).
template <typename T>
constexpr int group_of() { return sizeof(T) == 4 ? 4 : 2; }

// Images are handled a group at a time (G links, or G/2 plaquettes in both
// directions): the G orbit-table loads are issued together, then the G x-row
// loads, then the arithmetic, so that each thread keeps several independent
// gathers in flight instead of one dependent pair per image.
template <int ZN, typename T, int NV>
__global__ void __launch_bounds__(kMvThreads, 2) zn_matvec_k(const __grid_constant__ edg_zn_lattice L, const edg_zn_basis B,
                                                          const double* __restrict__ coup, const T* __restrict__ x,
                                                          T* __restrict__ y) {
  using Z = Zn<ZN>;
  constexpr int kGroup = group_of<T>();
  extern __shared__ uint64_t zsm[];
  __shared__ double c_t[NV], c_m[NV], c_e[NV], c_b[NV];
  __shared__ double sq_div[8], isq_div[8];
  const int n_chunks = (L.field_bits + 7) / 8;
  uint64_t* lut = zsm;
  uint32_t* rank = (uint32_t*)(zsm + n_chunks * 256);
  if (threadIdx.x < NV) {
    c_t[threadIdx.x] = -coup[4 * threadIdx.x + 0];
    c_m[threadIdx.x] = coup[4 * threadIdx.x + 1];
    c_e[threadIdx.x] = coup[4 * threadIdx.x + 2];
    c_b[threadIdx.x] = coup[4 * threadIdx.x + 3];
  }
  if (threadIdx.x < 8) {
    const double d = threadIdx.x < L.n_div ? (double)L.divisors[threadIdx.x] : 1.0;
    sq_div[threadIdx.x] = sqrt(d);
    isq_div[threadIdx.x] = 1.0 / sqrt(d);
  }
  load_tables(L, lut, rank);
  const int F = L.field_bits;
  const uint64_t pc = (uint64_t)L.pow_cot;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < B.n_rows; r += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t key = B.keys[r];
    const uint32_t occ = (uint32_t)(key >> F);
    const uint32_t self = B.orbit[gauss_index(lut, rank, key, F, n_chunks, pc)];
    const double inv_s = isq_div[(self >> 28) & 7u];
    double ah[NV], ap[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) ah[v] = ap[v] = 0.0;
    // hopping: c^dag_tail U c_head (tail empty, head full) and its conjugate;
    // links in groups (n_links = 2 * n_sites is a multiple of four)
    for (int l0 = 0; l0 < L.n_links; l0 += kGroup) {
      uint32_t e[kGroup];
      int neg[kGroup];
#pragma unroll
      for (int c = 0; c < kGroup; ++c) {
        const int l = l0 + c;
        const int ta = L.link_tail[l], he = L.link_head[l];
        const uint32_t nt = (occ >> ta) & 1u, nh = (occ >> he) & 1u;
        e[c] = 0xFFFFFFFFu;
        neg[c] = (int)(__popc(occ & L.link_between[l]) & 1) ^ (L.link_eta[l] < 0);
        if (nt != nh) {
          const int f = Z::field(key, l);
          uint64_t k2 = Z::set(key, l, nt == 0 ? Z::inc(f) : Z::dec(f));
          k2 ^= ((1ull << ta) | (1ull << he)) << F;
          e[c] = B.orbit[gauss_index(lut, rank, k2, F, n_chunks, pc)];
        }
      }
      T xv[kGroup][NV];
#pragma unroll
      for (int c = 0; c < kGroup; ++c)
        if (e[c] != 0xFFFFFFFFu) load_row<T, NV>(x + (int64_t)(e[c] & 0x0FFFFFFFu) * NV, xv[c]);
#pragma unroll
      for (int c = 0; c < kGroup; ++c)
        if (e[c] != 0xFFFFFFFFu) {
          const double s = sq_div[(e[c] >> 28) & 7u] * inv_s;
          const double a = (neg[c] ^ (int)(e[c] >> 31)) ? -s : s;
#pragma unroll
          for (int v = 0; v < NV; ++v) ah[v] = fma(a, (double)xv[c][v], ah[v]);
        }
    }
    // plaquettes U_p and U_p^dag, kGroup / 2 plaquettes per group
    for (int p0 = 0; p0 < L.n_sites; p0 += kGroup / 2) {
      uint32_t e[kGroup];
#pragma unroll
      for (int c = 0; c < kGroup; ++c) {
        const int p = p0 + c / 2, dir = c & 1;
        const int l0 = L.plaq[p][0], l1 = L.plaq[p][1], l2 = L.plaq[p][2], l3 = L.plaq[p][3];
        uint64_t k2 = key;
        k2 = Z::set(k2, l0, dir == 0 ? Z::inc(Z::field(key, l0)) : Z::dec(Z::field(key, l0)));
        k2 = Z::set(k2, l1, dir == 0 ? Z::inc(Z::field(key, l1)) : Z::dec(Z::field(key, l1)));
        k2 = Z::set(k2, l2, dir == 0 ? Z::dec(Z::field(key, l2)) : Z::inc(Z::field(key, l2)));
        k2 = Z::set(k2, l3, dir == 0 ? Z::dec(Z::field(key, l3)) : Z::inc(Z::field(key, l3)));
        e[c] = B.orbit[gauss_index(lut, rank, k2, F, n_chunks, pc)];
      }
      T xv[kGroup][NV];
#pragma unroll
      for (int c = 0; c < kGroup; ++c)
        if (e[c] != 0xFFFFFFFFu) load_row<T, NV>(x + (int64_t)(e[c] & 0x0FFFFFFFu) * NV, xv[c]);
#pragma unroll
      for (int c = 0; c < kGroup; ++c)
        if (e[c] != 0xFFFFFFFFu) {
          const double s = sq_div[(e[c] >> 28) & 7u] * inv_s;
          const double a = (e[c] >> 31) ? -s : s;
#pragma unroll
          for (int v = 0; v < NV; ++v) ap[v] = fma(a, (double)xv[c][v], ap[v]);
        }
    }
    double esq = 0.0;
    for (int l = 0; l < L.n_links; ++l) esq += L.esq[Z::field(key, l)];
    const double mass = (double)(__popc(occ & L.even_mask) - __popc(occ & ~L.even_mask));
    T xr[NV];
    load_row<T, NV>(x + r * NV, xr);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double d = c_e[v] * esq + c_m[v] * mass;
      y[r * NV + v] = (T)(fma(d, (double)xr[v], fma(c_t[v], ah[v], c_b[v] * ap[v])));
    }
  }
}

int check_lattice(const edg_zn_lattice* L, const char* where) {
  EDG_REQUIRE(L != nullptr, "%s: null lattice", where);
  EDG_REQUIRE(L->zn >= 2 && L->zn <= 4, "%s: zn must be 2, 3 or 4", where);
  EDG_REQUIRE(L->link_bits == (L->zn == 2 ? 1 : 2), "%s: link_bits must be %d", where, L->zn == 2 ? 1 : 2);
  EDG_REQUIRE(L->n_sites >= 4 && L->n_sites <= EDG_ZN_MAX_SITES && L->n_sites == L->lx * L->ly,
              "%s: need 4 <= lx * ly <= %d", where, EDG_ZN_MAX_SITES);
  EDG_REQUIRE(L->lx % 2 == 0 && L->ly >= 2, "%s: need lx even and ly >= 2", where);
  EDG_REQUIRE(L->n_links == 2 * L->n_sites && L->field_bits == L->link_bits * L->n_links &&
                  L->field_bits + L->n_sites <= 64,
              "%s: inconsistent link/field sizes", where);
  EDG_REQUIRE(L->n_group >= 1 && L->n_group <= EDG_ZN_MAX_GROUP, "%s: n_group must be 1..%d", where, EDG_ZN_MAX_GROUP);
  EDG_REQUIRE(L->n_div >= 1 && L->n_div <= 8, "%s: n_div must be 1..8", where);
  EDG_REQUIRE(L->n_gauss > 0 && L->n_gauss <= 0xFFFFFFFFll, "%s: Gauss index range must fit 32 bits", where);
  EDG_REQUIRE(L->pow_cot > 0 && L->pow_cot <= 0xFFFFFFFFll && L->n_gauss % L->pow_cot == 0,
              "%s: bad pow_cot", where);
  EDG_REQUIRE(L->n_cot == L->n_links - L->n_sites + 1, "%s: n_cot must be links - sites + 1", where);
  EDG_REQUIRE(L->chunk_lut != nullptr && L->occ_rank != nullptr && L->rank_occ != nullptr,
              "%s: null lookup table", where);
  return EDG_OK;
}

size_t table_smem(const edg_zn_lattice* L) {
  return sizeof(uint64_t) * 256 * (size_t)((L->field_bits + 7) / 8) + sizeof(uint32_t) * ((size_t)1 << L->n_sites);
}

template <typename K>
int set_smem(K kernel, size_t smem, const char* where) {
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return edg::cuda_status(e, where);
  }
  return EDG_OK;
}

// Persistent grid: resident CTAs per SM times the SM count.
template <typename K>
unsigned persistent_grid(K kernel, int threads, size_t smem, int64_t n_items) {
  int per_sm = 1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  return edg::grid_for(n_items, threads, per_sm);
}

template <int ZN, typename T, int NV>
int launch_matvec(const edg_zn_lattice* L, const edg_zn_basis* B, const double* coup, const void* x, void* y,
                  cudaStream_t stream) {
  const size_t smem = table_smem(L);
  auto kern = zn_matvec_k<ZN, T, NV>;
  int st = set_smem(kern, smem, "edg_zn_matvec");
  if (st != EDG_OK) return st;
  const unsigned grid = persistent_grid(kern, kMvThreads, smem, B->n_rows);
  kern<<<grid, kMvThreads, smem, stream>>>(*L, *B, coup, (const T*)x, (T*)y);
  EDG_CHECK_LAUNCH("edg_zn_matvec");
  return EDG_OK;
}

template <int ZN>
int dispatch_matvec(const edg_zn_lattice* L, const edg_zn_basis* B, const double* coup, int nvec, int dtype,
                    const void* x, void* y, cudaStream_t s) {
#define EDG_ZN_MV(NV)                                                           \
  case NV:                                                                      \
    return dtype == 0 ? launch_matvec<ZN, double, NV>(L, B, coup, x, y, s)      \
                      : launch_matvec<ZN, float, NV>(L, B, coup, x, y, s);
  switch (nvec) {
    EDG_ZN_MV(1)
    EDG_ZN_MV(2)
    EDG_ZN_MV(4)
    EDG_ZN_MV(8)
  }
#undef EDG_ZN_MV
  edg::set_error("edg_zn_matvec: nvec must be 1, 2, 4 or 8");
  return EDG_ERR_ARG;
}

}  // namespace

extern "C" int64_t edg_zn_bitmap_words(const edg_zn_lattice* L) {
  if (L == nullptr || L->n_gauss <= 0) return -1;
  return (L->n_gauss + 63) / 64;
}

extern "C" int edg_zn_mark(const edg_zn_lattice* L, uint64_t* bitmap, int64_t* counts, cudaStream_t stream) {
  int st = check_lattice(L, "edg_zn_mark");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(bitmap != nullptr && counts != nullptr, "edg_zn_mark: null output");
  const int64_t words = (L->n_gauss + 63) / 64;
  const unsigned grid = edg::grid_for(words, 256);
  switch (L->zn) {
    case 2: zn_mark_k<2><<<grid, 256, 0, stream>>>(*L, bitmap, counts, words); break;
    case 3: zn_mark_k<3><<<grid, 256, 0, stream>>>(*L, bitmap, counts, words); break;
    default: zn_mark_k<4><<<grid, 256, 0, stream>>>(*L, bitmap, counts, words); break;
  }
  EDG_CHECK_LAUNCH("edg_zn_mark");
  return EDG_OK;
}

extern "C" int edg_zn_fill(const edg_zn_lattice* L, const uint64_t* bitmap, const int64_t* offsets, uint64_t* keys,
                           cudaStream_t stream) {
  int st = check_lattice(L, "edg_zn_fill");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(bitmap != nullptr && offsets != nullptr && keys != nullptr, "edg_zn_fill: null argument");
  const int64_t words = (L->n_gauss + 63) / 64;
  const unsigned grid = edg::grid_for(words, 256);
  switch (L->zn) {
    case 2: zn_fill_k<2><<<grid, 256, 0, stream>>>(*L, bitmap, offsets, keys, words); break;
    case 3: zn_fill_k<3><<<grid, 256, 0, stream>>>(*L, bitmap, offsets, keys, words); break;
    default: zn_fill_k<4><<<grid, 256, 0, stream>>>(*L, bitmap, offsets, keys, words); break;
  }
  EDG_CHECK_LAUNCH("edg_zn_fill");
  return EDG_OK;
}

extern "C" int edg_zn_orbit_table(const edg_zn_lattice* L, const uint64_t* keys, int64_t n_rows, uint32_t* orbit,
                                  cudaStream_t stream) {
  int st = check_lattice(L, "edg_zn_orbit_table");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(keys != nullptr && orbit != nullptr, "edg_zn_orbit_table: null argument");
  EDG_REQUIRE(n_rows >= 0 && n_rows < 0x0FFFFFFFll, "edg_zn_orbit_table: n_rows must be below 2^28 - 1");
  cudaError_t e = cudaMemsetAsync(orbit, 0xFF, sizeof(uint32_t) * (size_t)L->n_gauss, stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_zn_orbit_table: memset");
  if (n_rows == 0) return EDG_OK;
  const size_t smem = table_smem(L);
  st = set_smem(zn_orbit_k, smem, "edg_zn_orbit_table");
  if (st != EDG_OK) return st;
  const unsigned grid = persistent_grid(zn_orbit_k, 256, smem, n_rows);
  zn_orbit_k<<<grid, 256, smem, stream>>>(*L, keys, n_rows, orbit);
  EDG_CHECK_LAUNCH("edg_zn_orbit_table");
  return EDG_OK;
}

extern "C" int edg_zn_matvec(const edg_zn_lattice* L, const edg_zn_basis* B, const double* couplings, int32_t nvec,
                             int32_t dtype, const void* x, void* y, cudaStream_t stream) {
  int st = check_lattice(L, "edg_zn_matvec");
  if (st != EDG_OK) return st;
  EDG_REQUIRE(B != nullptr && couplings != nullptr && x != nullptr && y != nullptr, "edg_zn_matvec: null argument");
  EDG_REQUIRE(dtype == 0 || dtype == 1, "edg_zn_matvec: dtype must be 0 (f64) or 1 (f32)");
  EDG_REQUIRE(B->n_rows >= 0 && B->n_rows < 0x0FFFFFFFll, "edg_zn_matvec: n_rows must be below 2^28 - 1");
  EDG_REQUIRE(B->keys != nullptr && B->orbit != nullptr, "edg_zn_matvec: null basis arrays");
  EDG_REQUIRE(((uintptr_t)x & 15u) == 0, "edg_zn_matvec: x must be 16-byte aligned");
  if (B->n_rows == 0) return EDG_OK;
  switch (L->zn) {
    case 2: return dispatch_matvec<2>(L, B, couplings, nvec, dtype, x, y, stream);
    case 3: return dispatch_matvec<3>(L, B, couplings, nvec, dtype, x, y, stream);
    default: return dispatch_matvec<4>(L, B, couplings, nvec, dtype, x, y, stream);
  }
}
