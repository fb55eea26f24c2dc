// Two-body correlators: corr[i][j] = corr[j][i] = Re <psi| A_i B_j |psi> for
// a list of site pairs i < j, in a symmetry sector.  This is
// TwoBodyTerm.get_expval with lattice_twobody_exp_val
// (edlgt/modeling/twobody_term.py:160-264): for each pair the reference
// rebuilds the two-site triplets (nbody_data_2sites,
// edlgt/symmetries/sym_qmb_operations.py:490-562) and contracts them with psi
// (exp_val_data, edlgt/modeling/qmb_state.py:631-654).
//
// Here no triplet is stored and the sector is read once for all pairs.  A warp
// takes 32 rows at a time: each lane loads one row's key and amplitude and
// decodes the key into its local states (one mixed-radix division chain per
// row, staged in shared memory).  The warp then walks the 32 rows together,
// every lane owning up to kPairsPerLane pairs of the current pair tile: it
// applies the nonzero transitions of A at site i and B at site j from the
// local-state tables, finds the ket (the row itself when both transitions are
// diagonal, the bucketed key search otherwise) and accumulates
// conj(psi_row) * a * b * psi_ket in f64 registers.  Blocks reduce their warps
// per pair in shared memory; a second kernel sums the block partials in a
// fixed order, so results do not depend on scheduling.
#include "internal.cuh"
#include "lookup.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kPairsPerLane = 4;
constexpr int kTilePairs = 32 * kPairsPerLane;
constexpr int kBlocks = edg::kSmCount * 3;
constexpr int kTableSmemCap = 24 * 1024;  // transition tables larger than this stay in global memory

template <int PT>
__device__ __forceinline__ double2 load_psi(const void* psi, int64_t r, int64_t stride) {
  if (PT == 0) return make_double2(((const double*)psi)[r * stride], 0.0);
  if (PT == 1) return make_double2((double)((const float*)psi)[r * stride], 0.0);
  if (PT == 2) return ((const double2*)psi)[r * stride];
  const float2 a = ((const float2*)psi)[r * stride];
  return make_double2((double)a.x, (double)a.y);
}

struct Args {
  edg_lookup_table sec;
  const uint64_t* strides;
  const int32_t* loc_dims;
  const int32_t* count;  // [2][n_sites][dmax]
  const uint8_t* ket;    // [2][n_sites][dmax][dmax]
  const double2* amp;    // [2][n_sites][dmax][dmax]
  const int32_t* pair_i;
  const int32_t* pair_j;
  const void* psi;
  int64_t psi_stride;
  double* partial;  // [kBlocks][n_pairs][2]
  int32_t* err;
  int n_sites, dmax, n_pairs;
  int tables_in_smem, diag_in_smem;
};

// Shared memory, in this order: the transition tables [amp | diagonal values
// | count | ket] when they fit (kTableSmemCap); the real diagonal table when
// it fits (kDiagCap entries); the local dimensions with their multiply-high
// reciprocals; the row staging (keys, amplitudes, local states); the per-warp
// pair partials.  In the transition tables a count carries kDiagBit when its
// bra state has exactly one transition, to itself, and the diagonal values
// hold that element.  The real diagonal table is stored local state major,
// [b][operator * n_sites + site] with a row pitch rounded to 16 doubles: the
// lanes of a warp read one row's values at different sites, which then fall
// in different banks whatever the local states are.
constexpr int kDiagBit = 1 << 16;
constexpr int kDiagCap = 2048;
__host__ __device__ inline int64_t round16(int64_t b) { return (b + 15) / 16 * 16; }
__host__ __device__ inline int diag_pitch(int n_sites) { return (2 * n_sites + 15) / 16 * 16; }
__host__ __device__ inline int64_t table_bytes(int n_sites, int dmax) {
  const int64_t e = 2LL * n_sites * dmax;
  return e * dmax * 16 + e * 16 + e * 4 + e * dmax;
}
struct Layout {
  int64_t tables, diag, aux, staging, red, total;
};
__host__ __device__ inline Layout layout(int ns, int dm, int tables_in_smem, int diag_in_smem) {
  Layout l;
  int64_t off = 0;
  l.tables = off;
  off += tables_in_smem ? round16(table_bytes(ns, dm)) : 0;
  l.diag = off;
  off += diag_in_smem ? (int64_t)dm * diag_pitch(ns) * 8 : 0;
  l.aux = off;
  off += round16((int64_t)ns * 12);
  l.staging = off;
  off += (int64_t)kWarps * 32 * (8 + 16) + round16((int64_t)kWarps * 32 * ns);
  l.red = off;
  off += (int64_t)kWarps * kTilePairs * 16;
  l.total = off;
  return l;
}

template <int PT>
__global__ void __launch_bounds__(kThreads, 3) twobody_k(const Args a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int ns = a.n_sites, dm = a.dmax;
  const int e = 2 * ns * dm;  // table entries (operator, site, bra state)
  const Layout L = layout(ns, dm, a.tables_in_smem, a.diag_in_smem);
  double2* s_amp = reinterpret_cast<double2*>(smem + L.tables);
  double2* s_dv = s_amp + (int64_t)e * dm;
  int32_t* s_count = reinterpret_cast<int32_t*>(s_dv + e);
  uint8_t* s_ket = reinterpret_cast<uint8_t*>(s_count + e);
  double* s_dre = reinterpret_cast<double*>(smem + L.diag);
  uint64_t* s_magic = reinterpret_cast<uint64_t*>(smem + L.aux);
  uint32_t* s_ld = reinterpret_cast<uint32_t*>(s_magic + ns);
  uint64_t* s_key = reinterpret_cast<uint64_t*>(smem + L.staging);
  double2* s_psi = reinterpret_cast<double2*>(s_key + kWarps * 32);
  uint8_t* s_dig = reinterpret_cast<uint8_t*>(s_psi + kWarps * 32);
  double2* s_red = reinterpret_cast<double2*>(smem + L.red);

  // local dimensions and ceil(2^64 / d): floor(x / d) = umulhi(x, that) for
  // every x < 2^32 (Lemire, Kaser, Kurz, "Faster remainder by direct
  // computation", 2019, theorem 1 with N = 32, F = 64)
  for (int s = threadIdx.x; s < ns; s += kThreads) {
    uint32_t d = (uint32_t)a.loc_dims[s];
    if (d < 1) {
      atomicExch(a.err, 1);
      d = 1;
    }
    s_ld[s] = d;
    s_magic[s] = d > 1 ? ~0ull / d + 1 : 0;
  }
  const double2* amp = a.amp;
  const int32_t* count = a.count;
  const uint8_t* ket = a.ket;
  if (a.tables_in_smem) {
    for (int k = threadIdx.x; k < e * dm; k += kThreads) {
      s_amp[k] = a.amp[k];
      s_ket[k] = a.ket[k];
    }
    for (int k = threadIdx.x; k < e; k += kThreads) {
      const int c = a.count[k];
      const bool diag = c == 1 && a.ket[k * dm] == k % dm;
      s_count[k] = c | (diag ? kDiagBit : 0);
      s_dv[k] = diag ? a.amp[k * dm] : make_double2(0.0, 0.0);
    }
    amp = s_amp;
    count = s_count;
    ket = s_ket;
  }
  // both operators diagonal and real on every local state: the block takes
  // the real diagonal path, <psi| A_i B_j |psi> = sum_r |psi_r|^2 a_i(r) b_j(r)
  const int pitch = diag_pitch(ns);
  int real_diag = a.diag_in_smem;
  if (a.diag_in_smem) {
    for (int k = threadIdx.x; k < e; k += kThreads) {
      const int c = a.count[k];
      const double2 v = c > 0 ? a.amp[k * dm] : make_double2(0.0, 0.0);
      real_diag &= c == 0 || (c == 1 && a.ket[k * dm] == k % dm && v.y == 0.0);
      s_dre[(k % dm) * pitch + k / dm] = v.x;  // k / dm = operator * n_sites + site
    }
  }
  const bool fast = __syncthreads_and(real_diag) != 0;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t n = a.sec.n;
  const int64_t n_groups = (n + 31) / 32;
  const int64_t gwarp = (int64_t)blockIdx.x * kWarps + warp, nwarps = (int64_t)gridDim.x * kWarps;
  uint64_t* wkey = s_key + warp * 32;
  double2* wpsi = s_psi + warp * 32;
  uint8_t* wdig = s_dig + warp * 32 * ns;

  for (int tile = 0; tile < a.n_pairs; tile += kTilePairs) {
    int si[kPairsPerLane], sj[kPairsPerLane];
    bool live[kPairsPerLane];
    double acc_re[kPairsPerLane], acc_im[kPairsPerLane];
#pragma unroll
    for (int k = 0; k < kPairsPerLane; ++k) {
      const int p = tile + lane + 32 * k;
      const int pi = p < a.n_pairs ? a.pair_i[p] : 0, pj = p < a.n_pairs ? a.pair_j[p] : 0;
      const bool ok = pi >= 0 && pj >= 0 && pi < ns && pj < ns && pi != pj;
      if (p < a.n_pairs && !ok && blockIdx.x == 0) atomicExch(a.err, 2);
      live[k] = p < a.n_pairs && ok;
      si[k] = live[k] ? pi : 0;
      sj[k] = live[k] ? pj : 1;
      acc_re[k] = 0.0;
      acc_im[k] = 0.0;
    }
    for (int64_t g = gwarp; g < n_groups; g += nwarps) {
      const int64_t r0 = g * 32;
      const int rows = n - r0 < 32 ? (int)(n - r0) : 32;
      if (lane < rows) {
        uint64_t x = __ldg(a.sec.keys + r0 + lane);
        wkey[lane] = x;
        wpsi[lane] = load_psi<PT>(a.psi, r0 + lane, a.psi_stride);
        for (int s = ns - 1; s >= 0; --s) {  // last site fastest
          const uint32_t d = s_ld[s];
          const uint64_t q = (x >> 32) ? x / d : (d > 1 ? __umul64hi(s_magic[s], x) : x);
          uint32_t c = (uint32_t)(x - q * d);
          if (c >= (uint32_t)dm) {  // a local state beyond the operators' dimension
            atomicExch(a.err, 1);
            c = 0;
          }
          wdig[lane * ns + s] = (uint8_t)c;
          x = q;
        }
      }
      __syncwarp();
      if (fast) {
        for (int t = 0; t < rows; ++t) {
          const double2 pr = wpsi[t];
          const double w = fma(pr.x, pr.x, pr.y * pr.y);
          const uint8_t* drow = wdig + t * ns;
#pragma unroll
          for (int k = 0; k < kPairsPerLane; ++k) {
            const double va = s_dre[drow[si[k]] * pitch + si[k]];
            const double vb = s_dre[drow[sj[k]] * pitch + ns + sj[k]];
            acc_re[k] = fma(va * w, vb, acc_re[k]);
          }
        }
      } else {
        for (int t = 0; t < rows; ++t) {
          const uint64_t key = wkey[t];
          const double2 pr = wpsi[t];
          const double w = fma(pr.x, pr.x, pr.y * pr.y);
          const uint8_t* drow = wdig + t * ns;
#pragma unroll
          for (int k = 0; k < kPairsPerLane; ++k) {
            if (!live[k]) continue;
            const int ci = drow[si[k]], cj = drow[sj[k]];
            const int ea = si[k] * dm + ci, eb = (ns + sj[k]) * dm + cj;
            const int na = count[ea], nb = count[eb];
            if (na & nb & kDiagBit) {  // both diagonal here: <r| a b |r> |psi_r|^2
              const double2 av = s_dv[ea], bv = s_dv[eb];
              acc_re[k] = fma(w, av.x * bv.x - av.y * bv.y, acc_re[k]);
              acc_im[k] = fma(w, av.x * bv.y + av.y * bv.x, acc_im[k]);
              continue;
            }
            const int ca = na & (kDiagBit - 1), cb = nb & (kDiagBit - 1);
            for (int ta = 0; ta < ca; ++ta) {
              const int ia = ea * dm + ta;
              const int ka = ket[ia];
              const double2 av = amp[ia];
              for (int tbi = 0; tbi < cb; ++tbi) {
                const int ib = eb * dm + tbi;
                const int kb = ket[ib];
                const double2 bv = amp[ib];
                double2 pc;
                if (ka == ci && kb == cj) {
                  pc = pr;  // both factors diagonal: the ket is this row
                } else {
                  // a padded local state (beyond the site's dimension) is no configuration
                  const bool inside = (uint32_t)ka < s_ld[si[k]] && (uint32_t)kb < s_ld[sj[k]];
                  const uint64_t q = key + ((uint64_t)ka - (uint64_t)ci) * __ldg(a.strides + si[k]) +
                                     ((uint64_t)kb - (uint64_t)cj) * __ldg(a.strides + sj[k]);
                  const int64_t col = inside ? edg::find_key(a.sec, q) : -1;
                  if (col < 0) {
                    atomicExch(a.err, 1);
                    continue;
                  }
                  pc = load_psi<PT>(a.psi, col, a.psi_stride);
                }
                // acc += conj(pr) * (a * b) * pc
                const double vr = av.x * bv.x - av.y * bv.y, vi = av.x * bv.y + av.y * bv.x;
                const double tr = vr * pc.x - vi * pc.y, ti = vr * pc.y + vi * pc.x;
                acc_re[k] = fma(pr.x, tr, fma(pr.y, ti, acc_re[k]));
                acc_im[k] = fma(pr.x, ti, fma(-pr.y, tr, acc_im[k]));
              }
            }
          }
        }
      }
      __syncwarp();
    }
    // block partial per pair of the tile, warps summed in a fixed order
#pragma unroll
    for (int k = 0; k < kPairsPerLane; ++k) s_red[warp * kTilePairs + lane + 32 * k] = make_double2(acc_re[k], acc_im[k]);
    __syncthreads();
    for (int q = threadIdx.x; q < kTilePairs; q += kThreads) {
      const int p = tile + q;
      if (p < a.n_pairs) {
        double re = 0.0, im = 0.0;
        for (int w = 0; w < kWarps; ++w) {
          re += s_red[w * kTilePairs + q].x;
          im += s_red[w * kTilePairs + q].y;
        }
        a.partial[((int64_t)blockIdx.x * a.n_pairs + p) * 2] = re;
        a.partial[((int64_t)blockIdx.x * a.n_pairs + p) * 2 + 1] = im;
      }
    }
    __syncthreads();
  }
}

// corr[i][j] = corr[j][i] = Re sum_b partial[b][p]; one warp per pair, the
// lanes' strided sums combined by a fixed butterfly.
__global__ void twobody_reduce_k(const double* __restrict__ partial, int nblk, int n_pairs,
                                 const int32_t* __restrict__ pair_i, const int32_t* __restrict__ pair_j, int n_sites,
                                 double* __restrict__ corr) {
  const int p = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= n_pairs) return;
  double s = 0.0;
  for (int b = lane; b < nblk; b += 32) s += partial[((int64_t)b * n_pairs + p) * 2];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  const int pi = pair_i[p], pj = pair_j[p];
  if (lane == 0 && pi >= 0 && pj >= 0 && pi < n_sites && pj < n_sites) {
    corr[(int64_t)pi * n_sites + pj] = s;
    corr[(int64_t)pj * n_sites + pi] = s;
  }
}

template <int PT>
cudaError_t launch(const Args& a, int64_t smem, cudaStream_t stream) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(twobody_k<PT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  twobody_k<PT><<<kBlocks, kThreads, (size_t)smem, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

extern "C" int64_t edg_twobody_scratch_elems(int32_t n_pairs) {
  if (n_pairs < 0) return -1;
  return (int64_t)n_pairs * kBlocks * 2 + 1;  // + the missing-ket flag
}

extern "C" int edg_twobody_expval(const edg_lookup_table* sector, const uint64_t* strides, const int32_t* loc_dims,
                                  int32_t n_sites, const int32_t* t_count, const uint8_t* t_ket, const double* t_amp,
                                  int32_t dmax, const int32_t* pair_i, const int32_t* pair_j, int32_t n_pairs,
                                  const void* psi, int32_t psi_dtype, int64_t psi_stride, double* corr,
                                  double* scratch, int64_t scratch_elems, cudaStream_t stream) {
  EDG_REQUIRE(sector != nullptr && strides != nullptr && loc_dims != nullptr && t_count != nullptr &&
                  t_ket != nullptr && t_amp != nullptr && corr != nullptr && scratch != nullptr,
              "edg_twobody_expval: null argument");
  EDG_REQUIRE(n_sites >= 2 && n_sites <= EDG_MAX_SITES && dmax >= 1 && dmax <= 256 && psi_stride >= 1,
              "edg_twobody_expval: bad sizes");
  EDG_REQUIRE(psi_dtype >= 0 && psi_dtype <= 3, "edg_twobody_expval: psi_dtype must be 0..3");
  EDG_REQUIRE(sector->key_words <= 1, "edg_twobody_expval: one-word keys only (key space below 2^63)");
  EDG_REQUIRE(n_pairs >= 0 && n_pairs <= n_sites * (n_sites - 1) / 2 && (n_pairs == 0 || (pair_i && pair_j)),
              "edg_twobody_expval: bad pair list");
  EDG_REQUIRE(((uintptr_t)t_amp & 15) == 0, "edg_twobody_expval: t_amp must be 16-byte aligned");
  EDG_REQUIRE(scratch_elems >= edg_twobody_scratch_elems(n_pairs), "edg_twobody_expval: scratch too small");
  cudaError_t e = cudaMemsetAsync(corr, 0, sizeof(double) * (size_t)n_sites * n_sites, stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_twobody_expval: reset");
  if (n_pairs == 0 || sector->n == 0) return EDG_OK;
  int32_t* err = reinterpret_cast<int32_t*>(scratch + (int64_t)n_pairs * kBlocks * 2);
  e = cudaMemsetAsync(err, 0, sizeof(int32_t), stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_twobody_expval: flag");
  Args a{*sector, strides, loc_dims, t_count, t_ket, reinterpret_cast<const double2*>(t_amp), pair_i, pair_j, psi,
         psi_stride, scratch, err, n_sites, dmax, n_pairs, 0, 0};
  a.tables_in_smem = table_bytes(n_sites, dmax) <= kTableSmemCap;
  a.diag_in_smem = dmax * diag_pitch(n_sites) <= kDiagCap;
  const int64_t smem = layout(n_sites, dmax, a.tables_in_smem, a.diag_in_smem).total;
  switch (psi_dtype) {
    case 0: e = launch<0>(a, smem, stream); break;
    case 1: e = launch<1>(a, smem, stream); break;
    case 2: e = launch<2>(a, smem, stream); break;
    default: e = launch<3>(a, smem, stream); break;
  }
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_twobody_expval");
  twobody_reduce_k<<<(n_pairs + 7) / 8, 256, 0, stream>>>(scratch, kBlocks, n_pairs, pair_i, pair_j, n_sites, corr);
  EDG_CHECK_LAUNCH("edg_twobody_expval: reduce");
  // the missing-ket flag decides the status: one small synchronous read
  int32_t h_err = 0;
  e = cudaMemcpyAsync(&h_err, err, sizeof(int32_t), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return edg::cuda_status(e, "edg_twobody_expval: flag read");
  if (h_err == 2) {
    edg::set_error("edg_twobody_expval: a pair names a site outside [0, n_sites) or the same site twice");
    return EDG_ERR_ARG;
  }
  if (h_err) {
    edg::set_error("edg_twobody_expval: an operator maps a sector configuration outside the sector");
    return EDG_ERR_MISSING_KET;
  }
  return EDG_OK;
}
