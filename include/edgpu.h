/*
 * edgpu.h -- C ABI of libedgpu, the sm_100a exact-diagonalization engine for
 * lattice gauge theories (sector enumeration, config->index lookup, sector
 * Hamiltonian assembly, matvec, Lanczos and Krylov time evolution).
 *
 * Conventions for every entry point:
 *   - all array arguments are DEVICE pointers owned by the caller (typically
 *     torch tensors passed as data_ptr()); the library never allocates,
 *     frees or retains them;
 *   - sizes are int64_t; configurations are packed into uint64 keys
 *     key = sum_s c_s * stride_s with the last site the fastest digit, so that
 *     ascending keys == lexicographic configuration order;
 *   - work is enqueued on the given stream and is asynchronous unless the
 *     comment says the call synchronizes;
 *   - the return value is EDG_OK (0) or a negative status; the message of the
 *     last failure on the calling thread is returned by edg_get_last_error.
 *
 * Each entry point cites the ed-lgt (edlgt 0.2.3) function it replaces.
 */
#ifndef EDGPU_H
#define EDGPU_H

#include <stdint.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EDG_OK 0
#define EDG_ERR_ARG -1          /* invalid argument / unsupported shape        */
#define EDG_ERR_CUDA -2         /* CUDA runtime error                          */
#define EDG_ERR_OVERFLOW -3     /* a count or key does not fit its type       */
#define EDG_ERR_MISSING_KET -4  /* an operator maps a sector state outside it */
#define EDG_ERR_NOT_CONVERGED -5
#define EDG_ERR_BREAKDOWN -6    /* Krylov space exhausted before convergence  */
#define EDG_ERR_TIMEOUT -7      /* a grid-wide wait of a persistent kernel    */
                                /* ran out (the launch returned early)        */

#define EDG_MAX_OPS 4           /* max operator factors of one term instance  */
#define EDG_MAX_SITES 64        /* max lattice sites of one configuration     */

/* ------------------------------------------------------------------------ */
/* Library                                                                  */
/* ------------------------------------------------------------------------ */

/* Copies the last failure message of the calling thread into buf. */
int edg_get_last_error(char* buf, int len);
/* ABI version (major * 100 + minor). */
int edg_version(void);

/* ------------------------------------------------------------------------ */
/* Tuning context (no counterpart in the reference, which has no autotuner). */
/* Autotuners store their launch-shape choices here, keyed by a hash of the  */
/* problem shape; the caller creates, passes and destroys the context, so    */
/* the library holds no global tuning state.  Thread-safe.                   */
/* ------------------------------------------------------------------------ */

#define EDG_CTX_MAX_PARAMS 8
typedef struct edg_ctx edg_ctx;

/* NULL when out of host memory. */
edg_ctx* edg_ctx_create(void);
void edg_ctx_destroy(edg_ctx* ctx);
/* Stores n_params (1..EDG_CTX_MAX_PARAMS) int32 values under key. */
int edg_ctx_put(edg_ctx* ctx, uint64_t key, const int32_t* params,
                int32_t n_params);
/* Copies up to n_params values stored under key; returns how many (0 when
 * the key is absent) or a negative status. */
int edg_ctx_get(edg_ctx* ctx, uint64_t key, int32_t* params, int32_t n_params);
/* Number of stored keys (-1 for a null context). */
int64_t edg_ctx_size(edg_ctx* ctx);

/* ------------------------------------------------------------------------ */
/* Exclusive prefix sum of int64 counts (the two-pass count/scan/fill idiom  */
/* of edlgt/symmetries/sym_qmb_operations.py:139-164, with int64 offsets).   */
/* ------------------------------------------------------------------------ */

/* Scratch elements (int64) edg_scan_i64 needs for n inputs. */
int64_t edg_scan_scratch_elems(int64_t n);
/* out[i] = sum_{k<i} in[i] for i in [0, n]; out has n+1 entries (out[n] is the
 * total). in and out may alias. */
int edg_scan_i64(const int64_t* in, int64_t* out, int64_t n, int64_t* scratch,
                 cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Sector keys                                                               */
/* A configuration (c_0 .. c_{n-1}) is the mixed-radix number                */
/* sum_s c_s * stride_s with the last site fastest (edlgt/tools/magic.py:     */
/* 41-140).  When the product of the local dimensions is below 2^63 a key is */
/* one uint64 word (key_words = 1).  Otherwise (key_words = 2) the sites are */
/* split at n_hi: the high word holds sites [0, n_hi), the low word sites    */
/* [n_hi, n_sites), each a mixed-radix number below 2^63 whose strides are    */
/* relative to its own word (stride of site n_hi-1 and of site n_sites-1 is  */
/* 1).  A two-word key takes 16 bytes, low word first, 16-byte aligned: the   */
/* unsigned 128-bit integer hi * 2^64 + lo, whose order is the               */
/* lexicographic order of the configurations.  Key arrays passed as          */
/* "uint64_t*" hold key_words words per key.  Up to 126 bits of key space.   */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* Sector enumeration                                                        */
/* Replaces iterative_sitebased_sym_sector_configs,                          */
/* iterative_sitebased_sym_sector_configs1, iterative_link_sector_configs,    */
/* iterative_link_sector_configs_plus (edlgt/symmetries/symmetry_sector.py:   */
/* 785-967, 970-1164, 1237-1326, 1329-1469) and global_abelian_sector          */
/* (edlgt/symmetries/global_abelian_sym.py:147-244).                          */
/* Generator diagonals are passed as integers (the dyadic values times a     */
/* power of two), which makes every accept/reject decision exact.            */
/* ------------------------------------------------------------------------ */

typedef struct {
  int32_t n_sites;
  int32_t dmax;                   /* padded local dimension                  */
  int32_t loc_dims[EDG_MAX_SITES];   /* by value: local dimension per site   */
  uint64_t strides[EDG_MAX_SITES];   /* by value: key stride per site        */
  const uint8_t* site_allowed;    /* [n_sites][dmax] 1 = state allowed       */
  /* global symmetries: U(1) sums or Z2 parities (type 0 / 1)                */
  int32_t n_glob;                 /* <= 4                                    */
  int32_t glob_type;
  const int32_t* glob_val;        /* [n_glob][n_sites][dmax] (Z2: 0/1 bits)  */
  const int32_t* glob_target;     /* [n_glob]                                */
  const int32_t* glob_rem_min;    /* [n_glob][n_sites+1] reachable minimum   */
  const int32_t* glob_rem_max;    /* [n_glob][n_sites+1] reachable maximum   */
  /* link constraints val0[dir][site0][c0] + val1[dir][site1][c1] == target  */
  int32_t n_dirs;
  const int32_t* link_val;        /* [n_dirs][2][n_sites][dmax]              */
  const int32_t* link_target;     /* [n_dirs]                                */
  const int32_t* pair_start;      /* [n_sites+1] pairs grouped by activation */
  const int32_t* pair_s0;         /* [n_pairs]                               */
  const int32_t* pair_s1;         /* [n_pairs]                               */
  const int32_t* pair_dir;        /* [n_pairs]                               */
  /* n-body constraints: sum (type 0) or parity (type 1) over a site set     */
  int32_t nbody_type;
  const int32_t* nb_val;          /* [n_nb][n_sites][dmax]                   */
  const int32_t* nb_target;       /* [n_nb]                                  */
  const int32_t* nb_start;        /* [n_sites+1] constraints by activation   */
  const int32_t* nb_id;           /* [n_act] constraint id                   */
  const int32_t* nb_site_start;   /* [n_nb+1] site list offsets              */
  const int32_t* nb_sites;        /* flattened site lists                    */
  /* key layout (see "Sector keys" above): 1 word, or 2 words split at n_hi  */
  int32_t key_words;              /* 1 or 2                                  */
  int32_t n_hi;                   /* sites [0, n_hi) in the high word (W=2)  */
} edg_sector_tables;

/* Number of per-block counters (int64) the level kernels need for n
 * candidate prefixes; scratch for edg_sector_level_count must hold this many
 * elements plus edg_scan_scratch_elems of it. */
int64_t edg_sector_level_blocks(int64_t n_candidates);

/* Level `depth` of the prefix expansion: every parent prefix (depth-1 sites,
 * n_prev of them; n_prev = 1 with an empty parent at depth 0) is extended by
 * each state of site `depth`; survivors keep the parent order and the state
 * order, so the final level is sorted.  Count writes, into block_offsets
 * (edg_sector_level_blocks(n_prev*d)+1 entries), the exclusive per-block
 * offsets and, at block_offsets[n_blocks], the number of survivors. */
int edg_sector_level_count(const edg_sector_tables* t, int32_t depth,
                           const uint64_t* prev_keys, const int32_t* prev_sums,
                           int64_t n_prev, int64_t* block_offsets,
                           int64_t* scratch, cudaStream_t stream);
/* Writes the survivors counted by edg_sector_level_count. */
int edg_sector_level_fill(const edg_sector_tables* t, int32_t depth,
                          const uint64_t* prev_keys, const int32_t* prev_sums,
                          int64_t n_prev, const int64_t* block_offsets,
                          uint64_t* next_keys, int32_t* next_sums,
                          cudaStream_t stream);

/* keys -> uint16 configurations [n][n_sites] (index_to_config over a sector,
 * edlgt/symmetries/generate_configs.py:30-54). */
int edg_keys_to_configs(const uint64_t* keys, int64_t n, int32_t n_sites,
                        const int32_t* loc_dims, uint16_t* configs,
                        cudaStream_t stream);
/* uint16 configurations -> keys (encode_all_configs,
 * edlgt/tools/magic.py:111-140). */
int edg_configs_to_keys(const uint16_t* configs, int64_t n, int32_t n_sites,
                        const uint64_t* strides, uint64_t* keys,
                        cudaStream_t stream);
/* The same for two-word keys split at n_hi (keys: 2n words; strides within
 * each word, device array of n_sites). */
int edg_keys_to_configs_wide(const uint64_t* keys, int64_t n, int32_t n_sites,
                             int32_t n_hi, const int32_t* loc_dims,
                             uint16_t* configs, cudaStream_t stream);
int edg_configs_to_keys_wide(const uint16_t* configs, int64_t n,
                             int32_t n_sites, int32_t n_hi,
                             const uint64_t* strides, uint64_t* keys,
                             cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* config -> index lookup                                                    */
/* Replaces config_to_index_binarysearch (edlgt/symmetries/                   */
/* generate_configs.py:145-173): index of the key in the sorted sector, or   */
/* -1 when absent.  A bucket table over the top key bits narrows each search.*/
/* ------------------------------------------------------------------------ */

typedef struct {
  const uint64_t* keys;         /* [n] sorted ascending, unique              */
  int64_t n;
  const int64_t* bucket_start;  /* [n_buckets+1]                             */
  int32_t shift;                /* bucket = dense key >> shift               */
  int64_t n_buckets;
  /* key layout; zero-initialised tables read as one-word keys              */
  int32_t key_words;            /* 0 or 1: one word; 2: two words            */
  int32_t n_hi;                 /* sites [0, n_hi) in the high word          */
  uint64_t lo_space;            /* product of the low word's dimensions: the */
                                /* dense key is hi * lo_space + lo (W = 2)   */
} edg_lookup_table;

/* Fills bucket_start (n_buckets+1 entries) for keys < n_buckets << shift. */
int edg_lookup_build(const uint64_t* keys, int64_t n, int32_t shift,
                     int64_t n_buckets, int64_t* bucket_start,
                     cudaStream_t stream);
/* Bucket table for keys of key_words words (1 or 2): bucket_start[b] is
 * the first row whose dense key (hi * lo_space + lo for two words) is
 * >= b << shift, and bucket_start[n_buckets] = n.  shift < 64 for one-word
 * keys, < 127 for two; every dense key must be < n_buckets << shift. */
int edg_lookup_build_wide(const uint64_t* keys, int64_t n, int32_t key_words,
                          uint64_t lo_space, int32_t shift, int64_t n_buckets,
                          int64_t* bucket_start, cudaStream_t stream);
int edg_lookup(const edg_lookup_table* table, const uint64_t* queries,
               int64_t m, int64_t* index_out, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Sector Hamiltonian assembly                                               */
/* Replaces nbody_term / nbody_data / nbody_data_2sites / nbody_data_4sites /  */
/* localbody_data_par (edlgt/symmetries/sym_qmb_operations.py:32-602), the     */
/* term site loops (edlgt/modeling/{local,twobody,plaquette}_term.py) and the */
/* triplet -> matrix build (edlgt/modeling/qmb_hamiltonian.py:173-225,          */
/* 667-702).  Output is the canonical matrix: off-diagonal entries as CSR      */
/* with duplicate (row, col) summed and columns ascending, and the diagonal as */
/* a dense vector with a presence flag per row.                               */
/* ------------------------------------------------------------------------ */

typedef struct {
  int32_t n_sites;
  int32_t dmax;
  int32_t loc_dims[EDG_MAX_SITES];   /* by value                              */
  uint64_t strides[EDG_MAX_SITES];   /* by value                              */
  edg_lookup_table sector;        /* sorted sector keys = matrix rows        */
  int32_t complex_values;         /* 0: real double, 1: interleaved complex  */
  /* local transition tables (nonzero entries of one site operator)         */
  const int32_t* t_count;         /* [n_tables][dmax]                        */
  const uint8_t* t_ket;           /* [n_tables][dmax][dmax]                  */
  const double* t_amp;            /* [n_tables][dmax][dmax](x2 if complex)   */
  /* off-diagonal term instances: product of n_ops site operators           */
  int32_t n_terms;
  const int32_t* term_nops;       /* [n_terms] in 1..EDG_MAX_OPS             */
  const int32_t* term_site;       /* [n_terms][EDG_MAX_OPS]                  */
  const int32_t* term_table;      /* [n_terms][EDG_MAX_OPS]                  */
  const double* term_coef;        /* [n_terms] (x2 if complex)               */
  /* diagonal terms: coef * op[c_site][c_site] (only the diagonal is used)   */
  int32_t n_dterms;
  const int32_t* dterm_site;      /* [n_dterms]                              */
  const double* dterm_diag;       /* [n_dterms][dmax] (x2 if complex)        */
  const double* dterm_coef;       /* [n_dterms] (x2 if complex)              */
} edg_assembly;

/* Per-row upper bound of off-diagonal entries (before merging duplicates). */
int edg_assemble_count(const edg_assembly* a, int64_t* row_bound,
                       cudaStream_t stream);
/* Generates the entries of each row into its [offsets[r], offsets[r+1])
 * window of tmp_cols/tmp_vals, merges duplicate columns, and writes the
 * merged count to row_nnz; the diagonal goes to diag/diag_present.
 * error_flag (one int32, zero-initialised by the caller) receives
 * EDG_ERR_MISSING_KET when a ket is outside the sector. */
int edg_assemble_fill(const edg_assembly* a, const int64_t* offsets,
                      int32_t* tmp_cols, double* tmp_vals, int64_t* row_nnz,
                      double* diag, uint8_t* diag_present, int32_t* error_flag,
                      cudaStream_t stream);
/* Copies the merged windows into the final CSR (rowptr from a scan of
 * row_nnz). */
int edg_assemble_compact(int64_t n_rows, int32_t complex_values,
                         const int64_t* offsets, const int32_t* tmp_cols,
                         const double* tmp_vals, const int64_t* rowptr,
                         int32_t* cols, double* vals, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Matvec y = (A_offdiag + diag) x                                           */
/* Replaces csr_spmv / csr_matmat (edlgt/modeling/qmb_hamiltonian.py:705-764)*/
/* and the SciPy CSC matvec behind eigsh / expm_multiply.                    */
/* dtype: 0 = f64, 1 = f32, 2 = complex128, 3 = complex64 (values, diag and */
/* vectors share the dtype; accumulation is in double precision).           */
/* Batched form: nvec right-hand sides stored interleaved x[row][vec],      */
/* sharing the off-diagonal matrix, with a per-vector diagonal diag[row][vec].*/
/* ------------------------------------------------------------------------ */

int edg_spmv(int32_t dtype, int64_t n_rows, int64_t nnz,
             const int64_t* rowptr, const int32_t* cols, const void* vals,
             const void* diag, int32_t nvec, const void* x, void* y,
             cudaStream_t stream);

/* Same with an explicit number of threads cooperating on a row (2, 4, 8, 16
 * or 32; 0 = heuristic from the mean row length): the knob the autotuner in
 * edgpu.solvers.tune_spmv_group sets. */
int edg_spmv_group(int32_t dtype, int64_t n_rows, int64_t nnz,
                   const int64_t* rowptr, const int32_t* cols, const void* vals,
                   const void* diag, int32_t nvec, const void* x, void* y,
                   int32_t group, cudaStream_t stream);

/* Sliced ELL (SELL-32-sigma) layout of the off-diagonal matrix for the f32
 * Krylov path (same product as csr_spmv, qmb_hamiltonian.py:705-730, with a
 * row layout built for coalesced loads): rows sorted by length (descending,
 * stable) inside windows of `window` rows (a multiple of 32, at most 4096;
 * 32 keeps the basis order), slices of 32 sorted rows, entries of a slice
 * stored column-major as 8-byte (int32 column, f32 value) pairs, padding
 * marked by column -1.  Build: edg_sell_order (perm [n_slices*32], -1 =
 * padding; width and counts [n_slices] = width * 32), exclusive scan of
 * counts into off [n_slices+1] (edg_scan_i64), then edg_sell_fill (entries
 * [off[n_slices]] pairs; dtype of vals 0 = f64, 1 = f32). */
int64_t edg_sell_slices(int64_t n_rows);
int edg_sell_order(const int64_t* rowptr, int64_t n_rows, int32_t window,
                   int32_t* perm, int32_t* width, int64_t* counts,
                   cudaStream_t stream);
int edg_sell_fill(int32_t dtype, const int64_t* rowptr, const int32_t* cols,
                  const void* vals, int64_t n_rows, const int32_t* perm,
                  const int32_t* width, const int64_t* off, void* entries,
                  cudaStream_t stream);
/* y[v * y_plane + r] (f64, planar; y_plane 0 = n_rows) = (A + diag) x with
 * x interleaved (f32 rows of x_stride entries: nvec, or 4 for nvec = 3),
 * diag [n_rows][nvec] (f32). */
int edg_spmv_sell(int64_t n_rows, int32_t nvec, const int32_t* perm,
                  const int32_t* width, const int64_t* off, const void* entries,
                  const float* diag, const float* x, int32_t x_stride,
                  double* y, int64_t y_plane, cudaStream_t stream);
/* Dictionary-packed tiled layout of the off-diagonal matrix (same product
 * as csr_spmv, qmb_hamiltonian.py:705-730, with 4 bytes an entry): the model
 * Hamiltonians have few distinct off-diagonal values, so an entry is the
 * word col | (value index << colbits), n_rows < 2^colbits, the values in an
 * ascending table of at most 2^(32 - colbits) and at most
 * EDG_PACK_MAX_VALUES entries.  Rows are grouped in tiles of 16; tile t is
 * w_t = its longest row wide, and its 16 w_t words [tile_off[t],
 * tile_off[t+1]) hold entry k of its row s at tile_off[t] + 16 k + s
 * (k-major, CSR order inside a row), shorter rows padded with the all-ones
 * word (its column, 2^colbits - 1, is never a real one).
 * Build: edg_pack_collect inserts the values' bit patterns (dtype 0 f64, 1
 * f32) into a caller-owned set of 2^log2_slots slots (8-byte slots for f64,
 * 4-byte for f32) pre-filled with 0xFF bytes, setting overflow[0] when the
 * set fills (more distinct values than it holds) or a value is a NaN; the
 * caller reads the set and sorts the distinct values into the table.
 * edg_pack_tile_counts writes counts [n_tiles] = 16 w_t (n_tiles =
 * edg_pack_tiles(n_rows)); their exclusive scan offsets [n_tiles+1]
 * (edg_scan_i64) gives total = offsets[n_tiles] < 2^31 - 4 words, and
 * edg_pack_encode writes tile_off [n_tiles+1] (int32) and words [total+4],
 * setting missing[0] if a value is not in the table.  The matvec (y f64
 * planar, x rows at x_stride, diag [n_rows][nvec], table, diag and x in the
 * dtype) stages each tile with one bulk copy: f64 gives the same sums, in
 * the same order, as the CSR kernel with two threads a row; f32 sums each
 * half row's products in f32 and the rest in f64.  err (device int, may be
 * NULL) receives EDG_ERR_TIMEOUT if a stage wait ran out (1 s; y is then
 * incomplete). */
#define EDG_PACK_MAX_VALUES 4096
int64_t edg_pack_tiles(int64_t n_rows);
int edg_pack_tile_counts(int64_t n_rows, const int64_t* rowptr,
                         int64_t* counts, cudaStream_t stream);
int edg_pack_collect(int32_t dtype, const void* vals, int64_t nnz, void* set,
                     int32_t log2_slots, int32_t* overflow,
                     cudaStream_t stream);
int edg_pack_encode(int32_t dtype, int64_t n_rows, int64_t total,
                    const int64_t* rowptr, const int32_t* cols,
                    const void* vals, const void* table, int32_t count,
                    int32_t colbits, const int64_t* offsets,
                    int32_t* tile_off, uint32_t* words, int32_t* missing,
                    cudaStream_t stream);
int edg_spmv_packed(int32_t dtype, int64_t n_rows, int32_t nvec,
                    const int32_t* tile_off, const uint32_t* words,
                    const void* table, int32_t count, int32_t colbits,
                    const void* diag, const void* x, int32_t x_stride,
                    double* y, int64_t y_plane, int32_t* err,
                    cudaStream_t stream);
/* The CSR matvec in the same configuration (f32 values, diagonal and x, f64
 * planar y): the f32 Krylov path's CSR kernel, for layout comparisons. */
int edg_spmv_f32_planar(int64_t n_rows, int64_t nnz, const int64_t* rowptr,
                        const int32_t* cols, const float* vals,
                        const float* diag, int32_t nvec, const float* x,
                        int32_t x_stride, double* y, int64_t y_plane,
                        int32_t group, cudaStream_t stream);

/* Casts between f64 <-> f32 (or c128 <-> c64) arrays of n scalars. */
int edg_convert(int32_t dtype_in, const void* in, int32_t dtype_out, void* out,
                int64_t n_scalars, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Lanczos ground states                                                     */
/* Replaces scipy.sparse.linalg.eigsh(H, k, which="SA") as called from       */
/* QMB_hamiltonian.diagonalize (edlgt/modeling/qmb_hamiltonian.py:260-332).  */
/* Lanczos with full reorthogonalisation (delayed classical Gram-Schmidt,   */
/* two passes over the basis per step) on nvec independent problems that    */
/* share the off-diagonal matrix, vectors in f64 or f32 (dtype 0/1) and     */
/* every inner product, recurrence coefficient and the tridiagonal          */
/* eigensolve in f64 on the device.  Stops when the k lowest Ritz values of */
/* every problem have residual |beta_{j+1} s_j| <= tol * max(1, |theta|),   */
/* or after max_iter steps.  The step index, the convergence checks and     */
/* their schedule live on the device: the host records a few steps (and     */
/* their checks) in a CUDA graph and replays it, one replay ahead, polling  */
/* the progress words the device writes to host_progress; no stream         */
/* synchronisation happens inside the step loop.  With stats set, the steps */
/* are launched one by one with CUDA events around each phase instead.      */
/* A step that reorthogonalises against at most 8 vectors (reorth_window of  */
/* 1..7, or max_iter <= 8) does it in one cooperative launch (dots, a grid    */
/* barrier with a 1 s limit, update); the device must support cooperative   */
/* launches.                                                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
  int32_t dtype;          /* 0 f64, 1 f32 (real symmetric matrices)          */
  int64_t n_rows;
  int64_t nnz;
  const int64_t* rowptr;
  const int32_t* cols;
  const void* vals;
  const void* diag;       /* [n_rows][nvec]                                 */
  int32_t nvec;           /* independent problems, <= 4                     */
  int32_t k;              /* eigenpairs wanted per problem                  */
  int32_t max_iter;       /* Krylov dimension limit                         */
  double tol;
  int32_t check_every;    /* steps between convergence checks               */
  uint64_t seed;          /* start vector: uniform(-1,1) from this seed     */
  const void* v0;         /* optional start vectors [n_rows][nvec] or NULL  */
  int32_t spmv_group;     /* threads per matvec row, 0 = heuristic         */
  double* stats;          /* optional HOST array of 6 doubles, or NULL:     */
                          /* [0] matvec ms, [1] matvec launches, [2] reorth */
                          /* ms, [3] kernel launches, [4] Lanczos steps,    */
                          /* [5] check ms (CUDA events on the stream)       */
  int32_t* host_progress; /* optional PINNED host memory, >= 4 int32: the   */
                          /* device writes [0] steps done, [1] done flag;   */
                          /* NULL = the host synchronises once per replay   */
  const int32_t* sell_perm;   /* optional SELL layout of the off-diagonal   */
  const int32_t* sell_width;  /* matrix (edg_sell_*), used by the f32 path  */
  const int64_t* sell_off;    /* when sell_entries is not NULL              */
  const void* sell_entries;
  int32_t reorth_window;  /* 0: full reorthogonalisation; W > 0: each step */
                          /* orthogonalises against the last W Krylov      */
                          /* vectors only (local reorthogonalisation: the  */
                          /* lowest Ritz pair converges as with the full   */
                          /* one, later copies of it are not suppressed)   */
  const int32_t* pk_tile_off;  /* optional dictionary-packed layout of the  */
  const uint32_t* pk_words;    /* off-diagonal matrix (edg_pack_*) with its */
  const void* pk_table;        /* table in the problem dtype; used instead  */
  int32_t pk_count;            /* of the CSR (and SELL) arrays when         */
  int32_t pk_colbits;          /* pk_words is not NULL                      */
} edg_lanczos_problem;

/* Bytes of device workspace edg_lanczos needs. */
int64_t edg_lanczos_workspace_bytes(const edg_lanczos_problem* p);
/* Runs to convergence (synchronizes every check_every steps).  Outputs:
 * evals [nvec][k] (f64), evecs [k][n_rows][nvec] in the problem dtype (may be
 * NULL), iters_out [nvec] steps used, resid_out [nvec][k] residual bounds. */
int edg_lanczos(const edg_lanczos_problem* p, void* workspace,
                int64_t workspace_bytes, double* evals, void* evecs,
                int32_t* iters_out, double* resid_out, cudaStream_t stream);

/* Tridiagonal eigen-solve on the device (multisection + inverse iteration)
 * of T = tridiag(beta[1..m-1], alpha[0..m-1], beta[1..m-1]): the k <= 16
 * lowest eigenvalues and eigenvectors S [k][m] (f64; evecs may be NULL).
 * work holds 6*m doubles. */
int edg_tridiag_lowest(const double* alpha, const double* beta, int32_t m,
                       int32_t k, double* evals, double* evecs, double* work,
                       cudaStream_t stream);

/* Same as edg_tridiag_lowest, for callers that cannot allocate device memory
 * (code running where cudaMalloc is unavailable or forbidden, e.g. inside a
 * host callback or a memory-capped plugin host).  No counterpart in the
 * reference.  The 6*m doubles of scratch come from a static device array
 * compiled into the library, so m is limited to 4096 (larger m returns
 * EDG_ERR_ARG) and the call allocates nothing.  The first call on a device
 * looks up the array's device address (with that device current); make that
 * first call before any stream capture.  All calls share the one array:
 * calls that overlap on the GPU race, so serialise them (one stream, or
 * events).  Inputs and outputs are caller-owned device pointers.  The
 * address is cached per device for the life of the process: a device reset
 * (cudaDeviceReset, or destroying the primary context) between calls is not
 * supported. */
int edg_tridiag_lowest_noalloc(const double* alpha, const double* beta,
                               int32_t m, int32_t k, double* evals,
                               double* evecs, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Batched Lanczos over an (instance, row-tile) work queue: instances of any */
/* dimension (charge sectors, coupling sweeps, lattice sizes) in one         */
/* persistent cooperative launch.  Every phase of a Lanczos step (matvec,    */
/* dots, coefficients, update, convergence check) walks the list of          */
/* (instance, tile of tile_rows rows) items; phases are separated by         */
/* grid-wide barriers, so one instance spreads over many CTAs and small      */
/* instances share the grid.  Replaces the sequential loop of eigsh calls of */
/* QMB_hamiltonian.diagonalize (edlgt/modeling/qmb_hamiltonian.py:260-332)   */
/* over a sweep of instances.  dtype 1 keeps the Krylov basis and matvec     */
/* operands in f32 (dots, recurrence, reorthogonalisation coefficients and   */
/* the tridiagonal eigen-solve in f64); dtype 0 is f64 throughout.  The      */
/* launch does no host synchronisation and no allocation, so a whole solve   */
/* can be recorded in a CUDA graph.                                          */
/* ------------------------------------------------------------------------ */

#define EDG_TB_FIELDS 8  /* int64 fields per instance in the plan table   */

typedef struct {
  int32_t dtype;              /* 0: f64 vectors and matvec; 1: f32          */
  int32_t n_inst;
  int32_t n_items;            /* from edg_tiled_batch_plan                  */
  int32_t tile_rows;          /* rows per work item (multiple of 4)         */
  int32_t lanes;              /* threads per matrix row: 2, 4, 8, 16, 32    */
  int32_t k;                  /* lowest eigenpairs per instance (1..8)      */
  int32_t max_iter;           /* Krylov steps at most (<= 2000)             */
  int32_t reserved;
  double tol;                 /* |beta_m s_q(m)| <= tol * max(1, |theta_q|) */
  uint64_t seed;              /* random start vectors when v0 is NULL       */
  const int64_t* inst;        /* [n_inst][EDG_TB_FIELDS] plan table         */
  const int32_t* item_inst;   /* [n_items] instance of each item            */
  const uint8_t* check_at;    /* [max_iter] 1 = check after that step       */
  const int64_t* rowptr;      /* per-instance rowptr blocks, concatenated;  */
                              /* entries index the concatenated cols/vals   */
  const int32_t* cols;        /* instance-local columns                     */
  const void* vals;           /* off-diagonal values, f64 or f32 (dtype)    */
  const void* diag;           /* diagonals concatenated [sum dims] (dtype)  */
  const double* v0;           /* start vectors concatenated (f64) or NULL   */
  void* workspace;            /* plan's byte count, 256-byte aligned        */
  double* evals;              /* [n_inst][k] (NaN where never checked)      */
  double* resid;              /* [n_inst][k] residual bounds                */
  int32_t* iters;             /* [n_inst] Krylov dimension used             */
  double* evecs;              /* ground-state vectors concatenated (f64,    */
                              /* normalised) or NULL                        */
  int32_t* status;            /* device word: EDG_OK or EDG_ERR_TIMEOUT     */
} edg_tiled_batch;

/* Host-side plan: per-instance table (dims in rows), the item list, the
 * convergence-check schedule (every check_every steps, the last step, and
 * each instance's Krylov cap min(dim, max_iter)), the item count and the
 * workspace size.  inst_out / item_inst_out / check_at_out may be NULL
 * (query).  All pointers are host memory. */
int edg_tiled_batch_plan(int32_t n_inst, const int64_t* dims, int32_t dtype,
                         int32_t max_iter, int32_t k, int32_t tile_rows,
                         int32_t check_every, int64_t* inst_out,
                         int32_t* item_inst_out, uint8_t* check_at_out,
                         int32_t* n_items_out, int64_t* workspace_bytes_out);
/* Bytes at the start of the workspace that every launch resets. */
int edg_tiled_batch_header_bytes(int32_t n_inst);
/* One solve: resets the workspace header, one cooperative launch, copies the
 * launch status to b->status.  Asynchronous; converged instances leave the
 * queue, an unconverged one stops at its cap with its residual reported. */
int edg_lanczos_tiled_batch(const edg_tiled_batch* b, cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Batched Lanczos for many small instances (charge sectors, coupling        */
/* sweeps) in one persistent launch: CTAs pull instances from a device work  */
/* queue.  Replaces the sequential loop of eigsh calls (one per instance) of  */
/* QMB_hamiltonian.diagonalize (edlgt/modeling/qmb_hamiltonian.py:260-332)   */
/* that a sweep over instances performs.  f64 throughout, full               */
/* reorthogonalisation, device tridiagonal eigen-solve per instance.  The    */
/* launch (a queue reset + one kernel) can be captured in a CUDA graph.      */
/* ------------------------------------------------------------------------ */

typedef struct {
  int32_t n_inst;
  int32_t max_dim;            /* largest instance dimension (<= 4096)       */
  const int64_t* dims;        /* [n_inst]                                   */
  const int64_t* row_off;     /* [n_inst] first row of the instance in      */
                              /* diag / evecs                               */
  const int64_t* rowptr_off;  /* [n_inst] start of the instance's rowptr    */
                              /* block (dim+1 entries into cols / vals)     */
  const int64_t* rowptr;
  const int32_t* cols;        /* column indices local to the instance       */
  const double* vals;
  const double* diag;         /* [sum of dims]                              */
  double* work;               /* per-instance scratch, see                  */
  const int64_t* work_off;    /* edg_small_batch_work_elems; [n_inst]       */
  int32_t k;                  /* eigenvalues per instance (<= 16)           */
  int32_t max_iter;
  int32_t check_every;
  double tol;
  uint64_t seed;
  double* evals;              /* [n_inst][k]                                */
  double* evecs;              /* [sum of dims] ground states, or NULL       */
  int32_t* iters;             /* [n_inst] Krylov dimension used, or NULL    */
} edg_small_batch;

/* Scratch doubles one instance of dimension dim needs. */
int64_t edg_small_batch_work_elems(int64_t dim, int32_t max_iter, int32_t k);
/* queue: one int32 of device memory (reset by the call). */
int edg_lanczos_small_batched(const edg_small_batch* b, int32_t* queue,
                              cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Krylov time evolution psi <- exp(-i H dt) psi                             */
/* Replaces scipy.sparse.linalg.expm_multiply(-iH, psi0, ...) as called from */
/* QMB_hamiltonian.time_evolution (edlgt/modeling/qmb_hamiltonian.py:        */
/* 334-426).  Krylov vectors complex128 or complex64, Lanczos recurrence and  */
/* the small exponential in f64; no host synchronisation inside a step       */
/* unless err_out is given.                                                  */
/* ------------------------------------------------------------------------ */

typedef struct {
  int32_t vec_dtype;      /* 2 complex128, 3 complex64 (psi and the basis) */
  int32_t mat_dtype;      /* 0 f64, 1 f32 (real form), 2 c128, 3 c64; same  */
                          /* precision as the vectors                       */
  int64_t n_rows;
  int64_t nnz;
  const int64_t* rowptr;
  const int32_t* cols;
  const void* vals;
  const void* diag;       /* [n_rows]                                       */
  int32_t m;              /* Krylov dimension, <= 64                        */
  int32_t reorth_passes;  /* 0 local recurrence, 1 or 2 full Gram-Schmidt   */
  int32_t spmv_group;     /* threads per matvec row, 0 = heuristic         */
  const int32_t* pk_tile_off; /* optional dictionary-packed layout of the   */
  const uint32_t* pk_words;   /* real off-diagonal matrix (edg_pack_*, mat_ */
  const void* pk_table;       /* dtype 0 or 1, table in that dtype): the    */
  int32_t pk_count;           /* matvec treats each complex vector as two   */
  int32_t pk_colbits;         /* real right-hand sides; used when pk_words  */
                              /* is not NULL                                */
  int32_t* status;        /* optional device word: EDG_ERR_TIMEOUT when a   */
                          /* stage wait of the packed matvec ran out        */
} edg_krylov_problem;

int64_t edg_krylov_workspace_bytes(const edg_krylov_problem* p);
/* One step of length dt in place on psi [n_rows] (complex, vec_dtype).
 * err_out (host, may be NULL): a posteriori error estimate of the step. */
int edg_krylov_step(const edg_krylov_problem* p, void* psi, double dt,
                    void* workspace, int64_t workspace_bytes, double* err_out,
                    cudaStream_t stream);

/* ------------------------------------------------------------------------ */
/* Local (diagonal) observables                                              */
/* Replaces LocalTerm.get_expval in a symmetry sector (edlgt/modeling/       */
/* local_term.py:119-237, exp_val_data edlgt/modeling/qmb_state.py:631-654): */
/* out[s] = sum_r |psi_r|^2 diag[s][c_s(r)] for all sites at once.           */
/* ------------------------------------------------------------------------ */

typedef struct {
  int32_t d[EDG_MAX_SITES];   /* local dimension per site (by value)        */
} edg_site_dims;

/* psi: dtype 0 f64, 1 f32, 2 complex128, 3 complex64, element r at
 * psi[r * psi_stride]; diag: [n_sites][dmax] f64; out: [n_sites] f64. */
int edg_local_expval(const uint64_t* keys, int64_t n, const edg_site_dims* dims,
                     int32_t n_sites, const void* psi, int32_t psi_dtype,
                     int64_t psi_stride, const double* diag, int32_t dmax,
                     double* out, cudaStream_t stream);
/* The same over two-word keys split at n_hi (keys: 2n words). */
int edg_local_expval_wide(const uint64_t* keys, int64_t n, int32_t n_hi,
                          const edg_site_dims* dims, int32_t n_sites,
                          const void* psi, int32_t psi_dtype,
                          int64_t psi_stride, const double* diag,
                          int32_t dmax, double* out, cudaStream_t stream);

/* Two-body correlators, TwoBodyTerm.get_expval / lattice_twobody_exp_val
 * (edlgt/modeling/twobody_term.py:160-264): corr[i * n_sites + j] =
 * corr[j * n_sites + i] = Re <psi| A_i B_j |psi> for each listed pair i < j
 * (pair_i, pair_j device arrays), 0 elsewhere.  A and B come as transition
 * tables: t_count [2][n_sites][dmax], t_ket [2][n_sites][dmax][dmax] (uint8),
 * t_amp [2][n_sites][dmax][dmax][2] (re, im), first index 0 for A, 1 for B.
 * sector: the lookup table of the sorted sector keys; strides, loc_dims:
 * [n_sites] device arrays of the key format.  psi: dtype 0 f64, 1 f32,
 * 2 complex128, 3 complex64 at psi[r * psi_stride].  scratch: at least
 * edg_twobody_scratch_elems(n_pairs) doubles; t_amp 16-byte aligned.
 * Synchronizes the stream (one flag read); a ket outside the sector returns
 * EDG_ERR_MISSING_KET (the reference would read psi[-1] there), a pair with a
 * site outside [0, n_sites) or i == j returns EDG_ERR_ARG. */
int64_t edg_twobody_scratch_elems(int32_t n_pairs);
int edg_twobody_expval(const edg_lookup_table* sector, const uint64_t* strides,
                       const int32_t* loc_dims, int32_t n_sites, const int32_t* t_count,
                       const uint8_t* t_ket, const double* t_amp, int32_t dmax,
                       const int32_t* pair_i, const int32_t* pair_j, int32_t n_pairs,
                       const void* psi, int32_t psi_dtype, int64_t psi_stride, double* corr,
                       double* scratch, int64_t scratch_elems, cudaStream_t stream);

/* Dense row-major (n, n) form of a canonical sector matrix (off-diagonal CSR
 * plus its diagonal), for full diagonalisation: QMB_hamiltonian.
 * convert_hamiltonian("dense") (edlgt/modeling/qmb_hamiltonian.py:227-258).
 * dtype 0 f64 or 2 complex128 (interleaved); err_flag: one device int32.
 * Synchronizes the stream (one flag read). */
int edg_csr_to_dense(int32_t dtype, int64_t n, const int64_t* rowptr, const int32_t* cols,
                     const void* vals, const void* diag, void* out, int32_t* err_flag,
                     cudaStream_t stream);

/* ------------------------------------------------------------------------
 * Momentum basis.  Replaces build_all_translations, select_references and
 * momentum_basis_zero_k / momentum_basis_finite_k
 * (edlgt/symmetries/translational_sym.py:567-949, get_momentum_basis
 * :1307-1358) and the momentum-projected term builders
 * (nbody_data_momentum*, :1394-1969): the projector B is built on the device
 * (CSC, rows ascending, complex128 values) and H_k = B^dagger H B is applied
 * matrix-free around the sector matvec (expand, matvec, reduce).
 * ------------------------------------------------------------------------ */
typedef struct {
  int32_t lattice_dim;        /* 1..3                                         */
  int32_t n_shifts;           /* prod(shifts_per_dir) <= EDG_MAX_SITES        */
  int32_t shifts_per_dir[4];  /* R_d = L_d / unit cell d                      */
  int32_t shift_strides[4];   /* row-major strides over the shifts            */
  int32_t k_vals[4];          /* momentum labels                              */
} edg_momentum_group;

/* trans[r * n_shifts + t] = row of configuration r translated by shift t;
 * source_sites [n_shifts][n_sites] (device): the site whose local state lands
 * on each destination site.  local_map (nullable, device [map_dim]): a local
 * state map applied t times along with shift t, the translation-charge
 * generator of build_TC_translations (translational_sym.py:455-505; 1D, unit
 * cell 1); label_sign / row_sign (nullable together, device [map_dim] /
 * [n_rows]): row_sign[r] = prod_s label_sign[c_s(r)]
 * (precompute_C_sign_per_config, :108-128).  A translated configuration
 * outside the sector returns EDG_ERR_MISSING_KET.  Synchronizes the stream
 * (one flag read). */
int edg_momentum_translations(const edg_lookup_table* sector, const uint64_t* strides,
                              const int32_t* loc_dims, int32_t n_sites, const int32_t* source_sites,
                              int32_t n_shifts, const int32_t* local_map, int32_t map_dim,
                              const double* label_sign, double* row_sign, int32_t* trans,
                              int32_t* err_flag, cudaStream_t stream);
/* Scratch elements (int64) edg_momentum_references needs. */
int64_t edg_momentum_scratch_elems(int64_t n_rows);
/* refs[c] = reference row of column c (the smallest row of each orbit whose
 * axis periods are compatible with k_vals, ascending); pvec [n_rows][dim] =
 * axis periods of every row; *n_cols (host).  Synchronizes the stream. */
int edg_momentum_references(const int32_t* trans, int64_t n_rows, const edg_momentum_group* g,
                            int32_t* pvec, int64_t* refs, int64_t* n_cols, int64_t* scratch,
                            int64_t scratch_elems, cudaStream_t stream);
/* Columns of B.  phase_table [dim][max_r] complex128 = exp(-2 pi i k_d t / R_d)
 * by repeated products.  row_sign (nullable, [n_rows]): images at odd flat
 * shifts take the reference row's sign (the TC bases, :952-1303).  With
 * row_idx == NULL (count pass): col_ptr [n_cols+1]
 * = offsets, *nnz (host) = total, stream synchronized; scratch:
 * edg_scan_scratch_elems(n_cols).  Otherwise (fill pass): row_idx [nnz],
 * data [nnz] complex128. */
int edg_momentum_columns(const int32_t* trans, const int64_t* refs, int64_t n_cols, const int32_t* pvec,
                         const edg_momentum_group* g, const double* phase_table, int32_t max_r,
                         int32_t zero_k, const double* row_sign, int64_t* col_ptr, int64_t* nnz,
                         int32_t* row_idx, double* data, int64_t* scratch, int64_t scratch_elems,
                         cudaStream_t stream);
/* row_col[r] = column holding row r (-1 if none), row_val[r] its complex128
 * value.  A row in two columns returns EDG_ERR_ARG.  Synchronizes. */
int edg_momentum_rowmap(const int64_t* col_ptr, const int32_t* row_idx, const double* data, int64_t n_cols,
                        int64_t n_rows, int64_t* row_col, double* row_val, int32_t* err_flag,
                        cudaStream_t stream);
/* v = B x (complex128, v [n_rows], x [n_cols]). */
int edg_momentum_expand(int64_t n_rows, const int64_t* row_col, const double* row_val, const double* x,
                        double* v, cudaStream_t stream);
/* y = B^dagger w (complex128, w [n_rows], y [n_cols]), fixed summation order. */
int edg_momentum_reduce(int64_t n_cols, const int64_t* col_ptr, const int32_t* row_idx, const double* data,
                        const double* w, double* y, cudaStream_t stream);

/* ------------------------------------------------------------------------
 * Bipartitions.  Replaces QuantumModel._get_partition with
 * _unique_configs_with_inverse (edlgt/models/quantum_model.py:715-791,
 * 73-117) and build_psi_matrix (edlgt/modeling/qmb_state.py:596-627).  A part
 * (subsystem or environment) is a list of sites in ascending order; its key
 * packs their local states mixed radix, last part site fastest, so ascending
 * part keys are np.unique's order of the part configurations.
 * ------------------------------------------------------------------------ */
#define EDG_PART_MAX_KEY_SPACE (1ull << 34)

typedef struct {
  int32_t n_part;                       /* sites in the part, 0..EDG_MAX_SITES  */
  int32_t reserved;
  uint64_t key_space;                   /* product of the part's local dims     */
  uint64_t src_stride[EDG_MAX_SITES];   /* each part site's stride in the key   */
  uint64_t dim[EDG_MAX_SITES];          /* its local dimension                  */
  uint64_t part_stride[EDG_MAX_SITES];  /* its stride in the part key           */
} edg_part_spec;

/* Scratch elements (8-byte) edg_part_map needs; -1 when key_space is 0 or
 * above EDG_PART_MAX_KEY_SPACE. */
int64_t edg_part_scratch_elems(uint64_t key_space);
/* index[r] = position of row r's part configuration among the distinct part
 * configurations of the sector (ascending keys); *n_unique (host) = their
 * number; unique_keys (nullable, device, unique_cap entries) = those keys.
 * Synchronizes the stream (one count read). */
int edg_part_map(const uint64_t* keys, int64_t n, const edg_part_spec* spec, int64_t* index,
                 uint64_t* unique_keys, int64_t unique_cap, int64_t* n_unique, uint64_t* scratch,
                 int64_t scratch_elems, cudaStream_t stream);
/* out[sub_index[r] * env_dim + env_index[r]] = psi[r], zero elsewhere: the
 * dense (sub_dim, env_dim) state matrix.  psi_dtype 0 f64, 1 f32,
 * 2 complex128, 3 complex64; out_dtype 0 f64 (real states only) or
 * 2 complex128.  err_flag: one device int32.  An index out of range returns
 * EDG_ERR_ARG.  Synchronizes the stream (one flag read). */
int edg_psi_matrix(const void* psi, int32_t psi_dtype, int64_t n, const int64_t* sub_index,
                   const int64_t* env_index, int64_t sub_dim, int64_t env_dim, void* out,
                   int32_t out_dtype, int32_t* err_flag, cudaStream_t stream);

/* ------------------------------------------------------------------------
 * Matrix-free Z_n lattice gauge theory with staggered fermions (periodic
 * Lx x Ly, Gauss law, zero charge, optional zero momentum).
 *
 * No reference counterpart computes this model: ed-lgt raises for odd n
 * with matter (edlgt/operators/Zn_operators.py:153-157).  The pieces it
 * replaces are the momentum-basis builders (get_momentum_basis,
 * edlgt/symmetries/translational_sym.py:1307-1358; build_all_translations
 * :567-617; select_references :620-694; momentum_basis_zero_k :697-819), the
 * sector enumeration (symmetry_sector.py:785-967) and the projected n-body
 * triplets with their CSR matvec (nbody_data_momentum*,
 * translational_sym.py:1394-1969; csr_spmv, qmb_hamiltonian.py:705-730):
 * the Hamiltonian is never stored, each matvec recomputes its elements from
 * the packed representative configurations.
 *
 * Packed key: link l = 2 s + mu has its field at bits
 * [link_bits * l, link_bits * (l + 1)); site s's occupation at bit
 * field_bits + s.  Gauss index: colex rank of the occupied-site set times
 * zn^n_cot plus the cotree fields as base-zn digits.
 * ------------------------------------------------------------------------ */
#define EDG_ZN_MAX_SITES 14
#define EDG_ZN_MAX_GROUP 32

typedef struct {
  int32_t sf, sx;   /* field bits: lane-array rotation, rotation inside each lane */
  int32_t sm, smx;  /* occupation bits: the same two rotations */
  uint64_t hif, lof; /* field bits at lane positions >= sx / < sx */
  uint32_t him, lom; /* occupation bits at lane positions >= smx / < smx */
  uint32_t ylow, yhigh; /* occupied rows that stay below / wrap around in y */
  uint32_t xhead, xtail; /* row-0 sites that stay / wrap around in x */
} edg_zn_translation;

typedef struct {
  int32_t lx, ly, zn, link_bits;
  int32_t n_sites, n_links, field_bits, n_cot;
  int64_t n_gauss;  /* sector size before momentum: n_matter * zn^n_cot (< 2^32) */
  int64_t pow_cot;  /* zn^n_cot */
  uint32_t odd_mask;  /* sites with static charge offset 1 (x odd) */
  uint32_t even_mask; /* sites with eta = +1 */
  int32_t n_group;    /* translations, element 0 the identity */
  int32_t n_div;      /* stabiliser sizes (divisors of n_group), at most 8 */
  int32_t divisors[8];
  edg_zn_translation group[EDG_ZN_MAX_GROUP];
  int32_t cot_link[2 * EDG_ZN_MAX_SITES]; /* cotree link of digit c */
  /* Gauss-law peeling order, children before parents */
  int32_t peel_site[EDG_ZN_MAX_SITES], peel_link[EDG_ZN_MAX_SITES], peel_sign[EDG_ZN_MAX_SITES];
  int32_t peel_other[EDG_ZN_MAX_SITES][3], peel_osign[EDG_ZN_MAX_SITES][3];
  /* Hamiltonian geometry: link tail/head sites, Kogut-Susskind phase,
   * occupation mask strictly between tail and head (Jordan-Wigner order) */
  int32_t link_tail[2 * EDG_ZN_MAX_SITES], link_head[2 * EDG_ZN_MAX_SITES];
  int32_t link_eta[2 * EDG_ZN_MAX_SITES];
  uint32_t link_between[2 * EDG_ZN_MAX_SITES];
  int32_t plaq[EDG_ZN_MAX_SITES][4]; /* links raised, raised, lowered, lowered by U_p */
  double esq[4];                     /* E^2 of each field value */
  const uint64_t* chunk_lut;  /* device [ceil(field_bits / 8)][256]: cotree digits of a key byte */
  const uint32_t* occ_rank;   /* device [2^n_sites]: colex rank, 0xFFFFFFFF off-sector */
  const uint32_t* rank_occ;   /* device [n_matter]: occupation bits of a rank */
} edg_zn_lattice;

typedef struct {
  int64_t n_rows;
  const uint64_t* keys;   /* [n_rows] representatives, ascending Gauss index */
  const uint32_t* orbit;  /* [n_gauss] row | divisor index << 28 | sign << 31, or 0xFFFFFFFF */
} edg_zn_basis;

/* Number of 64-bit bitmap words over the Gauss index range. */
int64_t edg_zn_bitmap_words(const edg_zn_lattice* L);
/* Marks the zero-momentum representatives (smallest key of their orbit, no
 * stabiliser element of sign -1): bitmap [words], counts [words] = popcount. */
int edg_zn_mark(const edg_zn_lattice* L, uint64_t* bitmap, int64_t* counts, cudaStream_t stream);
/* keys[offsets[w] + j] = the j-th representative of word w (offsets: exclusive scan of counts). */
int edg_zn_fill(const edg_zn_lattice* L, const uint64_t* bitmap, const int64_t* offsets,
                uint64_t* keys, cudaStream_t stream);
/* orbit[gidx(T_g r)] = (row of r, stabiliser size, sign of T_g on r) for all g;
 * 0xFFFFFFFF elsewhere.  n_rows < 2^28 - 1. */
int edg_zn_orbit_table(const edg_zn_lattice* L, const uint64_t* keys, int64_t n_rows,
                       uint32_t* orbit, cudaStream_t stream);
/* y = H x for nvec instances at once, x and y interleaved [row][nvec]
 * (dtype 0 f64, 1 f32; nvec 1, 2, 4 or 8); couplings [nvec][4] = (t, m,
 * g^2/2, -1/(2 g^2)) in device memory; f64 accumulation. */
int edg_zn_matvec(const edg_zn_lattice* L, const edg_zn_basis* B, const double* couplings,
                  int32_t nvec, int32_t dtype, const void* x, void* y, cudaStream_t stream);

/* ------------------------------------------------------------------------
 * Batched interleaved vectors: nvec instances stored [row][nvec], the total
 * element count n_elems a multiple of 4 with padding entries zero; basis
 * vector i at V + i * stride elements (stride a multiple of 4).
 * Building blocks of the thick-restart Lanczos that drives the matrix-free
 * matvec (scipy eigsh's role, qmb_hamiltonian.py:313).
 * ------------------------------------------------------------------------ */
int64_t edg_iv_scratch_elems(int64_t n_elems, int32_t m);
/* h[i * nvec + v] = sum over rows of V_i * w for instance v, i < m (f64). */
int edg_iv_dots(int32_t dtype, int64_t n_elems, int32_t nvec, const void* V, int64_t stride,
                int32_t m, const void* w, double* h, double* scratch, cudaStream_t stream);
/* w -= sum_i V_i h[i * nvec + v] per instance v. */
int edg_iv_update(int32_t dtype, int64_t n_elems, int32_t nvec, const void* V, int64_t stride,
                  int32_t m, const double* h, void* w, cudaStream_t stream);
/* Second Gram-Schmidt pass fused with the norm: w -= sum_i V_i h[i * nvec + v]
 * (i < m), then sq[v] = w . w per instance. */
int edg_iv_update_norm(int32_t dtype, int64_t n_elems, int32_t nvec, const void* V, int64_t stride,
                       int32_t m, const double* h, void* w, double* sq, double* scratch,
                       cudaStream_t stream);
/* Dots against two vectors in one read of the basis: h1[i * nvec + v] = V_i . x1,
 * h2[i * nvec + v] = V_i . x2 (i < m).  scratch: edg_iv_scratch_elems(n_elems, m). */
int edg_iv_dots2(int32_t dtype, int64_t n_elems, int32_t nvec, const void* V, int64_t stride,
                 int32_t m, const void* x1, const void* x2, double* h1, double* h2, double* scratch,
                 cudaStream_t stream);
/* One delayed classical Gram-Schmidt step (the second pass of the previous
 * vector lagged into this one), one read of V_0..V_{j-1}.  Inputs: hu = dots
 * of V_0..V_j with u = V_j (s = hu[0..j), alpha = hu[j]), hw = dots of
 * V_0..V_j with w (z = hw[0..j), omega = hw[j]).  Writes
 * V_j = (u - sum_i V_i s_i) / r with r = sqrt(alpha - s.s), then
 * w -= sum_i V_i z_i + V_j (omega - s.z) / r, and sq[v] = w . w.  j < 32. */
int edg_iv_dcgs_update(int32_t dtype, int64_t n_elems, int32_t nvec, void* V, int64_t stride,
                       int32_t j, const double* hu, const double* hw, void* w, double* sq,
                       double* scratch, cudaStream_t stream);
/* out = w / sqrt(sq[v]) per instance (0 where sq <= 0). */
int edg_iv_scale(int32_t dtype, int64_t n_elems, int32_t nvec, const void* w, const double* sq,
                 void* out, cudaStream_t stream);
/* In place, per row: V_q <- sum_{i<m} V_i S[v][i][q] for q < k (S device f64 [nvec][m][k]);
 * m <= 32, k <= m. */
int edg_iv_combine(int32_t dtype, int64_t n_elems, int32_t nvec, void* V, int64_t stride,
                   int32_t m, const double* S, int32_t k, cudaStream_t stream);
/* x = uniform(-1, 1) from (seed, element) for rows < n_rows, 0 in the padding. */
int edg_iv_random(int32_t dtype, int64_t n_rows, int64_t n_elems, int32_t nvec, uint64_t seed,
                  void* x, cudaStream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* EDGPU_H */
