/*
 * bclx — B200 (sm_100a) sparse tile multiply for BCL containers: the C ABI.
 *
 * This is the drop-in boundary under the BCL container API.  The reference
 * (berkeley-container-library/bcl) runs these operations as header-only C++
 * inside its SUMMA-style tile loop; every entry point below replaces one of
 * those local kernels (or the whole loop) with device-resident tiles and
 * hand-written CUDA kernels.  Paths are relative to the BCL tree.
 *
 *   bclx_spgemm_symbolic / _numeric   BCL::gemm(SPMatrix, SPMatrix, SPMatrix&)
 *                                     bcl/containers/algorithms/spgemm.hpp:182-242
 *                                     (a 1x1x1 grid is the local tile product
 *                                     CSRMatrix::dot -> gemm(CSR, CSR, CSR&),
 *                                     spgemm.hpp:41-76, CSRMatrix.hpp:229-235)
 *   bclx_tile_accumulate_*            SparseHashAccumulator::accumulate/get_matrix
 *                                     bcl/containers/sequential/SparseHashAccumulator.hpp:86-183
 *   bclx_spmm_tile                    spmm_wrapper(m, n, k, nnz, c, b, vals, rowptr,
 *                                     colind, ldb, ldc), spgemm.hpp:140-149 (80-96)
 *   bclx_spmm_grid                    BCL::gemm(SPMatrix, DMatrix, DMatrix&)
 *                                     spgemm.hpp:153-179
 *   bclx_spmm_grid_sub                one process's C tiles of that product
 *                                     (the same loop under c.tile_rank)
 *   bclx_csr_to_tiles                 SPMatrix(fname, blocking) slicing,
 *                                     SPMatrix.hpp:194-271
 *   bclx_tiles_to_csr                 SPMatrix::get, SPMatrix.hpp:516-546
 *
 * Semantics kept from the reference:
 *   - output structure is the symbolic pattern (entries that sum to zero are
 *     kept), columns sorted within each row (CSRMatrix.hpp:107-165);
 *   - per output entry, a tile product sums from 0 in stored A-row order with
 *     fused multiply-adds; C tile (i, j) adds its partial products for
 *     k = (k_ + i + j) mod G, k_ = 0..G-1, in that order (spgemm.hpp:204-224,
 *     SimpleHash.hpp:88-119).  FP32 results are therefore bit-identical to
 *     the reference CPU build (which contracts `c += a*b` to an FMA), and
 *     int32 results are exact;
 *   - SpMM accumulates into C in place (beta = 1), C tiles in rotated k order.
 *
 * Conventions: all matrix pointers are DEVICE pointers; index arrays are
 * int32 (the reference's default index type); row_ptr holds m+1 entries.
 * No exceptions cross this boundary: every call returns a bclx_status_t
 * (the C++ layer in include/bclx/ turns errors into std::runtime_error, as
 * the reference does for bad shapes and out-of-memory).  Calls on one context
 * are ordered on the context's stream and are not thread-safe against each
 * other; distinct contexts are independent.
 */
#ifndef BCLX_H
#define BCLX_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define BCLX_API __attribute__((visibility("default")))
#else
#define BCLX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  BCLX_OK = 0,
  BCLX_ERR_INVALID = 1,         /* bad argument or shape mismatch */
  BCLX_ERR_DTYPE = 2,           /* unsupported value type for this call */
  BCLX_ERR_CUDA = 3,            /* a CUDA runtime call failed (see bclx_last_error) */
  BCLX_ERR_NO_MEMORY = 4,       /* device allocation failed */
  BCLX_ERR_INDEX_OVERFLOW = 5,  /* a tile's nnz does not fit the int32 index type */
  BCLX_ERR_DEVICE_TIMEOUT = 6,  /* reserved for a bounded device-side wait that gives up; no kernel of
                                   this library waits on a flag set by another kernel, so none returns it */
  BCLX_ERR_NO_DEVICE = 7        /* no usable sm_100 device */
} bclx_status_t;

typedef enum {
  BCLX_F32 = 0,   /* float */
  BCLX_I32 = 1,   /* int32_t */
  BCLX_BF16 = 2   /* bfloat16 storage (SpMM B and C only) */
} bclx_dtype_t;

/* One CSR tile (CSRMatrix<T, int>): m x n, nnz entries, device pointers. */
typedef struct {
  int64_t m, n, nnz;
  int32_t* row_ptr; /* [m+1] */
  int32_t* col_ind; /* [nnz], tile-local columns, sorted per row */
  void* vals;       /* [nnz] of dtype */
  int32_t dtype;
  int32_t pad_;
} bclx_csr_t;

/* A tile grid of CSR tiles (SPMatrix<T, int>): tile (i, j) holds rows
 * [i*tile_m, min((i+1)*tile_m, m)) and columns [j*tile_n, min(.., n)),
 * as in SPMatrix::tile_shape(index) (SPMatrix.hpp:401-405).
 * `tiles` is a DEVICE array of grid_m*grid_n descriptors, row-major. */
typedef struct {
  int64_t m, n;
  int64_t tile_m, tile_n;
  int64_t grid_m, grid_n;
  const bclx_csr_t* tiles;
  int32_t dtype;
  int32_t pad_;
} bclx_spgrid_t;

/* Output tile grid of a sparse product, packed in one allocation per array:
 * tile t = i*grid_n + j owns entries [tile_offset[t], tile_offset[t+1]) of
 * col_ind/vals, and its local row_ptr is tile_row_ptr + t*(tile_m+1)
 * (edge tiles repeat their nnz past their last row). */
typedef struct {
  int64_t m, n;
  int64_t tile_m, tile_n;
  int64_t grid_m, grid_n;
  int32_t* tile_row_ptr; /* [grid_m*grid_n*(tile_m+1)], written by symbolic */
  int64_t* tile_offset;  /* [grid_m*grid_n+1], written by symbolic */
  int32_t* col_ind;      /* [nnz], written by numeric */
  void* vals;            /* [nnz], written by numeric */
  int32_t dtype;
  int32_t pad_;
} bclx_spgrid_out_t;

/* A tile grid of dense tiles (DMatrix<T>): every tile is a row-major
 * tile_m x tile_n block with leading dimension tile_n, padded to full size
 * even at the edges (DMatrix.hpp:55-95, 151-173).  `tiles` is a DEVICE array
 * of grid_m*grid_n base pointers, row-major. */
typedef struct {
  int64_t m, n;
  int64_t tile_m, tile_n;
  int64_t grid_m, grid_n;
  void* const* tiles;
  int32_t dtype;
  int32_t pad_;
} bclx_dgrid_t;

typedef struct bclx_context_s* bclx_context_t;
typedef struct bclx_spgemm_plan_s* bclx_spgemm_plan_t;

/* ---- context: device, stream, stream-ordered scratch pool ------------- */
/* Replaces the backend/segment set-up of BCL::init (backends/mpi/backend.hpp:78-118):
 * one context per device; scratch comes from a stream-ordered pool. */
BCLX_API int bclx_context_create(int device, bclx_context_t* ctx);
BCLX_API int bclx_context_destroy(bclx_context_t ctx);
/* Use `stream` (a cudaStream_t; NULL = legacy default) for every later call. */
BCLX_API int bclx_context_set_stream(bclx_context_t ctx, void* stream);
BCLX_API int bclx_context_synchronize(bclx_context_t ctx);
/* Wait for the context's stream, then return the scratch pool's cached
 * device memory to the driver (the pool keeps freed scratch for reuse).
 * Counterpart of freeing a BCL segment (BCL::finalize, backends/mpi/backend.hpp:120-130). */
BCLX_API int bclx_context_release_cached(bclx_context_t ctx);
/* Tuning knobs of a context, read by the later calls on it (no reference
 * counterpart; the autotuner, bcl_b200/autotune.py, searches them).  A value
 * below 0 restores the default; out-of-range values are BCLX_ERR_INVALID. */
typedef enum {
  BCLX_TUNE_LIGHT_UB = 0,          /* SpGEMM: a row with at most this many products is light (32..512; 512) */
  BCLX_TUNE_LEARN_TARGET = 1,      /* learned product: outputs aimed at per heavy item (64..448; 320) */
  BCLX_TUNE_BTABLE_MAX_BYTES = 2,  /* SpGEMM: largest B-row table built (0..; 2 GiB, or BCLX_BTABLE_MAX_BYTES) */
  BCLX_TUNE_SPMM_ROWS = 3,         /* SpMM: rows per warp item (0 = by product size, 1, 2, 4) */
  BCLX_TUNE_SPMM_LONG_ROW = 4,     /* SpMM: entries from which a row goes to the long-row kernel (0 = 512 FP32 / 1024 BF16, 64..) */
  BCLX_TUNE_SPMM_LONG_BLOCKS = 5,  /* SpMM: blocks of the long-row kernel (0 = a quarter of the SMs per panel up to half, 1..SMs) */
  BCLX_TUNE_SPMM_SCHEDULE = 6,     /* SpMM: 0 = long rows on the side stream, 1 = dependent launch (0 or 1; 0) */
  BCLX_TUNE_ITEM_OUTPUTS = 7,      /* SpGEMM: outputs per heavy-row work item (512 or 1024; 512) */
  BCLX_TUNE_WIDE_LIGHT = 8,        /* SpGEMM: 1 = rows of tiles wider than 8192 columns may be light (0 or 1; 0) */
  BCLX_TUNE_SPMM_PANEL_MAJOR = 9,  /* SpMM: 1 = every row's first column panel before any row's second (0 or 1; 0) */
  BCLX_TUNE_KEYS = 10
} bclx_tune_key_t;
BCLX_API int bclx_context_set_tuning(bclx_context_t ctx, int32_t key, int64_t value);
BCLX_API int bclx_context_get_tuning(bclx_context_t ctx, int32_t key, int64_t* value);
/* Text of the last CUDA error seen on this thread (empty if none). */
BCLX_API const char* bclx_last_error(void);
/* Library version, e.g. 100 for 0.1.0. */
BCLX_API int bclx_version(void);
/* Number of CUDA kernels this library has launched in this process (no
 * reference counterpart; used for launch accounting in benchmarks). */
BCLX_API long long bclx_launch_count(void);

/* ---- sparse x sparse ---------------------------------------------------
 * C = A * B over tile grids: A is m x k with grid (gm x gk), B is k x n with
 * grid (gk x gn), C is m x n with grid (gm x gn); A's tile_n must equal B's
 * tile_m, C's tile_m/tile_n must equal A's tile_m / B's tile_n
 * (BCL::gemm(SPMatrix, SPMatrix, SPMatrix&), spgemm.hpp:182-242).
 *
 * Two phases.  symbolic sizes every output row (the union of all partial
 * products of the row's tile), writes c->tile_row_ptr and c->tile_offset,
 * returns the total nnz in *nnz (one device->host read) and a plan that holds
 * the work decomposition.  The caller then provides c->col_ind and c->vals of
 * that size, and numeric fills them.  numeric may run the SUMMA stages
 * k_ in [stage_begin, stage_end) only: stage_begin == 0 starts C from zero,
 * later ranges add onto the values already in c->vals, so running the stages
 * one call at a time gives bit-identical results to one call over all of them
 * (stage_end <= 0 means all stages). */
BCLX_API int bclx_spgemm_symbolic(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                         bclx_spgrid_out_t* c, bclx_spgemm_plan_t* plan, int64_t* nnz);
BCLX_API int bclx_spgemm_numeric(bclx_context_t ctx, bclx_spgemm_plan_t plan, const bclx_spgrid_t* a,
                        const bclx_spgrid_t* b, bclx_spgrid_out_t* c, int32_t stage_begin,
                        int32_t stage_end);
BCLX_API int bclx_spgemm_plan_destroy(bclx_spgemm_plan_t plan);
/* A sub-grid of C's tiles, as one process of the reference's distributed
 * loop computes its own C tiles (stationary C, spgemm.hpp:194-224, with
 * tile (i, j) owned by process (j mod pn) + (i mod pm) * pn,
 * SPMatrix.hpp:230-237): c is the grid_m x grid_n block of C tiles whose
 * global tile rows / columns are tile_rows[0..grid_m) / tile_cols[0..grid_n)
 * (host arrays, increasing); a holds A's tiles of those tile rows (all k),
 * b holds B's tiles of those tile columns (all k), in that order, as
 * descriptor arrays (a sub-grid view: no copy).  Every C tile keeps the
 * global product's stage order k = (k_ + i + j) mod G with its global
 * (i, j), so the sub-grid is bit-identical to those tiles of the whole
 * product.  Then bclx_spgemm_numeric as usual. */
BCLX_API int bclx_spgemm_symbolic_sub(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                                      bclx_spgrid_out_t* c, const int64_t* tile_rows, const int64_t* tile_cols,
                                      bclx_spgemm_plan_t* plan, int64_t* nnz);
/* Batched SUMMA form: the numeric pass as one launch per stage k_ (each launch
 * covers all grid_m*grid_n tile products of that stage, adding into C), in
 * order.  use_graph = 1 captures the G launches once into a CUDA graph kept
 * by the plan and replays it on later calls with the same plan, grids and
 * output arrays (a replay recomputes the values for the same structure; the
 * call that captures also computes C).  Bit-identical to bclx_spgemm_numeric.
 * The batched stage loop has no single reference counterpart; it runs the
 * stages of spgemm.hpp:209-224 for all C tiles at once. */
BCLX_API int bclx_spgemm_numeric_staged(bclx_context_t ctx, bclx_spgemm_plan_t plan, const bclx_spgrid_t* a,
                                        const bclx_spgrid_t* b, bclx_spgrid_out_t* c, int32_t use_graph);
/* Numeric-pass tuning of a plan: grab = work items a warp takes from the
 * device work queue at a time (1..64), blocks_per_sm (1..4), long_seg = B
 * segments of at least this many products are walked lane-parallel.  Chosen
 * by the autotuner (bcl_b200/autotune.py); no reference counterpart. */
BCLX_API int bclx_spgemm_plan_tune(bclx_spgemm_plan_t plan, int32_t grab, int32_t blocks_per_sm,
                                   int32_t long_seg);
/* Plan statistics: [0] intermediate products, [1] row items, [2] work items,
 * [3] work items in the large-accumulator class, [4] stages, [5] output nnz. */
BCLX_API int bclx_spgemm_plan_stats(bclx_spgemm_plan_t plan, int64_t* out6);

/* ---- learned product --------------------------------------------------------
 * The same product without a separate symbolic pass: a row-nnz predictor
 * (bclx_mlp_*) sizes the work.  run: classifies rows and computes their
 * features, predicts each heavy row's output count, cuts heavy rows into
 * column items from the prediction, runs one numeric pass that also builds
 * every item's structure (outputs to plan-owned temp slots), redoes every row
 * with an item whose real count exceeded the accumulator by the exact
 * two-phase path, and writes c->tile_row_ptr / tile_offset and *nnz.  The
 * caller then provides c->col_ind / c->vals and finish compacts the result
 * into them.  Output bit-identical to bclx_spgemm_symbolic/_numeric.
 * mlp_params: device array of bclx_mlp_num_params() floats, or NULL to size
 * items from the product count (an upper bound) instead of a prediction.
 * Destroy the plan with bclx_spgemm_plan_destroy.  No reference counterpart
 * (the reference has no predictor); it replaces spgemm.hpp:182-242 as the
 * symbolic/numeric pair does. */
BCLX_API int bclx_spgemm_learned_run(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                                     bclx_spgrid_out_t* c, const float* mlp_params, bclx_spgemm_plan_t* plan,
                                     int64_t* nnz);
BCLX_API int bclx_spgemm_learned_finish(bclx_context_t ctx, bclx_spgemm_plan_t plan, bclx_spgrid_out_t* c);
/* The learned product of a sub-grid of C's tiles (tile_rows / tile_cols as
 * in bclx_spgemm_symbolic_sub): a process's own C tiles, or one block of C
 * tile rows of a product whose temporary slots would not fit beside the
 * whole C (the blocks are computed and kept one after another).  Then
 * bclx_spgemm_learned_finish. */
BCLX_API int bclx_spgemm_learned_run_sub(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                                         bclx_spgrid_out_t* c, const int64_t* tile_rows, const int64_t* tile_cols,
                                         const float* mlp_params, bclx_spgemm_plan_t* plan, int64_t* nnz);
/* [0] heavy rows, [1] predicted heavy items, [2] rows redone exactly
 * (mispredictions), [3] temp entries allocated, [4] nnz, [5] redo items. */
BCLX_API int bclx_spgemm_learned_stats(bclx_spgemm_plan_t plan, int64_t* out6);
/* Per C-tile row (grid_m*grid_n*tile_m rows, tile-major): the predictor's
 * features X[row*5 + 0..4] (log2(1+A-row nnz), log2(1+products),
 * log2(1+longest referenced B row), tile-row and tile-column coordinate in
 * (0,1)) and the product count ub[row] (device arrays). */
BCLX_API int bclx_spgemm_row_features(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                                      const bclx_spgrid_out_t* c, float* X, int32_t* ub);
/* The exact per-row output counts of a symbolic plan (device array of
 * grid_m*grid_n*tile_m int32): the predictor's training targets. */
BCLX_API int bclx_spgemm_plan_row_counts(bclx_spgemm_plan_t plan, int32_t* counts);

/* ---- row-nnz predictor: 5 -> 64 -> 64 -> 1 MLP (ReLU, FP32) -------------------
 * No reference counterpart.  Parameters: device float array of
 * bclx_mlp_num_params() values, layout W1[5][64] b1[64] W2[64][64] b2[64]
 * w3[64] b3.  X: device [n][5]; y: device [n] targets log2(1 + row nnz). */
BCLX_API int bclx_mlp_num_params(void);
BCLX_API int bclx_mlp_predict(bclx_context_t ctx, const float* X, int64_t n, const float* params, float* out);
/* grad[0..P) = dL/dparams of L = mean (yhat - y)^2, grad[P] = sum of squared errors. */
BCLX_API int bclx_mlp_gradient(bclx_context_t ctx, const float* X, const float* y, int64_t n, const float* params,
                               float* grad);
/* `steps` full-batch Adam steps on (X, y) from `params` (updated in place);
 * loss_host (host, may be NULL) receives the loss before each step. */
BCLX_API int bclx_mlp_train(bclx_context_t ctx, const float* X, const float* y, int64_t n, float* params,
                            int32_t steps, float lr, float* loss_host);

/* ---- tile accumulation ---------------------------------------------------
 * C = parts[0] + parts[1] + ... (all m x n), per entry summed in list order
 * from 0, union structure (SparseHashAccumulator::get_matrix,
 * SparseHashAccumulator.hpp:101-182).  `parts` is a DEVICE array of nparts
 * descriptors.  symbolic writes c_row_ptr[m+1] and returns *nnz; numeric
 * fills c->col_ind / c->vals (c->row_ptr = the same c_row_ptr). */
BCLX_API int bclx_tile_accumulate_symbolic(bclx_context_t ctx, const bclx_csr_t* parts, int32_t nparts,
                                  int64_t m, int64_t n, int32_t dtype, int32_t* c_row_ptr,
                                  bclx_spgemm_plan_t* plan, int64_t* nnz);
BCLX_API int bclx_tile_accumulate_numeric(bclx_context_t ctx, bclx_spgemm_plan_t plan, const bclx_csr_t* parts,
                                 int32_t nparts, bclx_csr_t* c);

/* ---- one tile pair, without allocating -----------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory when they call (a framework that has
 * reserved the device's memory for its own allocator, or code that must not
 * call cudaMalloc/cudaFree because they synchronize the device).
 * C = A * B for one pair of CSR tiles (A m x k, B k x n, both BCLX_F32 or both
 * BCLX_I32; host structs holding device pointers), with the same results as
 * bclx_spgemm_symbolic/_numeric on 1x1 grids.  The caller provides
 * c_row_ptr[m+1] and c_col_ind/c_vals with room for c_capacity entries; the
 * call writes c_row_ptr and *c_nnz, and returns BCLX_ERR_INVALID without
 * touching c_col_ind/c_vals when *c_nnz > c_capacity (retry with more room).
 * No cudaMalloc/cudaFree: all work arrays come from a 32 MiB device array
 * that the library holds on every GPU it runs on; a tile product that needs
 * more (or B wider than 16384 columns) is rejected with BCLX_ERR_INVALID and
 * nothing written to c_col_ind/c_vals.  The first call on a device looks that
 * array up (cudaGetSymbolAddress) and should come before any stream capture.
 * Calls share the array and each clears the parts that must start at zero:
 * calls whose work overlaps on the GPU (different streams) race.  Runs on
 * `stream` on the current device.  The host reads sizes back twice (after
 * the row classification and after the row counts), synchronizing `stream`
 * each time; the values are ready when the stream reaches the end of the
 * call.  m == 0, k == 0 or n == 0 writes an all-zero c_row_ptr. */
BCLX_API int bclx_spgemm_tile_noalloc(const bclx_csr_t* a, const bclx_csr_t* b, int32_t* c_row_ptr,
                                      int32_t* c_col_ind, void* c_vals, int64_t c_capacity, int64_t* c_nnz,
                                      void* stream);

/* ---- whole matrix <-> tile grid ---------------------------------------------
 * Slice a CSR matrix (device arrays, columns ascending within each row, as
 * CSRMatrix holds them) into the packed tile layout of `out` (m, n,
 * tile_m, tile_n, grid_m, grid_n and all four arrays set by the caller;
 * col_ind and vals hold a->nnz entries; dtype F32 or I32).  Replaces the
 * SPMatrix(fname, blocking) constructor's slicing (SPMatrix.hpp:194-271,
 * CSRMatrix::get_slice_impl_ CSRMatrix.hpp:238-276), done on the device.
 * Rows whose columns are not ascending or out of range: BCLX_ERR_INVALID,
 * nothing written to col_ind/vals.  Synchronizes the context's stream. */
BCLX_API int bclx_csr_to_tiles(bclx_context_t ctx, const bclx_csr_t* a, bclx_spgrid_out_t* out);
/* Gather every tile of `g` into one CSR matrix: row_ptr [m+1], col_ind and
 * vals [nnz] (nnz = sum of tile nnz), global columns, each row's tiles in
 * column order.  Replaces SPMatrix::get (SPMatrix.hpp:516-546), on the
 * device; FP32 values come back as that call returns them (it adds each to
 * 0 in a SparseHashAccumulator: -0.0 becomes +0.0, a signalling NaN becomes
 * quiet).  Reads nnz back once (synchronizes). */
BCLX_API int bclx_tiles_to_csr(bclx_context_t ctx, const bclx_spgrid_t* g, int32_t* row_ptr, int32_t* col_ind,
                               void* vals);

/* ---- sparse x dense ------------------------------------------------------
 * C += A * B for one tile (spmm_wrapper, spgemm.hpp:140-149): A is m x k CSR
 * (FP32 values), B is k x n row-major with leading dimension ldb, C is m x n
 * row-major with leading dimension ldc.  bc_dtype: BCLX_F32 (bit-identical to
 * the reference), or BCLX_BF16 (B and C stored as bfloat16, products chained
 * in FP32 and each C row rounded once). */
BCLX_API int bclx_spmm_tile(bclx_context_t ctx, int64_t m, int64_t n, int64_t k, int64_t nnz, void* c,
                   const void* b, const float* a_values, const int32_t* a_rowptr,
                   const int32_t* a_colind, int64_t ldb, int64_t ldc, int32_t bc_dtype);
/* C += A * B over tile grids, every C tile over all k in rotated order, in
 * one launch (BCL::gemm(SPMatrix, DMatrix, DMatrix&), spgemm.hpp:153-179).
 * b->dtype == c->dtype selects FP32 or BF16 storage. */
BCLX_API int bclx_spmm_grid(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_dgrid_t* b,
                   const bclx_dgrid_t* c);
/* The C tiles (tile_rows[x], tile_cols[y]) of a larger product C += A * B,
 * in one launch: what one process of the reference's stationary-C loop
 * computes (spgemm.hpp:153-179 with c.tile_rank({i, j}) == rank; the GPU
 * driver cuda/algorithms/spmm.hpp:20-115).  `c` is the grid of those tiles
 * (grid_m = number of tile_rows, grid_n = number of tile_cols), `a` holds
 * A's tile rows tile_rows over every k, `b` B's tile columns tile_cols over
 * every k (grids of gathered tile pointers or compact copies).  Each C tile
 * takes the k tiles in the rotated order of its global position,
 * k = (k_ + tile_rows[x] + tile_cols[y]) mod G, so it is bit-identical to
 * that tile of bclx_spmm_grid on the whole grids.  tile_rows / tile_cols:
 * host arrays of global tile indices, increasing (only the last can be a
 * ragged edge tile), else BCLX_ERR_INVALID.  Copies the two index maps to
 * the device (synchronizes the context's stream once). */
BCLX_API int bclx_spmm_grid_sub(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_dgrid_t* b,
                                const bclx_dgrid_t* c, const int64_t* tile_rows, const int64_t* tile_cols);
/* The row-wise variants rowwise_gemm / cached_rowwise_gemm /
 * batched_rowwise_gemm (bcl/containers/algorithms/experimental_gemm.hpp:
 * 83-214): C += A * B with C in one tile column (c->grid_n == 1, else
 * BCLX_ERR_INVALID) and each C tile row taking the k tiles in ascending
 * order (all three variants give these sums: the cache only changes how
 * B rows are fetched, the batched sort only reorders entries of different
 * rows).  Same tile-grid rules and dtypes as bclx_spmm_grid. */
BCLX_API int bclx_spmm_grid_rowwise(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_dgrid_t* b,
                                    const bclx_dgrid_t* c);

/* ---- dense and elementwise container operations -------------------------
 * DMatrix::sum (DMatrix.hpp:537-554): the sum of every element of the
 * grid's tiles (padding excluded), written to *result_host (float for
 * BCLX_F32 and BCLX_BF16 storage, int32_t for BCLX_I32).  int32: the exact
 * sum modulo 2^32 (what the reference's int accumulator wraps to).  Floating
 * point: accumulated in FP64 on the device and rounded once to FP32; the
 * reference adds in tile, row, column order in FP32, so the two agree within
 * that sequential sum's own rounding error (|error| <= (n-1) u sum |x|,
 * u = 2^-24).  Synchronizes the context's stream. */
BCLX_API int bclx_dmatrix_sum(bclx_context_t ctx, const bclx_dgrid_t* a, void* result_host);

/* SPMatrix::binary_op_inplace(DMatrix other, fn) (SPMatrix.hpp:571-616):
 * every stored entry a(i, j) of the sparse grid becomes op(a(i, j), b(i, j)),
 * b read at the same global (i, j) through its own tile grid (any blocking:
 * the reference's same-layout and sliced branches give the same result).
 * Values FP32 (b F32) or int32 (b I32).  The structure is unchanged. */
typedef enum {
  BCLX_OP_PLUS = 0,        /* a + b   (std::plus)       */
  BCLX_OP_MINUS = 1,       /* a - b   (std::minus)      */
  BCLX_OP_MULTIPLIES = 2,  /* a * b   (std::multiplies) */
  BCLX_OP_DIVIDES = 3,     /* a / b   (std::divides; int32: b == 0 gives 0) */
  BCLX_OP_MIN = 4,         /* b < a ? b : a (std::min)  */
  BCLX_OP_MAX = 5,         /* a < b ? b : a (std::max)  */
  BCLX_OP_SECOND = 6       /* b (assignment)            */
} bclx_binary_op_t;
BCLX_API int bclx_spmatrix_binary_op(bclx_context_t ctx, const bclx_spgrid_t* a, const bclx_dgrid_t* b, int32_t op);

#ifdef __cplusplus
}
#endif

#endif /* BCLX_H */
