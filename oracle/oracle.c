/*
 * CPU restatement of the reference's sparse tile multiply — TEST
 * INFRASTRUCTURE ONLY (the checker for the CUDA path; never shipped or timed
 * as the product).
 *
 * Pinned against the reference itself: tests compare every function below
 * bit-for-bit with oracle/_ref/bcl_ref, the reference's unmodified CPU code
 * built from its headers, and against the committed golden fixtures that
 * tests/golden/make_golden.py produced from it.
 *
 * What it restates (reference paths relative to the BCL tree):
 *
 *  - Local SpGEMM, bcl/containers/algorithms/spgemm.hpp:41-76 with the output
 *    assembly of bcl/containers/sequential/CSRMatrix.hpp:107-165.  Row by row
 *    (Gustavson): every output entry starts at T{} = 0 and takes
 *    `c += a_ik * b_kj` in stored A-row order, then within the stored B-row
 *    order.  Entries whose sum is zero are kept (the map never drops keys);
 *    columns are sorted.  With a contracting compiler (`-ffp-contract=fast`,
 *    GCC's default for GNU C++ with FMA available) `c += a*b` is one fused
 *    multiply-add; `use_fma` selects that (1) or the separately rounded form (0).
 *
 *  - Tile accumulation, bcl/containers/sequential/SparseHashAccumulator.hpp:
 *    101-182 with SimpleHash.hpp:88-119: partial tiles are summed per entry
 *    in the order they were pushed, starting from T{} = 0 (`acc = acc + v`).
 *
 *  - The stationary-C SUMMA loop, spgemm.hpp:182-242: C tile (i, j) pushes
 *    the partial products A_ik * B_kj for k = (k_ + i + j) mod G,
 *    k_ = 0 .. G-1, G = number of tile columns of A; the partials are then
 *    accumulated as above.
 *
 *  - SpMM, spgemm.hpp:80-96 and 153-179: C[i, j] = C[i, j] + v * B[k, j] in
 *    stored A-row order, per C tile over k in the same rotated order, in
 *    place (beta = 1).
 *
 * FP64 variants accumulate FP32 inputs in double to state the error of the
 * FP32 (and BF16) results.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

/* ------------------------------------------------------------------------ */
/* Per-thread scratch: a dense sparse accumulator over the output columns.   */
/* ------------------------------------------------------------------------ */
typedef struct {
  unsigned char* seen;   /* n flags: column present in the accumulated row */
  unsigned char* pseen;  /* n flags: column touched by the current partial */
  int32_t* cols;         /* touched columns of the accumulated row */
  int32_t* pcols;        /* touched columns of the current partial */
  void* acc;             /* n values: accumulated row */
  void* part;            /* n values: current partial row */
} spa_t;

static void spa_init(spa_t* s, int64_t n, size_t vsize) {
  s->seen = (unsigned char*)calloc((size_t)n, 1);
  s->pseen = (unsigned char*)calloc((size_t)n, 1);
  s->cols = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  s->pcols = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  s->acc = calloc((size_t)(n > 0 ? n : 1), vsize);
  s->part = calloc((size_t)(n > 0 ? n : 1), vsize);
}

static void spa_free(spa_t* s) {
  free(s->seen); free(s->pseen); free(s->cols); free(s->pcols); free(s->acc); free(s->part);
}

/* Column-block start of every B row: bstart[r*(gn+1) + j] = first entry of
 * row r with column >= j*tn (B rows are sorted). */
static int64_t* block_starts(int64_t k, const int32_t* brp, const int32_t* bci, int64_t tn, int64_t gn) {
  int64_t* bs = (int64_t*)malloc(sizeof(int64_t) * (size_t)(k * (gn + 1) + 1));
  #pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < k; r++) {
    int64_t p = brp[r];
    for (int64_t j = 0; j <= gn; j++) {
      int64_t lim = j * tn;
      while (p < brp[r + 1] && bci[p] < lim) p++;
      bs[r * (gn + 1) + j] = (j == gn) ? brp[r + 1] : p;
    }
  }
  return bs;
}

/* ------------------------------------------------------------------------ */
/* Structure of C = A*B (symbolic; identical for tiled and untiled forms).    */
/* rows == NULL means all rows 0..m-1; counts[i] receives nnz of row rows[i]. */
/* Returns the total.                                                        */
/* ------------------------------------------------------------------------ */
int64_t oracle_spgemm_count(int64_t m, int64_t n, const int32_t* arp, const int32_t* aci,
                            const int32_t* brp, const int32_t* bci,
                            const int64_t* rows, int64_t nrows, int64_t* counts) {
  if (!rows) nrows = m;
  int64_t total = 0;
  #pragma omp parallel reduction(+ : total)
  {
    unsigned char* seen = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
    int32_t* list = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    #pragma omp for schedule(dynamic, 64)
    for (int64_t ii = 0; ii < nrows; ii++) {
      int64_t i = rows ? rows[ii] : ii;
      int64_t cnt = 0;
      for (int32_t p = arp[i]; p < arp[i + 1]; p++) {
        int32_t k = aci[p];
        for (int32_t q = brp[k]; q < brp[k + 1]; q++) {
          int32_t j = bci[q];
          if (!seen[j]) { seen[j] = 1; list[cnt++] = j; }
        }
      }
      for (int64_t t = 0; t < cnt; t++) seen[list[t]] = 0;
      counts[ii] = cnt;
      total += cnt;
    }
    free(seen); free(list);
  }
  return total;
}

/* ------------------------------------------------------------------------ */
/* Tiled SUMMA product, numeric.  A is m x K with tiles tm x tk, B is K x n   */
/* with tiles tk x tn, C tiles tm x tn.  offsets[ii] = output start of row    */
/* rows[ii] (prefix sum of the counts above).  Columns are global.           */
/* The same body is stamped out for float (FMA or not), int32 and double.   */
/* ------------------------------------------------------------------------ */
#define ORACLE_GEMM_TILED(NAME, VT, OT, UPDATE)                                                      \
  void NAME(int64_t m, int64_t K, int64_t n, const int32_t* arp, const int32_t* aci, const VT* av,   \
            const int32_t* brp, const int32_t* bci, const VT* bv, int64_t tm, int64_t tk, int64_t tn, \
            const int64_t* rows, int64_t nrows, const int64_t* offsets, int32_t* cci, OT* cv,        \
            int use_fma) {                                                                          \
    (void)use_fma;                                                                                  \
    if (!rows) nrows = m;                                                                           \
    int64_t gk = (K + tk - 1) / tk, gn = (n + tn - 1) / tn;                                         \
    if (gk < 1) gk = 1;                                                                             \
    int64_t* bs = block_starts(K, brp, bci, tn, gn);                                                \
    _Pragma("omp parallel")                                                                         \
    {                                                                                               \
      spa_t s;                                                                                      \
      spa_init(&s, n, sizeof(OT));                                                                  \
      OT* acc = (OT*)s.acc;                                                                         \
      OT* part = (OT*)s.part;                                                                       \
      int64_t* akstart = (int64_t*)malloc(sizeof(int64_t) * (size_t)(gk + 1));                      \
      _Pragma("omp for schedule(dynamic, 16)")                                                      \
      for (int64_t ii = 0; ii < nrows; ii++) {                                                      \
        int64_t r = rows ? rows[ii] : ii;                                                           \
        int64_t ti = r / tm;                                                                        \
        /* split A row r by k block (columns sorted) */                                             \
        int64_t p = arp[r];                                                                         \
        for (int64_t kb = 0; kb <= gk; kb++) {                                                      \
          int64_t lim = kb * tk;                                                                    \
          while (p < arp[r + 1] && aci[p] < lim) p++;                                               \
          akstart[kb] = (kb == gk) ? arp[r + 1] : p;                                                \
        }                                                                                           \
        int64_t ncols = 0;                                                                          \
        for (int64_t tj = 0; tj < gn; tj++) {                                                       \
          for (int64_t kk = 0; kk < gk; kk++) {                                                     \
            int64_t kb = (kk + ti + tj) % gk;                                                       \
            int64_t np = 0;                                                                         \
            for (int64_t pa = akstart[kb]; pa < akstart[kb + 1]; pa++) {                            \
              int32_t k = aci[pa];                                                                  \
              OT a = (OT)av[pa];                                                                    \
              for (int64_t q = bs[k * (gn + 1) + tj]; q < bs[k * (gn + 1) + tj + 1]; q++) {         \
                int32_t j = bci[q];                                                                 \
                OT b = (OT)bv[q];                                                                   \
                if (!s.pseen[j]) { s.pseen[j] = 1; s.pcols[np++] = j; part[j] = (OT)0; }            \
                UPDATE;                                                                             \
              }                                                                                     \
            }                                                                                       \
            /* accumulate the partial tile row in push order: acc = acc + v */                      \
            for (int64_t t = 0; t < np; t++) {                                                      \
              int32_t j = s.pcols[t];                                                               \
              s.pseen[j] = 0;                                                                       \
              if (!s.seen[j]) { s.seen[j] = 1; s.cols[ncols++] = j; acc[j] = (OT)0; }               \
              acc[j] = acc[j] + part[j];                                                            \
            }                                                                                       \
          }                                                                                         \
        }                                                                                           \
        qsort(s.cols, (size_t)ncols, sizeof(int32_t), cmp_i32);                                     \
        int64_t o = offsets[ii];                                                                    \
        for (int64_t t = 0; t < ncols; t++) {                                                       \
          int32_t j = s.cols[t];                                                                    \
          cci[o + t] = j;                                                                           \
          cv[o + t] = acc[j];                                                                       \
          s.seen[j] = 0;                                                                            \
        }                                                                                           \
      }                                                                                             \
      free(akstart);                                                                                \
      spa_free(&s);                                                                                 \
    }                                                                                               \
    free(bs);                                                                                       \
  }

ORACLE_GEMM_TILED(oracle_gemm_tiled_f32, float, float,
                  part[j] = use_fma ? fmaf(a, b, part[j]) : (float)(part[j] + (float)(a * b)))
ORACLE_GEMM_TILED(oracle_gemm_tiled_i32, int32_t, int32_t,
                  part[j] = (int32_t)((uint32_t)part[j] + (uint32_t)a * (uint32_t)b))
ORACLE_GEMM_TILED(oracle_gemm_tiled_f64, float, double, part[j] = part[j] + a * b)

/* ------------------------------------------------------------------------ */
/* Tile accumulation of P partial CSRs (all m x n), summed in list order.     */
/* Two calls: count (row nnz of the union), then fill at offsets.            */
/* ------------------------------------------------------------------------ */
int64_t oracle_accumulate_count(int64_t m, int64_t n, int64_t nparts, const int32_t* const* rps,
                                const int32_t* const* cis, int64_t* counts) {
  int64_t total = 0;
  #pragma omp parallel reduction(+ : total)
  {
    unsigned char* seen = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);
    int32_t* list = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    #pragma omp for schedule(dynamic, 256)
    for (int64_t i = 0; i < m; i++) {
      int64_t cnt = 0;
      for (int64_t t = 0; t < nparts; t++)
        for (int32_t p = rps[t][i]; p < rps[t][i + 1]; p++) {
          int32_t j = cis[t][p];
          if (!seen[j]) { seen[j] = 1; list[cnt++] = j; }
        }
      for (int64_t q = 0; q < cnt; q++) seen[list[q]] = 0;
      counts[i] = cnt;
      total += cnt;
    }
    free(seen); free(list);
  }
  return total;
}

#define ORACLE_ACCUMULATE(NAME, VT)                                                                  \
  void NAME(int64_t m, int64_t n, int64_t nparts, const int32_t* const* rps, const int32_t* const* cis, \
            const VT* const* vs, const int64_t* offsets, int32_t* cci, VT* cv) {                       \
    _Pragma("omp parallel")                                                                          \
    {                                                                                                \
      unsigned char* seen = (unsigned char*)calloc((size_t)(n > 0 ? n : 1), 1);                      \
      int32_t* list = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));                   \
      VT* acc = (VT*)calloc((size_t)(n > 0 ? n : 1), sizeof(VT));                                    \
      _Pragma("omp for schedule(dynamic, 256)")                                                      \
      for (int64_t i = 0; i < m; i++) {                                                              \
        int64_t cnt = 0;                                                                             \
        for (int64_t t = 0; t < nparts; t++)                                                         \
          for (int32_t p = rps[t][i]; p < rps[t][i + 1]; p++) {                                      \
            int32_t j = cis[t][p];                                                                   \
            if (!seen[j]) { seen[j] = 1; list[cnt++] = j; acc[j] = (VT)0; }                          \
            acc[j] = acc[j] + vs[t][p];                                                              \
          }                                                                                          \
        qsort(list, (size_t)cnt, sizeof(int32_t), cmp_i32);                                          \
        for (int64_t q = 0; q < cnt; q++) {                                                          \
          cci[offsets[i] + q] = list[q];                                                             \
          cv[offsets[i] + q] = acc[list[q]];                                                         \
          seen[list[q]] = 0;                                                                         \
        }                                                                                            \
      }                                                                                              \
      free(seen); free(list); free(acc);                                                             \
    }                                                                                                \
  }

ORACLE_ACCUMULATE(oracle_accumulate_f32, float)
ORACLE_ACCUMULATE(oracle_accumulate_i32, int32_t)

/* ------------------------------------------------------------------------ */
/* SpMM, tiled and in place: C (m x N, row-major, ldc) += A (m x K CSR) * B   */
/* (K x N, row-major, ldb).  Tiles tm x tk (A), tk x tn (B), tm x tn (C);     */
/* per C tile the k blocks run in rotated order.  rows == NULL: all rows.     */
/* For the rows subset form, C points at an nrows x N block (row ii).         */
/* ------------------------------------------------------------------------ */
/* natural = 0: the SUMMA loop's rotated stage order; natural = 1: stages in
 * ascending k, the order of rowwise_gemm / cached_rowwise_gemm /
 * batched_rowwise_gemm (experimental_gemm.hpp:83-214: for k, for each A
 * entry of the row in stored order, local_c[..] += row[j_]*value, an FMA
 * with the same operands). */
static void spmm_tiled_f32_impl(int64_t m, int64_t K, int64_t N, const int32_t* arp, const int32_t* aci,
                                const float* av, const float* b, int64_t ldb, float* c, int64_t ldc,
                                int64_t tm, int64_t tk, int64_t tn, const int64_t* rows, int64_t nrows,
                                int use_fma, int natural) {
  if (!rows) nrows = m;
  int64_t gk = (K + tk - 1) / tk, gn = (N + tn - 1) / tn;
  if (gk < 1) gk = 1;
  #pragma omp parallel
  {
    int64_t* akstart = (int64_t*)malloc(sizeof(int64_t) * (size_t)(gk + 1));
    #pragma omp for schedule(dynamic, 16)
    for (int64_t ii = 0; ii < nrows; ii++) {
      int64_t r = rows ? rows[ii] : ii;
      int64_t ti = r / tm;
      int64_t p = arp[r];
      for (int64_t kb = 0; kb <= gk; kb++) {
        int64_t lim = kb * tk;
        while (p < arp[r + 1] && aci[p] < lim) p++;
        akstart[kb] = (kb == gk) ? arp[r + 1] : p;
      }
      float* crow = c + ii * ldc;
      for (int64_t tj = 0; tj < gn; tj++) {
        int64_t j0 = tj * tn, j1 = j0 + tn < N ? j0 + tn : N;
        for (int64_t kk = 0; kk < gk; kk++) {
          int64_t kb = natural ? kk : (kk + ti + tj) % gk;
          for (int64_t pa = akstart[kb]; pa < akstart[kb + 1]; pa++) {
            float v = av[pa];
            const float* brow = b + (int64_t)aci[pa] * ldb;
            if (use_fma)
              for (int64_t j = j0; j < j1; j++) crow[j] = fmaf(v, brow[j], crow[j]);
            else
              for (int64_t j = j0; j < j1; j++) crow[j] = crow[j] + v * brow[j];
          }
        }
      }
    }
    free(akstart);
  }
}

void oracle_spmm_tiled_f32(int64_t m, int64_t K, int64_t N, const int32_t* arp, const int32_t* aci,
                           const float* av, const float* b, int64_t ldb, float* c, int64_t ldc,
                           int64_t tm, int64_t tk, int64_t tn, const int64_t* rows, int64_t nrows,
                           int use_fma) {
  spmm_tiled_f32_impl(m, K, N, arp, aci, av, b, ldb, c, ldc, tm, tk, tn, rows, nrows, use_fma, 0);
}

void oracle_spmm_rowwise_f32(int64_t m, int64_t K, int64_t N, const int32_t* arp, const int32_t* aci,
                             const float* av, const float* b, int64_t ldb, float* c, int64_t ldc,
                             int64_t tm, int64_t tk, int64_t tn, const int64_t* rows, int64_t nrows) {
  spmm_tiled_f32_impl(m, K, N, arp, aci, av, b, ldb, c, ldc, tm, tk, tn, rows, nrows, 1, 1);
}

/* DMatrix::sum (DMatrix.hpp:537-554) on a row-major m x n matrix cut into
 * tm x tn tiles: tiles in row-major grid order, each tile's rows, each row's
 * columns, `local_sum += value` in FP32 from 0 (out[0]); also the FP64 sum
 * (out[1]) and the sum of magnitudes (out[2]) for the error bound. */
void oracle_dsum_f32(int64_t m, int64_t n, int64_t tm, int64_t tn, const float* x, double* out) {
  float s = 0.0f;
  double d = 0.0, a = 0.0;
  for (int64_t i0 = 0; i0 < m; i0 += tm)
    for (int64_t j0 = 0; j0 < n; j0 += tn)
      for (int64_t i = i0; i < i0 + tm && i < m; i++)
        for (int64_t j = j0; j < j0 + tn && j < n; j++) {
          const float v = x[i * n + j];
          s = s + v;
          d += (double)v;
          a += fabs((double)v);
        }
  out[0] = (double)s;
  out[1] = d;
  out[2] = a;
}

/* Same loop in double over FP32 inputs (error reference); c is double. */
void oracle_spmm_tiled_f64(int64_t m, int64_t K, int64_t N, const int32_t* arp, const int32_t* aci,
                           const float* av, const float* b, int64_t ldb, double* c, int64_t ldc,
                           const int64_t* rows, int64_t nrows) {
  (void)K;
  if (!rows) nrows = m;
  #pragma omp parallel for schedule(dynamic, 16)
  for (int64_t ii = 0; ii < nrows; ii++) {
    int64_t r = rows ? rows[ii] : ii;
    double* crow = c + ii * ldc;
    for (int32_t pa = arp[r]; pa < arp[r + 1]; pa++) {
      double v = av[pa];
      const float* brow = b + (int64_t)aci[pa] * ldb;
      for (int64_t j = 0; j < N; j++) crow[j] += v * (double)brow[j];
    }
  }
}

/* BF16 storage: round-to-nearest-even of an FP32 value to its upper 16 bits. */
static inline uint16_t f32_to_bf16(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  if ((u & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((u >> 16) | 0x40); /* quiet NaN */
  uint32_t lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  return (uint16_t)(u >> 16);
}
static inline float bf16_to_f32(uint16_t h) {
  uint32_t u = (uint32_t)h << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

/* BF16-storage SpMM: B and C hold bf16; every C row is read once, the
 * products of all stages (rotated k order per C tile, A-row order inside a
 * stage) are chained in FP32 with fused multiply-adds, and the row is rounded
 * once to bf16 at the end. */
void oracle_spmm_tiled_bf16(int64_t m, int64_t K, int64_t N, const int32_t* arp, const int32_t* aci,
                            const float* av, const uint16_t* b, int64_t ldb, uint16_t* c, int64_t ldc,
                            int64_t tm, int64_t tk, int64_t tn, const int64_t* rows, int64_t nrows) {
  if (!rows) nrows = m;
  int64_t gk = (K + tk - 1) / tk, gn = (N + tn - 1) / tn;
  if (gk < 1) gk = 1;
  #pragma omp parallel
  {
    int64_t* akstart = (int64_t*)malloc(sizeof(int64_t) * (size_t)(gk + 1));
    float* acc = (float*)malloc(sizeof(float) * (size_t)(N > 0 ? N : 1));
    #pragma omp for schedule(dynamic, 16)
    for (int64_t ii = 0; ii < nrows; ii++) {
      int64_t r = rows ? rows[ii] : ii;
      int64_t ti = r / tm;
      int64_t p = arp[r];
      for (int64_t kb = 0; kb <= gk; kb++) {
        int64_t lim = kb * tk;
        while (p < arp[r + 1] && aci[p] < lim) p++;
        akstart[kb] = (kb == gk) ? arp[r + 1] : p;
      }
      uint16_t* crow = c + ii * ldc;
      for (int64_t j = 0; j < N; j++) acc[j] = bf16_to_f32(crow[j]);
      for (int64_t tj = 0; tj < gn; tj++) {
        int64_t j0 = tj * tn, j1 = j0 + tn < N ? j0 + tn : N;
        for (int64_t kk = 0; kk < gk; kk++) {
          int64_t kb = (kk + ti + tj) % gk;
          for (int64_t pa = akstart[kb]; pa < akstart[kb + 1]; pa++) {
            float v = av[pa];
            const uint16_t* brow = b + (int64_t)aci[pa] * ldb;
            for (int64_t j = j0; j < j1; j++) acc[j] = fmaf(v, bf16_to_f32(brow[j]), acc[j]);
          }
        }
      }
      for (int64_t j = 0; j < N; j++) crow[j] = f32_to_bf16(acc[j]);
    }
    free(akstart);
    free(acc);
  }
}

void oracle_f32_to_bf16(const float* x, uint16_t* y, int64_t count) {
  #pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < count; i++) y[i] = f32_to_bf16(x[i]);
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
