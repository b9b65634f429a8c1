// Sparse x dense: C += A * B, for one tile (spmm_wrapper,
// bcl/containers/algorithms/spgemm.hpp:80-96 and 140-149) and for the whole
// tile loop of BCL::gemm(SPMatrix, DMatrix, DMatrix&) (spgemm.hpp:153-179) in
// one launch.
//
// Layout: one warp per (C tile row, column panel).  Lane l owns VEC
// consecutive columns per chunk (a 16-byte vector: 4 floats or 8 bfloat16),
// so a warp covers 128 FP32 / 256 BF16 columns per chunk, CH chunks per
// panel.  The warp reads 32 (column, value) pairs of the A row at once and
// broadcasts them with shuffles; for each entry every lane issues its 16-byte
// loads of the B row (coalesced: the warp reads whole 512-byte row segments),
// UNROLL entries' loads in flight before their multiply-adds are applied.
//
// Order: per output element the multiply-adds run in stored A-row order, and
// over the C tile's stages k = (k_ + i + j) mod G in that order, starting
// from the C value already stored (beta = 1, in place) — the reference's
// sequence, so FP32 results are bit-identical.  BF16 storage keeps the chain
// in FP32 registers and rounds each C element once when it is stored.
#include "common.cuh"

namespace bclx {

constexpr int kSpmmWarps = 8;

template <typename ST>
struct Vec;

template <>
struct Vec<float> {
  static constexpr int N = 4;
  __device__ __forceinline__ static void load(const float* p, float* out) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
  }
  __device__ __forceinline__ static void load_c(const float* p, float* out) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
  }
  __device__ __forceinline__ static void store(float* p, const float* in) {
    *reinterpret_cast<float4*>(p) = make_float4(in[0], in[1], in[2], in[3]);
  }
  __device__ __forceinline__ static float to_f(float x) { return x; }
  __device__ __forceinline__ static float from_f(float x) { return x; }
};

template <>
struct Vec<__nv_bfloat16> {
  static constexpr int N = 8;
  __device__ __forceinline__ static void unpack(uint4 v, float* out) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < 4; i++) {
      out[2 * i] = __uint_as_float(w[i] << 16);
      out[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
    }
  }
  __device__ __forceinline__ static void load(const __nv_bfloat16* p, float* out) {
    unpack(__ldg(reinterpret_cast<const uint4*>(p)), out);
  }
  __device__ __forceinline__ static void load_c(const __nv_bfloat16* p, float* out) {
    unpack(*reinterpret_cast<const uint4*>(p), out);
  }
  __device__ __forceinline__ static void store(__nv_bfloat16* p, const float* in) {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(in[2 * i]));
      const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(in[2 * i + 1]));
      w[i] = lo | (hi << 16);
    }
    *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  __device__ __forceinline__ static float to_f(__nv_bfloat16 x) { return __bfloat162float(x); }
  __device__ __forceinline__ static __nv_bfloat16 from_f(float x) { return __float2bfloat16_rn(x); }
};

// One (C row, panel) with all loads of B and C as 16-byte vectors.
template <typename ST, int CH, bool VECTOR>
__device__ __forceinline__ void spmm_row(const SpGridView& A, const DGridView& B, const DGridView& C, int64_t ti,
                                         int64_t tj, int64_t r, int c0, int W) {
  using V = Vec<ST>;
  constexpr int VN = V::N;
  // entries whose B loads are in flight together: 16 floats of B per lane
  constexpr int kUnroll = VN * CH >= 16 ? 1 : (VN * CH >= 8 ? 2 : 4);
  const int lane = lane_id();
  ST* __restrict__ crow = reinterpret_cast<ST*>(C.tile(ti, tj)) + r * C.ld;
  float acc[CH][VN];
  bool own[CH];
#pragma unroll
  for (int q = 0; q < CH; q++) {
    const int col = c0 + (q * 32 + lane) * VN;
    own[q] = col < W;
    if (VECTOR) {
      if (own[q]) V::load_c(crow + col, acc[q]);
    } else {
#pragma unroll
      for (int x = 0; x < VN; x++) acc[q][x] = (col + x < W) ? V::to_f(crow[col + x]) : 0.f;
    }
  }
  const int64_t gk = A.gn;
  for (int64_t kk = 0; kk < gk; kk++) {
    const int64_t k = (kk + ti + tj) % gk;
    const bclx_csr_t At = A.tile(ti, k);
    const int32_t a0 = __ldg(At.row_ptr + r), a1 = __ldg(At.row_ptr + r + 1);
    if (a0 == a1) continue;
    const ST* __restrict__ bt = reinterpret_cast<const ST*>(B.tile(k, tj));
    const bool bvec = VECTOR && (reinterpret_cast<uintptr_t>(bt) & 15) == 0;
    const float* __restrict__ av = reinterpret_cast<const float*>(At.vals);
    for (int32_t cb = a0; cb < a1; cb += 32) {
      const int32_t p = cb + lane;
      const int32_t kc = p < a1 ? __ldg(At.col_ind + p) : 0;
      const float vv = p < a1 ? __ldg(av + p) : 0.f;
      const int ne = min(32, a1 - cb);
      for (int e = 0; e < ne; e += kUnroll) {
        float bvals[kUnroll][CH][VN];
        float vs[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
          const int32_t kr = __shfl_sync(kFull, kc, (e + u) & 31);
          vs[u] = __shfl_sync(kFull, vv, (e + u) & 31);
          const ST* brow = bt + (int64_t)kr * B.ld;
#pragma unroll
          for (int q = 0; q < CH; q++) {
            const int col = c0 + (q * 32 + lane) * VN;
            if (e + u < ne && own[q]) {
              if (bvec) {
                V::load(brow + col, bvals[u][q]);
              } else {
#pragma unroll
                for (int x = 0; x < VN; x++) bvals[u][q][x] = (col + x < W) ? V::to_f(brow[col + x]) : 0.f;
              }
            }
          }
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
          if (e + u < ne) {
#pragma unroll
            for (int q = 0; q < CH; q++)
#pragma unroll
              for (int x = 0; x < VN; x++) acc[q][x] = __fmaf_rn(vs[u], bvals[u][q][x], acc[q][x]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < CH; q++) {
    const int col = c0 + (q * 32 + lane) * VN;
    if (VECTOR) {
      if (own[q]) V::store(crow + col, acc[q]);
    } else {
#pragma unroll
      for (int x = 0; x < VN; x++)
        if (col + x < W) crow[col + x] = V::from_f(acc[q][x]);
    }
  }
}

template <typename ST, int CH>
__global__ void __launch_bounds__(kSpmmWarps * 32)
    k_spmm(SpGridView A, DGridView B, DGridView C, int64_t n_items, int npanels, int row_align_ok) {
  constexpr int PW = 32 * Vec<ST>::N * CH;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t item = warp; item < n_items; item += nwarps) {
    const int64_t ri = item / npanels;
    const int panel = (int)(item - ri * npanels);
    const int64_t t = ri / C.tm;
    const int64_t r = ri - t * C.tm;
    const int64_t ti = t / C.gn, tj = t - ti * C.gn;
    if (r >= C.rows_of(ti)) continue;
    const int W = (int)C.cols_of(tj);
    const int c0 = panel * PW;
    if (c0 >= W) continue;
    bool vec = row_align_ok && (W % Vec<ST>::N) == 0;
    if (vec) {
      const uintptr_t pc = reinterpret_cast<uintptr_t>(C.tile(ti, tj));
      vec = (pc & 15) == 0;
    }
    // (a B tile that is not 16-byte aligned is read with scalar loads)
    if (vec)
      spmm_row<ST, CH, true>(A, B, C, ti, tj, r, c0, W);
    else
      spmm_row<ST, CH, false>(A, B, C, ti, tj, r, c0, W);
  }
}

template <typename ST>
static int launch_spmm(Context* ctx, const SpGridView& A, const DGridView& B, const DGridView& C, int align_ok) {
  constexpr int VN = Vec<ST>::N;
  const int64_t W = C.tn;
  int ch = W <= 32 * VN ? 1 : (W <= 64 * VN ? 2 : 4);
  const int64_t pw = 32 * VN * ch;
  const int npanels = (int)ceil_div(W, pw);
  const int64_t n_items = C.gm * C.gn * C.tm * npanels;
  if (n_items == 0) return BCLX_OK;
  int64_t want = ceil_div(n_items, kSpmmWarps);
  int64_t cap = (int64_t)ctx->num_sms * 8;
  const unsigned blocks = (unsigned)(want < cap ? want : cap);
  switch (ch) {
    case 1: k_spmm<ST, 1><<<blocks, kSpmmWarps * 32, 0, ctx->stream>>>(A, B, C, n_items, npanels, align_ok); break;
    case 2: k_spmm<ST, 2><<<blocks, kSpmmWarps * 32, 0, ctx->stream>>>(A, B, C, n_items, npanels, align_ok); break;
    default: k_spmm<ST, 4><<<blocks, kSpmmWarps * 32, 0, ctx->stream>>>(A, B, C, n_items, npanels, align_ok); break;
  }
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

static int run_spmm(Context* ctx, const SpGridView& A, const DGridView& B, const DGridView& C, int dtype) {
  const int es = dtype == BCLX_F32 ? 4 : 2;
  const int align_ok = ((B.ld * es) % 16 == 0) && ((C.ld * es) % 16 == 0);
  if (dtype == BCLX_F32) return launch_spmm<float>(ctx, A, B, C, align_ok);
  return launch_spmm<__nv_bfloat16>(ctx, A, B, C, align_ok);
}

}  // namespace bclx

using namespace bclx;

extern "C" {

int bclx_spmm_tile(bclx_context_t c, int64_t m, int64_t n, int64_t k, int64_t nnz, void* cp, const void* bp,
                   const float* a_values, const int32_t* a_rowptr, const int32_t* a_colind, int64_t ldb,
                   int64_t ldc, int32_t bc_dtype) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || m < 0 || n < 0 || k < 0 || nnz < 0) return BCLX_ERR_INVALID;
  if (bc_dtype != BCLX_F32 && bc_dtype != BCLX_BF16) return BCLX_ERR_DTYPE;
  if (m == 0 || n == 0) return BCLX_OK;
  if (!cp || !bp || !a_rowptr || (nnz > 0 && (!a_values || !a_colind)) || ldb < n || ldc < n)
    return BCLX_ERR_INVALID;
  if (n > INT32_MAX || m > INT32_MAX) return BCLX_ERR_INDEX_OVERFLOW;
  BCLX_CK(cudaSetDevice(ctx->device));
  SpGridView A{};
  A.tiles = nullptr;
  A.single.m = m; A.single.n = k; A.single.nnz = nnz;
  A.single.row_ptr = const_cast<int32_t*>(a_rowptr);
  A.single.col_ind = const_cast<int32_t*>(a_colind);
  A.single.vals = const_cast<float*>(a_values);
  A.single.dtype = BCLX_F32;
  A.m = m; A.n = k > 0 ? k : 1; A.tm = m; A.tn = A.n; A.gm = 1; A.gn = 1;
  DGridView B{};
  B.tiles = nullptr; B.single = const_cast<void*>(bp);
  B.m = A.n; B.n = n; B.tm = A.n; B.tn = n; B.gm = 1; B.gn = 1; B.ld = ldb;
  DGridView C{};
  C.tiles = nullptr; C.single = cp;
  C.m = m; C.n = n; C.tm = m; C.tn = n; C.gm = 1; C.gn = 1; C.ld = ldc;
  return run_spmm(ctx, A, B, C, bc_dtype);
}

int bclx_spmm_grid(bclx_context_t c, const bclx_spgrid_t* a, const bclx_dgrid_t* b, const bclx_dgrid_t* cg) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !a || !b || !cg || !a->tiles || !b->tiles || !cg->tiles) return BCLX_ERR_INVALID;
  if (a->dtype != BCLX_F32) return BCLX_ERR_DTYPE;
  if (b->dtype != cg->dtype || (b->dtype != BCLX_F32 && b->dtype != BCLX_BF16)) return BCLX_ERR_DTYPE;
  auto grid_ok = [](int64_t m, int64_t n, int64_t tm, int64_t tn, int64_t gm, int64_t gn) {
    return m >= 0 && n >= 0 && tm > 0 && tn > 0 && gm == ceil_div(m, tm) && gn == ceil_div(n, tn);
  };
  if (!grid_ok(a->m, a->n, a->tile_m, a->tile_n, a->grid_m, a->grid_n) ||
      !grid_ok(b->m, b->n, b->tile_m, b->tile_n, b->grid_m, b->grid_n) ||
      !grid_ok(cg->m, cg->n, cg->tile_m, cg->tile_n, cg->grid_m, cg->grid_n))
    return BCLX_ERR_INVALID;
  if (a->m != cg->m || a->n != b->m || b->n != cg->n) return BCLX_ERR_INVALID;
  if (a->tile_m != cg->tile_m || a->tile_n != b->tile_m || b->tile_n != cg->tile_n) return BCLX_ERR_INVALID;
  if (cg->tile_n > INT32_MAX) return BCLX_ERR_INDEX_OVERFLOW;
  BCLX_CK(cudaSetDevice(ctx->device));
  SpGridView A = make_view(*a);
  DGridView B{};
  B.tiles = b->tiles; B.m = b->m; B.n = b->n; B.tm = b->tile_m; B.tn = b->tile_n; B.gm = b->grid_m;
  B.gn = b->grid_n; B.ld = b->tile_n;
  DGridView C{};
  C.tiles = cg->tiles; C.m = cg->m; C.n = cg->n; C.tm = cg->tile_m; C.tn = cg->tile_n; C.gm = cg->grid_m;
  C.gn = cg->grid_n; C.ld = cg->tile_n;
  return run_spmm(ctx, A, B, C, b->dtype);
}

}  // extern "C"
