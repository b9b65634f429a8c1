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

#include <algorithm>
#include <cstdlib>

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
  __device__ __forceinline__ static void unpack_raw(uint4 v, float* out) {
    out[0] = __uint_as_float(v.x); out[1] = __uint_as_float(v.y);
    out[2] = __uint_as_float(v.z); out[3] = __uint_as_float(v.w);
  }
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
  __device__ __forceinline__ static void unpack_raw(uint4 v, float* out) { unpack(v, out); }
};

constexpr int kSpmmUnroll = 4;  // B-row loads in flight per lane (with 32 warps per SM)

// Ask L2 for the 128-byte lines of [p, p + bytes) (no-op for null).
__device__ __forceinline__ void l2_prefetch_slice(const void* p, int bytes) {
  if (p == nullptr) return;
  const char* q = reinterpret_cast<const char*>(p);
  for (int o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L2 [%0];\n" ::"l"(q + o));
}

// Per-warp entry tables (two 32-entry buffers of 16 bytes per warp).
__shared__ uint4 spmm_tables[kSpmmWarps * 64];

// The stages of C-tile row (ti, tj, r), one lane per stage of the group
// [g0, g0+32), in the reference's rotated order k = (k_ + ti + tj) mod gk:
// the A-row segment of that stage and its B tile.
template <typename ST>
struct StageLane {
  int32_t alen;
  const int32_t* acol;
  const float* aval;
  const ST* bt;
};

template <typename ST>
__device__ __forceinline__ StageLane<ST> stage_lane(const SpGridView& A, const DGridView& B, int64_t ti, int64_t tj,
                                                    int64_t r, int64_t g0) {
  StageLane<ST> s{0, nullptr, nullptr, nullptr};
  const int64_t kk = g0 + lane_id();
  const int64_t gk = A.gn;
  if (kk < gk) {
    const int64_t k = (kk + ti + tj) % gk;
    const bclx_csr_t At = A.tile(ti, k);
    const int32_t as = __ldg(At.row_ptr + r);
    s.alen = __ldg(At.row_ptr + r + 1) - as;
    s.acol = At.col_ind + as;
    s.aval = reinterpret_cast<const float*>(At.vals) + as;
    s.bt = reinterpret_cast<const ST*>(B.tile(k, tj));
  }
  return s;
}

// C tile (ti, tj) and every B tile of its column start on 16 bytes.
__device__ __forceinline__ bool tiles_aligned(const DGridView& B, const DGridView& C, int64_t ti, int64_t tj) {
  bool ok = (reinterpret_cast<uintptr_t>(C.tile(ti, tj)) & 15) == 0;
  for (int64_t k = lane_id(); k < B.gm; k += 32) ok &= (reinterpret_cast<uintptr_t>(B.tile(k, tj)) & 15) == 0;
  return __all_sync(kFull, ok);
}

// One warp per (C row, panel of 32 16-byte vectors).  The A entries of all
// stages are taken 32 at a time (one lane each finds its B row), then
// broadcast kSpmmUnroll at a time so that that many B-row loads (raw
// 16-byte vectors) are in flight before their multiply-adds are applied in
// entry order.  `vec`: every B and C row slice of this tile pair is 16-byte
// aligned; otherwise element-wise access.
template <typename ST, int UNROLL = kSpmmUnroll>
__device__ __forceinline__ void spmm_row(const SpGridView& A, const DGridView& B, const DGridView& C, int64_t ti,
                                         int64_t tj, int64_t r, int c0, int W, bool vec) {
  using V = Vec<ST>;
  constexpr int VN = V::N;
  const int lane = lane_id();
  ST* __restrict__ crow = reinterpret_cast<ST*>(C.tile(ti, tj)) + r * C.ld;
  const int col = c0 + lane * VN;
  const bool own = col < W;
  float acc[VN];
  if (vec) {
    if (own) V::load_c(crow + col, acc);
  } else {
#pragma unroll
    for (int x = 0; x < VN; x++) acc[x] = (col + x < W) ? V::to_f(crow[col + x]) : 0.f;
  }
  // Entry table of one 32-entry chunk per buffer: B row address (column 0
  // of the tile) and A value, written lane-parallel one chunk ahead and read
  // back with broadcast 16-byte shared loads.
  uint4* tb = spmm_tables + (threadIdx.x >> 5) * 64;
  // bytes of this warp's panel in one B row
  const int pbytes = min(32 * VN, W - c0) * (int)sizeof(ST);
  for (int64_t g0 = 0; g0 < A.gn; g0 += 32) {
    const StageLane<ST> sl = stage_lane<ST>(A, B, ti, tj, r, g0);
    const int32_t aincl = warp_inclusive_scan(sl.alen);
    const int32_t atot = __shfl_sync(kFull, aincl, 31);
    const int32_t aexcl = aincl - sl.alen;
    // entry e0 + lane of the flattened stages: its A value and B row
    auto chunk = [&](int32_t e0, float& v, const ST*& brow) {
      const int32_t e = e0 + lane;
      int src = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int32_t t = __shfl_sync(kFull, aincl, src + step - 1);
        if (t <= e) src += step;
      }
      src = min(src, 31);
      const int32_t off = e - __shfl_sync(kFull, aexcl, src);
      const int32_t* sacol = reinterpret_cast<const int32_t*>(
          __shfl_sync(kFull, reinterpret_cast<unsigned long long>(sl.acol), src));
      const float* saval = reinterpret_cast<const float*>(
          __shfl_sync(kFull, reinterpret_cast<unsigned long long>(sl.aval), src));
      const ST* sbt = reinterpret_cast<const ST*>(__shfl_sync(kFull, reinterpret_cast<unsigned long long>(sl.bt), src));
      v = 0.f;
      brow = sbt;
      if (e < atot) {
        v = __ldg(saval + off);
        brow = sbt + (int64_t)__ldg(sacol + off) * B.ld;
      }
    };
    auto put = [&](int buf, float v, const ST* brow) {
      const uint64_t pa = reinterpret_cast<uint64_t>(brow);
      tb[buf * 32 + lane] = make_uint4((uint32_t)pa, (uint32_t)(pa >> 32), __float_as_uint(v), 0u);
    };
    // Chunk c is applied from the table while the rows of chunk c+2 are
    // asked into L2 (each lane its own entry's panel slice) and the A loads
    // of chunk c+3 are in flight.
    float v0, v1, v2, v3;
    const ST *b0, *b1, *b2, *b3;
    chunk(0, v0, b0);
    chunk(32, v1, b1);
    chunk(64, v2, b2);
    put(0, v0, b0);
    l2_prefetch_slice(vec && lane < atot ? b0 + c0 : nullptr, pbytes);
    l2_prefetch_slice(vec && 32 + lane < atot ? b1 + c0 : nullptr, pbytes);
    __syncwarp();
    int buf = 0;
    for (int32_t e0 = 0; e0 < atot; e0 += 32) {
      const bool more = e0 + 32 < atot;
      if (e0 + 96 < atot) chunk(e0 + 96, v3, b3);  // A loads three chunks ahead
      l2_prefetch_slice(vec && e0 + 64 + lane < atot ? b2 + c0 : nullptr, pbytes);
      const int ne = min(32, atot - e0);
      const uint4* t = tb + buf * 32;
      if (vec) {
        for (int u0 = 0; u0 < ne; u0 += UNROLL) {
          uint4 ent[UNROLL];
          uint4 raw[UNROLL];
#pragma unroll
          for (int u = 0; u < UNROLL; u++) ent[u] = t[(u0 + u) & 31];
#pragma unroll
          for (int u = 0; u < UNROLL; u++) {
            const ST* rp = reinterpret_cast<const ST*>((uint64_t)ent[u].x | ((uint64_t)ent[u].y << 32));
            if (u0 + u < ne && own) raw[u] = __ldg(reinterpret_cast<const uint4*>(rp + col));
          }
#pragma unroll
          for (int u = 0; u < UNROLL; u++) {
            if (u0 + u < ne && own) {
              float b[VN];
              V::unpack_raw(raw[u], b);
              const float vs = __uint_as_float(ent[u].z);
#pragma unroll
              for (int x = 0; x < VN; x++) acc[x] = __fmaf_rn(vs, b[x], acc[x]);
            }
          }
        }
      } else {
        for (int u = 0; u < ne; u++) {
          const uint4 en = t[u];
          const ST* rp = reinterpret_cast<const ST*>((uint64_t)en.x | ((uint64_t)en.y << 32));
          const float vs = __uint_as_float(en.z);
#pragma unroll
          for (int x = 0; x < VN; x++)
            if (col + x < W) acc[x] = __fmaf_rn(vs, V::to_f(rp[col + x]), acc[x]);
        }
      }
      if (more) {
        buf ^= 1;
        put(buf, v1, b1);
      }
      __syncwarp();
      v1 = v2;
      b1 = b2;
      v2 = v3;
      b2 = b3;
    }
  }
  if (vec) {
    if (own) V::store(crow + col, acc);
  } else {
#pragma unroll
    for (int x = 0; x < VN; x++)
      if (col + x < W) crow[col + x] = V::from_f(acc[x]);
  }
}

template <typename ST>
__global__ void __launch_bounds__(kSpmmWarps * 32, 4)
    k_spmm(SpGridView A, DGridView B, DGridView C, int64_t n_items, int npanels, int row_align_ok,
           const uint8_t* __restrict__ long_flag) {
  constexpr int PW = 32 * Vec<ST>::N;
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
    const bool vec = row_align_ok && (W % Vec<ST>::N) == 0 && tiles_aligned(B, C, ti, tj);
    if (long_flag && vec && long_flag[ti * C.tm + r]) continue;  // k_spmm_long takes it
    spmm_row<ST>(A, B, C, ti, tj, r, c0, W, vec);
  }
}

// ---- long rows ----------------------------------------------------------------
//
// A row with thousands of entries is one chain of multiply-adds per output
// element (the reference's order), so a warp with a few B-row loads in flight
// spends milliseconds on it.  Such rows are found first (k_spmm_find_long),
// skipped by k_spmm and run by k_spmm_long on the context's side stream at
// the same time: one warp per (row, C tile column, panel), the same walk
// with kLongUnroll B-row loads in flight per lane (warps with the registers
// for it: few of them, each on one long chain).

constexpr int kLongUnroll = 32;  // B-row loads in flight per lane on long rows (half for BF16: registers)
constexpr int kLongWarps = 4;
constexpr int kSpmmLongRow = 1024;         // entries over all stages
constexpr int64_t kSpmmLongMinRows = 65536;  // smaller products do not use the long-row path

// Thread per A row (ti, r): entries over all stages; rows with at least
// long_row are flagged and listed.
__global__ void k_spmm_find_long(SpGridView A, int long_row, uint8_t* __restrict__ flag, int64_t* __restrict__ list,
                                 int32_t* __restrict__ count) {
  const int64_t rows = A.gm * A.tm;
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < rows; x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ti = x / A.tm, r = x - ti * A.tm;
    int64_t tot = 0;
    if (r < A.rows_of(ti))
      for (int64_t k = 0; k < A.gn; k++) {
        const int32_t* rp = A.tile(ti, k).row_ptr;
        tot += __ldg(rp + r + 1) - __ldg(rp + r);
      }
    const bool lng = tot >= long_row;
    flag[x] = lng ? 1 : 0;
    if (lng) list[atomicAdd(count, 1)] = x;
  }
}

template <typename ST>
__global__ void __launch_bounds__(kLongWarps * 32)
    k_spmm_long(SpGridView A, DGridView B, DGridView C, const int64_t* __restrict__ list,
                const int32_t* __restrict__ count, int npanels, int row_align_ok) {
  constexpr int PW = 32 * Vec<ST>::N;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t nl = *count;
  const int64_t n = nl * C.gn * npanels;
  for (int64_t w = warp; w < n; w += nwarps) {
    // consecutive warps take different rows; a row's panels are spread out
    const int64_t li = w % nl;
    const int64_t pt = w / nl;
    const int panel = (int)(pt % npanels);
    const int64_t tj = pt / npanels;
    const int64_t x = list[li];
    const int64_t ti = x / A.tm, r = x - ti * A.tm;
    const int W = (int)C.cols_of(tj);
    if (panel * PW >= W) continue;
    const bool vec = row_align_ok && (W % Vec<ST>::N) == 0 && tiles_aligned(B, C, ti, tj);
    if (!vec) continue;  // k_spmm did this one element-wise
    spmm_row<ST, sizeof(ST) == 4 ? kLongUnroll : kLongUnroll / 2>(A, B, C, ti, tj, r, panel * PW, W, true);
  }
}

static int64_t spmm_long_min_rows() {
  const char* e = std::getenv("BCLX_SPMM_LONG_MIN_ROWS");
  return e && *e ? std::strtoll(e, nullptr, 10) : kSpmmLongMinRows;
}

template <typename ST>
static int launch_spmm(Context* ctx, const SpGridView& A, const DGridView& B, const DGridView& C, int align_ok) {
  constexpr int VN = Vec<ST>::N;
  const int npanels = (int)ceil_div(C.tn, 32 * VN);
  const int64_t n_items = C.gm * C.gn * C.tm * npanels;
  if (n_items == 0) return BCLX_OK;
  const int64_t want = ceil_div(n_items, kSpmmWarps);
  const int64_t cap = (int64_t)ctx->num_sms * 8;
  const int64_t arows = A.gm * A.tm;
  const bool long_path = align_ok && A.gn <= 32 && arows >= spmm_long_min_rows();
  uint8_t* flag = nullptr;
  int64_t* list = nullptr;
  int32_t* cnt = nullptr;
  if (long_path) {
    // find the long rows, then run them on the side stream beside k_spmm
    BCLX_TRY(ensure_side_stream(ctx));
    BCLX_TRY(scratch_alloc_n(ctx, &flag, (size_t)arows));
    BCLX_TRY(scratch_alloc_n(ctx, &list, (size_t)arows));
    BCLX_TRY(scratch_alloc_n(ctx, &cnt, 1));
    BCLX_CK(cudaMemsetAsync(cnt, 0, sizeof(int32_t), ctx->stream));
    k_spmm_find_long<<<(unsigned)std::min<int64_t>(ceil_div(arows, 256), (int64_t)ctx->num_sms * 16), 256, 0,
                       ctx->stream>>>(A, kSpmmLongRow, flag, list, cnt);
    note_launch();
    BCLX_CK_LAUNCH();
    BCLX_CK(cudaEventRecord(ctx->fork_ev, ctx->stream));
    BCLX_CK(cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0));
    k_spmm_long<ST><<<(unsigned)ctx->num_sms, kLongWarps * 32, 0, ctx->side>>>(A, B, C, list, cnt, npanels,
                                                                                align_ok);
    note_launch();
    BCLX_CK_LAUNCH();
    BCLX_CK(cudaEventRecord(ctx->join_ev, ctx->side));
  }
  k_spmm<ST><<<(unsigned)(want < cap ? want : cap), kSpmmWarps * 32, 0, ctx->stream>>>(A, B, C, n_items, npanels,
                                                                                        align_ok, flag);
  note_launch();
  BCLX_CK_LAUNCH();
  if (long_path) {
    BCLX_CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0));
    scratch_free(ctx, flag);
    scratch_free(ctx, list);
    scratch_free(ctx, cnt);
  }
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
