// Sparse x sparse product over tile grids (the SUMMA tile loop of
// BCL::gemm(SPMatrix, SPMatrix, SPMatrix&), bcl/containers/algorithms/
// spgemm.hpp:182-242, with its local kernel spgemm.hpp:41-76 and the tile
// accumulation of SparseHashAccumulator.hpp:101-182), and tile accumulation.
//
// Work decomposition.  A "row item" is one row r of one C tile (i, j); it
// owns every product A_ik[r, :] * B_kj over all k.  Long row items are split
// into column slices ("work items") so that no work item sees more than a
// few thousand products or more than kSliceCols output columns.
//
// Per work item, one warp:
//   symbolic: sets one bit per product column in a shared-memory bitmap of
//             the slice; the popcount is the output count.
//   numeric:  rebuilds the bitmap (or reads the already-written columns),
//             turns it into per-word prefix counts so that the output
//             position of column j is rank(j) = prefix[j/32] + popc(lower
//             bits); writes the sorted columns directly; then walks the
//             products again in the reference's order and accumulates
//             values into a shared-memory row indexed by rank.
//
// Order.  Products are enumerated 32 at a time in exactly the reference's
// sequence: stages k = (k_ + i + j) mod G; inside a stage the A-row entries
// in stored order; inside an entry the B-row entries in stored order.  In a
// batch, lanes holding the same column are grouped with __match_any_sync and
// the lowest lane applies the group's multiply-adds in lane order; batches
// are separated by __syncwarp.  Every output entry therefore sees the same
// chain of fused multiply-adds (from 0) per stage and the same chain of adds
// across stages as the reference, so FP32 results are bit-identical.
#include "common.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace bclx {

constexpr int kSliceCols = 8192;                 // bitmap capacity per work item (columns)
constexpr int kBitmapWords = kSliceCols / 32;    // 256
constexpr int64_t kSliceTarget = 4096;           // products per work item before a row is split
constexpr int kMaxSlices = 64;
constexpr int kVcapSmall = 512;                  // outputs per work item, small-accumulator kernel
constexpr int kVcapBig = kSliceCols;             // outputs per work item, large kernel (= slice width)
constexpr int kWarpsSym = 8;
constexpr int kWarpsSmall = 8;
constexpr int kWarpsBig = 2;

struct Geom {
  int64_t gm, gk, gn;  // C grid is gm x gn; the k grid has gk tiles
  int64_t tm, tn;      // C tile shape
  int64_t m, n;        // C shape
  int64_t n_row_items; // gm * gn * tm
};

struct ItemInfo {
  int64_t ri, ti, tj, r;
  int s, ns, lo, hi;
};

__device__ __forceinline__ void decode_row_item(const Geom& g, int64_t ri, int64_t& ti, int64_t& tj,
                                                int64_t& r) {
  int64_t t = ri / g.tm;
  r = ri - t * g.tm;
  ti = t / g.gn;
  tj = t - ti * g.gn;
}

__device__ __forceinline__ int64_t encode_item(int64_t ri, int s, int ns) {
  return ri | ((int64_t)s << 40) | ((int64_t)ns << 50);
}

__device__ __forceinline__ ItemInfo decode_item(const Geom& g, int64_t code) {
  ItemInfo it;
  it.ri = code & ((1LL << 40) - 1);
  it.s = (int)((code >> 40) & 1023);
  it.ns = (int)((code >> 50) & 1023);
  decode_row_item(g, it.ri, it.ti, it.tj, it.r);
  int64_t w = g.n - it.tj * g.tn;
  if (w > g.tn) w = g.tn;
  it.lo = (int)(w * it.s / it.ns);
  it.hi = (int)(w * (it.s + 1) / it.ns);
  return it;
}

template <typename VT>
__device__ __forceinline__ VT load_val(const void* p, int64_t i) {
  return __ldg(reinterpret_cast<const VT*>(p) + i);
}

// Walk the products of C tile row r for one stage (A tile At, B tile Bt),
// restricted to columns [lo, hi) when SLICED, 32 at a time in the reference's
// order.  Every lane calls f(valid, j, a, b) once per batch (warp-uniform
// control flow), valid lanes form a prefix of the warp.
template <typename VT, bool SLICED, bool VALUES, typename F>
__device__ __forceinline__ void for_each_product(const bclx_csr_t& At, const bclx_csr_t& Bt, int64_t r,
                                                 int lo, int hi, F&& f) {
  const int lane = lane_id();
  const int32_t a0 = __ldg(At.row_ptr + r), a1 = __ldg(At.row_ptr + r + 1);
  for (int32_t c0 = a0; c0 < a1; c0 += 32) {
    const int32_t p = c0 + lane;
    int32_t bs = 0, len = 0;
    VT av = VT(0);
    if (p < a1) {
      const int32_t kc = __ldg(At.col_ind + p);
      if (VALUES) av = load_val<VT>(At.vals, p);
      bs = __ldg(Bt.row_ptr + kc);
      int32_t be = __ldg(Bt.row_ptr + kc + 1);
      if (SLICED) {
        const int32_t s0 = lower_bound_i32(Bt.col_ind, bs, be, lo);
        be = lower_bound_i32(Bt.col_ind, s0, be, hi);
        bs = s0;
      }
      len = be - bs;
    }
    const int32_t incl = warp_inclusive_scan(len);
    const int32_t total = __shfl_sync(kFull, incl, 31);
    const int32_t excl = incl - len;
    for (int32_t base = 0; base < total; base += 32) {
      const int32_t q = base + lane;
      int src = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const int32_t v = __shfl_sync(kFull, incl, src + step - 1);
        if (v <= q) src += step;
      }
      const int32_t sbs = __shfl_sync(kFull, bs, src);
      const int32_t sex = __shfl_sync(kFull, excl, src);
      const VT a = __shfl_sync(kFull, av, src);
      const bool valid = q < total;
      int32_t j = -1;
      VT bv = VT(0);
      if (valid) {
        const int32_t bpos = sbs + (q - sex);
        j = __ldg(Bt.col_ind + bpos);
        if (VALUES) bv = load_val<VT>(Bt.vals, bpos);
      }
      f(valid, j, a, bv);
    }
  }
}

// ---- planning -------------------------------------------------------------------

__global__ void k_spgemm_ub(SpGridView A, SpGridView B, Geom g, int64_t* __restrict__ ub,
                            int32_t* __restrict__ nslices, unsigned long long* __restrict__ products) {
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  int64_t mine = 0;
  for (int64_t ri = warp; ri < g.n_row_items; ri += nwarps) {
    int64_t ti, tj, r;
    decode_row_item(g, ri, ti, tj, r);
    int64_t tot = 0;
    if (r < A.rows_of(ti)) {
      for (int64_t k = 0; k < g.gk; k++) {
        const bclx_csr_t At = A.tile(ti, k);
        const bclx_csr_t Bt = B.tile(k, tj);
        const int32_t a0 = __ldg(At.row_ptr + r), a1 = __ldg(At.row_ptr + r + 1);
        for (int32_t p = a0 + lane; p < a1; p += 32) {
          const int32_t kc = __ldg(At.col_ind + p);
          tot += __ldg(Bt.row_ptr + kc + 1) - __ldg(Bt.row_ptr + kc);
        }
      }
      tot = warp_sum(tot);
    }
    if (lane == 0) {
      ub[ri] = tot;
      mine += tot;
      int ns = 0;
      if (tot > 0) {
        int64_t w = g.n - tj * g.tn;
        if (w > g.tn) w = g.tn;
        int64_t by_cols = (w + kSliceCols - 1) / kSliceCols;
        int64_t by_work = (tot + kSliceTarget - 1) / kSliceTarget;
        if (by_work > kMaxSlices) by_work = kMaxSlices;
        int64_t s = by_cols > by_work ? by_cols : by_work;
        if (s > w) s = w;
        ns = (int)s;
      }
      nslices[ri] = ns;
    }
  }
  if (lane == 0 && mine) atomicAdd(products, (unsigned long long)mine);
}

__global__ void k_build_items(Geom g, const int32_t* __restrict__ nslices, const int64_t* __restrict__ first,
                              int64_t* __restrict__ items) {
  for (int64_t ri = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ri < g.n_row_items;
       ri += (int64_t)gridDim.x * blockDim.x) {
    const int ns = nslices[ri];
    const int64_t f = first[ri];
    for (int s = 0; s < ns; s++) items[f + s] = encode_item(ri, s, ns);
  }
}

// ---- symbolic ------------------------------------------------------------------------

template <typename VT>
__global__ void __launch_bounds__(kWarpsSym * 32)
    k_spgemm_symbolic(SpGridView A, SpGridView B, Geom g, const int64_t* __restrict__ items, int64_t n_items,
                      int32_t* __restrict__ item_count, int32_t* __restrict__ row_count,
                      int64_t* __restrict__ big_list, int32_t* __restrict__ big_n) {
  __shared__ uint32_t bm_all[kWarpsSym][kBitmapWords];
  uint32_t* bm = bm_all[threadIdx.x >> 5];
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t idx = warp; idx < n_items; idx += nwarps) {
    const ItemInfo it = decode_item(g, items[idx]);
    const int words = (it.hi - it.lo + 31) >> 5;
    for (int w = lane; w < words; w += 32) bm[w] = 0u;
    __syncwarp();
    const int lo = it.lo;
    auto setbit = [&](bool valid, int32_t j, VT, VT) {
      if (valid) atomicOr(&bm[(j - lo) >> 5], 1u << ((j - lo) & 31));
    };
    for (int64_t k = 0; k < g.gk; k++) {
      const bclx_csr_t At = A.tile(it.ti, k);
      const bclx_csr_t Bt = B.tile(k, it.tj);
      if (it.ns > 1)
        for_each_product<VT, true, false>(At, Bt, it.r, it.lo, it.hi, setbit);
      else
        for_each_product<VT, false, false>(At, Bt, it.r, it.lo, it.hi, setbit);
    }
    __syncwarp();
    int cnt = 0;
    for (int w = lane; w < words; w += 32) cnt += __popc(bm[w]);
    cnt = warp_sum(cnt);
    if (lane == 0) {
      item_count[idx] = cnt;
      if (cnt) atomicAdd(&row_count[it.ri], cnt);
      if (cnt > kVcapSmall) big_list[atomicAdd(big_n, 1)] = idx;
    }
    __syncwarp();
  }
}

// tile_row_ptr / tile_offset from the row offsets (row items are tile-major).
__global__ void k_tile_ptrs(Geom g, const int64_t* __restrict__ row_offset, int32_t* __restrict__ tile_row_ptr,
                            int64_t* __restrict__ tile_offset, int32_t* __restrict__ overflow) {
  const int64_t ntiles = g.gm * g.gn;
  const int64_t total = ntiles * (g.tm + 1);
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = x / (g.tm + 1), r = x - t * (g.tm + 1);
    const int64_t base = row_offset[t * g.tm];
    const int64_t v = row_offset[t * g.tm + r] - base;
    if (v > INT32_MAX) *overflow = 1;
    tile_row_ptr[x] = (int32_t)v;
    if (r == 0) tile_offset[t] = base;
    if (t == ntiles - 1 && r == g.tm) tile_offset[ntiles] = row_offset[g.n_row_items];
  }
}

// ---- numeric -------------------------------------------------------------------------

template <typename VT, int VCAP>
struct WarpSmem {
  uint32_t bm[kBitmapWords];
  uint32_t pre[kBitmapWords];
  VT part[VCAP];
  VT acc[VCAP];
  VT sa[32];
  VT sb[32];
};

template <typename VT, int VCAP, int WARPS, bool BIG>
__global__ void __launch_bounds__(WARPS * 32)
    k_spgemm_numeric(SpGridView A, SpGridView B, Geom g, const int64_t* __restrict__ items, int64_t n_items,
                     const int64_t* __restrict__ big_list, const int32_t* __restrict__ big_n,
                     const int32_t* __restrict__ item_count, const int64_t* __restrict__ row_offset,
                     int32_t* __restrict__ out_col, VT* __restrict__ out_val, int stage_begin, int stage_end) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem<VT, VCAP>& S = reinterpret_cast<WarpSmem<VT, VCAP>*>(smem_raw)[threadIdx.x >> 5];
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t limit = BIG ? (int64_t)*big_n : n_items;
  for (int64_t w_i = warp; w_i < limit; w_i += nwarps) {
    const int64_t idx = BIG ? big_list[w_i] : w_i;
    const int cnt = item_count[idx];
    if (!BIG && (cnt == 0 || cnt > VCAP)) continue;
    const ItemInfo it = decode_item(g, items[idx]);
    const int lo = it.lo;
    const int words = (it.hi - it.lo + 31) >> 5;

    // output offset: the row's offset plus the counts of the earlier slices
    int64_t off = 0;
    for (int q = lane; q < it.s; q += 32) off += item_count[idx - it.s + q];
    off = warp_sum(off) + row_offset[it.ri];

    // 1. bitmap of the item's output columns
    for (int w = lane; w < words; w += 32) S.bm[w] = 0u;
    __syncwarp();
    if (stage_begin == 0) {
      auto setbit = [&](bool valid, int32_t j, VT, VT) {
        if (valid) atomicOr(&S.bm[(j - lo) >> 5], 1u << ((j - lo) & 31));
      };
      for (int64_t k = 0; k < g.gk; k++) {
        const bclx_csr_t At = A.tile(it.ti, k);
        const bclx_csr_t Bt = B.tile(k, it.tj);
        if (it.ns > 1)
          for_each_product<VT, true, false>(At, Bt, it.r, it.lo, it.hi, setbit);
        else
          for_each_product<VT, false, false>(At, Bt, it.r, it.lo, it.hi, setbit);
      }
    } else {
      for (int q = lane; q < cnt; q += 32) {
        const int x = out_col[off + q] - lo;
        atomicOr(&S.bm[x >> 5], 1u << (x & 31));
      }
    }
    __syncwarp();

    // 2. per-word exclusive prefix of the popcounts
    {
      const int per = (words + 31) >> 5;
      const int w0 = lane * per;
      int loc = 0;
      for (int w = w0; w < w0 + per && w < words; w++) loc += __popc(S.bm[w]);
      int ex = warp_inclusive_scan(loc) - loc;
      for (int w = w0; w < w0 + per && w < words; w++) {
        S.pre[w] = ex;
        ex += __popc(S.bm[w]);
      }
    }
    __syncwarp();

    // 3. sorted columns (first pass only) and accumulator start values
    if (stage_begin == 0) {
      for (int w = lane; w < words; w += 32) {
        uint32_t bits = S.bm[w];
        int pos = S.pre[w];
        while (bits) {
          const int b = __ffs(bits) - 1;
          bits &= bits - 1;
          out_col[off + pos++] = lo + w * 32 + b;
        }
      }
    }
    VT* acc = S.acc;
    VT* part = S.part;
    for (int q = lane; q < cnt; q += 32) {
      acc[q] = stage_begin == 0 ? VT(0) : out_val[off + q];
      part[q] = VT(0);
    }
    bool acc_zero = stage_begin == 0;
    __syncwarp();

    // 4. values, stage by stage in rotated order
    for (int kk = stage_begin; kk < stage_end; kk++) {
      const int64_t k = (kk + it.ti + it.tj) % g.gk;
      const bclx_csr_t At = A.tile(it.ti, k);
      const bclx_csr_t Bt = B.tile(k, it.tj);
      bool any = false;
      auto update = [&](bool valid, int32_t j, VT a, VT b) {
        any = true;
        int rank = 0;
        if (valid) {
          const int x = j - lo;
          rank = S.pre[x >> 5] + __popc(S.bm[x >> 5] & ((1u << (x & 31)) - 1u));
        }
        const unsigned peers = __match_any_sync(kFull, valid ? j : -1);
        S.sa[lane] = a;
        S.sb[lane] = b;
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) {
          VT v = part[rank];
          unsigned gmask = peers;
          do {
            const int mbr = __ffs(gmask) - 1;
            gmask &= gmask - 1;
            v = madd(S.sa[mbr], S.sb[mbr], v);
          } while (gmask);
          part[rank] = v;
        }
        __syncwarp();
      };
      if (it.ns > 1)
        for_each_product<VT, true, true>(At, Bt, it.r, it.lo, it.hi, update);
      else
        for_each_product<VT, false, true>(At, Bt, it.r, it.lo, it.hi, update);
      if (!any) continue;
      if (acc_zero) {
        // 0 + partial == partial: swap roles instead of adding (the old
        // accumulator is all zeros and becomes the next partial).
        VT* t = acc;
        acc = part;
        part = t;
        acc_zero = false;
      } else {
        for (int q = lane; q < cnt; q += 32) {
          acc[q] = vadd(acc[q], part[q]);
          part[q] = VT(0);
        }
      }
      __syncwarp();
    }

    // 5. values out
    for (int q = lane; q < cnt; q += 32) out_val[off + q] = acc[q];
    __syncwarp();
  }
}

// ---- identity tiles (tile accumulation as a product) ------------------------------

template <typename VT>
__global__ void k_identity(int64_t m, int32_t* __restrict__ rp, int32_t* __restrict__ ci, VT* __restrict__ v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += (int64_t)gridDim.x * blockDim.x) {
    rp[i] = (int32_t)i;
    if (i < m) {
      ci[i] = (int32_t)i;
      v[i] = VT(1);
    }
  }
}

__global__ void k_fill_desc(bclx_csr_t* __restrict__ d, int n, bclx_csr_t v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = v;
}

}  // namespace bclx

using namespace bclx;

struct bclx_spgemm_plan_s {
  Context* ctx = nullptr;
  Geom g{};
  int dtype = BCLX_F32;
  int64_t products = 0, n_items = 0, nnz = 0, n_big = 0;
  int64_t* ub = nullptr;
  int32_t* nslices = nullptr;
  int64_t* first = nullptr;
  int64_t* items = nullptr;
  int32_t* item_count = nullptr;
  int32_t* row_count = nullptr;
  int64_t* row_offset = nullptr;
  int64_t* big_list = nullptr;
  int32_t* flags = nullptr;  // [0] big count, [1] overflow
  unsigned long long* products_dev = nullptr;
  // tile accumulation: identity A tiles and their descriptors, 1x1 C offsets
  int32_t* id_rp = nullptr;
  int32_t* id_ci = nullptr;
  void* id_v = nullptr;
  bclx_csr_t* id_desc = nullptr;
  int64_t* acc_tile_offset = nullptr;

  void release() {
    void* ps[] = {ub, nslices, first, items, item_count, row_count, row_offset, big_list, flags, products_dev,
                  id_rp, id_ci, id_v, id_desc, acc_tile_offset};
    for (void* p : ps) scratch_free(ctx, p);
    ub = nullptr; nslices = nullptr; first = nullptr; items = nullptr; item_count = nullptr;
    row_count = nullptr; row_offset = nullptr; big_list = nullptr; flags = nullptr; products_dev = nullptr;
    id_rp = nullptr; id_ci = nullptr; id_v = nullptr; id_desc = nullptr; acc_tile_offset = nullptr;
  }
};

namespace bclx {

static int value_size(int dtype) { return dtype == BCLX_F32 || dtype == BCLX_I32 ? 4 : 0; }

static int check_grids(const bclx_spgrid_t* a, const bclx_spgrid_t* b, const bclx_spgrid_out_t* c) {
  if (!a || !b || !c || !a->tiles || !b->tiles) return BCLX_ERR_INVALID;
  auto grid_ok = [](int64_t m, int64_t n, int64_t tm, int64_t tn, int64_t gm, int64_t gn) {
    return m >= 0 && n >= 0 && tm > 0 && tn > 0 && gm == ceil_div(m, tm) && gn == ceil_div(n, tn);
  };
  if (!grid_ok(a->m, a->n, a->tile_m, a->tile_n, a->grid_m, a->grid_n)) return BCLX_ERR_INVALID;
  if (!grid_ok(b->m, b->n, b->tile_m, b->tile_n, b->grid_m, b->grid_n)) return BCLX_ERR_INVALID;
  if (!grid_ok(c->m, c->n, c->tile_m, c->tile_n, c->grid_m, c->grid_n)) return BCLX_ERR_INVALID;
  if (a->n != b->m || a->m != c->m || b->n != c->n) return BCLX_ERR_INVALID;
  if (a->tile_n != b->tile_m || a->grid_n != b->grid_m) return BCLX_ERR_INVALID;
  if (a->tile_m != c->tile_m || b->tile_n != c->tile_n) return BCLX_ERR_INVALID;
  if (a->grid_n < 1 || a->grid_n > INT32_MAX) return BCLX_ERR_INVALID;
  if (c->tile_n > (int64_t)1023 * kSliceCols) return BCLX_ERR_INVALID;
  if (a->tile_m > INT32_MAX || b->tile_n > INT32_MAX) return BCLX_ERR_INDEX_OVERFLOW;
  if (a->dtype != b->dtype || a->dtype != c->dtype || !value_size(a->dtype)) return BCLX_ERR_DTYPE;
  return BCLX_OK;
}

static unsigned grid_for(Context* ctx, int64_t work_warps, int warps_per_block, int blocks_per_sm) {
  int64_t want = (work_warps + warps_per_block - 1) / warps_per_block;
  int64_t cap = (int64_t)ctx->num_sms * blocks_per_sm;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return (unsigned)want;
}

template <typename VT>
static int launch_symbolic(Context* ctx, const SpGridView& A, const SpGridView& B, bclx_spgemm_plan_s* P) {
  unsigned blocks = grid_for(ctx, P->n_items, kWarpsSym, 16);
  k_spgemm_symbolic<VT><<<blocks, kWarpsSym * 32, 0, ctx->stream>>>(A, B, P->g, P->items, P->n_items,
                                                                   P->item_count, P->row_count, P->big_list,
                                                                   P->flags);
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

template <typename VT>
static int launch_numeric(Context* ctx, const SpGridView& A, const SpGridView& B, bclx_spgemm_plan_s* P,
                          int32_t* out_col, void* out_val, int s0, int s1) {
  constexpr size_t small_smem = sizeof(WarpSmem<VT, kVcapSmall>) * kWarpsSmall;
  constexpr size_t big_smem = sizeof(WarpSmem<VT, kVcapBig>) * kWarpsBig;
  auto ks = k_spgemm_numeric<VT, kVcapSmall, kWarpsSmall, false>;
  auto kb = k_spgemm_numeric<VT, kVcapBig, kWarpsBig, true>;
  BCLX_CK(cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)small_smem));
  BCLX_CK(cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)big_smem));
  unsigned blocks = grid_for(ctx, P->n_items, kWarpsSmall, 4);
  ks<<<blocks, kWarpsSmall * 32, small_smem, ctx->stream>>>(A, B, P->g, P->items, P->n_items, P->big_list,
                                                           P->flags, P->item_count, P->row_offset, out_col,
                                                           reinterpret_cast<VT*>(out_val), s0, s1);
  BCLX_CK_LAUNCH();
  if (P->n_big > 0) {
    unsigned bb = grid_for(ctx, P->n_big, kWarpsBig, 1);
    kb<<<bb, kWarpsBig * 32, big_smem, ctx->stream>>>(A, B, P->g, P->items, P->n_items, P->big_list, P->flags,
                                                     P->item_count, P->row_offset, out_col,
                                                     reinterpret_cast<VT*>(out_val), s0, s1);
    BCLX_CK_LAUNCH();
  }
  return BCLX_OK;
}

// Plan + symbolic over validated views; fills the plan and the C offsets.
static int symbolic_impl(Context* ctx, const SpGridView& A, const SpGridView& B, const Geom& g, int dtype,
                         int32_t* tile_row_ptr, int64_t* tile_offset, bclx_spgemm_plan_s* P) {
  P->g = g;
  P->dtype = dtype;
  const int64_t nri = g.n_row_items;
  BCLX_TRY(scratch_alloc_n(ctx, &P->ub, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->nslices, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->first, nri + 1));
  BCLX_TRY(scratch_alloc_n(ctx, &P->flags, 4));
  BCLX_TRY(scratch_alloc_n(ctx, &P->products_dev, 1));
  BCLX_CK(cudaMemsetAsync(P->flags, 0, 4 * sizeof(int32_t), ctx->stream));
  BCLX_CK(cudaMemsetAsync(P->products_dev, 0, sizeof(unsigned long long), ctx->stream));
  if (nri > 0) {
    k_spgemm_ub<<<grid_for(ctx, nri, 8, 16), 256, 0, ctx->stream>>>(A, B, g, P->ub, P->nslices, P->products_dev);
    BCLX_CK_LAUNCH();
  }
  BCLX_TRY(exclusive_scan_i32(ctx, P->nslices, P->first, nri));
  BCLX_CK(cudaMemcpyAsync(ctx->pinned, P->first + nri, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaMemcpyAsync(ctx->pinned + 1, P->products_dev, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  P->n_items = ctx->pinned[0];
  P->products = ctx->pinned[1];

  BCLX_TRY(scratch_alloc_n(ctx, &P->items, P->n_items));
  BCLX_TRY(scratch_alloc_n(ctx, &P->item_count, P->n_items));
  BCLX_TRY(scratch_alloc_n(ctx, &P->big_list, P->n_items));
  BCLX_TRY(scratch_alloc_n(ctx, &P->row_count, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->row_offset, nri + 1));
  BCLX_CK(cudaMemsetAsync(P->row_count, 0, sizeof(int32_t) * (nri > 0 ? nri : 1), ctx->stream));
  if (nri > 0) {
    k_build_items<<<grid_for(ctx, nri / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(g, P->nslices, P->first, P->items);
    BCLX_CK_LAUNCH();
  }
  if (P->n_items > 0) {
    if (dtype == BCLX_F32) BCLX_TRY(launch_symbolic<float>(ctx, A, B, P));
    else BCLX_TRY(launch_symbolic<int32_t>(ctx, A, B, P));
  }
  BCLX_TRY(exclusive_scan_i32(ctx, P->row_count, P->row_offset, nri));
  const int64_t ntiles = g.gm * g.gn;
  k_tile_ptrs<<<grid_for(ctx, ntiles * (g.tm + 1) / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(
      g, P->row_offset, tile_row_ptr, tile_offset, P->flags + 1);
  BCLX_CK_LAUNCH();
  BCLX_CK(cudaMemcpyAsync(ctx->pinned, P->row_offset + nri, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaMemcpyAsync(ctx->pinned + 1, P->flags, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  P->nnz = ctx->pinned[0];
  int32_t fl[2];
  std::memcpy(fl, ctx->pinned + 1, sizeof(fl));
  P->n_big = fl[0];
  if (fl[1]) {
    set_last_error("a C tile has more than 2^31-1 nonzeros; use a finer tile grid");
    return BCLX_ERR_INDEX_OVERFLOW;
  }
  // ub and nslices are not needed after planning
  scratch_free(ctx, P->ub);
  scratch_free(ctx, P->nslices);
  P->ub = nullptr;
  P->nslices = nullptr;
  return BCLX_OK;
}

static int numeric_impl(Context* ctx, bclx_spgemm_plan_s* P, const SpGridView& A, const SpGridView& B,
                        int32_t* out_col, void* out_val, int s0, int s1) {
  if (s1 <= 0 || s1 > P->g.gk) s1 = (int)P->g.gk;
  if (s0 < 0 || s0 > s1) return BCLX_ERR_INVALID;
  if (P->n_items == 0 || s0 == s1) return BCLX_OK;
  if (P->dtype == BCLX_F32) return launch_numeric<float>(ctx, A, B, P, out_col, out_val, s0, s1);
  return launch_numeric<int32_t>(ctx, A, B, P, out_col, out_val, s0, s1);
}

static Geom make_geom(const bclx_spgrid_out_t* c, int64_t gk) {
  Geom g;
  g.gm = c->grid_m; g.gn = c->grid_n; g.gk = gk;
  g.tm = c->tile_m; g.tn = c->tile_n; g.m = c->m; g.n = c->n;
  g.n_row_items = g.gm * g.gn * g.tm;
  return g;
}

}  // namespace bclx

extern "C" {

int bclx_spgemm_symbolic(bclx_context_t c, const bclx_spgrid_t* a, const bclx_spgrid_t* b, bclx_spgrid_out_t* out,
                         bclx_spgemm_plan_t* plan, int64_t* nnz) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !plan || !nnz) return BCLX_ERR_INVALID;
  *plan = nullptr;
  BCLX_TRY(check_grids(a, b, out));
  if (!out->tile_row_ptr || !out->tile_offset) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  auto* P = new bclx_spgemm_plan_s();
  P->ctx = ctx;
  int rc = symbolic_impl(ctx, make_view(*a), make_view(*b), make_geom(out, a->grid_n), a->dtype,
                         out->tile_row_ptr, out->tile_offset, P);
  if (rc != BCLX_OK) {
    P->release();
    delete P;
    return rc;
  }
  *nnz = P->nnz;
  *plan = P;
  return BCLX_OK;
}

int bclx_spgemm_numeric(bclx_context_t c, bclx_spgemm_plan_t P, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                        bclx_spgrid_out_t* out, int32_t stage_begin, int32_t stage_end) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !P) return BCLX_ERR_INVALID;
  BCLX_TRY(check_grids(a, b, out));
  if (a->grid_n != P->g.gk || out->grid_m != P->g.gm || out->grid_n != P->g.gn || a->dtype != P->dtype)
    return BCLX_ERR_INVALID;
  if (P->nnz > 0 && (!out->col_ind || !out->vals)) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  return numeric_impl(ctx, P, make_view(*a), make_view(*b), out->col_ind, out->vals, stage_begin, stage_end);
}

int bclx_spgemm_plan_destroy(bclx_spgemm_plan_t P) {
  if (!P) return BCLX_OK;
  cudaSetDevice(P->ctx->device);
  P->release();
  delete P;
  return BCLX_OK;
}

int bclx_spgemm_plan_stats(bclx_spgemm_plan_t P, int64_t* out6) {
  if (!P || !out6) return BCLX_ERR_INVALID;
  out6[0] = P->products;
  out6[1] = P->g.n_row_items;
  out6[2] = P->n_items;
  out6[3] = P->n_big;
  out6[4] = P->g.gk;
  out6[5] = P->nnz;
  return BCLX_OK;
}

// Tile accumulation as a product: A = [I I ... I] (1 x nparts identity
// tiles, value 1), B = [parts] (nparts x 1).  With a 1x1 C grid the stage
// order is the list order, each partial value passes through fma(1, v, 0) == v
// exactly, and the partials are added from 0 in list order: the
// SparseHashAccumulator sum.
static int accumulate_views(bclx_spgemm_plan_s* P, Context* ctx, const bclx_csr_t* parts, int32_t nparts,
                            int64_t m, int64_t n, int32_t dtype, SpGridView* A, SpGridView* B, Geom* g) {
  A->tiles = P->id_desc;
  A->m = m; A->n = m * (int64_t)nparts; A->tm = m; A->tn = m; A->gm = 1; A->gn = nparts;
  B->tiles = parts;
  B->m = m * (int64_t)nparts; B->n = n; B->tm = m; B->tn = n; B->gm = nparts; B->gn = 1;
  g->gm = 1; g->gn = 1; g->gk = nparts; g->tm = m; g->tn = n; g->m = m; g->n = n; g->n_row_items = m;
  (void)ctx; (void)dtype;
  return BCLX_OK;
}

int bclx_tile_accumulate_symbolic(bclx_context_t c, const bclx_csr_t* parts, int32_t nparts, int64_t m, int64_t n,
                                  int32_t dtype, int32_t* c_row_ptr, bclx_spgemm_plan_t* plan, int64_t* nnz) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !plan || !nnz || !parts || nparts < 1 || m < 1 || n < 1 || !c_row_ptr) return BCLX_ERR_INVALID;
  if (m > INT32_MAX || n > (int64_t)1023 * kSliceCols) return BCLX_ERR_INVALID;
  if (!value_size(dtype)) return BCLX_ERR_DTYPE;
  *plan = nullptr;
  BCLX_CK(cudaSetDevice(ctx->device));
  auto* P = new bclx_spgemm_plan_s();
  P->ctx = ctx;
  int rc = BCLX_OK;
  do {
    if ((rc = scratch_alloc_n(ctx, &P->id_rp, m + 1))) break;
    if ((rc = scratch_alloc_n(ctx, &P->id_ci, m))) break;
    if ((rc = scratch_alloc(ctx, &P->id_v, 4 * (size_t)m))) break;
    if ((rc = scratch_alloc_n(ctx, &P->id_desc, nparts))) break;
    if ((rc = scratch_alloc_n(ctx, &P->acc_tile_offset, 2))) break;
    unsigned blocks = grid_for(ctx, m / 256 + 1, 8, 8);
    if (dtype == BCLX_F32)
      k_identity<float><<<blocks, 256, 0, ctx->stream>>>(m, P->id_rp, P->id_ci, (float*)P->id_v);
    else
      k_identity<int32_t><<<blocks, 256, 0, ctx->stream>>>(m, P->id_rp, P->id_ci, (int32_t*)P->id_v);
    bclx_csr_t d{};
    d.m = m; d.n = m; d.nnz = m; d.row_ptr = P->id_rp; d.col_ind = P->id_ci; d.vals = P->id_v; d.dtype = dtype;
    k_fill_desc<<<1, 256, 0, ctx->stream>>>(P->id_desc, nparts, d);
    if (cudaGetLastError() != cudaSuccess) { rc = BCLX_ERR_CUDA; break; }
    SpGridView A{}, B{};
    Geom g{};
    accumulate_views(P, ctx, parts, nparts, m, n, dtype, &A, &B, &g);
    rc = symbolic_impl(ctx, A, B, g, dtype, c_row_ptr, P->acc_tile_offset, P);
  } while (0);
  if (rc != BCLX_OK) {
    P->release();
    delete P;
    return rc;
  }
  *nnz = P->nnz;
  *plan = P;
  return BCLX_OK;
}

int bclx_tile_accumulate_numeric(bclx_context_t c, bclx_spgemm_plan_t P, const bclx_csr_t* parts, int32_t nparts,
                                 bclx_csr_t* out) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !P || !parts || !out || !P->id_desc || nparts != P->g.gk) return BCLX_ERR_INVALID;
  if (out->m != P->g.m || out->n != P->g.n || out->dtype != P->dtype) return BCLX_ERR_INVALID;
  if (P->nnz > 0 && (!out->col_ind || !out->vals)) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  SpGridView A{}, B{};
  Geom g{};
  accumulate_views(P, ctx, parts, nparts, out->m, out->n, P->dtype, &A, &B, &g);
  return numeric_impl(ctx, P, A, B, out->col_ind, out->vals, 0, nparts);
}

}  // extern "C"
