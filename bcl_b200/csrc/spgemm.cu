// Sparse x sparse product over tile grids (the SUMMA tile loop of
// BCL::gemm(SPMatrix, SPMatrix, SPMatrix&), bcl/containers/algorithms/
// spgemm.hpp:182-242, with its local kernel spgemm.hpp:41-76 and the tile
// accumulation of SparseHashAccumulator.hpp:101-182), and tile accumulation.
//
// Work decomposition.  A "row" is one row r of one C tile (i, j); it owns the
// products A_ik[r, :] * B_kj over every stage k.  Its intermediate-product
// count (ub) classifies it:
//   light (ub <= kLightUb):  one warp does the symbolic count and, later, the
//                            whole numeric row (at most kLightUb outputs);
//   heavy:                   one block does the symbolic pass (no ordering is
//                            needed there) and leaves the row's column bitmap
//                            in global memory; the row is then cut at
//                            kFineCols-column block boundaries into items of
//                            at most kVcap outputs, one warp each.
// B rows are cut at the same block boundaries by a per-row table, so a heavy
// item finds its part of every B row with two loads.
//
// Numeric, per item (one warp): the item's column bitmap (rebuilt from the
// products for light rows, loaded for heavy items) is turned into per-word
// prefix counts, so that column j's output position is
// rank(j) = prefix[j/32] + popc(lower bits of its word); sorted columns are
// written directly.  Then the products are walked in the reference's order
// and values are accumulated in shared memory at rank(j).
//
// Order.  The product stream of a row is: stages k = (k_ + i + j) mod G for
// k_ = 0..G-1; inside a stage the A-row entries in stored order; inside an
// entry the B-row entries in stored order.  It is walked 32 products at a
// time, packed across A entries and stages.  Lanes holding the same column
// are grouped with __match_any_sync and the lowest lane applies the group's
// updates in lane order; batches are separated by __syncwarp.  Every column
// keeps a running stage partial (`part`, started at 0 and advanced with a
// fused multiply-add per product) and the sum of its finished stage partials
// (`acc`, started at 0); when a product of a later stage arrives the partial
// is added to acc first.  That is exactly the reference's arithmetic: each
// tile product is an FMA chain from 0 in A-row order, and the partial tiles
// are added from 0 in stage order.  FP32 results are bit-identical; int32
// uses wrapping arithmetic and is exact.
#include "common.cuh"

#include <cstdlib>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <initializer_list>
#include <mutex>
#include <tuple>
#include <vector>

namespace bclx {

constexpr int kLightUb = 512;        // products of a light row (so <= 512 outputs)
constexpr int kVcap = 512;           // outputs per numeric item (the default; BCLX_TUNE_ITEM_OUTPUTS: 512 or 1024)
constexpr int kFineCols = 256;       // column block of heavy rows and of the B-row table
constexpr int kMaxWords = 512;       // bitmap words per warp (tiles up to 16384 columns)
constexpr int kMaxCols = kMaxWords * 32;
constexpr int kWarpsSym = 8;
constexpr int kWarpsNum = 8;
constexpr int kNoStage = 0xff;
constexpr int kLongSegDefault = 32;       // B segments at least this long are walked in direct mode
constexpr int kQueueSlots = 256;          // work-queue heads in a plan (one per stage launch)
constexpr int64_t kVeryHeavyUb = 32768;  // rows above this many products get a whole block in the symbolic pass

struct Geom {
  int64_t gm, gk, gn;   // C grid is gm x gn; the k grid has gk tiles
  int64_t tm, tn, tk;   // C tile shape; A tile width (= B tile height)
  int64_t m, n;         // C shape
  int64_t n_row_items;  // gm * gn * tm
  int64_t nfb;          // fine blocks per (full) tile width: ceil(tn / kFineCols)
  // Stage map (or null: every stage): for C tile t = ti*gn + tj, scount[t]
  // positions kk (ascending) of the rotated order k = (kk + rotation) mod gk
  // whose A_ik and B_kj tiles both have entries, in smap[t*gk ...].
  const int32_t* smap = nullptr;
  const int32_t* scount = nullptr;
  // Sub-grid products (or null: C's tile (ti, tj) is global tile (ti, tj)):
  // the global tile row / column of each C tile row / column, which sets
  // the rotated stage order k = (kk + gi + gj) mod gk.
  const int32_t* rot_i = nullptr;
  const int32_t* rot_j = nullptr;
};

// Rotation of C tile (ti, tj): stage position kk is k = (kk + rotation) mod gk.
__device__ __forceinline__ int64_t tile_rotation(const Geom& g, int64_t ti, int64_t tj) {
  const int64_t gi = g.rot_i ? (int64_t)__ldg(g.rot_i + ti) : ti;
  const int64_t gj = g.rot_j ? (int64_t)__ldg(g.rot_j + tj) : tj;
  return (gi + gj) % g.gk;
}

__device__ __forceinline__ int stage_count(const Geom& g, int64_t ti, int64_t tj) {
  return g.scount ? __ldg(g.scount + ti * g.gn + tj) : (int)g.gk;
}
__device__ __forceinline__ int stage_at(const Geom& g, int64_t ti, int64_t tj, int s) {
  return g.smap ? __ldg(g.smap + (ti * g.gn + tj) * g.gk + s) : s;
}
// Stage-list window [lo, hi) of the positions kk in [s0, s1) (warp-uniform).
__device__ __forceinline__ void stage_window(const Geom& g, int64_t ti, int64_t tj, int s0, int s1, int& lo,
                                             int& hi) {
  if (!g.smap) {
    lo = s0;
    hi = s1;
    return;
  }
  const int ns = stage_count(g, ti, tj);
  if (s0 <= 0 && s1 >= g.gk) {
    lo = 0;
    hi = ns;
    return;
  }
  int c0 = 0, c1 = 0;
  for (int b = 0; b < ns; b += 32) {
    const int si = b + (int)(threadIdx.x & 31);
    const int kk = si < ns ? stage_at(g, ti, tj, si) : INT_MAX;
    c0 += __popc(__ballot_sync(0xffffffffu, kk < s0));
    c1 += __popc(__ballot_sync(0xffffffffu, kk < s1));
  }
  lo = c0;
  hi = c1;
}

// Entries [bs, be) of B row kc whose columns lie in fine blocks
// [fb_lo, fb_hi): from the B-row table rows `trows` of the tile when there is
// one, otherwise by binary search of the row's sorted columns.
__device__ __forceinline__ void b_block_range(const int32_t* trows, const int32_t* brp, const int32_t* bci,
                                              int32_t kc, int fb_lo, int fb_hi, int64_t nfb, int32_t& bs,
                                              int32_t& be) {
  if (trows) {
    const int32_t* trow = trows + (int64_t)kc * (nfb + 1);
    bs = __ldg(trow + fb_lo);
    be = __ldg(trow + fb_hi);
  } else {
    const int32_t b0 = __ldg(brp + kc), b1 = __ldg(brp + kc + 1);
    bs = fb_lo == 0 ? b0 : lower_bound_i32(bci, b0, b1, fb_lo * kFineCols);
    be = fb_hi >= nfb ? b1 : lower_bound_i32(bci, bs, b1, fb_hi * kFineCols);
  }
}

struct RowInfo {
  int64_t ti, tj, r;
  int64_t rot;  // the C tile's stage rotation (tile_rotation)
  int w;        // width of the C tile (columns)
};

__device__ __forceinline__ RowInfo decode_row(const Geom& g, int64_t ri) {
  RowInfo x;
  const int64_t t = ri / g.tm;
  x.r = ri - t * g.tm;
  x.ti = t / g.gn;
  x.tj = t - x.ti * g.gn;
  x.rot = tile_rotation(g, x.ti, x.tj);
  int64_t w = g.n - x.tj * g.tn;
  x.w = (int)(w < g.tn ? w : g.tn);
  return x;
}

template <typename VT>
__device__ __forceinline__ VT load_val(const void* p, int64_t i) {
  return __ldg(reinterpret_cast<const VT*>(p) + i);
}

// Number of lanes whose inclusive prefix is <= q (incl is nondecreasing).
__device__ __forceinline__ int warp_search(int32_t incl, int32_t q) {
  int src = 0;
#pragma unroll
  for (int step = 16; step >= 1; step >>= 1) {
    const int32_t v = __shfl_sync(kFull, incl, src + step - 1);
    if (v <= q) src += step;
  }
  return src;
}

template <typename P>
__device__ __forceinline__ P* shfl_ptr(P* p, int src) {
  unsigned long long u = reinterpret_cast<unsigned long long>(p);
  u = __shfl_sync(kFull, u, src);
  return reinterpret_cast<P*>(u);
}

// Walk the product stream of C-tile row `x` over stages [s0, s1), restricted
// to fine blocks [fb_lo, fb_hi) of the row when RANGED (through the B-row
// table `tab`), in the reference's order.
//
// One lane per stage first reads that stage's A-row segment and B-tile
// pointers.  The A entries of the row (all stages, flattened) are then taken
// 32 at a time, one per lane, each finding its B segment.  An entry whose B
// segment has at least kLongSeg products is walked in "direct" mode: lanes
// stride over the segment and each lane calls fd(j, a, b, stage) for its own
// products (the columns of one B row are distinct, so lanes never touch the
// same column; a __syncwarp follows the segment).  Runs of shorter entries
// are packed 32 products per batch and every lane calls f(valid, j, a, b,
// stage) once per batch (warp-uniform); valid lanes form a prefix of the warp
// and lane order is product order.  The loads of batch n+1 are issued before
// f runs on batch n.
template <typename VT, bool RANGED, typename F, typename FD>
__device__ __forceinline__ void walk_products(const SpGridView& A, const SpGridView& B, const Geom& g,
                                              const RowInfo& x, int s0, int s1, int fb_lo, int fb_hi,
                                              const int32_t* __restrict__ tab, int long_seg, F&& f, FD&& fd) {
  const int lane = lane_id();
  int w0, w1;
  stage_window(g, x.ti, x.tj, s0, s1, w0, w1);
  for (int g0 = w0; g0 < w1; g0 += 32) {
    // one lane per stage: its A-row segment and its B tile
    const int si = g0 + lane;
    int kk = 0;
    int32_t as = 0, alen = 0;
    const int32_t* acol = nullptr;
    const VT* aval = nullptr;
    const int32_t* brow = nullptr;   // B row_ptr
    const int32_t* btrows = nullptr;  // the stage's B-row table block (RANGED, when there is a table)
    const int32_t* bci = nullptr;
    const VT* bva = nullptr;
    if (si < w1) {
      kk = stage_at(g, x.ti, x.tj, si);
      const int64_t k = (kk + x.rot) % g.gk;
      const bclx_csr_t At = A.tile(x.ti, k);
      as = __ldg(At.row_ptr + x.r);
      alen = __ldg(At.row_ptr + x.r + 1) - as;
      acol = At.col_ind + as;
      aval = reinterpret_cast<const VT*>(At.vals) + as;
      const bclx_csr_t Bt = B.tile(k, x.tj);
      brow = Bt.row_ptr;
      if (RANGED && tab) btrows = tab + (k * g.gn + x.tj) * g.tk * (g.nfb + 1);
      bci = Bt.col_ind;
      bva = reinterpret_cast<const VT*>(Bt.vals);
    }
    const int32_t aincl = warp_inclusive_scan(alen);
    const int32_t atot = __shfl_sync(kFull, aincl, 31);
    const int32_t aexcl = aincl - alen;
    for (int32_t e0 = 0; e0 < atot; e0 += 32) {
      // one lane per A entry of the flattened stage stream
      const int32_t e = e0 + lane;
      const int sl = warp_search(aincl, e);
      const int32_t off = e - __shfl_sync(kFull, aexcl, sl);
      const int32_t* sacol = shfl_ptr(acol, sl);
      const VT* saval = shfl_ptr(aval, sl);
      const int32_t* sbrow = shfl_ptr(brow, sl);
      const int32_t* sbci = shfl_ptr(bci, sl);
      const VT* sbva = shfl_ptr(bva, sl);
      const int32_t* sbtr = RANGED ? shfl_ptr(btrows, sl) : nullptr;
      const int stage = __shfl_sync(kFull, kk, sl);
      int32_t len = 0;
      VT av = VT(0);
      const int32_t* bcol = nullptr;
      const VT* bval = nullptr;
      if (e < atot) {
        const int32_t kc = __ldg(sacol + off);
        av = __ldg(saval + off);
        int32_t bs, be;
        if (RANGED) {
          b_block_range(sbtr, sbrow, sbci, kc, fb_lo, fb_hi, g.nfb, bs, be);
        } else {
          bs = __ldg(sbrow + kc);
          be = __ldg(sbrow + kc + 1);
        }
        len = be - bs;
        bcol = sbci + bs;
        bval = sbva + bs;
      }
      const int nent = min(32, atot - e0);
      const unsigned longm = __ballot_sync(kFull, len >= long_seg);
      int e_start = 0;
      while (e_start < nent) {
        const unsigned lm = longm & (kFull << e_start);
        const int e_long = lm ? __ffs(lm) - 1 : nent;
        if (e_long > e_start) {
          // packed batches over the short entries [e_start, e_long), software pipelined
          const int32_t lenm = (lane >= e_start && lane < e_long) ? len : 0;
          const int32_t incl = warp_inclusive_scan(lenm);
          const int32_t total = __shfl_sync(kFull, incl, 31);
          const int32_t excl = incl - lenm;
          int32_t nj = -1;
          VT na = VT(0), nb = VT(0);
          int nst = 0;
          auto fetch = [&](int32_t base) {
            const int32_t q = base + lane;
            const int src = warp_search(incl, q);
            const int32_t pos = q - __shfl_sync(kFull, excl, src);
            const int32_t* sbcol = shfl_ptr(bcol, src);
            const VT* sbval = shfl_ptr(bval, src);
            na = __shfl_sync(kFull, av, src);
            nst = __shfl_sync(kFull, stage, src);
            nj = -1;
            nb = VT(0);
            if (q < total) {
              nj = __ldg(sbcol + pos);
              nb = __ldg(sbval + pos);
            }
          };
          if (total > 0) fetch(0);
          for (int32_t base = 0; base < total; base += 32) {
            const int32_t j = nj;
            const VT a = na, b = nb;
            const int st = nst;
            if (base + 32 < total) fetch(base + 32);
            f(j >= 0, j, a, b, st);
          }
        }
        if (e_long < nent) {
          // direct mode over one long segment
          const int32_t dl = __shfl_sync(kFull, len, e_long);
          const int32_t* dcol = shfl_ptr(bcol, e_long);
          const VT* dval = shfl_ptr(bval, e_long);
          const VT da = __shfl_sync(kFull, av, e_long);
          const int dst = __shfl_sync(kFull, stage, e_long);
          int32_t q = lane;
          for (; q + 32 < dl; q += 64) {
            const int32_t j0 = __ldg(dcol + q), j1 = __ldg(dcol + q + 32);
            const VT b0 = __ldg(dval + q), b1 = __ldg(dval + q + 32);
            fd(j0, da, b0, dst);
            fd(j1, da, b1, dst);
          }
          if (q < dl) fd(__ldg(dcol + q), da, __ldg(dval + q), dst);
          __syncwarp();
        }
        e_start = e_long + 1;
      }
    }
  }
}

// Order-free walk for the symbolic pass: calls fs(j) for every product
// column of C-tile row `x` (all stages).  Short B segments are looped over by
// their own lane, long ones by the whole warp.  With nparts walkers (the warps
// of a block): when the row has at least 2 * nparts chunks of 32 A entries,
// each walker takes every nparts-th chunk whole (short and long segments);
// otherwise every walker reads every chunk and takes every nparts-th chunk of
// short segments and an interleaved share of every long segment.
template <typename FS>
__device__ __forceinline__ void walk_columns(const SpGridView& A, const SpGridView& B, const Geom& g,
                                             const RowInfo& x, int part, int nparts, FS&& fs) {
  const int lane = lane_id();
  const int ns = stage_count(g, x.ti, x.tj);
  for (int g0 = 0; g0 < ns; g0 += 32) {
    const int si = g0 + lane;
    int32_t as = 0, alen = 0;
    const int32_t* acol = nullptr;
    const int32_t* brp = nullptr;
    const int32_t* bci = nullptr;
    if (si < ns) {
      const int64_t k = (stage_at(g, x.ti, x.tj, si) + x.rot) % g.gk;
      const bclx_csr_t At = A.tile(x.ti, k);
      as = __ldg(At.row_ptr + x.r);
      alen = __ldg(At.row_ptr + x.r + 1) - as;
      acol = At.col_ind;
      const bclx_csr_t Bt = B.tile(k, x.tj);
      brp = Bt.row_ptr;
      bci = Bt.col_ind;
    }
    const int32_t aincl = warp_inclusive_scan(alen);
    const int32_t atot = __shfl_sync(kFull, aincl, 31);
    const int32_t aexcl = aincl - alen;
    // chunk x's A column (one entry per lane) and its B tile, loaded one
    // chunk ahead so the column load of the next chunk is in flight while
    // the current chunk's B rows are read
    struct Ent {
      int32_t kc;
      const int32_t* brp;
      const int32_t* bci;
    };
    auto load_ent = [&](int32_t e0) {
      Ent t{0, nullptr, nullptr};
      const int32_t e = e0 + lane;
      const int sl = warp_search(aincl, e);
      const int32_t sas = __shfl_sync(kFull, as, sl);
      const int32_t sax = __shfl_sync(kFull, aexcl, sl);
      const int32_t* sacol = shfl_ptr(acol, sl);
      t.brp = shfl_ptr(brp, sl);
      t.bci = shfl_ptr(bci, sl);
      if (e < atot) t.kc = __ldg(sacol + sas + (e - sax));
      return t;
    };
    // whole chunks per walker, or every chunk read by every walker
    const bool own = nparts > 1 && atot >= 64 * nparts;
    const int32_t first = own ? 32 * part : 0;
    const int32_t stride = own ? 32 * nparts : 32;
    const int wpart = own ? 0 : part;  // this walker's share within a chunk
    const int wparts = own ? 1 : nparts;
    Ent nxt = first < atot ? load_ent(first) : Ent{0, nullptr, nullptr};
    for (int32_t e0 = first, chunk = 0; e0 < atot; e0 += stride, chunk++) {
      const Ent cur = nxt;
      const int32_t e = e0 + lane;
      if (e0 + stride < atot) nxt = load_ent(e0 + stride);
      const int32_t* sbci = cur.bci;
      int32_t bs = 0, be = 0;
      if (e < atot) {
        bs = __ldg(cur.brp + cur.kc);
        be = __ldg(cur.brp + cur.kc + 1);
      }
      const bool lng = be - bs >= 32;
      if (!lng && chunk % wparts == wpart) {
        int32_t q = bs;
        for (; q + 4 <= be; q += 4) {  // four column loads in flight
          const int32_t j0 = __ldg(sbci + q), j1 = __ldg(sbci + q + 1);
          const int32_t j2 = __ldg(sbci + q + 2), j3 = __ldg(sbci + q + 3);
          fs(j0);
          fs(j1);
          fs(j2);
          fs(j3);
        }
        for (; q < be; q++) fs(__ldg(sbci + q));
      }
      unsigned longm = __ballot_sync(kFull, lng);
      while (longm) {
        const int src = __ffs(longm) - 1;
        longm &= longm - 1;
        const int32_t lb = __shfl_sync(kFull, bs, src), le = __shfl_sync(kFull, be, src);
        const int32_t* lci = shfl_ptr(sbci, src);
        const int32_t step = 32 * wparts;
        int32_t q = lb + lane + 32 * wpart;
        for (; q + 3 * step < le; q += 4 * step) {
          const int32_t j0 = __ldg(lci + q), j1 = __ldg(lci + q + step);
          const int32_t j2 = __ldg(lci + q + 2 * step), j3 = __ldg(lci + q + 3 * step);
          fs(j0);
          fs(j1);
          fs(j2);
          fs(j3);
        }
        for (; q < le; q += step) fs(__ldg(lci + q));
      }
    }
  }
}

// Order-free walk over the products of C-tile row `x` whose columns lie in
// fine blocks [fb_lo, fb_hi) (B-row table `tab`): calls fs(j) for each.
template <typename FS>
__device__ __forceinline__ void walk_columns_ranged(const SpGridView& A, const SpGridView& B, const Geom& g,
                                                    const RowInfo& x, int fb_lo, int fb_hi,
                                                    const int32_t* __restrict__ tab, FS&& fs) {
  const int lane = lane_id();
  const int ns = stage_count(g, x.ti, x.tj);
  for (int g0 = 0; g0 < ns; g0 += 32) {
    const int si = g0 + lane;
    int32_t as = 0, alen = 0;
    const int32_t* acol = nullptr;
    const int32_t* trows = nullptr;
    const int32_t* brp = nullptr;
    const int32_t* bci = nullptr;
    if (si < ns) {
      const int64_t k = (stage_at(g, x.ti, x.tj, si) + x.rot) % g.gk;
      const bclx_csr_t At = A.tile(x.ti, k);
      as = __ldg(At.row_ptr + x.r);
      alen = __ldg(At.row_ptr + x.r + 1) - as;
      acol = At.col_ind;
      if (tab) trows = tab + (k * g.gn + x.tj) * g.tk * (g.nfb + 1);
      const bclx_csr_t Bt = B.tile(k, x.tj);
      brp = Bt.row_ptr;
      bci = Bt.col_ind;
    }
    const int32_t aincl = warp_inclusive_scan(alen);
    const int32_t atot = __shfl_sync(kFull, aincl, 31);
    const int32_t aexcl = aincl - alen;
    for (int32_t e0 = 0; e0 < atot; e0 += 32) {
      const int32_t e = e0 + lane;
      const int sl = warp_search(aincl, e);
      const int32_t sas = __shfl_sync(kFull, as, sl);
      const int32_t sax = __shfl_sync(kFull, aexcl, sl);
      const int32_t* sacol = shfl_ptr(acol, sl);
      const int32_t* strows = shfl_ptr(trows, sl);
      const int32_t* sbrp = shfl_ptr(brp, sl);
      const int32_t* sbci = shfl_ptr(bci, sl);
      int32_t bs = 0, be = 0;
      if (e < atot) {
        const int32_t kc = __ldg(sacol + sas + (e - sax));
        b_block_range(strows, sbrp, sbci, kc, fb_lo, fb_hi, g.nfb, bs, be);
      }
      const bool lng = be - bs >= 32;
      if (!lng)
        for (int32_t q = bs; q < be; q++) fs(__ldg(sbci + q));
      unsigned longm = __ballot_sync(kFull, lng);
      while (longm) {
        const int src = __ffs(longm) - 1;
        longm &= longm - 1;
        const int32_t lb = __shfl_sync(kFull, bs, src), le = __shfl_sync(kFull, be, src);
        const int32_t* lci = shfl_ptr(sbci, src);
        for (int32_t q = lb + lane; q < le; q += 32) fs(__ldg(lci + q));
      }
    }
  }
}

// ---- host reads ----------------------------------------------------------------------
//
// The planning passes read a few sizes back to the host.  A one-warp kernel
// stores them into the context's mapped page-locked slots instead of a
// device-to-host copy, which would queue behind any large copy the caller
// has running in the same direction (a previous product's output on its way
// to the host).

struct ReadBack {
  const void* src[4];
  int32_t bytes[4];  // at most 8 each
  int32_t slot[4];   // 8-byte destination slot
  int32_t n;
};

__global__ void k_read_back(ReadBack r, int64_t* __restrict__ dst) {
  const int t = threadIdx.x;
  for (int i = 0; i < r.n; i++)
    if (t < r.bytes[i])
      reinterpret_cast<volatile unsigned char*>(dst + r.slot[i])[t] = reinterpret_cast<const unsigned char*>(r.src[i])[t];
}

// Store up to four values (each at most 8 bytes) into ctx->pinned[slot] on
// the context's stream; the host reads them after synchronizing the stream.
static int read_back(Context* ctx, std::initializer_list<std::tuple<const void*, int, int>> items) {
  ReadBack r{};
  for (const auto& it : items) {
    if (r.n == 4 || std::get<1>(it) > 8) return BCLX_ERR_INVALID;
    r.src[r.n] = std::get<0>(it);
    r.bytes[r.n] = std::get<1>(it);
    r.slot[r.n] = std::get<2>(it);
    r.n++;
  }
  k_read_back<<<1, 32, 0, ctx->stream>>>(r, ctx->pinned_dev);
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

// ---- planning --------------------------------------------------------------------

// Per row: intermediate products; light/heavy classification into two lists.
// One warp per row: one lane per stage reads the A-row segment, then the
// flattened entries are read 32 at a time.
// With FEATURES it also writes, per row, the predictor's five features
// X[ri*5 + 0..4] = log2(1 + A-row nnz over all stages), log2(1 + products),
// log2(1 + longest referenced B row), (i + 1/2)/grid_m, (j + 1/2)/grid_n,
// and the row's product count (capped at 2^31-1) to ub_out[ri].
// `live` (or null: every C tile): the n_live[0] C tiles with at least one
// stage; only their rows are walked (the others have no products).
template <bool FEATURES>
__global__ void k_classify(SpGridView A, SpGridView B, Geom g, int32_t* __restrict__ light_list,
                           int32_t* __restrict__ heavy_list, int32_t* __restrict__ vheavy_list,
                           int32_t* __restrict__ counters, unsigned long long* __restrict__ products,
                           int heavy_min_cols, int light_ub, float* __restrict__ X,
                           int32_t* __restrict__ ub_out, unsigned long long* __restrict__ queue, int grab,
                           const int32_t* __restrict__ live = nullptr, const int32_t* __restrict__ n_live = nullptr) {
  const int lane = lane_id();
  // row item of walk position `it`
  auto row_of = [&](unsigned long long it) -> int64_t {
    if (!live) return (int64_t)it;
    const int64_t lt = (int64_t)(it / (unsigned long long)g.tm);
    return (int64_t)__ldg(live + lt) * g.tm + (int64_t)(it - (unsigned long long)lt * g.tm);
  };
  unsigned long long mine = 0;
  // rows from a device counter, `grab` (at most 32) consecutive rows per
  // atomic (one atomic per row serialises on the counter when a fine grid has
  // hundreds of millions of mostly empty row items); the next grab is in
  // flight while the current rows are walked.  Lane q keeps the class of row
  // base + q, and the grab's rows are appended to each list with one atomic.
  grab = min(grab, 32);
  const unsigned long long n_rows =
      live ? (unsigned long long)__ldg(n_live) * (unsigned long long)g.tm : (unsigned long long)g.n_row_items;
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(queue, (unsigned long long)grab);
  base = __shfl_sync(kFull, base, 0);
  while (base < n_rows) {
    unsigned long long nx = 0;
    if (lane == 0) nx = atomicAdd(queue, (unsigned long long)grab);
    const unsigned long long end = min(base + (unsigned long long)grab, n_rows);
    int cls = -1;  // list of row base + lane: 0 light, 1 heavy, 3 very heavy
    for (unsigned long long it = base; it < end; it++) {
    const int64_t ri = row_of(it);
    const RowInfo x = decode_row(g, ri);
    int64_t tot = 0, annz = 0;
    int32_t bmax = 0;
    if (x.r < A.rows_of(x.ti)) {
      const int ns = stage_count(g, x.ti, x.tj);
      for (int g0 = 0; g0 < ns; g0 += 32) {
        const int si = g0 + lane;
        int32_t as = 0, alen = 0;
        const int32_t* acol = nullptr;
        const int32_t* brp = nullptr;
        if (si < ns) {
          const int64_t k = (stage_at(g, x.ti, x.tj, si) + x.rot) % g.gk;
          const bclx_csr_t At = A.tile(x.ti, k);
          as = __ldg(At.row_ptr + x.r);
          alen = __ldg(At.row_ptr + x.r + 1) - as;
          acol = At.col_ind;
          brp = B.tile(k, x.tj).row_ptr;
        }
        const int32_t aincl = warp_inclusive_scan(alen);
        const int32_t atot = __shfl_sync(kFull, aincl, 31);
        for (int32_t e0 = 0; e0 < atot; e0 += 32) {
          const int32_t e = e0 + lane;
          const int sl = warp_search(aincl, e);
          const int32_t sas = __shfl_sync(kFull, as, sl);
          const int32_t sax = __shfl_sync(kFull, aincl - alen, sl);
          const int32_t* sacol = shfl_ptr(acol, sl);
          const int32_t* sbrp = shfl_ptr(brp, sl);
          if (e < atot) {
            const int32_t kc = __ldg(sacol + sas + (e - sax));
            const int32_t bl = __ldg(sbrp + kc + 1) - __ldg(sbrp + kc);
            tot += bl;
            if (FEATURES) bmax = max(bmax, bl);
          }
        }
        if (FEATURES) annz += atot;
      }
      tot = warp_sum(tot);
      if (FEATURES) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) bmax = max(bmax, __shfl_xor_sync(kFull, bmax, d));
      }
    }
    if (FEATURES && lane == 0) {
      float* xr = X + ri * 5;
      xr[0] = log2f(1.f + (float)annz);
      xr[1] = log2f(1.f + (float)tot);
      xr[2] = log2f(1.f + (float)bmax);
      xr[3] = ((float)x.ti + 0.5f) / (float)g.gm;
      xr[4] = ((float)x.tj + 0.5f) / (float)g.gn;
      ub_out[ri] = (int32_t)(tot < INT32_MAX ? tot : INT32_MAX);
    }
    if (tot > 0) {
      if (lane == 0) mine += (unsigned long long)tot;
      if (lane == (int)(it - base)) cls = (tot <= light_ub && x.w < heavy_min_cols) ? 0 : (tot <= kVeryHeavyUb ? 1 : 3);
    }
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
      if (c == 2) continue;
      const unsigned m = __ballot_sync(kFull, cls == c);
      if (m == 0) continue;
      int pos = 0;
      if (lane == 0) pos = atomicAdd(&counters[c], __popc(m));
      pos = __shfl_sync(kFull, pos, 0) + __popc(m & ((1u << lane) - 1u));
      int32_t* list = c == 0 ? light_list : (c == 1 ? heavy_list : vheavy_list);
      if (cls == c) list[pos] = (int32_t)row_of(base + lane);
    }
    base = __shfl_sync(kFull, nx, 0);
  }
  if (lane == 0 && mine) atomicAdd(products, mine);
}

// B-row table: for every row of every B tile (k, j), the position of the
// first entry in each fine column block: tab[((k*gn + j)*tk + r)*(nfb+1) + b]
// = first entry with column >= b*kFineCols (b = nfb: the row end).
// One thread per B row (rows of a tile are short on average).
__global__ void k_btable(SpGridView B, Geom g, int32_t* __restrict__ tab) {
  const int64_t nrows = g.gk * g.gn * g.tk;
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < nrows; x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t kt = x / g.tk, r = x - kt * g.tk;
    const int64_t k = kt / g.gn, j = kt - k * g.gn;
    const bclx_csr_t Bt = B.tile(k, j);
    if (r >= Bt.m) continue;  // the tile's own row count (sub-grids may reorder B's tiles)
    int32_t* trow = tab + x * (g.nfb + 1);
    const int32_t b0 = __ldg(Bt.row_ptr + r), b1 = __ldg(Bt.row_ptr + r + 1);
    int b = 0;
    for (int32_t q = b0; q < b1; q++) {
      const int blk = __ldg(Bt.col_ind + q) / kFineCols;
      while (b <= blk) trow[b++] = q;
    }
    while (b <= g.nfb) trow[b++] = b1;
  }
}

// ---- symbolic ----------------------------------------------------------------------

// Symbolic pass.  Heavy rows are numbered 0..n_heavy-1 (the very heavy ones
// first); a row's column bitmap is built in shared memory, its popcount is
// the row's output count, and heavy rows also store the bitmap for the
// numeric pass (hbm_words words per row).
//
// One warp per row for the light and ordinary heavy rows (heavy first),
// rows taken from a device counter (each warp grabs its next row while it
// walks the current one) ...
// Four blocks per SM: 64 registers without spills (R-MAT s16: 5.50-5.52 ms
// per product against 5.52-5.54 with 48 registers and spills, 5.66 with 40).
__global__ void __launch_bounds__(kWarpsSym * 32, 4)
    k_symbolic(SpGridView A, SpGridView B, Geom g, const int32_t* __restrict__ light_list,
               const int32_t* __restrict__ heavy_list, int n_light, int n_heavy, int n_vheavy,
               int32_t* __restrict__ row_count, uint32_t* __restrict__ heavy_bitmaps, int64_t hbm_words,
               int16_t* __restrict__ heavy_span, unsigned long long* __restrict__ queue, int grab) {
  __shared__ uint32_t bm_all[kWarpsSym][kMaxWords];
  uint32_t* bm = bm_all[threadIdx.x >> 5];
  const int lane = lane_id();
  const unsigned long long n_items = (unsigned long long)((int64_t)n_light + n_heavy - n_vheavy);
  unsigned long long base = 0;
  if (lane == 0) base = atomicAdd(queue, (unsigned long long)grab);
  base = __shfl_sync(kFull, base, 0);
  while (base < n_items) {
    unsigned long long nx = 0;
    if (lane == 0) nx = atomicAdd(queue, (unsigned long long)grab);
    const unsigned long long end = min(base + (unsigned long long)grab, n_items);
    for (unsigned long long it = base; it < end; it++) {
    const int64_t idx = n_vheavy + (int64_t)it;
    const bool heavy = idx < n_heavy;
    const int64_t ri = heavy ? heavy_list[idx] : light_list[idx - n_heavy];
    const RowInfo x = decode_row(g, ri);
    const int words = (x.w + 31) >> 5;
    for (int w = lane; w < words; w += 32) bm[w] = 0u;
    __syncwarp();
    walk_columns(A, B, g, x, 0, 1, [&](int32_t j) { atomicOr(&bm[j >> 5], 1u << (j & 31)); });
    __syncwarp();
    int cnt = 0, w0 = INT_MAX, w1 = -1;
    uint32_t* out = heavy ? heavy_bitmaps + idx * hbm_words : nullptr;
    for (int w = lane; w < words; w += 32) {
      const uint32_t v = bm[w];
      if (heavy) out[w] = v;
      cnt += __popc(v);
      if (v) {
        w0 = min(w0, w);
        w1 = max(w1, w);
      }
    }
    cnt = warp_sum(cnt);
    if (heavy && heavy_span) {
      w0 = __reduce_min_sync(kFull, w0);
      w1 = __reduce_max_sync(kFull, w1);
    }
    if (lane == 0) {
      row_count[ri] = cnt;
      if (heavy && heavy_span) {
        heavy_span[2 * idx] = (int16_t)(cnt > 0 ? w0 / (kFineCols / 32) : 0);
        heavy_span[2 * idx + 1] = (int16_t)(cnt > 0 ? w1 / (kFineCols / 32) + 1 : 0);
      }
    }
    __syncwarp();
    }
    base = __shfl_sync(kFull, nx, 0);
  }
}

// ... and one block per very heavy row, its warps sharing the bitmap.
__global__ void __launch_bounds__(kWarpsSym * 32)
    k_symbolic_block(SpGridView A, SpGridView B, Geom g, const int32_t* __restrict__ heavy_list, int n_vheavy,
                     int32_t* __restrict__ row_count, uint32_t* __restrict__ heavy_bitmaps, int64_t hbm_words,
                     int16_t* __restrict__ heavy_span) {
  __shared__ uint32_t bm[kMaxWords];
  __shared__ int red[kWarpsSym];
  __shared__ int first_word, last_word;
  const int wid = threadIdx.x >> 5;
  for (int64_t h = blockIdx.x; h < n_vheavy; h += gridDim.x) {
    const int64_t ri = heavy_list[h];
    const RowInfo x = decode_row(g, ri);
    const int words = (x.w + 31) >> 5;
    for (int w = threadIdx.x; w < words; w += blockDim.x) bm[w] = 0u;
    if (threadIdx.x == 0) {
      first_word = INT_MAX;
      last_word = -1;
    }
    __syncthreads();
    walk_columns(A, B, g, x, wid, kWarpsSym, [&](int32_t j) { atomicOr(&bm[j >> 5], 1u << (j & 31)); });
    __syncthreads();
    int cnt = 0, w0 = INT_MAX, w1 = -1;
    uint32_t* out = heavy_bitmaps + h * hbm_words;
    for (int w = threadIdx.x; w < words; w += blockDim.x) {
      const uint32_t v = bm[w];
      out[w] = v;
      cnt += __popc(v);
      if (v) {
        w0 = min(w0, w);
        w1 = max(w1, w);
      }
    }
    if (heavy_span) {
      w0 = __reduce_min_sync(kFull, w0);
      w1 = __reduce_max_sync(kFull, w1);
      if ((threadIdx.x & 31) == 0 && w0 != INT_MAX) {
        atomicMin(&first_word, w0);
        atomicMax(&last_word, w1);
      }
    }
    cnt = warp_sum(cnt);
    if ((threadIdx.x & 31) == 0) red[wid] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
      int t = 0;
      for (int q = 0; q < kWarpsSym; q++) t += red[q];
      row_count[ri] = t;
      if (heavy_span) {
        heavy_span[2 * h] = (int16_t)(t > 0 ? first_word / (kFineCols / 32) : 0);
        heavy_span[2 * h + 1] = (int16_t)(t > 0 ? last_word / (kFineCols / 32) + 1 : 0);
      }
    }
    __syncthreads();
  }
}

// tile_row_ptr / tile_offset from the row offsets (rows are tile-major).
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

// Heavy rows are cut at fine-block boundaries into items of <= vcap outputs
// (greedy left to right; leading empty blocks are skipped).  One warp per
// heavy row (blocks of 256 threads): lanes count the fine blocks' outputs
// from the row's bitmap, lane 0 cuts.  FILL = false counts the items,
// FILL = true writes them.
struct HeavyItem {
  int32_t h;       // heavy slot
  int16_t fb_lo;   // first fine block
  int16_t fb_hi;   // one past the last
  int32_t rel;     // output offset inside the row
  int32_t count;   // outputs
};

template <bool FILL>
__global__ void __launch_bounds__(256)
    k_cut_heavy(Geom g, const int32_t* __restrict__ heavy_list, int n_heavy,
                const uint32_t* __restrict__ heavy_bitmaps, int64_t hbm_words, int32_t* __restrict__ n_items,
                const int64_t* __restrict__ first, HeavyItem* __restrict__ items, int vcap,
                const int32_t* __restrict__ row_count = nullptr, const int16_t* __restrict__ span = nullptr) {
  __shared__ int32_t cnt_all[8][kMaxCols / kFineCols];
  int32_t* cnt = cnt_all[threadIdx.x >> 5];
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  constexpr int kWordsPerBlock = kFineCols / 32;
  for (int64_t h = warp; h < n_heavy; h += nwarps) {
    const int64_t ri = heavy_list[h];
    const RowInfo x = decode_row(g, ri);
    const int nfb = (x.w + kFineCols - 1) / kFineCols;
    if (span && row_count) {
      // counted by the symbolic pass: a row whose outputs fit one item needs
      // no look at its bitmap; the item spans its first to its last block
      // with outputs
      const int tot = __ldg(row_count + ri);
      if (tot <= vcap) {
        if (lane == 0) {
          if (FILL && tot > 0)
            items[first[h]] = HeavyItem{(int32_t)h, __ldg(span + 2 * h), __ldg(span + 2 * h + 1), 0, tot};
          if (!FILL) n_items[h] = tot > 0 ? 1 : 0;
        }
        continue;
      }
    }
    const uint32_t* bm = heavy_bitmaps + h * hbm_words;
    const int words = (x.w + 31) >> 5;
    int tot = 0, first_nz = INT_MAX, last_nz = -1;
    for (int b = lane; b < nfb; b += 32) {
      int c = 0;
#pragma unroll
      for (int q = 0; q < kWordsPerBlock; q++) {
        const int w = b * kWordsPerBlock + q;
        if (w < words) c += __popc(__ldg(bm + w));
      }
      cnt[b] = c;
      tot += c;
      if (c > 0) {
        first_nz = min(first_nz, b);
        last_nz = max(last_nz, b);
      }
    }
    tot = warp_sum(tot);
    first_nz = __reduce_min_sync(kFull, first_nz);
    last_nz = __reduce_max_sync(kFull, last_nz);
    __syncwarp();
    if (tot <= vcap) {
      // one item, from the first to the last block with outputs: what the
      // block-by-block cut below gives for such a row
      if (lane == 0) {
        if (FILL && tot > 0)
          items[first[h]] = HeavyItem{(int32_t)h, (int16_t)first_nz, (int16_t)(last_nz + 1), 0, tot};
        if (!FILL) n_items[h] = tot > 0 ? 1 : 0;
      }
    } else if (lane == 0) {
      int nit = 0, cur = 0, start = 0, rel = 0, last = -1;
      int64_t out = FILL ? first[h] : 0;
      for (int b = 0; b < nfb; b++) {
        const int c = cnt[b];
        if (c > 0) last = b;
        if (cur > 0 && cur + c > vcap) {
          if (FILL) items[out++] = HeavyItem{(int32_t)h, (int16_t)start, (int16_t)b, rel, cur};
          nit++;
          rel += cur;
          cur = 0;
          start = b;
        }
        if (cur == 0 && c == 0) start = b + 1;
        cur += c;
      }
      if (cur > 0) {  // the last item ends after the row's last block with outputs
        if (FILL) items[out++] = HeavyItem{(int32_t)h, (int16_t)start, (int16_t)(last + 1), rel, cur};
        nit++;
      }
      if (!FILL) n_items[h] = nit;
    }
    __syncwarp();
  }
}

// ---- numeric ------------------------------------------------------------------------------

template <typename VT, int WORDS, int VCAP>
struct WarpSmem {
  uint32_t bm[WORDS];
  uint16_t pre[WORDS];
  VT acc[VCAP];
  VT part[VCAP];
  unsigned char tag[VCAP];
  VT sa[32];
  VT sb[32];
  int32_t ss[32];
};

#ifndef BCLX_NUMERIC_MIN_BLOCKS
#define BCLX_NUMERIC_MIN_BLOCKS 4
#endif
// LEARNED: the learned product's single pass.  Heavy items come from the
// predicted cut (their counts are unknown): each builds its bitmap from its
// own products, and an item with more than kVcap outputs marks its row in
// row_failed and stops (that row is redone by the exact path).  Outputs go
// to temp slots (light row l at light_slot[l], heavy item idx at
// heavy_slot_base + item_off[idx], after all light slots; an item's slot
// count, at most kVcap, comes from the prediction),
// counts to item_count / row_count_w.
template <typename VT, int WORDS, bool LEARNED, int VCAP>
__global__ void __launch_bounds__(kWarpsNum * 32, BCLX_NUMERIC_MIN_BLOCKS)
    k_numeric(SpGridView A, SpGridView B, Geom g, const int32_t* __restrict__ light_list,
              const int32_t* __restrict__ heavy_list, int n_light, int64_t n_heavy_items,
              const HeavyItem* __restrict__ heavy_items,
              const uint32_t* __restrict__ heavy_bitmaps, int64_t hbm_words, const int32_t* __restrict__ tab,
              const int32_t* __restrict__ row_count, const int64_t* __restrict__ row_offset,
              int32_t* __restrict__ out_col, VT* __restrict__ out_val, int s0, int s1,
              unsigned long long* __restrict__ queue, int grab, int long_seg,
              const int64_t* __restrict__ light_slot, int32_t* __restrict__ item_count,
              int32_t* __restrict__ row_count_w, int32_t* __restrict__ row_failed, int64_t heavy_slot_base,
              const int64_t* __restrict__ item_off) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpSmem<VT, WORDS, VCAP>& S = reinterpret_cast<WarpSmem<VT, WORDS, VCAP>*>(smem_raw)[threadIdx.x >> 5];
  const int lane = lane_id();
  const int64_t n_total = n_heavy_items + n_light;
  // persistent warps: take `grab` consecutive items at a time from the queue
  int64_t next = 0, stop = 0;
  for (;;) {
    if (next >= stop) {
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(queue, (unsigned long long)grab);
      b = __shfl_sync(kFull, b, 0);
      if ((int64_t)b >= n_total) break;
      next = (int64_t)b;
      stop = min((int64_t)b + grab, n_total);
    }
    const int64_t idx = next++;
    // heavy items first (they are the larger ones)
    const bool heavy = idx < n_heavy_items;
    int64_t ri;
    int cnt = 0, fb_lo = 0, fb_hi = 0, lo = 0, hi, hslot = 0, icap = VCAP;
    int64_t off;
    const uint32_t* hb = nullptr;
    if (heavy) {
      const HeavyItem it = heavy_items[idx];
      ri = heavy_list[it.h];
      hslot = it.h;
      fb_lo = it.fb_lo;
      fb_hi = it.fb_hi;
      if (LEARNED) {
        off = heavy_slot_base + item_off[idx];
        icap = it.count;  // temp slots sized from the prediction
      } else {
        cnt = it.count;
        off = row_offset[ri] + it.rel;
        hb = heavy_bitmaps + (int64_t)it.h * hbm_words;
      }
    } else {
      ri = light_list[idx - n_heavy_items];
      if (LEARNED) {
        off = light_slot[idx - n_heavy_items];
      } else {
        cnt = row_count[ri];
        off = row_offset[ri];
      }
    }
    const RowInfo x = decode_row(g, ri);
    if (heavy) {
      lo = fb_lo * kFineCols;
      hi = min(fb_hi * kFineCols, x.w);
    } else {
      hi = x.w;
    }
    const int w0 = lo >> 5;
    const int words = ((hi - lo) + 31) >> 5;

    // 1. column bitmap of the item (word w covers columns lo + 32w ..)
    if (heavy && LEARNED) {
      for (int w = lane; w < words; w += 32) S.bm[w] = 0u;
      __syncwarp();
      walk_columns_ranged(A, B, g, x, fb_lo, fb_hi, tab, [&](int32_t j) {
        const int xx = j - lo;
        atomicOr(&S.bm[xx >> 5], 1u << (xx & 31));
      });
    } else if (heavy) {
      for (int w = lane; w < words; w += 32) S.bm[w] = __ldg(hb + w0 + w);
    } else {
      for (int w = lane; w < words; w += 32) S.bm[w] = 0u;
      __syncwarp();
      if (s0 == 0) {
        walk_columns(A, B, g, x, 0, 1, [&](int32_t j) { atomicOr(&S.bm[j >> 5], 1u << (j & 31)); });
      } else {
        for (int q = lane; q < cnt; q += 32) {
          const int j = out_col[off + q];
          atomicOr(&S.bm[j >> 5], 1u << (j & 31));
        }
      }
    }
    __syncwarp();

    // 2. per-word exclusive prefix counts
    {
      const int per = (words + 31) >> 5;
      const int wa = lane * per;
      int loc = 0;
      for (int w = wa; w < wa + per && w < words; w++) loc += __popc(S.bm[w]);
      const int inc = warp_inclusive_scan(loc);
      int ex = inc - loc;
      for (int w = wa; w < wa + per && w < words; w++) {
        S.pre[w] = (uint16_t)ex;
        ex += __popc(S.bm[w]);
      }
      if (LEARNED) cnt = __shfl_sync(kFull, inc, 31);
    }
    __syncwarp();
    if (LEARNED) {
      if (heavy && cnt > icap) {  // the prediction cut this item too wide, or sized it too small
        if (lane == 0) row_failed[hslot] = 1;
        continue;
      }
      if (lane == 0) {
        if (heavy) {
          item_count[idx] = cnt;
          atomicAdd(&row_count_w[ri], cnt);
        } else {
          row_count_w[ri] = cnt;
        }
      }
    }

    // 3. sorted columns (first stage range only) and the accumulators
    if (s0 == 0) {
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
    for (int q = lane; q < cnt; q += 32) {
      S.acc[q] = s0 == 0 ? VT(0) : out_val[off + q];
      S.part[q] = VT(0);
      S.tag[q] = (unsigned char)kNoStage;
    }
    __syncwarp();

    // 4. values in the reference's order, with a lazy per-column stage fold
    auto update = [&](bool valid, int32_t j, VT a, VT b, int stage) {
      int rank = 0;
      if (valid) {
        const int xx = j - lo;
        rank = S.pre[xx >> 5] + __popc(S.bm[xx >> 5] & ((1u << (xx & 31)) - 1u));
      }
      const unsigned peers = __match_any_sync(kFull, valid ? j : -1);
      const bool single = peers == (1u << lane);
      if (__any_sync(kFull, valid && !single)) {
        S.sa[lane] = a;
        S.sb[lane] = b;
        S.ss[lane] = stage;
        __syncwarp();
      }
      if (valid && single) {
        // the only product of its column in this batch
        VT v = S.part[rank];
        const int t = S.tag[rank];
        if (t != stage) {
          if (t != kNoStage) S.acc[rank] = vadd(S.acc[rank], v);
          v = VT(0);
          S.tag[rank] = (unsigned char)stage;
        }
        S.part[rank] = madd(a, b, v);
      } else if (valid && lane == __ffs(peers) - 1) {
        VT v = S.part[rank];
        int t = S.tag[rank];
        VT ac = S.acc[rank];
        unsigned gmask = peers;
        do {
          const int mb = __ffs(gmask) - 1;
          gmask &= gmask - 1;
          const int st = S.ss[mb];
          if (st != t) {
            if (t != kNoStage) ac = vadd(ac, v);
            v = VT(0);
            t = st;
          }
          v = madd(S.sa[mb], S.sb[mb], v);
        } while (gmask);
        S.part[rank] = v;
        S.tag[rank] = (unsigned char)t;
        S.acc[rank] = ac;
      }
      __syncwarp();
    };
    // direct mode: the lanes hold distinct columns, each updates its own
    auto update_direct = [&](int32_t j, VT a, VT b, int stage) {
      const int xx = j - lo;
      const int rank = S.pre[xx >> 5] + __popc(S.bm[xx >> 5] & ((1u << (xx & 31)) - 1u));
      VT v = S.part[rank];
      const int t = S.tag[rank];
      if (t != stage) {
        if (t != kNoStage) S.acc[rank] = vadd(S.acc[rank], v);
        v = VT(0);
        S.tag[rank] = (unsigned char)stage;
      }
      S.part[rank] = madd(a, b, v);
    };
    if (heavy)
      walk_products<VT, true>(A, B, g, x, s0, s1, fb_lo, fb_hi, tab, long_seg, update, update_direct);
    else
      walk_products<VT, false>(A, B, g, x, s0, s1, 0, 0, nullptr, long_seg, update, update_direct);

    // 5. last fold and values out
    for (int q = lane; q < cnt; q += 32) {
      VT v = S.acc[q];
      if (S.tag[q] != kNoStage) v = vadd(v, S.part[q]);
      out_val[off + q] = v;
    }
    __syncwarp();
  }
}

// ---- learned product ---------------------------------------------------------------------

// outputs aimed at per heavy item (the accumulator holds kVcap): the
// context's BCLX_TUNE_LEARN_TARGET, 320 by default
constexpr float kLearnMargin = 1.15f;  // head room on the predicted count
constexpr float kCapMargin = 1.25f;    // head room of an item's temp slots over its estimate
constexpr float kCapSlack = 32.f;

// Products of every heavy row per fine column block: bub[h*nfb + b].  One
// warp per heavy row; lanes take A entries (all stages) and add each entry's
// per-block segment lengths (from the B-row table) into shared counters.
__global__ void __launch_bounds__(256) k_heavy_block_ub(SpGridView A, SpGridView B, Geom g,
                                                        const int32_t* __restrict__ heavy_list,
                                                        int n_heavy, const int32_t* __restrict__ tab,
                                                        int32_t* __restrict__ bub) {
  __shared__ int32_t cnt_all[8][64];
  int32_t* cnt = cnt_all[threadIdx.x >> 5];
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int nfb = (int)g.nfb;
  for (int64_t h = warp; h < n_heavy; h += nwarps) {
    const RowInfo x = decode_row(g, heavy_list[h]);
    cnt[lane] = 0;
    cnt[lane + 32] = 0;
    __syncwarp();
    const int ns = stage_count(g, x.ti, x.tj);
    for (int si = 0; si < ns; si++) {
      const int64_t k = (stage_at(g, x.ti, x.tj, si) + x.rot) % g.gk;
      const bclx_csr_t At = A.tile(x.ti, k);
      const int32_t a0 = __ldg(At.row_ptr + x.r), a1 = __ldg(At.row_ptr + x.r + 1);
      // per A entry: a B row shorter than the block count is counted column
      // by column, a longer one from the B-row table's block starts
      const bclx_csr_t Bt = B.tile(k, x.tj);
      const int32_t* trows = tab ? tab + (k * g.gn + x.tj) * g.tk * (g.nfb + 1) : nullptr;
      for (int32_t p = a0 + lane; p < a1; p += 32) {
        const int32_t kc = __ldg(At.col_ind + p);
        const int32_t b0 = __ldg(Bt.row_ptr + kc), b1 = __ldg(Bt.row_ptr + kc + 1);
        if (!trows || b1 - b0 <= nfb) {
          for (int32_t q = b0; q < b1; q++) atomicAdd(&cnt[__ldg(Bt.col_ind + q) / kFineCols], 1);
        } else {
          const int32_t* trow = trows + (int64_t)kc * (g.nfb + 1);
          int32_t prev = b0;
          for (int b = 0; b < nfb; b++) {
            const int32_t nx = __ldg(trow + b + 1);
            if (nx != prev) atomicAdd(&cnt[b], nx - prev);
            prev = nx;
          }
        }
      }
    }
    __syncwarp();
    if (lane < nfb) bub[h * nfb + lane] = cnt[lane];
    if (lane + 32 < nfb) bub[h * nfb + lane + 32] = cnt[lane + 32];
    __syncwarp();
  }
}

// Heavy rows cut into fine-block ranges of about `target` expected
// outputs, greedy left to right.  A block of width w receiving p products is
// expected to hold w*(1 - exp(-p/w)) distinct columns (p products spread over
// w columns); the network's predicted row count (pred = log2(1 + count))
// rescales these block estimates so that they add up to the prediction.
// Without a network a block's product count (capped at its width) is used:
// an upper bound, so no item can overflow.  FILL = false counts the items,
// FILL = true writes them.
// Temp slots of a heavy item from its expected outputs: a predicted estimate
// gets head room (an item that outgrows it is redone exactly); without a
// network the estimate is already an upper bound.
__device__ __forceinline__ int item_capacity(float est, bool predicted) {
  const float want = predicted ? est * kCapMargin + kCapSlack : est;
  const int c = ((int)ceilf(want) + 15) & ~15;
  return c < 16 ? 16 : (c > kVcap ? kVcap : c);
}

template <bool FILL>
__global__ void k_learned_cut(Geom g, const int32_t* __restrict__ heavy_list, int n_heavy,
                              const float* __restrict__ pred, const int32_t* __restrict__ ub,
                              const int32_t* __restrict__ bub, int32_t* __restrict__ n_items,
                              const int64_t* __restrict__ first, HeavyItem* __restrict__ items,
                              int32_t* __restrict__ item_cap, float target) {
  const int nfb_g = (int)g.nfb;
  for (int64_t h = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; h < n_heavy; h += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ri = heavy_list[h];
    const RowInfo x = decode_row(g, ri);
    const int nfb = (x.w + kFineCols - 1) / kFineCols;
    const int32_t* bu = bub + h * nfb_g;
    float kappa = 1.f;
    if (pred) {
      float est = 0.f;
      for (int b = 0; b < nfb; b++) {
        const float w = (float)min(kFineCols, x.w - b * kFineCols);
        est += w * (1.f - __expf(-(float)bu[b] / w));
      }
      const float c = exp2f(pred[ri]) - 1.f;
      kappa = fminf(fmaxf(c * kLearnMargin / fmaxf(est, 1.f), 0.25f), 4.f);
    }
    int n = 0, start = 0;
    float cur = 0.f;
    int64_t out = FILL ? first[h] : 0;
    for (int b = 0; b < nfb; b++) {
      const float w = (float)min(kFineCols, x.w - b * kFineCols);
      const float p = (float)bu[b];
      const float e = pred ? fminf(w, kappa * w * (1.f - __expf(-p / w))) : fminf(w, p);
      if (b > start && cur + e > target) {
        if (FILL) {
          const int cap = item_capacity(cur, pred != nullptr);
          item_cap[out] = cap;
          items[out++] = HeavyItem{(int32_t)h, (int16_t)start, (int16_t)b, 0, cap};
        }
        n++;
        start = b;
        cur = 0.f;
      }
      cur += e;
    }
    if (FILL) {
      const int cap = item_capacity(cur, pred != nullptr);
      item_cap[out] = cap;
      items[out++] = HeavyItem{(int32_t)h, (int16_t)start, (int16_t)nfb, 0, cap};
    }
    n++;
    if (!FILL) n_items[h] = n;
  }
}

__global__ void k_gather_features(const int32_t* __restrict__ list, int n, const float* __restrict__ feat,
                                  float* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int64_t ri = list[i];
#pragma unroll
    for (int f = 0; f < 5; f++) out[(int64_t)i * 5 + f] = feat[ri * 5 + f];
  }
}

__global__ void k_scatter_pred(const int32_t* __restrict__ list, int n, const float* __restrict__ pred_in,
                               float* __restrict__ pred) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) pred[list[i]] = pred_in[i];
}

__global__ void k_gather_ub(const int32_t* __restrict__ list, int n, const int32_t* __restrict__ ub,
                            int32_t* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = ub[list[i]];
}

// Failed heavy rows -> their row indices, and their heavy-list slots marked.
__global__ void k_collect_failed(const int32_t* __restrict__ heavy_list, int n_heavy,
                                 const int32_t* __restrict__ row_failed, int32_t* __restrict__ failed_list,
                                 int32_t* __restrict__ n_failed) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < n_heavy; h += gridDim.x * blockDim.x)
    if (row_failed[h]) failed_list[atomicAdd(n_failed, 1)] = heavy_list[h];
}

__global__ void k_take_counts(const int32_t* __restrict__ failed_list, int n_failed,
                              const int32_t* __restrict__ redo_count, int32_t* __restrict__ row_count) {
  for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n_failed; f += gridDim.x * blockDim.x) {
    const int ri = failed_list[f];
    row_count[ri] = redo_count[ri];
  }
}

// Compaction into the final CSR: one warp per light row, heavy item (of a row
// that did not fail) and failed row; lanes copy the contiguous run.
template <typename VT>
__global__ void k_compact(Geom g, const int32_t* __restrict__ light_list, int n_light,
                          const int64_t* __restrict__ light_slot, const int32_t* __restrict__ heavy_list,
                          const HeavyItem* __restrict__ items, int64_t n_items, const int64_t* __restrict__ first,
                          const int32_t* __restrict__ item_count, const int64_t* __restrict__ item_pos,
                          const int32_t* __restrict__ row_failed, const int32_t* __restrict__ failed_list,
                          int n_failed, int64_t heavy_slot_base, const int64_t* __restrict__ item_off,
                          const int64_t* __restrict__ redo_off,
                          const int32_t* __restrict__ row_count,
                          const int64_t* __restrict__ row_offset, const int32_t* __restrict__ tcol,
                          const VT* __restrict__ tval, const int32_t* __restrict__ rcol, const VT* __restrict__ rval,
                          int32_t* __restrict__ out_col, VT* __restrict__ out_val) {
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t total = (int64_t)n_light + n_items + n_failed;
  for (int64_t u = warp; u < total; u += nwarps) {
    int64_t src, dst;
    int cnt;
    const int32_t* sc = tcol;
    const VT* sv = tval;
    if (u < n_light) {
      const int ri = light_list[u];
      src = light_slot[u];
      dst = row_offset[ri];
      cnt = row_count[ri];
    } else if (u < n_light + n_items) {
      const int64_t idx = u - n_light;
      const HeavyItem it = items[idx];
      if (row_failed[it.h]) continue;
      const int ri = heavy_list[it.h];
      src = heavy_slot_base + item_off[idx];
      dst = row_offset[ri] + (item_pos[idx] - item_pos[first[it.h]]);
      cnt = item_count[idx];
    } else {
      const int ri = failed_list[u - n_light - n_items];
      src = redo_off[ri];
      dst = row_offset[ri];
      cnt = row_count[ri];
      sc = rcol;
      sv = rval;
    }
    for (int q = lane; q < cnt; q += 32) {
      out_col[dst + q] = sc[src + q];
      out_val[dst + q] = sv[src + q];
    }
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
  int64_t products = 0, nnz = 0, n_light = 0, n_heavy = 0, n_vheavy = 0, n_heavy_items = 0;
  int64_t hbm_words = 0;
  int32_t* light_list = nullptr;
  int32_t* heavy_list = nullptr;   // very heavy rows first, then the other heavy rows
  int32_t* vheavy_list = nullptr;
  int32_t* heavy_tmp = nullptr;
  int32_t* counters = nullptr;  // [0] light rows, [1] heavy rows (total after planning), [2] overflow, [3] very heavy
  unsigned long long* products_dev = nullptr;
  int32_t* row_count = nullptr;
  int64_t* row_offset = nullptr;
  uint32_t* heavy_bitmaps = nullptr;
  int16_t* heavy_span = nullptr;  // per heavy row: first fine block with outputs, one past the last (or null)
  int32_t* heavy_nitems = nullptr;
  int64_t* heavy_first = nullptr;
  HeavyItem* heavy_items = nullptr;
  int32_t* tab = nullptr;
  int32_t* smap_own = nullptr;    // stage map (Geom::smap / scount) owned by this plan
  int32_t* scount_own = nullptr;
  int32_t* rot_own = nullptr;     // sub-grid tile maps (Geom::rot_i, then rot_j) owned by this plan
  unsigned long long* queue = nullptr;  // work-queue heads, one per stage launch
  // numeric tuning (bclx_spgemm_plan_tune)
  int grab = 1, blocks_per_sm = 4, long_seg = kLongSegDefault;
  int light_ub_max = kLightUb;         // light-row class bound (products), set at symbolic time
  int vcap = kVcap;                    // outputs per heavy item (512 or 1024), set at symbolic time
  // CUDA graph of the staged numeric pass (bclx_spgemm_numeric_staged)
  cudaGraphExec_t graph = nullptr;
  const void* graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaStream_t gstream = nullptr;  // capture/replay stream (the caller's may be the legacy default stream)
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // learned product (bclx_spgemm_learned_run / _finish)
  bool learned = false;
  float* feat = nullptr;            // [nri*5]
  int32_t* ub = nullptr;            // [nri]
  float* pred = nullptr;            // [nri]
  int64_t* light_slot = nullptr;    // [n_light+1]
  int32_t* light_ub = nullptr;      // [n_light]
  int32_t* item_count = nullptr;    // [n_heavy_items]
  int32_t* item_cap = nullptr;      // [n_heavy_items] temp slots per heavy item
  int64_t* item_off = nullptr;      // [n_heavy_items+1] their offsets
  int64_t* item_pos = nullptr;      // [n_heavy_items+1]
  int32_t* row_failed = nullptr;    // [n_heavy]
  int32_t* block_ub = nullptr;      // [n_heavy*nfb] products per fine block
  int32_t* failed_list = nullptr;   // [n_heavy] row indices of failed rows
  int32_t* temp_col = nullptr;
  void* temp_val = nullptr;
  int64_t temp_entries = 0, n_failed = 0, heavy_slot_base = 0;
  bclx_spgemm_plan_s* redo = nullptr;  // exact plan over the failed rows
  int64_t* redo_off = nullptr;         // [nri+1]
  int32_t* redo_col = nullptr;
  void* redo_val = nullptr;
  // tile accumulation: identity A tiles and their descriptors, 1x1 C offsets
  int32_t* id_rp = nullptr;
  int32_t* id_ci = nullptr;
  void* id_v = nullptr;
  bclx_csr_t* id_desc = nullptr;
  int64_t* acc_tile_offset = nullptr;

  void release() {
    // planning work on the side stream must be done before its scratch goes
    if (ctx && ctx->side) cudaStreamSynchronize(ctx->side);
    if (graph) {
      cudaGraphExecDestroy(graph);
      graph = nullptr;
    }
    if (gstream) {
      cudaStreamSynchronize(gstream);
      cudaStreamDestroy(gstream);
      gstream = nullptr;
    }
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    ev_in = ev_out = nullptr;
    if (redo) {
      redo->heavy_list = nullptr;  // borrowed from this plan
      redo->light_list = nullptr;
      redo->row_offset = nullptr;
      redo->tab = nullptr;
      redo->release();
      delete redo;
      redo = nullptr;
    }
    void* lp[] = {feat, ub, pred, light_slot, light_ub, item_count, item_cap, item_off, item_pos, row_failed, block_ub,
                  failed_list,
                  temp_col,
                  temp_val, redo_off, redo_col, redo_val};
    for (void* p : lp) scratch_free(ctx, p);
    feat = pred = nullptr;
    ub = light_ub = item_count = item_cap = row_failed = block_ub = failed_list = temp_col = redo_col = nullptr;
    light_slot = item_pos = item_off = redo_off = nullptr;
    temp_val = redo_val = nullptr;
    void* ps[] = {queue, light_list, heavy_list, vheavy_list, heavy_tmp, counters, products_dev, row_count, row_offset, heavy_bitmaps,
                  heavy_nitems, heavy_first, heavy_items, tab, id_rp, id_ci, id_v, id_desc, acc_tile_offset,
                  smap_own, scount_own, rot_own, heavy_span};
    for (void* p : ps) scratch_free(ctx, p);
    queue = nullptr;
    heavy_span = nullptr;
    smap_own = scount_own = rot_own = nullptr;
    light_list = heavy_list = vheavy_list = heavy_tmp = counters = row_count = heavy_nitems = tab = id_rp = id_ci = nullptr;
    products_dev = nullptr;
    row_offset = heavy_first = acc_tile_offset = nullptr;
    heavy_bitmaps = nullptr;
    heavy_items = nullptr;
    id_v = nullptr;
    id_desc = nullptr;
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
  if (a->grid_n < 1 || a->grid_n >= kNoStage) {
    set_last_error("the k dimension must have between 1 and 254 tiles");
    return BCLX_ERR_INVALID;
  }
  if (c->tile_n > kMaxCols) {
    set_last_error("tiles wider than 16384 columns are not supported; use a finer tile grid");
    return BCLX_ERR_INVALID;
  }
  if (c->grid_m * c->grid_n * c->tile_m > INT32_MAX) return BCLX_ERR_INDEX_OVERFLOW;
  if (a->dtype != b->dtype || a->dtype != c->dtype || !value_size(a->dtype)) return BCLX_ERR_DTYPE;
  return BCLX_OK;
}

// Rows a warp takes from a device counter at a time: about `per_warp` grabs
// per resident warp over the pass, at least 1 and at most `cap`.
static int queue_grab(Context* ctx, int64_t rows, int warps_per_block, int blocks_per_sm, int cap,
                      int per_warp = 32) {
  const int64_t warps = (int64_t)ctx->num_sms * blocks_per_sm * warps_per_block;
  const int64_t g = rows / (warps * per_warp);
  return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

static unsigned grid_for(Context* ctx, int64_t work_warps, int warps_per_block, int blocks_per_sm) {
  int64_t want = (work_warps + warps_per_block - 1) / warps_per_block;
  int64_t cap = (int64_t)ctx->num_sms * blocks_per_sm;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return (unsigned)want;
}

// With `side`, the very heavy rows (a block per row, few blocks) run on the
// context's side stream beside the warp-per-row kernel; the caller joins the
// side stream back before reading the counts.
static int launch_symbolic(Context* ctx, const SpGridView& A, const SpGridView& B, bclx_spgemm_plan_s* P,
                           bool side = false) {
  if (P->n_vheavy > 0) {
    cudaStream_t st = ctx->stream;
    if (side) {
      BCLX_CK(cudaEventRecord(ctx->fork2_ev, ctx->stream));
      BCLX_CK(cudaStreamWaitEvent(ctx->side, ctx->fork2_ev, 0));
      st = ctx->side;
    }
    k_symbolic_block<<<grid_for(ctx, P->n_vheavy, 1, 8), kWarpsSym * 32, 0, st>>>(
        A, B, P->g, P->heavy_list, (int)P->n_vheavy, P->row_count, P->heavy_bitmaps, P->hbm_words, P->heavy_span);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  const int64_t rows = P->n_light + P->n_heavy - P->n_vheavy;
  if (rows > 0) {
    // queue head 0 (each numeric launch clears its head before use)
    BCLX_CK(cudaMemsetAsync(P->queue, 0, sizeof(unsigned long long), ctx->stream));
    k_symbolic<<<grid_for(ctx, rows, kWarpsSym, 8), kWarpsSym * 32, 0, ctx->stream>>>(
        A, B, P->g, P->light_list, P->heavy_list, (int)P->n_light, (int)P->n_heavy, (int)P->n_vheavy,
        P->row_count, P->heavy_bitmaps, P->hbm_words, P->heavy_span, P->queue, queue_grab(ctx, rows, kWarpsSym, 8, 8));
    note_launch();
    BCLX_CK_LAUNCH();
  }
  return BCLX_OK;
}

template <typename VT, int WORDS, bool LEARNED = false, int VCAP = kVcap>
static int launch_numeric_w(Context* ctx, const SpGridView& A, const SpGridView& B, bclx_spgemm_plan_s* P,
                            int32_t* out_col, void* out_val, int s0, int s1) {
  constexpr size_t smem = sizeof(WarpSmem<VT, WORDS, VCAP>) * kWarpsNum;
  auto kern = k_numeric<VT, WORDS, LEARNED, VCAP>;
  static std::atomic<unsigned long long> configured{0};  // one bit per device
  const unsigned long long bit = 1ull << (ctx->device & 63);
  if (!(configured.load() & bit)) {
    BCLX_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    configured.fetch_or(bit);
  }
  const int64_t n_total = P->n_light + P->n_heavy_items;
  unsigned long long* q = P->queue + (s0 % kQueueSlots);
  BCLX_CK(cudaMemsetAsync(q, 0, sizeof(unsigned long long), ctx->stream));
  const int bps = P->blocks_per_sm < 1 ? 1 : (P->blocks_per_sm > 4 ? 4 : P->blocks_per_sm);
  kern<<<grid_for(ctx, n_total, kWarpsNum, bps), kWarpsNum * 32, smem, ctx->stream>>>(
      A, B, P->g, P->light_list, P->heavy_list, (int)P->n_light, P->n_heavy_items, P->heavy_items, P->heavy_bitmaps,
      P->hbm_words, P->tab, P->row_count, P->row_offset, out_col, reinterpret_cast<VT*>(out_val), s0, s1, q,
      P->grab < 1 ? 1 : P->grab, P->long_seg < 1 ? 1 : P->long_seg, LEARNED ? P->light_slot : nullptr,
      LEARNED ? P->item_count : nullptr, LEARNED ? P->row_count : nullptr, LEARNED ? P->row_failed : nullptr,
      P->heavy_slot_base, LEARNED ? P->item_off : nullptr);
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

template <typename VT>
static int launch_numeric(Context* ctx, const SpGridView& A, const SpGridView& B, bclx_spgemm_plan_s* P,
                          int32_t* out_col, void* out_val, int s0, int s1) {
  if (P->vcap == 1024) {
    if (P->g.tn <= 8192) return launch_numeric_w<VT, 256, false, 1024>(ctx, A, B, P, out_col, out_val, s0, s1);
    return launch_numeric_w<VT, kMaxWords, false, 1024>(ctx, A, B, P, out_col, out_val, s0, s1);
  }
  if (P->g.tn <= 8192) return launch_numeric_w<VT, 256>(ctx, A, B, P, out_col, out_val, s0, s1);
  return launch_numeric_w<VT, kMaxWords>(ctx, A, B, P, out_col, out_val, s0, s1);
}

// Stage map for fine grids: per C tile, the rotated stage positions whose A
// and B tiles both have entries (a banded matrix on a fine grid has a few of
// gk).  Coarse grids (gk <= 16) walk every stage.
__global__ void k_stage_map(SpGridView A, SpGridView B, Geom g, int32_t* __restrict__ smap,
                            int32_t* __restrict__ scount) {
  const int64_t nt = g.gm * g.gn;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ti = t / g.gn, tj = t - ti * g.gn;
    int32_t c = 0;
    const int64_t rot = tile_rotation(g, ti, tj);
    for (int64_t kk = 0; kk < g.gk; kk++) {
      const int64_t k = (kk + rot) % g.gk;
      if (A.tile(ti, k).nnz > 0 && B.tile(k, tj).nnz > 0) smap[t * g.gk + c++] = (int32_t)kk;
    }
    scount[t] = c;
  }
}

// C tiles with at least one stage (scount[t] > 0) into live[], their number
// to *n_live (one atomic per warp; the order is immaterial).
__global__ void k_live_tiles(const int32_t* __restrict__ scount, int64_t nt, int32_t* __restrict__ live,
                             int32_t* __restrict__ n_live) {
  const int lane = lane_id();
  const int64_t end = (nt + 31) & ~int64_t(31);  // whole warps run every iteration
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < end; t += (int64_t)gridDim.x * blockDim.x) {
    const bool on = t < nt && scount[t] > 0;
    const unsigned m = __ballot_sync(kFull, on);
    if (m == 0) continue;
    int base = 0;
    if (lane == 0) base = atomicAdd(n_live, __popc(m));
    base = __shfl_sync(kFull, base, 0);
    if (on) live[base + __popc(m & ((1u << lane) - 1u))] = (int32_t)t;
  }
}

constexpr int64_t kStageMapMinGrid = 17;

static int build_stage_map(Context* ctx, const SpGridView& A, const SpGridView& B, bclx_spgemm_plan_s* P, Geom& g) {
  g.smap = g.scount = nullptr;
  if (g.gk < kStageMapMinGrid) return BCLX_OK;
  const int64_t nt = g.gm * g.gn;
  BCLX_TRY(scratch_alloc_n(ctx, &P->smap_own, (size_t)(nt * g.gk)));
  BCLX_TRY(scratch_alloc_n(ctx, &P->scount_own, (size_t)nt));
  k_stage_map<<<grid_for(ctx, nt / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(A, B, g, P->smap_own, P->scount_own);
  note_launch();
  BCLX_CK_LAUNCH();
  g.smap = P->smap_own;
  g.scount = P->scount_own;
  return BCLX_OK;
}

// With a stage map: the C tiles that have stages, into a new scratch array
// (their number in its last slot, written by the device); *live stays null
// without a map (every tile is walked).
static int build_live_tiles(Context* ctx, const Geom& g, int32_t** live) {
  *live = nullptr;
  if (!g.scount) return BCLX_OK;
  const int64_t nt = g.gm * g.gn;
  BCLX_TRY(scratch_alloc_n(ctx, live, (size_t)nt + 1));
  BCLX_CK(cudaMemsetAsync(*live + nt, 0, sizeof(int32_t), ctx->stream));
  k_live_tiles<<<grid_for(ctx, nt / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(g.scount, nt, *live, *live + nt);
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

// B-row table (k_btable) when it fits the context's BCLX_TUNE_BTABLE_MAX_BYTES
// (default 2 GiB); otherwise none and the walks find column-block ranges by
// binary search.  (A larger table pays where memory allows: R-MAT s20 on
// 64x64 tiles, 17.4 GB, 638 against 679 ms per product; but the table is
// sized before the product's bitmaps and C are, so the default stays small.)
static int64_t btable_cap(const Context* ctx) { return tuning(ctx, BCLX_TUNE_BTABLE_MAX_BYTES); }

// With `side`, the table is allocated in stream order on the main stream and
// built on `side` after a fork event.
static int build_btable(Context* ctx, const SpGridView& B, const Geom& g, bclx_spgemm_plan_s* P,
                        cudaStream_t side = nullptr) {
  const int64_t nbrows = g.gk * g.gn * g.tk;
  if ((int64_t)sizeof(int32_t) * nbrows * (g.nfb + 1) > btable_cap(ctx)) {
    P->tab = nullptr;
    return BCLX_OK;
  }
  BCLX_TRY(scratch_alloc_n(ctx, &P->tab, (size_t)nbrows * (g.nfb + 1)));
  cudaStream_t st = ctx->stream;
  if (side) {
    BCLX_CK(cudaEventRecord(ctx->fork_ev, ctx->stream));
    BCLX_CK(cudaStreamWaitEvent(side, ctx->fork_ev, 0));
    st = side;
  }
  k_btable<<<grid_for(ctx, nbrows / 32 + 1, 8, 16), 256, 0, st>>>(B, g, P->tab);
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

// Classification, symbolic, row offsets and the heavy-row cut.
static int symbolic_impl(Context* ctx, const SpGridView& A, const SpGridView& B, Geom g, int dtype,
                         int32_t* tile_row_ptr, int64_t* tile_offset, bclx_spgemm_plan_s* P) {
  BCLX_TRY(build_stage_map(ctx, A, B, P, g));
  P->g = g;
  // The B-row table depends on B alone: it is built on the side stream from
  // the start, beside classification and the symbolic pass.
  BCLX_TRY(ensure_side_stream(ctx));
  BCLX_TRY(build_btable(ctx, B, g, P, ctx->side));
  P->dtype = dtype;
  const int64_t nri = g.n_row_items;
  P->hbm_words = (g.tn + 31) / 32;
  BCLX_TRY(scratch_alloc_n(ctx, &P->light_list, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_list, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->vheavy_list, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_tmp, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->counters, 4));
  BCLX_TRY(scratch_alloc_n(ctx, &P->products_dev, 1));
  BCLX_TRY(scratch_alloc_n(ctx, &P->row_count, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->row_offset, nri + 1));
  BCLX_TRY(scratch_alloc_n(ctx, &P->queue, kQueueSlots));
  BCLX_CK(cudaMemsetAsync(P->counters, 0, 4 * sizeof(int32_t), ctx->stream));
  BCLX_CK(cudaMemsetAsync(P->products_dev, 0, sizeof(unsigned long long), ctx->stream));
  BCLX_CK(cudaMemsetAsync(P->row_count, 0, sizeof(int32_t) * (nri > 0 ? nri : 1), ctx->stream));
  // rows of tiles wider than 8192 columns take the heavy path unless the
  // context allows light rows there (BCLX_TUNE_WIDE_LIGHT)
  const int heavy_min_cols = tuning(ctx, BCLX_TUNE_WIDE_LIGHT) ? INT_MAX : 8192 + 1;
  P->light_ub_max = (int)tuning(ctx, BCLX_TUNE_LIGHT_UB);
  P->vcap = (int)tuning(ctx, BCLX_TUNE_ITEM_OUTPUTS);
  int32_t* live = nullptr;  // C tiles with stages (when the stage map says which)
  if (nri > 0) {
    BCLX_CK(cudaMemsetAsync(P->queue + 1, 0, sizeof(unsigned long long), ctx->stream));
    const int64_t nt = g.gm * g.gn;
    BCLX_TRY(build_live_tiles(ctx, g, &live));
    k_classify<false><<<grid_for(ctx, nri, 8, 16), 256, 0, ctx->stream>>>(
        A, B, g, P->light_list, P->heavy_tmp, P->vheavy_list, P->counters, P->products_dev, heavy_min_cols, P->light_ub_max,
        nullptr, nullptr, P->queue + 1, queue_grab(ctx, nri, 8, 16, 32, 8), live, live ? live + nt : nullptr);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  BCLX_TRY(read_back(ctx, {{P->counters, 8, 0}, {P->counters + 2, 8, 1}, {P->products_dev, 8, 2}}));
  if (live) scratch_free(ctx, live);
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  int32_t cnts[4];
  std::memcpy(cnts, ctx->pinned, sizeof(cnts));
  P->n_light = cnts[0];
  P->n_vheavy = cnts[3];
  P->n_heavy = cnts[1] + cnts[3];
  P->products = ctx->pinned[2];
  // heavy slots: the very heavy rows first, then the others
  if (P->n_vheavy > 0)
    BCLX_CK(cudaMemcpyAsync(P->heavy_list, P->vheavy_list, sizeof(int32_t) * P->n_vheavy, cudaMemcpyDeviceToDevice,
                            ctx->stream));
  if (cnts[1] > 0)
    BCLX_CK(cudaMemcpyAsync(P->heavy_list + P->n_vheavy, P->heavy_tmp, sizeof(int32_t) * cnts[1],
                            cudaMemcpyDeviceToDevice, ctx->stream));

  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_bitmaps, (size_t)P->n_heavy * P->hbm_words));
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_span, 2 * (size_t)P->n_heavy));
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_nitems, P->n_heavy));
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_first, P->n_heavy + 1));
  BCLX_TRY(launch_symbolic(ctx, A, B, P, true));
  // the side stream (B-row table, very heavy rows) joins before the scan
  BCLX_CK(cudaEventRecord(ctx->join_ev, ctx->side));
  BCLX_CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0));
  BCLX_TRY(exclusive_scan_i32(ctx, P->row_count, P->row_offset, nri));
  const int64_t ntiles = g.gm * g.gn;
  k_tile_ptrs<<<grid_for(ctx, ntiles * (g.tm + 1) / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(
      g, P->row_offset, tile_row_ptr, tile_offset, P->counters + 2);
  note_launch();
  BCLX_CK_LAUNCH();
  if (P->n_heavy > 0) {
    const unsigned blocks = grid_for(ctx, P->n_heavy, 8, 8);
    k_cut_heavy<false><<<blocks, 256, 0, ctx->stream>>>(g, P->heavy_list, (int)P->n_heavy, P->heavy_bitmaps,
                                                        P->hbm_words, P->heavy_nitems, nullptr, nullptr, P->vcap,
                                                        P->row_count, P->heavy_span);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  BCLX_TRY(exclusive_scan_i32(ctx, P->heavy_nitems, P->heavy_first, P->n_heavy));
  BCLX_TRY(read_back(ctx, {{P->row_offset + nri, 8, 0}, {P->heavy_first + P->n_heavy, 8, 1}, {P->counters + 2, 4, 2}}));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  P->nnz = ctx->pinned[0];
  P->n_heavy_items = ctx->pinned[1];
  int32_t overflow;
  std::memcpy(&overflow, ctx->pinned + 2, sizeof(overflow));
  if (overflow) {
    set_last_error("a C tile has more than 2^31-1 nonzeros; use a finer tile grid");
    return BCLX_ERR_INDEX_OVERFLOW;
  }
  if (P->n_heavy > 0) {
    BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_items, P->n_heavy_items));
    const unsigned blocks = grid_for(ctx, P->n_heavy, 8, 8);
    k_cut_heavy<true><<<blocks, 256, 0, ctx->stream>>>(g, P->heavy_list, (int)P->n_heavy, P->heavy_bitmaps,
                                                       P->hbm_words, nullptr, P->heavy_first, P->heavy_items, P->vcap,
                                                       P->row_count, P->heavy_span);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  if (P->n_heavy == 0 && P->tab) {  // no heavy item reads the table
    scratch_free(ctx, P->tab);
    P->tab = nullptr;
  }
  return BCLX_OK;
}

static int numeric_impl(Context* ctx, bclx_spgemm_plan_s* P, const SpGridView& A, const SpGridView& B,
                        int32_t* out_col, void* out_val, int s0, int s1) {
  if (s1 <= 0 || s1 > P->g.gk) s1 = (int)P->g.gk;
  if (s0 < 0 || s0 > s1) return BCLX_ERR_INVALID;
  if (P->n_light + P->n_heavy_items == 0 || s0 == s1) return BCLX_OK;
  if (P->dtype == BCLX_F32) return launch_numeric<float>(ctx, A, B, P, out_col, out_val, s0, s1);
  return launch_numeric<int32_t>(ctx, A, B, P, out_col, out_val, s0, s1);
}

static Geom make_geom(const bclx_spgrid_out_t* c, int64_t gk, int64_t tk) {
  Geom g;
  g.gm = c->grid_m; g.gn = c->grid_n; g.gk = gk;
  g.tm = c->tile_m; g.tn = c->tile_n; g.tk = tk; g.m = c->m; g.n = c->n;
  g.n_row_items = g.gm * g.gn * g.tm;
  g.nfb = ceil_div(g.tn, kFineCols);
  return g;
}

}  // namespace bclx

extern "C" {

// Sub-grid tile maps: global tile indices increasing (so only the last may
// be a ragged edge tile) and in range.
static bool maps_ok(const bclx_spgrid_out_t* out, const int64_t* tile_rows, const int64_t* tile_cols) {
  for (int64_t i = 0; i < out->grid_m; i++)
    if (tile_rows[i] < 0 || tile_rows[i] >= INT32_MAX || (i > 0 && tile_rows[i] <= tile_rows[i - 1])) return false;
  for (int64_t j = 0; j < out->grid_n; j++)
    if (tile_cols[j] < 0 || tile_cols[j] >= INT32_MAX || (j > 0 && tile_cols[j] <= tile_cols[j - 1])) return false;
  return true;
}

// Device copies of the maps (owned by the plan) into g.rot_i / g.rot_j.
static int attach_maps(Context* ctx, bclx_spgemm_plan_s* P, Geom& g, const bclx_spgrid_out_t* out,
                       const int64_t* tile_rows, const int64_t* tile_cols) {
  std::vector<int32_t> maps((size_t)(out->grid_m + out->grid_n));
  for (int64_t i = 0; i < out->grid_m; i++) maps[(size_t)i] = (int32_t)(tile_rows[i] % g.gk);
  for (int64_t j = 0; j < out->grid_n; j++) maps[(size_t)(out->grid_m + j)] = (int32_t)(tile_cols[j] % g.gk);
  BCLX_TRY(scratch_alloc_n(ctx, &P->rot_own, maps.size()));
  BCLX_CK(cudaMemcpyAsync(P->rot_own, maps.data(), sizeof(int32_t) * maps.size(), cudaMemcpyHostToDevice,
                          ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));  // the host vector goes out of scope
  g.rot_i = P->rot_own;
  g.rot_j = P->rot_own + out->grid_m;
  return BCLX_OK;
}

static int symbolic_entry(bclx_context_t c, const bclx_spgrid_t* a, const bclx_spgrid_t* b, bclx_spgrid_out_t* out,
                          const int64_t* tile_rows, const int64_t* tile_cols, bclx_spgemm_plan_t* plan,
                          int64_t* nnz) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !plan || !nnz) return BCLX_ERR_INVALID;
  *plan = nullptr;
  BCLX_TRY(check_grids(a, b, out));
  if (!out->tile_row_ptr || !out->tile_offset) return BCLX_ERR_INVALID;
  if (tile_rows && !maps_ok(out, tile_rows, tile_cols)) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  auto* P = new bclx_spgemm_plan_s();
  P->ctx = ctx;
  Geom g = make_geom(out, a->grid_n, a->tile_n);
  int rc = tile_rows ? attach_maps(ctx, P, g, out, tile_rows, tile_cols) : BCLX_OK;
  if (rc == BCLX_OK)
    rc = symbolic_impl(ctx, make_view(*a), make_view(*b), g, a->dtype, out->tile_row_ptr, out->tile_offset, P);
  if (rc != BCLX_OK) {
    P->release();
    delete P;
    return rc;
  }
  *nnz = P->nnz;
  *plan = P;
  return BCLX_OK;
}

int bclx_spgemm_symbolic(bclx_context_t c, const bclx_spgrid_t* a, const bclx_spgrid_t* b, bclx_spgrid_out_t* out,
                         bclx_spgemm_plan_t* plan, int64_t* nnz) {
  return symbolic_entry(c, a, b, out, nullptr, nullptr, plan, nnz);
}

int bclx_spgemm_symbolic_sub(bclx_context_t c, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                             bclx_spgrid_out_t* out, const int64_t* tile_rows, const int64_t* tile_cols,
                             bclx_spgemm_plan_t* plan, int64_t* nnz) {
  if (!tile_rows || !tile_cols) return BCLX_ERR_INVALID;
  return symbolic_entry(c, a, b, out, tile_rows, tile_cols, plan, nnz);
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
  out6[1] = P->n_light;
  out6[2] = P->n_heavy;
  out6[3] = P->n_heavy_items;
  out6[4] = P->g.gk;
  out6[5] = P->nnz;
  return BCLX_OK;
}

int bclx_spgemm_plan_tune(bclx_spgemm_plan_t P, int32_t grab, int32_t blocks_per_sm, int32_t long_seg) {
  if (!P || grab < 1 || grab > 64 || blocks_per_sm < 1 || blocks_per_sm > 4 || long_seg < 1)
    return BCLX_ERR_INVALID;
  P->grab = grab;
  P->blocks_per_sm = blocks_per_sm;
  P->long_seg = long_seg;
  if (P->graph) {  // the captured launches carry the old parameters
    cudaGraphExecDestroy(P->graph);
    P->graph = nullptr;
  }
  return BCLX_OK;
}

int bclx_spgemm_numeric_staged(bclx_context_t c, bclx_spgemm_plan_t P, const bclx_spgrid_t* a,
                               const bclx_spgrid_t* b, bclx_spgrid_out_t* out, int32_t use_graph) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !P) return BCLX_ERR_INVALID;
  BCLX_TRY(check_grids(a, b, out));
  if (a->grid_n != P->g.gk || out->grid_m != P->g.gm || out->grid_n != P->g.gn || a->dtype != P->dtype)
    return BCLX_ERR_INVALID;
  if (P->nnz > 0 && (!out->col_ind || !out->vals)) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  const SpGridView A = make_view(*a), B = make_view(*b);
  const int G = (int)P->g.gk;
  auto run_all = [&]() -> int {
    for (int s = 0; s < G; s++) BCLX_TRY(numeric_impl(ctx, P, A, B, out->col_ind, out->vals, s, s + 1));
    return BCLX_OK;
  };
  if (!use_graph) return run_all();
  const void* key[4] = {a->tiles, b->tiles, out->col_ind, out->vals};
  if (P->graph && std::memcmp(key, P->graph_key, sizeof(key)) != 0) {
    cudaGraphExecDestroy(P->graph);
    P->graph = nullptr;
  }
  if (!P->gstream) {
    BCLX_CK(cudaStreamCreateWithFlags(&P->gstream, cudaStreamNonBlocking));
    BCLX_CK(cudaEventCreateWithFlags(&P->ev_in, cudaEventDisableTiming));
    BCLX_CK(cudaEventCreateWithFlags(&P->ev_out, cudaEventDisableTiming));
  }
  if (!P->graph) {
    // this call computes C directly (which also configures the kernels), then
    // captures the G launches on the plan's stream for later replays
    BCLX_TRY(run_all());
    BCLX_CK(cudaEventRecord(P->ev_in, ctx->stream));
    BCLX_CK(cudaStreamWaitEvent(P->gstream, P->ev_in, 0));
    Context cap = *ctx;
    cap.stream = P->gstream;
    cudaGraph_t graph = nullptr;
    BCLX_CK(cudaStreamBeginCapture(P->gstream, cudaStreamCaptureModeThreadLocal));
    int rc = BCLX_OK;
    for (int s = 0; s < G && rc == BCLX_OK; s++)
      rc = numeric_impl(&cap, P, A, B, out->col_ind, out->vals, s, s + 1);
    const cudaError_t e = cudaStreamEndCapture(P->gstream, &graph);
    if (rc != BCLX_OK) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) {
      set_last_error(std::string("cudaStreamEndCapture: ") + cudaGetErrorString(e));
      return BCLX_ERR_CUDA;
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      set_last_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
      return BCLX_ERR_CUDA;
    }
    P->graph = exec;
    std::memcpy(P->graph_key, key, sizeof(key));
    return BCLX_OK;
  }
  BCLX_CK(cudaEventRecord(P->ev_in, ctx->stream));
  BCLX_CK(cudaStreamWaitEvent(P->gstream, P->ev_in, 0));
  BCLX_CK(cudaGraphLaunch(P->graph, P->gstream));
  BCLX_CK(cudaEventRecord(P->ev_out, P->gstream));
  BCLX_CK(cudaStreamWaitEvent(ctx->stream, P->ev_out, 0));
  note_launch(G);
  return BCLX_OK;
}

// Tile accumulation as a product: A = [I I ... I] (1 x nparts identity
// tiles, value 1), B = [parts] (nparts x 1).  With a 1x1 C grid the stage
// order is the list order, each partial value passes through fma(1, v, 0) == v
// exactly, and the partials are added from 0 in list order: the
// SparseHashAccumulator sum.
static void accumulate_views(bclx_spgemm_plan_s* P, const bclx_csr_t* parts, int32_t nparts, int64_t m, int64_t n,
                             SpGridView* A, SpGridView* B, Geom* g) {
  A->tiles = P->id_desc;
  A->m = m; A->n = m * (int64_t)nparts; A->tm = m; A->tn = m; A->gm = 1; A->gn = nparts;
  B->tiles = parts;
  B->m = m * (int64_t)nparts; B->n = n; B->tm = m; B->tn = n; B->gm = nparts; B->gn = 1;
  g->gm = 1; g->gn = 1; g->gk = nparts; g->tm = m; g->tn = n; g->tk = m; g->m = m; g->n = n; g->n_row_items = m;
  g->nfb = ceil_div(n, kFineCols);
}

int bclx_tile_accumulate_symbolic(bclx_context_t c, const bclx_csr_t* parts, int32_t nparts, int64_t m, int64_t n,
                                  int32_t dtype, int32_t* c_row_ptr, bclx_spgemm_plan_t* plan, int64_t* nnz) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !plan || !nnz || !parts || nparts < 1 || m < 1 || n < 1 || !c_row_ptr) return BCLX_ERR_INVALID;
  if (nparts >= kNoStage || m > INT32_MAX) return BCLX_ERR_INVALID;
  if (n > kMaxCols) {
    set_last_error("tiles wider than 16384 columns are not supported");
    return BCLX_ERR_INVALID;
  }
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
    note_launch(2);
    if (cudaGetLastError() != cudaSuccess) { rc = BCLX_ERR_CUDA; break; }
    SpGridView A{}, B{};
    Geom g{};
    accumulate_views(P, parts, nparts, m, n, &A, &B, &g);
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
  accumulate_views(P, parts, nparts, out->m, out->n, &A, &B, &g);
  return numeric_impl(ctx, P, A, B, out->col_ind, out->vals, 0, nparts);
}

}  // extern "C"

// ---- product of one tile pair without allocating -----------------------------------
//
// For callers that cannot allocate device memory at the time of the call: a
// framework that has reserved the device's memory for its own allocator, or
// code that must not call cudaMalloc/cudaFree because those calls
// synchronize the device.  Every work array of the two phases comes from one
// file-scope device array of kNoAllocScratchBytes, which every GPU that loads
// this library holds until the process exits.  The first call on a device
// looks up that array's device address (cudaGetSymbolAddress, with the device
// current); that first call should come before any stream capture.  Every
// call uses the same array, and whatever the last call left in it: the parts
// that must start at zero are cleared by each call, and calls whose work
// overlaps on the GPU (for instance on two streams) race with each other.
// The host reads two sizes back during a call (cudaStreamSynchronize on the
// caller's stream each time).

namespace bclx {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
static void* g_noalloc_base[kNoAllocMaxDevices];
static std::mutex g_noalloc_mutex;

struct ScratchArena {
  unsigned char* base;
  size_t cap;
  size_t used = 0;
  bool ok = true;
  template <typename T>
  T* take(size_t count) {
    const size_t bytes = (sizeof(T) * (count > 0 ? count : 1) + 255) & ~size_t(255);
    if (!ok || used + bytes > cap) {
      ok = false;
      return nullptr;
    }
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};

static int noalloc_base(int device, void** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (device < 0 || device >= kNoAllocMaxDevices) {
    set_last_error("device ordinal out of range for the no-allocation scratch");
    return BCLX_ERR_NO_DEVICE;
  }
  if (!g_noalloc_base[device]) {
    void* p = nullptr;
    BCLX_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_base[device] = p;
  }
  *out = g_noalloc_base[device];
  return BCLX_OK;
}

static int noalloc_exhausted() {
  set_last_error("this product needs more than the 32 MiB no-allocation scratch; use "
                 "bclx_spgemm_symbolic/bclx_spgemm_numeric instead");
  return BCLX_ERR_INVALID;
}

static int noalloc_product(Context* ctx, ScratchArena& ar, const bclx_csr_t* a, const bclx_csr_t* b,
                           int32_t* c_row_ptr, int32_t* c_col_ind, void* c_vals, int64_t c_capacity,
                           int64_t* c_nnz) {
  const int64_t m = a->m, k = a->n, n = b->n;
  bclx_csr_t* dA = ar.take<bclx_csr_t>(1);
  bclx_csr_t* dB = ar.take<bclx_csr_t>(1);
  if (!ar.ok) return noalloc_exhausted();
  BCLX_CK(cudaMemcpyAsync(dA, a, sizeof(bclx_csr_t), cudaMemcpyHostToDevice, ctx->stream));
  BCLX_CK(cudaMemcpyAsync(dB, b, sizeof(bclx_csr_t), cudaMemcpyHostToDevice, ctx->stream));
  SpGridView A{}, B{};
  A.tiles = dA; A.m = m; A.n = k; A.tm = m; A.tn = k; A.gm = 1; A.gn = 1;
  B.tiles = dB; B.m = k; B.n = n; B.tm = k; B.tn = n; B.gm = 1; B.gn = 1;
  Geom g;
  g.gm = 1; g.gn = 1; g.gk = 1; g.tm = m; g.tn = n; g.tk = k; g.m = m; g.n = n;
  g.n_row_items = m;
  g.nfb = ceil_div(n, kFineCols);

  bclx_spgemm_plan_s P;  // its arrays live in the arena; it is never released
  P.ctx = ctx;
  P.g = g;
  P.dtype = a->dtype;
  P.hbm_words = (n + 31) / 32;
  const int64_t nri = m;
  P.light_list = ar.take<int32_t>(nri);
  P.heavy_list = ar.take<int32_t>(nri);
  P.vheavy_list = ar.take<int32_t>(nri);
  P.heavy_tmp = ar.take<int32_t>(nri);
  P.counters = ar.take<int32_t>(4);
  P.products_dev = ar.take<unsigned long long>(1);
  P.row_count = ar.take<int32_t>(nri);
  P.row_offset = ar.take<int64_t>(nri + 1);
  int64_t* tile_offset = ar.take<int64_t>(2);
  int64_t* sums = ar.take<int64_t>(exclusive_scan_sums_len(nri));
  P.queue = ar.take<unsigned long long>(kQueueSlots);
  if (!ar.ok) return noalloc_exhausted();
  BCLX_CK(cudaMemsetAsync(P.counters, 0, 4 * sizeof(int32_t), ctx->stream));
  BCLX_CK(cudaMemsetAsync(P.products_dev, 0, sizeof(unsigned long long), ctx->stream));
  BCLX_CK(cudaMemsetAsync(P.row_count, 0, sizeof(int32_t) * nri, ctx->stream));
  BCLX_CK(cudaMemsetAsync(P.queue + 1, 0, sizeof(unsigned long long), ctx->stream));
  k_classify<false><<<grid_for(ctx, nri, 8, 16), 256, 0, ctx->stream>>>(
      A, B, g, P.light_list, P.heavy_tmp, P.vheavy_list, P.counters, P.products_dev, 8192 + 1, kLightUb, nullptr, nullptr,
      P.queue + 1, queue_grab(ctx, nri, 8, 16, 32, 8));
  note_launch();
  BCLX_CK_LAUNCH();
  int32_t cnts[4];
  BCLX_CK(cudaMemcpyAsync(cnts, P.counters, sizeof(cnts), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  P.n_light = cnts[0];
  P.n_vheavy = cnts[3];
  P.n_heavy = cnts[1] + cnts[3];
  if (P.n_vheavy > 0)
    BCLX_CK(cudaMemcpyAsync(P.heavy_list, P.vheavy_list, sizeof(int32_t) * P.n_vheavy, cudaMemcpyDeviceToDevice,
                            ctx->stream));
  if (cnts[1] > 0)
    BCLX_CK(cudaMemcpyAsync(P.heavy_list + P.n_vheavy, P.heavy_tmp, sizeof(int32_t) * cnts[1],
                            cudaMemcpyDeviceToDevice, ctx->stream));
  P.heavy_bitmaps = ar.take<uint32_t>((size_t)P.n_heavy * P.hbm_words);
  P.heavy_nitems = ar.take<int32_t>(P.n_heavy);
  P.heavy_first = ar.take<int64_t>(P.n_heavy + 1);
  int64_t* sums_h = ar.take<int64_t>(exclusive_scan_sums_len(P.n_heavy));
  if (!ar.ok) return noalloc_exhausted();
  BCLX_TRY(launch_symbolic(ctx, A, B, &P));
  BCLX_TRY(exclusive_scan_i32_buf(ctx, P.row_count, P.row_offset, nri, sums));
  k_tile_ptrs<<<grid_for(ctx, (g.tm + 1) / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(g, P.row_offset, c_row_ptr,
                                                                                 tile_offset, P.counters + 2);
  note_launch();
  BCLX_CK_LAUNCH();
  if (P.n_heavy > 0) {
    k_cut_heavy<false><<<grid_for(ctx, P.n_heavy, 8, 8), 256, 0, ctx->stream>>>(
        g, P.heavy_list, (int)P.n_heavy, P.heavy_bitmaps, P.hbm_words, P.heavy_nitems, nullptr, nullptr, P.vcap);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  BCLX_TRY(exclusive_scan_i32_buf(ctx, P.heavy_nitems, P.heavy_first, P.n_heavy, sums_h));
  int64_t tail[3];
  BCLX_CK(cudaMemcpyAsync(&tail[0], P.row_offset + nri, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaMemcpyAsync(&tail[1], P.heavy_first + P.n_heavy, sizeof(int64_t), cudaMemcpyDeviceToHost,
                          ctx->stream));
  BCLX_CK(cudaMemcpyAsync(&tail[2], P.counters + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  int32_t overflow;
  std::memcpy(&overflow, &tail[2], sizeof(overflow));
  if (overflow) {
    set_last_error("the product has more than 2^31-1 nonzeros");
    return BCLX_ERR_INDEX_OVERFLOW;
  }
  P.nnz = tail[0];
  P.n_heavy_items = tail[1];
  *c_nnz = P.nnz;
  if (P.nnz > c_capacity) {
    set_last_error("output capacity too small: the product has " + std::to_string(P.nnz) +
                   " nonzeros (c_row_ptr and *c_nnz are written; retry with larger c_col_ind/c_vals)");
    return BCLX_ERR_INVALID;
  }
  if (P.n_heavy > 0) {
    P.heavy_items = ar.take<HeavyItem>(P.n_heavy_items);
    if (!ar.ok) return noalloc_exhausted();
    // The B-row table is optional: when what is left of the scratch cannot
    // hold it, heavy items find their column blocks by binary search.
    ScratchArena probe = ar;
    P.tab = probe.take<int32_t>((size_t)g.tk * (g.nfb + 1));
    if (probe.ok) ar = probe;
    else P.tab = nullptr;
    k_cut_heavy<true><<<grid_for(ctx, P.n_heavy, 8, 8), 256, 0, ctx->stream>>>(
        g, P.heavy_list, (int)P.n_heavy, P.heavy_bitmaps, P.hbm_words, nullptr, P.heavy_first, P.heavy_items, P.vcap);
    note_launch();
    BCLX_CK_LAUNCH();
    if (P.tab && g.tk > 0) {
      k_btable<<<grid_for(ctx, g.tk / 32 + 1, 8, 16), 256, 0, ctx->stream>>>(B, g, P.tab);
      note_launch();
      BCLX_CK_LAUNCH();
    }
  }
  if (P.n_light + P.n_heavy_items == 0) return BCLX_OK;
  if (P.dtype == BCLX_F32) return launch_numeric<float>(ctx, A, B, &P, c_col_ind, c_vals, 0, 1);
  return launch_numeric<int32_t>(ctx, A, B, &P, c_col_ind, c_vals, 0, 1);
}

}  // namespace bclx

extern "C" int bclx_spgemm_tile_noalloc(const bclx_csr_t* a, const bclx_csr_t* b, int32_t* c_row_ptr,
                                        int32_t* c_col_ind, void* c_vals, int64_t c_capacity, int64_t* c_nnz,
                                        void* stream) {
  if (!a || !b || !c_row_ptr || !c_nnz || c_capacity < 0) return BCLX_ERR_INVALID;
  *c_nnz = 0;
  if (a->n != b->m || a->m < 0 || a->n < 0 || b->n < 0) {
    set_last_error("shape mismatch: A is m x k and B must be k x n");
    return BCLX_ERR_INVALID;
  }
  if (a->dtype != b->dtype || !value_size(a->dtype)) return BCLX_ERR_DTYPE;
  if (b->n > kMaxCols || a->m > INT32_MAX || a->n > INT32_MAX) {
    set_last_error("tile too large for the no-allocation product (at most 16384 columns)");
    return BCLX_ERR_INVALID;
  }
  if (a->m > 0 && (!a->row_ptr || (a->nnz > 0 && (!a->col_ind || !a->vals)))) return BCLX_ERR_INVALID;
  if (a->n > 0 && (!b->row_ptr || (b->nnz > 0 && (!b->col_ind || !b->vals)))) return BCLX_ERR_INVALID;
  if (c_capacity > 0 && (!c_col_ind || !c_vals)) return BCLX_ERR_INVALID;
  int device = 0;
  BCLX_CK(cudaGetDevice(&device));
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (a->m == 0 || b->n == 0 || a->n == 0) {
    BCLX_CK(cudaMemsetAsync(c_row_ptr, 0, sizeof(int32_t) * (a->m + 1), st));
    return BCLX_OK;
  }
  void* base = nullptr;
  BCLX_TRY(noalloc_base(device, &base));
  int nsm = 148;
  BCLX_CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  Context ctx;
  ctx.device = device;
  ctx.num_sms = nsm;
  ctx.stream = st;
  ctx.pinned = nullptr;
  ScratchArena ar{reinterpret_cast<unsigned char*>(base), kNoAllocScratchBytes};
  return noalloc_product(&ctx, ar, a, b, c_row_ptr, c_col_ind, c_vals, c_capacity, c_nnz);
}

// ---- learned product: orchestration ---------------------------------------------------

namespace bclx {

template <typename VT>
static int learned_numeric(Context* ctx, const SpGridView& A, const SpGridView& B, bclx_spgemm_plan_s* P) {
  if (P->g.tn <= 8192) return launch_numeric_w<VT, 256, true>(ctx, A, B, P, P->temp_col, P->temp_val, 0, (int)P->g.gk);
  return launch_numeric_w<VT, kMaxWords, true>(ctx, A, B, P, P->temp_col, P->temp_val, 0, (int)P->g.gk);
}

template <typename VT>
static int exact_numeric_into(Context* ctx, const SpGridView& A, const SpGridView& B, bclx_spgemm_plan_s* R,
                              int32_t* col, void* val) {
  if (R->g.tn <= 8192) return launch_numeric_w<VT, 256>(ctx, A, B, R, col, val, 0, (int)R->g.gk);
  return launch_numeric_w<VT, kMaxWords>(ctx, A, B, R, col, val, 0, (int)R->g.gk);
}

// Everything up to the final offsets: predict, cut, one numeric pass into
// temp slots, redo the failed rows exactly, row offsets.  nnz in P->nnz.
static int learned_impl(Context* ctx, const SpGridView& A, const SpGridView& B, Geom g, int dtype,
                        const float* params, int32_t* tile_row_ptr, int64_t* tile_offset, bclx_spgemm_plan_s* P) {
  P->learned = true;
  BCLX_TRY(build_stage_map(ctx, A, B, P, g));
  P->g = g;
  P->dtype = dtype;
  // The B-row table depends on B alone: built on the side stream from the
  // start, beside classification and the prediction.
  BCLX_TRY(ensure_side_stream(ctx));
  BCLX_TRY(build_btable(ctx, B, g, P, ctx->side));
  P->hbm_words = (g.tn + 31) / 32;
  const int64_t nri = g.n_row_items;
  BCLX_TRY(scratch_alloc_n(ctx, &P->light_list, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_list, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->vheavy_list, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_tmp, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->counters, 4));
  BCLX_TRY(scratch_alloc_n(ctx, &P->products_dev, 1));
  BCLX_TRY(scratch_alloc_n(ctx, &P->row_count, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->row_offset, nri + 1));
  BCLX_TRY(scratch_alloc_n(ctx, &P->queue, kQueueSlots));
  BCLX_TRY(scratch_alloc_n(ctx, &P->feat, (size_t)nri * 5));
  BCLX_TRY(scratch_alloc_n(ctx, &P->ub, nri));
  BCLX_TRY(scratch_alloc_n(ctx, &P->pred, nri));
  BCLX_CK(cudaMemsetAsync(P->counters, 0, 4 * sizeof(int32_t), ctx->stream));
  BCLX_CK(cudaMemsetAsync(P->products_dev, 0, sizeof(unsigned long long), ctx->stream));
  BCLX_CK(cudaMemsetAsync(P->row_count, 0, sizeof(int32_t) * (nri > 0 ? nri : 1), ctx->stream));
  int32_t* live = nullptr;  // C tiles with stages (rows of the others have no products)
  if (nri > 0) {
    BCLX_CK(cudaMemsetAsync(P->queue + 1, 0, sizeof(unsigned long long), ctx->stream));
    BCLX_TRY(build_live_tiles(ctx, g, &live));
    const int64_t nt = g.gm * g.gn;
    k_classify<true><<<grid_for(ctx, nri, 8, 16), 256, 0, ctx->stream>>>(
        A, B, g, P->light_list, P->heavy_tmp, P->vheavy_list, P->counters, P->products_dev, tuning(ctx, BCLX_TUNE_WIDE_LIGHT) ? INT_MAX : 8192 + 1,
        (int)tuning(ctx, BCLX_TUNE_LIGHT_UB), P->feat, P->ub,
        P->queue + 1, queue_grab(ctx, nri, 8, 16, 32, 8), live, live ? live + nt : nullptr);
    note_launch();
    BCLX_CK_LAUNCH();
    if (live) scratch_free(ctx, live);
  }
  int32_t cnts[4];
  int64_t prod = 0;
  BCLX_CK(cudaMemcpyAsync(cnts, P->counters, sizeof(cnts), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaMemcpyAsync(&prod, P->products_dev, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  P->n_light = cnts[0];
  P->n_vheavy = 0;  // the learned cut treats every heavy row alike
  P->n_heavy = cnts[1] + cnts[3];
  P->products = prod;
  if (cnts[3] > 0)
    BCLX_CK(cudaMemcpyAsync(P->heavy_list, P->vheavy_list, sizeof(int32_t) * cnts[3], cudaMemcpyDeviceToDevice,
                            ctx->stream));
  if (cnts[1] > 0)
    BCLX_CK(cudaMemcpyAsync(P->heavy_list + cnts[3], P->heavy_tmp, sizeof(int32_t) * cnts[1],
                            cudaMemcpyDeviceToDevice, ctx->stream));
  if (params && P->n_heavy > 0) {
    // predictions are needed for the heavy rows only
    float* hx = nullptr;
    BCLX_TRY(scratch_alloc_n(ctx, &hx, (size_t)P->n_heavy * 6));
    k_gather_features<<<grid_for(ctx, P->n_heavy / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(
        P->heavy_list, (int)P->n_heavy, P->feat, hx);
    note_launch();
    int rc = bclx_mlp_predict(reinterpret_cast<bclx_context_t>(ctx), hx, P->n_heavy, params, hx + 5 * P->n_heavy);
    if (rc == BCLX_OK) {
      k_scatter_pred<<<grid_for(ctx, P->n_heavy / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(
          P->heavy_list, (int)P->n_heavy, hx + 5 * P->n_heavy, P->pred);
      note_launch();
    }
    scratch_free(ctx, hx);
    BCLX_TRY(rc);
    BCLX_CK_LAUNCH();
  }

  // heavy rows: predicted cut; light rows: slots of their product count
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_nitems, P->n_heavy));
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_first, P->n_heavy + 1));
  BCLX_TRY(scratch_alloc_n(ctx, &P->light_ub, P->n_light));
  BCLX_TRY(scratch_alloc_n(ctx, &P->light_slot, P->n_light + 1));
  const unsigned hb = grid_for(ctx, P->n_heavy / 32 + 1, 8, 8);
  // the side stream (B-row table) joins before the table is read
  BCLX_CK(cudaEventRecord(ctx->join_ev, ctx->side));
  BCLX_CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0));
  if (P->n_heavy > 0) {
    BCLX_TRY(scratch_alloc_n(ctx, &P->block_ub, (size_t)P->n_heavy * g.nfb));
    k_heavy_block_ub<<<grid_for(ctx, P->n_heavy, 8, 16), 256, 0, ctx->stream>>>(A, B, g, P->heavy_list,
                                                                               (int)P->n_heavy, P->tab, P->block_ub);
    note_launch();
    BCLX_CK_LAUNCH();
    k_learned_cut<false><<<hb, 256, 0, ctx->stream>>>(g, P->heavy_list, (int)P->n_heavy, params ? P->pred : nullptr,
                                                      P->ub, P->block_ub, P->heavy_nitems, nullptr, nullptr, nullptr,
                                                      (float)tuning(ctx, BCLX_TUNE_LEARN_TARGET));
    note_launch();
    BCLX_CK_LAUNCH();
  }
  BCLX_TRY(exclusive_scan_i32(ctx, P->heavy_nitems, P->heavy_first, P->n_heavy));
  if (P->n_light > 0) {
    k_gather_ub<<<grid_for(ctx, P->n_light / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(P->light_list, (int)P->n_light,
                                                                                    P->ub, P->light_ub);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  BCLX_TRY(exclusive_scan_i32(ctx, P->light_ub, P->light_slot, P->n_light));
  int64_t tails[2];
  BCLX_CK(cudaMemcpyAsync(&tails[0], P->heavy_first + P->n_heavy, sizeof(int64_t), cudaMemcpyDeviceToHost,
                          ctx->stream));
  BCLX_CK(cudaMemcpyAsync(&tails[1], P->light_slot + P->n_light, sizeof(int64_t), cudaMemcpyDeviceToHost,
                          ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  P->n_heavy_items = tails[0];
  const int64_t light_total = tails[1];
  BCLX_TRY(scratch_alloc_n(ctx, &P->heavy_items, P->n_heavy_items));
  BCLX_TRY(scratch_alloc_n(ctx, &P->item_cap, P->n_heavy_items));
  BCLX_TRY(scratch_alloc_n(ctx, &P->item_off, P->n_heavy_items + 1));
  if (P->n_heavy > 0) {
    k_learned_cut<true><<<hb, 256, 0, ctx->stream>>>(g, P->heavy_list, (int)P->n_heavy, params ? P->pred : nullptr,
                                                     P->ub, P->block_ub, nullptr, P->heavy_first, P->heavy_items,
                                                     P->item_cap, (float)tuning(ctx, BCLX_TUNE_LEARN_TARGET));
    note_launch();
    BCLX_CK_LAUNCH();
  }
  // heavy items' temp slots: their sizes, in item order
  BCLX_TRY(exclusive_scan_i32(ctx, P->item_cap, P->item_off, P->n_heavy_items));
  int64_t heavy_total = 0;
  BCLX_CK(cudaMemcpyAsync(&heavy_total, P->item_off + P->n_heavy_items, sizeof(int64_t), cudaMemcpyDeviceToHost,
                          ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));

  // one numeric pass into temp slots
  P->heavy_slot_base = light_total;  // heavy item slots follow the light rows' slots
  P->temp_entries = light_total + heavy_total;
  BCLX_TRY(scratch_alloc_n(ctx, &P->temp_col, P->temp_entries));
  BCLX_TRY(scratch_alloc(ctx, &P->temp_val, 4 * (size_t)(P->temp_entries > 0 ? P->temp_entries : 1)));
  BCLX_TRY(scratch_alloc_n(ctx, &P->item_count, P->n_heavy_items));
  BCLX_TRY(scratch_alloc_n(ctx, &P->row_failed, P->n_heavy));
  BCLX_TRY(scratch_alloc_n(ctx, &P->failed_list, P->n_heavy));
  BCLX_CK(cudaMemsetAsync(P->item_count, 0, sizeof(int32_t) * (P->n_heavy_items > 0 ? P->n_heavy_items : 1),
                          ctx->stream));
  BCLX_CK(cudaMemsetAsync(P->row_failed, 0, sizeof(int32_t) * (P->n_heavy > 0 ? P->n_heavy : 1), ctx->stream));
  if (P->n_light + P->n_heavy_items > 0) {
    if (dtype == BCLX_F32) BCLX_TRY(learned_numeric<float>(ctx, A, B, P));
    else BCLX_TRY(learned_numeric<int32_t>(ctx, A, B, P));
  }
  BCLX_CK(cudaMemsetAsync(P->counters + 2, 0, sizeof(int32_t), ctx->stream));
  if (P->n_heavy > 0) {
    k_collect_failed<<<hb, 256, 0, ctx->stream>>>(P->heavy_list, (int)P->n_heavy, P->row_failed, P->failed_list,
                                                  P->counters + 2);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  int32_t nf = 0;
  BCLX_CK(cudaMemcpyAsync(&nf, P->counters + 2, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  P->n_failed = nf;

  // the exact two-phase path for the failed rows (symbolic, cut, numeric)
  if (nf > 0) {
    auto* R = new bclx_spgemm_plan_s();
    P->redo = R;
    R->ctx = ctx;
    R->g = g;
    R->dtype = dtype;
    R->hbm_words = P->hbm_words;
    R->grab = P->grab;
    R->blocks_per_sm = P->blocks_per_sm;
    R->long_seg = P->long_seg;
    R->heavy_list = P->failed_list;  // borrowed
    R->light_list = P->light_list;   // borrowed (unused: no light rows)
    R->n_light = 0;
    R->n_vheavy = 0;
    R->n_heavy = nf;
    BCLX_TRY(scratch_alloc_n(ctx, &R->row_count, nri));
    BCLX_TRY(scratch_alloc_n(ctx, &R->heavy_bitmaps, (size_t)nf * R->hbm_words));
    BCLX_TRY(scratch_alloc_n(ctx, &R->heavy_nitems, nf));
    BCLX_TRY(scratch_alloc_n(ctx, &R->heavy_first, nf + 1));
    BCLX_TRY(scratch_alloc_n(ctx, &R->queue, kQueueSlots));
    BCLX_TRY(scratch_alloc_n(ctx, &P->redo_off, nri + 1));
    BCLX_CK(cudaMemsetAsync(R->row_count, 0, sizeof(int32_t) * nri, ctx->stream));
    BCLX_TRY(launch_symbolic(ctx, A, B, R));
    BCLX_TRY(exclusive_scan_i32(ctx, R->row_count, P->redo_off, nri));
    R->row_offset = P->redo_off;  // borrowed
    const unsigned rb = grid_for(ctx, nf, 8, 8);
    k_cut_heavy<false><<<rb, 256, 0, ctx->stream>>>(g, R->heavy_list, nf, R->heavy_bitmaps, R->hbm_words,
                                                    R->heavy_nitems, nullptr, nullptr, R->vcap);
    note_launch();
    BCLX_CK_LAUNCH();
    BCLX_TRY(exclusive_scan_i32(ctx, R->heavy_nitems, R->heavy_first, nf));
    int64_t rt[2];
    BCLX_CK(cudaMemcpyAsync(&rt[0], R->heavy_first + nf, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    BCLX_CK(cudaMemcpyAsync(&rt[1], P->redo_off + nri, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
    BCLX_CK(cudaStreamSynchronize(ctx->stream));
    R->n_heavy_items = rt[0];
    BCLX_TRY(scratch_alloc_n(ctx, &R->heavy_items, R->n_heavy_items));
    k_cut_heavy<true><<<rb, 256, 0, ctx->stream>>>(g, R->heavy_list, nf, R->heavy_bitmaps, R->hbm_words, nullptr,
                                                   R->heavy_first, R->heavy_items, R->vcap);
    note_launch();
    BCLX_CK_LAUNCH();
    R->tab = P->tab;  // borrowed
    BCLX_TRY(scratch_alloc_n(ctx, &P->redo_col, rt[1]));
    BCLX_TRY(scratch_alloc(ctx, &P->redo_val, 4 * (size_t)(rt[1] > 0 ? rt[1] : 1)));
    if (R->n_heavy_items > 0) {
      if (dtype == BCLX_F32) BCLX_TRY(exact_numeric_into<float>(ctx, A, B, R, P->redo_col, P->redo_val));
      else BCLX_TRY(exact_numeric_into<int32_t>(ctx, A, B, R, P->redo_col, P->redo_val));
    }
    k_take_counts<<<rb, 256, 0, ctx->stream>>>(P->failed_list, nf, R->row_count, P->row_count);
    note_launch();
    BCLX_CK_LAUNCH();
  }

  // final row offsets and the C tile pointers (counters[3] becomes the overflow flag)
  BCLX_TRY(exclusive_scan_i32(ctx, P->row_count, P->row_offset, nri));
  BCLX_CK(cudaMemsetAsync(P->counters + 3, 0, sizeof(int32_t), ctx->stream));
  const int64_t ntiles = g.gm * g.gn;
  k_tile_ptrs<<<grid_for(ctx, ntiles * (g.tm + 1) / 32 + 1, 8, 8), 256, 0, ctx->stream>>>(
      g, P->row_offset, tile_row_ptr, tile_offset, P->counters + 3);
  note_launch();
  BCLX_CK_LAUNCH();
  BCLX_TRY(scratch_alloc_n(ctx, &P->item_pos, P->n_heavy_items + 1));
  BCLX_TRY(exclusive_scan_i32(ctx, P->item_count, P->item_pos, P->n_heavy_items));
  int64_t nnz = 0;
  int32_t ovf = 0;
  BCLX_CK(cudaMemcpyAsync(&nnz, P->row_offset + nri, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaMemcpyAsync(&ovf, P->counters + 3, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  if (ovf) {
    set_last_error("a C tile has more than 2^31-1 nonzeros; use a finer tile grid");
    return BCLX_ERR_INDEX_OVERFLOW;
  }
  P->nnz = nnz;
  return BCLX_OK;
}

template <typename VT>
static int learned_finish_impl(Context* ctx, bclx_spgemm_plan_s* P, int32_t* out_col, void* out_val) {
  const int64_t units = P->n_light + P->n_heavy_items + P->n_failed;
  if (units == 0) return BCLX_OK;
  k_compact<VT><<<grid_for(ctx, units, 8, 8), 256, 0, ctx->stream>>>(
      P->g, P->light_list, (int)P->n_light, P->light_slot, P->heavy_list, P->heavy_items, P->n_heavy_items,
      P->heavy_first, P->item_count, P->item_pos, P->row_failed, P->failed_list, (int)P->n_failed,
      P->heavy_slot_base, P->item_off, P->redo_off,
      P->row_count, P->row_offset, P->temp_col, reinterpret_cast<const VT*>(P->temp_val), P->redo_col,
      reinterpret_cast<const VT*>(P->redo_val), out_col, reinterpret_cast<VT*>(out_val));
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

}  // namespace bclx

extern "C" {

static int learned_entry(bclx_context_t c, const bclx_spgrid_t* a, const bclx_spgrid_t* b, bclx_spgrid_out_t* out,
                         const int64_t* tile_rows, const int64_t* tile_cols, const float* mlp_params,
                         bclx_spgemm_plan_t* plan, int64_t* nnz) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !plan || !nnz) return BCLX_ERR_INVALID;
  *plan = nullptr;
  BCLX_TRY(check_grids(a, b, out));
  if (!out->tile_row_ptr || !out->tile_offset) return BCLX_ERR_INVALID;
  if (tile_rows && !maps_ok(out, tile_rows, tile_cols)) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  auto* P = new bclx_spgemm_plan_s();
  P->ctx = ctx;
  Geom g = make_geom(out, a->grid_n, a->tile_n);
  int rc = tile_rows ? attach_maps(ctx, P, g, out, tile_rows, tile_cols) : BCLX_OK;
  if (rc == BCLX_OK)
    rc = learned_impl(ctx, make_view(*a), make_view(*b), g, a->dtype, mlp_params, out->tile_row_ptr,
                      out->tile_offset, P);
  if (rc != BCLX_OK) {
    P->release();
    delete P;
    return rc;
  }
  *nnz = P->nnz;
  *plan = P;
  return BCLX_OK;
}

int bclx_spgemm_learned_run(bclx_context_t c, const bclx_spgrid_t* a, const bclx_spgrid_t* b, bclx_spgrid_out_t* out,
                            const float* mlp_params, bclx_spgemm_plan_t* plan, int64_t* nnz) {
  return learned_entry(c, a, b, out, nullptr, nullptr, mlp_params, plan, nnz);
}

int bclx_spgemm_learned_run_sub(bclx_context_t c, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                                bclx_spgrid_out_t* out, const int64_t* tile_rows, const int64_t* tile_cols,
                                const float* mlp_params, bclx_spgemm_plan_t* plan, int64_t* nnz) {
  if (!tile_rows || !tile_cols) return BCLX_ERR_INVALID;
  return learned_entry(c, a, b, out, tile_rows, tile_cols, mlp_params, plan, nnz);
}

int bclx_spgemm_learned_finish(bclx_context_t c, bclx_spgemm_plan_t P, bclx_spgrid_out_t* out) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !P || !out || !P->learned) return BCLX_ERR_INVALID;
  if (P->nnz > 0 && (!out->col_ind || !out->vals)) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  if (P->dtype == BCLX_F32) return learned_finish_impl<float>(ctx, P, out->col_ind, out->vals);
  return learned_finish_impl<int32_t>(ctx, P, out->col_ind, out->vals);
}

int bclx_spgemm_learned_stats(bclx_spgemm_plan_t P, int64_t* out6) {
  if (!P || !out6 || !P->learned) return BCLX_ERR_INVALID;
  out6[0] = P->n_heavy;
  out6[1] = P->n_heavy_items;
  out6[2] = P->n_failed;
  out6[3] = P->temp_entries;
  out6[4] = P->nnz;
  out6[5] = P->redo ? P->redo->n_heavy_items : 0;
  return BCLX_OK;
}

int bclx_spgemm_row_features(bclx_context_t c, const bclx_spgrid_t* a, const bclx_spgrid_t* b,
                             const bclx_spgrid_out_t* out, float* X, int32_t* ub) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !X || !ub) return BCLX_ERR_INVALID;
  BCLX_TRY(check_grids(a, b, out));
  BCLX_CK(cudaSetDevice(ctx->device));
  const Geom g = make_geom(out, a->grid_n, a->tile_n);
  const int64_t nri = g.n_row_items;
  if (nri == 0) return BCLX_OK;
  int32_t* lists = nullptr;
  int32_t* cnt = nullptr;
  unsigned long long* prod = nullptr;
  BCLX_TRY(scratch_alloc_n(ctx, &lists, 3 * (size_t)nri));
  int rc = scratch_alloc_n(ctx, &cnt, 4);
  if (rc == BCLX_OK) rc = scratch_alloc_n(ctx, &prod, 2);  // products, row counter
  if (rc == BCLX_OK) {
    cudaMemsetAsync(cnt, 0, 4 * sizeof(int32_t), ctx->stream);
    cudaMemsetAsync(prod, 0, 2 * sizeof(unsigned long long), ctx->stream);
    k_classify<true><<<grid_for(ctx, nri, 8, 16), 256, 0, ctx->stream>>>(
        make_view(*a), make_view(*b), g, lists, lists + nri, lists + 2 * nri, cnt, prod, 8192 + 1, kLightUb, X, ub, prod + 1,
        queue_grab(ctx, nri, 8, 16, 32, 8));
    note_launch();
    if (cudaGetLastError() != cudaSuccess) rc = BCLX_ERR_CUDA;
  }
  scratch_free(ctx, lists);
  scratch_free(ctx, cnt);
  scratch_free(ctx, prod);
  return rc;
}

int bclx_spgemm_plan_row_counts(bclx_spgemm_plan_t P, int32_t* counts) {
  if (!P || !counts || !P->row_count) return BCLX_ERR_INVALID;
  Context* ctx = P->ctx;
  BCLX_CK(cudaMemcpyAsync(counts, P->row_count, sizeof(int32_t) * P->g.n_row_items, cudaMemcpyDeviceToDevice,
                          ctx->stream));
  return BCLX_OK;
}

}  // extern "C"
