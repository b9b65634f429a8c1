// Sparse x dense: C += A * B, for one tile (spmm_wrapper,
// bcl/containers/algorithms/spgemm.hpp:80-96 and 140-149) and for the whole
// tile loop of BCL::gemm(SPMatrix, DMatrix, DMatrix&) (spgemm.hpp:153-179) in
// one launch.
//
// Layout: one warp per (group of 1, 2 or 4 rows of one C tile, column panel
// of 32 16-byte vectors: 128 FP32 / 256 BF16 columns); lane l owns one
// vector.  The group's A entries are flattened over rows and stages and put
// 32 at a time into a per-warp shared-memory table (B-row address, value,
// row); every lane then issues its 16-byte loads of the B rows (the warp
// reads whole 512-byte row segments), UNROLL entries' loads in flight before
// their multiply-adds are applied.  Rows with thousands of entries run in
// k_spmm_long beside it.
//
// Order: per output element the multiply-adds run in stored A-row order, and
// over the C tile's stages k = (k_ + i + j) mod G in that order, starting
// from the C value already stored (beta = 1, in place) — the reference's
// sequence, so FP32 results are bit-identical.  BF16 storage keeps the chain
// in FP32 registers and rounds each C element once when it is stored.
#include "common.cuh"

#include <algorithm>
#include <cstdlib>
#include <vector>

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

constexpr int kSpmmMaxRows = 4;  // rows of one C tile a warp walks together
constexpr int kARing = 4;        // A-entry staging slots (chunks of 32 entries) per warp
constexpr int kTabBufs = 3;      // entry-table buffers per warp: applied, next, being built

// Per-warp shared memory of the walk:
//  * entry tables: per chunk of 32 entries, (B-row address, A value, row) of
//    each entry, read back with broadcast 16-byte loads;
//  * A staging ring: the (column, value) pair of each entry, copied by
//    cp.async kARing - 1 chunks ahead, with the entry's stage lane;
//  * C staging: the C row slices the item updates (one 16-byte vector per
//    lane and row), copied by cp.async while the A and B loads are in flight.
__shared__ uint4 spmm_tables[kSpmmWarps * kTabBufs * 32];
__shared__ uint2 spmm_aring[kSpmmWarps * kARing * 32];
__shared__ uint8_t spmm_asrc[kSpmmWarps * kARing * 32];
__shared__ uint4 spmm_cstage[kSpmmWarps * kSpmmMaxRows * 32];

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// Copies without a compiler memory barrier, for the pipelined loops:
// there every earlier access to the target shared memory is ordered before the
// copy by a __syncwarp, and every later one after it by a wait (which is a
// barrier), so the loads around the copies may be scheduled freely.
__device__ __forceinline__ void cp_async16_nb(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

__device__ __forceinline__ void cp_async4_nb(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }

template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// One stage of one row of C tile (ti, tj): for stage slot kk of the
// reference's rotated order k = (k_ + ti + tj) mod gk, the A-row segment of
// row r in tile (ti, k) and the B tile (k, tj).  Empty when !valid.
template <typename ST>
struct StageLane {
  int32_t alen;
  const int32_t* acol;
  const float* aval;
  const ST* bt;
};

template <typename ST, bool SUB>
__device__ __forceinline__ StageLane<ST> stage_lane(const SpGridView& A, const DGridView& B, int64_t ti, int64_t tj,
                                                    int64_t r, int64_t kk, bool valid) {
  StageLane<ST> s{0, nullptr, nullptr, nullptr};
  const int64_t gk = A.gn;
  if (valid && kk < gk) {
    const int64_t rot = SUB ? (int64_t)__ldg(B.rot_i + ti) + __ldg(B.rot_j + tj) : ti + tj;
    const int64_t k = B.natural_order ? kk : (kk + rot) % gk;
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

// One warp per (R consecutive rows of C tile (ti, tj) from r0, panel of 32
// 16-byte vectors from column c0).  The A entries of the rows' stages are
// flattened (row by row, each row's stages in rotated order) and taken in
// chunks of 32, one entry per lane, through a software pipeline:
//   * chunk c + kARing + 1: each lane finds its entry's stage and copies the
//     entry's (column, value) into the warp's staging ring by cp.async;
//   * chunk c + 2: each lane turns its staged entry into a table entry
//     (B-row address, value, row) and asks L2 for that B-row slice;
//   * chunk c: the warp reads the table UNROLL entries at a time, so that
//     many B-row loads (raw 16-byte vectors) are in flight before their
//     multiply-adds are applied in entry order.
// No load result is waited for before it is used, so the A loads of later
// chunks never stall the current one.  A row's chain starts from its C
// value, staged in shared memory by cp.async once the row is known to have
// entries; rows without entries are not touched.  R > 1 needs R * gk <= 32
// (one lane per (row, stage)); R == 1 takes the stages 32 at a time.
// GROUP = false compiles the one-row walk alone (R == 1, no row changes to
// test for inside the unrolled loop).  `skip` (or null): rows flagged there
// are left to another kernel.  `vec`: every B and C row slice of this tile
// pair is 16-byte aligned; otherwise element-wise access.
template <typename ST, bool GROUP, bool SUB, int UNROLL = kSpmmUnroll>
__device__ __forceinline__ void spmm_rows(const SpGridView& A, const DGridView& B, const DGridView& C, int64_t ti,
                                          int64_t tj, int64_t r0, int R, int c0, int W, bool vec,
                                          const uint8_t* __restrict__ skip) {
  if (!GROUP) R = 1;
  using V = Vec<ST>;
  constexpr int VN = V::N;
  const int lane = lane_id();
  const int64_t nrows = min((int64_t)R, C.rows_of(ti) - r0);
  ST* __restrict__ crow0 = reinterpret_cast<ST*>(C.tile(ti, tj)) + r0 * C.ld;
  const int col = c0 + lane * VN;
  const bool own = col < W;
  const int bcol = own ? col : 0;  // lanes past the tile edge load column 0 (in bounds) and store nothing
  const int wib = threadIdx.x >> 5;
  uint4* tb = spmm_tables + wib * (kTabBufs * 32);
  uint2* ar = spmm_aring + wib * (kARing * 32);
  uint8_t* asrc = spmm_asrc + wib * (kARing * 32);
  uint4* cs = spmm_cstage + wib * (kSpmmMaxRows * 32);
  // bytes of this warp's panel in one B row
  const int pbytes = min(32 * VN, W - c0) * (int)sizeof(ST);
  const int gk = (int)A.gn;
  float acc[VN];
  int cur = -1;  // row whose chain is in acc
  bool staged = false;
  auto flush = [&]() {
    if (cur < 0 || !own) return;
    ST* p = crow0 + cur * C.ld;
    if (vec) {
      V::store(p + col, acc);
    } else {
#pragma unroll
      for (int x = 0; x < VN; x++)
        if (col + x < W) p[col + x] = V::from_f(acc[x]);
    }
  };
  auto enter = [&](int q) {
    flush();
    cur = q;
    if (!own) return;
    if (vec) {
      cp_async_wait_all();
      V::unpack_raw(cs[q * 32 + lane], acc);
    } else {
      const ST* p = crow0 + q * C.ld;
#pragma unroll
      for (int x = 0; x < VN; x++) acc[x] = (col + x < W) ? V::to_f(p[col + x]) : 0.f;
    }
  };
  for (int64_t g0 = 0; g0 < gk; g0 += 32) {
    const int ql = GROUP ? lane / gk : 0;
    const int64_t kk = GROUP ? lane - ql * gk : g0 + lane;
    bool valid = ql < nrows;
    if (valid && skip) valid = skip[ti * C.tm + r0 + ql] == 0;
    const StageLane<ST> sl = stage_lane<ST, SUB>(A, B, ti, tj, r0 + ql, kk, valid);
    const int32_t aincl = warp_inclusive_scan(sl.alen);
    const int32_t atot = __shfl_sync(kFull, aincl, 31);
    if (atot == 0) continue;
    const int32_t aexcl = aincl - sl.alen;
    // stage the C slices of the rows that have entries
    if (!GROUP) {
      if (vec && !staged) {
        if (own) cp_async16(cs + lane, crow0 + col);
        staged = true;
      }
    } else {
      for (int q = 0; q < R; q++) {
        const int32_t hi = __shfl_sync(kFull, aincl, q * gk + gk - 1);
        const int32_t lo = __shfl_sync(kFull, aexcl, q * gk);
        if (vec && own && hi > lo) cp_async16(cs + q * 32 + lane, crow0 + q * C.ld + col);
      }
    }
    const int32_t nch = (atot + 31) >> 5;
    // chunk x: each lane's entry x*32 + lane into ring slot x % kARing (one
    // commit group per chunk, empty past the end)
    auto issue_a = [&](int32_t x) {
      if (x < nch) {
        const int32_t e = x * 32 + lane;
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
        const int slot = (x % kARing) * 32 + lane;
        asrc[slot] = (uint8_t)src;
        if (e < atot) {
          cp_async4_nb(&ar[slot].x, sacol + off);
          cp_async4_nb(&ar[slot].y, saval + off);
        }
      }
      cp_async_commit();
    };
    // chunk x (staged): table entries and L2 requests for the B-row slices.
    // Entries past the end point at the last entry's B row with value 0 (an
    // in-bounds load whose product is never applied).
    auto build = [&](int32_t x) {
      if (x >= nch) return;
      const int slot = (x % kARing) * 32 + lane;
      const int src = asrc[slot];
      const ST* sbt = reinterpret_cast<const ST*>(__shfl_sync(kFull, reinterpret_cast<unsigned long long>(sl.bt), src));
      const int32_t e = x * 32 + lane;
      float v = 0.f;
      const ST* brow = sbt;
      if (e < atot) {
        const uint2 a = ar[slot];
        v = __uint_as_float(a.y);
        brow = sbt + (int64_t)(int32_t)a.x * B.ld;
      }
      const ST* last = reinterpret_cast<const ST*>(
          __shfl_sync(kFull, reinterpret_cast<unsigned long long>(brow), (atot - 1) & 31));
      if (e >= atot) brow = last;
      const uint64_t pa = reinterpret_cast<uint64_t>(brow);
      tb[(x % kTabBufs) * 32 + lane] =
          make_uint4((uint32_t)pa, (uint32_t)(pa >> 32), __float_as_uint(v), GROUP ? (uint32_t)(src / gk) : 0u);
      l2_prefetch_slice(vec && e < atot ? brow + c0 : nullptr, pbytes);
    };
    // pipeline fill: chunks 0 .. kARing-1 staged, 0 and 1 built, kARing staged
    for (int x = 0; x < kARing; x++) issue_a(x);
    cp_async_wait_group<kARing - 2>();
    build(0);
    build(1);
    issue_a(kARing);
    __syncwarp();
    if (!GROUP && cur < 0) enter(0);
    for (int32_t c = 0; c < nch; c++) {
      issue_a(c + kARing + 1);
      cp_async_wait_group<kARing - 1>();
      build(c + 2);
      const int ne = min(32, atot - c * 32);
      const uint4* t = tb + (c % kTabBufs) * 32;
      if (vec) {
        for (int u0 = 0; u0 < ne; u0 += UNROLL) {
          uint4 ent[UNROLL];
          uint4 raw[UNROLL];
#pragma unroll
          for (int u = 0; u < UNROLL; u++) ent[u] = t[(u0 + u) & 31];
#pragma unroll
          for (int u = 0; u < UNROLL; u++) {
            const ST* rp = reinterpret_cast<const ST*>((uint64_t)ent[u].x | ((uint64_t)ent[u].y << 32));
            raw[u] = __ldg(reinterpret_cast<const uint4*>(rp + bcol));
          }
          auto apply = [&](int u) {
            if (GROUP && (int)ent[u].w != cur) enter((int)ent[u].w);
            float b[VN];
            V::unpack_raw(raw[u], b);
            const float vs = __uint_as_float(ent[u].z);
#pragma unroll
            for (int x = 0; x < VN; x++) acc[x] = __fmaf_rn(vs, b[x], acc[x]);
          };
          if (u0 + UNROLL <= ne) {  // whole group: no test between the loads and their use
#pragma unroll
            for (int u = 0; u < UNROLL; u++) apply(u);
          } else {
#pragma unroll
            for (int u = 0; u < UNROLL; u++)
              if (u0 + u < ne) apply(u);
          }
        }
      } else {
        for (int u = 0; u < ne; u++) {
          const uint4 en = t[u];
          if (GROUP && (int)en.w != cur) enter((int)en.w);
          const ST* rp = reinterpret_cast<const ST*>((uint64_t)en.x | ((uint64_t)en.y << 32));
          const float vs = __uint_as_float(en.z);
#pragma unroll
          for (int x = 0; x < VN; x++)
            if (col + x < W) acc[x] = __fmaf_rn(vs, V::to_f(rp[col + x]), acc[x]);
        }
      }
      __syncwarp();
    }
  }
  flush();
}

// Warp items come from a device counter (one grab per item, the next grab in
// flight while the current item runs), so warps that draw short rows take
// more of them: the cost of a (row group, panel) item varies by orders of
// magnitude on power-law matrices.
template <typename ST, bool GROUP, bool SUB>
__global__ void __launch_bounds__(kSpmmWarps * 32, 4)
    k_spmm(SpGridView A, DGridView B, DGridView C, int64_t n_items, int npanels, int R, int64_t ngroups,
           int row_align_ok, int panel_major, const uint8_t* __restrict__ long_flag,
           unsigned long long* __restrict__ next_item) {
  constexpr int PW = 32 * Vec<ST>::N;
  const int lane = lane_id();
  unsigned long long it = 0;
  if (lane == 0) it = atomicAdd(next_item, 1ULL);
  it = __shfl_sync(kFull, it, 0);
  while (it < (unsigned long long)n_items) {
    unsigned long long nx = 0;
    if (lane == 0) nx = atomicAdd(next_item, 1ULL);
    const int64_t item = (int64_t)it;
    int64_t rg;
    int panel;
    if (panel_major) {  // all row groups of panel 0, then of panel 1, ...
      const int64_t n_rg = n_items / npanels;
      panel = (int)(item / n_rg);
      rg = item - panel * n_rg;
    } else {  // the panels of a row group one after another
      rg = item / npanels;
      panel = (int)(item - rg * npanels);
    }
    const int64_t t = rg / ngroups;
    const int64_t r0 = (rg - t * ngroups) * R;
    const int64_t ti = t / C.gn, tj = t - ti * C.gn;
    const int W = (int)C.cols_of(tj);
    const int c0 = panel * PW;
    if (r0 < C.rows_of(ti) && c0 < W) {
      const bool vec = row_align_ok && (W % Vec<ST>::N) == 0 && tiles_aligned(B, C, ti, tj);
      // rows flagged long are k_spmm_long's (it takes the aligned ones)
      spmm_rows<ST, GROUP, SUB>(A, B, C, ti, tj, r0, R, c0, W, vec, vec ? long_flag : nullptr);
    }
    it = __shfl_sync(kFull, nx, 0);
  }
  // launched as k_spmm_long's programmatic dependent: finish only after it
  // (a normal launch returns here at once)
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
}

// ---- long rows ----------------------------------------------------------------
//
// A row with thousands of entries is one chain of multiply-adds per output
// element (the reference's order): it cannot be split, only fed faster.  Such
// rows are found first (k_spmm_find_long), skipped by k_spmm and run by
// k_spmm_long on the context's side stream at the same time, one warp per
// (row, C tile column, panel), with the B-row slices themselves copied into
// shared memory by cp.async two chunks (64 entries) ahead: the loads in
// flight cost no registers, and a chunk's multiply-adds read shared memory.
// Rows of 8 times the long-row threshold or more are listed first, so that
// the longest chains start first.

constexpr int kLongWarps = 4;
constexpr int kLongBSlots = 3;  // chunks of B slices per warp: applied, in flight, being issued
constexpr int kLongTSlots = 3;  // chunks of table entries per warp (with the B slices)
constexpr int kLongASlots = 6;  // chunks of staged A entries per warp
// A row is long from BCLX_TUNE_SPMM_LONG_ROW entries over all stages (512
// for FP32, 1024 for BF16 by default).
constexpr int64_t kSpmmLongMinRows = 65536;  // smaller products do not use the long-row path

struct LongSmem {
  uint4 b[kLongBSlots][32][32];  // [chunk slot][entry][lane]: each lane's 16 bytes of the entry's B row
  uint4 tab[kLongTSlots][32];    // [chunk slot][entry]: B-row address, A value
  uint2 a[kLongASlots][32];      // [chunk slot][entry]: staged A (column, value)
  uint8_t src[kLongASlots][32];  // the entry's stage lane
};

// Thread per A row (ti, r): entries over all stages; rows with at least
// long_row are flagged and listed: very long rows from list[0] up
// (count[0]), the others from list[rows-1] down (count[1]).
__global__ void k_spmm_find_long(SpGridView A, int long_row, int very_long_row, uint8_t* __restrict__ flag,
                                 int64_t* __restrict__ list, int32_t* __restrict__ count) {
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
    if (lng) {
      if (tot >= very_long_row)
        list[atomicAdd(count, 1)] = x;
      else
        list[rows - 1 - atomicAdd(count + 1, 1)] = x;
    }
  }
}

// One long row r of C tile (ti, tj), panel from column c0 (16-byte aligned
// access: the caller checked).  Pipeline at chunk c (32 entries, one per
// lane when staged or built):
//   * A of chunk c + 6 staged (cp.async, 8 bytes per lane);
//   * chunk c + 2 built: each lane's entry -> table (B-row address, value),
//     then every lane copies its 16 bytes of each of the chunk's 32 B rows
//     into the chunk's B slot (cp.async);
//   * chunk c applied: the multiply-adds in entry order from shared memory.
// One commit group per chunk step holds A(c+6) and B(c+2); B(c) is in the
// group two steps back.  The stages are at most 32 (one lane each).
template <typename ST, bool SUB>
__device__ __forceinline__ void spmm_long_row(LongSmem& S, const SpGridView& A, const DGridView& B,
                                              const DGridView& C, int64_t ti, int64_t tj, int64_t r, int c0, int W) {
  using V = Vec<ST>;
  constexpr int VN = V::N;
  const int lane = lane_id();
  ST* __restrict__ crow = reinterpret_cast<ST*>(C.tile(ti, tj)) + r * C.ld;
  const int col = c0 + lane * VN;
  const bool own = col < W;
  float acc[VN];
  if (own) V::load_c(crow + col, acc);
  const StageLane<ST> sl = stage_lane<ST, SUB>(A, B, ti, tj, r, lane, true);
  const int32_t aincl = warp_inclusive_scan(sl.alen);
  const int32_t atot = __shfl_sync(kFull, aincl, 31);
  const int32_t aexcl = aincl - sl.alen;
  const int32_t nch = (atot + 31) >> 5;
  auto issue_a = [&](int32_t x) {
    if (x >= nch) return;
    const int32_t e = x * 32 + lane;
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
    const int slot = x % kLongASlots;
    S.src[slot][lane] = (uint8_t)src;
    if (e < atot) {
      cp_async4_nb(&S.a[slot][lane].x, sacol + off);
      cp_async4_nb(&S.a[slot][lane].y, saval + off);
    }
  };
  auto build = [&](int32_t x) {  // A(x) has landed
    if (x >= nch) return;
    const int slot = x % kLongASlots;
    const int src = S.src[slot][lane];
    const ST* sbt = reinterpret_cast<const ST*>(__shfl_sync(kFull, reinterpret_cast<unsigned long long>(sl.bt), src));
    const int32_t e = x * 32 + lane;
    if (e < atot) {
      const uint2 a = S.a[slot][lane];
      const uint64_t pa = reinterpret_cast<uint64_t>(sbt + (int64_t)(int32_t)a.x * B.ld);
      S.tab[x % kLongTSlots][lane] = make_uint4((uint32_t)pa, (uint32_t)(pa >> 32), a.y, 0u);
    }
  };
  auto issue_b = [&](int32_t x) {  // table of chunk x built, then a __syncwarp
    if (x >= nch || !own) return;
    const int ne = min(32, atot - x * 32);
    const int bslot = x % kLongBSlots, tslot = x % kLongTSlots;
    auto copy = [&](int u, const uint4& t) {
      const ST* rp = reinterpret_cast<const ST*>((uint64_t)t.x | ((uint64_t)t.y << 32));
      cp_async16_nb(&S.b[bslot][u][lane], rp + col);
    };
    if (ne == 32) {
#pragma unroll
      for (int u0 = 0; u0 < 32; u0 += 8) {
        uint4 t[8];
#pragma unroll
        for (int k = 0; k < 8; k++) t[k] = S.tab[tslot][u0 + k];
#pragma unroll
        for (int k = 0; k < 8; k++) copy(u0 + k, t[k]);
      }
    } else {
      for (int u = 0; u < ne; u++) copy(u, S.tab[tslot][u]);
    }
  };
  // fill: A(0..5) staged, chunks 0 and 1 built and their B slices asked for
  issue_a(0);
  issue_a(1);
  cp_async_commit();
  issue_a(2);
  issue_a(3);
  cp_async_commit();
  cp_async_wait_group<1>();
  build(0);
  build(1);
  __syncwarp();
  issue_b(0);
  issue_a(4);
  cp_async_commit();
  issue_b(1);
  issue_a(5);
  cp_async_commit();
  cp_async_wait_group<2>();
  for (int32_t c = 0; c < nch; c++) {
    issue_a(c + 6);
    build(c + 2);
    __syncwarp();
    issue_b(c + 2);
    cp_async_commit();
    cp_async_wait_group<2>();  // B(c) and A(c + 4) have landed
    const int ne = min(32, atot - c * 32);
    const int bslot = c % kLongBSlots, tslot = c % kLongTSlots;
    if (own) {
      if (ne == 32) {
#pragma unroll 8
        for (int u = 0; u < 32; u++) {
          float b[VN];
          V::unpack_raw(S.b[bslot][u][lane], b);
          const float vs = __uint_as_float(S.tab[tslot][u].z);
#pragma unroll
          for (int x = 0; x < VN; x++) acc[x] = __fmaf_rn(vs, b[x], acc[x]);
        }
      } else {
        for (int u = 0; u < ne; u++) {
          float b[VN];
          V::unpack_raw(S.b[bslot][u][lane], b);
          const float vs = __uint_as_float(S.tab[tslot][u].z);
#pragma unroll
          for (int x = 0; x < VN; x++) acc[x] = __fmaf_rn(vs, b[x], acc[x]);
        }
      }
    }
    __syncwarp();
  }
  cp_async_wait_all();
  if (own) V::store(crow + col, acc);
}

// Items (listed row, C tile column, panel), a row's items consecutive, taken
// from a device counter in list order.  Every block, once placed, lets a
// programmatic dependent (k_spmm under the dependent-launch schedule) launch.
template <typename ST, bool SUB>
__global__ void __launch_bounds__(kLongWarps * 32)
    k_spmm_long(SpGridView A, DGridView B, DGridView C, const int64_t* __restrict__ list,
                const int32_t* __restrict__ count, int npanels, int row_align_ok,
                unsigned long long* __restrict__ next_item) {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  extern __shared__ __align__(16) unsigned char long_smem[];
  LongSmem& S = reinterpret_cast<LongSmem*>(long_smem)[threadIdx.x >> 5];
  constexpr int PW = 32 * Vec<ST>::N;
  const int lane = lane_id();
  const int64_t rows = A.gm * A.tm;
  const int64_t nv = count[0];
  const int64_t nl = nv + count[1];
  const int64_t per_row = C.gn * npanels;
  const unsigned long long n = (unsigned long long)(nl * per_row);
  unsigned long long it = 0;
  if (lane == 0) it = atomicAdd(next_item, 1ULL);
  it = __shfl_sync(kFull, it, 0);
  while (it < n) {
    unsigned long long nx = 0;
    if (lane == 0) nx = atomicAdd(next_item, 1ULL);
    const int64_t li = (int64_t)it / per_row;
    const int64_t pt = (int64_t)it - li * per_row;
    const int panel = (int)(pt % npanels);
    const int64_t tj = pt / npanels;
    const int64_t x = li < nv ? list[li] : list[rows - 1 - (li - nv)];
    const int64_t ti = x / A.tm, r = x - ti * A.tm;
    const int W = (int)C.cols_of(tj);
    if (panel * PW < W) {
      const bool vec = row_align_ok && (W % Vec<ST>::N) == 0 && tiles_aligned(B, C, ti, tj);
      if (vec) spmm_long_row<ST, SUB>(S, A, B, C, ti, tj, r, panel * PW, W);  // otherwise k_spmm did it element-wise
    }
    it = __shfl_sync(kFull, nx, 0);
  }
}

// Launch delay of the short-row kernel under the side-stream schedule: a
// one-warp kernel on the main stream that returns after `ns` (global timer,
// bounded by an iteration cap; it waits for nothing), so that the long-row
// blocks, which each need a whole SM's shared memory, are placed first.
constexpr unsigned kLongHeadStartNs = 4000;

__global__ void k_spmm_launch_delay(unsigned ns) {
  uint64_t t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (int i = 0; i < 4096; i++) {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 >= ns) break;
    __nanosleep(256);
  }
}

// Blocks of k_spmm_long (one per SM: its shared memory fills the SM); the
// other SMs run k_spmm.  By default a quarter of the SMs per column panel of
// a long row, at most half (R-MAT s21 x 256: FP32, two panels, 74 blocks;
// BF16, one panel, 37 blocks, measured 2.39 against 2.75 ms with 74);
// BCLX_TUNE_SPMM_LONG_BLOCKS sets the count.
static int spmm_long_blocks(const Context* ctx, int npanels) {
  int b = (int)tuning(ctx, BCLX_TUNE_SPMM_LONG_BLOCKS);
  if (b <= 0) b = std::min(ctx->num_sms / 2, ctx->num_sms / 4 * npanels);
  return std::max(1, std::min(b, ctx->num_sms));
}

static int64_t spmm_long_min_rows() {
  const char* e = std::getenv("BCLX_SPMM_LONG_MIN_ROWS");
  return e && *e ? std::strtoll(e, nullptr, 10) : kSpmmLongMinRows;
}

// Rows per k_spmm warp item: grouping short rows shares one prologue (tile
// descriptors, row pointers, A loads) among them, while the items still
// cover every resident warp.  BCLX_TUNE_SPMM_ROWS (1, 2, 4) overrides.
static int spmm_rows_per_item(const Context* ctx, const DGridView& C, int64_t gk, int npanels) {
  auto fits = [&](int r) { return r <= kSpmmMaxRows && r * gk <= 32; };
  const int want = (int)tuning(ctx, BCLX_TUNE_SPMM_ROWS);
  if ((want == 1 || want == 2 || want == 4) && fits(want)) return want;
  const int64_t resident = (int64_t)ctx->num_sms * 4 * kSpmmWarps;
  int r = 1;
  while (fits(2 * r) && C.gm * C.gn * ceil_div(C.tm, (int64_t)(2 * r)) * npanels >= resident) r *= 2;
  return r;
}

// Two schedules of the long-row and short-row kernels (BCLX_TUNE_SPMM_SCHEDULE):
//  0 (default): the long rows on the context's side stream at the highest
//    priority; k_spmm on the main stream after the list is ready and a
//    4-microsecond launch delay, so the long-row blocks take their SMs first;
//  1: one stream; k_spmm launched as k_spmm_long's programmatic dependent
//    (it launches once every long-row block has started, and finishes only
//    after k_spmm_long).
// Measured on R-MAT s21 x 256 (one B200): schedule 0 4.14 ms FP32 / 2.45 ms
// BF16, schedule 1 4.63 / 3.45 ms.  Also measured, and slower: one-warp
// long-row blocks small enough to share every SM with four k_spmm blocks
// (k_spmm capped at 56 registers, both kernels at the largest shared-memory
// carveout): 5.08 / 3.91 ms, k_spmm alone losing 15 % to the smaller L1;
// and one cp.async.bulk copy per 512-byte B slice, completing on an
// mbarrier, in place of the per-lane copies: 6.8 ms for k_spmm_long alone
// against 1.9.
template <typename ST, bool SUB>
static int launch_spmm(Context* ctx, const SpGridView& A, const DGridView& B, const DGridView& C, int align_ok) {
  constexpr int VN = Vec<ST>::N;
  const int npanels = (int)ceil_div(C.tn, 32 * VN);
  const int R = spmm_rows_per_item(ctx, C, A.gn, npanels);
  const int64_t ngroups = ceil_div(C.tm, (int64_t)R);
  const int64_t n_items = C.gm * C.gn * ngroups * npanels;
  if (n_items == 0) return BCLX_OK;
  const int64_t want = ceil_div(n_items, kSpmmWarps);
  const int64_t cap = (int64_t)ctx->num_sms * 4;  // resident blocks: warps take items from a counter
  const int64_t arows = A.gm * A.tm;
  const bool long_path = align_ok && A.gn <= 32 && arows >= spmm_long_min_rows();
  // rows of at least long_row entries go to the long-row kernel: by default
  // 512 for FP32 and 1024 for BF16 (R-MAT s21 x 256: FP32 4.00 against
  // 4.21 ms with 1024; BF16 2.42 against 3.11 ms with 512)
  int long_row = (int)tuning(ctx, BCLX_TUNE_SPMM_LONG_ROW);
  if (long_row <= 0) long_row = sizeof(ST) == 4 ? 512 : 1024;
  const bool dependent = tuning(ctx, BCLX_TUNE_SPMM_SCHEDULE) == 1;
  // counters: [0] k_spmm items, [1] k_spmm_long items, [2] listed very long / other long rows (2 x int32)
  unsigned long long* ctr = nullptr;
  BCLX_TRY(scratch_alloc_n(ctx, &ctr, 3));
  BCLX_CK(cudaMemsetAsync(ctr, 0, 3 * sizeof(unsigned long long), ctx->stream));
  int32_t* cnt = reinterpret_cast<int32_t*>(ctr + 2);
  uint8_t* flag = nullptr;
  int64_t* list = nullptr;
  if (long_path) {
    BCLX_TRY(scratch_alloc_n(ctx, &flag, (size_t)arows));
    BCLX_TRY(scratch_alloc_n(ctx, &list, (size_t)arows));
    cudaStream_t ls = ctx->stream;
    if (!dependent) {
      BCLX_TRY(ensure_side_stream(ctx));
      BCLX_CK(cudaEventRecord(ctx->fork_ev, ctx->stream));
      BCLX_CK(cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0));
      ls = ctx->side;
    }
    k_spmm_find_long<<<(unsigned)std::min<int64_t>(ceil_div(arows, 256), (int64_t)ctx->num_sms * 16), 256, 0,
                       ls>>>(A, long_row, long_row * 8, flag, list, cnt);
    note_launch();
    BCLX_CK_LAUNCH();
    if (!dependent) BCLX_CK(cudaEventRecord(ctx->fork2_ev, ctx->side));
    const size_t lsmem = sizeof(LongSmem) * kLongWarps;
    BCLX_CK(cudaFuncSetAttribute(k_spmm_long<ST, SUB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsmem));
    k_spmm_long<ST, SUB><<<(unsigned)spmm_long_blocks(ctx, npanels), kLongWarps * 32, lsmem, ls>>>(A, B, C, list, cnt, npanels,
                                                                                    align_ok, ctr + 1);
    note_launch();
    BCLX_CK_LAUNCH();
    if (!dependent) {
      BCLX_CK(cudaEventRecord(ctx->join_ev, ctx->side));
      BCLX_CK(cudaStreamWaitEvent(ctx->stream, ctx->fork2_ev, 0));
      k_spmm_launch_delay<<<1, 32, 0, ctx->stream>>>(kLongHeadStartNs);
      note_launch();
      BCLX_CK_LAUNCH();
    }
  }
  const unsigned grid = (unsigned)(want < cap ? want : cap);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kSpmmWarps * 32);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = (long_path && dependent) ? 1 : 0;
  const uint8_t* lflag = flag;
  const int pmajor = (int)tuning(ctx, BCLX_TUNE_SPMM_PANEL_MAJOR);
  if (R > 1)
    BCLX_CK(cudaLaunchKernelEx(&cfg, k_spmm<ST, true, SUB>, A, B, C, n_items, npanels, R, ngroups, align_ok, pmajor, lflag,
                               ctr));
  else
    BCLX_CK(cudaLaunchKernelEx(&cfg, k_spmm<ST, false, SUB>, A, B, C, n_items, npanels, 1, ngroups, align_ok, pmajor, lflag,
                               ctr));
  note_launch();
  BCLX_CK_LAUNCH();
  if (long_path) {
    if (!dependent) BCLX_CK(cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0));
    scratch_free(ctx, flag);
    scratch_free(ctx, list);
  }
  scratch_free(ctx, ctr);
  return BCLX_OK;
}

static int run_spmm(Context* ctx, const SpGridView& A, const DGridView& B, const DGridView& C, int dtype) {
  const int es = dtype == BCLX_F32 ? 4 : 2;
  const int align_ok = ((B.ld * es) % 16 == 0) && ((C.ld * es) % 16 == 0);
  if (B.rot_i) {  // a sub-grid (bclx_spmm_grid_sub): stage maps
    if (dtype == BCLX_F32) return launch_spmm<float, true>(ctx, A, B, C, align_ok);
    return launch_spmm<__nv_bfloat16, true>(ctx, A, B, C, align_ok);
  }
  if (dtype == BCLX_F32) return launch_spmm<float, false>(ctx, A, B, C, align_ok);
  return launch_spmm<__nv_bfloat16, false>(ctx, A, B, C, align_ok);
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

static int spmm_grid_impl(bclx_context_t c, const bclx_spgrid_t* a, const bclx_dgrid_t* b, const bclx_dgrid_t* cg,
                          int natural_order, const int64_t* tile_rows = nullptr,
                          const int64_t* tile_cols = nullptr) {
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
  B.natural_order = natural_order;
  DGridView C{};
  C.tiles = cg->tiles; C.m = cg->m; C.n = cg->n; C.tm = cg->tile_m; C.tn = cg->tile_n; C.gm = cg->grid_m;
  C.gn = cg->grid_n; C.ld = cg->tile_n;
  if (!tile_rows || a->grid_n == 0 || cg->grid_m == 0 || cg->grid_n == 0) return run_spmm(ctx, A, B, C, b->dtype);
  // sub-grid: the stage maps, on the device for the launch
  std::vector<int32_t> maps((size_t)(cg->grid_m + cg->grid_n));
  for (int64_t i = 0; i < cg->grid_m; i++) maps[(size_t)i] = (int32_t)(tile_rows[i] % a->grid_n);
  for (int64_t j = 0; j < cg->grid_n; j++) maps[(size_t)(cg->grid_m + j)] = (int32_t)(tile_cols[j] % a->grid_n);
  int32_t* dmaps = nullptr;
  BCLX_TRY(scratch_alloc_n(ctx, &dmaps, maps.size()));
  cudaError_t e = cudaMemcpyAsync(dmaps, maps.data(), sizeof(int32_t) * maps.size(), cudaMemcpyHostToDevice,
                                  ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);  // the host vector goes out of scope
  if (e != cudaSuccess) {
    scratch_free(ctx, dmaps);
    set_last_error(std::string("stage maps: ") + cudaGetErrorString(e));
    return BCLX_ERR_CUDA;
  }
  B.rot_i = dmaps;
  B.rot_j = dmaps + cg->grid_m;
  const int rc = run_spmm(ctx, A, B, C, b->dtype);
  scratch_free(ctx, dmaps);  // stream-ordered: after the launches (the side stream is joined)
  return rc;
}

int bclx_spmm_grid(bclx_context_t c, const bclx_spgrid_t* a, const bclx_dgrid_t* b, const bclx_dgrid_t* cg) {
  return spmm_grid_impl(c, a, b, cg, 0);
}

int bclx_spmm_grid_rowwise(bclx_context_t c, const bclx_spgrid_t* a, const bclx_dgrid_t* b, const bclx_dgrid_t* cg) {
  return spmm_grid_impl(c, a, b, cg, 1);
}

int bclx_spmm_grid_sub(bclx_context_t c, const bclx_spgrid_t* a, const bclx_dgrid_t* b, const bclx_dgrid_t* cg,
                       const int64_t* tile_rows, const int64_t* tile_cols) {
  if (!cg || !tile_rows || !tile_cols) return BCLX_ERR_INVALID;
  // global tile indices increasing (so only the last may be a ragged edge tile)
  for (int64_t i = 0; i < cg->grid_m; i++)
    if (tile_rows[i] < 0 || tile_rows[i] >= INT32_MAX || (i > 0 && tile_rows[i] <= tile_rows[i - 1]))
      return BCLX_ERR_INVALID;
  for (int64_t j = 0; j < cg->grid_n; j++)
    if (tile_cols[j] < 0 || tile_cols[j] >= INT32_MAX || (j > 0 && tile_cols[j] <= tile_cols[j - 1]))
      return BCLX_ERR_INVALID;
  return spmm_grid_impl(c, a, b, cg, 0, tile_rows, tile_cols);
}

}  // extern "C"
