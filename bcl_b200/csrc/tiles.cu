// Whole matrix <-> tile grid on the device: the slicing of a CSR matrix into
// the packed SPMatrix tile layout (what the SPMatrix(fname, blocking)
// constructor does on the host, SPMatrix.hpp:194-271 with
// CSRMatrix::get_slice_impl_, CSRMatrix.hpp:238-276), and its inverse, the
// gather of every tile back into one CSR matrix (SPMatrix::get,
// SPMatrix.hpp:516-546).  Both are byte moves bound by HBM bandwidth:
//
//   tiling   1. thread per row: the row's entries per tile column (columns
//               are sorted, so a tile column is one run found by binary
//               search) into counts[t][local row];
//            2. one exclusive scan over all counts gives every entry's tile
//               offset and local row pointer at once;
//            3. warp per row: each entry goes to its tile at
//               start(tile, row) + (position - start of its run).
//   gather   1. thread per row: the row's length over its tile columns;
//            2. scan -> row_ptr;  3. warp per row: copy the runs in tile
//               column order, columns shifted to global.
#include "common.cuh"

#include <string>

namespace bclx {

// Thread per global row: entries per tile column.  cnt has (tm+1) slots per
// tile (the last stays 0, so that one scan yields the tile's row pointer
// including its end).
__global__ void k_tile_count(int64_t m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci, int64_t tm,
                             int64_t tn, int64_t gn, int32_t* __restrict__ cnt) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ti = r / tm, lr = r - ti * tm;
    const int32_t rs = __ldg(rp + r), re = __ldg(rp + r + 1);
    int32_t p = rs;
    while (p < re) {  // columns are ascending (k_check_rows): a tile column is one run
      const int64_t tj = __ldg(ci + p) / tn;
      const int32_t q = tj == gn - 1 ? re : lower_bound_i32(ci, p, re, (int32_t)((tj + 1) * tn));
      cnt[(ti * gn + tj) * (tm + 1) + lr] = q - p;
      p = q;
    }
  }
}

// Warp per row: columns strictly ascending and within [0, n); else *bad.
__global__ void k_check_rows(int64_t m, int64_t n, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                             int32_t* __restrict__ bad) {
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps) {
    const int32_t rs = __ldg(rp + r), re = __ldg(rp + r + 1);
    bool ok = rs <= re;
    for (int32_t p = rs + lane; ok && p < re; p += 32) {
      const int32_t c = __ldg(ci + p);
      ok = c >= 0 && c < n && (p == rs || __ldg(ci + p - 1) < c);
    }
    if (__any_sync(kFull, !ok) && lane == 0) atomicExch(bad, 1);
  }
}

// Local row pointers and tile offsets from the scanned counts E.
__global__ void k_tile_ptrs(const int64_t* __restrict__ E, int64_t ntiles, int64_t tm, int32_t* __restrict__ trp,
                            int64_t* __restrict__ toff) {
  const int64_t total = ntiles * (tm + 1);
  for (int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; x < total; x += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = x / (tm + 1), lr = x - t * (tm + 1);
    const int64_t base = E[t * (tm + 1)];
    trp[x] = (int32_t)(E[x] - base);
    if (lr == 0) toff[t] = base;
    if (x == total - 1) toff[ntiles] = E[total];
  }
}

// Warp per global row: scatter the entries into their tiles.
template <typename VT>
__global__ void k_tile_scatter(int64_t m, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                               const VT* __restrict__ va, int64_t tm, int64_t tn, int64_t gn,
                               const int64_t* __restrict__ E, int32_t* __restrict__ oci, VT* __restrict__ ova) {
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < m; r += nwarps) {
    const int64_t ti = r / tm, lr = r - ti * tm;
    const int32_t rs = __ldg(rp + r), re = __ldg(rp + r + 1);
    int32_t carry = rs;  // start of the run the previous chunk ended in
    for (int32_t p0 = rs; p0 < re; p0 += 32) {
      const int32_t p = p0 + lane;
      int64_t tj = -1;
      int32_t c = 0;
      bool start = false;
      if (p < re) {
        c = __ldg(ci + p);
        tj = c / tn;
        start = p == rs || (int64_t)(__ldg(ci + p - 1) / tn) != tj;
      }
      // start of this entry's run: the latest run start at or before it
      int32_t s = start ? p : -1;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int32_t o = __shfl_up_sync(kFull, s, d);
        if (lane >= d) s = max(s, o);
      }
      if (s < 0) s = carry;
      carry = __shfl_sync(kFull, s, 31);
      if (p < re) {
        const int64_t dst = E[(ti * gn + tj) * (tm + 1) + lr] + (p - s);
        oci[dst] = (int32_t)(c - tj * tn);
        ova[dst] = __ldg(va + p);
      }
    }
  }
}

// Thread per global row: entries over the row's tiles.
__global__ void k_gather_len(SpGridView g, int32_t* __restrict__ len) {
  const int64_t m = g.m;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < m; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t ti = r / g.tm, lr = r - ti * g.tm;
    int64_t tot = 0;
    for (int64_t tj = 0; tj < g.gn; tj++) {
      const int32_t* trp = g.tile(ti, tj).row_ptr;
      tot += __ldg(trp + lr + 1) - __ldg(trp + lr);
    }
    len[r] = (int32_t)tot;
  }
}

__global__ void k_rowptr32(const int64_t* __restrict__ off, int64_t m, int32_t* __restrict__ rp) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= m; r += (int64_t)gridDim.x * blockDim.x)
    rp[r] = (int32_t)off[r];
}

// A value as SPMatrix::get returns it: the reference gathers through
// SparseHashAccumulator, which adds each value to a zero-initialised slot
// (SparseHashAccumulator.hpp:50-53) on the host, so -0.0 comes back as +0.0
// and a signalling NaN comes back quiet (its payload kept); every other
// value is unchanged.  int32 values pass through.
__device__ __forceinline__ int32_t gathered(int32_t v) { return v; }
__device__ __forceinline__ float gathered(float v) {
  uint32_t b = __float_as_uint(v);
  if (b == 0x80000000u) b = 0u;
  else if ((b & 0x7f800000u) == 0x7f800000u && (b & 0x007fffffu)) b |= 0x00400000u;
  return __uint_as_float(b);
}

// Warp per global row: copy its runs in tile-column order.
template <typename VT>
__global__ void k_gather_rows(SpGridView g, const int64_t* __restrict__ off, int32_t* __restrict__ oci,
                              VT* __restrict__ ova) {
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < g.m; r += nwarps) {
    const int64_t ti = r / g.tm, lr = r - ti * g.tm;
    int64_t dst = off[r];
    for (int64_t tj = 0; tj < g.gn; tj++) {
      const bclx_csr_t t = g.tile(ti, tj);
      const int32_t s = __ldg(t.row_ptr + lr), e = __ldg(t.row_ptr + lr + 1);
      const int32_t shift = (int32_t)(tj * g.tn);
      const VT* tv = reinterpret_cast<const VT*>(t.vals);
      for (int32_t p = s + lane; p < e; p += 32) {
        oci[dst + (p - s)] = __ldg(t.col_ind + p) + shift;
        ova[dst + (p - s)] = gathered(__ldg(tv + p));
      }
      dst += e - s;
    }
  }
}

static unsigned blocks_for(Context* ctx, int64_t work, int per_block) {
  int64_t b = ceil_div(work > 0 ? work : 1, per_block);
  const int64_t cap = (int64_t)ctx->num_sms * 16;
  return (unsigned)(b < cap ? b : cap);
}

}  // namespace bclx

using namespace bclx;

extern "C" {

int bclx_csr_to_tiles(bclx_context_t c, const bclx_csr_t* a, bclx_spgrid_out_t* out) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !a || !out) return BCLX_ERR_INVALID;
  if (a->dtype != BCLX_F32 && a->dtype != BCLX_I32) return BCLX_ERR_DTYPE;
  const int64_t m = a->m, n = a->n, tm = out->tile_m, tn = out->tile_n;
  if (m < 0 || n < 0 || tm <= 0 || tn <= 0 || out->m != m || out->n != n || out->grid_m != ceil_div(m, tm) ||
      out->grid_n != ceil_div(n, tn) || !out->tile_row_ptr || !out->tile_offset) {
    set_last_error("bclx_csr_to_tiles: output grid does not match the matrix and tile shape");
    return BCLX_ERR_INVALID;
  }
  if (n > INT32_MAX || (a->nnz > 0 && (!a->row_ptr || !a->col_ind || !a->vals || !out->col_ind || !out->vals))) {
    set_last_error("bclx_csr_to_tiles: missing arrays");
    return BCLX_ERR_INVALID;
  }
  BCLX_CK(cudaSetDevice(ctx->device));
  const int64_t gm = out->grid_m, gn = out->grid_n, ntiles = gm * gn;
  const int64_t slots = ntiles * (tm + 1);
  if (slots == 0) return BCLX_OK;
  int32_t* cnt = nullptr;
  int32_t* bad = nullptr;
  int64_t* E = nullptr;
  BCLX_TRY(scratch_alloc_n(ctx, &cnt, (size_t)slots));
  BCLX_TRY(scratch_alloc_n(ctx, &bad, 1));
  BCLX_TRY(scratch_alloc_n(ctx, &E, (size_t)slots + 1));
  BCLX_CK(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * slots, ctx->stream));
  BCLX_CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), ctx->stream));
  if (m > 0) {
    // the matrix is checked before anything is placed by its column indices
    k_check_rows<<<blocks_for(ctx, m, 8), 256, 0, ctx->stream>>>(m, n, a->row_ptr, a->col_ind, bad);
    note_launch();
    BCLX_CK_LAUNCH();
    int32_t hbad = 0;
    BCLX_CK(cudaMemcpyAsync(&hbad, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    BCLX_CK(cudaStreamSynchronize(ctx->stream));
    if (hbad) {
      scratch_free(ctx, cnt);
      scratch_free(ctx, bad);
      scratch_free(ctx, E);
      set_last_error("bclx_csr_to_tiles: column indices must be ascending and within [0, n) in every row");
      return BCLX_ERR_INVALID;
    }
    k_tile_count<<<blocks_for(ctx, m, 256), 256, 0, ctx->stream>>>(m, a->row_ptr, a->col_ind, tm, tn, gn, cnt);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  BCLX_TRY(exclusive_scan_i32(ctx, cnt, E, slots));
  k_tile_ptrs<<<blocks_for(ctx, slots, 256), 256, 0, ctx->stream>>>(E, ntiles, tm, out->tile_row_ptr,
                                                                    out->tile_offset);
  note_launch();
  BCLX_CK_LAUNCH();
  if (m > 0 && a->nnz > 0) {
    const unsigned blocks = blocks_for(ctx, m, 8);
    if (a->dtype == BCLX_F32)
      k_tile_scatter<float><<<blocks, 256, 0, ctx->stream>>>(m, a->row_ptr, a->col_ind,
                                                             reinterpret_cast<const float*>(a->vals), tm, tn, gn, E,
                                                             out->col_ind, reinterpret_cast<float*>(out->vals));
    else
      k_tile_scatter<int32_t><<<blocks, 256, 0, ctx->stream>>>(m, a->row_ptr, a->col_ind,
                                                               reinterpret_cast<const int32_t*>(a->vals), tm, tn, gn,
                                                               E, out->col_ind, reinterpret_cast<int32_t*>(out->vals));
    note_launch();
    BCLX_CK_LAUNCH();
  }
  scratch_free(ctx, cnt);
  scratch_free(ctx, bad);
  scratch_free(ctx, E);
  return BCLX_OK;
}

int bclx_tiles_to_csr(bclx_context_t c, const bclx_spgrid_t* g, int32_t* row_ptr, int32_t* col_ind, void* vals) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !g || !row_ptr || !g->tiles) return BCLX_ERR_INVALID;
  if (g->dtype != BCLX_F32 && g->dtype != BCLX_I32) return BCLX_ERR_DTYPE;
  if (g->m < 0 || g->n < 0 || g->tile_m <= 0 || g->tile_n <= 0 || g->grid_m != ceil_div(g->m, g->tile_m) ||
      g->grid_n != ceil_div(g->n, g->tile_n)) {
    set_last_error("bclx_tiles_to_csr: inconsistent tile grid");
    return BCLX_ERR_INVALID;
  }
  BCLX_CK(cudaSetDevice(ctx->device));
  const SpGridView v = make_view(*g);
  const int64_t m = g->m;
  int32_t* len = nullptr;
  int64_t* off = nullptr;
  BCLX_TRY(scratch_alloc_n(ctx, &len, (size_t)(m > 0 ? m : 1)));
  BCLX_TRY(scratch_alloc_n(ctx, &off, (size_t)m + 1));
  if (m > 0) {
    k_gather_len<<<blocks_for(ctx, m, 256), 256, 0, ctx->stream>>>(v, len);
    note_launch();
    BCLX_CK_LAUNCH();
  }
  BCLX_TRY(exclusive_scan_i32(ctx, len, off, m));
  int64_t nnz = 0;
  BCLX_CK(cudaMemcpyAsync(&nnz, off + m, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  if (nnz > INT32_MAX) {
    scratch_free(ctx, len);
    scratch_free(ctx, off);
    set_last_error("bclx_tiles_to_csr: more than 2^31-1 entries do not fit an int32 row_ptr");
    return BCLX_ERR_INDEX_OVERFLOW;
  }
  if (nnz > 0 && (!col_ind || !vals)) return BCLX_ERR_INVALID;
  k_rowptr32<<<blocks_for(ctx, m + 1, 256), 256, 0, ctx->stream>>>(off, m, row_ptr);
  note_launch();
  BCLX_CK_LAUNCH();
  if (nnz > 0) {
    const unsigned blocks = blocks_for(ctx, m, 8);
    if (g->dtype == BCLX_F32)
      k_gather_rows<float><<<blocks, 256, 0, ctx->stream>>>(v, off, col_ind, reinterpret_cast<float*>(vals));
    else
      k_gather_rows<int32_t><<<blocks, 256, 0, ctx->stream>>>(v, off, col_ind, reinterpret_cast<int32_t*>(vals));
    note_launch();
    BCLX_CK_LAUNCH();
  }
  scratch_free(ctx, len);
  scratch_free(ctx, off);
  return BCLX_OK;
}

}  // extern "C"
