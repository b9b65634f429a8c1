// Shared pieces of the bclx CUDA library: status handling, the context
// (device, stream, stream-ordered scratch pool, pinned readback slot), tile
// grid views read by the kernels, and warp/block primitives.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include <string>

#include "../../include/bclx.h"

namespace bclx {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarp = 32;

// ---- status ---------------------------------------------------------------

void set_last_error(const std::string& msg);

// Kernel launches issued by this library (all contexts), for launch accounting.
void note_launch(int n = 1);

#define BCLX_CK(call)                                                              \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess) {                                                      \
      ::bclx::set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      return e_ == cudaErrorMemoryAllocation ? BCLX_ERR_NO_MEMORY : BCLX_ERR_CUDA; \
    }                                                                             \
  } while (0)

#define BCLX_CK_LAUNCH() BCLX_CK(cudaGetLastError())

#define BCLX_TRY(expr)            \
  do {                            \
    int s_ = (expr);              \
    if (s_ != BCLX_OK) return s_; \
  } while (0)

// ---- context ----------------------------------------------------------------

struct Context {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  int64_t* pinned = nullptr;      // host readback slots (page-locked, mapped)
  int64_t* pinned_dev = nullptr;  // the same slots as the device addresses them
  // A second stream for planning work that overlaps the main stream (created
  // on first use), with events to fork from and join back to the main stream.
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, fork2_ev = nullptr, join_ev = nullptr;
  // bclx_context_set_tuning values (-1: the default)
  int64_t tune[BCLX_TUNE_KEYS] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1};
};

// The value in effect for a tuning knob (the context's, else the default).
int64_t tuning(const Context* ctx, int key);

// Create ctx->side and its events if they do not exist yet.
int ensure_side_stream(Context* ctx);

// Stream-ordered scratch from the device's default memory pool (kept cached:
// the release threshold is raised at context creation).
int scratch_alloc(Context* ctx, void** p, size_t bytes);
void scratch_free(Context* ctx, void* p);

template <typename T>
int scratch_alloc_n(Context* ctx, T** p, size_t count) {
  return scratch_alloc(ctx, reinterpret_cast<void**>(p), sizeof(T) * (count > 0 ? count : 1));
}

// Exclusive prefix sum of `in` (int32 or int64 values) into int64 `out`
// [count+1]; out[count] is the total.
int exclusive_scan_i32(Context* ctx, const int32_t* in, int64_t* out, int64_t count);
int exclusive_scan_i64(Context* ctx, const int64_t* in, int64_t* out, int64_t count);
// The same scan with a caller-provided block-sums buffer of
// exclusive_scan_sums_len(count) entries (allocates nothing).
int64_t exclusive_scan_sums_len(int64_t count);
int exclusive_scan_i32_buf(Context* ctx, const int32_t* in, int64_t* out, int64_t count, int64_t* sums);

// ---- grid views (kernel parameters) -------------------------------------------

struct SpGridView {
  const bclx_csr_t* tiles;  // device array, or null: use `single`
  bclx_csr_t single;
  int64_t m, n, tm, tn, gm, gn;

  __device__ __forceinline__ bclx_csr_t tile(int64_t i, int64_t j) const {
    return tiles ? tiles[i * gn + j] : single;
  }
  __host__ __device__ __forceinline__ int64_t rows_of(int64_t i) const {
    int64_t r = m - i * tm;
    return r < tm ? r : tm;
  }
  __host__ __device__ __forceinline__ int64_t cols_of(int64_t j) const {
    int64_t c = n - j * tn;
    return c < tn ? c : tn;
  }
};

inline SpGridView make_view(const bclx_spgrid_t& g) {
  SpGridView v{};
  v.tiles = g.tiles;
  v.m = g.m; v.n = g.n; v.tm = g.tile_m; v.tn = g.tile_n; v.gm = g.grid_m; v.gn = g.grid_n;
  return v;
}

struct DGridView {
  void* const* tiles;  // device array, or null: use `single`
  void* single;
  int64_t m, n, tm, tn, gm, gn;
  int64_t ld;  // leading dimension in elements
  // SpMM stage order: 0 = the SUMMA loop's rotated order k = (k_ + i + j) mod
  // G (spgemm.hpp:162-175), 1 = ascending k (the row-wise variants,
  // experimental_gemm.hpp:83-214).  Read from the B view.
  int32_t natural_order;
  // Sub-grid stage maps (bclx_spmm_grid_sub), read from the B view: the
  // global tile row of each C grid row and the global tile column of each C
  // grid column, both mod G, so that the rotation is that of the tile's
  // global position; null when the grids are the whole product.
  const int32_t* rot_i;
  const int32_t* rot_j;

  __device__ __forceinline__ void* tile(int64_t i, int64_t j) const {
    return tiles ? tiles[i * gn + j] : single;
  }
  __host__ __device__ __forceinline__ int64_t rows_of(int64_t i) const {
    int64_t r = m - i * tm;
    return r < tm ? r : tm;
  }
  __host__ __device__ __forceinline__ int64_t cols_of(int64_t j) const {
    int64_t c = n - j * tn;
    return c < tn ? c : tn;
  }
};

// ---- device helpers -----------------------------------------------------------

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
  const int lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T t = __shfl_up_sync(kFull, v, d);
    if (lane >= d) v += t;
  }
  return v;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(kFull, v, d);
  return v;
}

// Multiply-add in the value type: one fused multiply-add for float (what the
// reference's `c += a*b` compiles to), wrapping arithmetic for int32.
__device__ __forceinline__ float madd(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ int32_t madd(int32_t a, int32_t b, int32_t c) {
  return (int32_t)((uint32_t)a * (uint32_t)b + (uint32_t)c);
}
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ int32_t vadd(int32_t a, int32_t b) {
  return (int32_t)((uint32_t)a + (uint32_t)b);
}

// First position in sorted col[lo, hi) whose value is >= key.
__device__ __forceinline__ int32_t lower_bound_i32(const int32_t* __restrict__ col, int32_t lo, int32_t hi,
                                                   int32_t key) {
  while (lo < hi) {
    int32_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(col + mid) < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace bclx
