// Dense-tile and elementwise container operations:
//   DMatrix::sum                     (bcl/containers/DMatrix.hpp:537-554)
//   SPMatrix::binary_op_inplace      (bcl/containers/SPMatrix.hpp:571-616)
//
// Both are single passes over HBM (bound by its bandwidth): the sum reads
// every tile element once; the binary op reads a sparse grid's column
// indices and values and one dense element per stored entry, and writes the
// values back.
#include "common.cuh"

#include <algorithm>
#include <cstring>
#include <type_traits>

namespace bclx {

__device__ __forceinline__ double to_double(float v) { return (double)v; }
__device__ __forceinline__ double to_double(__nv_bfloat16 v) { return (double)__bfloat162float(v); }

// Sum of the valid (unpadded) part of every tile.  Blocks take (tile, row)
// pairs grid-stride; threads stride over the row's columns.  Floating point
// accumulates in FP64 per thread, then per block, then one FP64 atomic per
// block; int32 accumulates in 64-bit wrapping integers (the low 32 bits are
// the exact sum modulo 2^32 whatever the order).
template <typename T, typename Acc>
__global__ void __launch_bounds__(256) k_dsum(DGridView D, Acc* __restrict__ out) {
  __shared__ Acc red[8];
  Acc acc = Acc(0);
  const int64_t nrows = D.gm * D.gn * D.tm;
  for (int64_t x = blockIdx.x; x < nrows; x += gridDim.x) {
    const int64_t t = x / D.tm, r = x - t * D.tm;
    const int64_t ti = t / D.gn, tj = t - ti * D.gn;
    if (r >= D.rows_of(ti)) continue;
    const int64_t w = D.cols_of(tj);
    const T* row = reinterpret_cast<const T*>(D.tile(ti, tj)) + r * D.ld;
    for (int64_t c = threadIdx.x; c < w; c += blockDim.x) {
      if constexpr (std::is_same<T, int32_t>::value)
        acc = (Acc)((unsigned long long)acc + (unsigned long long)(long long)__ldg(row + c));
      else
        acc += to_double(row[c]);
    }
  }
  // block reduction
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const Acc o = __shfl_xor_sync(kFull, acc, d);
    if constexpr (std::is_same<T, int32_t>::value)
      acc = (Acc)((unsigned long long)acc + (unsigned long long)o);
    else
      acc += o;
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    if constexpr (std::is_same<T, int32_t>::value) {
      unsigned long long b = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); q++) b += (unsigned long long)red[q];
      atomicAdd(reinterpret_cast<unsigned long long*>(out), b);
    } else {
      Acc b = Acc(0);
      for (int q = 0; q < (int)(blockDim.x >> 5); q++) b += red[q];
      atomicAdd(out, b);
    }
  }
}

__device__ __forceinline__ float wrap_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float wrap_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float wrap_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ int32_t wrap_add(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
__device__ __forceinline__ int32_t wrap_sub(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
__device__ __forceinline__ int32_t wrap_mul(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }

// One rounding per operation (no contraction), int32 wrapping: what the
// reference's functor computes on the host.
template <typename T>
__device__ __forceinline__ T apply_op(int op, T a, T b) {
  switch (op) {
    case BCLX_OP_PLUS: return wrap_add(a, b);
    case BCLX_OP_MINUS: return wrap_sub(a, b);
    case BCLX_OP_MULTIPLIES: return wrap_mul(a, b);
    case BCLX_OP_MIN: return b < a ? b : a;
    case BCLX_OP_MAX: return a < b ? b : a;
    case BCLX_OP_SECOND: return b;
    default: return a;
  }
}
__device__ __forceinline__ float apply_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ int32_t apply_div(int32_t a, int32_t b) {
  if (b == 0) return 0;
  if (b == -1) return (int32_t)(0u - (uint32_t)a);  // INT32_MIN / -1 wraps
  return a / b;
}

// Every stored entry (row r of tile (ti, tj), column c) becomes
// op(value, B(global row, global column)); one warp per tile row, lanes over
// the row's entries.
template <typename T>
__global__ void __launch_bounds__(256) k_binary_op(SpGridView A, DGridView B, int op) {
  const int lane = lane_id();
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  const int64_t nrows = A.gm * A.gn * A.tm;
  for (int64_t x = warp; x < nrows; x += nwarps) {
    const int64_t t = x / A.tm, r = x - t * A.tm;
    const int64_t ti = t / A.gn, tj = t - ti * A.gn;
    if (r >= A.rows_of(ti)) continue;
    const bclx_csr_t At = A.tile(ti, tj);
    const int32_t p0 = __ldg(At.row_ptr + r), p1 = __ldg(At.row_ptr + r + 1);
    const int64_t gr = ti * A.tm + r;
    const int64_t bi = gr / B.tm, br = gr - bi * B.tm;
    T* vals = reinterpret_cast<T*>(At.vals);
    for (int32_t p = p0 + lane; p < p1; p += 32) {
      const int64_t gc = tj * A.tn + __ldg(At.col_ind + p);
      const int64_t bj = gc / B.tn, bc = gc - bj * B.tn;
      const T b = __ldg(reinterpret_cast<const T*>(B.tile(bi, bj)) + br * B.ld + bc);
      const T a = vals[p];
      vals[p] = op == BCLX_OP_DIVIDES ? apply_div(a, b) : apply_op(op, a, b);
    }
  }
}

static bool dgrid_ok(const bclx_dgrid_t* d) {
  return d && d->tiles && d->m >= 0 && d->n >= 0 && d->tile_m > 0 && d->tile_n > 0 &&
         d->grid_m == ceil_div(d->m, d->tile_m) && d->grid_n == ceil_div(d->n, d->tile_n);
}

static DGridView dview(const bclx_dgrid_t& d) {
  DGridView v{};
  v.tiles = d.tiles;
  v.m = d.m; v.n = d.n; v.tm = d.tile_m; v.tn = d.tile_n; v.gm = d.grid_m; v.gn = d.grid_n; v.ld = d.tile_n;
  return v;
}

}  // namespace bclx

using namespace bclx;

extern "C" {

int bclx_dmatrix_sum(bclx_context_t c, const bclx_dgrid_t* a, void* result_host) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !dgrid_ok(a) || !result_host) return BCLX_ERR_INVALID;
  if (a->dtype != BCLX_F32 && a->dtype != BCLX_BF16 && a->dtype != BCLX_I32) return BCLX_ERR_DTYPE;
  BCLX_CK(cudaSetDevice(ctx->device));
  const DGridView D = dview(*a);
  void* acc = nullptr;
  BCLX_TRY(scratch_alloc(ctx, &acc, 8));
  BCLX_CK(cudaMemsetAsync(acc, 0, 8, ctx->stream));
  const int64_t rows = D.gm * D.gn * D.tm;
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(rows, (int64_t)ctx->num_sms * 8));
  if (a->dtype == BCLX_F32)
    k_dsum<float, double><<<blocks, 256, 0, ctx->stream>>>(D, reinterpret_cast<double*>(acc));
  else if (a->dtype == BCLX_BF16)
    k_dsum<__nv_bfloat16, double><<<blocks, 256, 0, ctx->stream>>>(D, reinterpret_cast<double*>(acc));
  else
    k_dsum<int32_t, long long><<<blocks, 256, 0, ctx->stream>>>(D, reinterpret_cast<long long*>(acc));
  note_launch();
  cudaError_t le = cudaGetLastError();
  int64_t raw = 0;
  cudaError_t ce = le == cudaSuccess ? cudaMemcpyAsync(&raw, acc, 8, cudaMemcpyDeviceToHost, ctx->stream) : le;
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx->stream);
  scratch_free(ctx, acc);
  if (ce != cudaSuccess) {
    set_last_error(std::string("bclx_dmatrix_sum: ") + cudaGetErrorString(ce));
    return BCLX_ERR_CUDA;
  }
  if (a->dtype == BCLX_I32) {
    const int32_t v = (int32_t)(uint32_t)(uint64_t)raw;
    std::memcpy(result_host, &v, sizeof(v));
  } else {
    double d;
    std::memcpy(&d, &raw, sizeof(d));
    const float v = (float)d;
    std::memcpy(result_host, &v, sizeof(v));
  }
  return BCLX_OK;
}

int bclx_spmatrix_binary_op(bclx_context_t c, const bclx_spgrid_t* a, const bclx_dgrid_t* b, int32_t op) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !a || !a->tiles || !dgrid_ok(b)) return BCLX_ERR_INVALID;
  if (a->m != b->m || a->n != b->n || a->tile_m <= 0 || a->tile_n <= 0 ||
      a->grid_m != ceil_div(a->m, a->tile_m) || a->grid_n != ceil_div(a->n, a->tile_n))
    return BCLX_ERR_INVALID;
  if (op < BCLX_OP_PLUS || op > BCLX_OP_SECOND) return BCLX_ERR_INVALID;
  if (!((a->dtype == BCLX_F32 && b->dtype == BCLX_F32) || (a->dtype == BCLX_I32 && b->dtype == BCLX_I32)))
    return BCLX_ERR_DTYPE;
  BCLX_CK(cudaSetDevice(ctx->device));
  const SpGridView A = make_view(*a);
  const DGridView B = dview(*b);
  const int64_t rows = A.gm * A.gn * A.tm;
  if (rows == 0) return BCLX_OK;
  const unsigned blocks = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(rows, 8), (int64_t)ctx->num_sms * 16));
  if (a->dtype == BCLX_F32) k_binary_op<float><<<blocks, 256, 0, ctx->stream>>>(A, B, op);
  else k_binary_op<int32_t><<<blocks, 256, 0, ctx->stream>>>(A, B, op);
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

}  // extern "C"
