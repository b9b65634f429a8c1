// Context (device, stream, scratch pool), status text and the device-wide
// exclusive scan used to turn per-row counts into CSR offsets.
#include "common.cuh"

#include <cstdlib>

#include <atomic>
#include <cstring>
#include <string>

namespace bclx {

static int64_t env_or(const char* name, int64_t dflt) {
  const char* e = std::getenv(name);
  return e && *e ? std::strtoll(e, nullptr, 10) : dflt;
}

// Defaults of the tuning knobs (environment variables override some, for
// experiments without code changes).
static int64_t tuning_default(const Context* ctx, int key) {
  switch (key) {
    case BCLX_TUNE_LIGHT_UB: return 512;
    case BCLX_TUNE_LEARN_TARGET: return 320;
    case BCLX_TUNE_BTABLE_MAX_BYTES: return env_or("BCLX_BTABLE_MAX_BYTES", int64_t(2) << 30);
    case BCLX_TUNE_SPMM_ROWS: return env_or("BCLX_SPMM_ROWS", 0);
    case BCLX_TUNE_SPMM_LONG_ROW: return env_or("BCLX_SPMM_LONG_ROW", 0);
    case BCLX_TUNE_SPMM_LONG_BLOCKS: return env_or("BCLX_SPMM_LONG_BLOCKS", 0);
    case BCLX_TUNE_SPMM_SCHEDULE: return env_or("BCLX_SPMM_SCHEDULE", 0);
    case BCLX_TUNE_ITEM_OUTPUTS: return env_or("BCLX_ITEM_OUTPUTS", 512);
    case BCLX_TUNE_WIDE_LIGHT: return env_or("BCLX_WIDE_LIGHT", 0);
    case BCLX_TUNE_SPMM_PANEL_MAJOR: return env_or("BCLX_SPMM_PANEL_MAJOR", 0);
    default: return 0;
  }
}

static bool tuning_in_range(const Context* ctx, int key, int64_t v) {
  switch (key) {
    case BCLX_TUNE_LIGHT_UB: return v >= 32 && v <= 512;
    case BCLX_TUNE_LEARN_TARGET: return v >= 64 && v <= 448;
    case BCLX_TUNE_BTABLE_MAX_BYTES: return true;
    case BCLX_TUNE_SPMM_ROWS: return v == 0 || v == 1 || v == 2 || v == 4;
    case BCLX_TUNE_SPMM_LONG_ROW: return v == 0 || (v >= 64 && v <= INT32_MAX);
    case BCLX_TUNE_SPMM_LONG_BLOCKS: return v >= 0 && v <= ctx->num_sms;
    case BCLX_TUNE_SPMM_SCHEDULE: return v == 0 || v == 1;
    case BCLX_TUNE_ITEM_OUTPUTS: return v == 512 || v == 1024;
    case BCLX_TUNE_WIDE_LIGHT: return v == 0 || v == 1;
    case BCLX_TUNE_SPMM_PANEL_MAJOR: return v == 0 || v == 1;
    default: return false;
  }
}

int64_t tuning(const Context* ctx, int key) {
  if (key < 0 || key >= BCLX_TUNE_KEYS) return 0;
  return ctx->tune[key] >= 0 ? ctx->tune[key] : tuning_default(ctx, key);
}


static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

static std::atomic<long long> g_launches{0};
void note_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int scratch_alloc(Context* ctx, void** p, size_t bytes) {
  cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
  if (e != cudaSuccess) {
    set_last_error(std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    *p = nullptr;
    return e == cudaErrorMemoryAllocation ? BCLX_ERR_NO_MEMORY : BCLX_ERR_CUDA;
  }
  return BCLX_OK;
}

void scratch_free(Context* ctx, void* p) {
  if (p) cudaFreeAsync(p, ctx->stream);
}

// ---- exclusive scan: reduce per block, scan the block sums, scan again ----

constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 16;
constexpr int kScanChunk = kScanThreads * kScanPerThread;

template <typename TIn>
__device__ __forceinline__ int64_t load_or_zero(const TIn* in, int64_t i, int64_t n) {
  return i < n ? (int64_t)in[i] : 0;
}

__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* total) {
  __shared__ int64_t warp_tot[kScanThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int64_t incl = warp_inclusive_scan(v);
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    int64_t w = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
    int64_t wi = warp_inclusive_scan(w);
    if (lane < kScanThreads / 32) warp_tot[lane] = wi - w;
    if (lane == kScanThreads / 32 - 1) *total = wi;  // written by one lane; read after the barrier
  }
  __syncthreads();
  int64_t r = warp_tot[warp] + incl - v;
  __syncthreads();
  return r;
}

template <typename TIn>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const TIn* __restrict__ in, int64_t n,
                                                              int64_t* __restrict__ block_sums) {
  int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanPerThread;
  int64_t s = 0;
#pragma unroll
  for (int q = 0; q < kScanPerThread; q++) s += load_or_zero(in, base + q, n);
  __shared__ int64_t tot;
  block_exclusive_scan(s, &tot);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

// One block scans the block sums in place (exclusive), looping over chunks.
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(int64_t* __restrict__ sums, int64_t nb) {
  __shared__ int64_t tot;
  int64_t carry = 0;
  for (int64_t base = 0; base < nb; base += kScanThreads) {
    int64_t i = base + threadIdx.x;
    int64_t v = i < nb ? sums[i] : 0;
    int64_t ex = block_exclusive_scan(v, &tot);
    if (i < nb) sums[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[nb] = carry;
}

template <typename TIn>
__global__ void __launch_bounds__(kScanThreads) k_scan_final(const TIn* __restrict__ in, int64_t n,
                                                             const int64_t* __restrict__ block_sums,
                                                             int64_t* __restrict__ out) {
  int64_t base = (int64_t)blockIdx.x * kScanChunk + (int64_t)threadIdx.x * kScanPerThread;
  int64_t vals[kScanPerThread];
  int64_t s = 0;
#pragma unroll
  for (int q = 0; q < kScanPerThread; q++) {
    vals[q] = load_or_zero(in, base + q, n);
    s += vals[q];
  }
  __shared__ int64_t tot;
  int64_t run = block_exclusive_scan(s, &tot) + block_sums[blockIdx.x];
#pragma unroll
  for (int q = 0; q < kScanPerThread; q++) {
    if (base + q < n) out[base + q] = run;
    run += vals[q];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) out[n] = block_sums[gridDim.x];
}

template <typename TIn>
static int exclusive_scan_impl(Context* ctx, const TIn* in, int64_t* out, int64_t n) {
  if (n == 0) {
    BCLX_CK(cudaMemsetAsync(out, 0, sizeof(int64_t), ctx->stream));
    return BCLX_OK;
  }
  int64_t nb = ceil_div(n, kScanChunk);
  int64_t* sums = nullptr;
  BCLX_TRY(scratch_alloc_n(ctx, &sums, nb + 1));
  k_scan_reduce<TIn><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(in, n, sums);
  k_scan_sums<<<1, kScanThreads, 0, ctx->stream>>>(sums, nb);
  k_scan_final<TIn><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(in, n, sums, out);
  note_launch(3);
  cudaError_t e = cudaGetLastError();
  scratch_free(ctx, sums);
  if (e != cudaSuccess) {
    set_last_error(std::string("scan launch: ") + cudaGetErrorString(e));
    return BCLX_ERR_CUDA;
  }
  return BCLX_OK;
}

int64_t exclusive_scan_sums_len(int64_t n) { return ceil_div(n > 0 ? n : 1, kScanChunk) + 1; }

int exclusive_scan_i32_buf(Context* ctx, const int32_t* in, int64_t* out, int64_t n, int64_t* sums) {
  if (n == 0) {
    BCLX_CK(cudaMemsetAsync(out, 0, sizeof(int64_t), ctx->stream));
    return BCLX_OK;
  }
  const int64_t nb = ceil_div(n, kScanChunk);
  k_scan_reduce<int32_t><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(in, n, sums);
  k_scan_sums<<<1, kScanThreads, 0, ctx->stream>>>(sums, nb);
  k_scan_final<int32_t><<<(unsigned)nb, kScanThreads, 0, ctx->stream>>>(in, n, sums, out);
  note_launch(3);
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

int exclusive_scan_i32(Context* ctx, const int32_t* in, int64_t* out, int64_t n) {
  return exclusive_scan_impl(ctx, in, out, n);
}
int exclusive_scan_i64(Context* ctx, const int64_t* in, int64_t* out, int64_t n) {
  return exclusive_scan_impl(ctx, in, out, n);
}

int ensure_side_stream(Context* ctx) {
  if (ctx->side) return BCLX_OK;
  // highest priority: work forked to the side stream (long SpMM rows, the
  // SpGEMM B-row table) gets SMs ahead of the main stream's blocks
  int lo = 0, hi = 0;
  BCLX_CK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  BCLX_CK(cudaStreamCreateWithPriority(&ctx->side, cudaStreamNonBlocking, hi));
  BCLX_CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
  BCLX_CK(cudaEventCreateWithFlags(&ctx->fork2_ev, cudaEventDisableTiming));
  BCLX_CK(cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming));
  return BCLX_OK;
}

}  // namespace bclx

using namespace bclx;

extern "C" {

const char* bclx_last_error(void) { return g_last_error.c_str(); }

int bclx_version(void) { return 100; }

long long bclx_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int bclx_context_create(int device, bclx_context_t* out) {
  if (!out) return BCLX_ERR_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    set_last_error("no CUDA device with that ordinal");
    return BCLX_ERR_NO_DEVICE;
  }
  BCLX_CK(cudaSetDevice(device));
  cudaDeviceProp prop;
  BCLX_CK(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    set_last_error("bclx kernels are built for sm_100a (B200); this device is sm_" +
                   std::to_string(prop.major) + std::to_string(prop.minor));
    return BCLX_ERR_NO_DEVICE;
  }
  Context* ctx = new Context();
  ctx->device = device;
  ctx->num_sms = prop.multiProcessorCount;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  if (cudaHostAlloc(&ctx->pinned, 8 * sizeof(int64_t), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer(&ctx->pinned_dev, ctx->pinned, 0) != cudaSuccess) {
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    delete ctx;
    set_last_error("cudaHostAlloc (mapped readback slots) failed");
    return BCLX_ERR_NO_MEMORY;
  }
  *out = reinterpret_cast<bclx_context_t>(ctx);
  return BCLX_OK;
}

int bclx_context_destroy(bclx_context_t c) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx) return BCLX_OK;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  if (ctx->side) {
    cudaStreamSynchronize(ctx->side);
    cudaStreamDestroy(ctx->side);
  }
  for (cudaEvent_t e : {ctx->fork_ev, ctx->fork2_ev, ctx->join_ev})
    if (e) cudaEventDestroy(e);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  delete ctx;
  return BCLX_OK;
}

int bclx_context_set_tuning(bclx_context_t c, int32_t key, int64_t value) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || key < 0 || key >= BCLX_TUNE_KEYS) return BCLX_ERR_INVALID;
  if (value >= 0 && !tuning_in_range(ctx, key, value)) return BCLX_ERR_INVALID;
  ctx->tune[key] = value < 0 ? -1 : value;
  return BCLX_OK;
}

int bclx_context_get_tuning(bclx_context_t c, int32_t key, int64_t* value) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || !value || key < 0 || key >= BCLX_TUNE_KEYS) return BCLX_ERR_INVALID;
  *value = tuning(ctx, key);
  return BCLX_OK;
}

int bclx_context_set_stream(bclx_context_t c, void* stream) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx) return BCLX_ERR_INVALID;
  ctx->stream = reinterpret_cast<cudaStream_t>(stream);
  return BCLX_OK;
}

int bclx_context_release_cached(bclx_context_t c) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  cudaMemPool_t pool;
  BCLX_CK(cudaDeviceGetDefaultMemPool(&pool, ctx->device));
  BCLX_CK(cudaMemPoolTrimTo(pool, 0));
  return BCLX_OK;
}

int bclx_context_synchronize(bclx_context_t c) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx) return BCLX_ERR_INVALID;
  BCLX_CK(cudaStreamSynchronize(ctx->stream));
  return BCLX_OK;
}

}  // extern "C"
