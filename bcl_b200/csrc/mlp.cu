// Row-nnz predictor: a 5 -> 64 -> 64 -> 1 multilayer perceptron (ReLU, FP32)
// with hand-written training (forward, backward, Adam) and inference kernels.
//
// It predicts y = log2(1 + nnz of one C-tile row) from five features of the
// row (see k_row_features in spgemm.cu), so that the learned product can cut
// heavy rows into accumulator-sized items without a symbolic pass.
//
// Parameter layout (kMlpParams floats, row-major):
//   W1[5][64] | b1[64] | W2[64][64] | b2[64] | w3[64] | b3[1]
// Loss: mean squared error over the n samples, L = (1/n) sum (yhat - y)^2.
#include "common.cuh"

namespace bclx {

constexpr int kIn = 5, kH = 64;
constexpr int kOffW1 = 0, kOffB1 = kIn * kH, kOffW2 = kOffB1 + kH, kOffB2 = kOffW2 + kH * kH,
              kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kH, kMlpParams = kOffB3 + 1;
constexpr int kMlpBlock = 128;  // samples per block in the gradient kernel
constexpr int kS = kH + 1;      // padded row stride of the per-sample activations (no bank conflicts)

// Inference: one thread per sample, weights in shared memory.
__global__ void __launch_bounds__(256) k_mlp_forward(const float* __restrict__ X, int64_t n,
                                                     const float* __restrict__ prm, float* __restrict__ out) {
  __shared__ float w[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) w[i] = prm[i];
  __syncthreads();
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
    float x[kIn];
#pragma unroll
    for (int f = 0; f < kIn; f++) x[f] = X[s * kIn + f];
    float h1[kH];
#pragma unroll
    for (int u = 0; u < kH; u++) {
      float a = w[kOffB1 + u];
#pragma unroll
      for (int f = 0; f < kIn; f++) a = fmaf(x[f], w[kOffW1 + f * kH + u], a);
      h1[u] = fmaxf(a, 0.f);
    }
    float y = w[kOffB3];
    for (int u = 0; u < kH; u++) {
      float a = w[kOffB2 + u];
#pragma unroll
      for (int v = 0; v < kH; v++) a = fmaf(h1[v], w[kOffW2 + v * kH + u], a);
      y = fmaf(fmaxf(a, 0.f), w[kOffW3 + u], y);
    }
    out[s] = y;
  }
}

// Gradient of L over all samples, accumulated into grad[kMlpParams] (which
// the caller zeroes).  One block per kMlpBlock samples: each thread runs the
// forward and backward pass of one sample, keeps its layer activations and
// deltas in shared memory, and the block then reduces the weight gradients
// (dW = sum over its samples of activation x delta) before one atomic add per
// weight.  Also accumulates the loss sum into grad[kMlpParams].
__global__ void __launch_bounds__(kMlpBlock) k_mlp_grad(const float* __restrict__ X, const float* __restrict__ Y,
                                                        int64_t n, const float* __restrict__ prm,
                                                        float* __restrict__ grad) {
  extern __shared__ float sm[];
  float* w = sm;                              // kMlpParams
  float* h1 = w + kMlpParams;                 // [kMlpBlock][kS]
  float* d2 = h1 + kMlpBlock * kS;            // [kMlpBlock][kS]  delta at layer 2 pre-activation
  float* d1 = d2 + kMlpBlock * kS;            // [kMlpBlock][kS]  delta at layer 1 pre-activation
  float* xs = d1 + kMlpBlock * kS;            // [kMlpBlock][kIn]
  float* h2 = xs + kMlpBlock * kIn;           // [kMlpBlock][kS]
  float* dy = h2 + kMlpBlock * kS;            // [kMlpBlock]
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) w[i] = prm[i];
  __syncthreads();
  const float inv_n = 1.f / (float)n;
  for (int64_t base = (int64_t)blockIdx.x * kMlpBlock; base < n; base += (int64_t)gridDim.x * kMlpBlock) {
    const int t = threadIdx.x;
    const int64_t s = base + t;
    const bool live = s < n;
    float x[kIn];
#pragma unroll
    for (int f = 0; f < kIn; f++) {
      x[f] = live ? X[s * kIn + f] : 0.f;
      xs[t * kIn + f] = x[f];
    }
    for (int u = 0; u < kH; u++) {
      float a = w[kOffB1 + u];
#pragma unroll
      for (int f = 0; f < kIn; f++) a = fmaf(x[f], w[kOffW1 + f * kH + u], a);
      h1[t * kS + u] = fmaxf(a, 0.f);
    }
    float yhat = w[kOffB3];
    for (int u = 0; u < kH; u++) {
      float a = w[kOffB2 + u];
      for (int v = 0; v < kH; v++) a = fmaf(h1[t * kS + v], w[kOffW2 + v * kH + u], a);
      const float hv = fmaxf(a, 0.f);
      h2[t * kS + u] = hv;
      yhat = fmaf(hv, w[kOffW3 + u], yhat);
    }
    const float err = live ? yhat - Y[s] : 0.f;
    const float g = 2.f * err * inv_n;  // dL/dyhat
    dy[t] = g;
    for (int u = 0; u < kH; u++) d2[t * kS + u] = h2[t * kS + u] > 0.f ? g * w[kOffW3 + u] : 0.f;
    for (int v = 0; v < kH; v++) {
      float a = 0.f;
      for (int u = 0; u < kH; u++) a = fmaf(d2[t * kS + u], w[kOffW2 + v * kH + u], a);
      d1[t * kS + v] = h1[t * kS + v] > 0.f ? a : 0.f;
    }
    // loss sum (thread 0 of each warp adds its warp's share)
    float l = err * err;
    l = warp_sum(l);
    if ((t & 31) == 0) atomicAdd(&grad[kMlpParams], l);
    __syncthreads();
    // weight gradients of this block of samples: each thread owns some weights
    for (int p = t; p < kMlpParams; p += kMlpBlock) {
      float acc = 0.f;
      if (p < kOffB1) {  // W1[f][u]
        const int f = p / kH, u = p % kH;
        for (int q = 0; q < kMlpBlock; q++) acc = fmaf(xs[q * kIn + f], d1[q * kS + u], acc);
      } else if (p < kOffW2) {  // b1[u]
        const int u = p - kOffB1;
        for (int q = 0; q < kMlpBlock; q++) acc += d1[q * kS + u];
      } else if (p < kOffB2) {  // W2[v][u]
        const int v = (p - kOffW2) / kH, u = (p - kOffW2) % kH;
        for (int q = 0; q < kMlpBlock; q++) acc = fmaf(h1[q * kS + v], d2[q * kS + u], acc);
      } else if (p < kOffW3) {  // b2[u]
        const int u = p - kOffB2;
        for (int q = 0; q < kMlpBlock; q++) acc += d2[q * kS + u];
      } else if (p < kOffB3) {  // w3[u]
        const int u = p - kOffW3;
        for (int q = 0; q < kMlpBlock; q++) acc = fmaf(h2[q * kS + u], dy[q], acc);
      } else {  // b3
        for (int q = 0; q < kMlpBlock; q++) acc += dy[q];
      }
      atomicAdd(&grad[p], acc);
    }
    __syncthreads();
  }
}

// Adam step: prm -= lr * mhat / (sqrt(vhat) + eps); moments in mom[0..2P).
__global__ void k_mlp_adam(float* __restrict__ prm, const float* __restrict__ grad, float* __restrict__ mom,
                           float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kMlpParams; p += gridDim.x * blockDim.x) {
    const float g = grad[p];
    const float m = b1 * mom[p] + (1.f - b1) * g;
    const float v = b2 * mom[kMlpParams + p] + (1.f - b2) * g * g;
    mom[p] = m;
    mom[kMlpParams + p] = v;
    prm[p] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
  }
}

static size_t grad_smem() {
  return sizeof(float) * ((size_t)kMlpParams + 4 * (size_t)kMlpBlock * kS + (size_t)kMlpBlock * kIn + kMlpBlock);
}

static int launch_grad(Context* ctx, const float* X, const float* Y, int64_t n, const float* prm, float* grad) {
  BCLX_CK(cudaMemsetAsync(grad, 0, sizeof(float) * (kMlpParams + 1), ctx->stream));
  BCLX_CK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)grad_smem()));
  int64_t blocks = ceil_div(n, kMlpBlock);
  if (blocks > (int64_t)ctx->num_sms * 4) blocks = (int64_t)ctx->num_sms * 4;
  if (blocks < 1) blocks = 1;
  k_mlp_grad<<<(unsigned)blocks, kMlpBlock, grad_smem(), ctx->stream>>>(X, Y, n, prm, grad);
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

}  // namespace bclx

using namespace bclx;

extern "C" {

int bclx_mlp_num_params(void) { return kMlpParams; }

int bclx_mlp_predict(bclx_context_t c, const float* X, int64_t n, const float* params, float* out) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || n < 0 || (n > 0 && (!X || !params || !out))) return BCLX_ERR_INVALID;
  if (n == 0) return BCLX_OK;
  BCLX_CK(cudaSetDevice(ctx->device));
  int64_t blocks = ceil_div(n, 256);
  if (blocks > (int64_t)ctx->num_sms * 8) blocks = (int64_t)ctx->num_sms * 8;
  k_mlp_forward<<<(unsigned)blocks, 256, 0, ctx->stream>>>(X, n, params, out);
  note_launch();
  BCLX_CK_LAUNCH();
  return BCLX_OK;
}

int bclx_mlp_gradient(bclx_context_t c, const float* X, const float* y, int64_t n, const float* params,
                      float* grad) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || n <= 0 || !X || !y || !params || !grad) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  return launch_grad(ctx, X, y, n, params, grad);
}

int bclx_mlp_train(bclx_context_t c, const float* X, const float* y, int64_t n, float* params, int32_t steps,
                   float lr, float* loss_host) {
  Context* ctx = reinterpret_cast<Context*>(c);
  if (!ctx || n <= 0 || !X || !y || !params || steps < 0) return BCLX_ERR_INVALID;
  BCLX_CK(cudaSetDevice(ctx->device));
  float* work = nullptr;  // grad[P+1] | moments[2P]
  BCLX_TRY(scratch_alloc_n(ctx, &work, 3 * (size_t)kMlpParams + 1));
  float* grad = work;
  float* mom = work + kMlpParams + 1;
  int rc = BCLX_OK;
  if (cudaMemsetAsync(mom, 0, sizeof(float) * 2 * kMlpParams, ctx->stream) != cudaSuccess) rc = BCLX_ERR_CUDA;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float p1 = 1.f, p2 = 1.f;
  for (int32_t t = 0; t < steps && rc == BCLX_OK; t++) {
    rc = launch_grad(ctx, X, y, n, params, grad);
    if (rc != BCLX_OK) break;
    p1 *= b1;
    p2 *= b2;
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, ctx->stream>>>(params, grad, mom, lr, b1, b2, eps, 1.f - p1,
                                                                 1.f - p2);
    note_launch();
    if (cudaGetLastError() != cudaSuccess) rc = BCLX_ERR_CUDA;
    if (loss_host && rc == BCLX_OK) {
      float l = 0.f;
      if (cudaMemcpyAsync(&l, grad + kMlpParams, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
          cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        rc = BCLX_ERR_CUDA;
      loss_host[t] = l / (float)n;
    }
  }
  scratch_free(ctx, work);
  if (rc == BCLX_OK) BCLX_CK(cudaStreamSynchronize(ctx->stream));
  return rc;
}

}  // extern "C"
