// Learned (m, s) selector: a small MLP 8 -> 64 -> 64 -> (5 Pade-degree logits + scalar s).
//
// Weights (FP32 masters, 5126 values, this order): W1 [64 x 8], b1 [64], W2 [64 x 64], b2 [64],
// W3 [6 x 64], b3 [6]; ReLU after the two hidden layers.  Output o[0..4] are the logits of
// m in {3, 5, 7, 9, 13}, o[5] the predicted number of squarings.
//
// Kernels:
//   k_mlp_infer     inference with BF16 weights and FP32 accumulation; one warp per sample,
//                   the weights staged once per CTA in shared memory.
//   k_mlp_fwd_bwd   fused forward + backward of a minibatch in FP32: 32 samples per CTA, the
//                   activations kept in shared memory, the weight gradient of the CTA reduced
//                   in shared memory and added to the global gradient once per CTA.
//                   Loss per sample: cross-entropy of the m logits + lambda (s_hat - s)^2.
//   k_adam          Adam update of the FP32 weights from the accumulated gradient.
// The host loop (fx_mlp_train) draws minibatches from a seeded permutation and runs
// fwd_bwd + adam per step on one stream; nothing crosses to the host until the end.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "fx_kernels.cuh"

namespace fx {
namespace {

constexpr int kIn = 8, kH = 64, kOut = 6, kCls = 5;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH, kParams = oB3 + kOut;
static_assert(kParams == 5126, "parameter count");

// ------------------------------------------------------------------------- inference
__global__ void __launch_bounds__(256) k_mlp_infer(const float* __restrict__ w, const float* __restrict__ x, int n,
                                                   float* __restrict__ out) {
  __shared__ __nv_bfloat16 sw[kParams];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) sw[i] = __float2bfloat16_rn(w[i]);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sample = blockIdx.x * (blockDim.x >> 5) + warp;
  if (sample >= n) return;
  const float* xs = x + (size_t)sample * kIn;
  // lane j owns hidden units j and j + 32
  float h1[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int j = lane + 32 * u;
    float a = __bfloat162float(sw[oB1 + j]);
#pragma unroll
    for (int k = 0; k < kIn; ++k) a += __bfloat162float(sw[oW1 + j * kIn + k]) * xs[k];
    h1[u] = fmaxf(a, 0.f);
  }
  float h2[2];
#pragma unroll
  for (int u = 0; u < 2; ++u) {
    const int j = lane + 32 * u;
    float a = __bfloat162float(sw[oB2 + j]);
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
#pragma unroll
      for (int kk = 0; kk < 32; ++kk) {
        const float hk = __shfl_sync(0xffffffffu, h1[hh], kk);
        a += __bfloat162float(sw[oW2 + j * kH + 32 * hh + kk]) * hk;
      }
    }
    h2[u] = fmaxf(a, 0.f);
  }
  for (int o = 0; o < kOut; ++o) {
    float a = __bfloat162float(sw[oW3 + o * kH + lane]) * h2[0] + __bfloat162float(sw[oW3 + o * kH + lane + 32]) * h2[1];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) a += __shfl_xor_sync(0xffffffffu, a, d);
    if (lane == 0) out[(size_t)sample * kOut + o] = a + __bfloat162float(sw[oB3 + o]);
  }
}

// ------------------------------------------------------------------- fused forward/backward
// 32 samples per CTA of 256 threads.  idx: sample indices of the minibatch (into x, ym, ys).
// grad (kParams floats) and loss (1 float) are accumulated with atomics, once per CTA.
constexpr int kSamplesPerCta = 32;
__global__ void __launch_bounds__(256) k_mlp_fwd_bwd(const float* __restrict__ w, const float* __restrict__ x,
                                                     const int* __restrict__ ym, const float* __restrict__ ys,
                                                     const int* __restrict__ idx, int nb, float lambda, float inv_nb,
                                                     float* __restrict__ grad, float* __restrict__ loss) {
  extern __shared__ float sm[];
  float* sw = sm;                                  // kParams
  float* sg = sw + kParams;                        // kParams (gradient of this CTA)
  float* a0 = sg + kParams;                        // 32 x 8   inputs
  float* z1 = a0 + kSamplesPerCta * kIn;           // 32 x 64  pre-activations
  float* z2 = z1 + kSamplesPerCta * kH;            // 32 x 64
  float* o3 = z2 + kSamplesPerCta * kH;            // 32 x 6   outputs, then their gradients
  float* d2 = o3 + kSamplesPerCta * kOut;          // 32 x 64  dL/dz2
  float* d1 = d2 + kSamplesPerCta * kH;            // 32 x 64  dL/dz1
  __shared__ float s_loss;
  const int tid = threadIdx.x;
  for (int i = tid; i < kParams; i += blockDim.x) {
    sw[i] = w[i];
    sg[i] = 0.f;
  }
  if (tid == 0) s_loss = 0.f;
  const int first = blockIdx.x * kSamplesPerCta;
  const int cnt = min(kSamplesPerCta, nb - first);
  for (int i = tid; i < kSamplesPerCta * kIn; i += blockDim.x) {
    const int s = i / kIn;
    a0[i] = s < cnt ? x[(size_t)idx[first + s] * kIn + (i % kIn)] : 0.f;
  }
  __syncthreads();
  // layer 1 and 2 forward: thread t -> (sample t / 8, units (t % 8) + 8 u)
  for (int i = tid; i < kSamplesPerCta * kH; i += blockDim.x) {
    const int s = i / kH, j = i % kH;
    float a = sw[oB1 + j];
#pragma unroll
    for (int k = 0; k < kIn; ++k) a += sw[oW1 + j * kIn + k] * a0[s * kIn + k];
    z1[i] = a;
  }
  __syncthreads();
  for (int i = tid; i < kSamplesPerCta * kH; i += blockDim.x) {
    const int s = i / kH, j = i % kH;
    float a = sw[oB2 + j];
    for (int k = 0; k < kH; ++k) a += sw[oW2 + j * kH + k] * fmaxf(z1[s * kH + k], 0.f);
    z2[i] = a;
  }
  __syncthreads();
  for (int i = tid; i < kSamplesPerCta * kOut; i += blockDim.x) {
    const int s = i / kOut, o = i % kOut;
    float a = sw[oB3 + o];
    for (int k = 0; k < kH; ++k) a += sw[oW3 + o * kH + k] * fmaxf(z2[s * kH + k], 0.f);
    o3[i] = a;
  }
  __syncthreads();
  // loss and dL/do (one thread per sample), scaled by 1 / minibatch size
  if (tid < kSamplesPerCta) {
    const int s = tid;
    float* o = o3 + s * kOut;
    const int g = s < cnt ? idx[first + s] : 0;
    const int c = s < cnt ? ym[g] : -1;
    if (s < cnt && (unsigned)c < (unsigned)kCls) {   // a label outside 0..4 contributes nothing
      float mx = o[0];
      for (int k = 1; k < kCls; ++k) mx = fmaxf(mx, o[k]);
      float se = 0.f;
      for (int k = 0; k < kCls; ++k) se += expf(o[k] - mx);
      const float lse = mx + logf(se);
      const float ds = o[kCls] - ys[g];
      atomicAdd(&s_loss, (lse - o[c] + lambda * ds * ds) * inv_nb);
      for (int k = 0; k < kCls; ++k) o[k] = (expf(o[k] - lse) - (k == c ? 1.f : 0.f)) * inv_nb;
      o[kCls] = 2.f * lambda * ds * inv_nb;
    } else {
      for (int k = 0; k < kOut; ++k) o[k] = 0.f;
    }
  }
  __syncthreads();
  // backward through layer 3: dW3, db3, d2 = W3^T do * relu'(z2)
  for (int i = tid; i < kOut * kH; i += blockDim.x) {
    const int o = i / kH, k = i % kH;
    float a = 0.f;
    for (int s = 0; s < kSamplesPerCta; ++s) a += o3[s * kOut + o] * fmaxf(z2[s * kH + k], 0.f);
    sg[oW3 + i] += a;
  }
  for (int o = tid; o < kOut; o += blockDim.x) {
    float a = 0.f;
    for (int s = 0; s < kSamplesPerCta; ++s) a += o3[s * kOut + o];
    sg[oB3 + o] += a;
  }
  for (int i = tid; i < kSamplesPerCta * kH; i += blockDim.x) {
    const int s = i / kH, k = i % kH;
    float a = 0.f;
#pragma unroll
    for (int o = 0; o < kOut; ++o) a += sw[oW3 + o * kH + k] * o3[s * kOut + o];
    d2[i] = z2[i] > 0.f ? a : 0.f;
  }
  __syncthreads();
  // layer 2: dW2, db2, d1 = W2^T d2 * relu'(z1)
  for (int i = tid; i < kH * kH; i += blockDim.x) {
    const int j = i / kH, k = i % kH;
    float a = 0.f;
    for (int s = 0; s < kSamplesPerCta; ++s) a += d2[s * kH + j] * fmaxf(z1[s * kH + k], 0.f);
    sg[oW2 + i] += a;
  }
  for (int j = tid; j < kH; j += blockDim.x) {
    float a = 0.f;
    for (int s = 0; s < kSamplesPerCta; ++s) a += d2[s * kH + j];
    sg[oB2 + j] += a;
  }
  for (int i = tid; i < kSamplesPerCta * kH; i += blockDim.x) {
    const int s = i / kH, k = i % kH;
    float a = 0.f;
    for (int j = 0; j < kH; ++j) a += sw[oW2 + j * kH + k] * d2[s * kH + j];
    d1[i] = z1[i] > 0.f ? a : 0.f;
  }
  __syncthreads();
  // layer 1: dW1, db1
  for (int i = tid; i < kH * kIn; i += blockDim.x) {
    const int j = i / kIn, k = i % kIn;
    float a = 0.f;
    for (int s = 0; s < kSamplesPerCta; ++s) a += d1[s * kH + j] * a0[s * kIn + k];
    sg[oW1 + i] += a;
  }
  for (int j = tid; j < kH; j += blockDim.x) {
    float a = 0.f;
    for (int s = 0; s < kSamplesPerCta; ++s) a += d1[s * kH + j];
    sg[oB1 + j] += a;
  }
  __syncthreads();
  for (int i = tid; i < kParams; i += blockDim.x) atomicAdd(grad + i, sg[i]);
  if (tid == 0) atomicAdd(loss, s_loss);
}

constexpr size_t kFwdBwdSmem =
    sizeof(float) * (2 * kParams + kSamplesPerCta * (kIn + 2 * kH + kOut + 2 * kH));

__global__ void k_adam(float* w, float* m, float* v, float* grad, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  grad[i] = 0.f;
}

std::string g_sel_err;
int sel_fail(const Error& e) {
  g_sel_err = e.msg;
  return e.code;
}

}  // namespace

void launch_mlp_infer(const float* w, const float* x, int n, float* out, cudaStream_t s) {
  if (n <= 0) return;
  k_mlp_infer<<<cdiv(n, 8), 256, 0, s>>>(w, x, n, out);
  FX_LAUNCH_CHECK();
}

}  // namespace fx

extern "C" {

int fx_mlp_param_count(void) { return fx::kParams; }

int fx_mlp_infer(const float* dw, const float* dx, int64_t n, float* dout, void* stream) {
  try {
    if (!dw || !dx || !dout || n < 0) throw fx::Error{FX_ERR_VALUE, "mlp: null argument or negative count"};
    fx::launch_mlp_infer(dw, dx, (int)n, dout, (cudaStream_t)stream);
  } catch (const fx::Error& e) {
    return fx::sel_fail(e);
  }
  return FX_OK;
}

int fx_mlp_loss_grad(const float* dw, const float* dx, const int32_t* dym, const float* dys, int64_t n,
                     float lambda, float* dgrad, float* dloss, void* stream) {
  try {
    if (!dw || !dx || !dym || !dys || !dgrad || !dloss || n <= 0)
      throw fx::Error{FX_ERR_VALUE, "mlp: null argument or empty batch"};
    cudaStream_t s = (cudaStream_t)stream;
    std::vector<int> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    int* didx = nullptr;
    FX_CUDA(cudaMallocAsync((void**)&didx, sizeof(int) * n, s));
    FX_CUDA(cudaMemcpyAsync(didx, idx.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
    FX_CUDA(cudaMemsetAsync(dgrad, 0, sizeof(float) * fx::kParams, s));
    FX_CUDA(cudaMemsetAsync(dloss, 0, sizeof(float), s));
    FX_CUDA(cudaFuncSetAttribute(fx::k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fx::kFwdBwdSmem));
    fx::k_mlp_fwd_bwd<<<fx::cdiv(n, fx::kSamplesPerCta), 256, fx::kFwdBwdSmem, s>>>(
        dw, dx, dym, dys, didx, (int)n, lambda, 1.f / (float)n, dgrad, dloss);
    FX_LAUNCH_CHECK();
    FX_CUDA(cudaFreeAsync(didx, s));
    FX_CUDA(cudaStreamSynchronize(s));
  } catch (const fx::Error& e) {
    return fx::sel_fail(e);
  }
  return FX_OK;
}

int fx_mlp_train(float* dw, const float* dx, const int32_t* dym, const float* dys, int64_t n, int epochs, int batch,
                 float lr, float lambda, uint64_t seed, float* epoch_loss, void* stream) {
  try {
    if (!dw || !dx || !dym || !dys || n <= 0 || epochs <= 0 || batch <= 0)
      throw fx::Error{FX_ERR_VALUE, "mlp: bad training arguments"};
    cudaStream_t s = (cudaStream_t)stream;
    const int P = fx::kParams;
    float *m = nullptr, *v = nullptr, *g = nullptr, *loss = nullptr;
    int* didx = nullptr;
    FX_CUDA(cudaMallocAsync((void**)&m, sizeof(float) * 3 * P + sizeof(float) * epochs, s));
    v = m + P;
    g = v + P;
    loss = g + P;
    FX_CUDA(cudaMallocAsync((void**)&didx, sizeof(int) * n * epochs, s));
    FX_CUDA(cudaMemsetAsync(m, 0, sizeof(float) * 3 * P + sizeof(float) * epochs, s));
    // one seeded permutation per epoch, uploaded once
    std::mt19937_64 rng(seed);
    std::vector<int> perm((size_t)n * epochs);
    for (int e = 0; e < epochs; ++e) {
      std::iota(perm.begin() + (size_t)e * n, perm.begin() + (size_t)(e + 1) * n, 0);
      std::shuffle(perm.begin() + (size_t)e * n, perm.begin() + (size_t)(e + 1) * n, rng);
    }
    FX_CUDA(cudaMemcpyAsync(didx, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice, s));
    FX_CUDA(cudaFuncSetAttribute(fx::k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fx::kFwdBwdSmem));
    const float b1 = 0.9f, b2 = 0.999f;
    int step = 0;
    for (int e = 0; e < epochs; ++e) {
      for (int64_t first = 0; first < n; first += batch) {
        const int nb = (int)std::min<int64_t>(batch, n - first);
        ++step;
        fx::k_mlp_fwd_bwd<<<fx::cdiv(nb, fx::kSamplesPerCta), 256, fx::kFwdBwdSmem, s>>>(
            dw, dx, dym, dys, didx + (size_t)e * n + first, nb, lambda, 1.f / (float)nb, g, loss + e);
        FX_LAUNCH_CHECK();
        const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
        fx::k_adam<<<fx::cdiv(P, 256), 256, 0, s>>>(dw, m, v, g, P, lr, b1, b2, 1e-8f, c1, c2);
        FX_LAUNCH_CHECK();
      }
    }
    if (epoch_loss) {
      std::vector<float> h(epochs);
      FX_CUDA(cudaMemcpyAsync(h.data(), loss, sizeof(float) * epochs, cudaMemcpyDeviceToHost, s));
      FX_CUDA(cudaStreamSynchronize(s));
      const int steps_per_epoch = (int)((n + batch - 1) / batch);
      for (int e = 0; e < epochs; ++e) epoch_loss[e] = h[e] / (float)steps_per_epoch;
    }
    FX_CUDA(cudaFreeAsync(m, s));
    FX_CUDA(cudaFreeAsync(didx, s));
    FX_CUDA(cudaStreamSynchronize(s));
  } catch (const fx::Error& e) {
    return fx::sel_fail(e);
  }
  return FX_OK;
}

const char* fx_mlp_error(void) { return fx::g_sel_err.c_str(); }

}  // extern "C"
