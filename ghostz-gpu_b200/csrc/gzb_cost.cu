// gzb_cost.cu -- training and inference kernels of the gapped-stage cost
// model (8 -> 32 -> 32 -> 1 MLP, ReLU, mean squared error on log2(1+cells)).
//
// Training is FP32 and deterministic: each block computes the per-sample
// forward and backward pass of its slice of the minibatch (one thread per
// sample), stores the activations in shared memory and then reduces the
// weight gradients over its samples as small outer-product sums (one thread
// per parameter group); a second kernel sums the block partials in a fixed
// order and applies Adam.  Inference rounds weights and activations to BF16
// and accumulates in FP32.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "ghostz_b200.h"
#include "gzb_common.h"
#include "gzb_cost.cuh"

namespace gzb {

constexpr int kGradBlock = 128;  // samples per gradient block
// per-sample shared activations: x, h1, dh1, h2, dh2, dy
constexpr int kActStride = kFeat + 4 * kHid + 1;

__global__ void __launch_bounds__(kGradBlock)
mlp_grad_kernel(const float *__restrict__ params, const float *__restrict__ X,
                const float *__restrict__ Y, const uint32_t *__restrict__ idx, uint32_t n,
                float *__restrict__ partial, float *__restrict__ partial_loss) {
  extern __shared__ float smem[];
  float *P = smem;                          // kParams
  float *A = smem + ((kParams + 3) & ~3);   // kGradBlock * kActStride
  __shared__ float loss_s[kGradBlock];
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  const uint32_t s = blockIdx.x * kGradBlock + threadIdx.x;
  float *a = A + threadIdx.x * kActStride;
  float *x = a, *h1 = a + kFeat, *dh1 = h1 + kHid, *h2 = dh1 + kHid, *dh2 = h2 + kHid,
        *dy = dh2 + kHid;
  float lsum = 0.f;
  if (s < n) {
    const uint32_t i = idx ? idx[s] : s;
    for (int k = 0; k < kFeat; ++k) x[k] = X[(size_t)i * kFeat + k];
    for (int j = 0; j < kHid; ++j) {
      float acc = P[kOffB1 + j];
      for (int k = 0; k < kFeat; ++k) acc = fmaf(P[kOffW1 + j * kFeat + k], x[k], acc);
      h1[j] = acc > 0.f ? acc : 0.f;
    }
    for (int j = 0; j < kHid; ++j) {
      float acc = P[kOffB2 + j];
      for (int k = 0; k < kHid; ++k) acc = fmaf(P[kOffW2 + j * kHid + k], h1[k], acc);
      h2[j] = acc > 0.f ? acc : 0.f;
    }
    float y = P[kOffB3];
    for (int k = 0; k < kHid; ++k) y = fmaf(P[kOffW3 + k], h2[k], y);
    const float d = y - Y[i];
    lsum = d * d;
    const float g = 2.f * d / (float)n;
    dy[0] = g;
    for (int j = 0; j < kHid; ++j) dh2[j] = h2[j] > 0.f ? g * P[kOffW3 + j] : 0.f;
    for (int k = 0; k < kHid; ++k) {
      float acc = 0.f;
      for (int j = 0; j < kHid; ++j) acc = fmaf(P[kOffW2 + j * kHid + k], dh2[j], acc);
      dh1[k] = h1[k] > 0.f ? acc : 0.f;
    }
  } else {
    for (int k = 0; k < kActStride; ++k) a[k] = 0.f;
  }
  loss_s[threadIdx.x] = lsum;
  __syncthreads();
  // parameter gradients as sums over this block's samples
  float *out = partial + (size_t)blockIdx.x * kParams;
  for (int p = threadIdx.x; p < kParams; p += blockDim.x) {
    float acc = 0.f;
    if (p < kOffB1) {  // W1[j][k]
      const int j = p / kFeat, k = p % kFeat;
      for (int t = 0; t < kGradBlock; ++t)
        acc = fmaf(A[t * kActStride + kFeat + kHid + j], A[t * kActStride + k], acc);
    } else if (p < kOffW2) {  // b1[j]
      const int j = p - kOffB1;
      for (int t = 0; t < kGradBlock; ++t) acc += A[t * kActStride + kFeat + kHid + j];
    } else if (p < kOffB2) {  // W2[j][k]
      const int q = p - kOffW2, j = q / kHid, k = q % kHid;
      for (int t = 0; t < kGradBlock; ++t)
        acc = fmaf(A[t * kActStride + kFeat + 3 * kHid + j], A[t * kActStride + kFeat + k], acc);
    } else if (p < kOffW3) {  // b2[j]
      const int j = p - kOffB2;
      for (int t = 0; t < kGradBlock; ++t) acc += A[t * kActStride + kFeat + 3 * kHid + j];
    } else if (p < kOffB3) {  // W3[k]
      const int k = p - kOffW3;
      for (int t = 0; t < kGradBlock; ++t)
        acc = fmaf(A[t * kActStride + kFeat + 4 * kHid], A[t * kActStride + kFeat + 2 * kHid + k],
                   acc);
    } else {  // b3
      for (int t = 0; t < kGradBlock; ++t) acc += A[t * kActStride + kFeat + 4 * kHid];
    }
    out[p] = acc;
  }
  if (threadIdx.x == 0) {
    float l = 0.f;
    for (int t = 0; t < kGradBlock; ++t) l += loss_s[t];
    partial_loss[blockIdx.x] = l;
  }
}

// grad[p] = sum of block partials (fixed order); loss = sum / n
__global__ void mlp_reduce_kernel(const float *partial, const float *partial_loss, int blocks,
                                  uint32_t n, float *grad, float *loss) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kParams; p += gridDim.x * blockDim.x) {
    float acc = 0.f;
    for (int b = 0; b < blocks; ++b) acc += partial[(size_t)b * kParams + p];
    grad[p] = acc;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && loss) {
    float l = 0.f;
    for (int b = 0; b < blocks; ++b) l += partial_loss[b];
    *loss = l / (float)n;
  }
}

__global__ void mlp_adam_kernel(float *params, const float *grad, float *m, float *v, float lr,
                                float beta1, float beta2, float eps, float c1, float c2) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kParams; p += gridDim.x * blockDim.x) {
    const float g = grad[p];
    const float mm = beta1 * m[p] + (1.f - beta1) * g;
    const float vv = beta2 * v[p] + (1.f - beta2) * g * g;
    m[p] = mm;
    v[p] = vv;
    params[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
  }
}

// BF16 inference: weights and activations rounded to bf16, FP32 accumulate.
__device__ __forceinline__ float bf16_round(float v) {
  return __bfloat162float(__float2bfloat16(v));
}

// BF16 inference: parameters, inputs and both hidden layers rounded to
// bf16, products accumulated in fp32.  The parameters sit in shared memory
// as the fp32 values of their bf16 roundings (exact), the second layer's
// weights also transposed, and are read as float4 broadcasts.  Each thread
// takes two samples (s and s + T, T threads in the grid), so every weight
// read feeds both.  The first layer's units are taken one at a time and
// each is added at once into all 32 second-layer sums (kept in registers),
// which adds the same products in the same order (unit by unit) as summing
// each second-layer unit over the first layer's.
__global__ void __launch_bounds__(256, 2)
mlp_predict_kernel(const float *__restrict__ params, const float *__restrict__ X, uint32_t n,
                   float *__restrict__ out, const uint64_t *n_dev) {
  if (n_dev) n = (uint32_t)*n_dev;
  __shared__ __align__(16) float P[(kParams + 3) & ~3];
  __shared__ __align__(16) float W2T[kHid * kHid];  // W2T[i][j] = W2[j][i]
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) P[i] = bf16_round(params[i]);
  for (int t = threadIdx.x; t < kHid * kHid; t += blockDim.x) {
    const int i = t / kHid, j = t % kHid;
    W2T[t] = bf16_round(params[kOffW2 + j * kHid + i]);
  }
  __syncthreads();
  const float4 *P4 = reinterpret_cast<const float4 *>(P);
  const float4 *T4 = reinterpret_cast<const float4 *>(W2T);
  static_assert(kOffW1 % 4 == 0 && kOffW2 % 4 == 0 && kFeat % 4 == 0 && kHid % 4 == 0,
                "float4 rows");
  const uint32_t T = gridDim.x * blockDim.x;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += 2 * T) {
    const uint32_t s1 = s + T;
    const bool two = s1 < n;
    float x0[kFeat], x1[kFeat], a0[kHid], a1[kHid];
    const float4 *u4 = reinterpret_cast<const float4 *>(X + (size_t)s * kFeat);
    const float4 *v4 = reinterpret_cast<const float4 *>(X + (size_t)(two ? s1 : s) * kFeat);
#pragma unroll
    for (int k = 0; k < kFeat / 4; ++k) {
      const float4 u = u4[k], v = v4[k];
      x0[4 * k] = bf16_round(u.x);
      x0[4 * k + 1] = bf16_round(u.y);
      x0[4 * k + 2] = bf16_round(u.z);
      x0[4 * k + 3] = bf16_round(u.w);
      x1[4 * k] = bf16_round(v.x);
      x1[4 * k + 1] = bf16_round(v.y);
      x1[4 * k + 2] = bf16_round(v.z);
      x1[4 * k + 3] = bf16_round(v.w);
    }
#pragma unroll
    for (int j = 0; j < kHid; ++j) a0[j] = a1[j] = P[kOffB2 + j];
#pragma unroll 1
    for (int i = 0; i < kHid; ++i) {
      // first-layer unit i of both samples
      float h0 = P[kOffB1 + i], h1 = h0;
#pragma unroll
      for (int k = 0; k < kFeat / 4; ++k) {
        const float4 w = P4[(kOffW1 + i * kFeat) / 4 + k];
        h0 = fmaf(w.x, x0[4 * k], h0);
        h1 = fmaf(w.x, x1[4 * k], h1);
        h0 = fmaf(w.y, x0[4 * k + 1], h0);
        h1 = fmaf(w.y, x1[4 * k + 1], h1);
        h0 = fmaf(w.z, x0[4 * k + 2], h0);
        h1 = fmaf(w.z, x1[4 * k + 2], h1);
        h0 = fmaf(w.w, x0[4 * k + 3], h0);
        h1 = fmaf(w.w, x1[4 * k + 3], h1);
      }
      h0 = bf16_round(h0 > 0.f ? h0 : 0.f);
      h1 = bf16_round(h1 > 0.f ? h1 : 0.f);
      // ... added into every second-layer sum
#pragma unroll
      for (int q = 0; q < kHid / 4; ++q) {
        const float4 w = T4[(i * kHid) / 4 + q];
        a0[4 * q] = fmaf(w.x, h0, a0[4 * q]);
        a1[4 * q] = fmaf(w.x, h1, a1[4 * q]);
        a0[4 * q + 1] = fmaf(w.y, h0, a0[4 * q + 1]);
        a1[4 * q + 1] = fmaf(w.y, h1, a1[4 * q + 1]);
        a0[4 * q + 2] = fmaf(w.z, h0, a0[4 * q + 2]);
        a1[4 * q + 2] = fmaf(w.z, h1, a1[4 * q + 2]);
        a0[4 * q + 3] = fmaf(w.w, h0, a0[4 * q + 3]);
        a1[4 * q + 3] = fmaf(w.w, h1, a1[4 * q + 3]);
      }
    }
    float y0 = P[kOffB3], y1 = y0;
#pragma unroll
    for (int j = 0; j < kHid; ++j) {
      const float w3 = P[kOffW3 + j];
      y0 = fmaf(w3, bf16_round(a0[j] > 0.f ? a0[j] : 0.f), y0);
      y1 = fmaf(w3, bf16_round(a1[j] > 0.f ? a1[j] : 0.f), y1);
    }
    out[s] = y0;
    if (two) out[s1] = y1;
  }
}

// permutation keys for minibatch shuffling
__global__ void shuffle_keys_kernel(uint32_t n, uint64_t seed, uint64_t *keys, uint32_t *vals) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint64_t z = seed + 0x9e3779b97f4a7c15ull * (uint64_t)(i + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    keys[i] = z;
    vals[i] = i;
  }
}

static size_t grad_smem_bytes() {
  return sizeof(float) * (((kParams + 3) & ~3) + (size_t)kGradBlock * kActStride);
}

int cost_gradients(const float *d_params, const float *d_x, const float *d_y,
                   const uint32_t *d_idx, uint32_t n, float *d_grad, float *d_loss,
                   float *d_partial, float *d_partial_loss, cudaStream_t s) {
  const int blocks = (int)((n + kGradBlock - 1) / kGradBlock);
  static bool attr_set = false;
  if (!attr_set) {
    GZB_CUDA(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)grad_smem_bytes()));
    attr_set = true;
  }
  mlp_grad_kernel<<<blocks, kGradBlock, grad_smem_bytes(), s>>>(d_params, d_x, d_y, d_idx, n,
                                                                d_partial, d_partial_loss);
  GZB_CUDA(cudaGetLastError());
  mlp_reduce_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(d_partial, d_partial_loss, blocks, n,
                                                          d_grad, d_loss);
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}

int cost_predict(const float *d_params, const float *d_x, uint32_t n, float *d_out,
                 cudaStream_t s, const uint64_t *n_dev) {
  if (n == 0) return GZB_OK;
  GZB_CHECK(((uintptr_t)d_x & 15) == 0, GZB_ERR_INVALID, "features must be 16-byte aligned");
  unsigned g = (unsigned)((n + 255) / 256);
  if (g > 148 * 16) g = 148 * 16;
  mlp_predict_kernel<<<g, 256, 0, s>>>(d_params, d_x, n, d_out, n_dev);
  GZB_CUDA(cudaGetLastError());
  return GZB_OK;
}

// Minibatch Adam over device-resident (x, y); params in/out on the host.
int cost_train(const float *d_x, const float *d_y, uint32_t n, float *params, int epochs,
               int batch, float lr, uint64_t seed, float *final_loss, cudaStream_t s);

}  // namespace gzb

#include <cub/cub.cuh>

namespace gzb {

int cost_train(const float *d_x, const float *d_y, uint32_t n, float *params, int epochs,
               int batch, float lr, uint64_t seed, float *final_loss, cudaStream_t s) {
  GZB_CHECK(n > 0 && epochs > 0 && batch > 0, GZB_ERR_INVALID, "empty training set");
  const int max_blocks = (batch + kGradBlock - 1) / kGradBlock;
  float *P = nullptr, *G = nullptr, *M = nullptr, *V = nullptr, *part = nullptr, *pl = nullptr,
        *loss = nullptr;
  uint64_t *keys = nullptr, *keys2 = nullptr;
  uint32_t *vals = nullptr, *vals2 = nullptr;
  void *tmp = nullptr;
  size_t tb = 0;
  int rc = GZB_OK;
  auto fail = [&](cudaError_t e, const char *what) {
    rc = cuda_error(e, what, __FILE__, __LINE__);
  };
  cudaError_t e = cudaSuccess;
  if ((e = cudaMalloc(&P, 4 * kParams)) != cudaSuccess) fail(e, "params");
  if (!rc && (e = cudaMalloc(&G, 4 * kParams)) != cudaSuccess) fail(e, "grad");
  if (!rc && (e = cudaMalloc(&M, 4 * kParams)) != cudaSuccess) fail(e, "adam m");
  if (!rc && (e = cudaMalloc(&V, 4 * kParams)) != cudaSuccess) fail(e, "adam v");
  if (!rc && (e = cudaMalloc(&part, 4 * (size_t)kParams * max_blocks)) != cudaSuccess) fail(e, "partials");
  if (!rc && (e = cudaMalloc(&pl, 4 * max_blocks)) != cudaSuccess) fail(e, "partial loss");
  if (!rc && (e = cudaMalloc(&loss, 4)) != cudaSuccess) fail(e, "loss");
  if (!rc && (e = cudaMalloc(&keys, 8 * (size_t)n)) != cudaSuccess) fail(e, "keys");
  if (!rc && (e = cudaMalloc(&keys2, 8 * (size_t)n)) != cudaSuccess) fail(e, "keys");
  if (!rc && (e = cudaMalloc(&vals, 4 * (size_t)n)) != cudaSuccess) fail(e, "vals");
  if (!rc && (e = cudaMalloc(&vals2, 4 * (size_t)n)) != cudaSuccess) fail(e, "vals");
  if (!rc) {
    cub::DeviceRadixSort::SortPairs(nullptr, tb, keys, keys2, vals, vals2, (int64_t)n, 0, 64, s);
    if ((e = cudaMalloc(&tmp, tb)) != cudaSuccess) fail(e, "sort temp");
  }
  if (!rc && (e = cudaMemcpyAsync(P, params, 4 * kParams, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    fail(e, "upload params");
  if (!rc && (e = cudaMemsetAsync(M, 0, 4 * kParams, s)) != cudaSuccess) fail(e, "zero m");
  if (!rc && (e = cudaMemsetAsync(V, 0, 4 * kParams, s)) != cudaSuccess) fail(e, "zero v");
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  int step = 0;
  for (int ep = 0; ep < epochs && !rc; ++ep) {
    shuffle_keys_kernel<<<(n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096, 256, 0, s>>>(
        n, seed + 1315423911ull * (uint64_t)(ep + 1), keys, vals);
    if ((e = cudaGetLastError()) != cudaSuccess) {
      fail(e, "shuffle");
      break;
    }
    if ((e = cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, vals, vals2, (int64_t)n, 0, 64,
                                             s)) != cudaSuccess) {
      fail(e, "shuffle sort");
      break;
    }
    for (uint32_t b0 = 0; b0 < n && !rc; b0 += (uint32_t)batch) {
      const uint32_t bn = (n - b0) < (uint32_t)batch ? (n - b0) : (uint32_t)batch;
      rc = cost_gradients(P, d_x, d_y, vals2 + b0, bn, G, loss, part, pl, s);
      if (rc) break;
      ++step;
      const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
      mlp_adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(P, G, M, V, lr, b1, b2, eps, c1, c2);
      if ((e = cudaGetLastError()) != cudaSuccess) fail(e, "adam");
    }
  }
  if (!rc) {
    // final loss over the whole set
    float *fpart = nullptr, *fpl = nullptr;
    const int fb = (int)((n + kGradBlock - 1) / kGradBlock);
    if ((e = cudaMalloc(&fpart, 4 * (size_t)kParams * fb)) != cudaSuccess) fail(e, "final partials");
    if (!rc && (e = cudaMalloc(&fpl, 4 * (size_t)fb)) != cudaSuccess) fail(e, "final loss");
    if (!rc) rc = cost_gradients(P, d_x, d_y, nullptr, n, G, loss, fpart, fpl, s);
    if (!rc && final_loss && (e = cudaMemcpyAsync(final_loss, loss, 4, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      fail(e, "read loss");
    if (!rc && (e = cudaMemcpyAsync(params, P, 4 * kParams, cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      fail(e, "read params");
    if (!rc && (e = cudaStreamSynchronize(s)) != cudaSuccess) fail(e, "sync");
    cudaFree(fpart);
    cudaFree(fpl);
  }
  cudaFree(P);
  cudaFree(G);
  cudaFree(M);
  cudaFree(V);
  cudaFree(part);
  cudaFree(pl);
  cudaFree(loss);
  cudaFree(keys);
  cudaFree(keys2);
  cudaFree(vals);
  cudaFree(vals2);
  cudaFree(tmp);
  return rc;
}

}  // namespace gzb

using namespace gzb;

extern "C" int gzb_cost_model_param_count(void) { return kParams; }

extern "C" int gzb_cost_model_init(float *params, uint64_t seed) {
  GZB_CHECK(params, GZB_ERR_INVALID, "null params");
  // He-normal weights from a fixed generator (Box-Muller on splitmix64)
  uint64_t st = seed ^ 0x2545f4914f6cdd1dull;
  auto next = [&]() {
    uint64_t z = (st += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return (double)((z ^ (z >> 31)) >> 11) * (1.0 / 9007199254740992.0);
  };
  auto normal = [&]() {
    const double u1 = next() + 1e-300, u2 = next();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  };
  for (int i = 0; i < kParams; ++i) params[i] = 0.f;
  for (int i = 0; i < kHid * kFeat; ++i) params[kOffW1 + i] = (float)(normal() * std::sqrt(2.0 / kFeat));
  for (int i = 0; i < kHid * kHid; ++i) params[kOffW2 + i] = (float)(normal() * std::sqrt(2.0 / kHid));
  for (int i = 0; i < kHid; ++i) params[kOffW3 + i] = (float)(normal() * std::sqrt(1.0 / kHid));
  params[kOffB3] = 8.f;  // typical log2(cells) of an extension
  return GZB_OK;
}

extern "C" int gzb_cost_model_gradients(const float *d_params, const float *d_x,
                                        const float *d_y, uint32_t n, float *d_grad,
                                        float *d_loss, void *stream) {
  GZB_CHECK(d_params && d_x && d_y && d_grad && n > 0, GZB_ERR_INVALID, "null argument");
  cudaStream_t s = (cudaStream_t)stream;
  const int blocks = (int)((n + kGradBlock - 1) / kGradBlock);
  float *part = nullptr, *pl = nullptr;
  GZB_CUDA(cudaMalloc(&part, 4 * (size_t)kParams * blocks));
  cudaError_t e = cudaMalloc(&pl, 4 * (size_t)blocks);
  if (e != cudaSuccess) {
    cudaFree(part);
    return cuda_error(e, "partial loss", __FILE__, __LINE__);
  }
  int rc = cost_gradients(d_params, d_x, d_y, nullptr, n, d_grad, d_loss, part, pl, s);
  if (!rc) {
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_error(e, "sync", __FILE__, __LINE__);
  }
  cudaFree(part);
  cudaFree(pl);
  return rc;
}

extern "C" int gzb_cost_model_predict(const float *d_params, const float *d_x, uint32_t n,
                                      float *d_out, void *stream) {
  GZB_CHECK(d_params && d_x && d_out, GZB_ERR_INVALID, "null argument");
  return cost_predict(d_params, d_x, n, d_out, (cudaStream_t)stream, nullptr);
}

extern "C" int gzb_cost_model_train(const float *d_x, const float *d_y, uint32_t n,
                                    float *params, int epochs, int batch, float lr,
                                    uint64_t seed, float *final_loss, void *stream) {
  GZB_CHECK(d_x && d_y && params, GZB_ERR_INVALID, "null argument");
  return cost_train(d_x, d_y, n, params, epochs, batch, lr, seed, final_loss,
                    (cudaStream_t)stream);
}
