// The quasiparticle-shift network: 4 -> H -> H -> 1 perceptron with SiLU,
// FP32, H <= 64. Forward: one thread per sample with the parameters staged
// in shared memory. Backward: a block of 32 samples stages its per-sample
// error vectors in shared memory and reduces the weight gradients over them
// before one atomic add per parameter and block. AdamW: elementwise.
#include <cmath>

#include "common.cuh"

namespace mbpt {
namespace {

constexpr int kMaxH = 64;
constexpr int kIn = 4;
constexpr int kTile = 32;  // samples per backward block

__host__ __device__ inline int param_count(int H) { return H * H + 7 * H + 1; }

struct Off {
  int W1, b1, W2, b2, W3, b3;
  __host__ __device__ explicit Off(int H)
      : W1(0), b1(H * kIn), W2(H * kIn + H), b2(H * kIn + H + H * H),
        W3(H * kIn + 2 * H + H * H), b3(H * kIn + 3 * H + H * H) {}
};

__device__ __forceinline__ float sigm(float z) { return 1.f / (1.f + expf(-z)); }

__global__ void mlp_forward_kernel(const float *params, int H, const float *x, int B, float *y,
                                   float *act) {
  extern __shared__ float sp[];
  const int np = param_count(H);
  for (int i = threadIdx.x; i < np; i += blockDim.x) sp[i] = params[i];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= B) return;
  const Off o(H);
  float xi[kIn];
  for (int k = 0; k < kIn; ++k) xi[k] = x[s * kIn + k];
  float h1[kMaxH], h2[kMaxH];
  float *a = act ? act + static_cast<int64_t>(s) * 4 * H : nullptr;
  for (int i = 0; i < H; ++i) {
    float z = sp[o.b1 + i];
    for (int k = 0; k < kIn; ++k) z = fmaf(sp[o.W1 + i * kIn + k], xi[k], z);
    h1[i] = z * sigm(z);
    if (a) {
      a[i] = z;
      a[H + i] = h1[i];
    }
  }
  float out = sp[o.b3];
  for (int i = 0; i < H; ++i) {
    float z = sp[o.b2 + i];
    for (int j = 0; j < H; ++j) z = fmaf(sp[o.W2 + i * H + j], h1[j], z);
    h2[i] = z * sigm(z);
    if (a) {
      a[2 * H + i] = z;
      a[3 * H + i] = h2[i];
    }
    out = fmaf(sp[o.W3 + i], h2[i], out);
  }
  y[s] = out;
}

__global__ void mlp_backward_kernel(const float *params, int H, const float *x, int B,
                                    const float *act, const float *y, const float *t,
                                    float *grad, float *loss) {
  __shared__ float W3s[kMaxH];
  __shared__ float dz1[kTile][kMaxH + 1];
  __shared__ float dz2[kTile][kMaxH + 1];
  __shared__ float h1s[kTile][kMaxH + 1];
  __shared__ float h2s[kTile][kMaxH + 1];
  __shared__ float xs[kTile][kIn];
  __shared__ float dys[kTile];
  const Off o(H);
  for (int i = threadIdx.x; i < H; i += blockDim.x) W3s[i] = params[o.W3 + i];
  __syncthreads();
  const int s0 = blockIdx.x * kTile;
  const int ls = threadIdx.x;  // local sample
  const int s = s0 + ls;
  const float invB = 1.f / static_cast<float>(B);
  if (s < B) {
    const float *a = act + static_cast<int64_t>(s) * 4 * H;
    const float diff = y[s] - t[s];
    const float dy = diff * invB;
    atomicAdd(loss, 0.5f * diff * diff * invB);
    dys[ls] = dy;
    for (int k = 0; k < kIn; ++k) xs[ls][k] = x[s * kIn + k];
    for (int i = 0; i < H; ++i) {
      h1s[ls][i] = a[H + i];
      h2s[ls][i] = a[3 * H + i];
      const float z2 = a[2 * H + i];
      const float sg = sigm(z2);
      dz2[ls][i] = dy * W3s[i] * sg * (1.f + z2 * (1.f - sg));
    }
    for (int j = 0; j < H; ++j) {
      float g = 0.f;
      for (int i = 0; i < H; ++i) g = fmaf(__ldg(params + o.W2 + i * H + j), dz2[ls][i], g);
      const float z1 = a[j];
      const float sg = sigm(z1);
      dz1[ls][j] = g * sg * (1.f + z1 * (1.f - sg));
    }
  } else {
    dys[ls] = 0.f;
    for (int k = 0; k < kIn; ++k) xs[ls][k] = 0.f;
    for (int i = 0; i < H; ++i) {
      h1s[ls][i] = h2s[ls][i] = dz1[ls][i] = dz2[ls][i] = 0.f;
    }
  }
  __syncthreads();
  // thread i reduces row i of every weight matrix over the block's samples
  for (int i = threadIdx.x; i < H; i += blockDim.x) {
    float db1 = 0.f, db2 = 0.f, dw3 = 0.f;
    float dw1[kIn] = {0.f, 0.f, 0.f, 0.f};
    for (int q = 0; q < kTile; ++q) {
      db1 += dz1[q][i];
      db2 += dz2[q][i];
      dw3 = fmaf(dys[q], h2s[q][i], dw3);
      for (int k = 0; k < kIn; ++k) dw1[k] = fmaf(dz1[q][i], xs[q][k], dw1[k]);
    }
    atomicAdd(grad + o.b1 + i, db1);
    atomicAdd(grad + o.b2 + i, db2);
    atomicAdd(grad + o.W3 + i, dw3);
    for (int k = 0; k < kIn; ++k) atomicAdd(grad + o.W1 + i * kIn + k, dw1[k]);
    for (int j = 0; j < H; ++j) {
      float g = 0.f;
      for (int q = 0; q < kTile; ++q) g = fmaf(dz2[q][i], h1s[q][j], g);
      atomicAdd(grad + o.W2 + i * H + j, g);
    }
  }
  if (threadIdx.x == 0) {
    float db3 = 0.f;
    for (int q = 0; q < kTile; ++q) db3 += dys[q];
    atomicAdd(grad + o.b3, db3);
  }
}

__global__ void adamw_kernel(float *p, const float *g, float *m, float *v, int n, float lr,
                             float b1, float b2, float eps, float wd, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / c1, vh = vi / c2;
  p[i] -= lr * (mh / (sqrtf(vh) + eps) + wd * p[i]);
}

}  // namespace
}  // namespace mbpt

using namespace mbpt;

extern "C" {

int mbpt_mlp_param_count(int hidden) { return param_count(hidden); }

int mbpt_mlp_forward(const float *params, int H, const float *x, int B, float *y, float *act,
                     void *stream) {
  if (H < 1 || H > kMaxH || B < 0) return MBPT_ERR_SHAPE;
  if (B == 0) return MBPT_OK;
  const size_t smem = sizeof(float) * param_count(H);
  count_launch(); mlp_forward_kernel<<<(B + 127) / 128, 128, smem, reinterpret_cast<cudaStream_t>(stream)>>>(
      params, H, x, B, y, act);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int mbpt_mlp_backward(const float *params, int H, const float *x, int B, const float *act,
                      const float *y, const float *t, float *grad, float *loss, void *stream) {
  if (H < 1 || H > kMaxH || B < 1) return MBPT_ERR_SHAPE;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaMemsetAsync(grad, 0, sizeof(float) * param_count(H), st);
  cudaMemsetAsync(loss, 0, sizeof(float), st);
  count_launch(); mlp_backward_kernel<<<(B + kTile - 1) / kTile, kTile, 0, st>>>(params, H, x, B, act, y, t,
                                                                 grad, loss);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

int mbpt_mlp_adamw(float *p, const float *g, float *m, float *v, int n, float lr, float b1,
                   float b2, float eps, float wd, int step, void *stream) {
  if (n < 1 || step < 1) return MBPT_ERR_SHAPE;
  const float c1 = 1.f - powf(b1, static_cast<float>(step));
  const float c2 = 1.f - powf(b2, static_cast<float>(step));
  count_launch(); adamw_kernel<<<(n + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      p, g, m, v, n, lr, b1, b2, eps, wd, c1, c2);
  return cudaGetLastError() == cudaSuccess ? MBPT_OK : MBPT_ERR_CUDA;
}

}  // extern "C"
