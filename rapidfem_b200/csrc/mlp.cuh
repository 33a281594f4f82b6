// mlp.cuh -- the small MLP of the learned ETD step controller: n_in -> H -> H
// -> n_out with tanh hidden layers and a linear output, trained by mean squared
// error with Adam, all on the device.
//
// Parameter vector (f32), in this order:
//   W1[H][n_in], b1[H], W2[H][H], b2[H], W3[n_out][H], b3[n_out]
// Forward: one block of H threads per sample, hidden unit per thread.
// Backward: per-sample gradients (one block per sample) into G[b][P], then a
// fixed-order reduction over the batch, so the gradient is deterministic.
#pragma once
#include <cstdint>

namespace dgtd {

constexpr int kMlpMaxIn = 64;
constexpr int kMlpMaxHidden = 128;
constexpr int kMlpMaxOut = 8;

struct MlpShape {
  int n_in, n_hidden, n_out;
  __host__ __device__ int o_w1() const { return 0; }
  __host__ __device__ int o_b1() const { return n_hidden * n_in; }
  __host__ __device__ int o_w2() const { return o_b1() + n_hidden; }
  __host__ __device__ int o_b2() const { return o_w2() + n_hidden * n_hidden; }
  __host__ __device__ int o_w3() const { return o_b2() + n_hidden; }
  __host__ __device__ int o_b3() const { return o_w3() + n_out * n_hidden; }
  __host__ __device__ int n_params() const { return o_b3() + n_out; }
};

// Forward for a batch: y[b][o]; the hidden activations a1, a2 [b][H] are kept
// for the backward pass when non-null.
__global__ void k_mlp_forward(MlpShape S, const float* __restrict__ p, const float* __restrict__ x, int64_t batch,
                              float* __restrict__ y, float* __restrict__ a1, float* __restrict__ a2) {
  __shared__ float sx[kMlpMaxIn], h1[kMlpMaxHidden], h2[kMlpMaxHidden];
  const int64_t b = blockIdx.x;
  if (b >= batch) return;
  const int k = threadIdx.x;
  for (int i = k; i < S.n_in; i += blockDim.x) sx[i] = x[b * S.n_in + i];
  __syncthreads();
  if (k < S.n_hidden) {
    float acc = p[S.o_b1() + k];
    const float* w = p + S.o_w1() + k * S.n_in;
    for (int i = 0; i < S.n_in; ++i) acc = fmaf(w[i], sx[i], acc);
    h1[k] = tanhf(acc);
    if (a1) a1[b * S.n_hidden + k] = h1[k];
  }
  __syncthreads();
  if (k < S.n_hidden) {
    float acc = p[S.o_b2() + k];
    const float* w = p + S.o_w2() + k * S.n_hidden;
    for (int i = 0; i < S.n_hidden; ++i) acc = fmaf(w[i], h1[i], acc);
    h2[k] = tanhf(acc);
    if (a2) a2[b * S.n_hidden + k] = h2[k];
  }
  __syncthreads();
  if (k < S.n_out) {
    float acc = p[S.o_b3() + k];
    const float* w = p + S.o_w3() + k * S.n_hidden;
    for (int i = 0; i < S.n_hidden; ++i) acc = fmaf(w[i], h2[i], acc);
    y[b * S.n_out + k] = acc;
  }
}

// Per-sample gradient of L = (1/B) sum_b sum_o (y_bo - t_bo)^2 into G[b][P];
// loss_b[b] = sum_o (y_bo - t_bo)^2.
__global__ void k_mlp_backward(MlpShape S, const float* __restrict__ p, const float* __restrict__ x,
                               const float* __restrict__ t, const float* __restrict__ y,
                               const float* __restrict__ a1, const float* __restrict__ a2, int64_t batch,
                               float* __restrict__ G, float* __restrict__ loss_b) {
  __shared__ float sx[kMlpMaxIn], h1[kMlpMaxHidden], h2[kMlpMaxHidden];
  __shared__ float d3[kMlpMaxOut], d2[kMlpMaxHidden], d1[kMlpMaxHidden];
  const int64_t b = blockIdx.x;
  if (b >= batch) return;
  const int k = threadIdx.x;
  const float inv_b = 1.0f / (float)batch;
  float* g = G + b * (int64_t)S.n_params();
  for (int i = k; i < S.n_in; i += blockDim.x) sx[i] = x[b * S.n_in + i];
  if (k < S.n_hidden) {
    h1[k] = a1[b * S.n_hidden + k];
    h2[k] = a2[b * S.n_hidden + k];
  }
  if (k < S.n_out) {
    const float r = y[b * S.n_out + k] - t[b * S.n_out + k];
    d3[k] = 2.0f * r * inv_b;
  }
  __syncthreads();
  if (k == 0) {
    float l = 0.f;
    for (int o = 0; o < S.n_out; ++o) {
      const float r = y[b * S.n_out + o] - t[b * S.n_out + o];
      l += r * r;
    }
    loss_b[b] = l;
  }
  // output layer
  if (k < S.n_hidden) {
    for (int o = 0; o < S.n_out; ++o) g[S.o_w3() + o * S.n_hidden + k] = d3[o] * h2[k];
    float s = 0.f;
    for (int o = 0; o < S.n_out; ++o) s = fmaf(p[S.o_w3() + o * S.n_hidden + k], d3[o], s);
    d2[k] = s * (1.0f - h2[k] * h2[k]);
  }
  if (k < S.n_out) g[S.o_b3() + k] = d3[k];
  __syncthreads();
  // second hidden layer
  if (k < S.n_hidden) {
    for (int i = 0; i < S.n_hidden; ++i) g[S.o_w2() + k * S.n_hidden + i] = d2[k] * h1[i];
    g[S.o_b2() + k] = d2[k];
    float s = 0.f;
    for (int j = 0; j < S.n_hidden; ++j) s = fmaf(p[S.o_w2() + j * S.n_hidden + k], d2[j], s);
    d1[k] = s * (1.0f - h1[k] * h1[k]);
  }
  __syncthreads();
  // first hidden layer
  if (k < S.n_hidden) {
    for (int i = 0; i < S.n_in; ++i) g[S.o_w1() + k * S.n_in + i] = d1[k] * sx[i];
    g[S.o_b1() + k] = d1[k];
  }
}

// grad[q] = sum_b G[b][q] in batch order; loss = (1/B) sum_b loss_b[b].
__global__ void k_mlp_reduce(const float* __restrict__ G, int64_t batch, int np, float* __restrict__ grad,
                             const float* __restrict__ loss_b, float* __restrict__ loss) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < np) {
    float s = 0.f;
    for (int64_t b = 0; b < batch; ++b) s += G[b * (int64_t)np + q];
    grad[q] = s;
  }
  if (q == 0 && loss) {
    float l = 0.f;
    for (int64_t b = 0; b < batch; ++b) l += loss_b[b];
    *loss = l / (float)batch;
  }
}

// Adam (Kingma & Ba 2015) with bias correction; step t >= 1.
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ grad, int np, float lr, float beta1, float beta2, float eps,
                           int t) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= np) return;
  const float g = grad[q];
  const float mq = beta1 * m[q] + (1.0f - beta1) * g;
  const float vq = beta2 * v[q] + (1.0f - beta2) * g * g;
  m[q] = mq;
  v[q] = vq;
  const float mh = mq / (1.0f - powf(beta1, (float)t));
  const float vh = vq / (1.0f - powf(beta2, (float)t));
  p[q] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace dgtd
