// mlp_kernels.cu — training and inference kernels of the schedule cost model.
//
// The cost model is a multilayer perceptron  x -> ReLU(x W1 + b1) -> ReLU(. W2 + b2)
// -> . w3 + b3  predicting the log run time of a fused pass under a schedule from
// the pass's features (op mix, stencil reach, dtypes, grid) and the schedule's
// (tile, threads, z-segment, boundary strategy). It is trained on the autotuner's
// own timings and only ranks schedules: results never depend on it.
//
// Parameters live in one FP32 buffer, layout (row-major):
//   W1[in][h], b1[h], W2[h][h], b2[h], w3[h], b3[1]
// Kernels are plain CUDA (the matrices are tiny: in <= 64, h = 64): one thread per
// output element, loops in a fixed order, no atomics — deterministic.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>

#include "../../include/stenpy_b200.h"

extern "C" void sten_internal_set_error(const char* msg);  // stenpy_abi.cu

namespace {

struct Layout {
  int in, h;
  size_t w1, b1, w2, b2, w3, b3, total;
};

Layout layout(int in, int h) {
  Layout L;
  L.in = in;
  L.h = h;
  L.w1 = 0;
  L.b1 = L.w1 + (size_t)in * h;
  L.w2 = L.b1 + h;
  L.b2 = L.w2 + (size_t)h * h;
  L.w3 = L.b2 + h;
  L.b3 = L.w3 + h;
  L.total = L.b3 + 1;
  return L;
}

// Y[r][o] = act(b[o] + sum_i X[r][i] W[i][o]); Z keeps the pre-activation.
__global__ void dense_fwd(const float* __restrict__ X, int n, int din, const float* __restrict__ W,
                          const float* __restrict__ b, int dout, float* __restrict__ Z, float* __restrict__ Y,
                          int relu) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * dout) return;
  const int r = (int)(t / dout), o = (int)(t - (long long)r * dout);
  const float* x = X + (size_t)r * din;
  float acc = b[o];
  for (int i = 0; i < din; ++i) acc = fmaf(x[i], W[(size_t)i * dout + o], acc);
  if (Z) Z[t] = acc;
  Y[t] = relu ? fmaxf(acc, 0.0f) : acc;
}

// dY for the output layer of the mean-squared error, and the loss terms.
__global__ void mse_grad(const float* __restrict__ pred, const float* __restrict__ target, int n,
                         float* __restrict__ dpred, float* __restrict__ sq) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const float d = pred[r] - target[r];
  dpred[r] = 2.0f * d / (float)n;
  sq[r] = d * d;
}

// dX[r][i] = sum_o dY[r][o] W[i][o], masked by relu'(Zx) when Zx is given.
__global__ void dense_bwd_input(const float* __restrict__ dY, int n, int dout, const float* __restrict__ W, int din,
                                const float* __restrict__ Zx, float* __restrict__ dX) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * din) return;
  const int r = (int)(t / din), i = (int)(t - (long long)r * din);
  const float* dy = dY + (size_t)r * dout;
  const float* w = W + (size_t)i * dout;
  float acc = 0.0f;
  for (int o = 0; o < dout; ++o) acc = fmaf(dy[o], w[o], acc);
  if (Zx && Zx[t] <= 0.0f) acc = 0.0f;
  dX[t] = acc;
}

// dW[i][o] = sum_r X[r][i] dY[r][o]; db[o] = sum_r dY[r][o]  (thread per weight, fixed row order)
__global__ void dense_bwd_weights(const float* __restrict__ X, const float* __restrict__ dY, int n, int din,
                                  int dout, float* __restrict__ dW, float* __restrict__ db) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nw = din * dout;
  if (t < nw) {
    const int i = t / dout, o = t - (t / dout) * dout;
    float acc = 0.0f;
    for (int r = 0; r < n; ++r) acc = fmaf(X[(size_t)r * din + i], dY[(size_t)r * dout + o], acc);
    dW[t] = acc;
  } else if (t < nw + dout) {
    const int o = t - nw;
    float acc = 0.0f;
    for (int r = 0; r < n; ++r) acc += dY[(size_t)r * dout + o];
    db[o] = acc;
  }
}

__global__ void sum_reduce(const float* __restrict__ x, int n, float* __restrict__ out) {
  __shared__ float s[256];
  float acc = 0.0f;
  for (int i = threadIdx.x; i < n; i += 256) acc += x[i];
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = s[0] / (float)n;
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float bc1,
                            float bc2, float wd) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t] + wd * p[t];
  const float mt = b1 * m[t] + (1.0f - b1) * gt;
  const float vt = b2 * v[t] + (1.0f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * (mt / bc1) / (sqrtf(vt / bc2) + eps);
}

inline unsigned blocks(long long n, int t = 256) { return (unsigned)((n + t - 1) / t); }

int check(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    static thread_local char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    sten_internal_set_error(buf);
    return STENPY_E_RUNTIME;
  }
  return STENPY_OK;
}

}  // namespace

extern "C" {

int stenpy_mlp_param_count(int in_dim, int hidden) {
  if (in_dim <= 0 || hidden <= 0) return -1;
  return (int)layout(in_dim, hidden).total;
}

int stenpy_mlp_workspace_floats(int n, int hidden) {
  if (n <= 0 || hidden <= 0) return -1;
  return 6 * n * hidden + 3 * n + 1;
}

int stenpy_mlp_forward(const float* params, int in_dim, int hidden, const float* X, int n, float* out,
                       float* workspace, void* stream) {
  if (!params || !X || !out || !workspace || n <= 0) {
    sten_internal_set_error("mlp_forward: bad argument");
    return STENPY_E_INVALID;
  }
  Layout L = layout(in_dim, hidden);
  cudaStream_t s = (cudaStream_t)stream;
  float* a1 = workspace;
  float* a2 = a1 + (size_t)n * hidden;
  dense_fwd<<<blocks((long long)n * hidden), 256, 0, s>>>(X, n, in_dim, params + L.w1, params + L.b1, hidden,
                                                           nullptr, a1, 1);
  dense_fwd<<<blocks((long long)n * hidden), 256, 0, s>>>(a1, n, hidden, params + L.w2, params + L.b2, hidden,
                                                           nullptr, a2, 1);
  dense_fwd<<<blocks(n), 256, 0, s>>>(a2, n, hidden, params + L.w3, params + L.b3, 1, nullptr, out, 0);
  return check("mlp_forward");
}

int stenpy_mlp_loss_grad(const float* params, int in_dim, int hidden, const float* X, const float* target, int n,
                         float* grad, float* loss, float* workspace, void* stream) {
  if (!params || !X || !target || !grad || !loss || !workspace || n <= 0) {
    sten_internal_set_error("mlp_loss_grad: bad argument");
    return STENPY_E_INVALID;
  }
  Layout L = layout(in_dim, hidden);
  cudaStream_t s = (cudaStream_t)stream;
  const size_t nh = (size_t)n * hidden;
  float* z1 = workspace;
  float* a1 = z1 + nh;
  float* z2 = a1 + nh;
  float* a2 = z2 + nh;
  float* d2 = a2 + nh;   // dL/dz2 (n x h)
  float* d1 = d2 + nh;   // dL/dz1 (n x h)
  float* pred = d1 + nh;
  float* dpred = pred + n;
  float* sq = dpred + n;
  dense_fwd<<<blocks((long long)nh), 256, 0, s>>>(X, n, in_dim, params + L.w1, params + L.b1, hidden, z1, a1, 1);
  dense_fwd<<<blocks((long long)nh), 256, 0, s>>>(a1, n, hidden, params + L.w2, params + L.b2, hidden, z2, a2, 1);
  dense_fwd<<<blocks(n), 256, 0, s>>>(a2, n, hidden, params + L.w3, params + L.b3, 1, nullptr, pred, 0);
  mse_grad<<<blocks(n), 256, 0, s>>>(pred, target, n, dpred, sq);
  sum_reduce<<<1, 256, 0, s>>>(sq, n, loss);
  // output layer: dw3 = a2^T dpred, db3 = sum dpred; d2 = dpred w3^T * relu'(z2)
  dense_bwd_weights<<<blocks(hidden + 1), 256, 0, s>>>(a2, dpred, n, hidden, 1, grad + L.w3, grad + L.b3);
  dense_bwd_input<<<blocks((long long)nh), 256, 0, s>>>(dpred, n, 1, params + L.w3, hidden, z2, d2);
  dense_bwd_weights<<<blocks((long long)hidden * hidden + hidden), 256, 0, s>>>(a1, d2, n, hidden, hidden,
                                                                               grad + L.w2, grad + L.b2);
  dense_bwd_input<<<blocks((long long)nh), 256, 0, s>>>(d2, n, hidden, params + L.w2, hidden, z1, d1);
  dense_bwd_weights<<<blocks((long long)in_dim * hidden + hidden), 256, 0, s>>>(X, d1, n, in_dim, hidden,
                                                                               grad + L.w1, grad + L.b1);
  return check("mlp_loss_grad");
}

int stenpy_adam_step(float* params, const float* grad, float* m, float* v, int n_params, float lr, float beta1,
                     float beta2, float eps, int step, float weight_decay, void* stream) {
  if (!params || !grad || !m || !v || n_params <= 0 || step <= 0) {
    sten_internal_set_error("adam_step: bad argument");
    return STENPY_E_INVALID;
  }
  const float bc1 = 1.0f - powf(beta1, (float)step), bc2 = 1.0f - powf(beta2, (float)step);
  adam_kernel<<<blocks(n_params), 256, 0, (cudaStream_t)stream>>>(params, grad, m, v, n_params, lr, beta1, beta2,
                                                                   eps, bc1, bc2, weight_decay);
  return check("adam_step");
}

}  // extern "C"
