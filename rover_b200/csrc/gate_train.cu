// gate_train.cu -- training kernels of the learned gate (5 -> 64 -> 64 -> 2).
//
// The forward pass reproduces the inference arithmetic of pq_batched.cu:
// standardised inputs, weights and hidden activations rounded to BF16,
// FP32 accumulation, ReLU hidden layers, two logits.  The backward pass
// treats the BF16 roundings as identity (gradients flow to the FP32 master
// weights).  Loss: per head, masked binary cross-entropy on the logit with a
// positive-class weight, averaged over the rows of the batch.
//
// Parameter vector (FP32, row-major [in][out]):
//   w1[5][64] b1[64] w2[64][64] b2[64] w3[64][2] b3[2]

#include <algorithm>
#include <cuda_bf16.h>

#include "kernels.h"

namespace rover {

constexpr int kP_W1 = 0;
constexpr int kP_B1 = kP_W1 + kGateIn * kGateHidden;
constexpr int kP_W2 = kP_B1 + kGateHidden;
constexpr int kP_B2 = kP_W2 + kGateHidden * kGateHidden;
constexpr int kP_W3 = kP_B2 + kGateHidden;
constexpr int kP_B3 = kP_W3 + kGateHidden * kGateOut;
constexpr int kGateParams = kP_B3 + kGateOut;
static_assert(kGateParams == 4674, "gate parameter count");

constexpr int kRows = 64;       // rows per block
constexpr int kHS = kGateHidden + 1;  // padded activation row

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float softplus(float z) { return z > 0.f ? z + log1pf(__expf(-z)) : log1pf(__expf(z)); }

// Column sums and sums of squares of x[n][5] (FP64 accumulation).
__global__ void gate_stats_kernel(const float* __restrict__ x, int64_t n, double* __restrict__ acc) {
  double s[kGateIn] = {}, s2[kGateIn] = {};
  for (int64_t r = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<int64_t>(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int i = 0; i < kGateIn; ++i) {
      const double v = x[r * kGateIn + i];
      s[i] += v;
      s2[i] += v * v;
    }
  }
#pragma unroll
  for (int i = 0; i < kGateIn; ++i) {
    double a = s[i], b = s2[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      a += __shfl_xor_sync(kFullMask, a, off);
      b += __shfl_xor_sync(kFullMask, b, off);
    }
    if ((threadIdx.x & 31) == 0) {
      atomicAdd(acc + i, a);
      atomicAdd(acc + kGateIn + i, b);
    }
  }
}

// Forward + backward for rows idx[0..n) (or 0..n when idx is null).  Adds
// the parameter gradients (already divided by `denom`) into grad and the
// loss sum into loss.
__global__ void __launch_bounds__(kRows) gate_fwd_bwd_kernel(const float* __restrict__ params,
                                                             const float* __restrict__ mu,
                                                             const float* __restrict__ sigma,
                                                             const float* __restrict__ x, const float* __restrict__ y,
                                                             const float* __restrict__ m,
                                                             const int64_t* __restrict__ idx, int64_t n,
                                                             float pw0, float pw1, float denom,
                                                             float* __restrict__ grad, double* __restrict__ loss) {
  extern __shared__ __align__(16) float sm[];
  float* W1 = sm;                                   // [5][64]
  float* W2 = W1 + kGateIn * kGateHidden;           // [64][64]
  float* W3 = W2 + kGateHidden * kGateHidden;       // [64][2]
  float* B1 = W3 + kGateHidden * kGateOut;
  float* B2 = B1 + kGateHidden;
  float* B3 = B2 + kGateHidden;                     // [2] (+2 pad)
  float* X = B3 + 4;                                // [64][5]
  float* H1 = X + kRows * kGateIn;                  // [64][65]
  float* H2 = H1 + kRows * kHS;
  float* DH1 = H2 + kRows * kHS;
  float* DH2 = DH1 + kRows * kHS;
  float* DZ = DH2 + kRows * kHS;                    // [64][2]
  const int t = threadIdx.x;
  for (int i = t; i < kGateIn * kGateHidden; i += kRows) W1[i] = bf16r(params[kP_W1 + i]);
  for (int i = t; i < kGateHidden * kGateHidden; i += kRows) W2[i] = bf16r(params[kP_W2 + i]);
  for (int i = t; i < kGateHidden * kGateOut; i += kRows) W3[i] = bf16r(params[kP_W3 + i]);
  for (int i = t; i < kGateHidden; i += kRows) {
    B1[i] = params[kP_B1 + i];
    B2[i] = params[kP_B2 + i];
  }
  if (t < kGateOut) B3[t] = params[kP_B3 + t];
  const int64_t r0 = static_cast<int64_t>(blockIdx.x) * kRows;
  const int64_t rr = r0 + t;
  const bool live = rr < n;
  const int64_t row = live ? (idx ? idx[rr] : rr) : 0;
  float lsum = 0.0f;
  __syncthreads();
  // forward
  float xin[kGateIn];
#pragma unroll
  for (int i = 0; i < kGateIn; ++i) {
    xin[i] = live ? bf16r((x[row * kGateIn + i] - mu[i]) / sigma[i]) : 0.0f;
    X[t * kGateIn + i] = xin[i];
  }
  for (int j = 0; j < kGateHidden; ++j) {
    float a = B1[j];
#pragma unroll
    for (int i = 0; i < kGateIn; ++i) a += xin[i] * W1[i * kGateHidden + j];
    H1[t * kHS + j] = a > 0.f ? bf16r(a) : 0.f;
  }
  for (int j = 0; j < kGateHidden; ++j) {
    float a = B2[j];
    for (int i = 0; i < kGateHidden; ++i) a += H1[t * kHS + i] * W2[i * kGateHidden + j];
    H2[t * kHS + j] = a > 0.f ? bf16r(a) : 0.f;
  }
  float z[kGateOut];
#pragma unroll
  for (int k = 0; k < kGateOut; ++k) {
    float a = B3[k];
    for (int i = 0; i < kGateHidden; ++i) a += H2[t * kHS + i] * W3[i * kGateOut + k];
    z[k] = a;
  }
  // masked weighted BCE and its logit gradient
#pragma unroll
  for (int k = 0; k < kGateOut; ++k) {
    float dz = 0.0f;
    if (live) {
      const float mk = m[row * kGateOut + k], yk = y[row * kGateOut + k];
      const float pw = k == 0 ? pw0 : pw1;
      if (mk != 0.0f) {
        lsum += mk * (pw * yk * softplus(-z[k]) + (1.0f - yk) * softplus(z[k]));
        const float sg = 1.0f / (1.0f + __expf(-z[k]));
        dz = mk * (pw * yk * (sg - 1.0f) + (1.0f - yk) * sg) / denom;
      }
    }
    DZ[t * kGateOut + k] = dz;
  }
  // backward through the hidden layers
  for (int j = 0; j < kGateHidden; ++j) {
    float a = 0.0f;
#pragma unroll
    for (int k = 0; k < kGateOut; ++k) a += DZ[t * kGateOut + k] * W3[j * kGateOut + k];
    DH2[t * kHS + j] = H2[t * kHS + j] > 0.f ? a : 0.f;
  }
  for (int j = 0; j < kGateHidden; ++j) {
    float a = 0.0f;
    for (int k = 0; k < kGateHidden; ++k) a += DH2[t * kHS + k] * W2[j * kGateHidden + k];
    DH1[t * kHS + j] = H1[t * kHS + j] > 0.f ? a : 0.f;
  }
  __syncthreads();
  // parameter gradients: thread t owns input unit t of W2 / W3 and output
  // unit t of W1 and the biases
  const int nr = static_cast<int>(n - r0 < kRows ? n - r0 : kRows);
  for (int j = 0; j < kGateHidden; ++j) {
    float a = 0.0f;
    for (int r = 0; r < nr; ++r) a += H1[r * kHS + t] * DH2[r * kHS + j];
    atomicAdd(grad + kP_W2 + t * kGateHidden + j, a);
  }
#pragma unroll
  for (int i = 0; i < kGateIn; ++i) {
    float a = 0.0f;
    for (int r = 0; r < nr; ++r) a += X[r * kGateIn + i] * DH1[r * kHS + t];
    atomicAdd(grad + kP_W1 + i * kGateHidden + t, a);
  }
#pragma unroll
  for (int k = 0; k < kGateOut; ++k) {
    float a = 0.0f;
    for (int r = 0; r < nr; ++r) a += H2[r * kHS + t] * DZ[r * kGateOut + k];
    atomicAdd(grad + kP_W3 + t * kGateOut + k, a);
  }
  {
    float a1 = 0.0f, a2 = 0.0f;
    for (int r = 0; r < nr; ++r) {
      a1 += DH1[r * kHS + t];
      a2 += DH2[r * kHS + t];
    }
    atomicAdd(grad + kP_B1 + t, a1);
    atomicAdd(grad + kP_B2 + t, a2);
  }
  if (t < kGateOut) {
    float a = 0.0f;
    for (int r = 0; r < nr; ++r) a += DZ[r * kGateOut + t];
    atomicAdd(grad + kP_B3 + t, a);
  }
  // loss
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) lsum += __shfl_xor_sync(kFullMask, lsum, off);
  if ((t & 31) == 0) atomicAdd(loss, static_cast<double>(lsum));
}

// Adam with decoupled weight decay on the FP32 master parameters.
__global__ void gate_adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                                 float* __restrict__ m2, int count, float lr, float b1, float b2, float eps,
                                 float wd, float bc1, float bc2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.0f - b1) * gi;
  const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = v;
  p[i] -= lr * ((a / bc1) / (sqrtf(v / bc2) + eps) + wd * p[i]);
}

size_t gate_fwd_bwd_smem() {
  return sizeof(float) * (kGateIn * kGateHidden + kGateHidden * kGateHidden + kGateHidden * kGateOut +
                          2 * kGateHidden + 4 + kRows * kGateIn + 4 * kRows * kHS + kRows * kGateOut);
}

void launch_gate_stats(const float* x, int64_t n, double* acc, cudaStream_t s) {
  const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 148 * 8));
  gate_stats_kernel<<<std::max(1, blocks), 256, 0, s>>>(x, n, acc);
}

cudaError_t launch_gate_fwd_bwd(const float* params, const float* mu, const float* sigma, const float* x,
                                const float* y, const float* m, const int64_t* idx, int64_t n, float pw0, float pw1,
                                float denom, float* grad, double* loss, cudaStream_t s) {
  static bool configured = false;
  const size_t smem = gate_fwd_bwd_smem();
  if (!configured) {
    const cudaError_t e = cudaFuncSetAttribute(gate_fwd_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const int64_t blocks = (n + kRows - 1) / kRows;
  gate_fwd_bwd_kernel<<<static_cast<unsigned>(blocks), kRows, smem, s>>>(params, mu, sigma, x, y, m, idx, n, pw0,
                                                                         pw1, denom, grad, loss);
  return cudaGetLastError();
}

void launch_gate_adam(float* p, const float* g, float* m1, float* m2, int count, float lr, float b1, float b2,
                      float eps, float wd, float bc1, float bc2, cudaStream_t s) {
  gate_adam_kernel<<<(count + 255) / 256, 256, 0, s>>>(p, g, m1, m2, count, lr, b1, b2, eps, wd, bc1, bc2);
}

}  // namespace rover
