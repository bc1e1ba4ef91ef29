// Learned auxiliary-field proposal (sm_100a): a small MLP that proposes the grid point of a
// coupling from environment features, its online training on pairs the grid walk generates,
// and the in-sweep inference.  No counterpart in the reference, whose PropagateSeparately
// samples the exact grid PDF (MPSQMC2.cpp:551-588).
//
// Network: features f (32) -> relu(f W1 + b1) (128) -> relu(. W2 + b2) (128) -> z = . W3 + b3 (G)
// -> q = softmax(z).  Parameters form one flat FP32 vector, W input-major (W[i * out + o]):
// W1 32x128, b1, W2 128x128, b2, W3 128xG, b3.  The sweep reads a BF16 copy (FP32 accumulation);
// training keeps the FP32 master, Adam moments and gradients in the same layout.
//
// Features of coupling (i, j) (both scale-free): 4 C_kl / ov, the 16 coefficients of the overlap
// ratio rho(x) = <Psi_T|B(x)phi> / <Psi_T|phi> = sum_kl f_kl x_k x_l, and 4 M / ov, the 16 closures
// of the left and right environment branches the C_kl are formed from.
//
// Use in the walk (exact-ratio reweighting, so the estimator stays unbiased): the exact PDF
// P(x) = max(0, rho(x)) / G over the grid is still formed; the network's q is restricted to the
// support of P (q~ = q [P > 0] / sum), the point is drawn from q~ with the walker's uniform by the
// same CDF scan, and the weight is multiplied by P(x) / q~(x) instead of sum_x P(x).  With q~ = P /
// sum P this is the grid method exactly; every other q~ adds variance, so the grid PDF is both
// the fallback and the yardstick the network is trained towards (loss KL(P / sum P || q)).
#pragma once

#include <cuda_bf16.h>

#include "walker_kernels.cuh"

namespace mq {

constexpr int kMlpIn = 32, kMlpHid = 128, kMlpMaxOut = 256;

__host__ __device__ inline long mlp_off_b1() { return (long)kMlpIn * kMlpHid; }
__host__ __device__ inline long mlp_off_w2() { return mlp_off_b1() + kMlpHid; }
__host__ __device__ inline long mlp_off_b2() { return mlp_off_w2() + (long)kMlpHid * kMlpHid; }
__host__ __device__ inline long mlp_off_w3() { return mlp_off_b2() + kMlpHid; }
__host__ __device__ inline long mlp_off_b3(int G) { return mlp_off_w3() + (long)kMlpHid * G; }
__host__ __device__ inline long mlp_params(int G) { return mlp_off_b3(G) + G; }

// Forward pass of one feature vector by the whole CTA.  f: 32 floats (smem); h: 2 x 128 floats
// and part: 2 x 128 floats of smem scratch; z: G floats (smem) on exit.  Starts after a barrier
// the caller placed behind f; ends with a barrier.
__device__ __forceinline__ void mlp_forward_cta(const __nv_bfloat16 *__restrict__ wb, int G, const float *f,
                                                float *h, float *part, float *z) {
  const int tid = threadIdx.x;
  const int o = tid & (kMlpHid - 1), half = tid >> 7;  // 256 threads: two halves of the input range
  {
    const __nv_bfloat16 *W1 = wb;
    float a = 0.f;
#pragma unroll 4
    for (int i = half * (kMlpIn / 2); i < (half + 1) * (kMlpIn / 2); ++i)
      a += __bfloat162float(W1[i * kMlpHid + o]) * f[i];
    part[half * kMlpHid + o] = a;
  }
  __syncthreads();
  if (tid < kMlpHid)
    h[tid] = fmaxf(part[tid] + part[kMlpHid + tid] + __bfloat162float(wb[mlp_off_b1() + tid]), 0.f);
  __syncthreads();
  {
    const __nv_bfloat16 *W2 = wb + mlp_off_w2();
    float a = 0.f;
#pragma unroll 8
    for (int i = half * (kMlpHid / 2); i < (half + 1) * (kMlpHid / 2); ++i)
      a += __bfloat162float(W2[i * kMlpHid + o]) * h[i];
    part[half * kMlpHid + o] = a;
  }
  __syncthreads();
  if (tid < kMlpHid)
    h[kMlpHid + tid] = fmaxf(part[tid] + part[kMlpHid + tid] + __bfloat162float(wb[mlp_off_b2() + tid]), 0.f);
  __syncthreads();
  {
    const __nv_bfloat16 *W3 = wb + mlp_off_w3();
    for (int x = tid; x < G; x += kThreads) {
      float a = __bfloat162float(wb[mlp_off_b3(G) + x]);
#pragma unroll 8
      for (int i = 0; i < kMlpHid; ++i) a += __bfloat162float(W3[(long)i * G + x]) * h[kMlpHid + i];
      z[x] = a;
    }
  }
  __syncthreads();
}

#ifndef MQ_DEVICE_ONLY

// ------------------------------------------------------------------------------------------
// Training kernels (one launch each, captured into the step's graph when training is on).
// Row-major matrices; the batch size is read from device memory (*Bdev), grids are sized for
// the capacity and blocks beyond the batch return at once.
// ------------------------------------------------------------------------------------------

// C (M x N, ldc) = op(A) op(B) (+ bias[n]) (relu), or += when accumulate.  A(m, k) = ta ?
// A[k * lda + m] : A[m * lda + k]; B(k, n) = tb ? B[n * ldb + k] : B[k * ldb + n].  M, N or K may
// be the batch size: mdev / kdev (nullable) override M / K from device memory.  64x64 tiles,
// 16-deep K slices, 4x4 outputs per thread; FP32 throughout.
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const int *mdev, const int *kdev,
                                                       const float *A, int lda, int ta, const float *B, int ldb,
                                                       int tb, float *C, int ldc, const float *bias, int relu) {
  if (mdev) M = *mdev;
  if (kdev) K = *kdev;
  const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
  if (m0 >= M || n0 >= N) return;
  __shared__ float As[16][65], Bs[16][65];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      const int kk = e & 15, mm = e >> 4;
      const int m = m0 + mm, k = k0 + kk;
      As[kk][mm] = (m < M && k < K) ? (ta ? A[(long)k * lda + m] : A[(long)m * lda + k]) : 0.f;
      const int nn = e >> 4, n = n0 + nn;
      Bs[kk][nn] = (n < N && k < K) ? (tb ? B[(long)n * ldb + k] : B[(long)k * ldb + n]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a[u] = As[kk][ty + 16 * u];
        b[u] = Bs[kk][tx + 16 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] += a[u] * b[v];
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int m = m0 + ty + 16 * u, n = n0 + tx + 16 * v;
      if (m < M && n < N) {
        float r = acc[u][v] + (bias ? bias[n] : 0.f);
        if (relu) r = fmaxf(r, 0.f);
        C[(long)m * ldc + n] = r;
      }
    }
}

// Per row of the batch: q = softmax(z), dZ = (q - p) / B, loss += sum p (log p - log q) / B.
// One warp per row.  loss: one double, zeroed by the caller.
__global__ void __launch_bounds__(256) mlp_softmax_grad_kernel(const int *Bdev, int G, const float *Z,
                                                               const float *P, float *dZ, double *loss) {
  const int B = *Bdev;
  const int row = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= B) return;
  const float *z = Z + (long)row * G, *p = P + (long)row * G;
  float mx = -INFINITY;
  for (int x = lane; x < G; x += 32) mx = fmaxf(mx, z[x]);
  for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  float se = 0.f;
  for (int x = lane; x < G; x += 32) se += expf(z[x] - mx);
  for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
  const float lse = mx + logf(se);
  double l = 0.0;
  const float invB = 1.f / (float)B;
  for (int x = lane; x < G; x += 32) {
    const float lq = z[x] - lse;
    dZ[(long)row * G + x] = (expf(lq) - p[x]) * invB;
    if (p[x] > 0.f) l += (double)p[x] * ((double)logf(p[x]) - (double)lq);
  }
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if (lane == 0) atomicAdd(loss, l / B);
}

// dH *= (H > 0), B x n.
__global__ void mlp_relu_back_kernel(const int *Bdev, int n, const float *H, float *dH) {
  const long total = (long)(*Bdev) * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x)
    if (H[e] <= 0.f) dH[e] = 0.f;
}

// g[n] = sum over the batch rows of D[., n].
__global__ void mlp_colsum_kernel(const int *Bdev, int n, const float *D, float *g) {
  const int B = *Bdev;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  float s = 0.f;
  for (int r = 0; r < B; ++r) s += D[(long)r * n + col];
  g[col] = s;
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 master; refreshes the BF16 copy the sweep
// reads.  t: update counter (device), incremented by block 0 after the grid finished reading it
// (the kernel reads it once per thread; the increment is a separate single-thread launch).
__global__ void mlp_adam_kernel(long n, float lr, const int *t, const float *g, float *w, float *m, float *v,
                                __nv_bfloat16 *wb) {
  const int step = *t + 1;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f / (1.f - powf(b1, (float)step)), c2 = 1.f / (1.f - powf(b2, (float)step));
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const float gi = g[e];
    const float mi = b1 * m[e] + (1.f - b1) * gi, vi = b2 * v[e] + (1.f - b2) * gi * gi;
    m[e] = mi;
    v[e] = vi;
    const float wi = w[e] - lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
    w[e] = wi;
    wb[e] = __float2bfloat16(wi);
  }
}

__global__ void mlp_count_kernel(int *t) { *t += 1; }

__global__ void mlp_to_bf16_kernel(long n, const float *w, __nv_bfloat16 *wb) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
    wb[e] = __float2bfloat16(w[e]);
}

#endif  // MQ_DEVICE_ONLY

}  // namespace mq
