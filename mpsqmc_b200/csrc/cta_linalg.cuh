// CTA-cooperative FP64 dense linear algebra for the walker kernels (sm_100a).
//
// All matrices are column-major with an explicit leading dimension and may live in shared or
// global memory (generic pointers).  Every routine is called by all threads of the CTA and
// returns without a trailing barrier unless stated; callers place __syncthreads() between
// dependent calls.
//
// FP64 products use the tensor-core DMMA instruction mma.sync.m8n8k4.f64 (tcgen05 has no f64
// kind, so this is Blackwell's FP64 tensor path).  Fragment layouts follow the PTX ISA for
// .f64 m8n8k4: A (8x4, row): lane holds A[lane>>2][lane&3]; B (4x8, col): B[lane&3][lane>>2];
// C/D (8x8): C[lane>>2][2*(lane&3) + i], i = 0,1.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mq {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

// Check-free path for M, N, K multiples of 16: each warp computes 16x16 blocks; the K loop runs
// in chunks of four k-steps whose 16 fragment loads are issued one chunk ahead of the DMMAs.
template <bool TA, bool TB>
static __device__ __forceinline__ void gemm16(int M, int N, int K, double alpha, const double *A, int lda,
                                              const double *B, int ldb, double beta, double *C, int ldc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int bm = M >> 4, bn = N >> 4;
  const long sa = TA ? 4 : 4L * lda, sb = TB ? 4L * ldb : 4;
  for (int blk = warp; blk < bm * bn; blk += kWarps) {
    const int m0 = (blk % bm) << 4, n0 = (blk / bm) << 4;
    const int ma = m0 + g, mb = m0 + 8 + g, na = n0 + g, nb = n0 + 8 + g;
    const double *pa0 = TA ? A + (long)lda * ma + t : A + ma + (long)lda * t;
    const double *pa1 = TA ? A + (long)lda * mb + t : A + mb + (long)lda * t;
    const double *pb0 = TB ? B + na + (long)ldb * t : B + t + (long)ldb * na;
    const double *pb1 = TB ? B + nb + (long)ldb * t : B + t + (long)ldb * nb;
    double acc[2][2][2] = {{{0.0, 0.0}, {0.0, 0.0}}, {{0.0, 0.0}, {0.0, 0.0}}};
    double a0[4], a1[4], b0[4], b1[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      a0[u] = pa0[u * sa];
      a1[u] = pa1[u * sa];
      b0[u] = pb0[u * sb];
      b1[u] = pb1[u * sb];
    }
    for (int k0 = 0; k0 < K; k0 += 16) {
      double c0[4], c1[4], d0[4], d1[4];
      const bool more = k0 + 16 < K;
      const long off = (long)(k0 / 4 + 4);
      if (more) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          c0[u] = pa0[(off + u) * sa];
          c1[u] = pa1[(off + u) * sa];
          d0[u] = pb0[(off + u) * sb];
          d1[u] = pb1[(off + u) * sb];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        dmma884(acc[0][0][0], acc[0][0][1], a0[u], b0[u]);
        dmma884(acc[0][1][0], acc[0][1][1], a0[u], b1[u]);
        dmma884(acc[1][0][0], acc[1][0][1], a1[u], b0[u]);
        dmma884(acc[1][1][0], acc[1][1][1], a1[u], b1[u]);
      }
      if (more) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          a0[u] = c0[u];
          a1[u] = c1[u];
          b0[u] = d0[u];
          b1[u] = d1[u];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          double *c = C + (m0 + 8 * i + g) + (long)ldc * (n0 + 8 * j + 2 * t + e);
          const double v = alpha * acc[i][j][e];
          *c = (beta == 0.0) ? v : v + beta * (*c);
        }
  }
}

// C (M x N, ldc) = alpha * op(A) * op(B) + beta * C, op(A) M x K, op(B) K x N.
//   ta == false: A[m + lda*k];  ta == true: A[k + lda*m]
//   tb == false: B[k + ldb*n];  tb == true: B[n + ldb*k]
// Each warp owns 16x16 output blocks (2x2 DMMA tiles).  When M, N and K are multiples of 16 the
// check-free gemm16 path runs; otherwise element bounds are checked, so any M, N, K >= 0 is
// valid.  Output element (m, n) is always written by the same thread for a given (M, N), so two
// calls with the same M, N may accumulate into C without a barrier.
static __device__ __noinline__ void cta_gemm(int M, int N, int K, double alpha, const double *A, int lda,
                                      bool ta, const double *B, int ldb, bool tb, double beta,
                                      double *C, int ldc) {
  if (((M | N | K) & 15) == 0) {
    if (ta) {
      if (tb) gemm16<true, true>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
      else gemm16<true, false>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    } else {
      if (tb) gemm16<false, true>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
      else gemm16<false, false>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    }
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int bm = (M + 15) >> 4, bn = (N + 15) >> 4;
  for (int blk = warp; blk < bm * bn; blk += kWarps) {
    const int m0 = (blk % bm) << 4, n0 = (blk / bm) << 4;
    double acc[2][2][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int ma = m0 + g, mb = m0 + 8 + g;
    const int na = n0 + g, nb = n0 + 8 + g;
    for (int k0 = 0; k0 < K; k0 += 4) {
      const int k = k0 + t;
      const bool kin = k < K;
      double a0 = 0.0, a1 = 0.0, b0 = 0.0, b1 = 0.0;
      if (kin) {
        if (ma < M) a0 = ta ? A[k + (long)lda * ma] : A[ma + (long)lda * k];
        if (mb < M) a1 = ta ? A[k + (long)lda * mb] : A[mb + (long)lda * k];
        if (na < N) b0 = tb ? B[na + (long)ldb * k] : B[k + (long)ldb * na];
        if (nb < N) b1 = tb ? B[nb + (long)ldb * k] : B[k + (long)ldb * nb];
      }
      dmma884(acc[0][0][0], acc[0][0][1], a0, b0);
      dmma884(acc[0][1][0], acc[0][1][1], a0, b1);
      dmma884(acc[1][0][0], acc[1][0][1], a1, b0);
      dmma884(acc[1][1][0], acc[1][1][1], a1, b1);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int m = m0 + 8 * i + g, n = n0 + 8 * j + 2 * t + e;
          if (m < M && n < N) {
            double *c = C + m + (long)ldc * n;
            const double v = alpha * acc[i][j][e];
            *c = (beta == 0.0) ? v : v + beta * (*c);
          }
        }
  }
}

// Sixteen closures of two-site branch products, fused with the GEMM that forms them:
//   out[k + 4 (s + 2 t)] = sum_{m < M, n < N} (A_s B_t)[m, n] P_k[m, n],   s, t in {0, 1}, k < 4,
// A_s = A + s*sa (M x K, ld lda), B_t = B + t*sb (K x N, ld ldb), P_k = P + k*sp (ld ldp).
// The products A_s B_t are never stored: each warp multiplies its 16x16 output blocks by the four
// P blocks in the DMMA epilogue, and one CTA reduction writes the 16 sums to out (shared memory).
// FAST requires M, N, K multiples of 16 (fragments loaded a chunk of four k-steps at a time);
// otherwise every element access is bounds-checked.  red: >= 16*kWarps doubles.  Starts and ends with a
// barrier inside the reduction.
template <bool FAST>
static __device__ __noinline__ void cta_closure16(int M, int N, int K, const double *A, int lda, long sa,
                                                  const double *B, int ldb, long sb, const double *P, int ldp,
                                                  long sp, double *red, double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int bm = (M + 15) >> 4, bn = (N + 15) >> 4;
  double v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = 0.0;
  for (int blk = warp; blk < bm * bn; blk += kWarps) {
    const int m0 = (blk % bm) << 4, n0 = (blk / bm) << 4;
    const int ma = m0 + g, mb = m0 + 8 + g, na = n0 + g, nb = n0 + 8 + g;
#pragma unroll 1
    for (int s = 0; s < 2; ++s) {
      const double *As = A + s * sa;
      double acc[2][2][2][2], w[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) w[q] = 0.0;
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 2; ++j) acc[u][i][j][0] = acc[u][i][j][1] = 0.0;
      if (FAST) {
        // per chunk of four k-steps: all fragment loads first, then the 32 DMMAs
        const double *pa0 = As + ma + (long)lda * t, *pa1 = As + mb + (long)lda * t;
        const double *pb00 = B + t + (long)ldb * na, *pb01 = B + t + (long)ldb * nb;
        const double *pb10 = pb00 + sb, *pb11 = pb01 + sb;
        const long sA = 4L * lda;
        for (int k0 = 0; k0 < K; k0 += 16) {
          const int off = k0 / 4;
          double a0[4], a1[4], b00[4], b01[4], b10[4], b11[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            a0[u] = pa0[(off + u) * sA];
            a1[u] = pa1[(off + u) * sA];
            b00[u] = pb00[4 * (off + u)];
            b01[u] = pb01[4 * (off + u)];
            b10[u] = pb10[4 * (off + u)];
            b11[u] = pb11[4 * (off + u)];
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            dmma884(acc[0][0][0][0], acc[0][0][0][1], a0[u], b00[u]);
            dmma884(acc[0][0][1][0], acc[0][0][1][1], a0[u], b01[u]);
            dmma884(acc[0][1][0][0], acc[0][1][0][1], a1[u], b00[u]);
            dmma884(acc[0][1][1][0], acc[0][1][1][1], a1[u], b01[u]);
            dmma884(acc[1][0][0][0], acc[1][0][0][1], a0[u], b10[u]);
            dmma884(acc[1][0][1][0], acc[1][0][1][1], a0[u], b11[u]);
            dmma884(acc[1][1][0][0], acc[1][1][0][1], a1[u], b10[u]);
            dmma884(acc[1][1][1][0], acc[1][1][1][1], a1[u], b11[u]);
          }
        }
      } else {
        for (int k0 = 0; k0 < K; k0 += 4) {
          const int k = k0 + t;
          const bool kin = k < K;
          double a0 = 0.0, a1 = 0.0, b[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
          if (kin) {
            if (ma < M) a0 = As[ma + (long)lda * k];
            if (mb < M) a1 = As[mb + (long)lda * k];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              if (na < N) b[u][0] = B[u * sb + k + (long)ldb * na];
              if (nb < N) b[u][1] = B[u * sb + k + (long)ldb * nb];
            }
          }
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            dmma884(acc[u][0][0][0], acc[u][0][0][1], a0, b[u][0]);
            dmma884(acc[u][0][1][0], acc[u][0][1][1], a0, b[u][1]);
            dmma884(acc[u][1][0][0], acc[u][1][0][1], a1, b[u][0]);
            dmma884(acc[u][1][1][0], acc[u][1][1][1], a1, b[u][1]);
          }
        }
      }
      // epilogue: dot the product blocks with the four P blocks
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int m = m0 + 8 * i + g, n = n0 + 8 * j + 2 * t + e;
            if (FAST || (m < M && n < N)) {
              const double *pp = P + m + (long)ldp * n;
#pragma unroll
              for (int k = 0; k < 4; ++k) {
                const double pk = pp[k * sp];
                w[k] += acc[0][i][j][e] * pk;
                w[k + 4] += acc[1][i][j][e] * pk;
              }
            }
          }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (s == 0) {
          v[k] += w[k];
          v[k + 8] += w[k + 4];
        } else {
          v[k + 4] += w[k];
          v[k + 12] += w[k + 4];
        }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 16; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 16; ++q) red[q * kWarps + warp] = v[q];
  __syncthreads();
  if (threadIdx.x < 16) {
    double sum = 0.0;
    for (int w = 0; w < kWarps; ++w) sum += red[threadIdx.x * kWarps + w];
    out[threadIdx.x] = sum;
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------------------------
// FP32 storage, TF32 tensor cores (the mixed-precision sweep)
//
// mma.sync.m16n8k8 .tf32 with FP32 accumulation.  Fragment layouts (PTX ISA, m16n8k8 .tf32),
// g = lane >> 2, t = lane & 3:
//   A (16x8, row):  a0 A[g][t], a1 A[g+8][t], a2 A[g][t+4], a3 A[g+8][t+4]
//   B (8x8, col):   b0 B[t][g], b1 B[t+4][g]
//   C/D (16x8):     c0 C[g][2t], c1 C[g][2t+1], c2 C[g+8][2t], c3 C[g+8][2t+1]
// NP = 1: operands rounded to TF32 (10-bit mantissa) once.  NP = 3: each operand split into a
// TF32 head and a TF32 tail, three products (tail*head + head*tail + head*head), which carries
// the FP32 operands' precision through the tensor cores.
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t tf32_bits(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// One k-step of 8 for a 16x16 output block: A fragment a[4] (FP32 values), B fragments of the
// two 8-column halves b[2][2]; acc[j] is the 16x8 half j.
template <int NP>
__device__ __forceinline__ void mma_block16(float (&acc)[2][4], const float (&a)[4], const float (&b)[2][2]) {
  uint32_t ah[4], bh[2][2];
#pragma unroll
  for (int q = 0; q < 4; ++q) ah[q] = tf32_bits(a[q]);
#pragma unroll
  for (int j = 0; j < 2; ++j)
#pragma unroll
    for (int q = 0; q < 2; ++q) bh[j][q] = tf32_bits(b[j][q]);
  if (NP == 3) {
    uint32_t at[4], bt[2][2];
#pragma unroll
    for (int q = 0; q < 4; ++q) at[q] = tf32_bits(a[q] - __uint_as_float(ah[q]));
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 2; ++q) bt[j][q] = tf32_bits(b[j][q] - __uint_as_float(bh[j][q]));
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      mma_tf32(acc[j], at[0], at[1], at[2], at[3], bh[j][0], bh[j][1]);
      mma_tf32(acc[j], ah[0], ah[1], ah[2], ah[3], bt[j][0], bt[j][1]);
    }
  }
#pragma unroll
  for (int j = 0; j < 2; ++j) mma_tf32(acc[j], ah[0], ah[1], ah[2], ah[3], bh[j][0], bh[j][1]);
}

// C (M x N, ldc) = alpha * op(A) * op(B) + beta * C in FP32 with TF32 tensor cores; the same
// operand conventions, block ownership (16x16 output blocks per warp, so two calls with the same
// M, N may accumulate without a barrier) and bounds rules as the FP64 cta_gemm.
template <int NP>
static __device__ __noinline__ void cta_gemm_tf32(int M, int N, int K, float alpha, const float *A, int lda,
                                                  bool ta, const float *B, int ldb, bool tb, float beta,
                                                  float *C, int ldc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int bm = (M + 15) >> 4, bn = (N + 15) >> 4;
  const bool full = ((M | N | K) & 15) == 0;
  const long sam = ta ? lda : 1, sak = ta ? 1 : lda;  // A(m, k) = A[m*sam + k*sak]
  const long sbk = tb ? ldb : 1, sbn = tb ? 1 : ldb;  // B(k, n) = B[k*sbk + n*sbn]
  for (int blk = warp; blk < bm * bn; blk += kWarps) {
    const int m0 = (blk % bm) << 4, n0 = (blk / bm) << 4;
    const int ma = m0 + g, mb = m0 + 8 + g;
    float acc[2][4];
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[j][q] = 0.f;
    if (full) {
      const float *pa = A + ma * sam + t * sak, *pb = B + t * sbk + (n0 + g) * sbn;
      const long a8 = 8 * sam, k4a = 4 * sak, k4b = 4 * sbk, n8 = 8 * sbn;
#pragma unroll 2
      for (int k0 = 0; k0 < K; k0 += 8) {
        const float *qa = pa + k0 * sak, *qb = pb + k0 * sbk;
        const float a[4] = {qa[0], qa[a8], qa[k4a], qa[a8 + k4a]};
        const float b[2][2] = {{qb[0], qb[k4b]}, {qb[n8], qb[n8 + k4b]}};
        mma_block16<NP>(acc, a, b);
      }
    } else {
      for (int k0 = 0; k0 < K; k0 += 8) {
        const int ka = k0 + t, kb = k0 + t + 4;
        float a[4] = {0.f, 0.f, 0.f, 0.f}, b[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
        if (ka < K) {
          if (ma < M) a[0] = A[ma * sam + ka * sak];
          if (mb < M) a[1] = A[mb * sam + ka * sak];
        }
        if (kb < K) {
          if (ma < M) a[2] = A[ma * sam + kb * sak];
          if (mb < M) a[3] = A[mb * sam + kb * sak];
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int n = n0 + 8 * j + g;
          if (n < N) {
            if (ka < K) b[j][0] = B[ka * sbk + n * sbn];
            if (kb < K) b[j][1] = B[kb * sbk + n * sbn];
          }
        }
        mma_block16<NP>(acc, a, b);
      }
    }
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int m = (q < 2) ? ma : mb, n = n0 + 8 * j + 2 * t + (q & 1);
        if (full || (m < M && n < N)) {
          float *c = C + m + (long)ldc * n;
          const float v = alpha * acc[j][q];
          *c = (beta == 0.f) ? v : v + beta * (*c);
        }
      }
  }
}

// Sixteen closures (the FP32/TF32 counterpart of cta_closure16):
//   out[k + 4 (s + 2 t)] = sum_{m < M, n < N} (A_s B_t)[m, n] P_k[m, n],   s, t in {0, 1}, k < 4,
// A_s = A + s*sa (M x K, ld lda, not transposed), B_t = B + t*sb (K x N, ld ldb), P_k = P + k*sp.
// Partial sums leave the warps in FP64.  red: >= 16*kWarps doubles.  Ends with a barrier.
template <int NP>
static __device__ __noinline__ void cta_closure16_tf32(int M, int N, int K, const float *A, int lda, long sa,
                                                       const float *B, int ldb, long sb, const float *P, int ldp,
                                                       long sp, double *red, double *out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int bm = (M + 15) >> 4, bn = (N + 15) >> 4;
  double v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = 0.0;
  for (int blk = warp; blk < bm * bn; blk += kWarps) {
    const int m0 = (blk % bm) << 4, n0 = (blk / bm) << 4;
    const int ma = m0 + g, mb = m0 + 8 + g;
#pragma unroll 1
    for (int s = 0; s < 2; ++s) {
      const float *As = A + s * sa;
      float acc[2][2][4];  // [t][n half][fragment]
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
          for (int q = 0; q < 4; ++q) acc[u][j][q] = 0.f;
      for (int k0 = 0; k0 < K; k0 += 8) {
        const int ka = k0 + t, kb = k0 + t + 4;
        float a[4] = {0.f, 0.f, 0.f, 0.f};
        if (ka < K) {
          if (ma < M) a[0] = As[ma + (long)lda * ka];
          if (mb < M) a[1] = As[mb + (long)lda * ka];
        }
        if (kb < K) {
          if (ma < M) a[2] = As[ma + (long)lda * kb];
          if (mb < M) a[3] = As[mb + (long)lda * kb];
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          float b[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int n = n0 + 8 * j + g;
            if (n < N) {
              if (ka < K) b[j][0] = B[u * sb + ka + (long)ldb * n];
              if (kb < K) b[j][1] = B[u * sb + kb + (long)ldb * n];
            }
          }
          mma_block16<NP>(acc[u], a, b);
        }
      }
      // epilogue: dot the product blocks with the four P blocks
      float w[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) w[q] = 0.f;
#pragma unroll
      for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int m = (q < 2) ? ma : mb, n = n0 + 8 * j + 2 * t + (q & 1);
          if (m < M && n < N) {
            const float *pp = P + m + (long)ldp * n;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const float pk = pp[k * sp];
              w[k] += acc[0][j][q] * pk;
              w[k + 4] += acc[1][j][q] * pk;
            }
          }
        }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        v[k + 4 * s] += w[k];
        v[k + 8 + 4 * s] += w[k + 4];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 16; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 16; ++q) red[q * kWarps + warp] = v[q];
  __syncthreads();
  if (threadIdx.x < 16) {
    double sum = 0.0;
    for (int w = 0; w < kWarps; ++w) sum += red[threadIdx.x * kWarps + w];
    out[threadIdx.x] = sum;
  }
  __syncthreads();
}

// Overloads that let the sweep be written once for FP64 (DMMA) and FP32 (TF32) work buffers.
template <int NP>
__device__ __forceinline__ void gemm_t(int M, int N, int K, double alpha, const double *A, int lda, bool ta,
                                       const double *B, int ldb, bool tb, double beta, double *C, int ldc) {
  cta_gemm(M, N, K, alpha, A, lda, ta, B, ldb, tb, beta, C, ldc);
}
template <int NP>
__device__ __forceinline__ void gemm_t(int M, int N, int K, float alpha, const float *A, int lda, bool ta,
                                       const float *B, int ldb, bool tb, float beta, float *C, int ldc) {
  cta_gemm_tf32<NP>(M, N, K, alpha, A, lda, ta, B, ldb, tb, beta, C, ldc);
}

// Sum of v over the CTA; result returned to every thread.  red: >= kWarps doubles of smem.
__device__ __forceinline__ double cta_sum(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) s += red[w];
  return s;
}

// Four sums at once (one pair of barriers).  red: >= 4*kWarps doubles.
__device__ __forceinline__ void cta_sum4(double v[4], double *red) {
#pragma unroll
  for (int q = 0; q < 4; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 4; ++q) red[q * kWarps + warp] = v[q];
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    double s = 0.0;
    for (int w = 0; w < kWarps; ++w) s += red[q * kWarps + w];
    v[q] = s;
  }
}

// dlarfg's coefficients for a column with head alpha and squared tail norm xnorm2 > 0:
// beta = -sign(alpha) ||(alpha, x)||, tau = (beta - alpha) / beta, scale of the tail 1/(alpha - beta).
// FP64 square roots and divisions are long dependent sequences on this GPU, and this sits on the
// QR's critical path (once per column): one sqrt of alpha^2 + xnorm2 (no overflow at the
// magnitudes of normalised MPS tensors) and one division serve all three.
__device__ __forceinline__ void reflector_coeffs(double alpha, double xnorm2, double &beta, double &tau,
                                                 double &scale) {
  const double mag = sqrt(fma(alpha, alpha, xnorm2));
  beta = (alpha >= 0.0) ? -mag : mag;
  const double dd = alpha - beta;  // nonzero: |beta| > 0 and of opposite sign to alpha
  const double r = 1.0 / (beta * dd);
  tau = -dd * dd * r;               // (beta - alpha) / beta
  scale = beta * r;                 // 1 / (alpha - beta)
}

// Apply H = I - tau v v^T (v = (1, col[i+1..m)) stored below the diagonal of column i) to the
// columns j > i that this warp owns (j = warp mod kWarps), all of them at once: partial dot
// products for every owned column first, then one interleaved butterfly, then the updates.
// MAXC bounds the owned columns (n <= MAXC * kWarps).
template <int MAXC>
static __device__ __forceinline__ void warp_apply_reflector(int m, int n, int i, const double *col,
                                                            double tau, double *A, int lda) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int first = i + 1 + (((warp - (i + 1)) % kWarps) + kWarps) % kWarps;
  double part[MAXC], head[MAXC];
#pragma unroll
  for (int c = 0; c < MAXC; ++c) {
    const int j = first + c * kWarps;
    part[c] = 0.0;
    head[c] = 0.0;
    if (j < n) {
      const double *cj = A + (long)lda * j;
      head[c] = cj[i];
      for (int r = i + 1 + lane; r < m; r += 32) part[c] += col[r] * cj[r];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int c = 0; c < MAXC; ++c) part[c] += __shfl_xor_sync(0xffffffffu, part[c], o);
#pragma unroll
  for (int c = 0; c < MAXC; ++c) {
    const int j = first + c * kWarps;
    if (j < n) {
      double *cj = A + (long)lda * j;
      const double f = tau * (part[c] + head[c]);
      for (int r = i + 1 + lane; r < m; r += 32) cj[r] -= f * col[r];
      if (lane == 0) cj[i] = head[c] - f;
    }
  }
  __syncwarp();
}

// Register-resident Householder QR (same conventions and results as cta_householder_qr below).
// Column j belongs to warp j % kWarps; the warp keeps rows lane + 32*q (q < RPL) of its columns
// (at most MAXC of them) in registers for the whole factorisation, so updates never go through
// shared memory.  Reflector vectors are published in A below the diagonal (and tau[]), one
// barrier per column in the factorisation; forming Q reads the published reflectors only and
// needs no barrier.  Requires m <= 32*RPL and n <= kWarps*MAXC.
template <int RPL, int MAXC>
static __device__ __noinline__ void cta_qr_reg(int m, int n, double *__restrict__ A, int lda,
                                               double *__restrict__ R, int ldr, double *__restrict__ tau) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu;
  double x[MAXC][RPL];
  __syncthreads();
#pragma unroll
  for (int c = 0; c < MAXC; ++c) {
    const int j = warp + c * kWarps;
#pragma unroll
    for (int q = 0; q < RPL; ++q) {
      const int r = lane + 32 * q;
      x[c][q] = (j < n && r < m) ? A[r + (long)lda * j] : 0.0;
    }
  }
  // dgeqr2
  for (int i = 0; i < n; ++i) {
    const int ci = i / kWarps;  // slot of column i in its owner's registers
    if (warp == i % kWarps) {
      double part = 0.0, alpha = 0.0;
#pragma unroll
      for (int c = 0; c < MAXC; ++c)
        if (c == ci) {
#pragma unroll
          for (int q = 0; q < RPL; ++q) {
            const int r = lane + 32 * q;
            if (r > i && r < m) part += x[c][q] * x[c][q];
            if (r == i) alpha = x[c][q];
          }
        }
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(full, part, o);
      alpha = __shfl_sync(full, alpha, i & 31);
      double ti = 0.0, beta = alpha, sc = 1.0;
      if (m - i > 1 && part > 0.0) reflector_coeffs(alpha, part, beta, ti, sc);
#pragma unroll
      for (int c = 0; c < MAXC; ++c)
        if (c == ci) {
#pragma unroll
          for (int q = 0; q < RPL; ++q) {
            const int r = lane + 32 * q;
            if (r > i && r < m) {
              if (ti != 0.0) x[c][q] *= sc;
              A[r + (long)lda * i] = x[c][q];  // published reflector below the diagonal
            }
            if (r == i) x[c][q] = beta;
          }
        }
      if (lane == 0) tau[i] = ti;
    }
    __syncthreads();
    const double ti = tau[i];
    if (ti != 0.0) {
      double v[RPL];
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const int r = lane + 32 * q;
        v[q] = (r > i && r < m) ? A[r + (long)lda * i] : (r == i ? 1.0 : 0.0);
      }
      double part[MAXC];
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        part[c] = 0.0;
#pragma unroll
        for (int q = 0; q < RPL; ++q) part[c] += v[q] * x[c][q];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < MAXC; ++c) part[c] += __shfl_xor_sync(full, part[c], o);
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        const int j = warp + c * kWarps;
        if (j > i && j < n) {
          const double f = ti * part[c];
#pragma unroll
          for (int q = 0; q < RPL; ++q) x[c][q] -= f * v[q];
        }
      }
    }
  }
  // R: upper triangle of the reduced columns
#pragma unroll
  for (int c = 0; c < MAXC; ++c) {
    const int j = warp + c * kWarps;
    if (j < n) {
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const int r = lane + 32 * q;
        if (r < n) R[r + (long)ldr * j] = (r <= j) ? x[c][q] : 0.0;
      }
    }
  }
  // dorg2r: columns start as unit vectors, H_i applied for i = n-1 .. 0
#pragma unroll
  for (int c = 0; c < MAXC; ++c) {
    const int j = warp + c * kWarps;
#pragma unroll
    for (int q = 0; q < RPL; ++q) x[c][q] = (lane + 32 * q == j) ? 1.0 : 0.0;
  }
  for (int i = n - 1; i >= 0; --i) {
    const double ti = tau[i];
    double v[RPL];
#pragma unroll
    for (int q = 0; q < RPL; ++q) {
      const int r = lane + 32 * q;
      v[q] = (r > i && r < m) ? A[r + (long)lda * i] : (r == i ? 1.0 : 0.0);
    }
    if (ti != 0.0) {
      double part[MAXC];
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        part[c] = 0.0;
#pragma unroll
        for (int q = 0; q < RPL; ++q) part[c] += v[q] * x[c][q];
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < MAXC; ++c) part[c] += __shfl_xor_sync(full, part[c], o);
#pragma unroll
      for (int c = 0; c < MAXC; ++c) {
        const int j = warp + c * kWarps;
        if (j > i && j < n) {
          const double f = ti * part[c];
#pragma unroll
          for (int q = 0; q < RPL; ++q) x[c][q] -= f * v[q];
        }
      }
    }
    // column i := H_i e_i
#pragma unroll
    for (int c = 0; c < MAXC; ++c) {
      const int j = warp + c * kWarps;
      if (j == i) {
#pragma unroll
        for (int q = 0; q < RPL; ++q) {
          const int r = lane + 32 * q;
          x[c][q] = (r > i) ? -ti * v[q] : (r == i ? 1.0 - ti : 0.0);
        }
      }
    }
  }
  __syncthreads();  // every warp has read the published reflectors
#pragma unroll
  for (int c = 0; c < MAXC; ++c) {
    const int j = warp + c * kWarps;
    if (j < n) {
#pragma unroll
      for (int q = 0; q < RPL; ++q) {
        const int r = lane + 32 * q;
        if (r < m) A[r + (long)lda * j] = x[c][q];
      }
    }
  }
  __syncthreads();
}

// Householder QR of A (m x n, m >= n, ld lda, shared memory) in LAPACK's conventions
// (dgeqr2 + dorg2r, with dlarfg's beta = -sign(alpha)*||x||, tau = 0 when the column below the
// diagonal is zero or m - i == 1).  On exit A holds Q (m x n, orthonormal columns) and R
// (n x n, ld ldr, upper triangular) holds the triangular factor.  tau: >= n doubles of shared
// memory; w and red are not used.  Starts and ends with a barrier.
//
// Column j belongs to warp j % kWarps for the whole factorisation: the owner builds reflector j
// and every warp applies published reflectors to its own columns, so one barrier per column
// and pass is enough (a warp updates its columns in program order).
static __device__ __noinline__ void cta_householder_qr(int m, int n, double *A, int lda, double *R, int ldr,
                                                double *tau, double *w, double *red) {
  (void)w;
  (void)red;
  if (m <= 64 && n <= 4 * kWarps) {
    cta_qr_reg<2, 4>(m, n, A, lda, R, ldr, tau);
    return;
  }
  if (m <= 128 && n <= 8 * kWarps) {
    cta_qr_reg<4, 8>(m, n, A, lda, R, ldr, tau);
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu;
  __syncthreads();
  // dgeqr2
  for (int i = 0; i < n; ++i) {
    double *col = A + (long)lda * i;
    if (warp == i % kWarps) {
      double part = 0.0;
      for (int r = i + 1 + lane; r < m; r += 32) part += col[r] * col[r];
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(full, part, o);
      const double alpha = col[i];
      double ti = 0.0;
      if (m - i > 1 && part > 0.0) {
        double beta, sc;
        reflector_coeffs(alpha, part, beta, ti, sc);
        for (int r = i + 1 + lane; r < m; r += 32) col[r] *= sc;
        __syncwarp();
        if (lane == 0) col[i] = beta;
      }
      if (lane == 0) tau[i] = ti;
    }
    __syncthreads();
    const double ti = tau[i];
    if (ti != 0.0) {
      if (n <= 4 * kWarps) warp_apply_reflector<4>(m, n, i, col, ti, A, lda);
      else if (n <= 8 * kWarps) warp_apply_reflector<8>(m, n, i, col, ti, A, lda);
      else warp_apply_reflector<16>(m, n, i, col, ti, A, lda);
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < n * n; q += kThreads) {
    const int r = q % n, c = q / n;
    R[r + (long)ldr * c] = (r <= c) ? A[r + (long)lda * c] : 0.0;
  }
  __syncthreads();
  // dorg2r, k = n: Q = H_0 ... H_{n-1} applied to the first n unit columns
  for (int i = n - 1; i >= 0; --i) {
    const double *col = A + (long)lda * i;
    const double ti = tau[i];
    if (ti != 0.0 && i < n - 1) {
      if (n <= 4 * kWarps) warp_apply_reflector<4>(m, n, i, col, ti, A, lda);
      else if (n <= 8 * kWarps) warp_apply_reflector<8>(m, n, i, col, ti, A, lda);
      else warp_apply_reflector<16>(m, n, i, col, ti, A, lda);
    }
    __syncthreads();
    if (warp == i % kWarps) {
      double *ci = A + (long)lda * i;
      for (int r = lane; r < m; r += 32) {
        if (r > i) ci[r] *= -ti;
        else if (r == i) ci[r] = 1.0 - ti;
        else ci[r] = 0.0;
      }
    }
  }
  __syncthreads();
}

}  // namespace mq
