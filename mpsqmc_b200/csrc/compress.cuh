// Walker recompression on the device (sm_100a, FP64): MPSstate::CompressState(truncD)
// (MPSstate.cpp:379-404) for every walker of the population, one CTA per walker.
//
// A sweep left to right and one right to left over the bonds.  At bond (k, k+1) the two-site
// object Theta (rows alpha + D_k sigma_k, columns beta + D_{k+2} sigma_{k+1};
// TwoSiteObject.cpp:71-115) is factorised by a one-sided Jacobi SVD, truncated to
// min(truncD, number of singular values >= 1e-13) (TwoSiteObject.cpp:145-157), and split as
// U | S V^T moving right, U S | V^T moving left (TwoSiteObject.cpp:164-182).  The SVD's column
// signs are this implementation's, so the tensors differ from LAPACK's by signs on the bonds; the
// state is the same.
//
// The walker is unpacked into a fixed layout (site k at the offset it has in the largest walker
// layout) so that sites can change shape in place, then packed back with its new bond dims.
#pragma once

#include "walker_kernels.cuh"

namespace mq {

constexpr double kSchmidtCut = 1e-13;  // TwoSiteObject.cpp:16

// One-sided (Hestenes) Jacobi SVD of A (p x q, p >= q, ld lda): on exit A V = U Sigma, i.e. the
// columns of A are sigma_j u_j, V (q x q, ld ldv) is orthogonal, sig[j] = ||A_j|| and order[r]
// is the column of the r-th largest singular value.  Column pairs of one round (round-robin
// tournament) are disjoint, so every warp rotates its pairs without synchronisation; one barrier
// per round.  sig/order/red in shared memory (q, q and kWarps+1 entries).
static __device__ __noinline__ void cta_jacobi_svd(int p, int q, double *A, int lda, double *V, int ldv,
                                                   double *sig, int *order, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int e = threadIdx.x; e < q * q; e += kThreads) V[(e % q) + (long)ldv * (e / q)] = (e % q == e / q) ? 1.0 : 0.0;
  __syncthreads();
  const int nq = q + (q & 1);  // a dummy column pads odd q
  for (int sweep = 0; sweep < 60 && q > 1; ++sweep) {
    double off = 0.0;
    for (int r = 0; r < nq - 1; ++r) {
      for (int k = warp; k < nq / 2; k += kWarps) {
        // circle method: position 0 fixed, positions 1..nq-1 rotate by r
        auto at = [&](int pos) { return pos == 0 ? 0 : 1 + (pos - 1 + r) % (nq - 1); };
        int cp = at(k), cq = at(nq - 1 - k);
        if (cp >= q || cq >= q) continue;
        if (cp > cq) {
          const int t = cp;
          cp = cq;
          cq = t;
        }
        double *ap = A + (long)lda * cp, *aq = A + (long)lda * cq;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = lane; i < p; i += 32) {
          const double x = ap[i], y = aq[i];
          al += x * x;
          be += y * y;
          ga += x * y;
        }
        for (int o = 16; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga += __shfl_xor_sync(0xffffffffu, ga, o);
        }
        if (ga == 0.0 || al == 0.0 || be == 0.0) continue;
        const double ratio = fabs(ga) / sqrt(al * be);
        if (ratio <= 1e-15) continue;
        off = fmax(off, ratio);
        const double zeta = (be - al) / (2.0 * ga);
        const double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
        for (int i = lane; i < p; i += 32) {
          const double x = ap[i], y = aq[i];
          ap[i] = c * x - s * y;
          aq[i] = s * x + c * y;
        }
        double *vp = V + (long)ldv * cp, *vq = V + (long)ldv * cq;
        for (int i = lane; i < q; i += 32) {
          const double x = vp[i], y = vq[i];
          vp[i] = c * x - s * y;
          vq[i] = s * x + c * y;
        }
      }
      __syncthreads();
    }
    // converged when no pair of the sweep was rotated
    if (lane == 0) red[warp] = off;
    __syncthreads();
    double mx = 0.0;
    for (int w = 0; w < kWarps; ++w) mx = fmax(mx, red[w]);
    __syncthreads();
    if (mx == 0.0) break;
  }
  // singular values and their descending order (ties by column index)
  for (int j = warp; j < q; j += kWarps) {
    const double *aj = A + (long)lda * j;
    double s2 = 0.0;
    for (int i = lane; i < p; i += 32) s2 += aj[i] * aj[i];
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    if (lane == 0) sig[j] = sqrt(s2);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < q; j += kThreads) {
    int rank = 0;
    for (int i = 0; i < q; ++i) rank += (sig[i] > sig[j] || (sig[i] == sig[j] && i < j)) ? 1 : 0;
    order[rank] = j;
  }
  __syncthreads();
}

#ifndef MQ_DEVICE_ONLY

// Compress walker w to bond dimension targets[w] (<= 0: unchanged).  Per-CTA scratch: the walker
// in the fixed layout (p.woff offsets), Theta (m x n), its transpose and V, each sized for the
// largest two-site object.  Dynamic shared memory: sig, order (2*maxB each), reductions, dims.
__global__ void __launch_bounds__(kThreads, 1) compress_kernel(Dev p, const int *targets, double *cscr,
                                                               long cstride) {
  extern __shared__ double smem_raw[];
  const int L = p.L, d = kMaxD, tid = threadIdx.x;
  const int q2 = 2 * p.maxB;
  double *sig = smem_raw;
  double *red = sig + q2;
  int *order = reinterpret_cast<int *>(red + kWarps + 2);
  int *dims = order + q2;
  int *wsel = dims + L + 2;
  long *wofs_new = reinterpret_cast<long *>(smem_raw) + (q2 + kWarps + 2) + (q2 + L + 4) / 2 + 1;
  double *Wk = cscr + (long)blockIdx.x * cstride;
  const long wmax = p.woff[L - 1] + (long)p.bW[L - 1] * p.bW[L] * d;
  double *T = Wk + ((wmax + 31) & ~31L);
  double *M2 = T + (long)q2 * q2;
  double *Vm = M2 + (long)q2 * q2;
  const int N = *p.n_cur;
  for (;;) {
    __syncthreads();
    if (tid == 0) *wsel = atomicAdd(p.ctr + kCtrCompress, 1);
    __syncthreads();
    const int w = *wsel;
    if (w >= N) break;
    const int truncD = targets[w];
    if (truncD <= 0) continue;
    const int slot = p.slot_of[w];
    double *W = p.walkers + (long)slot * p.wstride;
    int *gd = const_cast<int *>(p.wdims) + (long)slot * (L + 1);
    long *go = const_cast<long *>(p.wofs) + (long)slot * L;
    for (int k = tid; k <= L; k += kThreads) dims[k] = gd[k];
    __syncthreads();
    {  // SetupWalkers compresses only when the target is below the walker's bond dimension
      int dmax = 1;
      for (int k = 0; k <= L; ++k) dmax = max(dmax, dims[k]);
      if (truncD >= dmax) continue;
    }
    // unpack: site k of the walker (packed at go[k]) to the fixed offset p.woff[k]
    for (int k = 0; k < L; ++k) {
      const long n = (long)dims[k] * dims[k + 1] * d;
      for (long e = tid; e < n; e += kThreads) Wk[p.woff[k] + e] = W[go[k] + e];
    }
    __syncthreads();
    for (int pass = 0; pass < 2; ++pass) {
      const bool right = pass == 0;
      for (int it = 0; it < L - 1; ++it) {
        const int k = right ? it : L - 2 - it;
        const int DL = dims[k], DM = dims[k + 1], DR = dims[k + 2];
        const int m = DL * d, n = DR * d;
        double *Al = Wk + p.woff[k], *Ar = Wk + p.woff[k + 1];
        // Theta (TwoSiteObject.cpp:111-115, 126-134)
        for (int il = 0; il < d; ++il)
          for (int ir = 0; ir < d; ++ir)
            cta_gemm(DL, DR, DM, 1.0, Al + (long)il * DL * DM, DL, false, Ar + (long)ir * DM * DR, DM, false, 0.0,
                     T + DL * il + (long)m * DR * ir, m);
        __syncthreads();
        const bool tall = m >= n;
        double *Mx = T;
        int pp = m, qq = n;
        if (!tall) {
          for (long e = tid; e < (long)m * n; e += kThreads) {
            const int i = (int)(e % m), j = (int)(e / m);
            M2[j + (long)n * i] = T[e];
          }
          __syncthreads();
          Mx = M2;
          pp = n;
          qq = m;
        }
        cta_jacobi_svd(pp, qq, Mx, pp, Vm, qq, sig, order, red);
        // truncation (TwoSiteObject.cpp:145-157), never beyond the slot layout's bond
        int idx = qq;
        for (int c = 0; c < qq; ++c)
          if (sig[order[c]] < kSchmidtCut) {
            idx = c;
            break;
          }
        int tr = min(truncD, idx);
        tr = min(tr, p.bW[k + 1]);
        tr = max(tr, 1);
        // U (m x tr) and VT (tr x n) columns: tall -> U_j = Mx_j / sig_j, V_j = Vm_j;
        //                                     wide -> U_j = Vm_j,         V_j = Mx_j / sig_j
        for (long e = tid; e < (long)m * tr; e += kThreads) {
          const int row = (int)(e % m), b = (int)(e / m);  // row = alpha + DL*sigma
          const int j = order[b];
          const double sj = sig[j];
          const double u = tall ? (sj > 0.0 ? Mx[row + (long)pp * j] / sj : 0.0) : Vm[row + (long)qq * j];
          const int alpha = row % DL, sg = row / DL;
          Al[alpha + (long)DL * (b + (long)tr * sg)] = right ? u : u * sj;
        }
        for (long e = tid; e < (long)n * tr; e += kThreads) {
          const int col = (int)(e % n), b = (int)(e / n);  // col = beta + DR*sigma
          const int j = order[b];
          const double sj = sig[j];
          const double v = tall ? Vm[col + (long)qq * j] : (sj > 0.0 ? Mx[col + (long)pp * j] / sj : 0.0);
          const int beta = col % DR, sg = col / DR;
          Ar[b + (long)tr * (beta + (long)DR * sg)] = right ? v * sj : v;
        }
        __syncthreads();
        if (tid == 0) dims[k + 1] = tr;
        __syncthreads();
      }
    }
    // pack back with the new dims; the walker's dims and offsets follow
    if (tid == 0) {
      long o = 0;
      for (int k = 0; k < L; ++k) {
        wofs_new[k] = o;
        o += (long)dims[k] * dims[k + 1] * d;
      }
    }
    __syncthreads();
    for (int k = 0; k < L; ++k) {
      const long n = (long)dims[k] * dims[k + 1] * d;
      for (long e = tid; e < n; e += kThreads) W[wofs_new[k] + e] = Wk[p.woff[k] + e];
    }
    for (int k = tid; k <= L; k += kThreads) gd[k] = dims[k];
    for (int k = tid; k < L; k += kThreads) go[k] = wofs_new[k];
    __syncthreads();
  }
}

// Dynamic shared memory of compress_kernel (bytes).
inline size_t compress_smem_bytes(int L, int maxB) {
  const int q2 = 2 * maxB;
  return sizeof(double) * ((size_t)(q2 + kWarps + 2) + (size_t)(q2 + L + 4) / 2 + 1 + (size_t)L + 4);
}

#endif  // MQ_DEVICE_ONLY

}  // namespace mq
