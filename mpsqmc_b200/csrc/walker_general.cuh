// Walker step for couplings of any range (sm_100a): 2D lattices on a snake path and other
// long-range Heisenberg models, with the coupling order of MPSQMC2.cpp:286-299 (by first site,
// then by second site).
//
// One CTA per walker, as in walker_step_kernel.  The centre of the walker moves left to right;
// while it sits on site i every coupling (i, j) is processed:
//   1. right environment R[j+1] = <Psi_T|phi> over sites j+1..L-1, recomputed from the first
//      still-valid one when an earlier coupling changed a site beyond j;
//   2. four left branches P[s,t] = B_i[s]^T L C[t] on the centre, carried through the middle
//      sites i+1..j-1 by ordinary transfer steps, four right branches at j and 16 closures give
//      C_kl = <Psi_T|(sqrt(s_k)U_k)_i (sqrt(s_l)V_l)_j|phi> (MPSQMC2.cpp:540-549); for
//      nearest-neighbour couplings the right branches come from the right-environment sweep, so
//      the closures are dot products only;
//   3. PDF, weight, CDF sample (551-588), O1 on the centre and O2 on site j (MPSstate.cpp:575-633).
// Then one Householder QR moves the centre to i+1, and the final site i enters the left
// environments: the trial overlap and the energy channels of the compact MPO of
// H = sum_c J_c S_i.S_j - h sum_k S^z_k (one "done" channel plus Sx, iSy, Sz per site that still
// has a partner to the right).
//
// Normalisation is deferred to the end of the step.  Every quantity the reference derives from
// the normalised walker is a ratio in which the norm cancels: PDF[x] = max(0, sum C x x) 4/(ov G)
// with C and ov of the same state, and the new overlap <Psi_T|B(x)phi> = 4 sum_kl C_kl x_k x_l.
// So the walk carries the unnormalised overlap and normalises once, when the centre reaches
// site L-1 and the norm is that of the centre.  The reference's per-coupling setOverlap
// (MPSQMC2.cpp:592) rescales by a positive number and never flips a sign here: the sampled x
// has sum C x x > 0, so the overlap stays positive.
//
// QR-free variant (p.nloff >= 0): no site is orthonormalised during the sweep.  The centre is
// stored as it is once its couplings are done, rescaled so that its squared Frobenius norm is
// its right bond dimension (that of an isometry: a per-site scale factor, carried into the FP64
// overlap), and a left norm environment Nl = sum_s A[s]^T Nl A[s] of the stored sites gives the
// norm at site L-1.  Every quantity above is gauge invariant, so the walk is the same; the host
// restores the left-canonical form (Walker::setOverlap's LeftNormalize, set_overlap_kernel) every
// few steps, which bounds the growth of the bond gauges' condition numbers.
//
// Work-buffer precision T: double (FP64 DMMA, the parity mode) or float (the mixed-precision
// sweep: site tensors, environments and branches in FP32, products on the TF32 tensor cores with
// FP32 accumulation, NP = 1 or 3 passes; the closures, PDF, sampling, weights, overlaps, norms and
// energies in FP64; walkers stay FP64 in HBM).  The mixed sweep is always QR-free.
#pragma once

#include <type_traits>

#include "proposal.cuh"
#include "walker_kernels.cuh"

namespace mq {

template <typename T>
__device__ __forceinline__ const T *trial_of(const Dev &p) {
  if constexpr (std::is_same<T, double>::value) return p.trial;
  else return p.trial32;
}

// R[k] = sum_s B_k[s] R[k+1] A_k[s]^T from the walker's site k as stored in global memory.
// With ZB (nearest-neighbour couplings) also the right branches of site k,
// Z[s' + 2 t'] = B_k[s'] R[k+1] A_k[t']^T (a_k x b_k, ld a_k, block stride a_k * (the slot
// layout's b_k)), and R[k] = Z[0] + Z[3]: the coupling (k-1, k) then closes its left branches
// against Z[k] without products of its own (closures).  Uses Nxt and Xb.  Ends with a barrier.
template <typename T, int NP = 0, bool ZB = false>
static __device__ void right_env_step(const Dev &p, SmemT<T> &s, const double *W, T *scr, int k) {
  const int d = kMaxD;
  const int al = p.aT[k], ar = p.aT[k + 1], bl = s.bW[k], br = s.bW[k + 1];
  load_site(s.Nxt, p.pb, s.sbC, W + s.woff[k], bl, br);
  if (k > 1) prefetch_l2(W + s.woff[k - 1], (long)s.bW[k - 1] * bl * kMaxD);  // the next site of the sweep
  __syncthreads();
  const T *Rn = scr + p.roff[k + 1];
  T *Rk = scr + p.roff[k];
  T *Z = scr + p.zoff[k];
  const long zb = (long)al * p.bW[k];
  const T *Bk = trial_of<T>(p) + p.toff[k];
  for (int sg = 0; sg < d; ++sg)
    gemm_t<NP>(ar, bl, br, T(1), Rn, ar, false, s.Nxt + sg * s.sbC, p.pb, true, T(0), s.Xb + sg * s.sbX, p.pa);
  __syncthreads();
  if constexpr (ZB) {
    for (int sg = 0; sg < d; ++sg)
      for (int tau = 0; tau < d; ++tau)
        gemm_t<NP>(al, bl, ar, T(1), Bk + (long)sg * al * ar, al, false, s.Xb + tau * s.sbX, p.pa, false, T(0),
                   Z + (sg + d * tau) * zb, al);
    __syncthreads();
    for (int q = threadIdx.x; q < al * bl; q += kThreads) Rk[q] = Z[q] + Z[3 * zb + q];
  } else {
    for (int sg = 0; sg < d; ++sg)
      gemm_t<NP>(al, bl, ar, T(1), Bk + (long)sg * al * ar, al, false, s.Xb + sg * s.sbX, p.pa, false,
                 sg == 0 ? T(0) : T(1), Rk, al);
  }
  __syncthreads();
}

// E <- sum_s B[s]^T E T[s] in place (E: al x bl -> ar x br, leading dimension lde).  T[s] is
// bl x br with column stride cs and sigma stride ss.  Uses Xb.  Ends with a barrier.
template <typename T, int NP = 0>
static __device__ void transfer_in_place(const Dev &p, SmemT<T> &s, const T *B, int al, int ar, int bl, int br,
                                         const T *Tm, int cs, int ss, T *E, int lde) {
  const int d = kMaxD;
  for (int sg = 0; sg < d; ++sg)
    gemm_t<NP>(al, br, bl, T(1), E, lde, false, Tm + sg * ss, cs, false, T(0), s.Xb + sg * s.sbX, p.pa);
  __syncthreads();
  for (int sg = 0; sg < d; ++sg)
    gemm_t<NP>(ar, br, al, T(1), B + (long)sg * al * ar, al, true, s.Xb + sg * s.sbX, p.pa, false,
               sg == 0 ? T(0) : T(1), E, lde);
  __syncthreads();
}

// Left environments through the final tensor Tm of site k (Tm[s] bl x br, column stride cs,
// sigma stride ss): trial overlap Lenv, "done" channel Fd -> Fdn, open channels in Fch
// (slot q, operator a at Fch + (3q + a) * maxA * maxB, leading dimension maxA).
// Order: branches P; done' from Fd, the channels that close on k and the field; channels that
// stay open; then Lenv' and the channel site k opens (its slot may be one that closed on k).
// have_P: the branches P of Tm are already in Pb (the caller derived them), skip their products.
template <typename T, int NP = 0>
static __device__ void env_update_general(const Dev &p, SmemT<T> &s, int k, const T *B, int al, int ar, int bl,
                                          int br, const T *Tm, int cs, int ss, const T *Fd, T *Fdn, T *Fch,
                                          bool have_P = false) {
  const int d = kMaxD, lda = p.maxA;
  const long fm = (long)p.maxA * p.maxB;
  // P[s + d t] = B[s]^T Lenv Tm[t]    (ar x br)
  if (!have_P) {
    for (int tau = 0; tau < d; ++tau)
      gemm_t<NP>(al, br, bl, T(1), s.Lenv, p.pa, false, Tm + tau * ss, cs, false, T(0), s.Xb + tau * s.sbX, p.pa);
    __syncthreads();
    for (int sg = 0; sg < d; ++sg)
      for (int tau = 0; tau < d; ++tau)
        gemm_t<NP>(ar, br, al, T(1), B + (long)sg * al * ar, al, true, s.Xb + tau * s.sbX, p.pa, false, T(0),
                   s.Pb + (sg + d * tau) * s.sbX, p.pa);
    __syncthreads();
  }
  // done' = -h sum Sz P + sum_s B[s]^T (sum_t G_st Tm[t]),
  // G_st = delta_st Fd + sum_{i closing on k} J_ik (Sx F_i,x - iSy F_i,iy + Sz F_i,z)(s,t)
  for (int q = threadIdx.x; q < ar * br; q += kThreads) {
    const int r = q % ar, c = q / ar;
    T fz = T(0);
#pragma unroll
    for (int e = 0; e < kN2; ++e) fz += T(p.opSz[e]) * s.Pb[e * s.sbX + r + p.pa * c];
    Fdn[r + lda * c] = T(-p.h) * fz;
  }
  __syncthreads();
  const int e0 = p.ech_off[k], e1 = p.ech_off[k + 1];
  if (k > 0) {
    for (int sg = 0; sg < d; ++sg) {
      for (int q = threadIdx.x; q < al * bl; q += kThreads) {
        const int r = q % al, c = q / al;
        const T fd = Fd[r + lda * c];
        T gx = T(0), gy = T(0), gz = T(0);
        for (int e = e0; e < e1; ++e) {
          const T J = T(p.ech_J[e]);
          if (J == T(0)) continue;
          const T *F = Fch + 3L * p.ech_slot[e] * fm;
          gx += J * F[r + lda * c];
          gy += J * F[fm + r + lda * c];
          gz += J * F[2 * fm + r + lda * c];
        }
        for (int tau = 0; tau < d; ++tau) {
          const int o = sg + d * tau;
          s.Xb[tau * s.sbX + r + p.pa * c] =
              ((sg == tau) ? fd : T(0)) + T(p.opSx[o]) * gx - T(p.opISy[o]) * gy + T(p.opSz[o]) * gz;
        }
      }
      __syncthreads();
      gemm_t<NP>(al, br, bl, T(1), s.Xb, p.pa, false, Tm, cs, false, T(0), s.Qt, p.pa);
      for (int tau = 1; tau < d; ++tau)
        gemm_t<NP>(al, br, bl, T(1), s.Xb + tau * s.sbX, p.pa, false, Tm + tau * ss, cs, false, T(1), s.Qt, p.pa);
      __syncthreads();
      gemm_t<NP>(ar, br, al, T(1), B + (long)sg * al * ar, al, true, s.Qt, p.pa, false, T(1), Fdn, lda);
      __syncthreads();
    }
  }
  // channels that stay open: identity on site k
  for (int e = e0; e < e1; ++e) {
    if (!p.ech_cont[e]) continue;
    T *F = Fch + 3L * p.ech_slot[e] * fm;
    for (int a = 0; a < 3; ++a) transfer_in_place<T, NP>(p, s, B, al, ar, bl, br, Tm, cs, ss, F + a * fm, lda);
  }
  // Lenv' = sum_s P[s,s]; the channels opened on site k
  const int op = p.eopen[k];
  T *Fo = (op >= 0) ? Fch + 3L * op * fm : nullptr;
  for (int q = threadIdx.x; q < ar * br; q += kThreads) {
    const int r = q % ar, c = q / ar;
    T P[kN2];
#pragma unroll
    for (int e = 0; e < kN2; ++e) P[e] = s.Pb[e * s.sbX + r + p.pa * c];
    T l = T(0), fx = T(0), fy = T(0), fz = T(0);
#pragma unroll
    for (int e = 0; e < kN2; ++e) {
      if ((e % d) == (e / d)) l += P[e];
      fx += T(p.opSx[e]) * P[e];
      fy += T(p.opISy[e]) * P[e];
      fz += T(p.opSz[e]) * P[e];
    }
    s.Lenv[r + p.pa * c] = l;
    if (Fo) {
      Fo[r + lda * c] = fx;
      Fo[fm + r + lda * c] = fy;
      Fo[2 * fm + r + lda * c] = fz;
    }
  }
  __syncthreads();
}

// Closures of the four left branches in Pb (cut j, a_j x b_j) with the right branches Z of site
// j (right_env_step): M[p + 4q] = <P_p, Z[q]> = <P_p, B_j[s'] R[j+1] A_j[t']^T>, q = s' + 2t'.
// Sixteen dot products in one pass, reduced in FP64.  Ends with a barrier.
template <typename T, int NP = 0>
static __device__ void closures_z(const Dev &p, SmemT<T> &s, int j, const T *Z) {
  const int aj = p.aT[j], bj = s.bW[j];
  const long zb = (long)aj * p.bW[j];
  double v[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) v[q] = 0.0;
  for (int e = threadIdx.x; e < aj * bj; e += kThreads) {
    const int m = e % aj, n = e / aj;
    T pk[4], zq[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) pk[k] = s.Pb[k * s.sbX + m + p.pa * n];
#pragma unroll
    for (int q = 0; q < 4; ++q) zq[q] = Z[q * zb + e];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k + 4 * q] += (double)pk[k] * (double)zq[q];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 16; ++q)
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < 16; ++q) s.red[q * kWarps + warp] = v[q];
  __syncthreads();
  if (threadIdx.x < 16) {
    double sum = 0.0;
    for (int w = 0; w < kWarps; ++w) sum += s.red[threadIdx.x * kWarps + w];
    s.M[threadIdx.x] = sum;
  }
  __syncthreads();
}

// The same closures for couplings of any range: the right branches of site j (walker site in
// Nxt, R[j+1] at Rn) formed and dotted with P in one pass of products.
template <typename T, int NP = 0>
static __device__ void closures_products(const Dev &p, SmemT<T> &s, int j, const T *Rn) {
  const int d = kMaxD;
  const int aj = p.aT[j], a2 = p.aT[j + 1], bj = s.bW[j], b2 = s.bW[j + 1];
  const T *Bj = trial_of<T>(p) + p.toff[j];
  for (int tau = 0; tau < d; ++tau)
    gemm_t<NP>(a2, bj, b2, T(1), Rn, a2, false, s.Nxt + tau * s.sbC, p.pb, true, T(0), s.Xb + tau * s.sbX, p.pa);
  __syncthreads();
  // M[k + 4 (s' + 2 t')] = <P_k, B_j[s'] Y[t']>, the products formed and dotted in one pass
  if constexpr (std::is_same<T, double>::value) {
    if (((aj | bj | a2) & 15) == 0)
      cta_closure16<true>(aj, bj, a2, Bj, aj, (long)aj * a2, s.Xb, p.pa, s.sbX, s.Pb, p.pa, s.sbX, s.red, s.M);
    else
      cta_closure16<false>(aj, bj, a2, Bj, aj, (long)aj * a2, s.Xb, p.pa, s.sbX, s.Pb, p.pa, s.sbX, s.red, s.M);
  } else {
    cta_closure16_tf32<NP>(aj, bj, a2, Bj, aj, (long)aj * a2, s.Xb, p.pa, s.sbX, s.Pb, p.pa, s.sbX, s.red, s.M);
  }
}

// The 16 closures of coupling (i, j), left branches in Pb: against the stored right branches of
// site j (ZB) or formed here (site j from W, R[j+1] from the scratch).  Uses Nxt and Xb.
template <typename T, int NP = 0, bool ZB = false>
static __device__ void closures(const Dev &p, SmemT<T> &s, int j, const double *W, T *scr) {
  if constexpr (ZB) {
    closures_z<T, NP>(p, s, j, scr + p.zoff[j]);
  } else {
    load_site(s.Nxt, p.pb, s.sbC, W + s.woff[j], s.bW[j], s.bW[j + 1]);
    __syncthreads();
    closures_products<T, NP>(p, s, j, scr + p.roff[j + 1]);
  }
}

// Largest v over the CTA (every thread gets it).  red: >= kWarps doubles.
__device__ __forceinline__ double cta_max(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double m = red[0];
#pragma unroll
  for (int w = 1; w < kWarps; ++w) m = fmax(m, red[w]);
  return m;
}

// C_kl from the closures, PDF over the grid, weight update, CDF sample with the walker's uniform
// for coupling c, and the site operators O1, O2 (MPSQMC2.cpp:551-588, MPSstate.cpp:575-633).
// Returns 4 sum_kl C_kl x_k x_l of the sampled point (the new unnormalised overlap).
// Learned proposal (p.prop_mode == 1, proposal.cuh): the point is drawn from the network's q~ on
// the support of the PDF and the weight takes P(x) / q~(x); with p.prop_collect the grid walk
// stores the features and the normalised PDF of coupling w % nC as a training pair.
template <typename T>
static __device__ double sample_coupling(const Dev &p, SmemT<T> &s, int w, int c, int jq, double ov, double &wt) {
  const int tid = threadIdx.x;
  const double *U = p.tabU + 16 * jq, *Sq = p.tabSq + 4 * jq, *VT = p.tabVT + 16 * jq;
  if (tid < 16) {
    const int k = tid & 3, l = tid >> 2;
    double acc = 0.0;
    for (int qq = 0; qq < 4; ++qq) {
      double inner = 0.0;
      for (int pp = 0; pp < 4; ++pp) inner += U[pp + 4 * k] * s.M[pp + 4 * qq];
      acc += inner * VT[l + 4 * qq];
    }
    s.Cm[k + 4 * l] = Sq[k] * Sq[l] * acc;
  }
  __syncthreads();
  const double fac = 4.0 / (ov * p.G);
  double part = 0.0;
  for (int g = tid; g < p.G; g += kThreads) {
    const double *x = p.grid + 4 * g;
    double v = 0.0;
    for (int l = 0; l < 4; ++l)
      for (int r = 0; r < 4; ++r) v += s.Cm[l + 4 * r] * x[l] * x[r];
    v = fmax(0.0, v) * fac;
    s.pdf[g] = v;
    part += v;
  }
  const double pnorm = cta_sum(part, s.red);
  const bool learned = p.prop_mode == 1;
  const bool collect = !learned && p.prop_collect && c == w % p.nC;
  if (learned || collect) {  // the 32 features
    float *f = s.mlp;
    if (tid < 16) f[tid] = (float)(4.0 * s.Cm[tid] / ov);
    else if (tid < 32) f[tid] = (float)(4.0 * s.M[tid - 16] / ov);
    __syncthreads();
    if (collect)
      for (int e = tid; e < kMlpIn; e += kThreads) p.prop_feat[(long)w * kMlpIn + e] = f[e];
  }
  if (!learned) {
    const double pinv = 1.0 / pnorm;
    for (int g = tid; g < p.G; g += kThreads) {
      s.pdf[g] *= pinv;
      if (collect) p.prop_target[(long)w * p.G + g] = (float)s.pdf[g];
    }
    wt *= pnorm;
    __syncthreads();
  } else {
    float *z = s.mlp + kMlpIn + 4 * kMlpHid;
    mlp_forward_cta(p.prop_w, p.G, s.mlp, s.mlp + kMlpIn, s.mlp + kMlpIn + 2 * kMlpHid, z);
    double zmax = -INFINITY;
    for (int g = tid; g < p.G; g += kThreads)
      if (s.pdf[g] > 0.0) zmax = fmax(zmax, (double)z[g]);
    zmax = cta_max(zmax, s.red);
    double se = 0.0;
    for (int g = tid; g < p.G; g += kThreads) {
      const double e = (s.pdf[g] > 0.0) ? exp((double)z[g] - zmax) : 0.0;
      s.qprop[g] = e;
      se += e;
    }
    // the defensive mixture (1 - alpha) q~ + alpha P / sum P: P / q_mix <= sum P / alpha
    const double qinv = (1.0 - p.prop_mix) / cta_sum(se, s.red), pinv = pnorm > 0.0 ? p.prop_mix / pnorm : 0.0;
    for (int g = tid; g < p.G; g += kThreads) s.qprop[g] = s.qprop[g] * qinv + s.pdf[g] * pinv;
    __syncthreads();
  }
  if (tid == 0) {
    const double u = p.uni[(long)w * p.nC + c];
    int count = 0;
    double factor = pnorm;
    if (!learned) {
      double cum = s.pdf[0];
      while ((cum <= u) && (count < p.G - 1)) {
        count += 1;
        cum += s.pdf[count];
      }
    } else {
      // first support point whose cumulative q~ exceeds u (the last one if rounding leaves u above)
      double cum = 0.0;
      int last = 0;
      for (int g = 0; g < p.G; ++g) {
        if (s.qprop[g] <= 0.0) continue;
        last = g;
        cum += s.qprop[g];
        if (cum > u) break;
      }
      count = last;
      factor = s.pdf[count] / s.qprop[count];
      wt *= factor;
    }
    const double *x = p.grid + 4 * count;
    double nm = 0.0;
    for (int l = 0; l < 4; ++l)
      for (int r = 0; r < 4; ++r) nm += s.Cm[l + 4 * r] * x[l] * x[r];
    s.sc[1] = 4.0 * nm;
    s.sc[2] = count;
    s.sc[3] = u;
    s.sc[4] = factor;
    s.sc[5] = wt;
    for (int q = 0; q < 4; ++q) {
      double o1 = 0.0, o2 = 0.0;
      for (int k = 0; k < 4; ++k) {
        const double pf = 2.0 * Sq[k] * x[k];  // sqrt(4 s_k) x_k
        o1 += pf * U[q + 4 * k];
        o2 += pf * VT[k + 4 * q];
      }
      s.O1[q] = o1;
      s.O2[q] = o2;
    }
  }
  __syncthreads();
  if (learned) wt = s.sc[5];  // thread 0 updated it
  return s.sc[1];
}

// Site operator O (2x2, O[s + 2t]) on a site held in smem (rows r < dl, columns < dr, sigma
// stride sb, column stride ld), in place.  No barrier.
template <typename T>
__device__ __forceinline__ void apply_site_op(T *X, int ld, int sb, int dl, int dr, const double *O) {
  const T o0 = T(O[0]), o1 = T(O[1]), o2 = T(O[2]), o3 = T(O[3]);
  for (int q = threadIdx.x; q < dl * dr; q += kThreads) {
    const int r = q % dl, cc = q / dl;
    const T x0 = X[r + ld * cc], x1 = X[sb + r + ld * cc];
    X[r + ld * cc] = o0 * x0 + o2 * x1;
    X[sb + r + ld * cc] = o1 * x0 + o3 * x1;
  }
}

// The same on a site as stored in HBM (X[r + dl (c + dr sigma)], FP64), in place.  No barrier.
__device__ __forceinline__ void apply_site_op_stored(double *X, int dl, int dr, const double *O) {
  const int blk = dl * dr;
  for (int q = threadIdx.x; q < blk; q += kThreads) {
    const double x0 = X[q], x1 = X[blk + q];
    X[q] = O[0] * x0 + O[2] * x1;
    X[blk + q] = O[1] * x0 + O[3] * x1;
  }
}

// ||phi||^2 of the walker with the centre C on site i (sites > i as stored in global memory):
// N = sum_s A_k[s] N A_k[s]^T from site L-1 down to i+1 (in the norm-environment scratch), then
// sum_s tr(C[s]^T Nl C[s] N) with the left norm environment Nl of sites < i (ld pb), or the
// identity when those sites are orthonormal (Nl == nullptr).  Uses Nxt, Xb, Pb.  Only the trace
// mode calls it, to report the reference's normalised C_kl and overlaps.
template <typename T, int NP = 0>
static __device__ double norm_from_centre(const Dev &p, SmemT<T> &s, const double *W, T *scr, int i,
                                          const T *Nl = nullptr) {
  const int L = p.L, d = kMaxD, tid = threadIdx.x;
  if (tid == 0) scr[p.nroff[L]] = T(1);
  __syncthreads();
  for (int k = L - 1; k > i; --k) {
    const int bl = s.bW[k], br = s.bW[k + 1];
    load_site(s.Nxt, p.pb, s.sbC, W + s.woff[k], bl, br);
    __syncthreads();
    const T *Nn = scr + p.nroff[k + 1];
    T *Nk = scr + p.nroff[k];
    for (int sg = 0; sg < d; ++sg)
      gemm_t<NP>(br, bl, br, T(1), Nn, br, false, s.Nxt + sg * s.sbC, p.pb, true, T(0), s.Pb + sg * s.sbX, p.pa);
    __syncthreads();
    for (int sg = 0; sg < d; ++sg)
      gemm_t<NP>(bl, bl, br, T(1), s.Nxt + sg * s.sbC, p.pb, false, s.Pb + sg * s.sbX, p.pa, false,
                 sg == 0 ? T(0) : T(1), Nk, bl);
    __syncthreads();
  }
  const int bl = s.bW[i], br = s.bW[i + 1];
  const T *N1 = scr + p.nroff[i + 1];
  for (int sg = 0; sg < d; ++sg)
    gemm_t<NP>(bl, br, br, T(1), s.Cen + sg * s.sbC, p.pb, false, N1, br, false, T(0), s.Xb + sg * s.sbX, p.pa);
  __syncthreads();
  const T *Z = s.Xb;
  if (Nl != nullptr) {
    for (int sg = 0; sg < d; ++sg)
      gemm_t<NP>(bl, br, bl, T(1), Nl, p.pb, false, s.Xb + sg * s.sbX, p.pa, false, T(0), s.Pb + sg * s.sbX, p.pa);
    __syncthreads();
    Z = s.Pb;
  }
  double part = 0.0;
  for (int q = tid; q < bl * br * d; q += kThreads) {
    const int r = q % bl, rest = q / bl, cc = rest % br, sg = rest / br;
    part += (double)s.Cen[sg * s.sbC + r + p.pb * cc] * (double)Z[sg * s.sbX + r + p.pa * cc];
  }
  return cta_sum(part, s.red);
}

#ifndef MQ_DEVICE_ONLY

// The walker step (all walkers of the population, one CTA per walker at a time).
// QM: 1 the QR-free sweep, 2 the QR per site, 0 either, chosen by p.nloff at run time.  TR: the
// per-coupling trace is compiled in (recorded when p.trace is set).  The chain sweeps run as
// separate instantiations (fewer registers spilled); for couplings of any range one
// instantiation choosing at run time measured faster.
template <typename T, int NP, bool ZB, int QM, bool TR = true>
__device__ __forceinline__ void general_step(const Dev &p, double *smem_raw) {
  const bool QF = QM == 1 || (QM == 0 && p.nloff >= 0);
  const bool traced = TR && p.trace != nullptr;
  constexpr bool kMixed = !std::is_same<T, double>::value;
  SmemT<T> s;
  if constexpr (kMixed) carve(p, s, smem_raw);
  else carve(p, s, smem_raw, !QF);  // the QR-free sweep has no Householder buffers
  const int L = p.L, d = kMaxD, tid = threadIdx.x;
  const int N = *p.n_cur;
  T *scr = reinterpret_cast<T *>(p.scratch) + (long)blockIdx.x * p.scr_stride;
  const long fm = (long)p.maxA * p.maxB;
  T *Fdone[2] = {scr + p.choff, scr + p.choff + fm};
  T *Fch = scr + p.choff + 2 * fm;
  T *Nl = QF ? scr + p.nloff : nullptr;  // left norm environment (QR-free sweep)
  const T *trial = trial_of<T>(p);
  for (int w = next_walker(s, p.ctr + kCtrStep); w < N; w = next_walker(s, p.ctr + kCtrStep)) {
    const int slot = p.slot_of[w];
    load_walker_dims(p, s, slot);
    double *W = p.walkers + (long)slot * p.wstride;
    // right environments of the walker as stored
    if (tid == 0) {
      scr[p.roff[L]] = T(1);
      if (QF) Nl[0] = T(1);
    }
    for (int k = L - 1; k >= 1; --k) right_env_step<T, NP, ZB>(p, s, W, scr, k);
    int rv = 1;  // R[k] is valid for k >= rv
    // centre on site 0: overlap <Psi_T|phi> (the stored walker is normalised, overlap > 0)
    double ov;
    {
      const int a1 = p.aT[1], b1 = s.bW[1];
      load_site(s.Cen, p.pb, s.sbC, W + s.woff[0], 1, b1);
      __syncthreads();
      const T *R1 = scr + p.roff[1], *B0 = trial + p.toff[0];
      double part = 0.0;
      for (int q = tid; q < a1 * b1 * d; q += kThreads) {
        const int a = q % a1, rest = q / a1, b = rest % b1, sg = rest / b1;
        part += (double)B0[a + a1 * sg] * (double)R1[a + a1 * b] * (double)s.Cen[sg * s.sbC + p.pb * b];
      }
      ov = cta_sum(part, s.red);
    }
    double wt = p.weight[slot];
    double nrm_prev = 1.0;  // trace mode: norm of the walker before the current coupling
    if (traced) nrm_prev = sqrt(norm_from_centre<T, NP>(p, s, W, scr, 0));
    if (tid == 0) s.Lenv[0] = T(1);
    int cur = 0;
    __syncthreads();
    for (int i = 0; i < L; ++i) {
      const int al = p.aT[i], ar = p.aT[i + 1], bl = s.bW[i], br = s.bW[i + 1];
      const T *Bi = trial + p.toff[i];
      // the walker's next site, and on chains the right branches this site's coupling closes with
      // (formed in the right-environment sweep, since evicted from L2): fetched ahead
      if (i + 1 < L) {
        prefetch_l2(W + s.woff[i + 1], (long)br * s.bW[i + 2] * d);
        if constexpr (ZB) prefetch_l2(scr + p.zoff[i + 1], 4L * ar * br);
      }
      // Pb still holds the last coupling's left branches at cut i+1 (its partner was i+1, so they
      // were not carried further, and the trace did not use Pb as scratch)
      bool branches_kept = false;
      for (int c = p.site_c0[i]; c < p.site_c0[i + 1]; ++c) {
        const int j = p.cp_j[c];
        while (rv > (ZB ? j : j + 1)) {  // R[j+1] (and the right branches of site j) up to date
          --rv;
          right_env_step<T, NP, ZB>(p, s, W, scr, rv);
        }
        if constexpr (!ZB) {  // what the closures read after the middle sites: site j and R[j+1]
          if (j > i + 1) prefetch_l2(W + s.woff[j], (long)s.bW[j] * s.bW[j + 1] * d);
          prefetch_l2(scr + p.roff[j + 1], (long)p.aT[j + 1] * s.bW[j + 1]);
        }
        // left branches P[s + d t] = B_i[s]^T Lenv C[t] (a_{i+1} x b_{i+1})
        for (int tau = 0; tau < d; ++tau)
          gemm_t<NP>(al, br, bl, T(1), s.Lenv, p.pa, false, s.Cen + tau * s.sbC, p.pb, false, T(0),
                     s.Xb + tau * s.sbX, p.pa);
        __syncthreads();
        for (int sg = 0; sg < d; ++sg)
          for (int tau = 0; tau < d; ++tau)
            gemm_t<NP>(ar, br, al, T(1), Bi + (long)sg * al * ar, al, true, s.Xb + tau * s.sbX, p.pa, false, T(0),
                       s.Pb + (sg + d * tau) * s.sbX, p.pa);
        __syncthreads();
        // through the middle sites
        for (int m = i + 1; m < j; ++m) {
          const int am = p.aT[m], am1 = p.aT[m + 1], bm = s.bW[m], bm1 = s.bW[m + 1];
          load_site(s.Nxt, p.pb, s.sbC, W + s.woff[m], bm, bm1);
          if (m + 1 < j) prefetch_l2(W + s.woff[m + 1], (long)bm1 * s.bW[m + 2] * d);
          __syncthreads();
          const T *Bm = trial + p.toff[m];
          for (int q = 0; q < kN2; ++q)
            transfer_in_place<T, NP>(p, s, Bm, am, am1, bm, bm1, s.Nxt, p.pb, s.sbC, s.Pb + q * s.sbX, p.pa);
        }
        // closures with the right branches of site j, sample, site operators
        const int bj = s.bW[j], bj1 = s.bW[j + 1];
        __syncthreads();
        closures<T, NP, ZB>(p, s, j, W, scr);
        const double num = sample_coupling(p, s, w, c, p.cp_q[c], ov, wt);
        apply_site_op(s.Cen, p.pb, s.sbC, bl, br, s.O1);
        // O2 acts on site j as stored in HBM; in the mixed sweep the walker itself stays FP64, so
        // O1 acts on its stored site i as well (the FP32 centre only feeds the contractions)
        if constexpr (kMixed) apply_site_op_stored(W + s.woff[i], bl, br, s.O1);
        apply_site_op_stored(W + s.woff[j], bj, bj1, s.O2);
        __syncthreads();
        if (rv < j + 1) rv = j + 1;
        ov = num;
        branches_kept = (j == i + 1) && !traced;
        if (traced) {
          // the reference normalises after every coupling: report C of the normalised walker
          // and the normalised overlap (the walk itself does not need the norm)
          __syncthreads();
          const double nrm_after = sqrt(norm_from_centre<T, NP>(p, s, W, scr, i, Nl));
          if (tid == 0) {
            double *t = p.trace + ((long)w * p.nC + c) * kTraceStride;
            for (int k = 0; k < 16; ++k) t[k] = s.Cm[k] / nrm_prev;
            t[16] = s.sc[4];
            t[17] = s.sc[3];
            t[18] = s.sc[2];
            t[19] = wt;
            t[20] = ov / nrm_after;
          }
          nrm_prev = nrm_after;
        }
        __syncthreads();
      }
      if (QF && i < L - 1) {
        // QR-free: the centre itself becomes the final site i, rescaled to the Frobenius norm of
        // an isometry (sqrt(br)) so that the tensor scales cannot drift over the steps (the
        // overlap takes the same factor), and the left norm environment takes it in:
        // Nl' = sum_s C[s]^T Nl C[s]
        double *Wi = W + s.woff[i];
        double part = 0.0;
        for (int q = tid; q < bl * br * d; q += kThreads) {
          const int r = q % bl, rest = q / bl, cc = rest % br, sg = rest / br;
          const double x = kMixed ? Wi[q] : (double)s.Cen[sg * s.sbC + r + p.pb * cc];
          part += x * x;
        }
        const double inv = sqrt((double)br / cta_sum(part, s.red));
        for (int q = tid; q < bl * br * d; q += kThreads) {
          const int r = q % bl, rest = q / bl, cc = rest % br, sg = rest / br;
          s.Cen[sg * s.sbC + r + p.pb * cc] *= T(inv);
          if (kMixed) Wi[q] *= inv;
        }
        ov *= inv;
        nrm_prev *= inv;
        if (branches_kept) {
          // the left branches of the final site, without their products: P is linear in the
          // centre's sigma blocks, so P'[s, t] = inv sum_t' O1(t, t') P[s, t'] (O1 of the last coupling)
          const T o0 = T(inv * s.O1[0]), o1 = T(inv * s.O1[1]), o2 = T(inv * s.O1[2]), o3 = T(inv * s.O1[3]);
          for (int q = tid; q < ar * br; q += kThreads) {
            const int off = q % ar + p.pa * (q / ar);
#pragma unroll
            for (int sg = 0; sg < d; ++sg) {
              T *P0 = s.Pb + sg * s.sbX + off, *P1 = s.Pb + (sg + d) * s.sbX + off;
              const T x0 = *P0, x1 = *P1;
              *P0 = o0 * x0 + o2 * x1;
              *P1 = o1 * x0 + o3 * x1;
            }
          }
        }
        __syncthreads();
        if (!kMixed) store_site(Wi, s.Cen, p.pb, s.sbC, bl, br);
        for (int sg = 0; sg < d; ++sg)
          gemm_t<NP>(bl, br, bl, T(1), Nl, p.pb, false, s.Cen + sg * s.sbC, p.pb, false, T(0), s.Xb + sg * s.sbX,
                     p.pa);
        __syncthreads();
        for (int sg = 0; sg < d; ++sg)
          gemm_t<NP>(br, br, bl, T(1), s.Cen + sg * s.sbC, p.pb, true, s.Xb + sg * s.sbX, p.pa, false,
                     sg == 0 ? T(0) : T(1), Nl, p.pb);
        __syncthreads();
        env_update_general<T, NP>(p, s, i, Bi, al, ar, bl, br, s.Cen, p.pb, s.sbC, Fdone[cur], Fdone[1 - cur],
                                  Fch, branches_kept);
        cur = 1 - cur;
        load_site(s.Cen, p.pb, s.sbC, W + s.woff[i + 1], br, s.bW[i + 2]);
        __syncthreads();
      } else if (i < L - 1) {
        if constexpr (std::is_same<T, double>::value && QM != 1) {
          // QR of the centre: Q is the final site i, R moves into site i+1
          for (int q = tid; q < bl * br; q += kThreads) {
            const int r = q % bl, cc = q / bl;
            s.QRb[(r + bl * 0) + p.pq * cc] = s.Cen[r + p.pb * cc];
            s.QRb[(r + bl * 1) + p.pq * cc] = s.Cen[s.sbC + r + p.pb * cc];
          }
          __syncthreads();
          cta_householder_qr(bl * d, br, s.QRb, p.pq, s.Rf, p.pb, s.tau, s.wv, s.red);
          {
            double *Wi = W + s.woff[i];
            for (int q = tid; q < bl * br * d; q += kThreads) {
              const int r = q % bl, rest = q / bl, cc = rest % br, sg = rest / br;
              Wi[q] = s.QRb[(r + bl * sg) + p.pq * cc];
            }
          }
          const int b2 = s.bW[i + 2];
          load_site(s.Nxt, p.pb, s.sbC, W + s.woff[i + 1], br, b2);
          __syncthreads();
          for (int sg = 0; sg < d; ++sg)
            cta_gemm(br, b2, br, 1.0, s.Rf, p.pb, false, s.Nxt + sg * s.sbC, p.pb, false, 0.0, s.Cen + sg * s.sbC,
                     p.pb);
          __syncthreads();
          env_update_general<T, NP>(p, s, i, Bi, al, ar, bl, br, s.QRb, p.pq, bl, Fdone[cur], Fdone[1 - cur], Fch);
          cur = 1 - cur;
        }
      } else {
        // last site: energy and overlap of the unnormalised walker, then normalise the centre
        env_update_general<T, NP>(p, s, i, Bi, al, 1, bl, 1, s.Cen, p.pb, s.sbC, Fdone[cur], Fdone[1 - cur], Fch);
        double *Wi = W + s.woff[i];
        double part = 0.0;
        for (int q = tid; q < bl * d; q += kThreads) {  // site L-1: bl x 1 per sigma
          const T *cs = s.Cen + (q / bl) * s.sbC;
          const double *ws = Wi + (q / bl) * bl;  // the FP64 walker (mixed sweep)
          const double x = kMixed ? ws[q % bl] : (double)cs[q % bl];
          if (!QF) {
            part += x * x;
          } else {  // x (Nl c)_r
            double y = 0.0;
            for (int k = 0; k < bl; ++k) y += (double)Nl[(q % bl) + p.pb * k] * (kMixed ? ws[k] : (double)cs[k]);
            part += x * y;
          }
        }
        const double nrm = sqrt(cta_sum(part, s.red));
        const double ovr = s.Lenv[0];
        const double en = Fdone[1 - cur][0];
        const double scale = (ovr < 0.0) ? -1.0 / nrm : 1.0 / nrm;
        if (kMixed) {
          for (int q = tid; q < bl * d; q += kThreads) Wi[q] *= scale;
        } else {
          for (int q = tid; q < bl * d; q += kThreads) s.Cen[(q / bl) * s.sbC + (q % bl)] *= T(scale);
          __syncthreads();
          store_site(Wi, s.Cen, p.pb, s.sbC, bl, 1);
        }
        if (tid == 0) {
          const double ovf = fabs(ovr) / nrm;
          const double ew = en / ovr;
          p.overlap[slot] = ovf;
          p.weight[slot] = wt;
          p.energy[w] = ew;
          p.ov_out[w] = ovf;
          p.wt_out[w] = wt;
          if (!(isfinite(wt) && isfinite(ovf) && isfinite(ew))) atomicOr(p.err, kErrNumeric);
        }
        __syncthreads();
      }
    }
  }
}

// ZB: nearest-neighbour couplings, right branches stored per site (a separate instantiation, so
// the register allocation of each sweep carries one closure path only).
template <bool ZB, int QM, bool TR = true>
__global__ void __launch_bounds__(kThreads, 1) walker_step_general_kernel(Dev p) {
  extern __shared__ double smem_raw[];
  general_step<double, 0, ZB, QM, TR>(p, smem_raw);
}

// Mixed precision: FP32 work buffers, TF32 tensor cores (NP passes), always QR-free.  Half the
// shared memory of the FP64 sweep, so two CTAs fit on an SM where the FP64 sweep fits one.
template <int NP, bool ZB>
__global__ void __launch_bounds__(kThreads, 2) walker_step_mixed_kernel(Dev p) {
  extern __shared__ double smem_raw[];
  general_step<float, NP, ZB, 1, true>(p, smem_raw);
}

// <Psi_T|H|phi> / overlap for every walker (any coupling range), tensors as stored.
__global__ void __launch_bounds__(kThreads, 1) energy_general_kernel(Dev p) {
  extern __shared__ double smem_raw[];
  Smem s;
  carve(p, s, smem_raw);
  const int L = p.L, tid = threadIdx.x;
  const int N = *p.n_cur;
  double *scr = p.scratch + (long)blockIdx.x * p.scr_stride;
  const long fm = (long)p.maxA * p.maxB;
  double *Fdone[2] = {scr + p.choff, scr + p.choff + fm};
  double *Fch = scr + p.choff + 2 * fm;
  for (int w = next_walker(s, p.ctr + kCtrEnergy); w < N; w = next_walker(s, p.ctr + kCtrEnergy)) {
    const int slot = p.slot_of[w];
    load_walker_dims(p, s, slot);
    const double *W = p.walkers + (long)slot * p.wstride;
    if (tid == 0) s.Lenv[0] = 1.0;
    __syncthreads();
    int cur = 0;
    for (int k = 0; k < L; ++k) {
      const int al = p.aT[k], ar = p.aT[k + 1], bl = s.bW[k], br = s.bW[k + 1];
      env_update_general<double, 0>(p, s, k, p.trial + p.toff[k], al, ar, bl, br, W + s.woff[k], bl, bl * br,
                                    Fdone[cur], Fdone[1 - cur], Fch);
      cur = 1 - cur;
    }
    if (tid == 0) {
      const double en = Fdone[cur][0];
      p.energy[w] = en / p.overlap[slot];
      p.ov_out[w] = p.overlap[slot];
      p.wt_out[w] = p.weight[slot];
    }
    __syncthreads();
  }
}

#endif  // MQ_DEVICE_ONLY

}  // namespace mq
