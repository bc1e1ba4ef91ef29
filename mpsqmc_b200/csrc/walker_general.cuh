// Walker step for couplings of any range (sm_100a, FP64): 2D lattices on a snake path and other
// long-range Heisenberg models, with the coupling order of MPSQMC2.cpp:286-299 (by first site,
// then by second site).
//
// One CTA per walker, as in walker_step_kernel.  The centre of the walker moves left to right;
// while it sits on site i every coupling (i, j) is processed:
//   1. right environment R[j+1] = <Psi_T|phi> over sites j+1..L-1, recomputed from the first
//      still-valid one when an earlier coupling changed a site beyond j;
//   2. four left branches P[s,t] = B_i[s]^T L C[t] on the centre, carried through the middle
//      sites i+1..j-1 by ordinary transfer steps, four right branches at j and 16 closures give
//      C_kl = <Psi_T|(sqrt(s_k)U_k)_i (sqrt(s_l)V_l)_j|phi> (MPSQMC2.cpp:540-549);
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
#pragma once

#include "walker_kernels.cuh"

namespace mq {

// R[k] = sum_s B_k[s] R[k+1] A_k[s]^T from the walker's site k as stored in global memory.
// Uses Nxt and Xb.  Ends with a barrier.
static __device__ void right_env_step(const Dev &p, Smem &s, const double *W, double *scr, int k) {
  const int d = kMaxD;
  const int al = p.aT[k], ar = p.aT[k + 1], bl = s.bW[k], br = s.bW[k + 1];
  load_site(s.Nxt, p.pb, s.sbC, W + s.woff[k], bl, br);
  __syncthreads();
  const double *Rn = scr + p.roff[k + 1];
  double *Rk = scr + p.roff[k];
  const double *Bk = p.trial + p.toff[k];
  for (int sg = 0; sg < d; ++sg)
    cta_gemm(ar, bl, br, 1.0, Rn, ar, false, s.Nxt + sg * s.sbC, p.pb, true, 0.0, s.Xb + sg * s.sbX, p.pa);
  __syncthreads();
  for (int sg = 0; sg < d; ++sg)
    cta_gemm(al, bl, ar, 1.0, Bk + (long)sg * al * ar, al, false, s.Xb + sg * s.sbX, p.pa, false,
             sg == 0 ? 0.0 : 1.0, Rk, al);
  __syncthreads();
}

// E <- sum_s B[s]^T E T[s] in place (E: al x bl -> ar x br, leading dimension lde).  T[s] is
// bl x br with column stride cs and sigma stride ss.  Uses Xb.  Ends with a barrier.
static __device__ void transfer_in_place(const Dev &p, Smem &s, const double *B, int al, int ar, int bl,
                                         int br, const double *T, int cs, int ss, double *E, int lde) {
  const int d = kMaxD;
  for (int sg = 0; sg < d; ++sg)
    cta_gemm(al, br, bl, 1.0, E, lde, false, T + sg * ss, cs, false, 0.0, s.Xb + sg * s.sbX, p.pa);
  __syncthreads();
  for (int sg = 0; sg < d; ++sg)
    cta_gemm(ar, br, al, 1.0, B + (long)sg * al * ar, al, true, s.Xb + sg * s.sbX, p.pa, false,
             sg == 0 ? 0.0 : 1.0, E, lde);
  __syncthreads();
}

// Left environments through the final tensor T of site k (T[s] bl x br, column stride cs,
// sigma stride ss): trial overlap Lenv, "done" channel Fd -> Fdn, open channels in Fch
// (slot q, operator a at Fch + (3q + a) * maxA * maxB, leading dimension maxA).
// Order: branches P; done' from Fd, the channels that close on k and the field; channels that
// stay open; then Lenv' and the channel site k opens (its slot may be one that closed on k).
static __device__ void env_update_general(const Dev &p, Smem &s, int k, const double *B, int al, int ar,
                                          int bl, int br, const double *T, int cs, int ss, const double *Fd,
                                          double *Fdn, double *Fch) {
  const int d = kMaxD, lda = p.maxA;
  const long fm = (long)p.maxA * p.maxB;
  // P[s + d t] = B[s]^T Lenv T[t]    (ar x br)
  for (int tau = 0; tau < d; ++tau)
    cta_gemm(al, br, bl, 1.0, s.Lenv, p.pa, false, T + tau * ss, cs, false, 0.0, s.Xb + tau * s.sbX, p.pa);
  __syncthreads();
  for (int sg = 0; sg < d; ++sg)
    for (int tau = 0; tau < d; ++tau)
      cta_gemm(ar, br, al, 1.0, B + (long)sg * al * ar, al, true, s.Xb + tau * s.sbX, p.pa, false, 0.0,
               s.Pb + (sg + d * tau) * s.sbX, p.pa);
  __syncthreads();
  // done' = -h sum Sz P + sum_s B[s]^T (sum_t G_st T[t]),
  // G_st = delta_st Fd + sum_{i closing on k} J_ik (Sx F_i,x - iSy F_i,iy + Sz F_i,z)(s,t)
  for (int q = threadIdx.x; q < ar * br; q += kThreads) {
    const int r = q % ar, c = q / ar;
    double fz = 0.0;
#pragma unroll
    for (int e = 0; e < kN2; ++e) fz += p.opSz[e] * s.Pb[e * s.sbX + r + p.pa * c];
    Fdn[r + lda * c] = -p.h * fz;
  }
  __syncthreads();
  const int e0 = p.ech_off[k], e1 = p.ech_off[k + 1];
  if (k > 0) {
    for (int sg = 0; sg < d; ++sg) {
      for (int q = threadIdx.x; q < al * bl; q += kThreads) {
        const int r = q % al, c = q / al;
        const double fd = Fd[r + lda * c];
        double gx = 0.0, gy = 0.0, gz = 0.0;
        for (int e = e0; e < e1; ++e) {
          const double J = p.ech_J[e];
          if (J == 0.0) continue;
          const double *F = Fch + 3L * p.ech_slot[e] * fm;
          gx += J * F[r + lda * c];
          gy += J * F[fm + r + lda * c];
          gz += J * F[2 * fm + r + lda * c];
        }
        for (int tau = 0; tau < d; ++tau) {
          const int o = sg + d * tau;
          s.Xb[tau * s.sbX + r + p.pa * c] =
              ((sg == tau) ? fd : 0.0) + p.opSx[o] * gx - p.opISy[o] * gy + p.opSz[o] * gz;
        }
      }
      __syncthreads();
      cta_gemm(al, br, bl, 1.0, s.Xb, p.pa, false, T, cs, false, 0.0, s.Qt, p.pa);
      for (int tau = 1; tau < d; ++tau)
        cta_gemm(al, br, bl, 1.0, s.Xb + tau * s.sbX, p.pa, false, T + tau * ss, cs, false, 1.0, s.Qt, p.pa);
      __syncthreads();
      cta_gemm(ar, br, al, 1.0, B + (long)sg * al * ar, al, true, s.Qt, p.pa, false, 1.0, Fdn, lda);
      __syncthreads();
    }
  }
  // channels that stay open: identity on site k
  for (int e = e0; e < e1; ++e) {
    if (!p.ech_cont[e]) continue;
    double *F = Fch + 3L * p.ech_slot[e] * fm;
    for (int a = 0; a < 3; ++a) transfer_in_place(p, s, B, al, ar, bl, br, T, cs, ss, F + a * fm, lda);
  }
  // Lenv' = sum_s P[s,s]; the channels opened on site k
  const int op = p.eopen[k];
  double *Fo = (op >= 0) ? Fch + 3L * op * fm : nullptr;
  for (int q = threadIdx.x; q < ar * br; q += kThreads) {
    const int r = q % ar, c = q / ar;
    double P[kN2];
#pragma unroll
    for (int e = 0; e < kN2; ++e) P[e] = s.Pb[e * s.sbX + r + p.pa * c];
    double l = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
#pragma unroll
    for (int e = 0; e < kN2; ++e) {
      if ((e % d) == (e / d)) l += P[e];
      fx += p.opSx[e] * P[e];
      fy += p.opISy[e] * P[e];
      fz += p.opSz[e] * P[e];
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

// Closures of the four left branches in Pb (cut j, a_j x b_j) with the right branches of site j
// (walker site in Nxt, R[j+1] at Rn): M[p + 4q] = <P_p, B_j[s'] R[j+1] A_j[t']^T>, q = s' + 2t'.
static __device__ void closures(const Dev &p, Smem &s, int j, const double *Rn) {
  const int d = kMaxD;
  const int aj = p.aT[j], a2 = p.aT[j + 1], bj = s.bW[j], b2 = s.bW[j + 1];
  const double *Bj = p.trial + p.toff[j];
  for (int tau = 0; tau < d; ++tau)
    cta_gemm(a2, bj, b2, 1.0, Rn, a2, false, s.Nxt + tau * s.sbC, p.pb, true, 0.0, s.Xb + tau * s.sbX, p.pa);
  __syncthreads();
  // M[k + 4 (s' + 2 t')] = <P_k, B_j[s'] Y[t']>, the products formed and dotted in one pass
  if (((aj | bj | a2) & 15) == 0)
    cta_closure16<true>(aj, bj, a2, Bj, aj, (long)aj * a2, s.Xb, p.pa, s.sbX, s.Pb, p.pa, s.sbX, s.red, s.M);
  else
    cta_closure16<false>(aj, bj, a2, Bj, aj, (long)aj * a2, s.Xb, p.pa, s.sbX, s.Pb, p.pa, s.sbX, s.red, s.M);
}

// C_kl from the closures, PDF over the grid, weight update, CDF sample with the walker's uniform
// for coupling c, and the site operators O1, O2 (MPSQMC2.cpp:551-588, MPSstate.cpp:575-633).
// Returns 4 sum_kl C_kl x_k x_l of the sampled point (the new unnormalised overlap).
static __device__ double sample_coupling(const Dev &p, Smem &s, int w, int c, int jq, double ov, double &wt) {
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
  const double pinv = 1.0 / pnorm;
  for (int g = tid; g < p.G; g += kThreads) s.pdf[g] *= pinv;
  wt *= pnorm;
  __syncthreads();
  if (tid == 0) {
    const double u = p.uni[(long)w * p.nC + c];
    int count = 0;
    double cum = s.pdf[0];
    while ((cum <= u) && (count < p.G - 1)) {
      count += 1;
      cum += s.pdf[count];
    }
    const double *x = p.grid + 4 * count;
    double nm = 0.0;
    for (int l = 0; l < 4; ++l)
      for (int r = 0; r < 4; ++r) nm += s.Cm[l + 4 * r] * x[l] * x[r];
    s.sc[1] = 4.0 * nm;
    s.sc[2] = count;
    s.sc[3] = u;
    s.sc[4] = pnorm;
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
  return s.sc[1];
}

// Site operator O (2x2, O[s + 2t]) on a site held in smem (rows r < dl, columns < dr, sigma
// stride sb, column stride ld), in place.  No barrier.
__device__ __forceinline__ void apply_site_op(double *X, int ld, int sb, int dl, int dr, const double *O) {
  for (int q = threadIdx.x; q < dl * dr; q += kThreads) {
    const int r = q % dl, cc = q / dl;
    const double x0 = X[r + ld * cc], x1 = X[sb + r + ld * cc];
    X[r + ld * cc] = O[0] * x0 + O[2] * x1;
    X[sb + r + ld * cc] = O[1] * x0 + O[3] * x1;
  }
}

// ||phi||^2 of the walker with the centre C on site i (sites < i orthonormal, sites > i as stored
// in global memory): N = sum_s A_k[s] N A_k[s]^T from site L-1 down to i+1 (in the norm-environment
// scratch), then sum_s tr(C[s] N C[s]^T).  Uses Nxt, Xb, Pb.  Only the trace mode calls it, to
// report the reference's normalised C_kl and overlaps.
static __device__ double norm_from_centre(const Dev &p, Smem &s, const double *W, double *scr, int i) {
  const int L = p.L, d = kMaxD, tid = threadIdx.x;
  if (tid == 0) scr[p.nroff[L]] = 1.0;
  __syncthreads();
  for (int k = L - 1; k > i; --k) {
    const int bl = s.bW[k], br = s.bW[k + 1];
    load_site(s.Nxt, p.pb, s.sbC, W + s.woff[k], bl, br);
    __syncthreads();
    const double *Nn = scr + p.nroff[k + 1];
    double *Nk = scr + p.nroff[k];
    for (int sg = 0; sg < d; ++sg)
      cta_gemm(br, bl, br, 1.0, Nn, br, false, s.Nxt + sg * s.sbC, p.pb, true, 0.0, s.Pb + sg * s.sbX, p.pa);
    __syncthreads();
    for (int sg = 0; sg < d; ++sg)
      cta_gemm(bl, bl, br, 1.0, s.Nxt + sg * s.sbC, p.pb, false, s.Pb + sg * s.sbX, p.pa, false,
               sg == 0 ? 0.0 : 1.0, Nk, bl);
    __syncthreads();
  }
  const int bl = s.bW[i], br = s.bW[i + 1];
  const double *N1 = scr + p.nroff[i + 1];
  for (int sg = 0; sg < d; ++sg)
    cta_gemm(bl, br, br, 1.0, s.Cen + sg * s.sbC, p.pb, false, N1, br, false, 0.0, s.Xb + sg * s.sbX, p.pa);
  __syncthreads();
  double part = 0.0;
  for (int q = tid; q < bl * br * d; q += kThreads) {
    const int r = q % bl, rest = q / bl, cc = rest % br, sg = rest / br;
    part += s.Cen[sg * s.sbC + r + p.pb * cc] * s.Xb[sg * s.sbX + r + p.pa * cc];
  }
  return cta_sum(part, s.red);
}

#ifndef MQ_DEVICE_ONLY

__global__ void __launch_bounds__(kThreads, 1) walker_step_general_kernel(Dev p) {
  extern __shared__ double smem_raw[];
  Smem s;
  carve(p, s, smem_raw);
  const int L = p.L, d = kMaxD, tid = threadIdx.x;
  const int N = *p.n_cur;
  double *scr = p.scratch + (long)blockIdx.x * p.scr_stride;
  const long fm = (long)p.maxA * p.maxB;
  double *Fdone[2] = {scr + p.choff, scr + p.choff + fm};
  double *Fch = scr + p.choff + 2 * fm;
  for (int w = next_walker(s, p.ctr + kCtrStep); w < N; w = next_walker(s, p.ctr + kCtrStep)) {
    const int slot = p.slot_of[w];
    load_walker_dims(p, s, slot);
    double *W = p.walkers + (long)slot * p.wstride;
    // right environments of the walker as stored
    if (tid == 0) scr[p.roff[L]] = 1.0;
    for (int k = L - 1; k >= 1; --k) right_env_step(p, s, W, scr, k);
    int rv = 1;  // R[k] is valid for k >= rv
    // centre on site 0: overlap <Psi_T|phi> (the stored walker is normalised, overlap > 0)
    double ov;
    {
      const int a1 = p.aT[1], b1 = s.bW[1];
      load_site(s.Cen, p.pb, s.sbC, W + s.woff[0], 1, b1);
      __syncthreads();
      const double *R1 = scr + p.roff[1], *B0 = p.trial + p.toff[0];
      double part = 0.0;
      for (int q = tid; q < a1 * b1 * d; q += kThreads) {
        const int a = q % a1, rest = q / a1, b = rest % b1, sg = rest / b1;
        part += B0[a + a1 * sg] * R1[a + a1 * b] * s.Cen[sg * s.sbC + p.pb * b];
      }
      ov = cta_sum(part, s.red);
    }
    double wt = p.weight[slot];
    double nrm_prev = 1.0;  // trace mode: norm of the walker before the current coupling
    if (p.trace != nullptr) nrm_prev = sqrt(norm_from_centre(p, s, W, scr, 0));
    if (tid == 0) s.Lenv[0] = 1.0;
    int cur = 0;
    __syncthreads();
    for (int i = 0; i < L; ++i) {
      const int al = p.aT[i], ar = p.aT[i + 1], bl = s.bW[i], br = s.bW[i + 1];
      const double *Bi = p.trial + p.toff[i];
      for (int c = p.site_c0[i]; c < p.site_c0[i + 1]; ++c) {
        const int j = p.cp_j[c];
        while (rv > j + 1) {
          --rv;
          right_env_step(p, s, W, scr, rv);
        }
        // left branches P[s + d t] = B_i[s]^T Lenv C[t] (a_{i+1} x b_{i+1})
        for (int tau = 0; tau < d; ++tau)
          cta_gemm(al, br, bl, 1.0, s.Lenv, p.pa, false, s.Cen + tau * s.sbC, p.pb, false, 0.0,
                   s.Xb + tau * s.sbX, p.pa);
        __syncthreads();
        for (int sg = 0; sg < d; ++sg)
          for (int tau = 0; tau < d; ++tau)
            cta_gemm(ar, br, al, 1.0, Bi + (long)sg * al * ar, al, true, s.Xb + tau * s.sbX, p.pa, false, 0.0,
                     s.Pb + (sg + d * tau) * s.sbX, p.pa);
        __syncthreads();
        // through the middle sites
        for (int m = i + 1; m < j; ++m) {
          const int am = p.aT[m], am1 = p.aT[m + 1], bm = s.bW[m], bm1 = s.bW[m + 1];
          load_site(s.Nxt, p.pb, s.sbC, W + s.woff[m], bm, bm1);
          __syncthreads();
          const double *Bm = p.trial + p.toff[m];
          for (int q = 0; q < kN2; ++q)
            transfer_in_place(p, s, Bm, am, am1, bm, bm1, s.Nxt, p.pb, s.sbC, s.Pb + q * s.sbX, p.pa);
        }
        // right branches at j, closures, sample
        const int bj = s.bW[j], bj1 = s.bW[j + 1];
        load_site(s.Nxt, p.pb, s.sbC, W + s.woff[j], bj, bj1);
        __syncthreads();
        closures(p, s, j, scr + p.roff[j + 1]);
        const double num = sample_coupling(p, s, w, c, p.cp_q[c], ov, wt);
        apply_site_op(s.Cen, p.pb, s.sbC, bl, br, s.O1);
        apply_site_op(s.Nxt, p.pb, s.sbC, bj, bj1, s.O2);
        __syncthreads();
        store_site(W + s.woff[j], s.Nxt, p.pb, s.sbC, bj, bj1);
        if (rv < j + 1) rv = j + 1;
        ov = num;
        if (p.trace != nullptr) {
          // the reference normalises after every coupling: report C of the normalised walker
          // and the normalised overlap (the walk itself does not need the norm)
          __syncthreads();
          const double nrm_after = sqrt(norm_from_centre(p, s, W, scr, i));
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
      if (i < L - 1) {
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
        env_update_general(p, s, i, Bi, al, ar, bl, br, s.QRb, p.pq, bl, Fdone[cur], Fdone[1 - cur], Fch);
        cur = 1 - cur;
      } else {
        // last site: energy and overlap of the unnormalised walker, then normalise the centre
        env_update_general(p, s, i, Bi, al, 1, bl, 1, s.Cen, p.pb, s.sbC, Fdone[cur], Fdone[1 - cur], Fch);
        double part = 0.0;
        for (int q = tid; q < bl * d; q += kThreads) {  // site L-1: bl x 1 per sigma
          const double x = s.Cen[(q / bl) * s.sbC + (q % bl)];
          part += x * x;
        }
        const double nrm = sqrt(cta_sum(part, s.red));
        const double ovr = s.Lenv[0];
        const double en = Fdone[1 - cur][0];
        const double scale = (ovr < 0.0) ? -1.0 / nrm : 1.0 / nrm;
        for (int q = tid; q < bl * d; q += kThreads) s.Cen[(q / bl) * s.sbC + (q % bl)] *= scale;
        __syncthreads();
        store_site(W + s.woff[i], s.Cen, p.pb, s.sbC, bl, 1);
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
      env_update_general(p, s, k, p.trial + p.toff[k], al, ar, bl, br, W + s.woff[k], bl, bl * br, Fdone[cur],
                         Fdone[1 - cur], Fch);
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
