// The MPO-term projector of MPSQMC::PropagateSeparately (MPSQMC.cpp:322-369), one CTA per walker.
//
// exp(-dtau H) is sampled one Hamiltonian term at a time: with the terms t of the MPO's
// term list (HeisenbergMPO.cpp:456-553: per coupling J Sx Sx, -J iSy iSy, J Sz Sz; per site
// -h Sz), PDF[0] = 1 (identity) and PDF[t+1] = max(-dtau <t Psi_T|phi> / ov, 0); the walker's
// weight takes the PDF norm, one uniform picks a term, and a picked term is applied to the walker,
// which is then left-normalised with its overlap recomputed and its sign fixed (Walker-free
// setOverlap of MPSQMC.cpp:356-364, done by set_overlap_kernel for the walkers flagged here).
//
// The reference stores nTerms copies of Psi_T with each term applied and takes one full-chain
// InnerProduct per term.  Here one sweep over the unchanged walker gives every term's overlap:
// right environments R[k], left environment L and, per coupling (i, j), the four left branches
// carried to j and closed with the right branches (the 16 closures M of the Trotter walk); a term
// A_i B_j then has <Psi_T|A_i B_j|phi> = sum A(s,t) B(s',t') M[(s,t),(s',t')].  Field terms close
// the left branches of site k with R[k+1].
#pragma once

#include "walker_general.cuh"

namespace mq {

struct LegacyDev {
  int nterms;
  const int *term_slot;    // [nterms]: index of the term's overlap in the per-walker table
  const double *term_pref; // [nterms]: prefactor
  const int *term_site;    // [nterms][2]: sites (second -1 for a one-site term)
  const int *term_op;      // [nterms][2]: 1 Sx, 2 iSy, 3 Sz
  double dtau;
  long loff;               // per-CTA table of term overlaps and PDF inside the scratch
  int *changed;            // [N]: 1 if the walker was hit by a term this step
  double *tr;              // optional per-walker trace: [N][3] = PDF norm, uniform, picked index
};

__device__ __forceinline__ const double *legacy_op(const Dev &p, int code) {
  return code == 1 ? p.opSx : (code == 2 ? p.opISy : p.opSz);
}

#ifndef MQ_DEVICE_ONLY

__global__ void __launch_bounds__(kThreads, 1) legacy_step_kernel(Dev p, LegacyDev lp) {
  extern __shared__ double smem_raw[];
  Smem s;
  carve(p, s, smem_raw);
  const int L = p.L, d = kMaxD, tid = threadIdx.x;
  const int N = *p.n_cur;
  double *scr = p.scratch + (long)blockIdx.x * p.scr_stride;
  double *tov = scr + lp.loff;             // overlaps: 3 per coupling, then one per site
  double *pdf = tov + 3 * p.nC + L;        // nterms + 1
  for (int w = next_walker(s, p.ctr + kCtrStep); w < N; w = next_walker(s, p.ctr + kCtrStep)) {
    const int slot = p.slot_of[w];
    load_walker_dims(p, s, slot);
    double *W = p.walkers + (long)slot * p.wstride;
    if (tid == 0) scr[p.roff[L]] = 1.0;
    for (int k = L - 1; k >= 1; --k) right_env_step(p, s, W, scr, k);
    if (tid == 0) s.Lenv[0] = 1.0;
    __syncthreads();
    for (int i = 0; i < L; ++i) {
      const int al = p.aT[i], ar = p.aT[i + 1], bl = s.bW[i], br = s.bW[i + 1];
      const double *Bi = p.trial + p.toff[i];
      load_site(s.Cen, p.pb, s.sbC, W + s.woff[i], bl, br);
      __syncthreads();
      auto left_branches = [&]() {
        for (int tau = 0; tau < d; ++tau)
          cta_gemm(al, br, bl, 1.0, s.Lenv, p.pa, false, s.Cen + tau * s.sbC, p.pb, false, 0.0,
                   s.Xb + tau * s.sbX, p.pa);
        __syncthreads();
        for (int sg = 0; sg < d; ++sg)
          for (int tau = 0; tau < d; ++tau)
            cta_gemm(ar, br, al, 1.0, Bi + (long)sg * al * ar, al, true, s.Xb + tau * s.sbX, p.pa, false, 0.0,
                     s.Pb + (sg + d * tau) * s.sbX, p.pa);
        __syncthreads();
      };
      for (int c = p.site_c0[i]; c < p.site_c0[i + 1]; ++c) {
        const int j = p.cp_j[c];
        left_branches();
        for (int m = i + 1; m < j; ++m) {
          const int am = p.aT[m], am1 = p.aT[m + 1], bm = s.bW[m], bm1 = s.bW[m + 1];
          load_site(s.Nxt, p.pb, s.sbC, W + s.woff[m], bm, bm1);
          __syncthreads();
          const double *Bm = p.trial + p.toff[m];
          for (int q = 0; q < kN2; ++q)
            transfer_in_place(p, s, Bm, am, am1, bm, bm1, s.Nxt, p.pb, s.sbC, s.Pb + q * s.sbX, p.pa);
        }
        __syncthreads();
        closures(p, s, j, W, scr);
        if (tid < 3) {  // <Psi_T| A_i A_j |phi> for A = Sx, iSy, Sz
          const double *op = legacy_op(p, tid + 1);
          double v = 0.0;
          for (int a = 0; a < kN2; ++a)
            for (int b = 0; b < kN2; ++b) v += op[a] * op[b] * s.M[a + 4 * b];
          tov[3 * c + tid] = v;
        }
        __syncthreads();
      }
      if (p.h != 0.0) {  // <Psi_T| Sz_i |phi>
        left_branches();
        const double *R1 = scr + p.roff[i + 1];
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int q = tid; q < ar * br; q += kThreads) {
          const int r = q % ar, cc = q / ar;
          const double rv = R1[r + ar * cc];
#pragma unroll
          for (int e = 0; e < kN2; ++e) v[e] += s.Pb[e * s.sbX + r + p.pa * cc] * rv;
        }
        cta_sum4(v, s.red);
        if (tid == 0) {
          double z = 0.0;
          for (int e = 0; e < kN2; ++e) z += p.opSz[e] * v[e];
          tov[3 * p.nC + i] = z;
        }
        __syncthreads();
      }
      // left environment through site i
      if (i < L - 1) transfer_in_place(p, s, Bi, al, ar, bl, br, s.Cen, p.pb, s.sbC, s.Lenv, p.pa);
    }
    // PDF, weight, sample (MPSQMC.cpp:336-353): one thread, the reference's order and divisions
    if (tid == 0) {
      const double ov = p.overlap[slot];
      double norm = 1.0;
      pdf[0] = 1.0;
      for (int t = 0; t < lp.nterms; ++t) {
        const double v = fmax(-lp.dtau * (lp.term_pref[t] * tov[lp.term_slot[t]]) / ov, 0.0);
        pdf[t + 1] = v;
        norm += v;
      }
      for (int t = 0; t <= lp.nterms; ++t) pdf[t] /= norm;
      const double u = p.uni[w];
      int count = 0;
      double cum = pdf[0];
      while ((cum <= u) && (count < lp.nterms)) {
        count += 1;
        cum += pdf[count];
      }
      p.weight[slot] *= norm;
      lp.changed[w] = count > 0 ? 1 : 0;
      s.sc[0] = count;
      if (lp.tr != nullptr) {
        lp.tr[3 * w + 0] = norm;
        lp.tr[3 * w + 1] = u;
        lp.tr[3 * w + 2] = count;
      }
    }
    __syncthreads();
    const int count = (int)s.sc[0];
    if (count > 0) {  // MPSstate::ApplyMPOterm (MPSstate.cpp:473-498) on the walker in memory
      const int t = count - 1;
      for (int e = 0; e < 2; ++e) {
        const int k = lp.term_site[2 * t + e];
        if (k < 0) continue;
        const double *op = legacy_op(p, lp.term_op[2 * t + e]);
        const int blk = s.bW[k] * s.bW[k + 1];
        double *site = W + s.woff[k];
        for (int q = tid; q < blk; q += kThreads) {
          const double x0 = site[q], x1 = site[blk + q];
          site[q] = op[0] * x0 + op[2] * x1;
          site[blk + q] = op[1] * x0 + op[3] * x1;
        }
        __syncthreads();
      }
      // ScalarMultiplication (MPSstate.cpp:286-305): |prefactor|^(1/L) per site, its sign on site 0.
      // The magnitude drops out of the normalisation that follows; the sign decides the gauge.
      if (lp.term_pref[t] < 0.0) {
        const int n0 = s.bW[0] * s.bW[1] * d;
        for (int q = tid; q < n0; q += kThreads) W[s.woff[0] + q] = -W[s.woff[0] + q];
      }
      __syncthreads();
    }
  }
}

#endif  // MQ_DEVICE_ONLY

}  // namespace mq
