// Walker-propagation kernels (sm_100a, FP64).
//
// One CTA owns one walker at a time (persistent grid striding over walkers) and runs the whole
// timestep of MPSQMC2::PropagateSeparately (MPSQMC2.cpp:518-611) for it:
//
//   phase A  right environments (site L-1 .. 1) of the walker as stored: R[k] = <Psi_T|phi> and
//            N[k] = <phi|phi> contracted over sites k..L-1; overlap, norm and sign fix with the
//            centre on site 0 (Walker::setOverlap, Walker.cpp:54-66, at MPSQMC2.cpp:534);
//   phase B  left-to-right sweep over the bonds.  For a bond (i, i+1) that carries a coupling:
//            the 16 numbers C_kl = <Psi_T|(sqrt(s_k)U_k)_i (sqrt(s_l)V_l)_j|phi> from the left
//            environment, 4 left branches, 4 right branches and 16 closures (the reference gets
//            them from 16 full-chain InnerProducts against stored trial copies, 540-549); the
//            grid PDF, weight update and CDF sample (551-588); the auxiliary-field site
//            operators (MPSstate.cpp:575-633); renormalisation and new overlap (592).  The centre
//            moves to i+1 by one Householder QR; the new norm closes against N[i+2].  Compact-MPO left environments built from
//            the final site tensors give <Psi_T|H|phi> at the end of the sweep, i.e. the local
//            energy of Walker::calcIndividualProjectedEnergy (Walker.cpp:72-77).
//
// Between steps each walker is left-canonical with a normalised centre on site L-1, which is
// the state Walker::setOverlap leaves behind.  Gauge differs from the reference's after the
// first coupling (orthogonal transformations on the bonds); every quantity the walk uses
// (C_kl, PDF, weights, overlaps, energies) is gauge invariant.
#pragma once

#include <cuda_bf16.h>

#include "cta_linalg.cuh"

namespace mq {

constexpr int kMaxD = 2;  // local dimension implemented by the kernels
constexpr int kN2 = kMaxD * kMaxD;
constexpr int kTraceStride = kN2 * kN2 + 5;

struct Dev {
  int L, d, nC, G, nJ;
  int maxA, maxB;   // largest trial / walker bond dimension
  int pa, pb, pq;   // padded shared-memory leading dimensions
  const int *aT;    // trial bond dims [L+1]
  const int *bW;    // largest walker bond dims [L+1] (the slot layout)
  const long *toff; // trial site offsets [L]
  const long *woff; // walker site offsets of the slot layout [L]
  const int *wdims; // per slot: the walker's own bond dims [capacity][L+1] (<= bW)
  const long *wofs; // per slot: the walker's site offsets [capacity][L]
  int *ctr;         // work counters of the persistent kernels (zeroed before each launch)
  const int *sel;   // set_overlap_kernel: only walkers w with sel[w] != 0 (nullptr: all)
  const double *trial;
  const float *trial32;  // FP32 copy of the trial (mixed-precision sweep), or nullptr
  long wstride;     // doubles per walker slot
  double *walkers;
  const int *slot_of;  // logical walker -> slot
  const int *n_cur;    // current number of walkers (device scalar)
  double *weight, *overlap, *ehist;  // per slot
  double *energy;      // per logical walker (last step)
  double *ov_out;      // per logical walker (last step)
  double *wt_out;      // per logical walker (last step)
  const double *uni;   // propagation uniforms [N][nC], logical order
  const int *bond_c;   // coupling index of bond (i, i+1), or -1  [L-1]
  const int *bond_j;   // distinct-J index of the bond's coupling      [L-1]
  const double *bondJ; // coupling strength of bond (i, i+1) or 0     [L-1]
  const double *tabU, *tabS, *tabVT;  // [nJ][16], [nJ][4], [nJ][16]
  const double *tabSq;                 // [nJ][4]: sqrt(S)
  const double *grid;  // [G][4]
  double opSx[4], opISy[4], opSz[4];  // [sigma + d*tau]
  double h;
  double onesite[kMaxD];  // diagonal of exp(0.5 h dtau S^z) (TrotterHeisenberg.cpp:80-88)
  double *scratch;     // per-CTA global scratch
  long scr_stride;
  const long *roff;    // right-environment offsets [L+1] inside a CTA's scratch
  const long *nroff;   // norm-environment offsets [L+1] inside a CTA's scratch
  const long *zoff;    // right-branch offsets [L] inside a CTA's scratch (general sweep)
  long foff;           // compact-MPO environments (2 x 4 x maxA*maxB) inside the scratch
  double *trace;       // optional [N][nC][kTraceStride]
  int *err;            // device error word (bit flags)
  // couplings (i, j) of any range (walker_general.cuh)
  const int *cp_j, *cp_q;  // per coupling: second site, distinct-J index
  const int *site_c0;      // [L+1]: couplings whose first site is i are site_c0[i] .. site_c0[i+1]-1
  const int *ech_off;      // [L+1]: energy-channel entries of site k are ech_off[k] .. ech_off[k+1]-1
  const int *ech_slot;     // per entry: channel slot of an open site i < k
  const double *ech_J;     // per entry: J_ik (0 if i and k are not coupled)
  const int *ech_cont;     // per entry: 1 if site i still has a partner beyond k
  const int *eopen;        // [L]: slot of the channel that site k opens, or -1
  long choff;              // energy channels inside a CTA's scratch: 2 "done" + 3 per slot
  long gwoff;              // matrix work buffers inside a CTA's scratch, or -1 (shared memory)
  // QR-free general sweep: sites are stored as they leave the centre (rescaled to an isometry's Frobenius
  // norm) and a left norm environment (maxB x maxB, ld pb) inside the scratch gives the norm
  long nloff;              // its offset inside a CTA's scratch, or -1 (Householder QR per site)
  // learned proposal (proposal.cuh)
  int prop_mode;                 // 0: the exact grid PDF; 1: the network's proposal, exact-ratio weights
  int prop_collect;              // 1: store (features, PDF) of coupling w % nC of every walker w
  double prop_mix;               // learned proposal: weight of the exact PDF in the drawn mixture
  const __nv_bfloat16 *prop_w;   // network parameters (BF16 copy)
  float *prop_feat, *prop_target;  // [capacity][32], [capacity][G]
};

enum : int { kErrNumeric = 1, kErrCapacity = 2 };

__host__ __device__ inline int padld(int x) {
  int p = (x + 3) & ~3;
  if ((p & 7) == 0) p += 4;
  return p;
}

// Work buffers of one CTA.  T: precision of the matrix buffers (double, or float in the
// mixed-precision sweep); the small buffers (reductions, closures, PDF) are always FP64.
template <typename T>
struct SmemT {
  T *Lenv, *Cen, *Nxt, *Xb, *Pb, *Qt, *QRb, *Rf;
  double *red, *tau, *wv, *M, *Cm, *O1, *O2, *pdf, *sc;
  float *mlp;   // learned proposal: features (32), hidden (256), partial sums (256), logits (256)
  double *qprop;  // learned proposal: q~ over the grid (G)
  int *bW;      // bond dims of the walker being processed [L+1]
  long *woff;   // its site offsets [L]
  int *wsel;    // the walker index handed out by the work counter
  int sbC, sbX;  // sigma-block strides of Cen/Nxt and of Xb/Pb
};
using Smem = SmemT<double>;

// Work buffers of one CTA.  The small ones always live in shared memory.  The matrix buffers
// (environments, site tensors, branches, QR panel) follow them in shared memory when they fit;
// for large bond dimensions they live in the CTA's global scratch instead (big != nullptr), where
// the GEMMs read them through L1/L2.  Returns the doubles placed in shared memory; *big_doubles
// (if given) receives the size of the matrix buffers.  mlp: the learned proposal's buffers.
__host__ __device__ inline long smem_doubles(int L, int maxA, int maxB, int G, int pa, int pb, int pq,
                                              Smem *s, double *base, double *big = nullptr,
                                              long *big_doubles = nullptr, bool mlp = false, bool qr = true) {
  (void)maxA;  // the blocks are sized by the padded pa, pb
  long off = 0, boff = 0;
  double *dummy;
  auto take = [&](double *&p, long n) {
    if (s) p = base + off;
    off += (n + 3) & ~3L;
  };
  auto take_big = [&](double *&p, long n) {
    const long r = (n + 3) & ~3L;
    if (big) {
      if (s) p = big + boff;
    } else {
      if (s) p = base + off;
      off += r;
    }
    boff += r;
  };
  const int d = kMaxD;
  take(s ? s->red : dummy, 16 * kWarps);
  take(s ? s->tau : dummy, maxB);
  take(s ? s->wv : dummy, maxB);
  take(s ? s->M : dummy, 16);
  take(s ? s->Cm : dummy, 16);
  take(s ? s->O1 : dummy, 4);
  take(s ? s->O2 : dummy, 4);
  take(s ? s->pdf : dummy, G);
  take(s ? s->sc : dummy, 16);
  {
    double *b, *o, *q, *m;
    take(b, (L + 2) / 2);
    take(o, L);
    take(q, 1);
    take(m, mlp ? 400 : 0);
    if (s) {
      s->bW = reinterpret_cast<int *>(b);
      s->woff = reinterpret_cast<long *>(o);
      s->wsel = reinterpret_cast<int *>(q);
      s->mlp = reinterpret_cast<float *>(m);
    }
  }
  take(s ? s->qprop : dummy, mlp ? G : 0);
  take_big(s ? s->Lenv : dummy, (long)pa * maxB);
  take_big(s ? s->Cen : dummy, (long)pb * maxB * d);
  take_big(s ? s->Nxt : dummy, (long)pb * maxB * d);
  take_big(s ? s->Xb : dummy, (long)pa * maxB * d);
  take_big(s ? s->Pb : dummy, (long)pa * maxB * kN2);
  take_big(s ? s->Qt : dummy, (long)pa * maxB);
  if (qr) {  // the Householder panel and R factor, last: the QR-free sweep goes without them
    take_big(s ? s->QRb : dummy, (long)pq * maxB);
    take_big(s ? s->Rf : dummy, (long)pb * maxB);
  } else if (s) {
    s->QRb = nullptr;
    s->Rf = nullptr;
  }
  if (big_doubles) *big_doubles = boff;
  if (s) {
    s->sbC = pb * maxB;
    s->sbX = pa * maxB;
  }
  return off;
}

// The same buffers for the mixed-precision sweep: FP64 small buffers as above, FP32 matrix
// buffers, no QR panel (that sweep is QR-free).  Sizes in bytes; *big_floats (if given)
// receives the size of the matrix buffers in floats.
__host__ __device__ inline long smem_bytes_f32(int L, int maxA, int maxB, int G, int pa, int pb,
                                               SmemT<float> *s, double *base, float *big = nullptr,
                                               long *big_floats = nullptr, bool mlp = false) {
  (void)maxA;  // the blocks are sized by the padded pa, pb
  long off = 0, boff = 0;  // doubles of the small buffers; floats of the matrix buffers
  double *dummy;
  float *fdummy;
  auto take = [&](double *&p, long n) {
    if (s) p = base + off;
    off += (n + 3) & ~3L;
  };
  const int d = kMaxD;
  take(s ? s->red : dummy, 16 * kWarps);
  take(s ? s->tau : dummy, maxB);
  take(s ? s->wv : dummy, maxB);
  take(s ? s->M : dummy, 16);
  take(s ? s->Cm : dummy, 16);
  take(s ? s->O1 : dummy, 4);
  take(s ? s->O2 : dummy, 4);
  take(s ? s->pdf : dummy, G);
  take(s ? s->sc : dummy, 16);
  {
    double *b, *o, *q, *m;
    take(b, (L + 2) / 2);
    take(o, L);
    take(q, 1);
    take(m, mlp ? 400 : 0);
    if (s) {
      s->bW = reinterpret_cast<int *>(b);
      s->woff = reinterpret_cast<long *>(o);
      s->wsel = reinterpret_cast<int *>(q);
      s->mlp = reinterpret_cast<float *>(m);
    }
  }
  take(s ? s->qprop : dummy, mlp ? G : 0);
  float *fbase = reinterpret_cast<float *>(base + off);
  long soff = 0;  // floats placed in shared memory after the small buffers
  auto take_big = [&](float *&p, long n) {
    const long r = (n + 7) & ~7L;
    if (big) {
      if (s) p = big + boff;
    } else {
      if (s) p = fbase + soff;
      soff += r;
    }
    boff += r;
  };
  take_big(s ? s->Lenv : fdummy, (long)pa * maxB);
  take_big(s ? s->Cen : fdummy, (long)pb * maxB * d);
  take_big(s ? s->Nxt : fdummy, (long)pb * maxB * d);
  take_big(s ? s->Xb : fdummy, (long)pa * maxB * d);
  take_big(s ? s->Pb : fdummy, (long)pa * maxB * kN2);
  take_big(s ? s->Qt : fdummy, (long)pa * maxB);
  if (s) {
    s->QRb = nullptr;
    s->Rf = nullptr;
    s->sbC = pb * maxB;
    s->sbX = pa * maxB;
  }
  if (big_floats) *big_floats = boff;
  return (long)sizeof(double) * off + (long)sizeof(float) * soff;
}

// Carve the work buffers of the calling CTA (shared memory, plus its global scratch when the
// matrix buffers do not fit on chip).
// qr: the kernel uses the Householder buffers (all but the QR-free general sweep).
__device__ __forceinline__ void carve(const Dev &p, Smem &s, double *smem_raw, bool qr = true) {
  double *big = (p.gwoff >= 0) ? p.scratch + (long)blockIdx.x * p.scr_stride + p.gwoff : nullptr;
  smem_doubles(p.L, p.maxA, p.maxB, p.G, p.pa, p.pb, p.pq, &s, smem_raw, big, nullptr,
               p.prop_mode != 0 || p.prop_collect != 0, qr);
}
// Mixed precision: the CTA's scratch is read as floats with the same element offsets.
__device__ __forceinline__ void carve(const Dev &p, SmemT<float> &s, double *smem_raw) {
  float *big = (p.gwoff >= 0) ? reinterpret_cast<float *>(p.scratch) + (long)blockIdx.x * p.scr_stride + p.gwoff
                              : nullptr;
  smem_bytes_f32(p.L, p.maxA, p.maxB, p.G, p.pa, p.pb, &s, smem_raw, big, nullptr,
                 p.prop_mode != 0 || p.prop_collect != 0);
}

// Bond dims and site offsets of the walker in `slot` into shared memory.  Ends with a barrier.
template <typename T>
__device__ __forceinline__ void load_walker_dims(const Dev &p, SmemT<T> &s, int slot) {
  for (int k = threadIdx.x; k <= p.L; k += kThreads) s.bW[k] = p.wdims[(long)slot * (p.L + 1) + k];
  for (int k = threadIdx.x; k < p.L; k += kThreads) s.woff[k] = p.wofs[(long)slot * p.L + k];
  __syncthreads();
}

// Dynamic scheduling of the persistent grid: the next logical walker from the kernel's work
// counter (walkers of uneven bond dimension cost unevenly).  Starts with a barrier, so the
// previous walker's shared data is no longer in use.
template <typename T>
__device__ __forceinline__ int next_walker(SmemT<T> &s, int *ctr) {
  __syncthreads();
  if (threadIdx.x == 0) *s.wsel = atomicAdd(ctr, 1);
  __syncthreads();
  return *s.wsel;
}

enum : int { kCtrStep = 0, kCtrSetOverlap = 1, kCtrEnergy = 2, kCtrCompress = 3, kNumCtr = 8 };

// dst[sigma*sb + r + ld*c] = src[r + dl*(c + dr*sigma)]   (site storage -> padded smem; an
// FP32 destination rounds the FP64 walker)
template <typename T>
__device__ __forceinline__ void load_site(T *dst, int ld, int sb, const double *src, int dl, int dr) {
  const int n = dl * dr * kMaxD;
  for (int q = threadIdx.x; q < n; q += kThreads) {
    const int r = q % dl, rest = q / dl, c = rest % dr, s = rest / dr;
    dst[s * sb + r + ld * c] = T(src[q]);
  }
}
// Hint the L2 to fetch the n elements at p (global memory) ahead of their use: one prefetch per
// 128-byte line, spread over the CTA's threads.  Nothing waits for it.
template <typename T>
__device__ __forceinline__ void prefetch_l2(const T *p, long n) {
  const char *b = reinterpret_cast<const char *>(p);
  const long bytes = n * (long)sizeof(T);
  for (long o = 128L * threadIdx.x; o < bytes; o += 128L * kThreads)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(b + o));
}
template <typename T>
__device__ __forceinline__ void store_site(double *dst, const T *src, int ld, int sb, int dl, int dr) {
  const int n = dl * dr * kMaxD;
  for (int q = threadIdx.x; q < n; q += kThreads) {
    const int r = q % dl, rest = q / dl, c = rest % dr, s = rest / dr;
    dst[q] = double(src[s * sb + r + ld * c]);
  }
}

// Compact-MPO / overlap environment update through one site (all threads; ends with barrier).
//   site tensor T(r, c, sigma) = T[sigma*ss + r + cs*c], r < bl, c < br
//   Lenv (al x bl, ld pa) -> Lenv' = sum_s B[s]^T Lenv T[s]               (ar x br)
//   Fcur[0..3] (done, Sx, iSy, Sz; ld maxA) -> Fnxt[0..3]
// Bond coupling into the site: Jprev (0 if none).  first: Fcur is zero (site 0).
static __device__ void env_update(const Dev &p, Smem &s, const double *B, int al, int ar, int bl, int br,
                           const double *T, int cs, int ss, const double *Fcur, double *Fnxt,
                           double Jprev, bool first) {
  const int d = kMaxD, lda = p.maxA, fstride = p.maxA * p.maxB;
  // X[tau] = Lenv * T[tau]      (al x br)
  for (int tau = 0; tau < d; ++tau)
    cta_gemm(al, br, bl, 1.0, s.Lenv, p.pa, false, T + tau * ss, cs, false, 0.0, s.Xb + tau * s.sbX,
             p.pa);
  __syncthreads();
  // P[sigma + d*tau] = B[sigma]^T X[tau]   (ar x br)
  for (int sg = 0; sg < d; ++sg)
    for (int tau = 0; tau < d; ++tau)
      cta_gemm(ar, br, al, 1.0, B + (long)sg * al * ar, al, true, s.Xb + tau * s.sbX, p.pa, false,
               0.0, s.Pb + (sg + d * tau) * s.sbX, p.pa);
  __syncthreads();
  // Lenv' and the operator channels opened on this site; field closes immediately.
  for (int q = threadIdx.x; q < ar * br; q += kThreads) {
    const int r = q % ar, c = q / ar;
    double P[kN2];
#pragma unroll
    for (int k = 0; k < kN2; ++k) P[k] = s.Pb[k * s.sbX + r + p.pa * c];
    double l = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
#pragma unroll
    for (int k = 0; k < kN2; ++k) {
      if ((k % d) == (k / d)) l += P[k];
      fx += p.opSx[k] * P[k];
      fy += p.opISy[k] * P[k];
      fz += p.opSz[k] * P[k];
    }
    s.Lenv[r + p.pa * c] = l;
    Fnxt[0 * fstride + r + lda * c] = -p.h * fz;
    Fnxt[1 * fstride + r + lda * c] = fx;
    Fnxt[2 * fstride + r + lda * c] = fy;
    Fnxt[3 * fstride + r + lda * c] = fz;
  }
  __syncthreads();
  if (first) return;
  // Fdone' += sum_s B[s]^T ( sum_t G_st T[t] ),
  // G_st = delta_st Fdone + Jprev (Sx(s,t) F_Sx - iSy(s,t) F_iSy + Sz(s,t) F_Sz)
  for (int sg = 0; sg < d; ++sg) {
    for (int q = threadIdx.x; q < al * bl; q += kThreads) {
      const int r = q % al, c = q / al;
      const double fd = Fcur[0 * fstride + r + lda * c];
      const double fx = Fcur[1 * fstride + r + lda * c];
      const double fy = Fcur[2 * fstride + r + lda * c];
      const double fz = Fcur[3 * fstride + r + lda * c];
      for (int tau = 0; tau < d; ++tau) {
        const int k = sg + d * tau;
        const double g = ((sg == tau) ? fd : 0.0) +
                         Jprev * (p.opSx[k] * fx - p.opISy[k] * fy + p.opSz[k] * fz);
        s.Xb[tau * s.sbX + r + p.pa * c] = g;
      }
    }
    __syncthreads();
    cta_gemm(al, br, bl, 1.0, s.Xb, p.pa, false, T, cs, false, 0.0, s.Qt, p.pa);
    for (int tau = 1; tau < d; ++tau)
      cta_gemm(al, br, bl, 1.0, s.Xb + tau * s.sbX, p.pa, false, T + tau * ss, cs, false, 1.0, s.Qt,
               p.pa);
    __syncthreads();
    cta_gemm(ar, br, al, 1.0, B + (long)sg * al * ar, al, true, s.Qt, p.pa, false, 1.0, Fnxt, lda);
    __syncthreads();
  }
}

// Translation units that only need the device helpers above define MQ_DEVICE_ONLY, so that
// the kernels below are compiled once, in capi.cu.
#ifndef MQ_DEVICE_ONLY

// ---------------------------------------------------------------------------------------------
// The walker-step kernel
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1) walker_step_kernel(Dev p) {
  extern __shared__ double smem_raw[];
  Smem s;
  carve(p, s, smem_raw);
  const int L = p.L, d = kMaxD, tid = threadIdx.x;
  const int N = *p.n_cur;
  double *scr = p.scratch + (long)blockIdx.x * p.scr_stride;
  double *Fbuf = scr + p.foff;
  const int fst = 4 * p.maxA * p.maxB;
  for (int w = next_walker(s, p.ctr + kCtrStep); w < N; w = next_walker(s, p.ctr + kCtrStep)) {
    const int slot = p.slot_of[w];
    load_walker_dims(p, s, slot);
    double *W = p.walkers + (long)slot * p.wstride;
    // ---------------- phase A: right environments ------------------------------------------
    // The walker is read as stored (between steps: left-canonical).  For k = L-1 .. 1:
    //   R[k] = sum_s B_k[s] R[k+1] A_k[s]^T        (a_k x b_k, trial-walker overlap)
    //   N[k] = sum_s A_k[s] N[k+1] A_k[s]^T        (b_k x b_k, walker norm)
    // so that <Psi_T|phi> and ||phi||^2 of any state that differs from phi only on sites < k
    // close against R[k] and N[k].  Then the centre is site 0: normalise, overlap, sign fix
    // (Walker::setOverlap at MPSQMC2.cpp:534).
    {
      if (tid == 0) {
        scr[p.roff[L]] = 1.0;
        scr[p.nroff[L]] = 1.0;
      }
      for (int k = L - 1; k >= 1; --k) {
        const int al = p.aT[k], ar = p.aT[k + 1], bl = s.bW[k], br = s.bW[k + 1];
        load_site(s.Nxt, p.pb, s.sbC, W + s.woff[k], bl, br);
        __syncthreads();
        const double *Rn = scr + p.roff[k + 1], *Nn = scr + p.nroff[k + 1];
        double *Rk = scr + p.roff[k], *Nk = scr + p.nroff[k];
        const double *Bk = p.trial + p.toff[k];
        for (int sg = 0; sg < d; ++sg) {
          // Y[s] = R[k+1] A_k[s]^T (ar x bl),  Z[s] = N[k+1] A_k[s]^T (br x bl)
          cta_gemm(ar, bl, br, 1.0, Rn, ar, false, s.Nxt + sg * s.sbC, p.pb, true, 0.0,
                   s.Xb + sg * s.sbX, p.pa);
          cta_gemm(br, bl, br, 1.0, Nn, br, false, s.Nxt + sg * s.sbC, p.pb, true, 0.0,
                   s.Pb + sg * s.sbX, p.pa);
        }
        __syncthreads();
        for (int sg = 0; sg < d; ++sg) {
          cta_gemm(al, bl, ar, 1.0, Bk + (long)sg * al * ar, al, false, s.Xb + sg * s.sbX, p.pa, false,
                   sg == 0 ? 0.0 : 1.0, Rk, al);
          cta_gemm(bl, bl, br, 1.0, s.Nxt + sg * s.sbC, p.pb, false, s.Pb + sg * s.sbX, p.pa, false,
                   sg == 0 ? 0.0 : 1.0, Nk, bl);
        }
        __syncthreads();
      }
      // centre = site 0 (1 x b1): ||phi||^2 = sum_s C[s] N[1] C[s]^T, ov = sum_s B_0[s] R[1] C[s]^T
      {
        const int a1 = p.aT[1], b1 = s.bW[1];
        load_site(s.Cen, p.pb, s.sbC, W + s.woff[0], 1, b1);
        __syncthreads();
        const double *R1 = scr + p.roff[1], *N1 = scr + p.nroff[1];
        const double *B0 = p.trial + p.toff[0];
        double v2[4] = {0.0, 0.0, 0.0, 0.0};
        for (int q = tid; q < b1 * b1 * d; q += kThreads) {
          const int a = q % b1, rest = q / b1, b = rest % b1, sg = rest / b1;
          v2[0] += s.Cen[sg * s.sbC + p.pb * a] * N1[a + b1 * b] * s.Cen[sg * s.sbC + p.pb * b];
        }
        for (int q = tid; q < a1 * b1 * d; q += kThreads) {
          const int a = q % a1, rest = q / a1, b = rest % b1, sg = rest / b1;
          v2[1] += B0[a + a1 * sg] * R1[a + a1 * b] * s.Cen[sg * s.sbC + p.pb * b];
        }
        cta_sum4(v2, s.red);
        const double nrm = sqrt(v2[0]);
        double ov = v2[1] / nrm;
        const double scale = (ov < 0.0) ? -1.0 / nrm : 1.0 / nrm;  // ChangePhase, MPSstate.cpp:307-315
        if (ov < 0.0) ov = -ov;
        for (int q = tid; q < b1 * d; q += kThreads) s.Cen[(q / b1) * s.sbC + p.pb * (q % b1)] *= scale;
        if (tid == 0) s.sc[0] = ov;
        __syncthreads();
      }
    }
    // ---------------- phase B: coupling sweep -----------------------------------------------
    double ov = s.sc[0];
    double wt = p.weight[slot];
    if (tid == 0) s.Lenv[0] = 1.0;
    int cur = 0;
    __syncthreads();
    for (int i = 0; i < L - 1; ++i) {
      const int al = p.aT[i], ar = p.aT[i + 1], a2 = p.aT[i + 2];
      const int bl = s.bW[i], br = s.bW[i + 1], b2 = s.bW[i + 2];
      const double *Bi = p.trial + p.toff[i];
      const double *Bj = p.trial + p.toff[i + 1];
      load_site(s.Nxt, p.pb, s.sbC, W + s.woff[i + 1], br, b2);
      __syncthreads();
      const int c = p.bond_c[i];
      double num = ov;  // overlap numerator after the bond (no coupling: unchanged)
      if (c >= 0) {
        const int jq = p.bond_j[i];
        const double *U = p.tabU + 16 * jq, *Sq = p.tabSq + 4 * jq, *VT = p.tabVT + 16 * jq;
        // left branches P[s + d t] = B_i[s]^T Lenv C[t]
        for (int tau = 0; tau < d; ++tau)
          cta_gemm(al, br, bl, 1.0, s.Lenv, p.pa, false, s.Cen + tau * s.sbC, p.pb, false, 0.0,
                   s.Xb + tau * s.sbX, p.pa);
        __syncthreads();
        for (int sg = 0; sg < d; ++sg)
          for (int tau = 0; tau < d; ++tau)
            cta_gemm(ar, br, al, 1.0, Bi + (long)sg * al * ar, al, true, s.Xb + tau * s.sbX, p.pa,
                     false, 0.0, s.Pb + (sg + d * tau) * s.sbX, p.pa);
        __syncthreads();
        // right branches Y[t'] = R[i+2] N[t']^T, Q = B_j[s'] Y[t'], closures M[p + 4q]
        const double *R2 = scr + p.roff[i + 2];
        for (int tau = 0; tau < d; ++tau)
          cta_gemm(a2, br, b2, 1.0, R2, a2, false, s.Nxt + tau * s.sbC, p.pb, true, 0.0,
                   s.Xb + tau * s.sbX, p.pa);
        __syncthreads();
        for (int sg = 0; sg < d; ++sg)
          for (int tau = 0; tau < d; ++tau) {
            cta_gemm(ar, br, a2, 1.0, Bj + (long)sg * ar * a2, ar, false, s.Xb + tau * s.sbX, p.pa,
                     false, 0.0, s.Qt, p.pa);
            __syncthreads();
            double v[4] = {0.0, 0.0, 0.0, 0.0};
            for (int q = tid; q < ar * br; q += kThreads) {
              const int r = q % ar, cc = q / ar;
              const double qv = s.Qt[r + p.pa * cc];
#pragma unroll
              for (int k = 0; k < 4; ++k) v[k] += s.Pb[k * s.sbX + r + p.pa * cc] * qv;
            }
            cta_sum4(v, s.red);
            if (tid == 0)
              for (int k = 0; k < 4; ++k) s.M[k + 4 * (sg + d * tau)] = v[k];
          }
        __syncthreads();
        // C[k + 4 l] = sqrt(s_k s_l) sum_{p,q} U[p + 4k] VT[l + 4q] M[p + 4q]
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
        // PDF over the grid (MPSQMC2.cpp:554-567)
        const double fac = 4.0 / (ov * p.G);
        double part = 0.0;
        for (int g = tid; g < p.G; g += kThreads) {
          const double *x = p.grid + 4 * g;
          double v = 0.0;
          for (int l = 0; l < 4; ++l)
            for (int r = 0; r < 4; ++r) v += s.Cm[l + 4 * r] * x[l] * x[r];
          v = fmax(0.0, v);
          v *= fac;
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
          // O1(s,t) = sum_k sqrt(4 s_k) x_k U[s + 2(t + 2k)], O2(s,t) = sum_l sqrt(4 s_l) x_l VT[l + 4(s + 2t)]
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
        num = s.sc[1];
        // apply O1 to the centre (into the QR layout), O2 to site j in place
        for (int q = tid; q < bl * br; q += kThreads) {
          const int r = q % bl, cc = q / bl;
          const double c0 = s.Cen[r + p.pb * cc], c1 = s.Cen[s.sbC + r + p.pb * cc];
          s.QRb[(r + bl * 0) + p.pq * cc] = s.O1[0] * c0 + s.O1[2] * c1;
          s.QRb[(r + bl * 1) + p.pq * cc] = s.O1[1] * c0 + s.O1[3] * c1;
        }
        for (int q = tid; q < br * b2; q += kThreads) {
          const int r = q % br, cc = q / br;
          const double n0 = s.Nxt[r + p.pb * cc], n1 = s.Nxt[s.sbC + r + p.pb * cc];
          s.Nxt[r + p.pb * cc] = s.O2[0] * n0 + s.O2[2] * n1;
          s.Nxt[s.sbC + r + p.pb * cc] = s.O2[1] * n0 + s.O2[3] * n1;
        }
      } else {
        for (int q = tid; q < bl * br; q += kThreads) {
          const int r = q % bl, cc = q / bl;
          s.QRb[(r + bl * 0) + p.pq * cc] = s.Cen[r + p.pb * cc];
          s.QRb[(r + bl * 1) + p.pq * cc] = s.Cen[s.sbC + r + p.pb * cc];
        }
      }
      __syncthreads();
      // move the centre: QR of site i, R into site i+1
      cta_householder_qr(bl * d, br, s.QRb, p.pq, s.Rf, p.pb, s.tau, s.wv, s.red);
      for (int sg = 0; sg < d; ++sg)
        cta_gemm(br, b2, br, 1.0, s.Rf, p.pb, false, s.Nxt + sg * s.sbC, p.pb, false, 0.0,
                 s.Cen + sg * s.sbC, p.pb);
      // site i <- Q
      {
        double *Wi = W + s.woff[i];
        for (int q = tid; q < bl * br * d; q += kThreads) {
          const int r = q % bl, rest = q / bl, cc = rest % br, sg = rest / br;
          Wi[q] = s.QRb[(r + bl * sg) + p.pq * cc];
        }
      }
      __syncthreads();
      if (c >= 0) {
        // ||B(x) phi||^2 = sum_s tr(C[s] N[i+2] C[s]^T): sites < i+1 are orthonormal now
        const double *N2 = scr + p.nroff[i + 2];
        for (int sg = 0; sg < d; ++sg)
          cta_gemm(br, b2, b2, 1.0, s.Cen + sg * s.sbC, p.pb, false, N2, b2, false, 0.0, s.Xb + sg * s.sbX,
                   p.pa);
        __syncthreads();
        double part = 0.0;
        for (int q = tid; q < br * b2 * d; q += kThreads) {
          const int r = q % br, rest = q / br, cc = rest % b2, sg = rest / b2;
          part += s.Cen[sg * s.sbC + r + p.pb * cc] * s.Xb[sg * s.sbX + r + p.pa * cc];
        }
        const double nrm = sqrt(cta_sum(part, s.red));
        ov = num / nrm;
        const double scale = (ov < 0.0) ? -1.0 / nrm : 1.0 / nrm;
        if (ov < 0.0) ov = -ov;
        for (int q = tid; q < br * b2 * d; q += kThreads) {
          const int r = q % br, rest = q / br, cc = rest % b2, sg = rest / b2;
          s.Cen[sg * s.sbC + r + p.pb * cc] *= scale;
        }
        if (p.trace != nullptr && tid == 0) {
          double *t = p.trace + ((long)w * p.nC + c) * kTraceStride;
          for (int k = 0; k < 16; ++k) t[k] = s.Cm[k];
          t[16] = s.sc[4];
          t[17] = s.sc[3];
          t[18] = s.sc[2];
          t[19] = wt;
          t[20] = ov;
        }
      }
      // environments through the final site i
      env_update(p, s, Bi, al, ar, bl, br, s.QRb, p.pq, bl, Fbuf + cur * fst, Fbuf + (1 - cur) * fst,
                 (i > 0) ? p.bondJ[i - 1] : 0.0, i == 0);
      cur = 1 - cur;
    }
    // last site: centre; overlap and energy (final setOverlap, MPSQMC2.cpp:598; Walker.cpp:76)
    {
      const int i = L - 1;
      const int al = p.aT[i], bl = s.bW[i];
      env_update(p, s, p.trial + p.toff[i], al, 1, bl, 1, s.Cen, p.pb, s.sbC, Fbuf + cur * fst,
                 Fbuf + (1 - cur) * fst, p.bondJ[i - 1], false);
      store_site(W + s.woff[i], s.Cen, p.pb, s.sbC, bl, 1);
      const double ovf = s.Lenv[0];
      const double en = Fbuf[(1 - cur) * fst + 0];
      if (tid == 0) {
        p.overlap[slot] = ovf;
        p.weight[slot] = wt;
        p.energy[w] = en / ovf;
        p.ov_out[w] = ovf;
        p.wt_out[w] = wt;
        if (!(isfinite(wt) && isfinite(ovf) && isfinite(en))) atomicOr(p.err, kErrNumeric);
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Walker::setOverlap exactly as the reference does it (Walker.cpp:54-66): Householder
// LeftNormalize (MPSstate.cpp:216-229), overlap <Psi_T|phi>, ChangePhase if negative.
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1) set_overlap_kernel(Dev p) {
  extern __shared__ double smem_raw[];
  Smem s;
  carve(p, s, smem_raw);
  const int L = p.L, d = kMaxD, tid = threadIdx.x;
  const int N = *p.n_cur;
  for (int w = next_walker(s, p.ctr + kCtrSetOverlap); w < N; w = next_walker(s, p.ctr + kCtrSetOverlap)) {
    if (p.sel != nullptr && p.sel[w] == 0) continue;
    const int slot = p.slot_of[w];
    load_walker_dims(p, s, slot);
    double *W = p.walkers + (long)slot * p.wstride;
    load_site(s.Cen, p.pb, s.sbC, W + s.woff[0], s.bW[0], s.bW[1]);
    __syncthreads();
    for (int k = 0; k < L; ++k) {
      const int bl = s.bW[k], br = s.bW[k + 1];
      for (int q = tid; q < bl * br; q += kThreads) {
        const int r = q % bl, cc = q / bl;
        for (int sg = 0; sg < d; ++sg) s.QRb[(r + bl * sg) + p.pq * cc] = s.Cen[sg * s.sbC + r + p.pb * cc];
      }
      __syncthreads();
      cta_householder_qr(bl * d, br, s.QRb, p.pq, s.Rf, p.pb, s.tau, s.wv, s.red);
      double *Wk = W + s.woff[k];
      for (int q = tid; q < bl * br * d; q += kThreads) {
        const int r = q % bl, rest = q / bl, cc = rest % br, sg = rest / br;
        Wk[q] = s.QRb[(r + bl * sg) + p.pq * cc];
      }
      if (k < L - 1) {
        const int b2 = s.bW[k + 2];
        load_site(s.Nxt, p.pb, s.sbC, W + s.woff[k + 1], br, b2);
        __syncthreads();
        for (int sg = 0; sg < d; ++sg)
          cta_gemm(br, b2, br, 1.0, s.Rf, p.pb, false, s.Nxt + sg * s.sbC, p.pb, false, 0.0,
                   s.Cen + sg * s.sbC, p.pb);
      }
      __syncthreads();
    }
    // overlap sweep: Lenv' = sum_s B[s]^T Lenv A[s]
    if (tid == 0) s.Lenv[0] = 1.0;
    __syncthreads();
    for (int k = 0; k < L; ++k) {
      const int al = p.aT[k], ar = p.aT[k + 1], bl = s.bW[k], br = s.bW[k + 1];
      const double *A = W + s.woff[k];
      const double *B = p.trial + p.toff[k];
      for (int sg = 0; sg < d; ++sg)
        cta_gemm(al, br, bl, 1.0, s.Lenv, p.pa, false, A + (long)sg * bl * br, bl, false, 0.0,
                 s.Xb + sg * s.sbX, p.pa);
      __syncthreads();
      cta_gemm(ar, br, al, 1.0, B, al, true, s.Xb, p.pa, false, 0.0, s.Qt, p.pa);
      for (int sg = 1; sg < d; ++sg)
        cta_gemm(ar, br, al, 1.0, B + (long)sg * al * ar, al, true, s.Xb + sg * s.sbX, p.pa, false,
                 1.0, s.Qt, p.pa);
      __syncthreads();
      for (int q = tid; q < ar * br; q += kThreads) s.Lenv[(q % ar) + p.pa * (q / ar)] = s.Qt[(q % ar) + p.pa * (q / ar)];
      __syncthreads();
    }
    double ov = s.Lenv[0];
    __syncthreads();
    if (ov < 0.0) {
      const int n0 = s.bW[0] * s.bW[1] * d;
      for (int q = tid; q < n0; q += kThreads) W[s.woff[0] + q] *= -1.0;
      ov = -ov;
    }
    if (tid == 0) p.overlap[slot] = ov;
    __syncthreads();
  }
}

// <Psi_T|H|phi> / overlap for every walker, walker tensors taken as stored (any gauge).
__global__ void __launch_bounds__(kThreads, 1) energy_kernel(Dev p) {
  extern __shared__ double smem_raw[];
  Smem s;
  carve(p, s, smem_raw);
  const int L = p.L, tid = threadIdx.x;
  const int N = *p.n_cur;
  double *scr = p.scratch + (long)blockIdx.x * p.scr_stride;
  double *Fbuf = scr + p.foff;
  const int fst = 4 * p.maxA * p.maxB;
  for (int w = next_walker(s, p.ctr + kCtrEnergy); w < N; w = next_walker(s, p.ctr + kCtrEnergy)) {
    const int slot = p.slot_of[w];
    load_walker_dims(p, s, slot);
    const double *W = p.walkers + (long)slot * p.wstride;
    if (tid == 0) s.Lenv[0] = 1.0;
    __syncthreads();
    int cur = 0;
    for (int k = 0; k < L; ++k) {
      const int al = p.aT[k], ar = p.aT[k + 1], bl = s.bW[k], br = s.bW[k + 1];
      env_update(p, s, p.trial + p.toff[k], al, ar, bl, br, W + s.woff[k], bl, bl * br,
                 Fbuf + cur * fst, Fbuf + (1 - cur) * fst, (k > 0) ? p.bondJ[k - 1] : 0.0, k == 0);
      cur = 1 - cur;
    }
    if (tid == 0) {
      const double en = Fbuf[cur * fst];
      p.energy[w] = en / p.overlap[slot];
      p.ov_out[w] = p.overlap[slot];
      p.wt_out[w] = p.weight[slot];
    }
    __syncthreads();
  }
}

// ApplyOneSiteTrotterTermEverywhere (MPSstate.cpp:635-659): every site's sigma block scaled by
// the diagonal single-site propagator.  One CTA per walker (grid-stride).
__global__ void onesite_kernel(Dev p) {
  const int N = *p.n_cur;
  for (int w = blockIdx.x; w < N; w += gridDim.x) {
    const int slot = p.slot_of[w];
    double *W = p.walkers + (long)slot * p.wstride;
    const int *bW = p.wdims + (long)slot * (p.L + 1);
    const long *woff = p.wofs + (long)slot * p.L;
    for (int k = 0; k < p.L; ++k) {
      const int blk = bW[k] * bW[k + 1];
      double *site = W + woff[k];
      for (int q = threadIdx.x; q < blk * kMaxD; q += blockDim.x) site[q] *= p.onesite[q / blk];
    }
  }
}

// ---------------------------------------------------------------------------------------------
// MT19937 (Matsumoto & Nishimura 1998), one CTA, the reference's single random stream.
// ---------------------------------------------------------------------------------------------
struct MtState {
  uint32_t mt[624];
  int idx;
  int pad;
  unsigned long long draws;
};

__device__ __forceinline__ uint32_t mt_temper(uint32_t y) {
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= (y >> 18);
  return y;
}

__device__ void mt_twist_range(uint32_t *mt, int lo, int hi) {
  // new mt[i] for i in [lo, hi), all inputs already final for this phase
  uint32_t v = 0;
  const int i = lo + threadIdx.x;
  const bool act = i < hi;
  if (act) {
    const uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
    v = mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
  }
  __syncthreads();
  if (act) mt[i] = v;
  __syncthreads();
}

// Produce the next n uniforms (n from *n_dev when non-null) into out.  blockDim = 1024.
__global__ void mt_generate_kernel(MtState *st, const int *n_dev, long n_host, long mult,
                                   double *out) {
  __shared__ uint32_t mt[624];
  __shared__ int s_idx;
  const long n = n_dev ? (long)(*n_dev) * mult : n_host;
  for (int q = threadIdx.x; q < 624; q += blockDim.x) mt[q] = st->mt[q];
  if (threadIdx.x == 0) s_idx = st->idx;
  __syncthreads();
  long pos = 0;
  while (pos < n) {
    if (s_idx >= 624) {
      mt_twist_range(mt, 0, 227);
      mt_twist_range(mt, 227, 454);
      mt_twist_range(mt, 454, 623);
      mt_twist_range(mt, 623, 624);
      if (threadIdx.x == 0) s_idx = 0;
      __syncthreads();
    }
    const int idx = s_idx;
    const long take = min((long)(624 - idx), n - pos);
    for (int q = threadIdx.x; q < take; q += blockDim.x)
      out[pos + q] = (double)mt_temper(mt[idx + q]) / 4294967296.0;
    __syncthreads();
    if (threadIdx.x == 0) s_idx = idx + (int)take;
    pos += take;
    __syncthreads();
  }
  for (int q = threadIdx.x; q < 624; q += blockDim.x) st->mt[q] = mt[q];
  if (threadIdx.x == 0) {
    st->idx = s_idx;
    st->draws += (unsigned long long)n;
  }
}

// ---------------------------------------------------------------------------------------------
// Statistics and population control (one CTA, 1024 threads)
// ---------------------------------------------------------------------------------------------
struct StepDev {
  int n_cur, n_flag, n_new, n_extra, n_free, step, status, pad;
  double sumw, EP, ET, omega, scaling;
};

template <typename T>
__device__ T block_scan_excl(T v, T *buf, T &total) {  // blockDim.x == 1024
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  T x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __syncthreads();
  if (lane == 31) buf[warp] = x;
  __syncthreads();
  if (warp == 0) {
    T t = buf[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    buf[lane] = t;
  }
  __syncthreads();
  total = buf[31];
  const T before = (warp > 0) ? buf[warp - 1] : T(0);
  __syncthreads();
  return before + x - v;
}

__device__ double block_sum_d(double v, double *buf) {  // blockDim.x == 1024
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) buf[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int q = 0; q < 32; ++q) s += buf[q];
  __syncthreads();
  return s;
}

// Population control modes (mpsqmc_set_option): threshold branching of the reference, or comb
// (systematic) resampling to Ndesired equal-weight walkers; either every `interval` steps, with
// the weights only rescaled by Ndesired / sum(w) on the steps in between.
enum : int { kResampleThreshold = 0, kResampleComb = 1, kResampleLegacy = 2 };

// Weight sum, E_T, E_P, energy history, fluctuation metric (MPSQMC2.cpp:468-487, 688-747),
// then the branching flags of SeparatePopulationControl (613-648).
// The step number (1-based, for e_j = Ehist_j / step) is sd->step + 1; finish_branch_kernel
// advances sd->step, so a captured step graph needs no per-step argument.
// Uniforms needed by the branching (n_flag): one per walker whose scaled weight leaves
// [0.25, 1.5] (threshold), one per resampling (comb), none on steps without population control.
// ext (a walk split over ranks): the sums of all ranks' walkers [Sum w, Sum w E, Sum e, Sum e^2,
// N, Ndesired of all ranks] replace this rank's own, whose history local_sums_kernel updated.
__global__ void __launch_bounds__(1024) stats_kernel(Dev p, StepDev *sd, int Ndesired, double dtau,
                                                     int update_history, int *flag_pos, double *sw_out,
                                                     int interval, int mode, const double *ext = nullptr) {
  const int step = sd->step + 1;
  const bool branch_now = (step % interval) == 0;
  __shared__ double dbuf[32];
  __shared__ int ibuf[32];
  const int N = sd->n_cur;
  double sw = 0.0, num = 0.0;
  for (int w = threadIdx.x; w < N; w += 1024) {
    const double wt = p.wt_out[w];
    sw += wt;
    num += wt * p.energy[w];
  }
  const double sumw_full = ext ? ext[0] : block_sum_d(sw, dbuf);
  const double numer = ext ? ext[1] : block_sum_d(num, dbuf);
  // the MPO-term projector sums the weights into an int (MPSQMC.cpp:364-366)
  const double sumw = (mode == kResampleLegacy) ? (double)(int)sumw_full : sumw_full;
  const double Nall = ext ? ext[4] : (double)N;
  const double avgW = sumw / Nall;
  const double scaling = (ext ? ext[5] : (double)Ndesired) / (Nall * avgW);
  double se = 0.0, se2 = 0.0;
  if (update_history && !ext) {
    for (int w = threadIdx.x; w < N; w += 1024) {
      const int slot = p.slot_of[w];
      const double h = p.ehist[slot] + p.energy[w];
      p.ehist[slot] = h;
      const double e = h / step;
      se += e;
      se2 += e * e;
    }
  }
  const double sE = ext ? ext[2] : block_sum_d(se, dbuf);
  const double sE2 = ext ? ext[3] : block_sum_d(se2, dbuf);
  // flags: walkers whose scaled weight leaves [0.25, 1.5] draw one uniform, in walker order
  int nflag_total = 0;
  for (int base = 0; base < N; base += 1024) {
    const int w = base + threadIdx.x;
    int f = 0;
    double s = 0.0;
    if (w < N) {
      s = p.wt_out[w] * scaling;
      sw_out[w] = s;
      f = (branch_now && ((mode == kResampleThreshold && (s < 0.25 || s > 1.5)) || mode == kResampleLegacy)) ? 1 : 0;
    }
    int tot;
    const int ex = block_scan_excl<int>(f, ibuf, tot);
    if (w < N) flag_pos[w] = f ? nflag_total + ex : -1;
    nflag_total += tot;
  }
  if (threadIdx.x == 0) {
    sd->sumw = sumw;
    sd->scaling = scaling;
    sd->ET = log(scaling) / dtau;
    sd->EP = numer / sumw_full;
    sd->omega = update_history ? (sE2 - sE * sE / Nall) / Nall : 0.0;
    sd->n_flag = (branch_now && mode == kResampleComb) ? 1 : nflag_total;
    if (!(isfinite(sumw) && sumw > 0.0 && isfinite(numer))) atomicOr(p.err, kErrNumeric);
  }
}

// Branching with a slot table: the first copy of a surviving walker keeps its slot, extra copies
// take free slots, killed walkers free theirs.  Copies per walker:
//   threshold (MPSQMC2.cpp:620-686): int(s + u) for flagged walkers, else 1;
//   comb: the teeth k + u (k = 0, 1, ...) that fall in [S_w, S_w + s_w), S_w the running sum of
//         the scaled weights in walker order (summed sequentially, as the oracle does), weight 1;
//   steps without population control: one copy with the scaled weight.
__global__ void __launch_bounds__(1024) branch_kernel(Dev p, StepDev *sd, const int *flag_pos,
                                                      const double *sw_in, const double *ubr,
                                                      int *slot_of_new, int *free_slots,
                                                      int *copy_src, int *copy_dst, int *parent,
                                                      int capacity, int *ncop, int interval, int mode) {
  __shared__ int ibuf[32];
  const int N = sd->n_cur;
  const bool comb = mode == kResampleComb && ((sd->step + 1) % interval) == 0;
  int nfree = sd->n_free;
  int new_total = 0, extra_total = 0, killed_total = 0;
  if (comb) {
    if (threadIdx.x == 0) {
      const double u = ubr[0];
      double S = 0.0;
      for (int w = 0; w < N; ++w) {
        const double s = sw_in[w];
        ncop[w] = (int)(ceil(S + s - u) - ceil(S - u));
        S += s;
      }
    }
  } else {
    for (int w = threadIdx.x; w < N; w += 1024)
      ncop[w] = (flag_pos[w] >= 0) ? (int)(sw_in[w] + ubr[flag_pos[w]]) : 1;
  }
  __syncthreads();
  // pass 1: killed slots onto the free stack (in walker order)
  for (int base = 0; base < N; base += 1024) {
    const int w = base + threadIdx.x;
    const int nc = (w < N) ? ncop[w] : 1;
    int tot;
    const int k = block_scan_excl<int>((w < N && nc == 0) ? 1 : 0, ibuf, tot);
    if (w < N && nc == 0) free_slots[nfree + killed_total + k] = p.slot_of[w];
    killed_total += tot;
  }
  __syncthreads();
  nfree += killed_total;
  // pass 2: new logical order
  for (int base = 0; base < N; base += 1024) {
    const int w = base + threadIdx.x;
    int nc = 0;
    double s = 0.0, neww = 0.0;
    if (w < N) {
      s = sw_in[w];
      nc = ncop[w];
      neww = s;
      if (comb || mode == kResampleLegacy) neww = 1.0;  // MPSQMC.cpp:413: every copy gets weight 1
      else if (flag_pos[w] >= 0) neww = (s < 0.25) ? 1.0 : s / nc;
    }
    int tot_new, tot_extra;
    const int pos = block_scan_excl<int>(nc, ibuf, tot_new);
    const int ex = block_scan_excl<int>(nc > 1 ? nc - 1 : 0, ibuf, tot_extra);
    if (w < N && nc >= 1) {
      const int slot = p.slot_of[w];
      const int dst0 = new_total + pos;
      if (dst0 < capacity) {
        slot_of_new[dst0] = slot;
        parent[dst0] = w;
      }
      p.weight[slot] = neww;
      for (int c = 1; c < nc; ++c) {
        const int e = extra_total + ex + (c - 1);
        const int fs = nfree - 1 - e;
        const int dst = dst0 + c;
        if (fs >= 0 && dst < capacity) {
          const int ns = free_slots[fs];
          slot_of_new[dst] = ns;
          parent[dst] = w;
          copy_src[e] = slot;
          copy_dst[e] = ns;
        }
      }
    }
    new_total += tot_new;
    extra_total += tot_extra;
  }
  if (threadIdx.x == 0) {
    sd->n_new = new_total;
    sd->n_extra = extra_total;
    if (extra_total > nfree || new_total > capacity) {
      atomicOr(p.err, kErrCapacity);
      sd->n_free = nfree;
    } else {
      sd->n_free = nfree - extra_total;
    }
  }
}

// Copy walker slots for the extra copies: tensors and scalar state.
__global__ void copy_walkers_kernel(Dev p, const StepDev *sd, const int *copy_src,
                                    const int *copy_dst) {
  const int n = sd->n_extra;
  if (p.err != nullptr && (*p.err & kErrCapacity)) return;
  const long per = p.wstride;
  for (long q = blockIdx.x; q < (long)n; q += gridDim.x) {
    const int src = copy_src[q], dst = copy_dst[q];
    const double *a = p.walkers + (long)src * per;
    double *b = p.walkers + (long)dst * per;
    for (long e = threadIdx.x; e < per; e += blockDim.x) b[e] = a[e];
    for (int k = threadIdx.x; k <= p.L; k += blockDim.x)
      const_cast<int *>(p.wdims)[(long)dst * (p.L + 1) + k] = p.wdims[(long)src * (p.L + 1) + k];
    for (int k = threadIdx.x; k < p.L; k += blockDim.x)
      const_cast<long *>(p.wofs)[(long)dst * p.L + k] = p.wofs[(long)src * p.L + k];
    if (threadIdx.x == 0) {
      p.weight[dst] = p.weight[src];
      p.overlap[dst] = p.overlap[src];
      p.ehist[dst] = p.ehist[src];
    }
  }
}

// Walkers [w0, w0 + m) in logical order into dst (stride per doubles each).
__global__ void gather_walkers_kernel(Dev p, int w0, int m, long per, double *dst) {
  for (int q = blockIdx.x; q < m; q += gridDim.x) {
    const double *a = p.walkers + (long)p.slot_of[w0 + q] * p.wstride;
    double *b = dst + (long)q * per;
    for (long e = threadIdx.x; e < per; e += blockDim.x) b[e] = a[e];
  }
}

// New population becomes current: slot table copied back, counts updated (one CTA).
__global__ void finish_branch_kernel(StepDev *sd, int *n_cur, int *slot_of, const int *slot_of_new,
                                     const int *err, int capacity) {
  if (*err & kErrCapacity) return;
  const int nn = min(sd->n_new, capacity);
  for (int q = threadIdx.x; q < nn; q += blockDim.x) slot_of[q] = slot_of_new[q];
  if (threadIdx.x == 0) {
    sd->n_cur = nn;
    sd->step += 1;
    *n_cur = nn;
  }
}

#endif  // MQ_DEVICE_ONLY

}  // namespace mq
