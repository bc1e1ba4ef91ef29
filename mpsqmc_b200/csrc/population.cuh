// Walks split over ranks (one context per rank and GPU): the device side of the reference's MPI
// path through MPSQMC2::Walk (MPSQMC2.cpp:465-511 with USE_MPI_IN_MPSQMC).
//
// A step splits where the reference all-reduces: after the propagation every rank reduces its
// walkers to five sums (MPSQMC2.cpp:475 the weights, 716-731 the projected energy and the
// fluctuation metric), the host sums them over the ranks, and every rank runs its own population
// control with the global scaling (MPSQMC2.cpp:613-686 with totalSumOfWalkerWeights).  Walkers
// then move between ranks as packed records (MPSQMC2::PopulationBalancing, MPSQMC2.cpp:778-934,
// which sends weight, overlap, energy history and the site tensors of the last walkers).
//
// Record of one walker (rec doubles): [0] weight, [1] overlap, [2] energy history,
// [3 .. 3+L] bond dims (as doubles), then the site tensors packed for those dims.
#pragma once

#include "walker_kernels.cuh"

namespace mq {

enum { kSumW = 0, kSumWE = 1, kSumE = 2, kSumE2 = 3, kSumN = 4, kNumSums = 5 };

__host__ __device__ inline long record_doubles(int L, long wsize) { return (4 + (long)L + 1 + wsize + 31) & ~31L; }

#ifndef MQ_DEVICE_ONLY

// This rank's sums after the propagation, and the energy-history update that stats_kernel makes
// on a one-rank step (e_j = Ehist_j / step, step = sd->step + 1).  One CTA of 1024.
__global__ void __launch_bounds__(1024) local_sums_kernel(Dev p, const StepDev *sd, double *out) {
  __shared__ double dbuf[32];
  const int N = sd->n_cur, step = sd->step + 1;
  double sw = 0.0, num = 0.0, se = 0.0, se2 = 0.0;
  for (int w = threadIdx.x; w < N; w += 1024) {
    const double wt = p.wt_out[w];
    sw += wt;
    num += wt * p.energy[w];
    const int slot = p.slot_of[w];
    const double h = p.ehist[slot] + p.energy[w];
    p.ehist[slot] = h;
    const double e = h / step;
    se += e;
    se2 += e * e;
  }
  const double a = block_sum_d(sw, dbuf), b = block_sum_d(num, dbuf), c = block_sum_d(se, dbuf),
               d = block_sum_d(se2, dbuf);
  if (threadIdx.x == 0) {
    out[kSumW] = a;
    out[kSumWE] = b;
    out[kSumE] = c;
    out[kSumE2] = d;
    out[kSumN] = N;
  }
}

// The last k walkers (logical order) into records; one CTA per walker.
__global__ void export_walkers_kernel(Dev p, const StepDev *sd, int k, long rec, double *buf) {
  const int N = sd->n_cur, L = p.L;
  for (int q = blockIdx.x; q < k; q += gridDim.x) {
    const int w = N - k + q;
    const int slot = p.slot_of[w];
    double *r = buf + (long)q * rec;
    const int *dims = p.wdims + (long)slot * (L + 1);
    const long n = p.wofs[(long)slot * L + L - 1] + (long)dims[L - 1] * dims[L] * kMaxD;
    const double *src = p.walkers + (long)slot * p.wstride;
    for (long e = threadIdx.x; e < n; e += blockDim.x) r[4 + L + 1 + e] = src[e];
    for (int e = threadIdx.x; e <= L; e += blockDim.x) r[3 + e] = dims[e];
    if (threadIdx.x == 0) {
      r[0] = p.weight[slot];
      r[1] = p.overlap[slot];
      r[2] = p.ehist[slot];
    }
  }
}

// Records into free slots as walkers N .. N+k-1.  One CTA per walker.  The host has checked that
// k free slots exist.
__global__ void import_walkers_kernel(Dev p, const StepDev *sd, const int *free_slots, int *slot_of, int k,
                                      long rec, const double *buf) {
  const int L = p.L, N = sd->n_cur, nfree = sd->n_free;
  for (int q = blockIdx.x; q < k; q += gridDim.x) {
    const int slot = free_slots[nfree - 1 - q];
    const double *r = buf + (long)q * rec;
    int *dims = const_cast<int *>(p.wdims) + (long)slot * (L + 1);
    long *ofs = const_cast<long *>(p.wofs) + (long)slot * L;
    for (int e = threadIdx.x; e <= L; e += blockDim.x) dims[e] = (int)r[3 + e];
    if (threadIdx.x == 0) {
      long o = 0;
      for (int s = 0; s < L; ++s) {
        ofs[s] = o;
        o += (long)r[3 + s] * (long)r[4 + s] * kMaxD;
      }
      p.weight[slot] = r[0];
      p.overlap[slot] = r[1];
      p.ehist[slot] = r[2];
      slot_of[N + q] = slot;
    }
    __syncthreads();
    const long n = ofs[L - 1] + (long)dims[L - 1] * dims[L] * kMaxD;
    double *dst = p.walkers + (long)slot * p.wstride;
    for (long e = threadIdx.x; e < n; e += blockDim.x) dst[e] = r[4 + L + 1 + e];
  }
}

// Counts after an export (dk = -k: the last k walkers' slots go onto the free stack) or an
// import (dk = +k: k slots were taken from its top).  One CTA.
__global__ void population_count_kernel(StepDev *sd, int *n_cur, const int *slot_of, int *free_slots, int dk) {
  const int N = sd->n_cur, nfree = sd->n_free;
  if (dk < 0)
    for (int q = threadIdx.x; q < -dk; q += blockDim.x) free_slots[nfree + q] = slot_of[N + dk + q];
  __syncthreads();
  if (threadIdx.x == 0) {
    sd->n_cur = N + dk;
    sd->n_free = nfree - dk;
    *n_cur = N + dk;
  }
}

#endif  // MQ_DEVICE_ONLY

}  // namespace mq
