// The walker-batched mixed-precision sweep (MPSQMC_PRECISION_TF32X3_TC): every walker of the
// population moves through the same sequence of sites and couplings in lockstep, and every
// contraction of the step is ONE launch of the tcgen05 product (tc_gemm.cuh) over all walkers.
// Products whose left factor is the trial tensor become wide GEMMs (M = trial bond, N = walkers
// x walker bond, K = trial bond); the walker-by-walker ones are batched GEMMs.  Host-side
// interface used by capi.cu; the implementation is in batched.cu.
#pragma once

#include <cuda_runtime.h>

#include <vector>

namespace mq {
namespace bs {

// Classes of right factors that may be stored split (Tiles::split_out bits): Y (right
// environments and closures), X (left branches), X4 (branch carries), Q (energy), Xch (energy
// channels).
constexpr int kSplitY = 1, kSplitX = 2, kSplitX4 = 4, kSplitQ = 8, kSplitXch = 16, kSplitAll = 31;

// Tile choices of the plan's products (what the autotuner varies per bond-profile bucket).
struct Tiles {
  int stack_tn = 256;   // widest N tile of products whose A (a trial tensor) is shared: walkers are
                        // stacked along N up to this width (64, 128 or 256; 64 with N = 64 means
                        // one walker per tile)
  int wide_tn = 256;    // widest N tile of the walker-by-walker products (64, 128 or 256)
  int max_stages = 8;   // load-ring depth cap (2 .. 8; fewer when shared memory is short)
  int kc_trial = 32;    // k-values per stage of the trial products (32, or 16: half the stage
                        // and twice the ring depth)
  int split_out = 0;    // three passes: bits (kSplit*) of the classes of right factors of the trial
                        // products that are written as TF32 head and tail arrays and loaded
                        // split (no conversion in their consumers, twice the bytes written by
                        // their producers)
  bool operator==(const Tiles &o) const {
    return stack_tn == o.stack_tn && wide_tn == o.wide_tn && max_stages == o.max_stages && split_out == o.split_out &&
           kc_trial == o.kc_trial;
  }
  bool operator!=(const Tiles &o) const { return !(*this == o); }
};

// What one walk needs (filled by the engine).  The population must share one bond profile bW.
struct Problem {
  int L = 0, nC = 0, G = 0;
  std::vector<int> aT, bW;         // trial and walker bond dims [L+1]
  std::vector<long> toff, woff;    // FP64 site offsets of the trial and of a walker slot [L]
  std::vector<int> ci, cj, cq;     // couplings (ordered by i, then j) and their distinct-J index
  std::vector<int> ech_off, ech_slot, ech_cont, eopen;  // compact-MPO channels (as the engine's)
  std::vector<double> ech_J;
  int nslots = 0;
  double h = 0.0;
  double opSx[4], opISy[4], opSz[4];
  const double *trial = nullptr;   // device, FP64, reference layout
  double *walkers = nullptr;       // device slots
  long wstride = 0;
  const int *slot_of = nullptr, *n_cur = nullptr;
  double *weight = nullptr, *overlap = nullptr;      // per slot
  double *energy = nullptr, *ov_out = nullptr, *wt_out = nullptr;  // per logical walker
  const double *uni = nullptr;     // [N][nC] uniforms, logical order
  const double *tabU = nullptr, *tabSq = nullptr, *tabVT = nullptr, *grid = nullptr;
  int *err = nullptr;
  int capacity = 0;                // walkers the batched buffers hold
  int passes = 3;                  // 3: FP32-accurate products, 1: TF32 (or BF16 with bf16)
  bool bf16 = false;               // one BF16 pass (kind::f16) instead of TF32
  Tiles tiles;
};

struct Plan;

// Bit of the engine's device error word set when a tcgen05 pipeline wait timed out.
constexpr int kErrTimeout = 4;

// Allocates the batched work buffers (FP32 site forms, environments, branches, channels) and
// records the step's launch sequence.  Returns 0 or a negative MPSQMC status.
int build(const Problem &pr, Plan **out);
// Enqueues one step's propagation and local energies on `stream` (capturable).  trace: optional
// [N][nC][21] per-coupling record (C/ov, factor, uniform, index, weight).
int enqueue(Plan *p, cudaStream_t stream, double *trace, int *launches);
void destroy(Plan *p);
size_t device_bytes(const Plan *p);
// Device bytes build() would allocate for this problem.
size_t bytes_needed(const Problem &pr);

}  // namespace bs
}  // namespace mq
