// Host implementation of the C ABI declared in include/mpsqmc_gpu.h.
//
// The context owns every device buffer; walkers live in `capacity` fixed-size slots in HBM and
// a logical->slot table gives the population order the reference's theWalkers array has
// (MPSQMC2.h:119-123).  One call of mpsqmc_walk issues, per step, the kernels of
// walker_kernels.cuh on one stream and reads back a small statistics record.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <map>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mpsqmc_gpu.h"
#include "walker_kernels.cuh"
#include "walker_general.cuh"
#include "compress.cuh"
#include "legacy.cuh"
#include "proposal.cuh"
#include "population.cuh"
#include "batched.h"

namespace {

thread_local std::string g_err = "";

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

}  // namespace

// Lets the other translation unit of the library (noalloc.cu) report through mpsqmc_last_error.
namespace mq_host {
__attribute__((visibility("hidden"))) void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace mq_host

namespace {

#define CK(call)                                                                             \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(MPSQMC_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));         \
  } while (0)

template <typename T>
int dalloc(T **p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
  if (e != cudaSuccess) return fail(MPSQMC_E_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return 0;
}

double op_sz(int d, int i, int j) { return (i == j) ? 0.5 * (1 - d) + i : 0.0; }
double ladder(int d, int k) { return 0.25 * std::sqrt(d * d - 1.0 - (1.0 - d + 2 * k) * (3.0 - d + 2 * k)); }
double op_sx(int d, int i, int j) {
  if (i == j + 1) return ladder(d, j);
  if (i + 1 == j) return ladder(d, i);
  return 0.0;
}
double op_isy(int d, int i, int j) {
  if (i == j + 1) return ladder(d, j);
  if (i + 1 == j) return -ladder(d, i);
  return 0.0;
}

bool valid_dims(const int *dims, int L, int d) {
  if (dims[0] != 1 || dims[L] != 1) return false;
  for (int k = 0; k < L; ++k) {
    if (dims[k] < 1 || dims[k + 1] < 1) return false;
    if (dims[k + 1] > d * dims[k] || dims[k] > d * dims[k + 1]) return false;
  }
  return true;
}

}  // namespace

struct mpsqmc_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int L = 0, d = 2, nC = 0, G = 0, nJ = 0, Ndesired = 0, capacity = 0;
  double dtau = 0.0, h = 0.0;
  std::vector<int> aT, bW;
  std::vector<long> toff, woff, roff, nroff, zoff;
  long wsize = 0, wstride = 0, scr_stride = 0, foff = 0, gwoff = -1;
  long scr_base = 0;                    // scratch doubles per CTA before the matrix work buffers
  long all_doubles = 0, big_doubles = 0;  // work buffers: all of them / the matrix ones
  long mlp_doubles = 0;                 // the learned proposal's small buffers (on chip while it is in use)
  size_t smem_optin = 0;
  bool global_work = false;             // matrix work buffers in global scratch
  int maxA = 1, maxB = 1, pa = 4, pb = 4, pq = 4;
  size_t smem_bytes = 0;
  size_t smem_bytes_noqr = 0;           // the QR-free general sweep's (no Householder buffers)
  int sm_count = 1, max_ctas = 1;
  // mixed-precision sweep (FP32 work buffers, TF32 tensor cores): its own shared memory and grid
  int precision = MPSQMC_PRECISION_FP64;
  size_t smem_bytes_mixed = 0;
  int max_ctas_mixed = 1;
  float *d_trial32 = nullptr;
  // learned proposal: FP32 master parameters, Adam moments, gradient, BF16 copy, training pairs
  // and activations (allocated on first use)
  int proposal = MPSQMC_PROPOSAL_GRID;
  bool prop_train = false;
  int prop_mix = 100;  // thousandths of the exact PDF in the learned proposal's mixture
  long nparams = 0;
  float *d_pw = nullptr, *d_pm = nullptr, *d_pv = nullptr, *d_pg = nullptr;
  __nv_bfloat16 *d_pwb = nullptr;
  int *d_pt = nullptr, *d_pb = nullptr;
  double *d_ploss = nullptr;
  float *d_pfeat = nullptr, *d_ptarget = nullptr, *d_ph1 = nullptr, *d_ph2 = nullptr, *d_pz = nullptr,
        *d_pdz = nullptr, *d_pdh2 = nullptr, *d_pdh1 = nullptr;
  // device memory
  int *d_aT = nullptr, *d_bW = nullptr;
  long *d_toff = nullptr, *d_woff = nullptr, *d_roff = nullptr, *d_nroff = nullptr, *d_zoff = nullptr;
  double *d_trial = nullptr, *d_walkers = nullptr;
  int *d_slot_of = nullptr, *d_slot_new = nullptr, *d_free = nullptr, *d_copy_src = nullptr,
      *d_copy_dst = nullptr, *d_parent = nullptr, *d_flag_pos = nullptr, *d_ncur = nullptr;
  double *d_weight = nullptr, *d_overlap = nullptr, *d_ehist = nullptr, *d_energy = nullptr,
         *d_ovout = nullptr, *d_wtout = nullptr, *d_sw = nullptr, *d_uni = nullptr, *d_ubr = nullptr;
  int *d_bond_c = nullptr, *d_bond_j = nullptr;
  // couplings of any range and the energy channels of their compact MPO
  bool nn = true;   // every coupling is (i, i+1)
  int sweep = MPSQMC_SWEEP_AUTO;
  int workspace = MPSQMC_WORKSPACE_AUTO;
  int pc_interval = 1;                  // population control every pc_interval steps
  int resample = MPSQMC_RESAMPLE_THRESHOLD;
  int canon_interval = 16;              // QR-free general sweep, LeftNormalize every K steps (0: off)
  bool gauge_dirty = false;             // the last step left the walkers un-normalised (QR-free)
  // walks split over ranks: between mpsqmc_step_propagate and mpsqmc_step_control
  bool split_pending = false, split_canon = false;
  int split_launches = 0;
  double *d_sums = nullptr;             // [0..4] this rank's sums, [8..13] the global ones
  long nloff = 0;                       // its left norm environment inside a CTA's scratch
  int *d_ncop = nullptr;                // copies per walker in the branching step
  int *d_wdims = nullptr;               // per slot: the walker's bond dims [capacity][L+1]
  long *d_wofs = nullptr;               // per slot: its site offsets [capacity][L]
  int *d_ctr = nullptr;                 // work counters of the persistent kernels
  double *d_stage = nullptr;            // mpsqmc_get_walkers: walkers gathered into logical order
  int stage_walkers = 0;
  // MPO-term projector (MPSQMC::Walk)
  int projector = MPSQMC_PROJECTOR_TROTTER;
  int nterms = 0;
  long loff = 0;
  int *d_term_slot = nullptr, *d_term_site = nullptr, *d_term_op = nullptr, *d_changed = nullptr;
  double *d_term_pref = nullptr;
  double *d_cscr = nullptr;             // mpsqmc_compress_walkers: per-CTA scratch
  long cstride = 0;
  int *d_targets = nullptr;
  long choff = 0;
  int *d_cp_j = nullptr, *d_cp_q = nullptr, *d_site_c0 = nullptr, *d_ech_off = nullptr, *d_ech_slot = nullptr,
      *d_ech_cont = nullptr, *d_eopen = nullptr;
  double *d_ech_J = nullptr;
  double *d_bondJ = nullptr, *d_tabU = nullptr, *d_tabS = nullptr, *d_tabVT = nullptr, *d_grid = nullptr,
         *d_tabSq = nullptr;
  double *d_scratch = nullptr, *d_trace = nullptr;
  int *d_err = nullptr;
  mq::MtState *d_mt = nullptr;
  mq::StepDev *d_sd = nullptr;
  bool trace_on = false;
  int n_cur = 0, step_count = 0, last_n_before = 0, last_n_after = 0;
  unsigned long long draws = 0;
  double last_kernel_ms = 0.0, last_total_ms = 0.0;
  int last_launches = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  double opSx[4], opISy[4], opSz[4];
  // one timestep captured as a CUDA graph (re-captured when the trace setting changes)
  bool use_graph = true;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraphExec_t graph_exec_canon = nullptr;  // QR-free sweep: the step that also left-normalises
  int graph_launches[2] = {0, 0};
  bool graph_trace = false;
  mq::StepDev *h_sd = nullptr;  // pinned copies read back after every step
  int *h_err = nullptr;
  // walker-batched tcgen05 sweep (MPSQMC_PRECISION_TF32X3_TC / TF32_TC): host copies of the
  // coupling and channel tables, and the plan (its buffers hold bcap walkers)
  std::vector<int> h_ci, h_cj, h_cq, h_ech_off, h_ech_slot, h_ech_cont, h_eopen;
  std::vector<double> h_ech_J;
  int nslots = 0;
  mq::bs::Plan *bplan = nullptr;
  int bplan_passes = 0;
  int bcap = 0;
  mq::bs::Tiles tc_tiles;     // tile choices for the next plan (options, autotuner)
  mq::bs::Tiles bplan_tiles;  // those the current plan was built with
};

namespace {

bool general_sweep(const mpsqmc_ctx *c);
bool qr_free(const mpsqmc_ctx *c);
bool mixed(const mpsqmc_ctx *c);

mq::Dev make_dev(mpsqmc_ctx *c) {
  mq::Dev p;
  std::memset(&p, 0, sizeof p);
  p.L = c->L;
  p.d = c->d;
  p.nC = c->nC;
  p.G = c->G;
  p.nJ = c->nJ;
  p.maxA = c->maxA;
  p.maxB = c->maxB;
  p.pa = c->pa;
  p.pb = c->pb;
  p.pq = c->pq;
  p.aT = c->d_aT;
  p.bW = c->d_bW;
  p.toff = c->d_toff;
  p.woff = c->d_woff;
  p.trial = c->d_trial;
  p.trial32 = c->d_trial32;
  p.wstride = c->wstride;
  p.walkers = c->d_walkers;
  p.slot_of = c->d_slot_of;
  p.n_cur = c->d_ncur;
  p.weight = c->d_weight;
  p.overlap = c->d_overlap;
  p.ehist = c->d_ehist;
  p.energy = c->d_energy;
  p.ov_out = c->d_ovout;
  p.wt_out = c->d_wtout;
  p.uni = c->d_uni;
  p.bond_c = c->d_bond_c;
  p.bond_j = c->d_bond_j;
  p.bondJ = c->d_bondJ;
  p.tabU = c->d_tabU;
  p.tabS = c->d_tabS;
  p.tabVT = c->d_tabVT;
  p.tabSq = c->d_tabSq;
  p.grid = c->d_grid;
  for (int k = 0; k < 4; ++k) {
    p.opSx[k] = c->opSx[k];
    p.opISy[k] = c->opISy[k];
    p.opSz[k] = c->opSz[k];
  }
  p.h = c->h;
  for (int sg = 0; sg < mq::kMaxD; ++sg) p.onesite[sg] = std::exp(0.5 * c->h * c->dtau * op_sz(c->d, sg, sg));
  p.scratch = c->d_scratch;
  p.scr_stride = c->scr_stride;
  p.roff = c->d_roff;
  p.nroff = c->d_nroff;
  p.zoff = c->d_zoff;
  p.foff = c->foff;
  p.trace = c->trace_on ? c->d_trace : nullptr;
  p.err = c->d_err;
  p.cp_j = c->d_cp_j;
  p.cp_q = c->d_cp_q;
  p.site_c0 = c->d_site_c0;
  p.ech_off = c->d_ech_off;
  p.ech_slot = c->d_ech_slot;
  p.ech_J = c->d_ech_J;
  p.ech_cont = c->d_ech_cont;
  p.eopen = c->d_eopen;
  p.choff = c->choff;
  p.gwoff = c->gwoff;
  p.wdims = c->d_wdims;
  p.wofs = c->d_wofs;
  p.ctr = c->d_ctr;
  p.nloff = qr_free(c) ? c->nloff : -1;
  const bool trotter = c->projector == MPSQMC_PROJECTOR_TROTTER;
  p.prop_mode = (c->proposal == MPSQMC_PROPOSAL_LEARNED && trotter && c->d_pwb) ? 1 : 0;
  p.prop_collect = (c->prop_train && c->proposal == MPSQMC_PROPOSAL_GRID && trotter && c->d_pwb) ? 1 : 0;
  p.prop_mix = c->prop_mix * 1e-3;
  p.prop_w = c->d_pwb;
  p.prop_feat = c->d_pfeat;
  p.prop_target = c->d_ptarget;
  return p;
}

// The general sweep (walker_general.cuh) runs unless the nearest-neighbour sweep is requested
// (it needs every coupling to be (i, i+1)); it is the faster of the two on chains as well.
bool general_sweep(const mpsqmc_ctx *c) { return c->sweep != MPSQMC_SWEEP_NEAREST; }

// The mixed-precision sweep (MPSQMC_OPT_PRECISION, general sweep of the Trotter projector).
bool mixed(const mpsqmc_ctx *c) {
  return c->precision != MPSQMC_PRECISION_FP64 && general_sweep(c) && c->projector == MPSQMC_PROJECTOR_TROTTER;
}

// The QR-free variant of the general sweep (MPSQMC_OPT_CANONICAL_INTERVAL > 0, Trotter projector;
// always for the mixed-precision sweep).
bool qr_free(const mpsqmc_ctx *c) {
  return (c->canon_interval > 0 || mixed(c)) && general_sweep(c) && c->projector == MPSQMC_PROJECTOR_TROTTER;
}

// The walker-batched sweep on the tcgen05 tensor cores (batched.h).
bool tc_sweep(const mpsqmc_ctx *c) {
  return (c->precision == MPSQMC_PRECISION_TF32X3_TC || c->precision == MPSQMC_PRECISION_TF32_TC ||
          c->precision == MPSQMC_PRECISION_BF16_TC) &&
         mixed(c);
}

// Steps between two left-normalisations of the QR-free sweep.
constexpr int kMixedCanonInterval = 4;  // default of the mixed-precision sweep
int canon_every(const mpsqmc_ctx *c) { return c->canon_interval > 0 ? c->canon_interval : kMixedCanonInterval; }

// Doubles of per-CTA scratch for the largest grid of any walker kernel (the mixed sweep reads a
// CTA's scratch as floats with the same stride).
size_t scratch_doubles(const mpsqmc_ctx *c) {
  return std::max((size_t)c->max_ctas * c->scr_stride, ((size_t)c->max_ctas_mixed * c->scr_stride + 1) / 2);
}

int layout_workspace(mpsqmc_ctx *c, bool force_global);

// Recompute the work-buffer layout (after an option that changes it) and grow the scratch if needed.
int relayout(mpsqmc_ctx *c, bool force_global) {
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  const size_t before = c->d_scratch ? scratch_doubles(c) : 0;
  const int rc = layout_workspace(c, force_global);
  if (rc) return rc;
  if (scratch_doubles(c) > before) {
    cudaFree(c->d_scratch);
    c->d_scratch = nullptr;
    if (dalloc(&c->d_scratch, scratch_doubles(c))) return MPSQMC_E_CUDA;
  }
  return 0;
}

void drop_graphs(mpsqmc_ctx *c) {
  for (cudaGraphExec_t *g : {&c->graph_exec, &c->graph_exec_canon})
    if (*g) {
      cudaGraphExecDestroy(*g);
      *g = nullptr;
    }
}

int grid_for(const mpsqmc_ctx *c, int n) { return std::max(1, std::min(n, c->max_ctas)); }

int check_err(mpsqmc_ctx *c) {
  int e = 0;
  CK(cudaMemcpyAsync(&e, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (e & mq::bs::kErrTimeout) return fail(MPSQMC_E_CUDA, "a tcgen05 pipeline wait timed out");
  if (e & mq::kErrCapacity)
    return fail(MPSQMC_E_CAPACITY, "population control exceeded the walker capacity");
  if (e & mq::kErrNumeric) return fail(MPSQMC_E_NUMERIC, "non-finite weight, overlap or energy");
  return 0;
}

void free_all(mpsqmc_ctx *c) {
  if (c->bplan) {
    mq::bs::destroy(c->bplan);
    c->bplan = nullptr;
  }
  void *ptrs[] = {c->d_zoff, c->d_sums, c->d_pw, c->d_pm, c->d_pv, c->d_pg, c->d_pwb, c->d_pt, c->d_pb, c->d_ploss, c->d_pfeat,
                  c->d_ptarget, c->d_ph1, c->d_ph2, c->d_pz, c->d_pdz, c->d_pdh2, c->d_pdh1, c->d_trial32, c->d_aT, c->d_bW, c->d_toff, c->d_woff, c->d_roff, c->d_nroff, c->d_trial, c->d_walkers,
                  c->d_slot_of, c->d_slot_new, c->d_free, c->d_copy_src, c->d_copy_dst, c->d_parent,
                  c->d_flag_pos, c->d_ncur, c->d_weight, c->d_overlap, c->d_ehist, c->d_energy,
                  c->d_ovout, c->d_wtout, c->d_sw, c->d_uni, c->d_ubr, c->d_bond_c, c->d_bond_j,
                  c->d_bondJ, c->d_tabU, c->d_tabS, c->d_tabVT, c->d_grid, c->d_scratch, c->d_trace,
                  c->d_err, c->d_mt, c->d_sd, c->d_cp_j, c->d_cp_q, c->d_site_c0, c->d_ech_off,
                  c->d_ech_slot, c->d_ech_cont, c->d_eopen, c->d_ech_J, c->d_ncop, c->d_wdims, c->d_wofs,
                  c->d_ctr, c->d_stage, c->d_cscr, c->d_targets, c->d_tabSq, c->d_term_slot,
                  c->d_term_site, c->d_term_op, c->d_changed, c->d_term_pref};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  drop_graphs(c);
  if (c->h_sd) cudaFreeHost(c->h_sd);
  if (c->h_err) cudaFreeHost(c->h_err);
  for (auto &e : c->ev)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
}

// Where the matrix work buffers of a CTA live: shared memory when they fit (and are not forced
// out), else the CTA's global scratch.  Sets the scratch stride, the dynamic shared memory of
// every walker kernel and the persistent grid size.
// The learned proposal's buffers are on chip while the proposal samples or trains (the same
// condition make_dev gives the kernels).
bool mlp_on(const mpsqmc_ctx *c) {
  return c->d_pwb != nullptr && c->projector == MPSQMC_PROJECTOR_TROTTER &&
         (c->proposal == MPSQMC_PROPOSAL_LEARNED || c->prop_train);
}

int layout_workspace(mpsqmc_ctx *c, bool force_global) {
  const bool mlp = mlp_on(c);
  const long all = c->all_doubles + (mlp ? c->mlp_doubles : 0);
  const bool global = force_global || sizeof(double) * (size_t)all > c->smem_optin;
  c->scr_stride = (c->scr_base + 31) & ~31L;
  c->gwoff = -1;
  c->smem_bytes = sizeof(double) * (size_t)all;
  if (global) {
    c->gwoff = c->scr_stride;
    c->scr_stride = (c->gwoff + c->big_doubles + 31) & ~31L;
    c->smem_bytes = sizeof(double) * (size_t)(all - c->big_doubles);
  }
  c->global_work = global;
  c->smem_bytes_noqr = global ? c->smem_bytes
                              : sizeof(double) * (size_t)mq::smem_doubles(c->L, c->maxA, c->maxB, c->G, c->pa, c->pb,
                                                                          c->pq, nullptr, nullptr, nullptr, nullptr,
                                                                          mlp, false);
  if (c->smem_bytes > c->smem_optin)
    return fail(MPSQMC_E_UNSUPPORTED, "grid too large for the shared-memory budget of one CTA");
  const void *kernels[] = {(const void *)mq::walker_step_kernel, (const void *)mq::set_overlap_kernel,
                           (const void *)mq::energy_kernel, (const void *)mq::walker_step_general_kernel<true, 1>,
                           (const void *)mq::walker_step_general_kernel<true, 1, false>,
                           (const void *)mq::walker_step_general_kernel<true, 2>,
                           (const void *)mq::walker_step_general_kernel<false, 0>,
                           (const void *)mq::energy_general_kernel, (const void *)mq::legacy_step_kernel};
  for (const void *k : kernels)
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem_bytes));
  int occ = 1;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, mq::walker_step_kernel, mq::kThreads, c->smem_bytes));
  c->max_ctas = std::max(1, occ) * c->sm_count;
  // mixed-precision sweep: FP32 matrix buffers next to the small FP64 ones, on chip unless the
  // FP64 buffers were placed in global scratch
  long big_floats = 0;
  const long mixed_all = mq::smem_bytes_f32(c->L, c->maxA, c->maxB, c->G, c->pa, c->pb, nullptr, nullptr, nullptr,
                                            &big_floats, mlp);
  c->smem_bytes_mixed = global ? (size_t)(mixed_all - (long)sizeof(float) * big_floats) : (size_t)mixed_all;
  const void *mk[] = {(const void *)mq::walker_step_mixed_kernel<1, true>, (const void *)mq::walker_step_mixed_kernel<3, true>,
                      (const void *)mq::walker_step_mixed_kernel<1, false>, (const void *)mq::walker_step_mixed_kernel<3, false>};
  for (const void *k : mk)
    CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->smem_bytes_mixed));
  int occm = 1;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occm, mq::walker_step_mixed_kernel<3, true>, mq::kThreads,
                                                   c->smem_bytes_mixed));
  c->max_ctas_mixed = std::max(1, std::min(occm, 2)) * c->sm_count;
  return 0;
}

}  // namespace

extern "C" {

const char *mpsqmc_last_error(void) { return g_err.c_str(); }

const char *mpsqmc_version(void) { return "mpsqmc_b200 0.1 (sm_100a, fp64 dmma)"; }

long mpsqmc_walker_size(const mpsqmc_ctx *ctx) { return ctx ? ctx->wsize : -1; }

int mpsqmc_create(const mpsqmc_config *cfg, mpsqmc_ctx **out) {
  if (!cfg || !out) return fail(MPSQMC_E_ARG, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(MPSQMC_E_NODEVICE, "no CUDA device visible; the engine has no CPU fallback");
  if (cfg->device < 0 || cfg->device >= ndev) return fail(MPSQMC_E_ARG, "device ordinal out of range");
  if (cfg->d != mq::kMaxD) return fail(MPSQMC_E_UNSUPPORTED, "only d = 2 (spin 1/2) is implemented");
  const int L = cfg->L, d = cfg->d;
  if (L < 3) return fail(MPSQMC_E_ARG, "L must be >= 3 (HeisenbergMPO.cpp:10)");
  if (cfg->nC < 1 || !cfg->ci || !cfg->cj || !cfg->cJ) return fail(MPSQMC_E_ARG, "no couplings");
  if (cfg->G < 1 || !cfg->grid) return fail(MPSQMC_E_ARG, "empty grid");
  if (cfg->nJ < 1 || !cfg->Jvals || !cfg->U || !cfg->S || !cfg->VT)
    return fail(MPSQMC_E_ARG, "missing Trotter tables");
  if (cfg->capacity < 1 || cfg->Ndesired < 1) return fail(MPSQMC_E_ARG, "bad walker counts");
  if (!cfg->trial_dims || !cfg->trial || !cfg->walker_dims) return fail(MPSQMC_E_ARG, "missing MPS data");
  if (!valid_dims(cfg->trial_dims, L, d) || !valid_dims(cfg->walker_dims, L, d))
    return fail(MPSQMC_E_ARG, "bond dimensions inconsistent with the chain");
  // Couplings in the order MPSQMC2.cpp:286-299 lists them: by first site, then by second site.
  std::vector<int> bond_c(L - 1, -1), bond_j(L - 1, -1), cp_j(cfg->nC), cp_q(cfg->nC), site_c0(L + 1, 0);
  std::vector<double> bondJ(L - 1, 0.0);
  bool nn = true;
  for (int c = 0; c < cfg->nC; ++c) {
    const int i = cfg->ci[c], j = cfg->cj[c];
    if (i < 0 || j >= L || i >= j) return fail(MPSQMC_E_ARG, "coupling indices out of order");
    if (c > 0 && (cfg->ci[c - 1] > i || (cfg->ci[c - 1] == i && cfg->cj[c - 1] >= j)))
      return fail(MPSQMC_E_ARG, "couplings must be ordered by first site, then by second site, without repeats");
    int q = -1;
    for (int t = 0; t < cfg->nJ; ++t)
      if (cfg->Jvals[t] == cfg->cJ[c]) {
        q = t;
        break;
      }
    if (q < 0) return fail(MPSQMC_E_ARG, "coupling strength without Trotter tables");
    cp_j[c] = j;
    cp_q[c] = q;
    site_c0[i + 1] += 1;
    if (j != i + 1) {
      nn = false;
    } else {
      bond_c[i] = c;
      bond_j[i] = q;
      bondJ[i] = cfg->cJ[c];
    }
  }
  for (int i = 0; i < L; ++i) site_c0[i + 1] += site_c0[i];
  // Energy channels: a site i is open on the cut before site k when it couples to some j >= k.
  // Site k closes the couplings (i, k) and opens its own channel if it has a partner beyond k.
  // A slot freed on site k can be taken by the channel site k opens (the kernel reads closing
  // channels before it writes the new one).
  std::vector<int> last_partner(L, -1);
  for (int c = 0; c < cfg->nC; ++c) last_partner[cfg->ci[c]] = std::max(last_partner[cfg->ci[c]], cfg->cj[c]);
  std::vector<int> ech_off(L + 1, 0), ech_slot, ech_cont, eopen(L, -1), slot_of_site(L, -1), free_slots;
  std::vector<double> ech_J;
  std::vector<int> open_sites;
  int nslots = 0;
  for (int k = 0; k < L; ++k) {
    ech_off[k] = (int)ech_slot.size();
    std::vector<int> still;
    for (int i : open_sites) {
      double J = 0.0;
      for (int c = site_c0[i]; c < site_c0[i + 1]; ++c)
        if (cp_j[c] == k) J += cfg->cJ[c];
      const bool cont = last_partner[i] > k;
      ech_slot.push_back(slot_of_site[i]);
      ech_J.push_back(J);
      ech_cont.push_back(cont ? 1 : 0);
      if (cont) still.push_back(i);
      else free_slots.push_back(slot_of_site[i]);
    }
    open_sites.swap(still);
    if (last_partner[k] > k) {
      int sl;
      if (!free_slots.empty()) {
        sl = free_slots.back();
        free_slots.pop_back();
      } else {
        sl = nslots++;
      }
      slot_of_site[k] = sl;
      eopen[k] = sl;
      open_sites.push_back(k);
    }
  }
  ech_off[L] = (int)ech_slot.size();
  if (ech_slot.empty()) {  // keep the device arrays non-empty
    ech_slot.push_back(0);
    ech_J.push_back(0.0);
    ech_cont.push_back(0);
  }

  std::vector<int> h_ci(cfg->ci, cfg->ci + cfg->nC), h_cj(cfg->cj, cfg->cj + cfg->nC);
  // Terms of the MPO-term projector, in the order HeisenbergMPO::findNonZeroContributions lists
  // them (HeisenbergMPO.cpp:456-553): per coupling J Sx Sx, -J iSy iSy, J Sz Sz; then -h Sz on
  // every site.  slot: where the sweep stores the term's overlap without prefactor.
  std::vector<int> term_slot, term_site, term_op;
  std::vector<double> term_pref;
  for (int c = 0; c < cfg->nC; ++c)
    for (int a = 0; a < 3; ++a) {
      term_slot.push_back(3 * c + a);
      term_site.push_back(cfg->ci[c]);
      term_site.push_back(cfg->cj[c]);
      term_op.push_back(a + 1);
      term_op.push_back(a + 1);
      term_pref.push_back(a == 1 ? -cfg->cJ[c] : cfg->cJ[c]);
    }
  if (cfg->h != 0.0)
    for (int k = 0; k < L; ++k) {
      term_slot.push_back(3 * cfg->nC + k);
      term_site.push_back(k);
      term_site.push_back(-1);
      term_op.push_back(3);
      term_op.push_back(0);
      term_pref.push_back(-cfg->h);
    }

  mpsqmc_ctx *c = new mpsqmc_ctx();
  c->device = cfg->device;
  if (cudaSetDevice(c->device) != cudaSuccess) {
    delete c;
    return fail(MPSQMC_E_CUDA, "cudaSetDevice failed");
  }
  c->L = L;
  c->d = d;
  c->nC = cfg->nC;
  c->G = cfg->G;
  c->nJ = cfg->nJ;
  c->Ndesired = cfg->Ndesired;
  c->capacity = cfg->capacity;
  c->dtau = cfg->dtau;
  c->h = cfg->h;
  c->nn = nn;
  c->nterms = (int)term_pref.size();
  c->h_ci = h_ci;
  c->h_cj = h_cj;
  c->h_cq = cp_q;
  c->h_ech_off = ech_off;
  c->h_ech_slot = ech_slot;
  c->h_ech_cont = ech_cont;
  c->h_eopen = eopen;
  c->h_ech_J = ech_J;
  c->nslots = nslots;
  c->aT.assign(cfg->trial_dims, cfg->trial_dims + L + 1);
  c->bW.assign(cfg->walker_dims, cfg->walker_dims + L + 1);
  c->toff.resize(L);
  c->woff.resize(L);
  long to = 0, wo = 0;
  for (int k = 0; k < L; ++k) {
    c->toff[k] = to;
    c->woff[k] = wo;
    to += (long)c->aT[k] * c->aT[k + 1] * d;
    wo += (long)c->bW[k] * c->bW[k + 1] * d;
  }
  c->wsize = wo;
  c->wstride = (wo + 31) & ~31L;
  c->maxA = *std::max_element(c->aT.begin(), c->aT.end());
  c->maxB = *std::max_element(c->bW.begin(), c->bW.end());
  c->pa = mq::padld(std::max(c->maxA, c->maxB));  // slots also hold walker-row matrices
  c->pb = mq::padld(c->maxB);
  c->pq = mq::padld(d * c->maxB);
  c->all_doubles =
      mq::smem_doubles(L, c->maxA, c->maxB, c->G, c->pa, c->pb, c->pq, nullptr, nullptr, nullptr, &c->big_doubles);
  c->mlp_doubles = mq::smem_doubles(L, c->maxA, c->maxB, c->G, c->pa, c->pb, c->pq, nullptr, nullptr, nullptr,
                                    nullptr, true) - c->all_doubles;
  c->roff.resize(L + 1);
  long ro = 0;
  for (int k = 0; k <= L; ++k) {
    c->roff[k] = ro;
    ro += ((long)c->aT[k] * c->bW[k] + 3) & ~3L;
  }
  c->nroff.resize(L + 1);
  for (int k = 0; k <= L; ++k) {
    c->nroff[k] = ro;
    ro += ((long)c->bW[k] * c->bW[k] + 3) & ~3L;
  }
  c->foff = ro;
  c->choff = ro + 2L * 4 * c->maxA * c->maxB;
  c->loff = c->choff + (2L + 3L * nslots) * c->maxA * c->maxB;
  c->nloff = c->loff + ((2L * (3L * c->nC + L + 1) + 31) & ~31L);
  {  // nearest-neighbour couplings: right branches Z[k] (4 blocks of a_k x b_k) of every site
    long zo = c->nloff + (((long)c->pb * c->maxB + 31) & ~31L);
    c->zoff.resize(L);
    for (int k = 0; k < L; ++k) {
      c->zoff[k] = zo;
      if (nn) zo += (4L * c->aT[k] * c->bW[k] + 3) & ~3L;
    }
    c->scr_base = zo;
  }
  for (int s = 0; s < 2; ++s)
    for (int t = 0; t < 2; ++t) {
      c->opSx[s + 2 * t] = op_sx(d, s, t);
      c->opISy[s + 2 * t] = op_isy(d, s, t);
      c->opSz[s + 2 * t] = op_sz(d, s, t);
    }

  auto bail = [&](int code) {
    free_all(c);
    delete c;
    return code;
  };
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess) return bail(fail(MPSQMC_E_CUDA, "properties"));
  c->sm_count = prop.multiProcessorCount;
  c->smem_optin = prop.sharedMemPerBlockOptin;
  if (c->maxB > mq::kThreads / 2)
    return bail(fail(MPSQMC_E_UNSUPPORTED, "walker bond dimension above 128 (one QR column group per warp)"));
  {
    const int rc = layout_workspace(c, false);
    if (rc) return bail(rc);
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return bail(fail(MPSQMC_E_CUDA, "stream"));
  for (auto &e : c->ev)
    if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(MPSQMC_E_CUDA, "event"));
  const int cap = c->capacity;
  int rc = 0;
  rc |= dalloc(&c->d_aT, L + 1) | dalloc(&c->d_bW, L + 1) | dalloc(&c->d_toff, L) | dalloc(&c->d_woff, L) |
        dalloc(&c->d_roff, L + 1) | dalloc(&c->d_nroff, L + 1) | dalloc(&c->d_zoff, L) | dalloc(&c->d_trial, to) | dalloc(&c->d_walkers, (size_t)cap * c->wstride) |
        dalloc(&c->d_slot_of, cap) | dalloc(&c->d_slot_new, cap) | dalloc(&c->d_free, cap) |
        dalloc(&c->d_copy_src, cap) | dalloc(&c->d_copy_dst, cap) | dalloc(&c->d_parent, cap) |
        dalloc(&c->d_flag_pos, cap) | dalloc(&c->d_ncur, 1) | dalloc(&c->d_weight, cap) |
        dalloc(&c->d_overlap, cap) | dalloc(&c->d_ehist, cap) | dalloc(&c->d_energy, cap) |
        dalloc(&c->d_ovout, cap) | dalloc(&c->d_wtout, cap) | dalloc(&c->d_sw, cap) |
        dalloc(&c->d_uni, (size_t)cap * c->nC) | dalloc(&c->d_ubr, cap) | dalloc(&c->d_bond_c, L - 1) |
        dalloc(&c->d_bond_j, L - 1) | dalloc(&c->d_bondJ, L - 1) | dalloc(&c->d_tabU, 16 * c->nJ) |
        dalloc(&c->d_tabS, 4 * c->nJ) | dalloc(&c->d_tabVT, 16 * c->nJ) | dalloc(&c->d_grid, 4 * c->G) |
        dalloc(&c->d_tabSq, 4 * c->nJ) |
        dalloc(&c->d_scratch, scratch_doubles(c)) | dalloc(&c->d_err, 1) | dalloc(&c->d_trial32, to) |
        dalloc(&c->d_mt, 1) | dalloc(&c->d_sd, 1) | dalloc(&c->d_cp_j, c->nC) | dalloc(&c->d_cp_q, c->nC) |
        dalloc(&c->d_site_c0, L + 1) | dalloc(&c->d_ech_off, L + 1) | dalloc(&c->d_ech_slot, ech_slot.size()) |
        dalloc(&c->d_ech_cont, ech_cont.size()) | dalloc(&c->d_eopen, L) | dalloc(&c->d_ech_J, ech_J.size()) |
        dalloc(&c->d_ncop, cap) | dalloc(&c->d_wdims, (size_t)cap * (L + 1)) | dalloc(&c->d_wofs, (size_t)cap * L) |
        dalloc(&c->d_ctr, mq::kNumCtr) | dalloc(&c->d_term_slot, term_slot.size()) |
        dalloc(&c->d_term_site, term_site.size()) | dalloc(&c->d_term_op, term_op.size()) |
        dalloc(&c->d_term_pref, term_pref.size()) | dalloc(&c->d_changed, cap);
  if (rc) return bail(MPSQMC_E_CUDA);
  if (cudaMallocHost((void **)&c->h_sd, sizeof(mq::StepDev)) != cudaSuccess ||
      cudaMallocHost((void **)&c->h_err, sizeof(int)) != cudaSuccess)
    return bail(fail(MPSQMC_E_CUDA, "pinned host buffers"));
  std::vector<float> trial32(cfg->trial, cfg->trial + to);
  std::vector<double> sqS(4 * c->nJ);
  for (int q = 0; q < 4 * c->nJ; ++q) sqS[q] = std::sqrt(cfg->S[q]);
  auto up = [&](void *dst, const void *src, size_t bytes) {
    return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
  };
  bool ok = up(c->d_aT, c->aT.data(), sizeof(int) * (L + 1)) && up(c->d_bW, c->bW.data(), sizeof(int) * (L + 1)) &&
            up(c->d_toff, c->toff.data(), sizeof(long) * L) && up(c->d_woff, c->woff.data(), sizeof(long) * L) &&
            up(c->d_roff, c->roff.data(), sizeof(long) * (L + 1)) &&
            up(c->d_nroff, c->nroff.data(), sizeof(long) * (L + 1)) &&
            up(c->d_zoff, c->zoff.data(), sizeof(long) * L) &&
            up(c->d_trial, cfg->trial, sizeof(double) * to) && up(c->d_trial32, trial32.data(), sizeof(float) * to) &&
            up(c->d_bond_c, bond_c.data(), sizeof(int) * (L - 1)) &&
            up(c->d_bond_j, bond_j.data(), sizeof(int) * (L - 1)) &&
            up(c->d_bondJ, bondJ.data(), sizeof(double) * (L - 1)) &&
            up(c->d_tabU, cfg->U, sizeof(double) * 16 * c->nJ) && up(c->d_tabS, cfg->S, sizeof(double) * 4 * c->nJ) &&
            up(c->d_tabVT, cfg->VT, sizeof(double) * 16 * c->nJ) && up(c->d_grid, cfg->grid, sizeof(double) * 4 * c->G) &&
            up(c->d_tabSq, sqS.data(), sizeof(double) * 4 * c->nJ) &&
            up(c->d_cp_j, cp_j.data(), sizeof(int) * c->nC) && up(c->d_cp_q, cp_q.data(), sizeof(int) * c->nC) &&
            up(c->d_site_c0, site_c0.data(), sizeof(int) * (L + 1)) &&
            up(c->d_ech_off, ech_off.data(), sizeof(int) * (L + 1)) &&
            up(c->d_ech_slot, ech_slot.data(), sizeof(int) * ech_slot.size()) &&
            up(c->d_ech_cont, ech_cont.data(), sizeof(int) * ech_cont.size()) &&
            up(c->d_eopen, eopen.data(), sizeof(int) * L) &&
            up(c->d_ech_J, ech_J.data(), sizeof(double) * ech_J.size()) &&
            up(c->d_term_slot, term_slot.data(), sizeof(int) * term_slot.size()) &&
            up(c->d_term_site, term_site.data(), sizeof(int) * term_site.size()) &&
            up(c->d_term_op, term_op.data(), sizeof(int) * term_op.size()) &&
            up(c->d_term_pref, term_pref.data(), sizeof(double) * term_pref.size());
  if (!ok) return bail(fail(MPSQMC_E_CUDA, "upload failed"));
  {  // every slot starts with the common walker dims
    std::vector<int> wd((size_t)cap * (L + 1));
    std::vector<long> wf((size_t)cap * L);
    for (int q = 0; q < cap; ++q) {
      std::copy(c->bW.begin(), c->bW.end(), wd.begin() + (size_t)q * (L + 1));
      std::copy(c->woff.begin(), c->woff.end(), wf.begin() + (size_t)q * L);
    }
    if (!up(c->d_wdims, wd.data(), sizeof(int) * wd.size()) || !up(c->d_wofs, wf.data(), sizeof(long) * wf.size()))
      return bail(fail(MPSQMC_E_CUDA, "upload failed"));
  }
  if (cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess || cudaMemset(c->d_sd, 0, sizeof(mq::StepDev)) != cudaSuccess ||
      cudaMemset(c->d_ncur, 0, sizeof(int)) != cudaSuccess)
    return bail(fail(MPSQMC_E_CUDA, "memset failed"));
  *out = c;
  // default stream position: seed 5489 (std::mt19937 default), nothing skipped
  return mpsqmc_set_rng(c, 5489u, 0);
}

int mpsqmc_destroy(mpsqmc_ctx *ctx) {
  if (!ctx) return 0;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
  return 0;
}

int mpsqmc_set_rng(mpsqmc_ctx *c, uint32_t seed, uint64_t skip) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  std::mt19937 gen(seed);
  gen.discard(skip);
  std::stringstream ss;
  ss << gen;  // 624 state words followed by the position
  mq::MtState st;
  std::memset(&st, 0, sizeof st);
  for (int q = 0; q < 624; ++q) {
    unsigned long v;
    ss >> v;
    st.mt[q] = (uint32_t)v;
  }
  ss >> st.idx;
  st.draws = 0;
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(c->d_mt, &st, sizeof st, cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->draws = 0;
  return 0;
}

int mpsqmc_get_rng_draws(mpsqmc_ctx *c, uint64_t *draws) {
  if (!c || !draws) return fail(MPSQMC_E_ARG, "null argument");
  mq::MtState st;
  CK(cudaMemcpy(&st, c->d_mt, sizeof st, cudaMemcpyDeviceToHost));
  *draws = st.draws;
  return 0;
}

// Upload N walkers into slots 0..N-1.  dims == nullptr: every walker has the common dims and
// walker_size doubles (stride walker_size); else walker w has dims[w*(L+1) ..] and its tensors
// follow the previous walker's back to back.
static int set_walkers_impl(mpsqmc_ctx *c, int N, const int *dims, const double *walkers, const double *weights,
                            const double *overlaps, const double *ehist, int normalize) {
  if (!c || !walkers || !weights) return fail(MPSQMC_E_ARG, "null argument");
  if (N < 1 || N > c->capacity) return fail(MPSQMC_E_ARG, "walker count outside [1, capacity]");
  const int L = c->L, d = c->d;
  std::vector<int> wd((size_t)N * (L + 1));
  std::vector<long> wf((size_t)N * L);
  std::vector<long> src_off(N);
  long pos = 0;
  for (int w = 0; w < N; ++w) {
    const int *dw = dims ? dims + (size_t)w * (L + 1) : c->bW.data();
    if (dims) {
      if (!valid_dims(dw, L, d)) return fail(MPSQMC_E_ARG, "walker bond dimensions inconsistent with the chain");
      for (int k = 0; k <= L; ++k)
        if (dw[k] > c->bW[k]) return fail(MPSQMC_E_ARG, "walker bond dimension above the configured walker_dims");
    }
    long o = 0;
    for (int k = 0; k < L; ++k) {
      wf[(size_t)w * L + k] = o;
      o += (long)dw[k] * dw[k + 1] * d;
    }
    std::copy(dw, dw + L + 1, wd.begin() + (size_t)w * (L + 1));
    src_off[w] = pos;
    pos += dims ? o : c->wsize;
  }
  CK(cudaSetDevice(c->device));
  if (dims) {
    for (int w = 0; w < N; ++w) {
      const long n = (w + 1 < N ? src_off[w + 1] : pos) - src_off[w];
      CK(cudaMemcpyAsync(c->d_walkers + (size_t)w * c->wstride, walkers + src_off[w], sizeof(double) * n,
                         cudaMemcpyHostToDevice, c->stream));
    }
  } else {
    CK(cudaMemcpy2DAsync(c->d_walkers, sizeof(double) * c->wstride, walkers, sizeof(double) * c->wsize,
                         sizeof(double) * c->wsize, N, cudaMemcpyHostToDevice, c->stream));
  }
  CK(cudaMemcpyAsync(c->d_wdims, wd.data(), sizeof(int) * wd.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_wofs, wf.data(), sizeof(long) * wf.size(), cudaMemcpyHostToDevice, c->stream));
  std::vector<int> slots(N), freel(c->capacity - N);
  for (int w = 0; w < N; ++w) slots[w] = w;
  for (int q = 0; q < c->capacity - N; ++q) freel[q] = c->capacity - 1 - q;
  std::vector<double> zeros(N, 0.0), ones(N, 1.0);
  CK(cudaMemcpyAsync(c->d_slot_of, slots.data(), sizeof(int) * N, cudaMemcpyHostToDevice, c->stream));
  if (!freel.empty())
    CK(cudaMemcpyAsync(c->d_free, freel.data(), sizeof(int) * freel.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_weight, weights, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_overlap, overlaps ? overlaps : ones.data(), sizeof(double) * N,
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_ehist, ehist ? ehist : zeros.data(), sizeof(double) * N, cudaMemcpyHostToDevice,
                     c->stream));
  mq::StepDev sd;
  std::memset(&sd, 0, sizeof sd);
  sd.n_cur = N;
  sd.n_free = c->capacity - N;
  sd.step = c->step_count;
  CK(cudaMemcpyAsync(c->d_sd, &sd, sizeof sd, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_ncur, &N, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
  c->n_cur = N;
  c->gauge_dirty = false;
  if (normalize) {
    mq::Dev p = make_dev(c);
    CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(int) * mq::kNumCtr, c->stream));
    mq::set_overlap_kernel<<<grid_for(c, N), mq::kThreads, c->smem_bytes, c->stream>>>(p);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->stream));
  return check_err(c);
}

// Walkers left by a QR-free step are not left-canonical: set_overlap_kernel restores
// Walker::setOverlap's state (same quantum state, overlap recomputed) before they are read out
// or compressed.
static int restore_canonical(mpsqmc_ctx *c) {
  if (!c->gauge_dirty || c->n_cur < 1) return 0;
  CK(cudaSetDevice(c->device));
  mq::Dev p = make_dev(c);
  CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(int) * mq::kNumCtr, c->stream));
  mq::set_overlap_kernel<<<grid_for(c, c->n_cur), mq::kThreads, c->smem_bytes, c->stream>>>(p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  c->gauge_dirty = false;
  return check_err(c);
}

int mpsqmc_set_walkers(mpsqmc_ctx *c, int N, const double *walkers, const double *weights,
                       const double *overlaps, const double *ehist, int normalize) {
  return set_walkers_impl(c, N, nullptr, walkers, weights, overlaps, ehist, normalize);
}

int mpsqmc_set_walkers_dims(mpsqmc_ctx *c, int N, const int *dims, const double *walkers, const double *weights,
                            const double *overlaps, const double *ehist, int normalize) {
  if (!dims) return fail(MPSQMC_E_ARG, "null dims");
  return set_walkers_impl(c, N, dims, walkers, weights, overlaps, ehist, normalize);
}

int mpsqmc_compress_walkers(mpsqmc_ctx *c, const int *target_D, int normalize) {
  if (!c || !target_D) return fail(MPSQMC_E_ARG, "null argument");
  const int n = c->n_cur;
  if (n < 1) return fail(MPSQMC_E_ARG, "no walkers");
  {
    const int rc = restore_canonical(c);
    if (rc) return rc;
  }
  CK(cudaSetDevice(c->device));
  if (!c->d_cscr) {
    const long q2 = 2L * c->maxB;
    const long wmax = c->woff[c->L - 1] + (long)c->bW[c->L - 1] * c->bW[c->L] * c->d;
    c->cstride = ((wmax + 31) & ~31L) + 3 * q2 * q2;
    c->cstride = (c->cstride + 31) & ~31L;
    if (dalloc(&c->d_cscr, (size_t)c->max_ctas * c->cstride) || dalloc(&c->d_targets, c->capacity))
      return MPSQMC_E_CUDA;
  }
  CK(cudaMemcpyAsync(c->d_targets, target_D, sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(int) * mq::kNumCtr, c->stream));
  mq::Dev p = make_dev(c);
  mq::compress_kernel<<<grid_for(c, n), mq::kThreads, mq::compress_smem_bytes(c->L, c->maxB), c->stream>>>(
      p, c->d_targets, c->d_cscr, c->cstride);
  CK(cudaGetLastError());
  if (normalize) {
    CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(int) * mq::kNumCtr, c->stream));
    mq::set_overlap_kernel<<<grid_for(c, n), mq::kThreads, c->smem_bytes, c->stream>>>(p);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(c->stream));
  return check_err(c);
}

int mpsqmc_get_walker_dims(mpsqmc_ctx *c, int *N, int *dims) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  CK(cudaSetDevice(c->device));
  const int n = c->n_cur, L = c->L;
  if (N) *N = n;
  if (!dims) return 0;
  std::vector<int> slots(n), all((size_t)c->capacity * (L + 1));
  CK(cudaMemcpy(slots.data(), c->d_slot_of, sizeof(int) * n, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(all.data(), c->d_wdims, sizeof(int) * all.size(), cudaMemcpyDeviceToHost));
  for (int w = 0; w < n; ++w)
    std::copy(all.begin() + (size_t)slots[w] * (L + 1), all.begin() + (size_t)(slots[w] + 1) * (L + 1),
              dims + (size_t)w * (L + 1));
  return 0;
}

int mpsqmc_get_walkers(mpsqmc_ctx *c, int *N, double *walkers, double *weights, double *overlaps,
                       double *ehist) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  if (walkers || overlaps) {
    const int rc = restore_canonical(c);
    if (rc) return rc;
  }
  CK(cudaSetDevice(c->device));
  const int n = c->n_cur;
  if (N) *N = n;
  std::vector<int> slots(n);
  CK(cudaMemcpy(slots.data(), c->d_slot_of, sizeof(int) * n, cudaMemcpyDeviceToHost));
  std::vector<double> buf(c->capacity);
  auto gather = [&](double *dst, const double *src) -> int {
    if (!dst) return 0;
    CK(cudaMemcpy(buf.data(), src, sizeof(double) * c->capacity, cudaMemcpyDeviceToHost));
    for (int w = 0; w < n; ++w) dst[w] = buf[slots[w]];
    return 0;
  };
  int rc = gather(weights, c->d_weight) | gather(overlaps, c->d_overlap) | gather(ehist, c->d_ehist);
  if (rc) return rc;
  if (walkers && n > 0) {
    // gather the slots into logical order on the device, then one copy per chunk
    if (!c->d_stage) {
      const long per = c->wsize;
      c->stage_walkers = (int)std::max(1L, std::min<long>(c->capacity, (256L << 20) / (8 * per)));
      if (dalloc(&c->d_stage, (size_t)c->stage_walkers * per)) return MPSQMC_E_CUDA;
    }
    mq::Dev p = make_dev(c);
    for (int w0 = 0; w0 < n; w0 += c->stage_walkers) {
      const int m = std::min(c->stage_walkers, n - w0);
      mq::gather_walkers_kernel<<<std::min(m, 4 * c->sm_count), 256, 0, c->stream>>>(p, w0, m, c->wsize, c->d_stage);
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(walkers + (size_t)w0 * c->wsize, c->d_stage, sizeof(double) * (size_t)m * c->wsize,
                         cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
  }
  return 0;
}

int mpsqmc_energy(mpsqmc_ctx *c, double *E_P) {
  if (!c || !E_P) return fail(MPSQMC_E_ARG, "null argument");
  if (c->n_cur < 1) return fail(MPSQMC_E_ARG, "no walkers");
  CK(cudaSetDevice(c->device));
  mq::Dev p = make_dev(c);
  CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(int) * mq::kNumCtr, c->stream));
  if (general_sweep(c))
    mq::energy_general_kernel<<<grid_for(c, c->n_cur), mq::kThreads, c->smem_bytes, c->stream>>>(p);
  else
    mq::energy_kernel<<<grid_for(c, c->n_cur), mq::kThreads, c->smem_bytes, c->stream>>>(p);
  CK(cudaGetLastError());
  mq::stats_kernel<<<1, 1024, 0, c->stream>>>(p, c->d_sd, c->Ndesired, c->dtau, 0, c->d_flag_pos, c->d_sw, 1,
                                              mq::kResampleThreshold);
  CK(cudaGetLastError());
  mq::StepDev sd;
  CK(cudaMemcpyAsync(&sd, c->d_sd, sizeof sd, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  int rc = check_err(c);
  if (rc) return rc;
  *E_P = sd.EP;
  return 0;
}

// ---------------------------------------------------------------------------------------------
// Learned proposal (proposal.cuh)
// ---------------------------------------------------------------------------------------------
constexpr float kPropLr = 1e-3f;  // Adam step size of the online training

// Parameters and buffers on first use: He-uniform weights (seeded mt19937), zero biases and moments.
static int prop_alloc(mpsqmc_ctx *c) {
  if (c->d_pw) return 0;
  if (c->G > mq::kMlpMaxOut) return fail(MPSQMC_E_UNSUPPORTED, "the learned proposal takes grids of up to 256 points");
  CK(cudaSetDevice(c->device));
  const long n = mq::mlp_params(c->G);
  const size_t cap = c->capacity, G = c->G, H = mq::kMlpHid;
  if (dalloc(&c->d_pw, n) || dalloc(&c->d_pm, n) || dalloc(&c->d_pv, n) || dalloc(&c->d_pg, n) ||
      dalloc(&c->d_pwb, n) || dalloc(&c->d_pt, 1) || dalloc(&c->d_pb, 1) || dalloc(&c->d_ploss, 1) ||
      dalloc(&c->d_pfeat, cap * mq::kMlpIn) || dalloc(&c->d_ptarget, cap * G) || dalloc(&c->d_ph1, cap * H) ||
      dalloc(&c->d_ph2, cap * H) || dalloc(&c->d_pz, cap * G) || dalloc(&c->d_pdz, cap * G) ||
      dalloc(&c->d_pdh2, cap * H) || dalloc(&c->d_pdh1, cap * H))
    return MPSQMC_E_CUDA;
  c->nparams = n;
  std::vector<float> w(n, 0.f);
  std::mt19937 gen(20131015u);
  const long offs[3] = {0, mq::mlp_off_w2(), mq::mlp_off_w3()};
  const int fan_in[3] = {mq::kMlpIn, mq::kMlpHid, mq::kMlpHid}, fan_out[3] = {mq::kMlpHid, mq::kMlpHid, c->G};
  for (int l = 0; l < 3; ++l) {
    std::uniform_real_distribution<float> u(-std::sqrt(6.f / fan_in[l]), std::sqrt(6.f / fan_in[l]));
    for (long e = 0; e < (long)fan_in[l] * fan_out[l]; ++e) w[offs[l] + e] = u(gen);
  }
  CK(cudaMemcpy(c->d_pw, w.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
  CK(cudaMemset(c->d_pm, 0, sizeof(float) * n));
  CK(cudaMemset(c->d_pv, 0, sizeof(float) * n));
  CK(cudaMemset(c->d_pt, 0, sizeof(int)));
  CK(cudaMemset(c->d_ploss, 0, sizeof(double)));
  mq::mlp_to_bf16_kernel<<<64, 256, 0, c->stream>>>(n, c->d_pw, c->d_pwb);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

// Forward and backward pass over the pairs in d_pfeat / d_ptarget (batch size *Bdev): mean
// KL(p || q) into d_ploss, its gradient into d_pg; with update, one Adam step on the parameters
// (and their BF16 copy).  Adds the number of launches to *n.
static int enqueue_training(mpsqmc_ctx *c, const int *Bdev, bool update, int *n) {
  const int cap = c->capacity, G = c->G, H = mq::kMlpHid, I = mq::kMlpIn;
  float *W1 = c->d_pw, *b1 = c->d_pw + mq::mlp_off_b1(), *W2 = c->d_pw + mq::mlp_off_w2(),
        *b2 = c->d_pw + mq::mlp_off_b2(), *W3 = c->d_pw + mq::mlp_off_w3(), *b3 = c->d_pw + mq::mlp_off_b3(G);
  float *gW1 = c->d_pg, *gb1 = c->d_pg + mq::mlp_off_b1(), *gW2 = c->d_pg + mq::mlp_off_w2(),
        *gb2 = c->d_pg + mq::mlp_off_b2(), *gW3 = c->d_pg + mq::mlp_off_w3(), *gb3 = c->d_pg + mq::mlp_off_b3(G);
  int k = 0;
  // M == 0 with md: M is the batch size; K == 0 with kd: K is the batch size
  auto gemm = [&](int M, int N, int K, const int *md, const int *kd, const float *A, int lda, int ta, const float *B,
                  int ldb, int tb, float *C, int ldc, const float *bias, int relu) {
    const dim3 grid((N + 63) / 64, ((md ? cap : M) + 63) / 64);
    mq::mlp_gemm_kernel<<<grid, 256, 0, c->stream>>>(M, N, K, md, kd, A, lda, ta, B, ldb, tb, C, ldc, bias, relu);
    ++k;
  };
  const int rows_blocks = std::min(1024, (cap * H + 255) / 256);
  CK(cudaMemsetAsync(c->d_ploss, 0, sizeof(double), c->stream));
  gemm(0, H, I, Bdev, nullptr, c->d_pfeat, I, 0, W1, H, 0, c->d_ph1, H, b1, 1);
  gemm(0, H, H, Bdev, nullptr, c->d_ph1, H, 0, W2, H, 0, c->d_ph2, H, b2, 1);
  gemm(0, G, H, Bdev, nullptr, c->d_ph2, H, 0, W3, G, 0, c->d_pz, G, b3, 0);
  mq::mlp_softmax_grad_kernel<<<(cap + 7) / 8, 256, 0, c->stream>>>(Bdev, G, c->d_pz, c->d_ptarget, c->d_pdz,
                                                                     c->d_ploss);
  gemm(H, G, 0, nullptr, Bdev, c->d_ph2, H, 1, c->d_pdz, G, 0, gW3, G, nullptr, 0);
  mq::mlp_colsum_kernel<<<(G + 255) / 256, 256, 0, c->stream>>>(Bdev, G, c->d_pdz, gb3);
  gemm(0, H, G, Bdev, nullptr, c->d_pdz, G, 0, W3, G, 1, c->d_pdh2, H, nullptr, 0);
  mq::mlp_relu_back_kernel<<<rows_blocks, 256, 0, c->stream>>>(Bdev, H, c->d_ph2, c->d_pdh2);
  gemm(H, H, 0, nullptr, Bdev, c->d_ph1, H, 1, c->d_pdh2, H, 0, gW2, H, nullptr, 0);
  mq::mlp_colsum_kernel<<<1, 256, 0, c->stream>>>(Bdev, H, c->d_pdh2, gb2);
  gemm(0, H, H, Bdev, nullptr, c->d_pdh2, H, 0, W2, H, 1, c->d_pdh1, H, nullptr, 0);
  mq::mlp_relu_back_kernel<<<rows_blocks, 256, 0, c->stream>>>(Bdev, H, c->d_ph1, c->d_pdh1);
  gemm(I, H, 0, nullptr, Bdev, c->d_pfeat, I, 1, c->d_pdh1, H, 0, gW1, H, nullptr, 0);
  mq::mlp_colsum_kernel<<<1, 256, 0, c->stream>>>(Bdev, H, c->d_pdh1, gb1);
  k += 6;
  if (update) {
    mq::mlp_adam_kernel<<<128, 256, 0, c->stream>>>(c->nparams, kPropLr, c->d_pt, c->d_pg, c->d_pw, c->d_pm, c->d_pv,
                                                    c->d_pwb);
    mq::mlp_count_kernel<<<1, 1, 0, c->stream>>>(c->d_pt);
    k += 2;
  }
  CK(cudaGetLastError());
  *n += k;
  return 0;
}

// Issue one timestep on c->stream (also used under stream capture): every grid has its fixed
// maximal size and every kernel reads the current walker count from device memory.
static int enqueue_legacy_step(mpsqmc_ctx *c, int *launches) {
  mq::Dev p = make_dev(c);
  const int grid = c->max_ctas;
  mq::LegacyDev lp;
  lp.nterms = c->nterms;
  lp.term_slot = c->d_term_slot;
  lp.term_pref = c->d_term_pref;
  lp.term_site = c->d_term_site;
  lp.term_op = c->d_term_op;
  lp.dtau = c->dtau;
  lp.loff = c->loff;
  lp.changed = c->d_changed;
  lp.tr = c->trace_on ? c->d_trace : nullptr;
  CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(int) * mq::kNumCtr, c->stream));
  // one uniform per walker for the term choice (MPSQMC.cpp:342), in walker order
  mq::mt_generate_kernel<<<1, 1024, 0, c->stream>>>(c->d_mt, c->d_ncur, 0, 1, c->d_uni);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(c->stream, &cap));
  const unsigned evflags = (cap == cudaStreamCaptureStatusActive) ? cudaEventRecordExternal : 0u;
  CK(cudaEventRecordWithFlags(c->ev[0], c->stream, evflags));
  mq::legacy_step_kernel<<<grid, mq::kThreads, c->smem_bytes, c->stream>>>(p, lp);
  CK(cudaEventRecordWithFlags(c->ev[1], c->stream, evflags));
  // LeftNormalize + overlap + sign of the walkers a term hit (MPSQMC.cpp:355-362)
  mq::Dev ps = p;
  ps.sel = c->d_changed;
  mq::set_overlap_kernel<<<grid, mq::kThreads, c->smem_bytes, c->stream>>>(ps);
  mq::energy_general_kernel<<<grid, mq::kThreads, c->smem_bytes, c->stream>>>(p);
  mq::stats_kernel<<<1, 1024, 0, c->stream>>>(p, c->d_sd, c->Ndesired, c->dtau, 1, c->d_flag_pos, c->d_sw, 1,
                                              mq::kResampleLegacy);
  mq::mt_generate_kernel<<<1, 1024, 0, c->stream>>>(c->d_mt, &c->d_sd->n_flag, 0, 1, c->d_ubr);
  mq::branch_kernel<<<1, 1024, 0, c->stream>>>(p, c->d_sd, c->d_flag_pos, c->d_sw, c->d_ubr, c->d_slot_new,
                                               c->d_free, c->d_copy_src, c->d_copy_dst, c->d_parent,
                                               c->capacity, c->d_ncop, 1, mq::kResampleLegacy);
  mq::copy_walkers_kernel<<<4 * c->sm_count, 256, 0, c->stream>>>(p, c->d_sd, c->d_copy_src, c->d_copy_dst);
  mq::finish_branch_kernel<<<1, 1024, 0, c->stream>>>(c->d_sd, c->d_ncur, c->d_slot_of, c->d_slot_new, c->d_err,
                                                      c->capacity);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->h_sd, c->d_sd, sizeof(mq::StepDev), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  *launches = 10;
  return 0;
}

// canon: the QR-free sweep's step that also restores the left-canonical form (LeftNormalize,
// overlap and sign of Walker::setOverlap) after the couplings.
static int enqueue_control(mpsqmc_ctx *c, const double *ext, int *launches);

// The propagation part of a step: everything before the statistics.
// The walker-batched sweep's plan, built before any stream capture: the population must share
// the slot layout's bond profile (branching keeps it), and the grid proposal samples.
static int ensure_batched(mpsqmc_ctx *c) {
  if (!tc_sweep(c)) return 0;
  if (c->proposal != MPSQMC_PROPOSAL_GRID || c->prop_train)
    return fail(MPSQMC_E_UNSUPPORTED, "the tcgen05 sweep samples the grid PDF (no learned proposal or training)");
  const int L = c->L, N = c->n_cur;
  std::vector<int> dims((size_t)std::max(1, N) * (L + 1));
  std::vector<int> slots(std::max(1, N));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(slots.data(), c->d_slot_of, sizeof(int) * N, cudaMemcpyDeviceToHost));
  std::vector<int> all((size_t)c->capacity * (L + 1));
  CK(cudaMemcpy(all.data(), c->d_wdims, sizeof(int) * all.size(), cudaMemcpyDeviceToHost));
  for (int w = 0; w < N; ++w)
    for (int k = 0; k <= L; ++k)
      if (all[(size_t)slots[w] * (L + 1) + k] != c->bW[k])
        return fail(MPSQMC_E_UNSUPPORTED, "the tcgen05 sweep needs every walker in the slot layout's bond profile");
  const bool bf16 = c->precision == MPSQMC_PRECISION_BF16_TC;
  const int passes = (c->precision == MPSQMC_PRECISION_TF32_TC || bf16) ? 1 : 3;
  const int kind = bf16 ? 16 : passes;  // what the plan was built for
  if (c->bplan && c->bplan_passes == kind && c->bplan_tiles == c->tc_tiles) return 0;
  if (c->bplan) {
    mq::bs::destroy(c->bplan);
    c->bplan = nullptr;
  }
  mq::bs::Problem pr;
  pr.L = L;
  pr.nC = c->nC;
  pr.G = c->G;
  pr.aT = c->aT;
  pr.bW = c->bW;
  pr.toff = c->toff;
  pr.woff = c->woff;
  pr.ci = c->h_ci;
  pr.cj = c->h_cj;
  pr.cq = c->h_cq;
  pr.ech_off = c->h_ech_off;
  pr.ech_slot = c->h_ech_slot;
  pr.ech_cont = c->h_ech_cont;
  pr.eopen = c->h_eopen;
  pr.ech_J = c->h_ech_J;
  pr.nslots = c->nslots;
  pr.h = c->h;
  for (int k = 0; k < 4; ++k) {
    pr.opSx[k] = c->opSx[k];
    pr.opISy[k] = c->opISy[k];
    pr.opSz[k] = c->opSz[k];
  }
  pr.trial = c->d_trial;
  pr.walkers = c->d_walkers;
  pr.wstride = c->wstride;
  pr.slot_of = c->d_slot_of;
  pr.n_cur = c->d_ncur;
  pr.weight = c->d_weight;
  pr.overlap = c->d_overlap;
  pr.energy = c->d_energy;
  pr.ov_out = c->d_ovout;
  pr.wt_out = c->d_wtout;
  pr.uni = c->d_uni;
  pr.tabU = c->d_tabU;
  pr.tabSq = c->d_tabSq;
  pr.tabVT = c->d_tabVT;
  pr.grid = c->d_grid;
  pr.err = c->d_err;
  pr.passes = passes;
  pr.bf16 = bf16;
  pr.tiles = c->tc_tiles;
  // buffers for the whole slot capacity when they fit in half the free memory, else for 1.5x the
  // target population (a step with more walkers then stops with MPSQMC_E_CAPACITY)
  size_t free_b = 0, total_b = 0;
  CK(cudaMemGetInfo(&free_b, &total_b));
  pr.capacity = c->capacity;
  if (mq::bs::bytes_needed(pr) > free_b / 2)
    pr.capacity = std::min(c->capacity, std::max(64, (3 * c->Ndesired + 1) / 2));
  if (mq::bs::bytes_needed(pr) > free_b * 9 / 10)
    return fail(MPSQMC_E_CAPACITY, "the tcgen05 sweep's work buffers do not fit in device memory");
  const int rc = mq::bs::build(pr, &c->bplan);
  if (rc) return rc;
  c->bplan_passes = kind;
  c->bplan_tiles = pr.tiles;
  c->bcap = pr.capacity;
  drop_graphs(c);
  return 0;
}

static int enqueue_propagation(mpsqmc_ctx *c, int *launches, bool canon) {
  mq::Dev p = make_dev(c);
  const int grid = c->max_ctas;
  CK(cudaMemsetAsync(c->d_ctr, 0, sizeof(int) * mq::kNumCtr, c->stream));
  mq::mt_generate_kernel<<<1, 1024, 0, c->stream>>>(c->d_mt, c->d_ncur, 0, c->nC, c->d_uni);
  const bool field = c->h != 0.0;
  int n = 7;
  if (field) {  // single-site propagator before the couplings (MPSQMC2.cpp:533)
    mq::onesite_kernel<<<grid, 256, 0, c->stream>>>(p);
    n += 1;
  }
  // external event records: they become event-record nodes under capture, so they time the
  // step kernel inside the graph (outside a capture they are plain records)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  CK(cudaStreamIsCapturing(c->stream, &cap));
  const unsigned evflags = (cap == cudaStreamCaptureStatusActive) ? cudaEventRecordExternal : 0u;
  CK(cudaEventRecordWithFlags(c->ev[0], c->stream, evflags));
  const bool gen = general_sweep(c);
  if (tc_sweep(c)) {
    int nb = 0;
    const int rc = mq::bs::enqueue(c->bplan, c->stream, c->trace_on ? c->d_trace : nullptr, &nb);
    if (rc) return rc;
    n += nb - 1;
  } else if (mixed(c)) {
    const int g = c->max_ctas_mixed;
    const size_t sm = c->smem_bytes_mixed;
    if (c->precision == MPSQMC_PRECISION_TF32) {
      if (c->nn) mq::walker_step_mixed_kernel<1, true><<<g, mq::kThreads, sm, c->stream>>>(p);
      else mq::walker_step_mixed_kernel<1, false><<<g, mq::kThreads, sm, c->stream>>>(p);
    } else {
      if (c->nn) mq::walker_step_mixed_kernel<3, true><<<g, mq::kThreads, sm, c->stream>>>(p);
      else mq::walker_step_mixed_kernel<3, false><<<g, mq::kThreads, sm, c->stream>>>(p);
    }
  } else if (gen) {
    const size_t sm = qr_free(c) ? c->smem_bytes_noqr : c->smem_bytes;
    if (!c->nn) mq::walker_step_general_kernel<false, 0><<<grid, mq::kThreads, sm, c->stream>>>(p);
    else if (qr_free(c) && !c->trace_on)
      mq::walker_step_general_kernel<true, 1, false><<<grid, mq::kThreads, sm, c->stream>>>(p);
    else if (qr_free(c)) mq::walker_step_general_kernel<true, 1><<<grid, mq::kThreads, sm, c->stream>>>(p);
    else mq::walker_step_general_kernel<true, 2><<<grid, mq::kThreads, sm, c->stream>>>(p);
  } else
    mq::walker_step_kernel<<<grid, mq::kThreads, c->smem_bytes, c->stream>>>(p);
  CK(cudaEventRecordWithFlags(c->ev[1], c->stream, evflags));
  if (field) {
    // single-site propagator after the couplings, setOverlap, and the local energy of the
    // resulting state (MPSQMC2.cpp:597-598, then 698)
    mq::onesite_kernel<<<grid, 256, 0, c->stream>>>(p);
    mq::set_overlap_kernel<<<grid, mq::kThreads, c->smem_bytes, c->stream>>>(p);
    if (gen)
      mq::energy_general_kernel<<<grid, mq::kThreads, c->smem_bytes, c->stream>>>(p);
    else
      mq::energy_kernel<<<grid, mq::kThreads, c->smem_bytes, c->stream>>>(p);
    n += 3;
  } else if (canon && qr_free(c)) {
    mq::set_overlap_kernel<<<grid, mq::kThreads, c->smem_bytes, c->stream>>>(p);
    n += 1;
  }
  if (p.prop_collect) {  // online training of the proposal on this step's pairs
    const int rc = enqueue_training(c, c->d_ncur, true, &n);
    if (rc) return rc;
  }
  CK(cudaGetLastError());
  *launches = n - 5;  // the five statistics and branching launches are enqueue_control's
  return 0;
}

static int enqueue_step(mpsqmc_ctx *c, int *launches, bool canon) {
  if (c->projector == MPSQMC_PROJECTOR_MPO_TERMS) return enqueue_legacy_step(c, launches);
  int a = 0, b = 0;
  int rc = enqueue_propagation(c, &a, canon);
  if (!rc) rc = enqueue_control(c, nullptr, &b);
  *launches = a + b;
  return rc;
}

// Statistics, population control and the step's read-back (ext: sums over all ranks, or nullptr).
static int enqueue_control(mpsqmc_ctx *c, const double *ext, int *launches) {
  mq::Dev p = make_dev(c);
  mq::stats_kernel<<<1, 1024, 0, c->stream>>>(p, c->d_sd, c->Ndesired, c->dtau, 1, c->d_flag_pos, c->d_sw,
                                              c->pc_interval, c->resample, ext);
  mq::mt_generate_kernel<<<1, 1024, 0, c->stream>>>(c->d_mt, &c->d_sd->n_flag, 0, 1, c->d_ubr);
  mq::branch_kernel<<<1, 1024, 0, c->stream>>>(p, c->d_sd, c->d_flag_pos, c->d_sw, c->d_ubr, c->d_slot_new,
                                               c->d_free, c->d_copy_src, c->d_copy_dst, c->d_parent,
                                               c->capacity, c->d_ncop, c->pc_interval, c->resample);
  mq::copy_walkers_kernel<<<4 * c->sm_count, 256, 0, c->stream>>>(p, c->d_sd, c->d_copy_src, c->d_copy_dst);
  mq::finish_branch_kernel<<<1, 1024, 0, c->stream>>>(c->d_sd, c->d_ncur, c->d_slot_of, c->d_slot_new, c->d_err,
                                                      c->capacity);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(c->h_sd, c->d_sd, sizeof(mq::StepDev), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_err, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  *launches = 5;
  return 0;
}

static int build_graph(mpsqmc_ctx *c, bool canon) {
  cudaGraphExec_t &ge = canon ? c->graph_exec_canon : c->graph_exec;
  if (ge) {
    cudaGraphExecDestroy(ge);
    ge = nullptr;
  }
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(c, &c->graph_launches[canon ? 1 : 0], canon);
  cudaError_t e = cudaStreamEndCapture(c->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return fail(MPSQMC_E_CUDA, std::string("stream capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&ge, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(MPSQMC_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  c->graph_trace = c->trace_on;
  return 0;
}

// Host bookkeeping after a step's read-back: errors, random-stream position, population size.
static int finish_step(mpsqmc_ctx *c, int N, int step, bool canon, const mq::StepDev &sd, int err,
                       mpsqmc_step_stats *o) {
  if (err & mq::bs::kErrTimeout) return fail(MPSQMC_E_CUDA, "a tcgen05 pipeline wait timed out");
  if (err & mq::kErrNumeric) return fail(MPSQMC_E_NUMERIC, "non-finite weight, overlap or energy");
  if (err & mq::kErrCapacity) return fail(MPSQMC_E_CAPACITY, "population control exceeded the walker capacity");
  const int per_walker = (c->projector == MPSQMC_PROJECTOR_MPO_TERMS) ? 1 : c->nC;
  const unsigned long long dr = (unsigned long long)N * per_walker + (unsigned long long)sd.n_flag;
  c->draws += dr;
  c->last_n_before = N;
  c->last_n_after = sd.n_new;
  c->n_cur = sd.n_new;
  c->gauge_dirty = qr_free(c) && !canon && c->h == 0.0;
  if (o) {
    o->step = step;
    o->n_walkers = N;
    o->n_after = sd.n_new;
    o->sum_weight = sd.sumw;
    o->avg_weight = N > 0 ? sd.sumw / N : 0.0;
    o->E_P = sd.EP;
    o->E_T = sd.ET;
    o->omega = sd.omega;
    o->scaling = sd.scaling;
    o->draws = dr;
  }
  return 0;
}

int mpsqmc_walk(mpsqmc_ctx *c, int nsteps, mpsqmc_step_stats *stats) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  if (nsteps < 0) return fail(MPSQMC_E_ARG, "negative step count");
  if (c->n_cur < 1) return fail(MPSQMC_E_ARG, "no walkers");
  CK(cudaSetDevice(c->device));
  if (c->trace_on && !c->d_trace) {
    if (dalloc(&c->d_trace, (size_t)c->capacity * c->nC * mq::kTraceStride)) return MPSQMC_E_CUDA;
  }
  if (c->trace_on && mixed(c) && !tc_sweep(c))
    return fail(MPSQMC_E_UNSUPPORTED, "the per-coupling trace is recorded by the FP64 and tcgen05 sweeps only");
  {
    const int rc = ensure_batched(c);
    if (rc) return rc;
  }
  if (c->use_graph && c->graph_trace != c->trace_on) drop_graphs(c);
  int per_step = 0;
  double kernel_ms = 0.0;
  int launches = 0;
  CK(cudaEventRecord(c->ev[2], c->stream));
  for (int s = 0; s < nsteps; ++s) {
    const int N = c->n_cur;
    const int step = ++c->step_count;
    const bool canon = qr_free(c) && step % canon_every(c) == 0;
    if (c->use_graph) {
      if (!(canon ? c->graph_exec_canon : c->graph_exec)) {
        int rc = build_graph(c, canon);
        if (rc) return rc;
      }
      CK(cudaGraphLaunch(canon ? c->graph_exec_canon : c->graph_exec, c->stream));
      per_step = c->graph_launches[canon ? 1 : 0];
    } else {
      int rc = enqueue_step(c, &per_step, canon);
      if (rc) return rc;
    }
    launches += per_step;
    CK(cudaStreamSynchronize(c->stream));
    const mq::StepDev sd = *c->h_sd;
    const int err = *c->h_err;
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]));
    kernel_ms += ms;
    const int rc = finish_step(c, N, step, canon, sd, err, stats ? &stats[s] : nullptr);
    if (rc) return rc;
    if (sd.n_new == 0) return fail(MPSQMC_E_EXTINCT, "population control removed every walker");
  }
  CK(cudaEventRecord(c->ev[3], c->stream));
  CK(cudaEventSynchronize(c->ev[3]));
  float tot = 0.f;
  CK(cudaEventElapsedTime(&tot, c->ev[2], c->ev[3]));
  c->last_kernel_ms = kernel_ms;
  c->last_total_ms = tot;
  c->last_launches = launches;
  return 0;
}

// Autotuning: choices measured once per problem shape (L, trial and walker bond dims, coupling
// structure, projector, sweep family) and remembered for every later context of the same shape in
// this process.
namespace {
struct Tuned {
  int sweep, workspace;
  mq::bs::Tiles tiles;
};
std::mutex g_tune_mutex;
std::map<std::string, Tuned> g_tuned;  // shape -> choice

std::string tune_key(const mpsqmc_ctx *c) {
  std::ostringstream k;
  k << c->L << '|' << c->nC << '|' << c->nn << '|' << c->projector << '|' << (c->h != 0.0) << '|';
  for (int v : c->aT) k << v << ',';
  k << '|';
  for (int v : c->bW) k << v << ',';
  k << '|'
    << (tc_sweep(c) ? (c->precision == MPSQMC_PRECISION_TF32_TC   ? "tc1"
                       : c->precision == MPSQMC_PRECISION_BF16_TC ? "bf16"
                                                                  : "tc3")
                    : "cta");
  return k.str();
}

int apply_tuned(mpsqmc_ctx *c, const Tuned &t) {
  int rc = mpsqmc_set_option(c, MPSQMC_OPT_SWEEP, t.sweep);
  if (!rc) rc = mpsqmc_set_option(c, MPSQMC_OPT_WORKSPACE, t.workspace);
  if (!rc) rc = mpsqmc_set_option(c, MPSQMC_OPT_TC_STACK_TN, t.tiles.stack_tn);
  if (!rc) rc = mpsqmc_set_option(c, MPSQMC_OPT_TC_WIDE_TN, t.tiles.wide_tn);
  if (!rc) rc = mpsqmc_set_option(c, MPSQMC_OPT_TC_STAGES, t.tiles.max_stages);
  if (!rc) rc = mpsqmc_set_option(c, MPSQMC_OPT_TC_SPLIT_OUT, t.tiles.split_out);
  if (!rc) rc = mpsqmc_set_option(c, MPSQMC_OPT_TC_KC, t.tiles.kc_trial);
  return rc;
}
}  // namespace

int mpsqmc_autotune(mpsqmc_ctx *c, int steps, int *best_sweep, int *best_workspace) {
  if (!c || steps < 1) return fail(MPSQMC_E_ARG, "bad arguments");
  if (c->n_cur < 1) return fail(MPSQMC_E_ARG, "no walkers");
  CK(cudaSetDevice(c->device));
  const std::string key = tune_key(c);
  const bool tc = tc_sweep(c);
  {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      const int rc = apply_tuned(c, it->second);
      if (best_sweep) *best_sweep = it->second.sweep;
      if (best_workspace) *best_workspace = it->second.workspace;
      return rc;
    }
  }
  // measure on the first k walkers, with the population state saved and restored around every
  // trial: two waves of one CTA per SM for the per-walker sweeps; for the tcgen05 sweep, whose
  // tile counts grow with the population, up to 1024 walkers
  const int N = c->n_cur, k = std::min(N, tc ? 1024 : 2 * c->sm_count), cap = c->capacity, L = c->L;
  std::vector<int> slots(N), h_free(cap), wd((size_t)cap * (L + 1));
  std::vector<long> wf((size_t)cap * L);
  std::vector<double> wt(cap), ov(cap), eh(cap);
  mq::MtState mt;
  mq::StepDev sd;
  CK(cudaMemcpy(slots.data(), c->d_slot_of, sizeof(int) * N, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(h_free.data(), c->d_free, sizeof(int) * cap, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(wd.data(), c->d_wdims, sizeof(int) * wd.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(wf.data(), c->d_wofs, sizeof(long) * wf.size(), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(wt.data(), c->d_weight, sizeof(double) * cap, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(ov.data(), c->d_overlap, sizeof(double) * cap, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(eh.data(), c->d_ehist, sizeof(double) * cap, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&mt, c->d_mt, sizeof mt, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(&sd, c->d_sd, sizeof sd, cudaMemcpyDeviceToHost));
  double *snap = nullptr;
  if (dalloc(&snap, (size_t)k * c->wstride)) return MPSQMC_E_CUDA;
  for (int w = 0; w < k; ++w)
    CK(cudaMemcpyAsync(snap + (size_t)w * c->wstride, c->d_walkers + (size_t)slots[w] * c->wstride,
                       sizeof(double) * c->wstride, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const Tuned keep = {c->sweep, c->global_work ? MPSQMC_WORKSPACE_GLOBAL : MPSQMC_WORKSPACE_AUTO, c->tc_tiles};
  const int keep_nd = c->Ndesired, keep_step = c->step_count;
  const unsigned long long keep_draws = c->draws;
  const bool keep_trace = c->trace_on;
  const bool keep_dirty = c->gauge_dirty;
  auto restore = [&](int n_walkers) -> int {
    for (int w = 0; w < k; ++w)
      CK(cudaMemcpyAsync(c->d_walkers + (size_t)slots[w] * c->wstride, snap + (size_t)w * c->wstride,
                         sizeof(double) * c->wstride, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_slot_of, slots.data(), sizeof(int) * N, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_free, h_free.data(), sizeof(int) * cap, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_wdims, wd.data(), sizeof(int) * wd.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_wofs, wf.data(), sizeof(long) * wf.size(), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_weight, wt.data(), sizeof(double) * cap, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_overlap, ov.data(), sizeof(double) * cap, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_ehist, eh.data(), sizeof(double) * cap, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_mt, &mt, sizeof mt, cudaMemcpyHostToDevice, c->stream));
    mq::StepDev s2 = sd;
    s2.n_cur = n_walkers;
    CK(cudaMemcpyAsync(c->d_sd, &s2, sizeof s2, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->d_ncur, &n_walkers, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->n_cur = n_walkers;
    c->step_count = keep_step;
    c->draws = keep_draws;
    return 0;
  };
  c->trace_on = false;
  c->Ndesired = k;  // population control sized for the measured subset
  // one trial: the candidate's options, a warm-up step (graph capture, plan rebuild), `steps`
  // timed steps; returns the device time per walker-step
  auto trial = [&](const Tuned &cd, double *per) -> int {
    int rc = apply_tuned(c, cd);
    if (!rc) rc = restore(k);
    if (!rc) rc = mpsqmc_walk(c, 1, nullptr);
    if (!rc) rc = restore(k);
    if (!rc) rc = mpsqmc_walk(c, steps, nullptr);
    if (!rc) *per = c->last_kernel_ms / ((double)k * steps);
    return rc;
  };
  double best = 1e300;
  Tuned choice = keep;
  int rc = 0;
  if (!tc) {
    // every sweep that takes these couplings, both work-buffer placements (one when the buffers
    // do not fit on chip)
    const bool fits = sizeof(double) * (size_t)c->all_doubles <= c->smem_optin;
    for (int sw : {MPSQMC_SWEEP_GENERAL, MPSQMC_SWEEP_NEAREST}) {
      if (sw == MPSQMC_SWEEP_NEAREST && (!c->nn || c->projector != MPSQMC_PROJECTOR_TROTTER)) continue;
      for (int ws : {MPSQMC_WORKSPACE_AUTO, MPSQMC_WORKSPACE_GLOBAL}) {
        if (ws == MPSQMC_WORKSPACE_GLOBAL && !fits) continue;
        const Tuned cd = {sw, ws, keep.tiles};
        double per = 0.0;
        if ((rc = trial(cd, &per))) break;
        if (per < best) best = per, choice = cd;
      }
      if (rc) break;
    }
  } else {
    // tcgen05 sweep: coordinate search over the tile choices, one at a time from the defaults
    Tuned cur = {keep.sweep, keep.workspace, mq::bs::Tiles()};
    if (!(rc = trial(cur, &best))) choice = cur;
    // axes: 0 split right factors, 1 k-values per stage of the trial products, 2 stacked tile
    // width, 3 the walker products' tile width, 4 ring depth cap
    for (int axis = 0; axis < 5 && !rc; ++axis) {
      if (axis == 0 && c->precision != MPSQMC_PRECISION_TF32X3_TC) continue;  // one pass: nothing to split
      if (axis == 1 && c->precision == MPSQMC_PRECISION_BF16_TC) continue;    // BF16 stages take 32 values
      const std::vector<int> vals = axis == 0   ? std::vector<int>{mq::bs::kSplitX4, mq::bs::kSplitXch, mq::bs::kSplitY,
                                                                 mq::bs::kSplitX, mq::bs::kSplitQ}
                                    : axis == 1 ? std::vector<int>{16}
                                    : axis == 4 ? std::vector<int>{4, 2}
                                                : std::vector<int>{128, 64};
      for (int v : vals) {
        Tuned cd = choice;
        if (axis == 0) cd.tiles.split_out |= v;  // one class of right factors more, stored split
        else (axis == 1 ? cd.tiles.kc_trial : axis == 2 ? cd.tiles.stack_tn : axis == 3 ? cd.tiles.wide_tn
                                                                                      : cd.tiles.max_stages) = v;
        double per = 0.0;
        if ((rc = trial(cd, &per))) break;
        if (per < best) best = per, choice = cd;
      }
    }
  }
  c->Ndesired = keep_nd;
  c->trace_on = keep_trace;
  const int rr = restore(N);
  c->gauge_dirty = keep_dirty;
  cudaFree(snap);
  if (rc) {
    apply_tuned(c, keep);
    return rc;
  }
  if (rr) return rr;
  drop_graphs(c);  // captured with the subset's population size
  if (tc && c->bplan) {
    // the trials' plans were sized for the measured subset: the next walk builds one for the
    // population's own target
    mq::bs::destroy(c->bplan);
    c->bplan = nullptr;
  }
  rc = apply_tuned(c, choice);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lk(g_tune_mutex);
    g_tuned[key] = choice;
  }
  if (best_sweep) *best_sweep = choice.sweep;
  if (best_workspace) *best_workspace = choice.workspace;
  return 0;
}

int mpsqmc_set_step(mpsqmc_ctx *c, int completed_steps) {
  if (!c || completed_steps < 0) return fail(MPSQMC_E_ARG, "bad arguments");
  CK(cudaSetDevice(c->device));
  c->step_count = completed_steps;
  CK(cudaMemcpy((char *)c->d_sd + offsetof(mq::StepDev, step), &completed_steps, sizeof(int),
                cudaMemcpyHostToDevice));
  return 0;
}

int mpsqmc_last_step_walkers(mpsqmc_ctx *c, int *n_before, double *weight, double *overlap,
                             double *energy, int *n_after, int *parent) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  CK(cudaSetDevice(c->device));
  const int nb = c->last_n_before, na = c->last_n_after;
  if (n_before) *n_before = nb;
  if (n_after) *n_after = na;
  if (weight && nb) CK(cudaMemcpy(weight, c->d_wtout, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  if (overlap && nb) CK(cudaMemcpy(overlap, c->d_ovout, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  if (energy && nb) CK(cudaMemcpy(energy, c->d_energy, sizeof(double) * nb, cudaMemcpyDeviceToHost));
  if (parent && na) CK(cudaMemcpy(parent, c->d_parent, sizeof(int) * na, cudaMemcpyDeviceToHost));
  return 0;
}

int mpsqmc_set_trace(mpsqmc_ctx *c, int enable) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  c->trace_on = enable != 0;
  return 0;
}

int mpsqmc_get_trace(mpsqmc_ctx *c, double *trace, int *n_walkers) {
  if (!c || !trace) return fail(MPSQMC_E_ARG, "null argument");
  if (!c->d_trace) return fail(MPSQMC_E_ARG, "trace was not enabled for a step");
  CK(cudaSetDevice(c->device));
  const int nb = c->last_n_before;
  if (n_walkers) *n_walkers = nb;
  CK(cudaMemcpy(trace, c->d_trace, sizeof(double) * (size_t)nb * c->nC * mq::kTraceStride,
                cudaMemcpyDeviceToHost));
  return 0;
}

int mpsqmc_last_timing(mpsqmc_ctx *c, double *step_kernel_ms, double *total_ms, int *kernel_launches) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  if (step_kernel_ms) *step_kernel_ms = c->last_kernel_ms;
  if (total_ms) *total_ms = c->last_total_ms;
  if (kernel_launches) *kernel_launches = c->last_launches;
  return 0;
}

int mpsqmc_set_option(mpsqmc_ctx *c, int option, long value) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  switch (option) {
    case MPSQMC_OPT_SWEEP:
      if (value != MPSQMC_SWEEP_AUTO && value != MPSQMC_SWEEP_NEAREST && value != MPSQMC_SWEEP_GENERAL)
        return fail(MPSQMC_E_ARG, "unknown sweep");
      if (value == MPSQMC_SWEEP_NEAREST && !c->nn)
        return fail(MPSQMC_E_UNSUPPORTED, "the nearest-neighbour sweep needs every coupling to be (i, i+1)");
      c->sweep = (int)value;
      break;
    case MPSQMC_OPT_WORKSPACE: {
      if (value != MPSQMC_WORKSPACE_AUTO && value != MPSQMC_WORKSPACE_GLOBAL)
        return fail(MPSQMC_E_ARG, "unknown workspace placement");
      const int rc = relayout(c, value == MPSQMC_WORKSPACE_GLOBAL);
      if (rc) return rc;
      c->workspace = (int)value;
      break;
    }
    case MPSQMC_OPT_PROJECTOR:
      if (value != MPSQMC_PROJECTOR_TROTTER && value != MPSQMC_PROJECTOR_MPO_TERMS)
        return fail(MPSQMC_E_ARG, "unknown projector");
      c->projector = (int)value;
      break;
    case MPSQMC_OPT_POPCONTROL_INTERVAL:
      if (value < 1 || value > (1L << 30)) return fail(MPSQMC_E_ARG, "population-control interval must be >= 1");
      c->pc_interval = (int)value;
      break;
    case MPSQMC_OPT_RESAMPLING:
      if (value != MPSQMC_RESAMPLE_THRESHOLD && value != MPSQMC_RESAMPLE_COMB)
        return fail(MPSQMC_E_ARG, "unknown resampling");
      c->resample = (int)value;
      break;
    case MPSQMC_OPT_CANONICAL_INTERVAL:
      if (value < 0 || value > (1L << 30)) return fail(MPSQMC_E_ARG, "canonical interval must be >= 0");
      c->canon_interval = (int)value;
      break;
    case MPSQMC_OPT_PRECISION:
      if (value < MPSQMC_PRECISION_FP64 || value > MPSQMC_PRECISION_BF16_TC) return fail(MPSQMC_E_ARG, "unknown precision");
      c->precision = (int)value;
      if (c->bplan && !tc_sweep(c)) {
        CK(cudaStreamSynchronize(c->stream));
        mq::bs::destroy(c->bplan);
        c->bplan = nullptr;
      }
      break;
    case MPSQMC_OPT_PROPOSAL:
      if (value != MPSQMC_PROPOSAL_GRID && value != MPSQMC_PROPOSAL_LEARNED) return fail(MPSQMC_E_ARG, "unknown proposal");
      if (value == MPSQMC_PROPOSAL_LEARNED) {
        const int rc = prop_alloc(c);
        if (rc) return rc;
      }
      c->proposal = (int)value;
      {
        const int rc = relayout(c, c->workspace == MPSQMC_WORKSPACE_GLOBAL);
        if (rc) return rc;
      }
      break;
    case MPSQMC_OPT_PROPOSAL_TRAINING:
      if (value != 0 && value != 1) return fail(MPSQMC_E_ARG, "proposal training is 0 or 1");
      if (value) {
        const int rc = prop_alloc(c);
        if (rc) return rc;
      }
      c->prop_train = value != 0;
      {
        const int rc = relayout(c, c->workspace == MPSQMC_WORKSPACE_GLOBAL);
        if (rc) return rc;
      }
      break;
    case MPSQMC_OPT_PROPOSAL_MIX:
      if (value < 0 || value > 1000) return fail(MPSQMC_E_ARG, "proposal mixture is 0..1000 thousandths");
      c->prop_mix = (int)value;
      break;
    case MPSQMC_OPT_TC_STACK_TN:
    case MPSQMC_OPT_TC_WIDE_TN:
      if (value != 64 && value != 128 && value != 256) return fail(MPSQMC_E_ARG, "tile width is 64, 128 or 256");
      (option == MPSQMC_OPT_TC_STACK_TN ? c->tc_tiles.stack_tn : c->tc_tiles.wide_tn) = (int)value;
      break;
    case MPSQMC_OPT_TC_STAGES:
      if (value < 2 || value > 8) return fail(MPSQMC_E_ARG, "load-ring stages are 2..8");
      c->tc_tiles.max_stages = (int)value;
      break;
    case MPSQMC_OPT_TC_SPLIT_OUT:
      if (value < 0 || value > mq::bs::kSplitAll) return fail(MPSQMC_E_ARG, "split outputs are a mask 0..31");
      c->tc_tiles.split_out = (int)value;
      break;
    case MPSQMC_OPT_TC_KC:
      if (value != 16 && value != 32) return fail(MPSQMC_E_ARG, "k-values per stage are 16 or 32");
      c->tc_tiles.kc_trial = (int)value;
      break;
    default:
      return fail(MPSQMC_E_ARG, "unknown option");
  }
  drop_graphs(c);  // the captured steps no longer match
  return 0;
}

int mpsqmc_get_option(mpsqmc_ctx *c, int option, long *value) {
  if (!c || !value) return fail(MPSQMC_E_ARG, "null argument");
  switch (option) {
    case MPSQMC_OPT_SWEEP:
      *value = c->sweep;
      return 0;
    case MPSQMC_OPT_WORKSPACE:
      *value = c->global_work ? MPSQMC_WORKSPACE_GLOBAL : MPSQMC_WORKSPACE_AUTO;
      return 0;
    case MPSQMC_OPT_POPCONTROL_INTERVAL:
      *value = c->pc_interval;
      return 0;
    case MPSQMC_OPT_RESAMPLING:
      *value = c->resample;
      return 0;
    case MPSQMC_OPT_PROJECTOR:
      *value = c->projector;
      return 0;
    case MPSQMC_OPT_CANONICAL_INTERVAL:
      *value = c->canon_interval;
      return 0;
    case MPSQMC_OPT_PRECISION:
      *value = c->precision;
      return 0;
    case MPSQMC_OPT_PROPOSAL:
      *value = c->proposal;
      return 0;
    case MPSQMC_OPT_PROPOSAL_TRAINING:
      *value = c->prop_train ? 1 : 0;
      return 0;
    case MPSQMC_OPT_PROPOSAL_MIX:
      *value = c->prop_mix;
      return 0;
    case MPSQMC_OPT_TC_STACK_TN:
      *value = c->tc_tiles.stack_tn;
      return 0;
    case MPSQMC_OPT_TC_WIDE_TN:
      *value = c->tc_tiles.wide_tn;
      return 0;
    case MPSQMC_OPT_TC_STAGES:
      *value = c->tc_tiles.max_stages;
      return 0;
    case MPSQMC_OPT_TC_SPLIT_OUT:
      *value = c->tc_tiles.split_out;
      return 0;
    case MPSQMC_OPT_TC_KC:
      *value = c->tc_tiles.kc_trial;
      return 0;
    default:
      return fail(MPSQMC_E_ARG, "unknown option");
  }
}

// ---------------------------------------------------------------------------------------------
// Walks split over ranks (population.cuh)
// ---------------------------------------------------------------------------------------------
int mpsqmc_step_propagate(mpsqmc_ctx *c, double local_sums[5]) {
  if (!c || !local_sums) return fail(MPSQMC_E_ARG, "null argument");
  if (c->projector != MPSQMC_PROJECTOR_TROTTER)
    return fail(MPSQMC_E_UNSUPPORTED, "split steps run the Trotter projector");
  if (c->split_pending) return fail(MPSQMC_E_ARG, "mpsqmc_step_control is due first");
  if (c->trace_on) return fail(MPSQMC_E_UNSUPPORTED, "the per-coupling trace is recorded by mpsqmc_walk only");
  CK(cudaSetDevice(c->device));
  if (!c->d_sums && dalloc(&c->d_sums, 16)) return MPSQMC_E_CUDA;
  {
    const int rc = ensure_batched(c);
    if (rc) return rc;
  }
  const int step = ++c->step_count;
  c->split_canon = qr_free(c) && step % canon_every(c) == 0;
  int n = 0;
  int rc = enqueue_propagation(c, &n, c->split_canon);
  if (rc) return rc;
  mq::local_sums_kernel<<<1, 1024, 0, c->stream>>>(make_dev(c), c->d_sd, c->d_sums);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(local_sums, c->d_sums, sizeof(double) * mq::kNumSums, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->split_pending = true;
  c->split_launches = n + 1;
  return check_err(c);
}

int mpsqmc_step_control(mpsqmc_ctx *c, const double global_sums[5], long ndesired_total, mpsqmc_step_stats *stats) {
  if (!c || !global_sums) return fail(MPSQMC_E_ARG, "null argument");
  if (!c->split_pending) return fail(MPSQMC_E_ARG, "mpsqmc_step_propagate is due first");
  if (ndesired_total < 1 || !(global_sums[0] > 0.0) || !(global_sums[4] >= 1.0))
    return fail(MPSQMC_E_ARG, "global sums need a positive weight sum, walker count and target");
  CK(cudaSetDevice(c->device));
  double ext[6];
  std::copy(global_sums, global_sums + 5, ext);
  ext[5] = (double)ndesired_total;
  CK(cudaMemcpyAsync(c->d_sums + 8, ext, sizeof ext, cudaMemcpyHostToDevice, c->stream));
  const int N = c->n_cur;
  int n = 0;
  int rc = enqueue_control(c, c->d_sums + 8, &n);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->stream));
  c->split_pending = false;
  c->last_launches = c->split_launches + n;
  return finish_step(c, N, c->step_count, c->split_canon, *c->h_sd, *c->h_err, stats);
}

long mpsqmc_record_size(const mpsqmc_ctx *c) { return c ? mq::record_doubles(c->L, c->wsize) : -1; }

int mpsqmc_export_walkers(mpsqmc_ctx *c, int k, double *records) {
  if (!c || (!records && k > 0)) return fail(MPSQMC_E_ARG, "null argument");
  if (k < 0 || k > c->n_cur) return fail(MPSQMC_E_ARG, "export count outside [0, walkers]");
  if (c->split_pending) return fail(MPSQMC_E_ARG, "mpsqmc_step_control is due first");
  if (k == 0) return 0;
  int rc = restore_canonical(c);
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  mq::Dev p = make_dev(c);
  mq::export_walkers_kernel<<<std::min(k, 4 * c->sm_count), 256, 0, c->stream>>>(p, c->d_sd, k,
                                                                                  mq::record_doubles(c->L, c->wsize),
                                                                                  records);
  mq::population_count_kernel<<<1, 256, 0, c->stream>>>(c->d_sd, c->d_ncur, c->d_slot_of, c->d_free, -k);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  c->n_cur -= k;
  return 0;
}

int mpsqmc_import_walkers(mpsqmc_ctx *c, int k, const double *records) {
  if (!c || (!records && k > 0)) return fail(MPSQMC_E_ARG, "null argument");
  if (k < 0 || c->n_cur + k > c->capacity) return fail(MPSQMC_E_CAPACITY, "import beyond the walker capacity");
  if (c->split_pending) return fail(MPSQMC_E_ARG, "mpsqmc_step_control is due first");
  if (k == 0) return 0;
  CK(cudaSetDevice(c->device));
  mq::Dev p = make_dev(c);
  mq::import_walkers_kernel<<<std::min(k, 4 * c->sm_count), 256, 0, c->stream>>>(
      p, c->d_sd, c->d_free, c->d_slot_of, k, mq::record_doubles(c->L, c->wsize), records);
  mq::population_count_kernel<<<1, 256, 0, c->stream>>>(c->d_sd, c->d_ncur, c->d_slot_of, c->d_free, k);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  c->n_cur += k;
  return 0;
}

int mpsqmc_proposal_params(mpsqmc_ctx *c, float *out, const float *in, long *n_params) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  int rc = prop_alloc(c);
  if (rc) return rc;
  if (n_params) *n_params = c->nparams;
  CK(cudaSetDevice(c->device));
  if (out) CK(cudaMemcpy(out, c->d_pw, sizeof(float) * c->nparams, cudaMemcpyDeviceToHost));
  if (in) {
    CK(cudaMemcpy(c->d_pw, in, sizeof(float) * c->nparams, cudaMemcpyHostToDevice));
    CK(cudaMemset(c->d_pm, 0, sizeof(float) * c->nparams));
    CK(cudaMemset(c->d_pv, 0, sizeof(float) * c->nparams));
    CK(cudaMemset(c->d_pt, 0, sizeof(int)));
    mq::mlp_to_bf16_kernel<<<64, 256, 0, c->stream>>>(c->nparams, c->d_pw, c->d_pwb);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->stream));
  }
  return 0;
}

int mpsqmc_proposal_loss_grad(mpsqmc_ctx *c, int B, const float *features, const float *targets, double *loss,
                              float *grad) {
  if (!c || !features || !targets) return fail(MPSQMC_E_ARG, "null argument");
  if (B < 1 || B > c->capacity) return fail(MPSQMC_E_ARG, "batch size outside [1, capacity]");
  int rc = prop_alloc(c);
  if (rc) return rc;
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(c->d_pfeat, features, sizeof(float) * (size_t)B * mq::kMlpIn, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_ptarget, targets, sizeof(float) * (size_t)B * c->G, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_pb, &B, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  int n = 0;
  rc = enqueue_training(c, c->d_pb, false, &n);
  if (rc) return rc;
  if (loss) CK(cudaMemcpyAsync(loss, c->d_ploss, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  if (grad) CK(cudaMemcpyAsync(grad, c->d_pg, sizeof(float) * c->nparams, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return 0;
}

int mpsqmc_proposal_stats(mpsqmc_ctx *c, double *last_loss, int *updates) {
  if (!c) return fail(MPSQMC_E_ARG, "null context");
  if (!c->d_pw) {
    if (last_loss) *last_loss = 0.0;
    if (updates) *updates = 0;
    return 0;
  }
  CK(cudaSetDevice(c->device));
  if (last_loss) CK(cudaMemcpy(last_loss, c->d_ploss, sizeof(double), cudaMemcpyDeviceToHost));
  if (updates) CK(cudaMemcpy(updates, c->d_pt, sizeof(int), cudaMemcpyDeviceToHost));
  return 0;
}

}  // extern "C"
