/*
 * mpsqmc_gpu.h -- C ABI of the B200 walker-propagation engine (libmpsqmc_b200.so).
 *
 * Drop-in boundary for the reference's MPSQMC2 hot path.  The reference keeps the walk inside
 * C++ objects (MPSQMC2.h:13-166, Walker.h:13-52, MPSstate.h:19-102, TrotterHeisenberg.h:16-40);
 * these entry points are what those objects (or any FFI: ctypes, cgo, JNI) bind to.  Every call
 * returns an int status (0 = success, negative = MPSQMC_E_*); nothing throws, nothing aborts.
 * All arrays are plain host pointers; the library owns every device allocation.
 *
 * Data conventions (identical to the reference):
 *   - MPS bond dims dims[0..L], dims[0] = dims[L] = 1 (MPSstate.cpp:20-28);
 *   - site s stores dims[s]*dims[s+1]*d doubles, element [r + dims[s]*(c + dims[s+1]*sigma)]
 *     (MPStensor.cpp:91-96); sites are concatenated in order;
 *   - two-site propagator SVD tables per distinct coupling J: S[k], U[i + d*(j + d*k)],
 *     VT[k + d*d*(i + d*j)] (TrotterHeisenberg.cpp:345-431);
 *   - grid points grid[i + d*d*p] (GridGenerator.cpp:40-44);
 *   - couplings (ci[c] < cj[c], J_c != 0) in the order MPSQMC2.cpp:286-299 builds them.
 */
#ifndef MPSQMC_GPU_H
#define MPSQMC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define MPSQMC_OK 0
#define MPSQMC_E_ARG (-1)         /* invalid argument or size mismatch */
#define MPSQMC_E_CUDA (-2)        /* a CUDA call failed (message: mpsqmc_last_error) */
#define MPSQMC_E_NODEVICE (-3)    /* no CUDA device: there is no CPU fallback */
#define MPSQMC_E_UNSUPPORTED (-4) /* configuration outside what the kernels implement */
#define MPSQMC_E_CAPACITY (-5)    /* branching would exceed the walker capacity */
#define MPSQMC_E_NUMERIC (-6)     /* NaN/Inf or non-positive weight sum detected */
#define MPSQMC_E_EXTINCT (-7)     /* population control left no walker */

typedef struct mpsqmc_ctx mpsqmc_ctx;

/* Everything MPSQMC2's constructor (MPSQMC2.cpp:68-103) derives from its arguments. */
typedef struct {
  int L;                 /* chain length (HeisenbergMPO::gLength) */
  int d;                 /* local dimension; the kernels implement d = 2 */
  int nC;                /* number of couplings */
  const int *ci;         /* first site of each coupling */
  const int *cj;         /* second site of each coupling (any cj > ci) */
  const double *cJ;      /* coupling strength of each coupling */
  double h;              /* magnetic field (HeisenbergMPO::gField) */
  double dtau;           /* imaginary time step */
  const int *trial_dims; /* trial bond dims [L+1] (left-normalized trial, MPSQMC2.cpp:239) */
  const double *trial;   /* trial tensors */
  int nJ;                /* number of distinct couplings */
  const double *Jvals;   /* [nJ] */
  const double *U;       /* [nJ][d^4] */
  const double *S;       /* [nJ][d^2] */
  const double *VT;      /* [nJ][d^4] */
  int G;                 /* grid points */
  const double *grid;    /* [G][d^2] */
  int Ndesired;          /* totalNDesiredWalkers */
  int capacity;          /* walker slots (reference: max(1000, 3*Nwalkers), MPSQMC2.cpp:41) */
  const int *walker_dims;/* common walker bond dims [L+1] */
  int device;            /* CUDA device ordinal */
} mpsqmc_config;

/* Per-step statistics of Walk (MPSQMC2.cpp:465-498). */
typedef struct {
  int step;              /* step number (1-based, continues across calls) */
  int n_walkers;         /* totalNCurrentWalkers during the step (before branching) */
  int n_after;           /* walkers after population control */
  double sum_weight;     /* sum of walker weights after propagation */
  double avg_weight;     /* sum_weight / n_walkers */
  double E_P;            /* projected (mixed) energy */
  double E_T;            /* target energy log(scaling)/dtau */
  double omega;          /* fluctuation metric */
  double scaling;        /* Ndesired / sum_weight */
  uint64_t draws;        /* uniforms consumed by this step */
} mpsqmc_step_stats;

/* Creation copies every input to the device.  Replaces MPSQMC2::MPSQMC2 + SetupTrial
 * (MPSQMC2.cpp:68-103, 219-332) minus the trial-term copies, which the kernels do not need. */
int mpsqmc_create(const mpsqmc_config *cfg, mpsqmc_ctx **out);
int mpsqmc_destroy(mpsqmc_ctx *ctx);

/* Message of the last failure in this thread (static storage, never NULL). */
const char *mpsqmc_last_error(void);

/* Library version string. */
const char *mpsqmc_version(void);

/* Number of doubles in one walker (sum over sites of dims[s]*dims[s+1]*d). */
long mpsqmc_walker_size(const mpsqmc_ctx *ctx);

/* Upload N walkers in logical order (walkers: [N][walker_size]) with their weight, overlap and
 * energy history (Walker.h:224-234).  Replaces SetupWalkers (MPSQMC2.cpp:381-441) and
 * Walker(Walker*) copies.  When normalize != 0 each walker is first brought into the state
 * Walker::setOverlap leaves it in (Walker.cpp:54-66): left-normalized, overlap recomputed,
 * sign fixed; the given overlaps are then ignored. */
int mpsqmc_set_walkers(mpsqmc_ctx *ctx, int N, const double *walkers, const double *weights,
                       const double *overlaps, const double *ehist, int normalize);

/* Download the current population in logical order; *N receives the count.  Any pointer may
 * be NULL.  walkers must hold capacity*walker_size doubles (or the current N); walker w occupies
 * walker_size doubles from w*walker_size, its own tensors first (see mpsqmc_get_walker_dims). */
int mpsqmc_get_walkers(mpsqmc_ctx *ctx, int *N, double *walkers, double *weights,
                       double *overlaps, double *ehist);

/* Walkers of individual bond dimensions (the reference's MPSstate keeps its own VirtualD,
 * MPSstate.cpp:13-40, and InnerProduct handles differing dims, 264-267).  dims: [N][L+1], each
 * row valid for the chain and elementwise <= the configuration's walker_dims; walker w's tensors
 * (sum_s dims[w][s]*dims[w][s+1]*d doubles, reference layout) follow walker w-1's back to back.
 * Otherwise as mpsqmc_set_walkers.  One launch of every kernel serves all sizes; walkers are
 * handed to CTAs dynamically. */
int mpsqmc_set_walkers_dims(mpsqmc_ctx *ctx, int N, const int *dims, const double *walkers,
                            const double *weights, const double *overlaps, const double *ehist,
                            int normalize);
/* Bond dims of the current population in logical order: dims [N][L+1] (may be NULL). */
int mpsqmc_get_walker_dims(mpsqmc_ctx *ctx, int *N, int *dims);

/* MPSstate::CompressState(target_D[w]) (MPSstate.cpp:379-404; two-site SVD sweeps right then left,
 * truncation at target_D and at Schmidt values < 1e-13, TwoSiteObject.cpp:71-184) on the device for
 * every current walker w (logical order; target_D[w] <= 0, or >= the walker's largest bond
 * dimension, leaves walker w unchanged, as SetupWalkers compresses only when DW < DT).  With
 * normalize != 0 each walker then gets Walker::setOverlap, as SetupWalkers does after compressing
 * (MPSQMC2.cpp:404-409).  The walkers' bond dims shrink accordingly (mpsqmc_get_walker_dims).
 * Singular-vector signs are this implementation's: the states equal the reference's, the
 * tensors may differ by signs on the bonds. */
int mpsqmc_compress_walkers(mpsqmc_ctx *ctx, const int *target_D, int normalize);

/* Random stream: mt19937(seed) advanced by `skip` 32-bit outputs; every uniform is one output
 * divided by 2^32 (Random.cpp:28-59 with Boost's uniform_real_distribution). */
int mpsqmc_set_rng(mpsqmc_ctx *ctx, uint32_t seed, uint64_t skip);
int mpsqmc_get_rng_draws(mpsqmc_ctx *ctx, uint64_t *draws_since_set);

/* EnergyFunctionAndHistory(1, &E, false) (MPSQMC2.cpp:447, 688-747) on the current population. */
int mpsqmc_energy(mpsqmc_ctx *ctx, double *E_P);

/* Run `nsteps` iterations of the body of MPSQMC2::Walk (MPSQMC2.cpp:465-511): propagation of
 * every walker (PropagateSeparately, 518-611), weight sum, E_T, local energies and history
 * (688-747), threshold population control (613-686).  stats may be NULL or hold nsteps
 * entries.  Each step runs as one CUDA graph launch (captured on first use). */
int mpsqmc_walk(mpsqmc_ctx *ctx, int nsteps, mpsqmc_step_stats *stats);

/* Set the number of completed steps.  The next step is completed_steps + 1; it divides the
 * energy history in the fluctuation metric (MPSQMC2.cpp:708).  MPSQMC2::Walk restarts its step
 * loop at 1 on every call (MPSQMC2.cpp:465): call mpsqmc_set_step(ctx, 0) before mpsqmc_walk to
 * get that behaviour; by default the count continues across mpsqmc_walk calls. */
int mpsqmc_set_step(mpsqmc_ctx *ctx, int completed_steps);

/* Per-walker data of the most recent step, in the logical order used during that step (before
 * branching): weight, overlap and local energy after propagation; parent[k] is the pre-branch
 * index that walker k of the new population was copied from.  Any pointer may be NULL. */
int mpsqmc_last_step_walkers(mpsqmc_ctx *ctx, int *n_before, double *weight, double *overlap,
                             double *energy, int *n_after, int *parent);

/* Optional per-coupling trace of the next mpsqmc_walk step (for parity tests):
 * [N][nC][16 + 5] = C[16], PDF norm, uniform, grid index, weight, overlap after the coupling.
 * Enable before the step; read after.  Costs one device buffer of capacity*nC*21 doubles. */
int mpsqmc_set_trace(mpsqmc_ctx *ctx, int enable);
int mpsqmc_get_trace(mpsqmc_ctx *ctx, double *trace, int *n_walkers);

/* Device timing of the last mpsqmc_walk call: milliseconds spent in the walker-step kernel
 * (summed over steps), and the number of kernel launches the call made. */
int mpsqmc_last_timing(mpsqmc_ctx *ctx, double *step_kernel_ms, double *total_ms,
                       int *kernel_launches);

/* Engine options.  No counterpart in the reference (its choices are compile-time).  A new value
 * takes effect from the next mpsqmc_walk step; unknown options or values give MPSQMC_E_ARG. */
#define MPSQMC_OPT_SWEEP 1        /* walker-step kernel: */
#define MPSQMC_SWEEP_AUTO 0       /*   the general sweep (the faster one, also on chains) */
#define MPSQMC_SWEEP_NEAREST 1    /*   nearest-neighbour sweep (MPSQMC_E_UNSUPPORTED for longer couplings) */
#define MPSQMC_SWEEP_GENERAL 2    /*   couplings (i, j) of any range, e.g. 2D lattices on a snake path */
#define MPSQMC_OPT_WORKSPACE 2    /* where a CTA's matrix work buffers live: */
#define MPSQMC_WORKSPACE_AUTO 0   /*   shared memory when they fit, else global scratch (L2-cached) */
#define MPSQMC_WORKSPACE_GLOBAL 1 /*   always global scratch (reads the option back as the placement in use) */
#define MPSQMC_OPT_POPCONTROL_INTERVAL 3 /* population control every K >= 1 steps (default 1, as the
                                          * reference); on the steps between, weights are only
                                          * rescaled by Ndesired / sum(w) and no uniform is drawn */
#define MPSQMC_OPT_RESAMPLING 4   /* population control rule: */
#define MPSQMC_RESAMPLE_THRESHOLD 0 /* the reference's threshold branching (MPSQMC2.cpp:613-686) */
#define MPSQMC_RESAMPLE_COMB 1    /*   comb: one uniform u, walker w gets the teeth k + u in
                                   *   [S_w, S_w + s_w) of the running sum of scaled weights s,
                                   *   each copy with weight 1 (about Ndesired walkers) */
#define MPSQMC_OPT_PROJECTOR 5    /* what one mpsqmc_walk step does: */
#define MPSQMC_PROJECTOR_TROTTER 0    /* MPSQMC2::Walk: Trotter two-site propagators with auxiliary
                                       * fields (default) */
#define MPSQMC_PROJECTOR_MPO_TERMS 1  /* MPSQMC::Walk (MPSQMC.cpp:236-369): 1 - dtau H sampled one MPO
                                       * term at a time (identity or one of the terms J Sx Sx, -J iSy
                                       * iSy, J Sz Sz per coupling, -h Sz per site), weights summed
                                       * into an int as the reference does, and the reference's
                                       * population control (every walker: int(w s + u) copies of
                                       * weight 1); the trace then holds [N][3] = PDF norm, uniform,
                                       * picked term (0 = identity).  The population-control options
                                       * above do not apply. */
#define MPSQMC_OPT_CANONICAL_INTERVAL 6 /* K >= 1 (default 16): the general sweep stores each site
                                         * as it leaves the centre, without the per-site
                                         * Householder QR (the norm comes from a left norm
                                         * environment), and restores the left-canonical form of
                                         * Walker::setOverlap on every K-th step; 0: one QR per
                                         * site, the state the reference's per-coupling setOverlap
                                         * leaves.  Same walk (every quantity it uses is gauge
                                         * invariant).  mpsqmc_get_walkers and
                                         * mpsqmc_compress_walkers left-normalise first when the
                                         * last step did not.  Applies to the Trotter projector's
                                         * general sweep; with h != 0 the walkers are
                                         * left-normalised every step anyway. */
#define MPSQMC_OPT_PRECISION 7       /* arithmetic of the walker-step contractions (what a
                                      * set_precision(FP64 | TF32 | ...) entry point would select): */
#define MPSQMC_PRECISION_FP64 0      /*   FP64 tensor cores (DMMA), the reference's arithmetic (default) */
#define MPSQMC_PRECISION_TF32 1      /*   FP32 work buffers, one TF32 tensor-core pass per product */
#define MPSQMC_PRECISION_TF32X3 2    /*   FP32 work buffers, three TF32 passes (head/tail split):
                                      *   about FP32 accuracy.  Both mixed modes keep the walkers,
                                      *   closures, PDF, sampling, weights, overlaps, norms, energies
                                      *   and population control in FP64, run the QR-free sweep
                                      *   (left-normalising in FP64 every MPSQMC_OPT_CANONICAL_INTERVAL
                                      *   steps, 4 when that option is 0) and apply to the general
                                      *   sweep of the Trotter projector; the per-coupling trace is
                                      *   FP64-only (MPSQMC_E_UNSUPPORTED). */
#define MPSQMC_PRECISION_TF32X3_TC 3 /*   the walker-batched sweep on the tcgen05 tensor cores: all
                                      *   walkers move through the sites in lockstep and every
                                      *   contraction of the step is one batched tcgen05 product
                                      *   (TMA-fed, FP32 accumulators in TMEM) over the population,
                                      *   three TF32 passes (FP32 accuracy).  Same FP64 parts and
                                      *   QR-free sweep as TF32X3.  Needs walkers of one bond
                                      *   profile (MPSQMC_E_UNSUPPORTED otherwise) and the grid
                                      *   proposal; its trace records C/ov, the factor, uniform,
                                      *   index, weight and the overlap ratio per coupling. */
#define MPSQMC_PRECISION_TF32_TC 4   /*   the same with one TF32 pass per product */
#define MPSQMC_PRECISION_BF16_TC 5   /*   the same with one bfloat16 pass per product (tcgen05
                                      *   kind::f16, FP32 accumulation): operands rounded to 8
                                      *   mantissa bits, for callers that trade accuracy (local
                                      *   energies about 1e-2 relative) for speed */
#define MPSQMC_OPT_PROPOSAL 8        /* how a coupling's grid point is drawn (what a
                                      * set_proposal(GRID | LEARNED) entry point would select): */
#define MPSQMC_PROPOSAL_GRID 0       /*   the exact grid PDF, as MPSQMC2.cpp:551-588 (default) */
#define MPSQMC_PROPOSAL_LEARNED 1    /*   the learned proposal q: the point is drawn from q restricted
                                      *   to the PDF's support and the weight takes P(x) / q(x)
                                      *   (exact-ratio reweighting; unbiased).  The grid PDF is the
                                      *   zero-variance choice for one coupling, so q can at best
                                      *   match it; Trotter projector, grids of up to 256 points */
#define MPSQMC_OPT_PROPOSAL_TRAINING 9 /* 1: every grid step also stores (features, exact PDF) of one
                                        * coupling per walker and takes one Adam step (step size
                                        * 1e-3) of the network on them (mean KL(P || q)) */
#define MPSQMC_OPT_PROPOSAL_MIX 10   /* alpha in thousandths, 0..1000 (default 100): the learned
                                      * proposal draws from the defensive mixture
                                      * (1 - alpha) q + alpha P / sum P (Hesterberg, Technometrics
                                      * 37 (1995) 185), so the weight factor P(x) / q_mix(x) is at
                                      * most sum P / alpha and a poorly trained network cannot
                                      * give heavy-tailed weights.  1000 samples the grid PDF. */
#define MPSQMC_OPT_TC_STACK_TN 11     /* tile choices of the tcgen05 sweep's products (defaults
                                      * 256, 256, 8; mpsqmc_autotune picks them per bond profile):
                                      * widest N tile (64, 128, 256) of the products whose left
                                      * factor is a trial tensor, walkers stacked along N up to it */
#define MPSQMC_OPT_TC_WIDE_TN 12      /*   widest N tile (64, 128, 256) of the walker-by-walker
                                      *   products */
#define MPSQMC_OPT_TC_STAGES 13       /*   load-ring depth cap, 2..8 (fewer when shared memory is
                                      *   short; default 8) */
#define MPSQMC_OPT_TC_SPLIT_OUT 14    /*   mask 0..31 (default 0): with three passes, the classes
                                      *   of walker-side right factors of the trial products that
                                      *   are written as TF32 head and tail arrays and loaded split
                                      *   (the trial itself always is) instead of being split in
                                      *   shared memory: 1 right environments and closures, 2 left
                                      *   branches, 4 branch carries, 8 energy, 16 energy channels */
#define MPSQMC_OPT_TC_KC 15           /*   k-values per load stage of the trial products: 32
                                      *   (default, 128-byte swizzled rows) or 16 (64-byte rows:
                                      *   half the stage, twice the ring depth) */
int mpsqmc_set_option(mpsqmc_ctx *ctx, int option, long value);
int mpsqmc_get_option(mpsqmc_ctx *ctx, int option, long *value);

/* Walks split over ranks, one context per rank and GPU: the reference's MPI path through
 * MPSQMC2::Walk (MPSQMC2.cpp:465-511 with USE_MPI_IN_MPSQMC) and PopulationBalancing
 * (MPSQMC2.cpp:778-934).  A step is mpsqmc_step_propagate on every rank, a sum of the five
 * local sums over the ranks (the reference's MPI Allreduce calls), then mpsqmc_step_control on
 * every rank; mpsqmc_walk on one rank is the same as the pair with its own sums.
 *   mpsqmc_step_propagate: one step's propagation, local energies and energy-history update;
 *     local_sums = {sum w, sum w E, sum of Ehist/step, sum of (Ehist/step)^2, walker count}.
 *     A rank may hold no walkers.
 *   mpsqmc_step_control: statistics from the global sums and ndesired_total (scaling =
 *     ndesired_total / sum w, E_T, E_P, fluctuation metric), then this rank's population control
 *     with that scaling.  stats: sum_weight, E_P, E_T, omega and scaling are global, the walker
 *     counts this rank's.
 *   mpsqmc_export_walkers / mpsqmc_import_walkers: move the last k walkers (logical order) out
 *     as records of mpsqmc_record_size doubles (weight, overlap, energy history, bond dims, site
 *     tensors), or append k records; records are device memory (or memory the device can read
 *     and write).  Exported walkers are left-normalised first. */
int mpsqmc_step_propagate(mpsqmc_ctx *ctx, double local_sums[5]);
int mpsqmc_step_control(mpsqmc_ctx *ctx, const double global_sums[5], long ndesired_total,
                        mpsqmc_step_stats *stats);
long mpsqmc_record_size(const mpsqmc_ctx *ctx);
int mpsqmc_export_walkers(mpsqmc_ctx *ctx, int k, double *records);
int mpsqmc_import_walkers(mpsqmc_ctx *ctx, int k, const double *records);

/* Learned proposal (no counterpart in the reference).  The network maps 32 features of a
 * coupling (4 C_kl / ov and 4 M / ov: the overlap-ratio coefficients and the 16 closures of the
 * environment branches) through two hidden layers of 128 (ReLU) to logits over the G grid points.
 * Parameters: one FP32 vector of n = 32*128 + 128 + 128*128 + 128 + 128*G + G, W input-major
 * (W1[i*128 + o], then b1, W2, b2, W3[i*G + o], b3); the sweep reads a BF16 copy.
 *   mpsqmc_proposal_params: copies the parameters out (out != NULL) and/or in (in != NULL; resets
 *     the Adam state); *n_params receives n.  Parameters are created on first use (He-uniform,
 *     fixed seed).
 *   mpsqmc_proposal_loss_grad: mean KL(p || softmax(z)) over a batch of B <= capacity pairs
 *     (features [B][32], targets [B][G], each target a normalised PDF) and its gradient [n].
 *   mpsqmc_proposal_stats: the loss of the last training step and the number of Adam steps. */
int mpsqmc_proposal_params(mpsqmc_ctx *ctx, float *out, const float *in, long *n_params);
int mpsqmc_proposal_loss_grad(mpsqmc_ctx *ctx, int B, const float *features, const float *targets,
                              double *loss, float *grad);
int mpsqmc_proposal_stats(mpsqmc_ctx *ctx, double *last_loss, int *updates);

/* Autotuner (no counterpart in the reference): times `steps` steps of every applicable
 * (MPSQMC_OPT_SWEEP, MPSQMC_OPT_WORKSPACE) choice on the first walkers of the current population
 * (two waves of one CTA per SM), restores the population, random stream and step count after
 * each trial, and keeps the fastest.  Under the tcgen05 sweep (MPSQMC_PRECISION_TF32X3_TC,
 * TF32_TC, BF16_TC) it instead tunes that sweep's choices (MPSQMC_OPT_TC_SPLIT_OUT, _KC, _STACK_TN,
 * _WIDE_TN, _STAGES) by a coordinate search from the defaults, each timed on up to 1024 walkers (its tile counts
 * grow with the population).  The choice is remembered per problem shape (L, trial and walker
 * bond dims, couplings, projector, sweep family) for later contexts of this process, which then
 * skip the measurement.  best_* (may be NULL) receive the chosen sweep and workspace values. */
int mpsqmc_autotune(mpsqmc_ctx *ctx, int steps, int *best_sweep, int *best_workspace);

/* ---------------------------------------------------------------------------------------------
 * One batched FP32 product on the tcgen05 tensor cores (the building block of the walker-batched
 * mixed-precision sweep; no counterpart in the reference, whose products are dgemm_ calls, e.g.
 * MPSstate.cpp:271-274).  For z < Z:
 *   D_z[m, n] = alpha * sum_k A_{z/adiv}[m, k] B_{z/bdiv}[n, k]   (+ D_z[m, n] when beta = 1)
 * with A_x[m, k] = A[k + m lda + x a_zstride], B_x[n, k] = B[k + n ldb + x b_zstride] (k
 * contiguous) and D_z[m, n] = D[z dz + m dm + n dn]; adiv / bdiv = 0: the operand is shared by
 * every z.  bstack > 1 (A shared) puts bstack consecutive z side by side in one tile of N.
 * Operands are read in whole tiles and must be zero padded: k up to K rounded up to 32 (lda, ldb
 * cover it), A rows up to a multiple of 64 (M <= 64) or 128, B rows up to a multiple of the tile
 * width (N rounded up to 16, at most 256) when bstack = 1, and a_zcount / b_zcount operand
 * entries allocated (B: at least Z rounded up to bstack when stacked).  Strides are multiples of 4
 * and pointers 16-byte aligned.  passes = 3: FP32-accurate (head/tail TF32 split), 1: TF32,
 * 16: one bfloat16 pass (kind::f16; operands rounded to bfloat16, FP32 accumulation).
 * Device pointers; asynchronous on `stream`.  *err (device int) receives bit 4 if a pipeline wait
 * timed out.  Returns 0 or a negative status. */
int mpsqmc_tc_gemm(float *D, const float *A, const float *B, int M, int N, int K, long lda, long a_zstride,
                   int adiv, long a_zcount, long ldb, long b_zstride, int bdiv, long b_zcount, int Z, int bstack,
                   float alpha, int beta, int passes, long dz, long dm, long dn, int *err, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Local energies without any device allocation.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: code whose device memory is owned by someone else
 * (a framework's caching allocator, a fixed arena handed over by the application) or that runs
 * where allocating is not allowed.  The caller passes device pointers to its own inputs and
 * outputs; the environment scratch the kernel needs lives in one file-scope device array of
 * MPSQMC_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds until the process
 * exits.  The function calls no cudaMalloc, cudaFree or allocating library routine.
 *
 * Computes, for w < n_walkers, energies[w] = <Psi_T|H|phi_w> / overlaps[w] (the local energy of
 * the walk) for H = sum_c J_c S_i.S_j - h sum_k S^z_k on a nearest-neighbour chain, on `stream`
 * (a cudaStream_t, NULL = legacy default stream), asynchronously: results are valid once the
 * stream has been synchronised.
 *   trial:   device, reference layout for trial_dims;
 *   walkers: device, walker w at walkers + w * walker_stride, reference layout for walker_dims;
 *   overlaps, energies: device, n_walkers doubles each.
 * Limits: L <= MPSQMC_NOALLOC_MAX_L, d = 2, and one CTA's slice of the array must hold the
 * compact-MPO environments, 8 * max(trial_dims) * max(walker_dims) doubles, plus - when they do
 * not fit in the device's shared memory beside the small buffers (about max bond 32 x 64 on a
 * B200) - the matrix work buffers, about 12 * (max(trial_dims) + 4) * max(walker_dims) doubles:
 * up to trial and walker bond dimension ~180 in the 8 MiB array.  Larger problems are rejected
 * with MPSQMC_E_UNSUPPORTED and a message in mpsqmc_last_error(), also when n_walkers is 0.
 * The bond tables travel as a kernel argument: a call issues no host-to-device copy.
 * The first call on a device (with that device current) looks up the array's device address
 * and raises the kernel's shared-memory limit; make that first call before any stream capture.
 * Every call reuses the same array and leaves its contents behind; each call writes every
 * scratch element before reading it.  Calls that overlap on the GPU (different streams, or
 * different host threads without ordering) race on the array. */
#define MPSQMC_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)
#define MPSQMC_NOALLOC_MAX_L 128

typedef struct {
  int L;                   /* chain length */
  int d;                   /* local dimension (2) */
  const int *trial_dims;   /* host [L+1] */
  const int *walker_dims;  /* host [L+1] */
  int nC;                  /* couplings (nearest-neighbour, ordered by site) */
  const int *ci, *cj;      /* host [nC] */
  const double *cJ;        /* host [nC] */
  double h;                /* field */
} mpsqmc_energy_layout;

int mpsqmc_local_energy_noalloc(const mpsqmc_energy_layout *layout, const double *trial,
                                const double *walkers, long walker_stride,
                                const double *overlaps, int n_walkers, double *energies,
                                int device, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MPSQMC_GPU_H */
