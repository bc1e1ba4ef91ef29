/* Test infrastructure: C ABI of the CPU restatement of the reference's walker-propagation
 * path (oracle/mpsqmc_oracle.cpp).  Only tests, the fixture generator, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load this library, and only as the checker.
 *
 * MPS layout (as the reference stores it, MPStensor.cpp:91-96): bond dims dims[0..L],
 * dims[0] = dims[L] = 1; site s holds dims[s]*dims[s+1]*d doubles at element
 * [r + dims[s]*(c + dims[s+1]*sigma)]; sites are concatenated in order.
 */
#ifndef MPSQMC_ORACLE_H
#define MPSQMC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

long orc_mps_size(int L, int d, const int *dims);

/* MPSstate::InnerProduct, MPSstate.cpp:248-284: A.InnerProduct(B). */
double orc_inner_product(int L, int d, const int *dimsA, const double *A, const int *dimsB,
                         const double *B);

/* MPSstate::LeftNormalize, MPSstate.cpp:216-229 (Householder QR of MPStensor.cpp:100-135,
 * LeftMultiply 159-175).  In place; returns the last R factor (work1[0]). */
double orc_left_normalize(int L, int d, const int *dims, double *data);

/* MPSstate::ChangePhase, MPSstate.cpp:307-315. */
void orc_change_phase(int L, int d, const int *dims, double *data);

/* MPSstate::ApplyTwoSiteTrotterTerm(grid), MPSstate.cpp:575-633, for one coupling of strength
 * with tables S[d2], U[d2*d2], VT[d2*d2] (layouts of TrotterHeisenberg.cpp:391,425) and the
 * grid point x[d2]. */
void orc_apply_grid_op(int L, int d, const int *dims, double *data, int i, int j,
                       const double *S, const double *U, const double *VT, const double *x);

/* MPSstate::ApplyTwoSiteTrotterTerm(svd index), MPSstate.cpp:505-573. */
void orc_apply_svd_op(int L, int d, const int *dims, double *data, int i, int j,
                      const double *S, const double *U, const double *VT, int k, int l,
                      int doHC);

/* GridGenerator::FillMarsaglia / FillSimple, GridGenerator.cpp:167-308.  Writes points as
 * out[i + dim*p]; returns the number of points (or -1 if capacity is too small). */
int orc_grid_marsaglia(int dim, int pointsPerCo, double *out, int capacity);
int orc_grid_simple(int dim, int denominator, double *out, int capacity);

/* TrotterHeisenberg::SetTheTwoSitePropagators, TrotterHeisenberg.cpp:102-285, with a Jacobi
 * eigensolver and a Jacobi SVD in place of dsyev/dgesdd.  Singular vectors of degenerate
 * singular values are basis-dependent; only U*S*VT and S are comparable with LAPACK's. */
int orc_trotter(int d, double J, double dtau, double *U, double *S, double *VT);

/* <Psi_T|H|phi> for H = sum_{c} J_c S_i.S_j - h sum_k S^z_k, by a left-to-right sandwich with
 * a compact MPO.  Equals HPsi0->InnerProduct(phi) of MPSQMC2.cpp:255-257 and Walker.cpp:76. */
double orc_local_energy_numerator(int L, int d, const int *dimsT, const double *T,
                                  const int *dimsW, const double *W, int nC, const int *ci,
                                  const int *cj, const double *cJ, double h);

/* MPSstate::CompressState(truncD), MPSstate.cpp:379-404 with TwoSiteObject.cpp:71-184, using
 * a one-sided Jacobi SVD.  dims_inout is updated; data_out must hold orc_mps_size of the
 * input dims.  Returns the new maximal bond dimension. */
int orc_compress(int L, int d, int *dims_inout, const double *data_in, double *data_out,
                 int truncD);

/* Walk: MPSQMC2::Walk, MPSQMC2.cpp:443-513, with PropagateSeparately (518-611),
 * EnergyFunctionAndHistory (688-747) and SeparatePopulationControl (613-686).
 * All walkers share the bond dims dimsW.  RNG: one mt19937 seeded with `seed`, advanced by
 * `skip` 32-bit outputs, uniforms x/2^32 (Random.cpp:57 with Boost's uniform_real).
 * Per-step outputs have length nsteps; per-walker outputs are [nsteps][capacity];
 * trace (optional, may be null) is [nsteps][capacity][nC][16 + 5]:
 *   C[16], pdfnorm, u, index, weight, overlap after the coupling.
 * walkers/weights/overlaps/ehist are updated in place (capacity entries); *n_walkers too.
 * Returns 0, or a negative status: -1 capacity exceeded, -2 bad input. */
typedef struct {
  int L, d, nC, nJ, G, Ndesired, capacity, nsteps, nthreads;
  double dtau, h;
  unsigned int seed;
  unsigned long long skip;
  /* Population-control variants of the engine (no counterpart in the reference; 0, 0 is the
   * reference): popctl_interval K > 1 branches on steps divisible by K and only rescales the
   * weights by Ndesired / sum(w) in between; comb != 0 resamples with one uniform u, walker w
   * getting the teeth k + u inside [S_w, S_w + s_w) of the sequential running sum S of the
   * scaled weights s, each copy with weight 1. */
  int popctl_interval, comb;
} orc_walk_config;

/* As orc_walk, with walker w's own bond dims in wdims[w*(L+1) ..] (each <= dimsW elementwise;
 * walker slots keep the stride of dimsW, tensors packed from the slot start).  wdims is updated
 * by the branching (copies keep their parent's dims).  wdims == NULL: every walker has dimsW. */
int orc_walk_dims(const orc_walk_config *cfg, const int *dimsT, const double *trial, const int *ci,
                  const int *cj, const double *cJ, const double *Jvals, const double *Utab,
                  const double *Stab, const double *VTtab, const double *grid, const int *dimsW,
                  int *wdims, double *walkers, double *weights, double *overlaps, double *ehist,
                  int *n_walkers, double *E0, double *st_sumw, double *st_EP, double *st_ET,
                  double *st_omega, int *st_n, double *pw_weight, double *pw_overlap, double *pw_energy,
                  int *pw_parent, double *trace, unsigned long long *draws_used);

int orc_walk(const orc_walk_config *cfg, const int *dimsT, const double *trial, const int *ci,
             const int *cj, const double *cJ, const double *Jvals, const double *Utab,
             const double *Stab, const double *VTtab, const double *grid, const int *dimsW,
             double *walkers, double *weights, double *overlaps, double *ehist, int *n_walkers,
             double *E0, double *st_sumw, double *st_EP, double *st_ET, double *st_omega,
             int *st_n, double *pw_weight, double *pw_overlap, double *pw_energy,
             int *pw_parent, double *trace, unsigned long long *draws_used);

#ifdef __cplusplus
}
#endif

#endif
