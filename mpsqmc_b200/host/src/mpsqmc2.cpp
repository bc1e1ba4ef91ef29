// MPSQMC2 on the GPU engine: set-up on the host (trial, Trotter tables, grid, initial walkers),
// then every Walk() step is one mpsqmc_walk call (include/mpsqmc_gpu.h).  Console lines and the
// energy file follow MPSQMC2.cpp:449-498, 613-686 and 749-758.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <utility>
#include <vector>

#include "MPSQMC2.h"
#include "../../../include/mpsqmc_gpu.h"

MPSQMC2::MPSQMC2(HeisenbergMPO *mpo, GridGenerator *grid, Random *rn, const int DT_, const int DW_,
                 const int Nwalkers, const double dt)
    : theMPO(mpo), theTrotter(nullptr), theGrid(grid), RN(rn), DT(DT_), DW(DW_), totalNDesiredWalkers(Nwalkers),
      dtau(dt), Psi0(nullptr), ctx(nullptr) {
  // trial from DMRG, as SetupTrial(true) does (MPSQMC2.cpp:223-237)
  MPSstate trial(mpo->gLength(), DT, mpo->gPhys_d(), RN);
  DMRG solver(&trial, mpo);
  solver.Solve();
  Setup(&trial);
}

MPSQMC2::MPSQMC2(HeisenbergMPO *mpo, GridGenerator *grid, Random *rn, MPSstate *Psi0_in, const int DW_,
                 const int Nwalkers, const double dt)
    : theMPO(mpo), theTrotter(nullptr), theGrid(grid), RN(rn), DT(Psi0_in->gDtrunc()), DW(DW_),
      totalNDesiredWalkers(Nwalkers), dtau(dt), Psi0(nullptr), ctx(nullptr) {
  Setup(Psi0_in);
}

MPSQMC2::~MPSQMC2() {
  if (ctx) mpsqmc_destroy(ctx);
  delete theTrotter;
  delete Psi0;
}

void MPSQMC2::Setup(MPSstate *trial) {
  const int L = theMPO->gLength(), d = theMPO->gPhys_d();
  theTrotter = new TrotterHeisenberg(theMPO, dtau);
  Psi0 = new MPSstate(trial);
  Psi0->LeftNormalize();
  std::vector<int> ci, cj, tdims(L + 1), wdims(L + 1);
  std::vector<double> cJ, trialdata, U, S, VT, Jv, grid;
  for (int a = 0; a < L - 1; ++a)
    for (int b = a + 1; b < L; ++b) {
      const double J = theTrotter->gCoupling(a, b);
      if (J != 0.0) {
        ci.push_back(a);
        cj.push_back(b);
        cJ.push_back(J);
      }
    }
  const int n2 = d * d;
  for (int q = 0; q < theTrotter->gNDifferentCouplings(); ++q) {
    const double J = theTrotter->gDifferentCoupling(q);
    Jv.push_back(J);
    for (int k = 0; k < n2; ++k) S.push_back(theTrotter->gTwoSitePropSVD_Sing(J, k));
    const size_t u0 = U.size(), v0 = VT.size();
    U.resize(u0 + n2 * n2);
    VT.resize(v0 + n2 * n2);
    for (int k = 0; k < n2; ++k)
      for (int i = 0; i < d; ++i)
        for (int j = 0; j < d; ++j) {
          U[u0 + i + d * (j + d * k)] = theTrotter->gTwoSitePropSVD_Left(J, k, i, j);
          VT[v0 + k + n2 * (i + d * j)] = theTrotter->gTwoSitePropSVD_Right(J, k, i, j);
        }
  }
  if (n2 != theGrid->gDim())
    cerr << "trotterSVDsize = " << n2 << " and is not equal to theGrid->gDim() = " << theGrid->gDim() << endl;
  for (int p = 0; p < theGrid->gNPoints(); ++p)
    for (int k = 0; k < theGrid->gDim(); ++k) grid.push_back(theGrid->gCoOfPoint(p, k));
  for (int b = 0; b <= L; ++b) tdims[b] = Psi0->gDimAtBound(b);
  for (int s = 0; s < L; ++s) {
    MPStensor *t = Psi0->gMPStensor(s);
    const int n = tdims[s] * tdims[s + 1] * d;
    trialdata.insert(trialdata.end(), t->gStorage(), t->gStorage() + n);
  }
  // walkers: copies of the trial, compressed to DW when DW < DT (SetupWalkers, MPSQMC2.cpp:381-441)
  MPSstate walker(Psi0);
  if (DW < DT) walker.CompressState(DW);
  for (int b = 0; b <= L; ++b) wdims[b] = walker.gDimAtBound(b);
  std::vector<double> w0;
  for (int s = 0; s < L; ++s) {
    MPStensor *t = walker.gMPStensor(s);
    const int n = wdims[s] * wdims[s + 1] * d;
    w0.insert(w0.end(), t->gStorage(), t->gStorage() + n);
  }
  mpsqmc_config cfg;
  cfg.L = L;
  cfg.d = d;
  cfg.nC = (int)ci.size();
  cfg.ci = ci.data();
  cfg.cj = cj.data();
  cfg.cJ = cJ.data();
  cfg.h = theMPO->gField();
  cfg.dtau = dtau;
  cfg.trial_dims = tdims.data();
  cfg.trial = trialdata.data();
  cfg.nJ = (int)Jv.size();
  cfg.Jvals = Jv.data();
  cfg.U = U.data();
  cfg.S = S.data();
  cfg.VT = VT.data();
  cfg.G = theGrid->gNPoints();
  cfg.grid = grid.data();
  cfg.Ndesired = totalNDesiredWalkers;
  cfg.capacity = std::max(1000, 3 * totalNDesiredWalkers);
  cfg.walker_dims = wdims.data();
  cfg.device = 0;
  if (mpsqmc_create(&cfg, &ctx) != MPSQMC_OK) {
    cerr << "MPSQMC2: GPU engine unavailable: " << mpsqmc_last_error() << endl;
    ctx = nullptr;
    return;
  }
  // engine options from the environment, so that an unchanged main.cpp can choose them:
  //   MPSQMC_PRECISION = fp64 | tf32 | tf32x3 | tf32x3_tc | tf32_tc, MPSQMC_CANONICAL_INTERVAL = K,
  //   MPSQMC_POPCONTROL_INTERVAL = K, MPSQMC_RESAMPLING = threshold | comb
  {
    struct Named {
      const char *var;
      int option;
      const char *names[6];
      long values[6];
    };
    const Named named[] = {
        {"MPSQMC_PRECISION", MPSQMC_OPT_PRECISION, {"fp64", "tf32", "tf32x3", "tf32x3_tc", "tf32_tc", "bf16_tc"},
         {MPSQMC_PRECISION_FP64, MPSQMC_PRECISION_TF32, MPSQMC_PRECISION_TF32X3, MPSQMC_PRECISION_TF32X3_TC,
          MPSQMC_PRECISION_TF32_TC, MPSQMC_PRECISION_BF16_TC}},
        {"MPSQMC_RESAMPLING", MPSQMC_OPT_RESAMPLING, {"threshold", "comb", nullptr, nullptr, nullptr, nullptr},
         {MPSQMC_RESAMPLE_THRESHOLD, MPSQMC_RESAMPLE_COMB, 0, 0, 0, 0}}};
    for (const Named &o : named) {
      const char *v = getenv(o.var);
      if (!v) continue;
      int k = 0;
      while (k < 6 && o.names[k] && std::string(v) != o.names[k]) ++k;
      if (k == 6 || !o.names[k] || mpsqmc_set_option(ctx, o.option, o.values[k]) != MPSQMC_OK)
        cerr << "MPSQMC2: ignoring " << o.var << "=" << v << endl;
    }
    const std::pair<const char *, int> counts[] = {{"MPSQMC_CANONICAL_INTERVAL", MPSQMC_OPT_CANONICAL_INTERVAL},
                                                   {"MPSQMC_POPCONTROL_INTERVAL", MPSQMC_OPT_POPCONTROL_INTERVAL}};
    for (const auto &o : counts) {
      const char *v = getenv(o.first);
      if (v && mpsqmc_set_option(ctx, o.second, std::atol(v)) != MPSQMC_OK)
        cerr << "MPSQMC2: ignoring " << o.first << "=" << v << endl;
    }
  }
  const int N = totalNDesiredWalkers;
  std::vector<double> all((size_t)N * w0.size()), ones(N, 1.0), zeros(N, 0.0);
  for (int w = 0; w < N; ++w) std::copy(w0.begin(), w0.end(), all.begin() + (size_t)w * w0.size());
  if (mpsqmc_set_walkers(ctx, N, all.data(), ones.data(), ones.data(), zeros.data(), 1) != MPSQMC_OK)
    cerr << "MPSQMC2: " << mpsqmc_last_error() << endl;
}

void MPSQMC2::write(const int step, const int nwalkers, const double EP, const double ET, const double omega) {
  char filename[100];
  snprintf(filename, sizeof filename, "output/Heisenberg1D/ener_L%dDT%dDW%d.txt", theMPO->gLength(), DT, DW);
  std::ofstream out(filename, std::ios::app);
  out.precision(10);
  out << step << "\t\t" << nwalkers << "\t" << EP << "\t\t" << ET << "\t\t" << omega << endl;
}

void MPSQMC2::Walk(const int steps) {
  if (!ctx) {
    cerr << "MPSQMC2::Walk: no GPU engine (see the message at construction)." << endl;
    return;
  }
  double E = 0.0;
  if (mpsqmc_energy(ctx, &E) != MPSQMC_OK) cerr << "MPSQMC2::Walk: " << mpsqmc_last_error() << endl;
  {
    char filename[100];
    snprintf(filename, sizeof filename, "output/Heisenberg1D/ener_L%dDT%dDW%d.txt", theMPO->gLength(), DT, DW);
    std::ofstream out(filename, std::ios::trunc);
    out << "#Step\t\tE_P\t\tE_T\t\tFluctMetric" << endl;
  }
  cout << "Energy at start = " << E << endl;
  cout << "---------------------------------------------------------" << endl;
  // the device continues the host's random stream; the host skips what the device drew
  mpsqmc_set_rng(ctx, RN->gSeed(), RN->gDraws());
  mpsqmc_set_step(ctx, 0);
  std::vector<double> wt;
  std::vector<int> parent;
  for (int step = 1; step <= steps; ++step) {
    mpsqmc_step_stats st;
    const int rc = mpsqmc_walk(ctx, 1, &st);
    if (rc != MPSQMC_OK) {
      cerr << "MPSQMC::Walk -> " << mpsqmc_last_error() << endl;
      return;
    }
    RN->discard(st.draws);
    cout << "        Step = " << step << endl;
    cout << "   # walkers = " << st.n_walkers << endl;
    cout << " avg(weight) = " << st.avg_weight << endl;
    cout << "         E_P = " << st.E_P << endl;
    cout << "         E_T = " << st.E_T << endl;
    cout << "       Omega = " << st.omega << endl;
    write(step, st.n_walkers, st.E_P, st.E_T, st.omega);
    cout << "---------------------------------------------------------" << endl;
    // branching report of SeparatePopulationControl (MPSQMC2.cpp:620-670)
    int nb = 0, na = 0;
    mpsqmc_last_step_walkers(ctx, &nb, nullptr, nullptr, nullptr, &na, nullptr);
    wt.resize(nb);
    parent.resize(na > 0 ? na : 1);
    mpsqmc_last_step_walkers(ctx, &nb, wt.data(), nullptr, nullptr, &na, parent.data());
    std::vector<int> copies(nb, 0);
    for (int k = 0; k < na; ++k) copies[parent[k]] += 1;
    double minW = 1.0;
    for (int w = 0; w < nb; ++w) {
      const double s = wt[w] * st.scaling;
      if (s < minW) minW = s;
      if (s < 0.25)
        cout << "Walker with weight " << s << " will be " << copies[w] << " times copied with weight 1 ." << endl;
      else if (s > 1.5)
        cout << "Walker with weight " << s << " will be " << copies[w] << " times copied with weight "
             << s / copies[w] << " ." << endl;
    }
    cout << "The min. encountered weight on rank 0 is " << minW << " ." << endl;
  }
}
