// MPSQMC on the GPU engine: the trial from DMRG on the host (MPSQMC.cpp:125-150), walkers are
// trial copies with weight 1 and overlap 1 (MPSQMC.cpp:195-233), and every Walk() step is one
// mpsqmc_walk call with the MPO-term projector.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <vector>

#include "GridGenerator.h"
#include "HeisenbergMPO.h"
#include "MPSQMC.h"
#include "TrotterHeisenberg.h"
#include "../../../include/mpsqmc_gpu.h"

MPSQMC::MPSQMC(MPO *mpo, Random *rn, const int D, const int Nwalkers, const double dt)
    : theMPO(mpo), RN(rn), Dtrunc(D), totalNDesiredWalkers(Nwalkers), dtau(dt), bSetupTrial(false),
      bSetupWalkers(false), Psi0(nullptr), ctx(nullptr) {
  SetupTrial();
  SetupWalkers();
}

MPSQMC::~MPSQMC() {
  if (ctx) mpsqmc_destroy(ctx);
  delete Psi0;
}

void MPSQMC::SetupTrial() {
  if (bSetupTrial) return;
  bSetupTrial = true;
  const int L = theMPO->gLength(), d = theMPO->gPhys_d();
  Psi0 = new MPSstate(L, Dtrunc, d, RN);
  {
    DMRG solver(Psi0, theMPO);
    solver.Solve();
  }
  Psi0->LeftNormalize();
  HeisenbergMPO *h = dynamic_cast<HeisenbergMPO *>(theMPO);
  if (h == nullptr) {
    cerr << "MPSQMC: the GPU engine samples the terms of a HeisenbergMPO only." << endl;
    return;
  }
  if (theMPO->gRN_nTerms() == 0)
    cerr << "MPSQMC: the MPO has no term list (call findNonZeroContributions first)." << endl;
  std::vector<int> ci, cj, dims(L + 1);
  std::vector<double> cJ, trial, grid;
  for (int a = 0; a < L - 1; ++a)
    for (int b = a + 1; b < L; ++b) {
      const double J = h->gCoupling(a, b);
      if (J != 0.0) {
        ci.push_back(a);
        cj.push_back(b);
        cJ.push_back(J);
      }
    }
  for (int b = 0; b <= L; ++b) dims[b] = Psi0->gDimAtBound(b);
  for (int s = 0; s < L; ++s) {
    MPStensor *t = Psi0->gMPStensor(s);
    trial.insert(trial.end(), t->gStorage(), t->gStorage() + (long)dims[s] * dims[s + 1] * d);
  }
  // the engine's configuration also carries Trotter tables and a grid, which this projector
  // does not use
  TrotterHeisenberg trot(h, dtau);
  std::vector<double> Jv, U, S, VT;
  for (int q = 0; q < trot.gNDifferentCouplings(); ++q) {
    const double J = trot.gDifferentCoupling(q);
    Jv.push_back(J);
    for (int k = 0; k < 4; ++k) S.push_back(trot.gTwoSitePropSVD_Sing(J, k));
    const size_t u0 = U.size();
    U.resize(u0 + 16);
    VT.resize(u0 + 16);
    for (int k = 0; k < 4; ++k)
      for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) {
          U[u0 + i + 2 * (j + 2 * k)] = trot.gTwoSitePropSVD_Left(J, k, i, j);
          VT[u0 + k + 4 * (i + 2 * j)] = trot.gTwoSitePropSVD_Right(J, k, i, j);
        }
  }
  GridGenerator g(4);
  g.FillMarsaglia(4);
  for (int p = 0; p < g.gNPoints(); ++p)
    for (int k = 0; k < 4; ++k) grid.push_back(g.gCoOfPoint(p, k));
  mpsqmc_config cfg;
  cfg.L = L;
  cfg.d = d;
  cfg.nC = (int)ci.size();
  cfg.ci = ci.data();
  cfg.cj = cj.data();
  cfg.cJ = cJ.data();
  cfg.h = h->gField();
  cfg.dtau = dtau;
  cfg.trial_dims = dims.data();
  cfg.trial = trial.data();
  cfg.nJ = (int)Jv.size();
  cfg.Jvals = Jv.data();
  cfg.U = U.data();
  cfg.S = S.data();
  cfg.VT = VT.data();
  cfg.G = g.gNPoints();
  cfg.grid = grid.data();
  cfg.Ndesired = totalNDesiredWalkers;
  cfg.capacity = std::max(1000, 3 * totalNDesiredWalkers);
  cfg.walker_dims = dims.data();
  cfg.device = 0;
  if (mpsqmc_create(&cfg, &ctx) != MPSQMC_OK ||
      mpsqmc_set_option(ctx, MPSQMC_OPT_PROJECTOR, MPSQMC_PROJECTOR_MPO_TERMS) != MPSQMC_OK) {
    cerr << "MPSQMC: GPU engine unavailable: " << mpsqmc_last_error() << endl;
    if (ctx) mpsqmc_destroy(ctx);
    ctx = nullptr;
  }
}

void MPSQMC::SetupWalkers() {
  if (bSetupWalkers || !ctx) return;
  bSetupWalkers = true;
  const int N = totalNDesiredWalkers;
  const long size = mpsqmc_walker_size(ctx);
  std::vector<double> all((size_t)N * size), ones(N, 1.0), zeros(N, 0.0);
  std::vector<double> w0;
  for (int s = 0; s < Psi0->gLength(); ++s) {
    MPStensor *t = Psi0->gMPStensor(s);
    w0.insert(w0.end(), t->gStorage(),
              t->gStorage() + (long)Psi0->gDimAtBound(s) * Psi0->gDimAtBound(s + 1) * Psi0->gPhys_d());
  }
  for (int w = 0; w < N; ++w) std::copy(w0.begin(), w0.end(), all.begin() + (size_t)w * size);
  if (mpsqmc_set_walkers(ctx, N, all.data(), ones.data(), ones.data(), zeros.data(), 0) != MPSQMC_OK)
    cerr << "MPSQMC: " << mpsqmc_last_error() << endl;
}

double MPSQMC::EnergyFunction() {
  double E = NAN;
  if (!ctx || mpsqmc_energy(ctx, &E) != MPSQMC_OK) cerr << "MPSQMC::EnergyFunction: " << mpsqmc_last_error() << endl;
  return E;
}

void MPSQMC::write(const int step, const double projectedEnergy, const double targetEnergy, const double fluctMetric) {
  std::ofstream output("energies.txt", std::ios::app);
  output.precision(10);
  output << step << "\t\t" << projectedEnergy << "\t\t" << targetEnergy << "\t\t" << fluctMetric << endl;
}

void MPSQMC::Walk(const int steps) {
  if (!ctx) {
    cerr << "MPSQMC::Walk: no GPU engine (see the message at construction)." << endl;
    return;
  }
  const double E = EnergyFunction();
  {
    std::ofstream output("energies.txt", std::ios::trunc);
    output << "#Step\t\tE_P\t\tE_T\t\tFluctMetric" << endl;
  }
  cout << "Energy at start = " << E << endl;
  cout << "---------------------------------------------------------" << endl;
  mpsqmc_set_rng(ctx, RN->gSeed(), RN->gDraws());
  mpsqmc_set_step(ctx, 0);
  for (int step = 1; step <= steps; ++step) {
    mpsqmc_step_stats st;
    if (mpsqmc_walk(ctx, 1, &st) != MPSQMC_OK) {
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
    write(step, st.E_P, st.E_T, st.omega);
    cout << "---------------------------------------------------------" << endl;
  }
}
