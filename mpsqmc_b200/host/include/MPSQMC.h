// MPSQMC: the MPO-term projector QMC driver (1 - dtau H sampled one MPO term at a time).
// Interface of the reference's include/MPSQMC.h:10-31: constructor, SetupTrial, SetupWalkers,
// EnergyFunction, Walk.  The population lives on the GPU (include/mpsqmc_gpu.h, projector
// MPSQMC_PROJECTOR_MPO_TERMS); Walk() prints and writes the same per-step records as the
// reference (MPSQMC.cpp:236-318, 474-481).  The MPO must be a HeisenbergMPO with its term list
// built (findNonZeroContributions), as the reference's sampling requires.
#ifndef MPSQMC_H
#define MPSQMC_H

#include "DMRG.h"
#include "MPO.h"
#include "MPSstate.h"

struct mpsqmc_ctx;

class MPSQMC {
 public:
  MPSQMC(MPO *theMPO, Random *RN, const int Dtrunc, const int Nwalkers, const double dtau);
  ~MPSQMC();
  void SetupTrial();
  void SetupWalkers();
  double EnergyFunction();
  void Walk(const int steps);

 private:
  void write(const int step, const double projectedEnergy, const double targetEnergy, const double fluctMetric);
  MPO *theMPO;
  Random *RN;
  int Dtrunc;
  int totalNDesiredWalkers;
  double dtau;
  bool bSetupTrial, bSetupWalkers;
  MPSstate *Psi0;
  mpsqmc_ctx *ctx;
};

#endif
