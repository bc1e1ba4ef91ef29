// MPSQMC2: the MPS-walker projector QMC driver.  Interface of the reference's
// include/MPSQMC2.h:13-28: the two constructors and Walk().  The population lives on the GPU
// (libmpsqmc_b200.so, include/mpsqmc_gpu.h); Walk() prints and writes the same per-step
// records as the reference (MPSQMC2.cpp:449-498, 749-758).
#ifndef MPSQMC2_H
#define MPSQMC2_H

#include <cstdio>

#include "DMRG.h"
#include "GridGenerator.h"
#include "HeisenbergMPO.h"
#include "MPSstate.h"
#include "TrotterHeisenberg.h"
#include "Walker.h"

struct mpsqmc_ctx;

class MPSQMC2 {
 public:
  MPSQMC2(HeisenbergMPO *theMPO, GridGenerator *theGrid, Random *RN, const int DT, const int DW,
          const int Nwalkers, const double dtau);
  MPSQMC2(HeisenbergMPO *theMPO, GridGenerator *theGrid, Random *RN, MPSstate *Psi0_in, const int DW,
          const int Nwalkers, const double dtau);
  ~MPSQMC2();
  void Walk(const int steps);

 private:
  void Setup(MPSstate *trial);
  void write(const int step, const int nwalkers, const double projectedEnergy, const double targetEnergy,
             const double fluctMetric);
  HeisenbergMPO *theMPO;
  TrotterHeisenberg *theTrotter;
  GridGenerator *theGrid;
  Random *RN;
  int DT, DW;
  int totalNDesiredWalkers;
  double dtau;
  MPSstate *Psi0;
  mpsqmc_ctx *ctx;
};

#endif
