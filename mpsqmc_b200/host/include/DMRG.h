// DMRG: two-site ground-state solver that overwrites the given MPS (same bond dimensions) with
// the lowest-energy state of the MPO and returns its energy.  Interface of the reference's
// include/DMRG.h:11-23.  Environments of the MPO replace the reference's full MPO x MPS product,
// and a Lanczos iteration replaces Davidson.
#ifndef DMRG_H
#define DMRG_H

#include "MPO.h"
#include "MPSstate.h"
#include "MPStensor.h"
#include "TwoSiteObject.h"

class DMRG {
 public:
  DMRG(MPSstate *MPStrial, MPO *theMPO);
  ~DMRG();
  double Solve();

 private:
  MPSstate *MPSsolution;
  MPO *theMPO;
  int length;
};

#endif
