// Walker: one walker of the population (its MPS, weight, overlap with the trial, energy
// history).  Interface of the reference's include/Walker.h:9-55.  MPSQMC2 keeps its walkers on
// the GPU; this class serves host-side code that handles individual walkers.
#ifndef WALKER_H
#define WALKER_H

#include "MPSstate.h"

class Walker {
 public:
  Walker(MPSstate *theState, const double overlap, const double weight, const double energyHistory);
  Walker(Walker *theWalker);
  Walker(const int length, const int Dtrunc, const int phys_d, Random *RN);
  ~Walker();
  double gWeight() const;
  double gOverlap() const;
  double gEnergyHistory() const;
  MPSstate *gState();
  void setWeight(const double weight);
  void multiplyWeight(const double factor);
  void setOverlap(MPSstate *theTrial);
  void setEnergyHistory(const double energyHistory);
  void addEnergyToHistory(const double term);
  double calcIndividualProjectedEnergy(MPSstate *HamTimesTrial);

 private:
  MPSstate *theState;
  double overlap, weight, energyHistory;
};

#endif
