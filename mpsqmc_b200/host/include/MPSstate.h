// MPSstate: a matrix product state of `length` sites with bond dims VirtualD[0..length].
// Interface of the reference's include/MPSstate.h:15-100 (constructors, canonical forms,
// overlaps, compression, MPO and Trotter-term application, text output).
#ifndef MPSSTATE_H
#define MPSSTATE_H

#include <vector>

#include "GridGenerator.h"
#include "MPO.h"
#include "MPStensor.h"
#include "TrotterHeisenberg.h"
#include "TwoSiteObject.h"

class MPSstate {
  friend ostream &operator<<(ostream &output, MPSstate &mps);

 public:
  MPSstate(const int length, const int Dtrunc, const int phys_d, Random *RN);
  MPSstate(const int length, const int Dtrunc, const int phys_d, int *VirtualDims, Random *RN);
  MPSstate(MPSstate *toCopy);
  MPSstate(const char *filename, Random *RN);
  ~MPSstate();
  int gDtrunc() const;
  int gDimAtBound(const int bound) const;
  void printVdim() const;
  int gPhys_d() const;
  int gLength() const;
  MPStensor *gMPStensor(const int site);
  Random *gRN();
  double LeftNormalize();
  double RightNormalize();
  double InnerProduct(MPSstate *OtherState);
  void ScalarMultiplication(const double factor);
  void ResetContentsAndStoreSumOf(MPSstate *state1, MPSstate *state2);
  void ChangePhase();
  void CompressState(const int truncD);
  void CompressState() { CompressState(Dtrunc); }
  void ApplyMPO(MPO *theMPO, MPSstate *Psi0);
  void ApplyMPOterm(MPO *theMPO, const int SelectedTerm);
  void ApplyMPOtermHC(MPO *theMPO, const int SelectedTerm) {
    ApplyMPOterm(theMPO, theMPO->gRN_HCfriend(SelectedTerm));
  }
  void ApplyTwoSiteTrotterTerm(TrotterHeisenberg *theTrotter, const int firstSite, const int secondSite,
                               const int leftSVDindex, const int rightSVDindex, const bool doHC = false);
  void ApplyTwoSiteTrotterTerm(TrotterHeisenberg *theTrotter, const int firstSite, const int secondSite,
                               GridGenerator *theGrid, const int gridPoint);
  void ApplyOneSiteTrotterTermEverywhere(TrotterHeisenberg *theTrotter);
  void checkWork1(const int size);
  void checkWork2(const int size);
  void checkWork3(const int size);
  double *gWork1() { return work1.data(); }
  double *gWork2() { return work2.data(); }
  double *gWork3() { return work3.data(); }

 private:
  Random *RN;
  int length, Dtrunc, phys_d;
  std::vector<MPStensor *> theTensors;
  std::vector<int> VirtualD;
  std::vector<double> work1, work2, work3;
  void allocate(Random *RN);
  void applySiteOperator(const int site, const double *op);  // op[up + d * down]
};

#endif
