// HeisenbergMPO: H = sum_{i<j} J_ij S_i.S_j - h sum_i S^z_i as an MPO.
// Interface of the reference's include/HeisenbergMPO.h:16-104 (same constructor and accessors,
// so couplings set after construction take effect as in the reference).  The MPO itself is the
// compact form: channel 0 = finished terms, channels 1..3n = (site i, operator) waiting for a
// partner j >= bond, last channel = nothing placed yet; its bond dimension is 2 + 3 * (number of
// sites left of the bond that couple across it) instead of the reference's 2 + 3 min(k, L-k).
#ifndef HEISENBERGMPO_H
#define HEISENBERGMPO_H

#include <stdlib.h>
#include <iostream>
#include <vector>

#include "MPO.h"
#include "Op0.h"
#include "OpI.h"
#include "OpISy.h"
#include "OpSdown.h"
#include "OpSup.h"
#include "OpSx.h"
#include "OpSz.h"

using namespace std;

class HeisenbergMPO : public MPO {
 public:
  HeisenbergMPO(const int length, const int phys_d, const bool useLadder);
  ~HeisenbergMPO();
  void fillMPOdimensions();
  void fillMPOprefactorsMPOoperators();
  double gPrefactor(const int site, const int row, const int col) const;
  Operator *gOperator(const int site, const int row, const int col) const;
  double gCoupling(const int i, const int j) const;
  double gField() const;
  void sCoupling(const int i, const int j, const double value);
  void sField(const double value);
  void printOperators(ostream &os) const;
  void printOperatorTag(ostream &os, Operator *theOp) const;
  friend ostream &operator<<(ostream &os, const HeisenbergMPO &theMPO);
  void findNonZeroContributions();

 private:
  struct Entry {
    int row, col;
    double prefactor;
    Operator *op;
  };
  void refresh() const;
  bool useLadder;
  double fZero, fOne;
  Op0 *opZero;
  OpI *opOne;
  OpSx *opSx;
  OpISy *opISy;
  OpSz *opSz;
  OpSup *opSplus;
  OpSdown *opSminus;
  double MinusH;
  double *couplingMatrix;
  mutable bool dirty;
  mutable std::vector<std::vector<Entry> > entries;  // per site
};

#endif
