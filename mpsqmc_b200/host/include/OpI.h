// OpI: the local operator identity for spin (d-1)/2, basis ordered m = -S .. S.
// Interface of the reference's include/OpI.h (drop-in for main.cpp and MPSQMC2).
#ifndef OPI_H
#define OPI_H

#include "Operator.h"

class OpI : public Operator {
 public:
  OpI(const int phys_d);
  ~OpI();
  double operator()(const int i, const int j) const;
  bool AmIOp0() const { return false; }
  bool AmIOpI() const { return true; }
};

#endif
