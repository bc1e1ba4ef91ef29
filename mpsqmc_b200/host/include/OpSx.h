// OpSx: the local operator S^x for spin (d-1)/2, basis ordered m = -S .. S.
// Interface of the reference's include/OpSx.h (drop-in for main.cpp and MPSQMC2).
#ifndef OPSX_H
#define OPSX_H

#include "Operator.h"

class OpSx : public Operator {
 public:
  OpSx(const int phys_d);
  ~OpSx();
  double operator()(const int i, const int j) const;
  bool AmIOp0() const { return false; }
  bool AmIOpI() const { return false; }
};

#endif
