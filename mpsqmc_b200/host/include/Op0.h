// Op0: the local operator zero operator for spin (d-1)/2, basis ordered m = -S .. S.
// Interface of the reference's include/Op0.h (drop-in for main.cpp and MPSQMC2).
#ifndef OP0_H
#define OP0_H

#include "Operator.h"

class Op0 : public Operator {
 public:
  Op0(const int phys_d);
  ~Op0();
  double operator()(const int i, const int j) const;
  bool AmIOp0() const { return true; }
  bool AmIOpI() const { return false; }
};

#endif
