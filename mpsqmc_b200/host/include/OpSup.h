// OpSup: the local operator S^+ / sqrt(2) for spin (d-1)/2, basis ordered m = -S .. S.
// Interface of the reference's include/OpSup.h (drop-in for main.cpp and MPSQMC2).
#ifndef OPSUP_H
#define OPSUP_H

#include "Operator.h"

class OpSup : public Operator {
 public:
  OpSup(const int phys_d);
  ~OpSup();
  double operator()(const int i, const int j) const;
  bool AmIOp0() const { return false; }
  bool AmIOpI() const { return false; }
};

#endif
