// OpSdown: the local operator S^- / sqrt(2) for spin (d-1)/2, basis ordered m = -S .. S.
// Interface of the reference's include/OpSdown.h (drop-in for main.cpp and MPSQMC2).
#ifndef OPSDOWN_H
#define OPSDOWN_H

#include "Operator.h"

class OpSdown : public Operator {
 public:
  OpSdown(const int phys_d);
  ~OpSdown();
  double operator()(const int i, const int j) const;
  bool AmIOp0() const { return false; }
  bool AmIOpI() const { return false; }
};

#endif
