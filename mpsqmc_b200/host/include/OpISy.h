// OpISy: the local operator i S^y (real: S^+ part minus S^- part) for spin (d-1)/2, basis ordered m = -S .. S.
// Interface of the reference's include/OpISy.h (drop-in for main.cpp and MPSQMC2).
#ifndef OPISY_H
#define OPISY_H

#include "Operator.h"

class OpISy : public Operator {
 public:
  OpISy(const int phys_d);
  ~OpISy();
  double operator()(const int i, const int j) const;
  bool AmIOp0() const { return false; }
  bool AmIOpI() const { return false; }
};

#endif
