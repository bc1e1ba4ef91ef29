// OpSz: the local operator S^z for spin (d-1)/2, basis ordered m = -S .. S.
// Interface of the reference's include/OpSz.h (drop-in for main.cpp and MPSQMC2).
#ifndef OPSZ_H
#define OPSZ_H

#include "Operator.h"

class OpSz : public Operator {
 public:
  OpSz(const int phys_d);
  ~OpSz();
  double operator()(const int i, const int j) const;
  bool AmIOp0() const { return false; }
  bool AmIOpI() const { return false; }
};

#endif
