// Operator: a d x d local operator; element (i, j) acts as C_i = sum_j Op(i, j) C_j.
// Interface of the reference's include/Operator.h:13-41.
#ifndef OPERATOR_H
#define OPERATOR_H

#include <stdlib.h>
#include <iostream>

using namespace std;

class Operator {
 public:
  virtual ~Operator() {}
  int gPhys_d() const;
  virtual double operator()(const int i, const int j) const = 0;
  friend ostream &operator<<(ostream &os, const Operator &theOp);
  virtual bool AmIOp0() const = 0;
  virtual bool AmIOpI() const = 0;

 protected:
  int phys_d;
  double *storage;
};

#endif
