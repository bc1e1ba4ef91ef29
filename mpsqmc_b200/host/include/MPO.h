// MPO: an operator as a chain of dimL(site) x dimR(site) operator-valued matrices, plus the
// list of its nonzero product terms.  Interface of the reference's include/MPO.h:13-76.
#ifndef MPO_H
#define MPO_H

#include <stdlib.h>
#include <iostream>

#include "Operator.h"

using namespace std;

class MPO {
 public:
  virtual ~MPO() {}
  int gPhys_d() const;
  int gLength() const;
  int dimL(const int site) const;
  int dimR(const int site) const;
  virtual double gPrefactor(const int site, const int row, const int col) const = 0;
  virtual Operator *gOperator(const int site, const int row, const int col) const = 0;
  int gRN_nTerms() const;
  double gRN_prefactor(const int count) const;
  Operator *gRN_operator(const int count, const int site) const;
  int gRN_HCfriend(const int index) const;

 protected:
  // The MPO dimensions are derived lazily from the current couplings; subclasses keep them
  // up to date in refresh().
  virtual void refresh() const {}
  int length;
  int phys_d;
  mutable int *MPOdimensions;
  int RN_nTerms;
  double *RN_prefactors;
  Operator ***RN_operators;
  int *RN_HCfriends;
};

#endif
