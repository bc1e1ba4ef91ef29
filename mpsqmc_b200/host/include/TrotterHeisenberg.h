// TrotterHeisenberg: factorisation of the two-site propagator exp(-dtau J S_i.S_j) into sums of
// products of one-site operators (an SVD of the reshuffled d^2 x d^2 matrix), and the one-site
// field propagator exp(dtau h S^z / 2).  Interface of the reference's
// include/TrotterHeisenberg.h:14-40, with U[i + d (j + d k)] and VT[k + d^2 (i + d j)].
#ifndef TROTTERHEISENBERG_H
#define TROTTERHEISENBERG_H

#include <vector>

#include "HeisenbergMPO.h"
#include "OpISy.h"
#include "OpSx.h"
#include "OpSz.h"

class TrotterHeisenberg {
 public:
  TrotterHeisenberg(HeisenbergMPO *theMPO, double dtau);
  ~TrotterHeisenberg();
  bool gIsMagneticField() const;
  double gField() const;
  double gCoupling(const int i, const int j) const;
  double gTwoSitePropSVD_Sing(const double J, const int k) const;
  double gTwoSitePropSVD_Left(const double J, const int k, const int i, const int j) const;
  double gTwoSitePropSVD_Right(const double J, const int k, const int i, const int j) const;
  double gSingleSiteProp(const int i, const int j) const;
  // tables of every distinct coupling, in the order first met (i < j, i ascending)
  int gNDifferentCouplings() const;
  double gDifferentCoupling(const int q) const;

 private:
  int length, phys_d;
  double dtau, theField;
  bool isMagneticField;
  std::vector<double> couplingMx;
  std::vector<double> Jvals;
  std::vector<std::vector<double> > U, S, VT;
  std::vector<double> single;
  int find(const double J) const;
  void SetTheTwoSitePropagators();
};

#endif
