// Local spin operators for spin S = (d-1)/2 in the basis m = -S .. S (OpSz.cpp:9, OpSx.cpp:11,
// OpISy.cpp:11-21, OpSup.cpp:11, OpSdown.cpp:14 of the reference define the same matrices).
#include <cmath>

#include "Op0.h"
#include "OpI.h"
#include "OpISy.h"
#include "OpSdown.h"
#include "OpSup.h"
#include "OpSx.h"
#include "OpSz.h"

namespace {
// <m+1| S^+ |m> / 2 for the k-th pair of the ladder, k = 0 .. d-2
double half_ladder(int d, int k) {
  const double S = 0.5 * (d - 1), m = -S + k;
  return 0.5 * std::sqrt(S * (S + 1.0) - m * (m + 1.0));
}
}  // namespace

int Operator::gPhys_d() const { return phys_d; }

ostream &operator<<(ostream &os, const Operator &theOp) {
  os << "Operator, d = " << theOp.gPhys_d() << ", zero = " << theOp.AmIOp0() << ", identity = " << theOp.AmIOpI()
     << endl;
  for (int r = 0; r < theOp.gPhys_d(); ++r) {
    os << "\t";
    for (int c = 0; c < theOp.gPhys_d(); ++c) os << theOp(r, c) << "\t";
    os << endl;
  }
  return os;
}

Op0::Op0(const int d) { phys_d = d; storage = nullptr; }
Op0::~Op0() {}
double Op0::operator()(const int, const int) const { return 0.0; }

OpI::OpI(const int d) { phys_d = d; storage = nullptr; }
OpI::~OpI() {}
double OpI::operator()(const int i, const int j) const { return (i == j && i >= 0 && i < phys_d) ? 1.0 : 0.0; }

OpSz::OpSz(const int d) {
  phys_d = d;
  storage = new double[d];
  for (int k = 0; k < d; ++k) storage[k] = -0.5 * (d - 1) + k;
}
OpSz::~OpSz() { delete[] storage; }
double OpSz::operator()(const int i, const int j) const {
  return (i == j && i >= 0 && i < phys_d) ? storage[i] : 0.0;
}

OpSx::OpSx(const int d) {
  phys_d = d;
  storage = new double[d > 1 ? d - 1 : 1];
  for (int k = 0; k + 1 < d; ++k) storage[k] = half_ladder(d, k);
}
OpSx::~OpSx() { delete[] storage; }
double OpSx::operator()(const int i, const int j) const {
  if (i < 0 || j < 0 || i >= phys_d || j >= phys_d) return 0.0;
  if (i == j + 1) return storage[j];
  if (j == i + 1) return storage[i];
  return 0.0;
}

// i S^y = (S^+ - S^-)/2: +1/2 <m+1|S^+|m> below the diagonal, minus above.
OpISy::OpISy(const int d) {
  phys_d = d;
  storage = new double[d > 1 ? d - 1 : 1];
  for (int k = 0; k + 1 < d; ++k) storage[k] = half_ladder(d, k);
}
OpISy::~OpISy() { delete[] storage; }
double OpISy::operator()(const int i, const int j) const {
  if (i < 0 || j < 0 || i >= phys_d || j >= phys_d) return 0.0;
  if (i == j + 1) return storage[j];
  if (j == i + 1) return -storage[i];
  return 0.0;
}

// S^+ / sqrt(2): raises m, element (k+1, k).
OpSup::OpSup(const int d) {
  phys_d = d;
  storage = new double[d > 1 ? d - 1 : 1];
  for (int k = 0; k + 1 < d; ++k) storage[k] = std::sqrt(2.0) * half_ladder(d, k);
}
OpSup::~OpSup() { delete[] storage; }
double OpSup::operator()(const int i, const int j) const {
  if (i < 0 || j < 0 || i >= phys_d || j >= phys_d) return 0.0;
  return (i == j + 1) ? storage[j] : 0.0;
}

// S^- / sqrt(2): lowers m, element (k, k+1).
OpSdown::OpSdown(const int d) {
  phys_d = d;
  storage = new double[d > 1 ? d - 1 : 1];
  for (int k = 0; k + 1 < d; ++k) storage[k] = std::sqrt(2.0) * half_ladder(d, k);
}
OpSdown::~OpSdown() { delete[] storage; }
double OpSdown::operator()(const int i, const int j) const {
  if (i < 0 || j < 0 || i >= phys_d || j >= phys_d) return 0.0;
  return (j == i + 1) ? storage[i] : 0.0;
}
