// MPO base accessors and the compact Heisenberg MPO.
#include <cmath>

#include "HeisenbergMPO.h"

int MPO::gPhys_d() const { return phys_d; }
int MPO::gLength() const { return length; }
int MPO::dimL(const int site) const {
  if (site < 0 || site >= length) return 0;
  refresh();
  return MPOdimensions[site];
}
int MPO::dimR(const int site) const {
  if (site < 0 || site >= length) return 0;
  refresh();
  return MPOdimensions[site + 1];
}
int MPO::gRN_nTerms() const { return RN_nTerms; }
double MPO::gRN_prefactor(const int count) const {
  return (count < 0 || count >= RN_nTerms) ? 0.0 : RN_prefactors[count];
}
Operator *MPO::gRN_operator(const int count, const int site) const {
  if (count < 0 || count >= RN_nTerms || site < 0 || site >= length) return nullptr;
  return RN_operators[count][site];
}
int MPO::gRN_HCfriend(const int index) const {
  return (index < 0 || index >= RN_nTerms) ? -1 : RN_HCfriends[index];
}

HeisenbergMPO::HeisenbergMPO(const int L, const int d, const bool ladder) {
  if (L < 3) cerr << "HeisenbergMPO::HeisenbergMPO  :  The length must be at least three." << endl;
  length = L;
  phys_d = d;
  useLadder = ladder;
  fZero = 0.0;
  fOne = 1.0;
  opZero = new Op0(d);
  opOne = new OpI(d);
  opSx = new OpSx(d);
  opISy = new OpISy(d);
  opSz = new OpSz(d);
  opSplus = new OpSup(d);
  opSminus = new OpSdown(d);
  MinusH = -0.0;
  couplingMatrix = new double[(L * (L - 1)) / 2 + 1];
  for (int q = 0; q < (L * (L - 1)) / 2; ++q) couplingMatrix[q] = 0.0;
  MPOdimensions = new int[L + 1];
  RN_nTerms = 0;
  RN_prefactors = nullptr;
  RN_operators = nullptr;
  RN_HCfriends = nullptr;
  dirty = true;
  refresh();
}

HeisenbergMPO::~HeisenbergMPO() {
  delete opZero;
  delete opOne;
  delete opSx;
  delete opISy;
  delete opSz;
  delete opSplus;
  delete opSminus;
  delete[] couplingMatrix;
  delete[] MPOdimensions;
  if (RN_nTerms > 0) {
    delete[] RN_prefactors;
    for (int t = 0; t < RN_nTerms; ++t) delete[] RN_operators[t];
    delete[] RN_operators;
    delete[] RN_HCfriends;
  }
}

void HeisenbergMPO::fillMPOdimensions() { dirty = true; refresh(); }
void HeisenbergMPO::fillMPOprefactorsMPOoperators() { dirty = true; refresh(); }

void HeisenbergMPO::sField(const double value) {
  MinusH = -value;
  dirty = true;
}
double HeisenbergMPO::gField() const { return -MinusH; }

void HeisenbergMPO::sCoupling(const int i, const int j, const double value) {
  if (i == j || i < 0 || i >= length || j < 0 || j >= length) {
    cerr << "HeisenbergMPO::sCoupling  :  The combination of indices (" << i << "," << j << ") is not OK." << endl;
    return;
  }
  const int a = i < j ? i : j, b = i < j ? j : i;
  couplingMatrix[(b * (b - 1)) / 2 + a] = value;
  dirty = true;
}

double HeisenbergMPO::gCoupling(const int i, const int j) const {
  if (i == j || i < 0 || i >= length || j < 0 || j >= length) {
    cerr << "HeisenbergMPO::gCoupling  :  The combination of indices (" << i << "," << j << ") is not OK." << endl;
    return NAN;
  }
  const int a = i < j ? i : j, b = i < j ? j : i;
  return couplingMatrix[(b * (b - 1)) / 2 + a];
}

// Rebuild the compact MPO from the current couplings and field.
void HeisenbergMPO::refresh() const {
  if (!dirty) return;
  const int L = length;
  // open[b]: sites i < b with a nonzero coupling to some j >= b
  std::vector<std::vector<int> > open(L + 1);
  for (int b = 1; b < L; ++b)
    for (int i = 0; i < b; ++i)
      for (int j = b; j < L; ++j)
        if (gCoupling(i, j) != 0.0) {
          open[b].push_back(i);
          break;
        }
  MPOdimensions[0] = 1;
  MPOdimensions[L] = 1;
  for (int b = 1; b < L; ++b) MPOdimensions[b] = 2 + 3 * (int)open[b].size();
  auto done = [](int) { return 0; };  // the "done" channel is index 0 on every bond
  auto start = [&](int b) { return b == 0 ? 0 : 1 + 3 * (int)open[b].size(); };
  auto chan = [&](int b, int i, int op) {
    for (size_t q = 0; q < open[b].size(); ++q)
      if (open[b][q] == i) return 1 + 3 * (int)q + op;
    return -1;
  };
  Operator *left[3], *right[3];
  double sgn[3];
  if (useLadder) {
    left[0] = opSplus, right[0] = opSminus, sgn[0] = 1.0;
    left[1] = opSminus, right[1] = opSplus, sgn[1] = 1.0;
  } else {
    left[0] = opSx, right[0] = opSx, sgn[0] = 1.0;
    left[1] = opISy, right[1] = opISy, sgn[1] = -1.0;  // S^y S^y = -(iS^y)(iS^y)
  }
  left[2] = opSz, right[2] = opSz, sgn[2] = 1.0;
  entries.assign(L, std::vector<Entry>());
  const double h = -MinusH;
  for (int k = 0; k < L; ++k) {
    std::vector<Entry> &e = entries[k];
    const bool last = (k == L - 1);
    if (k > 0) e.push_back({done(k), done(k + 1), 1.0, opOne});
    if (h != 0.0) e.push_back({start(k), done(k + 1), MinusH, opSz});
    if (!last) e.push_back({start(k), start(k + 1), 1.0, opOne});
    for (int op = 0; op < 3; ++op) {
      const int c = chan(k + 1, k, op);
      if (c >= 0) e.push_back({start(k), c, 1.0, left[op]});
    }
    for (size_t q = 0; q < open[k].size(); ++q) {
      const int i = open[k][q];
      const double J = gCoupling(i, k);
      for (int op = 0; op < 3; ++op) {
        const int src = chan(k, i, op);
        if (J != 0.0) e.push_back({src, done(k + 1), sgn[op] * J, right[op]});
        const int dst = chan(k + 1, i, op);
        if (dst >= 0) e.push_back({src, dst, 1.0, opOne});
      }
    }
  }
  dirty = false;
}

double HeisenbergMPO::gPrefactor(const int site, const int row, const int col) const {
  if (site < 0 || site >= length || row < 0 || row >= dimL(site) || col < 0 || col >= dimR(site)) return 0.0;
  refresh();
  for (const Entry &e : entries[site])
    if (e.row == row && e.col == col) return e.prefactor;
  return 0.0;
}

Operator *HeisenbergMPO::gOperator(const int site, const int row, const int col) const {
  if (site < 0 || site >= length || row < 0 || row >= dimL(site) || col < 0 || col >= dimR(site)) return nullptr;
  refresh();
  for (const Entry &e : entries[site])
    if (e.row == row && e.col == col) return e.prefactor == 0.0 ? (Operator *)opZero : e.op;
  return opZero;
}

void HeisenbergMPO::printOperatorTag(ostream &os, Operator *op) const {
  if (op == opZero) os << "0";
  else if (op == opOne) os << "I";
  else if (op == opSx) os << "Sx";
  else if (op == opISy) os << "iSy";
  else if (op == opSz) os << "Sz";
  else if (op == opSplus) os << "S+/sqrt2";
  else if (op == opSminus) os << "S-/sqrt2";
  else os << "?";
}

void HeisenbergMPO::printOperators(ostream &os) const {
  os << *opZero << *opOne << *opSz;
  if (useLadder) os << *opSplus << *opSminus;
  else os << *opSx << *opISy;
}

ostream &operator<<(ostream &os, const HeisenbergMPO &m) {
  os << "HeisenbergMPO: L = " << m.gLength() << ", d = " << m.gPhys_d() << ", h = " << m.gField() << endl;
  for (int k = 0; k < m.gLength(); ++k) {
    os << "  site " << k << " (" << m.dimL(k) << " x " << m.dimR(k) << "):";
    m.refresh();
    for (const auto &e : m.entries[k]) {
      os << "  [" << e.row << "," << e.col << "] " << e.prefactor << " ";
      m.printOperatorTag(os, e.op);
    }
    os << endl;
  }
  for (int t = 0; t < m.gRN_nTerms(); ++t) {
    os << "  term " << t << ": " << m.gRN_prefactor(t) << " x";
    for (int k = 0; k < m.gLength(); ++k) {
      Operator *op = m.gRN_operator(t, k);
      if (op != m.opOne) {
        os << " ";
        m.printOperatorTag(os, op);
        os << "_" << k;
      }
    }
    os << "  (hc: " << m.gRN_HCfriend(t) << ")" << endl;
  }
  return os;
}

// The nonzero product terms of H: -h S^z_k for every site, and for every coupling the three
// products of the chosen operator basis (HeisenbergMPO.cpp:413-609 enumerates the same terms
// from the MPO paths).
void HeisenbergMPO::findNonZeroContributions() {
  if (RN_nTerms > 0) {
    delete[] RN_prefactors;
    for (int t = 0; t < RN_nTerms; ++t) delete[] RN_operators[t];
    delete[] RN_operators;
    delete[] RN_HCfriends;
    RN_nTerms = 0;
  }
  struct Term { double f; int i, j; Operator *a, *b; int hc; };
  std::vector<Term> terms;
  const double h = -MinusH;
  if (h != 0.0)
    for (int k = 0; k < length; ++k) terms.push_back({MinusH, k, -1, opSz, nullptr, -1});
  for (int i = 0; i < length; ++i)
    for (int j = i + 1; j < length; ++j) {
      const double J = gCoupling(i, j);
      if (J == 0.0) continue;
      const int base = (int)terms.size();
      if (useLadder) {
        terms.push_back({J, i, j, opSplus, opSminus, base + 1});
        terms.push_back({J, i, j, opSminus, opSplus, base});
      } else {
        terms.push_back({J, i, j, opSx, opSx, base});
        terms.push_back({-J, i, j, opISy, opISy, base + 1});
      }
      terms.push_back({J, i, j, opSz, opSz, base + 2});
    }
  RN_nTerms = (int)terms.size();
  if (RN_nTerms == 0) return;
  RN_prefactors = new double[RN_nTerms];
  RN_operators = new Operator **[RN_nTerms];
  RN_HCfriends = new int[RN_nTerms];
  for (int t = 0; t < RN_nTerms; ++t) {
    RN_prefactors[t] = terms[t].f;
    RN_operators[t] = new Operator *[length];
    for (int k = 0; k < length; ++k) RN_operators[t][k] = opOne;
    RN_operators[t][terms[t].i] = terms[t].a;
    if (terms[t].j >= 0) RN_operators[t][terms[t].j] = terms[t].b;
    RN_HCfriends[t] = terms[t].hc < 0 ? t : terms[t].hc;
  }
}
