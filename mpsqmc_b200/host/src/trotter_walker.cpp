// TrotterHeisenberg (propagator factor tables) and Walker (host-side walker object).
#include <cmath>

#include "TrotterHeisenberg.h"
#include "Walker.h"
#include "linalg.h"

TrotterHeisenberg::TrotterHeisenberg(HeisenbergMPO *mpo, double dt) {
  length = mpo->gLength();
  phys_d = mpo->gPhys_d();
  dtau = dt;
  couplingMx.assign((size_t)length * (length - 1) / 2 + 1, 0.0);
  for (int a = 0; a < length; ++a)
    for (int b = a + 1; b < length; ++b) {
      const double J = mpo->gCoupling(a, b);
      couplingMx[(size_t)(b * (b - 1)) / 2 + a] = J;
      if (J != 0.0 && find(J) < 0) Jvals.push_back(J);
    }
  theField = mpo->gField();
  isMagneticField = theField != 0.0;
  OpSz sz(phys_d);
  single.assign(phys_d, 1.0);
  if (isMagneticField)
    for (int s = 0; s < phys_d; ++s) single[s] = std::exp(0.5 * theField * dtau * sz(s, s));
  cout << "TrotterHeisenberg --> distinct couplings J_ij:";
  for (double J : Jvals) cout << " " << J;
  cout << "; field h = " << theField << endl;
  SetTheTwoSitePropagators();
}

TrotterHeisenberg::~TrotterHeisenberg() {}

int TrotterHeisenberg::find(const double J) const {
  for (size_t q = 0; q < Jvals.size(); ++q)
    if (Jvals[q] == J) return (int)q;
  return -1;
}

// exp(-dtau J S_1.S_2) from the eigen-decomposition of S_1.S_2, reshuffled to
// [(row1, col1), (row2, col2)] and split by an SVD into sum_k U_k (x) s_k V_k
// (TrotterHeisenberg.cpp:102-285).
void TrotterHeisenberg::SetTheTwoSitePropagators() {
  const int d = phys_d, n = d * d;
  OpSx sx(d);
  OpISy isy(d);
  OpSz sz(d);
  std::vector<double> H((size_t)n * n);
  for (int r1 = 0; r1 < d; ++r1)
    for (int c1 = 0; c1 < d; ++c1)
      for (int r2 = 0; r2 < d; ++r2)
        for (int c2 = 0; c2 < d; ++c2)
          H[(r1 + d * r2) + (size_t)n * (c1 + d * c2)] =
              sx(r1, c1) * sx(r2, c2) - isy(r1, c1) * isy(r2, c2) + sz(r1, c1) * sz(r2, c2);
  std::vector<double> lam, V;
  mqh::sym_eig(n, H, lam, V);
  U.assign(Jvals.size(), {});
  S.assign(Jvals.size(), {});
  VT.assign(Jvals.size(), {});
  for (size_t q = 0; q < Jvals.size(); ++q) {
    std::vector<double> W((size_t)n * n), P((size_t)n * n), Q((size_t)n * n);
    for (int c = 0; c < n; ++c) {
      const double f = std::exp(-0.5 * dtau * Jvals[q] * lam[c]);
      for (int r = 0; r < n; ++r) W[r + (size_t)n * c] = f * V[r + (size_t)n * c];
    }
    mqh::gemm(false, true, n, n, n, 1.0, W.data(), n, W.data(), n, 0.0, P.data(), n);
    for (int r1 = 0; r1 < d; ++r1)
      for (int c1 = 0; c1 < d; ++c1)
        for (int r2 = 0; r2 < d; ++r2)
          for (int c2 = 0; c2 < d; ++c2)
            Q[(r1 + d * c1) + (size_t)n * (r2 + d * c2)] = P[(r1 + d * r2) + (size_t)n * (c1 + d * c2)];
    mqh::svd(n, n, Q.data(), U[q], S[q], VT[q]);
  }
}

bool TrotterHeisenberg::gIsMagneticField() const { return isMagneticField; }
double TrotterHeisenberg::gField() const { return theField; }
int TrotterHeisenberg::gNDifferentCouplings() const { return (int)Jvals.size(); }
double TrotterHeisenberg::gDifferentCoupling(const int q) const { return Jvals[q]; }

double TrotterHeisenberg::gCoupling(const int i, const int j) const {
  if (i == j || i < 0 || i >= length || j < 0 || j >= length) {
    cerr << "TrotterHeisenberg::gCoupling  :  The combination of indices (" << i << "," << j << ") is not OK." << endl;
    return NAN;
  }
  const int a = i < j ? i : j, b = i < j ? j : i;
  return couplingMx[(size_t)(b * (b - 1)) / 2 + a];
}

double TrotterHeisenberg::gTwoSitePropSVD_Sing(const double J, const int k) const {
  const int q = find(J);
  if (k < 0 || k >= phys_d * phys_d || q < 0) return NAN;
  return S[q][k];
}
double TrotterHeisenberg::gTwoSitePropSVD_Left(const double J, const int k, const int i, const int j) const {
  const int q = find(J);
  if (k < 0 || k >= phys_d * phys_d || q < 0 || i < 0 || j < 0 || i >= phys_d || j >= phys_d) return NAN;
  return U[q][i + phys_d * (j + phys_d * k)];
}
double TrotterHeisenberg::gTwoSitePropSVD_Right(const double J, const int k, const int i, const int j) const {
  const int q = find(J);
  if (k < 0 || k >= phys_d * phys_d || q < 0 || i < 0 || j < 0 || i >= phys_d || j >= phys_d) return NAN;
  return VT[q][k + phys_d * phys_d * (i + phys_d * j)];
}
double TrotterHeisenberg::gSingleSiteProp(const int i, const int j) const {
  if (i < 0 || i >= phys_d || j < 0 || j >= phys_d) return NAN;
  return i == j ? single[i] : 0.0;
}

Walker::Walker(MPSstate *s, const double ov, const double w, const double eh)
    : theState(new MPSstate(s)), overlap(ov), weight(w), energyHistory(eh) {}
Walker::Walker(Walker *o)
    : theState(new MPSstate(o->gState())), overlap(o->gOverlap()), weight(o->gWeight()),
      energyHistory(o->gEnergyHistory()) {}
Walker::Walker(const int L, const int D, const int d, Random *RN)
    : theState(new MPSstate(L, D, d, RN)), overlap(NAN), weight(1.0), energyHistory(0.0) {}
Walker::~Walker() { delete theState; }
double Walker::gWeight() const { return weight; }
double Walker::gOverlap() const { return overlap; }
double Walker::gEnergyHistory() const { return energyHistory; }
MPSstate *Walker::gState() { return theState; }
void Walker::setWeight(const double w) { weight = w; }
void Walker::multiplyWeight(const double f) { weight *= f; }
void Walker::setEnergyHistory(const double e) { energyHistory = e; }
void Walker::addEnergyToHistory(const double e) { energyHistory += e; }
// LeftNormalize, overlap with the trial, and a sign flip if it is negative (Walker.cpp:54-66).
void Walker::setOverlap(MPSstate *trial) {
  theState->LeftNormalize();
  double v = trial->InnerProduct(theState);
  if (v < 0.0) {
    theState->ChangePhase();
    v = -v;
  }
  overlap = v;
}
double Walker::calcIndividualProjectedEnergy(MPSstate *HT) { return HT->InnerProduct(theState) / overlap; }
