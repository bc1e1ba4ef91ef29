// MPStensor, TwoSiteObject and MPSstate: host-side MPS algebra for set-up and for callers that
// handle single states.  Storage of a site: [r + dimL * (c + dimR * sigma)].
#include <cmath>
#include <cstring>
#include <fstream>

#include "MPSstate.h"
#include "Operator.h"
#include "linalg.h"

using std::endl;

// ---------------------------------------------------------------------------------------------
// MPStensor
// ---------------------------------------------------------------------------------------------
MPStensor::MPStensor(const int dL, const int dR, const int d, Random *rn)
    : RN(rn), dimL(dL), dimR(dR), phys_d(d), storageSize(dL * dR * d) {
  storage = new double[storageSize];
  random();
}

MPStensor::MPStensor(MPStensor *o)
    : RN(o->gRN()), dimL(o->gDimL()), dimR(o->gDimR()), phys_d(o->gPhys_d()), storageSize(o->gStorageSize()) {
  storage = new double[storageSize];
  std::memcpy(storage, o->gStorage(), sizeof(double) * storageSize);
}

MPStensor::MPStensor(const char *filename, Random *rn) : RN(rn) {
  ifstream in(filename);
  in >> dimL >> phys_d >> dimR >> storageSize;
  storage = new double[storageSize];
  for (int i = 0; i < storageSize; ++i) {
    int idx;
    in >> idx >> storage[i];
  }
}

MPStensor::~MPStensor() { delete[] storage; }

// Random fill with two draws per element: a sign, then a magnitude (MPStensor.cpp:75-79).
void MPStensor::random() {
  for (int q = 0; q < storageSize; ++q) {
    const double s = (RN->rand() < 0.5) ? -1.0 : 1.0;
    storage[q] = s * RN->rand();
  }
}

void MPStensor::Reset(const int dL, const int dR) {
  dimL = dL;
  dimR = dR;
  if (dL * dR * phys_d > storageSize) {
    storageSize = dL * dR * phys_d;
    delete[] storage;
    storage = new double[storageSize];
  }
  random();
}

int MPStensor::gDimL() const { return dimL; }
int MPStensor::gDimR() const { return dimR; }
int MPStensor::gPhys_d() const { return phys_d; }
int MPStensor::gStorageSize() const { return storageSize; }
double *MPStensor::gStorage() { return storage; }
double *MPStensor::gStorage(const int d_val) {
  if (d_val < 0 || d_val >= phys_d) return nullptr;
  return storage + d_val * dimL * dimR;
}
Random *MPStensor::gRN() { return RN; }

// Left-orthonormalise: the (dimL d) x dimR matrix with rows (r, sigma) = Q R (Householder,
// LAPACK signs); storage <- Q, Rmx (dimR x dimR, ld dimR) <- R.  mem, tau, work unused.
void MPStensor::QR(double *Rmx, double *, double *, double *) {
  const int m = dimL * phys_d, n = dimR;
  std::vector<double> A((size_t)m * n);
  for (int s = 0; s < phys_d; ++s)
    for (int r = 0; r < dimL; ++r)
      for (int c = 0; c < dimR; ++c) A[r + dimL * (s + phys_d * c)] = storage[r + dimL * (c + dimR * s)];
  mqh::householder_qr(m, n, A.data(), m, Rmx, n);
  for (int s = 0; s < phys_d; ++s)
    for (int r = 0; r < dimL; ++r)
      for (int c = 0; c < dimR; ++c) storage[r + dimL * (c + dimR * s)] = A[r + dimL * (s + phys_d * c)];
}

// Right-orthonormalise: the dimL x (dimR d) matrix = L Q via the QR of its transpose;
// storage <- Q, Lmx (dimL x dimL, ld dimL, lower triangular) <- L.
void MPStensor::LQ(double *Lmx, double *, double *) {
  const int m = dimL, n = dimR * phys_d;
  std::vector<double> At((size_t)n * m), R((size_t)m * m);
  for (int r = 0; r < m; ++r)
    for (int c = 0; c < n; ++c) At[c + (size_t)n * r] = storage[r + (size_t)m * c];
  mqh::householder_qr(n, m, At.data(), n, R.data(), m);
  for (int r = 0; r < m; ++r)
    for (int c = 0; c < n; ++c) storage[r + (size_t)m * c] = At[c + (size_t)n * r];
  for (int r = 0; r < m; ++r)
    for (int c = 0; c < m; ++c) Lmx[r + m * c] = R[c + m * r];
}

void MPStensor::LeftMultiply(double *Lmx, double *) {
  std::vector<double> tmp((size_t)dimL * dimR);
  for (int s = 0; s < phys_d; ++s) {
    mqh::gemm(false, false, dimL, dimR, dimL, 1.0, Lmx, dimL, gStorage(s), dimL, 0.0, tmp.data(), dimL);
    std::memcpy(gStorage(s), tmp.data(), sizeof(double) * tmp.size());
  }
}

void MPStensor::RightMultiply(double *Rmx, double *) {
  std::vector<double> tmp((size_t)dimL * dimR);
  for (int s = 0; s < phys_d; ++s) {
    mqh::gemm(false, false, dimL, dimR, dimR, 1.0, gStorage(s), dimL, Rmx, dimR, 0.0, tmp.data(), dimL);
    std::memcpy(gStorage(s), tmp.data(), sizeof(double) * tmp.size());
  }
}

ostream &operator<<(ostream &output, const MPStensor &t) {
  output << t.dimL << "\t" << t.phys_d << "\t" << t.dimR << "\t" << t.storageSize << endl;
  for (int i = 0; i < t.storageSize; ++i) output << i << "\t" << t.storage[i] << endl;
  return output;
}

// ---------------------------------------------------------------------------------------------
// TwoSiteObject
// ---------------------------------------------------------------------------------------------
const double TwoSiteObject::SchmidtTrunc = 1e-13;

TwoSiteObject::TwoSiteObject(const int dl, const int dr, const int d) : phys_d(d), DimL(dl), DimR(dr) {
  storage.assign((size_t)dl * dr * d * d, 0.0);
}
TwoSiteObject::~TwoSiteObject() {}
int TwoSiteObject::gDimL() const { return DimL; }
int TwoSiteObject::gDimR() const { return DimR; }
int TwoSiteObject::gPhys_d() const { return phys_d; }
int TwoSiteObject::gStorageSize() const { return (int)storage.size(); }
double *TwoSiteObject::gStorage() { return storage.data(); }
double *TwoSiteObject::gStorage(const int dl, const int dr) {
  if (dl < 0 || dl >= phys_d || dr < 0 || dr >= phys_d) return nullptr;
  return storage.data() + (size_t)DimL * DimR * (dl + phys_d * dr);
}

void TwoSiteObject::Compose(MPStensor *A, MPStensor *B) {
  if (A->gDimR() != B->gDimL() || A->gPhys_d() != phys_d || B->gPhys_d() != phys_d) return;
  DimL = A->gDimL();
  DimR = B->gDimR();
  const int M = A->gDimR();
  storage.assign((size_t)DimL * DimR * phys_d * phys_d, 0.0);
  for (int a = 0; a < phys_d; ++a)
    for (int b = 0; b < phys_d; ++b)
      mqh::gemm(false, false, DimL, DimR, M, 1.0, A->gStorage(a), DimL, B->gStorage(b), M, 0.0, gStorage(a, b), DimL);
}

// SVD split of the two-site tensor, rows (alpha, sigma_left), columns (beta, sigma_right);
// singular values go right when moving right, left otherwise (TwoSiteObject.cpp:119-184).
int TwoSiteObject::Decompose(MPStensor *A, MPStensor *B, const int Dtrunc, bool movingright, bool possiblyCompress) {
  const int d = phys_d, mL = DimL * d, mR = DimR * d;
  std::vector<double> mem((size_t)mL * mR);
  for (int a = 0; a < DimL; ++a)
    for (int il = 0; il < d; ++il)
      for (int b = 0; b < DimR; ++b)
        for (int ir = 0; ir < d; ++ir) mem[(a + DimL * il) + (size_t)mL * (b + DimR * ir)] = gStorage(il, ir)[a + DimL * b];
  std::vector<double> U, S, VT;
  mqh::svd(mL, mR, mem.data(), U, S, VT);
  const int dimMin = std::min(mL, mR);
  int keep = std::min(Dtrunc, dimMin);
  if (possiblyCompress)
    for (int c = 0; c < dimMin; ++c)
      if (S[c] < SchmidtTrunc) {
        keep = std::min(keep, c);
        break;
      }
  keep = std::max(keep, 1);
  if (keep != A->gDimR()) {
    A->Reset(DimL, keep);
    B->Reset(keep, DimR);
  }
  for (int s = 0; s < d; ++s) {
    double *t = A->gStorage(s);
    for (int a = 0; a < DimL; ++a)
      for (int b = 0; b < keep; ++b) t[a + DimL * b] = U[(a + DimL * s) + (size_t)mL * b] * (movingright ? 1.0 : S[b]);
  }
  for (int s = 0; s < d; ++s) {
    double *t = B->gStorage(s);
    for (int a = 0; a < keep; ++a)
      for (int b = 0; b < DimR; ++b) t[a + keep * b] = VT[a + (size_t)dimMin * (b + DimR * s)] * (movingright ? S[a] : 1.0);
  }
  return keep;
}

// ---------------------------------------------------------------------------------------------
// MPSstate
// ---------------------------------------------------------------------------------------------
void MPSstate::allocate(Random *rn) {
  RN = rn;
  theTensors.resize(length);
  for (int k = 0; k < length; ++k) theTensors[k] = new MPStensor(VirtualD[k], VirtualD[k + 1], phys_d, RN);
}

MPSstate::MPSstate(const int L, const int D, const int d, Random *rn) : length(L), Dtrunc(D), phys_d(d) {
  VirtualD.assign(L + 1, 1);
  for (int c = 1; c < L; ++c) VirtualD[c] = std::min(VirtualD[c - 1] * d, D);
  for (int c = L - 1; c > 0; --c) VirtualD[c] = std::min(std::min(VirtualD[c + 1] * d, D), VirtualD[c]);
  allocate(rn);
}

MPSstate::MPSstate(const int L, const int D, const int d, int *dims, Random *rn) : length(L), Dtrunc(D), phys_d(d) {
  VirtualD.assign(dims, dims + L + 1);
  allocate(rn);
}

MPSstate::MPSstate(MPSstate *o) : RN(o->gRN()), length(o->gLength()), Dtrunc(o->gDtrunc()), phys_d(o->gPhys_d()) {
  VirtualD.resize(length + 1);
  for (int b = 0; b <= length; ++b) VirtualD[b] = o->gDimAtBound(b);
  theTensors.resize(length);
  for (int k = 0; k < length; ++k) theTensors[k] = new MPStensor(o->gMPStensor(k));
}

// Text format of MPSstate.cpp:92-128 / 661-686: "L D d", then "i D_i" for every bond, then per
// site "i size" followed by "i j value" lines.  The tensors are first filled randomly (as the
// reference does), then overwritten.
MPSstate::MPSstate(const char *filename, Random *rn) {
  ifstream in(filename);
  in >> length >> Dtrunc >> phys_d;
  VirtualD.resize(length + 1);
  for (int b = 0; b <= length; ++b) {
    int idx;
    in >> idx >> VirtualD[b];
  }
  allocate(rn);
  for (int k = 0; k < length; ++k) {
    int idx, n;
    in >> idx >> n;
    for (int j = 0; j < n; ++j) {
      int a, b;
      in >> a >> b >> theTensors[k]->gStorage()[j];
    }
  }
}

MPSstate::~MPSstate() {
  for (MPStensor *t : theTensors) delete t;
}

int MPSstate::gLength() const { return length; }
int MPSstate::gPhys_d() const { return phys_d; }
int MPSstate::gDtrunc() const { return Dtrunc; }
int MPSstate::gDimAtBound(const int b) const { return (b < 0 || b > length) ? 0 : VirtualD[b]; }
MPStensor *MPSstate::gMPStensor(const int s) { return (s < 0 || s >= length) ? nullptr : theTensors[s]; }
Random *MPSstate::gRN() { return RN; }
void MPSstate::checkWork1(const int n) { if ((int)work1.size() < n) work1.resize(n); }
void MPSstate::checkWork2(const int n) { if ((int)work2.size() < n) work2.resize(n); }
void MPSstate::checkWork3(const int n) { if ((int)work3.size() < n) work3.resize(n); }

void MPSstate::printVdim() const {
  for (int b = 0; b <= length; ++b) cout << b << "\t" << VirtualD[b] << endl;
}

// QR sweep left to right, R pushed into the next site; returns the last R factor (the norm,
// with LAPACK's sign) as MPSstate.cpp:216-229 does.
double MPSstate::LeftNormalize() {
  double last = 0.0;
  for (int k = 0; k < length; ++k) {
    const int n = VirtualD[k + 1];
    std::vector<double> R((size_t)n * n);
    theTensors[k]->QR(R.data(), nullptr, nullptr, nullptr);
    last = R[0];
    if (k != length - 1) theTensors[k + 1]->LeftMultiply(R.data(), nullptr);
  }
  return last;
}

double MPSstate::RightNormalize() {
  double last = 0.0;
  for (int k = length - 1; k >= 0; --k) {
    const int m = VirtualD[k];
    std::vector<double> Lm((size_t)m * m);
    theTensors[k]->LQ(Lm.data(), nullptr, nullptr);
    last = Lm[0];
    if (k != 0) theTensors[k - 1]->RightMultiply(Lm.data(), nullptr);
  }
  return last;
}

// <this|other> by the transfer sweep of MPSstate.cpp:248-284 (environment other x this).
double MPSstate::InnerProduct(MPSstate *o) {
  if (phys_d != o->gPhys_d() || length != o->gLength()) return 0.0;
  std::vector<double> env(1, 1.0), nxt, tmp;
  for (int k = 0; k < length; ++k) {
    const int lt = VirtualD[k], rt = VirtualD[k + 1], lo = o->gDimAtBound(k), ro = o->gDimAtBound(k + 1);
    nxt.assign((size_t)ro * rt, 0.0);
    tmp.assign((size_t)lo * rt, 0.0);
    for (int s = 0; s < phys_d; ++s) {
      mqh::gemm(false, false, lo, rt, lt, 1.0, env.data(), lo, theTensors[k]->gStorage(s), lt, 0.0, tmp.data(), lo);
      mqh::gemm(true, false, ro, rt, lo, 1.0, o->gMPStensor(k)->gStorage(s), lo, tmp.data(), lo, 1.0, nxt.data(), ro);
    }
    env.swap(nxt);
  }
  return env[0];
}

void MPSstate::ScalarMultiplication(const double factor) {
  const double f = std::pow(std::fabs(factor), 1.0 / length);
  const double sign = factor > 0.0 ? 1.0 : (factor < 0.0 ? -1.0 : 0.0);
  for (int k = 0; k < length; ++k) {
    const int n = VirtualD[k] * VirtualD[k + 1] * phys_d;
    const double a = (k == 0 ? sign : 1.0) * f;
    double *st = theTensors[k]->gStorage();
    for (int q = 0; q < n; ++q) st[q] *= a;
  }
}

void MPSstate::ChangePhase() {
  const int n = VirtualD[0] * VirtualD[1] * phys_d;
  double *st = theTensors[0]->gStorage();
  for (int q = 0; q < n; ++q) st[q] = -st[q];
}

// Direct sum |state1> + |state2> (MPSstate.cpp:317-377): block-diagonal bulk tensors, row and
// column concatenation at the two ends.
void MPSstate::ResetContentsAndStoreSumOf(MPSstate *s1, MPSstate *s2) {
  if (s1->gPhys_d() != s2->gPhys_d() || s1->gLength() != s2->gLength()) return;
  length = s1->gLength();
  phys_d = s1->gPhys_d();
  Dtrunc = s1->gDtrunc() + s2->gDtrunc();
  for (int b = 1; b < length; ++b) VirtualD[b] = s1->gDimAtBound(b) + s2->gDimAtBound(b);
  for (int k = 0; k < length; ++k) theTensors[k]->Reset(VirtualD[k], VirtualD[k + 1]);
  for (int k = 0; k < length; ++k) {
    const int l1 = s1->gDimAtBound(k), l2 = s2->gDimAtBound(k), r1 = s1->gDimAtBound(k + 1), r2 = s2->gDimAtBound(k + 1);
    const int L = VirtualD[k], R = VirtualD[k + 1];
    for (int s = 0; s < phys_d; ++s) {
      double *t = theTensors[k]->gStorage(s);
      const double *a = s1->gMPStensor(k)->gStorage(s), *b = s2->gMPStensor(k)->gStorage(s);
      for (int q = 0; q < L * R; ++q) t[q] = 0.0;
      if (k == 0) {  // 1 x (r1 + r2)
        for (int c = 0; c < r1; ++c) t[c] = a[c];
        for (int c = 0; c < r2; ++c) t[r1 + c] = b[c];
      } else if (k == length - 1) {  // (l1 + l2) x 1
        for (int r = 0; r < l1; ++r) t[r] = a[r];
        for (int r = 0; r < l2; ++r) t[l1 + r] = b[r];
      } else {
        for (int r = 0; r < l1; ++r)
          for (int c = 0; c < r1; ++c) t[r + L * c] = a[r + l1 * c];
        for (int r = 0; r < l2; ++r)
          for (int c = 0; c < r2; ++c) t[(l1 + r) + L * (r1 + c)] = b[r + l2 * c];
      }
    }
  }
}

// Two sweeps of two-site SVD truncation (MPSstate.cpp:379-404).
void MPSstate::CompressState(const int truncD) {
  TwoSiteObject two(Dtrunc, Dtrunc, phys_d);
  for (int k = 0; k < length - 1; ++k) {
    two.Compose(theTensors[k], theTensors[k + 1]);
    VirtualD[k + 1] = two.Decompose(theTensors[k], theTensors[k + 1], truncD, true, true);
  }
  for (int k = length - 2; k >= 0; --k) {
    two.Compose(theTensors[k], theTensors[k + 1]);
    VirtualD[k + 1] = two.Decompose(theTensors[k], theTensors[k + 1], truncD, false, true);
  }
  Dtrunc = *std::max_element(VirtualD.begin(), VirtualD.end());
}

// H|Psi0> as an MPS of bond dim (MPO dim) x (Psi0 dim) (MPSstate.cpp:413-471).
void MPSstate::ApplyMPO(MPO *mpo, MPSstate *Psi0) {
  for (int b = 1; b < length; ++b) VirtualD[b] = mpo->dimL(b) * Psi0->gDimAtBound(b);
  VirtualD[0] = VirtualD[length] = 1;
  Dtrunc = *std::max_element(VirtualD.begin(), VirtualD.end());
  for (int k = 0; k < length; ++k) {
    theTensors[k]->Reset(VirtualD[k], VirtualD[k + 1]);
    double *t = theTensors[k]->gStorage();
    for (int q = 0; q < VirtualD[k] * VirtualD[k + 1] * phys_d; ++q) t[q] = 0.0;
    const int ls = Psi0->gDimAtBound(k), rs = Psi0->gDimAtBound(k + 1);
    const int lm = mpo->dimL(k), rm = mpo->dimR(k);
    for (int a = 0; a < lm; ++a)
      for (int b = 0; b < rm; ++b) {
        Operator *op = mpo->gOperator(k, a, b);
        if (!op || op->AmIOp0()) continue;
        const double f = mpo->gPrefactor(k, a, b);
        for (int up = 0; up < phys_d; ++up) {
          double *tg = theTensors[k]->gStorage(up);
          for (int dn = 0; dn < phys_d; ++dn) {
            const double v = f * (*op)(up, dn);
            if (v == 0.0) continue;
            const double *src = Psi0->gMPStensor(k)->gStorage(dn);
            for (int r = 0; r < ls; ++r)
              for (int c = 0; c < rs; ++c) tg[(a * ls + r) + (ls * lm) * (b * rs + c)] += v * src[r + ls * c];
          }
        }
      }
  }
}

void MPSstate::applySiteOperator(const int site, const double *op) {
  const int blk = VirtualD[site] * VirtualD[site + 1];
  std::vector<double> out((size_t)blk * phys_d, 0.0);
  const double *st = theTensors[site]->gStorage();
  for (int up = 0; up < phys_d; ++up)
    for (int dn = 0; dn < phys_d; ++dn) {
      const double v = op[up + phys_d * dn];
      if (v == 0.0) continue;
      for (int q = 0; q < blk; ++q) out[(size_t)up * blk + q] += v * st[(size_t)dn * blk + q];
    }
  std::memcpy(theTensors[site]->gStorage(), out.data(), sizeof(double) * out.size());
}

void MPSstate::ApplyMPOterm(MPO *mpo, const int t) {
  std::vector<double> op((size_t)phys_d * phys_d);
  for (int k = 0; k < length; ++k) {
    Operator *o = mpo->gRN_operator(t, k);
    if (!o || o->AmIOpI()) continue;
    for (int up = 0; up < phys_d; ++up)
      for (int dn = 0; dn < phys_d; ++dn) op[up + phys_d * dn] = (*o)(up, dn);
    applySiteOperator(k, op.data());
  }
  ScalarMultiplication(mpo->gRN_prefactor(t));
}

// sqrt(s_k) U_k on the first site and sqrt(s_l) V_l on the second, transposed when doHC
// (MPSstate.cpp:505-573).
void MPSstate::ApplyTwoSiteTrotterTerm(TrotterHeisenberg *T, const int i, const int j, const int k, const int l,
                                       const bool doHC) {
  const double J = T->gCoupling(i, j);
  std::vector<double> op((size_t)phys_d * phys_d);
  const double sk = std::sqrt(T->gTwoSitePropSVD_Sing(J, k)), sl = std::sqrt(T->gTwoSitePropSVD_Sing(J, l));
  for (int up = 0; up < phys_d; ++up)
    for (int dn = 0; dn < phys_d; ++dn)
      op[up + phys_d * dn] = sk * T->gTwoSitePropSVD_Left(J, k, doHC ? dn : up, doHC ? up : dn);
  applySiteOperator(i, op.data());
  for (int up = 0; up < phys_d; ++up)
    for (int dn = 0; dn < phys_d; ++dn)
      op[up + phys_d * dn] = sl * T->gTwoSitePropSVD_Right(J, l, doHC ? dn : up, doHC ? up : dn);
  applySiteOperator(j, op.data());
}

// Auxiliary-field operators O1(x) = sum_k sqrt(s_k dim) x_k U_k on the first site and
// O2(x) = sum_k sqrt(s_k dim) x_k V_k on the second (MPSstate.cpp:575-633).
void MPSstate::ApplyTwoSiteTrotterTerm(TrotterHeisenberg *T, const int i, const int j, GridGenerator *g,
                                       const int p) {
  const double J = T->gCoupling(i, j);
  const int D = g->gDim();
  std::vector<double> o1((size_t)phys_d * phys_d, 0.0), o2((size_t)phys_d * phys_d, 0.0);
  for (int k = 0; k < D; ++k) {
    const double pf = std::sqrt(T->gTwoSitePropSVD_Sing(J, k) * D) * g->gCoOfPoint(p, k);
    for (int up = 0; up < phys_d; ++up)
      for (int dn = 0; dn < phys_d; ++dn) {
        o1[up + phys_d * dn] += pf * T->gTwoSitePropSVD_Left(J, k, up, dn);
        o2[up + phys_d * dn] += pf * T->gTwoSitePropSVD_Right(J, k, up, dn);
      }
  }
  applySiteOperator(i, o1.data());
  applySiteOperator(j, o2.data());
}

void MPSstate::ApplyOneSiteTrotterTermEverywhere(TrotterHeisenberg *T) {
  if (!T->gIsMagneticField()) return;
  std::vector<double> op((size_t)phys_d * phys_d);
  for (int up = 0; up < phys_d; ++up)
    for (int dn = 0; dn < phys_d; ++dn) op[up + phys_d * dn] = T->gSingleSiteProp(up, dn);
  for (int k = 0; k < length; ++k) applySiteOperator(k, op.data());
}

ostream &operator<<(ostream &output, MPSstate &mps) {
  output << mps.length << "\t" << mps.Dtrunc << "\t" << mps.phys_d << endl;
  for (int b = 0; b <= mps.length; ++b) output << b << "\t" << mps.VirtualD[b] << endl;
  for (int k = 0; k < mps.length; ++k) {
    const int n = mps.VirtualD[k] * mps.VirtualD[k + 1] * mps.phys_d;
    output << k << "\t" << n << endl;
    const double *st = mps.theTensors[k]->gStorage();
    for (int j = 0; j < n; ++j) output << k << "\t" << j << "\t" << st[j] << endl;
  }
  return output;
}
