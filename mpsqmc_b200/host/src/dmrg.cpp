// Two-site DMRG on the MPO's environments with a Lanczos eigensolver.  The reference rebuilds
// the full MPO x MPS product every step (DMRG.cpp:70-100) and uses Davidson (232-479); the sweep
// order, the two-site update and the truncation back to the state's own bond dimensions are
// the same.
#include <cmath>
#include <cstdio>
#include <functional>
#include <vector>

#include "DMRG.h"
#include "linalg.h"

namespace {

struct Mpo {
  int L, d;
  std::vector<int> w;                    // bond widths
  std::vector<std::vector<double> > W;   // per site [a + wl (b + wr (up + d dn))]
};

Mpo dense_mpo(MPO *m) {
  Mpo o;
  o.L = m->gLength();
  o.d = m->gPhys_d();
  o.w.resize(o.L + 1);
  for (int k = 0; k < o.L; ++k) o.w[k] = m->dimL(k);
  o.w[o.L] = 1;
  o.W.resize(o.L);
  for (int k = 0; k < o.L; ++k) {
    const int wl = m->dimL(k), wr = m->dimR(k), d = o.d;
    o.W[k].assign((size_t)wl * wr * d * d, 0.0);
    for (int a = 0; a < wl; ++a)
      for (int b = 0; b < wr; ++b) {
        Operator *op = m->gOperator(k, a, b);
        if (!op || op->AmIOp0()) continue;
        const double f = m->gPrefactor(k, a, b);
        for (int up = 0; up < d; ++up)
          for (int dn = 0; dn < d; ++dn) o.W[k][a + wl * (b + wr * (up + d * dn))] = f * (*op)(up, dn);
      }
  }
  return o;
}

// site tensor element A[sigma](r, c) of an MPStensor
inline double at(MPStensor *t, int s, int r, int c) { return t->gStorage(s)[r + t->gDimL() * c]; }

// left environment E[k+1](c, b, c') = sum A(a,s,c) E[k](a, w, a') W(w, b, s, s') A(a', s', c')
std::vector<double> left_step(const std::vector<double> &E, MPStensor *A, const Mpo &m, int k) {
  const int Dl = A->gDimL(), Dr = A->gDimR(), d = m.d, wl = m.w[k], wr = m.w[k + 1];
  // T1(a, w, s', c') = sum_a' E(a, w, a') A(a', s', c')
  std::vector<double> T1((size_t)Dl * wl * d * Dr, 0.0);
  for (int sp = 0; sp < d; ++sp)
    for (int w = 0; w < wl; ++w)
      mqh::gemm(false, false, Dl, Dr, Dl, 1.0, E.data() + (size_t)Dl * Dl * w, Dl, A->gStorage(sp), Dl, 0.0,
                T1.data() + (size_t)Dl * Dr * (w + wl * sp), Dl);
  // T2(a, b, s, c') = sum_{w, s'} T1(a, w, s', c') W(w, b, s, s')
  std::vector<double> T2((size_t)Dl * wr * d * Dr, 0.0);
  for (int w = 0; w < wl; ++w)
    for (int b = 0; b < wr; ++b)
      for (int s = 0; s < d; ++s)
        for (int sp = 0; sp < d; ++sp) {
          const double v = m.W[k][w + wl * (b + wr * (s + d * sp))];
          if (v == 0.0) continue;
          const double *src = T1.data() + (size_t)Dl * Dr * (w + wl * sp);
          double *dst = T2.data() + (size_t)Dl * Dr * (b + wr * s);
          for (size_t q = 0; q < (size_t)Dl * Dr; ++q) dst[q] += v * src[q];
        }
  // E'(c, b, c') = sum_{a, s} A(a, s, c) T2(a, b, s, c')
  std::vector<double> out((size_t)Dr * wr * Dr, 0.0);
  for (int b = 0; b < wr; ++b)
    for (int s = 0; s < d; ++s)
      mqh::gemm(true, false, Dr, Dr, Dl, 1.0, A->gStorage(s), Dl, T2.data() + (size_t)Dl * Dr * (b + wr * s), Dl, 1.0,
                out.data() + (size_t)Dr * Dr * b, Dr);
  return out;
}

// right environment F[k](a, w, a') = sum A(a,s,c) W(w, b, s, s') F[k+1](c, b, c') A(a', s', c')
std::vector<double> right_step(const std::vector<double> &F, MPStensor *A, const Mpo &m, int k) {
  const int Dl = A->gDimL(), Dr = A->gDimR(), d = m.d, wl = m.w[k], wr = m.w[k + 1];
  // T1(a', s', c, b) = sum_c' A(a', s', c') F(c, b, c')  -> per (s', b): A[s'] (Dl x Dr) F_b^T (Dr x Dr)
  std::vector<double> T1((size_t)Dl * Dr * d * wr, 0.0);
  for (int sp = 0; sp < d; ++sp)
    for (int b = 0; b < wr; ++b)
      mqh::gemm(false, true, Dl, Dr, Dr, 1.0, A->gStorage(sp), Dl, F.data() + (size_t)Dr * Dr * b, Dr, 0.0,
                T1.data() + (size_t)Dl * Dr * (sp + d * b), Dl);
  // T2(a', c, w, s) = sum_{b, s'} W(w, b, s, s') T1(a', s', c, b)
  std::vector<double> T2((size_t)Dl * Dr * wl * d, 0.0);
  for (int w = 0; w < wl; ++w)
    for (int b = 0; b < wr; ++b)
      for (int s = 0; s < d; ++s)
        for (int sp = 0; sp < d; ++sp) {
          const double v = m.W[k][w + wl * (b + wr * (s + d * sp))];
          if (v == 0.0) continue;
          const double *src = T1.data() + (size_t)Dl * Dr * (sp + d * b);
          double *dst = T2.data() + (size_t)Dl * Dr * (w + wl * s);
          for (size_t q = 0; q < (size_t)Dl * Dr; ++q) dst[q] += v * src[q];
        }
  // F'(a, w, a') = sum_{s, c} A(a, s, c) T2(a', c, w, s)  -> A[s] (Dl x Dr) T2_ws^T (Dr x Dl)
  std::vector<double> out((size_t)Dl * wl * Dl, 0.0);
  for (int w = 0; w < wl; ++w)
    for (int s = 0; s < d; ++s)
      mqh::gemm(false, true, Dl, Dl, Dr, 1.0, A->gStorage(s), Dl, T2.data() + (size_t)Dl * Dr * (w + wl * s), Dl, 1.0,
                out.data() + (size_t)Dl * Dl * w, Dl);
  return out;
}

// y = H_eff x on the two-site tensor x(a, s, t, c) stored [a + Dl (s + d (t + d c))]
void heff(const std::vector<double> &E, const std::vector<double> &F, const Mpo &m, int k, int Dl, int Dr,
          const double *x, double *y) {
  const int d = m.d, w0 = m.w[k], w1 = m.w[k + 1], w2 = m.w[k + 2];
  const size_t n = (size_t)Dl * d * d * Dr;
  // X1(a, w, s', t', c) = sum_a' E(a, w, a') x(a', s', t', c)
  std::vector<double> X1((size_t)Dl * w0 * d * d * Dr, 0.0);
  for (int w = 0; w < w0; ++w)
    mqh::gemm(false, false, Dl, d * d * Dr, Dl, 1.0, E.data() + (size_t)Dl * Dl * w, Dl, x, Dl, 0.0,
              X1.data() + (size_t)w * Dl * d * d * Dr, Dl);
  // X2(a, v, s, t', c) = sum_{w, s'} W1(w, v, s, s') X1(a, w, s', t', c)
  const size_t blk = (size_t)Dl;  // stride of s' inside X1 block: [a + Dl (s' + d (t' + d c))]
  std::vector<double> X2((size_t)w1 * Dl * d * d * Dr, 0.0);
  for (int w = 0; w < w0; ++w)
    for (int v = 0; v < w1; ++v)
      for (int s = 0; s < d; ++s)
        for (int sp = 0; sp < d; ++sp) {
          const double f = m.W[k][w + w0 * (v + w1 * (s + d * sp))];
          if (f == 0.0) continue;
          const double *src = X1.data() + (size_t)w * Dl * d * d * Dr;
          double *dst = X2.data() + (size_t)v * Dl * d * d * Dr;
          for (int tc = 0; tc < d * Dr; ++tc)
            for (int a = 0; a < Dl; ++a) dst[a + blk * (s + d * tc)] += f * src[a + blk * (sp + d * tc)];
        }
  // X3(a, u, s, t, c) = sum_{v, t'} W2(v, u, t, t') X2(a, v, s, t', c)
  std::vector<double> X3((size_t)w2 * Dl * d * d * Dr, 0.0);
  for (int v = 0; v < w1; ++v)
    for (int u = 0; u < w2; ++u)
      for (int t = 0; t < d; ++t)
        for (int tp = 0; tp < d; ++tp) {
          const double f = m.W[k + 1][v + w1 * (u + w2 * (t + d * tp))];
          if (f == 0.0) continue;
          const double *src = X2.data() + (size_t)v * Dl * d * d * Dr;
          double *dst = X3.data() + (size_t)u * Dl * d * d * Dr;
          for (int c = 0; c < Dr; ++c)
            for (int s = 0; s < d; ++s)
              for (int a = 0; a < Dl; ++a)
                dst[a + Dl * (s + d * (t + d * c))] += f * src[a + Dl * (s + d * (tp + d * c))];
        }
  // y(a, s, t, c) = sum_{u, c'} X3(a, u, s, t, c') F(c, u, c')
  for (size_t q = 0; q < n; ++q) y[q] = 0.0;
  for (int u = 0; u < w2; ++u)
    mqh::gemm(false, true, Dl * d * d, Dr, Dr, 1.0, X3.data() + (size_t)u * Dl * d * d * Dr, Dl * d * d,
              F.data() + (size_t)Dr * Dr * u, Dr, 1.0, y, Dl * d * d);
}

// Lowest eigenpair by Lanczos with full reorthogonalisation, started from x (overwritten).
double lanczos(int n, const std::function<void(const double *, double *)> &op, double *x, int maxit = 60) {
  std::vector<std::vector<double> > Q;
  std::vector<double> alpha, beta;
  std::vector<double> v(x, x + n), w(n);
  double nrm = 0.0;
  for (double t : v) nrm += t * t;
  nrm = std::sqrt(nrm);
  if (nrm == 0.0) { v.assign(n, 0.0); v[0] = 1.0; nrm = 1.0; }
  for (double &t : v) t /= nrm;
  double eprev = 1e300, e = 0.0;
  std::vector<double> evec;
  const int m_max = std::min(maxit, n);
  for (int it = 0; it < m_max; ++it) {
    Q.push_back(v);
    op(v.data(), w.data());
    double a = 0.0;
    for (int q = 0; q < n; ++q) a += w[q] * v[q];
    alpha.push_back(a);
    for (const auto &qv : Q) {
      double dot = 0.0;
      for (int q = 0; q < n; ++q) dot += w[q] * qv[q];
      for (int q = 0; q < n; ++q) w[q] -= dot * qv[q];
    }
    double b = 0.0;
    for (double t : w) b += t * t;
    b = std::sqrt(b);
    const int m = (int)alpha.size();
    std::vector<double> T((size_t)m * m, 0.0), ev, V;
    for (int i = 0; i < m; ++i) {
      T[i + (size_t)m * i] = alpha[i];
      if (i + 1 < m) T[i + (size_t)m * (i + 1)] = T[(i + 1) + (size_t)m * i] = beta[i];
    }
    mqh::sym_eig(m, T, ev, V);
    e = ev[0];
    evec.assign(V.begin(), V.begin() + m);
    if (b < 1e-12 || std::fabs(e - eprev) < 1e-13 * std::max(1.0, std::fabs(e)) || it + 1 == m_max) break;
    eprev = e;
    beta.push_back(b);
    for (int q = 0; q < n; ++q) v[q] = w[q] / b;
  }
  for (int q = 0; q < n; ++q) x[q] = 0.0;
  for (size_t i = 0; i < evec.size(); ++i)
    for (int q = 0; q < n; ++q) x[q] += evec[i] * Q[i][q];
  return e;
}

}  // namespace

DMRG::DMRG(MPSstate *trial, MPO *mpo) : MPSsolution(trial), theMPO(mpo), length(trial->gLength()) {}
DMRG::~DMRG() {}

double DMRG::Solve() {
  const int L = length, d = MPSsolution->gPhys_d();
  const Mpo m = dense_mpo(theMPO);
  std::vector<int> dims(L + 1);
  for (int b = 0; b <= L; ++b) dims[b] = MPSsolution->gDimAtBound(b);
  MPSsolution->RightNormalize();
  std::vector<std::vector<double> > E(L + 1), F(L + 1);
  E[0].assign(1, 1.0);
  F[L].assign(1, 1.0);
  for (int k = L - 1; k >= 1; --k) F[k] = right_step(F[k + 1], MPSsolution->gMPStensor(k), m, k);
  double Eprev = 1e300, Ecur = 0.0;
  TwoSiteObject two(1, 1, d);
  auto update = [&](int k, bool right) {
    MPStensor *A = MPSsolution->gMPStensor(k), *B = MPSsolution->gMPStensor(k + 1);
    const int Dl = A->gDimL(), Dr = B->gDimR();
    two.Compose(A, B);
    const size_t n = (size_t)Dl * d * d * Dr;
    std::vector<double> x(n);
    for (int s = 0; s < d; ++s)
      for (int t = 0; t < d; ++t)
        for (int c = 0; c < Dr; ++c)
          for (int a = 0; a < Dl; ++a) x[a + Dl * (s + d * (t + d * c))] = two.gStorage(s, t)[a + Dl * c];
    Ecur = lanczos((int)n, [&](const double *in, double *out) { heff(E[k], F[k + 2], m, k, Dl, Dr, in, out); },
                   x.data());
    for (int s = 0; s < d; ++s)
      for (int t = 0; t < d; ++t)
        for (int c = 0; c < Dr; ++c)
          for (int a = 0; a < Dl; ++a) two.gStorage(s, t)[a + Dl * c] = x[a + Dl * (s + d * (t + d * c))];
    two.Decompose(A, B, dims[k + 1], right, false);
    if (right) E[k + 1] = left_step(E[k], A, m, k);
    else F[k + 1] = right_step(F[k + 2], B, m, k + 1);
  };
  for (int sweep = 0; sweep < 40; ++sweep) {
    for (int k = 0; k < L - 1; ++k) update(k, true);
    for (int k = L - 2; k >= 0; --k) update(k, false);
    cout << "DMRG :: sweep " << sweep << " energy = " << Ecur << endl;
    if (std::fabs(Ecur - Eprev) < 1e-10) break;
    Eprev = Ecur;
  }
  return Ecur;
}
