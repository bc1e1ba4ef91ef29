// Test infrastructure: CPU restatement of the reference's walker-propagation path, used as
// the checker for the CUDA implementation (tests, smoke check, CPU-baseline leg of the bench).
// It is never linked into or called by the product.
//
// Every routine restates the reference function it names (file:line in the reference tree),
// in plain C++ with its own dense linear algebra: Householder QR follows LAPACK's
// dgeqr2/dorg2r/dlarfg conventions (the reference calls dgeqrf/dorgqr with lwork=n, which
// selects exactly these unblocked routines), so LeftNormalize reproduces the reference's
// tensors element by element.  SVD and symmetric eigenproblems use Jacobi methods.
//
// Parity status: pinned.  tests/test_oracle_pin.py checks this file against outputs of the
// reference itself (built by oracle/Makefile) stored under tests/golden/.
#include "mpsqmc_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------------------
// MPS views
// ---------------------------------------------------------------------------------------
struct MpsView {
  int L, d;
  const int *dims;
  std::vector<double *> site;  // site pointers (may be overridden for trial terms)
};

MpsView make_view(int L, int d, const int *dims, const double *data) {
  MpsView v;
  v.L = L;
  v.d = d;
  v.dims = dims;
  v.site.resize(L);
  long off = 0;
  for (int s = 0; s < L; ++s) {
    v.site[s] = const_cast<double *>(data) + off;
    off += (long)dims[s] * dims[s + 1] * d;
  }
  return v;
}

// C(m x n) = op(A) * op(B) (+ beta*C), column-major, plain loops (dgemm semantics).
void gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda,
          const double *B, int ldb, double beta, double *C, int ldc) {
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < m; ++i) C[i + (long)ldc * j] *= beta;
    for (int p = 0; p < k; ++p) {
      const double b = tb ? B[j + (long)ldb * p] : B[p + (long)ldb * j];
      if (b == 0.0) continue;
      const double ab = alpha * b;
      if (!ta) {
        const double *a = A + (long)lda * p;
        double *c = C + (long)ldc * j;
        for (int i = 0; i < m; ++i) c[i] += ab * a[i];
      } else {
        double *c = C + (long)ldc * j;
        for (int i = 0; i < m; ++i) c[i] += ab * A[p + (long)lda * i];
      }
    }
  }
}

// MPSstate::InnerProduct, MPSstate.cpp:248-284 (this = A, other = B).
double inner_product(const MpsView &A, const MpsView &B, std::vector<double> &w1,
                     std::vector<double> &w2, std::vector<double> &w3) {
  const int L = A.L, d = A.d;
  int maxA = 1, maxB = 1;
  for (int b = 0; b <= L; ++b) {
    maxA = std::max(maxA, A.dims[b]);
    maxB = std::max(maxB, B.dims[b]);
  }
  const size_t ws = (size_t)maxA * maxB;
  if (w1.size() < ws) w1.resize(ws);
  if (w2.size() < ws) w2.resize(ws);
  if (w3.size() < ws) w3.resize(ws);
  double *work1 = w1.data(), *work2 = w2.data(), *work3 = w3.data();
  work1[0] = 1.0;
  for (int s = 0; s < L; ++s) {
    const int dLt = A.dims[s], dRt = A.dims[s + 1];
    const int dLo = B.dims[s], dRo = B.dims[s + 1];
    for (int q = 0; q < dRt * dRo; ++q) work2[q] = 0.0;
    for (int sg = 0; sg < d; ++sg) {
      // work3 (dLo x dRt) = work1 (dLo x dLt) * A[sg] (dLt x dRt)
      gemm(false, false, dLo, dRt, dLt, 1.0, work1, dLo, A.site[s] + (long)sg * dLt * dRt, dLt,
           0.0, work3, dLo);
      // work2 (dRo x dRt) += B[sg]^T (dRo x dLo) * work3
      gemm(true, false, dRo, dRt, dLo, 1.0, B.site[s] + (long)sg * dLo * dRo, dLo, work3, dLo,
           1.0, work2, dRo);
    }
    std::swap(work1, work2);
  }
  return work1[0];
}

// ---------------------------------------------------------------------------------------
// Householder QR in LAPACK's conventions (dlarfg / dlarf / dgeqr2 / dorg2r)
// ---------------------------------------------------------------------------------------
double dlapy2(double x, double y) {
  const double xa = std::fabs(x), ya = std::fabs(y);
  const double w = std::max(xa, ya), z = std::min(xa, ya);
  if (z == 0.0) return w;
  const double r = z / w;
  return w * std::sqrt(1.0 + r * r);
}

double dnrm2(int n, const double *x) {
  double scale = 0.0, ssq = 1.0;
  for (int i = 0; i < n; ++i) {
    if (x[i] != 0.0) {
      const double a = std::fabs(x[i]);
      if (scale < a) {
        const double r = scale / a;
        ssq = 1.0 + ssq * r * r;
        scale = a;
      } else {
        const double r = a / scale;
        ssq += r * r;
      }
    }
  }
  return scale * std::sqrt(ssq);
}

// dlarfg: on exit alpha = beta, x = v(2:n), returns tau.
double dlarfg(int n, double &alpha, double *x) {
  if (n <= 1) return 0.0;
  const double xnorm = dnrm2(n - 1, x);
  if (xnorm == 0.0) return 0.0;
  const double mag = dlapy2(alpha, xnorm);
  const double beta = (alpha >= 0.0) ? -mag : mag;
  const double tau = (beta - alpha) / beta;
  const double sc = 1.0 / (alpha - beta);
  for (int i = 0; i < n - 1; ++i) x[i] *= sc;
  alpha = beta;
  return tau;
}

// Apply H = I - tau v v^T from the left to C (m x n, ld ldc); v(0) is implicitly 1.
void dlarf_left(int m, int n, const double *v, double tau, double *C, int ldc, double *work) {
  if (tau == 0.0) return;
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    for (int i = 0; i < m; ++i) s += C[i + (long)ldc * j] * v[i];
    work[j] = s;
  }
  for (int j = 0; j < n; ++j) {
    const double t = -tau * work[j];
    for (int i = 0; i < m; ++i) C[i + (long)ldc * j] += t * v[i];
  }
}

// dgeqr2 followed by dorg2r on A (m x n, m >= n, ld m): A <- Q, R (n x n) returned.
void householder_qr(int m, int n, double *A, double *R, std::vector<double> &scratch) {
  scratch.resize((size_t)2 * n + m);
  double *tau = scratch.data(), *work = tau + n, *v = work + n;
  const int k = std::min(m, n);
  for (int i = 0; i < k; ++i) {
    double *col = A + (long)m * i;
    tau[i] = dlarfg(m - i, col[i], col + i + 1);
    if (i < n - 1) {
      const double aii = col[i];
      col[i] = 1.0;
      dlarf_left(m - i, n - i - 1, col + i, tau[i], A + i + (long)m * (i + 1), m, work);
      col[i] = aii;
    }
  }
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) R[r + (long)n * c] = (r <= c) ? A[r + (long)m * c] : 0.0;
  (void)v;
  // dorg2r with k = n
  for (int i = k - 1; i >= 0; --i) {
    double *col = A + (long)m * i;
    if (i < n - 1) {
      col[i] = 1.0;
      dlarf_left(m - i, n - i - 1, col + i, tau[i], A + i + (long)m * (i + 1), m, work);
    }
    if (i < m - 1)
      for (int r = i + 1; r < m; ++r) col[r] *= -tau[i];
    col[i] = 1.0 - tau[i];
    for (int r = 0; r < i; ++r) col[r] = 0.0;
  }
}

// MPSstate::LeftNormalize, MPSstate.cpp:216-229; MPStensor::QR 100-135; LeftMultiply 159-175.
double left_normalize(int L, int d, const int *dims, double *data, std::vector<double> &mem,
                      std::vector<double> &Rm, std::vector<double> &work) {
  long off = 0;
  double last = 0.0;
  for (int s = 0; s < L; ++s) {
    const int dl = dims[s], dr = dims[s + 1];
    double *st = data + off;
    const int m = dl * d, n = dr;
    mem.resize((size_t)m * n);
    Rm.resize((size_t)n * n);
    for (int sg = 0; sg < d; ++sg)
      for (int r = 0; r < dl; ++r)
        for (int c = 0; c < dr; ++c) mem[r + dl * (sg + d * c)] = st[r + dl * (c + dr * sg)];
    householder_qr(m, n, mem.data(), Rm.data(), work);
    for (int sg = 0; sg < d; ++sg)
      for (int r = 0; r < dl; ++r)
        for (int c = 0; c < dr; ++c) st[r + dl * (c + dr * sg)] = mem[r + dl * (sg + d * c)];
    last = Rm[0];
    off += (long)dl * dr * d;
    if (s != L - 1) {
      // next[sg] = R (dr x dr) * next[sg] (dr x dr2)
      const int dr2 = dims[s + 2];
      double *nx = data + off;
      std::vector<double> tmp((size_t)dr * dr2);
      for (int sg = 0; sg < d; ++sg) {
        double *blk = nx + (long)sg * dr * dr2;
        std::fill(tmp.begin(), tmp.end(), 0.0);
        gemm(false, false, dr, dr2, dr, 1.0, Rm.data(), dr, blk, dr, 0.0, tmp.data(), dr);
        std::copy(tmp.begin(), tmp.end(), blk);
      }
    }
  }
  return last;
}

// ---------------------------------------------------------------------------------------
// Local operators (OpSz.cpp:9, OpSx.cpp:11, OpISy.cpp:11-21)
// ---------------------------------------------------------------------------------------
double op_sz(int d, int i, int j) { return (i == j) ? 0.5 * (1 - d) + i : 0.0; }
double ladder(int d, int k) {
  return 0.25 * std::sqrt(d * d - 1.0 - (1.0 - d + 2 * k) * (3.0 - d + 2 * k));
}
double op_sx(int d, int i, int j) {
  if (i == j + 1) return ladder(d, j);
  if (i + 1 == j) return ladder(d, i);
  return 0.0;
}
double op_isy(int d, int i, int j) {
  if (i == j + 1) return ladder(d, j);
  if (i + 1 == j) return -ladder(d, i);
  return 0.0;
}

// One site, in place: T[up] <- sum_down Op(up,down) T[down] (daxpy order of MPSstate.cpp:523-538).
void apply_site_op(int d, int dl, int dr, double *T, const double *op /* [up + d*down] */,
                   std::vector<double> &work) {
  const int blk = dl * dr;
  work.assign((size_t)blk * d, 0.0);
  for (int up = 0; up < d; ++up)
    for (int dn = 0; dn < d; ++dn) {
      const double v = op[up + d * dn];
      if (v != 0.0)
        for (int q = 0; q < blk; ++q) work[(size_t)up * blk + q] += v * T[(size_t)dn * blk + q];
    }
  std::copy(work.begin(), work.end(), T);
}

// Site operator of ApplyTwoSiteTrotterTerm(grid), MPSstate.cpp:589-604 (left) / 615-628
// (right): daxpy accumulation in SVD-index-major order.
void apply_grid_site(int d, int dl, int dr, double *T, const double *S, const double *Mtab,
                     bool right, const double *x, std::vector<double> &work) {
  const int n = d * d, blk = dl * dr;
  work.assign((size_t)blk * d, 0.0);
  for (int k = 0; k < n; ++k) {
    const double pref = std::sqrt(S[k] * n) * x[k];
    if (pref == 0.0) continue;
    for (int up = 0; up < d; ++up)
      for (int dn = 0; dn < d; ++dn) {
        const double ov = right ? Mtab[k + n * (up + d * dn)] : Mtab[up + d * (dn + d * k)];
        const double v = pref * ov;
        if (v != 0.0)
          for (int q = 0; q < blk; ++q) work[(size_t)up * blk + q] += v * T[(size_t)dn * blk + q];
      }
  }
  std::copy(work.begin(), work.end(), T);
}

// Site operator of ApplyTwoSiteTrotterTerm(svd index, doHC), MPSstate.cpp:518-569.
void svd_site_op(int d, int k, const double *S, const double *Mtab, bool right, bool hc,
                 double *op /* [up + d*down] */) {
  const int n = d * d;
  const double sq = std::sqrt(S[k]);
  for (int up = 0; up < d; ++up)
    for (int dn = 0; dn < d; ++dn) {
      const int a = hc ? dn : up, b = hc ? up : dn;
      const double m = right ? Mtab[k + n * (a + d * b)] : Mtab[a + d * (b + d * k)];
      op[up + d * dn] = sq * m;
    }
}

long mps_size(int L, int d, const int *dims) {
  long n = 0;
  for (int s = 0; s < L; ++s) n += (long)dims[s] * dims[s + 1] * d;
  return n;
}

// ---------------------------------------------------------------------------------------
// Jacobi eigen / SVD (stand-ins for dsyev / dgesdd)
// ---------------------------------------------------------------------------------------
void jacobi_eig(int n, std::vector<double> A, std::vector<double> &w, std::vector<double> &V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[i + n * i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[p + n * q] * A[p + n * q];
    if (off < 1e-30) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p + n * q];
        if (std::fabs(apq) < 1e-300) continue;
        const double theta = (A[q + n * q] - A[p + n * p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = A[k + n * p], akq = A[k + n * q];
          A[k + n * p] = c * akp - s * akq;
          A[k + n * q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = A[p + n * k], aqk = A[q + n * k];
          A[p + n * k] = c * apk - s * aqk;
          A[q + n * k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[k + n * p], vkq = V[k + n * q];
          V[k + n * p] = c * vkp - s * vkq;
          V[k + n * q] = s * vkp + c * vkq;
        }
      }
  }
  w.resize(n);
  for (int i = 0; i < n; ++i) w[i] = A[i + n * i];
  // ascending order, like dsyev
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return w[a] < w[b]; });
  std::vector<double> w2(n), V2((size_t)n * n);
  for (int i = 0; i < n; ++i) {
    w2[i] = w[idx[i]];
    for (int k = 0; k < n; ++k) V2[k + n * i] = V[k + n * idx[i]];
  }
  w = w2;
  V = V2;
}

// One-sided Jacobi SVD of A (m x n, col-major): A = U diag(S) VT, min(m,n) = r columns,
// singular values descending.  U is m x r, VT is r x n.
void jacobi_svd(int m, int n, const double *Ain, std::vector<double> &U, std::vector<double> &S,
                std::vector<double> &VT) {
  const bool tr = m < n;
  const int M = tr ? n : m, N = tr ? m : n;  // work on B (M x N), M >= N
  std::vector<double> B((size_t)M * N), V((size_t)N * N, 0.0);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) B[i + (size_t)M * j] = tr ? Ain[j + (size_t)m * i] : Ain[i + (size_t)m * j];
  for (int i = 0; i < N; ++i) V[i + (size_t)N * i] = 1.0;
  for (int sweep = 0; sweep < 60; ++sweep) {
    double maxrot = 0.0;
    for (int p = 0; p < N; ++p)
      for (int q = p + 1; q < N; ++q) {
        double a = 0, b = 0, c = 0;
        for (int i = 0; i < M; ++i) {
          const double bp = B[i + (size_t)M * p], bq = B[i + (size_t)M * q];
          a += bp * bp;
          b += bq * bq;
          c += bp * bq;
        }
        if (std::fabs(c) <= 1e-15 * std::sqrt(a * b) || c == 0.0) continue;
        maxrot = std::max(maxrot, std::fabs(c) / std::sqrt(a * b));
        const double zeta = (b - a) / (2.0 * c);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = cs * t;
        for (int i = 0; i < M; ++i) {
          const double bp = B[i + (size_t)M * p], bq = B[i + (size_t)M * q];
          B[i + (size_t)M * p] = cs * bp - sn * bq;
          B[i + (size_t)M * q] = sn * bp + cs * bq;
        }
        for (int i = 0; i < N; ++i) {
          const double vp = V[i + (size_t)N * p], vq = V[i + (size_t)N * q];
          V[i + (size_t)N * p] = cs * vp - sn * vq;
          V[i + (size_t)N * q] = sn * vp + cs * vq;
        }
      }
    if (maxrot < 1e-15) break;
  }
  std::vector<double> sv(N);
  for (int j = 0; j < N; ++j) {
    double s = 0;
    for (int i = 0; i < M; ++i) s += B[i + (size_t)M * j] * B[i + (size_t)M * j];
    sv[j] = std::sqrt(s);
  }
  std::vector<int> idx(N);
  for (int i = 0; i < N; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return sv[a] > sv[b]; });
  // left vectors of B: B[:,j]/s_j ; right: V
  std::vector<double> Ub((size_t)M * N), Vb((size_t)N * N);
  S.resize(N);
  for (int jj = 0; jj < N; ++jj) {
    const int j = idx[jj];
    S[jj] = sv[j];
    for (int i = 0; i < M; ++i) Ub[i + (size_t)M * jj] = sv[j] > 0 ? B[i + (size_t)M * j] / sv[j] : 0.0;
    for (int i = 0; i < N; ++i) Vb[i + (size_t)N * jj] = V[i + (size_t)N * j];
  }
  // Complete zero columns of Ub to an orthonormal set (Gram-Schmidt against unit vectors).
  for (int jj = 0; jj < N; ++jj) {
    if (S[jj] > 0) continue;
    for (int e = 0; e < M; ++e) {
      std::vector<double> v(M, 0.0);
      v[e] = 1.0;
      for (int k = 0; k < N; ++k) {
        if (k == jj || (S[k] == 0 && k > jj)) continue;
        double dot = 0;
        for (int i = 0; i < M; ++i) dot += v[i] * Ub[i + (size_t)M * k];
        for (int i = 0; i < M; ++i) v[i] -= dot * Ub[i + (size_t)M * k];
      }
      double nv = 0;
      for (int i = 0; i < M; ++i) nv += v[i] * v[i];
      if (nv > 1e-6) {
        nv = std::sqrt(nv);
        for (int i = 0; i < M; ++i) Ub[i + (size_t)M * jj] = v[i] / nv;
        break;
      }
    }
  }
  const int r = N;
  if (!tr) {  // A = Ub S Vb^T
    U = Ub;
    VT.assign((size_t)r * n, 0.0);
    for (int k = 0; k < r; ++k)
      for (int j = 0; j < n; ++j) VT[k + (size_t)r * j] = Vb[j + (size_t)N * k];
  } else {  // A^T = Ub S Vb^T  =>  A = Vb S Ub^T
    U.assign((size_t)m * r, 0.0);
    for (int k = 0; k < r; ++k)
      for (int i = 0; i < m; ++i) U[i + (size_t)m * k] = Vb[i + (size_t)N * k];
    VT.assign((size_t)r * n, 0.0);
    for (int k = 0; k < r; ++k)
      for (int j = 0; j < n; ++j) VT[k + (size_t)r * j] = Ub[j + (size_t)M * k];
  }
}

// ---------------------------------------------------------------------------------------
// Compact MPO of H = sum_c J_c S_i.S_j - h sum_k Sz_k, channels per bond:
//   0 = done, 1..3*nopen = (site i, op in {Sx, iSy, Sz}) still waiting for its partner,
//   last = nothing placed yet.
// ---------------------------------------------------------------------------------------
struct MpoTerm {
  int a, b;       // source channel at bond k, target channel at bond k+1
  int op;         // 0 = I, 1 = Sx, 2 = iSy, 3 = Sz
  double coef;
};
struct CompactMpo {
  std::vector<int> width;                  // channels at each bond (L+1)
  std::vector<std::vector<MpoTerm>> terms;  // per site
};

CompactMpo build_mpo(int L, int nC, const int *ci, const int *cj, const double *cJ, double h) {
  CompactMpo m;
  m.width.assign(L + 1, 0);
  m.terms.resize(L);
  // open[b] = sorted list of sites i < b that couple to some j >= b.
  std::vector<std::vector<int>> open(L + 1);
  for (int b = 0; b <= L; ++b) {
    for (int i = 0; i < b; ++i) {
      bool any = false;
      for (int c = 0; c < nC; ++c)
        if (std::min(ci[c], cj[c]) == i && std::max(ci[c], cj[c]) >= b && cJ[c] != 0.0) any = true;
      if (any) open[b].push_back(i);
    }
  }
  auto chan = [&](int b, int i, int op) {  // op 1..3
    for (size_t q = 0; q < open[b].size(); ++q)
      if (open[b][q] == i) return 1 + 3 * (int)q + (op - 1);
    return -1;
  };
  for (int b = 0; b <= L; ++b) m.width[b] = 2 + 3 * (int)open[b].size();
  for (int k = 0; k < L; ++k) {
    const int lastL = m.width[k] - 1, lastR = m.width[k + 1] - 1;
    std::vector<MpoTerm> &t = m.terms[k];
    if (k > 0) t.push_back({0, 0, 0, 1.0});       // done -> done
    if (k < L - 1 || true) {
      if (k < L - 1) t.push_back({lastL, lastR, 0, 1.0});  // identity -> identity
    }
    if (h != 0.0) t.push_back({lastL, 0, 3, -h});  // field closes immediately
    for (size_t q = 0; q < open[k].size(); ++q) {
      const int i = open[k][q];
      double J = 0.0;
      for (int c = 0; c < nC; ++c)
        if (std::min(ci[c], cj[c]) == i && std::max(ci[c], cj[c]) == k) J += cJ[c];
      for (int op = 1; op <= 3; ++op) {
        const int src = chan(k, i, op);
        if (J != 0.0) t.push_back({src, 0, op, (op == 2) ? -J : J});
        const int dst = chan(k + 1, i, op);
        if (dst >= 0) t.push_back({src, dst, 0, 1.0});
      }
    }
    // start new channels at site k
    for (int op = 1; op <= 3; ++op) {
      const int dst = chan(k + 1, k, op);
      if (dst >= 0) t.push_back({lastL, dst, op, 1.0});
    }
  }
  return m;
}

double op_elem(int d, int op, int i, int j) {
  switch (op) {
    case 0: return i == j ? 1.0 : 0.0;
    case 1: return op_sx(d, i, j);
    case 2: return op_isy(d, i, j);
    default: return op_sz(d, i, j);
  }
}

double energy_numerator(const CompactMpo &mpo, const MpsView &T, const MpsView &W) {
  const int L = T.L, d = T.d;
  std::vector<std::vector<double>> F(mpo.width[0]), Fn;
  F[mpo.width[0] - 1].assign(1, 1.0);
  for (int c = 0; c + 1 < mpo.width[0]; ++c) F[c].assign(1, 0.0);
  std::vector<double> X;
  for (int k = 0; k < L; ++k) {
    const int aL = T.dims[k], aR = T.dims[k + 1], bL = W.dims[k], bR = W.dims[k + 1];
    Fn.assign(mpo.width[k + 1], std::vector<double>((size_t)aR * bR, 0.0));
    X.resize((size_t)aL * bR);
    for (const MpoTerm &t : mpo.terms[k]) {
      for (int tau = 0; tau < d; ++tau) {
        std::fill(X.begin(), X.end(), 0.0);
        gemm(false, false, aL, bR, bL, 1.0, F[t.a].data(), aL, W.site[k] + (long)tau * bL * bR, bL,
             0.0, X.data(), aL);
        for (int sg = 0; sg < d; ++sg) {
          const double v = t.coef * op_elem(d, t.op, sg, tau);
          if (v == 0.0) continue;
          gemm(true, false, aR, bR, aL, v, T.site[k] + (long)sg * aL * aR, aL, X.data(), aL, 1.0,
               Fn[t.b].data(), aR);
        }
      }
    }
    F.swap(Fn);
  }
  return F[0][0];
}

struct Rng {
  std::mt19937 gen;
  unsigned long long used = 0;
  double uniform() {
    ++used;
    const double numerator = (double)(gen() - 0u);
    const double divisor = (double)(0xffffffffu - 0u) + 1.0;
    return numerator / divisor * (1.0 - 0.0) + 0.0;
  }
};

}  // namespace

// =========================================================================================
// C ABI
// =========================================================================================
extern "C" {

long orc_mps_size(int L, int d, const int *dims) { return mps_size(L, d, dims); }

double orc_inner_product(int L, int d, const int *dimsA, const double *A, const int *dimsB,
                         const double *B) {
  std::vector<double> w1, w2, w3;
  return inner_product(make_view(L, d, dimsA, A), make_view(L, d, dimsB, B), w1, w2, w3);
}

double orc_left_normalize(int L, int d, const int *dims, double *data) {
  std::vector<double> mem, Rm, work;
  return left_normalize(L, d, dims, data, mem, Rm, work);
}

void orc_change_phase(int L, int d, const int *dims, double *data) {
  (void)L;
  const long n = (long)dims[0] * dims[1] * d;
  for (long q = 0; q < n; ++q) data[q] *= -1.0;
}

void orc_apply_grid_op(int L, int d, const int *dims, double *data, int i, int j, const double *S,
                       const double *U, const double *VT, const double *x) {
  MpsView v = make_view(L, d, dims, data);
  std::vector<double> work;
  apply_grid_site(d, dims[i], dims[i + 1], v.site[i], S, U, false, x, work);
  apply_grid_site(d, dims[j], dims[j + 1], v.site[j], S, VT, true, x, work);
}

void orc_apply_svd_op(int L, int d, const int *dims, double *data, int i, int j, const double *S,
                      const double *U, const double *VT, int k, int l, int doHC) {
  MpsView v = make_view(L, d, dims, data);
  std::vector<double> work, op((size_t)d * d);
  svd_site_op(d, k, S, U, false, doHC != 0, op.data());
  apply_site_op(d, dims[i], dims[i + 1], v.site[i], op.data(), work);
  svd_site_op(d, l, S, VT, true, doHC != 0, op.data());
  apply_site_op(d, dims[j], dims[j + 1], v.site[j], op.data(), work);
}

int orc_grid_marsaglia(int dim, int ppc, double *out, int capacity) {
  std::vector<double> one(ppc);
  for (int c = 0; c < ppc; ++c) one[c] = 2 * (c + 0.5) / ppc - 1.0;
  for (int c = 0; c < ppc; ++c) {
    // erf_inv by bisection + Newton (same stand-in the reference build uses)
    const double z = one[c];
    double r = 0.0;
    if (z != 0.0) {
      const double sgn = z < 0 ? -1.0 : 1.0, t = std::fabs(z);
      double lo = 0.0, hi = 6.0;
      for (int it = 0; it < 60; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (std::erf(mid) < t) lo = mid; else hi = mid;
      }
      double x = 0.5 * (lo + hi);
      for (int it = 0; it < 4; ++it) {
        const double f = std::erf(x) - t, df = 1.1283791670955126 * std::exp(-x * x);
        if (df == 0.0) break;
        x -= f / df;
      }
      r = sgn * x;
    }
    one[c] = r;
  }
  long est = 1;
  for (int c = 0; c < dim; ++c) est *= ppc;
  int n = 0;
  std::vector<double> att(dim);
  for (long cnt = 0; cnt < est; ++cnt) {
    long cc = cnt;
    double norm = 0.0;
    for (int k = 0; k < dim; ++k) {
      const int rem = (int)(cc % ppc);
      att[k] = one[rem];
      norm += att[k] * att[k];
      cc = (cc - rem) / ppc;
    }
    if (norm > 1e-16) {
      norm = 1.0 / std::sqrt(norm);
      for (int k = 0; k < dim; ++k) att[k] *= norm;
      bool copy = true;
      for (int s = 0; s < n && copy; ++s) {
        double d2 = 0.0;
        for (int k = 0; k < dim; ++k) {
          const double df = att[k] - out[k + dim * s];
          d2 += df * df;
        }
        if (d2 < 1e-16) copy = false;
      }
      if (copy) {
        if (n >= capacity) return -1;
        for (int k = 0; k < dim; ++k) out[k + dim * n] = att[k];
        ++n;
      }
    }
  }
  return n;
}

int orc_grid_simple(int dim, int denom, double *out, int capacity) {
  // GridGenerator::FillSimple / GenerateNextSimple, GridGenerator.cpp:227-341.
  std::vector<int> st(dim, 0);
  auto next = [&](std::vector<int> &s) {
    if (s[dim - 1] == denom) return false;
    int index = dim - 2;
    while (s[index] == 0) index--;
    if (s[dim - 1] == 0) {
      s[index] -= 1;
      s[index + 1] += 1;
    } else {
      const int last = s[dim - 1];
      s[dim - 1] -= last;
      s[index + 1] += 1 + last;
      s[index] -= 1;
    }
    return true;
  };
  st[0] = denom;
  if (capacity < 2) return -1;
  for (int k = 0; k < dim; ++k) out[k] = out[k + dim] = 0.0;
  out[0] = 1.0;
  out[dim] = -1.0;
  int n = 2;
  std::vector<int> nz(dim);
  while (next(st)) {
    int factor = 1, nnz = 0;
    for (int k = 0; k < dim; ++k)
      if (st[k] > 0) {
        factor *= 2;
        nz[nnz++] = k;
      }
    if (n + factor > capacity) return -1;
    for (int c = 0; c < factor; ++c) {
      for (int k = 0; k < dim; ++k) out[k + dim * (n + c)] = 0.0;
      int cc = c;
      for (int q = 0; q < nnz; ++q) {
        const int rem = cc % 2;
        out[nz[q] + dim * (n + c)] = (rem == 0 ? 1 : -1) * std::sqrt((double)st[nz[q]] / denom);
        cc = (cc - rem) / 2;
      }
    }
    n += factor;
  }
  return n;
}

int orc_trotter(int d, double J, double dtau, double *U, double *S, double *VT) {
  const int n = d * d;
  std::vector<double> H((size_t)n * n);
  for (int r1 = 0; r1 < d; ++r1)
    for (int c1 = 0; c1 < d; ++c1)
      for (int r2 = 0; r2 < d; ++r2)
        for (int c2 = 0; c2 < d; ++c2)
          H[r1 + d * (r2 + d * (c1 + d * c2))] = op_sx(d, r1, c1) * op_sx(d, r2, c2) -
                                                 op_isy(d, r1, c1) * op_isy(d, r2, c2) +
                                                 op_sz(d, r1, c1) * op_sz(d, r2, c2);
  std::vector<double> w, V;
  jacobi_eig(n, H, w, V);
  std::vector<double> work((size_t)n * n), P((size_t)n * n, 0.0);
  for (int c = 0; c < n; ++c) {
    const double pf = std::exp(-0.5 * dtau * J * w[c]);
    for (int r = 0; r < n; ++r) work[r + n * c] = pf * V[r + n * c];
  }
  gemm(false, true, n, n, n, 1.0, work.data(), n, work.data(), n, 0.0, P.data(), n);
  // reshuffle (TrotterHeisenberg.cpp:203-219)
  std::vector<double> Q((size_t)n * n);
  for (int r1 = 0; r1 < d; ++r1)
    for (int c1 = 0; c1 < d; ++c1)
      for (int r2 = 0; r2 < d; ++r2)
        for (int c2 = 0; c2 < d; ++c2)
          Q[r1 + d * (c1 + d * (r2 + d * c2))] = P[r1 + d * (r2 + d * (c1 + d * c2))];
  std::vector<double> Uv, Sv, VTv;
  jacobi_svd(n, n, Q.data(), Uv, Sv, VTv);
  std::copy(Uv.begin(), Uv.end(), U);
  std::copy(Sv.begin(), Sv.end(), S);
  std::copy(VTv.begin(), VTv.end(), VT);
  return 0;
}

double orc_local_energy_numerator(int L, int d, const int *dimsT, const double *T, const int *dimsW,
                                  const double *W, int nC, const int *ci, const int *cj,
                                  const double *cJ, double h) {
  CompactMpo mpo = build_mpo(L, nC, ci, cj, cJ, h);
  return energy_numerator(mpo, make_view(L, d, dimsT, T), make_view(L, d, dimsW, W));
}

int orc_compress(int L, int d, int *dims, const double *data_in, double *data_out, int truncD) {
  // Tensors kept as separate vectors while dims change.
  std::vector<std::vector<double>> site(L);
  {
    long off = 0;
    for (int s = 0; s < L; ++s) {
      const long n = (long)dims[s] * dims[s + 1] * d;
      site[s].assign(data_in + off, data_in + off + n);
      off += n;
    }
  }
  const double schmidt_cut = 1e-13;  // TwoSiteObject.cpp:16
  auto step = [&](int s, bool movingright) {
    const int DL = dims[s], DM = dims[s + 1], DR = dims[s + 2];
    // Compose (TwoSiteObject.cpp:111-115): two[dl,dr] = A[dl] (DL x DM) * B[dr] (DM x DR)
    const int mL = DL * d, mR = DR * d;
    std::vector<double> mem((size_t)mL * mR, 0.0), blk((size_t)DL * DR);
    for (int il = 0; il < d; ++il)
      for (int ir = 0; ir < d; ++ir) {
        std::fill(blk.begin(), blk.end(), 0.0);
        gemm(false, false, DL, DR, DM, 1.0, site[s].data() + (long)il * DL * DM, DL,
             site[s + 1].data() + (long)ir * DM * DR, DM, 0.0, blk.data(), DL);
        for (int a = 0; a < DL; ++a)
          for (int b = 0; b < DR; ++b) mem[(a + DL * il) + (size_t)mL * (b + DR * ir)] = blk[a + DL * b];
      }
    std::vector<double> Uv, Sv, VTv;
    jacobi_svd(mL, mR, mem.data(), Uv, Sv, VTv);
    const int dimMin = std::min(mL, mR);
    int trunc = truncD, idx = dimMin;
    for (int c = 0; c < dimMin; ++c)
      if (Sv[c] < schmidt_cut) {
        idx = c;
        break;
      }
    if (idx < trunc) trunc = idx;
    trunc = std::min(trunc, dimMin);
    std::vector<double> A((size_t)DL * trunc * d), B((size_t)trunc * DR * d);
    for (int ip = 0; ip < d; ++ip)
      for (int a = 0; a < DL; ++a)
        for (int b = 0; b < trunc; ++b)
          A[a + DL * (b + trunc * ip)] = Uv[(a + DL * ip) + (size_t)mL * b] * (movingright ? 1.0 : Sv[b]);
    for (int ip = 0; ip < d; ++ip)
      for (int a = 0; a < trunc; ++a)
        for (int b = 0; b < DR; ++b)
          B[a + trunc * (b + DR * ip)] = VTv[a + (size_t)dimMin * (b + DR * ip)] * (movingright ? Sv[a] : 1.0);
    site[s] = A;
    site[s + 1] = B;
    dims[s + 1] = trunc;
  };
  for (int s = 0; s < L - 1; ++s) step(s, true);
  for (int s = L - 2; s >= 0; --s) step(s, false);
  long off = 0;
  int maxD = dims[0];
  for (int s = 0; s < L; ++s) {
    std::copy(site[s].begin(), site[s].end(), data_out + off);
    off += (long)site[s].size();
    maxD = std::max(maxD, dims[s]);
  }
  return maxD;
}

int orc_walk(const orc_walk_config *cfg, const int *dimsT, const double *trial, const int *ci,
             const int *cj, const double *cJ, const double *Jvals, const double *Utab,
             const double *Stab, const double *VTtab, const double *grid, const int *dimsW,
             double *walkers, double *weights, double *overlaps, double *ehist, int *n_walkers,
             double *E0, double *st_sumw, double *st_EP, double *st_ET, double *st_omega, int *st_n,
             double *pw_weight, double *pw_overlap, double *pw_energy, int *pw_parent,
             double *trace, unsigned long long *draws_used) {
  return orc_walk_dims(cfg, dimsT, trial, ci, cj, cJ, Jvals, Utab, Stab, VTtab, grid, dimsW, nullptr, walkers,
                       weights, overlaps, ehist, n_walkers, E0, st_sumw, st_EP, st_ET, st_omega, st_n, pw_weight,
                       pw_overlap, pw_energy, pw_parent, trace, draws_used);
}

int orc_walk_dims(const orc_walk_config *cfg, const int *dimsT, const double *trial, const int *ci,
                  const int *cj, const double *cJ, const double *Jvals, const double *Utab,
                  const double *Stab, const double *VTtab, const double *grid, const int *dimsW,
                  int *wdims, double *walkers, double *weights, double *overlaps, double *ehist,
                  int *n_walkers, double *E0, double *st_sumw, double *st_EP, double *st_ET,
                  double *st_omega, int *st_n, double *pw_weight, double *pw_overlap, double *pw_energy,
                  int *pw_parent, double *trace, unsigned long long *draws_used) {
  const int L = cfg->L, d = cfg->d, nC = cfg->nC, G = cfg->G, cap = cfg->capacity;
  const int n2 = d * d;
  if (L < 2 || nC < 1 || G < 1 || *n_walkers < 1 || *n_walkers > cap) return -2;
  const long szW = mps_size(L, d, dimsW);
  const long szT = mps_size(L, d, dimsT);
  // walker w's own bond dims (MPSstate keeps its VirtualD, MPSstate.cpp:13-40)
  auto dims_of = [&](int w) -> const int * { return wdims ? wdims + (size_t)w * (L + 1) : dimsW; };
  (void)szT;
  std::vector<int> jidx(nC, -1);
  for (int c = 0; c < nC; ++c)
    for (int q = 0; q < cfg->nJ; ++q)
      if (cJ[c] == Jvals[q]) {
        jidx[c] = q;
        break;
      }
  for (int c = 0; c < nC; ++c)
    if (jidx[c] < 0 || ci[c] >= cj[c]) return -2;
  MpsView T = make_view(L, d, dimsT, trial);
  // Trial terms (MPSQMC2.cpp:303-330): site i gets sqrt(s_k) U_k^T, site j gets sqrt(s_l) V_l^T.
  std::vector<std::vector<double>> termI((size_t)nC * n2), termJ((size_t)nC * n2);
  {
    std::vector<double> work, op((size_t)d * d);
    for (int c = 0; c < nC; ++c) {
      const double *S = Stab + (size_t)n2 * jidx[c];
      const double *U = Utab + (size_t)n2 * n2 * jidx[c];
      const double *VT = VTtab + (size_t)n2 * n2 * jidx[c];
      const int i = ci[c], j = cj[c];
      for (int k = 0; k < n2; ++k) {
        termI[(size_t)c * n2 + k].assign(T.site[i], T.site[i] + (long)dimsT[i] * dimsT[i + 1] * d);
        svd_site_op(d, k, S, U, false, true, op.data());
        apply_site_op(d, dimsT[i], dimsT[i + 1], termI[(size_t)c * n2 + k].data(), op.data(), work);
        termJ[(size_t)c * n2 + k].assign(T.site[j], T.site[j] + (long)dimsT[j] * dimsT[j + 1] * d);
        svd_site_op(d, k, S, VT, true, true, op.data());
        apply_site_op(d, dimsT[j], dimsT[j + 1], termJ[(size_t)c * n2 + k].data(), op.data(), work);
      }
    }
  }
  CompactMpo mpo = build_mpo(L, nC, ci, cj, cJ, cfg->h);
  // Single-site propagator exp(0.5*h*dtau*Sz) (TrotterHeisenberg.cpp:80-88, 436-455).
  std::vector<double> onesite((size_t)d * d, 0.0);
  for (int s = 0; s < d; ++s) onesite[s + d * s] = std::exp(0.5 * cfg->h * cfg->dtau * op_sz(d, s, s));
  const bool field = cfg->h != 0.0;

  Rng rng;
  rng.gen.seed(cfg->seed);
  rng.gen.discard(cfg->skip);

  int N = *n_walkers;
  std::vector<double> energy(cap);
  auto energy_of = [&](int w) {
    const MpsView Wv = make_view(L, d, dims_of(w), walkers + (size_t)w * szW);
    return energy_numerator(mpo, T, Wv) / overlaps[w];
  };
  // Initial EnergyFunctionAndHistory(1, &E, false), MPSQMC2.cpp:447.
  {
    double num = 0.0, den = 0.0;
    for (int w = 0; w < N; ++w) {
      const double e = energy_of(w);
      num += weights[w] * e;
      den += weights[w];
    }
    *E0 = num / den;
  }
  const int nth = cfg->nthreads > 0 ? cfg->nthreads : 0;
  std::vector<double> newbuf((size_t)cap * szW);
  std::vector<double> uni;
  for (int step = 1; step <= cfg->nsteps; ++step) {
    // Uniforms of the propagation, in the order one thread would draw them (walker-major).
    uni.resize((size_t)N * nC);
    for (size_t q = 0; q < uni.size(); ++q) uni[q] = rng.uniform();
    double *tr_step = trace ? trace + (size_t)(step - 1) * cap * nC * (n2 * n2 + 5) : nullptr;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nth > 0 ? nth : omp_get_max_threads())
    for (int w = 0; w < N; ++w) {
      std::vector<double> w1, w2, w3, mem, Rm, qwork, work, pdf(G), C((size_t)n2 * n2);
      double *phi = walkers + (size_t)w * szW;
      const int *dW = dims_of(w);
      MpsView P = make_view(L, d, dW, phi);
      auto set_overlap = [&]() {  // Walker::setOverlap, Walker.cpp:54-66
        left_normalize(L, d, dW, phi, mem, Rm, qwork);
        double val = inner_product(T, P, w1, w2, w3);
        if (val < 0.0) {
          const long n0 = (long)dW[0] * dW[1] * d;
          for (long q = 0; q < n0; ++q) phi[q] *= -1.0;
          val *= -1;
        }
        overlaps[w] = val;
      };
      if (field)
        for (int s = 0; s < L; ++s) apply_site_op(d, dW[s], dW[s + 1], P.site[s], onesite.data(), work);
      set_overlap();
      MpsView term = T;
      for (int c = 0; c < nC; ++c) {
        const int i = ci[c], j = cj[c];
        for (int a = 0; a < n2; ++a)
          for (int b = 0; b < n2; ++b) {
            term.site[i] = termI[(size_t)c * n2 + a].data();
            term.site[j] = termJ[(size_t)c * n2 + b].data();
            C[a + n2 * b] = inner_product(term, P, w1, w2, w3);
          }
        term.site[i] = T.site[i];
        term.site[j] = T.site[j];
        double norm = 0.0;
        for (int p = 0; p < G; ++p) {
          double v = 0.0;
          for (int l = 0; l < n2; ++l)
            for (int r = 0; r < n2; ++r) v += C[l + n2 * r] * grid[l + n2 * p] * grid[r + n2 * p];
          v = std::max(0.0, v);
          v *= n2 / (overlaps[w] * G);
          pdf[p] = v;
          norm += v;
        }
        const double inv = 1.0 / norm;
        for (int p = 0; p < G; ++p) pdf[p] *= inv;
        weights[w] *= norm;
        const double u = uni[(size_t)w * nC + c];
        int count = 0;
        double cum = pdf[0];
        while ((cum <= u) && (count < G - 1)) {
          count += 1;
          cum += pdf[count];
        }
        const int q = jidx[c];
        apply_grid_site(d, dW[i], dW[i + 1], P.site[i], Stab + (size_t)n2 * q,
                        Utab + (size_t)n2 * n2 * q, false, grid + (size_t)n2 * count, work);
        apply_grid_site(d, dW[j], dW[j + 1], P.site[j], Stab + (size_t)n2 * q,
                        VTtab + (size_t)n2 * n2 * q, true, grid + (size_t)n2 * count, work);
        set_overlap();
        if (tr_step) {
          double *t = tr_step + ((size_t)w * nC + c) * (n2 * n2 + 5);
          for (int a = 0; a < n2 * n2; ++a) t[a] = C[a];
          t[n2 * n2 + 0] = norm;
          t[n2 * n2 + 1] = u;
          t[n2 * n2 + 2] = count;
          t[n2 * n2 + 3] = weights[w];
          t[n2 * n2 + 4] = overlaps[w];
        }
      }
      if (field)
        for (int s = 0; s < L; ++s) apply_site_op(d, dW[s], dW[s + 1], P.site[s], onesite.data(), work);
      set_overlap();
    }
    double sumw = 0.0;
    for (int w = 0; w < N; ++w) sumw += weights[w];
    const double avgW = sumw / N;
    const double scaling = cfg->Ndesired / (N * avgW);
    const double ET = std::log(scaling) / cfg->dtau;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nth > 0 ? nth : omp_get_max_threads())
    for (int w = 0; w < N; ++w) energy[w] = energy_of(w);
    double num = 0.0, den = 0.0, sE = 0.0, sE2 = 0.0;
    for (int w = 0; w < N; ++w) {
      num += weights[w] * energy[w];
      den += weights[w];
      ehist[w] += energy[w];
      const double e = ehist[w] / step;
      sE += e;
      sE2 += e * e;
    }
    const double omega = (sE2 - sE * sE / N) / N;
    const int s0 = step - 1;
    st_sumw[s0] = sumw;
    st_EP[s0] = num / den;
    st_ET[s0] = ET;
    st_omega[s0] = omega;
    st_n[s0] = N;
    for (int w = 0; w < N; ++w) {
      if (pw_weight) pw_weight[(size_t)s0 * cap + w] = weights[w];
      if (pw_overlap) pw_overlap[(size_t)s0 * cap + w] = overlaps[w];
      if (pw_energy) pw_energy[(size_t)s0 * cap + w] = energy[w];
    }
    // SeparatePopulationControl, MPSQMC2.cpp:613-686 (threshold), or the engine's comb and
    // interval variants (orc_walk_config).
    int Nn = 0;
    std::vector<double> nw, no, nh;
    std::vector<int> par;
    const int K = cfg->popctl_interval > 0 ? cfg->popctl_interval : 1;
    const bool branch_now = (step % K) == 0;
    const bool comb = branch_now && cfg->comb != 0;
    const double ucomb = comb ? rng.uniform() : 0.0;
    double Scomb = 0.0;
    for (int w = 0; w < N; ++w) {
      const double sw = weights[w] * scaling;
      int nCopies = 1;
      double newW = sw;
      if (comb) {
        nCopies = (int)(std::ceil(Scomb + sw - ucomb) - std::ceil(Scomb - ucomb));
        Scomb += sw;
        newW = 1.0;
      } else if (branch_now) {
        if (newW < 0.25) {
          nCopies = (int)(sw + rng.uniform());
          newW = 1.0;
        }
        if (newW > 1.5) {
          nCopies = (int)(sw + rng.uniform());
          newW = sw / nCopies;
        }
      }
      if (Nn + nCopies > cap) return -1;
      for (int c = 0; c < nCopies; ++c) {
        std::memcpy(newbuf.data() + (size_t)(Nn + c) * szW, walkers + (size_t)w * szW, sizeof(double) * szW);
        nw.push_back(newW);
        no.push_back(overlaps[w]);
        nh.push_back(ehist[w]);
        par.push_back(w);
      }
      Nn += nCopies;
    }
    std::memcpy(walkers, newbuf.data(), sizeof(double) * (size_t)Nn * szW);
    if (wdims) {  // copies keep their parent's bond dims
      std::vector<int> nd((size_t)Nn * (L + 1));
      for (int w = 0; w < Nn; ++w)
        std::memcpy(nd.data() + (size_t)w * (L + 1), wdims + (size_t)par[w] * (L + 1), sizeof(int) * (L + 1));
      std::memcpy(wdims, nd.data(), sizeof(int) * nd.size());
    }
    for (int w = 0; w < Nn; ++w) {
      weights[w] = nw[w];
      overlaps[w] = no[w];
      ehist[w] = nh[w];
      if (pw_parent) pw_parent[(size_t)s0 * cap + w] = par[w];
    }
    if (pw_parent)
      for (int w = Nn; w < cap; ++w) pw_parent[(size_t)s0 * cap + w] = -1;
    N = Nn;
    if (N == 0) {
      *n_walkers = 0;
      *draws_used = rng.used;
      return -3;
    }
  }
  *n_walkers = N;
  *draws_used = rng.used;
  return 0;
}

}  // extern "C"
