// Small dense FP64 linear algebra for the host-side set-up objects (column-major).
// Householder QR follows LAPACK's dgeqr2/dorg2r conventions (the reference calls dgeqrf/dorgqr
// with lwork = n, which selects those unblocked routines), so MPStensor::QR gives the
// reference's signs.  Eigen- and singular-value problems use Jacobi rotations.
#ifndef MQ_HOST_LINALG_H
#define MQ_HOST_LINALG_H

#include <algorithm>
#include <cmath>
#include <vector>

namespace mqh {

// C = alpha op(A) op(B) + beta C; A is m x k after op, B is k x n after op.
inline void gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double *A, int lda, const double *B,
                 int ldb, double beta, double *C, int ldc) {
  for (int j = 0; j < n; ++j) {
    double *c = C + (long)ldc * j;
    if (beta == 0.0)
      for (int i = 0; i < m; ++i) c[i] = 0.0;
    else if (beta != 1.0)
      for (int i = 0; i < m; ++i) c[i] *= beta;
    for (int p = 0; p < k; ++p) {
      const double b = alpha * (tb ? B[j + (long)ldb * p] : B[p + (long)ldb * j]);
      if (b == 0.0) continue;
      if (!ta) {
        const double *a = A + (long)lda * p;
        for (int i = 0; i < m; ++i) c[i] += b * a[i];
      } else {
        for (int i = 0; i < m; ++i) c[i] += b * A[p + (long)lda * i];
      }
    }
  }
}

inline double hypot2(double x, double y) {
  const double a = std::fabs(x), b = std::fabs(y);
  const double w = std::max(a, b), z = std::min(a, b);
  if (z == 0.0) return w;
  const double r = z / w;
  return w * std::sqrt(1.0 + r * r);
}

// Householder QR of A (m x n, m >= n, ld lda): on return A holds Q, R (n x n, ld ldr) holds R.
inline void householder_qr(int m, int n, double *A, int lda, double *R, int ldr) {
  std::vector<double> tau(n), w(n);
  for (int i = 0; i < n; ++i) {
    double *col = A + (long)lda * i;
    double ss = 0.0;
    for (int r = i + 1; r < m; ++r) ss += col[r] * col[r];
    double t = 0.0;
    if (m - i > 1 && ss > 0.0) {
      const double alpha = col[i];
      const double mag = hypot2(alpha, std::sqrt(ss));
      const double beta = alpha >= 0.0 ? -mag : mag;
      t = (beta - alpha) / beta;
      const double sc = 1.0 / (alpha - beta);
      for (int r = i + 1; r < m; ++r) col[r] *= sc;
      col[i] = beta;
    }
    tau[i] = t;
    if (t != 0.0)
      for (int j = i + 1; j < n; ++j) {
        double *cj = A + (long)lda * j;
        double s = cj[i];
        for (int r = i + 1; r < m; ++r) s += col[r] * cj[r];
        const double f = t * s;
        cj[i] -= f;
        for (int r = i + 1; r < m; ++r) cj[r] -= f * col[r];
      }
  }
  for (int c = 0; c < n; ++c)
    for (int r = 0; r < n; ++r) R[r + (long)ldr * c] = r <= c ? A[r + (long)lda * c] : 0.0;
  for (int i = n - 1; i >= 0; --i) {
    double *col = A + (long)lda * i;
    const double t = tau[i];
    if (t != 0.0)
      for (int j = i + 1; j < n; ++j) {
        double *cj = A + (long)lda * j;
        double s = cj[i];
        for (int r = i + 1; r < m; ++r) s += col[r] * cj[r];
        const double f = t * s;
        cj[i] -= f;
        for (int r = i + 1; r < m; ++r) cj[r] -= f * col[r];
      }
    for (int r = 0; r < m; ++r) col[r] = r > i ? -t * col[r] : (r == i ? 1.0 - t : 0.0);
  }
}

// Symmetric eigenproblem (cyclic Jacobi): eigenvalues ascending in w, eigenvectors in V columns.
inline void sym_eig(int n, std::vector<double> A, std::vector<double> &w, std::vector<double> &V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[i + (size_t)n * i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) off += A[p + (size_t)n * q] * A[p + (size_t)n * q];
    if (off < 1e-32) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p + (size_t)n * q];
        if (apq == 0.0) continue;
        const double th = (A[q + (size_t)n * q] - A[p + (size_t)n * p]) / (2.0 * apq);
        const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double a = A[k + (size_t)n * p], b = A[k + (size_t)n * q];
          A[k + (size_t)n * p] = c * a - s * b;
          A[k + (size_t)n * q] = s * a + c * b;
        }
        for (int k = 0; k < n; ++k) {
          const double a = A[p + (size_t)n * k], b = A[q + (size_t)n * k];
          A[p + (size_t)n * k] = c * a - s * b;
          A[q + (size_t)n * k] = s * a + c * b;
        }
        for (int k = 0; k < n; ++k) {
          const double a = V[k + (size_t)n * p], b = V[k + (size_t)n * q];
          V[k + (size_t)n * p] = c * a - s * b;
          V[k + (size_t)n * q] = s * a + c * b;
        }
      }
  }
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return A[a + (size_t)n * a] < A[b + (size_t)n * b]; });
  std::vector<double> V2((size_t)n * n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    w[i] = A[idx[i] + (size_t)n * idx[i]];
    for (int k = 0; k < n; ++k) V2[k + (size_t)n * i] = V[k + (size_t)n * idx[i]];
  }
  V.swap(V2);
}

// Thin SVD A (m x n) = U diag(S) VT with r = min(m, n) singular values, descending
// (one-sided Jacobi on the taller orientation).
inline void svd(int m, int n, const double *A, std::vector<double> &U, std::vector<double> &S,
                std::vector<double> &VT) {
  const bool tr = m < n;
  const int M = tr ? n : m, N = tr ? m : n;
  std::vector<double> B((size_t)M * N), V((size_t)N * N, 0.0);
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < M; ++i) B[i + (size_t)M * j] = tr ? A[j + (size_t)m * i] : A[i + (size_t)m * j];
  for (int i = 0; i < N; ++i) V[i + (size_t)N * i] = 1.0;
  for (int sweep = 0; sweep < 80; ++sweep) {
    double worst = 0.0;
    for (int p = 0; p < N; ++p)
      for (int q = p + 1; q < N; ++q) {
        double a = 0, b = 0, c = 0;
        for (int i = 0; i < M; ++i) {
          const double x = B[i + (size_t)M * p], y = B[i + (size_t)M * q];
          a += x * x;
          b += y * y;
          c += x * y;
        }
        if (c == 0.0 || std::fabs(c) <= 1e-15 * std::sqrt(a * b)) continue;
        worst = std::max(worst, std::fabs(c) / std::sqrt(a * b));
        const double z = (b - a) / (2.0 * c);
        const double t = (z >= 0 ? 1.0 : -1.0) / (std::fabs(z) + std::sqrt(1.0 + z * z));
        const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = cs * t;
        for (int i = 0; i < M; ++i) {
          const double x = B[i + (size_t)M * p], y = B[i + (size_t)M * q];
          B[i + (size_t)M * p] = cs * x - sn * y;
          B[i + (size_t)M * q] = sn * x + cs * y;
        }
        for (int i = 0; i < N; ++i) {
          const double x = V[i + (size_t)N * p], y = V[i + (size_t)N * q];
          V[i + (size_t)N * p] = cs * x - sn * y;
          V[i + (size_t)N * q] = sn * x + cs * y;
        }
      }
    if (worst < 1e-15) break;
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
  std::vector<double> Ub((size_t)M * N), Vb((size_t)N * N);
  S.resize(N);
  for (int jj = 0; jj < N; ++jj) {
    const int j = idx[jj];
    S[jj] = sv[j];
    for (int i = 0; i < M; ++i) Ub[i + (size_t)M * jj] = sv[j] > 0 ? B[i + (size_t)M * j] / sv[j] : 0.0;
    for (int i = 0; i < N; ++i) Vb[i + (size_t)N * jj] = V[i + (size_t)N * j];
  }
  // complete the columns of zero singular values to an orthonormal set
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
  if (!tr) {
    U = Ub;
    VT.assign((size_t)r * n, 0.0);
    for (int k = 0; k < r; ++k)
      for (int j = 0; j < n; ++j) VT[k + (size_t)r * j] = Vb[j + (size_t)N * k];
  } else {
    U.assign((size_t)m * r, 0.0);
    for (int k = 0; k < r; ++k)
      for (int i = 0; i < m; ++i) U[i + (size_t)m * k] = Vb[i + (size_t)N * k];
    VT.assign((size_t)r * n, 0.0);
    for (int k = 0; k < r; ++k)
      for (int j = 0; j < n; ++j) VT[k + (size_t)r * j] = Ub[j + (size_t)M * k];
  }
}

}  // namespace mqh

#endif
