// Test infrastructure only: minimal column-major LU routines with the LAPACK
// Fortran ABI that the reference declares (lib/include/basic_linear_systems.hpp:203-205).
// No LAPACK is installed here; the GMRES-FMM path only uses them for tiny geometric
// solves (circumcenters, 2x2/3x3 systems).  Partial pivoting, 1-based ipiv.
#include <cmath>
#include <utility>
#include <vector>

extern "C" void dgetrf_(const int* m_, const int* n_, double* a, const int* lda_, int* ipiv, int* info) {
  const int m = *m_, n = *n_, lda = *lda_;
  *info = 0;
  const int kmax = m < n ? m : n;
  for (int k = 0; k < kmax; ++k) {
    int piv = k;
    double best = std::abs(a[k + k * lda]);
    for (int i = k + 1; i < m; ++i)
      if (std::abs(a[i + k * lda]) > best) {
        best = std::abs(a[i + k * lda]);
        piv = i;
      }
    ipiv[k] = piv + 1;
    if (best == 0.0) {
      if (*info == 0) *info = k + 1;
      continue;
    }
    if (piv != k)
      for (int j = 0; j < n; ++j) std::swap(a[k + j * lda], a[piv + j * lda]);
    const double inv = 1.0 / a[k + k * lda];
    for (int i = k + 1; i < m; ++i) a[i + k * lda] *= inv;
    for (int j = k + 1; j < n; ++j) {
      const double akj = a[k + j * lda];
      for (int i = k + 1; i < m; ++i) a[i + j * lda] -= a[i + k * lda] * akj;
    }
  }
}

extern "C" void dgetrs_(const char* trans, const int* n_, const int* nrhs_, const double* a, const int* lda_, const int* ipiv, double* b,
                        const int* ldb_, int* info) {
  const int n = *n_, nrhs = *nrhs_, lda = *lda_, ldb = *ldb_;
  *info = 0;
  const bool T = (*trans == 'T' || *trans == 't' || *trans == 'C' || *trans == 'c');
  for (int r = 0; r < nrhs; ++r) {
    double* x = b + r * ldb;
    if (!T) {
      for (int k = 0; k < n; ++k)
        if (ipiv[k] - 1 != k) std::swap(x[k], x[ipiv[k] - 1]);
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < i; ++k) x[i] -= a[i + k * lda] * x[k];
      for (int i = n - 1; i >= 0; --i) {
        for (int k = i + 1; k < n; ++k) x[i] -= a[i + k * lda] * x[k];
        x[i] /= a[i + i * lda];
      }
    } else {  // A^T x = b: U^T y = b, L^T z = y, then undo the row swaps
      for (int i = 0; i < n; ++i) {
        for (int k = 0; k < i; ++k) x[i] -= a[k + i * lda] * x[k];
        x[i] /= a[i + i * lda];
      }
      for (int i = n - 1; i >= 0; --i)
        for (int k = i + 1; k < n; ++k) x[i] -= a[k + i * lda] * x[k];
      for (int k = n - 1; k >= 0; --k)
        if (ipiv[k] - 1 != k) std::swap(x[k], x[ipiv[k] - 1]);
    }
  }
}

extern "C" void dgetri_(const int* n_, double* a, const int* lda_, const int* ipiv, double* work, int* lwork, int* info) {
  const int n = *n_, lda = *lda_;
  if (*lwork == -1) {
    work[0] = n;
    *info = 0;
    return;
  }
  std::vector<double> inv((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) inv[j + j * n] = 1.0;
  int nn = n, one = n, ldb = n;
  dgetrs_("N", &nn, &one, a, lda_, ipiv, inv.data(), &ldb, info);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) a[i + j * lda] = inv[i + j * n];
}

// dgesvd_ with jobu = jobvt = 'A' (the only form the reference calls, lib/include/
// basic_linear_systems.hpp:773-830): one-sided Jacobi SVD (Hestenes 1958) of the tall
// orientation B (A, or A^T when m < n), singular values sorted descending, U completed to a
// square orthonormal basis by Gram-Schmidt against the unit vectors.  The geometric solves of
// the gradient fit (3x3 normal systems) are full rank, where every SVD gives the same solution.
extern "C" void dgesvd_(const char*, const char*, const int* m_, const int* n_, double* a, const int* lda_, double* s, double* u,
                        const int* ldu_, double* vt, const int* ldvt_, double* work, const int* lwork, int* info) {
  *info = 0;
  if (*lwork == -1) {
    work[0] = 1;
    return;
  }
  const int m = *m_, n = *n_, lda = *lda_, ldu = *ldu_, ldvt = *ldvt_;
  const bool tall = m >= n;
  const int M = tall ? m : n, N = tall ? n : m;
  std::vector<double> W((size_t)M * N), V((size_t)N * N, 0.0);  // column-major M x N, N x N
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < n; ++j) (tall ? W[i + (size_t)j * M] : W[j + (size_t)i * M]) = a[i + (size_t)j * lda];
  for (int j = 0; j < N; ++j) V[j + (size_t)j * N] = 1.0;
  const double eps = 1e-15;
  for (int sweep = 0; sweep < 60; ++sweep) {
    bool rotated = false;
    for (int p = 0; p < N - 1; ++p)
      for (int q = p + 1; q < N; ++q) {
        double al = 0, be = 0, ga = 0;
        for (int i = 0; i < M; ++i) {
          const double x = W[i + (size_t)p * M], y = W[i + (size_t)q * M];
          al += x * x;
          be += y * y;
          ga += x * y;
        }
        if (ga == 0.0 || std::abs(ga) <= eps * std::sqrt(al * be)) continue;
        rotated = true;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::abs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / std::sqrt(1.0 + t * t), sn = c * t;
        for (int i = 0; i < M; ++i) {
          const double x = W[i + (size_t)p * M], y = W[i + (size_t)q * M];
          W[i + (size_t)p * M] = c * x - sn * y;
          W[i + (size_t)q * M] = sn * x + c * y;
        }
        for (int i = 0; i < N; ++i) {
          const double x = V[i + (size_t)p * N], y = V[i + (size_t)q * N];
          V[i + (size_t)p * N] = c * x - sn * y;
          V[i + (size_t)q * N] = sn * x + c * y;
        }
      }
    if (!rotated) break;
  }
  std::vector<double> sig(N);
  std::vector<int> ord(N);
  for (int j = 0; j < N; ++j) {
    double ss = 0;
    for (int i = 0; i < M; ++i) ss += W[i + (size_t)j * M] * W[i + (size_t)j * M];
    sig[j] = std::sqrt(ss);
    ord[j] = j;
  }
  for (int i = 1; i < N; ++i)  // insertion sort, descending
    for (int k = i; k > 0 && sig[ord[k]] > sig[ord[k - 1]]; --k) std::swap(ord[k], ord[k - 1]);
  // Ub (M x M): normalised columns of W for non-zero values, then Gram-Schmidt completion
  std::vector<double> Ub((size_t)M * M, 0.0), Vb((size_t)N * N);
  int filled = 0;
  for (int k = 0; k < N; ++k) {
    const int j = ord[k];
    s[k] = sig[j];
    for (int i = 0; i < N; ++i) Vb[i + (size_t)k * N] = V[i + (size_t)j * N];
    if (sig[j] > 0) {
      for (int i = 0; i < M; ++i) Ub[i + (size_t)k * M] = W[i + (size_t)j * M] / sig[j];
      filled = k + 1;
    }
  }
  for (int e = 0; filled < M && e < M; ++e) {
    std::vector<double> c(M, 0.0);
    c[e] = 1.0;
    for (int pass = 0; pass < 2; ++pass)
      for (int k = 0; k < filled; ++k) {
        double d = 0;
        for (int i = 0; i < M; ++i) d += Ub[i + (size_t)k * M] * c[i];
        for (int i = 0; i < M; ++i) c[i] -= d * Ub[i + (size_t)k * M];
      }
    double nn = 0;
    for (int i = 0; i < M; ++i) nn += c[i] * c[i];
    nn = std::sqrt(nn);
    if (nn < 1e-8) continue;
    for (int i = 0; i < M; ++i) Ub[i + (size_t)filled * M] = c[i] / nn;
    ++filled;
  }
  // B = Ub S Vb^T; A = B (tall) or B^T = Vb S Ub^T
  if (tall) {
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) u[i + (size_t)j * ldu] = Ub[i + (size_t)j * M];
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) vt[i + (size_t)j * ldvt] = Vb[j + (size_t)i * N];
  } else {
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) u[i + (size_t)j * ldu] = Vb[i + (size_t)j * N];
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) vt[i + (size_t)j * ldvt] = Ub[j + (size_t)i * M];
  }
}
