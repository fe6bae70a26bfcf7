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
