// Roots of the GMRES polynomial preconditioner (host side).
//
// The reference preconditions its GMRES-FMM solve with incomplete factorisations (ILU0, ILUT,
// MILU, overlapping Schwarz blocks) of a sparse near-field matrix (buildSparseMatrixForILU,
// bem/BEM_solveBVP_GMRES_FMM.hpp:215-1050), applied on the left to every A.v and to b
// (:2124-2170).  Triangular solves are sequential; on the device the near-field matrix is used
// through a polynomial instead, applied on the right: p(B) with B = A_near D^{-1} is the GMRES polynomial of a
// short Krylov run on B, whose roots are the harmonic Ritz values of that run (the polynomial
// preconditioner of Loe and Morgan, "Toward efficient polynomial preconditioning for GMRES",
// Numer. Linear Algebra Appl. 2022).  This file turns the (k+1) x k Hessenberg matrix of the
// run into the roots, in a modified Leja order with conjugate pairs kept together.
#include <cmath>
#include <cstdint>
#include <complex>
#include <vector>

#include "poly.hpp"

namespace bemb200 {
namespace {

using cd = std::complex<double>;

// eigenvalues of an upper Hessenberg matrix (row-major n x n) by the complex shifted QR
// iteration: Givens sweeps on the active unreduced block, Wilkinson shifts, deflation at
// negligible subdiagonal entries, an exceptional shift after every 10 sweeps without one
int hessenberg_eigenvalues(int n, std::vector<cd> A, std::vector<cd>& ev) {
  ev.assign(n, cd(0, 0));
  auto a = [&](int i, int j) -> cd& { return A[(size_t)i * n + j]; };
  double norm = 0.0;
  for (const cd& z : A) norm = std::max(norm, std::abs(z));
  if (!(norm < INFINITY)) return -1;
  const double eps = 2.220446049250313e-16;
  std::vector<cd> cs(n), sn(n);
  int hi = n - 1, sweeps = 0, total = 0;
  while (hi >= 0) {
    if (hi == 0) {
      ev[0] = a(0, 0);
      break;
    }
    int lo = hi;
    while (lo > 0) {
      double s = std::abs(a(lo - 1, lo - 1)) + std::abs(a(lo, lo));
      if (s == 0.0) s = norm;
      if (std::abs(a(lo, lo - 1)) <= eps * s) {
        a(lo, lo - 1) = 0.0;
        break;
      }
      --lo;
    }
    if (lo == hi) {
      ev[hi] = a(hi, hi);
      --hi;
      sweeps = 0;
      continue;
    }
    if (++total > 60 * n) return -1;
    ++sweeps;
    const cd p = a(hi - 1, hi - 1), q = a(hi - 1, hi), r = a(hi, hi - 1), t = a(hi, hi);
    cd mu;
    if (sweeps % 11 == 10) {
      mu = t + cd(std::abs(r), 0.0);
    } else {
      const cd half = 0.5 * (p + t), disc = std::sqrt(0.25 * (p - t) * (p - t) + q * r);
      const cd m1 = half + disc, m2 = half - disc;
      mu = std::abs(m1 - t) < std::abs(m2 - t) ? m1 : m2;
    }
    for (int i = lo; i <= hi; ++i) a(i, i) -= mu;
    for (int k = lo; k < hi; ++k) {  // H - mu I = Q R: rotation k zeroes a(k+1, k)
      const cd x = a(k, k), y = a(k + 1, k);
      const double nr = std::hypot(std::abs(x), std::abs(y));
      const cd c = nr == 0.0 ? cd(1, 0) : x / nr, s = nr == 0.0 ? cd(0, 0) : y / nr;
      cs[k] = c;
      sn[k] = s;
      for (int j = k; j <= hi; ++j) {
        const cd u = a(k, j), v = a(k + 1, j);
        a(k, j) = std::conj(c) * u + std::conj(s) * v;
        a(k + 1, j) = -s * u + c * v;
      }
    }
    for (int k = lo; k < hi; ++k) {  // R Q
      const cd c = cs[k], s = sn[k];
      const int ie = std::min(k + 2, hi);
      for (int i = lo; i <= ie; ++i) {
        const cd u = a(i, k), v = a(i, k + 1);
        a(i, k) = u * c + v * s;
        a(i, k + 1) = -u * std::conj(s) + v * std::conj(c);
      }
    }
    for (int i = lo; i <= hi; ++i) a(i, i) += mu;
  }
  for (const cd& z : ev)
    if (!std::isfinite(z.real()) || !std::isfinite(z.imag())) return -1;
  return 0;
}

// Harmonic Ritz values of a k-step Arnoldi run: eigenvalues of H_k + h^2 f e_k^T with
// H_k^T f = e_k (h = H[k][k-1]); H row-major (k+1) x k with leading dimension ldh.
int harmonic_ritz(int k, const double* H, int ldh, std::vector<cd>& out) {
  out.clear();
  if (k <= 0 || k > 32 || !H || ldh < k) return -1;
  std::vector<double> M((size_t)k * (k + 1));  // [H_k^T | e_k], row-major k x (k+1)
  for (int i = 0; i < k; ++i) {
    for (int j = 0; j < k; ++j) M[(size_t)i * (k + 1) + j] = H[(size_t)j * ldh + i];
    M[(size_t)i * (k + 1) + k] = (i == k - 1) ? 1.0 : 0.0;
  }
  for (int c = 0; c < k; ++c) {  // Gaussian elimination, partial pivoting
    int piv = c;
    for (int r = c + 1; r < k; ++r)
      if (std::abs(M[(size_t)r * (k + 1) + c]) > std::abs(M[(size_t)piv * (k + 1) + c])) piv = r;
    if (M[(size_t)piv * (k + 1) + c] == 0.0) return -1;
    if (piv != c)
      for (int j = 0; j <= k; ++j) std::swap(M[(size_t)c * (k + 1) + j], M[(size_t)piv * (k + 1) + j]);
    for (int r = c + 1; r < k; ++r) {
      const double f = M[(size_t)r * (k + 1) + c] / M[(size_t)c * (k + 1) + c];
      for (int j = c; j <= k; ++j) M[(size_t)r * (k + 1) + j] -= f * M[(size_t)c * (k + 1) + j];
    }
  }
  std::vector<double> f(k);
  for (int r = k - 1; r >= 0; --r) {
    double s = M[(size_t)r * (k + 1) + k];
    for (int j = r + 1; j < k; ++j) s -= M[(size_t)r * (k + 1) + j] * f[j];
    f[r] = s / M[(size_t)r * (k + 1) + r];
  }
  const double h = H[(size_t)k * ldh + (k - 1)];
  std::vector<cd> T((size_t)k * k);
  for (int i = 0; i < k; ++i)
    for (int j = 0; j < k; ++j) T[(size_t)i * k + j] = H[(size_t)i * ldh + j] + (j == k - 1 ? h * h * f[i] : 0.0);
  return hessenberg_eigenvalues(k, T, out);
}

// Real roots and conjugate pairs (a + bi, b > 0 standing for both) of the k values, in the
// modified Leja order: the largest modulus first, then each next maximising the product of
// its distances to the roots already taken (sums of logarithms; a pair counts both members).
// Fails on a non-finite root or one that is tiny next to the largest.
int poly_roots_from_values(const std::vector<cd>& ev, PolyRoots& R) {
  R.n = 0;
  if (ev.empty() || ev.size() > 32) return -1;
  double big = 0.0;
  for (const cd& z : ev) big = std::max(big, std::abs(z));
  if (!(big > 0.0) || !std::isfinite(big)) return -1;
  std::vector<cd> units;  // real roots and the b > 0 member of each pair
  for (const cd& z : ev) {
    if (std::abs(z) < 1e-10 * big) return -1;
    const double tol = 1e-9 * std::abs(z);
    if (std::abs(z.imag()) <= tol)
      units.push_back(cd(z.real(), 0.0));
    else if (z.imag() > 0.0)
      units.push_back(z);
  }
  std::vector<cd> taken;
  std::vector<bool> used(units.size(), false);
  for (size_t step = 0; step < units.size(); ++step) {
    int best = -1;
    double best_score = -INFINITY;
    for (size_t u = 0; u < units.size(); ++u) {
      if (used[u]) continue;
      double score;
      if (taken.empty()) {
        score = std::abs(units[u]);
      } else {
        score = 0.0;
        for (const cd& t : taken) score += std::log(std::max(std::abs(units[u] - t), 1e-300));
      }
      if (score > best_score) {
        best_score = score;
        best = (int)u;
      }
    }
    used[best] = true;
    const cd z = units[best];
    taken.push_back(z);
    if (z.imag() != 0.0) taken.push_back(std::conj(z));
    R.re[R.n] = z.real();
    R.im[R.n] = z.imag();
    ++R.n;
  }
  return R.n > 0 ? 0 : -1;
}

}  // namespace

int harmonic_ritz_values(int k, const double* H, int ldh, std::vector<cd>& out) { return harmonic_ritz(k, H, ldh, out); }

int poly_roots_from_hessenberg(int k, const double* H, int ldh, PolyRoots& R) {
  std::vector<cd> ev;
  if (harmonic_ritz(k, H, ldh, ev) != 0) {
    R.n = 0;
    return -1;
  }
  return poly_roots_from_values(ev, R);
}

}  // namespace bemb200

extern "C" {

// Harmonic Ritz values of a (k+1) x k Arnoldi Hessenberg matrix (row-major, leading dimension
// ldh, k <= 32) into re[0..k-1], im[0..k-1]; returns 0, or -1 when H_k is singular or the QR
// iteration fails.
int bem_harmonic_ritz_values(int32_t k, const double* H, int32_t ldh, double* re, double* im) {
  if (!re || !im) return -1;
  std::vector<bemb200::cd> ev;
  if (bemb200::harmonic_ritz_values(k, H, ldh, ev) != 0) return -1;
  for (int i = 0; i < k; ++i) {
    re[i] = ev[i].real();
    im[i] = ev[i].imag();
  }
  return 0;
}

}  // extern "C"
