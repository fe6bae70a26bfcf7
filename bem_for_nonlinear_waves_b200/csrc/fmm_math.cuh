// Solid-harmonic helpers shared by the FMM kernels.
//
// Basis (no Condon-Shortley phase), m >= 0 stored, negative orders by symmetry:
//   F_n^m(x) = rho^n P_n^m(cos t) e^{i m phi} / (n+m)!      (regular)
//   S_n^m(x) = (n-m)! P_n^m(cos t) e^{i m phi} / rho^{n+1}  (irregular)
//   X_n^{-m} = (-1)^m conj(X_n^m)  for X in {F, S, multipole M, local L}.
// With 1/|x-y| = sum_{n,m} conj(F_n^m(y-c)) S_n^m(x-c) the translations are
//   P2M  M_n^m  += q conj(F_n^m(y-c)),  dipole: q conj(nu.grad F_n^m(y-c))
//   M2M  M'_n^m  = sum conj(F_{n'}^{m'}(c-c')) M_{n-n'}^{m-m'}
//   M2L  L_n^m   = (-1)^n sum S_{n+n'}^{m+m'}(c_L-c_M) M_{n'}^{m'}
//   L2L  L'_k^j  = sum_{n>=k} L_n^m conj(F_{n-k}^{m-j}(c'-c))
//   L2P  phi(x)  = sum L_n^m conj(F_n^m(x-c_L))
// The truncation (all degrees <= p on both sides) is the same as the reference's
// Greengard-Rokhlin tables (lib/include/moments.hpp:189-270), so both produce the same
// far field up to rounding; here no coefficient table is needed.
//   grad: dz F_n^m = F_{n-1}^m, (dx - i dy) F_n^m = F_{n-1}^{m-1}, (dx + i dy) F_n^m = -F_{n-1}^{m+1}
#pragma once
#include <cuda_runtime.h>

namespace bemb200 {

__host__ __device__ constexpr int ncoef(int p) { return (p + 1) * (p + 2) / 2; }
__host__ __device__ __forceinline__ int cidx(int n, int m) { return n * (n + 1) / 2 + m; }

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) { return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// acc += a * b
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}

// X_n^m for any m from the stored m >= 0 half
__device__ __forceinline__ double2 getsym(const double2* A, int n, int m) {
  if (m >= 0) return A[cidx(n, m)];
  const double2 c = A[cidx(n, -m)];
  return ((-m) & 1) ? make_double2(-c.x, c.y) : make_double2(c.x, -c.y);
}

__device__ __forceinline__ double2 shfl_up2(double2 v, int d, int width) {
  return make_double2(__shfl_up_sync(0xffffffffu, v.x, d, width), __shfl_up_sync(0xffffffffu, v.y, d, width));
}
__device__ __forceinline__ double2 shfl_down2(double2 v, int d, int width) {
  return make_double2(__shfl_down_sync(0xffffffffu, v.x, d, width), __shfl_down_sync(0xffffffffu, v.y, d, width));
}
__device__ __forceinline__ double2 shfl_xor2(double2 v, int d, int width = 32) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, d, width), __shfl_xor_sync(0xffffffffu, v.y, d, width));
}

// Lane m (< width) fills column m of F for vector (x,y,z) into Fout[cidx(n,m)], n = m..P.
template <int P>
__device__ __forceinline__ void F_column(int m, double x, double y, double z, double2* Fout) {
  if (m > P) return;
  const double r2 = x * x + y * y + z * z;
  double2 f = make_double2(1.0, 0.0);
  for (int k = 1; k <= m; ++k) f = cscale(cmul(f, make_double2(x, y)), 1.0 / (2.0 * k));
  Fout[cidx(m, m)] = f;
  double2 prev = make_double2(0.0, 0.0), cur = f;
  for (int n = m; n < P; ++n) {
    const double inv = 1.0 / double((n + 1) * (n + 1) - m * m);
    double2 nx = make_double2(((2 * n + 1) * z * cur.x - r2 * prev.x) * inv, ((2 * n + 1) * z * cur.y - r2 * prev.y) * inv);
    Fout[cidx(n + 1, m)] = nx;
    prev = cur;
    cur = nx;
  }
}

// Lane q fills column q of S for vector (x,y,z), degrees q..Q.
template <int Q>
__device__ __forceinline__ void S_column(int q, double x, double y, double z, double2* Sout) {
  if (q > Q) return;
  const double r2 = x * x + y * y + z * z;
  const double inv_r2 = 1.0 / r2;
  double2 s = make_double2(1.0 / sqrt(r2), 0.0);
  for (int k = 1; k <= q; ++k) s = cscale(cmul(s, make_double2(x, y)), (2.0 * k - 1.0) * inv_r2);
  Sout[cidx(q, q)] = s;
  double2 prev = make_double2(0.0, 0.0), cur = s;
  for (int l = q; l < Q; ++l) {
    const double a = (2 * l + 1) * z;
    const double b = double((l + q) * (l - q));
    double2 nx = make_double2((a * cur.x - b * prev.x) * inv_r2, (a * cur.y - b * prev.y) * inv_r2);
    Sout[cidx(l + 1, q)] = nx;
    prev = cur;
    cur = nx;
  }
}

// full (negative-order) table fill from one lane per column
template <int Q>
__device__ __forceinline__ void F_full_column(int m, double x, double y, double z, double2* T /*(Q+1)^2*/) {
  if (m > Q) return;
  const double r2 = x * x + y * y + z * z;
  double2 f = make_double2(1.0, 0.0);
  for (int k = 1; k <= m; ++k) f = cscale(cmul(f, make_double2(x, y)), 1.0 / (2.0 * k));
  double2 prev = make_double2(0.0, 0.0), cur = f;
  for (int n = m; n <= Q; ++n) {
    if (n > m) {
      const double inv = 1.0 / double(n * n - m * m);
      double2 nx = make_double2(((2 * n - 1) * z * cur.x - r2 * prev.x) * inv, ((2 * n - 1) * z * cur.y - r2 * prev.y) * inv);
      prev = cur;
      cur = nx;
    }
    T[n * (n + 1) + m] = cur;
    if (m > 0) T[n * (n + 1) - m] = (m & 1) ? make_double2(-cur.x, cur.y) : make_double2(cur.x, -cur.y);
  }
}

template <int Q>
__device__ __forceinline__ void S_full_column(int q, double x, double y, double z, double2* T /*(Q+1)^2*/) {
  if (q > Q) return;
  const double r2 = x * x + y * y + z * z;
  const double inv_r2 = 1.0 / r2;
  double2 s = make_double2(1.0 / sqrt(r2), 0.0);
  for (int k = 1; k <= q; ++k) s = cscale(cmul(s, make_double2(x, y)), (2.0 * k - 1.0) * inv_r2);
  double2 prev = make_double2(0.0, 0.0), cur = s;
  for (int l = q; l <= Q; ++l) {
    if (l > q) {
      const double a = (2 * l - 1) * z;
      const double b = double((l - 1 + q) * (l - 1 - q));
      double2 nx = make_double2((a * cur.x - b * prev.x) * inv_r2, (a * cur.y - b * prev.y) * inv_r2);
      prev = cur;
      cur = nx;
    }
    T[l * (l + 1) + q] = cur;
    if (q > 0) T[l * (l + 1) - q] = (q & 1) ? make_double2(-cur.x, cur.y) : make_double2(cur.x, -cur.y);
  }
}

}  // namespace bemb200
