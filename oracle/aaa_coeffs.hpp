// Test infrastructure only (oracle): Greengard & Rokhlin (1997) translation
// coefficients in the index convention of the reference's generated tables
// AAA_{M2M,M2L,L2L}_FMM[j][k+N][n][m+N]
// (lib/include/lib_multipole_expansion_constants.hpp:16-45, lib/include/moments.hpp:200-270).
//
// A_n^m = (-1)^n / sqrt((n-m)!(n+m)!)                         (constants.hpp:16-28)
// M2M[j][k][n][m] = i^{|k|-|m|-|k-m|} A_n^m A_{j-n}^{k-m} / A_j^k
// M2L[j][k][n][m] = i^{|k-m|-|k|-|m|} A_n^m A_j^k / ((-1)^n A_{j+n}^{m-k})
// L2L[j][k][n][m] = i^{|m|-|m-k|-|k|} A_{n-j}^{m-k} A_j^k / ((-1)^{n+j} A_n^m)
// Every exponent of i above is even, so each coefficient is a real +-ratio of
// factorial square roots.  Invalid index combinations are 0 (the reference skips
// exact zeros when it builds its sparse operator lists).
//
// The ratios are formed in __float128 (integer factorials up to 2p are exact in
// 113 bits) and rounded once to double, the way the reference's tables were
// generated from float128 literals.
#pragma once
#include <cstdlib>
#include <quadmath.h>

namespace bem_oracle_aaa {

inline __float128 fact_q(int n) {
  __float128 r = 1;
  for (int i = 2; i <= n; ++i) r *= i;
  return r;
}

// sqrt((a)!(b)!) / sqrt((c)!(d)!) * ... helpers: we form the product of
// factorials inside one sqrt to round once.
inline double ratio_sqrt(__float128 num, __float128 den) { return (double)sqrtq(num / den); }

inline int ipow_i_even_sign(int e) {  // i^e for even e
  // e even: i^e = (-1)^(e/2)
  int h = e / 2;
  return (h % 2 == 0) ? 1 : -1;
}

// A_n^m A_{n'}^{m'} / A_{n''}^{m''} = (-1)^{n+n'-n''} sqrt((n''-m'')!(n''+m'')!) / sqrt((n-m)!(n+m)!(n'-m')!(n'+m')!)
inline double m2m(int j, int k, int n, int m) {
  if (!(n >= 0 && n <= j && std::abs(m) <= n && std::abs(k) <= j && std::abs(k - m) <= j - n)) return 0.0;
  int e = std::abs(k) - std::abs(m) - std::abs(k - m);
  int s = ipow_i_even_sign(e);
  // A_n^m A_{j-n}^{k-m} / A_j^k, sign (-1)^{n + (j-n) - j} = +1
  __float128 num = fact_q(j - k) * fact_q(j + k);
  __float128 den = fact_q(n - m) * fact_q(n + m) * fact_q(j - n - (k - m)) * fact_q(j - n + (k - m));
  return s * ratio_sqrt(num, den);
}

inline double m2l(int j, int k, int n, int m) {
  if (!(std::abs(k) <= j && std::abs(m) <= n && std::abs(m - k) <= j + n)) return 0.0;
  int e = std::abs(k - m) - std::abs(k) - std::abs(m);
  int s = ipow_i_even_sign(e);
  // A_n^m A_j^k / ((-1)^n A_{j+n}^{m-k}): signs (-1)^n (-1)^j / ((-1)^n (-1)^{j+n}) = (-1)^{-n} = (-1)^n
  int sign_a = ((n % 2) == 0) ? 1 : -1;
  int l = j + n, q = m - k;
  __float128 num = fact_q(l - q) * fact_q(l + q);
  __float128 den = fact_q(n - m) * fact_q(n + m) * fact_q(j - k) * fact_q(j + k);
  return s * sign_a * ratio_sqrt(num, den);
}

inline double l2l(int j, int k, int n, int m) {
  if (!(n >= j && std::abs(k) <= j && std::abs(m) <= n && std::abs(m - k) <= n - j)) return 0.0;
  int e = std::abs(m) - std::abs(m - k) - std::abs(k);
  int s = ipow_i_even_sign(e);
  // A_{n-j}^{m-k} A_j^k / ((-1)^{n+j} A_n^m): (-1)^{n-j} (-1)^j / ((-1)^{n+j} (-1)^n) = (-1)^{-n-j}... evaluate explicitly
  int pa = (n - j) + j - (n + j) - n;  // exponent of (-1)
  int sign_a = ((std::abs(pa) % 2) == 0) ? 1 : -1;
  __float128 num = fact_q(n - m) * fact_q(n + m);
  __float128 den = fact_q(n - j - (m - k)) * fact_q(n - j + (m - k)) * fact_q(j - k) * fact_q(j + k);
  return s * sign_a * ratio_sqrt(num, den);
}

}  // namespace bem_oracle_aaa
