// Roots of the near-field polynomial preconditioner (host side, poly.cpp).
#pragma once

namespace bemb200 {

// Roots of a GMRES polynomial preconditioner, in the order they are applied: real roots
// (im == 0) and complex-conjugate pairs (one entry a + bi, b > 0, stands for both).
struct PolyRoots {
  int n = 0;  // entries
  double re[32], im[32];
};

// roots of the GMRES polynomial from a k-step Arnoldi run on B ((k+1) x k Hessenberg,
// row-major, leading dimension ldh): harmonic Ritz values in modified Leja order; -1 on failure
int poly_roots_from_hessenberg(int k, const double* H, int ldh, PolyRoots& R);

}  // namespace bemb200
