"""Host part of the near-field polynomial preconditioner: the harmonic Ritz values of an
Arnoldi run (eigenvalues of H_k + h^2 H_k^{-T} e_k e_k^T, by the library's own complex
Hessenberg QR iteration) against numpy's eigenvalue solver.  CPU only."""
import ctypes

import numpy as np

from bem_for_nonlinear_waves_b200 import _lib as L


def _arnoldi(A, k, rng):
    n = A.shape[0]
    v = rng.standard_normal(n)
    V = [v / np.linalg.norm(v)]
    H = np.zeros((k + 1, k))
    for j in range(k):
        w = A @ V[j]
        for i in range(j + 1):
            H[i, j] = V[i] @ w
            w = w - H[i, j] * V[i]
        H[j + 1, j] = np.linalg.norm(w)
        V.append(w / H[j + 1, j])
    return H


def test_harmonic_ritz_values_match_numpy(product_lib):
    rng = np.random.default_rng(5)
    worst = 0.0
    for trial in range(120):
        k = int(rng.integers(1, 25))
        n = 120
        A = rng.standard_normal((n, n)) / np.sqrt(n) + np.eye(n) * rng.uniform(0.5, 3.0)
        if trial % 4 == 0:  # symmetric: real values
            A = 0.5 * (A + A.T)
        H = np.ascontiguousarray(_arnoldi(A, k, rng))
        Hk = H[:k, :k]
        ek = np.zeros(k)
        ek[-1] = 1.0
        f = np.linalg.solve(Hk.T, ek)
        ref = np.linalg.eigvals(Hk + H[k, k - 1] ** 2 * np.outer(f, ek))
        re, im = np.zeros(k), np.zeros(k)
        rc = product_lib.bem_harmonic_ritz_values(k, L.ptr(H, L.P_dbl), k, L.ptr(re, L.P_dbl), L.ptr(im, L.P_dbl))
        assert rc == 0
        got = re + 1j * im
        scale = np.abs(ref).max()
        worst = max(worst, max(np.abs(got - r).min() for r in ref) / scale, max(np.abs(ref - g).min() for g in got) / scale)
    assert worst < 1e-11, worst


def test_harmonic_ritz_rejects_singular(product_lib):
    H = np.zeros((3, 2))
    re, im = np.zeros(2), np.zeros(2)
    assert product_lib.bem_harmonic_ritz_values(2, L.ptr(H, L.P_dbl), 2, L.ptr(re, L.P_dbl), L.ptr(im, L.P_dbl)) == -1
    assert product_lib.bem_harmonic_ritz_values(0, L.ptr(H, L.P_dbl), 2, L.ptr(re, L.P_dbl), L.ptr(im, L.P_dbl)) == -1
