"""bem_gpu_setup_refresh on the device: a set-up at new coordinates of the same mesh that keeps
the octree root (the reference's rebin path, bem/BEM_solveBVP_GMRES_FMM.hpp:3125-3346) and,
when the structure is unchanged, the device's structural arrays.  Where the bounding box (hence
the scaling and the root) does not change, the refreshed operator must be the operator of a
fresh set-up bit for bit (mixed precision with its fixed-order M2L reduction, tc_deterministic)."""
import dataclasses

import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, known_values, make_tank, point_normals

pytestmark = pytest.mark.gpu


def _tank(seed):
    t = make_tank(1.0, 0.5, 0.4, 0.05, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=seed)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    return t, d


def _known(t, d, X):
    t2 = dataclasses.replace(t, X=np.asarray(X, np.float64))
    return known_values(t2, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t2))


def _interior_shift(t, eps, seed):
    """Moves free-surface points whose coordinates are strictly inside the bounding box along x
    by eps * h: the bounding box, the scale factor and the root bucket stay the same.  Points on
    the mid-plane x = (min + max) / 2 lie exactly on bucket faces and are left in place."""
    X = np.array(t.X, np.float64)
    surf = np.unique(t.tri[np.asarray(t.face_dirichlet, bool)].reshape(-1))
    lo, hi = X.min(0), X.max(0)
    mid = 0.5 * (lo[0] + hi[0])  # a bucket face on every level (the root is centred on the box)
    inner = surf[(X[surf, 0] > lo[0] + 0.1) & (X[surf, 0] < hi[0] - 0.1) & (np.abs(X[surf, 0] - mid) > 1e-3) &
                 (X[surf, 2] < hi[2] - 1e-3) & (X[surf, 2] > lo[2] + 1e-3)]
    rng = np.random.default_rng(seed)
    X[inner, 0] += eps * 0.05 * rng.uniform(-1, 1, inner.size)
    assert np.array_equal(X.min(0), lo) and np.array_equal(X.max(0), hi)
    return X


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_refresh_same_coordinates_bit_exact(product_lib, precision):
    t, d = _tank(41)
    k = _known(t, d, t.X)
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=8, solver_tol=1e-10, tol_relative=True, preconditioner="jacobi",
                precision=precision, dofs=d, tc_deterministic=True)
    b.solve(k)
    a0 = b.ans.copy()
    assert b.refresh(np.array(t.X)) == 2
    b.solve(k)
    assert np.array_equal(b.ans, a0)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("eps", [1e-6, 0.2])
def test_refresh_equals_fresh_setup_in_the_same_root(product_lib, precision, eps):
    t, d = _tank(42)
    X1 = _interior_shift(t, eps, seed=5)
    k1 = _known(t, d, X1)
    kw = dict(expansion_order=8, solver_tol=1e-10, tol_relative=True, preconditioner="jacobi", precision=precision, dofs=d,
              tc_deterministic=True)
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, **kw)
    b.setup()
    kept = b.refresh(X1)
    if eps < 1e-3:
        assert kept == 2  # a tiny motion leaves the tree, lists and targets as they were
    b.solve(k1)
    fresh = BEM_BVP(X1, t.tri, t.face_dirichlet, **kw)
    fresh.solve(k1)
    assert np.array_equal(b.ans, fresh.ans)


def test_refresh_follows_the_geometry(product_lib):
    """A vertical free-surface motion (new bounding box, old root kept): the refreshed solve
    agrees with a fresh set-up to the FMM truncation level, and differs from the old geometry's
    solution by much more than that."""
    t, d = _tank(43)
    X1 = np.array(t.X, np.float64)
    surf = np.unique(t.tri[np.asarray(t.face_dirichlet, bool)].reshape(-1))
    X1[surf, 2] += 0.004 * np.sin(2 * np.pi * X1[surf, 0])
    k1 = _known(t, d, X1)
    kw = dict(expansion_order=10, solver_tol=1e-11, tol_relative=True, preconditioner="jacobi", dofs=d)
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, **kw)
    b.solve(k1)
    old = b.ans.copy()
    b.refresh(X1)
    b.solve(k1)
    fresh = BEM_BVP(X1, t.tri, t.face_dirichlet, **kw)
    fresh.solve(k1)
    scale = np.abs(fresh.ans).max()
    assert np.abs(b.ans - fresh.ans).max() / scale < 1e-6
    assert np.abs(old - fresh.ans).max() / scale > 1e-4
