"""Refresh of a set-up at new coordinates of the same mesh (bem_gpu_setup_refresh), host part:
the octree is regrown in the previous root bucket (the reference keeps its Buckets root across
time steps and rebins, bem/BEM_solveBVP_GMRES_FMM.hpp:3125-3346), and when the tree, lists and
targets come out unchanged the structural arrays are taken over from the previous plan.  The
taken-over plan must equal, array for array, the plan rebuilt in full in the same root.  CPU."""
import ctypes

import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import _lib as L
from bem_for_nonlinear_waves_b200 import build_dofs, make_tank


def _desc(X, t, d, keep):
    return L.Desc(X.shape[0], L.ptr(X, L.P_dbl), t.tri.shape[0], L.ptr(t.tri, L.P_int), L.ptr(t.face_dirichlet, L.P_u8),
                  keep[0].shape[0], L.ptr(keep[0], L.P_int), L.ptr(keep[1], L.P_int), L.ptr(keep[2], L.P_int), L.ptr(keep[3], L.P_int))


@pytest.fixture(scope="module")
def mesh():
    t = make_tank(1.0, 0.5, 0.4, 0.05, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=31)
    t.X = np.ascontiguousarray(t.X, np.float64)
    t.tri = np.ascontiguousarray(t.tri, np.int32)
    t.face_dirichlet = np.ascontiguousarray(t.face_dirichlet, np.uint8)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    keep = [np.ascontiguousarray(d[k], np.int32).reshape(-1) for k in ("dof_point", "dof_face", "dof_kind", "face_dof")]
    surf = np.unique(t.tri[t.face_dirichlet.astype(bool)].reshape(-1))
    return t, d, keep, surf


def _check(product_lib, t, keep, X0, X1, p=8):
    o = L.Opts()
    product_lib.bem_gpu_default_opts(ctypes.byref(o))
    o.expansion_order = p
    X0 = np.ascontiguousarray(X0)
    X1 = np.ascontiguousarray(X1)
    d0, d1 = _desc(X0, t, None, keep), _desc(X1, t, None, keep)
    out = np.zeros(3, np.int64)
    assert product_lib.bem_plan_refresh_inspect(ctypes.byref(o), ctypes.byref(d0), ctypes.byref(d1), L.ptr(out, L.P_i64)) == 0
    return out


def test_refresh_same_coordinates_keeps_everything(product_lib, mesh):
    t, d, keep, surf = mesh
    out = _check(product_lib, t, keep, t.X, t.X.copy())
    assert out.tolist() == [1, 2, 0]


def test_refresh_small_motion_takes_over_structure(product_lib, mesh):
    t, d, keep, surf = mesh
    X1 = t.X.copy()
    rng = np.random.default_rng(2)
    X1[surf, 2] += 1e-7 * rng.standard_normal(surf.size)  # a Runge-Kutta stage of a slow wave
    out = _check(product_lib, t, keep, t.X, X1)
    assert out.tolist() == [1, 2, 0]


@pytest.mark.parametrize("amp", [0.01, 0.05])
def test_refresh_larger_motion_equals_full_rebuild(product_lib, mesh, amp):
    t, d, keep, surf = mesh
    X1 = t.X.copy()
    rng = np.random.default_rng(3)
    X1[surf, 2] += amp * rng.standard_normal(surf.size)
    out = _check(product_lib, t, keep, t.X, X1)
    assert out[0] == 1 and out[2] == 0  # the structure may or may not change; the plans agree either way


def test_refresh_after_translation_takes_a_new_root(product_lib, mesh):
    t, d, keep, surf = mesh
    X1 = t.X.copy()
    X1[:, 0] += 3.0  # every centroid leaves the old root bucket
    out = _check(product_lib, t, keep, t.X, X1)
    assert out[0] == 0 and out[1] == 0 and out[2] == 0


def test_refresh_targets_moved_rebuilds_near_blocks_only(product_lib, mesh):
    """Free-surface points on the tank's mid-plane sit exactly on bucket faces: a tiny x motion
    moves them to the neighbouring leaf (new L2P targets) while the elements stay put."""
    t, d, keep, surf = mesh
    X1 = t.X.copy()
    lo, hi = t.X.min(0), t.X.max(0)
    mid = surf[np.abs(t.X[surf, 0] - 0.5 * (lo[0] + hi[0])) < 1e-12]
    assert mid.size > 0
    X1[mid, 0] -= 1e-9
    out = _check(product_lib, t, keep, t.X, X1)
    assert out.tolist() == [1, 1, 0]
