"""Autotuned tensor-core M2L work-item size (pairs per item = the MMA's N; items of more than
80 pairs run the one-table-slot kernel variant).  The item size
decides which CTA computes a pair and how many pairs share one MMA, not the pair's arithmetic,
so with the fixed-order reduction (tc_deterministic) every forced size and the tuned one give the
same solution bit for bit."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, known_values, make_tank, point_normals

pytestmark = pytest.mark.gpu


def test_item_size_does_not_change_the_result(product_lib):
    t = make_tank(1.0, 0.5, 0.4, 0.04, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=51)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    k = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    kw = dict(expansion_order=10, solver_tol=1e-10, tol_relative=True, preconditioner="jacobi", precision="mixed", dofs=d,
              tc_deterministic=True)
    ans = {}
    for pairs in (0, 16, 37, 80, 111, 128):
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, tc_item_pairs=pairs, **kw)
        b.solve(k)
        assert b.last_gmres_converged
        tune = b.tc_tuning()
        if pairs:
            assert tune["pairs_per_item"] == pairs
        else:
            assert tune["pairs_per_item"] in (64, 80, 112, 128)
            assert all(v > 0 for v in tune["candidates_ms"].values())
        ans[pairs] = b.ans.copy()
    for pairs in (16, 37, 80, 111, 128):
        assert np.array_equal(ans[pairs], ans[0]), pairs


def test_item_size_out_of_range_rejected(product_lib):
    t = make_tank(1.0, 0.5, 0.4, 0.1, amplitude=0.02, wavelength=0.7, seed=52)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    k = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    with pytest.raises(RuntimeError):
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=6, precision="mixed", tc_item_pairs=129, dofs=d)
        b.solve(k)


def test_wide_items_at_order_12_rejected(product_lib):
    t = make_tank(1.0, 0.5, 0.4, 0.1, amplitude=0.02, wavelength=0.7, seed=53)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    k = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    with pytest.raises(RuntimeError):
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=12, precision="mixed", tc_item_pairs=96, dofs=d)
        b.solve(k)
