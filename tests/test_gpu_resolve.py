"""Several right-hand sides on one set-up (the phi_t BVP of a floating-body step, or the next
Runge-Kutta stage with unchanged geometry, reuses the operator: BEM_solveBVP.hpp:922-1040).
A second solve on a set-up context must equal a fresh set-up + solve bit for bit (the set-up
is deterministic -- for mixed precision with the fixed-order M2L reduction -- and nothing of
the first solve leaks into the second), and the solution is
linear in the known boundary values (to the solve tolerance)."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, known_values, make_tank, point_normals

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_resolve_on_one_setup(product_lib, precision):
    t = make_tank(1.0, 0.5, 0.4, 0.05, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=11)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    k1 = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    rng = np.random.default_rng(4)
    k2 = -0.7 * k1 + 0.01 * rng.standard_normal(k1.shape)
    kw = dict(expansion_order=8, solver_tol=1e-11, tol_relative=True, solver_max_iter=1500, preconditioner="jacobi",
              precision=precision, dofs=d, tc_deterministic=True)
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, **kw)
    b.solve(k1)
    a1 = b.ans.copy()
    b.solve(k2)
    a2 = b.ans.copy()
    assert b.last_gmres_converged
    fresh = BEM_BVP(t.X, t.tri, t.face_dirichlet, **kw)
    fresh.solve(k2)
    assert np.array_equal(a2, fresh.ans)
    b.solve(k1 + k2)
    a12 = b.ans
    rel = np.abs(a12 - (a1 + a2)).max() / np.abs(a12).max()
    assert rel < 1e-8, rel


def test_warm_start_from_solution(product_lib):
    t = make_tank(1.0, 0.5, 0.4, 0.05, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=12)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    k1 = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=8, solver_tol=1e-10, tol_relative=True, preconditioner="jacobi", dofs=d)
    b.solve(k1)
    cold_iters, a1 = b.last_gmres_total_iter, b.ans.copy()
    b.solve(k1, x0=a1)  # the solution itself: already converged
    assert b.last_gmres_converged and b.last_gmres_total_iter <= 1
    assert np.abs(b.ans - a1).max() <= 1e-9 * np.abs(a1).max()
    b.solve(1.01 * k1, x0=a1)  # a nearby right-hand side starts close
    assert b.last_gmres_converged and b.last_gmres_total_iter < cold_iters
