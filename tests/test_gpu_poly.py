"""Near-field polynomial preconditioner (preconditioner="near_poly"): D^-1 p(A_near D^-1)
applied on the right, p the GMRES polynomial of a short Arnoldi run on A_near D^-1 (roots =
harmonic Ritz values).  It stands where the reference applies its near-field ILU / Schwarz
preconditioners (bem/BEM_solveBVP_GMRES_FMM.hpp:2124-2170); the solution of the BVP does not
depend on the preconditioner, so it must agree with the Jacobi-preconditioned solve (which the
parity tests pin to the oracle) to the solve tolerance, in fewer iterations."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, known_values, make_tank, point_normals

pytestmark = pytest.mark.gpu


def _problem(seed=21):
    t = make_tank(1.0, 0.5, 0.4, 0.05, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=seed)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    k = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    return t, d, k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_poly_agrees_with_jacobi_in_fewer_iterations(product_lib, precision):
    t, d, k = _problem()
    kw = dict(expansion_order=8, solver_tol=1e-11, tol_relative=True, solver_max_iter=1500, precision=precision, dofs=d)
    bj = BEM_BVP(t.X, t.tri, t.face_dirichlet, preconditioner="jacobi", **kw)
    bj.solve(k)
    bp = BEM_BVP(t.X, t.tri, t.face_dirichlet, preconditioner="near_poly", poly_degree=8, **kw)
    bp.solve(k)
    assert bj.last_gmres_converged and bp.last_gmres_converged
    roots = bp.poly_roots()
    assert 4 <= len(roots) <= 8 and np.all(np.isfinite(roots)) and np.all(roots.imag >= 0)
    # degree: a real root counts once, a conjugate pair twice
    assert sum(1 if r.imag == 0 else 2 for r in roots) <= 8
    rel = np.abs(bp.ans - bj.ans).max() / np.abs(bj.ans).max()
    assert rel < 1e-8, rel
    # on this 2.9k-DOF tank the polynomial cuts the iterations (58 -> 36 mixed); on fine meshes the
    # near-field spectrum of A_near D^-1 widens and it stops paying (Jacobi stays the default)
    assert bp.last_gmres_total_iter < 0.75 * bj.last_gmres_total_iter, (bp.last_gmres_total_iter, bj.last_gmres_total_iter)


@pytest.mark.parametrize("degree", [1, 3, 12])
def test_poly_degrees_converge(product_lib, degree):
    t, d, k = _problem(seed=22)
    kw = dict(expansion_order=6, solver_tol=1e-10, tol_relative=True, solver_max_iter=1500, dofs=d)
    ref = BEM_BVP(t.X, t.tri, t.face_dirichlet, preconditioner="jacobi", **kw)
    ref.solve(k)
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, preconditioner="near_poly", poly_degree=degree, **kw)
    b.solve(k)
    assert b.last_gmres_converged
    rel = np.abs(b.ans - ref.ans).max() / np.abs(ref.ans).max()
    assert rel < 1e-7, rel


def test_poly_resolve_and_warm_start(product_lib):
    t, d, k = _problem(seed=23)
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=8, solver_tol=1e-10, tol_relative=True, preconditioner="near_poly",
                precision="mixed", dofs=d, tc_deterministic=True)
    b.solve(k)
    a1, it1 = b.ans.copy(), b.last_gmres_total_iter
    b.solve(k)  # same set-up, same roots, fixed-order M2L reduction: bit for bit
    assert np.array_equal(b.ans, a1)
    b.solve(1.01 * k, x0=a1)
    assert b.last_gmres_converged and b.last_gmres_total_iter < it1


def test_poly_degree_out_of_range_rejected(product_lib):
    t, d, k = _problem(seed=24)
    with pytest.raises(RuntimeError):
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=6, preconditioner="near_poly", poly_degree=40, dofs=d)
        b.solve(k)
