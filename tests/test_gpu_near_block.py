"""The near-block preconditioner (opts.preconditioner = 3): block Jacobi whose cores are the
DOFs of each near block's targets, the counterpart of the reference's additive Schwarz on the
near-field matrix (bem/BEM_solveBVP_GMRES_FMM.hpp:899-1013) with bucket cores and no overlap.
Right preconditioning keeps the true residual as the GMRES residual, so the solution is the
same as with the Jacobi scaling: checked against it (1e-9 of the largest value, both at
relative residual 1e-12) and against the compiled reference's golden solution (3e-10: the
reference's iterate carries its own stopping error; measured 1.9e-10), with
fewer iterations than Jacobi; and in the mixed-precision solve (1e-8 of the FP64 solution)."""
import numpy as np
import pytest

import goldens
from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, known_values, make_tank, point_normals

pytestmark = pytest.mark.gpu


def _tank():
    fb = (0.5, 0.25, 0.2, 0.2, 0.1, (0.05, 0.0, 0.02), (0.0, 0.1, 0.0))
    t = make_tank(1.0, 0.5, 0.4, 0.03, amplitude=0.02, wavelength=0.7, noise_sigma=0.006, seed=4, floating_box=fb)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    kv = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    return t, d, kv


def _solve(t, d, kv, precond, precision="fp64"):
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, expansion_order=8, solver_tol=1e-12, tol_relative=True,
                preconditioner=precond, precision=precision, solver_max_iter=1000)
    b.solve(kv)
    assert b.last_gmres_converged
    return b.ans.copy(), b.last_gmres_total_iter


def test_near_block_matches_jacobi_with_fewer_iterations(product_lib):
    t, d, kv = _tank()
    xj, itj = _solve(t, d, kv, "jacobi")
    xb, itb = _solve(t, d, kv, "near_block")
    assert np.abs(xb - xj).max() <= 1e-9 * np.abs(xj).max()
    assert itb < itj, (itb, itj)
    xm, _ = _solve(t, d, kv, "near_block", precision="mixed")
    assert np.abs(xm - xj).max() <= 1e-8 * np.abs(xj).max()


def test_near_block_solution_matches_reference(product_lib):
    g = goldens.Golden("tank_h0p05_p8")
    d = build_dofs(g.tank.X, g.tank.tri, g.tank.face_dirichlet)
    kv = known_values(g.tank, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(g.tank))
    # one decade below the reference's stopping tolerance.  The reference's own iterate stops
    # inside its tolerance ball along the unpreconditioned Krylov path, which the Jacobi-scaled
    # solve follows closely (1e-10, tests/test_gpu_parity.py); the block-preconditioned solve
    # reaches the same solution from another direction: measured 1.9e-10 of the largest value
    # (at the reference's tolerance and one decade below alike)
    b = BEM_BVP(g.tank.X, g.tank.tri, g.tank.face_dirichlet, dofs=d, expansion_order=g.p, solver_tol=0.1 * g.tol, solver_max_iter=1000,
                preconditioner="near_block")
    b.solve(kv)
    assert b.last_gmres_converged
    ref = g.solution(d)
    assert np.abs(b.ans - ref).max() <= 3e-10 * np.abs(ref).max()
