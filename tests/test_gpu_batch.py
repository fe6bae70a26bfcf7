"""Batch / asynchronous solving (bem_gpu_batch_*): several tanks of different sizes queued on
two or three workers give exactly the solutions of one-at-a-time solves when every device
reduction has a fixed order (FP64, and mixed precision with tc_deterministic: bit-identical),
and the same solutions within the solve's tolerance with the tensor-core M2L's fused L2
reduction (whose FP32 summation order varies); tickets poll NOT_READY before they finish, and a
problem that fails set-up reports its error without stopping the others."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, BatchSolver, build_dofs, known_values, make_tank, point_normals

pytestmark = pytest.mark.gpu


def _problem(h, seed):
    t = make_tank(1.0, 0.5, 0.4, h, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=seed)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    known = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    return t, d, known


@pytest.mark.parametrize("precision,workers", [("fp64", 2), ("mixed", 3)])
def test_batch_matches_sequential(product_lib, precision, workers):
    kw = dict(expansion_order=8, solver_tol=1e-9, tol_relative=True, solver_max_iter=800, preconditioner="jacobi",
              precision=precision, tc_deterministic=True)
    probs = [_problem(h, s) for h, s in [(0.05, 1), (0.04, 2), (0.06, 3), (0.045, 4), (0.05, 5)]]
    ref = []
    for t, d, known in probs:
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, **kw)
        b.solve(known)
        assert b.last_gmres_converged
        ref.append((b.phi.copy(), b.phin.copy(), b.last_gmres_total_iter))
    bs = BatchSolver(workers, **kw)
    tickets = [bs.submit(t.X, t.tri, t.face_dirichlet, known, dofs=d) for t, d, known in probs]
    assert len(set(tickets)) == len(tickets)
    for (phi0, phin0, it0), tk in zip(ref, tickets):
        phi, phin, st = bs.result(tk)
        assert st.converged == 1
        assert st.iterations == it0
        assert np.array_equal(phi, phi0)
        assert np.array_equal(phin, phin0)
    bs.close()


def test_batch_matches_sequential_fused_reduction(product_lib):
    kw = dict(expansion_order=8, solver_tol=1e-10, tol_relative=True, solver_max_iter=800, preconditioner="jacobi",
              precision="mixed")
    probs = [_problem(h, s) for h, s in [(0.05, 1), (0.04, 2), (0.06, 3)]]
    ref = []
    for t, d, known in probs:
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, **kw)
        b.solve(known)
        assert b.last_gmres_converged
        ref.append(b.ans.copy())
    bs = BatchSolver(3, **kw)
    tickets = [bs.submit(t.X, t.tri, t.face_dirichlet, known, dofs=d) for t, d, known in probs]
    for a0, tk, (t, d, known) in zip(ref, tickets, probs):
        phi, phin, st = bs.result(tk)
        assert st.converged == 1
        ans = np.where(d["dof_kind"] == 0, phin, phi)
        assert np.abs(ans - a0).max() <= 1e-7 * np.abs(a0).max()
    bs.close()


def test_batch_poll_and_errors(product_lib):
    t, d, known = _problem(0.05, 7)
    bs = BatchSolver(2, expansion_order=8, solver_tol=1e-8, tol_relative=True, preconditioner="jacobi")
    bad = build_dofs(t.X, t.tri, t.face_dirichlet)
    bad["dof_kind"] = bad["dof_kind"].copy()
    bad["dof_kind"][0] = 9  # not a DOF kind: rejected by set-up on the host
    tk_bad = bs.submit(t.X, t.tri, t.face_dirichlet, known, dofs=bad)
    tk_ok = [bs.submit(t.X, t.tri, t.face_dirichlet, known, dofs=d) for _ in range(3)]
    pending_seen = not bs.done(tk_ok[-1])  # three solves queued behind two workers
    with pytest.raises(RuntimeError, match="invalid argument"):
        bs.result(tk_bad)
    first = None
    for tk in tk_ok:
        phi, phin, st = bs.result(tk)
        assert st.converged == 1
        if first is None:
            first = (phi, phin)
        else:
            assert np.array_equal(phi, first[0]) and np.array_equal(phin, first[1])
    assert pending_seen
    assert bs.lib.bem_gpu_batch_poll(bs.handle, 10**6, 0) == -1  # unknown ticket
    bs.close()
