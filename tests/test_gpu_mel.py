"""MEL stage update on the GPU (bem_gpu_mel_*) against the oracle's restatement
(oracle/mel_oracle.cpp): point phi and velocity on a noisy tank with arbitrary per-DOF phi /
phin, and four RK4 stages chained through moving positions, within 1e-12 relative (the fit's
3 x 3 solve differs: adjugate on the GPU, pivoted elimination in the oracle).  The linear
potential's velocity is exact on the GPU too.  Then one RK4 step of the BEM-MEL loop: BVP
solve, stage update, at the stage positions.  Pinned to the compiled reference's gradPhi and
DphiDt on the golden cases."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import oracle as O  # noqa: E402
import goldens  # noqa: E402

from bem_for_nonlinear_waves_b200 import BEM_BVP, MELStage, build_dofs, known_values, make_tank, point_normals  # noqa: E402
from test_mel_oracle import A, linear_field_surface  # noqa: E402

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _noisy():
    t = make_tank(1.0, 0.5, 0.4, 0.05, amplitude=0.02, wavelength=0.7, noise_sigma=0.004, seed=3)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    rng = np.random.default_rng(9)
    n = d["dof_point"].shape[0]
    return t, d, rng.standard_normal(n), rng.standard_normal(n)


def test_mel_velocity_matches_oracle(product_lib):
    t, d, phi, phin = _noisy()
    m = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d)
    pp, u = m.velocity(t.X, phi, phin)
    pp0, u0 = O.mel_velocity(t.X, t.tri, t.face_dirichlet, d["point_flags"], d["face_dof"], phi, phin)
    assert rel(pp, pp0) < 1e-13
    assert rel(u, u0) < 1e-12


def test_mel_linear_potential_exact(product_lib):
    t, d, phi, phin = linear_field_surface()
    m = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d)
    _, u = m.velocity(t.X, phi, phin)
    assert np.abs(u - A).max() < 1e-12


def test_mel_rk4_stages_match_oracle(product_lib):
    t, d, phi, phin = _noisy()
    m = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d)
    o = O.MelOracle(t.X.shape[0])
    rng = np.random.default_rng(2)
    X, Xo_ = t.X.copy(), t.X.copy()
    for k in range(4):
        ph = phi + 0.1 * k * rng.standard_normal(phi.shape)
        pn = phin + 0.1 * k * rng.standard_normal(phin.shape)
        Xg, pg, ug, dg = m.stage(k, 0.02, X, ph, pn)
        Xc, pc, uc, dc = o.stage(k, 0.02, 9.81, Xo_, t.tri, t.face_dirichlet, d["point_flags"], d["face_dof"], ph, pn)
        assert rel(ug, uc) < 1e-12, k
        assert rel(dg, dc) < 1e-12, k
        assert rel(pg, pc) < 1e-12, k
        assert rel(Xg - t.X, Xc - t.X) < 1e-11, k
        X, Xo_ = Xg, Xc  # the next stage at the stage positions of each side


def test_mel_rk4_step_with_bvp(product_lib):
    # the BEM-MEL loop for one RK4 step: solve the BVP at the stage positions with the stage's
    # free-surface phi, update, repeat; the step must stay finite and move the free surface
    t = make_tank(1.0, 0.5, 0.4, 0.05, amplitude=0.02, wavelength=0.7, seed=1)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    kv = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    m = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d)
    X = t.X.copy()
    known = kv.copy()
    dirichlet = d["dof_kind"] == 0
    prev = None
    for k in range(4):
        b = BEM_BVP(X, t.tri, t.face_dirichlet, expansion_order=8, solver_tol=1e-10, tol_relative=True, preconditioner="jacobi",
                    dofs=d)
        b.solve(known, x0=prev)  # warm start from the previous stage, as the reference does
        prev = b.ans.copy()
        assert b.last_gmres_converged
        X, pnext, u, dphi = m.stage(k, 0.01, X, b.phi, b.phin)
        known = known.copy()
        known[dirichlet] = pnext[d["dof_point"][dirichlet]]  # free-surface phi of the next stage; walls keep phin
    assert np.isfinite(X).all() and np.isfinite(pnext).all()
    top = (d["point_flags"] & 2) != 0
    assert np.abs(X[top] - t.X[top]).max() > 0


@pytest.mark.parametrize("name", goldens.names())
def test_mel_matches_reference(product_lib, name):
    """The device MEL update against the compiled reference's gradPhi / DphiDt of its own
    solution (golden fixtures): from the reference's per-DOF solution within 1e-11 of the largest
    value; and end to end, the device's own FP64 solve of the same problem followed by the device
    velocity fit, within 1e-8 (the solve agrees to 1e-10, the surface gradient divides by h)."""
    g = goldens.Golden(name)
    t = g.tank
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    phi, phin = g.surface_values(d)
    rphi, ru, rdp = g.mel()
    m = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d, gravity=t.g)
    pp, u = m.velocity(t.X, phi, phin)
    assert np.abs(pp - rphi).max() <= 1e-12 * np.abs(rphi).max()
    assert np.abs(u - ru).max() <= 1e-11 * np.abs(ru).max()
    _, _, _, dp = m.stage(0, 1e-3, t.X, phi, phin)
    pushed = (d["point_flags"] & 1) == 0
    assert np.abs(dp[pushed] - rdp[pushed]).max() <= 1e-11 * np.abs(rdp).max()
    kv = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, expansion_order=g.p, solver_tol=g.tol, solver_max_iter=1000)
    b.solve(kv)
    pp, u = m.velocity(t.X, b.phi, b.phin)
    assert np.abs(pp - rphi).max() <= 1e-8 * np.abs(rphi).max()
    assert np.abs(u - ru).max() <= 1e-8 * np.abs(ru).max()
