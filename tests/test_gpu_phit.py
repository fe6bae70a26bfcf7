"""Known values of the phi_t boundary-value problem (setPhiPhin_t, bem/BEM_setBoundaryTypes.hpp:
858-935) from bem_gpu_mel_phit_known, against a numpy restatement of the reference's formulas:
phi_t = -|u|^2/2 - g z on Dirichlet DOFs (aphiat(0), lib/include/Network.hpp:971-976), and on
Neumann DOFs phint_Neumann (bem/BEM_BoundaryValues.hpp:701-779): 0 on faces of no body, on a
rigid body's faces n.a + (Omega x n).(v - u) - (B v).H0 with the face basis B (OrthogonalBasis)
and H0 the first row of HessianOfPhi; point DOFs take the area-weighted mean over the point's
Neumann faces.  Checked: the device against the restatement on a floating-box tank (1e-12 of the
largest value, velocities given and computed), the known answer of a uniform flow with its
velocity given (the Hessian term vanishes), and the phi_t solve on the phi solve's set-up
(converges; linear in the data)."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, MELStage, build_dofs, make_tank
from bem_for_nonlinear_waves_b200.tank import face_normals

pytestmark = pytest.mark.gpu

G = 9.81


def _tank(h=0.05, seed=5):
    fb = (0.5, 0.25, 0.2, 0.2, 0.1, (0.05, 0.0, 0.02), (0.0, 0.1, 0.0))
    t = make_tank(1.0, 0.5, 0.4, h, amplitude=0.02, wavelength=0.7, noise_sigma=0.1 * h, seed=seed, floating_box=fb)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    face_body = np.where(t.body.face_mask, 0, -1).astype(np.int32)
    bodies = np.array([[*t.body.center, 0.05, -0.02, 0.01, 0.3, -0.2, 0.1, 0.4, 0.1, -0.3, 0.7, -0.5, 0.2]])
    return t, d, face_body, bodies


def _unit(v):
    n = np.linalg.norm(v)
    return v / n if n > 0 else v


def _grad_tri(x, v):
    e, f = x[1] - x[0], x[2] - x[0]
    ex = _unit(e)
    ez = _unit(np.cross(e, f))
    ey = _unit(np.cross(ez, ex))
    x1, x2, y2 = np.linalg.norm(e), f @ ex, f @ ey
    return (v[1] - v[0]) / x1 * ex + (v[2] * x1 - v[1] * x2 + v[0] * (x2 - x1)) / (x1 * y2) * ey


def _phint_face(t, p, F, n, u, face_body, bodies):
    b = face_body[F]
    if b < 0:
        return 0.0
    c, U, W, A, Al = (bodies[b, 3 * k:3 * k + 3] for k in range(5))
    r = t.X[p] - c
    v = U + np.cross(W, r)
    a = A + np.cross(Al, r) + np.cross(W, np.cross(W, r))
    s0 = np.array([1.0, 0, 0]) - n[0] * n
    if np.linalg.norm(s0) < 1e-3:
        s0 = np.array([0, 1.0, 0]) - n[1] * n
    s0 = _unit(s0)
    s1 = _unit(np.cross(n, s0))
    B = np.array([n, s0, s1])
    q = t.tri[F]
    xr = t.X[q] @ B.T
    ur = u[q] @ B.T
    g = np.array([_grad_tri(xr, ur[:, i]) for i in range(3)])
    H0 = np.array([-g[1, 1] - g[2, 2], 0.5 * (g[0, 1] + g[1, 0]), 0.5 * (g[0, 2] + g[2, 0])])
    return n @ a + np.cross(W, n) @ (v - u[p]) - (B @ v) @ H0


def _oracle(t, d, u, face_body, bodies):
    fn = face_normals(t)
    cr = np.cross(t.X[t.tri[:, 1]] - t.X[t.tri[:, 0]], t.X[t.tri[:, 2]] - t.X[t.tri[:, 0]])
    area = 0.5 * np.linalg.norm(cr, axis=1)
    faces_of = [[] for _ in range(t.X.shape[0])]
    for f, tr in enumerate(t.tri):
        for p in tr:
            faces_of[p].append(f)
    out = np.zeros(d["dof_point"].shape[0])
    for i, (p, F, k) in enumerate(zip(d["dof_point"], d["dof_face"], d["dof_kind"])):
        if k == 0:
            out[i] = -0.5 * u[p] @ u[p] - G * t.X[p, 2]
        elif F >= 0:
            out[i] = _phint_face(t, p, F, fn[F], u, face_body, bodies)
        else:
            fs = [f for f in faces_of[p] if not t.face_dirichlet[f]]
            w = sum(area[f] for f in fs)
            out[i] = sum(_phint_face(t, p, f, fn[f], u, face_body, bodies) * area[f] for f in fs) / w if w > 0 else 0.0
    return out


def _solve_phi(t, d):
    from bem_for_nonlinear_waves_b200 import known_values, point_normals

    k = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, expansion_order=8, solver_tol=1e-10, tol_relative=True, preconditioner="jacobi")
    b.solve(k)
    return b


def test_phit_known_matches_restatement(product_lib):
    t, d, face_body, bodies = _tank()
    b = _solve_phi(t, d)
    mel = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d, gravity=G)
    _, _, u, _ = mel.stage(0, 1e-3, t.X, b.phi, b.phin)  # the velocities of the solution
    got = mel.phit_known(t.X, b.phi, b.phin, face_body, bodies)
    exp = _oracle(t, d, u, face_body, bodies)
    assert np.isfinite(got).all()
    assert np.abs(got - exp).max() <= 1e-12 * np.abs(exp).max()
    # with the velocities given: a smooth field with a non-zero Hessian
    rng = np.random.default_rng(3)
    H = rng.normal(size=(3, 3))
    H = H + H.T
    H -= np.trace(H) / 3 * np.eye(3)
    ug = t.X @ H + np.array([0.1, -0.2, 0.05])
    got = mel.phit_known(t.X, b.phi, b.phin, face_body, bodies, u=ug)
    exp = _oracle(t, d, ug, face_body, bodies)
    assert np.abs(got - exp).max() <= 1e-12 * np.abs(exp).max()
    on_body = (d["dof_kind"] != 0) & (d["dof_face"] >= 0) & (face_body[np.maximum(d["dof_face"], 0)] >= 0)
    assert on_body.sum() > 0 and np.abs(got[on_body]).max() > 0


def test_phit_known_uniform_flow_and_solve(product_lib):
    t, d, face_body, bodies = _tank(h=0.05, seed=6)
    c = np.array([0.3, -0.1, 0.2])
    fn = face_normals(t)
    from bem_for_nonlinear_waves_b200 import point_normals

    pn = point_normals(t)
    dp, df, dk = d["dof_point"], d["dof_face"], d["dof_kind"]
    phi = t.X[dp] @ c
    nrm = np.where((df >= 0)[:, None], fn[np.maximum(df, 0)], pn[dp])
    phin = nrm @ c
    mel = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d, gravity=G)
    u = np.tile(c, (t.X.shape[0], 1))  # the flow's velocity at every point (a point DOF's single phin cannot carry it on an edge)
    got = mel.phit_known(t.X, phi, phin, face_body, bodies, u=u)
    exp = np.empty_like(got)
    dirichlet = dk == 0
    exp[dirichlet] = -0.5 * c @ c - G * t.X[dp[dirichlet], 2]
    # a uniform flow has no Hessian: phin_t = n.a + (Omega x n).(v - c) on the body, 0 on the walls
    exp[~dirichlet] = _oracle(t, d, u, face_body, bodies)[~dirichlet]
    face_dofs = (dk != 0) & (df >= 0)
    for i in np.nonzero(face_dofs)[0]:
        F = df[i]
        if face_body[F] < 0:
            assert got[i] == 0.0
            continue
        p = dp[i]
        cc, U, W, A, Al = (bodies[0, 3 * k:3 * k + 3] for k in range(5))
        r = t.X[p] - cc
        v = U + np.cross(W, r)
        a = A + np.cross(Al, r) + np.cross(W, np.cross(W, r))
        exp[i] = fn[F] @ a + np.cross(W, fn[F]) @ (v - c)
    assert np.abs(got - exp).max() <= 1e-9 * np.abs(exp).max()
    # the phi_t problem on the phi problem's set-up: converges, and is linear in its data
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, expansion_order=8, solver_tol=1e-11, tol_relative=True, preconditioner="jacobi")
    b.solve(got)
    a1 = b.ans.copy()
    assert b.last_gmres_converged and np.isfinite(a1).all()
    b.solve(2.0 * got)
    assert np.abs(b.ans - 2.0 * a1).max() <= 1e-8 * np.abs(a1).max()
