"""Known answers for the oracle's MEL stage update (mel_oracle.cpp): a linear potential
phi = a.x has the same velocity a at every point (each face's surface gradient plus phin
times its normal is a, at edges and CORNER points too), and with a fixed surface the four RK4
stages of a constant rate land on x0 + rate dt.  Pinned to the compiled reference: its point
phi, gradPhi velocity and Dphi/Dt on its own solution of each golden case."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle"))
import oracle as O  # noqa: E402

import goldens  # noqa: E402
from bem_for_nonlinear_waves_b200 import build_dofs, make_tank  # noqa: E402

A = np.array([0.3, -0.2, 0.5])


def linear_field_surface():
    t = make_tank(1.0, 0.5, 0.4, 0.1)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    X, tri = t.X, t.tri
    fn = np.cross(X[tri[:, 1]] - X[tri[:, 0]], X[tri[:, 2]] - X[tri[:, 0]])
    fn /= np.linalg.norm(fn, axis=1)[:, None]
    phi = X[d["dof_point"]] @ A
    # phin of every DOF: a.n of its face; a point DOF takes any face around its point (they
    # are coplanar there: points on edges and corners carry per-face DOFs)
    face_of = np.full(d["dof_point"].shape[0], -1)
    for f in range(tri.shape[0]):
        for a in range(3):
            k = d["face_dof"][f, a]
            if face_of[k] < 0:
                face_of[k] = f
    phin = np.einsum("ij,j->i", fn[face_of], A)
    return t, d, phi, phin


def test_oracle_velocity_of_linear_potential():
    t, d, phi, phin = linear_field_surface()
    pp, u = O.mel_velocity(t.X, t.tri, t.face_dirichlet, d["point_flags"], d["face_dof"], phi, phin)
    assert np.abs(u - A).max() < 1e-12
    assert np.abs(pp - t.X @ A).max() < 1e-12
    assert (d["point_flags"] & 4).any()  # CORNER points are covered


def test_oracle_rk4_constant_rate():
    t, d, phi, phin = linear_field_surface()
    m = O.MelOracle(t.X.shape[0])
    dt, g = 0.05, 9.81
    for k in range(4):
        Xo, po, u, dp = m.stage(k, dt, g, t.X, t.tri, t.face_dirichlet, d["point_flags"], d["face_dof"], phi, phin)
    assert np.abs(Xo - (t.X + A * dt)).max() < 1e-13
    nn = (d["point_flags"] & 1) == 0
    rate = 0.5 * A @ A - g * t.X[:, 2]
    assert np.abs(dp[nn] - rate[nn]).max() < 1e-13
    assert np.abs(po[nn] - (t.X[nn] @ A + rate[nn] * dt)).max() < 1e-13
    assert np.array_equal(po[~nn], (t.X @ A)[~nn]) or np.abs(po[~nn] - (t.X @ A)[~nn]).max() < 1e-14


@pytest.mark.parametrize("name", goldens.names())
def test_oracle_mel_matches_reference(name):
    """The oracle's velocity fit and Dphi/Dt against the compiled reference's gradPhi and DphiDt
    (bem/BEM_BoundaryValues.hpp:565, lib/include/Network.hpp:224-235) on its own solution."""
    g = goldens.Golden(name)
    t = g.tank
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    phi, phin = g.surface_values(d)
    rphi, ru, rdp = g.mel()
    pp, u = O.mel_velocity(t.X, t.tri, t.face_dirichlet, d["point_flags"], d["face_dof"], phi, phin)
    assert np.abs(pp - rphi).max() <= 1e-12 * np.abs(rphi).max()
    assert np.abs(u - ru).max() <= 1e-11 * np.abs(ru).max()
    m = O.MelOracle(t.X.shape[0])
    _, _, _, dp = m.stage(0, 1e-3, g.tank.g, t.X, t.tri, t.face_dirichlet, d["point_flags"], d["face_dof"], phi, phin)
    pushed = (d["point_flags"] & 1) == 0  # the stage pushes phi on the points that are not all-Neumann
    assert pushed.any()
    assert np.abs(dp[pushed] - rdp[pushed]).max() <= 1e-11 * np.abs(rdp).max()
    # the all-Neumann points: the reference's formula of the same velocities
    assert np.abs(0.5 * (u * u).sum(1) - g.tank.g * t.X[:, 2] - rdp).max() <= 1e-11 * np.abs(rdp).max()
