"""Synthetic tank meshes (CPU): the plain tank and the tank with a floating box piercing the
free surface are closed, consistently oriented surfaces (every edge used once in each
direction), enclose the fluid volume, and give the box's faces the rigid-body Neumann data."""
from collections import Counter

import numpy as np

from bem_for_nonlinear_waves_b200 import build_dofs, known_values, make_tank, point_normals


def _closed_and_oriented(t):
    E = Counter()
    for a, b, c in t.tri:
        for u, v in ((a, b), (b, c), (c, a)):
            E[(int(u), int(v))] += 1
    return all(n == 1 and E.get((v, u), 0) == 1 for (u, v), n in E.items())


def _volume(t):
    X, tri = t.X, t.tri
    n = np.cross(X[tri[:, 1]] - X[tri[:, 0]], X[tri[:, 2]] - X[tri[:, 0]]) * 0.5
    return float(np.einsum("ij,ij->i", X[tri].mean(axis=1), n).sum() / 3.0)


def test_plain_tank_closed():
    t = make_tank(2.0, 1.0, 0.5, 0.1)
    assert _closed_and_oriented(t)
    assert abs(_volume(t) - 1.0) < 1e-12


def test_floating_box_tank():
    U, Om = np.array([0.05, 0.0, -0.02]), np.array([0.0, 0.1, 0.05])
    t = make_tank(2.0, 1.0, 0.5, 0.05, floating_box=(1.0, 0.5, 0.3, 0.3, 0.2, U, Om))
    assert _closed_and_oriented(t)
    assert abs(_volume(t) - (1.0 - 0.3 * 0.3 * 0.2)) < 1e-9
    fb = t.body.face_mask
    assert fb.sum() > 0 and not t.face_dirichlet[fb].any()
    # box faces point into the box: towards its centre
    c = t.X[t.tri[fb]].mean(axis=1)
    n = np.cross(t.X[t.tri[fb, 1]] - t.X[t.tri[fb, 0]], t.X[t.tri[fb, 2]] - t.X[t.tri[fb, 0]])
    assert (np.einsum("ij,ij->i", n, t.body.center - c) > 0).all()
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    kv = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    # a per-face DOF of a box face carries the rigid velocity times the face normal
    k = np.nonzero((d["dof_face"] >= 0) & fb[np.maximum(d["dof_face"], 0)] & (d["dof_kind"] != 0))[0]
    assert k.size > 0
    f = d["dof_face"][k]
    nf = np.cross(t.X[t.tri[f, 1]] - t.X[t.tri[f, 0]], t.X[t.tri[f, 2]] - t.X[t.tri[f, 0]])
    nf /= np.linalg.norm(nf, axis=1)[:, None]
    x = t.X[d["dof_point"][k]]
    v = U[None, :] + np.cross(Om[None, :], x - t.body.center[None, :])
    np.testing.assert_allclose(kv[k], np.einsum("ij,ij->i", v, nf), rtol=0, atol=1e-15)
    # waterline points are CORNER points (free surface + body wall)
    assert (d["dof_kind"] == 2).sum() > 0
