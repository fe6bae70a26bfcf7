"""Synthetic rectangular wave tanks: closed surface meshes of linear triangles
plus the linear Stokes standing-wave potential used for boundary data.

The reference builds its BVP from a `Network` surface mesh whose faces carry
Dirichlet (free surface) or Neumann (walls, bottom) flags
(bem/BEM_setBoundaryTypes.hpp:447-586).  This module produces the same kind of
input as flat arrays: point coordinates, triangle connectivity with outward
normals, and a per-face Dirichlet flag.  Values are seeded and deterministic.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Tank:
    X: np.ndarray               # (n_points, 3) float64, physical coordinates
    tri: np.ndarray             # (n_faces, 3) int32, outward-oriented
    face_dirichlet: np.ndarray  # (n_faces,) uint8: 1 free surface (Dirichlet), 0 wall/bottom
    length: float
    width: float
    depth: float
    amplitude: float
    wavenumber: float
    g: float = 9.81
    body: "Body | None" = None

    @property
    def omega(self) -> float:
        k, h = self.wavenumber, self.depth
        return math.sqrt(self.g * k * math.tanh(k * h))

    def phi(self, X: np.ndarray) -> np.ndarray:
        """Linear Stokes potential (gA/w) cosh(k(z+h))/cosh(kh) sin(kx)."""
        k, h, A = self.wavenumber, self.depth, self.amplitude
        c = self.g * A / self.omega / math.cosh(k * h)
        return c * np.cosh(k * (X[..., 2] + h)) * np.sin(k * X[..., 0])

    def grad_phi(self, X: np.ndarray) -> np.ndarray:
        k, h, A = self.wavenumber, self.depth, self.amplitude
        c = self.g * A / self.omega / math.cosh(k * h)
        gx = c * k * np.cosh(k * (X[..., 2] + h)) * np.cos(k * X[..., 0])
        gz = c * k * np.sinh(k * (X[..., 2] + h)) * np.sin(k * X[..., 0])
        return np.stack([gx, np.zeros_like(gx), gz], axis=-1)

    @property
    def n_points(self) -> int:
        return int(self.X.shape[0])

    @property
    def n_faces(self) -> int:
        return int(self.tri.shape[0])


def make_tank(length: float = 2.0, width: float = 1.0, depth: float = 0.5, h: float = 0.05,
              amplitude: float = 0.01, wavelength: float = 1.0, noise_sigma: float = 0.0,
              seed: int = 0, floating_box=None) -> Tank:
    """Closed box [0,L]x[0,W]x[-D,0] meshed as structured right-triangle grids.

    `noise_sigma` perturbs the z of every free-surface node with seeded Gaussian
    noise (the points stay on the vertical wall planes).

    `floating_box` = (xc, yc, a, b, draft, U, Omega) cuts an a x b hole (snapped to the grid)
    centred at (xc, yc) into the free surface and closes it with the walls and bottom of a box of
    the given draft: a floating body piercing the free surface, its faces Neumann with the rigid
    velocity phin = (U + Omega x (x - c)) . n (bem/BEM_setBoundaryTypes.hpp:753-847), its
    normals pointing into the box (out of the fluid).  The waterline points are shared by the free
    surface and the body walls (CORNER points of the reference's classification)."""
    nx = max(1, int(round(length / h)))
    ny = max(1, int(round(width / h)))
    nz = max(1, int(round(depth / h)))
    xs = np.linspace(0.0, length, nx + 1)
    ys = np.linspace(0.0, width, ny + 1)
    zs = np.linspace(-depth, 0.0, nz + 1)

    pid = -np.ones((nx + 1, ny + 1, nz + 1), dtype=np.int64)
    coords = []

    def point(i, j, k):
        if pid[i, j, k] < 0:
            pid[i, j, k] = len(coords)
            coords.append((xs[i], ys[j], zs[k]))
        return pid[i, j, k]

    tris = []
    fdir = []

    def quad_grid(fixed_axis, fixed_index, outward_sign, dirichlet):
        axes = [a for a in range(3) if a != fixed_axis]
        n = [nx, ny, nz]
        for u in range(n[axes[0]]):
            for v in range(n[axes[1]]):
                def ijk(du, dv):
                    idx = [0, 0, 0]
                    idx[fixed_axis] = fixed_index
                    idx[axes[0]] = u + du
                    idx[axes[1]] = v + dv
                    return point(*idx)
                a, b, c, d = ijk(0, 0), ijk(1, 0), ijk(1, 1), ijk(0, 1)
                for t in ((a, b, c), (a, c, d)):
                    tris.append(t)
                    fdir.append(dirichlet)

    hole = None
    if floating_box is not None:
        xc, yc, a, b, draft = (float(v) for v in floating_box[:5])
        i0 = int(round((xc - a / 2) / (length / nx)))
        i1 = i0 + max(1, int(round(a / (length / nx))))
        j0 = int(round((yc - b / 2) / (width / ny)))
        j1 = j0 + max(1, int(round(b / (width / ny))))
        k0 = nz - max(1, int(round(draft / (depth / nz))))
        if not (0 < i0 < i1 < nx and 0 < j0 < j1 < ny and 0 < k0 < nz):
            raise ValueError("floating box does not fit inside the tank on this grid")
        hole = (i0, i1, j0, j1, k0)

    def box_faces(i0, i1, j0, j1, k0, k1):
        """The walls and bottom of the box [i0,i1]x[j0,j1]x[k0,k1] (lattice indices)."""
        def rect(fixed_axis, fixed_index, r0, r1):
            axes = [a for a in range(3) if a != fixed_axis]
            for u in range(r0[0], r1[0]):
                for v in range(r0[1], r1[1]):
                    def ijk(du, dv):
                        idx = [0, 0, 0]
                        idx[fixed_axis] = fixed_index
                        idx[axes[0]] = u + du
                        idx[axes[1]] = v + dv
                        return point(*idx)
                    a_, b_, c_, d_ = ijk(0, 0), ijk(1, 0), ijk(1, 1), ijk(0, 1)
                    for t in ((a_, b_, c_), (a_, c_, d_)):
                        tris.append(t)
                        fdir.append(0)
        rect(0, i0, (j0, k0), (j1, k1))
        rect(0, i1, (j0, k0), (j1, k1))
        rect(1, j0, (i0, k0), (i1, k1))
        rect(1, j1, (i0, k0), (i1, k1))
        rect(2, k0, (i0, j0), (i1, j1))

    if hole is None:
        quad_grid(2, nz, +1, 1)   # free surface z = 0
    else:  # free surface without the box's waterplane
        i0, i1, j0, j1, k0 = hole
        for u in range(nx):
            for v in range(ny):
                if i0 <= u < i1 and j0 <= v < j1:
                    continue
                a_, b_, c_, d_ = point(u, v, nz), point(u + 1, v, nz), point(u + 1, v + 1, nz), point(u, v + 1, nz)
                for t in ((a_, b_, c_), (a_, c_, d_)):
                    tris.append(t)
                    fdir.append(1)
    quad_grid(2, 0, -1, 0)    # bottom
    quad_grid(0, 0, -1, 0)    # x = 0
    quad_grid(0, nx, +1, 0)   # x = L
    quad_grid(1, 0, -1, 0)    # y = 0
    quad_grid(1, ny, +1, 0)   # y = W
    n_tank_faces = len(tris)
    if hole is not None:
        i0, i1, j0, j1, k0 = hole
        box_faces(i0, i1, j0, j1, k0, nz)

    X = np.asarray(coords, dtype=np.float64)
    tri = np.asarray(tris, dtype=np.int32)
    fdir = np.asarray(fdir, dtype=np.uint8)

    # orient every tank triangle outward: normal . (centroid - box centre) > 0 on a box; the
    # floating box's triangles point into the box (out of the fluid)
    centre = np.array([length / 2, width / 2, -depth / 2])
    n = np.cross(X[tri[:, 1]] - X[tri[:, 0]], X[tri[:, 2]] - X[tri[:, 0]])
    cen = X[tri].mean(axis=1)
    flip = np.einsum("ij,ij->i", n, cen - centre) < 0
    body = None
    if hole is not None:
        i0, i1, j0, j1, k0 = hole
        bc = np.array([(xs[i0] + xs[i1]) / 2, (ys[j0] + ys[j1]) / 2, zs[k0] / 2])
        fb = np.arange(tri.shape[0]) >= n_tank_faces
        flip[fb] = np.einsum("ij,ij->i", n[fb], cen[fb] - bc) > 0
        U = np.asarray(floating_box[5] if len(floating_box) > 5 else (0.0, 0.0, 0.0), np.float64)
        Om = np.asarray(floating_box[6] if len(floating_box) > 6 else (0.0, 0.0, 0.0), np.float64)
        body = Body(point_begin=-1, face_begin=n_tank_faces, center=bc, U=U, Omega=Om, face_mask=fb)
    tri[flip] = tri[flip][:, [0, 2, 1]]

    if noise_sigma > 0.0:
        rng = np.random.default_rng(seed)
        top = np.isclose(X[:, 2], 0.0)
        if body is not None:  # the waterline stays on the body walls
            top &= ~np.isin(np.arange(X.shape[0]), tri[body.face_mask].reshape(-1))
        X[top, 2] += rng.normal(0.0, noise_sigma, size=int(top.sum()))

    return Tank(X=X, tri=tri, face_dirichlet=fdir, length=length, width=width, depth=depth,
                amplitude=amplitude, wavenumber=2.0 * math.pi / wavelength, body=body)


@dataclasses.dataclass
class Body:
    """A rigid box in the fluid: its faces are Neumann with phin = (U + Omega x (x - c)) . n."""
    point_begin: int            # first point of the body surface in the tank's point array (-1: shared points)
    face_begin: int             # first face of the body surface
    center: np.ndarray
    U: np.ndarray
    Omega: np.ndarray
    face_mask: "np.ndarray | None" = None  # [n_faces] True on the body's faces (None: faces >= face_begin)


def add_box_body(tank: Tank, center, size, h: float, U=(0.0, 0.0, 0.0), Omega=(0.0, 0.0, 0.0)) -> Tank:
    """Adds a closed box surface (sizes `size`, centred at `center`, fully submerged) to a tank
    as a second boundary of the fluid.  Its triangles face into the box (out of the fluid),
    all Neumann; the tank's `body` carries the rigid velocity for the known values.  The
    floating bodies of the reference's BEM-MEL runs are such closed Neumann surfaces with
    phin = (U + Omega x r) . n (bem/BEM_setBoundaryTypes.hpp:753-847)."""
    c = np.asarray(center, dtype=np.float64)
    sz = np.asarray(size, dtype=np.float64)
    sub = make_tank(sz[0], sz[1], sz[2], h)  # outward box [0,a]x[0,b]x[-c,0]
    Xb = sub.X + (c - np.array([sz[0] / 2, sz[1] / 2, -sz[2] / 2]))
    tri_b = sub.tri[:, [0, 2, 1]] + tank.X.shape[0]  # reversed: normals into the box
    t = dataclasses.replace(tank, X=np.vstack([tank.X, Xb]), tri=np.vstack([tank.tri, tri_b]).astype(np.int32),
                            face_dirichlet=np.concatenate([tank.face_dirichlet, np.zeros(tri_b.shape[0], np.uint8)]))
    t.body = Body(point_begin=tank.X.shape[0], face_begin=tank.tri.shape[0], center=c, U=np.asarray(U, np.float64),
                  Omega=np.asarray(Omega, np.float64))
    return t


# Named workloads (tank sizes, spacing, expansion order).
CONFIGS = {
    # ~2,800 nodes / 5,600 triangles, p=8 (the reference's CPU-runnable case)
    "tank_2800": dict(length=2.0, width=1.0, depth=0.5, h=0.05, p=8, tol=1e-10),
    # ~60,000 nodes / 120,000 triangles, free surface z-noise 0.2h, p=10
    "tank_60k": dict(length=2.0, width=1.0, depth=0.5, h=2.0 / 185, p=10, tol=1e-8, noise=0.2),
}


def known_values(tank: Tank, dof_point: np.ndarray, dof_face: np.ndarray, dof_kind: np.ndarray,
                 point_normal: np.ndarray) -> np.ndarray:
    """Known boundary data per DOF in physical units: phi for Dirichlet DOFs, the
    analytic normal derivative grad(phi).n for Neumann DOFs (face normal for
    per-face DOFs, point normal otherwise)."""
    X = tank.X
    kv = np.zeros(dof_point.shape[0], dtype=np.float64)
    d = dof_kind == 0
    kv[d] = tank.phi(X[dof_point[d]])
    nd = ~d
    g = tank.grad_phi(X[dof_point[nd]])
    fn = face_normals(tank)
    f = dof_face[nd]
    nrm = np.where((f >= 0)[:, None], fn[np.maximum(f, 0)], point_normal[dof_point[nd]])
    kv[nd] = np.einsum("ij,ij->i", g, nrm)
    b = getattr(tank, "body", None)
    if b is not None:  # rigid-body Neumann data on the body surface
        fmask = b.face_mask if b.face_mask is not None else (np.arange(tank.tri.shape[0]) >= b.face_begin)
        # a point's DOF without a face belongs to the body if every face of the point does
        pt_all_body = np.ones(X.shape[0], bool)
        np.logical_and.at(pt_all_body, tank.tri[~fmask].reshape(-1), False)
        on_face = (dof_face >= 0) & fmask[np.maximum(dof_face, 0)]
        on = nd & (on_face | ((dof_face < 0) & pt_all_body[dof_point]))
        xb = X[dof_point[on]]
        vel = b.U[None, :] + np.cross(b.Omega[None, :], xb - b.center[None, :])
        kv[on] = np.einsum("ij,ij->i", vel, nrm[on[nd]])
    return kv


def face_normals(tank: Tank) -> np.ndarray:
    X, t = tank.X, tank.tri
    n = np.cross(X[t[:, 1]] - X[t[:, 0]], X[t[:, 2]] - X[t[:, 0]])
    return n / np.linalg.norm(n, axis=1)[:, None]


def point_normals(tank: Tank) -> np.ndarray:
    """Area-weighted point normals (networkPoint::getNormalAreaAveraged)."""
    X, t = tank.X, tank.tri
    n = np.cross(X[t[:, 1]] - X[t[:, 0]], X[t[:, 2]] - X[t[:, 0]]) * 0.5
    pn = np.zeros_like(X)
    for a in range(3):
        np.add.at(pn, t[:, a], n)
    return pn / np.maximum(np.linalg.norm(pn, axis=1), 1e-300)[:, None]
