"""ctypes wrapper of the oracle (test infrastructure only).

The oracle is a CPU restatement of the reference's GMRES-FMM Laplace BVP path
(see bem_oracle.cpp).  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module, as the checker.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        P = ctypes.c_void_p
        i32 = ctypes.c_int
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        llp = ctypes.POINTER(ctypes.c_longlong)
        L.oracle_build_dofs.restype = i32
        L.oracle_build_dofs.argtypes = [i32, dp, i32, ip, u8p, ip, ip, ip, ip, u8p]
        L.oracle_mel_velocity.restype = i32
        L.oracle_mel_velocity.argtypes = [i32, dp, i32, ip, u8p, u8p, ip, dp, dp, dp, dp]
        L.oracle_mel_stage.restype = i32
        L.oracle_mel_stage.argtypes = [i32, dp, i32, ip, u8p, u8p, ip, dp, dp, i32, ctypes.c_double, ctypes.c_double, dp, dp, dp,
                                       dp, dp, dp, dp]
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [i32, dp, i32, ip, u8p, i32, ip, ip, ip, ip, i32, ctypes.c_double, i32, i32]
        L.oracle_destroy.argtypes = [P]
        L.oracle_create_sampled.restype = P
        L.oracle_create_sampled.argtypes = [i32, dp, i32, ip, u8p, i32, ip, ip, ip, ip, i32, ctypes.c_double, i32, i32, i32]
        L.oracle_time_sample.argtypes = [P, i32, dp]
        L.oracle_time_stage.restype = ctypes.c_double
        L.oracle_time_stage.argtypes = [P, i32]
        L.oracle_setup_times.argtypes = [P, dp]
        L.oracle_compute_diag.argtypes = [P]
        L.oracle_get_diag.argtypes = [P, dp]
        L.oracle_point_integrals.argtypes = [P, dp, dp, dp, dp]
        L.oracle_point_integrals_direct.argtypes = [P, dp, dp, dp, dp]
        L.oracle_apply.argtypes = [P, dp, dp, dp]
        L.oracle_stats.argtypes = [P, llp, dp, llp]
        L.oracle_face_leaf.argtypes = [P, ip, dp]
        L.oracle_near_row.restype = i32
        L.oracle_near_row.argtypes = [P, i32, i32, ip, dp, dp]
        L.oracle_scale_factor.restype = ctypes.c_double
        L.oracle_scale_factor.argtypes = [P]
        L.oracle_solve.restype = i32
        L.oracle_solve.argtypes = [P, dp, dp, ctypes.c_double, i32, dp, dp, dp]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t))


def build_dofs(X, tri, face_dirichlet):
    X = np.ascontiguousarray(X, dtype=np.float64)
    tri = np.ascontiguousarray(tri, dtype=np.int32)
    fd = np.ascontiguousarray(face_dirichlet, dtype=np.uint8)
    np_, nf = X.shape[0], tri.shape[0]
    cap = np_ + 3 * nf
    dp_ = np.zeros(cap, np.int32)
    df = np.zeros(cap, np.int32)
    dk = np.zeros(cap, np.int32)
    fdof = np.zeros(3 * nf, np.int32)
    pflags = np.zeros(np_, np.uint8)
    n = lib().oracle_build_dofs(np_, _p(X, ctypes.c_double), nf, _p(tri, ctypes.c_int), _p(fd, ctypes.c_uint8),
                                _p(dp_, ctypes.c_int), _p(df, ctypes.c_int), _p(dk, ctypes.c_int),
                                _p(fdof, ctypes.c_int), _p(pflags, ctypes.c_uint8))
    return dict(dof_point=dp_[:n].copy(), dof_face=df[:n].copy(), dof_kind=dk[:n].copy(),
                face_dof=fdof.reshape(nf, 3), point_flags=pflags)


def mel_velocity(X, tri, face_dirichlet, point_flags, face_dof, phi, phin):
    """Oracle restatement of the MEL point velocities (mel_oracle.cpp)."""
    L = lib()
    X = np.ascontiguousarray(X, np.float64).reshape(-1)
    tri = np.ascontiguousarray(tri, np.int32).reshape(-1)
    fd = np.ascontiguousarray(face_dirichlet, np.uint8)
    fl = np.ascontiguousarray(point_flags, np.uint8)
    fdof = np.ascontiguousarray(face_dof, np.int32).reshape(-1)
    phi = np.ascontiguousarray(phi, np.float64)
    phin = np.ascontiguousarray(phin, np.float64)
    n = X.shape[0] // 3
    pp, u = np.zeros(n), np.zeros(3 * n)
    L.oracle_mel_velocity(n, _p(X, ctypes.c_double), tri.shape[0] // 3, _p(tri, ctypes.c_int), _p(fd, ctypes.c_uint8),
                          _p(fl, ctypes.c_uint8), _p(fdof, ctypes.c_int), _p(phi, ctypes.c_double), _p(phin, ctypes.c_double),
                          _p(pp, ctypes.c_double), _p(u, ctypes.c_double))
    return pp, u.reshape(-1, 3)


class MelOracle:
    """RK4 MEL stages on the CPU (mel_oracle.cpp), holding the step's RK state."""

    def __init__(self, n_points):
        self.n = n_points
        self.X0 = np.zeros(3 * n_points)
        self.phi0 = np.zeros(n_points)
        self.dX = np.zeros(4 * n_points * 4)

    def stage(self, k, dt, gravity, X, tri, face_dirichlet, point_flags, face_dof, phi, phin):
        L = lib()
        X = np.ascontiguousarray(X, np.float64).reshape(-1)
        tri = np.ascontiguousarray(tri, np.int32).reshape(-1)
        fd = np.ascontiguousarray(face_dirichlet, np.uint8)
        fl = np.ascontiguousarray(point_flags, np.uint8)
        fdof = np.ascontiguousarray(face_dof, np.int32).reshape(-1)
        phi = np.ascontiguousarray(phi, np.float64)
        phin = np.ascontiguousarray(phin, np.float64)
        n = self.n
        Xo, po, u, dp = np.zeros(3 * n), np.zeros(n), np.zeros(3 * n), np.zeros(n)
        L.oracle_mel_stage(n, _p(X, ctypes.c_double), tri.shape[0] // 3, _p(tri, ctypes.c_int), _p(fd, ctypes.c_uint8),
                           _p(fl, ctypes.c_uint8), _p(fdof, ctypes.c_int), _p(phi, ctypes.c_double), _p(phin, ctypes.c_double),
                           int(k), float(dt), float(gravity), _p(self.X0, ctypes.c_double), _p(self.phi0, ctypes.c_double),
                           _p(self.dX, ctypes.c_double), _p(Xo, ctypes.c_double), _p(po, ctypes.c_double), _p(u, ctypes.c_double),
                           _p(dp, ctypes.c_double))
        return Xo.reshape(-1, 3), po, u.reshape(-1, 3), dp


class Oracle:
    def __init__(self, X, tri, face_dirichlet, dofs, p=8, theta=0.25, max_points=30, max_level=7, near_stride=1):
        self.X = np.ascontiguousarray(X, dtype=np.float64)
        self.tri = np.ascontiguousarray(tri, dtype=np.int32)
        self.fd = np.ascontiguousarray(face_dirichlet, dtype=np.uint8)
        self.dof_point = np.ascontiguousarray(dofs["dof_point"], np.int32)
        self.dof_face = np.ascontiguousarray(dofs["dof_face"], np.int32)
        self.dof_kind = np.ascontiguousarray(dofs["dof_kind"], np.int32)
        self.face_dof = np.ascontiguousarray(dofs["face_dof"], np.int32).reshape(-1)
        self.ndof = int(self.dof_point.shape[0])
        self.np = int(self.X.shape[0])
        self.nf = int(self.tri.shape[0])
        self.p = p
        self.h = lib().oracle_create_sampled(self.np, _p(self.X, ctypes.c_double), self.nf, _p(self.tri, ctypes.c_int),
                                             _p(self.fd, ctypes.c_uint8), self.ndof, _p(self.dof_point, ctypes.c_int),
                                             _p(self.dof_face, ctypes.c_int), _p(self.dof_kind, ctypes.c_int),
                                             _p(self.face_dof, ctypes.c_int), p, theta, max_points, max_level, int(near_stride))
        self._diag = False

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().oracle_destroy(h)
            self.h = None

    @property
    def L(self):
        return lib().oracle_scale_factor(self.h)

    def compute_diag(self):
        lib().oracle_compute_diag(self.h)
        self._diag = True
        out = np.zeros(self.ndof)
        lib().oracle_get_diag(self.h, _p(out, ctypes.c_double))
        return out

    def point_integrals(self, phi, phin, direct=False):
        phi = np.ascontiguousarray(phi, np.float64)
        phin = np.ascontiguousarray(phin, np.float64)
        a = np.zeros(self.np)
        b = np.zeros(self.np)
        fn = lib().oracle_point_integrals_direct if direct else lib().oracle_point_integrals
        fn(self.h, _p(phi, ctypes.c_double), _p(phin, ctypes.c_double), _p(a, ctypes.c_double), _p(b, ctypes.c_double))
        return a, b

    def apply(self, phi, phin):
        if not self._diag:
            self.compute_diag()
        phi = np.ascontiguousarray(phi, np.float64)
        phin = np.ascontiguousarray(phin, np.float64)
        out = np.zeros(self.ndof)
        lib().oracle_apply(self.h, _p(phi, ctypes.c_double), _p(phin, ctypes.c_double), _p(out, ctypes.c_double))
        return out

    def time_sample(self, m2l_stride=1):
        """Seconds: p2m, m2m, m2l, l2l, near sums, l2p (one mat-vec), tree+lists, near
        quadrature; threads."""
        t = np.zeros(9)
        lib().oracle_time_sample(self.h, int(m2l_stride), _p(t, ctypes.c_double))
        keys = ["p2m", "m2m", "m2l", "l2l", "near", "l2p", "tree_lists", "near_setup", "threads"]
        return dict(zip(keys, t.tolist()))

    STAGES = ("p2m", "m2m", "m2l", "l2l", "near", "l2p")

    def time_stage(self, stage):
        """Wall seconds of one whole mat-vec stage (a name of STAGES) over the whole problem."""
        return lib().oracle_time_stage(self.h, self.STAGES.index(stage))

    def setup_times(self):
        """Measured set-up seconds: tree + lists, near-field quadrature; OpenMP threads."""
        out = np.zeros(3)
        lib().oracle_setup_times(self.h, _p(out, ctypes.c_double))
        return dict(tree_lists=float(out[0]), near_setup=float(out[1]), threads=int(out[2]))

    def stats(self, max_level=7):
        out = np.zeros(8, np.int64)
        d = np.zeros(2)
        per = np.zeros(3 * (max_level + 1), np.int64)
        lib().oracle_stats(self.h, _p(out, ctypes.c_longlong), _p(d, ctypes.c_double), _p(per, ctypes.c_longlong))
        return dict(nodes=int(out[0]), leaves=int(out[1]), depth=int(out[2]), n_added=int(out[3]),
                    m2l_pairs=int(out[4]), near_pairs=int(out[5]), nnz=int(out[6]), L=d[0], scale=d[1],
                    per_level=per.reshape(-1, 3))

    def face_leaf(self):
        lv = np.zeros(self.nf, np.int32)
        corner = np.zeros(3 * self.nf)
        lib().oracle_face_leaf(self.h, _p(lv, ctypes.c_int), _p(corner, ctypes.c_double))
        return lv, corner.reshape(-1, 3)

    def near_row(self, t):
        cap = 1 << 16
        idx = np.zeros(cap, np.int32)
        wg = np.zeros(cap)
        wgn = np.zeros(cap)
        n = lib().oracle_near_row(self.h, int(t), cap, _p(idx, ctypes.c_int), _p(wg, ctypes.c_double), _p(wgn, ctypes.c_double))
        n = min(n, cap)
        return idx[:n].copy(), wg[:n].copy(), wgn[:n].copy()

    def solve(self, known, tol=1e-10, max_iter=500, x0=None):
        known = np.ascontiguousarray(known, np.float64)
        phi = np.zeros(self.ndof)
        phin = np.zeros(self.ndof)
        st = np.zeros(4)
        x0p = None if x0 is None else _p(np.ascontiguousarray(x0, np.float64), ctypes.c_double)
        lib().oracle_solve(self.h, _p(known, ctypes.c_double), x0p, tol, max_iter, _p(phi, ctypes.c_double),
                           _p(phin, ctypes.c_double), _p(st, ctypes.c_double))
        return phi, phin, dict(iters=int(st[0]), r_true=st[1], r_est=st[2], converged=bool(st[3]))
