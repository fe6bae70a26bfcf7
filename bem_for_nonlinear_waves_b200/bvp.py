"""Host-side mirror of the reference's BEM_BVP for the GMRES + FMM path.

`BEM_BVP.solve()` keeps the reference's contract (bem/BEM_solveBVP.hpp:565-630): it
indexes the unknowns (setNodeFaceIndices), runs the GMRES-FMM solve and returns
`(time_setup, time_solve, unknowns)`; the per-DOF solution lands in `ans`, `phi`, `phin`
and the diagnostics in `last_gmres_*` (BEM_solveBVP.hpp:376-410).  Every operator
application runs in the sm_100a kernels of lib/libbem_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib as L

DOF_DIRICHLET, DOF_NEUMANN, DOF_CORNER_NEUMANN = 0, 1, 2


def build_dofs(X, tri, face_dirichlet):
    """DOF keys (point, face or -1), kinds and per-face-vertex DOF (pf2Index) from face flags,
    with the reference's rules (bem/BEM_setBoundaryTypes.hpp:29-254, 434-441)."""
    lib = L.load()
    X = np.ascontiguousarray(X, np.float64)
    tri = np.ascontiguousarray(tri, np.int32)
    fd = np.ascontiguousarray(face_dirichlet, np.uint8)
    npts, nf = X.shape[0], tri.shape[0]
    cap = npts + 3 * nf
    dp = np.zeros(cap, np.int32)
    df = np.zeros(cap, np.int32)
    dk = np.zeros(cap, np.int32)
    fdof = np.zeros(3 * nf, np.int32)
    pfl = np.zeros(npts, np.uint8)
    n = lib.bem_gpu_build_dofs(npts, L.ptr(X, L.P_dbl), nf, L.ptr(tri, L.P_int), L.ptr(fd, L.P_u8), L.ptr(dp, L.P_int),
                               L.ptr(df, L.P_int), L.ptr(dk, L.P_int), L.ptr(fdof, L.P_int), L.ptr(pfl, L.P_u8))
    if n < 0:
        raise ValueError("invalid mesh for DOF indexing: " + L.STATUS.get(n, str(n)))
    return dict(dof_point=dp[:n].copy(), dof_face=df[:n].copy(), dof_kind=dk[:n].copy(), face_dof=fdof.reshape(nf, 3),
                point_flags=pfl)


def _make_opts(lib, expansion_order, mac_theta, fmm_bucket_max_points, fmm_max_level, solver_tol, solver_max_iter, device,
               tol_relative, preconditioner, precision, poly_degree=8, tree_on_device=True, tc_item_pairs=0, overlap_near=True,
               refine_rtol=0.0, tc_deterministic=False):
    o = L.Opts()
    lib.bem_gpu_default_opts(ctypes.byref(o))
    o.expansion_order = int(expansion_order)
    o.mac_theta = float(mac_theta)
    o.leaf_max_elements = int(fmm_bucket_max_points)
    o.max_level = int(fmm_max_level)
    o.tol = float(solver_tol)
    o.max_iter = int(solver_max_iter)
    o.device = int(device)
    o.tol_relative = 1 if tol_relative else 0
    o.preconditioner = {"none": 0, "jacobi": 1, "near_poly": 2, "near_block": 3}[preconditioner]
    o.poly_degree = int(poly_degree)
    o.tree_on_host = 0 if tree_on_device else 1
    o.tc_item_pairs = int(tc_item_pairs)
    o.overlap_near = 1 if overlap_near else 0
    o.precision = {"fp64": 0, "mixed": 1}[precision]
    o.refine_rtol = float(refine_rtol)
    o.tc_deterministic = 1 if tc_deterministic else 0
    return o


class BEM_BVP:
    """GMRES-FMM Laplace BVP on one B200."""

    def __init__(self, X, tri, face_dirichlet, *, expansion_order=10, mac_theta=0.25, fmm_bucket_max_points=30,
                 fmm_max_level=7, solver_tol=1e-9, solver_max_iter=500, device=0, dofs=None, tol_relative=False, preconditioner="none",
                 precision="fp64", poly_degree=8, tree_on_device=True, tc_item_pairs=0, overlap_near=True, refine_rtol=0.0,
                 tc_deterministic=False):
        self.lib = L.load()
        if not self.lib.bem_gpu_is_available():
            raise RuntimeError("no sm_100 CUDA device visible: the GMRES-FMM solver runs only on the GPU")
        self.X = np.ascontiguousarray(X, np.float64)
        self.tri = np.ascontiguousarray(tri, np.int32)
        self.face_dirichlet = np.ascontiguousarray(face_dirichlet, np.uint8)
        o = _make_opts(self.lib, expansion_order, mac_theta, fmm_bucket_max_points, fmm_max_level, solver_tol, solver_max_iter,
                       device, tol_relative, preconditioner, precision, poly_degree, tree_on_device, tc_item_pairs,
                       overlap_near, refine_rtol, tc_deterministic)
        self.opts = o
        self.ctx = self.lib.bem_gpu_create(ctypes.byref(o))
        if not self.ctx:
            raise RuntimeError("bem_gpu_create failed")
        self.dofs = dofs
        self.matrix_size = 0
        self._setup_done = False
        self.ans = None
        self.phi = None
        self.phin = None
        self.last_gmres_total_iter = 0
        self.last_gmres_residual_norm = 0.0
        self.last_gmres_converged = False
        self.stats = None

    def __del__(self):
        ctx = getattr(self, "ctx", None)
        if ctx:
            self.lib.bem_gpu_destroy(ctx)
            self.ctx = None

    def _check(self, rc, what):
        if rc not in (L.BEM_OK,):
            msg = self.lib.bem_gpu_last_error(self.ctx)
            raise RuntimeError(f"{what}: {L.STATUS.get(rc, rc)}: {msg.decode() if msg else ''}")

    # setNodeFaceIndices (bem/BEM_setBoundaryTypes.hpp:134-254)
    def setNodeFaceIndices(self):
        if self.dofs is None:
            self.dofs = build_dofs(self.X, self.tri, self.face_dirichlet)
        self.matrix_size = int(self.dofs["dof_point"].shape[0])
        return self.matrix_size

    def setup(self):
        """Geometry part of solveGMRES (scaling, sources, tree, lists, near weights, diagonal)."""
        self.setNodeFaceIndices()
        d = self.dofs
        self._keep = [np.ascontiguousarray(d[k], np.int32).reshape(-1) for k in ("dof_point", "dof_face", "dof_kind", "face_dof")]
        desc = L.Desc(self.X.shape[0], L.ptr(self.X, L.P_dbl), self.tri.shape[0], L.ptr(self.tri, L.P_int),
                      L.ptr(self.face_dirichlet, L.P_u8), self.matrix_size, L.ptr(self._keep[0], L.P_int),
                      L.ptr(self._keep[1], L.P_int), L.ptr(self._keep[2], L.P_int), L.ptr(self._keep[3], L.P_int))
        self._check(self.lib.bem_gpu_setup(self.ctx, ctypes.byref(desc)), "setup")
        self._setup_done = True

    def refresh(self, X):
        """Set-up at new point coordinates X of the same mesh (a Runge-Kutta stage or the next time
        step), keeping the octree's root bucket as the reference's rebin path does
        (bem/BEM_solveBVP_GMRES_FMM.hpp:3125-3346).  Returns what the device kept: 2 (tree, lists
        and targets unchanged: only the geometry was uploaded), 1 (tree and lists; near-field
        blocks rebuilt) or 0 (full set-up)."""
        X = np.ascontiguousarray(X, np.float64)
        if X.shape != self.X.shape:
            raise ValueError("refresh needs the same points (n_points x 3)")
        if not self._setup_done:
            self.X = X
            self.setup()
            return 0
        self.X = X
        desc = L.Desc(self.X.shape[0], L.ptr(self.X, L.P_dbl), self.tri.shape[0], L.ptr(self.tri, L.P_int),
                      L.ptr(self.face_dirichlet, L.P_u8), self.matrix_size, L.ptr(self._keep[0], L.P_int),
                      L.ptr(self._keep[1], L.P_int), L.ptr(self._keep[2], L.P_int), L.ptr(self._keep[3], L.P_int))
        rc = self.lib.bem_gpu_setup_refresh(self.ctx, ctypes.byref(desc))
        self._check(min(rc, 0), "setup_refresh")
        return int(rc)

    def solve(self, known, x0=None):
        """known: per-DOF phi (Dirichlet DOFs) or phin (Neumann DOFs), physical units; x0: optional
        initial guess of the unknowns (phin for Dirichlet DOFs, phi for the others), e.g. the
        previous solution's `ans`.  Returns (time_setup, time_solve, unknowns) like BEM_BVP::solve()."""
        if not self._setup_done:
            self.setup()
        known = np.ascontiguousarray(known, np.float64)
        if known.shape[0] != self.matrix_size:
            raise ValueError("known values must have one entry per DOF")
        phi = np.zeros(self.matrix_size)
        phin = np.zeros(self.matrix_size)
        st = L.Stats()
        x0p = None if x0 is None else L.ptr(np.ascontiguousarray(x0, np.float64), L.P_dbl)
        rc = self.lib.bem_gpu_solve(self.ctx, L.ptr(known, L.P_dbl), x0p, L.ptr(phi, L.P_dbl), L.ptr(phin, L.P_dbl), ctypes.byref(st))
        if rc not in (L.BEM_OK, L.BEM_ERR_NOT_CONVERGED):
            self._check(rc, "solve")
        self.phi, self.phin = phi, phin
        kind = self.dofs["dof_kind"]
        self.ans = np.where(kind == DOF_DIRICHLET, phin, phi)
        self.stats = st
        self.last_gmres_total_iter = st.iterations
        self.last_gmres_residual_norm = st.residual
        self.last_gmres_converged = bool(st.converged)
        return (st.time_setup_s, st.time_solve_s, float(self.matrix_size))

    # ---- operator access (scaled units) ----
    def apply(self, phi, phin):
        phi = np.ascontiguousarray(phi, np.float64)
        phin = np.ascontiguousarray(phin, np.float64)
        out = np.zeros(self.matrix_size)
        self._check(self.lib.bem_gpu_apply(self.ctx, L.ptr(phi, L.P_dbl), L.ptr(phin, L.P_dbl), L.ptr(out, L.P_dbl)), "apply")
        return out

    def point_integrals(self, phi, phin):
        phi = np.ascontiguousarray(phi, np.float64)
        phin = np.ascontiguousarray(phin, np.float64)
        a = np.zeros(self.X.shape[0])
        b = np.zeros(self.X.shape[0])
        self._check(self.lib.bem_gpu_point_integrals(self.ctx, L.ptr(phi, L.P_dbl), L.ptr(phin, L.P_dbl), L.ptr(a, L.P_dbl),
                                                     L.ptr(b, L.P_dbl)), "point_integrals")
        return a, b

    def tc_tuning(self):
        """Tensor-core M2L work-item size in use and the autotuner's candidate timings (ms)."""
        used = ctypes.c_int(0)
        cand = np.zeros(4, np.int32)
        ms = np.zeros(4)
        rc = self.lib.bem_gpu_tc_tuning(self.ctx, ctypes.byref(used), L.ptr(cand, L.P_int), L.ptr(ms, L.P_dbl))
        self._check(min(rc, 0), "bem_gpu_tc_tuning")
        return {"pairs_per_item": int(used.value), "tuned_in_this_setup": bool(rc == 1),
                "candidates_ms": {int(c): round(float(m), 4) for c, m in zip(cand, ms)}}

    def setup_phases(self):
        """Seconds spent in each part of the last set-up (host plan phases, uploads, device part)."""
        out = np.zeros(16)
        self._check(self.lib.bem_gpu_setup_phases(self.ctx, L.ptr(out, L.P_dbl)), "bem_gpu_setup_phases")
        keys = ["sources", "octree", "lists", "order_nodes", "m2l_groups", "near_blocks", "dof_incidence", "upload", "device"]
        d = {k: float(v) for k, v in zip(keys, out)}
        d["tree_on_device"] = bool(int(out[9]) & 1)
        d["lists_on_device"] = bool(int(out[9]) & 2)
        up = ["upload_nodes", "upload_blocks", "upload_tc_items", "upload_p2m_lists", "upload_rest"]
        d.update({k: float(v) for k, v in zip(up, out[10:15])})
        d["device_near_weights"] = float(out[15])
        return d

    def poly_roots(self):
        """Roots of the near-field polynomial preconditioner (preconditioner="near_poly") formed by
        the last set-up, in the order they are applied; a conjugate pair is one complex entry
        with positive imaginary part.  Empty when none was formed (Jacobi scaling alone)."""
        re = np.zeros(32)
        im = np.zeros(32)
        n = self.lib.bem_gpu_poly_roots(self.ctx, 32, L.ptr(re, L.P_dbl), L.ptr(im, L.P_dbl))
        self._check(min(n, 0), "bem_gpu_poly_roots")
        return re[:n] + 1j * im[:n]

    def diag(self):
        out = np.zeros(self.matrix_size)
        self._check(self.lib.bem_gpu_get_diag(self.ctx, L.ptr(out, L.P_dbl)), "diag")
        return out

    @property
    def scale_factor(self):
        return self.lib.bem_gpu_scale_factor(self.ctx)

    def near_row(self, point):
        n = self.lib.bem_gpu_near_row(self.ctx, int(point), 0, None, None, None)
        if n < 0:
            self._check(n, "near_row")
        idx = np.zeros(max(n, 1), np.int32)
        g = np.zeros(max(n, 1))
        gn = np.zeros(max(n, 1))
        self.lib.bem_gpu_near_row(self.ctx, int(point), n, L.ptr(idx, L.P_int), L.ptr(g, L.P_dbl), L.ptr(gn, L.P_dbl))
        return idx[:n].copy(), g[:n].copy(), gn[:n].copy()

    def face_leaf(self):
        nf = self.tri.shape[0]
        lv = np.zeros(nf, np.int32)
        c = np.zeros(3 * nf)
        self._check(self.lib.bem_gpu_face_leaf(self.ctx, L.ptr(lv, L.P_int), L.ptr(c, L.P_dbl)), "face_leaf")
        return lv, c.reshape(-1, 3)

    def tree_stats(self):
        out = np.zeros(10, np.int64)
        self._check(self.lib.bem_gpu_tree_stats(self.ctx, L.ptr(out, L.P_i64)), "tree_stats")
        keys = ["nodes", "leaves", "depth", "n_added", "m2l_pairs", "near_pairs", "nnz", "near_blocks", "m2l_chunks", "m2l_groups"]
        return {k: int(v) for k, v in zip(keys, out)}

    def near_bytes(self):
        """Algorithmic bytes of one near-field SpMV of A.x: stored weight blocks in FP64 and in FP32
        (rows padded to 4 columns), the gathered unknowns (8 B per block column) and their DOF
        indices (4 B per block column), the per-target near sums (8 B per target) and the rows
        written (8 B per DOF)."""
        out = np.zeros(6, np.int64)
        self._check(self.lib.bem_gpu_near_stats(self.ctx, L.ptr(out, L.P_i64)), "near_stats")
        return {"weights_fp64": 8 * int(out[0]), "weights_fp32": 4 * int(out[1]), "x_gather": 8 * int(out[2]),
                "dof_index": 4 * int(out[2]), "near_sums": 8 * int(out[4]), "rows": 8 * int(out[5]), "blocks": int(out[3]),
                "targets": int(out[4])}

    def device_bytes(self):
        """Device bytes the context's buffers hold."""
        return int(self.lib.bem_gpu_device_bytes(self.ctx))

    def matvec_time_ms(self, repeats=10):
        return self.profile_matvec(repeats)["total"]

    def profile_matvec(self, repeats=10, mixed=False):
        """Per-stage mat-vec time in ms (CUDA events on the solver stream); mixed=True profiles
        the tensor-core operator of a precision="mixed" context."""
        st = np.zeros(10)
        fn = self.lib.bem_gpu_profile_matvec_mixed if mixed else self.lib.bem_gpu_profile_matvec
        self._check(fn(self.ctx, int(repeats), L.ptr(st, L.P_dbl)), "profile")
        keys = ["p2m", "m2m", "m2l", "l2l", "targets", "total"] + (["m2l_expand", "m2l_contract", "m2l_reduce", "near_sums"] if mixed else [])
        return dict(zip(keys, map(float, st)))

    def matvec_device(self, d_x, d_y, mixed=False):
        """y = A x on device buffers given as integer pointers (n_dof doubles each), on the
        solver's stream; mixed=True uses the tensor-core operator."""
        fn = self.lib.bem_gpu_matvec_device_mixed if mixed else self.lib.bem_gpu_matvec_device
        self._check(fn(self.ctx, int(d_x), int(d_y)), "matvec_device")
        self._check(self.lib.bem_gpu_check_device_status(self.ctx), "device status")


def inspect_plan(X, tri, face_dirichlet, dofs=None, *, expansion_order=10, mac_theta=0.25, fmm_bucket_max_points=30,
                 fmm_max_level=7):
    """Builds the host set-up plan without a GPU and returns (face_level, face_corner, stats):
    the leaf bucket of every element and the tree / list / near-field sizes."""
    lib = L.load()
    X = np.ascontiguousarray(X, np.float64)
    tri = np.ascontiguousarray(tri, np.int32)
    fd = np.ascontiguousarray(face_dirichlet, np.uint8)
    if dofs is None:
        dofs = build_dofs(X, tri, fd)
    keep = [np.ascontiguousarray(dofs[k], np.int32).reshape(-1) for k in ("dof_point", "dof_face", "dof_kind", "face_dof")]
    o = L.Opts()
    lib.bem_gpu_default_opts(ctypes.byref(o))
    o.expansion_order, o.mac_theta = int(expansion_order), float(mac_theta)
    o.leaf_max_elements, o.max_level = int(fmm_bucket_max_points), int(fmm_max_level)
    desc = L.Desc(X.shape[0], L.ptr(X, L.P_dbl), tri.shape[0], L.ptr(tri, L.P_int), L.ptr(fd, L.P_u8), keep[0].shape[0],
                  L.ptr(keep[0], L.P_int), L.ptr(keep[1], L.P_int), L.ptr(keep[2], L.P_int), L.ptr(keep[3], L.P_int))
    lv = np.zeros(tri.shape[0], np.int32)
    corner = np.zeros(3 * tri.shape[0])
    st = np.zeros(10, np.int64)
    rc = lib.bem_plan_inspect(ctypes.byref(o), ctypes.byref(desc), L.ptr(lv, L.P_int), L.ptr(corner, L.P_dbl), L.ptr(st, L.P_i64))
    if rc != 0:
        raise ValueError("plan construction failed: " + L.STATUS.get(rc, str(rc)))
    keys = ["nodes", "leaves", "depth", "n_added", "m2l_pairs", "near_pairs", "nnz", "near_blocks", "m2l_chunks", "m2l_groups"]
    return lv, corner.reshape(-1, 3), {k: int(v) for k, v in zip(keys, st)}


class BatchSolver:
    """Many independent BVPs through bem_gpu_batch_*: `n_workers` solver contexts, each with
    its own host thread and CUDA stream, take submitted problems in FIFO order, so the host
    set-up of one problem overlaps the GPU solve of another.  `submit` returns a ticket;
    `result(ticket)` waits for it and returns (phi, phin, stats) in physical units, like the
    phi / phin fields BEM_BVP::solve() leaves behind (bem/BEM_solveBVP.hpp:376-410)."""

    def __init__(self, n_workers=2, *, expansion_order=10, mac_theta=0.25, fmm_bucket_max_points=30, fmm_max_level=7,
                 solver_tol=1e-9, solver_max_iter=500, device=0, tol_relative=False, preconditioner="none", precision="fp64",
                 poly_degree=8, tc_deterministic=False):
        self.lib = L.load()
        if not self.lib.bem_gpu_is_available():
            raise RuntimeError("no sm_100 CUDA device visible: the GMRES-FMM solver runs only on the GPU")
        o = _make_opts(self.lib, expansion_order, mac_theta, fmm_bucket_max_points, fmm_max_level, solver_tol, solver_max_iter,
                       device, tol_relative, preconditioner, precision, poly_degree, tc_deterministic=tc_deterministic)
        self.handle = self.lib.bem_gpu_batch_create(ctypes.byref(o), int(n_workers))
        if not self.handle:
            raise RuntimeError("bem_gpu_batch_create failed")
        self._pending = {}  # ticket -> arrays the worker reads or writes until the ticket is done

    def submit(self, X, tri, face_dirichlet, known, dofs=None):
        X = np.ascontiguousarray(X, np.float64)
        tri = np.ascontiguousarray(tri, np.int32)
        fd = np.ascontiguousarray(face_dirichlet, np.uint8)
        if dofs is None:
            dofs = build_dofs(X, tri, fd)
        keep = [np.ascontiguousarray(dofs[k], np.int32).reshape(-1) for k in ("dof_point", "dof_face", "dof_kind", "face_dof")]
        n = keep[0].shape[0]
        known = np.ascontiguousarray(known, np.float64)
        if known.shape[0] != n:
            raise ValueError("known values must have one entry per DOF")
        phi, phin, st = np.zeros(n), np.zeros(n), L.Stats()
        desc = L.Desc(X.shape[0], L.ptr(X, L.P_dbl), tri.shape[0], L.ptr(tri, L.P_int), L.ptr(fd, L.P_u8), n,
                      L.ptr(keep[0], L.P_int), L.ptr(keep[1], L.P_int), L.ptr(keep[2], L.P_int), L.ptr(keep[3], L.P_int))
        t = ctypes.c_int64(0)
        rc = self.lib.bem_gpu_batch_submit(self.handle, ctypes.byref(desc), L.ptr(known, L.P_dbl), L.ptr(phi, L.P_dbl),
                                           L.ptr(phin, L.P_dbl), ctypes.byref(st), ctypes.byref(t))
        if rc != L.BEM_OK:
            raise RuntimeError(f"batch submit: {L.STATUS.get(rc, rc)}")
        self._pending[t.value] = (X, tri, fd, keep, known, phi, phin, st)
        return t.value

    def submit_chain(self, X, tri, face_dirichlet, known, n_steps, dt, dofs=None, gravity=9.81):
        """A whole RK4 time-stepping chain (n_steps x 4 stages of set-up, solve and MEL update) as one
        request; `result_chain(ticket)` returns (positions [n, 3], point phi, stats) at the end."""
        X = np.ascontiguousarray(X, np.float64)
        tri = np.ascontiguousarray(tri, np.int32)
        fd = np.ascontiguousarray(face_dirichlet, np.uint8)
        if dofs is None:
            dofs = build_dofs(X, tri, fd)
        keep = [np.ascontiguousarray(dofs[k], np.int32).reshape(-1) for k in ("dof_point", "dof_face", "dof_kind", "face_dof")]
        flags = np.ascontiguousarray(dofs["point_flags"], np.uint8)
        n = keep[0].shape[0]
        known = np.ascontiguousarray(known, np.float64)
        if known.shape[0] != n:
            raise ValueError("known values must have one entry per DOF")
        Xo, po, st = np.zeros(3 * X.shape[0]), np.zeros(X.shape[0]), L.Stats()
        desc = L.Desc(X.shape[0], L.ptr(X, L.P_dbl), tri.shape[0], L.ptr(tri, L.P_int), L.ptr(fd, L.P_u8), n,
                      L.ptr(keep[0], L.P_int), L.ptr(keep[1], L.P_int), L.ptr(keep[2], L.P_int), L.ptr(keep[3], L.P_int))
        t = ctypes.c_int64(0)
        rc = self.lib.bem_gpu_batch_submit_chain(self.handle, ctypes.byref(desc), L.ptr(flags, L.P_u8), L.ptr(known, L.P_dbl),
                                                 int(n_steps), float(dt), float(gravity), L.ptr(Xo, L.P_dbl), L.ptr(po, L.P_dbl),
                                                 ctypes.byref(st), ctypes.byref(t))
        if rc != L.BEM_OK:
            raise RuntimeError(f"batch submit_chain: {L.STATUS.get(rc, rc)}")
        self._pending[t.value] = (X, tri, fd, keep, flags, known, Xo, po, st)
        return t.value

    def result_chain(self, ticket):
        rc = self.lib.bem_gpu_batch_poll(self.handle, int(ticket), 1)
        item = self._pending.pop(int(ticket))
        msg = self.lib.bem_gpu_batch_last_error(self.handle) if rc not in (L.BEM_OK, L.BEM_ERR_NOT_CONVERGED) else None
        self.lib.bem_gpu_batch_release(self.handle, int(ticket))
        if msg is not None:
            raise RuntimeError(f"batch chain {ticket}: {L.STATUS.get(rc, rc)}: {msg.decode() if msg else ''}")
        return item[6].reshape(-1, 3), item[7], item[8]

    def set_budget(self, nbytes):
        """Admission by device memory (bytes held by the worker contexts); 0 = no limit."""
        rc = self.lib.bem_gpu_batch_set_budget(self.handle, int(nbytes))
        if rc != L.BEM_OK:
            raise RuntimeError(f"batch set_budget: {L.STATUS.get(rc, rc)}")

    def stats(self):
        out = np.zeros(6, np.int64)
        self.lib.bem_gpu_batch_stats(self.handle, L.ptr(out, L.P_i64))
        keys = ["admitted", "waited_for_memory", "contexts_recycled", "device_bytes_held", "budget", "queued"]
        return {k: int(v) for k, v in zip(keys, out)}

    def done(self, ticket):
        return self.lib.bem_gpu_batch_poll(self.handle, int(ticket), 0) != L.BEM_ERR_NOT_READY

    def result(self, ticket):
        rc = self.lib.bem_gpu_batch_poll(self.handle, int(ticket), 1)
        item = self._pending.pop(int(ticket))
        msg = self.lib.bem_gpu_batch_last_error(self.handle) if rc not in (L.BEM_OK, L.BEM_ERR_NOT_CONVERGED) else None
        self.lib.bem_gpu_batch_release(self.handle, int(ticket))
        if msg is not None:
            raise RuntimeError(f"batch solve {ticket}: {L.STATUS.get(rc, rc)}: {msg.decode() if msg else ''}")
        return item[5], item[6], item[7]

    def close(self):
        if getattr(self, "handle", None):
            self.lib.bem_gpu_batch_destroy(self.handle)  # finishes queued problems before the arrays go
            self.handle = None
            self._pending.clear()

    def __del__(self):
        self.close()


class MELStage:
    """The Mixed-Eulerian-Lagrangian update that follows each BVP solve of a BEM-MEL time step,
    on the GPU (bem_gpu_mel_*): point velocities u = grad phi (gradPhi(p),
    bem/BEM_BoundaryValues.hpp:500-563), Dphi/Dt on the points that are not all-Neumann
    (DphiDt_damped, lib/include/Network.hpp:224-235) and the RK4 stage push of phi and of the
    point positions (pushPhi / pushPosition, bem/main_time_domain.cpp:2410-2510).  Holds the RK
    state of one time step; `stage(k, ...)` for k = 0..3 returns the positions and point phi at
    which the next BVP is solved (after stage 3: the state at t + dt)."""

    def __init__(self, X, tri, face_dirichlet, dofs=None, device=0, gravity=9.81):
        self.lib = L.load()
        if not self.lib.bem_gpu_is_available():
            raise RuntimeError("no sm_100 CUDA device visible: the MEL update runs only on the GPU")
        self.tri = np.ascontiguousarray(tri, np.int32)
        self.fd = np.ascontiguousarray(face_dirichlet, np.uint8)
        self.dofs = dofs if dofs is not None else build_dofs(X, tri, face_dirichlet)
        self.flags = np.ascontiguousarray(self.dofs["point_flags"], np.uint8)
        self.face_dof = np.ascontiguousarray(self.dofs["face_dof"], np.int32).reshape(-1)
        self.np = int(np.asarray(X).shape[0])
        self.gravity = float(gravity)
        self.handle = self.lib.bem_gpu_mel_create(int(device))
        if not self.handle:
            raise RuntimeError("bem_gpu_mel_create failed")
        self.X0 = np.zeros(3 * self.np)
        self.phi0 = np.zeros(self.np)
        self.accX = np.zeros(3 * self.np)
        self.accphi = np.zeros(self.np)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h:
            self.lib.bem_gpu_mel_destroy(h)
            self.handle = None

    def _surface(self, X, phi, phin):
        X = np.ascontiguousarray(X, np.float64).reshape(-1)
        phi = np.ascontiguousarray(phi, np.float64)
        phin = np.ascontiguousarray(phin, np.float64)
        self._keep = (X, phi, phin)
        return L.MelSurface(self.np, L.ptr(X, L.P_dbl), self.tri.shape[0], L.ptr(self.tri, L.P_int), L.ptr(self.fd, L.P_u8),
                            L.ptr(self.flags, L.P_u8), phi.shape[0], L.ptr(self.face_dof, L.P_int), L.ptr(phi, L.P_dbl),
                            L.ptr(phin, L.P_dbl))

    def _check(self, rc, what):
        if rc != L.BEM_OK:
            msg = self.lib.bem_gpu_mel_last_error(self.handle)
            raise RuntimeError(f"{what}: {L.STATUS.get(rc, rc)}: {msg.decode() if msg else ''}")

    def velocity(self, X, phi, phin):
        """(phi per point, u per point [n, 3]) from per-DOF phi / phin at positions X."""
        s = self._surface(X, phi, phin)
        pp, u = np.zeros(self.np), np.zeros(3 * self.np)
        self._check(self.lib.bem_gpu_mel_velocity(self.handle, ctypes.byref(s), L.ptr(pp, L.P_dbl), L.ptr(u, L.P_dbl)), "mel velocity")
        return pp, u.reshape(-1, 3)

    def stage(self, k, dt, X, phi, phin, u_node=None, damping=None):
        """RK4 stage k (0..3): returns (X_next [n, 3], phi_next per point, u [n, 3], Dphi/Dt)."""
        s = self._surface(X, phi, phin)
        Xo, po, u, dp = np.zeros(3 * self.np), np.zeros(self.np), np.zeros(3 * self.np), np.zeros(self.np)
        un = None if u_node is None else np.ascontiguousarray(u_node, np.float64).reshape(-1)
        dm = None if damping is None else np.ascontiguousarray(damping, np.float64).reshape(-1)
        rc = self.lib.bem_gpu_mel_stage(self.handle, ctypes.byref(s), int(k), float(dt), self.gravity,
                                        None if un is None else L.ptr(un, L.P_dbl), None if dm is None else L.ptr(dm, L.P_dbl),
                                        L.ptr(self.X0, L.P_dbl), L.ptr(self.phi0, L.P_dbl), L.ptr(self.accX, L.P_dbl),
                                        L.ptr(self.accphi, L.P_dbl), L.ptr(Xo, L.P_dbl), L.ptr(po, L.P_dbl), L.ptr(u, L.P_dbl),
                                        L.ptr(dp, L.P_dbl))
        self._check(rc, "mel stage")
        return Xo.reshape(-1, 3), po, u.reshape(-1, 3), dp

    def phit_known(self, X, phi, phin, face_body=None, bodies=None, u=None):
        """Known values of the phi_t BVP (setPhiPhin_t, bem/BEM_setBoundaryTypes.hpp:858-935) for
        the solution (phi, phin per DOF) at positions X: phi_t = -|u|^2/2 - g z on Dirichlet DOFs,
        phin_t on Neumann DOFs (0 on faces of no body; on faces of rigid body b, face_body[f] = b,
        phint_Neumann with bodies[b] = (centre, velocity, angular velocity, acceleration, angular
        acceleration), 15 values).  u: point velocities, None to compute them from the solution.
        Solve with BEM_BVP.solve(known) on the same set-up: ans is phin_t on Dirichlet DOFs and
        phi_t on the others."""
        s = self._surface(X, phi, phin)
        d = self.dofs
        dp, df, dk = (np.ascontiguousarray(d[k], np.int32) for k in ("dof_point", "dof_face", "dof_kind"))
        nf = self.tri.shape[0]
        fb = np.full(nf, -1, np.int32) if face_body is None else np.ascontiguousarray(face_body, np.int32)
        bd = np.zeros((0, 15)) if bodies is None else np.ascontiguousarray(bodies, np.float64).reshape(-1, 15)
        bdf = np.ascontiguousarray(bd.reshape(-1)) if bd.size else np.zeros(15)
        uu = None if u is None else np.ascontiguousarray(u, np.float64).reshape(-1)
        out = np.zeros(dp.shape[0])
        rc = self.lib.bem_gpu_mel_phit_known(self.handle, ctypes.byref(s), L.ptr(dp, L.P_int), L.ptr(df, L.P_int), L.ptr(dk, L.P_int),
                                             L.ptr(fb, L.P_int), int(bd.shape[0]), L.ptr(bdf, L.P_dbl), self.gravity,
                                             None if uu is None else L.ptr(uu, L.P_dbl), L.ptr(out, L.P_dbl))
        self._check(rc, "phi_t known values")
        return out
