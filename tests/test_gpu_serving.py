"""Serving through the batch API: whole RK4 time-stepping chains as requests, continuous
batching with other requests, and admission by device memory.

A chain request (bem_gpu_batch_submit_chain) runs, per stage, a set-up at the stage positions
(the first in full, then bem_gpu_setup_refresh), a solve warm-started from the previous stage's
solution and the MEL stage update; the same steps driven one call at a time from Python give the
same positions and point phi bit for bit (FP64).  A chain gives the same result alone and among
other requests on three workers (mixed precision, whose fused M2L reduction varies in the last
bits: within 1e-8 relative).  With a device-memory budget for one request at a time, every
request still completes and some wait for memory; a request above the budget is refused."""
import ctypes

import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, BatchSolver, MELStage, build_dofs, known_values, make_tank, point_normals
from bem_for_nonlinear_waves_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _problem(h, seed, box=False):
    fb = (0.5, 0.25, 0.2, 0.2, 0.1, (0.05, 0.0, 0.02), (0.0, 0.1, 0.0)) if box else None
    t = make_tank(1.0, 0.5, 0.4, h, amplitude=0.02, wavelength=0.7, noise_sigma=0.1 * h, seed=seed, floating_box=fb)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    k = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    return t, d, k


def _python_chain(t, d, k, n_steps, dt, kw):
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, **kw)
    mel = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d)
    X, known, prev = np.array(t.X), k.copy(), None
    dirichlet = d["dof_kind"] == 0
    first = True
    for _ in range(n_steps):
        for s in range(4):
            if first:
                b.X = X
                b.setup()
                first = False
            else:
                b.refresh(X)
            b.solve(known, x0=prev)
            prev = b.ans.copy()
            X, pnext, _, _ = mel.stage(s, dt, X, b.phi, b.phin)
            known = known.copy()
            known[dirichlet] = pnext[d["dof_point"][dirichlet]]
    return X, pnext


def _desc(t, d, keep):
    X = np.ascontiguousarray(t.X, np.float64)
    tri = np.ascontiguousarray(t.tri, np.int32)
    fd = np.ascontiguousarray(t.face_dirichlet, np.uint8)
    arrs = [np.ascontiguousarray(d[k], np.int32).reshape(-1) for k in ("dof_point", "dof_face", "dof_kind", "face_dof")]
    keep.extend([X, tri, fd, arrs])
    return L.Desc(X.shape[0], L.ptr(X, L.P_dbl), tri.shape[0], L.ptr(tri, L.P_int), L.ptr(fd, L.P_u8), arrs[0].shape[0],
                  L.ptr(arrs[0], L.P_int), L.ptr(arrs[1], L.P_int), L.ptr(arrs[2], L.P_int), L.ptr(arrs[3], L.P_int))


def test_chain_request_matches_step_by_step(product_lib):
    t, d, k = _problem(0.05, 21, box=True)
    kw = dict(expansion_order=8, solver_tol=1e-10, tol_relative=True, preconditioner="jacobi", precision="fp64")
    Xr, pr = _python_chain(t, d, k, 2, 1e-3, kw)
    bs = BatchSolver(2, **kw)
    tk = bs.submit_chain(t.X, t.tri, t.face_dirichlet, k, n_steps=2, dt=1e-3, dofs=d)
    X, p, st = bs.result_chain(tk)
    bs.close()
    assert st.converged == 1 and st.iterations > 0
    assert np.array_equal(X, Xr)
    assert np.array_equal(p, pr)
    assert np.abs(X - t.X).max() > 0  # the free surface moved


def test_chain_same_alone_and_in_the_mix(product_lib):
    kw = dict(expansion_order=8, solver_tol=1e-10, tol_relative=True, preconditioner="jacobi", precision="mixed")
    t, d, k = _problem(0.05, 22)
    bs = BatchSolver(3, **kw)
    X0, p0, st0 = bs.result_chain(bs.submit_chain(t.X, t.tri, t.face_dirichlet, k, n_steps=2, dt=1e-3, dofs=d))
    others = [_problem(h, s, box=(s % 2 == 0)) for h, s in [(0.04, 23), (0.06, 24), (0.05, 25), (0.045, 26)]]
    tks = [bs.submit(o[0].X, o[0].tri, o[0].face_dirichlet, o[2], dofs=o[1]) for o in others[:2]]
    tc = bs.submit_chain(t.X, t.tri, t.face_dirichlet, k, n_steps=2, dt=1e-3, dofs=d)
    tks += [bs.submit_chain(o[0].X, o[0].tri, o[0].face_dirichlet, o[2], n_steps=1, dt=1e-3, dofs=o[1]) for o in others[2:]]
    X1, p1, st1 = bs.result_chain(tc)
    for tk in tks[:2]:
        assert bs.result(tk)[2].converged == 1
    for tk in tks[2:]:
        assert bs.result_chain(tk)[2].converged == 1
    bs.close()
    assert st0.converged == 1 and st1.converged == 1
    assert np.abs(X1 - X0).max() <= 1e-8 * np.abs(X0).max()
    assert np.abs(p1 - p0).max() <= 1e-8 * np.abs(p0).max()


def test_admission_by_device_memory(product_lib):
    kw = dict(expansion_order=8, solver_tol=1e-9, tol_relative=True, preconditioner="jacobi", precision="fp64")
    probs = [_problem(h, s) for h, s in [(0.04, 31), (0.045, 32), (0.05, 33), (0.04, 34)]]
    lib = L.load()
    # the estimate of the largest request, against the bytes its context really holds
    t, d, k = probs[0]
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, **kw)
    b.solve(k)
    keep = []
    est = lib.bem_gpu_estimate_bytes(ctypes.byref(b.opts), ctypes.byref(_desc(t, d, keep)))
    held = b.device_bytes()
    assert est > 0 and held > 0
    assert 0.3 * held <= est <= 3.0 * held, (est, held)
    ref = b.ans.copy()
    del b
    bs = BatchSolver(3, **kw)
    bs.set_budget(int(1.5 * max(est, held)))  # room for one request at a time
    tks = [bs.submit(t.X, t.tri, t.face_dirichlet, k, dofs=d) for t, d, k in probs]
    res = [bs.result(tk) for tk in tks]
    assert all(r[2].converged == 1 for r in res)
    got = np.where(probs[0][1]["dof_kind"] == 0, res[0][1], res[0][0])
    assert np.array_equal(got, ref)
    st = bs.stats()
    assert st["admitted"] == len(probs)
    assert st["waited_for_memory"] > 0 or st["contexts_recycled"] > 0
    bs.set_budget(1 << 20)  # 1 MiB: below any request
    t, d, k = probs[0]
    tk = bs.submit(t.X, t.tri, t.face_dirichlet, k, dofs=d)
    with pytest.raises(RuntimeError, match="out of memory"):
        bs.result(tk)
    bs.close()
