"""Host-side logic of the product library (no GPU): C-ABI exports, DOF keys and the
set-up plan (octree, lists, near-field sparsity) against the oracle."""
import re
import os

import numpy as np
import pytest

from conftest import ROOT
from bem_for_nonlinear_waves_b200 import build_dofs, make_tank
from bem_for_nonlinear_waves_b200.bvp import inspect_plan


def header_functions():
    with open(os.path.join(ROOT, "include", "bem_b200.h")) as fh:
        src = fh.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bem_\w+)\s*\(", src)))


def test_library_exports_every_header_symbol(product_lib):
    names = header_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(product_lib, n), n


TANKS = [dict(h=0.1), dict(h=0.1, noise_sigma=0.02, seed=3), dict(h=0.05), dict(length=1.3, width=0.7, depth=0.4, h=0.1)]


@pytest.mark.parametrize("spec", TANKS)
def test_dofs_match_oracle(product_lib, oracle_mod, spec):
    t = make_tank(**spec)
    a = build_dofs(t.X, t.tri, t.face_dirichlet)
    b = oracle_mod.build_dofs(t.X, t.tri, t.face_dirichlet)
    for k in ("dof_point", "dof_face", "dof_kind", "face_dof", "point_flags"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    # corner points carry one Dirichlet key plus one constrained key per Neumann face
    kinds = np.bincount(a["dof_kind"], minlength=3)
    assert kinds[0] > 0 and kinds[1] > 0 and kinds[2] > 0


@pytest.mark.parametrize("spec,p", [(TANKS[0], 8), (TANKS[1], 10), (TANKS[2], 8), (TANKS[3], 6)])
def test_plan_tree_and_lists_match_oracle(product_lib, oracle_mod, spec, p):
    t = make_tank(**spec)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    lv, corner, st = inspect_plan(t.X, t.tri, t.face_dirichlet, d, expansion_order=p)
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=p)
    ost = o.stats()
    olv, oc = o.face_leaf()
    np.testing.assert_array_equal(lv, olv)
    np.testing.assert_array_equal(corner, oc)  # bit-exact bucket bounds
    for k in ("nodes", "leaves", "depth", "n_added", "m2l_pairs", "near_pairs", "nnz"):
        assert st[k] == ost[k], k


def test_build_dofs_rejects_bad_connectivity(product_lib):
    t = make_tank(h=0.25)
    tri = t.tri.copy()
    tri[0, 0] = t.X.shape[0] + 5
    with pytest.raises(ValueError):
        build_dofs(t.X, tri, t.face_dirichlet)


def test_plan_rejects_nonfinite_coordinates(product_lib):
    t = make_tank(h=0.25)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    X = t.X.copy()
    X[3, 1] = np.nan
    with pytest.raises(ValueError):
        inspect_plan(X, t.tri, t.face_dirichlet, d)


def test_device_memory_estimate_counts_precision_and_preconditioner_buffers(product_lib):
    """bem_gpu_estimate_bytes (host arithmetic only): the mixed context adds the FP32 weights and
    the FP32 copy of the P2M operator, the near-block preconditioner its inverses (at most 64^2
    values per core of <= 64 DOFs) and core lists, the polynomial preconditioner its flexible
    basis."""
    import ctypes

    from bem_for_nonlinear_waves_b200 import _lib as L
    from bem_for_nonlinear_waves_b200.bvp import _make_opts

    t = make_tank(h=0.05)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    X = np.ascontiguousarray(t.X, np.float64)
    tri = np.ascontiguousarray(t.tri, np.int32)
    fd = np.ascontiguousarray(t.face_dirichlet, np.uint8)
    arrs = [np.ascontiguousarray(d[k], np.int32).reshape(-1) for k in ("dof_point", "dof_face", "dof_kind", "face_dof")]
    desc = L.Desc(X.shape[0], L.ptr(X, L.P_dbl), tri.shape[0], L.ptr(tri, L.P_int), L.ptr(fd, L.P_u8), arrs[0].shape[0],
                  L.ptr(arrs[0], L.P_int), L.ptr(arrs[1], L.P_int), L.ptr(arrs[2], L.P_int), L.ptr(arrs[3], L.P_int))

    def est(precond, precision):
        o = _make_opts(product_lib, 8, 0.25, 30, 7, 1e-9, 500, 0, True, precond, precision)
        return product_lib.bem_gpu_estimate_bytes(ctypes.byref(o), ctypes.byref(desc))

    ndof = arrs[0].shape[0]
    base = est("jacobi", "fp64")
    assert base > 0
    assert est("jacobi", "mixed") > base
    assert est("near_block", "fp64") - base == ndof * (64 * 8 + 16)
    assert est("near_poly", "fp64") - base == (500 + 2) * ndof * 8  # the flexible basis: max_iter + 2 more columns
