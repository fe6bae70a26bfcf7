"""Octree growth and interaction lists on the device (tree.cu, the default set-up path) against
the host's: both restate the reference's Buckets::generateTree
(lib/include/lib_spatial_partitioning.hpp:1078-1111) and list traversal (moments.hpp:950-997),
whose host versions the CPU tests pin to the oracle and the compiled reference.  The whole plan
built from the device tree and lists must equal the host one array for array."""
import ctypes

import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import _lib as L
from bem_for_nonlinear_waves_b200 import add_box_body, build_dofs, make_tank

pytestmark = pytest.mark.gpu


def _check(lib, t, leaf=30, max_level=7, p=8):
    X = np.ascontiguousarray(t.X, np.float64)
    tri = np.ascontiguousarray(t.tri, np.int32)
    fd = np.ascontiguousarray(t.face_dirichlet, np.uint8)
    d = build_dofs(X, tri, fd)
    keep = [np.ascontiguousarray(d[k], np.int32).reshape(-1) for k in ("dof_point", "dof_face", "dof_kind", "face_dof")]
    desc = L.Desc(X.shape[0], L.ptr(X, L.P_dbl), tri.shape[0], L.ptr(tri, L.P_int), L.ptr(fd, L.P_u8), keep[0].shape[0],
                  *[L.ptr(k, L.P_int) for k in keep])
    o = L.Opts()
    lib.bem_gpu_default_opts(ctypes.byref(o))
    o.expansion_order, o.leaf_max_elements, o.max_level = p, leaf, max_level
    out = np.zeros(4, np.int64)
    assert lib.bem_gpu_tree_check(ctypes.byref(o), ctypes.byref(desc), L.ptr(out, L.P_i64)) == 0
    return out


@pytest.mark.parametrize("h,noise,leaf,max_level", [(0.05, 0.0, 30, 7), (0.05, 0.2, 30, 7), (0.03, 0.2, 8, 7),
                                                    (0.03, 0.2, 100, 3), (0.02, 0.3, 30, 5)])
def test_device_tree_equals_host_tree(product_lib, h, noise, leaf, max_level):
    t = make_tank(2.0, 1.0, 0.5, h, amplitude=0.02, wavelength=0.9, noise_sigma=noise * h, seed=7)
    out = _check(product_lib, t, leaf, max_level)
    assert out[0] == 3 and out[1] == 0, out.tolist()


def test_device_tree_with_submerged_body(product_lib):
    t = make_tank(2.0, 1.0, 0.6, 0.04, amplitude=0.02, wavelength=0.9, noise_sigma=0.004, seed=9)
    t = add_box_body(t, (0.8, 0.5, -0.3), (0.3, 0.3, 0.2), 0.04, U=(0.05, 0.0, 0.0), Omega=(0.0, 0.0, 0.1))
    out = _check(product_lib, t)
    assert out[0] == 3 and out[1] == 0, out.tolist()
