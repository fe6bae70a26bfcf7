"""The low-precision A.x with its near field on a second stream (concurrent with the FMM
passes, far field added afterwards; opts.overlap_near = 1) against the single-stream fused
form: the same operator up to the association of one sum per row (near + far - diag x), so
one application agrees to 1e-13 relative (with the fixed-order M2L reduction, tc_deterministic),
and both solves converge to the same solution within the tolerance."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, known_values, make_tank, point_normals

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p", [8, 12])
def test_overlapped_operator_equals_fused(product_lib, p):
    import torch

    t = make_tank(1.0, 0.5, 0.4, 0.04, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=61)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    a = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=p, precision="mixed", dofs=d, overlap_near=True, tc_deterministic=True)
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=p, precision="mixed", dofs=d, overlap_near=False, tc_deterministic=True)
    a.setup()
    b.setup()
    n = a.matrix_size
    g = torch.Generator().manual_seed(7)
    for _ in range(3):  # repeated: the side stream's work of one application must not leak into the next
        x = torch.randn(n, dtype=torch.float64, generator=g).cuda()
        ya, yb = torch.empty_like(x), torch.empty_like(x)
        torch.cuda.synchronize()
        a.matvec_device(x.data_ptr(), ya.data_ptr(), mixed=True)
        b.matvec_device(x.data_ptr(), yb.data_ptr(), mixed=True)
        torch.cuda.synchronize()
        u, v = ya.cpu().numpy(), yb.cpu().numpy()
        assert np.abs(u - v).max() / np.abs(v).max() < 1e-13


def test_overlapped_solve(product_lib):
    t = make_tank(1.0, 0.5, 0.4, 0.04, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=62)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    k = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    kw = dict(expansion_order=10, solver_tol=1e-11, tol_relative=True, preconditioner="jacobi", precision="mixed", dofs=d,
              tc_deterministic=True)
    a = BEM_BVP(t.X, t.tri, t.face_dirichlet, overlap_near=True, **kw)
    b = BEM_BVP(t.X, t.tri, t.face_dirichlet, overlap_near=False, **kw)
    a.solve(k)
    b.solve(k)
    assert a.last_gmres_converged and b.last_gmres_converged
    first = a.ans.copy()
    a.solve(k)
    assert np.array_equal(a.ans, first)  # deterministic with two streams
    assert np.abs(a.ans - b.ans).max() / np.abs(b.ans).max() < 1e-8
