"""Mixed-precision operator and solve (tensor-core M2L with FP16 split operands and FP32
accumulation, FP64 refinement) against the FP64 path on the same context inputs.
Tolerances: one low-precision mat-vec within 1e-5 of the FP64 one (relative to the vector
maximum; the M2L carries ~2^-22 relative error per coefficient); solutions driven to a
relative residual of 1e-11 agree to 1e-8 relative."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, known_values, make_tank, point_normals

pytestmark = pytest.mark.gpu


def _tank(h=0.04, seed=5):
    return make_tank(1.0, 0.5, 0.4, h, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=seed)


@pytest.mark.parametrize("p", [6, 10, 11, 12])
def test_mixed_matvec_close_to_fp64(product_lib, p):
    import torch

    t = _tank()
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=p, precision="mixed")
    bvp.setup()
    assert bvp.tree_stats()["m2l_pairs"] > 0
    n = bvp.matrix_size
    g = torch.Generator().manual_seed(3)
    for _ in range(2):
        x = torch.randn(n, dtype=torch.float64, generator=g).cuda()
        y64 = torch.empty_like(x)
        ylo = torch.empty_like(x)
        torch.cuda.synchronize()
        bvp.matvec_device(x.data_ptr(), y64.data_ptr())
        bvp.matvec_device(x.data_ptr(), ylo.data_ptr(), mixed=True)
        torch.cuda.synchronize()
        a, b = ylo.cpu().numpy(), y64.cpu().numpy()
        rel = np.abs(a - b).max() / np.abs(b).max()
        assert rel < 1e-5, rel
        assert rel > 0.0  # the two operators are different code paths


def test_mixed_rejects_high_order(product_lib):
    # every order the solver accepts (1..12) has a tensor-core path; beyond it the context
    # is refused at creation, for either precision
    t = _tank(h=0.1)
    for prec in ("mixed", "fp64"):
        with pytest.raises(RuntimeError, match="bem_gpu_create failed"):
            BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=13, precision=prec)


@pytest.mark.parametrize("precond,tol,agree", [("jacobi", 1e-11, 1e-8), ("jacobi", 1e-8, 1e-5)])
def test_mixed_solve_matches_fp64(product_lib, precond, tol, agree):
    t = _tank()
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    known = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    sols = {}
    for prec in ("fp64", "mixed"):
        bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=10, solver_tol=tol, tol_relative=True, solver_max_iter=1500,
                      dofs=d, preconditioner=precond, precision=prec)
        bvp.solve(known)
        assert bvp.last_gmres_converged, (prec, bvp.last_gmres_residual_norm)
        sols[prec] = (bvp.ans.copy(), bvp.stats.matvecs, bvp.stats.matvecs_lo)
    a, b = sols["mixed"][0], sols["fp64"][0]
    assert np.abs(a - b).max() <= agree * np.abs(b).max()
    assert sols["mixed"][2] > 0 and sols["fp64"][2] == 0
    assert sols["mixed"][1] < sols["mixed"][2]  # most operator applications are low precision


@pytest.mark.parametrize("p", [10, 12])
def test_fused_reduction_matches_fixed_order(product_lib, p):
    """The tensor-core M2L's two reductions: each pair added into its target's FP32 accumulator in
    L2 (default; the summation order varies), or per-pair partials summed in a fixed order in FP64
    (tc_deterministic; repeated applications are bit-identical).  Both apply the same operator to
    FP32 rounding of the M2L sums: within 1e-6 of each other relative to the vector maximum."""
    import torch

    t = _tank()
    fused = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=p, precision="mixed")
    fixed = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=p, precision="mixed", tc_deterministic=True)
    fused.setup()
    fixed.setup()
    n = fused.matrix_size
    x = torch.randn(n, dtype=torch.float64, generator=torch.Generator().manual_seed(9)).cuda()
    ys = [torch.empty_like(x) for _ in range(4)]
    torch.cuda.synchronize()
    fused.matvec_device(x.data_ptr(), ys[0].data_ptr(), mixed=True)
    fused.matvec_device(x.data_ptr(), ys[1].data_ptr(), mixed=True)
    fixed.matvec_device(x.data_ptr(), ys[2].data_ptr(), mixed=True)
    fixed.matvec_device(x.data_ptr(), ys[3].data_ptr(), mixed=True)
    torch.cuda.synchronize()
    a, a2, b, b2 = (y.cpu().numpy() for y in ys)
    scale = np.abs(b).max()
    assert np.array_equal(b, b2)
    assert np.abs(a - b).max() <= 1e-6 * scale
    assert np.abs(a2 - b).max() <= 1e-6 * scale
