"""The Krylov operator A.x against the general operator it specialises.

A.x (bem_gpu_matvec_device, the operator of every GMRES iteration) takes three shortcuts of its
own: the P2M operator fused with each leaf's first M2M shift, no downward pass (the rows sum the
L2Ps of the M2L locals along each target bucket's path: L2L re-expands the same polynomial, so
the sum equals the L2P of the shifted local), and the near-field sums on a second stream beside
the FMM passes.  With the known values zero, A.x equals the general operator bem_gpu_apply
(per-level P2M/M2M, L2L launches, one targets kernel) fed phin = x on Dirichlet DOFs and phi = x
on the others.  Checked on a multi-level tank with a floating box to 1e-12 of the largest row,
with and without the second stream (bit for bit between those two)."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, make_tank

pytestmark = pytest.mark.gpu


def _tank():
    fb = (0.5, 0.25, 0.2, 0.2, 0.1, (0.05, 0.0, 0.02), (0.0, 0.1, 0.0))
    t = make_tank(1.0, 0.5, 0.4, 0.03, amplitude=0.02, wavelength=0.7, noise_sigma=0.003, seed=9, floating_box=fb)
    return t, build_dofs(t.X, t.tri, t.face_dirichlet)


@pytest.mark.parametrize("p", [6, 10])
def test_ax_equals_general_operator(product_lib, p):
    import torch

    t, d = _tank()
    ys = []
    for overlap in (True, False):
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, expansion_order=p, overlap_near=overlap)
        b.setup()
        assert b.tree_stats()["m2l_pairs"] > 0
        n = b.matrix_size
        x = torch.from_numpy(np.random.default_rng(7).standard_normal(n)).cuda()
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        b.matvec_device(x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        ys.append(y.cpu().numpy())
    np.testing.assert_array_equal(ys[0], ys[1])
    xv = np.random.default_rng(7).standard_normal(b.matrix_size)
    dirichlet = d["dof_kind"] == 0
    ref = b.apply(np.where(dirichlet, 0.0, xv), np.where(dirichlet, xv, 0.0))
    assert np.abs(ys[0] - ref).max() <= 1e-12 * np.abs(ref).max()
