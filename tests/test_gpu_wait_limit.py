"""Failure detection of the tensor-core M2L's bounded device-side waits, without a GPU fault.

Every mbarrier wait of k_m2l_tc has an iteration limit (a kernel argument).  With the limit set
to 0 through bem_gpu_set_wait_limit, the first pipeline wait of every CTA gives up at once: the
CTA records the failure, waits (with the default limit) for its own copies and MMAs already in
flight, frees its tensor memory and returns.  The host then reads BEM_ERR_DEVICE from
bem_gpu_check_device_status, and after restoring the limit the same context computes the same
mixed-precision mat-vec as before, bit for bit (fixed-order M2L reduction)."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, make_tank
from bem_for_nonlinear_waves_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_tc_wait_timeout_is_reported_and_context_recovers(product_lib):
    import torch

    t = make_tank(1.0, 0.5, 0.4, 0.04, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=3)
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=10, precision="mixed", tc_deterministic=True)
    bvp.setup()
    assert bvp.tree_stats()["m2l_pairs"] > 0
    lib = L.load()
    n = bvp.matrix_size
    x = torch.randn(n, dtype=torch.float64, generator=torch.Generator().manual_seed(4)).cuda()
    y0, y1, y2 = (torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(3))
    torch.cuda.synchronize()
    bvp.matvec_device(x.data_ptr(), y0.data_ptr(), mixed=True)  # checks the device status: OK
    assert lib.bem_gpu_set_wait_limit(bvp.ctx, 0) == L.BEM_OK
    assert lib.bem_gpu_matvec_device_mixed(bvp.ctx, x.data_ptr(), y1.data_ptr()) == L.BEM_OK
    assert lib.bem_gpu_check_device_status(bvp.ctx) == L.BEM_ERR_DEVICE
    assert b"bounded wait" in lib.bem_gpu_last_error(bvp.ctx)
    torch.cuda.synchronize()  # the context is still usable: no sticky CUDA error
    assert lib.bem_gpu_set_wait_limit(bvp.ctx, -1) == L.BEM_OK
    bvp.matvec_device(x.data_ptr(), y2.data_ptr(), mixed=True)
    torch.cuda.synchronize()
    a, b = y0.cpu().numpy(), y2.cpu().numpy()
    assert np.isfinite(a).all()
    np.testing.assert_array_equal(a, b)
