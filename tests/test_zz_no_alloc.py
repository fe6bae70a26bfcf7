"""bem_gpu_matvec_device_noalloc (M2L pair slots in the library's fixed device area) against
bem_gpu_matvec_device (slots in the context) on the same context and device inputs, two calls
in a row, through the C ABI.  Both paths run the same kernels in the same order, so the results
agree to rounding: tolerance 1e-13 relative to the vector maximum.  A problem whose slot area
exceeds the fixed 32 MiB is rejected with BEM_ERR_UNSUPPORTED."""
import ctypes

import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, make_tank
from bem_for_nonlinear_waves_b200 import _lib as L

pytestmark = pytest.mark.gpu

SLOT_BYTES = 32 << 20


def _ncoef(p):
    return (p + 1) * (p + 2) // 2


def _setup(h, p):
    t = make_tank(1.0, 0.5, 0.4, h, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=3)
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=p)
    bvp.setup()
    return bvp


def test_noalloc_matvec_matches_context_matvec(product_lib):
    import torch

    bvp = _setup(0.04, 10)
    pairs = bvp.tree_stats()["m2l_pairs"]
    assert pairs > 0 and pairs * 2 * _ncoef(10) * 16 <= SLOT_BYTES
    lib = L.load()
    n = bvp.matrix_size
    g = torch.Generator().manual_seed(11)
    xs = [torch.randn(n, dtype=torch.float64, generator=g).cuda() for _ in range(2)]
    y_na = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    y_ref = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    # two no-alloc calls in a row (the second reuses the slot area), then the context path
    for x, y in zip(xs, y_na):
        assert lib.bem_gpu_matvec_device_noalloc(bvp.ctx, x.data_ptr(), y.data_ptr()) == L.BEM_OK, \
            lib.bem_gpu_last_error(bvp.ctx)
    for x, y in zip(xs, y_ref):
        assert lib.bem_gpu_matvec_device(bvp.ctx, x.data_ptr(), y.data_ptr()) == L.BEM_OK
    torch.cuda.synchronize()
    for a, b in zip(y_na, y_ref):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    # the two inputs differ, so must the outputs (the second call did not return stale slots)
    assert np.abs(y_na[0].cpu().numpy() - y_na[1].cpu().numpy()).max() > 1e-3 * np.abs(y_ref[1].cpu().numpy()).max()


def test_noalloc_matvec_rejects_oversized_problem(product_lib):
    import torch

    bvp = _setup(0.025, 12)
    pairs = bvp.tree_stats()["m2l_pairs"]
    assert pairs * 2 * _ncoef(12) * 16 > SLOT_BYTES
    lib = L.load()
    x = torch.zeros(bvp.matrix_size, dtype=torch.float64, device="cuda")
    y = torch.zeros_like(x)
    torch.cuda.synchronize()
    rc = lib.bem_gpu_matvec_device_noalloc(bvp.ctx, x.data_ptr(), y.data_ptr())
    assert rc == L.BEM_ERR_UNSUPPORTED
    msg = lib.bem_gpu_last_error(bvp.ctx).decode()
    assert "exceeds" in msg and str(SLOT_BYTES) in msg
    assert lib.bem_gpu_matvec_device_noalloc(None, x.data_ptr(), y.data_ptr()) == L.BEM_ERR_INVALID_ARGUMENT
