"""bem_gpu_matvec_device_noalloc against bem_gpu_matvec_device, through the C ABI.

The no-alloc entry point is for callers that cannot allocate device memory while they apply
the operator: a time integrator or outer solver that runs out of a fixed device-memory
reservation, or a server that holds many small problems on one device and wants one shared
slot area instead of one per problem.  Its M2L pair slots live in a fixed 32 MiB area of the
library's device image, whose address the context looked up at set-up.

Checked here: two calls in a row with different inputs agree with the context's mat-vec
(same kernels in the same order: tolerance 1e-13 relative to the vector maximum), the
device's free memory and torch's reserved memory are the same before and after the calls,
a mixed-precision context gets the FP64 operator from it, and a problem whose slot area
exceeds 32 MiB is rejected with BEM_ERR_UNSUPPORTED.  This file is collected last, so a run
that stops at its first failure has run every other test before it."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, make_tank
from bem_for_nonlinear_waves_b200 import _lib as L

pytestmark = pytest.mark.gpu

SLOT_BYTES = 32 << 20


def _ncoef(p):
    return (p + 1) * (p + 2) // 2


def _setup(h, p, precision="fp64"):
    t = make_tank(1.0, 0.5, 0.4, h, amplitude=0.02, wavelength=0.7, noise_sigma=0.1, seed=3)
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=p, precision=precision)
    bvp.setup()
    return bvp


def _inputs(n, seed):
    import torch

    g = torch.Generator().manual_seed(seed)
    return [torch.randn(n, dtype=torch.float64, generator=g).cuda() for _ in range(2)]


def test_noalloc_matvec_matches_context_matvec(product_lib):
    import torch

    bvp = _setup(0.04, 10)
    pairs = bvp.tree_stats()["m2l_pairs"]
    assert pairs > 0 and pairs * 2 * _ncoef(10) * 16 <= SLOT_BYTES
    lib = L.load()
    n = bvp.matrix_size
    xs = _inputs(n, 11)
    y_na = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    y_ref = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    # two no-alloc calls in a row (the second reuses the slot area)
    for x, y in zip(xs, y_na):
        assert lib.bem_gpu_matvec_device_noalloc(bvp.ctx, x.data_ptr(), y.data_ptr()) == L.BEM_OK, \
            lib.bem_gpu_last_error(bvp.ctx)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"device free memory changed across the no-alloc calls: {free0} -> {free1}"
    assert torch.cuda.memory_reserved() == reserved0
    for x, y in zip(xs, y_ref):
        assert lib.bem_gpu_matvec_device(bvp.ctx, x.data_ptr(), y.data_ptr()) == L.BEM_OK
    torch.cuda.synchronize()
    for a, b in zip(y_na, y_ref):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.isfinite(a).all()
        assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
    # the two inputs differ, so must the outputs (the second call did not return stale slots)
    assert np.abs(y_na[0].cpu().numpy() - y_na[1].cpu().numpy()).max() > 1e-3 * np.abs(y_ref[1].cpu().numpy()).max()


def test_noalloc_matvec_is_fp64_on_mixed_context(product_lib):
    import torch

    lib = L.load()
    b64 = _setup(0.04, 10)
    bmx = _setup(0.04, 10, precision="mixed")
    n = b64.matrix_size
    assert bmx.matrix_size == n
    x = _inputs(n, 5)[0]
    y64 = torch.empty(n, dtype=torch.float64, device="cuda")
    ymx = torch.empty_like(y64)
    for _ in range(2):
        assert lib.bem_gpu_matvec_device_noalloc(bmx.ctx, x.data_ptr(), ymx.data_ptr()) == L.BEM_OK
    assert lib.bem_gpu_matvec_device(b64.ctx, x.data_ptr(), y64.data_ptr()) == L.BEM_OK
    torch.cuda.synchronize()
    a, b = ymx.cpu().numpy(), y64.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()


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
