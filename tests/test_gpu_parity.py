"""CUDA path (lib/libbem_b200.so through its C ABI) against the reference's golden outputs
and the oracle.  Tolerances: FP64 everywhere; near weights and single mat-vecs agree to
rounding (1e-11 relative to the row/vector maximum; near-row checksums 1e-11 against the
reference, which uses the same 15-digit 5x5 Gauss-Legendre constants), solutions to 1e-10
relative -- the parity bar for the plain FP64 path at the same order and tree -- with both
sides solved to an absolute residual of 1e-12."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import BEM_BVP, build_dofs, known_values, make_tank, point_normals
import goldens

pytestmark = pytest.mark.gpu
GOLDEN_NAMES = goldens.names()


@pytest.fixture(scope="module", params=GOLDEN_NAMES)
def case(request, product_lib, oracle_mod):
    g = goldens.Golden(request.param)
    t = g.tank
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=g.p, solver_tol=g.tol, solver_max_iter=1000, dofs=d)
    bvp.setup()
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=g.p)
    return g, d, bvp, o


def test_gpu_tree_matches_reference(case):
    g, d, bvp, o = case
    lv, corner = bvp.face_leaf()
    fl = g.z["face_leaf"]
    f = fl[:, 0].astype(int)
    np.testing.assert_array_equal(lv[f], fl[:, 1].astype(int))
    np.testing.assert_array_equal(corner[f], fl[:, 2:5])


def test_gpu_near_weights_match_oracle(case):
    g, d, bvp, o = case
    for p in range(bvp.X.shape[0]):
        i1, g1, n1 = bvp.near_row(p)
        i2, g2, n2 = o.near_row(p)
        np.testing.assert_array_equal(i1, i2)
        assert np.abs(g1 - g2).max() <= 1e-12 * np.abs(g2).max()
        # Gn weights of nearly coplanar elements are R.n / r^3 with R.n cancelling to rounding,
        # so their differences are measured against the row's l1 norm (its scale in a mat-vec)
        assert np.abs(n1 - n2).max() <= 1e-11 * max(np.abs(n2).sum(), 1e-300)


def test_gpu_near_weights_match_reference_checksums(case):
    g, d, bvp, o = case
    z = g.z
    for i, p in enumerate(z["near_points"]):
        idx, wg, wgn = bvp.near_row(p)
        assert len(idx) == z["near_count"][i]
        np.testing.assert_allclose(wg.sum(), z["near_sum_g"][i], rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(wgn.sum(), z["near_sum_gn"][i], rtol=1e-11, atol=1e-11 * np.abs(wgn).sum())


def test_gpu_diag_matches_reference(case):
    g, d, bvp, o = case
    np.testing.assert_allclose(bvp.diag(), g.diag(d), rtol=1e-12, atol=1e-12)


def test_gpu_matvec_matches_reference(case):
    g, d, bvp, o = case
    phi, phin, expect = g.matvec_input(d)
    got = bvp.apply(phi, phin)
    assert np.abs(got - expect).max() <= 1e-11 * np.abs(expect).max()


def test_gpu_point_integrals_match_oracle(case):
    g, d, bvp, o = case
    rng = np.random.default_rng(11)
    phi, phin = rng.normal(size=bvp.matrix_size), rng.normal(size=bvp.matrix_size)
    a1, b1 = bvp.point_integrals(phi, phin)
    a2, b2 = o.point_integrals(phi, phin)
    assert np.abs(a1 - a2).max() <= 1e-12 * np.abs(a2).max()
    assert np.abs(b1 - b2).max() <= 1e-11 * np.abs(b2).max()


def test_gpu_solution_matches_reference(case):
    g, d, bvp, o = case
    kv = known_values(g.tank, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(g.tank))
    bvp.solve(kv)
    assert bvp.last_gmres_converged, bvp.last_gmres_residual_norm
    ref = g.solution(d)
    err = np.abs(bvp.ans - ref).max() / np.abs(ref).max()
    assert err <= 1e-10, err
    # known values pass through unchanged
    kind = d["dof_kind"]
    np.testing.assert_array_equal(bvp.phi[kind == 0], kv[kind == 0])
    np.testing.assert_array_equal(bvp.phin[kind != 0], kv[kind != 0])


@pytest.mark.parametrize("p", [1, 5, 12])
def test_gpu_matvec_matches_oracle_other_orders(product_lib, oracle_mod, p):
    t = make_tank(length=1.5, width=0.8, depth=0.4, h=0.1, noise_sigma=0.01, seed=2)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=p, dofs=d, fmm_bucket_max_points=12)
    bvp.setup()
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=p, max_points=12)
    rng = np.random.default_rng(p)
    phi, phin = rng.normal(size=bvp.matrix_size), rng.normal(size=bvp.matrix_size)
    np.testing.assert_allclose(bvp.diag(), o.compute_diag(), rtol=1e-11, atol=1e-11)
    got, exp = bvp.apply(phi, phin), o.apply(phi, phin)
    assert np.abs(got - exp).max() <= 1e-10 * np.abs(exp).max()


def test_gpu_single_bucket_mesh(product_lib, oracle_mod):
    """Coarse mesh: the whole surface sits in few buckets, no M2L at all."""
    t = make_tank(h=0.5)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=6, dofs=d, solver_tol=1e-12)
    bvp.setup()
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=6)
    kv = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    bvp.solve(kv)
    phi, phin, st = o.solve(kv, tol=1e-12)
    ref = np.where(d["dof_kind"] == 0, phin, phi)
    assert np.abs(bvp.ans - ref).max() <= 1e-9 * np.abs(ref).max()


def test_gpu_near_quadrature_block_beyond_shared_memory(product_lib, oracle_mod):
    """The whole surface in one bucket, so one near block holds every element: its element
    list, column offsets and incidence map (nf + ndof + 1.5 nf words) exceed the near-quadrature
    kernel's 70 KB of shared memory, and the kernel searches the block's element ranges per
    target instead.  Diagonal and operator against the oracle."""
    t = make_tank(h=0.04)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    nf, ndof = t.tri.shape[0], d["dof_point"].shape[0]
    assert (nf + ndof + 1.5 * nf) * 4 > 70 * 1024
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=4, dofs=d, fmm_bucket_max_points=100000)
    bvp.setup()
    assert bvp.tree_stats()["m2l_pairs"] == 0
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=4, max_points=100000)
    np.testing.assert_allclose(bvp.diag(), o.compute_diag(), rtol=1e-11, atol=1e-11)
    rng = np.random.default_rng(4)
    phi, phin = rng.normal(size=bvp.matrix_size), rng.normal(size=bvp.matrix_size)
    got, exp = bvp.apply(phi, phin), o.apply(phi, phin)
    assert np.abs(got - exp).max() <= 1e-10 * np.abs(exp).max()


def test_gpu_rejects_nonfinite_boundary_values(product_lib):
    t = make_tank(h=0.25)
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=4)
    bvp.setup()
    kv = np.zeros(bvp.matrix_size)
    kv[3] = np.inf
    with pytest.raises(RuntimeError):
        bvp.solve(kv)


@pytest.mark.slow
def test_gpu_full_size_properties(product_lib):
    """60k-node tank (p=10): rigid-mode rows vanish, the operator is linear, GMRES converges."""
    t = make_tank(h=2.0 / 185, noise_sigma=0.2 * 2.0 / 185, seed=1)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=10, dofs=d, solver_tol=1e-8, tol_relative=True,
                  preconditioner="jacobi")
    bvp.setup()
    n = bvp.matrix_size
    kind = d["dof_kind"]
    rows = bvp.apply(np.ones(n), np.zeros(n))  # phi = 1, phin = 0: every BIE row is 0 by the diagonal
    diag = bvp.diag()
    assert np.abs(rows[kind != 2]).max() <= 1e-12 * np.abs(diag).max()
    rng = np.random.default_rng(3)
    a, b = rng.normal(size=(2, n)), rng.normal(size=(2, n))
    lhs = bvp.apply(2.0 * a[0] - 0.5 * b[0], 2.0 * a[1] - 0.5 * b[1])
    rhs = 2.0 * bvp.apply(a[0], a[1]) - 0.5 * bvp.apply(b[0], b[1])
    assert np.abs(lhs - rhs).max() <= 1e-12 * np.abs(rhs).max()
    kv = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    bvp.solve(kv)
    assert bvp.last_gmres_converged
    assert np.isfinite(bvp.ans).all()


def test_gpu_tank_with_submerged_body_matches_oracle(product_lib, oracle_mod):
    """Two boundaries: the tank and a closed box inside the fluid (Neumann, rigid-body
    velocity), the floating-body configuration; operator and solution against the oracle."""
    from bem_for_nonlinear_waves_b200 import add_box_body
    t = make_tank(1.0, 0.5, 0.4, 0.05, amplitude=0.02, wavelength=0.7, noise_sigma=0.003, seed=4)
    t = add_box_body(t, (0.45, 0.25, -0.2), (0.2, 0.15, 0.1), 0.05, U=(0.1, 0.0, -0.05), Omega=(0.0, 0.3, 0.1))
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    kv = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    bvp = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=8, dofs=d, solver_tol=1e-12, solver_max_iter=1500)
    bvp.setup()
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=8)
    rng = np.random.default_rng(8)
    phi, phin = rng.normal(size=bvp.matrix_size), rng.normal(size=bvp.matrix_size)
    got, exp = bvp.apply(phi, phin), o.apply(phi, phin)
    assert np.abs(got - exp).max() <= 1e-10 * np.abs(exp).max()
    bvp.solve(kv)
    assert bvp.last_gmres_converged
    ph, pn, st = o.solve(kv, tol=1e-12, max_iter=1500)
    ref = np.where(d["dof_kind"] == 0, pn, ph)
    assert np.abs(bvp.ans - ref).max() <= 1e-8 * np.abs(ref).max()
