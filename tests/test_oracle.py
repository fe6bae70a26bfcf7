"""The oracle (CPU restatement) against the compiled reference's golden outputs and
against direct summation.  CPU only."""
import numpy as np
import pytest

from bem_for_nonlinear_waves_b200 import build_dofs, make_tank, known_values, point_normals
import goldens

GOLDEN_NAMES = goldens.names()


@pytest.fixture(scope="module", params=GOLDEN_NAMES)
def golden_case(request, oracle_mod):
    g = goldens.Golden(request.param)
    t = g.tank
    d = oracle_mod.build_dofs(t.X, t.tri, t.face_dirichlet)
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=g.p)
    return g, d, o


def test_goldens_present():
    assert len(GOLDEN_NAMES) >= 2


def test_oracle_tree_matches_reference(golden_case):
    g, d, o = golden_case
    lv, corner = o.face_leaf()
    fl = g.z["face_leaf"]
    f = fl[:, 0].astype(int)
    np.testing.assert_array_equal(lv[f], fl[:, 1].astype(int))
    np.testing.assert_array_equal(corner[f], fl[:, 2:5])


def test_oracle_near_rows_match_reference(golden_case):
    g, d, o = golden_case
    _, ours = g.maps(d)
    z = g.z
    for i, p in enumerate(z["near_points"]):
        idx, wg, wgn = o.near_row(p)
        assert len(idx) == z["near_count"][i]
        np.testing.assert_allclose(wg.sum(), z["near_sum_g"][i], rtol=1e-11, atol=1e-14)
        np.testing.assert_allclose(np.abs(wg).sum(), z["near_sumabs_g"][i], rtol=1e-11)
        np.testing.assert_allclose(wgn.sum(), z["near_sum_gn"][i], rtol=1e-11, atol=1e-11 * np.abs(wgn).sum())
    off = z["sample_off"]
    for k, p in enumerate(z["sample_points"]):
        ridx = ours[z["sample_idx"][off[k]:off[k + 1]]]
        srt = np.argsort(ridx)
        idx, wg, wgn = o.near_row(p)
        np.testing.assert_array_equal(idx, ridx[srt])
        sc = np.abs(wg).max()
        np.testing.assert_allclose(wg, z["sample_g"][off[k]:off[k + 1]][srt], rtol=0, atol=1e-11 * sc)
        np.testing.assert_allclose(wgn, z["sample_gn"][off[k]:off[k + 1]][srt], rtol=0, atol=1e-11 * np.abs(wgn).max())


def test_oracle_diag_matches_reference(golden_case):
    g, d, o = golden_case
    np.testing.assert_allclose(o.compute_diag(), g.diag(d), rtol=1e-13, atol=1e-13)


def test_oracle_matvec_matches_reference(golden_case):
    g, d, o = golden_case
    phi, phin, expect = g.matvec_input(d)
    got = o.apply(phi, phin)
    assert np.abs(got - expect).max() <= 2e-12 * np.abs(expect).max()


@pytest.mark.slow
def test_oracle_solution_matches_reference(golden_case):
    g, d, o = golden_case
    if g.tank.X.shape[0] > 1000:
        # the 2,802-point golden takes the CPU oracle ~6 minutes (it passes at 1e-10); the CPU
        # suite keeps to the small tanks and the GPU parity tests cover every golden
        pytest.skip("large golden: solution parity checked by the GPU tests")
    kv = known_values(g.tank, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(g.tank))
    phi, phin, st = o.solve(kv, tol=g.tol, max_iter=1000)
    assert st["converged"]
    sol = np.where(d["dof_kind"] == 0, phin, phi)
    ref = g.solution(d)
    assert np.abs(sol - ref).max() <= 1e-10 * np.abs(ref).max()


@pytest.mark.parametrize("p,bound", [(4, 2e-4), (8, 5e-9), (12, 5e-12)])
def test_oracle_fmm_vs_direct(oracle_mod, p, bound):
    """Regenerated G&R translation tables: FMM far field vs direct summation over the same
    P2M points; error falls with p."""
    t = make_tank(h=0.1)
    d = oracle_mod.build_dofs(t.X, t.tri, t.face_dirichlet)
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=p, max_points=8)
    rng = np.random.default_rng(5)
    phi, phin = rng.normal(size=o.ndof), rng.normal(size=o.ndof)
    a, b = o.point_integrals(phi, phin)
    ad, bd = o.point_integrals(phi, phin, direct=True)
    assert np.abs(a - ad).max() <= bound * np.abs(ad).max()
    assert np.abs(b - bd).max() <= 10 * bound * np.abs(bd).max()


def test_oracle_rigid_mode_solid_angles(oracle_mod):
    """diag = -int dG/dn over the closed surface = interior solid angle: 2 pi on faces,
    pi on edges, pi/2 at box corners."""
    t = make_tank(h=0.1)
    d = oracle_mod.build_dofs(t.X, t.tri, t.face_dirichlet)
    o = oracle_mod.Oracle(t.X, t.tri, t.face_dirichlet, d, p=8)
    diag = o.compute_diag()
    X = t.X[d["dof_point"]]
    on = [np.isclose(X[:, 0], 0) | np.isclose(X[:, 0], t.length), np.isclose(X[:, 1], 0) | np.isclose(X[:, 1], t.width),
          np.isclose(X[:, 2], 0) | np.isclose(X[:, 2], -t.depth)]
    nb = sum(a.astype(int) for a in on)
    for k, ang in ((1, 2 * np.pi), (2, np.pi), (3, np.pi / 2)):
        np.testing.assert_allclose(diag[nb == k], ang, rtol=2e-3)  # quadrature error of the discrete operator
