"""J2 material and Newton-Raphson increments on the GPU against the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PROPS = np.array([200000.0, 0.3, 250.0, 1000.0])


def test_material_batch_matches_oracle(pkg, orc):
    rng = np.random.default_rng(12)
    n = 257
    sig_n = rng.standard_normal((n, 6)) * 120
    de = rng.standard_normal((n, 6)) * 2e-3
    sdv_n = np.zeros((n, 7))
    sdv_n[:, 0] = np.abs(rng.standard_normal(n)) * 1e-3
    sdv_n[:, 1:] = rng.standard_normal((n, 6)) * 1e-4
    m = pkg.FemModel()
    s, v, D, y = m.mat_update_batch(pkg.MAT_J2_ISO, PROPS, sig_n, de, sdv_n)
    for i in range(n):
        so, eo, lo, Do, yo = orc.j2_update(PROPS, de[i], sig_n[i], sdv_n[i, 0], sdv_n[i, 1:])
        assert yo == y[i]
        np.testing.assert_allclose(s[i], so, rtol=0, atol=1e-12 * np.abs(so).max())
        assert abs(v[i, 0] - eo) <= 1e-15
        np.testing.assert_allclose(v[i, 1:], lo, rtol=0, atol=1e-15)
        np.testing.assert_allclose(D[i], Do, rtol=0, atol=1e-12 * np.abs(Do).max())
    assert 0 < y.sum() < n
    # ufc_core/Testing/test_defn_invoke_umat.f90: sigma11 = 282.69230769230769
    s, _, _, _ = m.mat_update_batch(pkg.MAT_ELASTIC_ISO, [210000.0, 0.3], np.zeros(6), [1e-3, 0, 0, 0, 0, 0])
    assert abs(s[0, 0] - 282.69230769230769) <= 1e-12 * 282.7


def _bar_model(pkg, p):
    m = pkg.FemModel.from_problem(p)
    return m


def test_nr_increments_match_oracle(pkg, orc):
    p = pkg.mesh.j2_bar(4, 2, 2)
    steps, strain = 6, 0.006
    targets = [pkg.mesh.j2_bar_target(p, s, n_steps=steps, strain=strain) for s in range(1, steps + 1)]
    hist, state, logs = orc.nr_j2(orc.Model(p), targets)
    m = _bar_model(pkg, p)
    for s, tgt in enumerate(targets):
        res = m.nr_increment(tgt, tolerance_force=1e-8, lin=pkg.SolverAlgo(tolerance=1e-12))
        assert res.converged and res.iterations <= 8
        m.commit()
        u = m.displacement()
        np.testing.assert_allclose(u, hist[s], rtol=0, atol=1e-8 * np.abs(hist[s]).max())
    epeq, sig, epl = m.j2_state()
    np.testing.assert_allclose(sig.reshape(-1, 6), state["sig"].reshape(-1, 6), rtol=0,
                               atol=1e-7 * np.abs(state["sig"]).max())
    np.testing.assert_allclose(epeq.ravel(), state["epeq"], rtol=1e-6)


def test_nr_increments_fp32_refined_inner_solves(pkg, orc):
    """FP32 CG on the tangent rounded from its FP64 assembly, refined with the
    FP64 tangent residual, reaches the same Newton iterates as the oracle."""
    p = pkg.mesh.j2_bar(6, 3, 3)
    steps, strain = 5, 0.006
    targets = [pkg.mesh.j2_bar_target(p, s, n_steps=steps, strain=strain) for s in range(1, steps + 1)]
    hist, state, _ = orc.nr_j2(orc.Model(p), targets)
    m = _bar_model(pkg, p)
    lin = pkg.SolverAlgo(tolerance=1e-12, precision_mode=pkg.PRECISION_FP32_REFINE)
    for s, tgt in enumerate(targets):
        res = m.nr_increment(tgt, tolerance_force=1e-8, lin=lin)
        assert res.converged and res.iterations <= 8
        m.commit()
        np.testing.assert_allclose(m.displacement(), hist[s], rtol=0, atol=1e-8 * np.abs(hist[s]).max())
    epeq, sig, _ = m.j2_state()
    np.testing.assert_allclose(sig.reshape(-1, 6), state["sig"].reshape(-1, 6), rtol=0,
                               atol=1e-7 * np.abs(state["sig"]).max())


def test_rollback_restores_committed_state(pkg):
    p = pkg.mesh.j2_bar(3, 2, 2)
    m = _bar_model(pkg, p)
    m.nr_increment(pkg.mesh.j2_bar_target(p, 1, n_steps=2, strain=0.004))
    m.commit()
    u1 = m.displacement().copy()
    e1 = m.j2_state()[0].copy()
    m.nr_increment(pkg.mesh.j2_bar_target(p, 2, n_steps=2, strain=0.004))
    assert not np.allclose(m.displacement(), u1)
    m.rollback()
    np.testing.assert_array_equal(m.displacement(), u1)
    np.testing.assert_array_equal(m.j2_state()[0], e1)  # committed state unchanged until commit


def test_j2_bar_64x32x32_uniaxial(pkg):
    # 20 displacement increments to 1 % strain; the exact solution is homogeneous
    # uniaxial stress with sigma = sy + E H/(E+H) (eps - sy/E) once yielded.
    p = pkg.mesh.config3()
    m = _bar_model(pkg, p)
    E, nu, sy, H = PROPS
    total_iters = 0
    for s in range(1, 21):
        res = m.nr_increment(pkg.mesh.j2_bar_target(p, s), tolerance_force=1e-8,
                             lin=pkg.SolverAlgo(tolerance=1e-10))
        assert res.converged, (s, res)
        total_iters += res.iterations
        m.commit()
    eps = 0.01
    sigma = sy + E * H / (E + H) * (eps - sy / E)
    epeq, sig, _ = m.j2_state()
    np.testing.assert_allclose(sig[..., 0], sigma, rtol=1e-6)
    assert np.abs(sig[..., 1:]).max() <= 1e-5 * sigma
    np.testing.assert_allclose(epeq, (eps - sy / E) * E / (E + H), rtol=1e-5)
    # reaction on the pulled face equals sigma * area
    u = m.displacement()
    fint, _, _, _ = m.internal_force(u, update_state=False)
    pull = p.fixed[p.meta["pull_dofs"]]
    area = p.shape[1] * p.shape[2]
    assert abs(fint[pull].sum() - sigma * area) <= 1e-6 * sigma * area
    assert total_iters <= 20 * 6
