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
        np.testing.assert_allclose(u, hist[s], rtol=0, atol=1e-9 * np.abs(hist[s]).max())
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
    lin = pkg.SolverAlgo(tolerance=1e-12, precision_mode=pkg.PRECISION_FP32_REFINE,
                         refine_policy=pkg.REFINE_FORCE_FP32)
    for s, tgt in enumerate(targets):
        res = m.nr_increment(tgt, tolerance_force=1e-8, lin=lin)
        assert res.converged and res.iterations <= 8
        m.commit()
        np.testing.assert_allclose(m.displacement(), hist[s], rtol=0, atol=1e-9 * np.abs(hist[s]).max())
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


def _step_kw(**kw):
    base = dict(dt_min=1e-3, max_cutbacks=6, growth_factor=1.25, cutback_factor=0.5, target_iters=6,
                growth_threshold=0.8)
    base.update(kw)
    return base


def _compare_history(res, ref, iters_slack=0):
    assert len(res.history) == len(ref["history"])
    for (t, dt, it, ok), (t_o, dt_o, it_o, ok_o) in zip(res.history, ref["history"]):
        assert ok == ok_o and abs(it - it_o) <= iters_slack, ((t, dt, it, ok), (t_o, dt_o, it_o, ok_o))
        assert t == t_o and dt == dt_o  # the same IEEE operations on the same decisions


@pytest.mark.parametrize("max_iter,dt0,max_inc", [(2, 1.0, 60)])
def test_step_driver_history_matches_oracle(pkg, orc, max_iter, dt0, max_inc):
    """RT_StepDriver increment control: cutbacks after non-converged increments,
    growth after easy ones; the attempt history (time, dt, Newton iterations,
    converged) equals the oracle's.  With two Newton iterations an increment
    converges exactly when it stays elastic (one predictor solve) and fails when
    it crosses the yield point, so every decision is clear of the force
    tolerance; the histories must agree entry for entry."""
    p = pkg.mesh.j2_bar(4, 2, 2)
    u_end = pkg.mesh.j2_bar_target(p, 1, n_steps=1, strain=0.0107)
    kw = _step_kw(dt_initial=dt0, max_increments=max_inc)
    ref = orc.step_j2(orc.Model(p), u_end, max_iter=max_iter, lin_rtol=1e-12, **kw)
    m = _bar_model(pkg, p)
    res = m.nr_step(u_end, max_iterations=max_iter, lin=pkg.SolverAlgo(tolerance=1e-12), **kw)
    assert res.cutbacks == ref["cutbacks"] >= 3
    assert res.increments == ref["increments"] and res.attempts == ref["attempts"]
    assert not res.completed and res.status == pkg.STATUS_NOT_CONVERGED
    _compare_history(res, ref)
    # the context holds the last converged increment
    np.testing.assert_allclose(m.displacement(), ref["u"], rtol=0, atol=1e-8 * np.abs(ref["u"]).max())
    assert res.final_time == ref["final_time"]


def test_step_driver_completes_to_analytic_state(pkg, orc):
    p = pkg.mesh.j2_bar(4, 2, 2)
    strain = 0.01
    u_end = pkg.mesh.j2_bar_target(p, 1, n_steps=1, strain=strain)
    kw = _step_kw(dt_initial=0.05, dt_max=0.2, max_increments=80)
    m = _bar_model(pkg, p)
    res = m.nr_step(u_end, max_iterations=8, lin=pkg.SolverAlgo(tolerance=1e-12), **kw)
    ref = orc.step_j2(orc.Model(p), u_end, max_iter=8, lin_rtol=1e-12, **kw)
    assert res.completed and ref["completed"] and res.final_time == 1.0
    # plastic increments take 3 Newton iterations, or 4 when the third residual
    # lands within rounding of the force tolerance; dt grows either way
    _compare_history(res, ref, iters_slack=1)
    E, nu, sy, H = PROPS
    sigma = sy + E * H / (E + H) * (strain - sy / E)
    _, sig, _ = m.j2_state()
    np.testing.assert_allclose(sig[..., 0], sigma, rtol=1e-6)
    # every converged increment was committed: a rollback keeps the end-of-step state
    m.rollback()
    np.testing.assert_allclose(m.j2_state()[1][..., 0], sigma, rtol=1e-6)


def test_step_driver_elastic_growth(pkg):
    """Easy increments grow dt by 1.25 up to dt_max; the prescribed values
    reach their end values exactly."""
    p = pkg.mesh.j2_bar(3, 2, 2, sy=1e9)
    u_end = pkg.mesh.j2_bar_target(p, 1, n_steps=1, strain=0.001)
    m = _bar_model(pkg, p)
    res = m.nr_step(u_end, dt_initial=0.1, dt_max=0.3, max_increments=20, max_iterations=4,
                    lin=pkg.SolverAlgo(tolerance=1e-12))
    assert res.completed and res.cutbacks == 0
    dts = [h[1] for h in res.history]
    exp, t, dt = [], 0.0, 0.1
    while t < 1.0 - 1e-12:
        dt = min(dt, 1.0 - t)
        exp.append(dt)
        t += dt
        dt = min(dt * 1.25, 0.3)
    assert dts == exp
    u = m.displacement()
    np.testing.assert_array_equal(u[p.fixed], u_end)
