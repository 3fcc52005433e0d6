"""Geometric multigrid preconditioner (ufc_mg_setup) on the GPU: the Galerkin
coarse operators against P^T A P formed with scipy from the oracle's matrix,
symmetry and positivity of the V-cycle, and MG-PCG solutions against
Jacobi-PCG (linear elastic and J2 tangent)."""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


def _prolongation(nxc, nyc, nzc, fixed_f, fixed_c):
    """Trilinear P from the (nxc, nyc, nzc) box to the box twice as fine, zero
    at fixed fine rows and fixed coarse columns."""
    nxf, nyf, nzf = 2 * nxc, 2 * nyc, 2 * nzc
    rows, cols, vals = [], [], []
    par = lambda i: [(i // 2, 1.0)] if i % 2 == 0 else [(i // 2, 0.5), (i // 2 + 1, 0.5)]  # noqa: E731
    for k in range(nzf + 1):
        for j in range(nyf + 1):
            for i in range(nxf + 1):
                f = i + (nxf + 1) * (j + (nyf + 1) * k)
                for K, wk in par(k):
                    for J, wj in par(j):
                        for I, wi in par(i):
                            c = I + (nxc + 1) * (J + (nyc + 1) * K)
                            for d in range(3):
                                if not fixed_f[3 * f + d] and not fixed_c[3 * c + d]:
                                    rows.append(3 * f + d)
                                    cols.append(3 * c + d)
                                    vals.append(wi * wj * wk)
    nf, nc = 3 * (nxf + 1) * (nyf + 1) * (nzf + 1), 3 * (nxc + 1) * (nyc + 1) * (nzc + 1)
    return sp.csr_matrix((vals, (rows, cols)), shape=(nf, nc))


def _coarse_fixed(fixed_f, nxc, nyc, nzc):
    nxf, nyf = 2 * nxc, 2 * nyc
    out = np.zeros(3 * (nxc + 1) * (nyc + 1) * (nzc + 1), dtype=bool)
    for k in range(nzc + 1):
        for j in range(nyc + 1):
            for i in range(nxc + 1):
                c = i + (nxc + 1) * (j + (nyc + 1) * k)
                f = 2 * i + (nxf + 1) * (2 * j + (nyf + 1) * 2 * k)
                out[3 * c:3 * c + 3] = fixed_f[3 * f:3 * f + 3]
    return out


def _dense(rp, col, val, n):
    return sp.csr_matrix((val, col, rp), shape=(n, n)).toarray()


def _eliminated(Am, fixed):
    A = np.array(Am, dtype=np.float64)
    A[fixed, :] = 0.0
    A[:, fixed] = 0.0
    A[fixed, fixed] = 1.0
    return A


def test_galerkin_coarse_operators(pkg, orc):
    n = 4
    E = pkg.mesh.lognormal_moduli(n ** 3, seed=3)
    p = pkg.mesh.cantilever(n, n, n, float(n), float(n), float(n), E=E)
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    levels, cdof, _ = m.mg_setup(n, n, n, coarse_max=1)
    assert levels == 3 and cdof == 3 * 8
    A0 = orc.Model(p).assemble(eliminate=False)
    A = sp.csr_matrix((A0.val, A0.col, A0.row_ptr), shape=(p.n_dof, p.n_dof))
    fixed = np.zeros(p.n_dof, dtype=bool)
    fixed[p.fixed] = True
    # level 0 is the assembled matrix
    rp, col, val = m.mg_export(0)
    np.testing.assert_allclose(_dense(rp, col, val, p.n_dof), _eliminated(A.toarray(), fixed), rtol=0,
                               atol=1e-12 * abs(A).max())
    Af, ff, nc = A, fixed, n
    for lev in (1, 2):
        nc //= 2
        fc = _coarse_fixed(ff, nc, nc, nc)
        P = _prolongation(nc, nc, nc, ff, fc)
        Ac = (P.T @ Af @ P).toarray()
        rp, col, val = m.mg_export(lev)
        got = _dense(rp, col, val, Ac.shape[0])
        np.testing.assert_allclose(got, _eliminated(Ac, fc), rtol=0, atol=1e-12 * np.abs(Ac).max())
        # the pattern of the coarse level is the box pattern
        rpo, colo = orc.csr_pattern((nc + 1) ** 3, pkg.mesh.box_mesh(nc, nc, nc, 1.0, 1.0, 1.0)[1])
        assert np.array_equal(rp, rpo) and np.array_equal(col, colo)
        Af = sp.csr_matrix(Ac)  # the next level multiplies the masked, uneliminated operator
        ff = fc


def test_vcycle_symmetric_positive(pkg):
    p = pkg.mesh.lognormal_cantilever(8, 4, 4, seed=6)
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    m.mg_setup(8, 4, 4, coarse_max=30)
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal(p.n_dof), rng.standard_normal(p.n_dof)
    Ma, Mb = m.mg_apply(a), m.mg_apply(b)
    assert abs(a @ Mb - b @ Ma) <= 1e-11 * abs(a @ Mb)
    assert a @ Ma > 0 and b @ Mb > 0
    np.testing.assert_array_equal(m.mg_apply(a), Ma)  # deterministic


@pytest.mark.parametrize("storage", ["full", "symmetric"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name,make,dims", [
    ("cantilever_40x8x8", lambda mesh: mesh.config1(), (40, 8, 8)),
    ("lognormal_32x16x16", lambda mesh: mesh.lognormal_cantilever(32, 16, 16, seed=2), (32, 16, 16)),
])
def test_mg_pcg_matches_jacobi(pkg, orc, name, make, dims, precision, storage):
    """FP64 PCG around the V-cycle, the cycle in FP64 or FP32: the answer has
    the FP64 residual either way.  With symmetric storage the finest level's
    products (outer PCG, smoother, residual) take the half storage."""
    p = make(pkg.mesh)
    m = pkg.FemModel.from_problem(p)
    sym = pkg.BUILD_FP32_ROUNDED | pkg.BUILD_SYMMETRIC if storage == "symmetric" else 0
    m.assemble(pkg.BUILD_FP64 | sym)
    prec = pkg.PRECISION_FP64 if precision == "fp64" else pkg.PRECISION_FP32_REFINE
    levels, cdof, _ = m.mg_setup(*dims, precision=prec)
    assert levels >= 3
    b = pkg.lifted_rhs(m, p.f)
    if sym:
        # the cycle on the half storage is the cycle on the full storage, up to
        # the order of the row sums
        f = pkg.FemModel.from_problem(p)
        f.assemble(pkg.BUILD_FP64)
        f.mg_setup(*dims, precision=prec)
        r = np.random.default_rng(3).standard_normal(p.n_dof)
        zs, zf = m.mg_apply(r), f.mg_apply(r)
        np.testing.assert_allclose(zs, zf, rtol=0, atol=(1e-11 if precision == "fp64" else 1e-4) * np.abs(zf).max())
        f.close()
    xj, sj = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    xm, sm = m.solve(b, pkg.SolverAlgo(tolerance=1e-10, precond_type=pkg.SOLV_PREC_MG))
    assert sm.converged and sm.rnorm <= 1e-10
    # the residual of the multigrid solution with the oracle's matrix
    K = orc.Model(p).assemble()
    assert np.linalg.norm(b - K.matvec(xm)) <= 2e-10 * np.linalg.norm(b)
    # both solutions meet rtol 1e-10; they agree to the conditioning of K
    assert np.linalg.norm(xm - xj) <= 1e-6 * np.linalg.norm(xj)
    assert sm.niter * 8 <= sj.niter, (sm.niter, sj.niter)


def test_mg_on_j2_tangent(pkg):
    p = pkg.mesh.j2_bar(8, 4, 4)
    m = pkg.FemModel.from_problem(p)
    for s in (1, 2, 3):
        assert m.nr_increment(pkg.mesh.j2_bar_target(p, s, n_steps=3, strain=0.006)).converged
        m.commit()
    # the tangent of the committed plastic state, and a right-hand side on the free DOFs
    u = m.displacement()
    m.internal_force(u, update_state=True)
    m.assemble(pkg.BUILD_FP64)
    m.mg_setup(8, 4, 4, coarse_max=30)
    b = np.random.default_rng(4).standard_normal(p.n_dof)
    b[p.fixed] = 0.0
    xj, _ = m.solve(b, pkg.SolverAlgo(tolerance=1e-12))
    xm, sm = m.solve(b, pkg.SolverAlgo(tolerance=1e-10, precond_type=pkg.SOLV_PREC_MG))
    assert sm.converged
    assert np.linalg.norm(xm - xj) <= 1e-9 * np.linalg.norm(xj)


def test_mg_follows_reassembly(pkg):
    """After a reassembly with new moduli the hierarchy's numbers are rebuilt on
    the next multigrid solve (same boxes and patterns)."""
    p = pkg.mesh.lognormal_cantilever(16, 8, 8, seed=6)
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    m.mg_setup(16, 8, 8, coarse_max=100)
    b = pkg.lifted_rhs(m, p.f)
    mg = pkg.SolverAlgo(tolerance=1e-10, precond_type=pkg.SOLV_PREC_MG)
    x1, s1 = m.solve(b, mg)
    props = p.props.copy()
    props[:, 0] *= np.random.default_rng(9).uniform(0.5, 2.0, p.n_elems)
    m.set_material(p.mat_model_id, props)
    m.assemble(pkg.BUILD_FP64)
    x2, s2 = m.solve(b, mg)
    xj, _ = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    assert s1.converged and s2.converged and s2.niter <= 2 * s1.niter + 5
    assert np.linalg.norm(x2 - xj) <= 1e-6 * np.linalg.norm(xj)
    assert np.linalg.norm(x2 - x1) > 1e-3 * np.linalg.norm(x1)


def test_nr_increments_with_mg(pkg, orc):
    """Newton increments whose tangent solves use the multigrid preconditioner
    (the hierarchy follows every tangent reassembly) reach the oracle's iterates."""
    p = pkg.mesh.j2_bar(8, 4, 4)
    steps, strain = 4, 0.006
    targets = [pkg.mesh.j2_bar_target(p, s, n_steps=steps, strain=strain) for s in range(1, steps + 1)]
    hist, state, _ = orc.nr_j2(orc.Model(p), targets)
    m = pkg.FemModel.from_problem(p)
    m.internal_force(m.displacement(), update_state=True)
    m.assemble(pkg.BUILD_FP64)
    m.mg_setup(8, 4, 4, coarse_max=30)
    lin = pkg.SolverAlgo(tolerance=1e-12, precond_type=pkg.SOLV_PREC_MG)
    for s, tgt in enumerate(targets):
        res = m.nr_increment(tgt, tolerance_force=1e-8, lin=lin)
        assert res.converged and res.iterations <= 8
        m.commit()
        np.testing.assert_allclose(m.displacement(), hist[s], rtol=0, atol=1e-9 * np.abs(hist[s]).max())
        assert res.lin_iters_total <= 40 * max(res.iterations, 1)


def test_mg_errors(pkg):
    p = pkg.mesh.lognormal_cantilever(8, 4, 4, seed=6)
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    with pytest.raises(pkg.UfcError) as ei:
        m.mg_setup(4, 8, 4)  # not this box's numbering
    assert ei.value.status_code == 1
    q = pkg.mesh.unit_cube_uniaxial()
    m1 = pkg.FemModel.from_problem(q)
    m1.assemble(pkg.BUILD_FP64)
    with pytest.raises(pkg.UfcError):
        m1.mg_setup(1, 1, 1)  # cannot be coarsened
