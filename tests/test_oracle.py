"""The FP64 oracle against the reference's known answers and golden vectors (CPU)."""
import json
import os

import numpy as np
import pytest

from oracle import np_oracle as N

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KA = json.load(open(os.path.join(GOLD, "known_answers.json")))
REG = json.load(open(os.path.join(GOLD, "oracle_regression.json")))


def test_umat_elastic_282(orc):
    k = KA["umat_elastic_uniaxial_strain"]
    props = [k["props"][0], k["props"][1], 1e300, 0.0]
    s, _, _, D, y = orc.j2_update(props, k["dstrain"])
    assert not y
    assert abs(s[0] - k["sigma11"]) <= 1e-12 * k["sigma11"]  # reference tolerance 1e-5


def test_unit_cube_uniaxial(pkg, orc):
    k = KA["c3d8_unit_cube_uniaxial"]
    p = pkg.mesh.unit_cube_uniaxial(k["E"], k["nu"], k["sigma"])
    u, info = orc.Model(p).solve_linear(rtol=1e-15)
    a = p.conn[0]
    np.testing.assert_allclose(u[3 * a[[1, 2, 5, 6]]], k["u_x_face"], rtol=1e-12)
    np.testing.assert_allclose(u[3 * a[[2, 3, 6, 7]] + 1], k["u_y_face"], rtol=1e-10)


def test_j2_uniaxial_history(orc):
    k = KA["j2_uniaxial_history"]
    E, nu, sy, H = k["props"]
    sig, ep, epl, prev = np.zeros(6), 0.0, np.zeros(6), np.zeros(6)
    for e in k["eps11"]:
        tot = np.array([e, -nu * e, -nu * e, 0, 0, 0])
        sig, ep, epl, D, y = orc.j2_update(k["props"], tot - prev, sig, ep, epl)
        prev = tot
        if e <= sy / E:
            assert not y and ep == 0.0
            assert abs(sig[0] - E * e) <= 1e-12 * E * e
        else:
            assert y and ep > 0.0
            assert abs(orc.von_mises(sig) - (sy + H * ep)) <= 1e-10 * sy
    assert 0.0 < ep < k["eps11"][-1]


def test_perfect_plasticity(orc):
    k = KA["perfect_plasticity"]
    s, ep, epl, D, y = orc.j2_update(k["props"], [0.01, -0.002, 0.001, 0.004, -0.003, 0.002])
    assert y
    assert abs(orc.von_mises(s) - k["props"][2]) <= k["q_tol"]
    p = (s[0] + s[1] + s[2]) / 3
    st, *_ = orc.j2_update(k["props"][:2] + [1e300, 0.0], [0.01, -0.002, 0.001, 0.004, -0.003, 0.002])
    assert abs(p - (st[0] + st[1] + st[2]) / 3) <= 1e-12 * abs(p)  # hydrostatic stress preserved
    assert abs(np.sum(epl[:3])) <= 1e-15  # plastic flow is isochoric


def test_j2_consistent_tangent_fd(orc):
    props = [200000.0, 0.3, 250.0, 1000.0]
    rng = np.random.default_rng(4)
    for trial in range(5):
        sig_n = rng.standard_normal(6) * 50
        deps = rng.standard_normal(6) * 2e-3
        s0, _, _, Dep, y = orc.j2_update(props, deps, sig_n, 0.001)
        h = 1e-8
        Dfd = np.zeros((6, 6))
        for j in range(6):
            dp, dm = deps.copy(), deps.copy()
            dp[j] += h
            dm[j] -= h
            Dfd[:, j] = (orc.j2_update(props, dp, sig_n, 0.001)[0] - orc.j2_update(props, dm, sig_n, 0.001)[0]) / (2 * h)
        assert np.abs(Dfd - Dep).max() <= KA["fd_tangent"]["rel_tol"] * 1e-3 * np.abs(Dep).max()


def test_j2_tensor_form_agrees(orc):
    props = REG["j2_mixed_history"]["props"]
    sig, ep, prev = np.zeros(6), 0.0, np.zeros(6)
    epl = np.zeros(6)
    for st in REG["j2_mixed_history"]["steps"]:
        tot = np.array(st["strain"])
        s, e2, l2, D, y = orc.j2_update(props, tot - prev, sig, ep, epl)
        s_t, e_t = N.j2_tensor(props, tot - prev, sig, ep)
        np.testing.assert_allclose(s, st["sigma"], rtol=0, atol=1e-12 * np.abs(st["sigma"]).max())
        np.testing.assert_allclose(s, s_t, rtol=0, atol=1e-9 * np.abs(s).max())
        assert abs(e2 - st["epeq"]) <= 1e-15 and abs(e2 - e_t) <= 1e-15
        sig, ep, epl, prev = s, e2, l2, tot


def test_ke_against_numpy_and_golden(orc):
    g = REG["ke_distorted_hex"]
    X = np.array(g["X"])
    D = N.iso_D(g["E"], g["nu"])
    K = orc.c3d8_ke(X, D)
    np.testing.assert_allclose(K, np.array(g["Ke"]), rtol=0, atol=1e-12 * np.abs(K).max())
    np.testing.assert_allclose(K, N.ke(X, D), rtol=0, atol=1e-12 * np.abs(K).max())


def test_ke_patch_properties(orc):
    # tests/HARNESS_Elem_C3D8_PatchTest.f90: symmetry, non-negative diagonal, rigid-body null space
    X = np.array(REG["ke_distorted_hex"]["X"])
    K = orc.c3d8_ke(X, N.iso_D(1.0, 0.3))
    scale = np.abs(K).max()
    assert np.abs(K - K.T).max() <= 1e-14 * scale
    assert np.all(np.diag(K) > 0)
    modes = []
    for d in range(3):
        t = np.zeros((8, 3))
        t[:, d] = 1
        modes.append(t.ravel())
    for axis in range(3):
        w = np.zeros(3)
        w[axis] = 1
        modes.append(np.cross(w, X).ravel())
    for mvec in modes:
        assert np.abs(K @ mvec).max() <= 1e-12 * scale * np.abs(mvec).max()
    eig = np.linalg.eigvalsh(K)
    assert np.sum(eig < 1e-10 * eig.max()) == 6  # exactly the six rigid-body modes
    # patch test: a linear field gives constant strain and zero internal work error
    A = np.array([[1e-3, 2e-4, -1e-4], [3e-4, -5e-4, 2e-4], [-2e-4, 1e-4, 4e-4]])
    u = (X @ A.T).ravel()
    for ip in range(8):
        xi = N.GAUSS[ip]
        dN = N.shape_grad(xi)
        J = dN.T @ X
        dNx = (np.linalg.inv(J) @ dN.T).T
        eps = N.bmat(dNx) @ u
        exact = [A[0, 0], A[1, 1], A[2, 2], A[0, 1] + A[1, 0], A[1, 2] + A[2, 1], A[2, 0] + A[0, 2]]
        np.testing.assert_allclose(eps, exact, rtol=0, atol=1e-15)


def test_pattern_and_assembly_golden(pkg, orc):
    g = REG["cantilever_3x2x2"]
    p = pkg.mesh.cantilever(3, 2, 2, 3.0, 2.0, 2.0, E=np.linspace(1e3, 5e3, 12))
    m = orc.Model(p)
    assert np.array_equal(m.row_ptr, np.array(g["row_ptr"]))
    assert np.array_equal(m.col, np.array(g["col"]))
    K = m.assemble()
    np.testing.assert_allclose(K.val, np.array(g["val"]), rtol=0, atol=1e-12 * np.abs(K.val).max())
    A = K.to_dense()
    assert np.abs(A - A.T).max() <= 1e-14 * np.abs(A).max()
    u, info = m.solve_linear(rtol=1e-14)
    np.testing.assert_allclose(u, np.array(g["u"]), rtol=0, atol=1e-12 * np.abs(u).max())
    # against a dense FP64 solve
    u_dense = np.linalg.solve(A, m.lifted_rhs())
    assert np.abs(u - u_dense).max() <= 1e-11 * np.abs(u_dense).max()


def test_pattern_is_canonical(pkg, orc):
    # sorted unique columns per row; every element pair coupled; symmetric pattern
    p = pkg.mesh.lognormal_cantilever(5, 3, 4, seed=1)
    rp, col = orc.csr_pattern(p.n_nodes, p.conn)
    n = p.n_dof
    for i in range(0, n, 7):
        c = col[rp[i]:rp[i + 1]]
        assert np.all(np.diff(c) > 0)
    S = set()
    for e in p.conn:
        for a in e:
            for b in e:
                S.add((a, b))
    assert len(S) * 9 == col.size
    # structured-hex count: nnzb = prod(3 n_i - 2) over node counts
    nn = np.array([6, 4, 5])
    assert col.size == 9 * np.prod(3 * nn - 2)


def test_fint_equals_K_u(pkg, orc):
    p = pkg.mesh.lognormal_cantilever(4, 3, 3, seed=2)
    m = orc.Model(p)
    p_nobc = pkg.mesh.Problem(p.name, p.shape, p.coords, p.conn, p.mat_model_id, p.props,
                              np.zeros(0, np.int32), np.zeros(0), p.f)
    m0 = orc.Model(p_nobc)
    K = m0.assemble()
    u = np.random.default_rng(3).standard_normal(p.n_dof)
    np.testing.assert_allclose(m0.fint_elastic(u), K.matvec(u), rtol=0, atol=1e-12 * np.abs(K.matvec(u)).max())
    assert m.ncol == 8


def test_nr_j2_homogeneous_bar(pkg, orc):
    # uniaxial bar under displacement control: the exact solution is homogeneous
    p = pkg.mesh.j2_bar(4, 2, 2)
    model = orc.Model(p)
    steps = 6
    targets = [pkg.mesh.j2_bar_target(p, s, n_steps=steps, strain=0.006) for s in range(1, steps + 1)]
    hist, state, logs = orc.nr_j2(model, targets)
    E, nu, sy, H = p.props[0]
    eps = 0.006
    Et = E * H / (E + H)
    sigma_exact = sy + Et * (eps - sy / E)
    # the Newton tolerance (1e-8 on the force residual) bounds the stress error
    sig = state["sig"].reshape(-1, 6)
    np.testing.assert_allclose(sig[:, 0], sigma_exact, rtol=1e-7)
    assert np.abs(sig[:, 1:]).max() <= 1e-7 * sigma_exact
    epeq = state["epeq"]
    np.testing.assert_allclose(epeq, (eps - sy / E) * E / (E + H), rtol=1e-6)
    assert all(len(lg) <= 6 for lg in logs)


def test_face_loads_restatements_agree(pkg):
    """np_oracle.face_loads (3-D shape functions on the face, normal oriented
    from the centroid) against mesh.face_traction (bilinear face) on the
    cantilever end face, and the face-id table against the six box faces."""
    from oracle import np_oracle as NO

    p = pkg.mesh.config1()
    nx, ny, nz = p.shape
    e = pkg.mesh._face_elems(nx, ny, nz, "xmax")
    f = NO.face_loads(p.coords, p.conn, e, np.full(e.size, 6), np.tile([0.0, 0.0, -1.0], (e.size, 1)))
    np.testing.assert_allclose(f, p.f, rtol=0, atol=1e-15)
    X = NO.SIGNS * 0.5 + 0.5  # unit cube
    want = {1: [0, 0, 1], 2: [0, 0, -1], 3: [0, 1, 0], 4: [0, -1, 0], 5: [1, 0, 0], 6: [-1, 0, 0]}
    for fid, w in want.items():  # unit pressure pushes into the element
        np.testing.assert_allclose(NO.face_load(X, fid, pressure=1.0).sum(axis=0), w, atol=1e-15)


def test_extrapolation_matrix_closed_form():
    from oracle import np_oracle as NO

    Ex = NO.extrap_matrix()
    r3 = np.sqrt(3.0)
    closed = np.array([[np.prod([(1 + r3 * NO.SIGNS[a, d] * np.sign(NO.GAUSS[ip, d])) / 2 for d in range(3)])
                        for ip in range(8)] for a in range(8)])
    np.testing.assert_allclose(Ex, closed, rtol=0, atol=1e-14)
    np.testing.assert_allclose(Ex.sum(axis=1), 1.0, atol=1e-14)  # constants are reproduced
    s, vm = NO.nodal_stress(3 * 3 * 3, np.array([[0, 1, 4, 3, 9, 10, 13, 12]]), np.tile([1, 2, 3, 0, 0, 0.5], (1, 8, 1)))
    np.testing.assert_allclose(s[[0, 1, 4, 3, 9, 10, 13, 12]], np.tile([1, 2, 3, 0, 0, 0.5], (8, 1)), atol=1e-14)


def test_oracle_step_driver_growth_sequence(pkg, orc):
    """Elastic increments converge in one Newton iteration, so dt grows by the
    growth factor up to dt_max and the last increment is clipped at the end."""
    p = pkg.mesh.j2_bar(2, 1, 1, sy=1e9)
    u_end = pkg.mesh.j2_bar_target(p, 1, n_steps=1, strain=0.001)
    r = orc.step_j2(orc.Model(p), u_end, dt_initial=0.1, dt_max=0.3, max_increments=20)
    assert r["completed"] and r["cutbacks"] == 0
    dts = [h[1] for h in r["history"]]
    exp, t, dt = [], 0.0, 0.1
    while t < 1.0 - 1e-12:
        dt = min(dt, 1.0 - t)
        exp.append(dt)
        t += dt
        dt = min(dt * 1.25, 0.3)
    assert dts == exp and all(h[2] == 1 for h in r["history"])
    np.testing.assert_array_equal(r["u"][p.fixed], u_end)


def _penalty_solution(p, K_full):
    """The reference's Dirichlet treatment: penalty on the diagonal of the
    unreduced stiffness and penalty * value on the load
    (RT_Asm_ApplyBC_Displacement_Penalty, ufc_core/L5_RT/Assembly/
    RT_Asm_Solv.f90:427-483, with penalty = 1e20 max|K_ii| as
    RT_Asm_Core_Apply_BC, RT_Asm_Core.f90:265-274), solved directly."""
    sp = pytest.importorskip("scipy.sparse")
    spla = pytest.importorskip("scipy.sparse.linalg")
    A = sp.csr_matrix((K_full.val, K_full.col, K_full.row_ptr), shape=(K_full.n, K_full.n))
    pen = 1e20 * np.abs(A.diagonal()).max()
    add = np.zeros(K_full.n)
    add[p.fixed] = pen
    f = p.f.copy()
    f[p.fixed] += pen * p.fixed_values
    return spla.spsolve((A + sp.diags(add)).tocsc(), f)


@pytest.mark.parametrize("which", ["lognormal_8x4x4", "cantilever_40x8x8"])
def test_penalty_and_elimination_agree(pkg, orc, which):
    """This path eliminates the Dirichlet rows and columns (unit diagonal,
    lifted right-hand side) instead of the reference's 1e20 penalty: with both
    systems solved directly, the displacements differ by at most 1e-12
    relative (measured 4.5e-15 and 2.2e-13)."""
    spla = pytest.importorskip("scipy.sparse.linalg")
    sp = pytest.importorskip("scipy.sparse")
    p = pkg.mesh.lognormal_cantilever(8, 4, 4, seed=3) if which == "lognormal_8x4x4" else pkg.mesh.config1()
    m = orc.Model(p)
    u_pen = _penalty_solution(p, m.assemble(eliminate=False))
    Ke = m.assemble()
    u_el = spla.spsolve(sp.csc_matrix((Ke.val, Ke.col, Ke.row_ptr), shape=(Ke.n, Ke.n)), m.lifted_rhs())
    assert np.linalg.norm(u_pen - u_el) / np.linalg.norm(u_el) <= 1e-12
    assert np.abs(u_pen[p.fixed]).max() <= 1e-20
