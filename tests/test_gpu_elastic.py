"""Parity of the CUDA linear-elastic path with the FP64 oracle, through the C-ABI.

Pattern and index work are compared bit for bit; FP64 values to 1e-12
relative; solutions to the tolerances stated in each test.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _model(pkg, p, build=None):
    m = pkg.FemModel.from_problem(p)
    m.assemble(build or (pkg.BUILD_FP64 | pkg.BUILD_FP32))
    return m


SMALL = [
    ("unit_cube", lambda mesh: mesh.unit_cube_uniaxial()),
    ("box_3x2x2", lambda mesh: mesh.cantilever(3, 2, 2, 3.0, 2.0, 2.0, E=np.linspace(1e3, 5e3, 12))),
    ("cantilever_40x8x8", lambda mesh: mesh.config1()),
]


@pytest.mark.parametrize("name,make", SMALL)
def test_pattern_bit_exact(pkg, orc, name, make):
    p = make(pkg.mesh)
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    rp, col, _, _ = m.csr_export(index_base=0)
    rp_o, col_o = orc.csr_pattern(p.n_nodes, p.conn)
    assert np.array_equal(rp, rp_o)
    assert np.array_equal(col, col_o)
    rp1, col1, _, _ = m.csr_export(index_base=1)
    assert rp1[0] == 1 and np.array_equal(rp1 - 1, rp_o) and np.array_equal(col1 - 1, col_o)


def _shuffled_elements(p, seed):
    """The same problem with its elements listed in a random order."""
    perm = np.random.default_rng(seed).permutation(p.n_elems)
    return dataclasses.replace(p, name=p.name + "_shuffled", conn=np.ascontiguousarray(p.conn[perm]),
                               props=np.ascontiguousarray(p.props[perm]))


COLOURED = [
    ("cantilever_40x8x8", lambda mesh: mesh.config1()),
    ("lognormal_24x12x12", lambda mesh: mesh.lognormal_cantilever(24, 12, 12, seed=4)),
    ("shuffled_12x6x6", lambda mesh: _shuffled_elements(mesh.cantilever(12, 6, 6, 12.0, 6.0, 6.0), 7)),
    ("shuffled_10x2x2", lambda mesh: _shuffled_elements(mesh.config1(), 3)),
    ("strip_3000x1x1", lambda mesh: mesh.cantilever(3000, 1, 1, 3000.0, 1.0, 1.0)),
    ("strip_6000x1x1", lambda mesh: mesh.cantilever(6000, 1, 1, 6000.0, 1.0, 1.0)),
]


@pytest.mark.parametrize("name,make", COLOURED)
def test_element_colours_match_oracle(pkg, orc, name, make):
    """ufc_pattern_build colours the elements on the device by in-place sweeps
    of the greedy map; the colours equal the oracle's sequential greedy
    colouring (RT_AsmColor_Build) element for element, on structured and
    shuffled element orders and on strips one element thick, whose chains of
    lower neighbours are as long as the strip (the longer one may exceed the
    sweep limit, after which the host colouring finishes: the same colours)."""
    p = make(pkg.mesh)
    m = pkg.FemModel.from_problem(p)
    ref, ncol = orc.color_elements(p.n_nodes, p.conn)
    assert m.info.n_colors == ncol
    assert np.array_equal(m.colors(), ref)
    assert np.array_equal(m.colors(index_base=1), ref + 1)
    m.close()


@pytest.mark.parametrize("name,make", SMALL)
def test_assembly_values_fp64(pkg, orc, name, make):
    p = make(pkg.mesh)
    m = _model(pkg, p)
    _, _, v, _ = m.csr_export()
    K = orc.Model(p).assemble()
    err = np.abs(v - K.val).max() / np.abs(K.val).max()
    assert err <= 1e-12, err
    _, _, v32, _ = m.csr_export(values=False, values32=True)
    err32 = np.abs(v32.astype(np.float64) - K.val).max() / np.abs(K.val).max()
    assert err32 <= 1e-5, err32


def test_assembly_deterministic_and_symmetric(pkg):
    p = pkg.mesh.lognormal_cantilever(12, 6, 6, seed=7)
    m = _model(pkg, p)
    _, _, v1, _ = m.csr_export()
    m.assemble(pkg.BUILD_FP64 | pkg.BUILD_FP32)
    rp, col, v2, _ = m.csr_export()
    assert np.array_equal(v1, v2)  # bitwise: colour-ordered scatter, no float atomics
    n = p.n_dof
    import scipy.sparse as sp

    K = sp.csr_matrix((v2, col, rp), shape=(n, n))
    asym = abs(K - K.T).max() / abs(K).max()
    assert asym <= 1e-14, asym  # tests/integration/test_assembly_chain.f90:37-40


def test_unit_cube_uniaxial(pkg):
    # tests/ufc_core/test_c3d8_uniaxial.f90: u_x = sigma/E * L = 5e-4 (reference tolerance 1 %)
    p = pkg.mesh.unit_cube_uniaxial()
    m = _model(pkg, p)
    u, st = m.solve(pkg.lifted_rhs(m, p.f), pkg.SolverAlgo(tolerance=1e-14))
    a = p.conn[0]
    ux = u[3 * a[[1, 2, 5, 6]]]
    assert st.converged
    np.testing.assert_allclose(ux, 5e-4, rtol=1e-12)
    np.testing.assert_allclose(u[3 * a[[0, 1, 4, 5]] + 1], 0.0, atol=1e-15)  # uy on the y = 0 face
    # lateral contraction eps_y = -nu * eps_x on the y = 1 face
    np.testing.assert_allclose(u[3 * a[[3, 2, 6, 7]] + 1], -0.3 * 5e-4, rtol=1e-10)


def test_spmv_and_internal_force(pkg, orc):
    p = pkg.mesh.lognormal_cantilever(8, 4, 4, seed=3)
    m = _model(pkg, p)
    K = orc.Model(p).assemble()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(p.n_dof)
    y = m.spmv(x)
    y_o = K.matvec(x)
    assert np.abs(y - y_o).max() / np.abs(y_o).max() <= 1e-13
    y32 = m.spmv(x.astype(np.float32), precision=pkg.PRECISION_FP32_REFINE)
    assert np.abs(y32 - y_o).max() / np.abs(y_o).max() <= 1e-5
    # matrix-free FP64 internal force equals the oracle's F_int
    fint, r, rn, fn = m.internal_force(x)
    f_o = orc.Model(p).fint_elastic(x)
    assert np.abs(fint - f_o).max() / np.abs(f_o).max() <= 1e-13
    free = pkg.mesh.free_mask(p)
    np.testing.assert_allclose(r[free], -f_o[free], rtol=0, atol=1e-12 * np.abs(f_o).max())
    assert np.all(r[~free] == 0.0)


@pytest.mark.parametrize("prec", ["fp64", "fp32_refine", "fp32_forced"])
def test_cantilever_40x8x8_solve(pkg, orc, prec):
    p = pkg.mesh.config1()
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED)
    ref = orc.Model(p)
    u_ref, info = ref.solve_linear(rtol=1e-13)
    mode = pkg.PRECISION_FP64 if prec == "fp64" else pkg.PRECISION_FP32_REFINE
    policy = pkg.REFINE_FORCE_FP32 if prec == "fp32_forced" else pkg.REFINE_KEEP_DIRECTION
    b = pkg.lifted_rhs(m, p.f)
    u, st = m.solve(b, pkg.SolverAlgo(tolerance=1e-10, precision_mode=mode, refine_policy=policy))
    assert st.converged and st.rnorm <= 1e-10
    if prec == "fp32_refine":
        # 10k DOF: the FP64 matrix (8 MB) is read from L2, where FP32 storage
        # saves nothing, so the refined request runs FP64 iterations
        assert st.fp64_iters == st.niter
    if prec == "fp32_forced":
        # forced FP32 iterations on this slender, ill-conditioned cantilever: the
        # refined run converges with residual replacement, or hands its best
        # iterate on to FP64 when it stalls; either way to the same tolerance
        assert st.niter > 0
    # independent FP64 residual with the oracle's matrix
    r = b - info["K"].matvec(u)
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 2e-10
    # displacement error against the oracle solved to rtol 1e-13: at most 1e-9
    # relative (the accuracy target of the path; measured about 1e-12)
    err = np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref)
    assert err <= 1e-9, err
    if prec == "fp64":
        _, info10 = ref.solve_linear(rtol=1e-10)
        assert abs(st.niter - info10["iters"]) <= 3, (st.niter, info10["iters"])


@pytest.mark.parametrize("shape", [(8, 4, 4), (33, 5, 3)])
def test_symmetric_storage_matches_full(pkg, orc, shape):
    p = pkg.mesh.lognormal_cantilever(*shape, seed=6)
    full = _model(pkg, p, pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED)
    sym = _model(pkg, p, pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED | pkg.BUILD_SYMMETRIC)
    K = orc.Model(p).assemble()
    x = np.random.default_rng(1).standard_normal(p.n_dof)
    y_o = K.matvec(x)
    scale = np.abs(y_o).max()
    assert np.abs(sym.spmv(x) - y_o).max() <= 1e-13 * scale
    x32 = x.astype(np.float32)
    y32_full = full.spmv(x32, precision=pkg.PRECISION_FP32_REFINE)
    y32_sym = sym.spmv(x32, precision=pkg.PRECISION_FP32_REFINE)
    assert np.abs(y32_sym - y32_full).max() <= 1e-5 * scale
    assert np.abs(y32_sym - y_o).max() <= 1e-5 * scale
    b = pkg.lifted_rhs(sym, p.f)
    u_ref, _ = orc.Model(p).solve_linear(rtol=1e-13)
    for prec in (pkg.PRECISION_FP64, pkg.PRECISION_FP32_REFINE):
        # FP32 iterations forced on this small mesh, to exercise the FP32 kernels
        algo = pkg.SolverAlgo(tolerance=1e-10, precision_mode=prec, refine_policy=pkg.REFINE_FORCE_FP32)
        u, st = sym.solve(b, algo)
        assert st.converged and st.rnorm <= 1e-10
        assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) <= 1e-9
        # the solve is bitwise reproducible (no float atomics anywhere)
        u2, st2 = sym.solve(b, algo)
        assert np.array_equal(u, u2) and st2.niter == st.niter
    # the canonical export is unchanged by the symmetric copies
    _, _, v, _ = sym.csr_export()
    assert np.abs(v - K.val).max() <= 1e-12 * np.abs(K.val).max()


def test_cantilever_beam_theory(pkg):
    # E2E_C2_01 checks tip deflection against beam theory within 5 % (with
    # incompatible modes); full-integration C3D8 on 40x8x8 is within 5 % of
    # Euler-Bernoulli plus Timoshenko shear deflection.
    p = pkg.mesh.config1()
    m = _model(pkg, p)
    u, st = m.solve(pkg.lifted_rhs(m, p.f), pkg.SolverAlgo(tolerance=1e-10))
    tip = np.isclose(p.coords[:, 0], 10.0)
    delta = -u[3 * np.nonzero(tip)[0] + 2].mean()
    L, h, bw, P, E, nu = 10.0, 2.0, 2.0, 4.0, 210e3, 0.3
    I = bw * h ** 3 / 12
    G = E / (2 * (1 + nu))
    theory = P * L ** 3 / (3 * E * I) + P * L / (5.0 / 6.0 * G * bw * h)
    assert abs(delta - theory) / theory < 0.05, (delta, theory)


def test_von_mises_matches_oracle(pkg, orc):
    p = pkg.mesh.lognormal_cantilever(8, 4, 4, seed=5)
    m = _model(pkg, p)
    u = np.random.default_rng(1).standard_normal(p.n_dof) * 1e-3
    sig, vm = m.stress(u)
    sig_o, vm_o = orc.Model(p).elastic_vm(u)
    assert np.abs(sig - sig_o).max() / np.abs(sig_o).max() <= 1e-13
    assert np.abs(vm - vm_o).max() / np.abs(vm_o).max() <= 1e-13


def test_not_converged_and_errors(pkg):
    p = pkg.mesh.config1()
    m = _model(pkg, p)
    b = pkg.lifted_rhs(m, p.f)
    with pytest.raises(pkg.UfcError) as ei:
        m.solve(b, pkg.SolverAlgo(max_iter=3))
    assert ei.value.status_code == 4  # IF_STATUS_NOT_CONVERGED
    x, st = m.solve(b, pkg.SolverAlgo(max_iter=3), raise_on_not_converged=False)
    assert not st.converged and st.niter == 3 and st.status == 4
    # inverted element: Jacobian check reports IF_STATUS_ERROR, no device fault
    q = pkg.mesh.cantilever(2, 1, 1, 2.0, 1.0, 1.0)
    conn = q.conn.copy()
    conn[0] = conn[0][[4, 5, 6, 7, 0, 1, 2, 3]]  # top and bottom swapped: detJ < 0
    bad = pkg.FemModel()
    bad.set_mesh(q.coords, conn)
    bad.set_material(pkg.MAT_ELASTIC_ISO, q.props)
    bad.set_bc(q.fixed)
    bad.pattern_build()
    with pytest.raises(pkg.UfcError) as ei:
        bad.assemble()
    assert ei.value.status_code == 2 and "Jacobian" in ei.value.message
    # connectivity out of range is rejected on the host
    with pytest.raises(pkg.UfcError) as ei:
        bad.set_mesh(q.coords, conn + 100)
    assert ei.value.status_code == 1
    # the context stays usable after the failures
    m2 = _model(pkg, pkg.mesh.unit_cube_uniaxial())
    assert m2.solve(pkg.lifted_rhs(m2, m2.problem.f))[1].converged


@pytest.mark.parametrize("precond", ["jacobi", "multigrid", "block"])
def test_nan_load_returns_status(pkg, precond):
    """A load vector holding a NaN (or an Inf) is rejected with
    IF_STATUS_INVALID before any iteration (RT_Step_Exec.f90:560-600 reports a
    failed increment by status, never by hanging); the model stays usable."""
    p = pkg.mesh.lognormal_cantilever(8, 4, 4, seed=3)
    m = _model(pkg, p, pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED)
    b = pkg.lifted_rhs(m, p.f)
    bad = b.copy()
    bad[np.nonzero(b)[0][0]] = np.nan
    if precond == "multigrid":
        m.mg_setup(8, 4, 4)
        algos = [pkg.SolverAlgo(tolerance=1e-10, precond_type=pkg.SOLV_PREC_MG)]
    elif precond == "block":  # the block PCG is FP64 only
        algos = [pkg.SolverAlgo(tolerance=1e-10)]
    else:
        algos = [pkg.SolverAlgo(tolerance=1e-10, precision_mode=pm)
                 for pm in (pkg.PRECISION_FP64, pkg.PRECISION_FP32_REFINE)]
    for algo in algos:
        for v in (np.nan, np.inf):
            bad[np.nonzero(b)[0][0]] = v
            with pytest.raises(pkg.UfcError) as ei:
                if precond == "block":
                    m.solve_block(np.stack([b, bad]), algo)
                else:
                    m.solve(bad, algo)
            assert ei.value.status_code == pkg.STATUS_INVALID and "non-finite" in ei.value.message
        _, st = m.solve(b, algo)
        assert st.converged and st.rnorm <= 1e-10


@pytest.mark.parametrize("nrhs", [1, 2, 3, 8, 16, 32])
def test_block_solve_matches_single(pkg, orc, nrhs):
    p = pkg.mesh.density_problem(10, 5, 5, seed=5, n_rhs=max(nrhs, 1))
    m = _model(pkg, p, pkg.BUILD_FP64)
    F = np.ascontiguousarray(p.meta["F"][:nrhs])
    algo = pkg.SolverAlgo(tolerance=1e-10)
    X, states = m.solve_block(F, algo)
    K = orc.Model(p).assemble()
    for k in range(nrhs):
        assert states[k].converged and states[k].rnorm <= 1e-10
        r = F[k] - K.matvec(X[k])
        assert np.linalg.norm(r) / np.linalg.norm(F[k]) <= 2e-10
        x1, s1 = m.solve(F[k], algo)
        assert np.linalg.norm(X[k] - x1) <= 1e-9 * np.linalg.norm(x1)
        assert abs(states[k].niter - s1.niter) <= 2


def test_elimination_matches_reference_penalty(pkg, orc):
    """The GPU's eliminated solve against the reference's penalty treatment of
    the same Dirichlet set (1e20 max|K_ii| on the diagonal, solved directly on
    the CPU): within 1e-9 relative, the accuracy target of the path."""
    from test_oracle import _penalty_solution

    p = pkg.mesh.lognormal_cantilever(8, 4, 4, seed=3)
    m = _model(pkg, p, pkg.BUILD_FP64)
    u, st = m.solve(pkg.lifted_rhs(m, p.f), pkg.SolverAlgo(tolerance=1e-12))
    u_pen = _penalty_solution(p, orc.Model(p).assemble(eliminate=False))
    assert st.converged and np.linalg.norm(u - u_pen) / np.linalg.norm(u_pen) <= 1e-9


def test_symmetric_coded_indices_large_mesh(pkg, orc):
    """A mesh with more than 32 slices per SM takes the symmetric product with
    coded indices (per row 16 upper and 16 lower code bytes instead of 4-byte
    columns and lower references; stencil-like patterns only): its products in
    FP64 and FP32 against the oracle's CSR, a refined FP32 solve and an FP64
    solve against the full storage, and the bytes per product it reports."""
    p = pkg.mesh.lognormal_cantilever(64, 48, 48, seed=8)
    sym = _model(pkg, p, pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED | pkg.BUILD_SYMMETRIC)
    full = _model(pkg, p, pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED)
    K = orc.Model(p).assemble()
    x = np.random.default_rng(3).standard_normal(p.n_dof)
    y_o = K.matvec(x)
    scale = np.abs(y_o).max()
    assert np.abs(sym.spmv(x) - y_o).max() <= 1e-13 * scale
    x32 = x.astype(np.float32)
    assert np.abs(sym.spmv(x32, precision=pkg.PRECISION_FP32_REFINE) - y_o).max() <= 1e-5 * scale
    b = pkg.lifted_rhs(sym, p.f)
    for prec in (pkg.PRECISION_FP64, pkg.PRECISION_FP32_REFINE):
        algo = pkg.SolverAlgo(tolerance=1e-10, precision_mode=prec)
        us, ss = sym.solve(b, algo)
        uf, sf = full.solve(b, algo)
        assert ss.converged and sf.converged
        assert np.linalg.norm(us - uf) / np.linalg.norm(uf) <= 1e-9
    # the coded form reports its own bytes: 9 s per upper block + 32 code bytes per row + x and y
    sym.set_instrument(True)
    sym.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    t = sym.last_timing()
    sym.set_instrument(False)
    info = sym.info
    nrows = (p.n_nodes + 31) // 32 * 32
    upper = (info.nnzb + p.n_nodes) // 2
    assert t["spmv_bytes"] == upper * 72 + 32 * nrows + 16 * p.n_dof


def _renumbered(pkg, p, seed):
    """The same problem with its nodes numbered in a random order: the block
    pattern is then not stencil-like (many distinct offsets col - row), so the
    products read 4-byte column indices instead of the coded ones."""
    perm = np.random.default_rng(seed).permutation(p.n_nodes)  # new id of old node i
    coords = np.empty_like(p.coords)
    coords[perm] = p.coords
    conn = perm[p.conn].astype(np.int32)
    dof_map = (3 * perm[:, None] + np.arange(3)).ravel()  # old dof -> new dof
    order = np.argsort(dof_map[p.fixed])
    fixed = dof_map[p.fixed][order].astype(np.int32)
    f = np.empty_like(p.f)
    f[dof_map] = p.f
    return pkg.mesh.Problem(p.name + "_renumbered", p.shape, coords, conn, p.mat_model_id, p.props, fixed,
                            p.fixed_values[order], f), dof_map


def test_block_solve_tiles_match_plain_indices(pkg, orc):
    """16 right-hand sides on a structured numbering take the tiled block
    product (x nodes staged in shared memory by bulk copies, coded pattern); the
    same mesh randomly renumbered takes the pipelined one (4-byte columns).  Both
    block solves meet the tolerance against the oracle's matrix and agree with
    each other to 1e-9."""
    p = pkg.mesh.density_problem(12, 6, 6, seed=5, n_rhs=16)
    q, dof_map = _renumbered(pkg, p, seed=3)
    F = np.ascontiguousarray(p.meta["F"][:16])
    Fq = np.empty_like(F)
    Fq[:, dof_map] = F
    algo = pkg.SolverAlgo(tolerance=1e-10)
    Xp, sp = _model(pkg, p, pkg.BUILD_FP64).solve_block(F, algo)
    Xq, sq = _model(pkg, q, pkg.BUILD_FP64).solve_block(np.ascontiguousarray(Fq), algo)
    Kp, Kq = orc.Model(p).assemble(), orc.Model(q).assemble()
    for k in range(16):
        assert sp[k].converged and sq[k].converged
        assert np.linalg.norm(F[k] - Kp.matvec(Xp[k])) <= 2e-10 * np.linalg.norm(F[k])
        assert np.linalg.norm(Fq[k] - Kq.matvec(Xq[k])) <= 2e-10 * np.linalg.norm(Fq[k])
        assert np.linalg.norm(Xq[k][dof_map] - Xp[k]) <= 1e-9 * np.linalg.norm(Xp[k])


@pytest.mark.parametrize("shape", [(8, 4, 4), (64, 48, 48)])
def test_unstructured_numbering_uses_plain_indices(pkg, orc, shape):
    """Random node numbering: full and symmetric products and solves agree with
    the oracle and with the structured numbering of the same mesh (coded
    indices there, 4-byte indices here; 64x48x48 takes the one-warp-per-slice
    kernels, 8x4x4 the split ones)."""
    p = pkg.mesh.lognormal_cantilever(*shape, seed=4)
    q, dof_map = _renumbered(pkg, p, seed=11)
    K = orc.Model(q).assemble()
    x = np.random.default_rng(2).standard_normal(q.n_dof)
    y_o = K.matvec(x)
    scale = np.abs(y_o).max()
    u_ref = None
    for build in (pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED, pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED | pkg.BUILD_SYMMETRIC):
        m = _model(pkg, q, build)
        assert np.abs(m.spmv(x) - y_o).max() <= 1e-13 * scale
        u, st = m.solve(pkg.lifted_rhs(m, q.f), pkg.SolverAlgo(tolerance=1e-10))
        assert st.converged
        if u_ref is None:
            s = _model(pkg, p, build)
            us, _ = s.solve(pkg.lifted_rhs(s, p.f), pkg.SolverAlgo(tolerance=1e-10))
            u_ref = np.empty_like(us)
            u_ref[dof_map] = us  # structured solution in the renumbered order
        assert np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref) <= 1e-9
