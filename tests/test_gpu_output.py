"""Loads and output either side of the solve, on the GPU through the C-ABI:
face tractions and pressures (PH_Elem_C3D8_FormFacePressure), nodal stress by
Gauss-point extrapolation (PH_Elem_C3D8_GetExtrapMat / MapToNode) and
reaction forces, against the numpy oracle."""
import numpy as np
import pytest

from oracle import np_oracle as NO

pytestmark = pytest.mark.gpu


def _distorted_box(pkg, n=3, seed=7, amp=0.12):
    coords, conn = pkg.mesh.box_mesh(n, n, n, float(n), float(n), float(n))
    rng = np.random.default_rng(seed)
    coords = coords + amp * rng.uniform(-1.0, 1.0, coords.shape)
    ne = conn.shape[0]
    props = np.stack([rng.uniform(1e3, 5e3, ne), np.full(ne, 0.3)], axis=1)
    fixed = pkg.mesh._clamp(pkg.mesh._plane_nodes(n, n, n, 0, 0))
    return pkg.mesh.Problem("distorted", (n, n, n), coords, conn, pkg.MAT_ELASTIC_ISO, props, fixed,
                            np.zeros(fixed.size), np.zeros(3 * coords.shape[0]))


def test_face_traction_matches_cantilever_load(pkg):
    # the x = 10 face of the 40x8x8 cantilever: reference face 6 (xi = +1)
    p = pkg.mesh.config1()
    m = pkg.FemModel.from_problem(p)
    nx, ny, nz = p.shape
    elems = pkg.mesh._face_elems(nx, ny, nz, "xmax")
    f = m.load_faces(elems, np.full(elems.size, 6), traction=np.tile([0.0, 0.0, -1.0], (elems.size, 1)))
    np.testing.assert_allclose(f, p.f, rtol=0, atol=1e-14)
    assert abs(f[2::3].sum() + 4.0) <= 1e-12  # traction 1 on a 2 x 2 face
    # a pressure -1 on the same face: the force points along the outward normal +x
    fp = m.load_faces(elems, np.full(elems.size, 6), pressure=np.full(elems.size, -1.0))
    assert abs(fp[0::3].sum() - 4.0) <= 1e-12 and np.abs(fp[1::3]).max() <= 1e-15


def test_face_loads_distorted_mesh_match_oracle(pkg):
    p = _distorted_box(pkg)
    m = pkg.FemModel.from_problem(p)
    rng = np.random.default_rng(3)
    nf = 40
    elem = rng.integers(0, p.n_elems, nf).astype(np.int32)  # repeats: several faces per element
    face = rng.integers(1, 7, nf).astype(np.int32)
    tr = rng.standard_normal((nf, 3))
    pr = rng.standard_normal(nf)
    ref = NO.face_loads(p.coords, p.conn, elem, face, tr, pr)
    f = m.load_faces(elem, face, traction=tr, pressure=pr)
    np.testing.assert_allclose(f, ref, rtol=0, atol=1e-13 * np.abs(ref).max())
    f1 = m.load_faces(elem + 1, face, traction=tr, pressure=pr, index_base=1)
    np.testing.assert_array_equal(f1, f)  # deterministic, same order
    import torch

    dev = torch.device("cuda", 0)
    ft = m.load_faces(torch.tensor(elem, device=dev), torch.tensor(face, device=dev),
                      traction=torch.tensor(tr, device=dev), pressure=torch.tensor(pr, device=dev))
    np.testing.assert_array_equal(ft.cpu().numpy(), f)
    with pytest.raises(pkg.UfcError) as ei:
        m.load_faces(elem, np.full(nf, 7), pressure=pr)
    assert ei.value.status_code == 1


def test_uniform_pressure_on_closed_surface_balances(pkg):
    p = _distorted_box(pkg, n=3, seed=11)
    m = pkg.FemModel.from_problem(p)
    elem, face = [], []
    for name, fid in (("zmin", 1), ("zmax", 2), ("ymin", 3), ("ymax", 4), ("xmin", 5), ("xmax", 6)):
        e = pkg.mesh._face_elems(3, 3, 3, name)
        elem += list(e)
        face += [fid] * e.size
    f = m.load_faces(np.array(elem), np.array(face), pressure=np.full(len(elem), 2.5))
    scale = np.abs(f).max()
    for c in range(3):
        assert abs(f[c::3].sum()) <= 1e-12 * scale * len(elem)


def test_nodal_stress_uniform_field(pkg):
    p = pkg.mesh.unit_cube_uniaxial()
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    u, _ = m.solve(pkg.lifted_rhs(m, p.f), pkg.SolverAlgo(tolerance=1e-14))
    sig, vm = m.stress_nodal(u)
    np.testing.assert_allclose(sig[:, 0], 100e6, rtol=1e-10)
    assert np.abs(sig[:, 1:]).max() <= 1e-6 * 100e6
    np.testing.assert_allclose(vm, 100e6, rtol=1e-10)


def test_nodal_stress_matches_oracle(pkg, orc):
    p = _distorted_box(pkg, n=4, seed=5)
    m = pkg.FemModel.from_problem(p)
    u = np.random.default_rng(2).standard_normal(p.n_dof) * 1e-3
    sig, vm = m.stress_nodal(u)
    sgp, _ = orc.Model(p).elastic_vm(u)
    ref_s, ref_vm = NO.nodal_stress(p.n_nodes, p.conn, sgp)
    np.testing.assert_allclose(sig, ref_s, rtol=0, atol=1e-12 * np.abs(ref_s).max())
    np.testing.assert_allclose(vm, ref_vm, rtol=0, atol=1e-12 * np.abs(ref_vm).max())
    # u = None: the displacement held by the context
    m.set_displacement(u)
    sig2, _ = m.stress_nodal()
    np.testing.assert_array_equal(sig2, sig)


def test_nodal_stress_j2_committed_state(pkg, orc):
    p = pkg.mesh.j2_bar(4, 2, 2)
    m = pkg.FemModel.from_problem(p)
    for s in (1, 2):
        assert m.nr_increment(pkg.mesh.j2_bar_target(p, s, n_steps=2, strain=0.004)).converged
        m.commit()
    _, sig_gp, _ = m.j2_state()
    sig, vm = m.stress_nodal()
    ref_s, ref_vm = NO.nodal_stress(p.n_nodes, p.conn, sig_gp.reshape(p.n_elems, 8, 6))
    np.testing.assert_allclose(sig, ref_s, rtol=0, atol=1e-12 * np.abs(ref_s).max())
    np.testing.assert_allclose(vm, ref_vm, rtol=0, atol=1e-12 * np.abs(ref_vm).max())


def test_reactions_balance_and_match_oracle(pkg, orc):
    p = pkg.mesh.config1()
    m = pkg.FemModel.from_problem(p)
    m.assemble(pkg.BUILD_FP64)
    u, st = m.solve(pkg.lifted_rhs(m, p.f), pkg.SolverAlgo(tolerance=1e-10))
    rf = m.reactions(u, p.f)
    assert rf.shape == (p.fixed.size,)
    # equilibrium: the supports carry the applied load
    for c in range(3):
        sel = p.fixed % 3 == c
        assert abs(rf[sel].sum() + p.f[c::3].sum()) <= 1e-8 * 4.0
    K = orc.Model(p).assemble(eliminate=False)
    ref = (K.matvec(u) - p.f)[p.fixed]
    np.testing.assert_allclose(rf, ref, rtol=0, atol=1e-10 * np.abs(ref).max())
    m.set_displacement(u)
    np.testing.assert_array_equal(m.reactions(f_ext=p.f), rf)


def test_edge_cases(pkg):
    p = pkg.mesh.j2_bar(3, 2, 2)
    m = pkg.FemModel.from_problem(p)
    # no faces: a zero load vector
    f = m.load_faces(np.zeros(0, dtype=np.int32), np.zeros(0, dtype=np.int32), traction=np.zeros((0, 3)))
    assert f.shape == (p.n_dof,) and not f.any()
    # element id out of range
    with pytest.raises(pkg.UfcError) as ei:
        m.load_faces([p.n_elems], [1], pressure=[1.0])
    assert ei.value.status_code == 1
    # J2 before any increment: zero committed stress at the nodes, zero reactions
    sig, vm = m.stress_nodal()
    assert not sig.any() and not vm.any()
    assert not m.reactions().any()
    # invalid increment controls are rejected before any work
    for bad in (dict(cutback_factor=1.5), dict(dt_initial=0.0), dict(max_iterations=0), dict(dt_min=2.0)):
        with pytest.raises(pkg.UfcError) as ei:
            m.nr_step(pkg.mesh.j2_bar_target(p, 1, n_steps=1), **bad)
        assert ei.value.status_code == 1, bad
