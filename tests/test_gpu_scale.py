"""Full-size checks on the 128x64x64 and 192x96x96 lognormal cantilevers, the
adjoint at 128x64x64 and the J2 bar at 64x32x32, through properties that do not
need the oracle at that size: an independent FP64 residual (matrix-free element
operator against the assembled-matrix solve), agreement of the FP32+refine,
FP64 and symmetric-storage solutions, the compliance identity f.u = u.K.u,
bitwise reproducibility, and adjoint gradients against finite differences."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big(pkg):
    import torch

    out = {}
    for name, make in (("128x64x64", pkg.mesh.config2), ("192x96x96", pkg.mesh.config4)):
        p = make()
        m = pkg.FemModel.from_problem(p)
        m.assemble(pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED)
        b = torch.from_numpy(pkg.lifted_rhs(m, p.f)).cuda()
        out[name] = (p, m, b)
    yield out
    for _, m, _ in out.values():
        m.close()


@pytest.mark.parametrize("name", ["128x64x64", "192x96x96"])
def test_full_size_fp64_and_mixed(pkg, big, name):
    import torch

    p, m, b = big[name]
    u64, s64 = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    u32, s32 = m.solve(b, pkg.SolverAlgo(tolerance=1e-10, precision_mode=pkg.PRECISION_FP32_REFINE))
    assert s64.converged and s32.converged and s64.rnorm <= 1e-10 and s32.rnorm <= 1e-10
    bn = torch.linalg.vector_norm(b).item()
    for u in (u64, u32):
        # independent residual: matrix-free FP64 element operator, not the assembled matrix
        _, r, rn, _ = m.internal_force(u, f_ext=b)
        assert rn / bn <= 1.5e-10
    rel = (torch.linalg.vector_norm(u32 - u64) / torch.linalg.vector_norm(u64)).item()
    assert rel <= 1e-9, rel
    # compliance identity f.u = u.K.u (energy), through the SpMV
    Ku = m.spmv(u64)
    assert abs(torch.dot(b, u64).item() - torch.dot(u64, Ku).item()) <= 1e-9 * abs(torch.dot(b, u64).item())
    # von Mises of the two solutions
    _, vm64 = m.stress(u64, want_sigma=False)
    _, vm32 = m.stress(u32, want_sigma=False)
    assert (torch.max(torch.abs(vm32 - vm64)) / torch.max(vm64)).item() <= 1e-8
    # bitwise reproducible solve
    u64b, _ = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    assert torch.equal(u64, u64b)


def test_symmetric_storage_full_size(pkg, big):
    import torch

    p, m, b = big["128x64x64"]
    u_full, _ = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
    m.assemble(pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED | pkg.BUILD_SYMMETRIC)
    try:
        u_sym, s = m.solve(b, pkg.SolverAlgo(tolerance=1e-10))
        assert s.converged
        assert (torch.linalg.vector_norm(u_sym - u_full) / torch.linalg.vector_norm(u_full)).item() <= 1e-9
        x = torch.randn(p.n_dof, dtype=torch.float64, device="cuda")
        y_sym = m.spmv(x)
    finally:
        m.assemble(pkg.BUILD_FP64 | pkg.BUILD_FP32_ROUNDED)
    y_full = m.spmv(x)
    assert (torch.max(torch.abs(y_sym - y_full)) / torch.max(torch.abs(y_full))).item() <= 1e-13


def test_adjoint_autograd_128x64x64(pkg):
    """The density problem with its 16 tip-load cases through the
    torch.autograd.Function: forward as one block solve, then dJ/drho and dJ/dF
    of both objectives summed over the cases (compliance J1 = sum f.u, tip-centre
    displacement J2 = sum u_z(tip)).  dJ/drho is checked against central finite
    differences (h = 1e-6) on all 32 seeded elements for both objectives (each
    perturbed solve a multigrid correction), within 1e-6 relative; dJ2/dF by
    linearity of J2 in F."""
    import torch

    from ufc_fem_kernel_b200.adjoint import ElasticModel, central_differences, density_objectives

    p = pkg.mesh.config5()
    dev = torch.device("cuda", 0)
    model = ElasticModel(p, device=0)
    rho0 = torch.tensor(p.meta["rho"], dtype=torch.float64, device=dev)
    F0 = torch.tensor(p.meta["F"], dtype=torch.float64, device=dev) * model.free
    tip = 3 * int(p.meta["tip_node"]) + 2
    algo = pkg.SolverAlgo(tolerance=1e-10)
    rho = rho0.clone().requires_grad_(True)
    F = F0.clone().requires_grad_(True)
    J1, J2, U = density_objectives(rho, F, model, algo, tip)
    assert len(model.last_states) == 16 and all(s.converged for s in model.last_states)
    # the block solve agrees with a single solve of case 0
    u0, _ = model.fem.solve(F0[0].contiguous(), algo)
    assert (torch.linalg.vector_norm(U[0] - u0) / torch.linalg.vector_norm(u0)).item() <= 1e-9
    g1 = torch.autograd.grad(J1, [rho, F], retain_graph=True)
    g2 = torch.autograd.grad(J2, [rho, F])
    # compliance: dJ1/dF = 2 u on the free DOFs (J1 = f.K^-1 f)
    assert (torch.linalg.vector_norm(g1[1] - 2 * U.detach()) / torch.linalg.vector_norm(U)).item() <= 1e-9
    model.fem.mg_setup(*p.shape)
    mg = pkg.SolverAlgo(tolerance=1e-10, precond_type=pkg.SOLV_PREC_MG)
    elems = [int(e) for e in p.meta["fd_elems"]]
    fd1, fd2 = central_differences(model, rho0, F0, U.detach(), elems, mg, tip_dof=tip)
    scale2 = g2[0].abs().max().item()
    for e, f1, f2 in zip(elems, fd1, fd2):
        assert abs(g1[0][e].item() - f1) <= 1e-6 * abs(f1), (e, g1[0][e].item(), f1)
        assert abs(g2[0][e].item() - f2) <= 1e-6 * abs(f2) + 1e-9 * scale2, (e, g2[0][e].item(), f2)
    # dJ2/dF: J2 is linear in F, so J2(F + d) - J2(F) = d . dJ2/dF
    d = torch.randn(F0.shape, generator=torch.Generator(device=dev).manual_seed(7), device=dev,
                    dtype=torch.float64) * model.free
    with torch.no_grad():
        _, J2d, _ = density_objectives(rho0, F0 + d, model, algo, tip)
    lhs, rhs = J2d.item() - J2.item(), torch.sum(d * g2[1]).item()
    assert abs(lhs - rhs) <= 1e-7 * abs(rhs), (lhs, rhs)
    model.fem.close()
