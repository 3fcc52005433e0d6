"""Adjoint sensitivity kernel and the torch.autograd.Function against the
oracle and central finite differences (the reference adjoint is a stub, so
finite differences are the pin)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sensitivity_kernel_matches_oracle(pkg, orc):
    p = pkg.mesh.density_problem(6, 3, 3, seed=5, n_rhs=3)
    m = pkg.FemModel.from_problem(p)
    rng = np.random.default_rng(2)
    U = rng.standard_normal((3, p.n_dof))
    L = rng.standard_normal((3, p.n_dof))
    g = m.adjoint_sensitivity(U, L)
    g_o = orc.Model(p).adjoint_dJdE(U, L)
    np.testing.assert_allclose(g, g_o, rtol=0, atol=1e-12 * np.abs(g_o).max())


def _setup(pkg, nx=6, ny=3, nz=3, n_rhs=2):
    import torch

    from ufc_fem_kernel_b200.adjoint import ElasticModel

    p = pkg.mesh.density_problem(nx, ny, nz, seed=5, n_rhs=n_rhs)
    dev = torch.device("cuda", 0)
    model = ElasticModel(p, device=0)
    rho = torch.tensor(p.meta["rho"], dtype=torch.float64, device=dev)
    F = torch.tensor(p.meta["F"], dtype=torch.float64, device=dev)
    return p, model, rho, F


def _du(model, rho_pert, U0, F, algo):
    """Displacement change for perturbed densities, solved as a correction:
    K' d = P (F - K' u0) (so the finite difference is not swamped by the solver
    tolerance).  U0, F: [nrhs, n]."""
    import torch

    model.set_moduli(210e3 * rho_pert ** 3)
    D = torch.empty_like(U0)
    for k in range(U0.shape[0]):
        _, r, _, _ = model.fem.internal_force(U0[k].contiguous(), f_ext=F[k].contiguous(), update_state=False)
        D[k], _ = model.fem.solve(r, algo)
    return D


def test_compliance_gradient_vs_finite_differences(pkg):
    import torch

    from ufc_fem_kernel_b200.adjoint import UfcLinearElastic

    p, model, rho, F = _setup(pkg)
    algo = pkg.SolverAlgo(tolerance=1e-11, max_iter=20000)
    rho = rho.clone().requires_grad_(True)
    E = 210e3 * rho ** 3
    U = UfcLinearElastic.apply(E, F, model, algo)
    J = (F * U).sum()
    J.backward()
    g = rho.grad.clone()
    U0 = U.detach()
    h = 1e-6
    for e in p.meta["fd_elems"][:8]:
        rp, rm = rho.detach().clone(), rho.detach().clone()
        rp[e] += h
        rm[e] -= h
        fd = ((F * _du(model, rp, U0, F, algo)).sum() - (F * _du(model, rm, U0, F, algo)).sum()).item() / (2 * h)
        assert abs(g[e].item() - fd) <= 1e-6 * abs(fd), (e, g[e].item(), fd)


def test_tip_displacement_gradient_and_load_gradient(pkg):
    import torch

    from ufc_fem_kernel_b200.adjoint import UfcLinearElastic

    p, model, rho, F = _setup(pkg, n_rhs=1)
    algo = pkg.SolverAlgo(tolerance=1e-11, max_iter=20000)
    tip = 3 * p.meta["tip_node"] + 2
    rho = rho.clone().requires_grad_(True)
    F1 = F[0].clone().requires_grad_(True)
    U = UfcLinearElastic.apply(210e3 * rho ** 3, F1, model, algo)
    J = U[tip]
    J.backward()
    # dJ/dF = lambda = K^-1 e_tip (free DOFs); check by linearity: J(F + t d) - J(F) = t d.lambda
    d = torch.randn_like(F1) * model.free
    with torch.no_grad():
        U2 = UfcLinearElastic.apply(210e3 * rho.detach() ** 3, F1.detach() + d, model, algo)
    np.testing.assert_allclose((U2[tip] - U[tip]).item(), torch.dot(d, F1.grad).item(), rtol=1e-7)
    h = 1e-6
    g = rho.grad
    U0 = U.detach().reshape(1, -1)
    Fd = F1.detach().reshape(1, -1)
    for e in p.meta["fd_elems"][:4]:
        rp, rm = rho.detach().clone(), rho.detach().clone()
        rp[e] += h
        rm[e] -= h
        fd = (_du(model, rp, U0, Fd, algo)[0, tip] - _du(model, rm, U0, Fd, algo)[0, tip]).item() / (2 * h)
        assert abs(g[e].item() - fd) <= 1e-6 * abs(fd) + 1e-9 * abs(g).max().item(), (e, g[e].item(), fd)


def test_compliance_gradient_with_multigrid_preconditioner(pkg):
    """The adjoint through MG-PCG: the hierarchy is refreshed after each
    reassembly (set_moduli), so the gradient matches the Jacobi-PCG gradient
    and central finite differences."""
    import torch

    from ufc_fem_kernel_b200.adjoint import UfcLinearElastic

    p, model, rho, F = _setup(pkg, nx=16, ny=8, nz=8, n_rhs=2)
    model.set_moduli(210e3 * rho ** 3)
    levels, _, _ = model.fem.mg_setup(16, 8, 8, coarse_max=100)
    assert levels >= 2
    mg = pkg.SolverAlgo(tolerance=1e-11, max_iter=2000, precond_type=pkg.SOLV_PREC_MG)
    jac = pkg.SolverAlgo(tolerance=1e-11, max_iter=20000)
    grads = {}
    for name, algo in (("mg", mg), ("jacobi", jac)):
        r = rho.clone().requires_grad_(True)
        U = UfcLinearElastic.apply(210e3 * r ** 3, F, model, algo)
        (F * U).sum().backward()
        grads[name] = r.grad.clone()
        if name == "mg":
            assert all(st.converged and st.niter < 200 for st in model.last_states)
    g = grads["mg"]
    np.testing.assert_allclose(g.cpu().numpy(), grads["jacobi"].cpu().numpy(), rtol=1e-7,
                               atol=1e-9 * g.abs().max().item())
    U0 = UfcLinearElastic.apply(210e3 * rho ** 3, F, model, mg).detach()
    h = 1e-6
    for e in p.meta["fd_elems"][:4]:
        rp, rm = rho.clone(), rho.clone()
        rp[e] += h
        rm[e] -= h
        fd = ((F * _du(model, rp, U0, F, mg)).sum() - (F * _du(model, rm, U0, F, mg)).sum()).item() / (2 * h)
        assert abs(g[e].item() - fd) <= 1e-6 * abs(fd), (e, g[e].item(), fd)
